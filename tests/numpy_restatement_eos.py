"""An independent, vectorised numpy restatement of the Helmholtz evaluation
helm_rhoT_given_full (source/source.F90:23686-24232, without USE_COULOMB_CORRECTIONS, which no
configuration of the reference's tests defines) and of the table nodes of load_helm_table
(S:23094-23104), written from the Fortran separately from the C oracle, so that a bitwise match
pins the oracle's biquintic interpolation, its bicubic dP/drho, the ion and radiation terms and
the relativistic sound speed; helm_rhoT_given1 / given2 (S:24234-24941) and the two Newton
inversions helm_rhoP_given / helm_rhoe_given (S:24943-25019) likewise.  Test infrastructure
only.
"""
import numpy as np

RGAS = 8.31446261815324e7
RAD = 7.565767381646406e-15
C = 2.99792458e10
C2 = 8.987551787368177e20

# (rho order, T order) of the nine free-energy columns, in the table's order (S:520-528), and
# of the four dP/drho columns
_F_ORD = [(0, 0), (0, 1), (0, 2), (1, 0), (2, 0), (1, 1), (2, 1), (1, 2), (2, 2)]
_P_ORD = [(0, 0), (0, 1), (1, 0), (1, 1)]


def nodes(nT, nrho, ltlo, lthi, ldlo, ldhi):
    """helm_T, helm_rho and their log10 spacings as load_helm_table forms them."""
    dT = (lthi - ltlo) / float(nT - 1)
    drho = (ldhi - ldlo) / float(nrho - 1)
    # Fortran's 10**x is the C library's pow, which Python's float power calls (numpy's
    # vectorised power may round differently in the last place)
    T = np.array([10.0 ** (ltlo + float(j) * dT) for j in range(nT)])
    rho = np.array([10.0 ** (ldlo + float(i) * drho) for i in range(nrho)])
    return T, rho, dT, drho


def _sum_terms(terms):
    s = terms[0]
    for t in terms[1:]:
        s = s + t
    return s


def _quintic(x, omx, h, order):
    """The quintic Hermite basis (psi0, psi1, psi2 on both nodes) or its first / second
    derivative, scaled by the node spacing h as the reference writes them."""
    x2, x3 = x * x, x * x * x
    x4, x5 = x3 * x, x3 * x * x
    o2, o3 = omx * omx, omx * omx * omx
    o4, o5 = o3 * omx, o3 * omx * omx
    ih = 1.0 / h
    if order == 0:
        return ([-6.0 * x5 + 15.0 * x4 - 10.0 * x3 + 1.0, -6.0 * o5 + 15.0 * o4 - 10.0 * o3 + 1.0],
                [(-3.0 * x5 + 8.0 * x4 - 6.0 * x3 + x) * h, (3.0 * o5 - 8.0 * o4 + 6.0 * o3 - omx) * h],
                [(0.5 * (-x5 + 3.0 * x4 - 3.0 * x3 + x2)) * (h * h),
                 (0.5 * (-o5 + 3.0 * o4 - 3.0 * o3 + o2)) * (h * h)])
    if order == 1:
        return ([(-30.0 * x4 + 60.0 * x3 - 30.0 * x2) * ih, -(-30.0 * o4 + 60.0 * o3 - 30.0 * o2) * ih],
                [-15.0 * x4 + 32.0 * x3 - 18.0 * x2 + 1.0, -15.0 * o4 + 32.0 * o3 - 18.0 * o2 + 1.0],
                [(0.5 * (-5.0 * x4 + 12.0 * x3 - 9.0 * x2 + 2.0 * x)) * h,
                 -(0.5 * (-5.0 * o4 + 12.0 * o3 - 9.0 * o2 + 2.0 * omx)) * h])
    return ([(-120.0 * x3 + 180.0 * x2 - 60.0 * x) * (ih * ih), (-120.0 * o3 + 180.0 * o2 - 60.0 * omx) * (ih * ih)],
            [(-60.0 * x3 + 96.0 * x2 - 36.0 * x) * ih, -(-60.0 * o3 + 96.0 * o2 - 36.0 * omx) * ih],
            [0.5 * (-20.0 * x3 + 36.0 * x2 - 18.0 * x + 2.0), 0.5 * (-20.0 * o3 + 36.0 * o2 - 18.0 * omx + 2.0)])


def _cell(tab, nd, rho, T, abar, zbar):
    """The table cell of (rho Ye, T) and the biquintic sum over its 36 coefficients for a
    given pair of basis-derivative orders, as every helm_rhoT_given* routine forms them."""
    hT, hrho, ldT, ldrho = nd
    Ye = zbar / abar
    rhos = rho * Ye
    ih = ((np.log10(rhos) - np.log10(hrho[0])) / ldrho).astype(np.int64)   # 0-based ih - 1
    jh = ((np.log10(T) - np.log10(hT[0])) / ldT).astype(np.int64)
    r0 = hrho[ih]
    drho = hrho[ih + 1] - r0
    x = (rhos - r0) / drho
    omx = 1.0 - x
    t0 = hT[jh]
    dT = hT[jh + 1] - t0
    y = (T - t0) / dT
    omy = 1.0 - y
    corners = [(ih, jh), (ih + 1, jh), (ih, jh + 1), (ih + 1, jh + 1)]
    loc = [tab[v, i, j] for v in range(9) for i, j in corners]
    R = [_quintic(x, omx, drho, k) for k in range(2)]
    Tb = [_quintic(y, omy, dT, k) for k in range(3)]

    def biquintic(rk, tk):
        terms = []
        for v, (orr, ot) in enumerate(_F_ORD):
            rb, tb = R[rk][orr], Tb[tk][ot]
            for n, (a, b) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
                terms.append(loc[4 * v + n] * rb[a] * tb[b])
        return _sum_terms(terms)

    return Ye, rhos, corners, (x, omx, drho), (y, omy, dT), biquintic


def given2(tab, nd, rho, T, abar, zbar, deriv=True):
    """E and dE/dT of helm_rhoT_given2 (S:24571-24941); without `deriv` the table part of
    dE/dT is zero, as in the reference."""
    Ye, _, _, _, _, biquintic = _cell(tab, nd, rho, T, abar, zbar)
    f = biquintic(0, 0)
    df_dT = biquintic(0, 1)
    df_dT2 = biquintic(0, 2) if deriv else 0.0
    s = -Ye * df_dT
    ds_dT = -Ye * df_dT2
    E = Ye * f + T * s
    dE_dT = T * ds_dT
    T3 = T * T * T
    T4 = T3 * T
    tmp = 1.0 / abar
    E = E + 1.5 * RGAS * T * tmp + RAD * T4 / rho
    dE_dT = dE_dT + 1.5 * RGAS * tmp + 4.0 * RAD * T3 / rho
    return E, dE_dT


def given1(tab, nd, rho, T, abar, zbar, deriv=True):
    """P and dP/dT of helm_rhoT_given1 (S:24234-24569)."""
    _, rhos, _, _, _, biquintic = _cell(tab, nd, rho, T, abar, zbar)
    df_drho = biquintic(1, 0)
    df_drhodT = biquintic(1, 1) if deriv else 0.0
    tmp = rhos * rhos
    P = tmp * df_drho
    dP_dT = tmp * df_drhodT
    T3 = T * T * T
    T4 = T3 * T
    tmp = 1.0 / abar
    P = P + RGAS * rho * T * tmp + RAD * T4 * (1.0 / 3.0)
    dP_dT = dP_dT + RGAS * rho * tmp + (4.0 / 3.0) * RAD * T3
    return P, dP_dT


def _newton(fn, target, T0, tl, th, tol=1.0e-11):
    """helm_rhoe_given / helm_rhoP_given's loop (S:24943-25019) for every sample at once: at
    most 100 corrections T -= res / dres_dT, stop once |res / target| < tol, and back to the
    initial guess (and stop) when a correction leaves [Tl_eos, Th_eos].  Returns T and the
    number of evaluations."""
    T = np.array(T0, dtype=float)
    told = T.copy()
    active = np.ones(T.shape, dtype=bool)
    used = np.zeros(T.shape, dtype=np.int64)
    for _ in range(100):
        if not active.any():
            break
        val, dval = fn(T)
        res = val - target
        tn = T - res / dval
        err = np.abs(res / target)
        out = (tn < tl) | (tn > th)
        tn = np.where(out, told, tn)
        err = np.where(out, 1.0e-15, err)
        T = np.where(active, tn, T)
        used = used + active
        active = active & ~(err < tol)
    return T, used


def rhoe_given(tab, dpdr, nd, rho, E0, abar, zbar, T0, tl, th, return_sound=True):
    """helm_rhoe_given: T, P, sound speed (0 without return_sound, P then from given1) and the
    evaluation count."""
    T, used = _newton(lambda t: given2(tab, nd, rho, t, abar, zbar), E0, T0, tl, th)
    if not return_sound:
        return T, given1(tab, nd, rho, T, abar, zbar, deriv=False)[0], 0.0, used
    P, _, sound, _ = given_full(tab, dpdr, nd, rho, T, abar, zbar)
    return T, P, sound, used


def rhoP_given(tab, dpdr, nd, rho, P0, abar, zbar, T0, tl, th, return_sound=True):
    """helm_rhoP_given: T, E, sound speed (0 without return_sound, E then from given2) and the
    evaluation count."""
    T, used = _newton(lambda t: given1(tab, nd, rho, t, abar, zbar), P0, T0, tl, th)
    if not return_sound:
        return T, given2(tab, nd, rho, T, abar, zbar, deriv=False)[0], 0.0, used
    _, E, sound, _ = given_full(tab, dpdr, nd, rho, T, abar, zbar)
    return T, E, sound, used


def given_full(tab, dpdr, nd, rho, T, abar, zbar):
    """P, E, sound speed and c_v of helm_rhoT_given_full at arrays rho, T (abar, zbar scalars
    or arrays).  tab: (9, nrho, nT) columns, dpdr: (4, nrho, nT), nd: `nodes(...)`."""
    Ye, rhos, corners, (x, omx, drho), (y, omy, dT), biquintic = _cell(tab, nd, rho, T, abar, zbar)
    f = biquintic(0, 0)
    df_drho = biquintic(1, 0)
    df_dT = biquintic(0, 1)
    df_drhodT = biquintic(1, 1)
    df_dT2 = biquintic(0, 2)
    # bicubic Hermite of dP/drho
    x2, x3, o2, o3 = x * x, x * x * x, omx * omx, omx * omx * omx
    y2, y3, q2, q3 = y * y, y * y * y, omy * omy, omy * omy * omy
    cr = ([2.0 * x3 - 3.0 * x2 + 1.0, 2.0 * o3 - 3.0 * o2 + 1.0],
          [(x3 - 2.0 * x2 + x) * drho, -(o3 - 2.0 * o2 + omx) * drho])
    ct = ([2.0 * y3 - 3.0 * y2 + 1.0, 2.0 * q3 - 3.0 * q2 + 1.0],
          [(y3 - 2.0 * y2 + y) * dT, -(q3 - 2.0 * q2 + omy) * dT])
    terms = []
    for v, (orr, ot) in enumerate(_P_ORD):
        for a, b in [(0, 0), (1, 0), (0, 1), (1, 1)]:
            i, j = corners[a + 2 * b]
            terms.append(dpdr[v, i, j] * cr[orr][a] * ct[ot][b])
    dP_drho = Ye * _sum_terms(terms)
    tmp = rhos * rhos
    P = tmp * df_drho
    dP_dT = tmp * df_drhodT
    s = -Ye * df_dT
    ds_dT = -Ye * df_dT2
    E = Ye * f + T * s
    dE_dT = T * ds_dT
    tmp = 1.0 / abar
    T4 = T * T * T * T
    T3 = T * T * T
    pion = RGAS * rho * T * tmp
    P = P + pion + RAD * T4 * (1.0 / 3.0)
    dP_dT = dP_dT + RGAS * rho * tmp + (4.0 / 3.0) * RAD * T3
    dP_drho = dP_drho + RGAS * T * tmp
    E = E + 1.5 * RGAS * T * tmp + RAD * T4 / rho
    dE_dT = dE_dT + 1.5 * RGAS * tmp + 4.0 * RAD * T3 / rho
    zz = P / rho
    cv = dE_dT
    chiT = T / P * dP_dT
    chirho = dP_drho / zz
    xx = zz * chiT / (T * cv)
    gam1 = chiT * xx + chirho
    z = 1.0 + (E + C2) / zz
    return P, E, C * np.sqrt(gam1 / z), cv
