"""An independent, vectorised numpy restatement of the 2D ideal-gas hydro and MHD steps.

Written from the reference (source/source.F90) separately from the C oracle, in a different
style (whole-array operations on a ghost-padded grid instead of per-line loops), so that a
bitwise match between the two pins the oracle's sweep logic: ghost filling (periodic wrap and
reflective mirror, S:2293-2306 / S:7532-7958), well-balanced deviations (S:7151-7168),
LIM2ND PLM (S:8141-8181), x2 rotation (S:9715-9747, S:10101-10111), LHLLC (S:15681-16122),
WB momentum fix and EVOLVE_ETOT potential flux (S:8953-8966), gravity (S:12606-12644), RK3
(S:7018-7048, S:13518-13531), cons->prim (S:13533-13686) and the CFL dt (S:13707-13960).
With eps_sf set it adds USE_SHOCK_FLATTENING: the pressure-jump detector (S:8073-8136) and
the HLL flux on faces next to a flagged cell (S:15929-16010); LIM2ND cells need no fallback.
`mhd_2d_steps` and `mhd_3d_steps` restate the periodic ideal-MHD step with HLLD or LHLLD
and constrained transport, `wb_mhd_2d_steps` the MHD step of the well-balanced gravitating
box with reflective walls, and `stratified_steps` the stratified Helmholtz boxes of the
benchmark, hydro (LHLLC / HLLC, FLUX_IS_ALL_MACH) or magnetised (with the EoS of
numpy_restatement_eos), read from the same Fortran (their docstrings list the lines).
Test infrastructure only.
"""
import numpy as np

RGAS = 8.31446261815324e7


def _plm(qm, qc, qp):
    sf = qp - qc
    sb = qc - qm
    prod = sf * sb
    with np.errstate(divide="ignore", invalid="ignore"):
        slope = np.where(prod > 0.0, prod / (sf + sb), 0.0)
    t = 0.5 * slope
    return qc - t, qc + t


def _rec(q, kind, limited):
    """Edge values (left, right) of a row of cells from the views q = (q_{i-2}, q_{i-1}, q_i,
    q_{i+1}, q_{i+2}) (the outer two may be None for LIM2ND and PPH): LIM2ND PLM, PPH (third
    order, with the limiter only where `limited`) or LIM5TH (fifth order, always limited)
    (S:8141-8323)."""
    qmm, qm, qc, qp, qpp = q
    if kind == "lim2nd":
        return _plm(qm, qc, qp)
    if kind == "pph":
        tmp = (5.0 / 6.0) * qc
        am = (1.0 / 3.0) * qm + tmp - (1.0 / 6.0) * qp
        ap = -(1.0 / 6.0) * qm + tmp + (1.0 / 3.0) * qp
        if not limited:
            return am, ap
    else:
        tmp = 329.0 * qc
        am = (-21.0 * qmm + 189.0 * qm + tmp - 91.0 * qp + 14.0 * qpp) * (1.0 / 420.0)
        ap = (14.0 * qmm - 91.0 * qm + tmp + 189.0 * qp - 21.0 * qpp) * (1.0 / 420.0)
    am = np.minimum(np.maximum(am, np.minimum(qm, qc)), np.maximum(qm, qc))
    ap = np.minimum(np.maximum(ap, np.minimum(qc, qp)), np.maximum(qc, qp))
    am = am - qc
    ap = ap - qc
    flat = ap * am >= 0.0
    ap = np.where(~flat & (np.abs(ap) >= 2.0 * np.abs(am)), -2.0 * am, ap)
    am = np.where(~flat & (np.abs(am) >= 2.0 * np.abs(ap)), -2.0 * ap, am)
    ap = np.where(flat, 0.0, ap)
    am = np.where(flat, 0.0, am)
    return am + qc, ap + qc


def _lhllc(qL, qR, gm, mach_cutoff):
    igmm1 = 1.0 / (gm - 1.0)
    rhoL, v1L, v2L, pL = qL
    rhoR, v1R, v2R, pR = qR
    inv_rhoL = 1.0 / rhoL
    inv_rhoR = 1.0 / rhoR
    v2sL = v1L * v1L + v2L * v2L + 0.0 * 0.0
    v2sR = v1R * v1R + v2R * v2R + 0.0 * 0.0
    cL = np.sqrt(gm * pL * inv_rhoL)
    cR = np.sqrt(gm * pR * inv_rhoR)
    rhoeL = igmm1 * pL + 0.5 * rhoL * v2sL
    rhoeR = igmm1 * pR + 0.5 * rhoR * v2sR
    mc = np.maximum(cL, cR)
    sL = np.minimum(v1L, v1R) - mc
    sR = np.maximum(v1L, v1R) + mc
    dL = sL - v1L
    dR = sR - v1R
    us = (pR - pL + rhoL * v1L * dL - rhoR * v1R * dR) / (rhoL * dL - rhoR * dR)
    rsL = rhoL * (dL / (sL - us))
    resL = rsL * (rhoeL * inv_rhoL + (us - v1L) * (us + pL * inv_rhoL / dL))
    rsR = rhoR * (dR / (sR - us))
    resR = rsR * (rhoeR * inv_rhoR + (us - v1R) * (us + pR * inv_rhoR / dR))
    chi = np.minimum(1.0, np.maximum(np.sqrt(v2sL) / cL, np.sqrt(v2sR) / cR))
    chi = np.maximum(mach_cutoff, chi)
    phi = chi * (2.0 - chi)
    pstar = 0.5 * (pL + pR) - 0.5 * phi * (0.5 * (rhoL + rhoR)) * (0.5 * (cL + cR)) * (v1R - v1L)
    sgn = np.copysign(1.0, us)
    hp = 0.5 * (1.0 + sgn)
    hm = 0.5 * (1.0 - sgn)
    rs = hp * rsL + hm * rsR
    return [rs * us, rs * us * us + pstar, rs * us * (hp * v2L + hm * v2R), (hp * resL + hm * resR + pstar) * us]


def _hll(qL, qR, gm):
    """Two-wave HLL flux of the ideal-gas hydro solver on flattened faces."""
    igmm1 = 1.0 / (gm - 1.0)
    rhoL, v1L, v2L, pL = qL
    rhoR, v1R, v2R, pR = qR
    cL = np.sqrt(gm * pL * (1.0 / rhoL))
    cR = np.sqrt(gm * pR * (1.0 / rhoR))
    rhoeL = igmm1 * pL + 0.5 * rhoL * (v1L * v1L + v2L * v2L + 0.0 * 0.0)
    rhoeR = igmm1 * pR + 0.5 * rhoR * (v1R * v1R + v2R * v2R + 0.0 * 0.0)
    mc = np.maximum(cL, cR)
    sL = np.minimum(0.0, np.minimum(v1L, v1R) - mc)
    sR = np.maximum(0.0, np.maximum(v1L, v1R) + mc)
    UL = [rhoL, rhoL * v1L, rhoL * v2L, rhoeL]
    UR = [rhoR, rhoR * v1R, rhoR * v2R, rhoeR]
    fL = [rhoL * v1L, rhoL * v1L * v1L + pL, rhoL * v1L * v2L, (rhoeL + pL) * v1L]
    fR = [rhoR * v1R, rhoR * v1R * v1R + pR, rhoR * v1R * v2R, (rhoeR + pR) * v1R]
    d = 1.0 / (sR - sL)
    ph = sL * sR
    return [d * (sR * a - sL * b + ph * (ur - ul)) for a, b, ul, ur in zip(fL, fR, UL, UR)]


def _flags(p_full, G, nx, ny, eps_sf):
    """is_flattened of the padded cells G-1..G+n (2D): cells G-2..G+n+1 whose summed central
    pressure jumps exceed eps_sf * p mark their 3x3 neighbourhood."""
    c = p_full[G - 2:G + nx + 2, G - 2:G + ny + 2]
    tmp = (np.abs(p_full[G - 2:G + nx + 2, G - 1:G + ny + 3] - p_full[G - 2:G + nx + 2, G - 3:G + ny + 1]) +
           np.abs(p_full[G - 1:G + nx + 3, G - 2:G + ny + 2] - p_full[G - 3:G + nx + 1, G - 2:G + ny + 2])) / c
    mark = tmp > eps_sf
    f = np.zeros((nx + 2, ny + 2), dtype=bool)
    for a in range(3):
        for b in range(3):
            f |= mark[a:a + nx + 2, b:b + ny + 2]
    return f   # f[i, j] is padded cell (G - 1 + i, G - 1 + j)


def _fill(a, flip_y, G):
    """Ghosts of a (nx+2G, ny+2G) array: periodic in x, reflective in y (component flips)."""
    nx = a.shape[0] - 2 * G
    ny = a.shape[1] - 2 * G
    a[:G, :] = a[nx:nx + G, :]
    a[nx + G:, :] = a[G:2 * G, :]
    for g in range(1, G + 1):
        a[:, G - g] = (-1.0 if flip_y else 1.0) * a[:, G + g - 1]
        a[:, ny + G - 1 + g] = (-1.0 if flip_y else 1.0) * a[:, ny + G - g]


def hot_bubble_steps(h, nsteps, dt=None, eps_sf=None, rec="lim2nd"):
    """Advance the hot-bubble HostGrid `h` (2D, ideal, WB+ETOT+gravity, LHLLC, RK3) in place;
    eps_sf: USE_SHOCK_FLATTENING with that threshold (ngc >= 3); rec: LIM2ND, PPH or LIM5TH
    (ngc >= 3) edge values of the primitives (no scalars: PPH leaves them unlimited)."""
    c = h.cfg
    G = c.ngc
    gm = c.gamma_ad
    igmm1 = 1.0 / (gm - 1.0)
    inv_mu = 1.0 / c.mu
    dx1, dx2, _ = c.dx()
    idx1, idx2 = 1.0 / dx1, 1.0 / dx2
    nx, ny = c.nx1, c.nx2
    I = (slice(G, G + nx), slice(G, G + ny))
    W = [h.prim[v, :, :, 0].copy() for v in range(4)]
    eint = h.temp[:, :, 0].copy()
    # step-0 thermodynamics (ideal gas)
    rho = W[0][I]
    p = W[3][I]
    eint = p * igmm1
    temp = p / (RGAS * rho * inv_mu)
    eq_r = h.eq_prim_cc[0, :, :, 0][I]
    eq_p = h.eq_prim_cc[1, :, :, 0][I]
    phi_cc = h.phi_cc[:, :, 0][I]
    gy = h.grav[1, :, :, 0][I]
    gx = h.grav[0, :, :, 0][I]
    erx, epx, phx = h.eq_prim_x[0][0, :, :, 0], h.eq_prim_x[0][1, :, :, 0], h.phi_x[0][:, :, 0]
    ery, epy, phy = h.eq_prim_x[1][0, :, :, 0], h.eq_prim_x[1][1, :, :, 0], h.phi_x[1][:, :, 0]

    def cfl_dt(W):
        r, v1, v2, pp = (w[I] for w in W)
        cs = np.sqrt(gm * pp / r)
        s = (np.abs(v1) + cs) * idx1 + (np.abs(v2) + cs) * idx2
        smax = s.max()
        return c.cfl / smax

    dt = cfl_dt(W) if dt is None else dt
    rk = [(1.0, 0.0, -1.0), (0.75, 0.25, -0.25), (1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0))]
    for _ in range(nsteps):
        r, v1, v2 = W[0][I].copy(), W[1][I].copy(), W[2][I].copy()
        U0 = [r, r * v1, r * v2, eint + 0.5 * r * (v1 * v1 + v2 * v2 + 0.0 * 0.0) + r * phi_cc]
        U = [u.copy() for u in U0]
        for a1, a2, c3 in rk:
            Wd = [w.copy() for w in W]
            Wd[0][I] = W[0][I] - eq_r
            Wd[3][I] = W[3][I] - eq_p
            for v in range(4):
                _fill(Wd[v], v == 2, G)
            if eps_sf is not None:
                fl = _flags(Wd[3] + h.eq_prim_cc[1, :, :, 0], G, nx, ny, eps_sf)
            # x1 sweep: faces i = 0..nx (index of the low face of interior cell i)
            lo, hi = zip(*[_rec([w[G - 3 + o:G + nx - 1 + o, G:G + ny] if G - 3 + o >= 0 else None
                                 for o in range(5)], rec, False) for w in Wd])
            qL = [x[0:nx + 1] for x in hi]
            qR = [x[1:nx + 2] for x in lo]
            qL[0] = qL[0] + erx
            qR[0] = qR[0] + erx
            qL[3] = qL[3] + epx
            qR[3] = qR[3] + epx
            F = _lhllc(qL, qR, gm, c.mach_cutoff)
            if eps_sf is not None:
                flat = fl[0:nx + 1, 1:ny + 1] | fl[1:nx + 2, 1:ny + 1]
                F = [np.where(flat, a, b) for a, b in zip(_hll(qL, qR, gm), F)]
            F[1] = F[1] - epx
            F[3] = F[3] + F[0] * phx
            res = [(f[1:] - f[:-1]) * idx1 for f in F]
            # x2 sweep with rotation (v1, v2) <- (v2, -v1)
            lo, hi = zip(*[_rec([w[G:G + nx, G - 3 + o:G + ny - 1 + o] if G - 3 + o >= 0 else None
                                 for o in range(5)], rec, False) for w in Wd])
            qL = [x[:, 0:ny + 1] for x in hi]
            qR = [x[:, 1:ny + 2] for x in lo]
            qL = [qL[0], qL[2], -qL[1], qL[3]]
            qR = [qR[0], qR[2], -qR[1], qR[3]]
            qL[0] = qL[0] + ery
            qR[0] = qR[0] + ery
            qL[3] = qL[3] + epy
            qR[3] = qR[3] + epy
            F = _lhllc(qL, qR, gm, c.mach_cutoff)
            if eps_sf is not None:
                flat = fl[1:nx + 1, 0:ny + 1] | fl[1:nx + 1, 1:ny + 2]
                F = [np.where(flat, a, b) for a, b in zip(_hll(qL, qR, gm), F)]
            F = [F[0], -F[2], F[1], F[3]]
            F[2] = F[2] - epy
            F[3] = F[3] + F[0] * phy
            res = [rr + (f[:, 1:] - f[:, :-1]) * idx2 for rr, f in zip(res, F)]
            rdev = Wd[0][I]
            res[1] = res[1] - rdev * gx
            res[2] = res[2] - rdev * gy
            a3 = c3 * dt
            U = [a1 * u0 + a2 * u + a3 * rr for u0, u, rr in zip(U0, U, res)]
            rho = U[0]
            inv_rho = 1.0 / rho
            e = U[3] - 0.5 * (U[1] * U[1] + U[2] * U[2] + 0.0 * 0.0) * inv_rho
            e = e - rho * phi_cc
            p = (gm - 1.0) * e
            W[0][I] = rho
            W[1][I] = U[1] * inv_rho
            W[2][I] = U[2] * inv_rho
            W[3][I] = p
            temp = p / (rho * RGAS * inv_mu)
            eint = e
        dt = cfl_dt(W)
    return W, eint, temp, dt


# ------------------------------------------------------------------------------ ideal MHD
def _hlld(qL, qR, bL, bR, gm, mach_cutoff, low_mach, xL=(), xR=(), fasteos=None, side_eos=None, flat=None,
          all_mach=False):
    """HLLD (low_mach False, HLLD_FLUX) or LHLLD (low_mach True, LHLLD_FLUX) flux of one face
    array in the face frame, ideal gas (S:13969-15024).  q = (rho, v1, v2, v3, p), b = (B
    normal, B transverse 2, B transverse 3); in 2D v3 and B3 are zero arrays, as the reference
    sets them; x the passive scalars' edge values; fasteos = (gamma_e L, gamma_c L, gamma_e R,
    gamma_c R) replaces the ideal gas by USE_FASTEOS's face gammas (e = p / (gamma_e - 1),
    c^2 = gamma_c p / rho); side_eos = (e L, c^2 L, e R, c^2 R) takes each side's internal
    energy and sound speed squared as given (the Helmholtz solves without USE_FASTEOS); flat
    marks the faces of USE_SHOCK_FLATTENING, which take the two-wave HLL flux with
    sL = min(0, sL), sR = max(0, sR) (S:14386-14493); all_mach: FLUX_IS_ALL_MACH, LHLLD's
    fan extended by the outer states L (sL > 0) and R (sR <= 0) (S:14576-14661).  Returns the
    fluxes (rho, m1, m2, m3, E, then one per scalar) and fluxb(2), fluxb(3)."""
    (F, hF), (fb, hfb) = _hlld_fan(qL, qR, bL, bR, gm, mach_cutoff, low_mach, xL, xR, fasteos, side_eos,
                                   all_mach)
    if flat is None:
        return F, fb
    return [np.where(flat, a, b) for a, b in zip(hF, F)], [np.where(flat, a, b) for a, b in zip(hfb, fb)]


def _hlld_fan(qL, qR, bL, bR, gm, mach_cutoff, low_mach, xL, xR, fasteos, side_eos, all_mach=False):
    """`_hlld`'s arithmetic; returns ((F, HLL F), (fb, HLL fb))."""
    igmm1 = 1.0 / (gm - 1.0)
    rhoL, v1L, v2L, v3L, pL = qL
    rhoR, v1R, v2R, v3R, pR = qR
    iL = 1.0 / rhoL
    iR = 1.0 / rhoR
    v2sL = v1L * v1L + v2L * v2L + v3L * v3L
    v2sR = v1R * v1R + v2R * v2R + v3R * v3R
    if side_eos is not None:
        eL, c2L, eR, c2R = side_eos
        reL = eL + 0.5 * rhoL * v2sL
        reR = eR + 0.5 * rhoR * v2sR
    elif fasteos is None:
        c2L = gm * pL * iL
        c2R = gm * pR * iR
        reL = pL * igmm1 + 0.5 * rhoL * v2sL
        reR = pR * igmm1 + 0.5 * rhoR * v2sR
    else:
        geL, gcL, geR, gcR = fasteos
        reL = pL / (geL - 1.0) + 0.5 * rhoL * v2sL
        c2L = gcL * pL * iL
        reR = pR / (geR - 1.0) + 0.5 * rhoR * v2sR
        c2R = gcR * pR * iR
    b2L, b2R, b3L, b3R = bL[1], bR[1], bL[2], bR[2]
    bx1 = 0.5 * (bL[0] + bR[0])
    bx1_2 = bx1 * bx1
    pbL = 0.5 * (bx1_2 + b2L * b2L + b3L * b3L)
    pbR = 0.5 * (bx1_2 + b2R * b2R + b3R * b3R)
    reL = reL + pbL
    reR = reR + pbR
    ptL = pL + pbL
    ptR = pR + pbR
    a2L = 2.0 * pbL * iL
    a2R = 2.0 * pbR * iR
    an2L = bx1_2 * iL
    an2R = bx1_2 * iR
    d = c2L + a2L
    cL = np.sqrt(0.5 * (c2L + a2L + np.sqrt(d * d - 4.0 * c2L * an2L)))
    d = c2R + a2R
    cR = np.sqrt(0.5 * (c2R + a2R + np.sqrt(d * d - 4.0 * c2R * an2R)))
    mc = np.maximum(cL, cR)
    sL = np.minimum(v1L, v1R) - mc
    sR = np.maximum(v1L, v1R) + mc
    # the flattened faces' HLL flux
    hsL = np.minimum(0.0, sL)
    hsR = np.maximum(0.0, sR)
    hUL = [rhoL, rhoL * v1L, rhoL * v2L, rhoL * v3L, reL] + [rhoL * a for a in xL]
    hUR = [rhoR, rhoR * v1R, rhoR * v2R, rhoR * v3R, reR] + [rhoR * a for a in xR]
    hfL = [rhoL * v1L, rhoL * v1L * v1L + ptL - bx1_2, rhoL * v1L * v2L - bx1 * b2L, rhoL * v1L * v3L - bx1 * b3L,
           (reL + ptL) * v1L - bx1 * (bx1 * v1L + b2L * v2L + b3L * v3L)] + [u * v1L for u in hUL[5:]]
    hfR = [rhoR * v1R, rhoR * v1R * v1R + ptR - bx1_2, rhoR * v1R * v2R - bx1 * b2R, rhoR * v1R * v3R - bx1 * b3R,
           (reR + ptR) * v1R - bx1 * (bx1 * v1R + b2R * v2R + b3R * v3R)] + [u * v1R for u in hUR[5:]]
    hd = 1.0 / (hsR - hsL)
    hph = hsL * hsR
    hF = [hd * (hsR * a - hsL * b + hph * (ur - ul)) for a, b, ul, ur in zip(hfL, hfR, hUL, hUR)]
    hfb = [hd * (hsR * (v1L * b2L - v2L * bx1) - hsL * (v1R * b2R - v2R * bx1) + hph * (b2R - b2L)),
           hd * (hsR * (v1L * b3L - v3L * bx1) - hsL * (v1R * b3R - v3R * bx1) + hph * (b3R - b3L))]
    dsuL = sL - v1L
    dsuR = sR - v1R
    it1 = 1.0 / (dsuR * rhoR - dsuL * rhoL)
    us = (dsuR * rhoR * v1R - dsuL * rhoL * v1L - ptR + ptL) * it1
    dsumL = sL - us
    dsumR = sR - us
    if low_mach:
        d = v2sL + a2L
        cu2L = 0.5 * (v2sL + a2L + np.sqrt(d * d - 4.0 * v2sL * an2L))
        d = v2sR + a2R
        cu2R = 0.5 * (v2sR + a2R + np.sqrt(d * d - 4.0 * v2sR * an2R))
        mL = np.sqrt(cu2L) / cL
        mR = np.sqrt(cu2R) / cR
        mmax = np.maximum(mL, mR)
        chi = np.maximum(mach_cutoff, np.minimum(1.0, mmax))
        phi = np.where(mmax < 0.6, chi * (2.0 - chi), 1.0)
    else:
        phi = 1.0
    pst = (dsuR * rhoR * ptL - dsuL * rhoL * ptR - phi * rhoL * rhoR * dsuR * dsuL * (v1L - v1R)) * it1
    rsL = rhoL * dsuL / dsumL
    rsR = rhoR * dsuR / dsumR
    a1i = 1.0 / (rhoL * dsuL * dsumL - bx1_2)
    v2sL_ = v2L - bx1 * b2L * (us - v1L) * a1i
    b2sL = b2L * (rhoL * dsuL * dsuL - bx1_2) * a1i
    v3sL = v3L - bx1 * b3L * (us - v1L) * a1i
    b3sL = b3L * (rhoL * dsuL * dsuL - bx1_2) * a1i
    a2i = 1.0 / (rhoR * dsuR * dsumR - bx1_2)
    v2sR_ = v2R - bx1 * b2R * (us - v1R) * a2i
    b2sR = b2R * (rhoR * dsuR * dsuR - bx1_2) * a2i
    v3sR = v3R - bx1 * b3R * (us - v1R) * a2i
    b3sR = b3R * (rhoR * dsuR * dsuR - bx1_2) * a2i
    vbL = v1L * bx1 + v2L * b2L + v3L * b3L
    vbR = v1R * bx1 + v2R * b2R + v3R * b3R
    vbsL = us * bx1 + v2sL_ * b2sL + v3sL * b3sL
    vbsR = us * bx1 + v2sR_ * b2sR + v3sR * b3sR
    resL = (dsuL * reL - ptL * v1L + pst * us + bx1 * (vbL - vbsL)) / dsumL
    resR = (dsuR * reR - ptR * v1R + pst * us + bx1 * (vbR - vbsR)) / dsumR
    srL = np.sqrt(rsL)
    srR = np.sqrt(rsR)
    ab = np.abs(bx1)
    ssL = us - ab / srL
    ssR = us + ab / srR
    isb = 1.0 / (srL + srR)
    sgn = np.copysign(1.0, bx1)
    v22 = (srL * v2sL_ + srR * v2sR_ + (b2sR - b2sL) * sgn) * isb
    b22 = (srL * b2sR + srR * b2sL + srL * srR * (v2sR_ - v2sL_) * sgn) * isb
    v32 = (srL * v3sL + srR * v3sR + (b3sR - b3sL) * sgn) * isb
    b32 = (srL * b3sR + srR * b3sL + srL * srR * (v3sR - v3sL) * sgn) * isb
    vb2 = us * bx1 + v22 * b22 + v32 * b32
    re2L = resL - srL * (vbsL - vb2) * sgn
    re2R = resR + srR * (vbsR - vb2) * sgn
    if low_mach:
        # the state at x/t = 0 among L*, L**, R**, R* and its physical flux
        sel = [ssL > 0.0, us > 0.0, ssR > 0.0]

        def pick(a, b, c, d):
            return np.where(sel[0], a, np.where(sel[1], b, np.where(sel[2], c, d)))
        rho = pick(rsL, rsL, rsR, rsR)
        u = us
        v2 = pick(v2sL_, v22, v22, v2sR_)
        v3 = pick(v3sL, v32, v32, v3sR)
        re = pick(resL, re2L, re2R, resR)
        b2 = pick(b2sL, b22, b22, b2sR)
        b3 = pick(b3sL, b32, b32, b3sR)
        pres = pst
        if all_mach:
            outL = sL > 0.0
            outR = ~outL & ~sel[0] & ~sel[1] & ~sel[2] & ~(sR > 0.0)

            def outer(a, l_, r_):
                return np.where(outL, l_, np.where(outR, r_, a))
            rho, u, v2, v3 = outer(rho, rhoL, rhoR), outer(u, v1L, v1R), outer(v2, v2L, v2R), outer(v3, v3L, v3R)
            re, b2, b3, pres = outer(re, reL, reR), outer(b2, b2L, b2R), outer(b3, b3L, b3R), outer(pst, ptL, ptR)
        F = [rho * u, rho * u * u + pres - bx1_2, rho * u * v2 - bx1 * b2, rho * u * v3 - bx1 * b3,
             (re + pres) * u - bx1 * (bx1 * u + v2 * b2 + v3 * b3)]
        up = np.copysign(1.0, u)
        hp = 0.5 * (1.0 + up)
        hm = 0.5 * (1.0 - up)
        F += [rho * u * (hp * a + hm * b) for a, b in zip(xL, xR)]
        return (F, hF), ([u * b2 - bx1 * v2, u * b3 - bx1 * v3], hfb)
    # HLLD: f + s (U* - U) + s* (U** - U*) on the side of u*
    out = []
    for side in ("L", "R"):
        if side == "L":
            rho_, v1_, v2_, v3_, re_, pt_, b2_, b3_, vb_ = rhoL, v1L, v2L, v3L, reL, ptL, b2L, b3L, vbL
            s, ss, rs, v2s, v3s, b2s, b3s, res_ = sL, ssL, rsL, v2sL_, v3sL, b2sL, b3sL, resL
            ress, xs = re2L, xL
        else:
            rho_, v1_, v2_, v3_, re_, pt_, b2_, b3_, vb_ = rhoR, v1R, v2R, v3R, reR, ptR, b2R, b3R, vbR
            s, ss, rs, v2s, v3s, b2s, b3s, res_ = sR, ssR, rsR, v2sR_, v3sR, b2sR, b3sR, resR
            ress, xs = re2R, xR
        U = [rho_, rho_ * v1_, rho_ * v2_, rho_ * v3_, re_, b2_, b3_] + [rho_ * x for x in xs]
        f = [rho_ * v1_, rho_ * v1_ * v1_ + pt_ - bx1_2, rho_ * v1_ * v2_ - bx1 * b2_,
             rho_ * v1_ * v3_ - bx1 * b3_, (re_ + pt_) * v1_ - bx1 * vb_,
             v1_ * b2_ - bx1 * v2_, v1_ * b3_ - bx1 * v3_] + [rho_ * v1_ * x for x in xs]
        Us = [rs, rs * us, rs * v2s, rs * v3s, res_, b2s, b3s] + [rs * x for x in xs]
        Uss = [rs, rs * us, rs * v22, rs * v32, ress, b22, b32] + [rs * x for x in xs]
        outer = (s > 0.0) if side == "L" else (s < 0.0)
        inner = (ss > 0.0) if side == "L" else (ss < 0.0)
        out.append([np.where(outer, fi, np.where(inner, fi + s * (a - u0), fi + s * (a - u0) + ss * (b - a)))
                    for fi, u0, a, b in zip(f, U, Us, Uss)])
    left = us > 0.0
    F = [np.where(left, a, b) for a, b in zip(out[0], out[1])]
    return (F[:5] + F[7:], hF), (F[5:7], hfb)


def _fill_periodic(a, G):
    nx = a.shape[0] - 2 * G
    ny = a.shape[1] - 2 * G
    a[:G, :] = a[nx:nx + G, :]
    a[nx + G:, :] = a[G:2 * G, :]
    a[:, :G] = a[:, ny:ny + G]
    a[:, ny + G:] = a[:, G:2 * G]


def mhd_2d_steps(h, nsteps, low_mach):
    """Advance a 2D periodic ideal-gas MHD HostGrid `h` (LIM2ND, RK, no WB / gravity / scalars)
    in place of copies with HLLD (low_mach False) or LHLLD (True) and constrained transport:
    face EMFs and mass-flux signs (S:8926-8951, S:10101-10144), the upwinded corner EMF
    (S:11970-12029), the face-B update (S:12258-12380) and b_cc (S:12440-12470), the magnetic
    energy in prim->cons and cons->prim (S:7057-7117, S:13533-13560) and the magnetosonic CFL
    bound (S:13827-13836).  Returns (W, eint, temp, b1, b2, dt): padded primitives, interior
    eint and T, interior face fields (nx+1, ny) and (nx, ny+1), and the next dt."""
    c = h.cfg
    G = c.ngc
    gm = c.gamma_ad
    igmm1 = 1.0 / (gm - 1.0)
    inv_mu = 1.0 / c.mu
    dx1, dx2, _ = c.dx()
    idx1, idx2 = 1.0 / dx1, 1.0 / dx2
    nx, ny = c.nx1, c.nx2
    I = (slice(G, G + nx), slice(G, G + ny))
    W = [h.prim[v, :, :, 0].copy() for v in range(4)]
    b1 = h.b_x[0][1:nx + 2, 1:ny + 1, 0].copy()
    b2 = h.b_x[1][1:nx + 1, 1:ny + 2, 0].copy()
    B = [np.zeros_like(W[0]), np.zeros_like(W[0])]

    def cell_b():
        B[0][I] = 0.5 * (b1[1:] + b1[:-1])
        B[1][I] = 0.5 * (b2[:, 1:] + b2[:, :-1])
        for a in B:
            _fill_periodic(a, G)

    cell_b()
    eint = W[3][I] * igmm1
    temp = W[3][I] / (RGAS * W[0][I] * inv_mu)

    def cfl():
        r, v1, v2, pp = (w[I] for w in W)
        cs = np.sqrt(gm * pp / r)
        ca2 = B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0
        cs = np.sqrt(cs * cs + ca2 / r)
        smax = ((np.abs(v1) + cs) * idx1 + (np.abs(v2) + cs) * idx2).max()
        return smax, c.cfl / smax

    def mass_sign(f, rl, rr, smax):
        m = f / (0.5 * (rl + rr) * smax)
        return np.where(m > c.mach_ct, 1.0, np.where(m < -c.mach_ct, -1.0, 0.0))

    smax, dt = cfl()
    # RK2_STEPPER / RK3_STEPPER coefficients (S:7018-7038)
    rk = {2: [(1.0, 0.0, -1.0), (0.5, 0.5, -0.5)],
          3: [(1.0, 0.0, -1.0), (0.75, 0.25, -0.25), (1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0))]}[c.rk_stages]
    for _ in range(nsteps):
        r, v1, v2 = W[0][I].copy(), W[1][I].copy(), W[2][I].copy()
        U0 = [r, r * v1, r * v2,
              eint + 0.5 * r * (v1 * v1 + v2 * v2 + 0.0 * 0.0)
              + 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0)]
        U = [u.copy() for u in U0]
        b10, b20 = b1.copy(), b2.copy()
        for a1, a2, c3 in rk:
            for w in W:
                _fill_periodic(w, G)
            # x1 faces i = 1..nx+1: cells G-1+f | G+f
            lo, hi = zip(*[_plm(w[G - 2:G + nx, G:G + ny], w[G - 1:G + nx + 1, G:G + ny], w[G:G + nx + 2, G:G + ny])
                           for w in W + [B[1]]])
            qL = [x[0:nx + 1] for x in hi[:4]]
            qR = [x[1:nx + 2] for x in lo[:4]]
            z = np.zeros_like(b1)
            F, fb = _hlld(qL[:3] + [z, qL[3]], qR[:3] + [z, qR[3]], [b1, hi[4][0:nx + 1], z],
                          [b1, lo[4][1:nx + 2], z], gm, c.mach_cutoff, low_mach)
            F = F[:3] + F[4:]
            e1 = -fb[0]
            s1 = mass_sign(F[0], qL[0], qR[0], smax)
            res = [(f[1:] - f[:-1]) * idx1 for f in F]
            # x2 faces with (v1, v2) -> (v2, -v1) and (B1, B2) -> (B2, -B1)
            lo, hi = zip(*[_plm(w[G:G + nx, G - 2:G + ny], w[G:G + nx, G - 1:G + ny + 1], w[G:G + nx, G:G + ny + 2])
                           for w in W + [B[0]]])
            qL = [x[:, 0:ny + 1] for x in hi[:4]]
            qR = [x[:, 1:ny + 2] for x in lo[:4]]
            qL = [qL[0], qL[2], -qL[1], qL[3]]
            qR = [qR[0], qR[2], -qR[1], qR[3]]
            z = np.zeros_like(b2)
            F, fb = _hlld(qL[:3] + [z, qL[3]], qR[:3] + [z, qR[3]], [b2, -hi[4][:, 0:ny + 1], z],
                          [b2, -lo[4][:, 1:ny + 2], z], gm, c.mach_cutoff, low_mach)
            F = [F[0], -F[2], F[1], F[4]]
            e2 = -fb[0]
            s2 = mass_sign(F[0], qL[0], qR[0], smax)
            res = [rr + (f[:, 1:] - f[:, :-1]) * idx2 for rr, f in zip(res, F)]
            # corner EMFs (i = 1..nx+1, j = 1..ny+1), face arrays wrapped by one layer
            e1x = np.concatenate([e1[:, -1:], e1, e1[:, :1]], axis=1)
            s1x = np.concatenate([s1[:, -1:], s1, s1[:, :1]], axis=1)
            e2x = np.concatenate([e2[-1:], e2, e2[:1]], axis=0)
            s2x = np.concatenate([s2[-1:], s2, s2[:1]], axis=0)
            ec = -W[1] * B[1] + W[2] * B[0]
            eN, eS = e1x[:, 1:], e1x[:, :-1]
            eE, eW = e2x[1:], e2x[:-1]
            eSW = ec[G - 1:G + nx, G - 1:G + ny]
            eNW = ec[G - 1:G + nx, G:G + ny + 1]
            eNE = ec[G:G + nx + 1, G:G + ny + 1]
            eSE = ec[G:G + nx + 1, G - 1:G + ny]
            sg = s1x[:, :-1]
            dS = 0.5 * (1.0 + sg) * (eW - eSW) + 0.5 * (1.0 - sg) * (eE - eSE)
            sg = s1x[:, 1:]
            dN = 0.5 * (1.0 + sg) * (eNW - eW) + 0.5 * (1.0 - sg) * (eNE - eE)
            sg = s2x[:-1]
            dW = 0.5 * (1.0 + sg) * (eS - eSW) + 0.5 * (1.0 - sg) * (eN - eNW)
            sg = s2x[1:]
            dE = 0.5 * (1.0 + sg) * (eSE - eS) + 0.5 * (1.0 - sg) * (eNE - eN)
            cor = 0.25 * (eS + eW + eN + eE + dS - dN + dW - dE)
            a3 = c3 * dt
            b1 = a1 * b10 + a2 * b1 + a3 * ((cor[:, 1:] - cor[:, :-1]) * idx2)
            b2 = a1 * b20 + a2 * b2 + a3 * ((cor[:-1] - cor[1:]) * idx1)
            cell_b()
            U = [a1 * u0 + a2 * u + a3 * rr for u0, u, rr in zip(U0, U, res)]
            rho = U[0]
            inv_rho = 1.0 / rho
            e = U[3] - 0.5 * (U[1] * U[1] + U[2] * U[2] + 0.0 * 0.0) * inv_rho
            e = e - 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0)
            p = (gm - 1.0) * e
            W[0][I] = rho
            W[1][I] = U[1] * inv_rho
            W[2][I] = U[2] * inv_rho
            W[3][I] = p
            temp = p / (rho * RGAS * inv_mu)
            eint = e
        smax, dt = cfl()
    return W, eint, temp, b1, b2, dt


def _hllc3(qL, qR, gm, mach_cutoff, low_mach, all_mach=False, xL=(), xR=(), fasteos=None, side_eos=None,
           flat=None):
    """LHLLC (low_mach True) or HLLC flux of one face array in the face frame, 3D with
    scalars (S:15611-16260): q = (rho, v1, v2, v3, p); the side EoS as in `_hlld` (here
    side_eos carries the sound speed itself, as helm_rhoP_given returns it); all_mach:
    FLUX_IS_ALL_MACH, the upwind state's flux outside the fan (LHLLC only); flat: the faces of
    USE_SHOCK_FLATTENING, with the HLL flux (S:15929-16008)."""
    F, hF = _hllc3_fan(qL, qR, gm, mach_cutoff, low_mach, all_mach, xL, xR, fasteos, side_eos)
    return F if flat is None else [np.where(flat, a, b) for a, b in zip(hF, F)]


def _hllc3_fan(qL, qR, gm, mach_cutoff, low_mach, all_mach, xL, xR, fasteos, side_eos):
    """`_hllc3`'s arithmetic; returns (F, HLL F)."""
    rhoL, v1L, v2L, v3L, pL = qL
    rhoR, v1R, v2R, v3R, pR = qR
    iL = 1.0 / rhoL
    iR = 1.0 / rhoR
    w2L = v1L * v1L + v2L * v2L + v3L * v3L
    w2R = v1R * v1R + v2R * v2R + v3R * v3R
    if side_eos is not None:
        eL, cL, eR, cR = side_eos
    elif fasteos is not None:
        geL, gcL, geR, gcR = fasteos
        eL = pL / (geL - 1.0)
        cL = np.sqrt(gcL * pL * iL)
        eR = pR / (geR - 1.0)
        cR = np.sqrt(gcR * pR * iR)
    else:
        igmm1 = 1.0 / (gm - 1.0)
        eL = igmm1 * pL
        cL = np.sqrt(gm * pL * iL)
        eR = igmm1 * pR
        cR = np.sqrt(gm * pR * iR)
    reL = eL + 0.5 * rhoL * w2L
    reR = eR + 0.5 * rhoR * w2R
    mc = np.maximum(cL, cR)
    sL = np.minimum(v1L, v1R) - mc
    sR = np.maximum(v1L, v1R) + mc
    dL = sL - v1L
    dR = sR - v1R
    us = (pR - pL + rhoL * v1L * dL - rhoR * v1R * dR) / (rhoL * dL - rhoR * dR)
    rsL = rhoL * (dL / (sL - us))
    resL = rsL * (reL * iL + (us - v1L) * (us + pL * iL / dL))
    rsR = rhoR * (dR / (sR - us))
    resR = rsR * (reR * iR + (us - v1R) * (us + pR * iR / dR))
    hsL = np.minimum(0.0, sL)
    hsR = np.maximum(0.0, sR)
    hUL = [rhoL, rhoL * v1L, rhoL * v2L, rhoL * v3L, reL] + [rhoL * a for a in xL]
    hUR = [rhoR, rhoR * v1R, rhoR * v2R, rhoR * v3R, reR] + [rhoR * a for a in xR]
    hfL = [rhoL * v1L, rhoL * v1L * v1L + pL, rhoL * v1L * v2L, rhoL * v1L * v3L, (reL + pL) * v1L]
    hfL += [u * v1L for u in hUL[5:]]
    hfR = [rhoR * v1R, rhoR * v1R * v1R + pR, rhoR * v1R * v2R, rhoR * v1R * v3R, (reR + pR) * v1R]
    hfR += [u * v1R for u in hUR[5:]]
    hd = 1.0 / (hsR - hsL)
    hph = hsL * hsR
    hF = [hd * (hsR * a - hsL * b + hph * (ur - ul)) for a, b, ul, ur in zip(hfL, hfR, hUL, hUR)]
    if low_mach:
        chi = np.maximum(mach_cutoff, np.minimum(1.0, np.maximum(np.sqrt(w2L) / cL, np.sqrt(w2R) / cR)))
        phi = chi * (2.0 - chi)
        pst = 0.5 * (pL + pR) - 0.5 * phi * (0.5 * (rhoL + rhoR)) * (0.5 * (cL + cR)) * (v1R - v1L)
        sg = np.copysign(1.0, us)
        hp = 0.5 * (1.0 + sg)
        hm = 0.5 * (1.0 - sg)
        rs = hp * rsL + hm * rsR
        F = [rs * us, rs * us * us + pst, rs * us * (hp * v2L + hm * v2R), rs * us * (hp * v3L + hm * v3R),
             (hp * resL + hm * resR + pst) * us] + [rs * us * (hp * a + hm * b) for a, b in zip(xL, xR)]
        if all_mach:
            fL = [rhoL * v1L, rhoL * v1L * v1L + pL, rhoL * v1L * v2L, rhoL * v1L * v3L, (reL + pL) * v1L]
            fL += [rhoL * a * v1L for a in xL]
            fR = [rhoR * v1R, rhoR * v1R * v1R + pR, rhoR * v1R * v2R, rhoR * v1R * v3R, (reR + pR) * v1R]
            fR += [rhoR * a * v1R for a in xR]
            F = [np.where(sL > 0.0, a, np.where(sR < 0.0, b, c)) for a, b, c in zip(fL, fR, F)]
        return F, hF
    out = []
    for side in ("L", "R"):
        rho_, v1_, v2_, v3_, re_, p_, x_, s, rs, res_ = (
            (rhoL, v1L, v2L, v3L, reL, pL, xL, sL, rsL, resL) if side == "L" else
            (rhoR, v1R, v2R, v3R, reR, pR, xR, sR, rsR, resR))
        U = [rho_, rho_ * v1_, rho_ * v2_, rho_ * v3_, re_] + [rho_ * a for a in x_]
        f = [rho_ * v1_, rho_ * v1_ * v1_ + p_, rho_ * v1_ * v2_, rho_ * v1_ * v3_, (re_ + p_) * v1_]
        f += [rho_ * v1_ * a for a in x_]
        Us = [rs, rs * us, rs * v2_, rs * v3_, res_] + [rs * a for a in x_]
        outer = (s >= 0.0) if side == "L" else (s < 0.0)
        out.append([np.where(outer, fi, fi + s * (a - u0)) for fi, u0, a in zip(f, U, Us)])
    return [np.where(us > 0.0, a, b) for a, b in zip(out[0], out[1])], hF


def _wrap(a, axis):
    """One periodic layer on either side of `a` along `axis` (the self-copy of a face array's
    ghost layer, S:2293-2306)."""
    n = a.shape[axis]
    return np.concatenate([np.take(a, [n - 1], axis=axis), a, np.take(a, [0], axis=axis)], axis=axis)


def _corner(eA, eB, ec, sA, sB):
    """Upwinded corner EMF (S:11970-12029 and its x1 / x2 counterparts) from corner-aligned
    arrays: eA / sA the face EMF and mass-flux sign of the face array that varies along the
    corner's second axis (N = eA[q], S = eA[q-1]), eB / sB of the one that varies along its
    first axis (E = eB[p], W = eB[p-1]), ec = (SW, NW, NE, SE) the cell EMFs."""
    eN, eS, eE, eW, sgN, sgS, sgE, sgW = eA[1], eA[0], eB[1], eB[0], sA[1], sA[0], sB[1], sB[0]
    eSW, eNW, eNE, eSE = ec
    dS = 0.5 * (1.0 + sgS) * (eW - eSW) + 0.5 * (1.0 - sgS) * (eE - eSE)
    dN = 0.5 * (1.0 + sgN) * (eNW - eW) + 0.5 * (1.0 - sgN) * (eNE - eE)
    dW = 0.5 * (1.0 + sgW) * (eS - eSW) + 0.5 * (1.0 - sgW) * (eN - eNW)
    dE = 0.5 * (1.0 + sgE) * (eSE - eS) + 0.5 * (1.0 - sgE) * (eNE - eN)
    return 0.25 * (eS + eW + eN + eE + dS - dN + dW - dE)


class PeriodicHalo:
    """The ghost exchange of one triply periodic domain: the three operations
    `mhd_3d_steps` delegates, so that a decomposition can replace them."""

    dx = None                    # cell sizes; None: the configuration's

    @staticmethod
    def fill(a, G):
        """Ghost cells of a padded cell array."""
        _fill_periodic3(a, G)

    @staticmethod
    def wrap3(e):
        """One ghost layer along x3 of a face array whose x3 index is a cell index."""
        return _wrap(e, 2)

    @staticmethod
    def max(x):
        """The maximum over the whole domain of a local maximum (the dt reduction)."""
        return x


def mhd_3d_steps(h, nsteps, low_mach, halo=PeriodicHalo):
    """The 3D counterpart of `mhd_2d_steps` on a triply periodic box: the x2 and x3 frame
    rotations of states, fluxes and B (S:9715-9747, S:10101-10144, S:10845-10889,
    S:11241-11286), all three face-EMF components (S:8926-8951 and counterparts), the three
    corner EMFs (S:11970-12200), the three face-B updates (S:12258-12432) and the 3D dt sum
    sx3 + sx1 + sx2, with the passive scalars the configuration carries (upwinded by the sign
    of the contact speed) and its reconstruction (LIM2ND, PPH or LIM5TH; the cell B edges by
    the same formulas, S:8327-8469), and USE_CONSTANT_ACCELERATION when the configuration sets
    it (rho acc on the momenta and its work from the stage's input state, S:12806-12834).
    `halo` supplies the ghost exchange along x3 and the dt reduction (a slab of a
    decomposed domain).  Returns (W, eint, temp, [b1, b2, b3], dt)."""
    c = h.cfg
    G = c.ngc
    gm = c.gamma_ad
    igmm1 = 1.0 / (gm - 1.0)
    inv_mu = 1.0 / c.mu
    idx = [1.0 / d for d in (halo.dx or c.dx())]
    n = [c.nx1, c.nx2, c.nx3]
    I = tuple(slice(G, G + m) for m in n)
    nv = c.nvars
    W = [h.prim[v].copy() for v in range(nv)]
    b = [h.b_x[d][tuple(slice(1, 1 + n[a] + (a == d)) for a in range(3))].copy() for d in range(3)]
    B = [np.zeros_like(W[0]) for _ in range(3)]

    def cell_b():
        B[0][I] = 0.5 * (b[0][1:] + b[0][:-1])
        B[1][I] = 0.5 * (b[1][:, 1:] + b[1][:, :-1])
        B[2][I] = 0.5 * (b[2][:, :, 1:] + b[2][:, :, :-1])
        for a in B:
            halo.fill(a, G)

    cell_b()
    eint = W[4][I] * igmm1
    temp = W[4][I] / (RGAS * W[0][I] * inv_mu)

    def cfl():
        r, v1, v2, v3, pp = (w[I] for w in W[:5])
        cs = np.sqrt(gm * pp / r)
        ca2 = B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I]
        cs = np.sqrt(cs * cs + ca2 / r)
        sx1 = (np.abs(v1) + cs) * idx[0]
        sx2 = (np.abs(v2) + cs) * idx[1]
        sx3 = (np.abs(v3) + cs) * idx[2]
        smax = halo.max((sx3 + sx1 + sx2).max())
        return smax, c.cfl / smax

    def mass_sign(f, rl, rr, smax):
        m = f / (0.5 * (rl + rr) * smax)
        return np.where(m > c.mach_ct, 1.0, np.where(m < -c.mach_ct, -1.0, 0.0))

    def along(a, lo, hi):
        return tuple(slice(lo, hi) if x == a else I[x] for x in range(3))

    def sweep(a, trans):
        """Edge states of the faces normal to axis a (face f between padded cells G-1+f and
        G+f) for the five primitives and the two transverse cell-B components `trans`; with
        PPH only the scalars are limited."""
        m = n[a]
        arrs = W + [B[t] for t in trans]
        lim = [c.rec == "lim5th" or (c.rec == "pph" and 5 <= v < nv) for v in range(len(arrs))]
        lo, hi = zip(*[_rec([w[along(a, G - 3 + o, G + m - 1 + o)] if G - 3 + o >= 0 else None for o in range(5)],
                            c.rec, lv) for w, lv in zip(arrs, lim)])
        L = [np.take(x, range(0, m + 1), axis=a) for x in hi]
        R = [np.take(x, range(1, m + 2), axis=a) for x in lo]
        # primitives, transverse cell B, scalars
        return L[:5] + L[nv:] + L[5:nv], R[:5] + R[nv:] + R[5:nv]

    smax, dt = cfl()
    rk = {2: [(1.0, 0.0, -1.0), (0.5, 0.5, -0.5)],
          3: [(1.0, 0.0, -1.0), (0.75, 0.25, -0.25), (1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0))]}[c.rk_stages]
    for _ in range(nsteps):
        r, v1, v2, v3 = (W[v][I].copy() for v in range(4))
        U0 = [r, r * v1, r * v2, r * v3,
              eint + 0.5 * r * (v1 * v1 + v2 * v2 + v3 * v3)
              + 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I])]
        U0 += [r * W[v][I] for v in range(5, nv)]
        U = [u.copy() for u in U0]
        b0 = [x.copy() for x in b]
        for a1, a2, c3 in rk:
            for w in W:
                halo.fill(w, G)
            emf = [None, None, None]
            sgn = [None, None, None]
            res = None
            for a in range(3):
                trans = [t for t in range(3) if t != a]
                L, R = sweep(a, trans)
                # face frame: x1 as is, x2 (v1, v2, v3) -> (v2, -v1, v3), x3 -> (v3, v1, v2)
                if a == 0:
                    qL, qR = L[:5], R[:5]
                    bL, bR = [b[0], L[5], L[6]], [b[0], R[5], R[6]]
                elif a == 1:
                    qL = [L[0], L[2], -L[1], L[3], L[4]]
                    qR = [R[0], R[2], -R[1], R[3], R[4]]
                    bL, bR = [b[1], -L[5], L[6]], [b[1], -R[5], R[6]]
                else:
                    qL = [L[0], L[3], L[1], L[2], L[4]]
                    qR = [R[0], R[3], R[1], R[2], R[4]]
                    bL, bR = [b[2], L[5], L[6]], [b[2], R[5], R[6]]
                F, fb = _hlld(qL, qR, bL, bR, gm, c.mach_cutoff, low_mach, L[7:], R[7:], all_mach=c.all_mach)
                if a == 0:
                    emf[0] = (None, fb[1], -fb[0])
                elif a == 1:
                    F = [F[0], -F[2], F[1]] + F[3:]
                    emf[1] = (-fb[1], None, -fb[0])
                else:
                    F = [F[0], F[2], F[3], F[1]] + F[4:]
                    emf[2] = (fb[1], -fb[0], None)
                sgn[a] = mass_sign(F[0], qL[0], qR[0], smax)
                div = [np.diff(f, axis=a) * idx[a] for f in F]
                res = div if res is None else [rr + d for rr, d in zip(res, div)]
            if c.constant_acceleration:
                acc = c.acc
                for d in range(3):
                    res[1 + d] = res[1 + d] - U[0] * acc[d]
                res[4] = res[4] - U[3] * acc[2] - U[1] * acc[0] - U[2] * acc[1]
            # cell EMFs at the padded cells, then the corners of each axis
            ec3 = -W[1] * B[1] + W[2] * B[0]
            ec1 = W[3] * B[1] - W[2] * B[2]
            ec2 = W[1] * B[2] - W[3] * B[0]
            nx, ny, nz = n
            Ix, Iy, Iz = I
            e, s = _wrap(emf[0][2], 1), _wrap(sgn[0], 1)
            f, t = _wrap(emf[1][2], 0), _wrap(sgn[1], 0)
            cor3 = _corner((e[:, :-1], e[:, 1:]), (f[:-1], f[1:]),
                           (ec3[G - 1:G + nx, G - 1:G + ny, Iz], ec3[G - 1:G + nx, G:G + ny + 1, Iz],
                            ec3[G:G + nx + 1, G:G + ny + 1, Iz], ec3[G:G + nx + 1, G - 1:G + ny, Iz]),
                           (s[:, :-1], s[:, 1:]), (t[:-1], t[1:]))
            e, s = halo.wrap3(emf[1][0]), halo.wrap3(sgn[1])
            f, t = _wrap(emf[2][0], 1), _wrap(sgn[2], 1)
            cor1 = _corner((e[:, :, :-1], e[:, :, 1:]), (f[:, :-1], f[:, 1:]),
                           (ec1[Ix, G - 1:G + ny, G - 1:G + nz], ec1[Ix, G - 1:G + ny, G:G + nz + 1],
                            ec1[Ix, G:G + ny + 1, G:G + nz + 1], ec1[Ix, G:G + ny + 1, G - 1:G + nz]),
                           (s[:, :, :-1], s[:, :, 1:]), (t[:, :-1], t[:, 1:]))
            e, s = _wrap(emf[2][1], 0), _wrap(sgn[2], 0)
            f, t = halo.wrap3(emf[0][1]), halo.wrap3(sgn[0])
            cor2 = _corner((e[:-1], e[1:]), (f[:, :, :-1], f[:, :, 1:]),
                           (ec2[G - 1:G + nx, Iy, G - 1:G + nz], ec2[G:G + nx + 1, Iy, G - 1:G + nz],
                            ec2[G:G + nx + 1, Iy, G:G + nz + 1], ec2[G - 1:G + nx, Iy, G:G + nz + 1]),
                           (s[:-1], s[1:]), (t[:, :, :-1], t[:, :, 1:]))
            a3 = c3 * dt
            t1 = -(cor2[:, :, 1:] - cor2[:, :, :-1]) * idx[2] + (cor3[:, 1:] - cor3[:, :-1]) * idx[1]
            t2 = (cor1[:, :, 1:] - cor1[:, :, :-1]) * idx[2] + (cor3[:-1] - cor3[1:]) * idx[0]
            t3 = (cor2[1:] - cor2[:-1]) * idx[0] - (cor1[:, 1:] - cor1[:, :-1]) * idx[1]
            b = [a1 * x0 + a2 * x + a3 * tt for x0, x, tt in zip(b0, b, (t1, t2, t3))]
            cell_b()
            U = [a1 * u0 + a2 * u + a3 * rr for u0, u, rr in zip(U0, U, res)]
            rho = U[0]
            inv_rho = 1.0 / rho
            e = U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * inv_rho
            e = e - 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I])
            p = (gm - 1.0) * e
            W[0][I] = rho
            W[1][I] = U[1] * inv_rho
            W[2][I] = U[2] * inv_rho
            W[3][I] = U[3] * inv_rho
            W[4][I] = p
            for v in range(5, nv):
                W[v][I] = U[v] * inv_rho
            temp = p / (rho * RGAS * inv_mu)
            eint = e
        smax, dt = cfl()
    return W, eint, temp, b, dt


def _fill_periodic3(a, G):
    for ax in range(3):
        m = a.shape[ax] - 2 * G
        lo = [slice(None)] * 3
        src = [slice(None)] * 3
        lo[ax], src[ax] = slice(0, G), slice(m, m + G)
        a[tuple(lo)] = a[tuple(src)]
        lo[ax], src[ax] = slice(m + G, m + 2 * G), slice(G, 2 * G)
        a[tuple(lo)] = a[tuple(src)]


def wb_mhd_2d_steps(h, nsteps, low_mach):
    """The 2D MHD step with the hot bubble's well-balanced, gravitating set-up: periodic x,
    reflective y walls, USE_WB (deviations of rho and p reconstructed, S:7151-7168, and the
    equilibrium added back at the faces, S:8473-8486), EVOLVE_ETOT, gravity on rho', ideal gas;
    HLLD or LHLLD with constrained transport.  At the walls the cell values are mirrored with
    v2 and B2 negated (S:7640-7720) and the ghost face EMFs of the x1 faces take the
    reflective factor -1 on their E3 with the mass-flux sign copied (S:11494-11590).  Returns
    (W, eint, temp, b1, b2, dt)."""
    c = h.cfg
    G = c.ngc
    gm = c.gamma_ad
    igmm1 = 1.0 / (gm - 1.0)
    inv_mu = 1.0 / c.mu
    dx1, dx2, _ = c.dx()
    idx1, idx2 = 1.0 / dx1, 1.0 / dx2
    nx, ny = c.nx1, c.nx2
    I = (slice(G, G + nx), slice(G, G + ny))
    W = [h.prim[v, :, :, 0].copy() for v in range(4)]
    b1 = h.b_x[0][1:nx + 2, 1:ny + 1, 0].copy()
    b2 = h.b_x[1][1:nx + 1, 1:ny + 2, 0].copy()
    B = [np.zeros_like(W[0]), np.zeros_like(W[0])]
    eq_r = h.eq_prim_cc[0, :, :, 0][I]
    eq_p = h.eq_prim_cc[1, :, :, 0][I]
    phi_cc = h.phi_cc[:, :, 0][I]
    gx, gy = h.grav[0, :, :, 0][I], h.grav[1, :, :, 0][I]
    erx, epx, phx = h.eq_prim_x[0][0, :, :, 0], h.eq_prim_x[0][1, :, :, 0], h.phi_x[0][:, :, 0]
    ery, epy, phy = h.eq_prim_x[1][0, :, :, 0], h.eq_prim_x[1][1, :, :, 0], h.phi_x[1][:, :, 0]

    def cell_b():
        B[0][I] = 0.5 * (b1[1:] + b1[:-1])
        B[1][I] = 0.5 * (b2[:, 1:] + b2[:, :-1])
        _fill(B[0], False, G)
        _fill(B[1], True, G)

    cell_b()
    eint = W[3][I] * igmm1
    temp = W[3][I] / (RGAS * W[0][I] * inv_mu)

    def cfl():
        r, v1, v2, pp = (w[I] for w in W)
        cs = np.sqrt(gm * pp / r)
        ca2 = B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0
        cs = np.sqrt(cs * cs + ca2 / r)
        smax = ((np.abs(v1) + cs) * idx1 + (np.abs(v2) + cs) * idx2).max()
        return smax, c.cfl / smax

    def mass_sign(f, rl, rr, smax):
        m = f / (0.5 * (rl + rr) * smax)
        return np.where(m > c.mach_ct, 1.0, np.where(m < -c.mach_ct, -1.0, 0.0))

    smax, dt = cfl()
    rk = {2: [(1.0, 0.0, -1.0), (0.5, 0.5, -0.5)],
          3: [(1.0, 0.0, -1.0), (0.75, 0.25, -0.25), (1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0))]}[c.rk_stages]
    for _ in range(nsteps):
        r, v1, v2 = W[0][I].copy(), W[1][I].copy(), W[2][I].copy()
        U0 = [r, r * v1, r * v2,
              eint + 0.5 * r * (v1 * v1 + v2 * v2 + 0.0 * 0.0)
              + 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0) + r * phi_cc]
        U = [u.copy() for u in U0]
        b10, b20 = b1.copy(), b2.copy()
        for a1, a2, c3 in rk:
            Wd = [w.copy() for w in W]
            Wd[0][I] = W[0][I] - eq_r
            Wd[3][I] = W[3][I] - eq_p
            for v in range(4):
                _fill(Wd[v], v == 2, G)
            z = np.zeros((nx + 1, ny))
            lo, hi = zip(*[_plm(w[G - 2:G + nx, G:G + ny], w[G - 1:G + nx + 1, G:G + ny], w[G:G + nx + 2, G:G + ny])
                           for w in Wd + [B[1]]])
            qL = [x[0:nx + 1] for x in hi[:4]]
            qR = [x[1:nx + 2] for x in lo[:4]]
            qL[0] = qL[0] + erx
            qR[0] = qR[0] + erx
            qL[3] = qL[3] + epx
            qR[3] = qR[3] + epx
            F, fb = _hlld(qL[:3] + [z, qL[3]], qR[:3] + [z, qR[3]], [b1, hi[4][0:nx + 1], z],
                          [b1, lo[4][1:nx + 2], z], gm, c.mach_cutoff, low_mach)
            F = F[:3] + F[4:]
            e1 = -fb[0]
            s1 = mass_sign(F[0], qL[0], qR[0], smax)
            F[1] = F[1] - epx
            F[3] = F[3] + F[0] * phx
            res = [(f[1:] - f[:-1]) * idx1 for f in F]
            z = np.zeros((nx, ny + 1))
            lo, hi = zip(*[_plm(w[G:G + nx, G - 2:G + ny], w[G:G + nx, G - 1:G + ny + 1], w[G:G + nx, G:G + ny + 2])
                           for w in Wd + [B[0]]])
            qL = [x[:, 0:ny + 1] for x in hi[:4]]
            qR = [x[:, 1:ny + 2] for x in lo[:4]]
            qL = [qL[0], qL[2], -qL[1], qL[3]]
            qR = [qR[0], qR[2], -qR[1], qR[3]]
            qL[0] = qL[0] + ery
            qR[0] = qR[0] + ery
            qL[3] = qL[3] + epy
            qR[3] = qR[3] + epy
            F, fb = _hlld(qL[:3] + [z, qL[3]], qR[:3] + [z, qR[3]], [b2, -hi[4][:, 0:ny + 1], z],
                          [b2, -lo[4][:, 1:ny + 2], z], gm, c.mach_cutoff, low_mach)
            F = [F[0], -F[2], F[1], F[4]]
            e2 = -fb[0]
            s2 = mass_sign(F[0], qL[0], qR[0], smax)
            F[2] = F[2] - epy
            F[3] = F[3] + F[0] * phy
            res = [rr + (f[:, 1:] - f[:, :-1]) * idx2 for rr, f in zip(res, F)]
            rdev = Wd[0][I]
            res[1] = res[1] - rdev * gx
            res[2] = res[2] - rdev * gy
            # x1-face EMFs past the walls: E3 negated, the sign copied; x2 faces periodic in x
            e1x = np.concatenate([-e1[:, :1], e1, -e1[:, -1:]], axis=1)
            s1x = np.concatenate([s1[:, :1], s1, s1[:, -1:]], axis=1)
            e2x = _wrap(e2, 0)
            s2x = _wrap(s2, 0)
            ec = -Wd[1] * B[1] + Wd[2] * B[0]
            cor = _corner((e1x[:, :-1], e1x[:, 1:]), (e2x[:-1], e2x[1:]),
                          (ec[G - 1:G + nx, G - 1:G + ny], ec[G - 1:G + nx, G:G + ny + 1],
                           ec[G:G + nx + 1, G:G + ny + 1], ec[G:G + nx + 1, G - 1:G + ny]),
                          (s1x[:, :-1], s1x[:, 1:]), (s2x[:-1], s2x[1:]))
            a3 = c3 * dt
            b1 = a1 * b10 + a2 * b1 + a3 * ((cor[:, 1:] - cor[:, :-1]) * idx2)
            b2 = a1 * b20 + a2 * b2 + a3 * ((cor[:-1] - cor[1:]) * idx1)
            cell_b()
            U = [a1 * u0 + a2 * u + a3 * rr for u0, u, rr in zip(U0, U, res)]
            rho = U[0]
            inv_rho = 1.0 / rho
            e = U[3] - 0.5 * (U[1] * U[1] + U[2] * U[2] + 0.0 * 0.0) * inv_rho
            e = e - 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + 0.0 * 0.0)
            e = e - rho * phi_cc
            p = (gm - 1.0) * e
            W[0][I] = rho
            W[1][I] = U[1] * inv_rho
            W[2][I] = U[2] * inv_rho
            W[3][I] = p
            temp = p / (rho * RGAS * inv_mu)
            eint = e
        smax, dt = cfl()
    return W, eint, temp, b1, b2, dt


def _fill_strat(a, G, flip):
    """Ghosts of a padded 3D cell array of the stratified box: periodic along x1 and x3,
    mirrored at the x2 walls (negated when `flip`: v2, B2) over every x1 / x3 index
    (S:7640-7720)."""
    for ax in (0, 2):
        m = a.shape[ax] - 2 * G
        lo = [slice(None)] * 3
        src = [slice(None)] * 3
        lo[ax], src[ax] = slice(0, G), slice(m, m + G)
        a[tuple(lo)] = a[tuple(src)]
        lo[ax], src[ax] = slice(m + G, m + 2 * G), slice(G, 2 * G)
        a[tuple(lo)] = a[tuple(src)]
    ny = a.shape[1] - 2 * G
    f = -1.0 if flip else 1.0
    for g in range(1, G + 1):
        a[:, G - g] = f * a[:, G + g - 1]
        a[:, ny + G - 1 + g] = f * a[:, ny + G - g]


class StratifiedHalo(PeriodicHalo):
    """The ghost exchange of one whole stratified box (x1 / x3 periodic, x2 walls)."""

    @staticmethod
    def fill(a, G, flip=False):
        _fill_strat(a, G, flip)


def stratified_steps(h, tab, dpdr, nd, nsteps, halo=StratifiedHalo):
    """The stratified Helmholtz box (3D, x2 vertical between reflective walls, x1 / x3
    periodic), magnetised (HLLD / LHLLD with constrained transport) or not (HLLC / LHLLC, with
    FLUX_IS_ALL_MACH when the configuration sets it): USE_WB on rho, p and gamma_e (S:7151-7168, the equilibria added back at the
    faces, S:8473-8486, S:8714-8727), USE_FASTEOS face gammas in the Riemann solver
    (S:14223-14226), EVOLVE_ETOT, gravity on rho' (S:12606-12644), ADVECT_YE_IABAR scalars,
    LHLLD (or HLLD) with constrained transport and the reflective EMF ghosts of the x1 and x3
    faces (S:11494-11590), the step-0 thermodynamics through helm_rhoP_given (S:6350-6357),
    cons->prim through helm_rhoe_given from the previous temperature with the gammas renewed
    (S:13640-13647), and the dt from helm_rhoT_given_full.  Without USE_FASTEOS each Riemann
    side solves helm_rhoP_given from the face guess (T(i-1) + T(i)) / 2 of the stage input's
    temperatures (S:8488-8495, S:14250-14256) with its own reconstructed Ye and 1/Abar, and the
    gammas are neither reconstructed nor kept.  Returns (W, eint, temp, gammaf,
    [b1, b2, b3], dt).  `halo` supplies the ghost exchange along x3 and the dt reduction (a
    slab of a decomposed box).  LIM2ND, PPH or LIM5TH.  With USE_SHOCK_FLATTENING (3 ghost layers) a
    flagged cell's edges fall back to PLM, the flagged faces take the HLL flux and the x1
    sweep's gamma_e follows the reference's flattened branch."""
    from numpy_restatement_eos import given_full, rhoe_given, rhoP_given
    c = h.cfg
    G = c.ngc
    tl, th = 10.0 ** c.helm_ltlo, 10.0 ** c.helm_lthi
    idx = [1.0 / d for d in (halo.dx or c.dx())]
    n = [c.nx1, c.nx2, c.nx3]
    I = tuple(slice(G, G + m) for m in n)
    nv = c.nvars
    mhd = c.mhd
    low_mach = c.riemann in ("lhlld", "lhllc")
    W = [h.prim[v].copy() for v in range(nv)]
    temp = h.temp[I].copy()
    b = [h.b_x[d][tuple(slice(1, 1 + n[a] + (a == d)) for a in range(3))].copy() for d in range(3)] if mhd else None
    B = [np.zeros_like(W[0]) for _ in range(3)]
    ge, gc = np.zeros_like(W[0]), np.zeros_like(W[0])
    eq_r, eq_p, eq_ge = h.eq_prim_cc[0][I], h.eq_prim_cc[1][I], h.eq_gammae_cc[I]
    phi = h.phi_cc[I]
    grav = [h.grav[d][I] for d in range(3)]
    eqf = [(h.eq_prim_x[d][0], h.eq_prim_x[d][1], h.eq_gammae_x[d], h.phi_x[d]) for d in range(3)]

    def cell_b():
        B[0][I] = 0.5 * (b[0][1:] + b[0][:-1])
        B[1][I] = 0.5 * (b[1][:, 1:] + b[1][:, :-1])
        B[2][I] = 0.5 * (b[2][:, :, 1:] + b[2][:, :, :-1])
        for d, a in enumerate(B):
            halo.fill(a, G, d == 1)

    if mhd:
        cell_b()
    # step-0 thermodynamics
    rho, p = W[0][I], W[4][I]
    abar = 1.0 / W[6][I]
    zbar = abar * W[5][I]
    fast = c.fasteos
    temp, E, snd, _ = rhoP_given(tab, dpdr, nd, rho, p, abar, zbar, temp, tl, th, return_sound=fast)
    eint = rho * E
    if fast:
        ge[I] = p / eint + 1.0
        gc[I] = snd * snd * rho / p

    def cfl():
        r, v1, v2, v3 = (W[v][I] for v in range(4))
        ab = 1.0 / W[6][I]
        _, _, cs, _ = given_full(tab, dpdr, nd, r, temp, ab, W[5][I] * ab)
        if mhd:
            ca2 = B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I]
            cs = np.sqrt(cs * cs + ca2 / r)
        sx1 = (np.abs(v1) + cs) * idx[0]
        sx2 = (np.abs(v2) + cs) * idx[1]
        sx3 = (np.abs(v3) + cs) * idx[2]
        smax = halo.max((sx3 + sx1 + sx2).max())
        return smax, c.cfl / smax

    def mass_sign(f, rl, rr, smax):
        m = f / (0.5 * (rl + rr) * smax)
        return np.where(m > c.mach_ct, 1.0, np.where(m < -c.mach_ct, -1.0, 0.0))

    def along(a, lo, hi):
        return tuple(slice(lo, hi) if x == a else I[x] for x in range(3))

    def wall_wrap(e, flip):
        """One ghost layer of a face array along x2: the mirrored row times the wall factor."""
        f = -1.0 if flip else 1.0
        return np.concatenate([f * e[:, :1], e, f * e[:, -1:]], axis=1)

    smax, dt = cfl()
    rk = {2: [(1.0, 0.0, -1.0), (0.5, 0.5, -0.5)],
          3: [(1.0, 0.0, -1.0), (0.75, 0.25, -0.25), (1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0))]}[c.rk_stages]
    for _ in range(nsteps):
        r, v1, v2, v3 = (W[v][I].copy() for v in range(4))
        e0 = eint + 0.5 * r * (v1 * v1 + v2 * v2 + v3 * v3)
        if mhd:
            e0 = e0 + 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I])
        U0 = [r, r * v1, r * v2, r * v3, e0 + r * phi] + [r * W[v][I] for v in range(5, nv)]
        U = [u.copy() for u in U0]
        b0 = [x.copy() for x in b] if mhd else None
        for a1, a2, c3 in rk:
            Wd = [w.copy() for w in W]
            Wd[0][I] = W[0][I] - eq_r
            Wd[4][I] = W[4][I] - eq_p
            ged = ge.copy()
            ged[I] = ge[I] - eq_ge
            gcd = gc.copy()
            for v, w in enumerate(Wd):
                halo.fill(w, G, v == 2)
            halo.fill(ged, G)
            halo.fill(gcd, G)
            tpad = np.zeros_like(W[0])
            tpad[I] = temp
            halo.fill(tpad, G)
            fl = _flatten_flags(Wd[4] + h.eq_prim_cc[1], G, n, c.eps_sf) if c.shock_flattening else None
            emf = [None, None, None]
            sgn = [None, None, None]
            res = None
            for a in range(3):
                m = n[a]
                trans = [t for t in range(3) if t != a]
                nb = 2 if mhd else 0
                arrs = Wd + ([B[t] for t in trans] if mhd else []) + [ged, gcd]
                # PPH limits the scalars only; LIM5TH everything
                lim = [c.rec == "lim5th" or (c.rec == "pph" and 5 <= v < nv) for v in range(len(arrs))]

                def edges(kind):
                    lo, hi = zip(*[_rec([w[along(a, G - 3 + o, G + m - 1 + o)] if G - 3 + o >= 0 else None
                                         for o in range(5)], kind, lv) for w, lv in zip(arrs, lim)])
                    return ([np.take(x, range(0, m + 1), axis=a) for x in hi],
                            [np.take(x, range(1, m + 2), axis=a) for x in lo])
                L, R = edges(c.rec)
                flat = None
                if fl is not None:
                    ins = [slice(1, 1 + n[x]) for x in range(3)]
                    fleft = fl[tuple(slice(0, m + 1) if x == a else ins[x] for x in range(3))]
                    fright = fl[tuple(slice(1, m + 2) if x == a else ins[x] for x in range(3))]
                    flat = fleft | fright
                    # a flagged cell's edges fall back to LIM2ND PLM (S:8731-8878 and the x2 / x3
                    # counterparts)
                    pL, pR = edges("lim2nd")
                    rawL, rawR = L[nv + nb], R[nv + nb]
                    L = [np.where(fleft, u, v) for u, v in zip(pL, L)]
                    R = [np.where(fright, u, v) for u, v in zip(pR, R)]
                er, ep, eg, ph = eqf[a]
                devL, devR = L[nv + nb], R[nv + nb]
                for side in (L, R):
                    side[0] = side[0] + er
                    side[4] = side[4] + ep
                    side[nv + nb] = side[nv + nb] + eg
                if fl is not None and a == 0 and fast:
                    # the x1 sweep's flattened gamma_e (S:8834-8869): a flagged cell's PLM edge
                    # replaces the face value without the equilibrium, which is added to the
                    # other side of that face instead
                    gl = np.where(fleft, devL, rawL + eg)
                    L[nv + nb] = np.where(fright, gl + eg, gl)
                    R[nv + nb] = np.where(fright, devR, np.where(fleft, (rawR + eg) + eg, rawR + eg))
                if a == 0:
                    qL, qR = L[:5], R[:5]
                elif a == 1:
                    qL = [L[0], L[2], -L[1], L[3], L[4]]
                    qR = [R[0], R[2], -R[1], R[3], R[4]]
                else:
                    qL = [L[0], L[3], L[1], L[2], L[4]]
                    qR = [R[0], R[3], R[1], R[2], R[4]]
                if mhd:
                    bt = (L[nv], L[nv + 1]), (R[nv], R[nv + 1])
                    sg = -1.0 if a == 1 else 1.0
                    bL = [b[a], sg * bt[0][0], bt[0][1]]
                    bR = [b[a], sg * bt[1][0], bt[1][1]]
                if fast:
                    eos = dict(fasteos=(L[nv + nb], L[nv + nb + 1], R[nv + nb], R[nv + nb + 1]))
                else:
                    tg = 0.5 * (tpad[along(a, G - 1, G + m)] + tpad[along(a, G, G + m + 1)])
                    sides = []
                    for q in (L, R):
                        ab = 1.0 / q[6]
                        _, e1, s1, _ = rhoP_given(tab, dpdr, nd, q[0], q[4], ab, q[5] * ab, tg, tl, th)
                        sides += [e1 * q[0], s1 * s1 if mhd else s1]
                    eos = dict(side_eos=tuple(sides))
                if mhd:
                    F, fb = _hlld(qL, qR, bL, bR, c.gamma_ad, c.mach_cutoff, low_mach, L[5:nv], R[5:nv], flat=flat,
                                  all_mach=c.all_mach,
                                  **eos)
                    emf[a] = [(None, fb[1], -fb[0]), (-fb[1], None, -fb[0]), (fb[1], -fb[0], None)][a]
                else:
                    F = _hllc3(qL, qR, c.gamma_ad, c.mach_cutoff, low_mach, c.all_mach, L[5:nv], R[5:nv],
                               flat=flat, **eos)
                if a == 1:
                    F = [F[0], -F[2], F[1]] + F[3:]
                elif a == 2:
                    F = [F[0], F[2], F[3], F[1]] + F[4:]
                if mhd:
                    sgn[a] = mass_sign(F[0], qL[0], qR[0], smax)
                F[1 + a] = F[1 + a] - ep
                F[4] = F[4] + F[0] * ph
                div = [np.diff(f, axis=a) * idx[a] for f in F]
                res = div if res is None else [rr + d for rr, d in zip(res, div)]
            rdev = Wd[0][I]
            for d in range(3):
                res[1 + d] = res[1 + d] - rdev * grav[d]
            if mhd:
                b = _ct_walls(b, b0, emf, sgn, Wd, B, G, n, idx, a1, a2, c3 * dt, wall_wrap, halo.wrap3)
                cell_b()
            U = [a1 * u0 + a2 * u + c3 * dt * rr for u0, u, rr in zip(U0, U, res)]
            rho = U[0]
            inv_rho = 1.0 / rho
            e_ = U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * inv_rho
            if mhd:
                e_ = e_ - 0.5 * (B[0][I] * B[0][I] + B[1][I] * B[1][I] + B[2][I] * B[2][I])
            e_ = e_ - rho * phi
            ye = U[5] * inv_rho
            ab = rho / U[6]
            temp, p, snd, _ = rhoe_given(tab, dpdr, nd, rho, e_ * inv_rho, ab, ye * ab, temp, tl, th,
                                         return_sound=fast)
            if fast:
                ge[I] = p / e_ + 1.0
                gc[I] = snd * snd * rho / p
            W[0][I] = rho
            for d in range(3):
                W[1 + d][I] = U[1 + d] * inv_rho
            W[4][I] = p
            for v in range(5, nv):
                W[v][I] = U[v] * inv_rho
            eint = e_
        smax, dt = cfl()
    return W, eint, temp, (ge, gc), b, dt


def _flatten_flags(pf, G, n, eps_sf):
    """is_flattened of the padded cells G-1 .. G+n along every axis (S:8073-8136): a cell
    G-2 .. G+n+1 whose summed central jumps of the full pressure pf (deviation plus the stored
    equilibrium, ghosts included), x3 + x2 + x1, exceed eps_sf times its pressure marks its
    3 x 3 x 3 neighbourhood.  fl[i, j, k] is padded cell (G-1+i, G-1+j, G-1+k)."""
    def win(a, o):
        return tuple(slice(G - 2 + (o if x == a else 0), G + n[x] + 2 + (o if x == a else 0)) for x in range(3))
    d = [np.abs(pf[win(a, 1)] - pf[win(a, -1)]) for a in range(3)]
    tmp = (d[2] + d[1] + d[0]) / pf[win(0, 0)]
    mark = tmp > eps_sf
    fl = np.zeros(tuple(m + 2 for m in n), dtype=bool)
    for o0 in range(3):
        for o1 in range(3):
            for o2 in range(3):
                fl |= mark[o0:o0 + n[0] + 2, o1:o1 + n[1] + 2, o2:o2 + n[2] + 2]
    return fl


def _ct_walls(b, b0, emf, sgn, Wd, B, G, n, idx, a1, a2, a3, wall_wrap, wrap3):
    """Corner EMFs of the stratified box (reflective x2 walls, x1 / x3 periodic) and the RK
    update of the three face-B arrays."""
    I = tuple(slice(G, G + m) for m in n)
    ec3 = -Wd[1] * B[1] + Wd[2] * B[0]
    ec1 = Wd[3] * B[1] - Wd[2] * B[2]
    ec2 = Wd[1] * B[2] - Wd[3] * B[0]
    nx, ny, nz = n
    Ix, Iy, Iz = I
    e, s_ = wall_wrap(emf[0][2], True), wall_wrap(sgn[0], False)
    f, t = _wrap(emf[1][2], 0), _wrap(sgn[1], 0)
    cor3 = _corner((e[:, :-1], e[:, 1:]), (f[:-1], f[1:]),
                   (ec3[G - 1:G + nx, G - 1:G + ny, Iz], ec3[G - 1:G + nx, G:G + ny + 1, Iz],
                    ec3[G:G + nx + 1, G:G + ny + 1, Iz], ec3[G:G + nx + 1, G - 1:G + ny, Iz]),
                   (s_[:, :-1], s_[:, 1:]), (t[:-1], t[1:]))
    e, s_ = wrap3(emf[1][0]), wrap3(sgn[1])
    f, t = wall_wrap(emf[2][0], True), wall_wrap(sgn[2], False)
    cor1 = _corner((e[:, :, :-1], e[:, :, 1:]), (f[:, :-1], f[:, 1:]),
                   (ec1[Ix, G - 1:G + ny, G - 1:G + nz], ec1[Ix, G - 1:G + ny, G:G + nz + 1],
                    ec1[Ix, G:G + ny + 1, G:G + nz + 1], ec1[Ix, G:G + ny + 1, G - 1:G + nz]),
                   (s_[:, :, :-1], s_[:, :, 1:]), (t[:, :-1], t[:, 1:]))
    e, s_ = _wrap(emf[2][1], 0), _wrap(sgn[2], 0)
    f, t = wrap3(emf[0][1]), wrap3(sgn[0])
    cor2 = _corner((e[:-1], e[1:]), (f[:, :, :-1], f[:, :, 1:]),
                   (ec2[G - 1:G + nx, Iy, G - 1:G + nz], ec2[G:G + nx + 1, Iy, G - 1:G + nz],
                    ec2[G:G + nx + 1, Iy, G:G + nz + 1], ec2[G - 1:G + nx, Iy, G:G + nz + 1]),
                   (s_[:-1], s_[1:]), (t[:, :, :-1], t[:, :, 1:]))
    t1 = -(cor2[:, :, 1:] - cor2[:, :, :-1]) * idx[2] + (cor3[:, 1:] - cor3[:, :-1]) * idx[1]
    t2 = (cor1[:, :, 1:] - cor1[:, :, :-1]) * idx[2] + (cor3[:-1] - cor3[1:]) * idx[0]
    t3 = (cor2[1:] - cor2[:-1]) * idx[0] - (cor1[:, 1:] - cor1[:, :-1]) * idx[1]
    b = [a1 * x0 + a2 * x + a3 * tt for x0, x, tt in zip(b0, b, (t1, t2, t3))]
    return b
