"""An independent, vectorised numpy restatement of the 2D ideal-gas hydro step.

Written from the reference (source/source.F90) separately from the C oracle, in a different
style (whole-array operations on a ghost-padded grid instead of per-line loops), so that a
bitwise match between the two pins the oracle's sweep logic: ghost filling (periodic wrap and
reflective mirror, S:2293-2306 / S:7532-7958), well-balanced deviations (S:7151-7168),
LIM2ND PLM (S:8141-8181), x2 rotation (S:9715-9747, S:10101-10111), LHLLC (S:15681-16122),
WB momentum fix and EVOLVE_ETOT potential flux (S:8953-8966), gravity (S:12606-12644), RK3
(S:7018-7048, S:13518-13531), cons->prim (S:13533-13686) and the CFL dt (S:13707-13960).
With eps_sf set it adds USE_SHOCK_FLATTENING: the pressure-jump detector (S:8073-8136) and
the HLL flux on faces next to a flagged cell (S:15929-16010); LIM2ND cells need no fallback.
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


def hot_bubble_steps(h, nsteps, dt=None, eps_sf=None):
    """Advance the hot-bubble HostGrid `h` (2D, ideal, WB+ETOT+gravity, LHLLC, RK3) in place;
    eps_sf: USE_SHOCK_FLATTENING with that threshold (ngc >= 3)."""
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
            lo, hi = zip(*[_plm(w[G - 2:G + nx, G:G + ny], w[G - 1:G + nx + 1, G:G + ny], w[G:G + nx + 2, G:G + ny])
                           for w in Wd])
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
            lo, hi = zip(*[_plm(w[G:G + nx, G - 2:G + ny], w[G:G + nx, G - 1:G + ny + 1], w[G:G + nx, G:G + ny + 2])
                           for w in Wd])
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
