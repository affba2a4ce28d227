"""Electron-positron Helmholtz free-energy table from Fermi-Dirac integrals.

The reference evaluates its Helmholtz EoS (``helm_rhoT_given*``, ``source/source.F90:23686-24941``)
from Timmes' table of the electron-positron free energy (``helm_table.dat``, a third-party
file fetched by ``data/get_data.sh`` and absent here).  This module computes a table of the
same quantities, in the same layout as :func:`phlegethon_b200.helm_table.generate`, from the
ideal Fermi gas of electrons and positrons in pair equilibrium with arbitrary degeneracy and
special relativity, i.e. the physics the published table is built on (Timmes & Arnett 1999,
ApJS 125, 277; Timmes & Swesty 2000, ApJS 126, 501):

* per species, with x = kinetic energy / kT, beta = kT / (m_e c^2) and the degeneracy
  parameter eta (electrons) or eta_+ = -eta - 2/beta (positrons),

      n = K beta^(3/2) Int x^(1/2) (1 + beta x/2)^(1/2) (1 + beta x) F dx
      P = (2/3) K m_e c^2 beta^(5/2) Int x^(3/2) (1 + beta x/2)^(3/2) F dx
      E = K m_e c^2 beta^(5/2) Int x^(3/2) (1 + beta x/2)^(1/2) (1 + beta x) F dx
      S = k K beta^(3/2) Int x^(1/2) (1 + beta x/2)^(1/2) (1 + beta x) sigma dx

  with K = 8 pi sqrt(2) (m_e c / h)^3, the Fermi factor F = 1 / (exp(x - eta) + 1) and the
  entropy density sigma = -(F ln F + (1 - F) ln(1 - F));
* eta from charge neutrality n_- - n_+ = N_A d, d = rho Ye (the table's density variable);
* the free energy per unit d: f = N_A eta k T - P / d (the positrons' rest mass counted in the
  energy, the electrons' not), so that P = d^2 df/dd and E = Ye (f - T df/dT) as the reference
  combines them.

The integrals are evaluated by Gauss-Legendre quadrature on pieces placed around the Fermi
surface (a graded square-root substitution near x = 0, pieces of width <= 2 across
|x - eta| < 40, nothing beyond where F < e^-40).  Every table entry up to second order is
formed from integrals directly, without differencing (f_dd from dP/dd = n N_A kT / W0,
f_dT from dP/dT = S - n k W1 / W0, f_TT from the heat capacity
C_v / T = (k / T) (W2 - W1^2 / W0), with W_m = Int D (x - eta)^m F (1 - F) dx summed over the
species); the third and fourth derivatives are central differences in ln d of the second
ones, which carry no T-independent part, so nothing cancels even in degenerate matter.
"""
from __future__ import annotations

import math

import numpy as np

from .helm_table import CONST_AV, CONST_H, CONST_KB, M_E, nodes

CONST_C = 2.99792458e10
MC2 = M_E * CONST_C * CONST_C                               # electron rest energy [erg]
K_N = 8.0 * math.pi * math.sqrt(2.0) * (M_E * CONST_C / CONST_H) ** 3  # [cm^-3]

# quadrature layout: graded pieces in s = sqrt(x / xa) over [0, xa], equal pieces over [xa, xb]
_S_BREAKS = np.array([0.0, 1e-4, 1e-3, 1e-2, 3e-2, 0.1, 0.3, 0.6, 1.0])
_NA_PTS = 12
_NB_PIECES = 36
_NB_PTS = 8
_WINDOW = 40.0  # |x - eta| beyond which F or 1 - F is below e^-40


def _gauss(n):
    t, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (t + 1.0), 0.5 * w  # nodes and weights on [0, 1]


_TA, _WA = _gauss(_NA_PTS)
_TB, _WB = _gauss(_NB_PTS)


def _grid(eta):
    """Quadrature nodes x (n, m) and weights (dx included) for degeneracy parameters eta (n,)."""
    eta = np.asarray(eta, dtype=np.float64)
    xa = np.maximum(eta - 30.0, 2.0)
    xb = np.maximum(eta, 0.0) + _WINDOW
    xb = np.maximum(xb, xa + 2.0)
    # piece A: x = xa s^2, s in graded pieces of [0, 1]
    s_lo = _S_BREAKS[:-1, None]
    s_hi = _S_BREAKS[1:, None]
    s = (s_lo + (s_hi - s_lo) * _TA[None, :]).ravel()            # (8 * NA,)
    ws = ((s_hi - s_lo) * _WA[None, :]).ravel()
    xA = xa[:, None] * s[None, :] ** 2
    wA = 2.0 * xa[:, None] * s[None, :] * ws[None, :]
    # piece B: equal pieces over [xa, xb]
    k = np.arange(_NB_PIECES)[:, None]
    u = ((k + _TB[None, :]) / _NB_PIECES).ravel()
    wu = np.tile(_WB, _NB_PIECES) / _NB_PIECES
    span = (xb - xa)[:, None]
    xB = xa[:, None] + span * u[None, :]
    wB = span * wu[None, :]
    return np.concatenate([xA, xB], axis=1), np.concatenate([wA, wB], axis=1)


def _fermi(y):
    """F, F (1 - F) and the entropy density sigma of y = x - eta, overflow-free."""
    a = np.abs(y)
    e = np.exp(-a)
    inv = 1.0 / (1.0 + e)
    F = np.where(y > 0.0, e * inv, inv)
    w = e * inv * inv
    sigma = a * e * inv + np.log1p(e)
    return F, w, sigma


# Above this beta (T > 1.2e8 K) the solve runs in delta = eta + 1/beta, the electrons' chemical
# potential including the rest mass in units of kT: pairs can outnumber the net electrons by
# any factor there, and n_- - n_+ ~ sinh(delta) is resolved only through delta itself.  Below
# it the solve runs in eta (1/beta > 50: pairs are at most e^-26 of the electrons, and
# eta + 1/beta would round eta away in degenerate matter).
_BETA_HOT = 0.02


def _fermi_diff(u, dl):
    """F(u - dl) - F(u + dl) = sinh(dl) / (cosh(u) + cosh(dl)) with every exponent <= 0."""
    ad = np.abs(dl)
    a = np.maximum(u, ad)
    # 2 sinh(ad) e^-a: through sinh where the two exponentials would cancel
    small = ad < 1.0
    num = np.where(small, 2.0 * np.sinh(np.where(small, ad, 0.0)) * np.exp(-a), np.exp(ad - a) - np.exp(-ad - a))
    den = np.exp(u - a) + np.exp(-u - a) + np.exp(ad - a) + np.exp(-ad - a)
    return np.sign(dl) * num / den


def _split(z, beta):
    """(eta, delta, hot) of the solve variable z: delta where beta > _BETA_HOT, else eta."""
    hot = beta > _BETA_HOT
    eta = np.where(hot, z - 1.0 / beta, z)
    delta = np.where(hot, z, z + 1.0 / beta)
    return eta, delta, hot


def pair_integrals(z, beta, full=True):
    """Dimensionless integrals of the electron-positron gas at solve variable z (see _split),
    both species on the electrons' quadrature grid (positrons have the lower degeneracy
    parameter, so the grid that resolves the electrons' Fermi factor also covers theirs).

    Returns In (net number, n_- - n_+), In_pos (positrons), W0 = dIn/dz and, when full is set,
    Ip (pressure), Ie (kinetic energy), Is (entropy), W1 (first moment of F (1 - F) in the
    reduced energy, electrons minus positrons) and W2 (second moment, summed)."""
    z = np.asarray(z, dtype=np.float64).ravel()
    beta = np.asarray(beta, dtype=np.float64).ravel()
    eta, delta, hot = _split(z, beta)
    x, wx = _grid(eta)
    b = beta[:, None]
    h = hot[:, None]
    u = x + 1.0 / b
    dl = delta[:, None]
    y_m = np.where(h, u - dl, x - eta[:, None])
    y_p = np.where(h, u + dl, x + (eta + 2.0 / beta)[:, None])
    F_m, w_m, s_m = _fermi(y_m)
    F_p, w_p, s_p = _fermi(y_p)
    diff = np.where(h, _fermi_diff(u, dl), F_m - F_p)
    rel = np.sqrt(1.0 + 0.5 * b * x)
    D = np.sqrt(x) * rel * (1.0 + b * x) * wx
    out = {"In": np.sum(D * diff, axis=1), "In_pos": np.sum(D * F_p, axis=1),
           "W0": np.sum(D * (w_m + w_p), axis=1), "eta": eta}
    if full:
        x32 = x * np.sqrt(x) * wx
        out["Ip"] = np.sum(x32 * rel * rel * rel * (F_m + F_p), axis=1)
        out["Ie"] = np.sum(x32 * rel * (1.0 + b * x) * (F_m + F_p), axis=1)
        out["Is"] = np.sum(D * (s_m + s_p), axis=1)
        out["W1"] = np.sum(D * (y_m * w_m - y_p * w_p), axis=1)
        out["W2"] = np.sum(D * (y_m * y_m * w_m + y_p * y_p * w_p), axis=1)
    return out


def _net_density(z, beta):
    """n_- - n_+ and its derivative in the solve variable (cm^-3)."""
    pre = K_N * beta ** 1.5
    r = pair_integrals(z, beta, full=False)
    return pre * r["In"], pre * r["W0"]


def solve_eta(d, T, tol=1e-13, max_iter=100, z0=None):
    """Solve variable z (delta above _BETA_HOT, eta below) with N_A d = n_- - n_+; z0, when
    given, is the starting point (a solution at a nearby density)."""
    d = np.asarray(d, dtype=np.float64).ravel()
    T = np.asarray(T, dtype=np.float64).ravel()
    beta = CONST_KB * T / MC2
    target = CONST_AV * d
    hot = beta > _BETA_HOT
    if z0 is not None:
        return _newton(np.array(z0, dtype=np.float64), beta, target, hot, np.where(hot, 0.0, -1.0 / beta), tol,
                       max_iter)
    # initial guess: the larger of the non-degenerate and the cold degenerate estimates
    eta_nd = np.log(target / (K_N * beta ** 1.5 * 0.5 * math.sqrt(math.pi)))
    pf = CONST_H * (3.0 * target / (8.0 * math.pi)) ** (1.0 / 3.0)          # Fermi momentum
    xf2 = (pf / (M_E * CONST_C)) ** 2
    eta_deg = MC2 * xf2 / (np.sqrt(1.0 + xf2) + 1.0) / (CONST_KB * T)       # kinetic Fermi energy / kT
    eta0 = np.where(eta_deg > 1.0, np.maximum(eta_nd, eta_deg), eta_nd)
    lo = np.where(hot, 0.0, -1.0 / beta)    # n_- = n_+ there: below the root
    z = np.where(hot, eta0 + 1.0 / beta, eta0)
    z = np.maximum(z, np.where(hot, 0.0, lo + 1e-3))
    # pair-dominated nodes (delta < 1): n_- - n_+ is nearly linear in delta, start from the
    # slope at delta = 0
    pairs = np.nonzero(hot & (z < 1.0))[0]
    if pairs.size:
        _, dn0 = _net_density(np.zeros(pairs.size), beta[pairs])
        z[pairs] = np.minimum(target[pairs] / dn0, 1.0)
    return _newton(z, beta, target, hot, lo, tol, max_iter)


def _newton(z, beta, target, hot, lo, tol, max_iter):
    """Bracketed Newton iteration of n_- - n_+ = target in the solve variable z."""
    lo = np.array(lo, dtype=np.float64)
    hi = np.full_like(z, np.inf)
    active = np.ones(z.shape, dtype=bool)
    for _ in range(max_iter):
        idx = np.nonzero(active)[0]
        if idx.size == 0:
            break
        e, tg = z[idx], target[idx]
        n, dn = _net_density(e, beta[idx])
        above = n > tg
        hi[idx] = np.where(above, e, hi[idx])
        lo[idx] = np.where(above, lo[idx], e)
        # Newton on ln n (exact in the Boltzmann limit and linear in the pair limit, where
        # n ~ sinh(delta)); a step that leaves the bracket is replaced by bisection, or by an
        # expansion while no upper bound is known
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            step = np.where(n > 0.0, -(np.log(n) - np.log(tg)) * (n / dn), -(n - tg) / dn)
        cand = e + step
        lo_b, hi_b = lo[idx], hi[idx]
        bad = ~np.isfinite(cand) | (cand < lo_b) | (cand > hi_b)
        mid = np.where(np.isfinite(hi_b), 0.5 * (lo_b + hi_b), e + np.maximum(2.0 * np.abs(e), 10.0))
        cand = np.where(bad, mid, cand)
        z[idx] = cand
        active[idx] = np.abs(cand - e) > tol * np.maximum(np.abs(e), np.where(hot[idx], 0.0, 1.0))
    return z


def thermo(d, T, z0=None):
    """Electron-positron thermodynamics at (d = rho Ye, T): a dict of arrays with
    eta, n (net, cm^-3), P, E (per volume, pair rest mass included), S (per volume), and the
    derivatives P_d = dP/dd|T, P_T = dP/dT|d, Cv_T = dS/dT|d."""
    d = np.asarray(d, dtype=np.float64).ravel()
    T = np.asarray(T, dtype=np.float64).ravel()
    beta = CONST_KB * T / MC2
    z = solve_eta(d, T, z0=z0)
    r = pair_integrals(z, beta)
    eta = r["eta"]
    pre_n = K_N * beta ** 1.5
    pre_e = K_N * MC2 * beta ** 2.5
    n = pre_n * r["In"]
    n_p = pre_n * r["In_pos"]
    P = (2.0 / 3.0) * pre_e * r["Ip"]
    E = pre_e * r["Ie"] + 2.0 * MC2 * n_p
    S = CONST_KB * pre_n * r["Is"]
    W0 = pre_n * r["W0"]
    W1 = pre_n * r["W1"]
    W2 = pre_n * r["W2"]
    kT = CONST_KB * T
    P_d = n * CONST_AV * kT / W0
    P_T = S - n * CONST_KB * W1 / W0
    Cv_T = CONST_KB / T * (W2 - W1 * W1 / W0)
    return {"eta": eta, "n": n, "n_pos": n_p, "P": P, "E": E, "S": S, "P_d": P_d, "P_T": P_T,
            "Cv_T": Cv_T, "z": z}


def _second_order(d, T, z0=None):
    """f and its derivatives up to second order, plus c = dP/dd and dP/dT, at (d, T)."""
    th = thermo(d, T, z0)
    f = CONST_AV * th["eta"] * CONST_KB * T - th["P"] / d
    return {
        "f": f,
        "f_d": th["P"] / (d * d),
        "f_t": -th["S"] / d,
        "f_dd": th["P_d"] / (d * d) - 2.0 * th["P"] / (d * d * d),
        "f_dt": th["P_T"] / (d * d),
        "f_tt": -th["Cv_T"] / d,
        "c": th["P_d"],
        "p_t": th["P_T"],
        "z": th["z"],
    }


def _chunk(args):
    """Table quantities of one block of nodes: the node itself and its two neighbours in ln d."""
    dd, tt, dlog = args
    r0 = _second_order(dd, tt)
    rp = _second_order(dd * math.exp(dlog), tt, r0["z"])
    rm = _second_order(dd * math.exp(-dlog), tt, r0["z"])
    return r0, rp, rm


def generate(nrho=541, nT=201, ldlo=-12.0, ldhi=15.0, ltlo=3.0, lthi=13.0, dlog=1e-3, chunk=2048, workers=0):
    """Return ``(tab, dpdr)`` in the layout of :func:`phlegethon_b200.helm_table.generate`.

    The table's density variable is d = rho Ye over [10^ldlo, 10^ldhi] (the free energy per
    unit d does not depend on Ye).  Third and fourth derivatives are central differences in
    ln d with step ``dlog``.  ``workers`` > 1 spreads the node blocks over that many processes
    (started with "spawn", so it is safe after CUDA has been initialised; the calling script
    needs the usual ``if __name__ == "__main__":`` guard)."""
    rho, T, _, _ = nodes(nrho, nT, ldlo, ldhi, ltlo, lthi)
    dd = np.repeat(rho, nT)          # node (i, j) at i * nT + j
    tt = np.tile(T, nrho)
    blocks = [(dd[a:a + chunk], tt[a:a + chunk], dlog) for a in range(0, dd.size, chunk)]
    if workers and workers > 1:
        # spawned workers (safe after CUDA has been initialised); the executor raises instead of
        # waiting forever if a worker dies, e.g. when the main script lacks a __main__ guard
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_chunk, blocks))
    else:
        parts = [_chunk(b) for b in blocks]
    keys = ("f", "f_d", "f_t", "f_dd", "f_dt", "f_tt", "c", "p_t")
    res = {k: np.concatenate([p[0][k] for p in parts]) for k in keys}
    hi = {k: np.concatenate([p[1][k] for p in parts]) for k in ("f_dt", "f_tt", "c", "p_t")}
    lo = {k: np.concatenate([p[2][k] for p in parts]) for k in ("f_dt", "f_tt", "c", "p_t")}

    def d_dlnd(k):
        return (hi[k] - lo[k]) / (2.0 * dlog)

    def d2_dlnd2(k):
        return (hi[k] - 2.0 * res[k] + lo[k]) / (dlog * dlog)

    # d/dd g = g_L / d, d2/dd2 g = (g_LL - g_L) / d^2 with L = ln d
    f_ddt = d_dlnd("f_dt") / dd
    f_dtt = d_dlnd("f_tt") / dd
    f_ddtt = (d2_dlnd2("f_tt") - d_dlnd("f_tt")) / (dd * dd)
    c_d = d_dlnd("c") / dd
    c_t = d_dlnd("p_t") / dd
    c_dt = (d2_dlnd2("p_t") - d_dlnd("p_t")) / (dd * dd)

    def grid(v):
        return np.asarray(v).reshape(nrho, nT)

    tab = np.zeros((9, nrho, nT), order="F")
    for v, arr in enumerate([res["f"], res["f_t"], res["f_tt"], res["f_d"], res["f_dd"], res["f_dt"], f_ddt, f_dtt,
                             f_ddtt]):
        tab[v] = grid(arr)
    dpdr = np.zeros((4, nrho, nT), order="F")
    for v, arr in enumerate([res["c"], c_t, c_d, c_dt]):
        dpdr[v] = grid(arr)
    return np.asfortranarray(tab), np.asfortranarray(dpdr)
