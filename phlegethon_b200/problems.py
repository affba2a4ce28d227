"""Problem setups (the ``app.F90`` equivalents) for the benchmark configurations.

Each builder returns ``(cfg, grid)`` with every reference array filled on the ghost-padded
grid, exactly as an ``app.F90`` does before calling ``time_loop``:

* :func:`hot_bubble_2d`      2D hot bubble in an isothermal atmosphere (ideal gas, WB, LHLLC)
* :func:`orszag_tang_2d`     2D Orszag-Tang vortex (ideal MHD, CT, face B from A_z on nodes as
                             ``tests/orszag-tang/app.F90:28-79``)
* :func:`stratified_3d`      3D stratified convection box with the Helmholtz EoS (WB, LHLLC),
                             optionally magnetised (LHLLD + CT)
* :func:`eos_samples`        the (rho, T, Abar, Zbar) sample batch of the EoS inversion benchmark

All inputs are synthetic; random velocity perturbations come from a counter-based hash of
(seed, global i, j, k, component), so they do not depend on how the domain is split.
"""
from __future__ import annotations

import math

import numpy as np

from .grid import Config, HostGrid
from .helm_table import CONST_AV, CONST_H, CONST_KB, CONST_RGAS, M_E, X2_TABLE

CONST_RAD = 7.565767381646406e-15


# ------------------------------------------------------------------------------ hashing RNG
def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return z ^ (z >> np.uint64(31))


def hash_uniform(seed, i, j, k, comp):
    """Uniform [-1, 1) from a counter-based hash of (seed, i, j, k, comp)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x100000001B3)) & np.uint64(0xFFFFFFFFFFFFFFFF)
        x = _splitmix64(key ^ np.asarray(i, dtype=np.uint64))
        x = _splitmix64(x ^ (np.asarray(j, dtype=np.uint64) << np.uint64(21)))
        x = _splitmix64(x ^ (np.asarray(k, dtype=np.uint64) << np.uint64(42)))
        x = _splitmix64(x ^ np.uint64(comp + 1))
    return ((x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0


# ------------------------------------------------------------------------------ analytic EoS
# The closed-form electron free energy of helm_table.generate plus ions and radiation, used
# only to build initial states (the step itself uses the tabulated EoS).
def _kprime():
    hbar = CONST_H / (2.0 * math.pi)
    k_n = (3.0 * math.pi ** 2) ** (2.0 / 3.0) * hbar ** 2 / (5.0 * M_E)
    return 1.5 * k_n * CONST_AV ** (5.0 / 3.0)


def analytic_pressure(rho, T, abar, zbar):
    ye = zbar / abar
    d = rho * ye
    kp = _kprime()
    pe = (2.0 / 3.0) * kp * d ** (5.0 / 3.0) + CONST_RGAS * T * d
    return pe + CONST_RGAS * rho * T / abar + CONST_RAD * T ** 4 / 3.0


def analytic_energy(rho, T, abar, zbar):
    ye = zbar / abar
    d = rho * ye
    kp = _kprime()
    return ye * (kp * d ** (2.0 / 3.0) + 1.5 * CONST_RGAS * T) + 1.5 * CONST_RGAS * T / abar + CONST_RAD * T ** 4 / rho


def analytic_temperature(rho, p, abar, zbar, T0=1e8):
    T = np.full(np.shape(rho), T0, dtype=np.float64)
    for _ in range(60):
        f = analytic_pressure(rho, T, abar, zbar) - p
        dfdT = CONST_RGAS * rho * zbar / abar + CONST_RGAS * rho / abar + 4.0 / 3.0 * CONST_RAD * T ** 3
        T = np.clip(T - f / dfdT, 1e3, 1e13)
    return T


# The electron-positron Fermi gas of helm_fermi (the model of helm_fermi.generate's table)
# plus the same ions and radiation.
def fermi_pressure(rho, T, abar, zbar):
    from . import helm_fermi
    rho, T = np.broadcast_arrays(np.asarray(rho, dtype=np.float64), np.asarray(T, dtype=np.float64))
    th = helm_fermi.thermo((rho * (zbar / abar)).ravel(), T.ravel())
    pe = th["P"].reshape(rho.shape)
    return pe + CONST_RGAS * rho * T / abar + CONST_RAD * T ** 4 / 3.0


def fermi_energy(rho, T, abar, zbar):
    from . import helm_fermi
    rho, T = np.broadcast_arrays(np.asarray(rho, dtype=np.float64), np.asarray(T, dtype=np.float64))
    th = helm_fermi.thermo((rho * (zbar / abar)).ravel(), T.ravel())
    ee = th["E"].reshape(rho.shape) / rho
    return ee + 1.5 * CONST_RGAS * T / abar + CONST_RAD * T ** 4 / rho


def fermi_temperature(rho, p, abar, zbar, T0=1e8):
    from . import helm_fermi
    rho = np.asarray(rho, dtype=np.float64)
    T = np.full(rho.shape, T0, dtype=np.float64)
    d = (rho * (zbar / abar)).ravel()
    for _ in range(60):
        th = helm_fermi.thermo(d, T.ravel())
        f = th["P"].reshape(rho.shape) + CONST_RGAS * rho * T / abar + CONST_RAD * T ** 4 / 3.0 - p
        dfdT = th["P_T"].reshape(rho.shape) + CONST_RGAS * rho / abar + 4.0 / 3.0 * CONST_RAD * T ** 3
        dT = f / dfdT
        T = np.clip(T - dT, 1e3, 1e13)
        # the quadrature of the Fermi integrals leaves a rounding floor near 4e-14 in dT / T
        if np.all(np.abs(dT) <= 1e-12 * T):
            break
    return T


EOS_MODELS = {"synthetic": (analytic_pressure, analytic_energy, analytic_temperature),
              "fermi": (fermi_pressure, fermi_energy, fermi_temperature)}


# ------------------------------------------------------------------------------ hot bubble
def hot_bubble_2d(n=256, riemann="lhllc", seed=None, shock_flattening=False, eps_sf=0.25):
    """2D hot bubble: [0,1]^2, periodic x / reflecting y, g = -1 in y, isothermal atmosphere
    rho = exp(-y/H), H = 0.5, p = rho*H*|g|, Gaussian temperature bump
    dT/T = 0.05 exp(-r^2/0.1^2) at (0.5, 0.25) in pressure equilibrium; ideal gas gamma = 5/3."""
    cfg = Config(sdims=2, nx1=n, nx2=n, nx3=1, ngc=3 if shock_flattening else 2, nas=0, wb=True, gravity=True,
                 etot=True, riemann=riemann, rk_stages=3, shock_flattening=shock_flattening, eps_sf=eps_sf,
                 bc=[["periodic", "periodic"], ["reflective", "reflective"], ["periodic", "periodic"]],
                 x1l=0.0, x1u=1.0, x2l=0.0, x2u=1.0, x3l=0.0, x3u=1.0, gamma_ad=5.0 / 3.0, mu=1.0,
                 cfl=0.8, mach_cutoff=1e-4)
    h = HostGrid(cfg)
    H, g = 0.5, 1.0
    x, y, _ = h.coords()
    rho_eq = np.exp(-y / H)
    p_eq = rho_eq * H * g
    r2 = (x - 0.5) ** 2 + (y - 0.25) ** 2
    h.prim[0] = rho_eq / (1.0 + 0.05 * np.exp(-r2 / 0.01))
    h.prim[1] = 0.0
    h.prim[2] = 0.0
    h.prim[3] = p_eq
    h.grav[0] = 0.0
    h.grav[1] = -g
    h.phi_cc[...] = g * y
    h.eq_prim_cc[0] = rho_eq
    h.eq_prim_cc[1] = p_eq
    h.eq_prim_cc[2] = p_eq / (CONST_RGAS * rho_eq)
    for d in range(2):
        fx, fy, _ = h.face_coords(d)
        re = np.exp(-fy / H)
        h.eq_prim_x[d][0] = re
        h.eq_prim_x[d][1] = re * H * g
        h.eq_prim_x[d][2] = H * g / CONST_RGAS
        h.phi_x[d][...] = g * fy
    h.temp[...] = h.prim[3] / (CONST_RGAS * h.prim[0])
    return cfg, h


# ------------------------------------------------------------------------------ Orszag-Tang
def orszag_tang_2d(n=1024, riemann="hlld", rec="lim2nd", shock_flattening=False, eps_sf=0.25):
    """Orszag-Tang vortex on the periodic unit square (tests/orszag-tang/app.F90:13-79; the
    reference's test runs it with LIM5TH_REC, tests/orszag-tang/Makefile:29)."""
    cfg = Config(sdims=2, nx1=n, nx2=n, nx3=1, ngc=3 if (rec == "lim5th" or shock_flattening) else 2, nas=0,
                 mhd=True, riemann=riemann, rec=rec, shock_flattening=shock_flattening, eps_sf=eps_sf, rk_stages=3,
                 bc=[["periodic", "periodic"]] * 3, gamma_ad=5.0 / 3.0, mu=1.0, cfl=0.8,
                 mach_cutoff=1e-4, mach_ct=1e-6)
    h = HostGrid(cfg)
    B0 = 1.0 / math.sqrt(4.0 * math.pi)
    xn, yn, _ = h.node_coords()
    Az = B0 / (2.0 * math.pi) * np.cos(2.0 * math.pi * yn) + B0 / (4.0 * math.pi) * np.cos(4.0 * math.pi * xn)
    inv_dx1 = 1.0 / cfg.dx()[0]
    inv_dx2 = 1.0 / cfg.dx()[1]
    nx = n
    b1 = h.b_x[0]
    b2 = h.b_x[1]
    # b_x1(i,j) = (Az(i,j+1)-Az(i,j))*inv_dx2 for i=lx1..ux1+1, j=lx2..ux2 (array index +1)
    b1[1:nx + 2, 1:nx + 1, 0] = (Az[:, 1:, 0] - Az[:, :-1, 0]) * inv_dx2
    b2[1:nx + 1, 1:nx + 2, 0] = -(Az[1:, :, 0] - Az[:-1, :, 0]) * inv_dx1
    x, y, _ = h.coords()
    h.prim[0] = 25.0 / (36.0 * math.pi)
    h.prim[3] = 5.0 / (12.0 * math.pi)
    h.prim[1] = -np.sin(2.0 * math.pi * y)
    h.prim[2] = np.sin(2.0 * math.pi * x)
    return cfg, h


def blast_2d(n=128, riemann="hllc", rec="lim2nd", shock_flattening=True, eps_sf=0.25, p_in=10.0, p_out=0.1,
             nas=1):
    """Cylindrical blast wave on the periodic unit square: rho = 1, v = 0, p = p_in inside
    r < 0.1 of the centre and p_out outside, one passive scalar marking the hot gas; ideal gas
    gamma = 5/3.  A strong shock for the shock flattener (USE_SHOCK_FLATTENING)."""
    cfg = Config(sdims=2, nx1=n, nx2=n, nx3=1, ngc=3, nas=nas, riemann=riemann, rec=rec,
                 shock_flattening=shock_flattening, eps_sf=eps_sf, rk_stages=3,
                 bc=[["periodic", "periodic"]] * 3, gamma_ad=5.0 / 3.0, mu=1.0, cfl=0.8, mach_cutoff=1e-4)
    h = HostGrid(cfg)
    x, y, _ = h.coords()
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2
    inside = r2 < 0.01
    h.prim[0] = 1.0
    h.prim[1] = 0.0
    h.prim[2] = 0.0
    h.prim[3] = np.where(inside, p_in, p_out)
    for iv in range(nas):
        h.prim[4 + iv] = np.where(inside, 1.0, 0.0)
    h.temp[...] = h.prim[3] / (CONST_RGAS * h.prim[0])
    return cfg, h


# ------------------------------------------------------------------------------ stratified Helmholtz boxes
STRAT_ABAR = 13.7
STRAT_ZBAR = 6.9


def stratified_3d(n=256, ny=None, nz=None, mhd=False, beta=1.0e4, mach=1.0e-3, seed=12345,
                  riemann=None, table=X2_TABLE, fasteos=True, rec="lim2nd", shock_flattening=False, eps_sf=0.25,
                  eos_model="synthetic"):
    """3D stratified convection box with the Helmholtz EoS.

    x2 is vertical (reflecting walls), x1 and x3 periodic.  rho_eq(y) falls exponentially from
    1e6 to 1e5 g/cm^3 over the height, p_eq is the exact integral of dp/dy = -rho_eq g with g
    chosen so that T_eq spans ~1e8 (top) to ~3e8 K (bottom).  Abar = 13.7 and Zbar = 6.9 are
    advected as Ye and 1/Abar.  Velocities are mach * c_s * U[-1,1] per component from a
    counter-based hash (seed).  With mhd=True a uniform horizontal B_x1 of plasma beta `beta` at
    mid-height is added and the LHLLD solver with constrained transport is used.  fasteos=False
    selects the Helmholtz path without USE_FASTEOS (helm_rhoP_given per Riemann side); rec picks
    the reconstruction (lim2nd, pph, lim5th; lim5th uses 3 ghost layers); shock_flattening
    enables USE_SHOCK_FLATTENING with threshold eps_sf (3 ghost layers).  eos_model names the
    electron free energy the table is built from ("synthetic": helm_table.generate, "fermi":
    helm_fermi.generate); the hydrostatic background is computed with the same model.
    """
    pressure, energy, temperature = EOS_MODELS[eos_model]
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    abar, zbar = STRAT_ABAR, STRAT_ZBAR
    ye = zbar / abar
    rho_bot, rho_top = 1.0e6, 1.0e5
    Hrho = 1.0e8
    L = Hrho * math.log(rho_bot / rho_top)
    Lx = L
    p_top = float(pressure(rho_top, 1.0e8, abar, zbar))
    p_bot = float(pressure(rho_bot, 3.0e8, abar, zbar))
    g = (p_bot - p_top) / (rho_bot * Hrho * (1.0 - rho_top / rho_bot))
    cfg = Config(sdims=3, nx1=n, nx2=ny, nx3=nz, ngc=3 if (rec == "lim5th" or shock_flattening) else 2, nas=2,
                 mhd=mhd, wb=True, gravity=True, etot=True, rec=rec, helmholtz=True, fasteos=fasteos,
                 shock_flattening=shock_flattening, eps_sf=eps_sf,
                 riemann=riemann or ("lhlld" if mhd else "lhllc"), rk_stages=3,
                 bc=[["periodic", "periodic"], ["reflective", "reflective"], ["periodic", "periodic"]],
                 x1l=0.0, x1u=Lx * n / ny, x2l=0.0, x2u=L, x3l=0.0, x3u=Lx * nz / ny,
                 gamma_ad=5.0 / 3.0, mu=1.0, cfl=0.8, mach_cutoff=1e-4, mach_ct=1e-6,
                 helm_nT=table["nT"], helm_nrho=table["nrho"], helm_ltlo=table["ltlo"],
                 helm_lthi=table["lthi"], helm_ldlo=table["ldlo"], helm_ldhi=table["ldhi"])
    h = HostGrid(cfg)

    def rho_of(y):
        return rho_bot * np.exp(-y / Hrho)

    def p_of(y):
        return p_top + g * rho_bot * Hrho * (np.exp(-y / Hrho) - rho_top / rho_bot)

    def phi_of(y):
        return g * y

    # the background depends on height only: evaluate it on the x2 profile and broadcast
    dy = cfg.dx()[1]
    yc = cfg.x2l + (np.arange(1 - cfg.ngc, ny + cfg.ngc + 1) - 0.5) * dy
    re1, pe1 = rho_of(yc), p_of(yc)
    Te1 = temperature(re1, pe1, abar, zbar, T0=2e8)
    ee1 = re1 * energy(re1, Te1, abar, zbar)
    shp = (1, -1, 1)
    re, pe, Te, ee = (a.reshape(shp) for a in (re1, pe1, Te1, ee1))
    h.prim[0] = re
    h.prim[4] = pe
    h.prim[5] = ye
    h.prim[6] = 1.0 / abar
    cs = np.sqrt(5.0 / 3.0 * np.abs(pe) / re)
    gi = np.arange(h.cell_shape[0])[:, None, None] - cfg.ngc
    gj = np.arange(h.cell_shape[1])[None, :, None] - cfg.ngc
    gk = np.arange(h.cell_shape[2])[None, None, :] - cfg.ngc
    gi, gj, gk = np.broadcast_arrays(gi, gj, gk)
    gi = np.mod(gi, n).astype(np.uint64)
    gk = np.mod(gk, nz).astype(np.uint64)
    gj = np.clip(gj, 0, ny - 1).astype(np.uint64)
    for c in range(3):
        h.prim[1 + c] = mach * cs * hash_uniform(seed, gi, gj, gk, c)
    h.temp[...] = Te
    h.grav[0] = 0.0
    h.grav[1] = -g
    h.grav[2] = 0.0
    h.phi_cc[...] = phi_of(yc).reshape(shp)
    h.eq_prim_cc[0] = re
    h.eq_prim_cc[1] = pe
    h.eq_prim_cc[2] = Te
    h.eq_gammae_cc[...] = pe / ee + 1.0
    for d in range(3):
        nyf = ny + (d == 1)
        yf = cfg.x2l + (np.arange(1, nyf + 1) - (1.0 if d == 1 else 0.5)) * dy
        rf, pf = rho_of(yf), p_of(yf)
        Tf = temperature(rf, pf, abar, zbar, T0=2e8)
        gf = pf / (rf * energy(rf, Tf, abar, zbar)) + 1.0
        h.eq_prim_x[d][0] = rf.reshape(shp)
        h.eq_prim_x[d][1] = pf.reshape(shp)
        h.eq_prim_x[d][2] = Tf.reshape(shp)
        h.eq_gammae_x[d][...] = gf.reshape(shp)
        h.phi_x[d][...] = phi_of(yf).reshape(shp)
    if mhd:
        B = math.sqrt(2.0 * float(p_of(0.5 * L)) / beta)
        h.b_x[0][...] = B
        h.b_x[1][...] = 0.0
        h.b_x[2][...] = 0.0
    return cfg, h


# ------------------------------------------------------------------------------ EoS samples
def eos_samples(n, seed=20240601):
    """(rho, T, Abar, Zbar) with log10 rho ~ U[-2, 9], log10 T ~ U[4, 10], Abar ~ U[1, 56],
    Zbar ~ U[1, Abar/2]  (n samples, counter-based hash stream)."""
    idx = np.arange(n, dtype=np.uint64)
    u = [0.5 * (hash_uniform(seed, idx, 0, 0, c) + 1.0) for c in range(4)]
    lrho = -2.0 + 11.0 * u[0]
    lT = 4.0 + 6.0 * u[1]
    abar = 1.0 + 55.0 * u[2]
    # Zbar ~ U[1, Abar/2]; for Abar < 2 the range is empty and Zbar = 1 (hydrogen-like)
    zbar = 1.0 + np.maximum(abar / 2.0 - 1.0, 0.0) * u[3]
    return 10.0 ** lrho, 10.0 ** lT, abar, zbar


def config_by_name(name, **kw):
    """Named configurations: 'hot_bubble', 'orszag_tang', 'stratified', 'stratified_mhd'."""
    if name == "hot_bubble":
        return hot_bubble_2d(**kw)
    if name == "orszag_tang":
        return orszag_tang_2d(**kw)
    if name == "stratified":
        return stratified_3d(**kw)
    if name == "stratified_mhd":
        return stratified_3d(mhd=True, **kw)
    raise KeyError(name)
