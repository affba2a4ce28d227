"""Known-answer tests: the oracle (and, marked gpu, the CUDA forms) against exact solutions of the
equations, independent of any restatement of the reference.

* Sod's shock tube (ideal gas, gamma = 1.4) against the exact solution of the Riemann problem
  (Toro, "Riemann Solvers and Numerical Methods for Fluid Dynamics", ch. 4: Newton iteration on
  the pressure function for p*, then the self-similar wave pattern sampled at x / t): the
  density's L1 error is small and falls with resolution (first order, as at any shock).
* A circularly polarized Alfven wave (an exact nonlinear solution of ideal MHD: constant total
  pressure, travelling at the Alfven speed B_x / sqrt(rho) without change of shape), one period
  along x1 in a 3D box with HLLD and constrained transport: the transverse B and v come back in
  phase with second-order convergence, without exciting compressive motion, and div B stays at
  rounding.
* A stationary contact discontinuity (density jump at uniform pressure and zero velocity; with B
  uniform for MHD) is an exact steady solution that the contact-resolving solvers (HLLC and
  LHLLC, HLLD and LHLLD) keep without diffusing it: the mass flux through every face is zero.
* A linear sound wave travels one period at the sound speed: the convergence rate of the
  density's L1 error shows the order of each reconstruction.  LIM2ND_REC sets the edge values
  to q -+ slope / 2 with slope = df db / (df + db) (source.F90:8141-8181): half the van Leer
  slope, so on smooth data the scheme is first order (the error halves per doubling); PPH_REC
  and LIM5TH_REC converge faster than second order until their extremum limiters and the
  third-order Runge-Kutta stepper set the rate.
* The Gresho vortex, a steady rotating flow in pressure balance, at Mach 0.1 and 0.01: LHLLC
  keeps the same fraction of the kinetic energy at both Mach numbers, HLLC loses more at the
  lower one (the low-Mach dissipation problem the LHLLC solver addresses); threaded by a
  uniform axial field, LHLLD does the same while the Alfven speed stays below the flow speed.
* The Runge-Kutta steppers are second (RK2) and third (RK3) order in time.
"""
import math

import numpy as np
import pytest

from phlegethon_b200.grid import Config, HostGrid
from util import div_b_max

GAMMA_SOD = 1.4


# ------------------------------------------------------------------------------ exact Riemann solver
def _pressure_function(p, rho, pk, ck, g):
    """f_K(p) and f_K'(p) of one side (shock branch for p > p_K, rarefaction otherwise)."""
    if p > pk:
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        sq = math.sqrt(A / (p + B))
        return (p - pk) * sq, sq * (1.0 - 0.5 * (p - pk) / (p + B))
    r = p / pk
    f = 2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0)
    return f, 1.0 / (rho * ck) * r ** (-(g + 1.0) / (2.0 * g))


def exact_riemann(left, right, g, xi):
    """Exact solution (rho, u, p) at the similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _pressure_function(p, rl, pl, cl, g)
        fr, dr = _pressure_function(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(1e-10, p - dp)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = _pressure_function(p, rl, pl, cl, g)
    fr, _ = _pressure_function(p, rr, pr, cr, g)
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    gm1, gp1 = g - 1.0, g + 1.0
    out = np.zeros((3, xi.size))
    for n, s in enumerate(xi):
        if s <= us:  # left of the contact
            if p > pl:
                sl = ul - cl * math.sqrt(gp1 / (2 * g) * p / pl + gm1 / (2 * g))
                st = (rl * ((p / pl + gm1 / gp1) / (gm1 / gp1 * p / pl + 1.0)), us, p) if s > sl else left
            else:
                csl = cl * (p / pl) ** (gm1 / (2 * g))
                head, tail = ul - cl, us - csl
                if s <= head:
                    st = left
                elif s >= tail:
                    st = (rl * (p / pl) ** (1.0 / g), us, p)
                else:
                    u = 2.0 / gp1 * (cl + gm1 / 2.0 * ul + s)
                    c = 2.0 / gp1 * (cl + gm1 / 2.0 * (ul - s))
                    rho = rl * (c / cl) ** (2.0 / gm1)
                    st = (rho, u, pl * (c / cl) ** (2.0 * g / gm1))
        else:  # right of the contact
            if p > pr:
                sr = ur + cr * math.sqrt(gp1 / (2 * g) * p / pr + gm1 / (2 * g))
                st = (rr * ((p / pr + gm1 / gp1) / (gm1 / gp1 * p / pr + 1.0)), us, p) if s < sr else right
            else:
                csr = cr * (p / pr) ** (gm1 / (2 * g))
                head, tail = ur + cr, us + csr
                if s >= head:
                    st = right
                elif s <= tail:
                    st = (rr * (p / pr) ** (1.0 / g), us, p)
                else:
                    u = 2.0 / gp1 * (-cr + gm1 / 2.0 * ur + s)
                    c = 2.0 / gp1 * (cr - gm1 / 2.0 * (ur - s))
                    rho = rr * (c / cr) ** (2.0 / gm1)
                    st = (rho, u, pr * (c / cr) ** (2.0 * g / gm1))
        out[:, n] = st
    return out


def test_exact_riemann_solver_sod_star_state():
    """The exact solver reproduces the published star state of Sod's problem (Toro, Table 4.2:
    p* = 0.30313, u* = 0.92745)."""
    g = GAMMA_SOD
    sol = exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), g, np.array([0.5]))
    assert abs(sol[2, 0] - 0.30313) < 5e-5 and abs(sol[1, 0] - 0.92745) < 5e-5


def sod(n, riemann="hllc"):
    cfg = Config(sdims=2, nx1=n, nx2=4, nx3=1, ngc=2, nas=0, riemann=riemann, rk_stages=3,
                 bc=[["reflective", "reflective"], ["periodic", "periodic"], ["periodic", "periodic"]],
                 x1l=0.0, x1u=1.0, x2l=0.0, x2u=4.0 / n, x3l=0.0, x3u=1.0, gamma_ad=GAMMA_SOD, mu=1.0, cfl=0.8,
                 mach_cutoff=1e-4)
    h = HostGrid(cfg)
    x, _, _ = h.coords()
    left = x < 0.5
    h.prim[0] = np.where(left, 1.0, 0.125)
    h.prim[1] = 0.0
    h.prim[2] = 0.0
    h.prim[3] = np.where(left, 1.0, 0.1)
    h.temp[...] = h.prim[3] / h.prim[0]
    return cfg, h


def sod_error(h, t):
    x, _, _ = h.coords()
    xs = h.interior(x)[:, 0, 0]
    ex = exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), GAMMA_SOD, (xs - 0.5) / t)
    rho = h.interior(h.prim)[0][:, 0, 0]
    # every row along x2 is the same (the problem is uniform in x2)
    assert np.all(h.interior(h.prim)[0] == rho[:, None, None])
    return float(np.mean(np.abs(rho - ex[0])))


def run_oracle(oracle, cfg, h, tmax):
    o = oracle.OracleGrid(h, None)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(100000, tmax)
    assert abs(o.g.time - tmax) < 1e-12
    return h


@pytest.mark.parametrize("riemann", ["hllc", "lhllc"])
def test_sod_shock_tube_against_exact_solution(oracle, riemann):
    errs = []
    for n in (128, 256):
        cfg, h = sod(n, riemann)
        run_oracle(oracle, cfg, h, 0.2)
        errs.append(sod_error(h, 0.2))
    # PLM + RK3 on Sod: L1(rho) about 1e-2 at 128 cells (measured 0.0117 HLLC, 0.0097 LHLLC),
    # falling as N^-0.7 (the shock and contact are first order); a wrong wave speed or jump
    # condition puts whole cells of the profile off by O(0.1)
    assert errs[0] < 0.015 and errs[1] < 0.7 * errs[0], errs


# ------------------------------------------------------------------------------ Alfven wave
ALFVEN_AMP = 0.1


def alfven_wave(n, riemann="hlld"):
    """Circularly polarized Alfven wave along x1: rho = 1, p = 0.1, B = (1, A sin 2 pi x, A cos 2 pi x),
    v = -B_perp / sqrt(rho); it travels at v_A = 1 and returns after t = 1."""
    m = 4
    cfg = Config(sdims=3, nx1=n, nx2=m, nx3=m, ngc=2, nas=0, mhd=True, riemann=riemann, rk_stages=3,
                 bc=[["periodic", "periodic"]] * 3, x1l=0.0, x1u=1.0, x2l=0.0, x2u=m / n, x3l=0.0, x3u=m / n,
                 gamma_ad=5.0 / 3.0, mu=1.0, cfl=0.8, mach_cutoff=1e-4, mach_ct=1e-6)
    h = HostGrid(cfg)
    x, _, _ = h.coords()
    A, tp = ALFVEN_AMP, 2.0 * math.pi
    h.prim[0] = 1.0
    h.prim[1] = 0.0
    h.prim[2] = -A * np.sin(tp * x)
    h.prim[3] = -A * np.cos(tp * x)
    h.prim[4] = 0.1
    h.temp[...] = 0.1
    dx = 1.0 / n
    # face fields: B_x on x1 faces is uniform; B_y (B_z) on x2 (x3) faces depends on x1 only, so
    # div B vanishes exactly; the arrays' first index i holds cell i - 1 (one ghost layer)
    h.b_x[0][...] = 1.0
    xc = (np.arange(h.b_x[1].shape[0]) - 1 + 0.5) * dx
    h.b_x[1][...] = (A * np.sin(tp * xc))[:, None, None]
    xc = (np.arange(h.b_x[2].shape[0]) - 1 + 0.5) * dx
    h.b_x[2][...] = (A * np.cos(tp * xc))[:, None, None]
    return cfg, h


def fit_wave(a, n):
    """Amplitude and phase of a one-wavelength sinusoid a(x) = amp sin(2 pi x + phase) on n cells."""
    x = (np.arange(n) + 0.5) / n
    basis = np.array([np.sin(2 * np.pi * x), np.cos(2 * np.pi * x)]).T
    cs, cc = np.linalg.lstsq(basis, a[:n], rcond=None)[0]
    return float(np.hypot(cs, cc)), float(np.arctan2(cc, cs))


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_alfven_wave_returns_after_one_period(oracle, riemann):
    """After one period the wave is back in phase to second order (it travels at the Alfven
    speed); its amplitude decays at first order, as the LIM2ND limiter clips smooth extrema; the
    compressive fields it must not excite (v_x, rho) stay at the 1e-4 level; div B at rounding."""
    res = []
    for n in (32, 64, 128):
        cfg, h = alfven_wave(n, riemann)
        run_oracle(oracle, cfg, h, 1.0)
        amp, ph = fit_wave(h.bface_interior(1)[:, 0, 0], n)
        vamp, vph = fit_wave(-h.interior(h.prim)[2][:, 0, 0], n)
        res.append((amp / ALFVEN_AMP, abs(ph), vamp / ALFVEN_AMP, abs(vph)))
        assert float(np.abs(h.interior(h.prim)[1]).max()) < 2e-4
        assert float(np.abs(h.interior(h.prim)[0] - 1.0).max()) < 2e-4
        assert div_b_max(h) <= 1e-13
    (a1, p1, va1, vp1), (a2, p2, va2, vp2), (a3, p3, va3, vp3) = res
    # phase error: about 4x smaller per doubling (measured 0.011, 0.0026, 0.0006 with HLLD)
    assert p2 < 0.35 * p1 and p3 < 0.35 * p2 and p3 < 2e-3, res
    assert vp3 < 2e-3, res
    # amplitude loss 1 - amp about halves per doubling (measured 0.27, 0.14, 0.074)
    assert (1 - a2) < 0.6 * (1 - a1) and (1 - a3) < 0.6 * (1 - a2) and a3 > 0.9, res
    assert abs(va3 - a3) < 0.02, res


# ------------------------------------------------------------------------------ fast magnetosonic wave
FAST_EPS = 1e-6


def fast_wave(n, riemann):
    """Linear fast magnetosonic wave along x1 across a uniform B = (0, 1): rho = 1 + eps sin 2 pi x,
    v_x = c_f eps sin, p = 1 + c_s^2 eps sin, B_y = 1 + eps sin, with c_s^2 = gamma p / rho = 5/3,
    v_A = 1 and c_f = sqrt(c_s^2 + v_A^2); it returns in place after t = 1 / c_f.  (c_s differs
    from v_A on purpose: where they are equal along a face normal the reference's fast-speed
    discriminant is zero in exact arithmetic and can round negative.)"""
    g, p0, b0 = 5.0 / 3.0, 1.0, 1.0
    cfg = Config(sdims=2, nx1=n, nx2=4, nx3=1, ngc=2, nas=0, mhd=True, riemann=riemann, rk_stages=3,
                 bc=[["periodic", "periodic"]] * 3, x1l=0.0, x1u=1.0, x2l=0.0, x2u=4.0 / n, x3l=0.0, x3u=1.0,
                 gamma_ad=g, mu=1.0, cfl=0.8, mach_cutoff=1e-4, mach_ct=1e-6)
    h = HostGrid(cfg)
    x, _, _ = h.coords()
    cs2 = g * p0
    cf = math.sqrt(cs2 + b0 * b0)
    s = np.sin(2.0 * np.pi * x)
    h.prim[0] = 1.0 + FAST_EPS * s
    h.prim[1] = cf * FAST_EPS * s
    h.prim[2] = 0.0
    h.prim[3] = p0 + cs2 * FAST_EPS * s
    h.temp[...] = h.prim[3] / h.prim[0]
    h.b_x[0][...] = 0.0
    # B_y on x2 faces depends on x1 only; the arrays' first index i holds cell i - 1
    xc = (np.arange(h.b_x[1].shape[0]) - 1 + 0.5) / n
    h.b_x[1][...] = (b0 * (1.0 + FAST_EPS * np.sin(2.0 * np.pi * xc)))[:, None, None]
    return cfg, h, cf


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_fast_magnetosonic_wave_returns_after_one_period(oracle, riemann):
    """After t = 1 / c_f the compressive wave is back in phase to second order (it travels at the
    fast speed, which the magnetic pressure in the flux sets: at the sound speed alone it would
    lag by 2 pi (1 - c_s / c_f) = 0.66 rad), density and B_y stay in the eigenvector ratio
    dB_y / B_y = drho / rho, the amplitude decays at first order (the LIM2ND limiter) and no
    transverse velocity appears."""
    res = []
    for n in (32, 64, 128):
        cfg, h, cf = fast_wave(n, riemann)
        run_oracle(oracle, cfg, h, 1.0 / cf)
        amp, ph = fit_wave(h.interior(h.prim)[0][:, 0, 0] - 1.0, n)
        bamp, bph = fit_wave(h.bface_interior(1)[:n, 0, 0] - 1.0, n)
        res.append((amp / FAST_EPS, abs(ph), bamp / FAST_EPS, abs(bph)))
        assert float(np.abs(h.interior(h.prim)[2]).max()) == 0.0
    (a1, p1, b1, q1), (a2, p2, b2, q2), (a3, p3, b3, q3) = res
    # measured phase 0.0110, 0.0026, 0.00064; amplitude 0.731, 0.857, 0.926
    assert p2 < 0.3 * p1 and p3 < 0.3 * p2 and p3 < 1e-3, res
    assert (1 - a2) < 0.6 * (1 - a1) and (1 - a3) < 0.6 * (1 - a2) and a3 > 0.9, res
    assert abs(b3 - a3) < 1e-3 * a3 and abs(q3 - p3) < 1e-6, res


# ------------------------------------------------------------------------------ free fall
@pytest.mark.parametrize("etot", [False, True])
@pytest.mark.parametrize("riemann", ["hllc", "lhllc"])
def test_uniform_gas_falls_freely(oracle, riemann, etot):
    """A uniform gas at rest (rho = 1, p = 1) between reflecting walls under g = -1 (no
    well-balancing) falls freely away from the walls: after 5 steps the cells beyond the walls'
    numerical reach (3 stages x 2 cells per step) move at v = g t exactly (third-order
    Runge-Kutta integrates the constant acceleration exactly), at unchanged density and
    pressure: gravity's work (source.F90:12631-12638, or the potential carried by the mass flux
    under EVOLVE_ETOT) goes into kinetic energy alone."""
    from phlegethon_b200.problems import CONST_RGAS
    cfg = Config(sdims=2, nx1=16, nx2=128, nx3=1, ngc=2, nas=0, gravity=True, etot=etot, riemann=riemann,
                 rk_stages=3, bc=[["periodic", "periodic"], ["reflective", "reflective"], ["periodic", "periodic"]],
                 gamma_ad=5.0 / 3.0, mu=1.0, cfl=0.8, mach_cutoff=1e-4)
    h = HostGrid(cfg)
    _, y, _ = h.coords()
    h.prim[0] = 1.0
    h.prim[1] = 0.0
    h.prim[2] = 0.0
    h.prim[3] = 1.0
    h.grav[0] = 0.0
    h.grav[1] = -1.0
    if etot:
        h.phi_cc[...] = y
        for d in range(2):
            _, fy, _ = h.face_coords(d)
            h.phi_x[d][...] = fy
    h.temp[...] = 1.0 / CONST_RGAS
    o = oracle.OracleGrid(h, None)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(5)
    t = o.g.time
    w = h.interior(h.prim)[:, :, 40:88, 0]
    assert float(np.abs(w[2] + t).max()) <= 1e-14 and float(np.abs(w[1]).max()) == 0.0
    assert float(np.abs(w[0] - 1.0).max()) <= 1e-14 and float(np.abs(w[3] - 1.0).max()) <= 1e-14


# ------------------------------------------------------------------------------ stationary contact
def stationary_contact(n, riemann, mhd=False):
    """rho = 1 in 0.25 < x < 0.75 and 0.125 elsewhere (periodic), p = 1, v = 0; MHD: B = (0.75, 0.5)
    uniform, so the total pressure is uniform too."""
    cfg = Config(sdims=2, nx1=n, nx2=4, nx3=1, ngc=2, nas=0, riemann=riemann, rk_stages=3, mhd=mhd,
                 bc=[["periodic", "periodic"]] * 3, x1l=0.0, x1u=1.0, x2l=0.0, x2u=4.0 / n, x3l=0.0, x3u=1.0,
                 gamma_ad=1.4, mu=1.0, cfl=0.8, mach_cutoff=1e-4, mach_ct=1e-6)
    h = HostGrid(cfg)
    x, _, _ = h.coords()
    h.prim[0] = np.where((x > 0.25) & (x < 0.75), 1.0, 0.125)
    h.prim[1] = 0.0
    h.prim[2] = 0.0
    h.prim[3] = 1.0
    h.temp[...] = h.prim[3] / h.prim[0]
    if mhd:
        h.b_x[0][...] = 0.75
        h.b_x[1][...] = 0.5
    return cfg, h


@pytest.mark.parametrize("riemann,mhd", [("hllc", False), ("lhllc", False), ("hlld", True), ("lhlld", True)])
def test_stationary_contact_is_kept(oracle, riemann, mhd):
    """50 steps: density and pressure unchanged bit for bit, the velocity at rounding (LHLLD forms
    its star total pressure as a weighted mean of the two equal sides, which rounds)."""
    cfg, h = stationary_contact(64, riemann, mhd)
    w0 = h.interior(h.prim).copy()
    o = oracle.OracleGrid(h, None)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(50)
    w = h.interior(h.prim)
    assert np.array_equal(w[0], w0[0]) and np.array_equal(w[3], w0[3])
    assert float(np.abs(w[1:3]).max()) <= 1e-14


# ------------------------------------------------------------------------------ sound wave
SOUND_EPS = 1e-6


def sound_wave(n, rec="lim2nd", riemann="hllc"):
    """Linear sound wave rho = 1 + eps sin 2 pi x, v = c eps sin 2 pi x, p = 1 + gamma eps sin 2 pi x
    (gamma = 1.4, c = sqrt(1.4)); it returns in place after t = 1 / c."""
    g = 1.4
    cfg = Config(sdims=2, nx1=n, nx2=4, nx3=1, ngc=3 if rec == "lim5th" else 2, nas=0, riemann=riemann, rk_stages=3,
                 rec=rec, bc=[["periodic", "periodic"]] * 3, x1l=0.0, x1u=1.0, x2l=0.0, x2u=4.0 / n, x3l=0.0,
                 x3u=1.0, gamma_ad=g, mu=1.0, cfl=0.8, mach_cutoff=1e-4)
    h = HostGrid(cfg)
    x, _, _ = h.coords()
    s = np.sin(2 * np.pi * x)
    h.prim[0] = 1.0 + SOUND_EPS * s
    h.prim[1] = math.sqrt(g) * SOUND_EPS * s
    h.prim[2] = 0.0
    h.prim[3] = 1.0 + g * SOUND_EPS * s
    h.temp[...] = h.prim[3] / h.prim[0]
    return cfg, h


def sound_wave_error(oracle, n, rec):
    """L1 error of the density after one period against the exact cell averages, over eps."""
    cfg, h = sound_wave(n, rec)
    run_oracle(oracle, cfg, h, 1.0 / math.sqrt(1.4))
    x, _, _ = h.coords()
    xs = h.interior(x)[:, 0, 0]
    k = 2.0 * np.pi
    exact = 1.0 + SOUND_EPS * (np.cos(k * (xs - 0.5 / n)) - np.cos(k * (xs + 0.5 / n))) / (k / n)
    return float(np.mean(np.abs(h.interior(h.prim)[0][:, 0, 0] - exact))) / SOUND_EPS


def test_sound_wave_convergence_by_reconstruction(oracle):
    e2 = [sound_wave_error(oracle, n, "lim2nd") for n in (32, 64, 128)]
    # LIM2ND: first order (measured 0.170, 0.091, 0.047: rates 0.90, 0.95)
    r2 = [math.log2(e2[i] / e2[i + 1]) for i in range(2)]
    assert all(0.8 < r < 1.2 for r in r2) and 0.1 < e2[0] < 0.25, (e2, r2)
    # PPH and LIM5TH: at 64 cells over 10x below LIM2ND, above second order from 16 to 64 cells
    # (measured PPH 0.0160, 0.00157, 7.0e-5; LIM5TH 0.040, 0.0075, 0.0015)
    for rec in ("pph", "lim5th"):
        e = [sound_wave_error(oracle, n, rec) for n in (16, 32, 64)]
        rate = math.log2(e[0] / e[2]) / 2
        assert e[2] < 0.1 * e2[1] and rate > 2.2, (rec, e, rate)


# ------------------------------------------------------------------------------ conservation
def conserved_totals(h, gamma):
    """Sums over the interior of rho, rho v (per component) and the total energy e + rho v^2 / 2
    (+ B_cc^2 / 2), with e = p / (gamma - 1) (ideal gas)."""
    w = h.interior(h.prim)
    rho, v, p = w[0], w[1:1 + h.cfg.sdims], w[1 + h.cfg.sdims]
    E = p / (gamma - 1.0) + 0.5 * rho * np.sum(v * v, axis=0)
    if h.cfg.mhd:
        b = h.interior(h.b_cc)
        E = E + 0.5 * np.sum(b * b, axis=0)
    return float(rho.sum()), [float((rho * vd).sum()) for vd in v], float(E.sum()), \
        float(np.abs(rho * v).sum())


@pytest.mark.parametrize("case", ["blast_hllc", "blast_lhllc", "orszag_tang_hlld", "orszag_tang_lhlld"])
def test_periodic_box_conserves_mass_momentum_energy(oracle, case):
    """Finite-volume conservation: in a periodic box without sources every face flux leaves one
    cell and enters its neighbour, so the totals of mass, momentum and energy change only by
    rounding (a flux used with different values on its two sides, a wrong face index or a sign
    error shows up as a drift of order the flux)."""
    from phlegethon_b200 import problems
    if case.startswith("blast"):
        cfg, h = problems.blast_2d(64, riemann=case.split("_")[1], shock_flattening=False, nas=0)
    else:
        cfg, h = problems.orszag_tang_2d(64, riemann=case.split("_")[2])
    g = cfg.gamma_ad
    o = oracle.OracleGrid(h, None)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    m0, p0, e0, pabs0 = conserved_totals(h, g)
    o.time_loop(50)
    m1, p1, e1, pabs1 = conserved_totals(h, g)
    assert abs(m1 - m0) <= 1e-13 * m0, (m0, m1)
    scale = max(pabs0, pabs1)
    for a, b in zip(p0, p1):
        assert abs(b - a) <= 1e-13 * scale, (p0, p1)
    assert abs(e1 - e0) <= 1e-13 * e0, (e0, e1)


# ------------------------------------------------------------------------------ Gresho vortex
def gresho(n, riemann, mach, gamma=5.0 / 3.0):
    """The Gresho vortex, an exact steady solution of the Euler equations (Gresho & Chan 1990;
    the low-Mach form of Miczek et al. 2015): v_phi = 5r (r < 0.2), 2 - 5r (r < 0.4), 0 beyond,
    with the pressure that balances its centrifugal force, p = p0 + 12.5 r^2 (r < 0.2),
    p0 + 12.5 r^2 + 4 (1 - 5r - ln 0.2 + ln r) (r < 0.4), p0 - 2 + 4 ln 2 beyond; rho = 1 and
    p0 = 1 / (gamma M^2) - 1/2 sets the maximum Mach number M (the reference's tests/gresho
    set-up: 40^2, gamma 5/3, LIM2ND, Mach_cutoff 1e-4)."""
    cfg = Config(sdims=2, nx1=n, nx2=n, riemann=riemann, bc=[["periodic", "periodic"]] * 3,
                 gamma_ad=gamma, mach_cutoff=1e-4, cfl=0.8)
    h = HostGrid(cfg)
    x, y, _ = h.coords()
    dx, dy = x - 0.5, y - 0.5
    r = np.sqrt(dx * dx + dy * dy)
    rr = np.maximum(r, 1e-300)
    vphi = np.where(r < 0.2, 5.0 * r, np.where(r < 0.4, 2.0 - 5.0 * r, 0.0))
    p0 = 1.0 / gamma / mach ** 2 - 0.5
    p = np.where(r < 0.2, p0 + 12.5 * r * r,
                 np.where(r < 0.4, p0 + 12.5 * r * r + 4.0 * (1.0 - 5.0 * r - math.log(0.2) + np.log(rr)),
                          p0 - 2.0 + 4.0 * math.log(2.0)))
    h.prim[0] = 1.0
    h.prim[1] = -vphi * dy / rr
    h.prim[2] = vphi * dx / rr
    h.prim[3] = p
    return cfg, h


def test_gresho_vortex_low_mach_dissipation(oracle):
    """The low-dissipation solver's point (Minoshima & Miyoshi 2021): on the Gresho vortex the
    kinetic energy LHLLC keeps after t = 0.2 does not depend on the Mach number (the star
    pressure's dissipation scales with phi = chi (2 - chi)), while HLLC, whose dissipation does
    not fall with the Mach number, loses more of it the lower the Mach number."""
    kept = {}
    for riemann in ("lhllc", "hllc"):
        for mach in (0.1, 0.01):
            cfg, h = gresho(40, riemann, mach)
            ke0 = float((h.interior(h.prim)[1:3] ** 2).sum())
            o = oracle.OracleGrid(h, None, nthreads=4)
            o.init_thermo()
            o.compute_hyperbolic_dt()
            o.time_loop(100000, 0.2)
            kept[riemann, mach] = float((h.interior(h.prim)[1:3] ** 2).sum()) / ke0
    assert abs(kept["lhllc", 0.1] - kept["lhllc", 0.01]) < 2e-3
    assert kept["lhllc", 0.01] > 0.85
    assert kept["hllc", 0.01] < kept["hllc", 0.1] - 0.1
    assert kept["lhllc", 0.01] > kept["hllc", 0.01] + 0.3


def gresho_mhd(n, riemann, mach, bz):
    """The Gresho vortex in a thin periodic 3D box threaded by a uniform B_3 = bz sqrt(p0) along
    its axis: B is uniform and v does not vary along it, so the induction equation leaves it
    unchanged and the vortex stays an exact steady state of ideal MHD (Alfven speed over sound
    speed bz / sqrt(gamma))."""
    cfg2, h2 = gresho(n, riemann, mach)
    cfg = cfg2.replace(sdims=3, nx3=2, x3u=2.0 / n, mhd=True, mach_ct=1e-6)
    h = HostGrid(cfg)
    for v, w in ((0, 0), (1, 1), (2, 2), (4, 3)):
        h.prim[v] = h2.prim[w][:, :, :1]
    h.prim[3] = 0.0
    h.b_x[2][...] = bz * math.sqrt(1.0 / cfg.gamma_ad / mach ** 2 - 0.5)
    return cfg, h


def test_gresho_vortex_low_mach_dissipation_with_b(oracle):
    """LHLLD on the magnetised Gresho vortex: with a weak field (Alfven speed below the flow
    speed) it keeps the same fraction of the kinetic energy at Mach 0.1 and 0.01 while HLLD
    keeps less at the lower Mach number, as LHLLC does in hydro; with a field whose Alfven
    speed exceeds the flow speed the advantage is gone, because the reference's LHLLD measures
    its Mach number with cu^2 = (v^2 + a^2 + sqrt((v^2 + a^2)^2 - 4 v^2 a_n^2)) / 2, the Alfven
    speed a included (source.F90:14364-14384): then phi stays O(a / c_f) and the dissipation
    grows as the flow Mach number falls, like HLLD's."""
    kept = {}
    for riemann, bz in (("lhlld", 1e-3), ("hlld", 1e-3), ("lhlld", 0.3), ("hlld", 0.3)):
        for mach in (0.1, 0.01):
            if riemann == "hlld" and bz == 0.3 and mach == 0.1:
                continue
            cfg, h = gresho_mhd(24, riemann, mach, bz)
            ke0 = float((h.interior(h.prim)[1:3] ** 2).sum())
            o = oracle.OracleGrid(h, None, nthreads=4)
            o.init_thermo()
            o.compute_hyperbolic_dt()
            o.time_loop(100000, 0.2)
            assert float(np.abs(h.interior(h.prim)[3]).max()) == 0.0
            kept[riemann, bz, mach] = float((h.interior(h.prim)[1:3] ** 2).sum()) / ke0
    assert abs(kept["lhlld", 1e-3, 0.1] - kept["lhlld", 1e-3, 0.01]) < 3e-3
    assert kept["lhlld", 1e-3, 0.01] > kept["hlld", 1e-3, 0.01] + 0.25
    assert kept["hlld", 1e-3, 0.01] < kept["hlld", 1e-3, 0.1] - 0.03
    assert kept["lhlld", 0.3, 0.01] < kept["lhlld", 0.3, 0.1] - 0.1
    assert abs(kept["lhlld", 0.3, 0.01] - kept["hlld", 0.3, 0.01]) < 0.02


# ------------------------------------------------------------------------------ time order
def test_runge_kutta_order_in_time(oracle):
    """The Shu-Osher coefficients of RK2_STEPPER and RK3_STEPPER (source.F90:7018-7038) give
    second and third order in time: on one grid (64 cells, a density wave advected at unit
    speed, PPH_REC whose unlimited edges make the semi-discrete system smooth) the difference
    to a run at a 32 times smaller CFL number falls by 4x and 8x per halving of dt."""
    def run(stages, cfl):
        cfg = Config(sdims=2, nx1=64, nx2=4, x2u=4.0 / 64, riemann="hllc", rec="pph", rk_stages=stages,
                     bc=[["periodic", "periodic"]] * 3, cfl=cfl, gamma_ad=1.4)
        h = HostGrid(cfg)
        x, _, _ = h.coords()
        h.prim[0] = 1.0 + 0.2 * np.sin(2.0 * np.pi * x)
        h.prim[1] = 1.0
        h.prim[2] = 0.0
        h.prim[3] = 1.0
        run_oracle(oracle, cfg, h, 0.25)
        return h.interior(h.prim)[0][:, 0, 0].copy()

    for stages, order in ((2, 2.0), (3, 3.0)):
        ref = run(stages, 0.4 / 64)
        err = [float(np.abs(run(stages, c) - ref).max()) for c in (0.4, 0.2, 0.1, 0.05)]
        rates = [math.log2(err[i] / err[i + 1]) for i in range(3)]
        assert all(abs(r - order) < 0.1 for r in rates), (stages, rates)


def test_evolve_etot_conserves_total_energy_in_a_closed_box(oracle):
    """The hot bubble between reflective walls under gravity: with EVOLVE_ETOT the scheme
    evolves E + rho phi in conservation form (the potential flux F_rho phi_face,
    source.F90:8961-8966), so the box's total energy including the potential, and its mass,
    stay constant to rounding over 200 steps; with gravity as a momentum and work source
    instead (S:12631-12638) the total drifts by O(1e-5)."""
    from phlegethon_b200 import problems
    drift = {}
    for etot in (True, False):
        cfg, h = problems.hot_bubble_2d(32)
        h.cfg = cfg.replace(etot=etot)
        phi = h.interior(h.phi_cc)

        def totals():
            w, e = h.interior(h.prim), h.interior(h.eint)
            return float(w[0].sum()), float((e + 0.5 * w[0] * (w[1] ** 2 + w[2] ** 2) + w[0] * phi).sum())
        o = oracle.OracleGrid(h, None, nthreads=4)
        o.init_thermo()
        o.compute_hyperbolic_dt()
        m0, e0 = totals()
        o.time_loop(200)
        m1, e1 = totals()
        assert abs(m1 / m0 - 1.0) < 1e-13
        assert float(np.abs(h.interior(h.prim)[1:3]).max()) > 1e-2     # the bubble has risen
        drift[etot] = abs(e1 / e0 - 1.0)
    assert drift[True] < 1e-13
    assert drift[False] > 1e-6


# ------------------------------------------------------------------------------ the CUDA forms
def run_gpu(cfg, h, tmax, precision):
    from phlegethon_b200.abi import Simulation
    with Simulation(cfg.replace(precision=precision)) as sim:
        sim.upload(h)
        sim.init_thermo()
        sim.compute_hyperbolic_dt()
        t = 0.0
        while t < tmax:
            done, t = sim.time_loop(256, tmax)
            if done == 0:
                break
        sim.download(h)
    assert abs(t - tmax) < 1e-12
    return h


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_sod_on_the_gpu(gpu_lib, precision):
    cfg, h = sod(256, "hllc")
    run_gpu(cfg, h, 0.2, precision)
    # the FP64 form is bit-identical with the oracle (0.00726 at 256 cells)
    assert sod_error(h, 0.2) < 0.0075


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_alfven_wave_on_the_gpu(gpu_lib, precision):
    n = 128
    cfg, h = alfven_wave(n, "lhlld")
    run_gpu(cfg, h, 1.0, precision)
    amp, ph = fit_wave(h.bface_interior(1)[:, 0, 0], n)
    assert abs(ph) < 2e-3 and amp / ALFVEN_AMP > 0.9, (amp, ph)
    assert div_b_max(h) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("riemann,mhd", [("lhllc", False), ("lhlld", True)])
@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_stationary_contact_on_the_gpu(gpu_lib, riemann, mhd, precision):
    cfg, h = stationary_contact(64, riemann, mhd)
    w0 = h.interior(h.prim).copy()
    from phlegethon_b200.abi import Simulation
    with Simulation(cfg.replace(precision=precision)) as sim:
        sim.upload(h)
        sim.init_thermo()
        sim.compute_hyperbolic_dt()
        done, _ = sim.time_loop(50)
        sim.download(h)
    assert done == 50
    w = h.interior(h.prim)
    # FP64: the oracle's answer (density and pressure bit for bit); FP32 split: the FP32 state
    # carries the jump exactly and the mass flux vanishes, so density and pressure hold to FP32
    # rounding, and the velocity (sound speed ~1.2) stays at the level of FP32 rounding noise in
    # the LHLLD star pressure, accumulated over the 50 steps (measured 1.0e-7)
    tol = 0.0 if precision == "fp64" else 1e-7
    assert float(np.abs(w[0] - w0[0]).max()) <= tol and float(np.abs(w[3] - w0[3]).max()) <= tol
    assert float(np.abs(w[1:3]).max()) <= (1e-14 if precision == "fp64" else 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["blast_lhllc", "orszag_tang_lhlld"])
@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_conservation_on_the_gpu(gpu_lib, case, precision):
    """The periodic box's totals on the GPU: at rounding in the FP64 form; in the split form the
    flux divergence is formed from FP32 face fluxes in FP32 before it enters the FP64 state, so
    the sums over cells telescope to FP32 rounding of the fluxes (measured drifts are recorded
    in the assertion messages)."""
    from phlegethon_b200 import problems
    from phlegethon_b200.abi import Simulation
    if case.startswith("blast"):
        cfg, h = problems.blast_2d(64, riemann="lhllc", shock_flattening=False, nas=0)
    else:
        cfg, h = problems.orszag_tang_2d(64, riemann="lhlld")
    g = cfg.gamma_ad
    with Simulation(cfg.replace(precision=precision)) as sim:
        sim.upload(h)
        sim.init_thermo()
        sim.compute_hyperbolic_dt()
        sim.download(h)
        m0, p0, e0, pabs0 = conserved_totals(h, g)
        done, _ = sim.time_loop(50)
        sim.download(h)
    assert done == 50
    m1, p1, e1, pabs1 = conserved_totals(h, g)
    tol = 1e-13 if precision == "fp64" else 1e-6
    scale = max(pabs0, pabs1)
    assert abs(m1 - m0) <= tol * m0, (m0, m1)
    assert all(abs(b - a) <= tol * scale for a, b in zip(p0, p1)), (p0, p1)
    assert abs(e1 - e0) <= tol * e0, (e0, e1)
