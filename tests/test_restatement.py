"""The C oracle against the independent numpy restatement (bit for bit)."""
import numpy as np
import pytest

from phlegethon_b200 import problems
from numpy_restatement import hot_bubble_steps, mhd_2d_steps, mhd_3d_steps, stratified_steps, wb_mhd_2d_steps
from util import smooth_box


def test_oracle_matches_numpy_restatement(oracle):
    cfg, h = problems.hot_bubble_2d(40)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(4)
    W, eint, temp, dt = hot_bubble_steps(hn, 4)
    G = cfg.ngc
    I = (slice(G, G + cfg.nx1), slice(G, G + cfg.nx2))
    for v in range(4):
        np.testing.assert_array_equal(h.prim[v, :, :, 0][I], W[v][I])
    np.testing.assert_array_equal(h.interior(h.eint)[:, :, 0], eint)
    np.testing.assert_array_equal(h.interior(h.temp)[:, :, 0], temp)
    assert o.g.dt == dt


@pytest.mark.parametrize("rec", ["pph", "lim5th"])
def test_oracle_higher_order_reconstruction_matches_numpy_restatement(oracle, rec):
    """The hot bubble with PPH_REC (third order, unlimited primitives) or LIM5TH_REC (fifth
    order, limited), three ghost layers: bit for bit after five steps."""
    cfg, h = problems.hot_bubble_2d(32, shock_flattening=True, eps_sf=1e300)
    h.cfg = cfg = cfg.replace(shock_flattening=False, rec=rec)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(5)
    W, eint, temp, dt = hot_bubble_steps(hn, 5, rec=rec)
    G = cfg.ngc
    I = (slice(G, G + cfg.nx1), slice(G, G + cfg.nx2))
    for v in range(4):
        np.testing.assert_array_equal(h.prim[v, :, :, 0][I], W[v][I])
    np.testing.assert_array_equal(h.interior(h.eint)[:, :, 0], eint)
    assert o.g.dt == dt


@pytest.mark.parametrize("eps_sf", [0.1, 0.1251])
def test_oracle_shock_flattening_matches_numpy_restatement(oracle, eps_sf):
    """Detector over 3 ghost layers (deviation + ghost equilibrium) and HLL on flagged faces.
    For the 32^2 bubble the background jump 2 sinh(dy/H) = 0.12508 sits between the two
    thresholds: every cell is flagged at 0.1, only cells next to the bubble's disturbance at
    0.1251 once it has moved the pressure."""
    cfg, h = problems.hot_bubble_2d(32, shock_flattening=True, eps_sf=eps_sf)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(6)
    W, eint, temp, dt = hot_bubble_steps(hn, 6, eps_sf=eps_sf)
    G = cfg.ngc
    I = (slice(G, G + cfg.nx1), slice(G, G + cfg.nx2))
    for v in range(4):
        np.testing.assert_array_equal(h.prim[v, :, :, 0][I], W[v][I])
    np.testing.assert_array_equal(h.interior(h.eint)[:, :, 0], eint)
    assert o.g.dt == dt


@pytest.mark.parametrize("rk_stages", [3, 2])
@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_oracle_mhd_matches_numpy_restatement(oracle, riemann, rk_stages):
    """Orszag-Tang with HLLD / LHLLD and constrained transport: the C oracle and the numpy
    restatement (face EMFs, mass-flux signs, upwinded corner EMFs, face-B update, magnetic
    energy, magnetosonic dt) agree bit for bit in every primitive, e, T, both face-B arrays and
    the next dt after six steps."""
    cfg, h = problems.orszag_tang_2d(40, riemann=riemann)
    h.cfg = cfg = cfg.replace(rk_stages=rk_stages)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(6)
    W, eint, temp, b1, b2, dt = mhd_2d_steps(hn, 6, low_mach=riemann == "lhlld")
    G = cfg.ngc
    I = (slice(G, G + cfg.nx1), slice(G, G + cfg.nx2))
    for v in range(4):
        np.testing.assert_array_equal(h.prim[v, :, :, 0][I], W[v][I])
    np.testing.assert_array_equal(h.interior(h.eint)[:, :, 0], eint)
    np.testing.assert_array_equal(h.interior(h.temp)[:, :, 0], temp)
    np.testing.assert_array_equal(h.bface_interior(0)[:, :, 0], b1)
    np.testing.assert_array_equal(h.bface_interior(1)[:, :, 0], b2)
    assert o.g.dt == dt


@pytest.mark.parametrize("rec", ["lim2nd", "pph", "lim5th"])
@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_oracle_3d_mhd_matches_numpy_restatement(oracle, riemann, rec):
    """A smooth triply periodic MHD box (12 x 16 x 8, unequal extents, one passive scalar):
    the x2 / x3 frame rotations, the three face-EMF components, the three upwinded corner EMFs
    and face-B updates, the scalar's upwinded flux, the reconstruction of primitives, scalar
    (limited under PPH) and cell B, and the 3D dt sum of the C oracle equal the numpy
    restatement bit for bit after four steps."""
    h = smooth_box(3, riemann, rec, mhd=True)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(4)
    W, eint, temp, b, dt = mhd_3d_steps(hn, 4, low_mach=riemann == "lhlld")
    for v in range(h.cfg.nvars):
        np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
    np.testing.assert_array_equal(h.interior(h.eint), eint)
    np.testing.assert_array_equal(h.interior(h.temp), temp)
    for d in range(3):
        np.testing.assert_array_equal(h.bface_interior(d), b[d])
    assert o.g.dt == dt


def _magnetised_bubble(n, riemann):
    """The hot bubble (WB, EVOLVE_ETOT, gravity, reflective y walls) threaded by a field from
    the node potential A_z = 0.05 sin(2 pi x) sin^2(pi y) + 0.2 y: horizontal at the walls,
    divergence-free on the faces."""
    from phlegethon_b200.grid import HostGrid
    cfg, h0 = problems.hot_bubble_2d(n)
    cfg = cfg.replace(mhd=True, riemann=riemann, mach_ct=1e-6)
    h = HostGrid(cfg)
    for name, v in h0.__dict__.items():
        if isinstance(v, np.ndarray) and getattr(h, name) is not None:
            getattr(h, name)[...] = v
        elif isinstance(v, list) and name != "b_x":
            for d, a in enumerate(v):
                if a is not None:
                    getattr(h, name)[d][...] = a
    xn, yn, _ = h.node_coords()
    az = 0.05 * np.sin(2 * np.pi * xn) * np.sin(np.pi * yn) ** 2 + 0.2 * yn
    dx1, dx2, _ = cfg.dx()
    h.b_x[0][1:n + 2, 1:n + 1, 0] = (az[:, 1:, 0] - az[:, :-1, 0]) / dx2
    h.b_x[1][1:n + 1, 1:n + 2, 0] = -(az[1:, :, 0] - az[:-1, :, 0]) / dx1
    return cfg, h


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_oracle_wb_mhd_with_walls_matches_numpy_restatement(oracle, riemann):
    """The magnetised hot bubble: well-balanced deviations, the equilibrium added back at the
    faces, the WB momentum fix, the EVOLVE_ETOT potential flux, gravity on rho', mirrored cells
    with v2 and B2 negated, and the reflective EMF ghosts of the x1 faces (E3 negated, sign
    copied) agree with the numpy restatement bit for bit after six steps."""
    cfg, h = _magnetised_bubble(24, riemann)
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(6)
    W, eint, temp, b1, b2, dt = wb_mhd_2d_steps(hn, 6, low_mach=riemann == "lhlld")
    G = cfg.ngc
    I = (slice(G, G + cfg.nx1), slice(G, G + cfg.nx2))
    for v in range(4):
        np.testing.assert_array_equal(h.prim[v, :, :, 0][I], W[v][I])
    np.testing.assert_array_equal(h.interior(h.eint)[:, :, 0], eint)
    np.testing.assert_array_equal(h.interior(h.temp)[:, :, 0], temp)
    np.testing.assert_array_equal(h.bface_interior(0)[:, :, 0], b1)
    np.testing.assert_array_equal(h.bface_interior(1)[:, :, 0], b2)
    assert o.g.dt == dt


@pytest.fixture(scope="module")
def eos_case(oracle):
    from phlegethon_b200 import helm_table
    import numpy_restatement_eos as R
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    k = dict(nT=101, nrho=271, ltlo=3.0, lthi=13.0, ldlo=-12.0, ldhi=15.0)
    helm = oracle.Helm(tab, dpdr, **k)
    rng = np.random.default_rng(1)
    n = 2000
    rho = 10 ** rng.uniform(-2, 9, n)
    T = 10 ** rng.uniform(4, 10, n)
    abar = rng.uniform(1, 56, n)
    zbar = abar * rng.uniform(0.3, 0.6, n)
    return R, tab, dpdr, R.nodes(**k), helm, rng, (rho, T, abar, zbar)


def test_oracle_helmholtz_evaluation_matches_numpy_restatement(eos_case):
    """helm_rhoT_given_full, given1 and given2 of the C oracle equal the numpy restatement bit
    for bit over 2000 random (rho, T, Abar, Zbar) across the table, and so do the table nodes."""
    R, tab, dpdr, nd, helm, _, (rho, T, abar, zbar) = eos_case
    assert np.array_equal(nd[0], helm.T) and np.array_equal(nd[1], helm.rho)
    full = R.given_full(tab, dpdr, nd, rho, T, abar, zbar)
    o = np.array([helm.given_full(*a) for a in zip(rho, T, abar, zbar)])
    for i in range(4):
        np.testing.assert_array_equal(full[i], o[:, i])
    for deriv in (True, False):
        e2 = R.given2(tab, nd, rho, T, abar, zbar, deriv)
        o2 = np.array([helm.given2(*a, deriv=deriv) for a in zip(rho, T, abar, zbar)])
        p1 = R.given1(tab, nd, rho, T, abar, zbar, deriv)
        o1 = np.array([helm.given1(*a, deriv=deriv) for a in zip(rho, T, abar, zbar)])
        for i in range(2):
            np.testing.assert_array_equal(e2[i], o2[:, i])
            np.testing.assert_array_equal(p1[i], o1[:, i])


def test_oracle_newton_inversions_match_numpy_restatement(eos_case):
    """helm_rhoe_given and helm_rhoP_given from guesses 30% off: the same temperature, pressure
    or energy, sound speed and number of iterations for every sample."""
    R, tab, dpdr, nd, helm, rng, (rho, T, abar, zbar) = eos_case
    tl, th = 10.0 ** 3.0, 10.0 ** 13.0   # Tl_eos, Th_eos = 10**helm_ltlo, 10**helm_lthi
    T0 = T * rng.uniform(0.7, 1.3, T.size)
    E0 = R.given2(tab, nd, rho, T, abar, zbar)[0]
    got = R.rhoe_given(tab, dpdr, nd, rho, E0, abar, zbar, T0, tl, th)
    o = np.array([helm.rhoe_given(*a) for a in zip(rho, E0, abar, zbar, T0)])
    for i in range(4):
        np.testing.assert_array_equal(got[i], o[:, i])
    P0 = R.given1(tab, nd, rho, T, abar, zbar)[0]
    got = R.rhoP_given(tab, dpdr, nd, rho, P0, abar, zbar, T0, tl, th)
    o = np.array([helm.rhoP_given(*a) for a in zip(rho, P0, abar, zbar, T0)])
    for i in range(4):
        np.testing.assert_array_equal(got[i], o[:, i])


@pytest.mark.parametrize("fasteos", [True, False])
@pytest.mark.parametrize("riemann", ["lhlld", "hlld", "lhllc", "hllc"])
def test_oracle_stratified_helmholtz_matches_numpy_restatement(oracle, riemann, fasteos):
    """The benchmark's workloads in small: the stratified Helmholtz box (WB on rho, p and
    gamma_e, FASTEOS face gammas, EVOLVE_ETOT, gravity, Ye and 1/Abar, reflective x2 walls),
    magnetised (LHLLD / HLLD with constrained transport, a divergence-free perturbation of B_2
    and B_3 added to the uniform B_1 so that every EMF component and wall ghost matters) or not
    (LHLLC / HLLC).  The step-0 thermodynamics, three steps with the in-step Newton, the gammas,
    temperatures, face fields and dt equal the numpy restatement bit for bit; without
    USE_FASTEOS every Riemann side's helm_rhoP_given from the face temperature guess is part of
    it."""
    from phlegethon_b200 import helm_table
    import numpy_restatement_eos as RE
    from util import smooth_periodic
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    mhd = riemann in ("lhlld", "hlld")
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=mhd, mach=0.05, table=helm_table.X1_TABLE,
                                    riemann=riemann, fasteos=fasteos)
    if mhd:
        rng = np.random.default_rng(7)
        b0 = float(h.b_x[0][1, 1, 1])
        h.b_x[1][...] += 0.3 * b0 * smooth_periodic(h.b_x[1].shape, (8, None, 6), rng, stagger=1)
        h.b_x[2][...] += 0.3 * b0 * smooth_periodic(h.b_x[2].shape, (8, 12, None), rng, stagger=2)
    nd = RE.nodes(cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)
    hn = h.copy()
    o = oracle.OracleGrid(h, oracle.Helm.for_config(cfg, tab, dpdr), nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(3)
    W, eint, temp, (ge, gc), b, dt = stratified_steps(hn, tab, dpdr, nd, 3)
    for v in range(cfg.nvars):
        np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
    np.testing.assert_array_equal(h.interior(h.eint), eint)
    np.testing.assert_array_equal(h.interior(h.temp), temp)
    if fasteos:
        np.testing.assert_array_equal(h.interior(h.gammaf[0]), hn.interior(ge))
        np.testing.assert_array_equal(h.interior(h.gammaf[1]), hn.interior(gc))
    for d in range(3 if mhd else 0):
        np.testing.assert_array_equal(h.bface_interior(d), b[d])
    assert o.g.dt == dt


def test_oracle_supersonic_all_mach_matches_numpy_restatement(oracle):
    """The stratified hydro box streaming along x1 at twice its sound speed with
    FLUX_IS_ALL_MACH (LHLLC takes the upwind state's flux where the whole fan moves one way):
    bit for bit with the restatement, and different from the run without the switch."""
    from phlegethon_b200 import helm_table
    import numpy_restatement_eos as RE
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    out = []
    for all_mach in (True, False):
        cfg, h = problems.stratified_3d(8, ny=12, nz=6, mach=0.05, table=helm_table.X1_TABLE, riemann="lhllc")
        h.cfg = cfg = cfg.replace(all_mach=all_mach)
        v1 = h.interior(h.prim[1])
        v1 += 2.0 * np.sqrt(5.0 / 3.0 * h.interior(h.prim[4]) / h.interior(h.prim[0]))
        nd = RE.nodes(cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)
        hn = h.copy()
        o = oracle.OracleGrid(h, oracle.Helm.for_config(cfg, tab, dpdr), nthreads=2)
        o.init_thermo()
        o.compute_hyperbolic_dt()
        o.time_loop(3)
        W, eint, temp, _, _, dt = stratified_steps(hn, tab, dpdr, nd, 3)
        for v in range(cfg.nvars):
            np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
        np.testing.assert_array_equal(h.interior(h.temp), temp)
        assert o.g.dt == dt
        out.append(h.interior(h.prim).copy())
    assert not np.array_equal(out[0], out[1])


@pytest.mark.parametrize("rec", ["lim2nd", "pph", "lim5th"])
@pytest.mark.parametrize("riemann", ["lhlld", "hlld", "lhllc", "hllc"])
def test_oracle_shock_flattening_in_the_stratified_box_matches_numpy_restatement(oracle, riemann, rec):
    """USE_SHOCK_FLATTENING in the stratified Helmholtz box at eps_sf 0.6, where the
    background's vertical pressure jumps (0.42 ... 1.28 of p) flag part of the box: the
    detector on the full pressure with the ghosts' equilibria, the PLM fallback of a flagged
    cell's edges under PPH and LIM5TH, the HLL flux of the flagged faces (hydro and MHD) and
    the x1 sweep's gamma_e branch, which leaves the equilibrium off a flagged cell's side of the
    face and adds it to the other, agree with the restatement bit for bit; the flattening
    changes the result."""
    from phlegethon_b200 import helm_table
    import numpy_restatement_eos as RE
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=riemann.endswith("d"), mach=0.05,
                                    table=helm_table.X1_TABLE, riemann=riemann, rec=rec, shock_flattening=True,
                                    eps_sf=0.6)
    nd = RE.nodes(cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)
    helm = oracle.Helm.for_config(cfg, tab, dpdr)
    hn, h0 = h.copy(), h.copy()
    h0.cfg = cfg.replace(shock_flattening=False)
    for g in (h, h0):
        o = oracle.OracleGrid(g, helm, nthreads=2)
        o.init_thermo()
        o.compute_hyperbolic_dt()
        o.time_loop(3)
        if g is h:
            dt_oracle = o.g.dt
    W, eint, temp, _, b, dt = stratified_steps(hn, tab, dpdr, nd, 3)
    for v in range(cfg.nvars):
        np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
    np.testing.assert_array_equal(h.interior(h.temp), temp)
    for d in range(3 if cfg.mhd else 0):
        np.testing.assert_array_equal(h.bface_interior(d), b[d])
    assert dt_oracle == dt
    assert not np.array_equal(h.interior(h.prim), h0.interior(h0.prim))


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_oracle_constant_acceleration_matches_numpy_restatement(oracle, riemann):
    """USE_CONSTANT_ACCELERATION (acc = (0.3, -0.2, 0.15)) on the smooth 3D MHD box: the
    momentum source rho acc and its work, both from the stage's input state, bit for bit."""
    h = smooth_box(3, riemann, "lim2nd", mhd=True)
    h.cfg = h.cfg.replace(constant_acceleration=True, acc=(0.3, -0.2, 0.15))
    hn = h.copy()
    o = oracle.OracleGrid(h, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(3)
    W, eint, temp, b, dt = mhd_3d_steps(hn, 3, low_mach=riemann == "lhlld")
    for v in range(h.cfg.nvars):
        np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
    np.testing.assert_array_equal(h.interior(h.eint), eint)
    for d in range(3):
        np.testing.assert_array_equal(h.bface_interior(d), b[d])
    assert o.g.dt == dt


@pytest.mark.parametrize("rec", ["pph", "lim5th"])
@pytest.mark.parametrize("riemann", ["lhlld", "lhllc"])
def test_oracle_stratified_higher_order_matches_numpy_restatement(oracle, riemann, rec):
    """The stratified Helmholtz box with PPH_REC (primitives, cell B and gammas unlimited, the
    scalars limited) or LIM5TH_REC (all limited): bit for bit with the restatement."""
    from phlegethon_b200 import helm_table
    import numpy_restatement_eos as RE
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=riemann.endswith("d"), mach=0.05,
                                    table=helm_table.X1_TABLE, riemann=riemann, rec=rec)
    nd = RE.nodes(cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)
    hn = h.copy()
    o = oracle.OracleGrid(h, oracle.Helm.for_config(cfg, tab, dpdr), nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(3)
    W, eint, temp, (ge, gc), b, dt = stratified_steps(hn, tab, dpdr, nd, 3)
    for v in range(cfg.nvars):
        np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
    np.testing.assert_array_equal(h.interior(h.temp), temp)
    np.testing.assert_array_equal(h.interior(h.gammaf[0]), hn.interior(ge))
    for d in range(3 if cfg.mhd else 0):
        np.testing.assert_array_equal(h.bface_interior(d), b[d])
    assert o.g.dt == dt


def test_oracle_lhlld_all_mach_matches_numpy_restatement(oracle):
    """FLUX_IS_ALL_MACH with LHLLD on the smooth 3D MHD box streaming at Mach ~2 along x1: the
    outer states' fluxes where the whole fan moves one way, bit for bit with the restatement,
    and different from the run without the switch."""
    out = []
    for all_mach in (True, False):
        h = smooth_box(3, "lhlld", "lim2nd", mhd=True)
        h.cfg = h.cfg.replace(all_mach=all_mach)
        h.prim[1] += 2.5
        hn = h.copy()
        o = oracle.OracleGrid(h, nthreads=2)
        o.init_thermo()
        o.compute_hyperbolic_dt()
        o.time_loop(3)
        W, eint, temp, b, dt = mhd_3d_steps(hn, 3, low_mach=True)
        for v in range(h.cfg.nvars):
            np.testing.assert_array_equal(h.interior(h.prim[v]), hn.interior(W[v]))
        for d in range(3):
            np.testing.assert_array_equal(h.bface_interior(d), b[d])
        assert o.g.dt == dt
        out.append(h.interior(h.prim).copy())
    assert not np.array_equal(out[0], out[1])
