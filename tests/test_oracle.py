"""CPU tests of the oracle (the C restatement used as the parity checker).

The reference's own tests are compile-only (no golden vectors), so the oracle is pinned by
known answers of the scheme and by an independent numpy restatement of the same routines:
  * a uniform state stays uniform bit for bit,
  * an exact hydrostatic equilibrium stays at rest (well-balanced scheme), magnetised too,
  * the Riemann solvers are mirror symmetric (L<->R with v -> -v flips the flux),
  * constrained transport keeps div B at round-off,
  * the Helmholtz Newton inversions round-trip T -> e(rho,T) -> T and P(rho,T) -> T,
  * permuting or reflecting the axes of a state permutes or reflects the result of a step
    (every solver and reconstruction, and the gravitating Helmholtz box),
  * the checker gives the same bits on any number of threads.
The independent numpy restatement of the same routines is compared in test_restatement.py.
"""
import ctypes as C
import math

import numpy as np
import pytest

from phlegethon_b200 import helm_table, problems
from phlegethon_b200.grid import Config, HostGrid
from util import div_b_max, mirror_axis, permute_axes, smooth_box


def _run(oracle, h, helm=None, steps=3):
    o = oracle.OracleGrid(h, helm, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(steps)
    return o


def test_uniform_state_stays_uniform(oracle):
    cfg = Config(sdims=2, nx1=16, nx2=12, riemann="hllc", bc=[["periodic", "periodic"]] * 3)
    h = HostGrid(cfg)
    h.prim[0] = 1.3
    h.prim[1] = 0.2
    h.prim[2] = -0.1
    h.prim[3] = 0.7
    ref = h.interior(h.prim).copy()
    _run(oracle, h, steps=5)
    out = h.interior(h.prim)
    # translation invariance: every cell identical, density unchanged
    assert np.all(out == out[:, :1, :1, :1])
    assert np.all(out[0] == ref[0])


def test_hydrostatic_equilibrium_at_rest(oracle):
    cfg, h = problems.hot_bubble_2d(32)
    x, y, _ = h.coords()
    h.prim[0] = np.exp(-y / 0.5)
    p0 = h.interior(h.prim)[3].copy()
    _run(oracle, h, steps=10)
    v = h.interior(h.prim)[1:3]
    assert float(np.abs(v).max()) < 1e-14
    assert float(np.abs(h.interior(h.prim)[3] - p0).max() / p0.max()) < 1e-14


@pytest.mark.parametrize("riemann", ["lhlld", "hlld"])
def test_magnetised_hydrostatic_box_stays_at_rest(oracle, riemann):
    """The stratified Helmholtz box at rest (Mach 0) threaded by the uniform horizontal B_1 of
    plasma beta 1e4: the well-balanced scheme keeps it in equilibrium with B, ten steps leave
    every velocity below 1e-13 of the sound speed, the pressure within 1e-13 and B_1 uniform to
    1e-13 of itself, and B_2, B_3 exactly zero."""
    tab = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=True, mach=0.0, table=helm_table.X1_TABLE,
                                    riemann=riemann)
    p0 = h.interior(h.prim)[4].copy()
    cs = float(np.sqrt(p0 / h.interior(h.prim)[0]).min())
    b1 = float(h.bface_interior(0)[0, 0, 0])
    _run(oracle, h, oracle.Helm.for_config(cfg, *tab), steps=10)
    s = h.interior(h.prim)
    assert float(np.abs(s[1:4]).max()) < 1e-13 * cs
    assert float(np.abs(s[4] / p0 - 1.0).max()) < 1e-13
    assert float(np.abs(h.bface_interior(0) / b1 - 1.0).max()) < 1e-13
    assert not h.bface_interior(1).any() and not h.bface_interior(2).any()


@pytest.mark.parametrize("flat", [0, 1])
@pytest.mark.parametrize("riemann", ["lhllc", "hllc"])
def test_hydro_riemann_mirror_symmetry(oracle, riemann, flat):
    import ctypes as C
    cfg = Config(sdims=3, nx1=8, nx2=8, nx3=8, nas=2, riemann=riemann, mach_cutoff=1e-4,
                 bc=[["periodic", "periodic"]] * 3)
    h = HostGrid(cfg)
    og = oracle.OracleGrid(h)
    rng = np.random.default_rng(3)
    for _ in range(200):
        qL = np.array([rng.uniform(0.5, 2), rng.normal(), rng.normal(), rng.normal(), rng.uniform(0.5, 2),
                       rng.uniform(0, 1), rng.uniform(0, 1)])
        qR = np.array([rng.uniform(0.5, 2), rng.normal(), rng.normal(), rng.normal(), rng.uniform(0.5, 2),
                       rng.uniform(0, 1), rng.uniform(0, 1)])
        f = np.zeros(7)
        fm = np.zeros(7)
        P = C.POINTER(C.c_double)
        oracle.load().phlo_riemann_hydro(C.byref(og.g), qL.ctypes.data_as(P), qR.ctypes.data_as(P), None, None,
                                         f.ctypes.data_as(P), flat)
        mL = qR.copy()
        mR = qL.copy()
        mL[1] = -mL[1]
        mR[1] = -mR[1]
        oracle.load().phlo_riemann_hydro(C.byref(og.g), mL.ctypes.data_as(P), mR.ctypes.data_as(P), None, None,
                                         fm.ctypes.data_as(P), flat)
        # mirrored problem: mass, transverse momenta, energy, scalars flip sign; normal momentum not
        sgn = np.array([-1, 1, -1, -1, -1, -1, -1])
        np.testing.assert_allclose(fm, sgn * f, rtol=1e-12, atol=1e-12)


def test_lhllc_low_mach_dissipation_scales_with_phi(oracle):
    """LHLLC on a symmetric converging flow (u* = 0): the normal momentum flux is the star
    pressure p* = p + phi rho c v with phi = chi (2 - chi), chi = max(Mach_cutoff, min(1, M)) —
    the pressure dissipation falls with the Mach number instead of staying rho c v as in HLLC
    (source.F90:16012-16122)."""
    import ctypes as C
    cfg = Config(sdims=3, nx1=8, nx2=8, nx3=8, nas=0, riemann="lhllc", mach_cutoff=1e-4,
                 bc=[["periodic", "periodic"]] * 3)
    og = oracle.OracleGrid(HostGrid(cfg))
    P = C.POINTER(C.c_double)
    rho, p = 1.3, 0.7
    c = math.sqrt(cfg.gamma_ad * p / rho)
    for mach, chi in ((1e-6, 1e-4), (1e-3, 1e-3), (1e-2, 1e-2), (0.3, 0.3), (2.0, 1.0)):
        v = mach * c
        qL = np.array([rho, v, 0.0, 0.0, p])
        qR = np.array([rho, -v, 0.0, 0.0, p])
        f = np.zeros(5)
        oracle.load().phlo_riemann_hydro(C.byref(og.g), qL.ctypes.data_as(P), qR.ctypes.data_as(P), None, None,
                                         f.ctypes.data_as(P), 0)
        assert abs(f[0]) < 1e-15 * rho * c
        phi = chi * (2.0 - chi)
        # p* - p is formed from p* (rounded at ~1e-16 p): allow that cancellation
        assert abs((f[1] - p) - phi * rho * c * v) <= 1e-9 * phi * rho * c * v + 8 * np.finfo(float).eps * p


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_lhlld_low_mach_dissipation_scales_with_phi(oracle, riemann):
    """HLLD / LHLLD on a symmetric converging flow without B (u* = 0): the normal momentum flux
    is the star total pressure p + phi rho (c + 2v) v, with phi = 1 for HLLD and, for LHLLD,
    phi = chi (2 - chi) below a fast Mach number of 0.6 and 1 above it
    (source.F90:14364-14384, 14497-14498)."""
    import ctypes as C
    cfg = Config(sdims=3, nx1=8, nx2=8, nx3=8, mhd=True, riemann=riemann, mach_cutoff=1e-4,
                 bc=[["periodic", "periodic"]] * 3)
    og = oracle.OracleGrid(HostGrid(cfg))
    P = C.POINTER(C.c_double)
    rho, p = 1.3, 0.7
    c = math.sqrt(cfg.gamma_ad * p / rho)
    for mach in (1e-3, 1e-2, 0.3, 0.8):
        v = mach * c
        qL, qR = np.array([rho, v, 0.0, 0.0, p]), np.array([rho, -v, 0.0, 0.0, p])
        bL, bR = np.zeros(3), np.zeros(3)
        f, fb = np.zeros(5), np.zeros(3)
        oracle.load().phlo_riemann_mhd(C.byref(og.g), qL.ctypes.data_as(P), qR.ctypes.data_as(P),
                                       bL.ctypes.data_as(P), bR.ctypes.data_as(P), None, None,
                                       f.ctypes.data_as(P), fb.ctypes.data_as(P), 0)
        phi = mach * (2.0 - mach) if riemann == "lhlld" and mach < 0.6 else 1.0
        d = rho * (c + 2.0 * v) * v
        assert abs((f[1] - p) - phi * d) <= 1e-9 * phi * d + 8 * np.finfo(float).eps * p


@pytest.mark.parametrize("flat", [0, 1])
@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_mhd_riemann_mirror_symmetry(oracle, riemann, flat):
    import ctypes as C
    cfg = Config(sdims=3, nx1=8, nx2=8, nx3=8, mhd=True, riemann=riemann, mach_cutoff=1e-4,
                 bc=[["periodic", "periodic"]] * 3)
    h = HostGrid(cfg)
    og = oracle.OracleGrid(h)
    rng = np.random.default_rng(4)
    P = C.POINTER(C.c_double)
    for _ in range(200):
        qL = np.array([rng.uniform(0.5, 2), rng.normal(), rng.normal(), rng.normal(), rng.uniform(0.5, 2)])
        qR = np.array([rng.uniform(0.5, 2), rng.normal(), rng.normal(), rng.normal(), rng.uniform(0.5, 2)])
        bn = rng.normal()
        bL = np.array([bn, rng.normal(), rng.normal()])
        bR = np.array([bn, rng.normal(), rng.normal()])
        f, fb, fm, fbm = np.zeros(5), np.zeros(3), np.zeros(5), np.zeros(3)
        oracle.load().phlo_riemann_mhd(C.byref(og.g), qL.ctypes.data_as(P), qR.ctypes.data_as(P),
                                       bL.ctypes.data_as(P), bR.ctypes.data_as(P), None, None,
                                       f.ctypes.data_as(P), fb.ctypes.data_as(P), flat)
        mL, mR, bmL, bmR = qR.copy(), qL.copy(), bR.copy(), bL.copy()
        mL[1] = -mL[1]
        mR[1] = -mR[1]
        bmL[0] = -bmL[0]
        bmR[0] = -bmR[0]
        oracle.load().phlo_riemann_mhd(C.byref(og.g), mL.ctypes.data_as(P), mR.ctypes.data_as(P),
                                       bmL.ctypes.data_as(P), bmR.ctypes.data_as(P), None, None,
                                       fm.ctypes.data_as(P), fbm.ctypes.data_as(P), flat)
        np.testing.assert_allclose(fm, np.array([-1, 1, -1, -1, -1]) * f, rtol=1e-9, atol=1e-10)
        # induction flux v_n B_t - B_n v_t changes sign with v_n and B_n
        np.testing.assert_allclose(fbm[1:], -fb[1:], rtol=1e-9, atol=1e-10)


def test_orszag_tang_div_b(oracle):
    cfg, h = problems.orszag_tang_2d(48)
    _run(oracle, h, steps=20)
    assert div_b_max(h) <= 1e-13


def test_stratified_mhd_div_b_reflective(oracle):
    tab = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=True, table=helm_table.X1_TABLE)
    helm = oracle.Helm.for_config(cfg, *tab)
    _run(oracle, h, helm, steps=3)
    assert div_b_max(h) <= 1e-13


@pytest.mark.parametrize("sdims", [2, 3])
@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_magnetised_uniform_state_between_walls(oracle, riemann, sdims):
    """A uniform magnetised gas streaming along x1 between reflective x2 walls, with B parallel
    to the walls, is an exact steady state: the mirrored ghost cells equal the interior (v_x1
    and B are tangential), every face sees L = R, and the CT corner EMFs cancel.  Twenty RK3
    steps leave the density, the velocity and every face B unchanged to the bit; the pressure,
    recovered from E - rho v^2 / 2 - B^2 / 2, moves by rounding only."""
    cfg = Config(sdims=sdims, nx1=12, nx2=16, nx3=8 if sdims == 3 else 1, mhd=True,
                 riemann=riemann, gamma_ad=5.0 / 3.0, mu=1.0,
                 bc=[["periodic", "periodic"], ["reflective", "reflective"],
                     ["periodic", "periodic"]])
    h = HostGrid(cfg)
    h.prim[0] = 1.3
    h.prim[1] = 0.3
    h.prim[sdims + 1] = 0.7  # pressure
    h.temp[...] = 1.0
    h.b_x[0][...] = 0.6
    if sdims == 3:
        h.b_x[2][...] = -0.4
    w0 = h.interior(h.prim).copy()
    b0 = [h.bface_interior(d).copy() for d in range(sdims)]
    _run(oracle, h, steps=20)
    w = h.interior(h.prim)
    assert np.array_equal(w[:sdims + 1], w0[:sdims + 1])
    assert float(np.abs(w[sdims + 1] - 0.7).max()) <= 4 * np.finfo(float).eps * 0.7
    for d in range(sdims):
        assert np.array_equal(h.bface_interior(d), b0[d])



# ------------------------------------------------------------------------------ axis permutations
@pytest.mark.parametrize("rec", ["lim2nd", "pph", "lim5th"])
@pytest.mark.parametrize("riemann", ["hllc", "lhllc", "hlld", "lhlld"])
@pytest.mark.parametrize("sdims, perm", [(2, (1, 0, 2)), (3, (1, 2, 0))])
def test_axis_permutation_commutes_with_the_step(oracle, sdims, perm, riemann, rec):
    """The equations have no preferred axis: stepping a state whose axes were permuted (the
    2D transpose, the 3D cyclic x1 -> x3 -> x2 -> x1, on a box of unequal extents and cell
    counts) gives the permuted result of stepping the original.  The sweeps along each axis run
    the same code on re-indexed components, so this pins the component permutations of every
    direction: a transposed index or a swapped normal component shows up at O(1).  The two runs
    differ only in the order in which the directions' flux differences are summed (2D hydro
    happens to round identically)."""
    h = smooth_box(sdims, riemann, rec, mhd=riemann in ("hlld", "lhlld"))
    hp = permute_axes(h, perm)
    o1 = _run(oracle, h, steps=6)
    o2 = _run(oracle, hp, steps=6)
    assert abs(o2.g.time - o1.g.time) <= 1e-15 * o1.g.time
    ref = permute_axes(h, perm)
    assert float(np.abs(hp.interior(hp.prim) - ref.interior(ref.prim)).max()) <= 4e-15
    if h.cfg.mhd:
        for d in range(sdims):
            assert float(np.abs(hp.bface_interior(d) - ref.bface_interior(d)).max()) <= 2e-15


@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("perm", [(1, 2, 0), (2, 0, 1)])
def test_axis_permutation_of_the_stratified_helmholtz_box(oracle, perm, mhd):
    """The well-balanced, gravitating Helmholtz box (EVOLVE_ETOT, LHLLC / LHLLD with CT) with
    its vertical axis moved from x2 to x1 or x3: gravity, the reflective walls, the equilibrium
    face arrays and the potentials follow the axis, and four steps of the permuted box equal the
    permuted steps of the original to rounding (the Newton solves stop at the same residual)."""
    tab = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=mhd, mach=0.05, table=helm_table.X1_TABLE)
    helm = oracle.Helm.for_config(cfg, *tab)
    hp = permute_axes(h, perm)
    o1 = _run(oracle, h, helm, steps=4)
    o2 = _run(oracle, hp, helm, steps=4)
    assert abs(o2.g.time - o1.g.time) <= 1e-13 * o1.g.time
    ref = permute_axes(h, perm)
    a, b = hp.interior(hp.prim), ref.interior(ref.prim)
    for iv in range(a.shape[0]):
        assert float(np.abs(a[iv] - b[iv]).max()) <= 1e-12 * float(np.abs(b[iv]).max())
    t, tr = hp.interior(hp.temp), ref.interior(ref.temp)
    assert float(np.abs(t - tr).max()) <= 1e-12 * float(tr.max())
    if mhd:
        bscale = max(float(np.abs(ref.bface_interior(d)).max()) for d in range(3))
        for d in range(3):
            assert float(np.abs(hp.bface_interior(d) - ref.bface_interior(d)).max()) <= 1e-12 * bscale


@pytest.mark.parametrize("rec", ["lim2nd", "pph", "lim5th"])
@pytest.mark.parametrize("riemann", ["hllc", "lhllc", "hlld", "lhlld"])
@pytest.mark.parametrize("sdims, axis", [(2, 0), (2, 1), (3, 0), (3, 1), (3, 2)])
def test_mirror_commutes_with_the_step(oracle, sdims, axis, riemann, rec):
    """Reflecting a state along one axis (v_a and B_a change sign, every array reversed along
    a) reflects the result of a step: the reconstructions treat the left and right neighbours
    alike and the solvers the left and right states (their single-interface mirror symmetry is
    tested above), the CT corner averages are symmetric, and the update does not favour one
    end of a sweep.  Equal to 4e-15 in the state, 2e-15 in the face B."""
    h = smooth_box(sdims, riemann, rec, mhd=riemann in ("hlld", "lhlld"))
    hm = mirror_axis(h, axis)
    o1 = _run(oracle, h, steps=6)
    o2 = _run(oracle, hm, steps=6)
    assert abs(o2.g.time - o1.g.time) <= 1e-15 * o1.g.time
    ref = mirror_axis(h, axis)
    assert float(np.abs(hm.interior(hm.prim) - ref.interior(ref.prim)).max()) <= 4e-15
    if h.cfg.mhd:
        for d in range(sdims):
            assert float(np.abs(hm.bface_interior(d) - ref.bface_interior(d)).max()) <= 2e-15



def _offcentre_blast(riemann, rec):
    """A drifting blast off the centre of a 24 x 20 periodic box (p 10 inside r^2 < 0.02, 0.1
    outside; B = (0.5, 0.3) for the MHD solvers), run with USE_SHOCK_FLATTENING at eps_sf 0.25:
    the flattener flags the front, and its detector, PLM fallback and HLL faces enter the step."""
    mhd = riemann in ("hlld", "lhlld")
    cfg, _ = problems.blast_2d(24, riemann=riemann, rec=rec, shock_flattening=True, eps_sf=0.25)
    h = HostGrid(cfg.replace(nx2=20, x2u=20.0 / 24.0, mhd=mhd))
    x, y, _ = h.coords()
    inside = (x - 0.42) ** 2 + (y - 0.47) ** 2 < 0.02
    h.prim[0] = 1.0
    h.prim[1] = 0.1
    h.prim[2] = -0.05
    h.prim[3] = np.where(inside, 10.0, 0.1)
    h.prim[4] = np.where(inside, 1.0, 0.0)
    if mhd:
        h.b_x[0][...] = 0.5
        h.b_x[1][...] = 0.3
    return h


def _supersonic_box(sdims, riemann, rec):
    """The smooth periodic box streaming at Mach ~2 along x1 with FLUX_IS_ALL_MACH: the x1
    faces take the upwind flux where the whole fan moves one way."""
    h = smooth_box(sdims, riemann, rec, mhd=riemann == "lhlld")
    h.cfg = h.cfg.replace(all_mach=True)
    h.prim[1] += 2.5
    return h


@pytest.mark.parametrize("rec", ["lim2nd", "pph", "lim5th"])
@pytest.mark.parametrize("case", ["blast-hllc", "blast-lhllc", "blast-hlld", "blast-lhlld",
                                  "allmach2d-lhllc", "allmach2d-lhlld", "allmach3d-lhllc",
                                  "allmach3d-lhlld"])
def test_symmetries_with_flattening_and_all_mach(oracle, case, rec):
    """The permutation and reflection symmetries with the two options that change the face
    solve: shock flattening on a blast front, and FLUX_IS_ALL_MACH on a supersonic stream
    (both options change these states at O(1): with eps_sf out of reach, or without the
    all-Mach switch, the results differ).  Equal to 8e-15 (pressures up to 10, velocities up
    to 3)."""
    kind, riemann = case.split("-")
    if kind == "blast":
        h, sdims = _offcentre_blast(riemann, rec), 2
    else:
        sdims = int(kind[-2])
        h = _supersonic_box(sdims, riemann, rec)
    stepped = h.copy()
    _run(oracle, stepped, steps=6)
    without = h.copy()
    without.cfg = h.cfg.replace(eps_sf=1e300) if kind == "blast" else h.cfg.replace(all_mach=False)
    _run(oracle, without, steps=6)
    assert not np.allclose(without.interior(without.prim), stepped.interior(stepped.prim), atol=1e-6)
    transforms = [lambda g, a=a: mirror_axis(g, a) for a in range(sdims)]
    transforms.append(lambda g: permute_axes(g, (1, 0, 2) if sdims == 2 else (1, 2, 0)))
    for tr in transforms:
        moved = tr(h)
        _run(oracle, moved, steps=6)
        ref = tr(stepped)
        assert float(np.abs(moved.interior(moved.prim) - ref.interior(ref.prim)).max()) <= 8e-15
        if h.cfg.mhd:
            for d in range(sdims):
                assert float(np.abs(moved.bface_interior(d) - ref.bface_interior(d)).max()) <= 8e-15

@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_mirror_of_the_stratified_helmholtz_box(oracle, axis, mhd):
    """The gravitating Helmholtz box reflected along a horizontal axis, or upside down (gravity,
    the potentials and the equilibrium arrays reversed with it): four steps equal the reflected
    steps of the original to 1e-12 of each field's scale."""
    tab = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=mhd, mach=0.05, table=helm_table.X1_TABLE)
    helm = oracle.Helm.for_config(cfg, *tab)
    hm = mirror_axis(h, axis)
    o1 = _run(oracle, h, helm, steps=4)
    o2 = _run(oracle, hm, helm, steps=4)
    assert abs(o2.g.time - o1.g.time) <= 1e-13 * o1.g.time
    ref = mirror_axis(h, axis)
    a, b = hm.interior(hm.prim), ref.interior(ref.prim)
    for iv in range(a.shape[0]):
        assert float(np.abs(a[iv] - b[iv]).max()) <= 1e-12 * float(np.abs(b[iv]).max())
    if mhd:
        bscale = max(float(np.abs(ref.bface_interior(d)).max()) for d in range(3))
        for d in range(3):
            assert float(np.abs(hm.bface_interior(d) - ref.bface_interior(d)).max()) <= 1e-12 * bscale

def test_helmholtz_round_trips(oracle, table):
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    rho, T, abar, zbar = problems.eos_samples(400, seed=5)
    worst_e = worst_p = 0.0
    for i in range(len(rho)):
        E, _ = helm.given2(rho[i], T[i], abar[i], zbar[i])
        P, _ = helm.given1(rho[i], T[i], abar[i], zbar[i])
        Te, _, _, it = helm.rhoe_given(rho[i], E, abar[i], zbar[i], T[i] * 1.3)
        Tp, _, _, itp = helm.rhoP_given(rho[i], P, abar[i], zbar[i], T[i] * 0.8)
        # judge by the residual the Newton loop is built on (helm_tol = 1e-11)
        E2, _ = helm.given2(rho[i], Te, abar[i], zbar[i])
        P2, _ = helm.given1(rho[i], Tp, abar[i], zbar[i])
        worst_e = max(worst_e, abs(E2 - E) / abs(E))
        worst_p = max(worst_p, abs(P2 - P) / abs(P))
    assert worst_e < 1e-10
    assert worst_p < 1e-10


def test_helmholtz_interpolates_the_model(oracle, table):
    """Biquintic interpolation of the generated table reproduces the closed-form model."""
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    rho, T, abar, zbar = problems.eos_samples(300, seed=9)
    for i in range(len(rho)):
        P, E, s, cv = helm.given_full(rho[i], T[i], abar[i], zbar[i])
        Pm = problems.analytic_pressure(rho[i], T[i], abar[i], zbar[i])
        Em = problems.analytic_energy(rho[i], T[i], abar[i], zbar[i])
        assert abs(P - Pm) / Pm < 1e-6
        assert abs(E - Em) / Em < 1e-6
        assert s > 0 and cv > 0


def test_table_text_format_round_trip(tmp_path):
    tab, dpdr = helm_table.generate(nrho=20, nT=11, ldlo=1.0, ldhi=8.0, ltlo=5.0, lthi=9.0)
    p = tmp_path / "helm.dat"
    helm_table.write_text(str(p), tab, dpdr)
    t2, d2 = helm_table.read_text(str(p), 20, 11)
    np.testing.assert_array_equal(t2, tab)
    np.testing.assert_array_equal(d2, dpdr)


def test_table_thermodynamic_consistency():
    """The generated table's derivatives are consistent with finite differences of f."""
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    f = tab[0]
    rho, T, drho, dT = helm_table.nodes(271, 101, -12.0, 15.0, 3.0, 13.0)
    i, j = 150, 50
    h = 1e-6
    fr = (f[i + 1, j] - f[i - 1, j]) / (rho[i + 1] - rho[i - 1])
    assert abs(fr - tab[3, i, j]) / abs(tab[3, i, j]) < 1e-2
    ft = (f[i, j + 1] - f[i, j - 1]) / (T[j + 1] - T[j - 1])
    assert abs(ft - tab[1, i, j]) / abs(tab[1, i, j]) < 1e-2
    # c = dP/d(rho Ye) = 2 d f_d + d^2 f_dd
    c = 2 * rho[i] * tab[3, i, j] + rho[i] ** 2 * tab[4, i, j]
    assert abs(c - dpdr[0, i, j]) / abs(dpdr[0, i, j]) < 1e-12
    del h


def test_bracket_guess_batch_round_trip(oracle, table):
    """Cold bracket guess + helm_rhoe_given Newton recovers T over the EoS benchmark ranges."""
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    rho, T, abar, zbar = problems.eos_samples(2000, seed=31)
    e = np.array([helm.given2(rho[i], T[i], abar[i], zbar[i])[0] for i in range(rho.size)])
    Tb, it = helm.invert_batch(rho, e, abar, zbar, guess=2, nthreads=2)
    assert it.max() < 100
    E2 = np.array([helm.given2(rho[i], Tb[i], abar[i], zbar[i])[0] for i in range(rho.size)])
    assert np.max(np.abs(E2 - e) / np.abs(e)) < 1e-11
    # the guess itself lands between two table nodes: at most one node spacing (0.05 dex) off
    Tg = np.zeros(1)
    for i in range(0, rho.size, 97):
        nev = oracle.load().phlo_eos_bracket_guess(C.byref(helm.s), rho[i], e[i], abar[i], zbar[i],
                                                    Tg.ctypes.data_as(C.POINTER(C.c_double)))
        assert 1 <= nev <= 2 + 8
        assert abs(math.log10(Tg[0] / Tb[i])) < 0.06


@pytest.mark.parametrize("rec", ["pph", "lim5th"])
def test_higher_order_uniform_and_div_b(oracle, rec):
    """PPH_REC / LIM5TH_REC: a uniform state stays uniform; constrained transport keeps div B."""
    cfg = Config(sdims=2, nx1=16, nx2=12, riemann="hllc", rec=rec, ngc=3 if rec == "lim5th" else 2,
                 bc=[["periodic", "periodic"]] * 3)
    h = HostGrid(cfg)
    h.prim[0] = 1.3
    h.prim[1] = 0.2
    h.prim[2] = -0.1
    h.prim[3] = 0.7
    _run(oracle, h, steps=4)
    out = h.interior(h.prim)
    assert np.all(out == out[:, :1, :1, :1])
    cfg, h = problems.orszag_tang_2d(32, rec=rec)
    _run(oracle, h, steps=10)
    assert div_b_max(h) <= 1e-13


def test_lim5th_edges_reproduce_smooth_data():
    """The fifth-order edge formula of LIM5TH_REC is exact for quartic data (away from extrema)."""
    x = np.arange(-2, 3, dtype=float)
    f = lambda t: 1.0 + 0.1 * t + 0.01 * t ** 2 + 0.001 * t ** 3 + 0.0001 * t ** 4
    # cell averages of f over [i-1/2, i+1/2]
    from numpy.polynomial import polynomial as Pn
    coef = [1.0, 0.1, 0.01, 0.001, 0.0001]
    integ = Pn.polyint(coef)
    avg = np.array([Pn.polyval(i + 0.5, integ) - Pn.polyval(i - 0.5, integ) for i in x])
    am = (-21 * avg[0] + 189 * avg[1] + 329 * avg[2] - 91 * avg[3] + 14 * avg[4]) / 420.0
    ap = (14 * avg[0] - 91 * avg[1] + 329 * avg[2] + 189 * avg[3] - 21 * avg[4]) / 420.0
    assert abs(am - f(-0.5)) < 1e-12 and abs(ap - f(0.5)) < 1e-12


# ------------------------------------------------------------------------------ USE_SHOCK_FLATTENING
def _interior_state(h):
    return h.interior(h.prim).copy()


@pytest.mark.parametrize("rec", ["pph", "lim5th"])
def test_flattening_threshold_out_of_reach_changes_nothing(oracle, rec):
    """No cell reaches eps_sf = 1e300: the step equals the one without the option, bit for bit."""
    cfg, h = problems.blast_2d(32, rec=rec, shock_flattening=True, eps_sf=1e300)
    cfg0, h0 = problems.blast_2d(32, rec=rec, shock_flattening=False)
    _run(oracle, h, steps=8)
    _run(oracle, h0, steps=8)
    assert np.array_equal(_interior_state(h), _interior_state(h0))


@pytest.mark.parametrize("maker", ["blast", "orszag_tang"])
def test_flattening_everywhere_is_lim2nd(oracle, maker):
    """eps_sf < 0 flags every cell: every reconstruction falls back to LIM2ND PLM, so PPH and
    LIM5TH give exactly the LIM2ND result (hydro and MHD, including transverse B)."""
    out = {}
    for rec in ("lim2nd", "pph", "lim5th"):
        if maker == "blast":
            cfg, h = problems.blast_2d(32, rec=rec, shock_flattening=True, eps_sf=-1.0)
        else:
            cfg, h = problems.orszag_tang_2d(32, rec=rec, shock_flattening=True, eps_sf=-1.0)
        _run(oracle, h, steps=6)
        out[rec] = (_interior_state(h), None if h.b_cc is None else h.interior(h.b_cc).copy())
    for rec in ("pph", "lim5th"):
        assert np.array_equal(out[rec][0], out["lim2nd"][0])
        if out[rec][1] is not None:
            assert np.array_equal(out[rec][1], out["lim2nd"][1])


def test_flattening_removes_pph_overshoots(oracle):
    """Unlimited PPH rings at the blast front (p and rho undershoot their initial minima);
    with the shock flattener the flagged cells fall back to PLM + HLL and stay bounded."""
    res = {}
    for sf in (False, True):
        cfg, h = problems.blast_2d(64, rec="pph", shock_flattening=sf)
        _run(oracle, h, steps=20)
        s = _interior_state(h)
        res[sf] = (s[0].min(), s[3].min())
    assert res[False][0] < 0.3 and res[False][1] < 0.095   # ringing without the flattener
    assert res[True][0] > 0.4 and res[True][1] > 0.0999     # bounded with it


def test_flattening_conserves_mass_and_energy(oracle):
    cfg, h = problems.blast_2d(48, rec="lim5th", shock_flattening=True)
    dv = np.prod(cfg.dx()[:2])

    def totals():
        s = _interior_state(h)
        rho, v1, v2, p = s[0], s[1], s[2], s[3]
        return (rho.sum() * dv, (p / (cfg.gamma_ad - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2)).sum() * dv)

    m0, e0 = totals()
    _run(oracle, h, steps=15)
    m1, e1 = totals()
    assert abs(m1 - m0) <= 1e-13 * m0
    assert abs(e1 - e0) <= 1e-12 * e0


# ------------------------------------------------------------------------------ FLUX_IS_ALL_MACH
def test_all_mach_supersonic_face_takes_the_upwind_flux(oracle):
    """With FLUX_IS_ALL_MACH a face whose whole wave fan moves right (sL > 0) carries the left
    state's physical flux exactly; without it LHLLC keeps its star flux."""
    import ctypes as C
    P = C.POINTER(C.c_double)
    qL = np.array([1.0, 5.0, 0.3, -0.2, 1.0, 0.4])
    qR = np.array([0.8, 4.5, 0.1, 0.1, 0.7, 0.6])
    out = {}
    for am in (False, True):
        cfg = Config(sdims=3, nx1=8, nx2=8, nx3=8, nas=1, riemann="lhllc", all_mach=am, mach_cutoff=1e-4,
                     bc=[["periodic", "periodic"]] * 3)
        og = oracle.OracleGrid(HostGrid(cfg))
        f = np.zeros(6)
        oracle.load().phlo_riemann_hydro(C.byref(og.g), qL.ctypes.data_as(P), qR.ctypes.data_as(P), None, None,
                                         f.ctypes.data_as(P), 0)
        out[am] = f
    rho, v1, v2, v3, p, s = qL
    e = p / (5.0 / 3.0 - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3)
    exact = np.array([rho * v1, rho * v1 * v1 + p, rho * v1 * v2, rho * v1 * v3, (e + p) * v1, rho * s * v1])
    np.testing.assert_allclose(out[True], exact, rtol=1e-15)
    assert not np.allclose(out[False], exact, rtol=1e-6)


def test_all_mach_leaves_subsonic_flow_unchanged(oracle):
    res = []
    for am in (False, True):
        cfg, h = problems.hot_bubble_2d(32)
        h.cfg = cfg.replace(all_mach=am)
        _run(oracle, h, steps=10)
        res.append(h.interior(h.prim).copy())
    assert np.array_equal(res[0], res[1])


# ------------------------------------------------------------------------------ USE_CONSTANT_ACCELERATION
def test_constant_acceleration_uniform_state(oracle):
    """A uniform periodic state under a constant acceleration a: every cell gains momentum
    rho a t and kinetic energy (rho v + rho a t)^2 / (2 rho) - (rho v)^2 / (2 rho), exactly up
    to rounding (RK3 integrates the linear-in-time momentum exactly)."""
    cfg = Config(sdims=2, nx1=16, nx2=12, riemann="hllc", bc=[["periodic", "periodic"]] * 3,
                 constant_acceleration=True, acc=(0.3, -0.2, 0.0))
    h = HostGrid(cfg)
    h.prim[0] = 1.3
    h.prim[1] = 0.2
    h.prim[2] = -0.1
    h.prim[3] = 0.7
    o = _run(oracle, h, steps=5)
    t = o.g.time
    s = h.interior(h.prim)
    np.testing.assert_allclose(s[1], 0.2 + 0.3 * t, rtol=1e-13)
    np.testing.assert_allclose(s[2], -0.1 - 0.2 * t, rtol=1e-13)
    np.testing.assert_allclose(s[3], 0.7, rtol=1e-13)  # the work goes into kinetic energy only
    assert np.all(s == s[:, :1, :1, :1])


def test_face_temperature_guess_beats_a_learned_accuracy_guess(oracle, table):
    """Helmholtz without USE_FASTEOS solves helm_rhoP_given on both sides of every face from the
    guess 0.5 (T_L + T_R) (source.F90:8488-8495, 15777-15781).  On the stratified box that guess
    converges in fewer iterations (about 2.6) than a guess as accurate as the trained network's
    (0.2% in T, 3 iterations), so a learned guess cannot pay on these solves."""
    from phlegethon_b200 import problems
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, fasteos=False)
    helm = oracle.Helm.for_config(cfg, *table)
    o = oracle.OracleGrid(h, helm)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    oracle.face_newton_stats(reset=True)
    o.time_loop(2)
    calls, iters = oracle.face_newton_stats(reset=True)
    assert calls > 0
    face = iters / calls
    w, T = h.interior(h.prim), h.interior(h.temp)
    rho, p, ye, ia = (w[q].ravel() for q in (0, 4, 5, 6))
    abar = 1.0 / ia
    sel = range(0, rho.size, 7)
    learned_like = np.mean([helm.rhoP_given(rho[i], p[i], abar[i], ye[i] * abar[i], T.ravel()[i] * 1.002)[3]
                            for i in sel])
    assert face < learned_like, (face, learned_like)
    assert face < 2.8 and learned_like >= 3.0, (face, learned_like)


def test_helmholtz_evaluation_is_thermodynamically_consistent(oracle, table):
    """P and E of the oracle's helm_rhoT_given_full come from one interpolated free energy (the
    electron part) plus the analytic ions and radiation, so they obey the Maxwell relation
    (dE/drho)_T = (P - T (dP/dT)_rho) / rho^2, and c_v equals (dE/dT)_rho; both checked by central
    differences over the stratified boxes' and the EoS batch's (rho, T) ranges.  The c_v check
    allows for the rounding of E in the difference quotient where the electrons are degenerate
    (T c_v down to 1e-5 of E)."""
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    abar, zbar, h = 13.7, 6.9, 1e-5
    for lr in np.linspace(-1.0, 8.0, 10):
        for lt in np.linspace(5.0, 9.5, 10):
            rho, T = 10.0 ** lr, 10.0 ** lt
            P, E, _, cv = helm.given_full(rho, T, abar, zbar)
            dEdr = (helm.given_full(rho * (1 + h), T, abar, zbar)[1] -
                    helm.given_full(rho * (1 - h), T, abar, zbar)[1]) / (2 * rho * h)
            dPdT = (helm.given_full(rho, T * (1 + h), abar, zbar)[0] -
                    helm.given_full(rho, T * (1 - h), abar, zbar)[0]) / (2 * T * h)
            dEdT = (helm.given_full(rho, T * (1 + h), abar, zbar)[1] -
                    helm.given_full(rho, T * (1 - h), abar, zbar)[1]) / (2 * T * h)
            scale = (abs(P) + abs(T * dPdT)) / rho ** 2
            assert abs(dEdr - (P - T * dPdT) / rho ** 2) <= 1e-7 * scale, (lr, lt)
            assert abs(dEdT - cv) <= 1e-6 * cv + 1e-12 * abs(E) / (2 * T * h), (lr, lt, dEdT, cv)


def test_helmholtz_sound_speed_from_finite_differences(oracle, table):
    """The sound speed of helm_rhoT_given_full, formed from the bicubic dP/d(rho Ye) table, c_v
    and the biquintic dP/dT, equals the same relativistic expression (c^2 gamma_1 / z with
    gamma_1 = chi_T^2 P / (rho T c_v) + chi_rho and z = 1 + (E + c^2) rho / P, the quantities of
    source.F90:24223-24230) evaluated with central differences of P: a wrong derivative term
    shows up at the 1e-2 level, the two dP/drho interpolants agree to ~1e-6."""
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    abar, zbar, h, clight = 13.7, 6.9, 1e-5, 2.99792458e10
    for lr in np.linspace(-1.0, 8.0, 10):
        for lt in np.linspace(5.0, 9.5, 10):
            rho, T = 10.0 ** lr, 10.0 ** lt
            P, E, sound, cv = helm.given_full(rho, T, abar, zbar)
            dPdT = (helm.given_full(rho, T * (1 + h), abar, zbar)[0] -
                    helm.given_full(rho, T * (1 - h), abar, zbar)[0]) / (2 * T * h)
            dPdr = (helm.given_full(rho * (1 + h), T, abar, zbar)[0] -
                    helm.given_full(rho * (1 - h), T, abar, zbar)[0]) / (2 * rho * h)
            chi_t, chi_r = T * dPdT / P, rho * dPdr / P
            gam1 = chi_t * (P / rho) * chi_t / (T * cv) + chi_r
            z = 1.0 + (E + clight * clight) * rho / P
            assert abs(clight * math.sqrt(gam1 / z) - sound) <= 1e-5 * sound, (lr, lt)


# ------------------------------------------------------------------------------ determinism
def test_oracle_is_independent_of_its_thread_count(oracle):
    """The checker's OpenMP loops carry no order-dependent reduction (the dt reduction is a
    maximum): the magnetised stratified Helmholtz box with shock flattening gives the same bits
    on 1, 3 and 8 threads."""
    res = []
    for nt in (1, 3, 8):
        cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=True, mach=0.05, table=helm_table.X1_TABLE,
                                        shock_flattening=True, eps_sf=0.6)
        o = oracle.OracleGrid(h, oracle.Helm.for_config(cfg, *helm_table.generate(nrho=271, nT=101)),
                              nthreads=nt)
        o.init_thermo()
        o.compute_hyperbolic_dt()
        o.time_loop(3)
        res.append((h.interior(h.prim).copy(), [h.bface_interior(d).copy() for d in range(3)], o.g.dt))
    for r in res[1:]:
        assert np.array_equal(r[0], res[0][0]) and r[2] == res[0][2]
        for a, b in zip(r[1], res[0][1]):
            assert np.array_equal(a, b)
