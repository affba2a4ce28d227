"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the same inputs.

The FP64 path is compiled without FMA contraction and follows the reference's operation
order, so the expected agreement is bit-for-bit; the asserted bars are the ones the FP64 path
must meet in any case: relative L1 <= 1e-12 after one step and <= 1e-9 after many steps, and
div B <= 1e-13 (normalised by dx / max|B|) for constrained transport.
"""
import math

import numpy as np
import pytest

from phlegethon_b200 import problems
from phlegethon_b200.grid import Config, HostGrid
from util import div_b_max, field_errors, max_abs_diff

pytestmark = pytest.mark.gpu


def run_pair(cfg, h, nsteps, table=None, oracle=None):
    from phlegethon_b200.abi import Simulation
    hg, ho = h.copy(), h.copy()
    helm = oracle.Helm.for_config(cfg, *table) if cfg.helmholtz else None
    o = oracle.OracleGrid(ho, helm)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    o.time_loop(nsteps)
    with Simulation(cfg, table if cfg.helmholtz else None) as sim:
        sim.upload(hg)
        sim.init_thermo()
        dt0, smax0 = sim.compute_hyperbolic_dt()
        done, t = sim.time_loop(nsteps)
        assert done == nsteps
        sim.download(hg)
        tg, dtg, smaxg = sim.get_time()
        st = sim.status()
    assert abs(tg - o.g.time) <= 1e-14 * max(1.0, abs(o.g.time))
    assert abs(dtg - o.g.dt) <= 1e-12 * abs(o.g.dt)
    return hg, ho, st


def periodic_3d(n=12, mhd=False, riemann=None):
    cfg = Config(sdims=3, nx1=n, nx2=n + 2, nx3=n - 2, ngc=2, nas=0, mhd=mhd,
                 riemann=riemann or ("hlld" if mhd else "hllc"), bc=[["periodic", "periodic"]] * 3,
                 mach_cutoff=1e-4, mach_ct=1e-6)
    h = HostGrid(cfg)
    x, y, z = h.coords()
    tp = 2 * math.pi
    h.prim[0] = 1.0 + 0.3 * np.sin(tp * x) * np.sin(tp * y) * np.cos(tp * z)
    h.prim[1] = 0.5 * np.sin(tp * y + 0.3)
    h.prim[2] = 0.4 * np.cos(tp * z) * np.sin(tp * x)
    h.prim[3] = 0.3 * np.sin(tp * x + tp * y)
    h.prim[4] = 1.0 + 0.2 * np.cos(tp * x) * np.cos(tp * z)
    if mhd:
        xn, yn, zn = np.meshgrid(*(np.arange(m + 1) * d for m, d in zip((cfg.nx1, cfg.nx2, cfg.nx3), cfg.dx())),
                                 indexing="ij")
        Az = 0.1 * np.cos(tp * yn) + 0.05 * np.cos(2 * tp * xn)
        dx = cfg.dx()
        b1 = h.b_x[0]
        b2 = h.b_x[1]
        b3 = h.b_x[2]
        nx, ny, nz = cfg.nx1, cfg.nx2, cfg.nx3
        b1[1:nx + 2, 1:ny + 1, 1:nz + 1] = (Az[:, 1:, :nz] - Az[:, :-1, :nz]) / dx[1] + 0.2
        b2[1:nx + 1, 1:ny + 2, 1:nz + 1] = -(Az[1:, :, :nz] - Az[:-1, :, :nz]) / dx[0]
        b3[1:nx + 1, 1:ny + 1, 1:nz + 2] = 0.15
    return cfg, h


# ------------------------------------------------------------------------------ hot bubble
@pytest.mark.parametrize("riemann", ["lhllc", "hllc"])
def test_hot_bubble_one_step(gpu_lib, oracle, riemann):
    cfg, h = problems.hot_bubble_2d(64, riemann=riemann)
    hg, ho, _ = run_pair(cfg, h, 1, oracle=oracle)
    err = field_errors(hg, ho)
    assert max(err.values()) <= 1e-12, err
    assert max_abs_diff(hg, ho) == 0.0


def test_hot_bubble_many_steps(gpu_lib, oracle):
    cfg, h = problems.hot_bubble_2d(96)
    hg, ho, _ = run_pair(cfg, h, 100, oracle=oracle)
    err = field_errors(hg, ho)
    assert max(err.values()) <= 1e-9, err
    assert max_abs_diff(hg, ho) == 0.0  # same operation order: bit for bit


def test_hydrostatic_balance_kept(gpu_lib):
    """Well-balanced scheme: the exact equilibrium stays at rest to round-off."""
    from phlegethon_b200.abi import Simulation
    cfg, h = problems.hot_bubble_2d(64)
    x, y, _ = h.coords()
    h.prim[0] = np.exp(-y / 0.5)
    with Simulation(cfg) as sim:
        sim.upload(h)
        sim.init_thermo()
        sim.compute_hyperbolic_dt()
        sim.time_loop(20)
        out = h.copy()
        sim.download(out)
    v = out.interior(out.prim)[1:3]
    assert float(np.abs(v).max()) < 1e-14
    p0 = h.interior(h.prim)[3]
    assert float(np.abs(out.interior(out.prim)[3] - p0).max() / p0.max()) < 1e-14


# ------------------------------------------------------------------------------ Orszag-Tang
@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_orszag_tang(gpu_lib, oracle, riemann):
    cfg, h = problems.orszag_tang_2d(64, riemann=riemann)
    hg, ho, _ = run_pair(cfg, h, 30, oracle=oracle)
    err = field_errors(hg, ho)
    assert max(err.values()) <= 1e-9, err
    assert max_abs_diff(hg, ho) == 0.0
    assert div_b_max(hg) <= 1e-13


# ------------------------------------------------------------------------------ 3D ideal
@pytest.mark.parametrize("mhd,riemann", [(False, "hllc"), (False, "lhllc"), (True, "hlld"), (True, "lhlld")])
def test_periodic_3d(gpu_lib, oracle, mhd, riemann):
    cfg, h = periodic_3d(12, mhd=mhd, riemann=riemann)
    hg, ho, _ = run_pair(cfg, h, 5, oracle=oracle)
    err = field_errors(hg, ho)
    assert max(err.values()) <= 1e-12, err
    assert max_abs_diff(hg, ho) == 0.0
    if mhd:
        assert div_b_max(hg) <= 1e-13


# ------------------------------------------------------------------------------ stratified Helmholtz boxes
@pytest.mark.parametrize("mhd", [False, True])
def test_stratified_helmholtz(gpu_lib, oracle, table, mhd):
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd)
    hg, ho, st = run_pair(cfg, h, 3, table=table, oracle=oracle)
    err = field_errors(hg, ho)
    assert max(err.values()) <= 1e-12, err
    assert max_abs_diff(hg, ho) == 0.0
    assert st["newton_nonconverged"] == 0
    assert st["nonfinite"] == 0
    if mhd:
        assert div_b_max(hg) <= 1e-13


# ------------------------------------------------------------------------------ EoS batch
def test_eos_inversion_matches_oracle(gpu_lib, oracle, table):
    import torch
    from phlegethon_b200.abi import Simulation
    cfg, _ = problems.stratified_3d(8)
    n = 4096
    rho, T, abar, zbar = problems.eos_samples(n, seed=7)
    helm = oracle.Helm.for_config(cfg, *table)
    e = np.array([helm.given2(rho[i], T[i], abar[i], zbar[i], False)[0] for i in range(n)])
    T0 = T * np.exp(0.3 * np.sin(np.arange(n)))  # perturbed warm start
    with Simulation(cfg, table) as sim:
        Tg = T0.copy()
        p = np.zeros(n)
        cs = np.zeros(n)
        it = np.zeros(n, dtype=np.int32)
        import ctypes as C
        rc = sim.lib.phl_eos_invert_batch(sim.ctx, n, rho.ctypes.data, e.ctypes.data, abar.ctypes.data,
                                          zbar.ctypes.data, Tg.ctypes.data, p.ctypes.data, cs.ctypes.data,
                                          it.ctypes.data, 0)
        assert rc == 0
    mism = 0
    for i in range(0, n, 7):
        To, Po, so, ito = helm.rhoe_given(rho[i], e[i], abar[i], zbar[i], T0[i])
        if Tg[i] != To or it[i] != ito:
            mism += 1
    assert mism == 0


# ------------------------------------------------------------------------------ Helmholtz without USE_FASTEOS
@pytest.mark.parametrize("mhd,riemann", [(False, "lhllc"), (False, "hllc"), (True, "lhlld")])
def test_stratified_helmholtz_without_fasteos(gpu_lib, oracle, table, mhd, riemann):
    """helm_rhoP_given on each Riemann side from the face temperature guess, bit for bit."""
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd, riemann=riemann, fasteos=False)
    hg, ho, st = run_pair(cfg, h, 3, table=table, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["newton_nonconverged"] == 0 and st["nonfinite"] == 0
    if mhd:
        assert div_b_max(hg) <= 1e-13



# ------------------------------------------------------------------------------ PPH_REC / LIM5TH_REC
@pytest.mark.parametrize("rec", ["pph", "lim5th"])
def test_orszag_tang_higher_order(gpu_lib, oracle, rec):
    cfg, h = problems.orszag_tang_2d(48, rec=rec)
    hg, ho, _ = run_pair(cfg, h, 10, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert div_b_max(hg) <= 1e-13


@pytest.mark.parametrize("mhd,riemann,rec", [(False, "lhllc", "pph"), (False, "lhllc", "lim5th"),
                                             (True, "lhlld", "pph"), (True, "lhlld", "lim5th")])
def test_stratified_helmholtz_higher_order(gpu_lib, oracle, table, mhd, riemann, rec):
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd, riemann=riemann, rec=rec)
    hg, ho, st = run_pair(cfg, h, 3, table=table, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["newton_nonconverged"] == 0 and st["nonfinite"] == 0


# ------------------------------------------------------------------------------ USE_SHOCK_FLATTENING
@pytest.mark.parametrize("riemann,rec", [("hllc", "lim2nd"), ("lhllc", "lim2nd"), ("hllc", "pph"),
                                         ("hllc", "lim5th")])
def test_blast_shock_flattening(gpu_lib, oracle, riemann, rec):
    """Detector, PLM fallback in flagged cells and HLL on their faces, bit for bit."""
    cfg, h = problems.blast_2d(48, riemann=riemann, rec=rec)
    hg, ho, st = run_pair(cfg, h, 12, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["nonfinite"] == 0


@pytest.mark.parametrize("rec", ["lim2nd", "lim5th"])
def test_orszag_tang_shock_flattening(gpu_lib, oracle, rec):
    cfg, h = problems.orszag_tang_2d(48, rec=rec, shock_flattening=True)
    hg, ho, _ = run_pair(cfg, h, 10, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert div_b_max(hg) <= 1e-13


def test_hot_bubble_shock_flattening(gpu_lib, oracle):
    """WB ideal gas: the detector adds the cell equilibrium of the ghost layers to the pressure."""
    cfg, h = problems.hot_bubble_2d(32, shock_flattening=True, eps_sf=0.12)
    hg, ho, _ = run_pair(cfg, h, 3, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0


@pytest.mark.parametrize("mhd,rec,fasteos", [(False, "lim2nd", True), (False, "pph", True), (True, "lim2nd", True),
                                             (False, "lim2nd", False)])
def test_stratified_shock_flattening(gpu_lib, oracle, table, mhd, rec, fasteos):
    """eps_sf = 0.4 flags the upper half of the box (the pressure scale height shrinks upwards);
    with WB and USE_FASTEOS this includes the x1 sweep's handling of gamma_e on flagged faces."""
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd, rec=rec, fasteos=fasteos, shock_flattening=True,
                                    eps_sf=0.4)
    hg, ho, st = run_pair(cfg, h, 3, table=table, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["nonfinite"] == 0
    if mhd:
        assert div_b_max(hg) <= 1e-13


# ------------------------------------------------------------------------------ Fermi-gas table
@pytest.mark.parametrize("mhd", [False, True])
def test_stratified_on_fermi_table(gpu_lib, oracle, mhd):
    """The stratified box on the electron-positron Fermi-gas table (helm_fermi), bit for bit."""
    from phlegethon_b200 import helm_fermi
    from test_helm_fermi import SMALL
    table = helm_fermi.generate(**SMALL)
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd, table=dict(SMALL), eos_model="fermi")
    hg, ho, st = run_pair(cfg, h, 3, table=table, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["newton_nonconverged"] == 0 and st["nonfinite"] == 0
    if mhd:
        assert div_b_max(hg) <= 1e-13


# ------------------------------------------------------------------------------ FLUX_IS_ALL_MACH
@pytest.mark.parametrize("maker", ["orszag_tang", "blast"])
def test_all_mach_parity(gpu_lib, oracle, maker):
    """Upwind outer states of LHLLD / LHLLC (FLUX_IS_ALL_MACH) on flows with supersonic faces."""
    if maker == "orszag_tang":
        cfg, h = problems.orszag_tang_2d(48, riemann="lhlld")
    else:
        cfg, h = problems.blast_2d(48, riemann="lhllc")
    h.cfg = cfg = cfg.replace(all_mach=True)
    hg, ho, _ = run_pair(cfg, h, 12, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0


# ------------------------------------------------------------------------------ USE_CONSTANT_ACCELERATION
@pytest.mark.parametrize("maker", ["hot_bubble", "stratified_mhd"])
def test_constant_acceleration_parity(gpu_lib, oracle, table, maker):
    if maker == "hot_bubble":
        cfg, h = problems.hot_bubble_2d(48)
        acc = (0.05, -0.02, 0.0)
    else:
        cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=True)
        acc = (3.0e5, 0.0, -2.0e5)
    h.cfg = cfg = cfg.replace(constant_acceleration=True, acc=acc)
    hg, ho, st = run_pair(cfg, h, 4, table=table if cfg.helmholtz else None, oracle=oracle)
    assert max_abs_diff(hg, ho) == 0.0
    assert st["nonfinite"] == 0


def test_fp64_unchanged_after_split_contexts(gpu_lib, oracle, table):
    """Regression for a build defect: the FP64 and split units once instantiated the same
    dt / step-0 thermodynamics kernels under one weak host symbol, so after split contexts had
    run, an FP64 context could launch the split unit's FMA-contracted copy.  Run split contexts
    of the same option sets first, in this process, then require the FP64 boxes bit for bit."""
    from phlegethon_b200.abi import Simulation
    for mhd in (False, True):
        cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd)
        with Simulation(cfg.replace(precision="fp32_split"), table) as sim:
            sim.upload(h.copy())
            sim.init_thermo()
            sim.compute_hyperbolic_dt()
            sim.time_loop(2)
    for mhd in (False, True):
        cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=mhd)
        hg, ho, _ = run_pair(cfg, h, 3, table=table, oracle=oracle)
        assert max_abs_diff(hg, ho) == 0.0, field_errors(hg, ho)
