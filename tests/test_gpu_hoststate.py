"""GPU: the asynchronous host-state pipeline (phl_run_steps_host_async / phl_wait_host).

Each call uploads the dynamic state from host arrays, advances the requested steps and
downloads the state back, with the uploads of one call ordered chunk by chunk after the
downloads of the call before.  The result must equal the synchronous sequence
phl_upload_state -> phl_run_steps -> phl_download_state of the same steps bit for bit (same
kernels, same order), and the host arrays' ghost layers must be left as they were.
"""
import numpy as np
import pytest

from phlegethon_b200 import problems

pytestmark = pytest.mark.gpu

DYNAMIC = ("prim", "temp", "eint", "gammaf", "b_cc")


def dynamic_only(h):
    return h.dynamic_copy()


def arrays(h):
    out = [getattr(h, nm) for nm in DYNAMIC if getattr(h, nm) is not None]
    return out + [b for b in h.b_x if b is not None]


def start(cfg, h, table):
    from phlegethon_b200.abi import Simulation
    sim = Simulation(cfg, table)
    sim.upload(h)
    sim.init_thermo()
    sim.compute_hyperbolic_dt()
    dyn = dynamic_only(h)
    sim.download(dyn)
    return sim, dyn


@pytest.mark.parametrize("case", ["hot_bubble", "mhd_fp64", "mhd_split", "hydro_no_fasteos"])
def test_host_pipeline_matches_synchronous_steps(gpu_lib, table, case):
    if case == "hot_bubble":
        cfg, h = problems.hot_bubble_2d(48)
        tab = None
    else:
        cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=case.startswith("mhd"),
                                        fasteos=case != "hydro_no_fasteos")
        if case == "mhd_split":
            cfg = cfg.replace(precision="fp32_split")
            h.cfg = cfg
        tab = table
    nsteps = 4
    # synchronous reference: upload, one step, download, per step
    sim_a, dyn_a = start(cfg, h.copy(), tab)
    for _ in range(nsteps):
        sim_a.upload(dyn_a)
        sim_a.time_loop(1)
        sim_a.download(dyn_a)
    ta = sim_a.get_time()
    sim_a.close()
    # pipelined: queue every step, wait once
    sim_b, dyn_b = start(cfg, h.copy(), tab)
    for _ in range(nsteps):
        sim_b.time_loop_host_async(dyn_b, 1)
    sim_b.wait_host()
    tb = sim_b.get_time()
    sim_b.close()
    assert ta == tb
    # whole host arrays: interiors bit for bit, ghost layers untouched by both paths
    for x, y in zip(arrays(dyn_a), arrays(dyn_b)):
        assert np.array_equal(x, y)


def test_host_pipeline_then_synchronous_calls(gpu_lib, table):
    """Entry points called after queued host-state steps wait for their downloads first."""
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=True)
    sim, dyn = start(cfg, h.copy(), table)
    sim.time_loop_host_async(dyn, 2)
    dt, smax = sim.compute_hyperbolic_dt()  # drains the pipeline before it runs
    assert dt > 0 and smax > 0
    out = dynamic_only(h)
    sim.download(out)
    for x, y in zip(arrays(dyn), arrays(out)):
        assert np.array_equal(x, y)
    sim.close()


def test_host_pipeline_reads_and_writes_interiors_only(gpu_lib, table):
    """The pipeline moves only the interior of each host array: NaN in every ghost layer
    (cells and faces) changes nothing inside and stays NaN outside."""
    cfg, h = problems.stratified_3d(12, ny=16, nz=10, mhd=True)
    cfg = cfg.replace(precision="fp32_split")
    h.cfg = cfg
    sim_a, dyn_a = start(cfg, h.copy(), table)
    sim_b, dyn_b = start(cfg, h.copy(), table)
    ghost_masks = []
    for nm in DYNAMIC:
        a = getattr(dyn_b, nm)
        if a is None:
            continue
        keep = dyn_b.interior(a).copy()
        a[...] = np.nan
        dyn_b.interior(a)[...] = keep
        ghost_masks.append((nm, np.isnan(a)))
    for d in range(cfg.sdims):
        keep = dyn_b.bface_interior(d).copy()
        dyn_b.b_x[d][...] = np.nan
        dyn_b.bface_interior(d)[...] = keep
    for _ in range(3):
        sim_a.time_loop_host_async(dyn_a, 1)
        sim_b.time_loop_host_async(dyn_b, 1)
    sim_a.wait_host()
    sim_b.wait_host()
    sim_a.close()
    sim_b.close()
    for nm, mask in ghost_masks:
        a, b = getattr(dyn_a, nm), getattr(dyn_b, nm)
        assert np.array_equal(dyn_a.interior(a), dyn_b.interior(b)), nm
        assert np.isnan(b[mask]).all(), nm
    for d in range(cfg.sdims):
        assert np.array_equal(dyn_a.bface_interior(d), dyn_b.bface_interior(d))
        assert np.isnan(dyn_b.b_x[d]).sum() == dyn_b.b_x[d].size - dyn_b.bface_interior(d).size
