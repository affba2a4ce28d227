"""The allocation-free EoS inversion entry point against the allocating one.

phl_eos_invert_batch_noalloc serves callers that cannot call cudaMalloc during a run: a driver
that hands all free device memory to its own pool allocator at start-up, or one whose time loop
must not allocate because cudaMalloc/cudaFree can synchronise the whole device.  Its device
copies live in one array compiled into the library and shared by all calls, so calls in a row
must each give the same answer as phl_eos_invert_batch, with nothing carried over from the call
before -- including a call at the full capacity of PHL_NOALLOC_MAX_SAMPLES samples.  The file is
named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from phlegethon_b200 import problems

pytestmark = pytest.mark.gpu


def _invert(sim, fn, rho, e, abar, zbar, T0, guess):
    n = rho.size
    T = T0.copy()
    p = np.zeros(n)
    cs = np.zeros(n)
    it = np.zeros(n, dtype=np.int32)
    rc = fn(sim.ctx, n, rho.ctypes.data, e.ctypes.data, abar.ctypes.data, zbar.ctypes.data, T.ctypes.data,
            p.ctypes.data, cs.ctypes.data, it.ctypes.data, guess)
    return rc, T, p, cs, it


def test_noalloc_matches_allocating_entry_point(gpu_lib, table):
    from phlegethon_b200.abi import Simulation
    cfg, _ = problems.stratified_3d(8)
    with Simulation(cfg, table) as sim:
        lib = sim.lib
        assert lib.phl_mlp_train(sim.ctx, 1 << 16, 7, 4, 4096, C.c_double(3e-3), None) == 0
        # two calls in a row, then one at the array's capacity (65536 samples)
        for call, (n, seed) in enumerate([(5000, 11), (3000, 12), (65536, 13)]):
            rho, T, abar, zbar = problems.eos_samples(n, seed=seed)
            e = np.zeros(n)
            d = {}
            import torch
            for name, arr in (("rho", rho), ("T", T), ("abar", abar), ("zbar", zbar)):
                d[name] = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
            de = torch.zeros(n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            assert lib.phl_eos_energy_device(sim.ctx, n, d["rho"].data_ptr(), d["T"].data_ptr(),
                                             d["abar"].data_ptr(), d["zbar"].data_ptr(), de.data_ptr()) == 0
            e = de.cpu().numpy()
            T0 = T * np.exp(0.2 * np.cos(np.arange(n) + call))
            # warm, bracket and learned guesses (the learned one also uses the rejection queue)
            for guess in (0, 2, 1):
                rc_a, Ta, pa, csa, ita = _invert(sim, lib.phl_eos_invert_batch, rho, e, abar, zbar, T0, guess)
                rc_b, Tb, pb, csb, itb = _invert(sim, lib.phl_eos_invert_batch_noalloc, rho, e, abar, zbar, T0,
                                                 guess)
                assert rc_a == 0 and rc_b == 0
                # same kernels on the same inputs: identical results (tolerance of the EoS tests)
                np.testing.assert_allclose(Tb, Ta, rtol=1e-12, atol=0)
                np.testing.assert_allclose(pb, pa, rtol=1e-12, atol=0)
                np.testing.assert_allclose(csb, csa, rtol=1e-12, atol=0)
                assert np.array_equal(itb, ita)


def test_noalloc_rejects_oversize(gpu_lib, table):
    from phlegethon_b200.abi import Simulation
    cfg, _ = problems.stratified_3d(8)
    n = 65536 + 1
    a = np.ones(n)
    with Simulation(cfg, table) as sim:
        rc = sim.lib.phl_eos_invert_batch_noalloc(sim.ctx, n, a.ctypes.data, a.ctypes.data, a.ctypes.data,
                                                  a.ctypes.data, a.copy().ctypes.data, None, None, None, 0)
    assert rc == -7  # PHL_E_TOO_LARGE
