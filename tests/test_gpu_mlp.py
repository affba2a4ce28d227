"""The learned temperature guess: tensor-core MLP training and inference kernels against the CPU
reference, training on EoS-generated samples, and what the trained guess gains over the cold
bracket guess (the method without it) and over the untrained network."""
import ctypes as C

import numpy as np
import pytest

from phlegethon_b200 import problems

pytestmark = pytest.mark.gpu


def _sim(table):
    from phlegethon_b200.abi import Simulation
    cfg, _ = problems.stratified_3d(8)
    return Simulation(cfg, table)


def test_mlp_gradient_matches_cpu_reference(gpu_lib, table):
    import mlp_ref
    rng = np.random.default_rng(1)
    p = (rng.standard_normal(mlp_ref.NPARAM) * 0.2).astype(np.float32)
    n = 256
    X = rng.uniform(-1, 1, size=(n, 4)).astype(np.float32)
    t = rng.uniform(-1, 1, size=n).astype(np.float32)
    with _sim(table) as sim:
        assert sim.lib.phl_mlp_set_params(sim.ctx, p.ctypes.data_as(C.POINTER(C.c_float))) == 0
        g = np.zeros(mlp_ref.NPARAM, dtype=np.float32)
        loss = C.c_double()
        rc = sim.lib.phl_mlp_gradient(sim.ctx, n, X.ctypes.data, t.ctypes.data, g.ctypes.data, C.byref(loss))
        assert rc == 0
    lref, gref = mlp_ref.loss_and_grad(p.astype(np.float64), X, t, use_bf16=True)
    assert abs(loss.value - lref) / lref < 1e-4
    rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert rel < 1e-4, rel
    # against pure FP64 arithmetic the BF16 tensor-core operands cost a few percent at most
    _, g64 = mlp_ref.loss_and_grad(p.astype(np.float64), X, t, use_bf16=False)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 3e-2


def test_mlp_inference_matches_cpu_reference(gpu_lib, table):
    import torch
    import mlp_ref
    rng = np.random.default_rng(2)
    p = (rng.standard_normal(mlp_ref.NPARAM) * 0.2).astype(np.float32)
    n = 1000  # not a multiple of the 32-sample warp tile
    X = rng.uniform(-1, 1, size=(n, 4)).astype(np.float32)
    with _sim(table) as sim:
        assert sim.lib.phl_mlp_set_params(sim.ctx, p.ctypes.data_as(C.POINTER(C.c_float))) == 0
        dX = torch.from_numpy(X).cuda()
        out = torch.zeros(n, dtype=torch.float32, device="cuda")
        assert sim.lib.phl_mlp_infer_device(sim.ctx, n, dX.data_ptr(), out.data_ptr()) == 0
        got = out.cpu().numpy().astype(np.float64)
    ref = mlp_ref.guess_log10T(p, X)
    assert np.max(np.abs(got - ref)) < 2e-3 * max(1.0, np.max(np.abs(ref - mlp_ref.prior(X))))


def _invert(sim, n, rho, e, abar, zbar, guess):
    Tg = np.zeros(n)
    it = np.zeros(n, dtype=np.int32)
    sim.reset_status()
    rc = sim.lib.phl_eos_invert_batch(sim.ctx, n, rho.ctypes.data, e.ctypes.data, abar.ctypes.data,
                                      zbar.ctypes.data, Tg.ctypes.data, None, None, it.ctypes.data, guess)
    assert rc == 0
    return Tg, it, sim.status()


def _energy(sim, rho, T, abar, zbar):
    import torch
    d = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (rho, T, abar, zbar)]
    de = torch.zeros(len(rho), dtype=torch.float64, device="cuda")
    assert sim.lib.phl_eos_energy_device(sim.ctx, len(rho), *[x.data_ptr() for x in d], de.data_ptr()) == 0
    return de.cpu().numpy()


def test_mlp_training_gains_over_bracket_guess(gpu_lib, table):
    n = 8192
    rho, T, abar, zbar = problems.eos_samples(n, seed=77)
    with _sim(table) as sim:
        lib = sim.lib
        e = _energy(sim, rho, T, abar, zbar)
        # untrained network (initialisation only)
        assert lib.phl_mlp_train(sim.ctx, 1 << 16, 12345, 0, 8192, C.c_double(1e-2), None) == 0
        _, _, st0 = _invert(sim, n, rho, e, abar, zbar, 1)
        loss = C.c_double()
        assert lib.phl_mlp_train(sim.ctx, 1 << 22, 12345, 256, 8192, C.c_double(3e-3), C.byref(loss)) == 0
        assert loss.value < 1e-4, loss.value
        Tb, itb, stb = _invert(sim, n, rho, e, abar, zbar, 2)
        Tm, itm, stm = _invert(sim, n, rho, e, abar, zbar, 1)
        # conditioning kappa = |E / (T dE/dT)|: an energy residual r moves T by about kappa * r
        h = 1e-6
        dE = (_energy(sim, rho, Tb * (1 + h), abar, zbar) - _energy(sim, rho, Tb * (1 - h), abar, zbar)) / (2 * h)
        kappa = np.abs(e / dE)
        # both temperatures satisfy the reference tolerance on the energy
        for Tx in (Tb, Tm):
            assert np.max(np.abs(_energy(sim, rho, Tx, abar, zbar) - e) / np.abs(e)) < 1e-11
    assert stb["newton_nonconverged"] == 0 and stm["newton_nonconverged"] == 0
    assert stm["tensor_core_stalls"] == 0 and st0["tensor_core_stalls"] == 0
    assert stm["newton_calls"] == n and stb["newton_calls"] == n
    # same temperature: to 1e-10 where the inversion is well conditioned, and everywhere within
    # what the 1e-11 energy tolerance allows
    rel = np.abs(Tm - Tb) / Tb
    good = kappa < 10
    assert good.mean() > 0.5
    assert np.max(rel[good]) < 1e-10
    assert np.all(rel <= 1e-10 + 4e-11 * kappa)
    # training lifts the acceptance well above that of the fixed analytic part of the output alone
    # (the untrained network)
    assert stm["mlp_accepted"] > 0.8 * n, (stm, st0)
    assert stm["mlp_accepted"] > st0["mlp_accepted"] + 0.15 * n, (stm, st0)
    # gain: fewer EoS evaluations per inversion (guess construction + Newton iterations)
    cost_b = (stb["guess_evaluations"] + stb["newton_iterations"]) / n
    cost_m = (stm["guess_evaluations"] + stm["newton_iterations"]) / n
    cost_0 = (st0["guess_evaluations"] + st0["newton_iterations"]) / n
    assert stm["newton_iterations"] == int(itm.sum()) and stb["newton_iterations"] == int(itb.sum())
    assert cost_m < 0.75 * cost_b, (cost_m, cost_b)
    assert cost_m < cost_0, (cost_m, cost_0)


def test_bracket_guess_matches_oracle_bitwise(gpu_lib, oracle, table):
    """The GPU batch inversion from the bracket guess equals the C oracle's: same T, same count."""
    n = 4096
    rho, T, abar, zbar = problems.eos_samples(n, seed=21)
    cfg, _ = problems.stratified_3d(8)
    helm = oracle.Helm.for_config(cfg, *table)
    with _sim(table) as sim:
        e = _energy(sim, rho, T, abar, zbar)
        Tg, itg, _ = _invert(sim, n, rho, e, abar, zbar, 2)
    To, ito = helm.invert_batch(rho, e, abar, zbar, guess=2, nthreads=4)
    assert np.array_equal(Tg, To)
    assert np.array_equal(itg, ito)


# ------------------------------------------------------------------------------ learned guess in the step
def test_learned_guess_inside_the_split_mhd_step(gpu_lib, table):
    """eos_guess = PHL_GUESS_MLP: every cell's Newton starts from the trained network's guess,
    judged by at most 3 reference iterations with the warm start as the fallback.  The state
    equals the warm-start run to the Newton tolerance, and most guesses are accepted with a
    network fitted over the whole EoS benchmark range (about 70% in this moderately degenerate
    box, where the network's 0.2% error leaves the third Newton step just above the tolerance
    for the rest; fitted over the run's own range, all of them: the next test)."""
    import ctypes as C
    from phlegethon_b200.abi import Simulation
    from util import field_errors
    cfg, h = problems.stratified_3d(16, ny=16, nz=16, mhd=True)
    out, stats = {}, {}
    for guess in ("warm", "mlp"):
        c = cfg.replace(precision="fp32_split", eos_guess=guess)
        hg = h.copy()
        with Simulation(c, table) as sim:
            if guess == "mlp":
                loss = C.c_double()
                # the full training of the EoS benchmark (2^22 samples, 256 epochs, ~5 s)
                assert sim.lib.phl_mlp_train(sim.ctx, 1 << 22, 11, 256, 8192, C.c_double(3e-3), C.byref(loss)) == 0
            sim.upload(hg)
            sim.init_thermo()
            sim.compute_hyperbolic_dt()
            sim.reset_status()
            done, _ = sim.time_loop(10)
            assert done == 10
            sim.download(hg)
            stats[guess] = sim.status()
        out[guess] = hg
    err = field_errors(out["mlp"], out["warm"])
    assert max(err[f] for f in ("rho", "p", "e", "T")) <= 1e-9, err
    s = stats["mlp"]
    assert s["nonfinite"] == 0 and s["newton_nonconverged"] == 0
    assert s["mlp_accepted"] + s["mlp_rejected"] == s["newton_calls"]
    assert s["mlp_accepted"] > 0.5 * s["newton_calls"], s
    assert s["guess_evaluations"] == s["newton_calls"]


@pytest.mark.gpu
def test_learned_guess_trained_on_the_run_range(gpu_lib, table):
    """A network fitted over the run's own states (phl_mlp_set_sample_range with log10 rho and
    log10 T of the box widened by 0.1 dex and its Abar, Zbar) passes the 3-iteration judgment for
    every cell, and the state equals the warm-start run to the Newton tolerance.  Ranges that
    are empty or leave the table are refused."""
    import ctypes as C
    from phlegethon_b200.abi import PhlError, Simulation
    from phlegethon_b200.grid import helm_state_range
    from util import field_errors
    cfg, h = problems.stratified_3d(16, ny=16, nz=16, mhd=True)
    out, stats = {}, {}
    for guess in ("warm", "mlp"):
        c = cfg.replace(precision="fp32_split", eos_guess=guess)
        hg = h.copy()
        with Simulation(c, table) as sim:
            sim.upload(hg)
            sim.init_thermo()
            if guess == "mlp":
                with pytest.raises(PhlError):
                    sim.set_mlp_sample_range([5.0, 8.0, 2.0, 1.0], [4.0, 9.0, 2.0, 1.0])
                with pytest.raises(PhlError):
                    sim.set_mlp_sample_range([5.0, 8.0, 2.0, 1.0], [6.0, 14.0, 2.0, 1.0])
                h0 = h.copy()
                sim.download(h0)
                lo, hi = helm_state_range(h0, cfg)
                sim.set_mlp_sample_range(lo, hi)
                loss = C.c_double()
                assert sim.lib.phl_mlp_train(sim.ctx, 1 << 22, 11, 256, 8192, C.c_double(3e-3), C.byref(loss)) == 0
            sim.compute_hyperbolic_dt()
            sim.reset_status()
            done, _ = sim.time_loop(10)
            assert done == 10
            sim.download(hg)
            stats[guess] = sim.status()
        out[guess] = hg
    err = field_errors(out["mlp"], out["warm"])
    assert max(err[f] for f in ("rho", "p", "e", "T")) <= 1e-9, err
    s = stats["mlp"]
    assert s["nonfinite"] == 0 and s["newton_nonconverged"] == 0
    assert s["mlp_accepted"] + s["mlp_rejected"] == s["newton_calls"]
    assert s["mlp_accepted"] >= 0.99 * s["newton_calls"], s


def test_learned_rescue_of_poor_warm_starts(gpu_lib, table):
    """eos_guess = PHL_GUESS_MLP_RESCUE: every cell starts from the warm guess; a cell whose first
    warm Newton correction exceeds 2% of T is queued and finished from the network's judged
    guess (the warm guess as its fallback).  In the steady step no cell is queued and the state
    equals the warm-start run bit for bit.  After a restart from a temperature field 30% off
    (the stage input's T is the Newton's warm start) every cell of the first stage is rescued,
    the state equals the warm run to the Newton tolerance, and the rescued Newton needs fewer
    iterations than the one from the poor warm start.  The box (92,160 cells) fills more rescue
    tiles than the queue kernel has blocks, so blocks run several tensor-core tiles."""
    import ctypes as C
    from phlegethon_b200.abi import Simulation
    from phlegethon_b200.grid import helm_state_range
    from util import field_errors, max_abs_diff
    cfg, h = problems.stratified_3d(48, ny=40, nz=48, mhd=True)
    n = cfg.n_cells
    params = None
    out, stats = {}, {}
    for perturb in (False, True):
        for guess in ("warm", "mlp_rescue"):
            c = cfg.replace(precision="fp32_split", eos_guess=guess)
            hg = h.copy()
            with Simulation(c, table) as sim:
                sim.upload(hg)
                sim.init_thermo()
                if guess != "warm":
                    if params is None:
                        h0 = h.copy()
                        sim.download(h0)
                        lo, hi = helm_state_range(h0, cfg)
                        # wide enough in T for the perturbed restart's states
                        lo[1] -= 0.3
                        hi[1] += 0.3
                        sim.set_mlp_sample_range(lo, hi)
                        assert sim.lib.phl_mlp_train(sim.ctx, 1 << 22, 11, 256, 8192, C.c_double(3e-3), None) == 0
                        params = np.zeros(PHL_MLP_NPARAMS, dtype=np.float32)
                        assert sim.lib.phl_mlp_get_params(sim.ctx, params.ctypes.data_as(C.POINTER(C.c_float))) == 0
                    else:
                        assert sim.lib.phl_mlp_set_params(sim.ctx, params.ctypes.data_as(C.POINTER(C.c_float))) == 0
                if perturb:
                    dyn = h.dynamic_copy()
                    sim.download(dyn)
                    dyn.temp *= 1.3
                    sim.upload(dyn)
                sim.compute_hyperbolic_dt()
                sim.reset_status()
                done, _ = sim.time_loop(3)
                assert done == 3
                sim.download(hg)
                stats[perturb, guess] = sim.status()
            out[perturb, guess] = hg
    for perturb in (False, True):
        s = stats[perturb, "mlp_rescue"]
        assert s["nonfinite"] == 0 and s["newton_nonconverged"] == 0 and s["tensor_core_stalls"] == 0
        assert s["newton_calls"] == 9 * n  # 3 steps x 3 stages, one inversion per cell
    # steady step: nothing queued, identical to the warm start
    s = stats[False, "mlp_rescue"]
    assert s["mlp_accepted"] + s["mlp_rejected"] == 0, s
    assert max_abs_diff(out[False, "mlp_rescue"], out[False, "warm"]) == 0.0
    # poor warm start: the first stage goes through the network, the answer is unchanged
    s, w = stats[True, "mlp_rescue"], stats[True, "warm"]
    rescued = s["mlp_accepted"] + s["mlp_rejected"]
    assert rescued >= n, s
    assert s["mlp_accepted"] >= 0.95 * rescued, s
    err = field_errors(out[True, "mlp_rescue"], out[True, "warm"])
    assert max(err[f] for f in ("rho", "p", "e", "T")) <= 1e-9, err
    assert s["newton_iterations"] < w["newton_iterations"], (s, w)


PHL_MLP_NPARAMS = 4 * 64 + 64 + 64 * 64 + 64 + 64 + 1
