"""The x3 slab decomposition of the MHD step, checked on CPU with two gloo ranks.

The library keeps the whole domain on one GPU.  A decomposition into slabs along x3, one per
GPU, needs per RK stage: the ghost planes of every cell array the stencils read (primitives,
scalars, cell B), one plane on either side of the x1- and x2-face EMFs and mass-flux signs that
the corner EMFs of the slab's edges read, and a max-reduction of smax for dt -- the fields the
reference's MPI bricks (set up at source/source.F90:1160-1210) exchange at the start of a stage
(7183-7193) and before the corner EMFs (11374-11384), and its dt reduction (13954).  This
test runs the numpy restatement of the 3D MHD step on two slabs that exchange exactly that and
nothing else, and requires the assembled result to equal the single-domain step bit for bit:
the plan is complete, and the corners and faces on a slab boundary, computed by both
neighbours, agree.  The stratified Helmholtz box, with its reflective x2 walls, adds the
temperatures and the FASTEOS gammas to the exchanged cell arrays, as the reference does.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class SlabHalo:
    """Ghost exchange of one x3 slab over torch.distributed: x1 periodic, x2 periodic or (walls)
    mirrored at reflective walls, x3 periodic across the ranks."""

    def __init__(self, rank, world, dx, walls=False):
        self.rank, self.world, self.dx, self.walls = rank, world, dx, walls
        self.sent = 0          # bytes this rank has contributed to the exchanges

    def _neighbours(self, lo, hi):
        """All ranks' (lo, hi) boundary blocks; returns the lower neighbour's hi block and the
        upper neighbour's lo block."""
        t = torch.from_numpy(np.ascontiguousarray(np.stack([lo, hi])))
        got = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(got, t)
        self.sent += t.numel() * t.element_size()
        below = got[(self.rank - 1) % self.world][1].numpy()
        above = got[(self.rank + 1) % self.world][0].numpy()
        return below, above

    def fill(self, a, G, flip=False):
        # x1 and x2 are whole on every rank: their ghosts locally, then the x3 ghost planes
        # (whole padded planes, so the corner ghosts come along) from the neighbours
        for ax in ((0,) if self.walls else (0, 1)):
            m = a.shape[ax] - 2 * G
            lo = [slice(None)] * 3
            src = [slice(None)] * 3
            lo[ax], src[ax] = slice(0, G), slice(m, m + G)
            a[tuple(lo)] = a[tuple(src)]
            lo[ax], src[ax] = slice(m + G, m + 2 * G), slice(G, 2 * G)
            a[tuple(lo)] = a[tuple(src)]
        if self.walls:
            ny = a.shape[1] - 2 * G
            f = -1.0 if flip else 1.0
            for g in range(1, G + 1):
                a[:, G - g] = f * a[:, G + g - 1]
                a[:, ny + G - 1 + g] = f * a[:, ny + G - g]
        nz = a.shape[2] - 2 * G
        below, above = self._neighbours(a[:, :, G:2 * G], a[:, :, nz:nz + G])
        a[:, :, :G] = below
        a[:, :, nz + G:] = above

    def wrap3(self, e):
        below, above = self._neighbours(e[:, :, :1], e[:, :, -1:])
        return np.concatenate([below, e, above], axis=2)

    def max(self, x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())


def _worker(rank, world, port, riemann, steps, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from phlegethon_b200.grid import HostGrid
        from numpy_restatement import mhd_3d_steps
        from util import smooth_box
        full = smooth_box(3, riemann, "lim2nd", mhd=True)
        c = full.cfg
        G, nz = c.ngc, c.nx3
        nzl = nz // world
        k0 = rank * nzl
        loc = HostGrid(c.replace(nx3=nzl))
        loc.prim[...] = full.prim[:, :, :, k0:k0 + nzl + 2 * G]
        for d in range(3):
            bl, bf = loc.bface_interior(d), full.bface_interior(d)
            bl[...] = bf[:, :, k0:k0 + bl.shape[2]]
        halo = SlabHalo(rank, world, c.dx())
        W, eint, temp, b, dt = mhd_3d_steps(loc, steps, riemann == "lhlld", halo=halo)
        out[rank] = ([w[G:-G, G:-G, G:-G] for w in W], eint, b, dt, halo.sent)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("riemann", ["hlld", "lhlld"])
def test_two_slabs_reproduce_the_single_domain_step(riemann):
    sys.path.insert(0, HERE)
    from numpy_restatement import mhd_3d_steps
    from util import smooth_box
    steps = 3
    full = smooth_box(3, riemann, "lim2nd", mhd=True)
    Wf, eintf, _, bf, dtf = mhd_3d_steps(full.copy(), steps, riemann == "lhlld")
    G = full.cfg.ngc
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, riemann, steps, out), nprocs=2, start_method="spawn")
    W0, e0, b0, dt0, _ = out[0]
    W1, e1, b1, dt1, _ = out[1]
    assert dt0 == dt1 == dtf
    for v in range(full.cfg.nvars):
        np.testing.assert_array_equal(np.concatenate([W0[v], W1[v]], axis=2), Wf[v][G:-G, G:-G, G:-G])
    np.testing.assert_array_equal(np.concatenate([e0, e1], axis=2), eintf)
    for d in range(2):
        np.testing.assert_array_equal(np.concatenate([b0[d], b1[d]], axis=2), bf[d])
    # what crossed: per RK stage G ghost planes on either side of every cell array (nvars
    # primitives and scalars, 3 cell-B components) and one plane on either side of the x1- and
    # x2-face EMFs and signs, plus the cell-B planes of the step-0 set-up
    c = full.cfg
    plane = (c.nx1 + 2 * G) * (c.nx2 + 2 * G)
    per_stage = (c.nvars + 3) * 2 * G * plane + 2 * 2 * (c.nx1 * (c.nx2 + 1) + (c.nx1 + 1) * c.nx2)
    assert out[0][4] == out[1][4] == 8 * (steps * c.rk_stages * per_stage + 3 * 2 * G * plane)
    # the x3 faces on the slab boundaries are computed by both neighbours and must agree
    nzl = full.cfg.nx3 // 2
    np.testing.assert_array_equal(b0[2][:, :, :nzl], bf[2][:, :, :nzl])
    np.testing.assert_array_equal(b1[2][:, :, :nzl + 1], bf[2][:, :, nzl:])
    np.testing.assert_array_equal(b0[2][:, :, nzl], b1[2][:, :, 0])
    np.testing.assert_array_equal(b1[2][:, :, nzl], b0[2][:, :, 0])


def _slab_of(full, rank, world):
    """The x3 slab of host grid `full` that rank owns: every cell array with its ghost planes,
    every face array of its planes (the x3 faces on both of its ends)."""
    from phlegethon_b200.grid import HostGrid
    c = full.cfg
    G, nzl = c.ngc, c.nx3 // world
    k0 = rank * nzl
    loc = HostGrid(c.replace(nx3=nzl))
    for name in ("prim", "temp", "eint", "gammaf", "grav", "phi_cc", "eq_prim_cc", "eq_gammae_cc", "b_cc"):
        a = getattr(full, name)
        if a is not None:
            getattr(loc, name)[...] = a[..., k0:k0 + nzl + 2 * G]
    for name in ("phi_x", "eq_prim_x", "eq_gammae_x"):
        for d in range(3):
            a = getattr(full, name)[d]
            if a is not None:
                getattr(loc, name)[d][...] = a[..., k0:k0 + nzl + (d == 2)]
    if c.mhd:
        for d in range(3):
            bl = loc.bface_interior(d)
            bl[...] = full.bface_interior(d)[:, :, k0:k0 + bl.shape[2]]
    return loc


def _strat_case(riemann, flattening):
    from phlegethon_b200 import helm_table, problems
    import numpy_restatement_eos as RE
    tab, dpdr = helm_table.generate(nrho=271, nT=101)
    cfg, h = problems.stratified_3d(8, ny=12, nz=6, mhd=riemann.endswith("d"), mach=0.05,
                                    table=helm_table.X1_TABLE, riemann=riemann,
                                    shock_flattening=flattening, eps_sf=0.6)
    nd = RE.nodes(cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)
    return h, tab, dpdr, nd


def _strat_worker(rank, world, port, riemann, flattening, steps, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from numpy_restatement import stratified_steps
        full, tab, dpdr, nd = _strat_case(riemann, flattening)
        loc = _slab_of(full, rank, world)
        halo = SlabHalo(rank, world, full.cfg.dx(), walls=True)
        W, eint, temp, (ge, gc), b, dt = stratified_steps(loc, tab, dpdr, nd, steps, halo=halo)
        G = full.cfg.ngc
        out[rank] = ([w[G:-G, G:-G, G:-G] for w in W], temp, ge[G:-G, G:-G, G:-G], b, dt)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("riemann, flattening", [("lhlld", False), ("lhlld", True), ("lhllc", False)])
def test_two_slabs_of_the_stratified_box_reproduce_the_single_domain_step(riemann, flattening):
    """The stratified Helmholtz box (the benchmark's workloads, 8 x 12 x 6) split into two x3 slabs
    of 3 planes: ghost planes of the primitives, scalars, cell B, the gammas and the
    temperatures (the no-FASTEOS face guess and the Newton's warm start read the latter), the
    EMF planes and the dt maximum reproduce the single-domain step bit for bit, with
    shock flattening's detector reading the exchanged ghosts."""
    sys.path.insert(0, HERE)
    from numpy_restatement import stratified_steps
    steps = 2
    full, tab, dpdr, nd = _strat_case(riemann, flattening)
    Wf, _, Tf, (gef, _), bf, dtf = stratified_steps(full.copy(), tab, dpdr, nd, steps)
    G = full.cfg.ngc
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_strat_worker, args=(2, port, riemann, flattening, steps, out), nprocs=2,
                       start_method="spawn")
    (W0, T0, g0, b0, dt0), (W1, T1, g1, b1, dt1) = out[0], out[1]
    assert dt0 == dt1 == dtf
    for v in range(full.cfg.nvars):
        np.testing.assert_array_equal(np.concatenate([W0[v], W1[v]], axis=2), Wf[v][G:-G, G:-G, G:-G])
    np.testing.assert_array_equal(np.concatenate([T0, T1], axis=2), Tf)
    np.testing.assert_array_equal(np.concatenate([g0, g1], axis=2), gef[G:-G, G:-G, G:-G])
    if full.cfg.mhd:
        for d in range(2):
            np.testing.assert_array_equal(np.concatenate([b0[d], b1[d]], axis=2), bf[d])
        np.testing.assert_array_equal(np.concatenate([b0[2][:, :, :-1], b1[2]], axis=2), bf[2])
