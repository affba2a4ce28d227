"""Comparison helpers shared by the parity tests."""
import numpy as np


def rel_l1(a, b):
    """Relative L1 difference sum|a-b| / sum|b| (interior cells)."""
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def field_errors(hg, ho):
    """Per-field relative L1 of GPU grid `hg` against oracle grid `ho` (interior only)."""
    c = hg.cfg
    out = {}
    pg, po = hg.interior(hg.prim), ho.interior(ho.prim)
    out["rho"] = rel_l1(pg[0], po[0])
    for d in range(c.sdims):
        out["v%d" % (d + 1)] = rel_l1(pg[1 + d], po[1 + d])
    out["p"] = rel_l1(pg[1 + c.sdims], po[1 + c.sdims])
    out["e"] = rel_l1(hg.interior(hg.eint), ho.interior(ho.eint))
    out["T"] = rel_l1(hg.interior(hg.temp), ho.interior(ho.temp))
    if c.mhd:
        for d in range(c.sdims):
            out["b%d" % (d + 1)] = rel_l1(hg.bface_interior(d), ho.bface_interior(d))
    return out


def max_abs_diff(hg, ho):
    """Largest absolute difference over the dynamic interior fields."""
    m = float(np.abs(hg.interior(hg.prim) - ho.interior(ho.prim)).max())
    m = max(m, float(np.abs(hg.interior(hg.eint) - ho.interior(ho.eint)).max()))
    m = max(m, float(np.abs(hg.interior(hg.temp) - ho.interior(ho.temp)).max()))
    if hg.cfg.mhd:
        for d in range(hg.cfg.sdims):
            m = max(m, float(np.abs(hg.bface_interior(d) - ho.bface_interior(d)).max()))
    return m


def div_b_max(h):
    """max |div B| * dx / max|B| over interior cells (face fields)."""
    c = h.cfg
    dx = c.dx()
    div = 0.0
    n = [c.nx1, c.nx2, c.nx3]
    for d in range(c.sdims):
        b = h.bface_interior(d)
        sl_hi = [slice(None)] * 3
        sl_lo = [slice(None)] * 3
        sl_hi[d] = slice(1, n[d] + 1)
        sl_lo[d] = slice(0, n[d])
        div = div + (b[tuple(sl_hi)] - b[tuple(sl_lo)]) / dx[d]
    bmax = max(float(np.abs(h.bface_interior(d)).max()) for d in range(c.sdims))
    return float(np.abs(div).max() * min(dx[: c.sdims]) / bmax)


def permute_axes(h, perm):
    """A copy of host grid `h` with its coordinate axes permuted: new axis a is old axis
    perm[a] (perm a permutation of 0..2; in 2D perm[2] == 2).  Cell arrays are transposed,
    vector components (velocity, gravity, cell B) and per-direction face arrays (face B, face
    potentials and equilibria) are re-indexed, and the configuration's extents, boundary
    conditions and acceleration follow the axes."""
    from phlegethon_b200.grid import HostGrid
    cfg, sd = h.cfg, h.cfg.sdims
    ax = lambda *v: [v[perm[d]] for d in range(3)]
    nx, xl, xu = ax(cfg.nx1, cfg.nx2, cfg.nx3), ax(cfg.x1l, cfg.x2l, cfg.x3l), ax(cfg.x1u, cfg.x2u, cfg.x3u)
    c2 = cfg.replace(nx1=nx[0], nx2=nx[1], nx3=nx[2], x1l=xl[0], x2l=xl[1], x3l=xl[2],
                     x1u=xu[0], x2u=xu[1], x3u=xu[2], bc=[list(b) for b in ax(*cfg.bc)],
                     acc=tuple(ax(*cfg.acc)))
    h2 = HostGrid(c2)
    cell = lambda a: np.transpose(a, perm)
    comp = lambda a: np.transpose(a, (0,) + tuple(1 + p for p in perm))

    def vector(a, b, lo):
        for d in range(sd):
            b[lo + d] = cell(a[lo + perm[d]])

    vector(h.prim, h2.prim, 1)
    for iv in [0] + list(range(sd + 1, cfg.nvars)):
        h2.prim[iv] = cell(h.prim[iv])
    for name, tr in (("temp", cell), ("eint", cell), ("phi_cc", cell), ("eq_gammae_cc", cell),
                     ("gammaf", comp), ("eq_prim_cc", comp)):
        if getattr(h, name) is not None:
            getattr(h2, name)[...] = tr(getattr(h, name))
    for name in ("grav", "b_cc"):
        if getattr(h, name) is not None:
            vector(getattr(h, name), getattr(h2, name), 0)
    for name, tr in (("phi_x", cell), ("eq_gammae_x", cell), ("b_x", cell), ("eq_prim_x", comp)):
        a, b = getattr(h, name), getattr(h2, name)
        for d in range(sd):
            if a[perm[d]] is not None:
                b[d][...] = tr(a[perm[d]])
    return h2


def mirror_axis(h, a):
    """A copy of host grid `h` mirrored along axis a (x_a -> x_al + x_au - x_a): every array
    is reversed along a (ghost layers and staggered faces map onto themselves), and the a
    components of the vectors (velocity, gravity, face and cell B) change sign.  The boundary
    conditions of the two sides of axis a swap."""
    cfg, sd = h.cfg, h.cfg.sdims
    bc = [list(b) for b in cfg.bc]
    bc[a] = bc[a][::-1]
    h2 = h.copy()
    h2.cfg = cfg.replace(bc=bc)
    flip = lambda x, lead: np.flip(x, axis=a + lead)
    for name in ("prim", "gammaf", "eq_prim_cc", "grav", "b_cc"):
        x = getattr(h, name)
        if x is not None:
            getattr(h2, name)[...] = flip(x, 1)
    for name in ("temp", "eint", "phi_cc", "eq_gammae_cc"):
        x = getattr(h, name)
        if x is not None:
            getattr(h2, name)[...] = flip(x, 0)
    for name, lead in (("phi_x", 0), ("eq_gammae_x", 0), ("b_x", 0), ("eq_prim_x", 1)):
        for d in range(sd):
            x = getattr(h, name)[d]
            if x is not None:
                getattr(h2, name)[d][...] = flip(x, lead)
    h2.prim[1 + a] *= -1.0
    for name in ("grav", "b_cc"):
        if getattr(h2, name) is not None:
            getattr(h2, name)[a] *= -1.0
    if h2.b_x[a] is not None:
        h2.b_x[a] *= -1.0
    return h2


def smooth_periodic(shape, periods, rng, stagger=None):
    """Three random Fourier modes over the index grid of a padded array, periodic with the
    interior extent along every axis whose period is given (constant along the others);
    `stagger` marks the face axis, whose index 1 is the left face of cell 1."""
    idx = np.meshgrid(*[np.arange(s, dtype=float) for s in shape], indexing="ij")
    f = np.zeros(shape)
    for _ in range(3):
        ph, kk, a = rng.uniform(0, 2 * np.pi, 3), rng.integers(1, 3, 3), rng.normal()
        arg = sum(2 * np.pi * kk[d] * (idx[d] - (0.0 if stagger == d else 0.5)) / periods[d] + ph[d]
                  for d in range(3) if periods[d] is not None)
        f += a * np.cos(arg)
    return f / 3.0


def smooth_box(sdims, riemann, rec, mhd):
    """A smooth periodic box of unequal extents and cell counts (12 x 16 [x 8]) with one passive
    scalar: density, velocity, pressure, scalar and (mhd) face B from `smooth_periodic`, B_d
    independent of x_d so that div B = 0 on the faces."""
    from phlegethon_b200.grid import Config, HostGrid
    n = (12, 16, 8 if sdims == 3 else 1)
    cfg = Config(sdims=sdims, nx1=n[0], nx2=n[1], nx3=n[2], ngc=3 if rec == "lim5th" else 2, nas=1,
                 mhd=mhd, riemann=riemann, rec=rec, x1u=1.2, x2u=1.0, x3u=0.9, mach_cutoff=1e-4,
                 bc=[["periodic", "periodic"]] * 3)
    h = HostGrid(cfg)
    rng = np.random.default_rng(5)
    per = [n[d] if d < sdims else None for d in range(3)]
    h.prim[0] = 1.0 + 0.2 * smooth_periodic(h.cell_shape, per, rng)
    for d in range(sdims):
        h.prim[1 + d] = 0.3 * smooth_periodic(h.cell_shape, per, rng)
    h.prim[sdims + 1] = 1.0 + 0.2 * smooth_periodic(h.cell_shape, per, rng)
    h.prim[sdims + 2] = 0.5 + 0.2 * smooth_periodic(h.cell_shape, per, rng)
    if mhd:
        for d in range(sdims):
            # B_d independent of x_d: divergence-free on the faces
            pd = list(per)
            pd[d] = None
            h.b_x[d][...] = 0.4 + 0.3 * smooth_periodic(h.b_x[d].shape, pd, rng, stagger=d)
    return h
