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
