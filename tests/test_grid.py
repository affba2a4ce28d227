"""Host-side helpers of phlegethon_b200.grid (no GPU)."""
import numpy as np

from phlegethon_b200 import problems
from phlegethon_b200.grid import helm_state_range


def test_helm_state_range_covers_the_box():
    """The learned guess's sample range of the stratified box: log10 rho and log10 T of every
    interior cell inside [lo, hi] with the margin, Abar and Zbar the box's advected values, the
    temperatures clipped to the table."""
    cfg, h = problems.stratified_3d(8, ny=16, nz=4, mhd=True)
    lo, hi = helm_state_range(h, cfg, margin=0.1)
    w = h.interior(h.prim)
    lr, lt = np.log10(w[0]), np.log10(h.interior(h.temp))
    assert np.isclose(lo[0], lr.min() - 0.1) and np.isclose(hi[0], lr.max() + 0.1)
    assert np.isclose(lo[1], lt.min() - 0.1) and np.isclose(hi[1], lt.max() + 0.1)
    assert cfg.helm_ltlo <= lo[1] < hi[1] <= cfg.helm_lthi
    assert np.isclose(lo[2], problems.STRAT_ABAR) and np.isclose(hi[2], problems.STRAT_ABAR)
    assert np.isclose(lo[3], problems.STRAT_ZBAR) and np.isclose(hi[3], problems.STRAT_ZBAR)
    # a margin reaching past the table's temperatures is clipped to them
    lo2, hi2 = helm_state_range(h, cfg, margin=10.0)
    assert lo2[1] == cfg.helm_ltlo and hi2[1] == cfg.helm_lthi
