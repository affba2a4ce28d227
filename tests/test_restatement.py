"""The C oracle against the independent numpy restatement (bit for bit)."""
import numpy as np

from phlegethon_b200 import problems
from numpy_restatement import hot_bubble_steps


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
