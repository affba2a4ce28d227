"""The electron-positron Fermi-gas table generator (phlegethon_b200.helm_fermi).

Pinned by closed forms and identities of the ideal Fermi gas, by finite differences of its
own thermodynamics, and through the reference's table interpolation (the oracle's
helm_rhoT_given_full) against the exact model off the table nodes.
"""
import math

import numpy as np
import pytest

from phlegethon_b200 import helm_fermi as hf
from phlegethon_b200 import problems

# a small table around the stratified box (d = rho Ye 5e4..5e5 g/cm^3, T 1e8..4.5e8 K),
# 0.05 dex spacing like the 541 x 201 default table
SMALL = dict(nrho=51, nT=31, ldlo=4.0, ldhi=6.5, ltlo=7.5, lthi=9.0)


def test_cold_degenerate_limit():
    """T -> 0: number density and Chandrasekhar's zero-temperature pressure."""
    d = np.array([1e2, 1e4, 1e6, 1e8, 1e10, 1e12, 1e15])
    th = hf.thermo(d, np.full(d.shape, 1e3))
    n = hf.CONST_AV * d
    np.testing.assert_allclose(th["n"], n, rtol=1e-13)
    xf = hf.CONST_H * (3 * n / (8 * math.pi)) ** (1 / 3) / (hf.M_E * hf.CONST_C)
    p0 = (math.pi * hf.M_E ** 4 * hf.CONST_C ** 5 / (3 * hf.CONST_H ** 3) *
          (xf * (2 * xf ** 2 - 3) * np.sqrt(1 + xf ** 2) + 3 * np.arcsinh(xf)))
    # the finite-temperature correction ~ (pi / eta)^2 is 2e-7 at the lowest density
    np.testing.assert_allclose(th["P"], p0, rtol=3e-7)
    np.testing.assert_allclose(th["P"][2:], p0[2:], rtol=1e-11)


def test_boltzmann_limit():
    d = np.array([1e-12, 1e-10, 1e-8])
    T = np.array([1e5, 1e6, 1e7])
    th = hf.thermo(d, T)
    np.testing.assert_allclose(th["P"], th["n"] * hf.CONST_KB * T, rtol=1e-10)
    # kinetic energy 3/2 n kT up to the relativistic correction of order kT / m_e c^2
    beta = hf.CONST_KB * T / hf.MC2
    assert np.all(np.abs(th["E"] / (1.5 * th["n"] * hf.CONST_KB * T) - 1) < 2 * beta)


def test_euler_relation_and_pairs():
    """T S = E + P - mu n with the pair rest mass in E; net charge exact when pairs outnumber
    the net electrons by 16 orders of magnitude."""
    d = np.array([1e-2, 1e2, 1e5, 1e-6, 1e-12])
    T = np.array([1e9, 1e9, 1e10, 1e11, 1e13])
    th = hf.thermo(d, T)
    mu = th["eta"] * hf.CONST_KB * T
    np.testing.assert_allclose(T * th["S"], th["E"] + th["P"] - mu * th["n"], rtol=1e-12)
    np.testing.assert_allclose(th["n"], hf.CONST_AV * d, rtol=1e-12)
    assert th["n_pos"][3] / th["n"][3] > 1e15


def test_derivatives_match_finite_differences():
    """Analytic first and second derivatives of f and c = dP/dd against central differences,
    where differences resolve them (eta < 30, fewer pairs than net electrons)."""
    rng = np.random.default_rng(1)
    ld, lt = rng.uniform(-10, 12, 300), rng.uniform(4, 11, 300)
    d, T = 10 ** ld, 10 ** lt
    h = 1e-5

    def so(dd, tt):
        return hf._second_order(dd, tt)

    r0, rdp, rdm, rtp, rtm = so(d, T), so(d * (1 + h), T), so(d * (1 - h), T), so(d, T * (1 + h)), so(d, T * (1 - h))
    th = hf.thermo(d, T)
    ok = (th["eta"] < 30) & (th["n_pos"] < th["n"])
    assert ok.sum() > 100
    checks = [
        ((rdp["f"] - rdm["f"]) / (2 * h * d), r0["f_d"]),
        ((rtp["f"] - rtm["f"]) / (2 * h * T), r0["f_t"]),
        ((rdp["f_d"] - rdm["f_d"]) / (2 * h * d), r0["f_dd"]),
        ((rtp["f_d"] - rtm["f_d"]) / (2 * h * T), r0["f_dt"]),
        ((rtp["f_t"] - rtm["f_t"]) / (2 * h * T), r0["f_tt"]),
        ((rdp["f_d"] * (d * (1 + h)) ** 2 - rdm["f_d"] * (d * (1 - h)) ** 2) / (2 * h * d), r0["c"]),
    ]
    for fd, an in checks:
        np.testing.assert_allclose(fd[ok], an[ok], rtol=1e-6)


@pytest.fixture(scope="module")
def small_table():
    return hf.generate(**SMALL)


def test_table_interpolation_matches_the_model(oracle, small_table):
    """The reference's biquintic interpolation of the generated table reproduces the exact
    electron-positron gas (plus ions and radiation) between the nodes."""
    tab, dpdr = small_table
    helm = oracle.Helm(tab, dpdr, SMALL["nT"], SMALL["nrho"], SMALL["ltlo"], SMALL["lthi"], SMALL["ldlo"],
                       SMALL["ldhi"])
    abar, zbar = problems.STRAT_ABAR, problems.STRAT_ZBAR
    ye = zbar / abar
    rng = np.random.default_rng(3)
    rho = 10 ** rng.uniform(4.2, 6.2, 60) / ye
    T = 10 ** rng.uniform(7.7, 8.8, 60)
    for r, t in zip(rho, T):
        P, E, _, _ = helm.given_full(r, t, abar, zbar)
        assert abs(P / problems.fermi_pressure(r, t, abar, zbar) - 1) < 1e-6
        assert abs(E / problems.fermi_energy(r, t, abar, zbar) - 1) < 1e-6
        # and the Newton inversion of the reference returns the temperature
        T2, _, _, it = helm.rhoe_given(r, E, abar, zbar, 1.3 * t)
        assert abs(T2 / t - 1) < 1e-9 and it < 100


def test_stratified_box_on_the_fermi_table_is_hydrostatic(oracle, small_table):
    cfg, h = problems.stratified_3d(8, ny=16, nz=6, mach=0.0, table=dict(SMALL), eos_model="fermi")
    helm = oracle.Helm.for_config(cfg, *small_table)
    o = oracle.OracleGrid(h, helm, nthreads=2)
    o.init_thermo()
    o.compute_hyperbolic_dt()
    p0 = h.interior(h.prim)[4].copy()
    o.time_loop(3)
    s = h.interior(h.prim)
    assert float(np.abs(s[1:4]).max()) < 1e-6 * float(np.sqrt(p0 / s[0]).min())
    assert float(np.abs(s[4] / p0 - 1).max()) < 1e-12
