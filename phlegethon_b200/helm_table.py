"""Helmholtz free-energy table: synthetic generator and the reference's text format.

The reference reads a third-party table (Timmes' ``helm_table.dat``, fetched by
``data/get_data.sh:7-38``) with ``load_helm_table`` (``source/source.F90:23077-23156``):

* for every temperature row ``j = 1..nT`` and density column ``i = 1..nrho`` one line with
  ``f, df/drho, df/dT, d2f/drho2, d2f/dT2, d2f/drhodT, d3f/drho2dT, d3f/drhodT2,
  d4f/drho2dT2`` (``source.F90:23106-23115``);
* then, in the same order, ``c, dc/drho, dc/dT, d2c/drhodT`` with ``c = dP/d(rho Ye)``
  (``source.F90:23122-23126``).

"rho" in the table is the electron density variable ``d = rho*Ye`` and ``f`` is the
electron-positron free energy per unit ``d`` mass; ``helm_rhoT_given*`` combine it as
``P = d^2 df/dd`` and ``E = Ye (f - T df/dT)`` and add ions and radiation.

That table is not available here, so :func:`generate` fills the same layout from a closed-form,
thermodynamically consistent electron free energy:

    f(d, T) = 3/2 K d^(2/3) + R T (ln d - 3/2 ln T + C0)

a non-relativistic zero-temperature degenerate term plus a classical ideal electron gas
(``R`` = CONST_RGAS, ``C0`` from the thermal de Broglie wavelength).  Every derivative in the
table is exact, so the biquintic Hermite interpolation of the reference reproduces the model to
interpolation accuracy.  The physically faithful table (electron-positron Fermi gas from
Fermi-Dirac integrals) is built by :mod:`phlegethon_b200.helm_fermi`; :func:`make` returns
either, cached per process.
"""
from __future__ import annotations

import math

import numpy as np

# physical constants (source/source.F90:612-629)
CONST_RGAS = 8.31446261815324e7
CONST_AV = 6.02214076e23
CONST_KB = 1.380650424e-16
CONST_H = 6.62606896e-27
M_E = 9.10938356e-28

# table defaults: the "x2" table of tests/hotbubble-helmholtz/Makefile:41-46
X2_TABLE = dict(nrho=541, nT=201, ldlo=-12.0, ldhi=15.0, ltlo=3.0, lthi=13.0)
# module defaults (source/source.F90:191-233)
X1_TABLE = dict(nrho=271, nT=101, ldlo=-12.0, ldhi=15.0, ltlo=3.0, lthi=13.0)


def _model_constants():
    hbar = CONST_H / (2.0 * math.pi)
    # P_deg = K_n n_e^(5/3), n_e = d * N_A  ->  P_deg = K d^(5/3)
    k_n = (3.0 * math.pi ** 2) ** (2.0 / 3.0) * hbar ** 2 / (5.0 * M_E)
    k_d = k_n * CONST_AV ** (5.0 / 3.0)
    kprime = 1.5 * k_d  # f_deg = K' d^(2/3), P = d^2 f' = (2/3) K' d^(5/3) = K d^(5/3)
    # ln(n_e lambda^3 / 2) = ln d + ln(N_A/2) + 3/2 ln(h^2/(2 pi m_e k)) - 3/2 ln T
    c0 = math.log(CONST_AV / 2.0) + 1.5 * math.log(CONST_H ** 2 / (2.0 * math.pi * M_E * CONST_KB)) - 1.0
    return kprime, c0


def nodes(nrho, nT, ldlo, ldhi, ltlo, lthi):
    """Table nodes as load_helm_table builds them (source.F90:23091-23104)."""
    dT = (lthi - ltlo) / float(nT - 1)
    drho = (ldhi - ldlo) / float(nrho - 1)
    T = np.array([10.0 ** (ltlo + float(j) * dT) for j in range(nT)])
    rho = np.array([10.0 ** (ldlo + float(i) * drho) for i in range(nrho)])
    return rho, T, drho, dT


def generate(nrho=X2_TABLE["nrho"], nT=X2_TABLE["nT"], ldlo=X2_TABLE["ldlo"], ldhi=X2_TABLE["ldhi"],
             ltlo=X2_TABLE["ltlo"], lthi=X2_TABLE["lthi"]):
    """Return ``(tab, dpdr)`` with shapes ``(9, nrho, nT)`` and ``(4, nrho, nT)``.

    Both are Fortran-ordered arrays (variable index fastest), i.e. exactly the memory layout
    of ``helm_table_var`` and ``dpdrho_table_var`` (source.F90:558-567), and the variable
    order follows the ``id_*`` indices (source.F90:520-533): f, df/dT, d2f/dT2, df/drho,
    d2f/drho2, d2f/drhodT, d3f/drho2dT, d3f/drhodT2, d4f/drho2dT2 and c, dc/dT, dc/drho,
    d2c/drhodT.
    """
    kp, c0 = _model_constants()
    R = CONST_RGAS
    rho, T, _, _ = nodes(nrho, nT, ldlo, ldhi, ltlo, lthi)
    d = rho[:, None]
    t = T[None, :]
    lnd = np.log(d)
    lnt = np.log(t)
    f = kp * d ** (2.0 / 3.0) + R * t * (lnd - 1.5 * lnt + c0)
    f_d = (2.0 / 3.0) * kp * d ** (-1.0 / 3.0) + R * t / d
    f_t = R * (lnd - 1.5 * lnt + c0) - 1.5 * R + 0.0 * d
    f_dd = -(2.0 / 9.0) * kp * d ** (-4.0 / 3.0) - R * t / d ** 2
    f_tt = -1.5 * R / t + 0.0 * d
    f_dt = R / d + 0.0 * t
    f_ddt = -R / d ** 2 + 0.0 * t
    zero = np.zeros_like(f)
    c = (10.0 / 9.0) * kp * d ** (2.0 / 3.0) + R * t
    c_d = (20.0 / 27.0) * kp * d ** (-1.0 / 3.0) + 0.0 * t
    c_t = R + zero
    c_dt = zero
    tab = np.zeros((9, nrho, nT), order="F")
    for v, arr in enumerate([f, f_t, f_tt, f_d, f_dd, f_dt, f_ddt, zero, zero]):
        tab[v] = arr
    dpdr = np.zeros((4, nrho, nT), order="F")
    for v, arr in enumerate([c, c_t, c_d, c_dt]):
        dpdr[v] = arr
    return np.asfortranarray(tab), np.asfortranarray(dpdr)


def write_text(path, tab, dpdr):
    """Write ``tab``/``dpdr`` in the order ``load_helm_table`` reads them."""
    nv, nrho, nT = tab.shape
    # reading order: f, df/drho, df/dT, d2f/drho2, d2f/dT2, d2f/drhodT, d3f/drho2dT, d3f/drhodT2,
    # d4f/drho2dT2 -> id indices 1,4,2,5,3,6,7,8,9 (1-based)
    order = [0, 3, 1, 4, 2, 5, 6, 7, 8]
    corder = [0, 2, 1, 3]  # c, dc/drho, dc/dT, d2c/drhodT
    with open(path, "w") as fh:
        for j in range(nT):
            for i in range(nrho):
                fh.write(" ".join("%.17e" % tab[v, i, j] for v in order) + "\n")
        for j in range(nT):
            for i in range(nrho):
                fh.write(" ".join("%.17e" % dpdr[v, i, j] for v in corder) + "\n")


def read_text(path, nrho, nT):
    """Inverse of :func:`write_text` (the parse of load_helm_table)."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    a = np.array([[float(x) for x in ln.split()] for ln in lines[: nrho * nT]]).reshape(nT, nrho, 9)
    b = np.array([[float(x) for x in ln.split()] for ln in lines[nrho * nT: 2 * nrho * nT]]).reshape(nT, nrho, 4)
    tab = np.zeros((9, nrho, nT), order="F")
    dpdr = np.zeros((4, nrho, nT), order="F")
    order = [0, 3, 1, 4, 2, 5, 6, 7, 8]
    corder = [0, 2, 1, 3]
    for col, v in enumerate(order):
        tab[v] = a[:, :, col].T
    for col, v in enumerate(corder):
        dpdr[v] = b[:, :, col].T
    return tab, dpdr


_CACHE = {}


def make(model="synthetic", ranges=None, workers=None):
    """``(tab, dpdr)`` of the named electron free-energy model over ``ranges`` (a dict like
    X2_TABLE), computed once per process: "synthetic" (:func:`generate`) or "fermi"
    (:func:`phlegethon_b200.helm_fermi.generate`; ``workers`` > 1 spreads it over that many
    spawned processes, which needs a ``__main__`` guard in the calling script)."""
    r = dict(X2_TABLE if ranges is None else ranges)
    key = (model,) + tuple(sorted(r.items()))
    if key not in _CACHE:
        if model == "synthetic":
            _CACHE[key] = generate(**r)
        elif model == "fermi":
            from . import helm_fermi
            _CACHE[key] = helm_fermi.generate(workers=workers or 1, **r)
        else:
            raise KeyError(model)
    return _CACHE[key]
