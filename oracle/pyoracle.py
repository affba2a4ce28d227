"""ctypes driver of the CPU oracle (oracle/_build/libphl_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker and by bench.py's cpu_baseline / the
reference arm as the timed CPU restatement.  Parity status: unpinned against an execution of
the reference itself (no Fortran toolchain in this environment); see phl_oracle.h.

The oracle works in place on a ``phlegethon_b200.grid.HostGrid``: the same reference-layout
arrays that the C ABI uploads.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libphl_oracle.so")
_P = C.POINTER(C.c_double)


class _Helm(C.Structure):
    _fields_ = [("nT", C.c_int), ("nrho", C.c_int), ("ltlo", C.c_double), ("lthi", C.c_double),
                ("ldlo", C.c_double), ("ldhi", C.c_double), ("drho", C.c_double), ("dT", C.c_double),
                ("tab", _P), ("dpdr", _P), ("rho", _P), ("T", _P), ("Tl", C.c_double), ("Th", C.c_double)]


class _Grid(C.Structure):
    _fields_ = [
        ("sdims", C.c_int), ("nx1", C.c_int), ("nx2", C.c_int), ("nx3", C.c_int), ("ngc", C.c_int),
        ("nas", C.c_int), ("nvars", C.c_int), ("mhd", C.c_int), ("wb", C.c_int), ("gravity", C.c_int),
        ("etot", C.c_int), ("helm", C.c_int), ("fasteos", C.c_int), ("rec", C.c_int), ("sf", C.c_int),
        ("all_mach", C.c_int), ("use_acc", C.c_int), ("acc", C.c_double * 3),
        ("riemann", C.c_int), ("rk_stages", C.c_int), ("bc", (C.c_int * 2) * 3), ("gm", C.c_double), ("mu", C.c_double),
        ("cfl", C.c_double), ("mach_cutoff", C.c_double), ("mach_ct", C.c_double), ("eps_sf", C.c_double),
        ("dx1", C.c_double),
        ("dx2", C.c_double), ("dx3", C.c_double), ("inv_dx1", C.c_double), ("inv_dx2", C.c_double),
        ("inv_dx3", C.c_double), ("dt", C.c_double), ("smax", C.c_double), ("time", C.c_double),
        ("eos", C.POINTER(_Helm)), ("nthreads", C.c_int),
        ("prim", _P), ("temp", _P), ("eint", _P), ("gammaf", _P), ("grav", _P), ("phi_cc", _P),
        ("eq_prim_cc", _P), ("eq_gammae_cc", _P), ("b_cc", _P), ("phi_x", _P * 3), ("eq_prim_x", _P * 3),
        ("eq_gammae_x", _P * 3), ("b_x", _P * 3), ("scratch", _P),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        for n in ("phlo_hydro_step", "phlo_compute_hyperbolic_dt", "phlo_init_thermo", "phlo_helm_setup_nodes"):
            getattr(lib, n).restype = None
        lib.phlo_helm_rhoT_given_full.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double,
                                                  C.c_double, _P, _P, _P, _P]
        lib.phlo_helm_rhoT_given_full.restype = None
        lib.phlo_helm_rhoT_given2.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double,
                                              C.c_double, _P, _P, C.c_int]
        lib.phlo_helm_rhoT_given2.restype = None
        lib.phlo_helm_rhoT_given1.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double,
                                              C.c_double, _P, _P, C.c_int]
        lib.phlo_helm_rhoT_given1.restype = None
        lib.phlo_helm_rhoe_given.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double,
                                             C.c_double, _P, _P, _P, C.c_int]
        lib.phlo_helm_rhoe_given.restype = C.c_int
        lib.phlo_face_newton_stats.argtypes = [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.c_int]
        lib.phlo_face_newton_stats.restype = None
        lib.phlo_helm_rhoP_given.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double,
                                             C.c_double, _P, _P, _P, C.c_int]
        lib.phlo_helm_rhoP_given.restype = C.c_int
        lib.phlo_eos_invert_batch.argtypes = [C.POINTER(_Helm), C.c_long, _P, _P, _P, _P, _P,
                                              C.POINTER(C.c_int), C.c_int, C.c_int]
        lib.phlo_eos_invert_batch.restype = None
        lib.phlo_eos_bracket_guess.argtypes = [C.POINTER(_Helm), C.c_double, C.c_double, C.c_double, C.c_double,
                                               _P]
        lib.phlo_eos_bracket_guess.restype = C.c_int
        lib.phlo_riemann_hydro.argtypes = [C.POINTER(_Grid), _P, _P, _P, _P, _P, C.c_int]
        lib.phlo_riemann_hydro.restype = None
        lib.phlo_riemann_mhd.argtypes = [C.POINTER(_Grid), _P, _P, _P, _P, _P, _P, _P, _P, C.c_int]
        lib.phlo_riemann_mhd.restype = None
        _lib = lib
    return _lib


def _p(a):
    if a is None:
        return _P()
    assert a.dtype == np.float64
    return a.ctypes.data_as(_P)


class Helm:
    """Oracle-side Helmholtz table (load_helm_table)."""

    def __init__(self, tab, dpdr, nT, nrho, ltlo, lthi, ldlo, ldhi):
        lib = load()
        self.tab = np.asfortranarray(tab, dtype=np.float64)
        self.dpdr = np.asfortranarray(dpdr, dtype=np.float64)
        self.rho = np.zeros(nrho)
        self.T = np.zeros(nT)
        h = _Helm()
        h.nT, h.nrho, h.ltlo, h.lthi, h.ldlo, h.ldhi = nT, nrho, ltlo, lthi, ldlo, ldhi
        h.tab, h.dpdr, h.rho, h.T = _p(self.tab), _p(self.dpdr), _p(self.rho), _p(self.T)
        lib.phlo_helm_setup_nodes(C.byref(h))
        self.s = h

    @classmethod
    def for_config(cls, cfg, tab, dpdr):
        return cls(tab, dpdr, cfg.helm_nT, cfg.helm_nrho, cfg.helm_ltlo, cfg.helm_lthi, cfg.helm_ldlo, cfg.helm_ldhi)

    def given_full(self, rho, T, abar, zbar):
        P, E, s, cv = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        load().phlo_helm_rhoT_given_full(C.byref(self.s), rho, T, abar, zbar, C.byref(P), C.byref(E),
                                         C.byref(s), C.byref(cv))
        return P.value, E.value, s.value, cv.value

    def given2(self, rho, T, abar, zbar, deriv=True):
        E, dE = C.c_double(), C.c_double()
        load().phlo_helm_rhoT_given2(C.byref(self.s), rho, T, abar, zbar, C.byref(E), C.byref(dE), int(deriv))
        return E.value, dE.value

    def given1(self, rho, T, abar, zbar, deriv=True):
        P, dP = C.c_double(), C.c_double()
        load().phlo_helm_rhoT_given1(C.byref(self.s), rho, T, abar, zbar, C.byref(P), C.byref(dP), int(deriv))
        return P.value, dP.value

    def rhoe_given(self, rho, E0, abar, zbar, T0):
        T, P, s = C.c_double(T0), C.c_double(), C.c_double()
        it = load().phlo_helm_rhoe_given(C.byref(self.s), rho, E0, abar, zbar, C.byref(T), C.byref(P), C.byref(s), 1)
        return T.value, P.value, s.value, it

    def invert_batch(self, rho, e, abar, zbar, T0=None, guess=2, nthreads=0):
        """(rho, e) -> T for arrays of samples; guess 2 = bracket guess, 0 = warm start T0."""
        n = len(rho)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, e, abar, zbar)]
        T = np.zeros(n) if T0 is None else np.array(T0, dtype=np.float64)
        it = np.zeros(n, dtype=np.int32)
        load().phlo_eos_invert_batch(C.byref(self.s), n, *[a.ctypes.data_as(_P) for a in arrs],
                                     T.ctypes.data_as(_P), it.ctypes.data_as(C.POINTER(C.c_int)), guess, nthreads)
        return T, it

    def rhoP_given(self, rho, P0, abar, zbar, T0):
        T, E, s = C.c_double(T0), C.c_double(), C.c_double()
        it = load().phlo_helm_rhoP_given(C.byref(self.s), rho, P0, abar, zbar, C.byref(T), C.byref(E), C.byref(s), 1)
        return T.value, E.value, s.value, it


def face_newton_stats(reset=False):
    """(calls, iterations) of the per-face helm_rhoP_given solves since the last reset."""
    calls, iters = C.c_longlong(), C.c_longlong()
    load().phlo_face_newton_stats(C.byref(calls), C.byref(iters), int(reset))
    return calls.value, iters.value


class OracleGrid:
    """Runs the oracle on a HostGrid in place."""

    RIEM = {"lhllc": 0, "hllc": 1, "hlld": 2, "lhlld": 3}
    BCS = {"periodic": 0, "reflective": 1}

    def __init__(self, h, helm: Helm | None = None, nthreads: int = 0):
        self.lib = load()
        self.h = h
        self.helm = helm
        c = h.cfg
        g = _Grid()
        g.sdims, g.nx1, g.nx2, g.nx3, g.ngc, g.nas, g.nvars = c.sdims, c.nx1, c.nx2, c.nx3, c.ngc, c.nas, c.nvars
        g.mhd, g.wb, g.gravity, g.etot = int(c.mhd), int(c.wb), int(c.gravity), int(c.etot)
        g.helm = int(c.helmholtz)
        g.fasteos = int(c.helmholtz and c.fasteos)
        g.rec = {"lim2nd": 0, "pph": 1, "lim5th": 2}[c.rec]
        g.sf = int(c.shock_flattening)
        g.all_mach = int(c.all_mach)
        g.use_acc = int(c.constant_acceleration)
        for d in range(3):
            g.acc[d] = float(c.acc[d]) if c.constant_acceleration else 0.0
        g.eps_sf = c.eps_sf
        if c.shock_flattening and c.ngc < 3:
            raise ValueError("USE_SHOCK_FLATTENING reads 3 ghost layers: ngc >= 3")
        g.riemann = self.RIEM[c.riemann]
        g.rk_stages = c.rk_stages
        for d in range(3):
            for s in range(2):
                g.bc[d][s] = self.BCS[c.bc[d][s]]
        g.gm, g.mu, g.cfl, g.mach_cutoff, g.mach_ct = c.gamma_ad, c.mu, c.cfl, c.mach_cutoff, c.mach_ct
        dx1, dx2, dx3 = c.dx()
        g.dx1, g.dx2, g.dx3 = dx1, dx2, dx3
        g.inv_dx1, g.inv_dx2 = 1.0 / dx1, 1.0 / dx2
        g.inv_dx3 = 1.0 / dx3 if c.sdims == 3 else 0.0
        if helm is not None:
            g.eos = C.pointer(helm.s)
        g.nthreads = nthreads
        for n in ("prim", "temp", "eint", "gammaf", "grav", "phi_cc", "eq_prim_cc", "eq_gammae_cc", "b_cc"):
            setattr(g, n, _p(getattr(h, n)))
        for n in ("phi_x", "eq_prim_x", "eq_gammae_x", "b_x"):
            arr = getattr(g, n)
            for d in range(3):
                arr[d] = _p(getattr(h, n)[d])
        self.g = g

    def init_thermo(self):
        self.lib.phlo_init_thermo(C.byref(self.g))

    def compute_hyperbolic_dt(self):
        self.lib.phlo_compute_hyperbolic_dt(C.byref(self.g))
        return self.g.dt, self.g.smax

    def hydro_step(self):
        self.lib.phlo_hydro_step(C.byref(self.g))

    def time_loop(self, nsteps, tmax=float("inf")):
        """time_loop body without output (source.F90:6525-6748); returns steps taken."""
        n = 0
        while n < nsteps and self.g.time < tmax:
            if self.g.time + self.g.dt > tmax:
                self.g.dt = tmax - self.g.time
            self.hydro_step()
            self.g.time = self.g.time + self.g.dt
            self.compute_hyperbolic_dt()
            n += 1
        return n

    def free(self):
        if self.g.scratch:
            C.CDLL(None)  # noqa: keep libc reachable
            libc = C.CDLL("libc.so.6")
            libc.free(C.cast(self.g.scratch, C.c_void_p))
            self.g.scratch = _P()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
