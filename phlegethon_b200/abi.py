"""ctypes binding of ``include/phl_gpu.h`` and the ``Simulation`` host mirror.

``Simulation`` exposes the reference's call sites with the reference's names:

* ``init_thermo()``              step-0 thermodynamics of ``time_loop`` (source.F90:6271-6383)
* ``compute_hyperbolic_dt()``    ``compute_hyperbolic_dt`` (source.F90:13707-13960)
* ``hydro_step()``               ``hydro_step`` (source.F90:6847-13701)
* ``time_loop(nsteps, tmax)``    the output-free body of ``time_loop`` (source.F90:6525-6748)

The library is the in-tree ``_lib/libphl_b200.so``; there is no CPU fallback: loading fails
loudly when it is missing or when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .grid import BC, GUESS, PRECISION, RIEMANN, Config, HostGrid

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libphl_b200.so")
ABI_VERSION = 4

PHL_OK = 0
ERRORS = {-1: "PHL_E_INVALID", -2: "PHL_E_CUDA", -3: "PHL_E_NO_TABLE", -4: "PHL_E_STATE",
          -5: "PHL_E_NO_DEVICE", -6: "PHL_E_UNSUPPORTED", -7: "PHL_E_TOO_LARGE"}

# names of every exported entry point declared in include/phl_gpu.h
EXPORTS = [
    "phl_abi_version", "phl_error_string", "phl_init", "phl_finalize", "phl_load_helm_table",
    "phl_upload_state", "phl_download_state", "phl_init_thermo", "phl_compute_hyperbolic_dt",
    "phl_hydro_step", "phl_set_time", "phl_get_time", "phl_run_steps", "phl_get_status",
    "phl_reset_status", "phl_eos_invert_batch_device", "phl_eos_invert_batch",
    "phl_eos_energy_device", "phl_mlp_train", "phl_mlp_get_params", "phl_mlp_set_params",
    "phl_mlp_infer_device", "phl_mlp_gradient", "phl_device_field", "phl_stream", "phl_eos_invert_batch_noalloc",
    "phl_mlp_set_sample_range", "phl_run_steps_host_async", "phl_wait_host",
]


class PhlConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int), ("sdims", C.c_int), ("nx1", C.c_int), ("nx2", C.c_int),
        ("nx3", C.c_int), ("ngc", C.c_int), ("nas", C.c_int), ("nvars", C.c_int),
        ("flags", C.c_int), ("riemann", C.c_int), ("rk_stages", C.c_int),
        ("bc", (C.c_int * 2) * 3), ("precision", C.c_int), ("eos_guess", C.c_int),
        ("device", C.c_int),
        ("x1l", C.c_double), ("x1u", C.c_double), ("x2l", C.c_double), ("x2u", C.c_double),
        ("x3l", C.c_double), ("x3u", C.c_double), ("gamma_ad", C.c_double), ("mu", C.c_double),
        ("cfl", C.c_double), ("mach_cutoff", C.c_double), ("mach_ct", C.c_double),
        ("helm_nT", C.c_int), ("helm_nrho", C.c_int), ("helm_ltlo", C.c_double),
        ("helm_lthi", C.c_double), ("helm_ldlo", C.c_double), ("helm_ldhi", C.c_double),
        ("reconstruction", C.c_int), ("eps_sf", C.c_double), ("acc", C.c_double * 3),
    ]


_P = C.POINTER(C.c_double)


class PhlFields(C.Structure):
    _fields_ = [
        ("prim", _P), ("temp", _P), ("eint", _P), ("gammaf", _P), ("grav", _P), ("phi_cc", _P),
        ("eq_prim_cc", _P), ("eq_gammae_cc", _P), ("b_cc", _P), ("phi_x", _P * 3),
        ("eq_prim_x", _P * 3), ("eq_gammae_x", _P * 3), ("b_x", _P * 3),
    ]


class PhlStatus(C.Structure):
    _fields_ = [
        ("newton_calls", C.c_longlong), ("newton_iterations", C.c_longlong),
        ("newton_nonconverged", C.c_longlong), ("newton_clamped", C.c_longlong),
        ("mlp_accepted", C.c_longlong), ("mlp_rejected", C.c_longlong),
        ("nonfinite", C.c_longlong), ("guess_evaluations", C.c_longlong),
        ("tensor_core_stalls", C.c_longlong), ("steps", C.c_longlong),
        ("time", C.c_double),
        ("dt", C.c_double), ("smax", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("phlegethon_b200 CUDA library not built: %s (run __graft_entry__.build())" % path)
    try:
        from .build import _sources_newer
        if _sources_newer(path):
            import warnings
            warnings.warn("phlegethon_b200: CUDA sources are newer than %s; rebuild with "
                          "__graft_entry__.build()" % path, RuntimeWarning)
    except Exception:
        pass
    lib = C.CDLL(path)
    vp = C.c_void_p
    sig = {
        "phl_abi_version": ([], C.c_int),
        "phl_error_string": ([C.c_int], C.c_char_p),
        "phl_init": ([C.POINTER(PhlConfig), C.POINTER(vp)], C.c_int),
        "phl_finalize": ([vp], None),
        "phl_load_helm_table": ([vp, _P, _P], C.c_int),
        "phl_upload_state": ([vp, C.POINTER(PhlFields)], C.c_int),
        "phl_download_state": ([vp, C.POINTER(PhlFields)], C.c_int),
        "phl_init_thermo": ([vp], C.c_int),
        "phl_compute_hyperbolic_dt": ([vp, _P, _P], C.c_int),
        "phl_hydro_step": ([vp], C.c_int),
        "phl_set_time": ([vp, C.c_double, C.c_double, C.c_double], C.c_int),
        "phl_get_time": ([vp, _P, _P, _P], C.c_int),
        "phl_run_steps": ([vp, C.c_int, C.c_double, C.POINTER(C.c_int), _P], C.c_int),
        "phl_run_steps_host_async": ([vp, C.POINTER(PhlFields), C.c_int], C.c_int),
        "phl_wait_host": ([vp], C.c_int),
        "phl_get_status": ([vp, C.POINTER(PhlStatus)], C.c_int),
        "phl_reset_status": ([vp], C.c_int),
        "phl_eos_invert_batch_device": ([vp, C.c_longlong, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int], C.c_int),
        "phl_eos_invert_batch": ([vp, C.c_longlong, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int], C.c_int),
        "phl_eos_invert_batch_noalloc": ([vp, C.c_longlong, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int], C.c_int),
        "phl_eos_energy_device": ([vp, C.c_longlong, vp, vp, vp, vp, vp], C.c_int),
        "phl_mlp_train": ([vp, C.c_longlong, C.c_ulonglong, C.c_int, C.c_int, C.c_double, _P], C.c_int),
        "phl_mlp_get_params": ([vp, C.POINTER(C.c_float)], C.c_int),
        "phl_mlp_set_params": ([vp, C.POINTER(C.c_float)], C.c_int),
        "phl_mlp_infer_device": ([vp, C.c_longlong, vp, vp], C.c_int),
        "phl_mlp_gradient": ([vp, C.c_longlong, vp, vp, vp, _P], C.c_int),
        "phl_mlp_set_sample_range": ([vp, _P, _P], C.c_int),
        "phl_device_field": ([vp, C.c_char_p], vp),
        "phl_stream": ([vp], vp),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.phl_abi_version() != ABI_VERSION:
        raise RuntimeError("ABI version mismatch")
    _lib = lib
    return lib


class PhlError(RuntimeError):
    def __init__(self, code, where):
        lib = _lib
        msg = lib.phl_error_string(code).decode() if lib is not None else ERRORS.get(code, str(code))
        super().__init__("%s failed: %s (%s)" % (where, ERRORS.get(code, code), msg))
        self.code = code


def _check(rc, where):
    if rc != PHL_OK:
        raise PhlError(rc, where)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags["F_CONTIGUOUS"] or a.ndim <= 1), "reference-layout float64 array"
    return a.ctypes.data_as(_P)


def make_config_struct(cfg: Config) -> PhlConfig:
    s = PhlConfig()
    s.abi_version = ABI_VERSION
    s.sdims, s.nx1, s.nx2, s.nx3 = cfg.sdims, cfg.nx1, cfg.nx2, cfg.nx3
    s.ngc, s.nas, s.nvars = cfg.ngc, cfg.nas, cfg.nvars
    s.flags = cfg.flags
    s.riemann = RIEMANN[cfg.riemann]
    s.rk_stages = cfg.rk_stages
    for d in range(3):
        for side in range(2):
            s.bc[d][side] = BC[cfg.bc[d][side]]
    s.precision = PRECISION[cfg.precision]
    s.eos_guess = GUESS[cfg.eos_guess]
    s.reconstruction = {"lim2nd": 0, "pph": 1, "lim5th": 2}[cfg.rec]
    s.eps_sf = float(cfg.eps_sf)
    for d in range(3):
        s.acc[d] = float(cfg.acc[d])
    s.device = cfg.device
    for k in ("x1l", "x1u", "x2l", "x2u", "x3l", "x3u", "gamma_ad", "mu", "cfl", "mach_cutoff",
              "mach_ct", "helm_ltlo", "helm_lthi", "helm_ldlo", "helm_ldhi"):
        setattr(s, k, float(getattr(cfg, k)))
    s.helm_nT, s.helm_nrho = cfg.helm_nT, cfg.helm_nrho
    return s


def fields_struct(h: HostGrid) -> PhlFields:
    f = PhlFields()
    for name in ("prim", "temp", "eint", "gammaf", "grav", "phi_cc", "eq_prim_cc", "eq_gammae_cc", "b_cc"):
        setattr(f, name, _ptr(getattr(h, name)))
    for name in ("phi_x", "eq_prim_x", "eq_gammae_x", "b_x"):
        arr = getattr(f, name)
        for d in range(3):
            a = getattr(h, name)[d]
            arr[d] = _ptr(a) if a is not None else _P()
    return f


class Simulation:
    """A device-resident domain driven through the C ABI."""

    def __init__(self, cfg: Config, table=None):
        self.lib = load_library()
        self.cfg = cfg
        self._cs = make_config_struct(cfg)
        self.ctx = C.c_void_p()
        _check(self.lib.phl_init(C.byref(self._cs), C.byref(self.ctx)), "phl_init")
        if cfg.helmholtz:
            if table is None:
                raise ValueError("Helmholtz configuration needs a table (tab, dpdr)")
            self.load_helm_table(*table)

    def close(self):
        if self.ctx:
            self.lib.phl_finalize(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------- reference call sites
    def load_helm_table(self, tab, dpdr):
        tab = np.asfortranarray(tab, dtype=np.float64)
        dpdr = np.asfortranarray(dpdr, dtype=np.float64)
        _check(self.lib.phl_load_helm_table(self.ctx, _ptr(tab), _ptr(dpdr)), "phl_load_helm_table")

    def upload(self, h: HostGrid):
        self._fields = fields_struct(h)
        _check(self.lib.phl_upload_state(self.ctx, C.byref(self._fields)), "phl_upload_state")

    def download(self, h: HostGrid):
        f = fields_struct(h)
        _check(self.lib.phl_download_state(self.ctx, C.byref(f)), "phl_download_state")

    def init_thermo(self):
        _check(self.lib.phl_init_thermo(self.ctx), "phl_init_thermo")

    def compute_hyperbolic_dt(self):
        dt, smax = C.c_double(), C.c_double()
        _check(self.lib.phl_compute_hyperbolic_dt(self.ctx, C.byref(dt), C.byref(smax)), "phl_compute_hyperbolic_dt")
        return dt.value, smax.value

    def hydro_step(self):
        _check(self.lib.phl_hydro_step(self.ctx), "phl_hydro_step")

    def set_time(self, time, dt, smax):
        _check(self.lib.phl_set_time(self.ctx, time, dt, smax), "phl_set_time")

    def get_time(self):
        t, dt, smax = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.phl_get_time(self.ctx, C.byref(t), C.byref(dt), C.byref(smax)), "phl_get_time")
        return t.value, dt.value, smax.value

    def set_mlp_sample_range(self, lo=None, hi=None):
        """Range the learned guess is trained on: lo/hi = (log10 rho, log10 T, Abar, Zbar);
        None restores the default (the EoS benchmark range)."""
        if lo is None:
            rc = self.lib.phl_mlp_set_sample_range(self.ctx, None, None)
        else:
            rc = self.lib.phl_mlp_set_sample_range(self.ctx, (C.c_double * 4)(*lo), (C.c_double * 4)(*hi))
        _check(rc, "phl_mlp_set_sample_range")

    def time_loop(self, nsteps, tmax=float("inf")):
        done, t = C.c_int(), C.c_double()
        _check(self.lib.phl_run_steps(self.ctx, int(nsteps), float(tmax), C.byref(done), C.byref(t)), "phl_run_steps")
        return done.value, t.value

    def time_loop_host_async(self, h: HostGrid, nsteps=1):
        """Queue upload of h's dynamic state, `nsteps` steps and the download back into h
        (phl_run_steps_host_async); h must stay alive and untouched until wait_host()."""
        f = fields_struct(h)
        _check(self.lib.phl_run_steps_host_async(self.ctx, C.byref(f), int(nsteps)), "phl_run_steps_host_async")

    def wait_host(self):
        _check(self.lib.phl_wait_host(self.ctx), "phl_wait_host")

    def status(self):
        st = PhlStatus()
        _check(self.lib.phl_get_status(self.ctx, C.byref(st)), "phl_get_status")
        return st.as_dict()

    def reset_status(self):
        _check(self.lib.phl_reset_status(self.ctx), "phl_reset_status")

    def device_field(self, name):
        return self.lib.phl_device_field(self.ctx, name.encode())

    def stream(self):
        return self.lib.phl_stream(self.ctx)
