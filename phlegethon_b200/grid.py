"""Run-time configuration and host arrays in the reference's layout.

``Config`` carries the reference's compile-time options (``-D`` flags of the test Makefiles,
defaults in ``source/source.F90:31-477``) as run-time fields.  ``HostGrid`` allocates the
subset of ``locgrid`` (``source/source.F90:839-1130``) that the explicit step touches, with the
exact bounds of ``initialize_simulation`` (``source/source.F90:1219-1714``), as Fortran-ordered
numpy arrays: the first index varies fastest and ghost layers are included, so a pointer to
any of them is what the Fortran driver would pass through ISO_C_BINDING.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

RIEMANN = {"lhllc": 0, "hllc": 1, "hlld": 2, "lhlld": 3}
BC = {"periodic": 0, "reflective": 1}

FLAG_MHD = 1 << 0
FLAG_WB = 1 << 1
FLAG_GRAVITY = 1 << 2
FLAG_EVOLVE_ETOT = 1 << 3
FLAG_HELMHOLTZ = 1 << 4
FLAG_FASTEOS = 1 << 5
FLAG_ADVECT_YE_IABAR = 1 << 6
FLAG_SHOCK_FLATTENING = 1 << 7
FLAG_FLUX_IS_ALL_MACH = 1 << 8
FLAG_CONSTANT_ACCELERATION = 1 << 9

PRECISION = {"fp64": 0, "fp32_split": 1}
GUESS = {"warm": 0, "mlp": 1, "bracket": 2, "mlp_rescue": 3}


@dataclass
class Config:
    sdims: int = 2
    nx1: int = 64
    nx2: int = 64
    nx3: int = 1
    ngc: int = 2
    nas: int = 0
    mhd: bool = False
    wb: bool = False
    gravity: bool = False
    etot: bool = False
    helmholtz: bool = False          # HELMHOLTZ_EOS with ADVECT_YE_IABAR
    fasteos: bool = True             # USE_FASTEOS (with helmholtz): gamma_e/gamma_c at the faces
                                     # instead of helm_rhoP_given per Riemann side
    riemann: str = "lhllc"
    rec: str = "lim2nd"              # LIM2ND_REC, PPH_REC or LIM5TH_REC (needs ngc >= 3)
    shock_flattening: bool = False   # USE_SHOCK_FLATTENING (needs ngc >= 3)
    eps_sf: float = 0.25             # eps_sf_make
    all_mach: bool = False           # FLUX_IS_ALL_MACH (LHLLC / LHLLD: upwind states outside the fan)
    constant_acceleration: bool = False  # USE_CONSTANT_ACCELERATION with the vector acc
    acc: tuple = (0.0, 0.0, 0.0)
    rk_stages: int = 3
    bc: list = field(default_factory=lambda: [["periodic", "periodic"]] * 3)
    precision: str = "fp64"
    eos_guess: str = "warm"
    device: int = 0
    x1l: float = 0.0
    x1u: float = 1.0
    x2l: float = 0.0
    x2u: float = 1.0
    x3l: float = 0.0
    x3u: float = 1.0
    gamma_ad: float = 5.0 / 3.0
    mu: float = 1.0
    cfl: float = 0.8
    mach_cutoff: float = 1e-5
    mach_ct: float = 1e-6
    helm_nT: int = 201
    helm_nrho: int = 541
    helm_ltlo: float = 3.0
    helm_lthi: float = 13.0
    helm_ldlo: float = -12.0
    helm_ldhi: float = 15.0

    @property
    def nvars(self) -> int:
        return 2 + self.sdims + self.nas

    @property
    def flags(self) -> int:
        f = 0
        if self.mhd:
            f |= FLAG_MHD
        if self.wb:
            f |= FLAG_WB
        if self.gravity:
            f |= FLAG_GRAVITY
        if self.etot:
            f |= FLAG_EVOLVE_ETOT
        if self.helmholtz:
            f |= FLAG_HELMHOLTZ | FLAG_ADVECT_YE_IABAR
            if self.fasteos:
                f |= FLAG_FASTEOS
        if self.shock_flattening:
            f |= FLAG_SHOCK_FLATTENING
        if self.all_mach:
            f |= FLAG_FLUX_IS_ALL_MACH
        if self.constant_acceleration:
            f |= FLAG_CONSTANT_ACCELERATION
        return f

    @property
    def n_cells(self) -> int:
        return self.nx1 * self.nx2 * self.nx3

    def replace(self, **kw) -> "Config":
        return dataclasses.replace(self, **kw)

    def dx(self):
        # initialize_simulation (source.F90:1717-1735)
        return ((self.x1u - self.x1l) / self.nx1, (self.x2u - self.x2l) / self.nx2,
                (self.x3u - self.x3l) / self.nx3)


def _f(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


class HostGrid:
    """Reference-layout host arrays for one configuration (all float64, Fortran order)."""

    DYNAMIC = ("prim", "temp", "eint", "gammaf", "b_cc", "b_x")

    def __init__(self, cfg: Config):
        self.cfg = cfg
        g, sd = cfg.ngc, cfg.sdims
        g3 = g if sd == 3 else 0
        self.cell_shape = (cfg.nx1 + 2 * g, cfg.nx2 + 2 * g, cfg.nx3 + 2 * g3)
        cs = self.cell_shape
        self.prim = _f((cfg.nvars,) + cs)
        self.temp = _f(cs)
        self.eint = _f(cs)
        self.gammaf = _f((2,) + cs) if cfg.helmholtz else None
        self.grav = _f((sd,) + cs) if cfg.gravity else None
        self.phi_cc = _f(cs) if cfg.etot else None
        self.eq_prim_cc = _f((3,) + cs) if cfg.wb else None
        self.eq_gammae_cc = _f(cs) if (cfg.wb and cfg.helmholtz) else None
        self.b_cc = _f((sd,) + cs) if cfg.mhd else None
        self.phi_x = [None, None, None]
        self.eq_prim_x = [None, None, None]
        self.eq_gammae_x = [None, None, None]
        self.b_x = [None, None, None]
        for d in range(sd):
            fs = self.face_shape(d)
            if cfg.etot:
                self.phi_x[d] = _f(fs)
            if cfg.wb:
                self.eq_prim_x[d] = _f((3,) + fs)
                if cfg.helmholtz:
                    self.eq_gammae_x[d] = _f(fs)
            if cfg.mhd:
                self.b_x[d] = _f(self.bface_shape(d))

    # ------------------------------------------------------------------ shapes
    def face_shape(self, d):
        """x1 faces (lx1:ux1+1, lx2:ux2, lx3:ux3) etc."""
        n = [self.cfg.nx1, self.cfg.nx2, self.cfg.nx3]
        n[d] += 1
        return tuple(n)

    def bface_shape(self, d):
        """b_x1(lx1-1:ux1+2, lx2-1:ux2+1, lx3-1:ux3+1) etc. (2D: lx3:ux3)."""
        c = self.cfg
        n = [c.nx1 + 2, c.nx2 + 2, c.nx3 + 2 if c.sdims == 3 else c.nx3]
        n[d] += 1
        return tuple(n)

    # ------------------------------------------------------------------ views
    def interior(self, a):
        """Interior view of a ghost-padded cell array (leading component axis kept)."""
        c = self.cfg
        g, g3 = c.ngc, (c.ngc if c.sdims == 3 else 0)
        sl = (slice(g, g + c.nx1), slice(g, g + c.nx2), slice(g3, g3 + c.nx3))
        if a.ndim == 4:
            return a[(slice(None),) + sl]
        return a[sl]

    def bface_interior(self, d):
        c = self.cfg
        a = self.b_x[d]
        k0 = 1 if c.sdims == 3 else 0
        n = [c.nx1, c.nx2, c.nx3]
        n[d] += 1
        return a[1:1 + n[0], 1:1 + n[1], k0:k0 + n[2]]

    def coords(self):
        """Cell-centre coordinates of the ghost-padded grid (create_geometry, source.F90:16272-16371)."""
        c = self.cfg
        dx1, dx2, dx3 = c.dx()
        g, g3 = c.ngc, (c.ngc if c.sdims == 3 else 0)
        i = np.arange(1 - g, c.nx1 + g + 1)
        j = np.arange(1 - g, c.nx2 + g + 1)
        k = np.arange(1 - g3, c.nx3 + g3 + 1)
        x = c.x1l + (i - 0.5) * dx1
        y = c.x2l + (j - 0.5) * dx2
        z = c.x3l + (k - 0.5) * dx3
        return np.meshgrid(x, y, z, indexing="ij")

    def face_coords(self, d):
        """Coordinates of x_d faces over the face array's index range."""
        c = self.cfg
        dx1, dx2, dx3 = c.dx()
        n = self.face_shape(d)
        i = np.arange(1, n[0] + 1)
        j = np.arange(1, n[1] + 1)
        k = np.arange(1, n[2] + 1)
        x = c.x1l + (i - (1.0 if d == 0 else 0.5)) * dx1
        y = c.x2l + (j - (1.0 if d == 1 else 0.5)) * dx2
        z = c.x3l + (k - (1.0 if d == 2 else 0.5)) * dx3
        return np.meshgrid(x, y, z, indexing="ij")

    def node_coords(self):
        """Node coordinates over (lx1:ux1+1, lx2:ux2+1, lx3:ux3[+1])."""
        c = self.cfg
        dx1, dx2, dx3 = c.dx()
        i = np.arange(1, c.nx1 + 2)
        j = np.arange(1, c.nx2 + 2)
        k = np.arange(1, c.nx3 + (2 if c.sdims == 3 else 1))
        return np.meshgrid(c.x1l + (i - 1.0) * dx1, c.x2l + (j - 1.0) * dx2, c.x3l + (k - 1.0) * dx3,
                           indexing="ij")

    def copy(self) -> "HostGrid":
        h = HostGrid.__new__(HostGrid)
        h.__dict__.update(self.__dict__)
        for name, v in list(self.__dict__.items()):
            if isinstance(v, np.ndarray):
                setattr(h, name, v.copy(order="F"))
            elif isinstance(v, list):
                setattr(h, name, [a.copy(order="F") if isinstance(a, np.ndarray) else a for a in v])
        return h

    def dynamic_copy(self) -> "HostGrid":
        """A copy that carries only the dynamic state (background members None): what a driver
        passes to phl_upload_state to refresh the state without re-sending the background, and
        what phl_run_steps_host_async exchanges every call."""
        h = self.copy()
        for name in ("grav", "phi_cc", "eq_prim_cc", "eq_gammae_cc"):
            setattr(h, name, None)
        h.phi_x = [None] * 3
        h.eq_prim_x = [None] * 3
        h.eq_gammae_x = [None] * 3
        return h

    def dynamic_arrays(self):
        out = {"prim": self.prim, "temp": self.temp, "eint": self.eint}
        if self.gammaf is not None:
            out["gammaf"] = self.gammaf
        if self.b_cc is not None:
            out["b_cc"] = self.b_cc
            for d in range(self.cfg.sdims):
                out["b_x%d" % (d + 1)] = self.b_x[d]
        return out

    def state_bytes(self) -> int:
        return int(sum(a.nbytes for a in self.dynamic_arrays().values()))


def helm_state_range(h, cfg, margin=0.1):
    """(log10 rho, log10 T, Abar, Zbar) lower and upper bounds of a Helmholtz state with the
    ADVECT_YE_IABAR scalars, the two logarithms widened by ``margin`` dex and the temperatures
    clipped to the table's (the sample range of ``Simulation.set_mlp_sample_range``)."""
    w = h.interior(h.prim)
    ias = 2 + cfg.sdims
    abar = 1.0 / w[ias + 1]
    zbar = w[ias] * abar
    lr, lt = np.log10(w[0]), np.log10(h.interior(h.temp))
    lo = [float(lr.min()) - margin, max(float(lt.min()) - margin, float(cfg.helm_ltlo)), float(abar.min()),
          float(zbar.min())]
    hi = [float(lr.max()) + margin, min(float(lt.max()) + margin, float(cfg.helm_lthi)), float(abar.max()),
          float(zbar.max())]
    return lo, hi
