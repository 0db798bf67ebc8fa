"""ctypes wrappers for the CPU test oracles (TEST INFRASTRUCTURE ONLY).

* :class:`Oracle` -- the project's C restatement (``oracle/liboracle_o{ord}.so``).
* :class:`OracleLD` -- the same restatement in x87 long double
  (``oracle/liboracle_o5_ld.so``): a finite-difference reference for the adjoint.
* :class:`RefHarness` -- the reference's own code built on project-written stand-ins
  (``oracle/_ref/libawflref_o{ord}.so``, only where it has been built).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p
_I = ctypes.c_int

DATA_SPECS = {"thermal": 1, "collision": 2, "straka": 3, "igw": 4}
NGLL_OF = {5: 3, 9: 5}


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def build(ref: bool = False, ref_dir: str | None = None) -> None:
    """Build the oracle libraries (and, with ``ref``, the reference harness from the
    reference's source tree ``ref_dir``, default $AWFL_REFERENCE_DIR) via make."""
    targets = ["oracle"] + (["ref"] if ref else [])
    extra = []
    if ref:
        ref_dir = ref_dir or os.environ.get("AWFL_REFERENCE_DIR")
        if not ref_dir:
            raise RuntimeError("the reference's source tree is needed: set AWFL_REFERENCE_DIR")
        extra = ["REF=" + ref_dir]
    subprocess.run(["make", "-s", "-C", HERE] + targets + extra, check=True)


def oracle_path(ord_: int, crpow: bool = False) -> str:
    return os.path.join(HERE, "liboracle_o%d%s.so" % (ord_, "_crpow" if crpow else ""))


def ref_path(ord_: int, crpow: bool = False, tracers: bool = False) -> str:
    return os.path.join(HERE, "_ref", "libawflref_%so%d%s.so" % ("trc_" if tracers else "", ord_,
                                                                 "_crpow" if crpow else ""))


def ref_available(ord_: int = 5, crpow: bool = False, tracers: bool = False) -> bool:
    return os.path.exists(ref_path(ord_, crpow, tracers))


class _Grid:
    def __init__(self, ord_, nx, ny, nz):
        self.ord = ord_
        self.ngll = NGLL_OF[ord_]
        self.hs = (ord_ - 1) // 2
        self.nx, self.ny, self.nz = nx, ny, nz

    @property
    def state_shape(self):
        h = 2 * self.hs
        return (5, self.nz + h, self.ny + h, self.nx + h)

    @property
    def tend_shape(self):
        return (5, self.nz, self.ny, self.nx)

    def new_state(self):
        return np.zeros(self.state_shape, dtype=np.float64)

    def interior(self, st):
        h = self.hs
        return st[:, h:h + self.nz, h:h + self.ny, h:h + self.nx]


class Oracle(_Grid):
    """The project's C restatement of the path."""

    _libs: dict = {}

    @classmethod
    def lib(cls, ord_, crpow=False):
        key = (ord_, crpow)
        if key not in cls._libs:
            path = oracle_path(ord_, crpow)
            if not os.path.exists(path):
                build()
            L = ctypes.CDLL(path)
            L.oracle_create.restype = _VP
            L.oracle_create.argtypes = [_I] * 3 + [_D] * 3 + [_I] * 6
            L.oracle_destroy.argtypes = [_VP]
            L.oracle_state_size.restype = ctypes.c_long
            L.oracle_state_size.argtypes = [_VP]
            L.oracle_init_state.argtypes = [_VP, _DP]
            L.oracle_set_bubble.argtypes = [_VP, _DP, _I] + [_D] * 8
            L.oracle_add_theta_noise.argtypes = [_VP, _DP, ctypes.c_ulonglong, _D]
            L.oracle_init_tracers.argtypes = [_VP, _DP, _I]
            L.oracle_time_step_tracers.argtypes = [_VP, _DP, _DP, _I, ctypes.POINTER(_I), _D]
            L.oracle_split_tracers.argtypes = [_VP, _DP, _DP, _I, ctypes.POINTER(_I), _D, _I]
            L.oracle_limiter_chained_faces.restype = ctypes.c_long
            L.oracle_limiter_chained_faces.argtypes = [_VP]
            L.oracle_set_spacing.argtypes = [_VP, _D, _D, _D]
            L.oracle_compute_dt.restype = _D
            L.oracle_compute_dt.argtypes = [_VP, _DP, _D]
            L.oracle_compute_tendencies_dir.argtypes = [_VP, _DP, _DP, _D, _I]
            L.oracle_compute_tendencies.argtypes = [_VP, _DP, _DP, _D, _I]
            L.oracle_apply.argtypes = [_VP, _DP, _DP, _D]
            L.oracle_time_step.argtypes = [_VP, _DP, _D]
            L.oracle_get_dimswitch.restype = _I
            L.oracle_get_dimswitch.argtypes = [_VP]
            L.oracle_set_dimswitch.argtypes = [_VP, _I]
            L.oracle_get_tables.argtypes = [_VP, _DP, _DP, _DP, _DP]
            L.oracle_get_background.argtypes = [_VP] + [_DP] * 8
            L.oracle_coefs_to_tv.restype = _D
            L.oracle_coefs_to_tv.argtypes = [_DP, _I]
            L.oracle_weno_coefs.argtypes = [_VP, _DP, _DP]
            cls._libs[key] = L
        return cls._libs[key]

    def __init__(self, nx, ny, nz, xlen=20000.0, ylen=20000.0, zlen=10000.0, bc=(0, 0, 1),
                 weno_scalars=True, weno_winds=True, data="thermal", ord_=5, crpow=False):
        """crpow: the variant with correctly rounded pow/exp in place of glibc's."""
        super().__init__(ord_, nx, ny, nz)
        self.L = self.lib(ord_, crpow)
        self.h = self.L.oracle_create(nx, ny, nz, xlen, ylen, zlen, bc[0], bc[1], bc[2],
                                      int(weno_scalars), int(weno_winds), DATA_SPECS[data])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def init_state(self, st):
        self.L.oracle_init_state(self.h, _ptr(st))

    def set_bubble(self, st, shape, x0, y0, z0, xrad, yrad, zrad, amp, pwr=1.0):
        self.L.oracle_set_bubble(self.h, _ptr(st), shape, x0, y0, z0, xrad, yrad, zrad, amp, pwr)

    def add_theta_noise(self, st, seed, amp):
        self.L.oracle_add_theta_noise(self.h, _ptr(st), seed, amp)

    def new_tracers(self, ntr):
        hs = self.hs
        return np.zeros((ntr, self.nz + 2 * hs, self.ny + 2 * hs, self.nx + 2 * hs))

    def init_tracers(self, tr):
        """Spatial::initTracers on tr (ntr, nz+2hs, ny+2hs, nx+2hs)."""
        self.L.oracle_init_tracers(self.h, _ptr(tr), tr.shape[0])

    def time_step_tracers(self, st, tr, dt, pos=None):
        """One step of state and tracers with the reference's tracer code compiled in."""
        n = tr.shape[0]
        pos = [1] * n if pos is None else pos
        flags = (_I * max(n, 1))(*[int(bool(p)) for p in pos])
        self.L.oracle_time_step_tracers(self.h, _ptr(st), _ptr(tr), n, flags, dt)

    def set_spacing(self, dx, dy, dz):
        self.L.oracle_set_spacing(self.h, dx, dy, dz)

    def split_tracers(self, st, tr, dt, d, pos=None):
        """One split (direction d) of state and tracers with the tracer code compiled in."""
        n = tr.shape[0]
        pos = [1] * n if pos is None else pos
        flags = (_I * max(n, 1))(*[int(bool(p)) for p in pos])
        self.L.oracle_split_tracers(self.h, _ptr(st), _ptr(tr), n, flags, dt, d)

    def limiter_chained_faces(self):
        """Faces of the last tracer split whose limited flux depends on the serial order
        (differs from the value with every face read unscaled)."""
        return self.L.oracle_limiter_chained_faces(self.h)

    def compute_dt(self, st, cfl=0.8):
        return self.L.oracle_compute_dt(self.h, _ptr(st), cfl)

    def compute_tendencies_dir(self, st, tend, dt, d):
        self.L.oracle_compute_tendencies_dir(self.h, _ptr(st), _ptr(tend), dt, d)

    def compute_tendencies(self, st, tend, dt, split):
        self.L.oracle_compute_tendencies(self.h, _ptr(st), _ptr(tend), dt, split)

    def apply(self, st, tend, dt):
        self.L.oracle_apply(self.h, _ptr(st), _ptr(tend), dt)

    def time_step(self, st, dt):
        self.L.oracle_time_step(self.h, _ptr(st), dt)

    @property
    def dimswitch(self):
        return self.L.oracle_get_dimswitch(self.h)

    @dimswitch.setter
    def dimswitch(self, v):
        self.L.oracle_set_dimswitch(self.h, int(v))

    def tables(self):
        o, g, hs = self.ord, self.ngll, self.hs
        s2g = np.zeros(o * g); der = np.zeros(g * g); idl = np.zeros(hs + 2); sig = np.zeros(1)
        self.L.oracle_get_tables(self.h, _ptr(s2g), _ptr(der), _ptr(idl), _ptr(sig))
        return {"sten_to_gll": s2g, "deriv": der, "idl": idl, "sigma": sig}

    def background(self):
        nzc = self.nz + 2 * self.hs
        arrs = [np.zeros(nzc) for _ in range(4)] + [np.zeros(self.nz * self.ngll) for _ in range(4)]
        self.L.oracle_get_background(self.h, *[_ptr(a) for a in arrs])
        names = ["hyDensCells", "hyPressureCells", "hyThetaCells", "hyDensThetaCells",
                 "hyDensGLL", "hyPressureGLL", "hyThetaGLL", "hyDensThetaGLL"]
        return dict(zip(names, arrs))

    def coefs_to_tv(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.L.oracle_coefs_to_tv(_ptr(a), len(a))

    def weno_coefs(self, stencil):
        s = np.ascontiguousarray(stencil, dtype=np.float64)
        out = np.zeros(self.ord)
        self.L.oracle_weno_coefs(self.h, _ptr(s), _ptr(out))
        return out


class OracleLD(_Grid):
    """The C restatement compiled with ``oreal = long double`` (ord 5): states are numpy
    ``longdouble`` arrays (80-bit x87 values in 16-byte slots, the C ``long double``)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = os.path.join(HERE, "liboracle_o5_ld.so")
            if not os.path.exists(path):
                build()
            L = ctypes.CDLL(path)
            LD = ctypes.c_longdouble
            L.oracle_create.restype = _VP
            L.oracle_create.argtypes = [_I] * 3 + [LD] * 3 + [_I] * 6
            L.oracle_destroy.argtypes = [_VP]
            L.oracle_compute_dt.restype = LD
            L.oracle_compute_dt.argtypes = [_VP, _VP, LD]
            L.oracle_time_step.argtypes = [_VP, _VP, LD]
            L.oracle_set_dimswitch.argtypes = [_VP, _I]
            cls._lib = L
        return cls._lib

    def __init__(self, nx, ny, nz, xlen=20000.0, ylen=20000.0, zlen=10000.0, bc=(0, 0, 1),
                 weno_scalars=True, weno_winds=True, data="thermal"):
        super().__init__(5, nx, ny, nz)
        self.L = self.lib()
        self.h = self.L.oracle_create(nx, ny, nz, xlen, ylen, zlen, bc[0], bc[1], bc[2],
                                      int(weno_scalars), int(weno_winds), DATA_SPECS[data])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    @staticmethod
    def _p(a):
        assert a.dtype == np.longdouble and a.flags.c_contiguous
        return a.ctypes.data_as(_VP)

    def new_state(self):
        return np.zeros(self.state_shape, dtype=np.longdouble)

    def time_step(self, st, dt):
        self.L.oracle_time_step(self.h, self._p(st), dt)

    @property
    def dimswitch(self):
        raise AttributeError("write-only")

    @dimswitch.setter
    def dimswitch(self, v):
        self.L.oracle_set_dimswitch(self.h, int(v))


class RefHarness(_Grid):
    """The reference's own Spatial/Temporal operators (built from its sources)."""

    _libs: dict = {}

    @classmethod
    def lib(cls, ord_, crpow=False, tracers=False):
        key = (ord_, crpow, tracers)
        if key not in cls._libs:
            path = ref_path(ord_, crpow, tracers)
            if not os.path.exists(path):
                raise FileNotFoundError(path + " (build with: make -C oracle ref)")
            L = ctypes.CDLL(path)
            L.awflref_create.restype = _VP
            L.awflref_create.argtypes = [_I] * 3 + [_D] * 3 + [_I] * 5 + [ctypes.c_char_p]
            L.awflref_destroy.argtypes = [_VP]
            L.awflref_init_state.argtypes = [_VP]
            L.awflref_state_size.restype = ctypes.c_long
            L.awflref_state_size.argtypes = [_VP]
            L.awflref_get_state.argtypes = [_VP, _DP]
            L.awflref_set_state.argtypes = [_VP, _DP]
            L.awflref_set_bubble.argtypes = [_VP, _I] + [_D] * 8
            L.awflref_add_theta_noise.argtypes = [_VP, ctypes.c_ulonglong, _D]
            L.awflref_set_num_tracers.argtypes = [_I]
            L.awflref_init_tracers.argtypes = [_VP]
            L.awflref_tracer_size.restype = ctypes.c_long
            L.awflref_tracer_size.argtypes = [_VP]
            L.awflref_get_tracers.argtypes = [_VP, _DP]
            L.awflref_compute_dt.restype = _D
            L.awflref_compute_dt.argtypes = [_VP, _D]
            L.awflref_time_step.argtypes = [_VP, _D]
            L.awflref_compute_tendencies.argtypes = [_VP, _D, _I, _DP]
            L.awflref_get_dimswitch.restype = _I
            L.awflref_get_dimswitch.argtypes = [_VP]
            L.awflref_set_dimswitch.argtypes = [_VP, _I]
            L.awflref_get_tables.argtypes = [_VP] + [_DP] * 10
            L.awflref_get_background.argtypes = [_VP] + [_DP] * 8
            L.awflref_coefs_to_tv.restype = _D
            L.awflref_coefs_to_tv.argtypes = [_DP, _I]
            L.awflref_weno_coefs.argtypes = [_VP, _DP, _DP]
            L.awflref_set_tracer_pos.argtypes = [_I, ctypes.POINTER(_I)]
            L.awflref_has_tracer_transport.restype = _I
            L.awflref_set_tracers.argtypes = [_VP, _DP]
            L.awflref_split.argtypes = [_VP, _D, _I]
            L.awflref_output.argtypes = [_VP, _D]
            L.awflref_output_size.restype = ctypes.c_long
            L.awflref_output_size.argtypes = [ctypes.c_char_p]
            L.awflref_output_get.argtypes = [ctypes.c_char_p, _DP]
            cls._libs[key] = L
        return cls._libs[key]

    def __init__(self, nx, ny, nz, xlen=20000.0, ylen=20000.0, zlen=10000.0, bc=(0, 0, 1),
                 weno_scalars=True, weno_winds=True, data="thermal", ord_=5, crpow=False, ntracers=0,
                 tracer_transport=False, pos=None):
        """crpow: the reference's code with its pow/exp calls bound to a correctly rounded
        implementation instead of glibc's. ntracers: tracers registered with addTracer
        before init (the driver's names: uniform, theta, block), posDef flags `pos`
        (default all true). tracer_transport: the build with the reference's tracer code
        compiled in (its NO_TRACERS line blanked, serial loops)."""
        super().__init__(ord_, nx, ny, nz)
        self.L = self.lib(ord_, crpow, tracer_transport)
        self.L.awflref_set_num_tracers(ntracers)
        if pos is not None:
            arr = (_I * len(pos))(*[int(p) for p in pos])
            self.L.awflref_set_tracer_pos(len(pos), arr)
        self.ntracers = ntracers
        self.h = self.L.awflref_create(nx, ny, nz, xlen, ylen, zlen, bc[0], bc[1], bc[2],
                                       int(weno_scalars), int(weno_winds), data.encode())
        if not self.h:
            raise RuntimeError("reference init failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.awflref_destroy(self.h)
            self.h = None

    def init_state(self):
        self.L.awflref_init_state(self.h)

    def init_tracers(self):
        self.L.awflref_init_tracers(self.h)

    def get_tracers(self):
        hs = self.hs
        tr = np.zeros((self.ntracers, self.nz + 2 * hs, self.ny + 2 * hs, self.nx + 2 * hs))
        assert tr.size == self.L.awflref_tracer_size(self.h)
        self.L.awflref_get_tracers(self.h, _ptr(tr))
        return tr

    def set_tracers(self, tr):
        tr = np.ascontiguousarray(tr, dtype=np.float64)
        assert tr.size == self.L.awflref_tracer_size(self.h)
        self.L.awflref_set_tracers(self.h, _ptr(tr))

    def split(self, dt, spl):
        """One split of Temporal_ader::timeStep: computeTendencies(spl) on state and
        tracers, then both applies."""
        self.L.awflref_split(self.h, dt, spl)

    def output(self, etime):
        """Spatial::output on the current state: {variable name: values} of everything it
        wrote (the netCDF stand-in records them instead of writing a file)."""
        self.L.awflref_output(self.h, etime)
        names = ["x", "y", "z", "hyDens", "hyPressure", "hyTheta", "t", "dens_pert", "u", "v", "w",
                 "pot_temp_pert", "pressure_pert"] + ["tracer_" + n for n in ("uniform", "theta", "block")]
        out = {}
        for n in names:
            sz = self.L.awflref_output_size(n.encode())
            if sz >= 0:
                a = np.zeros(sz)
                self.L.awflref_output_get(n.encode(), _ptr(a))
                out[n] = a
        return out

    @property
    def has_tracer_transport(self):
        return bool(self.L.awflref_has_tracer_transport())

    def get_state(self):
        st = self.new_state()
        self.L.awflref_get_state(self.h, _ptr(st))
        return st

    def set_state(self, st):
        st = np.ascontiguousarray(st, dtype=np.float64)
        self.L.awflref_set_state(self.h, _ptr(st))

    def set_bubble(self, shape, x0, y0, z0, xrad, yrad, zrad, amp, pwr=1.0):
        self.L.awflref_set_bubble(self.h, shape, x0, y0, z0, xrad, yrad, zrad, amp, pwr)

    def add_theta_noise(self, seed, amp):
        self.L.awflref_add_theta_noise(self.h, seed, amp)

    def compute_dt(self, cfl=0.8):
        return self.L.awflref_compute_dt(self.h, cfl)

    def time_step(self, dt):
        self.L.awflref_time_step(self.h, dt)

    def compute_tendencies(self, dt, split):
        tend = np.zeros(self.tend_shape)
        self.L.awflref_compute_tendencies(self.h, dt, split, _ptr(tend))
        return tend

    @property
    def dimswitch(self):
        return self.L.awflref_get_dimswitch(self.h)

    @dimswitch.setter
    def dimswitch(self, v):
        self.L.awflref_set_dimswitch(self.h, int(v))

    def tables(self):
        o, g, hs = self.ord, self.ngll, self.hs
        W = np.zeros(o ** 3); c2g = np.zeros(o * g); s2g = np.zeros(o * g); der = np.zeros(g * g)
        idl = np.zeros(hs + 2); sig = np.zeros(1)
        po = np.zeros(o); wo = np.zeros(o); pn = np.zeros(g); wn = np.zeros(g)
        arrs = [W, c2g, s2g, der, idl, sig, po, wo, pn, wn]
        self.L.awflref_get_tables(self.h, *[_ptr(a) for a in arrs])
        names = ["weno_recon", "coefs_to_gll", "sten_to_gll", "deriv", "idl", "sigma",
                 "gll_pts_ord", "gll_wts_ord", "gll_pts_ngll", "gll_wts_ngll"]
        return dict(zip(names, arrs))

    def background(self):
        nzc = self.nz + 2 * self.hs
        arrs = [np.zeros(nzc) for _ in range(4)] + [np.zeros(self.nz * self.ngll) for _ in range(4)]
        self.L.awflref_get_background(self.h, *[_ptr(a) for a in arrs])
        names = ["hyDensCells", "hyPressureCells", "hyThetaCells", "hyDensThetaCells",
                 "hyDensGLL", "hyPressureGLL", "hyThetaGLL", "hyDensThetaGLL"]
        return dict(zip(names, arrs))

    def coefs_to_tv(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self.L.awflref_coefs_to_tv(_ptr(a), len(a))

    def weno_coefs(self, stencil):
        s = np.ascontiguousarray(stencil, dtype=np.float64)
        out = np.zeros(self.ord)
        self.L.awflref_weno_coefs(self.h, _ptr(s), _ptr(out))
        return out
