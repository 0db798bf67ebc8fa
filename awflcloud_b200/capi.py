"""ctypes bindings of the C ABI (include/awfl.h) and a thin context wrapper.

The CUDA library libawfl.so is REQUIRED: importing this module on a machine without it
raises. There is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; AWFL_LIBRARY names another build of the same library (a variant
# compiled with different options, for comparisons)
LIB_PATH = os.environ.get("AWFL_LIBRARY") or os.path.join(HERE, "lib", "libawfl.so")

AWFL_OK = 0
STATUS = {0: "AWFL_OK", -1: "AWFL_ERR_ARG", -2: "AWFL_ERR_CUDA", -3: "AWFL_ERR_NOMEM",
          -4: "AWFL_ERR_STATE", -5: "AWFL_ERR_TIMEOUT", -6: "AWFL_ERR_NOT_BUILT",
          -7: "AWFL_ERR_IO"}
BC = {"periodic": 0, "wall": 1}
BC_PERIODIC, BC_WALL = 0, 1
DATA = {"thermal": 1, "collision": 2, "straka": 3, "igw": 4}
FP64, FP32 = 0, 1
INIT_REFERENCE, INIT_BUBBLE = 0, 1
NOISE_UNIFORM, NOISE_NORMAL = 0, 1


class AwflConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xlen", ctypes.c_double), ("ylen", ctypes.c_double), ("zlen", ctypes.c_double),
                ("bc_x", ctypes.c_int), ("bc_y", ctypes.c_int), ("bc_z", ctypes.c_int),
                ("weno_scalars", ctypes.c_int), ("weno_winds", ctypes.c_int),
                ("data_spec", ctypes.c_int), ("ord", ctypes.c_int), ("precision", ctypes.c_int)]


class AwflInitSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("shape", ctypes.c_int),
                ("x0", ctypes.c_double), ("y0", ctypes.c_double), ("z0", ctypes.c_double),
                ("xrad", ctypes.c_double), ("yrad", ctypes.c_double), ("zrad", ctypes.c_double),
                ("amp", ctypes.c_double), ("pwr", ctypes.c_double),
                ("noise_amp", ctypes.c_double), ("noise_seed", ctypes.c_ulonglong),
                ("noise_kind", ctypes.c_int)]


class AwflError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


_VP, _I, _D, _L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
_DP = ctypes.POINTER(ctypes.c_double)
_SIGS = {
    "awfl_create": (_I, [ctypes.POINTER(AwflConfig), _I, ctypes.POINTER(_VP)]),
    "awfl_destroy": (_I, [_VP]),
    "awfl_last_error": (ctypes.c_char_p, [_VP]),
    "awfl_version": (ctypes.c_char_p, []),
    "awfl_sizes": (_I, [_VP, ctypes.POINTER(_L), ctypes.POINTER(_L), ctypes.POINTER(_I)]),
    "awfl_init_state": (_I, [_VP, _VP, ctypes.POINTER(AwflInitSpec), _VP]),
    "awfl_cfl": (_I, [_VP, _VP, _D, _DP, _VP]),
    "awfl_state_sums": (_I, [_VP, _VP, _DP, _VP]),
    "awfl_check_state": (_I, [_VP, _VP, ctypes.POINTER(_L), _VP]),
    "awfl_output_fields": (_I, [_VP, _VP, _VP, _VP]),
    "awfl_write_netcdf": (_I, [_VP, ctypes.c_char_p, _VP, _D, _VP]),
    "awfl_write_netcdf_fields": (_I, [_VP, ctypes.c_char_p, _DP, _D]),
    "awfl_init_tracers": (_I, [_VP, _VP, _I, _VP]),
    "awfl_split_tracers": (_I, [_VP, _VP, _VP, _I, ctypes.POINTER(_I), _D, _I, _VP]),
    "awfl_step_tracers": (_I, [_VP, _VP, _VP, _I, ctypes.POINTER(_I), _D, _VP]),
    "awfl_output_tracer_fields": (_I, [_VP, _VP, _VP, _I, _VP, _VP]),
    "awfl_write_netcdf_tracers": (_I, [_VP, ctypes.c_char_p, _VP, _VP, _I, ctypes.POINTER(ctypes.c_char_p), _D, _VP]),
    "awfl_write_netcdf_fields_tracers": (_I, [_VP, ctypes.c_char_p, _DP, _I, ctypes.POINTER(ctypes.c_char_p), _D]),
    "awfl_compute_tendencies": (_I, [_VP, _VP, _VP, _D, _I, _VP]),
    "awfl_apply_tendencies": (_I, [_VP, _VP, _VP, _D, _VP]),
    "awfl_split": (_I, [_VP, _VP, _D, _I, _VP]),
    "awfl_step": (_I, [_VP, _VP, _D, _VP]),
    "awfl_step_tlm": (_I, [_VP, _VP, _D, _VP]),
    "awfl_create_slab": (_I, [ctypes.POINTER(AwflConfig), _I, _I, _I, ctypes.POINTER(_VP)]),
    "awfl_slab_info": (_I, [_VP] + [ctypes.POINTER(_I)] * 4 + [ctypes.POINTER(_L)]),
    "awfl_slab_pack": (_I, [_VP, _VP, _VP, _VP]),
    "awfl_split_slab": (_I, [_VP, _VP, _VP, _D, _VP]),
    "awfl_step_adjoint": (_I, [_VP, _VP, _VP, _I, _D, _VP]),
    "awfl_adjoint_tape_bytes": (_I, [_VP, _I, ctypes.POINTER(_L)]),
    "awfl_set_adjoint_subwindow": (_I, [_VP, _I]),
    "awfl_get_dimswitch": (_I, [_VP, ctypes.POINTER(_I)]),
    "awfl_set_dimswitch": (_I, [_VP, _I]),
    "awfl_get_tables": (_I, [_VP] + [_DP] * 10),
    "awfl_get_background": (_I, [_VP] + [_DP] * 8),
    "awfl_selftest_pow": (_I, [_VP, _D, _VP, _L, _I, _VP]),
    "awfl_measure_fma_peak": (_I, [_I, _I, _DP]),
    "awfl_cfl_noalloc": (_I, [ctypes.POINTER(AwflConfig), _VP, _VP, _VP, _D, _DP, _VP]),
    "awfl_ensemble_create": (_I, [ctypes.POINTER(AwflConfig), _I, _I, ctypes.POINTER(_VP)]),
    "awfl_ensemble_destroy": (_I, [_VP]),
    "awfl_ensemble_last_error": (ctypes.c_char_p, [_VP]),
    "awfl_ensemble_size": (_I, [_VP, ctypes.POINTER(_I)]),
    "awfl_ensemble_member": (_I, [_VP, _I, ctypes.POINTER(_VP)]),
    "awfl_ensemble_bind": (_I, [_VP, _I, _VP, _D]),
    "awfl_ensemble_step": (_I, [_VP, _I, _VP]),
    "awfl_ensemble_tune": (_I, [_VP, _I, _VP]),
    "awfl_ensemble_num_shapes": (_I, [_VP, _I, ctypes.POINTER(_I)]),
    "awfl_ensemble_tuning": (_I, [_VP, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float)]),
    "awfl_ensemble_get_shape": (_I, [_VP, _I] + [ctypes.POINTER(_I)] * 4),
    "awfl_ensemble_set_shape": (_I, [_VP, _I, _I]),
    "awfl_ensemble_get_dimswitch": (_I, [_VP, ctypes.POINTER(_I)]),
    "awfl_ensemble_set_dimswitch": (_I, [_VP, _I]),
    "awfl_device_alloc": (_I, [ctypes.POINTER(_VP), _L]),
    "awfl_device_free": (_I, [_VP]),
    "awfl_copy_h2d": (_I, [_VP, _VP, _L, _VP]),
    "awfl_copy_d2h": (_I, [_VP, _VP, _L, _VP]),
    "awfl_memset_device": (_I, [_VP, _I, _L, _VP]),
    "awfl_stream_synchronize": (_I, [_VP]),
    "awfl_device_synchronize": (_I, []),
}

_lib = None


def lib():
    """Load libawfl.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(LIB_PATH + " is missing: build it with python -m awflcloud_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(x):
    """Device or host address of a torch tensor / numpy array / int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def _stream(s):
    if s is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except Exception:
            pass
        return None
    return s if isinstance(s, int) else s.cuda_stream


class Context:
    """An awfl_ctx: one grid configuration on one device (device < 0: host-only)."""

    def __init__(self, nx, ny, nz, xlen=20000.0, ylen=20000.0, zlen=10000.0,
                 bc=("periodic", "periodic", "wall"), weno_scalars=True, weno_winds=True,
                 data="thermal", ord_=5, precision=FP64, device=0):
        self.L = lib()
        bcv = [BC[b] if isinstance(b, str) else int(b) for b in bc]
        self.cfg = AwflConfig(nx, ny, nz, xlen, ylen, zlen, bcv[0], bcv[1], bcv[2],
                              int(weno_scalars), int(weno_winds),
                              DATA[data] if isinstance(data, str) else int(data), ord_, precision)
        h = _VP()
        rc = self.L.awfl_create(ctypes.byref(self.cfg), device, ctypes.byref(h))
        if rc != AWFL_OK:
            raise AwflError(rc, self.L.awfl_last_error(None).decode())
        self.h = h
        self.ord = ord_
        self.ngll = 3 if ord_ == 5 else 5
        self.hs = (ord_ - 1) // 2
        self.nx, self.ny, self.nz = nx, ny, nz
        self.precision = precision
        self.device = device

    @classmethod
    def slab(cls, nx, ny, nz, nslabs, slab, xlen=20000.0, ylen=20000.0, zlen=10000.0,
             bc=("periodic", "periodic", "wall"), weno_scalars=True, weno_winds=True, data="thermal", ord_=5,
             precision=FP64, device=0):
        """Slab `slab` of `nslabs` of the nx x ny x nz grid decomposed in x
        (awfl_create_slab); self.nx is the slab's own width, self.xoff its first cell."""
        self = cls.__new__(cls)
        self.L = lib()
        bcv = [BC[b] if isinstance(b, str) else int(b) for b in bc]
        self.cfg = AwflConfig(nx, ny, nz, xlen, ylen, zlen, bcv[0], bcv[1], bcv[2], int(weno_scalars),
                              int(weno_winds), DATA[data] if isinstance(data, str) else int(data), ord_, precision)
        h = _VP()
        rc = self.L.awfl_create_slab(ctypes.byref(self.cfg), nslabs, slab, device, ctypes.byref(h))
        if rc != AWFL_OK:
            raise AwflError(rc, self.L.awfl_last_error(None).decode())
        self.h = h
        self.ord = ord_
        self.ngll = 3 if ord_ == 5 else 5
        self.hs = (ord_ - 1) // 2
        self.precision = precision
        self.device = device
        info = self.slab_info()
        self.nslabs, self.slab_index, self.xoff, self.nx_global = (info[k] for k in
                                                                   ("nslabs", "slab", "xoff", "nx_global"))
        self.halo_elems = info["halo_elems"]
        self.nx = self._local_nx(nx, nslabs, slab)
        self.ny, self.nz = ny, nz
        return self

    @staticmethod
    def _local_nx(nx, nslabs, slab):
        return nx // nslabs + (1 if slab < nx % nslabs else 0)

    def slab_info(self):
        v = [_I() for _ in range(4)]
        n = _L()
        self._check(self.L.awfl_slab_info(self.h, *[ctypes.byref(x) for x in v], ctypes.byref(n)))
        return dict(nslabs=v[0].value, slab=v[1].value, xoff=v[2].value, nx_global=v[3].value,
                    halo_elems=n.value)

    def slab_pack(self, state, send, stream=None):
        """The slab's first and last hs+1 interior x columns into send
        ([2][5][nz][ny][hs+1], the state's element type)."""
        self._check_buf(send, (self.slab_info()["halo_elems"],), "send", plane_dtype=True)
        self._check(self.L.awfl_slab_pack(self.h, self._st(state), _ptr(send), _stream(stream)))

    def split_slab(self, state, recv, dt, stream=None):
        """The x split with the neighbouring slabs' columns (recv, the layout of send)."""
        self._check_buf(recv, (self.slab_info()["halo_elems"],), "recv", plane_dtype=True)
        self._check(self.L.awfl_split_slab(self.h, self._st(state), _ptr(recv), dt, _stream(stream)))

    @classmethod
    def _borrow(cls, handle, cfg, device):
        """A Context view of a member context owned by an ensemble (not destroyed here)."""
        self = cls.__new__(cls)
        self.L = lib()
        self.cfg = cfg
        self.h = handle
        self.ord = cfg.ord
        self.ngll = 3 if cfg.ord == 5 else 5
        self.hs = (cfg.ord - 1) // 2
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        self.precision = cfg.precision
        self.device = device
        self._owned = False
        return self

    def close(self):
        if getattr(self, "h", None) and getattr(self, "_owned", True):
            self.L.awfl_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != AWFL_OK:
            raise AwflError(rc, self.L.awfl_last_error(self.h).decode())

    # ---- shapes
    @property
    def state_shape(self):
        """FP64: (5, nz+2hs, ny+2hs, nx+2hs). FP32: (10, ...) -- the value plane (5
        variables) followed by the Kahan compensation plane."""
        h = 2 * self.hs
        return (5 if self.precision == FP64 else 10, self.nz + h, self.ny + h, self.nx + h)

    @property
    def tend_shape(self):
        return (5, self.nz, self.ny, self.nx)

    def new_state(self, **kw):
        import torch
        dt = torch.float64 if self.precision == FP64 else torch.float32
        return torch.zeros(self.state_shape, dtype=dt, device="cuda:%d" % max(self.device, 0), **kw)

    def new_tend(self):
        import torch
        dt = torch.float64 if self.precision == FP64 else torch.float32
        return torch.zeros(self.tend_shape, dtype=dt, device="cuda:%d" % max(self.device, 0))

    # ---- argument checks (the C ABI cannot see allocation sizes)
    def _dtype(self):
        import torch
        return torch.float64 if self.precision == FP64 else torch.float32

    def _check_buf(self, x, shape, what, plane_dtype=False):
        if isinstance(x, int) or x is None:
            return  # raw device address: the caller vouches for its size
        import math
        need = math.prod(shape)
        if x.numel() < need or not x.is_contiguous() or x.dtype != self._dtype() or not x.is_cuda:
            raise ValueError("%s must be a contiguous CUDA %s tensor with >= %d elements (got %s %s %s)"
                             % (what, self._dtype(), need, tuple(x.shape), x.dtype, x.device))

    def _st(self, x):
        self._check_buf(x, self.state_shape, "state")
        return _ptr(x)

    def _td(self, x):
        self._check_buf(x, self.tend_shape, "tendency")
        return _ptr(x)

    # ---- entry points
    def init_state(self, state, kind=INIT_REFERENCE, shape=1, x0=10000.0, y0=10000.0, z0=2000.0,
                   xrad=2000.0, yrad=2000.0, zrad=2000.0, amp=3.0, pwr=1.0, noise_amp=0.0,
                   noise_seed=20261203, noise_kind=NOISE_UNIFORM, stream=None):
        spec = AwflInitSpec(kind, shape, x0, y0, z0, xrad, yrad, zrad, amp, pwr, noise_amp, noise_seed, noise_kind)
        self._check(self.L.awfl_init_state(self.h, self._st(state), ctypes.byref(spec), _stream(stream)))

    def cfl(self, state, cfl=0.8, stream=None):
        out = ctypes.c_double()
        self._check(self.L.awfl_cfl(self.h, self._st(state), cfl, ctypes.byref(out), _stream(stream)))
        return out.value

    def state_sums(self, state, stream=None):
        """FP64 sums x dV of the five conserved variables over the interior."""
        import numpy as np
        out = np.zeros(5)
        self._check(self.L.awfl_state_sums(self.h, self._st(state), out.ctypes.data_as(_DP), _stream(stream)))
        return out

    def output_fields(self, state, fields=None, stream=None):
        """Spatial::output's diagnostics (dens_pert, u, v, w, pot_temp_pert, pressure_pert)
        as a (6, nz, ny, nx) FP64 CUDA tensor (allocated when `fields` is None)."""
        import torch
        shape = (6, self.nz, self.ny, self.nx)
        if fields is None:
            fields = torch.empty(shape, dtype=torch.float64, device="cuda:%d" % max(self.device, 0))
        elif (not isinstance(fields, int) and (fields.numel() < 6 * self.nz * self.ny * self.nx
                                               or not fields.is_contiguous() or fields.dtype != torch.float64
                                               or not fields.is_cuda)):
            raise ValueError("fields must be a contiguous CUDA float64 tensor with >= %d elements" % (6 * self.nz * self.ny * self.nx))
        self._check(self.L.awfl_output_fields(self.h, self._st(state), _ptr(fields), _stream(stream)))
        return fields

    def write_netcdf(self, path, state, etime, stream=None):
        """Spatial::output: create (etime == 0) or append to the netCDF output file."""
        self._check(self.L.awfl_write_netcdf(self.h, os.fsencode(path), self._st(state), float(etime),
                                             _stream(stream)))

    def write_netcdf_fields(self, path, fields, etime):
        """The same file from host fields, an array of shape (6, nz, ny, nx) (no device needed)."""
        import numpy as np
        a = np.ascontiguousarray(fields, dtype=np.float64)
        if a.size != 6 * self.nz * self.ny * self.nx:
            raise ValueError("fields must have 6*nz*ny*nx = %d elements" % (6 * self.nz * self.ny * self.nx))
        self._check(self.L.awfl_write_netcdf_fields(self.h, os.fsencode(path), a.ctypes.data_as(_DP), float(etime)))

    # ---- tracers (FP64 arrays of shape (ntracers, nz+2hs, ny+2hs, nx+2hs) for every precision)
    def tracer_shape(self, ntracers):
        h = 2 * self.hs
        return (ntracers, self.nz + h, self.ny + h, self.nx + h)

    def new_tracers(self, ntracers):
        import torch
        return torch.zeros(self.tracer_shape(ntracers), dtype=torch.float64, device="cuda:%d" % max(self.device, 0))

    def _tr(self, x, ntracers):
        import math
        import torch
        if isinstance(x, int) or x is None:
            return _ptr(x)
        need = math.prod(self.tracer_shape(ntracers))
        if x.numel() < need or not x.is_contiguous() or x.dtype != torch.float64 or not x.is_cuda:
            raise ValueError("tracers must be a contiguous CUDA float64 tensor with >= %d elements" % need)
        return _ptr(x)

    def init_tracers(self, tracers, ntracers=None, stream=None):
        """Spatial::initTracers: the driver's tracers (uniform, theta, block; any further zero)."""
        n = tracers.shape[0] if ntracers is None else ntracers
        self._check(self.L.awfl_init_tracers(self.h, self._tr(tracers, n), n, _stream(stream)))

    def _pos(self, pos, n):
        if pos is None:
            pos = [1] * n
        if len(pos) != n:
            raise ValueError("pos needs one flag per tracer")
        return (_I * max(n, 1))(*[int(bool(p)) for p in pos])

    def split_tracers(self, state, tracers, dt, d, pos=None, stream=None):
        """One split of state and tracers."""
        n = tracers.shape[0]
        self._check(self.L.awfl_split_tracers(self.h, self._st(state), self._tr(tracers, n), n, self._pos(pos, n),
                                              dt, d, _stream(stream)))

    def step_tracers(self, state, tracers, dt, pos=None, stream=None):
        """One time step of state and tracers (pos: positive-definite flags, default all)."""
        n = tracers.shape[0]
        self._check(self.L.awfl_step_tracers(self.h, self._st(state), self._tr(tracers, n), n, self._pos(pos, n),
                                             dt, _stream(stream)))

    def output_tracer_fields(self, state, tracers, ntracers=None, stream=None):
        """tracer / (rho' + rho_h) per tracer, as a (ntracers, nz, ny, nx) FP64 CUDA tensor."""
        import torch
        n = tracers.shape[0] if ntracers is None else ntracers
        out = torch.empty((n, self.nz, self.ny, self.nx), dtype=torch.float64, device="cuda:%d" % max(self.device, 0))
        self._check(self.L.awfl_output_tracer_fields(self.h, self._st(state), self._tr(tracers, n), n, _ptr(out),
                                                     _stream(stream)))
        return out

    def write_netcdf_tracers(self, path, state, tracers, names, etime, stream=None):
        """write_netcdf with the tracer_<name> record variables."""
        arr = (ctypes.c_char_p * max(len(names), 1))(*[n.encode() for n in names])
        self._check(self.L.awfl_write_netcdf_tracers(self.h, os.fsencode(path), self._st(state),
                                                     self._tr(tracers, len(names)) if names else None, len(names),
                                                     arr, float(etime), _stream(stream)))

    def write_netcdf_fields_tracers(self, path, fields, names, etime):
        """The same file from host fields of shape (6 + len(names), nz, ny, nx)."""
        import numpy as np
        a = np.ascontiguousarray(fields, dtype=np.float64)
        need = (6 + len(names)) * self.nz * self.ny * self.nx
        if a.size != need:
            raise ValueError("fields must have (6+ntracers)*nz*ny*nx = %d elements" % need)
        arr = (ctypes.c_char_p * max(len(names), 1))(*[n.encode() for n in names])
        self._check(self.L.awfl_write_netcdf_fields_tracers(self.h, os.fsencode(path), a.ctypes.data_as(_DP),
                                                            len(names), arr, float(etime)))

    def check_state(self, state, stream=None):
        """Number of interior cells with a non-finite value or a non-positive density (0 when
        healthy; the C call returns AWFL_ERR_STATE otherwise)."""
        n = _L()
        rc = self.L.awfl_check_state(self.h, self._st(state), ctypes.byref(n), _stream(stream))
        if rc not in (AWFL_OK, -4):
            self._check(rc)
        return n.value

    def compute_tendencies(self, state, tend, dt, d, stream=None):
        self._check(self.L.awfl_compute_tendencies(self.h, self._st(state), self._td(tend), dt, d, _stream(stream)))

    def apply_tendencies(self, state, tend, dt, stream=None):
        self._check(self.L.awfl_apply_tendencies(self.h, self._st(state), self._td(tend), dt, _stream(stream)))

    def split(self, state, dt, d, stream=None):
        self._check(self.L.awfl_split(self.h, self._st(state), dt, d, _stream(stream)))

    def step(self, state, dt, stream=None):
        self._check(self.L.awfl_step(self.h, self._st(state), dt, _stream(stream)))

    def step_tlm(self, state_tangent, dt, stream=None):
        """One tangent-linear step; state_tangent = (state plane, tangent plane), FP64."""
        shp = (2 * self.state_shape[0],) + self.state_shape[1:]
        self._check_buf(state_tangent, shp, "state+tangent")
        self._check(self.L.awfl_step_tlm(self.h, _ptr(state_tangent), dt, _stream(stream)))

    def step_adjoint(self, state_ckpt, lam, nsteps, dt, stream=None):
        """lam <- (d S_{n+nsteps} / d S_n)^T lam, S_n = state_ckpt (not modified), with the
        context's dimswitch holding its value at the checkpoint (unchanged on return)."""
        self._check_buf(state_ckpt, self.state_shape, "checkpoint state")
        self._check_buf(lam, self.state_shape, "adjoint")
        self._check(self.L.awfl_step_adjoint(self.h, _ptr(state_ckpt), _ptr(lam), int(nsteps), dt, _stream(stream)))

    def adjoint_tape_bytes(self, nsteps):
        out = _L()
        self._check(self.L.awfl_adjoint_tape_bytes(self.h, int(nsteps), ctypes.byref(out)))
        return out.value

    def set_adjoint_subwindow(self, steps):
        """Steps per recorded sub-window of step_adjoint (0: the whole window)."""
        self._check(self.L.awfl_set_adjoint_subwindow(self.h, int(steps)))

    @property
    def dimswitch(self):
        v = _I()
        self._check(self.L.awfl_get_dimswitch(self.h, ctypes.byref(v)))
        return v.value

    @dimswitch.setter
    def dimswitch(self, value):
        self._check(self.L.awfl_set_dimswitch(self.h, int(value)))

    def tables(self):
        import numpy as np
        o, g, hs = self.ord, self.ngll, self.hs
        arrs = [np.zeros(o ** 3), np.zeros(o * g), np.zeros(o * g), np.zeros(g * g), np.zeros(hs + 2),
                np.zeros(1), np.zeros(o), np.zeros(o), np.zeros(g), np.zeros(g)]
        self._check(self.L.awfl_get_tables(self.h, *[a.ctypes.data_as(_DP) for a in arrs]))
        names = ["weno_recon", "coefs_to_gll", "sten_to_gll", "deriv", "idl", "sigma",
                 "gll_pts_ord", "gll_wts_ord", "gll_pts_ngll", "gll_wts_ngll"]
        return dict(zip(names, arrs))

    def background(self):
        import numpy as np
        nzc = self.nz + 2 * self.hs
        arrs = [np.zeros(nzc) for _ in range(4)] + [np.zeros(self.nz * self.ngll) for _ in range(4)]
        self._check(self.L.awfl_get_background(self.h, *[a.ctypes.data_as(_DP) for a in arrs]))
        names = ["hyDensCells", "hyPressureCells", "hyThetaCells", "hyDensThetaCells",
                 "hyDensGLL", "hyPressureGLL", "hyThetaGLL", "hyDensThetaGLL"]
        return dict(zip(names, arrs))


class Ensemble:
    """An awfl_ensemble: members with their own configurations advanced together by one
    persistent kernel per split stage (replayed from a CUDA graph)."""

    def __init__(self, configs, device=0):
        """configs: a list of dicts of Context keyword arguments (nx, ny, nz, xlen, ...,
        ord_, precision); every member must share ord_ and precision."""
        self.L = lib()
        arr = (AwflConfig * len(configs))()
        self.members = []
        for i, kw in enumerate(configs):
            kw = dict(kw)
            bc = kw.pop("bc", ("periodic", "periodic", "wall"))
            bcv = [BC[b] if isinstance(b, str) else int(b) for b in bc]
            data = kw.pop("data", "thermal")
            arr[i] = AwflConfig(kw["nx"], kw["ny"], kw["nz"], kw.get("xlen", 20000.0), kw.get("ylen", 20000.0),
                                kw.get("zlen", 10000.0), bcv[0], bcv[1], bcv[2], int(kw.get("weno_scalars", True)),
                                int(kw.get("weno_winds", True)), DATA[data] if isinstance(data, str) else int(data),
                                kw.get("ord_", 5), kw.get("precision", FP64))
        h = _VP()
        rc = self.L.awfl_ensemble_create(arr, len(configs), device, ctypes.byref(h))
        if rc != AWFL_OK:
            raise AwflError(rc, self.L.awfl_ensemble_last_error(None).decode())
        self.h = h
        self.device = device
        for i in range(len(configs)):
            c = _VP()
            self._check(self.L.awfl_ensemble_member(self.h, i, ctypes.byref(c)))
            self.members.append(Context._borrow(c, arr[i], device))
        self.states = [None] * len(configs)

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None  # owned by the ensemble
            self.L.awfl_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != AWFL_OK:
            raise AwflError(rc, self.L.awfl_ensemble_last_error(self.h).decode())

    def __len__(self):
        return len(self.members)

    def bind(self, i, state, dt):
        self.members[i]._check_buf(state, self.members[i].state_shape, "state")
        self.states[i] = state  # keep the buffer alive while bound
        self._check(self.L.awfl_ensemble_bind(self.h, i, _ptr(state), float(dt)))

    def step(self, nsteps=1, stream=None):
        self._check(self.L.awfl_ensemble_step(self.h, int(nsteps), _stream(stream)))

    def tune(self, reps=3, stream=None):
        self._check(self.L.awfl_ensemble_tune(self.h, int(reps), _stream(stream)))
        return self.tuning()

    def tuning(self):
        """Per direction: list of (chunk, lines, ms per launch) of every candidate shape."""
        out = []
        for d in range(3):
            n = _I()
            self._check(self.L.awfl_ensemble_num_shapes(self.h, d, ctypes.byref(n)))
            rows = []
            for i in range(n.value):
                c, w, ms = _I(), _I(), ctypes.c_float()
                self._check(self.L.awfl_ensemble_tuning(self.h, d, i, ctypes.byref(c), ctypes.byref(w),
                                                        ctypes.byref(ms)))
                rows.append((c.value, w.value, ms.value))
            out.append(rows)
        return out

    def shape(self, d):
        """(shape index, chunk, lines, persistent grid) in use for direction d."""
        v = [_I() for _ in range(4)]
        self._check(self.L.awfl_ensemble_get_shape(self.h, d, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def set_shape(self, d, i):
        self._check(self.L.awfl_ensemble_set_shape(self.h, d, int(i)))

    @property
    def dimswitch(self):
        v = _I()
        self._check(self.L.awfl_ensemble_get_dimswitch(self.h, ctypes.byref(v)))
        return v.value

    @dimswitch.setter
    def dimswitch(self, value):
        self._check(self.L.awfl_ensemble_set_dimswitch(self.h, int(value)))


def header_symbols(path=None):
    """Function names declared in include/awfl.h."""
    import re
    path = path or os.path.join(os.path.dirname(HERE), "include", "awfl.h")
    src = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|void)\s*\*?\s*(awfl_\w+)\s*\(", src, re.M)))


PEAK_FP32_PAIRED = 2


def measure_fma_peak(precision=FP64, device=0):
    """Measured FMA throughput (TFLOP/s) of the FP64 or FP32 CUDA-core pipe; precision
    PEAK_FP32_PAIRED measures sm_100's paired FP32 FMA (two lanes per instruction)."""
    out = ctypes.c_double()
    rc = lib().awfl_measure_fma_peak(precision, device, ctypes.byref(out))
    if rc != AWFL_OK:
        raise AwflError(rc, "awfl_measure_fma_peak failed")
    return out.value
