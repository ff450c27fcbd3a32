"""Python binding of the B200 immersed-boundary coupling library.

The product is ``lib/libibk.so`` (hand-written sm_100a CUDA behind the C ABI
in ``include/ibk.h``).  This module binds that ABI with ctypes and mirrors the
reference's operator objects (sonwell/ib.cu ``include/ib/novel.h:193-250``
and ``include/ib/interpolate.h:88-138``):

    domain = Domain(Dimension(3.2, PERIODIC), Dimension(1.6, SOLID),
                    Dimension(3.2, PERIODIC))
    spread = Spread(Mac(64), domain, Bspline(3))
    interpolate = Interpolate(Mac(64), domain, Bspline(3))
    fe = spread(n, x, fl)          # list of device vectors, newly allocated
    spread(n, x, fl, fe)           # overwrites fe
    ul = interpolate(n, x, ue)

Arrays are torch CUDA float64 tensors (device memory and streams only; no
torch op is on the compute path).  There is no CPU fallback: every call
raises if the CUDA library is missing or a CUDA call fails.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libibk.so")

# ---------------------------------------------------------------- ABI enums
IBK_OK = 0
STATUS_NAMES = {
    0: "IBK_OK", 1: "IBK_ERR_INVALID_ARGUMENT", 2: "IBK_ERR_UNSUPPORTED",
    3: "IBK_ERR_OUT_OF_MEMORY", 4: "IBK_ERR_CUDA", 5: "IBK_ERR_CAPACITY",
    6: "IBK_ERR_DEVICE_CHECK",
}
PERIODIC, SOLID = 0, 1
TAG_MAC, TAG_CENTERED = 0, 1
BSPLINE, PESKIN, ROMA, COSINE, HAT = 0, 1, 2, 3, 4
FP64, FP32C = 0, 1
SKALAK, NEOHOOKEAN, HOOKEAN = 0, 1, 2    # ibk_tension_law

# Every symbol include/ibk.h declares (checked by the CPU test suite).
ABI_SYMBOLS = (
    "ibk_plan_create", "ibk_plan_destroy", "ibk_plan_info", "ibk_plan_reserve", "ibk_plan_set_tiles",
    "ibk_spread", "ibk_interpolate", "ibk_spread_interpolate", "ibk_sort_keys", "ibk_force_moments", "ibk_grid_totals",
    "ibk_plan_set_profiling", "ibk_plan_kernel_stats", "ibk_plan_reset_stats",
    "ibk_plan_launch_count", "ibk_plan_check", "ibk_interpolate_noalloc",
    "ibk_batch_create", "ibk_batch_destroy", "ibk_batch_info", "ibk_batch_bind",
    "ibk_batch_set_step", "ibk_batch_run", "ibk_batch_capture", "ibk_batch_configure",
    "ibk_batch_get_config", "ibk_batch_tune", "ibk_batch_launch_count", "ibk_batch_check",
    "ibk_server_create", "ibk_server_destroy", "ibk_server_admit", "ibk_server_retire",
    "ibk_server_submit", "ibk_server_progress", "ibk_server_drain", "ibk_server_clock",
    "ibk_server_read", "ibk_server_get_stats", "ibk_server_reset_stats", "ibk_server_run_poisson",
    "ibk_server_save", "ibk_server_admit_from",
    "ibk_io_write_dense", "ibk_io_write_scalar", "ibk_io_read_dense", "ibk_io_read_scalar",
    "ibk_io_write_sparse", "ibk_io_read_sparse",
    "ibk_surface_plan_create", "ibk_surface_plan_destroy", "ibk_surface_geometry", "ibk_membrane_tension",
    "ibk_membrane_bending", "ibk_membrane_dissipation", "ibk_membrane_tether", "ibk_membrane_repelling",
    "ibk_curve_plan_create", "ibk_curve_tension",
    "ibk_diffusion_create", "ibk_diffusion_destroy", "ibk_diffusion_apply", "ibk_diffusion_step",
    "ibk_diffusion_set_preconditioner", "ibk_diffusion_info",
    "ibk_last_error", "ibk_status_string", "ibk_version",
)
OP_SPREAD, OP_INTERPOLATE, OP_STEP, OP_SPREAD_INTERPOLATE = 1, 2, 3, 4


class IbkError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class _Domain(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int), ("length", ctypes.c_double * 3),
                ("boundary", ctypes.c_int * 3)]


class _Delta(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("order", ctypes.c_int)]


class KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_longlong),
                ("total_ms", ctypes.c_double)]


class GridInfo(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int), ("meshwidths", ctypes.c_int),
                ("unit", ctypes.c_double), ("resolution", ctypes.c_double),
                ("points", (ctypes.c_int * 3) * 3), ("cells", (ctypes.c_int * 3) * 3),
                ("shift", (ctypes.c_double * 3) * 3), ("size", ctypes.c_longlong * 3)]

    def comp_points(self, c):
        return [self.points[c][d] for d in range(self.dims)]


class _InstanceDesc(ctypes.Structure):
    _fields_ = [("domain", _Domain), ("tag", ctypes.c_int), ("refinement", ctypes.c_int)]


class _InstanceIO(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("x", ctypes.c_void_p), ("fl", ctypes.c_void_p),
                ("fe", ctypes.c_void_p * 3), ("ue", ctypes.c_void_p * 3), ("ul", ctypes.c_void_p),
                ("xn", ctypes.c_void_p), ("xref", ctypes.c_void_p), ("fs", ctypes.c_void_p)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("spread_tile", ctypes.c_int * 3), ("interp_tile", ctypes.c_int * 3),
                ("spread_ctas_per_sm", ctypes.c_int), ("interp_ctas_per_sm", ctypes.c_int),
                ("spread_threads", ctypes.c_int)]

    def as_dict(self):
        return {"spread_tile": list(self.spread_tile), "interp_tile": list(self.interp_tile),
                "spread_ctas_per_sm": self.spread_ctas_per_sm,
                "interp_ctas_per_sm": self.interp_ctas_per_sm,
                "spread_threads": self.spread_threads or 256}


class IoHeader(ctypes.Structure):
    _fields_ = [("magic", ctypes.c_int), ("matrix", ctypes.c_int), ("rows", ctypes.c_int),
                ("cols", ctypes.c_int), ("count", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("delta", _Delta), ("precision", ctypes.c_int), ("slots", ctypes.c_int),
                ("dt", ctypes.c_double), ("k", ctypes.c_double), ("hbm_budget", ctypes.c_longlong),
                ("max_points", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("points", ctypes.c_longlong), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("wall_s", ctypes.c_double),
                ("admitted_bytes", ctypes.c_longlong), ("host_ms_per_launch", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class _Surface(ctypes.Structure):
    _fields_ = [("position", ctypes.c_void_p), ("t", ctypes.c_void_p * 2), ("tt", ctypes.c_void_p * 3),
                ("normal", ctypes.c_void_p), ("sigma", ctypes.c_void_p)]


_lib = None
_vp = ctypes.c_void_p


def build(force: bool = False) -> str:
    """Compile lib/libibk.so for sm_100a with nvcc (in-tree)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """Load the CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"CUDA library not built: {LIB_PATH} (run build())")
        L = ctypes.CDLL(LIB_PATH)
        L.ibk_plan_create.argtypes = [ctypes.POINTER(_Domain), ctypes.c_int, ctypes.c_int,
                                      _Delta, ctypes.c_int, ctypes.POINTER(_vp)]
        L.ibk_plan_destroy.argtypes = [_vp]
        L.ibk_plan_info.argtypes = [_vp, ctypes.POINTER(GridInfo)]
        L.ibk_plan_reserve.argtypes = [_vp, ctypes.c_int]
        L.ibk_plan_set_tiles.argtypes = [_vp, ctypes.POINTER(ctypes.c_int * 3), ctypes.POINTER(ctypes.c_int * 3)]
        L.ibk_plan_set_tiles.restype = ctypes.c_int
        L.ibk_spread.argtypes = [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(_vp), _vp]
        L.ibk_interpolate.argtypes = [_vp, ctypes.c_int, _vp, ctypes.POINTER(_vp), _vp, _vp]
        L.ibk_spread_interpolate.argtypes = [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(_vp),
                                             ctypes.POINTER(_vp), _vp, _vp]
        L.ibk_sort_keys.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]
        L.ibk_force_moments.argtypes = [_vp, ctypes.c_int, _vp, _vp, _vp, _vp]
        L.ibk_force_moments.restype = ctypes.c_int
        L.ibk_grid_totals.argtypes = [_vp, ctypes.POINTER(_vp), _vp, _vp]
        L.ibk_grid_totals.restype = ctypes.c_int
        L.ibk_plan_set_profiling.argtypes = [_vp, ctypes.c_int]
        L.ibk_plan_kernel_stats.argtypes = [_vp, ctypes.POINTER(KernelStat), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int)]
        L.ibk_plan_reset_stats.argtypes = [_vp]
        L.ibk_plan_launch_count.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
        L.ibk_plan_check.argtypes = [_vp]
        L.ibk_interpolate_noalloc.argtypes = [ctypes.POINTER(_Domain), ctypes.c_int, ctypes.c_int,
                                              _Delta, ctypes.c_int, ctypes.c_int, _vp,
                                              ctypes.POINTER(_vp), _vp, _vp]
        L.ibk_interpolate_noalloc.restype = ctypes.c_int
        L.ibk_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(_InstanceDesc), _Delta, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(_vp)]
        L.ibk_batch_destroy.argtypes = [_vp]
        L.ibk_batch_info.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(GridInfo)]
        L.ibk_batch_bind.argtypes = [_vp, ctypes.POINTER(_InstanceIO), _vp]
        L.ibk_batch_set_step.argtypes = [_vp, ctypes.c_double, ctypes.c_double]
        L.ibk_batch_run.argtypes = [_vp, ctypes.c_int, _vp]
        L.ibk_batch_capture.argtypes = [_vp, ctypes.c_int]
        L.ibk_batch_configure.argtypes = [_vp, ctypes.POINTER(BatchConfig)]
        L.ibk_batch_get_config.argtypes = [_vp, ctypes.POINTER(BatchConfig)]
        L.ibk_batch_tune.argtypes = [_vp, ctypes.c_int, _vp, ctypes.POINTER(BatchConfig)]
        L.ibk_batch_launch_count.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
        L.ibk_batch_check.argtypes = [_vp]
        L.ibk_server_create.argtypes = [ctypes.c_int, ctypes.POINTER(_InstanceDesc),
                                        ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]
        L.ibk_server_destroy.argtypes = [_vp]
        L.ibk_server_admit.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.POINTER(_vp)]
        L.ibk_server_retire.argtypes = [_vp, ctypes.c_int]
        L.ibk_server_submit.argtypes = [_vp, ctypes.c_int, ctypes.c_double]
        L.ibk_server_progress.argtypes = [_vp, ctypes.POINTER(ctypes.c_int)]
        L.ibk_server_drain.argtypes = [_vp]
        L.ibk_server_clock.argtypes = [_vp]
        L.ibk_server_clock.restype = ctypes.c_double
        L.ibk_server_read.argtypes = [_vp, ctypes.c_int, _vp, ctypes.POINTER(_vp)]
        L.ibk_server_get_stats.argtypes = [_vp, ctypes.POINTER(ServerStats)]
        L.ibk_server_reset_stats.argtypes = [_vp]
        L.ibk_server_run_poisson.argtypes = [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong,
                                             ctypes.POINTER(ServerStats)]
        L.ibk_server_save.argtypes = [_vp, ctypes.c_int, ctypes.c_char_p]
        L.ibk_server_admit_from.argtypes = [_vp, ctypes.c_int, ctypes.c_char_p]
        L.ibk_io_write_dense.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, _vp]
        L.ibk_io_write_scalar.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
        L.ibk_io_read_dense.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.POINTER(IoHeader), _vp,
                                        ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
        L.ibk_io_read_scalar.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_longlong)]
        L.ibk_io_write_sparse.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _vp, _vp, _vp]
        L.ibk_io_read_sparse.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.POINTER(IoHeader), _vp, _vp,
                                         _vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
        L.ibk_surface_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp), _vp, ctypes.POINTER(_vp)]
        L.ibk_surface_plan_destroy.argtypes = [_vp]
        L.ibk_surface_geometry.argtypes = [_vp, ctypes.c_int, _vp, ctypes.POINTER(_Surface), _vp]
        L.ibk_membrane_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(_Surface), ctypes.POINTER(_Surface), _vp, _vp]
        L.ibk_diffusion_create.argtypes = [_vp, ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.POINTER(_vp)]
        L.ibk_diffusion_destroy.argtypes = [_vp]
        L.ibk_diffusion_apply.argtypes = [_vp, ctypes.c_int, _vp, _vp, _vp]
        L.ibk_diffusion_step.argtypes = [_vp, ctypes.c_double, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int), _vp]
        L.ibk_diffusion_set_preconditioner.argtypes = [_vp, ctypes.c_int]
        L.ibk_diffusion_info.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.ibk_membrane_bending.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                           ctypes.POINTER(_Surface), ctypes.POINTER(_Surface), _vp, _vp]
        L.ibk_membrane_dissipation.argtypes = [_vp, ctypes.c_double, ctypes.c_int, _vp, ctypes.POINTER(_Surface),
                                               _vp, _vp]
        L.ibk_curve_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp), _vp, ctypes.POINTER(_vp)]
        L.ibk_curve_tension.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.POINTER(_Surface), ctypes.POINTER(_Surface), _vp, _vp]
        L.ibk_membrane_tether.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.POINTER(_Surface),
                                          ctypes.POINTER(_Surface), _vp, _vp]
        L.ibk_membrane_repelling.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(_Surface), _vp, _vp]
        for name in ABI_SYMBOLS:
            if name.startswith(("ibk_batch_", "ibk_server_", "ibk_io_", "ibk_surface_", "ibk_membrane_",
                                "ibk_diffusion_", "ibk_curve_")) \
                    and name != "ibk_server_clock":
                getattr(L, name).restype = ctypes.c_int
        L.ibk_last_error.restype = ctypes.c_char_p
        L.ibk_status_string.restype = ctypes.c_char_p
        L.ibk_status_string.argtypes = [ctypes.c_int]
        for name in ("ibk_plan_create", "ibk_plan_destroy", "ibk_plan_info", "ibk_plan_reserve",
                     "ibk_spread", "ibk_interpolate", "ibk_sort_keys", "ibk_force_moments", "ibk_grid_totals", "ibk_plan_set_profiling",
                     "ibk_plan_kernel_stats", "ibk_plan_reset_stats", "ibk_plan_launch_count",
                     "ibk_plan_check"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != IBK_OK:
        msg = lib().ibk_last_error()
        raise IbkError(status, msg.decode() if msg else "")


def _stream_handle(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


# ------------------------------------------------ reference-shaped objects
class Dimension:
    """fd::dimension{length, boundary} (include/fd/dimension.h:32-80)."""

    def __init__(self, length: float, boundary: int = PERIODIC):
        self.length = float(length)
        self.boundary = int(boundary)


class Domain:
    """fd::domain{dims...} (include/fd/domain.h:15-33)."""

    def __init__(self, *dimensions: Dimension):
        if not 2 <= len(dimensions) <= 3:
            raise ValueError("domains have 2 or 3 dimensions")
        self.dimensions = list(dimensions)

    @property
    def dims(self) -> int:
        return len(self.dimensions)

    def _abi(self) -> _Domain:
        d = _Domain()
        d.dims = self.dims
        for i, dim in enumerate(self.dimensions):
            d.length[i] = dim.length
            d.boundary[i] = dim.boundary
        return d


class Mac:
    """fd::mac{refinement} (include/fd/cell.h:195)."""
    tag = TAG_MAC

    def __init__(self, refinement: int):
        self.refinement = int(refinement)


class Centered(Mac):
    """fd::centered{refinement} (include/fd/cell.h:194)."""
    tag = TAG_CENTERED


class DeltaFn:
    kind = BSPLINE
    order = 0


class Bspline(DeltaFn):
    """ib::delta::bspline<n> (include/ib/bspline.h:13-63)."""

    def __init__(self, order: int = 3):
        self.kind, self.order = BSPLINE, int(order)


class Peskin(DeltaFn):
    kind = PESKIN


class Roma(DeltaFn):
    kind = ROMA


class Cosine(DeltaFn):
    kind = COSINE


class Hat(DeltaFn):
    kind = HAT


class Plan:
    """Owner of one ``ibk_plan`` (grid geometry + device scratch)."""

    def __init__(self, tag: Mac, domain: Domain, delta: DeltaFn, precision: int = FP64):
        d = _Delta()
        d.kind, d.order = delta.kind, delta.order
        h = _vp()
        check(lib().ibk_plan_create(ctypes.byref(domain._abi()), tag.tag, tag.refinement,
                                    d, int(precision), ctypes.byref(h)))
        self._h = h
        self.domain = domain
        self.precision = precision
        info = GridInfo()
        check(lib().ibk_plan_info(h, ctypes.byref(info)))
        self.info = info
        self.dims = info.dims

    def close(self):
        if getattr(self, "_h", None):
            lib().ibk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def sizes(self):
        return [int(self.info.size[c]) for c in range(self.dims)]

    def reserve(self, max_points: int):
        check(lib().ibk_plan_reserve(self._h, int(max_points)))

    def set_tiles(self, spread_tile=None, interp_tile=None):
        """Preferred tile extents (cells per axis) of the spread / interpolation kernels."""
        def arr(t):
            return None if t is None else ctypes.byref((ctypes.c_int * 3)(*[int(v) for v in t]))
        check(lib().ibk_plan_set_tiles(self._h, arr(spread_tile), arr(interp_tile)))

    def _comp_ptrs(self, arrs):
        P = (_vp * 3)()
        for c in range(self.dims):
            P[c] = _ptr(arrs[c])
        return P

    def spread(self, n, x, fl, fe, stream=None):
        check(lib().ibk_spread(self._h, int(n), _ptr(x), _ptr(fl), self._comp_ptrs(fe),
                               _stream_handle(stream)))

    def interpolate(self, n, x, ue, ul, stream=None):
        check(lib().ibk_interpolate(self._h, int(n), _ptr(x), self._comp_ptrs(ue), _ptr(ul),
                                    _stream_handle(stream)))

    def spread_interpolate(self, n, x, fl, fe, ue, ul, stream=None):
        """spread(n, x, fl, fe) and interpolate(n, x, ue, ul) with one binning of x."""
        check(lib().ibk_spread_interpolate(self._h, int(n), _ptr(x), _ptr(fl), self._comp_ptrs(fe),
                                           self._comp_ptrs(ue), _ptr(ul), _stream_handle(stream)))

    def set_profiling(self, enable: bool):
        check(lib().ibk_plan_set_profiling(self._h, 1 if enable else 0))

    def kernel_stats(self):
        """{kernel name: (launches, total device ms)}; synchronises."""
        buf = (KernelStat * 64)()
        cnt = ctypes.c_int()
        check(lib().ibk_plan_kernel_stats(self._h, buf, 64, ctypes.byref(cnt)))
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].total_ms))
                for i in range(min(cnt.value, 64))}

    def reset_stats(self):
        check(lib().ibk_plan_reset_stats(self._h))

    def check(self):
        """Raise if a kernel's own device-side check tripped since the last call."""
        check(lib().ibk_plan_check(self._h))

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        check(lib().ibk_plan_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def force_moments(self, n, x, fl, stream=None):
        """FP64 total force and torque of the point forces (deterministic): 6 values."""
        import torch
        out = torch.empty(6, dtype=torch.float64, device=x.device)
        check(lib().ibk_force_moments(self._h, int(n), _ptr(x), _ptr(fl), _ptr(out), _stream_handle(stream)))
        return out.cpu().numpy()

    def grid_totals(self, fe, stream=None):
        """FP64 h^dims * sum over faces of each spread component (deterministic)."""
        import torch
        out = torch.empty(self.dims, dtype=torch.float64, device=fe[0].device)
        check(lib().ibk_grid_totals(self._h, self._comp_ptrs(fe), _ptr(out), _stream_handle(stream)))
        return out.cpu().numpy()

    def sort_keys(self, comp, n, x, keys, stream=None):
        check(lib().ibk_sort_keys(self._h, int(comp), int(n), _ptr(x), _ptr(keys),
                                  _stream_handle(stream)))


def _points(x, dims):
    return x.numel() // dims


class Spread:
    """ib::spread{tag, domain, delta} (include/ib/novel.h:193-250)."""

    def __init__(self, tag: Mac, domain: Domain, delta: DeltaFn, precision: int = FP64):
        self.plan = Plan(tag, domain, delta, precision)

    def __call__(self, *args, stream=None):
        import torch
        dims = self.plan.dims
        if len(args) == 4:                     # (n, x, fl, fe): overwrite fe
            n, x, fl, fe = args
        elif len(args) == 3 and isinstance(args[0], int):   # (n, x, fl): new fe
            n, x, fl = args
            fe = None
        elif len(args) == 3:                   # (x, fl, fe)
            x, fl, fe = args
            n = _points(x, dims)
        elif len(args) == 2:                   # (x, fl)
            x, fl = args
            n, fe = _points(x, dims), None
        else:
            raise TypeError("spread(n, x, fl[, fe]) or spread(x, fl[, fe])")
        if fe is None:
            fe = [torch.zeros(s, dtype=torch.float64, device=x.device) for s in self.plan.sizes()]
        self.plan.spread(n, x, fl, fe, stream)
        return fe


class Interpolate:
    """ib::interpolate{tag, domain, delta} (include/ib/interpolate.h:88-138)."""

    def __init__(self, tag: Mac, domain: Domain, delta: DeltaFn, precision: int = FP64):
        self.plan = Plan(tag, domain, delta, precision)

    def __call__(self, *args, stream=None):
        import torch
        dims = self.plan.dims
        if len(args) == 4:                     # (n, x, ue, ul)
            n, x, ue, ul = args
        elif len(args) == 3 and isinstance(args[0], int):   # (n, x, ue) -> ul
            n, x, ue = args
            ul = None
        elif len(args) == 3:                   # (x, ue, ul)
            x, ue, ul = args
            n = _points(x, dims)
        elif len(args) == 2:                   # (x, ue) -> ul
            x, ue = args
            n, ul = _points(x, dims), None
        else:
            raise TypeError("interpolate(n, x, ue[, ul]) or interpolate(x, ue[, ul])")
        if ul is None:
            ul = torch.empty(x.numel(), dtype=torch.float64, device=x.device)
        self.plan.interpolate(n, x, ue, ul, stream)
        return ul


# ------------------------------------------------------------------ batches
class Instance:
    """One grid of a batch: its domain and tag (fd::mac{refinement})."""

    def __init__(self, tag: Mac, domain: Domain):
        self.tag = tag
        self.domain = domain


class Batch:
    """Owner of one ``ibk_batch``: many independent grids, one persistent
    kernel per operator (no counterpart in the reference, which runs one
    operator object per grid).

    ``bind(io)`` takes one dict per instance with any of the keys ``n, x, fl,
    fe, ue, ul, xn, xref, fs`` (torch CUDA float64 tensors; fe and ue are
    per-component lists); ``run(op)`` runs OP_SPREAD, OP_INTERPOLATE or
    OP_STEP over every instance."""

    def __init__(self, instances, delta: DeltaFn, precision: int = FP32C, max_points: int = 0):
        count = len(instances)
        descs = (_InstanceDesc * count)()
        for i, inst in enumerate(instances):
            descs[i].domain = inst.domain._abi()
            descs[i].tag = inst.tag.tag
            descs[i].refinement = inst.tag.refinement
        d = _Delta()
        d.kind, d.order = delta.kind, delta.order
        h = _vp()
        check(lib().ibk_batch_create(count, descs, d, int(precision), int(max_points), ctypes.byref(h)))
        self._h = h
        self.count = count
        self.precision = precision
        self.infos = []
        for i in range(count):
            info = GridInfo()
            check(lib().ibk_batch_info(h, i, ctypes.byref(info)))
            self.infos.append(info)
        self._bound = None     # keeps the bound tensors alive

    def close(self):
        if getattr(self, "_h", None):
            lib().ibk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sizes(self, i):
        info = self.infos[i]
        return [int(info.size[c]) for c in range(info.dims)]

    def bind(self, io, stream=None):
        tab = (_InstanceIO * self.count)()
        for i, e in enumerate(io):
            t = tab[i]
            t.n = int(e.get("n", 0))
            for key in ("x", "fl", "ul", "xn", "xref", "fs"):
                setattr(t, key, _ptr(e.get(key)))
            for key in ("fe", "ue"):
                arrs = e.get(key)
                if arrs is not None:
                    for c, a in enumerate(arrs):
                        getattr(t, key)[c] = _ptr(a)
        check(lib().ibk_batch_bind(self._h, tab, _stream_handle(stream)))
        self._bound = io

    def set_step(self, dt: float, k: float):
        check(lib().ibk_batch_set_step(self._h, float(dt), float(k)))

    def run(self, op: int, stream=None):
        check(lib().ibk_batch_run(self._h, int(op), _stream_handle(stream)))

    def capture(self, op: int):
        check(lib().ibk_batch_capture(self._h, int(op)))

    def configure(self, spread_tile=(16, 16, 16), interp_tile=(16, 16, 16),
                  spread_ctas_per_sm=0, interp_ctas_per_sm=0, spread_threads=0):
        c = BatchConfig()
        for d in range(3):
            c.spread_tile[d] = int(spread_tile[d])
            c.interp_tile[d] = int(interp_tile[d])
        c.spread_ctas_per_sm = int(spread_ctas_per_sm)
        c.interp_ctas_per_sm = int(interp_ctas_per_sm)
        c.spread_threads = int(spread_threads)
        check(lib().ibk_batch_configure(self._h, ctypes.byref(c)))

    def config(self) -> dict:
        c = BatchConfig()
        check(lib().ibk_batch_get_config(self._h, ctypes.byref(c)))
        return c.as_dict()

    def tune(self, op: int, stream=None) -> dict:
        c = BatchConfig()
        check(lib().ibk_batch_tune(self._h, int(op), _stream_handle(stream), ctypes.byref(c)))
        return c.as_dict()

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        check(lib().ibk_batch_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def check(self):
        check(lib().ibk_batch_check(self._h))


# ------------------------------------------------------------------ serving
class Server:
    """Owner of one ``ibk_server``: device-resident ensemble members stepped
    (interpolate, advect, spring force, spread) as requests arrive, packed
    into batched launches on ``slots`` streams (continuous batching)."""

    def __init__(self, instances, delta: DeltaFn, precision: int = FP32C, slots: int = 2,
                 dt: float = 1e-3, k: float = 1e-3, hbm_budget: int = 150 * 10**9, max_points: int = 0):
        count = len(instances)
        descs = (_InstanceDesc * count)()
        for i, inst in enumerate(instances):
            descs[i].domain = inst.domain._abi()
            descs[i].tag = inst.tag.tag
            descs[i].refinement = inst.tag.refinement
        cfg = ServerConfig()
        cfg.delta.kind, cfg.delta.order = delta.kind, delta.order
        cfg.precision, cfg.slots, cfg.dt, cfg.k = int(precision), int(slots), float(dt), float(k)
        cfg.hbm_budget, cfg.max_points = int(hbm_budget), int(max_points)
        h = _vp()
        check(lib().ibk_server_create(count, descs, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.count = count

    def close(self):
        if getattr(self, "_h", None):
            lib().ibk_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, member: int, x, ue):
        """x: host float64 array (dims*n); ue: per-component host float64 arrays."""
        import numpy as np
        x = np.ascontiguousarray(x, dtype=np.float64)
        ue = [np.ascontiguousarray(u, dtype=np.float64) for u in ue]
        P = (_vp * 3)(*[u.ctypes.data for u in ue])
        check(lib().ibk_server_admit(self._h, int(member), x.size // len(ue), x.ctypes.data, P))

    def retire(self, member: int):
        check(lib().ibk_server_retire(self._h, int(member)))

    def submit(self, member: int, t_arrival: float = -1.0):
        check(lib().ibk_server_submit(self._h, int(member), float(t_arrival)))

    def progress(self) -> int:
        p = ctypes.c_int()
        check(lib().ibk_server_progress(self._h, ctypes.byref(p)))
        return int(p.value)

    def drain(self):
        check(lib().ibk_server_drain(self._h))

    def clock(self) -> float:
        return float(lib().ibk_server_clock(self._h))

    def read(self, member: int, n: int, sizes):
        """(positions, [force grid per component]) as host numpy arrays."""
        import numpy as np
        x = np.empty(3 * n, dtype=np.float64)
        fe = [np.empty(s, dtype=np.float64) for s in sizes]
        P = (_vp * 3)(*[a.ctypes.data for a in fe])
        check(lib().ibk_server_read(self._h, int(member), x.ctypes.data, P))
        return x, fe

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().ibk_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        check(lib().ibk_server_reset_stats(self._h))

    def save(self, member: int, path: str):
        """Checkpoint of one member in the linalg::io binary format."""
        check(lib().ibk_server_save(self._h, int(member), os.fsencode(path)))

    def admit_from(self, member: int, path: str):
        check(lib().ibk_server_admit_from(self._h, int(member), os.fsencode(path)))

    def run_poisson(self, rate: float, requests: int, seed: int = 0) -> dict:
        st = ServerStats()
        check(lib().ibk_server_run_poisson(self._h, float(rate), int(requests), int(seed), ctypes.byref(st)))
        return st.as_dict()


# ------------------------------------------- membrane forces on RBF surfaces
_SURFACE_FIELDS = ("position", "tu", "tv", "tuu", "tuv", "tvv", "normal", "sigma")


def _surface_struct(g):
    """ibk_surface from a dict of device tensors (missing keys: NULL)."""
    s = _Surface()
    s.position = _ptr(g.get("position"))
    s.t[0], s.t[1] = _ptr(g.get("tu")), _ptr(g.get("tv"))
    s.tt[0], s.tt[1], s.tt[2] = _ptr(g.get("tuu")), _ptr(g.get("tuv")), _ptr(g.get("tvv"))
    s.normal = _ptr(g.get("normal"))
    s.sigma = _ptr(g.get("sigma"))
    return s


class SurfacePlan:
    """Geometry of a family of shapes sharing one set of RBF operators
    (bases::geometry<2>, include/bases/geometry.h:74-124).  ops: six CUDA
    float64 ns x nd tensors (evaluation -- or None when the samples are the
    data sites -- d/du, d/dv, d2/du2, d2/dudv, d2/dv2); weights: ns quadrature
    weights.  The tensors are kept alive by the plan."""

    def __init__(self, ops, weights):
        import torch
        self.ns = int(weights.numel())
        self.nd = int(ops[1].shape[1])
        # column-major ns x nd: the transpose of a row-major (ns, nd) tensor
        self._ops = [None if o is None else o.t().contiguous().t() for o in ops]
        self._weights = weights.contiguous()
        arr = (_vp * 6)(*[None if o is None else o.data_ptr() for o in self._ops])
        h = _vp()
        check(lib().ibk_surface_plan_create(self.ns, self.nd, arr, self._weights.data_ptr(), ctypes.byref(h)))
        self.handle = h
        self._torch = torch

    def geometry(self, x, nc, stream=None):
        """x: 3*nd*nc positions [component][shape][site]; returns a dict of
        position, tu, tv, tuu, tuv, tvv, normal (3*ns*nc) and sigma (ns*nc)."""
        torch = self._torch
        m = self.ns * nc
        g = {k: torch.empty(m if k == "sigma" else 3 * m, dtype=torch.float64, device=x.device)
             for k in _SURFACE_FIELDS}
        s = _surface_struct(g)
        check(lib().ibk_surface_geometry(self.handle, nc, x.data_ptr(), ctypes.byref(s), _stream_handle(stream)))
        return g

    def __del__(self):
        if getattr(self, "handle", None):
            lib().ibk_surface_plan_destroy(self.handle)
            self.handle = None


_CURVE_FIELDS = ("position", "tu", "tuu", "normal", "sigma")


class CurvePlan(SurfacePlan):
    """Geometry of a family of closed curves in a two-dimensional run
    (bases::geometry<1>): ops = three CUDA float64 ns x nd tensors
    (evaluation or None, d/ds, d2/ds2), weights: ns."""

    def __init__(self, ops, weights):
        import torch
        self.ns = int(weights.numel())
        self.nd = int(ops[1].shape[1])
        self._ops = [None if o is None else o.t().contiguous().t() for o in ops]
        self._weights = weights.contiguous()
        arr = (_vp * 3)(*[None if o is None else o.data_ptr() for o in self._ops])
        h = _vp()
        check(lib().ibk_curve_plan_create(self.ns, self.nd, arr, self._weights.data_ptr(), ctypes.byref(h)))
        self.handle = h
        self._torch = torch

    def geometry(self, x, nc, stream=None):
        """x: 2*nd*nc positions [component][curve][site]; returns a dict of
        position, tu, tuu, normal (2*ns*nc) and sigma (ns*nc)."""
        torch = self._torch
        m = self.ns * nc
        g = {k: torch.empty(m if k == "sigma" else 2 * m, dtype=torch.float64, device=x.device)
             for k in _CURVE_FIELDS}
        s = _surface_struct(g)
        check(lib().ibk_surface_geometry(self.handle, nc, x.data_ptr(), ctypes.byref(s), _stream_handle(stream)))
        return g


def curve_tension(law, shear, bulk, rest, current, stream=None):
    """One-dimensional tension (forces::tension1d with skalak1d or
    hookean1d, include/forces/tension.h:160-200) from rest and current curve
    geometry dicts; returns 2*npoints forces [component][site]."""
    import torch
    n = int(rest["sigma"].numel())
    f = torch.empty(2 * n, dtype=torch.float64, device=rest["sigma"].device)
    r, c = _surface_struct(rest), _surface_struct(current)
    check(lib().ibk_curve_tension(law, shear, bulk, n, ctypes.byref(r), ctypes.byref(c), f.data_ptr(),
                                  _stream_handle(stream)))
    return f


def membrane_tension(law, shear, bulk, rest, current, stream=None):
    """Tension force at every sample site (forces::tension with the Skalak,
    neo-Hookean or Hookean law, include/forces/tension.h:55-116) from the
    rest and current geometry dicts; returns 3*npoints forces
    [component][site]."""
    import torch
    n = int(rest["sigma"].numel())
    f = torch.empty(3 * n, dtype=torch.float64, device=rest["sigma"].device)
    r, c = _surface_struct(rest), _surface_struct(current)
    check(lib().ibk_membrane_tension(law, shear, bulk, n, ctypes.byref(r), ctypes.byref(c), f.data_ptr(),
                                     _stream_handle(stream)))
    return f


def membrane_bending(data_plan, sample_plan, modulus, preferred, x_rest, x_current, rest, current, nc,
                     stream=None):
    """Bending force at every sample (forces::bending,
    include/forces/bending.h:145-229): data_plan holds the shape family's
    operators at its data sites, sample_plan those at its samples; rest /
    current are sample geometry dicts (SurfacePlan.geometry), x_rest /
    x_current the data-site positions.  Returns 3*ns*nc forces."""
    import torch
    n = sample_plan.ns * nc
    f = torch.empty(3 * n, dtype=torch.float64, device=x_current.device)
    r = _surface_struct(rest) if rest is not None else None
    c = _surface_struct(current)
    check(lib().ibk_membrane_bending(data_plan.handle, sample_plan.handle, modulus, int(bool(preferred)), nc,
                                     _ptr(x_rest), x_current.data_ptr(), ctypes.byref(r) if r is not None else None,
                                     ctypes.byref(c), f.data_ptr(), _stream_handle(stream)))
    return f


def membrane_dissipation(sample_plan, modulus, u, current, nc, stream=None):
    """Viscous dissipation at every sample (forces::dissipation,
    include/forces/dissipation.h:128-272): u is the data-site velocity
    (3*nd*nc, [component][shape][site]), current the sample geometry dict;
    returns 3*ns*nc forces."""
    import torch
    f = torch.empty(3 * sample_plan.ns * nc, dtype=torch.float64, device=u.device)
    c = _surface_struct(current)
    check(lib().ibk_membrane_dissipation(sample_plan.handle, modulus, nc, u.data_ptr(), ctypes.byref(c),
                                         f.data_ptr(), _stream_handle(stream)))
    return f


def membrane_tether(modulus, rest, current, stream=None):
    """Tether force modulus (rest position - current position) at every
    sample (forces::tether, include/forces/tether.h:9-26)."""
    import torch
    n = int(current["position"].numel()) // 3
    f = torch.empty(3 * n, dtype=torch.float64, device=current["position"].device)
    r, c = _surface_struct(rest), _surface_struct(current)
    check(lib().ibk_membrane_tether(modulus, n, ctypes.byref(r), ctypes.byref(c), f.data_ptr(),
                                    _stream_handle(stream)))
    return f


REPELLING_HEIGHT, REPELLING_RANGE = 1.6, 0.025     # 16 um and 0.25 um in units of 10 um


def membrane_repelling(modulus, current, height=REPELLING_HEIGHT, range_=REPELLING_RANGE, stream=None):
    """Repulsion from the wall y = height (forces::repelling,
    include/forces/repelling.h:9-49), reaching 2 range from it, at every
    sample of the current geometry dict (position and sigma read)."""
    import torch
    n = int(current["sigma"].numel())
    f = torch.empty(3 * n, dtype=torch.float64, device=current["sigma"].device)
    c = _surface_struct(current)
    check(lib().ibk_membrane_repelling(modulus, height, range_, n, ctypes.byref(c), f.data_ptr(),
                                       _stream_handle(stream)))
    return f


# ------------------------------------------- the fluid step: implicit diffusion
DIRICHLET, NEUMANN = (1.0, 0.0), (0.0, 1.0)    # Robin (a, b) of a wall: a u + b du/dn
CHEBYSHEV, JACOBI = 0, 1                        # ibk_preconditioner


class Diffusion:
    """ins::diffusion (include/ins/diffusion.h:12-78) on one component grid
    of a plan: step(u, rhs, f, gamma) = u + (I~ - lambda L)^-1 (k I~ f +
    k mu (L u + rhs)), k = gamma * timestep, lambda = timestep * mu / 2.
    robin[axis] = ((a, b) lower wall, (a, b) upper wall), ignored on periodic
    axes; default Dirichlet walls.  preconditioner: CHEBYSHEV (the
    reference's, the default) or JACOBI."""

    def __init__(self, plan, component, timestep, mu, tolerance=1e-11, max_iterations=10000, robin=None,
                 preconditioner=None):
        if robin is None:
            robin = [(DIRICHLET, DIRICHLET)] * 3
        flat = (ctypes.c_double * 12)(*[float(v) for axis in robin for side in axis for v in side])
        h = _vp()
        check(lib().ibk_diffusion_create(plan.handle, int(component), flat, float(timestep), float(mu),
                                         float(tolerance), int(max_iterations), ctypes.byref(h)))
        self.handle = h
        self.size = int(plan.info.size[component])
        self.iterations = 0
        if preconditioner is not None:
            check(lib().ibk_diffusion_set_preconditioner(self.handle, int(preconditioner)))

    def info(self):
        """(Gershgorin interval (lower, upper) of I~ - lambda L, the four
        Chebyshev weights)."""
        b = (ctypes.c_double * 2)()
        w = (ctypes.c_double * 4)()
        check(lib().ibk_diffusion_info(self.handle, b, w))
        return (b[0], b[1]), list(w)

    def apply(self, op, u, stream=None):
        """op 0: L u, 1: I~ u, 2: (I~ - lambda L) u."""
        import torch
        out = torch.empty(self.size, dtype=torch.float64, device=u.device)
        check(lib().ibk_diffusion_apply(self.handle, int(op), u.data_ptr(), out.data_ptr(), _stream_handle(stream)))
        return out

    def step(self, u, rhs, f, gamma=1.0, stream=None):
        import torch
        out = torch.empty(self.size, dtype=torch.float64, device=u.device)
        it = ctypes.c_int()
        check(lib().ibk_diffusion_step(self.handle, float(gamma), u.data_ptr(), rhs.data_ptr(), f.data_ptr(),
                                       out.data_ptr(), ctypes.byref(it), _stream_handle(stream)))
        self.iterations = it.value
        return out

    def __del__(self):
        if getattr(self, "handle", None):
            lib().ibk_diffusion_destroy(self.handle)
            self.handle = None


# ------------------------------------------------------- linalg::io files
def io_write(path, objects):
    """Write numpy arrays / floats to one file in the reference's binary
    format: 1-D arrays as vectors, 2-D arrays (n x m) as column-major
    matrices, Python floats as raw FP64 scalars."""
    import numpy as np
    for k, obj in enumerate(objects):
        append = 1 if k else 0
        if isinstance(obj, float):
            check(lib().ibk_io_write_scalar(os.fsencode(path), append, obj))
            continue
        a = np.asarray(obj, dtype=np.float64)
        if a.ndim == 1:
            v = np.ascontiguousarray(a)
            check(lib().ibk_io_write_dense(os.fsencode(path), append, 0, a.shape[0], 1, v.ctypes.data))
        elif a.ndim == 2:
            v = np.ascontiguousarray(a.T)          # column-major values
            check(lib().ibk_io_write_dense(os.fsencode(path), append, 1, a.shape[0], a.shape[1],
                                           v.ctypes.data))
        else:
            raise ValueError("only vectors and matrices")


def io_write_sparse(path, obj, append=False):
    """Write one sparse container in the reference's binary format: a
    scipy.sparse matrix (CSR), or a sparse vector given as (size, indices,
    values)."""
    import numpy as np
    if isinstance(obj, tuple):
        n, idx, val = obj
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        check(lib().ibk_io_write_sparse(os.fsencode(path), int(bool(append)), 0, int(n), 1, idx.size, None,
                                        idx.ctypes.data, val.ctypes.data))
        return
    m = obj.tocsr()
    starts = np.ascontiguousarray(m.indptr, dtype=np.int32)
    idx = np.ascontiguousarray(m.indices, dtype=np.int32)
    val = np.ascontiguousarray(m.data, dtype=np.float64)
    check(lib().ibk_io_write_sparse(os.fsencode(path), int(bool(append)), 1, m.shape[0], m.shape[1], idx.size,
                                    starts.ctypes.data, idx.ctypes.data, val.ctypes.data))


def _read_sparse(path, off):
    import numpy as np
    import scipy.sparse as sp
    h = IoHeader()
    check(lib().ibk_io_read_sparse(os.fsencode(path), off, ctypes.byref(h), None, None, None, 0, None))
    starts = np.empty(h.rows + 1 if h.matrix and h.rows > 0 else 1, dtype=np.int32)
    idx = np.empty(max(h.count, 1), dtype=np.int32)
    val = np.empty(max(h.count, 1), dtype=np.float64)
    nxt = ctypes.c_longlong()
    check(lib().ibk_io_read_sparse(os.fsencode(path), off, ctypes.byref(h), starts.ctypes.data, idx.ctypes.data,
                                   val.ctypes.data, idx.size, ctypes.byref(nxt)))
    idx, val = idx[:h.count], val[:h.count]
    if h.matrix:
        indptr = starts if h.rows > 0 else np.zeros(1, dtype=np.int32)
        obj = sp.csr_matrix((val, idx, indptr), shape=(h.rows, h.cols))
    else:
        obj = (h.rows, idx, val)
    return obj, nxt.value


def io_read(path, count=None):
    """Read consecutive containers: dense vectors as 1-D arrays, dense
    matrices as (rows, cols) arrays (values column-major in the file),
    sparse matrices as scipy.sparse CSR matrices and sparse vectors as
    (size, indices, values)."""
    import numpy as np
    out, off = [], 0
    size = os.path.getsize(path)
    while off < size and (count is None or len(out) < count):
        with open(path, "rb") as fh:
            fh.seek(off)
            magic = int.from_bytes(fh.read(4), "little")
        if magic & 0xff00 == 0x7300:            # sparse layout
            obj, off = _read_sparse(path, off)
            out.append(obj)
            continue
        h = IoHeader()
        check(lib().ibk_io_read_dense(os.fsencode(path), off, ctypes.byref(h), None, 0, None))
        buf = np.empty(max(h.count, 1), dtype=np.float64)
        nxt = ctypes.c_longlong()
        check(lib().ibk_io_read_dense(os.fsencode(path), off, ctypes.byref(h), buf.ctypes.data, buf.size,
                                      ctypes.byref(nxt)))
        buf = buf[:h.count]
        out.append(buf.reshape(h.cols, h.rows).T.copy() if h.matrix else buf)
        off = nxt.value
    return out
