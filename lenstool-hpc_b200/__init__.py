"""lenstool-hpc_b200 -- B200-native lensing-map hot path of Lenstool-HPC.

Python host mirror of the C ABI in include/lt_b200.h (library liblt_b200.so built by
build.py).  There is no CPU fallback: every call runs the CUDA kernels, and importing the
bindings fails loudly when the library is missing.

Reference-named wrappers at the bottom (gradient_grid_GPU, gradient2_grid_GPU,
map_grid_ampli_GPU, ...) take the same arguments as the reference's host functions
(src/grid_gradient_GPU.cuh:34-36, src/grid_gradient2_GPU.cuh:32-34,
src/grid_map_*_GPU.cuh) with a HaloCatalog in place of Potential_SOA.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from . import catalog, cosmo  # noqa: F401
from .catalog import Grid, HaloCatalog  # noqa: F401

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "liblt_b200.so"

# lt_status
STATUS = {0: "LT_OK", 1: "LT_ERR_INVALID_ARGUMENT", 2: "LT_ERR_UNKNOWN_PROFILE", 3: "LT_ERR_NONFINITE",
          4: "LT_ERR_CUDA", 5: "LT_ERR_OUT_OF_MEMORY", 6: "LT_ERR_BUDGET", 7: "LT_ERR_QUEUE_FULL",
          8: "LT_ERR_TIMEOUT", 9: "LT_ERR_NO_DEVICE", 10: "LT_ERR_NOT_READY"}
FP64, FP32C, FP64_FAST = 0, 1, 2
PRECISION = {"fp64": FP64, "fp32c": FP32C, "fp64fast": FP64_FAST, FP64: FP64, FP32C: FP32C, FP64_FAST: FP64_FAST}

# lt_map_kind
MAP = {"hess_a": 0, "hess_b": 1, "hess_c": 2, "hess_d": 3,
       "ampli1": 11, "ampli2": 12, "ampli3": 13, "ampli4": 14, "ampli5": 15, "ampli6": 16,
       "shear1": 21, "shear2": 22, "shear3": 23, "shear4": 24,
       "kappa": 31, "gamma1": 32, "gamma2": 33, "mu": 34, "mass": 41,
       # batch and serving requests only
       "potential": 51, "deflection_x": 61, "deflection_y": 62}
MAX_MAPS = 8

# physical constants of src/structure_hpc.hpp:62-73
CH2PIG = 0.11585881
CH4PIG = 0.057929405
CH0_4PIG = 2.7730112e-4
MCRIT12 = .2343165

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class LensError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {message}" if message else self.name)


class _Soa(C.Structure):
    _fields_ = [("nhalos", C.c_int32), ("type", _ip)] + [(f, _dp) for f in (
        "position_x", "position_y", "b0", "anglecos", "anglesin", "ellipticity_potential", "rcore", "rcut",
        "dlsds")]


class _Grid(C.Structure):
    _fields_ = [("xmin", C.c_double), ("ymin", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("nx", C.c_int32), ("ny", C.c_int32), ("istart", C.c_int32), ("jstart", C.c_int32)]


class _MapReq(C.Structure):
    _fields_ = [("kind", C.c_int32), ("out", C.c_void_p)]


class _Request(C.Structure):
    _fields_ = [("cat", C.c_void_p), ("grid", _Grid), ("kmap", C.c_int32), ("dlsds", C.c_double),
                ("mult", C.c_double), ("scale", C.c_double), ("nmaps", C.c_int32), ("maps", _MapReq * 8)]


class _ServerConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("slots", C.c_int32), ("window", C.c_int32), ("idle_us", C.c_int32),
                ("output_bytes", C.c_size_t), ("descriptor_wait_us", C.c_int32)]


class _ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("failed", C.c_uint64), ("loop_launches", C.c_uint64), ("max_inflight", C.c_int32),
                ("inflight", C.c_int32), ("queued", C.c_int32), ("loop_running", C.c_int32),
                ("arena_bytes", C.c_size_t), ("arena_peak", C.c_size_t), ("device_published", C.c_uint64),
                ("device_head", C.c_uint64), ("timed_out", C.c_uint64)]


class _HaloParams(C.Structure):
    _fields_ = [("nhalos", C.c_int32)] + [(f, _dp) for f in (
        "position_x", "position_y", "vdisp", "ellipticity", "ellipticity_angle", "rcore", "rcut", "anglecos",
        "anglesin")]


class _BayesModel(C.Structure):
    _fields_ = [("nhalos", C.c_int32), ("type", _ip)] + [(f, _dp) for f in (
        "position_x", "position_y", "ellipticity_potential", "ellipticity", "ellipticity_angle", "rcore", "vdisp",
        "rcut", "mag")]


class _Potfile(C.Structure):
    _fields_ = [("first", C.c_int32), ("count", C.c_int32)] + [(f, C.c_double) for f in (
        "mag0", "sigma", "cut", "core", "vdslope", "slope")]


class _Frame(C.Structure):
    _fields_ = [("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double)]


class _Systems(C.Structure):
    _fields_ = [("nsystems", C.c_int32), ("nimages", _ip), ("x", _dp), ("y", _dp), ("dlsds", _dp)]


MAX_IMAGES = 20


class _KernelConfig(C.Structure):
    _fields_ = [("pixels_per_thread", C.c_int32), ("ctas_per_sm", C.c_int32), ("threads", C.c_int32),
                ("chunk", C.c_int32)]


class _Cosmo(C.Structure):
    _fields_ = [("model", C.c_int32), ("omegaM", C.c_double), ("omegaX", C.c_double), ("curvature", C.c_double),
                ("wX", C.c_double), ("wa", C.c_double), ("H0", C.c_double)]


_LIB = None

# every symbol the C ABI exports (include/lt_b200.h)
EXPORTS = ("lt_create", "lt_destroy", "lt_catalog_upload", "lt_catalog_release", "lt_catalog_nhalos",
           "lt_gradient_grid", "lt_hessian_maps", "lt_potential_grid", "lt_lens_maps", "lt_synchronize",
           "lt_cosmo_distances", "lt_kernel_launch_count", "lt_status_string", "lt_last_error", "lt_abi_version",
           "lt_set_kernel_shape", "lt_get_kernel_shape", "lt_set_kernel_config", "lt_get_kernel_config",
           "lt_autotune", "lt_measure_fma_peak", "lt_set_pass_timing", "lt_pass_times", "lt_recompute_count",
           "lt_batch_create", "lt_batch_launch", "lt_batch_size", "lt_batch_config", "lt_batch_destroy",
           "lt_server_create",
           "lt_server_submit", "lt_server_poll", "lt_server_wait", "lt_server_request_times", "lt_server_release",
           "lt_server_get_stats", "lt_server_destroy", "lt_chi2", "lt_chi2_batch", "lt_delense",
           "lt_catalog_update", "lt_write_fits", "lt_eval_fast_math", "lt_eval_fast_math32",
           "lt_eval_approx32",
           "lt_bayes_create",
           "lt_bayes_apply", "lt_bayes_destroy", "lt_chi2_batch_precision", "lt_server_submit_chi2",
           "lt_server_chi2_result", "lt_server_inject_fault")
SUMS = {"deflection": 1, "hessian": 2, "potential": 4, "lens": 6}


def load_library(path=None):
    """Load liblt_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python lenstool-hpc_b200/build.py`")
    L = C.CDLL(str(p))
    vp = C.c_void_p
    L.lt_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(vp)]
    L.lt_destroy.argtypes = [vp]
    L.lt_catalog_upload.argtypes = [vp, C.POINTER(_Soa), C.POINTER(vp)]
    L.lt_catalog_release.argtypes = [vp, vp]
    L.lt_catalog_nhalos.argtypes = [vp]
    L.lt_gradient_grid.argtypes = [vp, vp, C.POINTER(_Grid), C.c_int32, C.c_double, vp, vp, vp]
    L.lt_hessian_maps.argtypes = [vp, vp, C.POINTER(_Grid), C.c_int32, C.c_int32, C.c_double, C.c_double,
                                  C.POINTER(_MapReq), C.c_int32, vp]
    L.lt_potential_grid.argtypes = [vp, vp, C.POINTER(_Grid), C.c_int32, C.c_double, vp, vp]
    L.lt_lens_maps.argtypes = [vp, vp, C.POINTER(_Grid), C.c_int32, C.c_double, vp, vp, vp, vp, vp, vp]
    L.lt_synchronize.argtypes = [vp, vp]
    L.lt_cosmo_distances.argtypes = [C.POINTER(_Cosmo), C.c_double, C.c_double, _dp, _dp, _dp]
    L.lt_set_kernel_shape.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.lt_get_kernel_shape.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.lt_set_kernel_config.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(_KernelConfig)]
    L.lt_get_kernel_config.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(_KernelConfig)]
    L.lt_autotune.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    L.lt_set_pass_timing.argtypes = [vp, C.c_int32]
    L.lt_pass_times.argtypes = [vp, _dp, _dp, _ip]
    L.lt_recompute_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.lt_measure_fma_peak.argtypes = [C.c_int, C.c_int]
    L.lt_measure_fma_peak.restype = C.c_double
    L.lt_batch_create.argtypes = [vp, C.POINTER(_Request), C.c_int32, C.c_int32, C.POINTER(vp)]
    L.lt_batch_launch.argtypes = [vp, vp, vp]
    L.lt_batch_size.argtypes = [vp]
    L.lt_batch_config.argtypes = [vp, C.POINTER(_KernelConfig)]
    L.lt_batch_destroy.argtypes = [vp, vp]
    L.lt_server_create.argtypes = [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]
    L.lt_server_submit.argtypes = [vp, C.POINTER(_Request), C.POINTER(C.c_uint64)]
    L.lt_server_poll.argtypes = [vp, C.c_uint64]
    L.lt_server_wait.argtypes = [vp, C.c_uint64, C.c_double]
    L.lt_server_request_times.argtypes = [vp, C.c_uint64, _dp, _dp, _dp]
    L.lt_server_release.argtypes = [vp, C.c_uint64]
    L.lt_server_get_stats.argtypes = [vp, C.POINTER(_ServerStats)]
    L.lt_server_destroy.argtypes = [vp]
    L.lt_server_inject_fault.argtypes = [vp, C.c_int32]
    L.lt_server_submit_chi2.argtypes = [vp, vp, C.POINTER(_Frame), C.c_int32, C.POINTER(_Systems),
                                        C.POINTER(C.c_uint64)]
    L.lt_server_chi2_result.argtypes = [vp, C.c_uint64, _dp, _ip]
    L.lt_catalog_update.argtypes = [vp, vp, C.POINTER(_HaloParams), vp]
    L.lt_bayes_create.argtypes = [vp, C.POINTER(_BayesModel), C.c_int32, C.POINTER(_Potfile), C.c_int32, _ip,
                                  C.POINTER(vp)]
    L.lt_bayes_apply.argtypes = [vp, vp, _dp, C.c_int32, C.POINTER(vp), vp]
    L.lt_bayes_destroy.argtypes = [vp, vp]
    L.lt_chi2.argtypes = [vp, vp, C.POINTER(_Frame), C.c_int32, C.POINTER(_Systems), _dp, _ip]
    L.lt_chi2_batch.argtypes = [vp, C.POINTER(vp), C.c_int32, C.POINTER(_Frame), C.c_int32, C.POINTER(_Systems), _dp,
                                _ip]
    L.lt_chi2_batch_precision.argtypes = [vp, C.POINTER(vp), C.c_int32, C.POINTER(_Frame), C.c_int32,
                                          C.POINTER(_Systems), C.c_int32, _dp, _ip]
    L.lt_delense.argtypes = [vp, vp, C.POINTER(_Frame), C.c_int32, C.c_int32, _dp, _dp, _dp, _ip, _dp, _dp]
    L.lt_kernel_launch_count.restype = C.c_uint64
    L.lt_status_string.restype = C.c_char_p
    L.lt_status_string.argtypes = [C.c_int]
    L.lt_last_error.restype = C.c_char_p
    L.lt_last_error.argtypes = [vp]
    if path is None:
        _LIB = L
    return L


def launch_count() -> int:
    """Kernels launched by the library in this process."""
    return int(load_library().lt_kernel_launch_count())


def cosmo_distances(zl: float, zs: float, cosmology: "cosmo.Cosmology | None" = None):
    """(D_LS, D_OS, D_OL) in units of c/H0, computed by the library (host only)."""
    c = cosmology or cosmo.Cosmology()
    s = _Cosmo(c.model, c.omegaM, c.omegaX, c.curvature, c.wX, c.wa, c.H0)
    a, b, d = C.c_double(), C.c_double(), C.c_double()
    st = load_library().lt_cosmo_distances(C.byref(s), zl, zs, C.byref(a), C.byref(b), C.byref(d))
    if st:
        raise LensError(st, "cosmology")
    return a.value, b.value, d.value


def _grid(g: Grid) -> _Grid:
    return _Grid(g.xmin, g.ymin, g.dx, g.dy, g.nx, g.ny, g.istart, g.jstart)


def _ptr(x):
    """(address, keep-alive) of a numpy array or a torch tensor."""
    if isinstance(x, np.ndarray):
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("output arrays must be C-contiguous float64")
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        if str(x.dtype) != "torch.float64" or not x.is_contiguous():
            raise ValueError("output tensors must be contiguous float64")
        return x.data_ptr()
    raise TypeError(f"unsupported output type {type(x)}")


def _stream_handle(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)


class Catalog:
    """A catalogue resident in HBM (lt_catalog handle)."""

    def __init__(self, ctx: "Context", handle, nhalos: int, source: HaloCatalog):
        self.ctx, self.handle, self.nhalos, self.source = ctx, handle, nhalos, source

    def release(self):
        if self.handle:
            self.ctx._lib.lt_catalog_release(self.ctx.handle, self.handle)
            self.handle = None

    def update(self, position_x, position_y, vdisp, ellipticity, ellipticity_angle, rcore, rcut, anglecos=None,
               anglesin=None, stream=None):
        """lt_catalog_update: re-derive this resident catalogue from a new sample's physical
        parameters (catalogue halo order; numpy arrays or all torch CUDA tensors)."""
        arrs = [position_x, position_y, vdisp, ellipticity, ellipticity_angle, rcore, rcut]
        trig = [anglecos, anglesin] if anglecos is not None and anglesin is not None else [None, None]
        for a in arrs + trig:
            if a is not None and (a.shape[0] if hasattr(a, "shape") else len(a)) != self.nhalos:
                raise LensError(1, f"lt_catalog_update: {self.nhalos} halos expected")
        keep, ptrs = [], []
        for a in arrs + trig:
            if a is None:
                ptrs.append(None)
            elif hasattr(a, "data_ptr"):
                keep.append(a)
                ptrs.append(C.cast(C.c_void_p(a.data_ptr()), _dp))
            else:
                a = np.ascontiguousarray(a, np.float64)
                keep.append(a)
                ptrs.append(a.ctypes.data_as(_dp))
        p = _HaloParams(self.nhalos, *ptrs)
        st = self.ctx._lib.lt_catalog_update(self.ctx.handle, self.handle, C.byref(p), _stream_handle(stream))
        self.ctx._check(st, "lt_catalog_update")
        self._keep = keep

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Context:
    """lt_context: one device, an HBM budget, resident catalogues."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        st = self._lib.lt_create(device, budget_bytes, C.byref(h))
        if st:
            raise LensError(st, "lt_create")
        self.handle = h

    def close(self):
        if self.handle:
            self._lib.lt_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st:
            msg = self._lib.lt_last_error(self.handle).decode()
            raise LensError(st, f"{what}: {msg}")

    def upload(self, cat: HaloCatalog) -> Catalog:
        c = cat.contiguous()
        keep = c.arrays()
        d = lambda a: a.ctypes.data_as(_dp)  # noqa: E731
        s = _Soa(c.n, c.type.ctypes.data_as(_ip), d(c.position_x), d(c.position_y), d(c.b0), d(c.anglecos),
                 d(c.anglesin), d(c.ellipticity_potential), d(c.rcore), d(c.rcut), d(c.dlsds))
        h = C.c_void_p()
        st = self._lib.lt_catalog_upload(self.handle, C.byref(s), C.byref(h))
        del keep
        self._check(st, "lt_catalog_upload")
        return Catalog(self, h, c.n, c)

    def _cat(self, cat):
        return cat if isinstance(cat, Catalog) else self.upload(cat)

    @staticmethod
    def _outs(grid: Grid, out, n):
        if out is None:
            return [np.empty((grid.ny, grid.nx)) for _ in range(n)]
        return list(out)

    def gradient_grid(self, cat, grid: Grid, precision="fp64", scale=1.0, out=None, stream=None):
        cat = self._cat(cat)
        ax, ay = self._outs(grid, out, 2)
        st = self._lib.lt_gradient_grid(self.handle, cat.handle, C.byref(_grid(grid)), PRECISION[precision], scale,
                                        _ptr(ax), _ptr(ay), _stream_handle(stream))
        self._check(st, "lt_gradient_grid")
        return ax, ay

    def hessian_maps(self, cat, grid: Grid, kinds, precision="fp64", kmap=False, dlsds=1.0, mult=1.0, out=None,
                     stream=None):
        cat = self._cat(cat)
        kinds = list(kinds)
        outs = self._outs(grid, out, len(kinds))
        req = (_MapReq * len(kinds))(*[_MapReq(MAP[k] if isinstance(k, str) else int(k), _ptr(o))
                                       for k, o in zip(kinds, outs)])
        st = self._lib.lt_hessian_maps(self.handle, cat.handle, C.byref(_grid(grid)), PRECISION[precision],
                                       int(bool(kmap)), dlsds, mult, req, len(kinds), _stream_handle(stream))
        self._check(st, "lt_hessian_maps")
        return dict(zip(kinds, outs))

    def potential_grid(self, cat, grid: Grid, precision="fp64", scale=1.0, out=None, stream=None):
        cat = self._cat(cat)
        (psi,) = self._outs(grid, None if out is None else [out], 1)
        st = self._lib.lt_potential_grid(self.handle, cat.handle, C.byref(_grid(grid)), PRECISION[precision], scale,
                                         _ptr(psi), _stream_handle(stream))
        self._check(st, "lt_potential_grid")
        return psi

    def lens_maps(self, cat, grid: Grid, precision="fp64", dlsds=1.0, out=None, stream=None,
                  which=("kappa", "gamma1", "gamma2", "mu", "psi")):
        """kappa, gamma1, gamma2, mu and psi*dlsds of one grid in one fused pass."""
        cat = self._cat(cat)
        names = ("kappa", "gamma1", "gamma2", "mu", "psi")
        if out is None:
            out = {k: np.empty((grid.ny, grid.nx)) for k in which}
        ptrs = [(_ptr(out[k]) if k in out else None) for k in names]
        st = self._lib.lt_lens_maps(self.handle, cat.handle, C.byref(_grid(grid)), PRECISION[precision], dlsds,
                                    *ptrs, _stream_handle(stream))
        self._check(st, "lt_lens_maps")
        return out

    def set_kernel_shape(self, precision, sums, pixels_per_thread, ctas_per_sm):
        st = self._lib.lt_set_kernel_shape(self.handle, PRECISION[precision], SUMS.get(sums, sums), pixels_per_thread,
                                           ctas_per_sm)
        self._check(st, "lt_set_kernel_shape")

    def kernel_shape(self, precision, sums):
        a, b = C.c_int32(), C.c_int32()
        st = self._lib.lt_get_kernel_shape(self.handle, PRECISION[precision], SUMS.get(sums, sums), C.byref(a),
                                           C.byref(b))
        self._check(st, "lt_get_kernel_shape")
        return a.value, b.value

    def set_kernel_config(self, precision, sums, pixels_per_thread, ctas_per_sm, threads=256, chunk=64):
        c = _KernelConfig(pixels_per_thread, ctas_per_sm, threads, chunk)
        st = self._lib.lt_set_kernel_config(self.handle, PRECISION[precision], SUMS.get(sums, sums), C.byref(c))
        self._check(st, "lt_set_kernel_config")

    def kernel_config(self, precision, sums) -> dict:
        c = _KernelConfig()
        st = self._lib.lt_get_kernel_config(self.handle, PRECISION[precision], SUMS.get(sums, sums), C.byref(c))
        self._check(st, "lt_get_kernel_config")
        return {f: getattr(c, f) for f, _ in _KernelConfig._fields_}

    def autotune(self, cat, precision="fp32c", sums="lens", grid_n=512):
        """Time every kernel configuration on a grid_n^2 grid over the catalogue; keep the
        fastest.  Returns (pixels_per_thread, ctas_per_sm, ms); kernel_config() gives the
        threads per CTA and the stage size too."""
        cat = self._cat(cat)
        ms = C.c_double()
        st = self._lib.lt_autotune(self.handle, cat.handle, PRECISION[precision], SUMS.get(sums, sums), grid_n,
                                   C.byref(ms))
        self._check(st, "lt_autotune")
        return self.kernel_shape(precision, sums) + (ms.value,)

    def set_pass_timing(self, on=True):
        self._check(self._lib.lt_set_pass_timing(self.handle, int(bool(on))), "lt_set_pass_timing")

    def pass_times(self):
        """(pass-1 ms, pass-2 ms, calls) summed over the FP32C calls since the last read."""
        a, b, n = C.c_double(), C.c_double(), C.c_int32()
        self._check(self._lib.lt_pass_times(self.handle, C.byref(a), C.byref(b), C.byref(n)), "lt_pass_times")
        return a.value, b.value, n.value

    def recompute_count(self):
        """Pixels of the FP32C calls recomputed in FP64 since the last read (lt_recompute_count)."""
        a = C.c_uint64()
        self._check(self._lib.lt_recompute_count(self.handle, C.byref(a)), "lt_recompute_count")
        return a.value

    def synchronize(self, stream=None):
        self._check(self._lib.lt_synchronize(self.handle, _stream_handle(stream)), "lt_synchronize")

    # ---- strong-lensing chi2 (frame = (xmin, xmax, ymin, ymax) of an n x n grid) ----

    def chi2(self, cats, frame, n, systems, precision="fp64"):
        """lt_chi2_batch_precision: chi2 of each catalogue (model) against `systems` (an
        images.ImageSystems), the deflection grid in `precision` ("fp64" or "fp32c"; the
        delensing and the chi2 are FP64).  Returns (chi2 array, predicted-image counts)."""
        single = not isinstance(cats, (list, tuple))
        cl = [self._cat(c) for c in ([cats] if single else cats)]
        s = systems.contiguous()
        sy = _Systems(s.nsys, s.nimg.ctypes.data_as(_ip), s.x.ctypes.data_as(_dp), s.y.ctypes.data_as(_dp),
                      s.dr.ctypes.data_as(_dp))
        handles = (C.c_void_p * len(cl))(*[c.handle.value if hasattr(c.handle, "value") else c.handle for c in cl])
        chi = np.empty(len(cl))
        found = np.empty(len(cl), np.int32)
        st = self._lib.lt_chi2_batch_precision(self.handle, handles, len(cl), C.byref(_Frame(*frame)), n,
                                               C.byref(sy), PRECISION[precision], chi.ctypes.data_as(_dp),
                                               found.ctypes.data_as(_ip))
        self._check(st, "lt_chi2_batch_precision")
        return (chi[0], int(found[0])) if single else (chi, found)

    def delense(self, cat, frame, n, bx, by, dlsds):
        """lt_delense: predicted images of the sources (bx, by, dlsds): (nfound, fx, fy)."""
        cat = self._cat(cat)
        bx, by, dr = (np.ascontiguousarray(np.broadcast_to(a, np.shape(bx)), np.float64) for a in (bx, by, dlsds))
        k = bx.size
        nf = np.zeros(k, np.int32)
        fx = np.zeros((k, MAX_IMAGES))
        fy = np.zeros((k, MAX_IMAGES))
        st = self._lib.lt_delense(self.handle, cat.handle, C.byref(_Frame(*frame)), n, k, bx.ctypes.data_as(_dp),
                                  by.ctypes.data_as(_dp), dr.ctypes.data_as(_dp), nf.ctypes.data_as(_ip),
                                  fx.ctypes.data_as(_dp), fy.ctypes.data_as(_dp))
        self._check(st, "lt_delense")
        return nf, fx, fy

    def batch(self, requests, precision="fp32c") -> "Batch":
        """lt_batch_create: `requests` are Request objects with device outputs."""
        reqs = list(requests)
        arr = (_Request * len(reqs))(*[r.to_c(self) for r in reqs])
        h = C.c_void_p()
        st = self._lib.lt_batch_create(self.handle, arr, len(reqs), PRECISION[precision], C.byref(h))
        self._check(st, "lt_batch_create")
        return Batch(self, h, reqs)

    def server(self, precision="fp32c", slots=0, window=0, idle_us=0, output_bytes=0,
               descriptor_wait_us=0) -> "Server":
        """lt_server_create: a continuous-batching serving loop on this context."""
        return Server(self, precision, slots, window, idle_us, output_bytes, descriptor_wait_us)

    def bayes(self, model, columns, potfiles=()) -> "Bayes":
        """lt_bayes_create: a bayes.dat model (bayes.BayesModel), its potfiles
        (bayes.Potfile) and the meaning of each row column ((field, target) pairs)."""
        return Bayes(self, model, columns, potfiles)


class Bayes:
    """lt_bayes: bayes.dat rows applied to resident catalogues on the device."""

    def __init__(self, ctx: Context, model, columns, potfiles=()):
        self.ctx, self.handle = ctx, None
        arrs = model.arrays()
        self._keep = [a for a in arrs if a is not None]
        t, *planes, mag = arrs
        m = _BayesModel(model.n, t.ctypes.data_as(_ip), *[a.ctypes.data_as(_dp) for a in planes],
                        None if mag is None else mag.ctypes.data_as(_dp))
        pots = list(potfiles)
        parr = (_Potfile * max(1, len(pots)))(*[_Potfile(p.first, p.count, p.mag0, p.sigma, p.cut, p.core, p.vdslope,
                                                         p.slope) for p in pots])
        cols = np.ascontiguousarray(np.asarray(columns, np.int32).reshape(-1, 2))
        self.ncolumns, self.nhalos = cols.shape[0], model.n
        h = C.c_void_p()
        st = ctx._lib.lt_bayes_create(ctx.handle, C.byref(m), len(pots), parr, cols.shape[0],
                                      cols.ctypes.data_as(_ip), C.byref(h))
        ctx._check(st, "lt_bayes_create")
        self.handle = h

    def apply(self, rows, cats, stream=None):
        """Row r of `rows` (numpy nrows x ncolumns, or a torch CUDA tensor) re-derives cats[r]."""
        cats = list(cats)
        if hasattr(rows, "data_ptr"):
            if tuple(rows.shape) != (len(cats), self.ncolumns) or not rows.is_contiguous():
                raise LensError(1, "lt_bayes_apply: rows must be contiguous (len(cats), ncolumns)")
            keep, ptr = rows, C.cast(C.c_void_p(rows.data_ptr()), _dp)
        else:
            keep = np.ascontiguousarray(rows, np.float64).reshape(-1, self.ncolumns)
            if keep.shape[0] != len(cats):
                raise LensError(1, "lt_bayes_apply: one row per catalogue")
            ptr = keep.ctypes.data_as(_dp)
        handles = (C.c_void_p * max(1, len(cats)))(*[c.handle for c in cats])
        st = self.ctx._lib.lt_bayes_apply(self.ctx.handle, self.handle, ptr, len(cats), handles,
                                          _stream_handle(stream))
        self.ctx._check(st, "lt_bayes_apply")
        self._rows = keep

    def destroy(self):
        if self.handle:
            self.ctx._lib.lt_bayes_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Request:
    """lt_request: one grid of output planes over one catalogue (batch / serving).

    maps: {kind name or lt_map_kind: output array/tensor}."""

    def __init__(self, cat, grid: Grid, maps, dlsds=1.0, kmap=False, mult=1.0, scale=1.0):
        self.cat, self.grid, self.maps = cat, grid, dict(maps)
        self.dlsds, self.kmap, self.mult, self.scale = dlsds, kmap, mult, scale
        if not 1 <= len(self.maps) <= MAX_MAPS:
            raise ValueError(f"a request has 1..{MAX_MAPS} maps")

    def to_c(self, ctx: "Context") -> _Request:
        cat = ctx._cat(self.cat)
        self._cat_keep = cat
        r = _Request()
        r.cat = cat.handle
        r.grid = _grid(self.grid)
        r.kmap = int(bool(self.kmap))
        r.dlsds, r.mult, r.scale = self.dlsds, self.mult, self.scale
        r.nmaps = len(self.maps)
        for i, (k, o) in enumerate(self.maps.items()):
            r.maps[i] = _MapReq(MAP[k] if isinstance(k, str) else int(k), _ptr(o))
        return r


class Batch:
    """lt_batch: requests evaluated by one graph-captured persistent launch."""

    def __init__(self, ctx: Context, handle, requests):
        self.ctx, self.handle, self.requests = ctx, handle, requests

    def __len__(self):
        return int(self.ctx._lib.lt_batch_size(self.handle))

    def config(self) -> dict:
        """lt_batch_config: the persistent kernel's shape for this batch."""
        c = _KernelConfig()
        self.ctx._check(self.ctx._lib.lt_batch_config(self.handle, C.byref(c)), "lt_batch_config")
        return {f: getattr(c, f) for f, _ in _KernelConfig._fields_}

    def launch(self, stream=None):
        self.ctx._check(self.ctx._lib.lt_batch_launch(self.ctx.handle, self.handle, _stream_handle(stream)),
                        "lt_batch_launch")

    def destroy(self):
        if self.handle:
            self.ctx._lib.lt_batch_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Server:
    """lt_server: continuous batching of map requests on one context."""

    def __init__(self, ctx: Context, precision="fp32c", slots=0, window=0, idle_us=0, output_bytes=0,
                 descriptor_wait_us=0):
        self.ctx, self._lib = ctx, ctx._lib
        cfg = _ServerConfig(PRECISION[precision], slots, window, idle_us, output_bytes, descriptor_wait_us)
        h = C.c_void_p()
        st = self._lib.lt_server_create(ctx.handle, C.byref(cfg), C.byref(h))
        ctx._check(st, "lt_server_create")
        self.handle = h
        self._keep = {}

    def submit(self, request: Request) -> int:
        r = request.to_c(self.ctx)
        t = C.c_uint64()
        st = self._lib.lt_server_submit(self.handle, C.byref(r), C.byref(t))
        self.ctx._check(st, "lt_server_submit")
        self._keep[t.value] = request
        return t.value

    def submit_chi2(self, cat, frame, n, systems) -> int:
        """lt_server_submit_chi2: the chi2 of the resident catalogue `cat` against `systems`
        (images.ImageSystems) on an n x n grid over `frame`; the result comes from
        chi2_result once the ticket completes."""
        s = systems.contiguous()
        sy = _Systems(s.nsys, s.nimg.ctypes.data_as(_ip), s.x.ctypes.data_as(_dp), s.y.ctypes.data_as(_dp),
                      s.dr.ctypes.data_as(_dp))
        t = C.c_uint64()
        st = self._lib.lt_server_submit_chi2(self.handle, cat.handle, C.byref(_Frame(*frame)), n, C.byref(sy),
                                             C.byref(t))
        self.ctx._check(st, "lt_server_submit_chi2")
        self._keep[t.value] = cat
        return t.value

    def chi2_result(self, ticket: int):
        """(chi2, predicted images) of a completed chi2 ticket."""
        chi, found = C.c_double(), C.c_int32()
        st = self._lib.lt_server_chi2_result(self.handle, ticket, C.byref(chi), C.byref(found))
        self.ctx._check(st, "lt_server_chi2_result")
        return chi.value, found.value

    def poll(self, ticket: int) -> bool:
        st = self._lib.lt_server_poll(self.handle, ticket)
        if st == 10:
            return False
        self.ctx._check(st, "lt_server_poll")
        return True

    def wait(self, ticket: int, timeout_s: float = 600.0):
        st = self._lib.lt_server_wait(self.handle, ticket, timeout_s)
        self.ctx._check(st, "lt_server_wait")

    def times(self, ticket: int):
        """(queued_ms, gpu_ms, total_ms) of a completed ticket."""
        q, g, t = C.c_double(), C.c_double(), C.c_double()
        st = self._lib.lt_server_request_times(self.handle, ticket, C.byref(q), C.byref(g), C.byref(t))
        self.ctx._check(st, "lt_server_request_times")
        return q.value, g.value, t.value

    def release(self, ticket: int):
        self._lib.lt_server_release(self.handle, ticket)
        self._keep.pop(ticket, None)

    def inject_fault(self, fault: int = 1):
        """lt_server_inject_fault (1: the next admitted request loses its descriptor)."""
        self.ctx._check(self._lib.lt_server_inject_fault(self.handle, fault), "lt_server_inject_fault")

    def stats(self) -> dict:
        s = _ServerStats()
        self.ctx._check(self._lib.lt_server_get_stats(self.handle, C.byref(s)), "lt_server_get_stats")
        return {f: getattr(s, f) for f, _ in _ServerStats._fields_}

    def close(self):
        if self.handle:
            self._lib.lt_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------
# Reference-named entry points (same argument meaning as the reference's host wrappers).
# ---------------------------------------------------------------------------------------

_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _frame_grid(frame, nbgridcells, nx=None, ny=None, dx=None, dy=None, istart=0, jstart=0) -> Grid:
    nx = nx or nbgridcells
    ny = ny or nbgridcells
    g = Grid(frame["xmin"], frame["xmax"], frame["ymin"], frame["ymax"], nx, ny, istart, jstart)
    if dx is not None:
        g.dx, g.dy = dx, dy
    return g


def gradient_grid_GPU(frame, lens: HaloCatalog, nbgridcells, **kw):
    """src/grid_gradient_GPU.cu:77-84: (grid_grad_x, grid_grad_y) over a square grid."""
    return default_context().gradient_grid(lens, _frame_grid(frame, nbgridcells, **kw))


def gradient2_grid_GPU(frame, lens: HaloCatalog, nbgridcells, **kw):
    """src/grid_gradient2_GPU.cu:77-183: the four Hessian planes (a, b, c, d)."""
    m = default_context().hessian_maps(lens, _frame_grid(frame, nbgridcells, **kw),
                                       ["hess_a", "hess_b", "hess_c", "hess_d"])
    return m["hess_a"], m["hess_b"], m["hess_c"], m["hess_d"]


def map_grid_ampli_GPU(mode, cosmology, frame, lens: HaloCatalog, nbgridcells, z, **kw):
    """src/grid_map_ampli_GPU.cu:93-192: amplification map mode 1-6 for sources at z."""
    if mode not in range(1, 7):
        raise LensError(1, f"amplification mode {mode} not supported")
    dls, dos, _ = cosmo_distances(lens.z, z, cosmology)
    k = f"ampli{mode}"
    return default_context().hessian_maps(lens, _frame_grid(frame, nbgridcells, **kw), [k], dlsds=dls / dos)[k]


def map_grid_shear_GPU(mode, cosmology, frame, lens: HaloCatalog, nbgridcells, z, **kw):
    """src/grid_map_shear_GPU.cu:87-187: shear map mode 1-4."""
    if mode not in range(1, 5):
        raise LensError(1, f"shear mode {mode} not supported")
    dls, dos, _ = cosmo_distances(lens.z, z, cosmology)
    k = f"shear{mode}"
    return default_context().hessian_maps(lens, _frame_grid(frame, nbgridcells, **kw), [k], dlsds=dls / dos)[k]


def mass_multiplier(mode, dl0s, ds, dl, h, dx, dy):
    """Unit factor of mass map modes 1-4 (src/grid_map_mass_GPU.cu:219-300)."""
    if mode == 1:
        return 1.
    if mode == 2:
        return CH4PIG * h / dl / dl0s * ds
    if mode == 3:
        return MCRIT12 / h * dx * dy * dl / dl0s * ds
    if mode == 4:
        return CH0_4PIG * h / dl / dl0s * ds
    raise LensError(1, f"mass mode {mode} not supported")


def map_grid_mass_GPU(mode, cosmology, frame, lens: HaloCatalog, nbgridcells, zl, zs, **kw):
    """src/grid_map_mass_GPU.cu:82-216: Kmap (per-halo dlsds weights) times the mode's unit."""
    c = cosmology or cosmo.Cosmology()
    zl = zl or lens.z
    dl0s, ds, dl = cosmo_distances(zl, zs, c)
    g = _frame_grid(frame, nbgridcells, **kw)
    mult = mass_multiplier(mode, dl0s, ds, dl, c.h, g.dx, g.dy)
    return default_context().hessian_maps(lens, g, ["mass"], kmap=True, mult=mult)["mass"]


def map_grid_potential_GPU(mode, cosmology, frame, lens: HaloCatalog, nbgridcells, z, **kw):
    """src/grid_map_pot_GPU.cu:83-273: potential mode 1 (x D_LS/D_OS) or 2 (x cH2piG h/D_OL)."""
    c = cosmology or cosmo.Cosmology()
    dl0s, ds, dl = cosmo_distances(lens.z, z, c)
    if mode == 1:
        scale = dl0s / ds
    elif mode == 2:
        scale = CH2PIG * c.h / dl
    else:
        raise LensError(1, f"potential mode {mode} not supported")
    return default_context().potential_grid(lens, _frame_grid(frame, nbgridcells, **kw), scale=scale)


def map_grid_dpl_GPU(cosmology, frame, lens: HaloCatalog, nbgridcells, z, **kw):
    """src/grid_map_dpl_GPU.cu:75-173: deflection x D_LS/D_OS, two planes."""
    dl0s, ds, _ = cosmo_distances(lens.z, z, cosmology)
    return default_context().gradient_grid(lens, _frame_grid(frame, nbgridcells, **kw), scale=dl0s / ds)
