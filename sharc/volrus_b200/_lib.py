"""ctypes binding of ``lib/libvolrus_b200.so`` (the C ABI in include/volrus_b200.h).

The library is loaded lazily on first use.  There is no fallback: if the
shared library is missing or a CUDA device is unavailable, calls raise.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libvolrus_b200.so"

VLR_OK = 0
ERROR_NAMES = {
    1: "VLR_ERR_INVALID", 2: "VLR_ERR_CUDA", 3: "VLR_ERR_CAPACITY", 4: "VLR_ERR_EXTENT",
    5: "VLR_ERR_REACH", 6: "VLR_ERR_NOMEM", 7: "VLR_ERR_FORMAT", 8: "VLR_ERR_TIMEOUT",
    9: "VLR_ERR_UNSUPPORTED",
}


class VolrusError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


class vlr_transform(C.Structure):
    _fields_ = [
        ("voxel_size", C.c_double),
        ("origin", C.c_double * 3),
        ("affine", C.c_double * 12),
        ("affine_voxel_size", C.c_double),
    ]


class vlr_velocity_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("constant", C.c_double * 3),
        ("voxel_size", C.c_double),
        ("w0", C.c_double * 3),
        ("period", C.c_double),
        ("octaves", C.c_int),
        ("amp", C.c_double * 4),
        ("wavenumber", C.c_double * 4),
        ("phase", (C.c_double * 3) * 4),
        ("dir", (C.c_double * 3) * 4),
        ("domain_lo", C.c_int32 * 3),
        ("domain_hi", C.c_int32 * 3),
    ]


class vlr_method_desc(C.Structure):
    _fields_ = [
        ("precision", C.c_int),
        ("half_width", C.c_float),
        ("integrator", C.c_int),
        ("reinit_iters", C.c_int),
        ("dt", C.c_double),
        ("t0", C.c_double),
        ("capacity", C.c_size_t),
        ("reinit_mode", C.c_int),
    ]


class vlr_sphere(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double)]


class vlr_batch_grid(C.Structure):
    _fields_ = [("spheres", C.POINTER(vlr_sphere)), ("n_spheres", C.c_int), ("velocity", vlr_velocity_desc)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
dbl_p = C.POINTER(C.c_double)
flt_p = C.POINTER(C.c_float)
i32_p = C.POINTER(C.c_int32)
u64_p = C.POINTER(C.c_uint64)
size_p = C.POINTER(C.c_size_t)

# name -> (restype, argtypes)
SIGNATURES = {
    "vlr_ctx_create": (C.c_int, [C.c_int, PP]),
    "vlr_ctx_destroy": (None, [P]),
    "vlr_last_error": (C.c_char_p, [P]),
    "vlr_ctx_synchronize": (C.c_int, [P]),
    "vlr_host_alloc": (C.c_int, [P, C.c_size_t, C.POINTER(C.c_void_p)]),
    "vlr_host_free": (C.c_int, [P, C.c_void_p]),
    "vlr_ctx_stream": (C.c_int, [P, PP]),
    "vlr_ctx_profile": (C.c_int, [P, C.c_int]),
    "vlr_ctx_profile_read": (C.c_int, [P, C.c_char_p, dbl_p, C.POINTER(C.c_longlong)]),
    "vlr_ctx_set_wait_limit": (C.c_int, [P, C.c_uint32]),
    "vlr_ctx_test_stall": (C.c_int, [P, C.c_int]),
    "vlr_grid_create": (C.c_int, [P, C.POINTER(vlr_transform), C.c_float, i32_p, u64_p, flt_p, C.c_size_t, PP]),
    "vlr_grid_create_device": (C.c_int, [P, C.POINTER(vlr_transform), C.c_float, P, P, P, C.c_size_t, PP]),
    "vlr_grid_info": (C.c_int, [P, P, size_p, C.POINTER(C.c_uint64), flt_p, C.POINTER(vlr_transform)]),
    "vlr_grid_download": (C.c_int, [P, P, i32_p, u64_p, flt_p, C.c_size_t]),
    "vlr_extend_velocity": (C.c_int, [P, P, P, P, P, C.c_float]),
    "vlr_advect_particles": (C.c_int, [P, P, P, P, dbl_p, C.c_size_t, C.c_double, C.c_int]),
    "vlr_advect_points": (C.c_int, [P, P, P, P, dbl_p, C.c_void_p, C.c_size_t, C.c_double, C.c_int, i32_p,
                                    C.POINTER(C.c_uint32), C.c_size_t, size_p]),
    "vlr_dilate": (C.c_int, [P, P, C.c_uint]),
    "vlr_flood_fill_sign": (C.c_int, [P, P]),
    "vlr_volume_to_mesh": (C.c_int, [P, P, C.c_float, dbl_p, C.c_size_t, C.POINTER(C.c_uint32), C.c_size_t, size_p,
                                     size_p]),
    "vlr_mc_triangle_table": (C.c_int, [C.POINTER(C.c_int8)]),
    "vlr_grid_from_vol": (C.c_int, [P, P, C.c_size_t, PP, C.POINTER(C.c_int)]),
    "vlr_grid_to_vol": (C.c_int, [P, P, C.c_int, P, C.c_size_t, size_p]),
    "vlr_grid_from_nano": (C.c_int, [P, P, C.c_size_t, PP, C.POINTER(C.c_int)]),
    "vlr_grid_to_nano": (C.c_int, [P, P, C.c_int, dbl_p, P, C.c_size_t, size_p]),
    "vlr_grid_destroy": (None, [P]),
    "vlr_make_level_set_sphere": (C.c_int, [P, C.c_double, dbl_p, C.c_double, C.c_double, PP]),
    "vlr_sample_trilinear": (C.c_int, [P, P, dbl_p, C.c_size_t, flt_p]),
    "vlr_advect_level_set": (C.c_int, [P, P, P, P, P, C.c_double, PP]),
    "vlr_find_zero_crossings": (C.c_int, [P, P, i32_p, C.c_size_t, size_p]),
    "vlr_find_zero_crossings_noalloc": (C.c_int, [P, P, C.c_void_p, C.c_size_t, C.c_void_p]),
    "vlr_trim_narrow_band": (C.c_int, [P, P, C.c_float]),
    "vlr_rebuild_narrow_band": (C.c_int, [P, P, C.c_float]),
    "vlr_advect_rebuild_host": (C.c_int, [P, C.POINTER(vlr_transform), C.c_float, i32_p, u64_p, flt_p, C.c_size_t,
                                          flt_p, C.c_double, C.c_float, i32_p, u64_p, flt_p, C.c_size_t, size_p]),
    "vlr_ls_create_sphere": (C.c_int, [P, C.POINTER(vlr_method_desc), C.POINTER(vlr_velocity_desc), C.c_double,
                                       dbl_p, C.c_double, dbl_p, PP]),
    "vlr_ls_create_from_leaves": (C.c_int, [P, C.POINTER(vlr_method_desc), C.POINTER(vlr_velocity_desc), i32_p, u64_p,
                                            flt_p, C.c_size_t, PP]),
    "vlr_ls_create_spheres": (C.c_int, [P, C.POINTER(vlr_method_desc), C.POINTER(vlr_batch_grid), C.c_int, PP]),
    "vlr_ls_download_grid": (C.c_int, [P, P, C.c_int, i32_p, i32_p, u64_p, flt_p, C.c_size_t, size_p]),
    "vlr_adj_create": (C.c_int, [P, i32_p, u64_p, flt_p, C.c_size_t, C.c_float, flt_p, C.c_int, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, PP]),
    "vlr_adj_band": (C.c_int, [P, P, i32_p, C.c_size_t, size_p]),
    "vlr_adj_create_level_set": (C.c_int, [P, P, C.c_int, C.c_int, PP]),
    "vlr_adj_displacement": (C.c_int, [P, P, flt_p]),
    "vlr_adj_shifted_phi0": (C.c_int, [P, P, C.c_int, C.c_int, C.c_int, P]),
    "vlr_adj_set_gather": (C.c_int, [P, P, C.c_int]),
    "vlr_adj_set_inputs": (C.c_int, [P, P, flt_p, flt_p]),
    "vlr_adj_forward": (C.c_int, [P, P, flt_p]),
    "vlr_adj_backward": (C.c_int, [P, P, flt_p, flt_p, flt_p]),
    "vlr_adj_forward_device": (C.c_int, [P, P, P]),
    "vlr_adj_backward_device": (C.c_int, [P, P, P, P, P]),
    "vlr_adj_destroy": (None, [P]),
    "vlr_ls_step": (C.c_int, [P, P, C.c_int]),
    "vlr_ls_enqueue": (C.c_int, [P, P, C.c_int]),
    "vlr_ls_set_launch_shape": (C.c_int, [P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "vlr_ls_get_launch_shape": (C.c_int, [P, P, C.POINTER(C.c_int), C.POINTER(C.c_int), flt_p, C.c_int]),
    "vlr_ctx_check": (C.c_int, [P]),
    "vlr_ls_step_host": (C.c_int, [P, P, i32_p, u64_p, flt_p, C.c_size_t, C.c_int, i32_p, u64_p, flt_p,
                                   C.c_size_t, size_p]),
    "vlr_ls_info": (C.c_int, [P, P, size_p, C.POINTER(C.c_uint64), dbl_p]),
    "vlr_ls_download": (C.c_int, [P, P, i32_p, u64_p, flt_p, C.c_size_t]),
    "vlr_ls_upload": (C.c_int, [P, P, i32_p, u64_p, flt_p, C.c_size_t]),
    "vlr_ls_set_step": (C.c_int, [P, P, C.c_int]),
    "vlr_ls_set_host_slabs": (C.c_int, [P, P, C.c_int]),
    "vlr_ls_volume_partials": (C.c_int, [P, P, dbl_p, P, C.c_size_t, size_p]),
    "vlr_ls_upload_device": (C.c_int, [P, P, P, P, P, C.c_size_t]),
    "vlr_ls_download_device": (C.c_int, [P, P, P, P, P, C.c_size_t, size_p]),
    "vlr_ls_gather_device": (C.c_int, [P, P, P, C.c_size_t, P, P, P]),
    "vlr_ls_edit_device": (C.c_int, [P, P, P, C.c_size_t, P, P, P, C.c_size_t]),
    "vlr_ls_volume": (C.c_int, [P, P, dbl_p, dbl_p]),
    "vlr_ls_destroy": (None, [P]),
}

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load the shared library and bind every declared entry point."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m sharc.volrus_b200.build` "
                    "(the CUDA path has no CPU fallback)")
            lib = C.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class _PinnedBlock:
    """A page-locked host allocation of a context, freed with the object."""

    def __init__(self, ctx, ptr: int, nbytes: int):
        self.ctx, self.ptr, self.nbytes = ctx, ptr, nbytes

    def __del__(self):
        if self.ptr and getattr(self.ctx, "handle", None):
            self.ctx.lib.vlr_host_free(self.ctx.handle, C.c_void_p(self.ptr))
            self.ptr = 0


class Context:
    """One CUDA device + stream; owns device grids created through it."""

    _default: dict[int, "Context"] = {}

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.vlr_ctx_create(device, C.byref(h))
        if rc != VLR_OK:
            raise VolrusError(rc, f"vlr_ctx_create(device={device}) failed (is a CUDA device present?)")
        self.handle = h
        self.device = device

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = cls(device)
        return cls._default[device]

    def check(self, rc: int, what: str = ""):
        if rc != VLR_OK:
            msg = self.lib.vlr_last_error(self.handle)
            raise VolrusError(rc, (what + ": " if what else "") + (msg.decode() if msg else ""))

    def synchronize(self):
        self.check(self.lib.vlr_ctx_synchronize(self.handle), "synchronize")

    def check_device(self):
        """Wait for the context stream and raise on device-side errors."""
        self.check(self.lib.vlr_ctx_check(self.handle), "vlr_ctx_check")

    def pinned(self, shape, dtype):
        """A numpy array in page-locked host memory (vlr_host_alloc), freed when
        the array and its views are gone: host buffers that host-resident
        calls copy at full rate (the slab pipeline of vlr_ls_step_host)."""
        import numpy as np
        dt = np.dtype(dtype)
        n = int(np.prod(shape)) * dt.itemsize
        p = C.c_void_p()
        self.check(self.lib.vlr_host_alloc(self.handle, max(n, 1), C.byref(p)), "vlr_host_alloc")
        holder = _PinnedBlock(self, p.value, max(n, 1))
        buf = (C.c_byte * max(n, 1)).from_address(p.value)
        buf._vlr_holder = holder  # the block lives as long as the buffer object
        return np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)

    def stream_ptr(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self.check(self.lib.vlr_ctx_stream(self.handle, C.byref(s)), "vlr_ctx_stream")
        return s.value or 0

    def profile(self, enable: bool):
        self.check(self.lib.vlr_ctx_profile(self.handle, 1 if enable else 0), "vlr_ctx_profile")

    def kernel_time(self, name: str):
        """(total milliseconds, launches) of kernel ``name`` since profiling was enabled."""
        ms = C.c_double()
        n = C.c_longlong()
        self.check(self.lib.vlr_ctx_profile_read(self.handle, name.encode(), C.byref(ms), C.byref(n)),
                   "vlr_ctx_profile_read")
        return ms.value, n.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.vlr_ctx_destroy(self.handle)
            self.handle = None
