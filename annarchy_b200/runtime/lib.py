"""ctypes binding of the C ABI in include/annarchy_b200.h.

The shared library is built in-tree (``annarchy_b200/_lib``) by
``annarchy_b200.build.build_all()``. There is no fallback: if the library
is missing or no GPU is visible, creating a network raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "_lib", "libannarchy_b200.so")

ANB_OK = 0
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_ALLOC", 3: "ERR_CUDA", 4: "ERR_COMPILE",
          5: "ERR_TIMEOUT", 6: "ERR_STATE"}

# name -> (restype, argtypes)
SIGNATURES = {
    "anb_abi_version": (C.c_int, []),
    "anb_last_error": (C.c_char_p, []),
    "anb_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "anb_device_sm_count": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "anb_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "anb_destroy": (C.c_int, [C.c_void_p]),
    "anb_initialize": (C.c_int, [C.c_void_p, C.c_double]),
    "anb_set_time": (C.c_int, [C.c_void_p, C.c_int64]),
    "anb_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "anb_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "anb_array_create": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "anb_array_free": (C.c_int, [C.c_void_p, C.c_char_p]),
    "anb_array_write": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_void_p, C.c_size_t]),
    "anb_array_read": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_void_p, C.c_size_t]),
    "anb_array_fill_zero": (C.c_int, [C.c_void_p, C.c_char_p]),
    "anb_array_info": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_size_t)]),
    "anb_module_load": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p]),
    "anb_array_fill": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]),
    "anb_connect_fixed_number_pre": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_int,
                                               C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_double,
                                               C.c_double, C.c_int, C.c_int]),
    "anb_connect_fixed_number_pre_rows": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_longlong,
                                                    C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                                    C.c_double, C.c_double, C.c_int, C.c_int]),
    "anb_connect_fixed_probability_rows": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int,
                                                     C.c_longlong, C.c_int, C.c_int, C.c_double,
                                                     C.c_uint64, C.c_int, C.c_double, C.c_double,
                                                     C.c_int, C.c_int, C.POINTER(C.c_longlong)]),
    "anb_csr_to_csc": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int]),
    "anb_set_stop_kernel": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_uint, C.c_uint, C.c_int]),
    "anb_module_set_constant": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double]),
    "anb_run_until": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int), C.c_int, C.c_int,
                                C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "anb_nvrtc_compile": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t,
                                    C.POINTER(C.c_size_t)]),
    "anb_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "anb_bsr_tc_pack_x": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "anb_bsr_spmm_tc_shape": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "anb_bsr_spmm_tc_prefetch": (C.c_int, [C.c_int]),
    "anb_stream_read": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(C.c_double)]),
    "anb_tile_fill": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.POINTER(C.c_double)]),
    "anb_array_copy_strided": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_size_t, C.c_char_p,
                                         C.c_size_t, C.c_size_t, C.c_size_t]),
    "anb_plan_add_concurrent": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.c_int]),
    "anb_bsr_spmm_tc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                  C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "anb_bsr_spmm_simt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "anb_monitor_decode": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64, C.c_int64, C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "anb_bank_interleave": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "anb_bitmap_decode": (C.c_int64, [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_int64]),
    "anb_plan_clear": (C.c_int, [C.c_void_p]),
    "anb_plan_add": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint, C.c_uint, C.c_uint]),
    "anb_set_local_kernel": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint, C.c_uint, C.c_uint]),
    "anb_set_local_kernel_ex": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint, C.c_uint, C.c_uint,
                                          C.c_uint]),
    "anb_set_graph_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "anb_set_pdl": (C.c_int, [C.c_void_p, C.c_int]),
    "anb_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "anb_step": (C.c_int, [C.c_void_p]),
    "anb_synchronize": (C.c_int, [C.c_void_p]),
    "anb_device_error": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "anb_clear_device_error": (C.c_int, [C.c_void_p]),
    "anb_flush_l2": (C.c_int, [C.c_void_p]),
    "anb_kernel_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "anb_kernel_time_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "anb_kernel_time_get": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t,
                                      C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "anb_selector_last_error": (C.c_char_p, []),
    "anb_mlp_param_count": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    "anb_mlp_loss_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "anb_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p]),
    "anb_mlp_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_void_p]),
    "anb_connect_distance_pattern": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                               C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                               C.POINTER(C.c_longlong)]),
    "anb_set_local_kernel_cooperative": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint, C.c_uint,
                                                   C.POINTER(C.c_uint)]),
    "anb_plan_add_bsr_tc": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_int]),
    "anb_set_seed": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_int]),
    "anb_record_declare": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64, C.c_int, C.c_int64]),
    "anb_estimate_record_size": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_size_t)]),
    "anb_init_from_lil": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                    C.POINTER(C.c_int64)]),
    "anb_mlp_noalloc_max_floats": (C.c_size_t, []),
    "anb_mlp_predict_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_void_p, C.c_void_p]),
}

_lib = None

# arrays every network has from anb_create on: step counter, dt, error words
BUILTIN_ARRAYS = {"t": (np.dtype(np.int64), (1,)), "dt": (np.dtype(np.float64), (1,)),
                  "err": (np.dtype(np.int32), (4,))}


class BackendError(RuntimeError):
    """A call of the native library failed."""

    def __init__(self, fn: str, status: int, message: str):
        super().__init__(f"{fn} -> {STATUS.get(status, status)}: {message}")
        self.status = status


def load():
    """Load libannarchy_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"native library not found at {LIB_PATH}; build it with "
                           "`python -c 'import annarchy_b200.build as b; b.build_all()'`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(fn: str, status: int):
    if status != ANB_OK:
        msg = load().anb_last_error()
        raise BackendError(fn, status, msg.decode(errors="replace") if msg else "")


def check_selector(fn: str, status: int):
    if status != ANB_OK:
        msg = load().anb_selector_last_error()
        raise BackendError(fn, status, msg.decode(errors="replace") if msg else "")


def device_count() -> int:
    n = C.c_int(0)
    check("anb_device_count", load().anb_device_count(C.byref(n)))
    return n.value


def device_sm_count(device: int = 0) -> int:
    n = C.c_int(0)
    check("anb_device_sm_count", load().anb_device_sm_count(int(device), C.byref(n)))
    return n.value


def nvrtc_compile(source: str, options: list[str]) -> tuple[int, str]:
    """Compile a generated module for sm_100a without a device; returns
    (cubin bytes, compiler log). Raises BackendError with the log on errors."""
    log = C.create_string_buffer(1 << 16)
    n = C.c_size_t(0)
    check("anb_nvrtc_compile", load().anb_nvrtc_compile(source.encode(), "\n".join(options).encode(),
                                                        log, len(log), C.byref(n)))
    return n.value, log.value.decode(errors="replace")


def bank_interleave(row_ptr: np.ndarray, post: np.ndarray) -> np.ndarray:
    """Permutation of the positions row_ptr[0]..row_ptr[-1]-1 that deals each
    row's synapses, by bank of their post rank, over the warp's atomic
    instructions (anb_bank_interleave)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    post = np.ascontiguousarray(post, dtype=np.int32)
    n = int(row_ptr[-1] - row_ptr[0]) if row_ptr.size else 0
    perm = np.arange(row_ptr[0] if row_ptr.size else 0, (row_ptr[0] if row_ptr.size else 0) + n,
                     dtype=np.int64)
    if n:
        check("anb_bank_interleave", load().anb_bank_interleave(
            row_ptr.ctypes.data_as(C.c_void_p), row_ptr.size - 1, post.ctypes.data_as(C.c_void_p),
            perm.ctypes.data_as(C.c_void_p)))
    return perm


def bitmap_decode(buf: np.ndarray, n: int):
    """(steps, words) uint32 spike bitmaps -> (step, rank) int64 arrays."""
    buf = np.ascontiguousarray(buf, dtype=np.uint32)
    steps, words = buf.shape
    lib = load()
    # first guess: one spike per word (np.empty does not touch the pages);
    # the decoder returns the true count and a second pass follows if needed
    cap = int(max(1024, buf.size))
    while True:
        s = np.empty(cap, dtype=np.int64)
        r = np.empty(cap, dtype=np.int64)
        k = lib.anb_bitmap_decode(buf.ctypes.data_as(C.c_void_p), steps, words, n,
                                  s.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p), cap)
        if k <= cap:
            return s[:k], r[:k]
        cap = int(k)


class NativeNet:
    """One network instance inside the native library."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check("anb_create", self.lib.anb_create(device, C.byref(h)))
        self.h = h
        self.arrays: dict[str, tuple[np.dtype, tuple]] = dict(BUILTIN_ARRAYS)

    def close(self):
        if self.h:
            self.lib.anb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- lifetime / time --------------------------------------------------
    def initialize(self, dt: float):
        check("anb_initialize", self.lib.anb_initialize(self.h, float(dt)))

    def set_time(self, t: int):
        check("anb_set_time", self.lib.anb_set_time(self.h, int(t)))

    def get_time(self) -> int:
        t = C.c_int64()
        check("anb_get_time", self.lib.anb_get_time(self.h, C.byref(t)))
        return t.value

    def set_stream(self, stream_ptr: int | None):
        check("anb_set_stream", self.lib.anb_set_stream(self.h, C.c_void_p(stream_ptr or None)))

    # -- arrays -------------------------------------------------------------
    def create(self, name: str, data: np.ndarray):
        """Create (or re-create) array `name` holding a copy of `data`."""
        data = np.ascontiguousarray(data)
        check("anb_array_create", self.lib.anb_array_create(self.h, name.encode(), data.nbytes))
        self.arrays[name] = (data.dtype, data.shape)
        if data.nbytes:
            self.write(name, data)

    def create_empty(self, name: str, dtype, shape):
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
        check("anb_array_create", self.lib.anb_array_create(self.h, name.encode(), nbytes))
        self.arrays[name] = (dtype, tuple(shape) if isinstance(shape, (tuple, list)) else (shape,))

    def write(self, name: str, data: np.ndarray, offset_bytes: int = 0):
        data = np.ascontiguousarray(data)
        check("anb_array_write", self.lib.anb_array_write(
            self.h, name.encode(), offset_bytes, data.ctypes.data_as(C.c_void_p), data.nbytes))

    def read(self, name: str, count: int | None = None, offset: int = 0) -> np.ndarray:
        dtype, shape = self.arrays[name]
        if count is None:
            out = np.empty(shape, dtype=dtype)
        else:
            out = np.empty(count, dtype=dtype)
        check("anb_array_read", self.lib.anb_array_read(
            self.h, name.encode(), offset * dtype.itemsize, out.ctypes.data_as(C.c_void_p),
            out.nbytes))
        return out

    def read_into(self, name: str, out: np.ndarray, offset_bytes: int = 0):
        check("anb_array_read", self.lib.anb_array_read(
            self.h, name.encode(), offset_bytes, out.ctypes.data_as(C.c_void_p), out.nbytes))

    def stream(self) -> int:
        """The cudaStream_t (as an integer) the network's work runs on."""
        out = C.c_void_p()
        check("anb_get_stream", self.lib.anb_get_stream(self.h, C.byref(out)))
        return out.value or 0

    def monitor_decode(self, name: str, steps: int, words: int, n: int):
        """(step, rank) int64 arrays of the spikes in the first `steps` rows of
        the spike ring `name`, decoded on the device (sorted by step, rank)."""
        cap = int(max(1024, steps * words))
        for _ in range(2):
            s = np.empty(cap, dtype=np.int32)
            r = np.empty(cap, dtype=np.int32)
            k = C.c_int64(0)
            check("anb_monitor_decode", self.lib.anb_monitor_decode(
                self.h, name.encode(), int(steps), int(words), int(n),
                s.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p), cap, C.byref(k)))
            if k.value <= cap:
                return s[:k.value].astype(np.int64), r[:k.value].astype(np.int64)
            cap = int(k.value)
        raise RuntimeError("monitor_decode: spike count changed between calls")

    def zero(self, name: str):
        check("anb_array_fill_zero", self.lib.anb_array_fill_zero(self.h, name.encode()))

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        n = C.c_size_t()
        check("anb_array_info", self.lib.anb_array_info(self.h, name.encode(), C.byref(p),
                                                       C.byref(n)))
        return p.value or 0

    def nbytes(self, name: str) -> int:
        p = C.c_void_p()
        n = C.c_size_t()
        check("anb_array_info", self.lib.anb_array_info(self.h, name.encode(), C.byref(p),
                                                       C.byref(n)))
        return int(n.value)

    def free(self, name: str):
        check("anb_array_free", self.lib.anb_array_free(self.h, name.encode()))
        self.arrays.pop(name, None)

    def stream_read_ms(self, nbytes: int, reps: int = 5) -> float:
        """Median cold streaming-read time (ms) of `nbytes` (anb_stream_read)."""
        out = C.c_double(0.0)
        check("anb_stream_read", self.lib.anb_stream_read(self.h, int(nbytes), reps, C.byref(out)))
        return out.value

    def tile_fill_ms(self, n_tiles: int, tile_bytes: int, copies: int, ctas_per_sm: int = 2,
                     stages: int = 3, reps: int = 5) -> float:
        """Median time (ms) of `copies` bulk copies of L2-resident tiles into
        shared memory (anb_tile_fill)."""
        out = C.c_double(0.0)
        check("anb_tile_fill", self.lib.anb_tile_fill(self.h, int(n_tiles), int(tile_bytes), int(copies),
                                                      int(ctas_per_sm), int(stages), int(reps),
                                                      C.byref(out)))
        return out.value

    def copy_strided(self, dst, dst_offset, dst_stride, src, src_offset, src_stride, count):
        """Device copy of `count` 4-byte elements between arrays (byte offsets
        and strides)."""
        check("anb_array_copy_strided", self.lib.anb_array_copy_strided(
            self.h, dst.encode(), dst_offset, dst_stride, src.encode(), src_offset, src_stride, count))

    def connect_distance_pattern(self, prefix: str, kind: int, post_coords, pre_coords,
                                 a_pos: float, den_pos: float, a_neg: float, den_neg: float,
                                 threshold: float, exclude_self: bool, weight_dtype) -> int:
        """Gaussian (kind 0) or difference-of-Gaussians (kind 1) pattern built
        on the device (anb_connect_distance_pattern); returns the synapse count."""
        qc = np.ascontiguousarray(post_coords, dtype=np.float64)
        pc = np.ascontiguousarray(pre_coords, dtype=np.float64)
        wb = np.dtype(weight_dtype).itemsize
        nnz = C.c_longlong()
        check("anb_connect_distance_pattern", self.lib.anb_connect_distance_pattern(
            self.h, prefix.encode(), int(kind), qc.shape[0], qc.ctypes.data_as(C.c_void_p),
            pc.shape[0], pc.ctypes.data_as(C.c_void_p), qc.shape[1], float(a_pos), float(den_pos),
            float(a_neg), float(den_neg), float(threshold), 1 if exclude_self else 0, wb,
            C.byref(nnz)))
        n = nnz.value
        for name, dt, count in (("__post_rank", np.int32, qc.shape[0]),
                                ("__row_ptr", np.int32, qc.shape[0] + 1), ("__col", np.int32, n)):
            self.arrays[prefix + name] = (np.dtype(dt), (count,))
        self.arrays[prefix + "__w"] = (np.dtype(weight_dtype), (n,))
        return int(n)

    def set_seed(self, seed: int, num_sources: int = 1, use_seed_seq: bool = True):
        """Key of the device's random draws (anb_set_seed)."""
        check("anb_set_seed", self.lib.anb_set_seed(self.h, int(seed) & (2**64 - 1),
                                                     int(num_sources), 1 if use_seed_seq else 0))
        self.arrays["rng_seed"] = (np.dtype(np.uint32), (2,))

    def record_declare(self, ring: str, values_per_record: int, value_bytes: int, period: int):
        check("anb_record_declare", self.lib.anb_record_declare(
            self.h, ring.encode(), int(values_per_record), int(value_bytes), int(period)))

    def estimate_record_size(self, nsteps: int) -> int:
        """MiB of the declared recorded variables after nsteps steps."""
        out = C.c_size_t()
        check("anb_estimate_record_size", self.lib.anb_estimate_record_size(
            self.h, int(nsteps), C.byref(out)))
        return int(out.value)

    def init_from_lil(self, prefix: str, post_ranks, pre_ranks, w, delays=None,
                      requires_sorting: bool = False, weight_bytes: int = 8) -> int:
        """Upload LIL connectivity (lists per dendrite) as CSR arrays through
        anb_init_from_lil; returns the synapse count."""
        sizes = np.array([len(r) for r in pre_ranks], dtype=np.int64)
        row_begin = np.zeros(len(sizes) + 1, dtype=np.int64)
        np.cumsum(sizes, out=row_begin[1:])
        post = np.ascontiguousarray(post_ranks, dtype=np.int32)
        cat = (lambda a, dt: np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=dt) for x in a])
                                                  if len(a) else np.zeros(0, dt)))
        pre = cat(pre_ranks, np.int32)
        ww = cat(w, np.float64)
        dd = cat(delays, np.int32) if delays is not None else None
        nnz = C.c_int64()
        check("anb_init_from_lil", self.lib.anb_init_from_lil(
            self.h, prefix.encode(), len(post), post.ctypes.data_as(C.c_void_p),
            row_begin.ctypes.data_as(C.c_void_p), pre.ctypes.data_as(C.c_void_p),
            ww.ctypes.data_as(C.c_void_p), dd.ctypes.data_as(C.c_void_p) if dd is not None else None,
            1 if requires_sorting else 0, int(weight_bytes), C.byref(nnz)))
        for name, dt, n in (("__post_rank", np.int32, len(post)), ("__row_ptr", np.int32, len(post) + 1),
                            ("__col", np.int32, nnz.value)):
            self.arrays[prefix + name] = (np.dtype(dt), (n,))
        wdt = {8: np.float64, 4: np.float32, 2: np.uint16}[int(weight_bytes)]
        self.arrays[prefix + "__w"] = (np.dtype(wdt), (nnz.value,))
        return int(nnz.value)

    def fill(self, name: str, value):
        v = np.asarray(value)
        check("anb_array_fill", self.lib.anb_array_fill(self.h, name.encode(),
                                                       v.ctypes.data_as(C.c_void_p), v.nbytes))

    def connect_fixed_number_pre(self, prefix, n_post, post_base, pre_lo, pre_hi, number, seed,
                                 weight_kind, a, b, weight_dtype, exclude_self, row_offset: int = 0):
        wb = {np.dtype(np.float64): 8, np.dtype(np.float32): 4, np.dtype(np.uint16): 2}[
            np.dtype(weight_dtype)]
        check("anb_connect_fixed_number_pre_rows", self.lib.anb_connect_fixed_number_pre_rows(
            self.h, prefix.encode(), n_post, post_base, int(row_offset), pre_lo, pre_hi, number, seed,
            weight_kind, float(a), float(b), wb, 1 if exclude_self else 0))
        nnz = n_post * number
        self.arrays[prefix + "__post_rank"] = (np.dtype(np.int32), (n_post,))
        self.arrays[prefix + "__row_ptr"] = (np.dtype(np.int32), (n_post + 1,))
        self.arrays[prefix + "__col"] = (np.dtype(np.int32), (nnz,))
        self.arrays[prefix + "__w"] = (np.dtype(weight_dtype), (nnz,))

    def connect_fixed_probability(self, prefix, n_post, post_base, pre_lo, pre_hi, probability,
                                  seed, weight_kind, a, b, weight_dtype, exclude_self,
                                  row_offset: int = 0) -> int:
        """Device-generated fixed-probability rows; returns the number of synapses."""
        wb = {np.dtype(np.float64): 8, np.dtype(np.float32): 4, np.dtype(np.uint16): 2}[
            np.dtype(weight_dtype)]
        nnz = C.c_longlong(0)
        check("anb_connect_fixed_probability_rows", self.lib.anb_connect_fixed_probability_rows(
            self.h, prefix.encode(), n_post, post_base, int(row_offset), pre_lo, pre_hi,
            float(probability), seed, weight_kind, float(a), float(b), wb,
            1 if exclude_self else 0, C.byref(nnz)))
        self.arrays[prefix + "__post_rank"] = (np.dtype(np.int32), (n_post,))
        self.arrays[prefix + "__row_ptr"] = (np.dtype(np.int32), (n_post + 1,))
        self.arrays[prefix + "__col"] = (np.dtype(np.int32), (nnz.value,))
        self.arrays[prefix + "__w"] = (np.dtype(weight_dtype), (nnz.value,))
        return int(nnz.value)

    def csr_to_csc(self, prefix, n_pre, with_weights):
        check("anb_csr_to_csc", self.lib.anb_csr_to_csc(self.h, prefix.encode(), n_pre,
                                                       1 if with_weights else 0))
        nnz = self.arrays[prefix + "__col"][1][0]
        self.arrays[prefix + "__col_ptr"] = (np.dtype(np.int32), (n_pre + 1,))
        self.arrays[prefix + "__post_idx"] = (np.dtype(np.int32), (nnz,))
        self.arrays[prefix + "__inv_idx"] = (np.dtype(np.int32), (nnz,))
        if with_weights:
            self.arrays[prefix + "__w_pre"] = (self.arrays[prefix + "__w"][0], (nnz,))

    # -- module and plan ------------------------------------------------------
    def load_module(self, source: str, options: list[str]):
        check("anb_module_load", self.lib.anb_module_load(self.h, source.encode(),
                                                         "\n".join(options).encode()))

    def plan(self, launches):
        """launches: (kernel, grid, block, shared bytes[, concurrency group])."""
        check("anb_plan_clear", self.lib.anb_plan_clear(self.h))
        for entry in launches:
            if isinstance(entry[0], dict):          # a library operation
                op = entry[0]
                check("anb_plan_add_bsr_tc", self.lib.anb_plan_add_bsr_tc(
                    self.h, op["prefix"].encode(), op["x"].encode(), op["y"].encode(),
                    op["n_block_rows"], op["batch"], op["n_pre"], op["n_post"],
                    entry[4] if len(entry) > 4 else 0))
                continue
            name, grid, block, smem = entry[:4]
            group = entry[4] if len(entry) > 4 else 0
            check("anb_plan_add_concurrent", self.lib.anb_plan_add_concurrent(
                self.h, name.encode(), grid, block, smem, group))

    def set_local_kernel(self, name, grid, block, smem, cluster: int = 1):
        if cluster == -1:                       # cooperative: the runtime sizes the grid
            g = C.c_uint()
            check("anb_set_local_kernel_cooperative", self.lib.anb_set_local_kernel_cooperative(
                self.h, name.encode(), block, smem, C.byref(g)))
            self.local_grid = int(g.value)
            return
        if cluster > 1:
            check("anb_set_local_kernel_ex", self.lib.anb_set_local_kernel_ex(
                self.h, name.encode(), grid, block, smem, cluster))
        else:
            check("anb_set_local_kernel", self.lib.anb_set_local_kernel(self.h, name.encode(),
                                                                       grid, block, smem))

    def set_graph_steps(self, steps: int):
        check("anb_set_graph_steps", self.lib.anb_set_graph_steps(self.h, steps))

    def set_pdl(self, on: bool):
        check("anb_set_pdl", self.lib.anb_set_pdl(self.h, 1 if on else 0))

    def run(self, steps: int):
        check("anb_run", self.lib.anb_run(self.h, int(steps)))

    def set_constant(self, name: str, value: float):
        check("anb_module_set_constant", self.lib.anb_module_set_constant(self.h, name.encode(),
                                                                        float(value)))

    def set_stop_kernel(self, pop: int, kernel: str, grid: int, block: int, all_mode: bool):
        check("anb_set_stop_kernel", self.lib.anb_set_stop_kernel(
            self.h, int(pop), kernel.encode(), int(grid), int(block), 1 if all_mode else 0))

    def run_until(self, steps: int, populations, or_and: bool) -> tuple[int, bool]:
        """(steps run, whether the stop conditions ended the run)."""
        pops = (C.c_int * max(1, len(populations)))(*[int(p) for p in populations])
        done, stopped = C.c_int64(0), C.c_int(0)
        check("anb_run_until", self.lib.anb_run_until(self.h, int(steps), pops, len(populations),
                                                      1 if or_and else 0, C.byref(done),
                                                      C.byref(stopped)))
        return int(done.value), bool(stopped.value)

    def synchronize(self):
        check("anb_synchronize", self.lib.anb_synchronize(self.h))

    def device_error(self) -> int:
        c = C.c_int()
        check("anb_device_error", self.lib.anb_device_error(self.h, C.byref(c)))
        return c.value

    def clear_device_error(self):
        check("anb_clear_device_error", self.lib.anb_clear_device_error(self.h))

    # -- timing -----------------------------------------------------------------
    def flush_l2(self):
        check("anb_flush_l2", self.lib.anb_flush_l2(self.h))

    def kernel_timing(self, enable: bool):
        check("anb_kernel_timing", self.lib.anb_kernel_timing(self.h, 1 if enable else 0))

    def kernel_times(self) -> dict[str, tuple[float, int]]:
        n = C.c_int()
        check("anb_kernel_time_count", self.lib.anb_kernel_time_count(self.h, C.byref(n)))
        out = {}
        buf = C.create_string_buffer(256)
        for i in range(n.value):
            ms = C.c_double()
            cnt = C.c_int64()
            check("anb_kernel_time_get", self.lib.anb_kernel_time_get(
                self.h, i, buf, 256, C.byref(ms), C.byref(cnt)))
            out[buf.value.decode()] = (ms.value, cnt.value)
        return out


class DryNative:
    """Stand-in for NativeNet that only records array names, types and
    shapes. It lets the code generator run on a machine without a GPU, so the
    generated module can be compiled (nvrtc_compile) and inspected there."""

    def __init__(self, device: int = 0):
        self.arrays: dict[str, tuple[np.dtype, tuple]] = dict(BUILTIN_ARRAYS)
        self.source = None
        self.options = None

    def initialize(self, dt):
        pass

    def create(self, name, data):
        data = np.asarray(data)
        self.arrays[name] = (data.dtype, data.shape)

    def create_empty(self, name, dtype, shape):
        self.arrays[name] = (np.dtype(dtype), tuple(np.atleast_1d(shape)))

    def write(self, *a, **k):
        pass

    def fill(self, name, value):
        pass

    def set_seed(self, seed, num_sources=1, use_seed_seq=True):
        self.arrays["rng_seed"] = (np.dtype(np.uint32), (2,))

    def connect_distance_pattern(self, prefix, kind, post_coords, pre_coords, *a):
        n = len(post_coords)
        self.arrays[prefix + "__post_rank"] = (np.dtype(np.int32), (n,))
        self.arrays[prefix + "__row_ptr"] = (np.dtype(np.int32), (n + 1,))
        self.arrays[prefix + "__col"] = (np.dtype(np.int32), (0,))
        self.arrays[prefix + "__w"] = (np.dtype(np.float64), (0,))
        return 0

    def record_declare(self, *a):
        pass

    def free(self, name):
        self.arrays.pop(name, None)

    def copy_strided(self, *a):
        pass

    def connect_fixed_number_pre(self, prefix, n_post, post_base, pre_lo, pre_hi, number, seed,
                                 weight_kind, a, b, weight_dtype, exclude_self, row_offset: int = 0):
        nnz = n_post * number
        self.arrays[prefix + "__post_rank"] = (np.dtype(np.int32), (n_post,))
        self.arrays[prefix + "__row_ptr"] = (np.dtype(np.int32), (n_post + 1,))
        self.arrays[prefix + "__col"] = (np.dtype(np.int32), (nnz,))
        self.arrays[prefix + "__w"] = (np.dtype(weight_dtype), (nnz,))

    def connect_fixed_probability(self, prefix, n_post, post_base, pre_lo, pre_hi, probability,
                                  seed, weight_kind, a, b, weight_dtype, exclude_self,
                                  row_offset: int = 0) -> int:
        nnz = int(round(n_post * (pre_hi - pre_lo) * probability))     # the expected count
        self.arrays[prefix + "__post_rank"] = (np.dtype(np.int32), (n_post,))
        self.arrays[prefix + "__row_ptr"] = (np.dtype(np.int32), (n_post + 1,))
        self.arrays[prefix + "__col"] = (np.dtype(np.int32), (nnz,))
        self.arrays[prefix + "__w"] = (np.dtype(weight_dtype), (nnz,))
        return nnz

    def csr_to_csc(self, prefix, n_pre, with_weights):
        nnz = self.arrays[prefix + "__col"][1][0]
        self.arrays[prefix + "__col_ptr"] = (np.dtype(np.int32), (n_pre + 1,))
        self.arrays[prefix + "__post_idx"] = (np.dtype(np.int32), (nnz,))
        self.arrays[prefix + "__inv_idx"] = (np.dtype(np.int32), (nnz,))
        if with_weights:
            self.arrays[prefix + "__w_pre"] = (self.arrays[prefix + "__w"][0], (nnz,))

    def load_module(self, source, options):
        self.source, self.options = source, options

    def plan(self, launches):
        self.launches = list(launches)

    def set_local_kernel(self, *a):
        self.local = a

    def set_constant(self, *a):
        pass

    def set_stop_kernel(self, *a):
        pass

    def set_graph_steps(self, steps):
        pass

    def set_pdl(self, on):
        pass

    def close(self):
        pass
