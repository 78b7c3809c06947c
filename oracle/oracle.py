"""ctypes wrapper over the FP64 oracle (fft_oracle.c) and the planned CPU
baseline (cpu_port.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product package never
imports this module.

Every function restates a reference function; the C file names the
reference file:line for each.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

FORWARD, INVERSE = 0, 1
NORM_NONE, NORM_FORWARD, NORM_INVERSE, NORM_ORTHO = 0, 1, 2, 3

_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def build() -> str:
    """Compiles liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or _stale():
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_fft_f64.argtypes = [_dp, _dp, ctypes.c_uint64, ctypes.c_int]
        L.oracle_c2c_nd_f64.argtypes = [_dp, _dp, _u64p, ctypes.c_int, _i32p, ctypes.c_int,
                                        ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_c2c_nd_f64.restype = ctypes.c_int
        L.oracle_c2c_nd_dft_f32.argtypes = [_fp, _fp, _u64p, ctypes.c_int, _i32p, ctypes.c_int,
                                            ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_c2c_nd_dft_f32.restype = ctypes.c_int
        L.oracle_r2c_packed_f64.argtypes = [_dp, _dp, _u64p, ctypes.c_int, ctypes.c_uint64,
                                            ctypes.c_int]
        L.oracle_c2r_from_packed_f64.argtypes = [_dp, _dp, _u64p, ctypes.c_int, ctypes.c_uint64,
                                                 ctypes.c_int]
        L.oracle_scale_f64.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_scale_f64.restype = ctypes.c_double
        L.oracle_scale_f32.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_scale_f32.restype = ctypes.c_float
        L.oracle_df64_split.argtypes = [_dp, _fp, ctypes.c_uint64]
        L.oracle_df64_join.argtypes = [_fp, _dp, ctypes.c_uint64]
        L.oracle_is_prime.argtypes = [ctypes.c_uint64]
        L.oracle_primitive_root.argtypes = [ctypes.c_uint64]
        L.oracle_primitive_root.restype = ctypes.c_uint64
        L.oracle_factor_supported_length.argtypes = [ctypes.c_uint64, _u32p, ctypes.c_int]
        L.oracle_rader_permutation.argtypes = [ctypes.c_uint64, _u32p]
        L.cpu_port_c2c_f32.argtypes = [_fp, _u64p, ctypes.c_int, _i32p, ctypes.c_int,
                                       ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cpu_port_lines_new_f32.argtypes = [_u64p, _u64p, ctypes.c_uint64, ctypes.c_int,
                                             ctypes.c_int]
        L.cpu_port_lines_new_f32.restype = ctypes.c_void_p
        L.cpu_port_lines_exec_f32.argtypes = [ctypes.c_void_p, _fp, ctypes.c_uint64,
                                              ctypes.c_uint64, ctypes.c_int]
        L.cpu_port_lines_free_f32.argtypes = [ctypes.c_void_p]
        L.cpu_port_max_threads.restype = ctypes.c_int
        L.cpu_port_line_f64.argtypes = [_dp, ctypes.c_uint64, ctypes.c_int]
        _lib = L
    return _lib


def _stale() -> bool:
    so = os.path.getmtime(_LIB_PATH)
    for name in ("fft_oracle.c", "cpu_port.c", "cpu_port_impl.h", "Makefile"):
        p = os.path.join(_HERE, name)
        if os.path.exists(p) and os.path.getmtime(p) > so:
            return True
    return False


def _arr_u64(values):
    return np.ascontiguousarray(np.asarray(values, dtype=np.uint64))


def _arr_i32(values):
    return np.ascontiguousarray(np.asarray(values, dtype=np.int32))


def fft_f64(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """fft_f64 (src/math/mod.rs:274): unnormalised DFT of one line."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().oracle_fft_f64(x.ctypes.data_as(_dp), out.ctypes.data_as(_dp), x.size, int(inverse))
    return out


def c2c_nd_f64(x: np.ndarray, shape, axes=None, batch: int = 1, inverse: bool = False,
               normalization: int = NORM_INVERSE) -> np.ndarray:
    """reference_c2c_nd_f64 (src/math/mod.rs:214): x is the flat interleaved
    buffer as complex128 with axis 0 fastest (`batch` blocks of prod(shape))."""
    shape = list(shape)
    axes = list(range(len(shape))) if axes is None else list(axes)
    x = np.ascontiguousarray(x, dtype=np.complex128).reshape(-1)
    assert x.size == int(np.prod(shape)) * batch
    out = np.empty_like(x)
    sh, ax = _arr_u64(shape), _arr_i32(axes)
    rc = lib().oracle_c2c_nd_f64(x.ctypes.data_as(_dp), out.ctypes.data_as(_dp),
                                 sh.ctypes.data_as(_u64p), len(shape), ax.ctypes.data_as(_i32p),
                                 len(axes), batch, int(inverse), normalization)
    if rc:
        raise ValueError("invalid oracle configuration")
    return out


def c2c_nd_dft_f32(x: np.ndarray, shape, axes=None, batch: int = 1, inverse: bool = False,
                   normalization: int = NORM_INVERSE) -> np.ndarray:
    """reference_c2c_nd (src/math/mod.rs:155): the f32 plain DFT."""
    shape = list(shape)
    axes = list(range(len(shape))) if axes is None else list(axes)
    x = np.ascontiguousarray(x, dtype=np.complex64).reshape(-1)
    out = np.empty_like(x)
    sh, ax = _arr_u64(shape), _arr_i32(axes)
    rc = lib().oracle_c2c_nd_dft_f32(x.view(np.float32).ctypes.data_as(_fp),
                                     out.view(np.float32).ctypes.data_as(_fp),
                                     sh.ctypes.data_as(_u64p), len(shape),
                                     ax.ctypes.data_as(_i32p), len(axes), batch, int(inverse),
                                     normalization)
    if rc:
        raise ValueError("invalid oracle configuration")
    return out


def packed_shape(shape):
    s = list(shape)
    s[0] = s[0] // 2 + 1
    return s


def r2c_packed_f64(real: np.ndarray, shape, batch: int = 1,
                   normalization: int = NORM_INVERSE) -> np.ndarray:
    """reference_r2c_packed_interleaved (src/math/mod.rs:81) in FP64."""
    real = np.ascontiguousarray(real, dtype=np.float64).reshape(-1)
    n_packed = int(np.prod(packed_shape(shape))) * batch
    out = np.empty(n_packed, dtype=np.complex128)
    sh = _arr_u64(shape)
    rc = lib().oracle_r2c_packed_f64(real.ctypes.data_as(_dp), out.ctypes.data_as(_dp),
                                     sh.ctypes.data_as(_u64p), len(shape), batch, normalization)
    if rc:
        raise ValueError("invalid oracle configuration")
    return out


def c2r_from_packed_f64(packed: np.ndarray, shape, batch: int = 1,
                        normalization: int = NORM_INVERSE) -> np.ndarray:
    """reference_c2r_from_packed_interleaved (src/math/mod.rs:115) in FP64."""
    packed = np.ascontiguousarray(packed, dtype=np.complex128).reshape(-1)
    out = np.empty(int(np.prod(shape)) * batch, dtype=np.float64)
    sh = _arr_u64(shape)
    rc = lib().oracle_c2r_from_packed_f64(packed.ctypes.data_as(_dp), out.ctypes.data_as(_dp),
                                          sh.ctypes.data_as(_u64p), len(shape), batch,
                                          normalization)
    if rc:
        raise ValueError("invalid oracle configuration")
    return out


def scale_f64(logical_len: int, inverse: bool, normalization: int) -> float:
    return lib().oracle_scale_f64(logical_len, int(inverse), normalization)


def scale_f32(logical_len: int, inverse: bool, normalization: int) -> float:
    return lib().oracle_scale_f32(logical_len, int(inverse), normalization)


def df64_split(values: np.ndarray) -> np.ndarray:
    """Complex128 -> float32 words [re_hi, re_lo, im_hi, im_lo] per value."""
    v = np.ascontiguousarray(values, dtype=np.complex128).view(np.float64).reshape(-1)
    words = np.empty(v.size * 2, dtype=np.float32)
    lib().oracle_df64_split(v.ctypes.data_as(_dp), words.ctypes.data_as(_fp), v.size)
    return words


def df64_join(words: np.ndarray) -> np.ndarray:
    """float32 df64 words -> complex128."""
    w = np.ascontiguousarray(words, dtype=np.float32).reshape(-1)
    v = np.empty(w.size // 2, dtype=np.float64)
    lib().oracle_df64_join(w.ctypes.data_as(_fp), v.ctypes.data_as(_dp), v.size)
    return v.view(np.complex128)


def is_prime(n: int) -> bool:
    return bool(lib().oracle_is_prime(n))


def primitive_root(p: int) -> int:
    return int(lib().oracle_primitive_root(p))


def factor_supported_length(n: int):
    buf = np.zeros(64, dtype=np.uint32)
    c = lib().oracle_factor_supported_length(n, buf.ctypes.data_as(_u32p), 64)
    return None if c < 0 else [int(v) for v in buf[:c]]


def rader_permutation(p: int) -> np.ndarray:
    perm = np.zeros(max(p - 1, 1), dtype=np.uint32)
    if lib().oracle_rader_permutation(p, perm.ctypes.data_as(_u32p)):
        raise ValueError("not a prime")
    return perm[: p - 1]


# ---- accuracy metrics (the style of the reference's tests/gpu_accuracy.rs:153-179)

def rel_l2(actual: np.ndarray, expected: np.ndarray) -> float:
    a = np.asarray(actual, dtype=np.complex128).reshape(-1)
    e = np.asarray(expected, dtype=np.complex128).reshape(-1)
    den = np.linalg.norm(e)
    return float(np.linalg.norm(a - e) / (den if den > 0 else 1.0))


def max_rel(actual: np.ndarray, expected: np.ndarray) -> float:
    a = np.asarray(actual, dtype=np.complex128).reshape(-1)
    e = np.asarray(expected, dtype=np.complex128).reshape(-1)
    scale = np.max(np.abs(e)) if e.size else 1.0
    return float(np.max(np.abs(a - e)) / (scale if scale > 0 else 1.0))


# ---- planned CPU baseline (cpu_port.c)

def cpu_c2c_f32_inplace(data: np.ndarray, shape, axes=None, batch=1, inverse=False,
                        normalization=NORM_INVERSE, threads=0):
    shape = list(shape)
    axes = list(range(len(shape))) if axes is None else list(axes)
    assert data.dtype == np.complex64 and data.flags.c_contiguous
    sh, ax = _arr_u64(shape), _arr_i32(axes)
    rc = lib().cpu_port_c2c_f32(data.view(np.float32).ctypes.data_as(_fp),
                                sh.ctypes.data_as(_u64p), len(shape), ax.ctypes.data_as(_i32p),
                                len(axes), batch, int(inverse), normalization, threads)
    if rc:
        raise ValueError("invalid cpu baseline configuration")
    return data


class CpuLines:
    """Planned mixed-length lines on the CPU (one contiguous buffer)."""

    def __init__(self, offsets, lengths, inverse=False, normalization=NORM_INVERSE):
        self._off = _arr_u64(offsets)
        self._len = _arr_u64(lengths)
        self.n = len(self._len)
        self._h = lib().cpu_port_lines_new_f32(self._off.ctypes.data_as(_u64p),
                                               self._len.ctypes.data_as(_u64p), self.n,
                                               int(inverse), normalization)

    def run(self, data: np.ndarray, first=0, count=None, threads=0):
        count = self.n - first if count is None else count
        assert data.dtype == np.complex64 and data.flags.c_contiguous
        rc = lib().cpu_port_lines_exec_f32(self._h, data.view(np.float32).ctypes.data_as(_fp),
                                           first, count, threads)
        if rc:
            raise ValueError("line range out of bounds")

    def close(self):
        if self._h:
            lib().cpu_port_lines_free_f32(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cpu_max_threads() -> int:
    return int(lib().cpu_port_max_threads())
