"""wgpufft_b200: the FFT transform path of the wgpu-fft crate
(MaximEremenko/wgpuFFT), rebuilt for NVIDIA B200 (sm_100a).

This module mirrors the crate's public plan API (src/plan.rs, src/config.rs,
src/tuning.rs) over the C ABI of ``libwgpufft_b200.so``
(``include/wgpufft_b200.h``):

    cfg = FftConfig.new(1024).with_batch(512)
    plan = FftPlan.c2c(cfg)                 # FftPlan::c2c (src/plan.rs:221)
    plan.execute_checked(inp, out)          # src/plan.rs:510
    plan.execute_in_place(buf)              # src/plan.rs:827
    with FftRecorder() as rec:              # FftRecorder (src/plan.rs:68-95)
        plan.record(rec, inp, out)
    rec.submit()

wgpu buffers become CUDA device memory: a torch CUDA tensor, or an
``(address, nbytes)`` pair.  There is no CPU fallback: without the built
library every call raises.
"""
from __future__ import annotations

import ctypes
import enum
import json
import os
from typing import Iterable, Optional, Sequence, Tuple, Union

__all__ = [
    "FftDirection", "Normalization", "FftPrecision", "FftTransformKind", "FftTuning",
    "FftConfig", "FftPlan", "FftRecorder", "FftBatch", "FftServer", "FftError", "lib",
    "FftLogicalLayout", "validate_df64_invariants",
    "library_path",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libwgpufft_b200.so")
_lib = None


def library_path() -> str:
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    """Loads libwgpufft_b200.so (built by wgpufft_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise FftError("LibraryMissing", 0,
                           f"{_LIB_PATH} is not built; run python wgpufft_b200/build.py")
        L = ctypes.CDLL(_LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L: ctypes.CDLL) -> None:
    vp, u64, i32, u32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32
    pvp = ctypes.POINTER(ctypes.c_void_p)
    st = ctypes.c_int32
    sig = {
        "b2f_config_new": (st, [pvp, ctypes.POINTER(u64), u32]),
        "b2f_config_free": (None, [vp]),
        "b2f_config_set_axes": (st, [vp, ctypes.POINTER(u32), u32]),
        "b2f_config_set_batch": (st, [vp, u64]),
        "b2f_config_set_direction": (st, [vp, i32]),
        "b2f_config_set_normalization": (st, [vp, i32]),
        "b2f_config_set_precision": (st, [vp, i32]),
        "b2f_config_set_tuning": (st, [vp, ctypes.c_char_p, ctypes.c_int64]),
        "b2f_config_get_tuning": (st, [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
        "b2f_autotune": (st, [vp, i32, i32, u32, ctypes.c_char_p, ctypes.POINTER(u64)]),
        "b2f_tuning_snapshot_record": (st, [vp, i32, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                            ctypes.c_double]),
        "b2f_tuning_snapshot_apply": (st, [vp, i32, ctypes.POINTER(i32)]),
        "b2f_tuning_snapshot_json": (st, [ctypes.c_char_p, ctypes.POINTER(u64)]),
        "b2f_tuning_snapshot_save": (st, [ctypes.c_char_p]),
        "b2f_tuning_snapshot_load": (st, [ctypes.c_char_p, i32]),
        "b2f_tuning_snapshot_clear": (None, []),
        "b2f_config_set_tuning_axes": (st, [vp, ctypes.c_char_p, ctypes.POINTER(u32), u32]),
        "b2f_config_validate": (st, [vp]),
        "b2f_config_required_buffer_size_bytes": (st, [vp, ctypes.POINTER(u64)]),
        "b2f_config_scale": (st, [vp, ctypes.POINTER(ctypes.c_float),
                                  ctypes.POINTER(ctypes.c_double)]),
        "b2f_plan_c2c": (st, [pvp, vp, i32]),
        "b2f_plan_r2c": (st, [pvp, vp, i32]),
        "b2f_plan_c2r": (st, [pvp, vp, i32]),
        "b2f_plan_free": (None, [vp]),
        "b2f_plan_kind": (i32, [vp]),
        "b2f_plan_required_buffer_size_bytes": (u64, [vp]),
        "b2f_plan_required_input_buffer_size_bytes": (u64, [vp]),
        "b2f_plan_required_output_buffer_size_bytes": (u64, [vp]),
        "b2f_plan_workspace_size_bytes": (u64, [vp]),
        "b2f_plan_supports_in_place": (i32, [vp]),
        "b2f_plan_execute_checked": (st, [vp, vp, vp, u64, vp, u64]),
        "b2f_plan_execute_in_place": (st, [vp, vp, vp, u64]),
        "b2f_plan_execute_logical_views": (st, [vp, vp, vp, u64, ctypes.POINTER(_Layout), vp, u64,
                                                ctypes.POINTER(_Layout)]),
        "b2f_plan_diagnostics_json": (st, [vp, ctypes.c_char_p, ctypes.POINTER(u64)]),
        "b2f_plan_device_status": (st, [vp]),
        "b2f_recorder_begin": (st, [pvp, vp]),
        "b2f_plan_record": (st, [vp, vp, vp, u64, vp, u64]),
        "b2f_plan_record_in_place": (st, [vp, vp, vp, u64]),
        "b2f_recorder_finish": (st, [vp]),
        "b2f_recorder_submit": (st, [vp, vp]),
        "b2f_recorder_free": (None, [vp]),
        "b2f_batch_new": (st, [pvp, ctypes.POINTER(u64), ctypes.POINTER(u64), u64, i32, i32, i32]),
        "b2f_batch_new_ex": (st, [pvp, ctypes.POINTER(u64), ctypes.POINTER(u64), u64, i32, i32, i32,
                                 u32]),
        "b2f_batch_free": (None, [vp]),
        "b2f_batch_required_buffer_size_bytes": (u64, [vp]),
        "b2f_batch_execute": (st, [vp, vp, vp, u64, vp, u64]),
        "b2f_batch_diagnostics_json": (st, [vp, ctypes.c_char_p, ctypes.POINTER(u64)]),
        "b2f_batch_execute_parts": (st, [vp, vp, vp, u64, vp, u64, u32, i32]),
        "b2f_batch_execute_host": (st, [vp, vp, vp, vp, vp, vp, u64]),
        "b2f_c2c_1d_f32_noalloc": (st, [vp, vp, u64, vp, u64, u64, u64, i32, i32]),
        "b2f_df64_canary": (st, [i32, ctypes.POINTER(u32), ctypes.POINTER(u64)]),
        "b2f_server_new": (st, [pvp, i32, u64, i32, i32]),
        "b2f_server_free": (None, [vp]),
        "b2f_server_submit": (st, [vp, vp, i32, vp, u64, vp, u64, ctypes.POINTER(u64)]),
        "b2f_server_submit_device": (st, [vp, vp, i32, vp, u64, vp, u64, ctypes.POINTER(u64)]),
        "b2f_server_wait": (st, [vp, u64, ctypes.c_double]),
        "b2f_server_drain": (st, [vp, ctypes.c_double]),
        "b2f_server_stats_json": (st, [vp, ctypes.c_char_p, ctypes.POINTER(u64)]),
        "b2f_server_reset_stats": (None, [vp]),
        "b2f_server_hold": (None, [vp, ctypes.c_int32]),
        "b2f_status_string": (ctypes.c_char_p, [st]),
        "b2f_last_error_message": (u64, [ctypes.c_char_p, u64]),
        "b2f_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


class FftError(Exception):
    """FftError (src/error.rs:12-177): `kind` is the variant name."""

    def __init__(self, kind: str, code: int, message: str):
        super().__init__(f"{kind}: {message}")
        self.kind = kind
        self.code = code
        self.message = message


def _check(status: int) -> None:
    if status == 0:
        return
    L = lib()
    kind = L.b2f_status_string(status).decode()
    buf = ctypes.create_string_buffer(4096)
    L.b2f_last_error_message(buf, 4096)
    raise FftError(kind, status, buf.value.decode())


class FftDirection(enum.IntEnum):
    """FftDirection (src/config.rs:43-57)."""
    Forward = 0
    Inverse = 1


class Normalization(enum.IntEnum):
    """Normalization (src/config.rs:61-71); default Inverse."""
    NONE = 0
    Forward = 1
    Inverse = 2
    Orthogonal = 3


class FftPrecision(enum.IntEnum):
    """FftPrecision (src/config.rs:6-38)."""
    F32 = 0
    F64 = 1
    Df64 = 2

    def as_str(self) -> str:
        return ("f32", "f64", "df64")[int(self)]

    def scalar_size_bytes(self) -> int:
        return 4 if self == FftPrecision.F32 else 8

    def complex_size_bytes(self) -> int:
        return 2 * self.scalar_size_bytes()


class FftTransformKind(enum.IntEnum):
    C2c = 0
    R2c = 1
    C2r = 2


_SCALAR_TUNING = (
    "workgroup_size", "fused_workgroup_size", "rader_max_prime", "direct_max_prime",
    "large_route", "large_chunk_max_batches", "grouped_batch", "swap_to_2_stage_4_step",
    "swap_to_3_stage_4_step", "segmented_burst_depth", "max_storage_buffer_binding_size",
    "max_buffer_size", "fused_min_convolution_length", "fuse_long_axes", "fuse_small_volumes",
    "lines_per_block", "threads_per_block", "twiddle_table", "tensor_cores", "radix_order",
    "tma_tiles",
)
_TUNING_DEFAULTS = {
    "workgroup_size": 64, "fused_workgroup_size": 256, "rader_max_prime": 8192,
    "direct_max_prime": 127, "large_route": 0, "large_chunk_max_batches": None,
    "grouped_batch": None, "swap_to_2_stage_4_step": 0, "swap_to_3_stage_4_step": 0,
    "segmented_burst_depth": 2, "max_storage_buffer_binding_size": None,
    "max_buffer_size": None, "fused_min_convolution_length": 128, "fuse_long_axes": True,
    "fuse_small_volumes": True, "lines_per_block": 0, "threads_per_block": 0,
    "twiddle_table": True, "tensor_cores": False, "radix_order": 0, "tma_tiles": False,
}


class FftTuning:
    """FftTuning (src/tuning.rs:35-268): immutable builder; `with_<knob>`
    returns a copy.  Adds the B200 launch knobs lines_per_block,
    threads_per_block (0 = planner's choice) and twiddle_table."""

    def __init__(self, **values):
        self._v = dict(_TUNING_DEFAULTS)
        self._v["force_rader_axes"] = []
        self._v["force_bluestein_axes"] = []
        for k, v in values.items():
            if k not in self._v:
                raise AttributeError(k)
            self._v[k] = v

    def __getattr__(self, name):
        if name.startswith("with_"):
            key = name[5:]
            if key in self._v:
                def setter(value):
                    t = FftTuning()
                    t._v = dict(self._v)
                    t._v[key] = list(value) if key.startswith("force_") else value
                    return t
                return setter
        if name in ("_v",):
            raise AttributeError(name)
        if name in self._v:
            return self._v[name]
        raise AttributeError(name)

    def __eq__(self, other):
        return isinstance(other, FftTuning) and self._v == other._v

    def as_dict(self):
        return dict(self._v)


class FftConfig:
    """FftConfig (src/config.rs:75-286): immutable builder."""

    def __init__(self, shape: Sequence[int], axes: Optional[Sequence[int]] = None, batch: int = 1,
                 direction: FftDirection = FftDirection.Forward,
                 normalization: Normalization = Normalization.Inverse,
                 precision: FftPrecision = FftPrecision.F32,
                 tuning: Optional[FftTuning] = None):
        self._shape = [int(s) for s in shape]
        self._axes = list(range(len(self._shape))) if axes is None else [int(a) for a in axes]
        self._batch = int(batch)
        self._direction = FftDirection(direction)
        self._normalization = Normalization(normalization)
        self._precision = FftPrecision(precision)
        self._tuning = tuning if tuning is not None else FftTuning()

    # constructors (src/config.rs:86-110)
    @classmethod
    def new(cls, length: int) -> "FftConfig":
        return cls([length])

    @classmethod
    def new_nd(cls, shape: Sequence[int]) -> "FftConfig":
        return cls(shape)

    @classmethod
    def inverse(cls, length: int) -> "FftConfig":
        return cls([length], direction=FftDirection.Inverse)

    @classmethod
    def inverse_nd(cls, shape: Sequence[int]) -> "FftConfig":
        return cls(shape, direction=FftDirection.Inverse)

    def _copy(self, **kw) -> "FftConfig":
        d = dict(shape=self._shape, axes=self._axes, batch=self._batch,
                 direction=self._direction, normalization=self._normalization,
                 precision=self._precision, tuning=self._tuning)
        d.update(kw)
        return FftConfig(**d)

    def with_direction(self, d) -> "FftConfig":
        return self._copy(direction=d)

    def with_normalization(self, n) -> "FftConfig":
        return self._copy(normalization=n)

    def with_axes(self, axes) -> "FftConfig":
        return self._copy(axes=list(axes))

    def with_batch(self, b) -> "FftConfig":
        return self._copy(batch=b)

    def with_precision(self, p) -> "FftConfig":
        return self._copy(precision=p)

    def with_tuning(self, t: FftTuning) -> "FftConfig":
        return self._copy(tuning=t)

    def shape(self):
        return list(self._shape)

    def axes(self):
        return list(self._axes)

    def batch(self):
        return self._batch

    def direction(self):
        return self._direction

    def normalization(self):
        return self._normalization

    def precision(self):
        return self._precision

    def tuning(self):
        return self._tuning

    def __len__(self):
        return self._shape[0] if self._shape else 0

    _FIELDS = ("_shape", "_axes", "_batch", "_direction", "_normalization", "_precision",
               "_tuning")

    def __eq__(self, other):
        return isinstance(other, FftConfig) and all(
            getattr(self, f) == getattr(other, f) for f in self._FIELDS)

    def _handle(self) -> "_ConfigHandle":
        # the native b2f_config of this (immutable) configuration, built on
        # first use and kept for the object's lifetime
        h = self.__dict__.get("_native")
        if h is None:
            h = _ConfigHandle(self)
            self.__dict__["_native"] = h
        return h

    def validate(self) -> None:
        with self._handle() as h:
            _check(lib().b2f_config_validate(h.ptr))

    def total_complex_len(self) -> int:
        n = self._batch
        for s in self._shape:
            n *= s
        return n

    def required_buffer_size_bytes(self) -> int:
        with self._handle() as h:
            out = ctypes.c_uint64()
            _check(lib().b2f_config_required_buffer_size_bytes(h.ptr, ctypes.byref(out)))
            return out.value

    def scale(self) -> float:
        with self._handle() as h:
            f, d = ctypes.c_float(), ctypes.c_double()
            _check(lib().b2f_config_scale(h.ptr, ctypes.byref(f), ctypes.byref(d)))
            return f.value

    def scale_f64(self) -> float:
        with self._handle() as h:
            f, d = ctypes.c_float(), ctypes.c_double()
            _check(lib().b2f_config_scale(h.ptr, ctypes.byref(f), ctypes.byref(d)))
            return d.value


class _ConfigHandle:
    """The b2f_config built from an FftConfig (freed with the handle)."""

    def __init__(self, cfg: FftConfig):
        L = lib()
        self.ptr = ctypes.c_void_p()
        shape = (ctypes.c_uint64 * len(cfg._shape))(*cfg._shape)
        _check(L.b2f_config_new(ctypes.byref(self.ptr), shape, len(cfg._shape)))
        axes = (ctypes.c_uint32 * max(1, len(cfg._axes)))(*[a & 0xFFFFFFFF for a in cfg._axes])
        _check(L.b2f_config_set_axes(self.ptr, axes, len(cfg._axes)))
        _check(L.b2f_config_set_batch(self.ptr, cfg._batch & 0xFFFFFFFFFFFFFFFF))
        _check(L.b2f_config_set_direction(self.ptr, int(cfg._direction)))
        _check(L.b2f_config_set_normalization(self.ptr, int(cfg._normalization)))
        _check(L.b2f_config_set_precision(self.ptr, int(cfg._precision)))
        for k in _SCALAR_TUNING:
            v = cfg._tuning._v[k]
            v = 0 if v is None else int(v)
            _check(L.b2f_config_set_tuning(self.ptr, k.encode(), v))
        for k in ("force_rader_axes", "force_bluestein_axes"):
            ax = cfg._tuning._v[k]
            arr = (ctypes.c_uint32 * max(1, len(ax)))(*ax)
            _check(L.b2f_config_set_tuning_axes(self.ptr, k.encode(), arr, len(ax)))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def __del__(self):
        try:
            if self.ptr:
                lib().b2f_config_free(self.ptr)
        except Exception:
            pass
        self.ptr = None


Buffer = Union["torch.Tensor", Tuple[int, int]]  # noqa: F821


def _buf(b) -> Tuple[int, int]:
    if isinstance(b, tuple):
        return int(b[0]), int(b[1])
    if hasattr(b, "data_ptr"):
        if not b.is_cuda:
            raise FftError("InvalidArgument", 15, "buffers must be CUDA device memory")
        return int(b.data_ptr()), int(b.numel() * b.element_size())
    raise TypeError("buffer must be a torch CUDA tensor or an (address, nbytes) pair")


def _stream(s) -> int:
    if s is None:
        try:
            import torch
            return int(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return 0
    if isinstance(s, int):
        return s
    return int(s.cuda_stream)


class _Layout(ctypes.Structure):
    _fields_ = [("element_offset", ctypes.c_uint64), ("element_stride", ctypes.c_uint64),
                ("batch_stride", ctypes.c_uint64)]


class FftLogicalLayout:
    """FftLogicalLayout (src/runtime/logical_io.rs:34-110): logical element i
    of batch b at element element_offset + b * batch_stride + i *
    element_stride of a view (batch_stride None = the per-batch span)."""

    def __init__(self, element_offset: int = 0, element_stride: int = 1,
                 batch_stride: Optional[int] = None):
        self.element_offset = int(element_offset)
        self.element_stride = int(element_stride)
        self.batch_stride = None if batch_stride is None else int(batch_stride)

    @classmethod
    def contiguous(cls) -> "FftLogicalLayout":
        return cls()

    def with_batch_stride(self, batch_stride: int) -> "FftLogicalLayout":
        return FftLogicalLayout(self.element_offset, self.element_stride, batch_stride)

    def _c(self) -> _Layout:
        return _Layout(self.element_offset, self.element_stride, self.batch_stride or 0)


class FftPlan:
    """FftPlan (src/plan.rs:32-1300)."""

    def __init__(self, ptr: ctypes.c_void_p, config: FftConfig, kind: FftTransformKind):
        self._ptr = ptr
        self._config = config
        self._kind = kind
        self._diag = None

    @classmethod
    def _make(cls, fn, config: FftConfig, device: Optional[int], kind) -> "FftPlan":
        L = lib()
        p = ctypes.c_void_p()
        dev = -1 if device is None else int(device)
        with config._handle() as h:
            _check(getattr(L, fn)(ctypes.byref(p), h.ptr, dev))
        return cls(p, config, kind)

    @classmethod
    def c2c(cls, config: FftConfig, device: Optional[int] = None) -> "FftPlan":
        return cls._make("b2f_plan_c2c", config, device, FftTransformKind.C2c)

    @classmethod
    def r2c(cls, config: FftConfig, device: Optional[int] = None) -> "FftPlan":
        return cls._make("b2f_plan_r2c", config, device, FftTransformKind.R2c)

    @classmethod
    def c2r(cls, config: FftConfig, device: Optional[int] = None) -> "FftPlan":
        return cls._make("b2f_plan_c2r", config, device, FftTransformKind.C2r)

    @classmethod
    def plan_only(cls, config: FftConfig, kind: FftTransformKind = FftTransformKind.C2c
                  ) -> "FftPlan":
        """Runs the planner without a device (diagnostics only; cannot execute)."""
        fn = {0: "b2f_plan_c2c", 1: "b2f_plan_r2c", 2: "b2f_plan_c2r"}[int(kind)]
        return cls._make(fn, config, -2, FftTransformKind(kind))

    def __del__(self):
        try:
            if self._ptr:
                lib().b2f_plan_free(self._ptr)
                self._ptr = None
        except Exception:
            pass

    def close(self):
        self.__del__()

    # sizes and introspection (src/plan.rs:390-492, 815)
    def kind(self) -> FftTransformKind:
        return self._kind

    def config(self) -> FftConfig:
        return self._config

    def required_buffer_size_bytes(self) -> int:
        return lib().b2f_plan_required_buffer_size_bytes(self._ptr)

    def required_input_buffer_size_bytes(self) -> int:
        return lib().b2f_plan_required_input_buffer_size_bytes(self._ptr)

    def required_output_buffer_size_bytes(self) -> int:
        return lib().b2f_plan_required_output_buffer_size_bytes(self._ptr)

    def workspace_size_bytes(self) -> int:
        return lib().b2f_plan_workspace_size_bytes(self._ptr)

    def supports_in_place(self) -> bool:
        return bool(lib().b2f_plan_supports_in_place(self._ptr))

    def packed_shape(self):
        if self._kind == FftTransformKind.C2c:
            return None
        s = self._config.shape()
        s[0] = s[0] // 2 + 1
        return s

    def diagnostics(self) -> dict:
        if self._diag is None:
            L = lib()
            n = ctypes.c_uint64(0)
            _check(L.b2f_plan_diagnostics_json(self._ptr, None, ctypes.byref(n)))
            buf = ctypes.create_string_buffer(n.value + 1)
            n2 = ctypes.c_uint64(n.value + 1)
            _check(L.b2f_plan_diagnostics_json(self._ptr, buf, ctypes.byref(n2)))
            self._diag = json.loads(buf.value.decode())
        return self._diag

    def device_status(self) -> None:
        """Synchronises the plan's device and raises FftError when a bounded
        device-side wait of its kernels gave up (b2f_plan_device_status)."""
        _check(lib().b2f_plan_device_status(self._ptr))

    def route(self) -> str:
        return self.diagnostics()["route"]

    def axis_kinds(self):
        return self.diagnostics()["axis_kinds"]

    def axis_factors(self):
        return self.diagnostics()["axis_factors"]

    def factors(self):
        f = self.axis_factors()
        return f[0] if f else []

    # execution (src/plan.rs:494-879)
    def execute_checked(self, input: Buffer, output: Buffer, stream=None) -> None:
        ip, ib = _buf(input)
        op, ob = _buf(output)
        _check(lib().b2f_plan_execute_checked(self._ptr, _stream(stream), ip, ib, op, ob))

    def execute(self, input: Buffer, output: Buffer, stream=None) -> None:
        """FftPlan::execute (src/plan.rs:494): the crate panics on invalid
        buffers; here the FftError propagates."""
        self.execute_checked(input, output, stream)

    def execute_in_place(self, buffer: Buffer, stream=None) -> None:
        bp, bb = _buf(buffer)
        _check(lib().b2f_plan_execute_in_place(self._ptr, _stream(stream), bp, bb))

    def execute_logical_views(self, input: Buffer, input_layout: Optional[FftLogicalLayout],
                              output: Buffer, output_layout: Optional[FftLogicalLayout],
                              stream=None) -> None:
        """FftPlan::execute_logical_views (src/plan.rs:580-806); None is the
        contiguous layout."""
        ip, ib = _buf(input)
        op, ob = _buf(output)
        li = ctypes.byref(input_layout._c()) if input_layout is not None else None
        lo = ctypes.byref(output_layout._c()) if output_layout is not None else None
        _check(lib().b2f_plan_execute_logical_views(self._ptr, _stream(stream), ip, ib, li, op,
                                                    ob, lo))

    def record(self, recorder: "FftRecorder", input: Buffer, output: Buffer) -> None:
        ip, ib = _buf(input)
        op, ob = _buf(output)
        _check(lib().b2f_plan_record(self._ptr, recorder._ptr, ip, ib, op, ob))

    def record_in_place(self, recorder: "FftRecorder", buffer: Buffer) -> None:
        bp, bb = _buf(buffer)
        _check(lib().b2f_plan_record_in_place(self._ptr, recorder._ptr, bp, bb))


class FftBatch:
    """Many 1D complex f32 lines of mixed lengths in one persistent launch
    (b2f_batch_*): line i has lengths[i] points at complex offset offsets[i]."""

    def __init__(self, lengths, offsets, direction=FftDirection.Forward,
                 normalization=Normalization.Inverse, device: Optional[int] = None,
                 clusters: bool = False):
        L = lib()
        n = len(lengths)
        la = (ctypes.c_uint64 * n)(*[int(x) for x in lengths])
        oa = (ctypes.c_uint64 * n)(*[int(x) for x in offsets])
        self._ptr = ctypes.c_void_p()
        _check(L.b2f_batch_new_ex(ctypes.byref(self._ptr), la, oa, n, int(direction),
                                  int(normalization), -1 if device is None else int(device),
                                  1 if clusters else 0))
        self.count = n

    def required_buffer_size_bytes(self) -> int:
        return lib().b2f_batch_required_buffer_size_bytes(self._ptr)

    def execute(self, input: Buffer, output: Buffer, stream=None) -> None:
        ip, ib = _buf(input)
        op, ob = _buf(output)
        _check(lib().b2f_batch_execute(self._ptr, _stream(stream), ip, ib, op, ob))

    def execute_parts(self, input: Buffer, output: Buffer, parts: int, sequential: bool = False,
                      stream=None) -> None:
        """Runs a subset of the lines: bit 0 the CTA-queue lines, bit 1 the
        cluster lines, bit 2 the column/row passes of the long lines."""
        ip, ib = _buf(input)
        op, ob = _buf(output)
        _check(lib().b2f_batch_execute_parts(self._ptr, _stream(stream), ip, ib, op, ob, parts,
                                             int(sequential)))

    def execute_host(self, host_in, host_out, dev_in, dev_out, stream=None) -> None:
        """From and to host memory (b2f_batch_execute_host): the chunks'
        copies in, transforms and copies out overlap.  host_in/host_out are
        CPU tensors (page-locked for the copies to overlap) or (address,
        nbytes) pairs; dev_in/dev_out are the device staging buffers.
        Asynchronous on `stream` like execute()."""
        def host(b):
            if isinstance(b, tuple):
                return int(b[0]), int(b[1])
            if hasattr(b, "data_ptr"):
                if b.is_cuda:
                    raise FftError("InvalidArgument", 15, "host buffers must be CPU memory")
                return int(b.data_ptr()), int(b.numel() * b.element_size())
            raise TypeError("buffer must be a torch CPU tensor or an (address, nbytes) pair")
        hi, hib = host(host_in)
        ho, hob = host(host_out)
        di, dib = _buf(dev_in)
        do, dob = _buf(dev_out)
        _check(lib().b2f_batch_execute_host(self._ptr, _stream(stream), hi, ho, di, do,
                                            min(hib, hob, dib, dob)))

    def diagnostics(self) -> dict:
        L = lib()
        n = ctypes.c_uint64(0)
        _check(L.b2f_batch_diagnostics_json(self._ptr, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        n2 = ctypes.c_uint64(n.value + 1)
        _check(L.b2f_batch_diagnostics_json(self._ptr, buf, ctypes.byref(n2)))
        return json.loads(buf.value.decode())

    def __del__(self):
        try:
            if self._ptr:
                lib().b2f_batch_free(self._ptr)
                self._ptr = None
        except Exception:
            pass


class FftServer:
    """Serving loop (b2f_server_*): resident plans, HBM-budget admission,
    continuous batching of same-configuration requests, several streams."""

    def __init__(self, device: Optional[int] = None, hbm_budget_bytes: int = 0, streams: int = 4,
                 coalesce: bool = True):
        self._ptr = ctypes.c_void_p()
        _check(lib().b2f_server_new(ctypes.byref(self._ptr), -1 if device is None else int(device),
                                    int(hbm_budget_bytes), int(streams), int(coalesce)))
        self._keep = {}

    def submit(self, config: FftConfig, kind: FftTransformKind, host_in, host_out) -> int:
        """host_in/host_out: numpy arrays or pinned torch CPU tensors (kept
        alive until the request is waited for)."""
        ip, ib = _host_buf(host_in)
        op, ob = _host_buf(host_out)
        rid = ctypes.c_uint64()
        with config._handle() as h:
            _check(lib().b2f_server_submit(self._ptr, h.ptr, int(kind), ip, ib, op, ob,
                                           ctypes.byref(rid)))
        self._keep[rid.value] = (host_in, host_out)
        return rid.value

    def submit_device(self, config: FftConfig, kind: FftTransformKind, dev_in, dev_out) -> int:
        """b2f_server_submit_device: dev_in/dev_out are CUDA tensors or
        (address, nbytes) pairs (kept alive until the request is waited for)."""
        ip, ib = _buf(dev_in)
        op, ob = _buf(dev_out)
        rid = ctypes.c_uint64()
        with config._handle() as h:
            _check(lib().b2f_server_submit_device(self._ptr, h.ptr, int(kind), ip, ib, op, ob,
                                                  ctypes.byref(rid)))
        self._keep[rid.value] = (dev_in, dev_out)
        return rid.value

    def wait(self, request_id: int, timeout_s: float = 0.0) -> None:
        try:
            _check(lib().b2f_server_wait(self._ptr, request_id, timeout_s))
        finally:
            self._keep.pop(request_id, None)

    def drain(self, timeout_s: float = 0.0) -> None:
        _check(lib().b2f_server_drain(self._ptr, timeout_s))

    def stats(self) -> dict:
        n = ctypes.c_uint64(0)
        _check(lib().b2f_server_stats_json(self._ptr, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        n2 = ctypes.c_uint64(n.value + 1)
        _check(lib().b2f_server_stats_json(self._ptr, buf, ctypes.byref(n2)))
        return json.loads(buf.value.decode())

    def reset_stats(self) -> None:
        lib().b2f_server_reset_stats(self._ptr)

    def hold(self, held: bool = True) -> None:
        """b2f_server_hold: while held, requests queue without being
        dispatched; releasing dispatches them coalesced."""
        lib().b2f_server_hold(self._ptr, 1 if held else 0)

    def close(self):
        if self._ptr:
            lib().b2f_server_free(self._ptr)
            self._ptr = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------- autotuner and snapshot
def _json_out(fn, *args, cap: int = 1 << 20) -> str:
    """One call into a buffer of `cap` bytes (the autotuner runs once per
    call, so its report is not sized by a first call); a second, larger call
    only when the text did not fit."""
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_uint64(cap)
    st = fn(*args, buf, ctypes.byref(n))
    if st == 12 and n.value >= cap:
        buf = ctypes.create_string_buffer(n.value + 1)
        n = ctypes.c_uint64(n.value + 1)
        st = fn(*args, buf, ctypes.byref(n))
    _check(st)
    return buf.value.decode()


def validate_df64_invariants(device: Optional[int] = None) -> dict:
    """validate_df64_invariants (src/df64_canary.rs): runs the df64 canary
    on the device; raises FftError (InvariantMismatch detail) when a device
    word differs from the host's error-free transform."""
    words = (ctypes.c_uint32 * 88)()
    exact = ctypes.c_uint64(0)
    _check(lib().b2f_df64_canary(-1 if device is None else int(device), words,
                                 ctypes.byref(exact)))
    return {"cases": 4, "exact_words": int(exact.value), "words": list(words)}


def autotune(config: FftConfig, kind: FftTransformKind = FftTransformKind.C2c,
             device: Optional[int] = None, reps: int = 20) -> dict:
    """Times candidate tunings of `config` on the device (b2f_autotune),
    records the fastest one that matches the default plan's results in the
    process-wide tuning snapshot and returns the report."""
    with _ConfigHandle(config) as h:
        dev = -1 if device is None else int(device)
        return json.loads(_json_out(lib().b2f_autotune, h.ptr, int(kind), dev, int(reps)))


def tuned_config(config: FftConfig, kind: FftTransformKind = FftTransformKind.C2c):
    """(config with the snapshot's tuning for its key applied, found)."""
    L = lib()
    with _ConfigHandle(config) as h:
        found = ctypes.c_int32(0)
        _check(L.b2f_tuning_snapshot_apply(h.ptr, int(kind), ctypes.byref(found)))
        if not found.value:
            return config, False
        vals = {}
        for k in ("lines_per_block", "threads_per_block", "twiddle_table", "radix_order"):
            v = ctypes.c_int64(0)
            _check(L.b2f_config_get_tuning(h.ptr, k.encode(), ctypes.byref(v)))
            vals[k] = int(v.value)
    t = config._tuning
    t = t.with_lines_per_block(vals["lines_per_block"]).with_threads_per_block(
        vals["threads_per_block"]).with_twiddle_table(bool(vals["twiddle_table"])).with_radix_order(
        vals["radix_order"])
    return config.with_tuning(t), True


def tuning_snapshot_record(config: FftConfig, kind: FftTransformKind, lines_per_block: int,
                           threads_per_block: int, twiddle_table: int, best_us: float = 0.0,
                           default_us: float = 0.0, radix_order: int = 0) -> None:
    with _ConfigHandle(config) as h:
        _check(lib().b2f_tuning_snapshot_record(h.ptr, int(kind), lines_per_block,
                                                threads_per_block, twiddle_table, radix_order,
                                                best_us, default_us))


def tuning_snapshot_json() -> dict:
    return json.loads(_json_out(lib().b2f_tuning_snapshot_json))


def tuning_snapshot_save(path: str) -> None:
    _check(lib().b2f_tuning_snapshot_save(os.fsencode(path)))


def tuning_snapshot_load(path: str, device: Optional[int] = None) -> None:
    """Loads a snapshot file after its schema, version, integrity and (with a
    device) device checks; raises FftError and keeps the current snapshot
    otherwise."""
    _check(lib().b2f_tuning_snapshot_load(os.fsencode(path), -1 if device is None else int(device)))


def tuning_snapshot_clear() -> None:
    lib().b2f_tuning_snapshot_clear()


def _host_buf(b) -> Tuple[int, int]:
    if isinstance(b, tuple):
        return int(b[0]), int(b[1])
    if hasattr(b, "data_ptr"):
        return int(b.data_ptr()), int(b.numel() * b.element_size())
    if hasattr(b, "ctypes"):
        return int(b.ctypes.data), int(b.nbytes)
    raise TypeError("host buffer must be a numpy array, a CPU tensor or (address, nbytes)")


class FftRecorder:
    """FftRecorder (src/plan.rs:68-95): records several plans' work into one
    CUDA graph; `submit` launches it (the crate's queue.submit)."""

    def __init__(self, stream=None):
        self._ptr = ctypes.c_void_p()
        _check(lib().b2f_recorder_begin(ctypes.byref(self._ptr), _stream(stream)))
        self._finished = False

    def finish(self) -> "FftRecorder":
        if not self._finished:
            self._finished = True
            _check(lib().b2f_recorder_finish(self._ptr))
        return self

    def submit(self, stream=None) -> None:
        self.finish()
        _check(lib().b2f_recorder_submit(self._ptr, _stream(stream)))

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc, tb):
        if exc_type is None:
            self.finish()

    def __del__(self):
        try:
            if self._ptr:
                lib().b2f_recorder_free(self._ptr)
                self._ptr = None
        except Exception:
            pass
