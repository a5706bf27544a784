"""ctypes bindings of the two native libraries of parafaft_b200.

* ``libb200fft.so`` — the transform engine's C ABI (include/b200fft.h).
* ``libparafaft_b200_drivers.so`` — ParaFaFT_C2C / ParaFaFT_R2C objects (the
  reference orchestrators, compiled against B200Backend / B200GridBackend).
* ``libparafaft_cufft_drivers.so`` — the same, also on the reference
  CuFFTBackend (the comparison on the same GPU; loaded only for it).

Nothing here computes on the CPU: if a library is missing the loaders raise,
and the engine itself refuses to create a handle without a CUDA device (except
in record-only mode, which plans and counts launches but moves no data).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
ENGINE_PATH = LIB_DIR / "libb200fft.so"
DRIVERS_PATH = LIB_DIR / "libparafaft_b200_drivers.so"
CUFFT_DRIVERS_PATH = LIB_DIR / "libparafaft_cufft_drivers.so"

F32, F64 = 0, 1
FORWARD, BACKWARD = 0, 1
PLAN_ESTIMATE, PLAN_MEASURE, PLAN_PATIENT = 0, 1, 2
FLAG_NO_DEFER, FLAG_RECORD_ONLY, FLAG_GENERIC_ONLY = 1, 2, 4
FLAG_SPLIT_TC = 8  # split-precision tensor-core C2C (FP32, lengths 256/512/1024)
KIND_C2C, KIND_R2C, KIND_C2R = 0, 1, 2

STATUS = {
    0: "SUCCESS", -1: "INVALID_ARG", -2: "UNSUPPORTED", -3: "NO_PLAN", -4: "CUDA",
    -5: "RANGE", -6: "NO_DEVICE", -7: "DEVICE_STATUS",
}

# Every symbol include/b200fft.h declares.
ENGINE_SYMBOLS = (
    "b200fft_last_error", "b200fft_version", "b200fft_device_count",
    "b200fft_create", "b200fft_destroy", "b200fft_set_stream",
    "b200fft_plan_c2c", "b200fft_exec_c2c", "b200fft_plan_r2c", "b200fft_exec_r2c",
    "b200fft_plan_c2r", "b200fft_exec_c2r", "b200fft_memcpy", "b200fft_memcpy2d",
    "b200fft_sync", "b200fft_flush", "b200fft_alloc", "b200fft_free",
    "b200fft_get_stats", "b200fft_reset_stats", "b200fft_get_log", "b200fft_set_profiling",
    "b200fft_describe", "b200fft_supported", "b200fft_c2c_noalloc",
    "b200fft_group_create", "b200fft_group_destroy", "b200fft_group_add",
    "b200fft_group_begin", "b200fft_group_end", "b200fft_group_capture",
    "b200fft_group_replay", "b200fft_group_sync", "b200fft_group_stats",
    "b200fft_set_work_buffer", "b200fft_plan_describe", "b200fft_export_wisdom",
    "b200fft_import_wisdom", "b200fft_forget_wisdom",
)


class B200FFTError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "kernel_launches", "exec_calls", "coalesced_calls", "memcpy_calls",
        "fused_copies", "copies_issued", "bytes_copied", "bytes_transformed")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class LaunchRecord(C.Structure):
    _fields_ = [("kind", C.c_int), ("direction", C.c_int), ("stage", C.c_int),
                ("family", C.c_int), ("length", C.c_int), ("fused_copy", C.c_int),
                ("transforms", C.c_longlong), ("slabs", C.c_longlong),
                ("bytes", C.c_longlong), ("ms", C.c_double)]

    def as_dict(self) -> dict:
        d = {n: int(getattr(self, n)) for n, _ in self._fields_ if n != "ms"}
        d["ms"] = float(self.ms)
        return d


_engine = None
_drivers = {}


def engine() -> C.CDLL:
    """Load libb200fft.so (raises if it has not been built)."""
    global _engine
    if _engine is None:
        if not ENGINE_PATH.exists():
            raise ImportError(f"{ENGINE_PATH} is missing: run `python -m parafaft_b200.build`")
        lib = C.CDLL(str(ENGINE_PATH))
        vp, i, sz, pd = C.c_void_p, C.c_int, C.c_size_t, C.c_ssize_t
        sig = {
            "b200fft_last_error": (C.c_char_p, []),
            "b200fft_version": (i, []),
            "b200fft_device_count": (i, []),
            "b200fft_create": (i, [i, i, i, C.c_uint, C.POINTER(vp)]),
            "b200fft_destroy": (i, [vp]),
            "b200fft_set_stream": (i, [vp, vp]),
            "b200fft_plan_c2c": (i, [vp, i, i, sz, pd, pd]),
            "b200fft_exec_c2c": (i, [vp, i, i, vp]),
            "b200fft_plan_r2c": (i, [vp, i, sz, pd, pd]),
            "b200fft_exec_r2c": (i, [vp, vp]),
            "b200fft_plan_c2r": (i, [vp, i, sz, pd, pd]),
            "b200fft_exec_c2r": (i, [vp, vp]),
            "b200fft_memcpy": (i, [vp, vp, vp, sz]),
            "b200fft_memcpy2d": (i, [vp, vp, sz, vp, sz, sz, sz]),
            "b200fft_sync": (i, [vp]),
            "b200fft_flush": (i, [vp]),
            "b200fft_alloc": (i, [sz, C.POINTER(vp)]),
            "b200fft_free": (i, [vp]),
            "b200fft_get_stats": (i, [vp, C.POINTER(Stats)]),
            "b200fft_reset_stats": (i, [vp]),
            "b200fft_get_log": (i, [vp, C.POINTER(LaunchRecord), i, C.POINTER(i)]),
            "b200fft_set_profiling": (i, [vp, i]),
            "b200fft_describe": (i, [i, i, i, sz, pd, pd, C.c_char_p, sz]),
            "b200fft_supported": (i, [i, i, i]),
            "b200fft_c2c_noalloc": (i, [i, i, i, sz, pd, pd, vp, vp, vp]),
            "b200fft_group_create": (i, [C.POINTER(vp)]),
            "b200fft_group_destroy": (i, [vp]),
            "b200fft_group_add": (i, [vp, vp]),
            "b200fft_group_begin": (i, [vp]),
            "b200fft_group_end": (i, [vp]),
            "b200fft_group_capture": (i, [vp]),
            "b200fft_group_replay": (i, [vp]),
            "b200fft_group_sync": (i, [vp]),
            "b200fft_group_stats": (i, [vp, C.POINTER(Stats)]),
            "b200fft_set_work_buffer": (i, [vp, vp, sz]),
            "b200fft_plan_describe": (i, [vp, i, i, C.c_char_p, sz]),
            "b200fft_export_wisdom": (i, [C.c_char_p]),
            "b200fft_import_wisdom": (i, [C.c_char_p]),
            "b200fft_forget_wisdom": (i, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _engine = lib
    return _engine


def drivers(cufft: bool = False) -> C.CDLL:
    """Load the ParaFaFT driver library (raises if it has not been built):
    the B200 one, or with `cufft` the comparator build that also holds
    CuFFTBackend objects."""
    path = CUFFT_DRIVERS_PATH if cufft else DRIVERS_PATH
    if path not in _drivers:
        engine()  # resolve libb200fft first
        if not path.exists():
            raise ImportError(f"{path} is missing: build it where the ParaFaFT headers exist")
        lib = C.CDLL(str(path))
        vp, i = C.c_void_p, C.c_int
        ip = C.POINTER(C.c_int)
        for name, res, args in (
            ("pfb_last_error", C.c_char_p, []),
            ("pfb_create", i, [i, i, i, i, ip, i, C.POINTER(vp)]),
            ("pfb_destroy", i, [vp]),
            ("pfb_forward", i, [vp, vp]),
            ("pfb_backward", i, [vp, vp]),
            ("pfb_forward_oop", i, [vp, vp, vp]),
            ("pfb_backward_oop", i, [vp, vp, vp]),
            ("pfb_required_size", C.c_longlong, [vp]),
            ("pfb_shapes", i, [vp, ip, ip, ip, ip]),
            ("pfb_b200_handle", vp, [vp]),
            ("pfb_buffer", vp, [vp]),
        ):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _drivers[path] = lib
    return _drivers[path]


def check(rc: int) -> None:
    if rc != 0:
        raise B200FFTError(rc, engine().b200fft_last_error().decode())


def _ptr(x) -> int:
    """Device/host address of a torch tensor, an int, or None."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


class Handle:
    """One engine handle (what a B200Backend<T> object owns)."""

    def __init__(self, precision: int = F32, num_stages: int = 1,
                 plan_flag: int = PLAN_ESTIMATE, flags: int = 0):
        self._lib = engine()
        h = C.c_void_p()
        check(self._lib.b200fft_create(precision, num_stages, plan_flag, flags, C.byref(h)))
        self._h = h
        self.precision = precision

    @classmethod
    def wrap(cls, raw: int) -> "Handle":
        """Borrow an existing handle (not destroyed by this object)."""
        obj = cls.__new__(cls)
        obj._lib = engine()
        obj._h = C.c_void_p(raw)
        obj.precision = None
        obj._borrowed = True
        return obj

    @property
    def raw(self) -> int:
        return self._h.value or 0

    def close(self) -> None:
        if getattr(self, "_borrowed", False):
            return
        if self._h:
            check(self._lib.b200fft_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan_c2c(self, stage, length, batch, stride, dist):
        check(self._lib.b200fft_plan_c2c(self._h, stage, length, batch, stride, dist))

    def exec_c2c(self, stage, direction, data):
        check(self._lib.b200fft_exec_c2c(self._h, stage, direction, _ptr(data)))

    def plan_r2c(self, length, batch, stride, dist):
        check(self._lib.b200fft_plan_r2c(self._h, length, batch, stride, dist))

    def exec_r2c(self, data):
        check(self._lib.b200fft_exec_r2c(self._h, _ptr(data)))

    def plan_c2r(self, length, batch, stride, dist):
        check(self._lib.b200fft_plan_c2r(self._h, length, batch, stride, dist))

    def exec_c2r(self, data):
        check(self._lib.b200fft_exec_c2r(self._h, _ptr(data)))

    def memcpy(self, dst, src, nbytes):
        check(self._lib.b200fft_memcpy(self._h, _ptr(dst), _ptr(src), nbytes))

    def memcpy2d(self, dst, dpitch, src, spitch, width, height):
        check(self._lib.b200fft_memcpy2d(self._h, _ptr(dst), dpitch, _ptr(src), spitch,
                                         width, height))

    def set_stream(self, stream: int | None):
        check(self._lib.b200fft_set_stream(self._h, stream or 0))

    def sync(self):
        check(self._lib.b200fft_sync(self._h))

    def flush(self):
        check(self._lib.b200fft_flush(self._h))

    def stats(self) -> dict:
        s = Stats()
        check(self._lib.b200fft_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        check(self._lib.b200fft_reset_stats(self._h))

    def set_work_buffer(self, data, nbytes: int = 0):
        check(self._lib.b200fft_set_work_buffer(self._h, _ptr(data), nbytes))

    def plan_describe(self, kind: int = KIND_C2C, stage: int = 0) -> str:
        buf = C.create_string_buffer(256)
        check(self._lib.b200fft_plan_describe(self._h, kind, stage, buf, 256))
        return buf.value.decode()

    def set_profiling(self, on: bool = True):
        check(self._lib.b200fft_set_profiling(self._h, 1 if on else 0))

    def log(self, cap: int = 4096) -> list[dict]:
        buf = (LaunchRecord * cap)()
        n = C.c_int()
        check(self._lib.b200fft_get_log(self._h, buf, cap, C.byref(n)))
        return [buf[i].as_dict() for i in range(n.value)]


class Group:
    """b200fft_group: transforms of many handles launched together."""

    def __init__(self, handles=()):
        self._lib = engine()
        g = C.c_void_p()
        check(self._lib.b200fft_group_create(C.byref(g)))
        self._g = g
        self.members = []
        for h in handles:
            self.add(h)

    def add(self, h: "Handle"):
        check(self._lib.b200fft_group_add(self._g, h.raw))
        self.members.append(h)

    def begin(self):
        check(self._lib.b200fft_group_begin(self._g))

    def end(self):
        check(self._lib.b200fft_group_end(self._g))

    def capture(self):
        check(self._lib.b200fft_group_capture(self._g))

    def replay(self):
        check(self._lib.b200fft_group_replay(self._g))

    def sync(self):
        check(self._lib.b200fft_group_sync(self._g))

    def stats(self) -> dict:
        s = Stats()
        check(self._lib.b200fft_group_stats(self._g, C.byref(s)))
        d = s.as_dict()
        d["passes_per_run"] = d.pop("coalesced_calls")
        d["runs"] = d.pop("exec_calls")
        return d

    def close(self):
        if self._g:
            check(self._lib.b200fft_group_destroy(self._g))
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def describe(precision: int, kind: int, length: int, batch: int = 1, stride: int = 1,
             dist: int | None = None) -> str:
    if dist is None:
        dist = length if kind == KIND_C2C else 2 * (length // 2 + 1)
    buf = C.create_string_buffer(256)
    check(engine().b200fft_describe(precision, kind, length, batch, stride, dist, buf, 256))
    return buf.value.decode()


def c2c_noalloc(precision: int, direction: int, length: int, batch: int, stride: int,
                dist: int, data_in, data_out, stream: int | None = None) -> None:
    """b200fft_c2c_noalloc: one batched C2C transform without a handle and
    without any device allocation (power-of-two lengths up to 4096)."""
    check(engine().b200fft_c2c_noalloc(precision, direction, length, batch, stride, dist,
                                       _ptr(data_in), _ptr(data_out), stream or 0))


def export_wisdom(path: str) -> None:
    check(engine().b200fft_export_wisdom(str(path).encode()))


def import_wisdom(path: str) -> int:
    n = engine().b200fft_import_wisdom(str(path).encode())
    if n < 0:
        check(n)
    return n


def forget_wisdom() -> None:
    check(engine().b200fft_forget_wisdom())


def supported(precision: int, kind: int, length: int) -> bool:
    return bool(engine().b200fft_supported(precision, kind, length))


class ParaFaFT:
    """A ParaFaFT_C2C<D, B> or ParaFaFT_R2C<D, B> object of the reference code.

    kind: "c2c" or "r2c" (the reference orchestrators), or "c2c_onerank" (the
    same backend call sequence with per-axis extents, for grids that are not
    hypercubic); backend: "b200" (B200Backend<T>), "b200grid"
    (B200GridBackend<D, T>, which owns the grid: forward/backward transform
    the buffer() it holds and ignore their argument) or "cufft" (the reference
    CuFFTBackend<T>, for comparison). Data arguments are device pointers (ints)
    or CUDA torch tensors.
    """

    def __init__(self, kind: str, shape, precision: int = F32, backend: str = "b200",
                 plan_flag: int = PLAN_ESTIMATE):
        self._lib = drivers(cufft=backend == "cufft")
        self.kind = kind
        self.shape = tuple(int(s) for s in shape)
        self.D = len(self.shape)
        self.precision = precision
        arr = (C.c_int * self.D)(*self.shape)
        h = C.c_void_p()
        kinds = {"c2c": 0, "r2c": 1, "c2c_onerank": 2}
        backends = {"b200": 0, "cufft": 1, "b200grid": 2}
        rc = self._lib.pfb_create(kinds[kind], self.D, precision, backends[backend], arr,
                                  plan_flag, C.byref(h))
        if rc != 0:
            raise RuntimeError("ParaFaFT construction failed: " + self._lib.pfb_last_error().decode())
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self._lib.pfb_last_error().decode())

    def close(self):
        if self._h:
            self._check(self._lib.pfb_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, data):
        """C2C forward() / R2C forward_in_place()."""
        self._check(self._lib.pfb_forward(self._h, _ptr(data)))

    def backward(self, data):
        """C2C backward() / R2C backward_in_place()."""
        self._check(self._lib.pfb_backward(self._h, _ptr(data)))

    def forward_oop(self, real_in, complex_out):
        self._check(self._lib.pfb_forward_oop(self._h, _ptr(real_in), _ptr(complex_out)))

    def backward_oop(self, complex_in, real_out):
        self._check(self._lib.pfb_backward_oop(self._h, _ptr(complex_in), _ptr(real_out)))

    @property
    def required_size(self) -> int:
        """get_required_output_size(): Complex elements (C2C) / FloatType scalars (R2C)."""
        return int(self._lib.pfb_required_size(self._h))

    def shapes(self) -> dict:
        a, b, c, d = ((C.c_int * self.D)() for _ in range(4))
        self._check(self._lib.pfb_shapes(self._h, a, b, c, d))
        return {"in_shape": list(a), "in_start": list(b), "out_shape": list(c),
                "out_start": list(d)}

    def buffer(self):
        """The grid a grid-owning backend holds, as a CUDA torch tensor viewing
        it (complex for C2C, the padded reals for R2C), or None."""
        import torch
        raw = self._lib.pfb_buffer(self._h)
        if not raw:
            return None
        n = self.shape[-1]
        rows = 1
        for s in self.shape[:-1]:
            rows *= s
        f64 = self.precision == F64
        if self.kind == "r2c":
            count, typestr = rows * 2 * (n // 2 + 1), "<f8" if f64 else "<f4"
        else:
            count, typestr = rows * n, "<c16" if f64 else "<c8"

        class _View:
            __cuda_array_interface__ = {"shape": (count,), "typestr": typestr,
                                        "data": (int(raw), False), "version": 2}
        return torch.as_tensor(_View(), device="cuda")

    def handle(self) -> Handle | None:
        raw = self._lib.pfb_b200_handle(self._h)
        return Handle.wrap(raw) if raw else None
