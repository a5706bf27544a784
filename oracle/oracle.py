"""FP64 oracle for the ParaFaFT transform hot path.

TEST INFRASTRUCTURE ONLY. This module is the parity checker of the repository:
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
and only to check or time; the product path (the CUDA kernels behind
include/b200fft.h) never calls it.

Contents
--------
* C restatement (dft_oracle.c, built into _build/liboracle.so): FP64
  mixed-radix DFTs with FFTW's conventions — sign -1 forward, +1 backward,
  unnormalised; R2C keeps N/2+1 outputs; C2R ignores Im of DC and Nyquist.
  FFTW itself (the arithmetic behind FFTWBackend,
  backend/fftw3/fft_backend_fftw.hpp:74-151) is third-party and not installed
  here; its published DFT definition is what is restated.
* ParaFaFT layouts on one rank: the in-place R2C buffer holds rows of
  2*(N/2+1) reals, N data reals then 2 pad reals (parafaft_r2c.hpp:804-847,
  :1173-1178); the complex result is the row-major [..., N/2+1] half spectrum
  in the same memory; C2C results stay in natural row-major order
  (get_final_shape == the global shape, parafaft_c2c.hpp:397-420).
* Input generators restated from the reference tests
  (test/test_helpers.hpp:106-270): Gaussian (sigma 4, centre N/2), step
  (sphere of radius N/4), random cubic polynomial from the tests' LCG; and the
  seeded synthetic inputs of the benchmark configurations.
* The reference orchestrators themselves, compiled with an FP64 oracle
  backend (_ref/libref_parafaft.so, see ref_parafaft.cpp), used to produce the
  golden fixtures under tests/golden/.

Parity is pinned by: the direct O(N^2) long-double DFT (small N), analytic
known answers (plane waves, delta, constant), scipy.fft (an independent FFT),
and fixtures produced by the reference's own orchestration code. FFTW's own
outputs cannot be produced on this machine (libfftw3 absent).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBORACLE = HERE / "_build" / "liboracle.so"
LIBREF = HERE / "_ref" / "libref_parafaft.so"

_lib = None
_ref = None


def build() -> None:
    """Compile the oracle (and, where the reference headers exist, _ref)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIBORACLE.exists():
            build()
        L = C.CDLL(str(LIBORACLE))
        dp, l, i = C.POINTER(C.c_double), C.c_long, C.c_int
        L.oracle_fft1d.argtypes = [dp, l, l, i]
        L.oracle_c2c_batch.argtypes = [dp, l, l, l, l, i]
        L.oracle_r2c_batch.argtypes = [dp, dp, l, l, l, l, l]
        L.oracle_c2r_batch.argtypes = [dp, dp, l, l, l, l, l]
        L.oracle_c2c_nd.argtypes = [dp, i, C.POINTER(l), i]
        L.oracle_dft_direct.argtypes = [dp, dp, l, i]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------------------
# 1D / batched transforms (C restatement)
# ---------------------------------------------------------------------------
def dft_direct(x: np.ndarray, sign: int = -1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    lib().oracle_dft_direct(_dp(x.view(np.float64)), _dp(y.view(np.float64)), x.size, sign)
    return y


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().oracle_fft1d(_dp(y.view(np.float64)), y.size, 1, sign)
    return y


def c2c_batch(data: np.ndarray, length: int, batch: int, stride: int, dist: int,
              sign: int) -> np.ndarray:
    """Backend stage-plan semantics on a flat complex128 buffer (in place on a copy)."""
    y = np.ascontiguousarray(data, dtype=np.complex128).copy()
    lib().oracle_c2c_batch(_dp(y.view(np.float64)), length, batch, stride, dist, sign)
    return y


def c2c_nd(x: np.ndarray, sign: int = -1, impl: str = "c") -> np.ndarray:
    """n-D C2C over all axes, unnormalised."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    if impl == "scipy":
        import scipy.fft as sf
        f = sf.fftn if sign < 0 else sf.ifftn
        return f(x, norm="backward" if sign < 0 else "forward", workers=os.cpu_count())
    y = x.copy()
    shape = (C.c_long * x.ndim)(*x.shape)
    lib().oracle_c2c_nd(_dp(y.view(np.float64)), x.ndim, shape, sign)
    return y


def r2c_nd(x: np.ndarray, impl: str = "c") -> np.ndarray:
    """n-D R2C: half spectrum [..., N/2+1] (FFTW / ParaFaFT output)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    if impl == "scipy":
        import scipy.fft as sf
        return sf.rfftn(x, workers=os.cpu_count())
    n = x.shape[-1]
    nc = n // 2 + 1
    rows = x.size // n
    out = np.empty(x.shape[:-1] + (nc,), dtype=np.complex128)
    lib().oracle_r2c_batch(_dp(x), _dp(out.view(np.float64)), n, rows, 1, n, nc)
    if x.ndim > 1:
        # remaining axes are C2C on the half spectrum
        shape = out.shape
        for ax in range(x.ndim - 1):
            inner = int(np.prod(shape[ax + 1:]))
            outer = int(np.prod(shape[:ax]))
            flat = out.reshape(-1)
            step = shape[ax] * inner
            for o in range(outer):
                seg = np.ascontiguousarray(flat[o * step:(o + 1) * step])
                lib().oracle_c2c_batch(_dp(seg.view(np.float64)), shape[ax], inner, inner, 1, -1)
                flat[o * step:(o + 1) * step] = seg
            out = flat.reshape(shape)
    return out


def c2c_planes(slab, n0: int, k0s, block: int = 16) -> np.ndarray:
    """Output planes X[k0, :, :] of the unnormalised forward 3-D C2C of a grid
    too large for a full FP64 copy, in FP64 (scipy.fft / pocketfft):

        X[k0, :, :] = sum_n0 exp(-2 pi i k0 n0 / N0) * fft2(x[n0, :, :]).

    `slab(a, b)` returns x[a:b] (any complex dtype; promoted to complex128).
    The phase is reduced exactly in integers ((k0 * n0) mod N0) before the
    FP64 exponential. Slabs are taken `block` at a time and the planes are
    accumulated as one (K x block) x (block x plane) product."""
    import scipy.fft as sf
    k0s = np.asarray(list(k0s), dtype=np.int64)
    acc = None
    for a in range(0, n0, block):
        b = min(a + block, n0)
        xs = np.asarray(slab(a, b), dtype=np.complex128)
        F = sf.fft2(xs, axes=(-2, -1), workers=os.cpu_count())
        m = (k0s[:, None] * np.arange(a, b, dtype=np.int64)[None, :]) % n0
        w = np.exp(-2j * np.pi * (m.astype(np.float64) / n0))
        part = (w @ F.reshape(b - a, -1)).reshape((len(k0s),) + F.shape[1:])
        acc = part if acc is None else acc + part
    return acc


def c2r_nd(X: np.ndarray, n_last: int, impl: str = "c") -> np.ndarray:
    """n-D C2R (unnormalised); Im of DC/Nyquist of the last axis ignored."""
    X = np.ascontiguousarray(X, dtype=np.complex128)
    shape_r = X.shape[:-1] + (n_last,)
    if impl == "scipy":
        import scipy.fft as sf
        Y = X.copy()
        # FFTW's c2r ignores Im(DC) and Im(Nyquist) of the last axis after the
        # other axes are transformed back; apply the C2C part first.
        if X.ndim > 1:
            Y = sf.ifftn(Y, axes=tuple(range(X.ndim - 1)), norm="forward", workers=os.cpu_count())
        Y[..., 0] = Y[..., 0].real
        if n_last % 2 == 0:
            Y[..., n_last // 2] = Y[..., n_last // 2].real
        return sf.irfft(Y, n=n_last, axis=-1, norm="forward", workers=os.cpu_count())
    Y = X.copy()
    shape = Y.shape
    flat = Y.reshape(-1)
    for ax in range(X.ndim - 1):
        inner = int(np.prod(shape[ax + 1:]))
        outer = int(np.prod(shape[:ax]))
        step = shape[ax] * inner
        for o in range(outer):
            seg = np.ascontiguousarray(flat[o * step:(o + 1) * step])
            lib().oracle_c2c_batch(_dp(seg.view(np.float64)), shape[ax], inner, inner, 1, +1)
            flat[o * step:(o + 1) * step] = seg
    Y = flat.reshape(shape)
    nc = shape[-1]
    rows = Y.size // nc
    out = np.empty(shape_r, dtype=np.float64)
    lib().oracle_c2r_batch(_dp(Y.view(np.float64)), _dp(out), n_last, rows, 1, nc, n_last)
    return out


# ---------------------------------------------------------------------------
# ParaFaFT layouts (one rank)
# ---------------------------------------------------------------------------
def pad_real(x: np.ndarray, dtype=np.float64) -> np.ndarray:
    """Real array [..., N] -> flat padded buffer [..., 2*(N/2+1)] (pad zero)."""
    n = x.shape[-1]
    p = 2 * (n // 2 + 1)
    out = np.zeros(x.shape[:-1] + (p,), dtype=dtype)
    out[..., :n] = x
    return out.reshape(-1)


def unpad_real(buf: np.ndarray, shape) -> np.ndarray:
    n = shape[-1]
    p = 2 * (n // 2 + 1)
    return np.asarray(buf).reshape(tuple(shape[:-1]) + (p,))[..., :n]


def complex_view(buf: np.ndarray, shape) -> np.ndarray:
    """Complex half spectrum stored in a padded real buffer."""
    nc = shape[-1] // 2 + 1
    return np.asarray(buf).view(np.complex128 if buf.dtype == np.float64 else np.complex64) \
        .reshape(tuple(shape[:-1]) + (nc,))


# ---------------------------------------------------------------------------
# Reference orchestrators with the oracle backend (_ref)
# ---------------------------------------------------------------------------
def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not LIBREF.exists():
            raise FileNotFoundError(f"{LIBREF} not built (needs the ParaFaFT headers)")
        L = C.CDLL(str(LIBREF))
        vp, i, ip = C.c_void_p, C.c_int, C.POINTER(C.c_int)
        L.ref_last_error.restype = C.c_char_p
        L.ref_create.argtypes = [i, i, ip, C.POINTER(vp)]
        L.ref_destroy.argtypes = [vp]
        L.ref_forward.argtypes = [vp, vp]
        L.ref_backward.argtypes = [vp, vp]
        L.ref_forward_oop.argtypes = [vp, vp, vp]
        L.ref_backward_oop.argtypes = [vp, vp, vp]
        L.ref_required_size.argtypes = [vp]
        L.ref_required_size.restype = C.c_longlong
        L.ref_shapes.argtypes = [vp, ip, ip, ip, ip]
        _ref = L
    return _ref


class RefParaFaFT:
    """ParaFaFT_{C2C,R2C}<D, OracleBackend<double>> of the reference code (CPU)."""

    def __init__(self, kind: str, shape):
        self.L = ref_lib()
        self.kind = kind
        self.shape = tuple(int(s) for s in shape)
        arr = (C.c_int * len(self.shape))(*self.shape)
        h = C.c_void_p()
        if self.L.ref_create(0 if kind == "c2c" else 1, len(self.shape), arr, C.byref(h)):
            raise RuntimeError(self.L.ref_last_error().decode())
        self.h = h

    def _ok(self, rc):
        if rc:
            raise RuntimeError(self.L.ref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    @property
    def required_size(self) -> int:
        return int(self.L.ref_required_size(self.h))

    def shapes(self):
        D = len(self.shape)
        a, b, c, d = ((C.c_int * D)() for _ in range(4))
        self._ok(self.L.ref_shapes(self.h, a, b, c, d))
        return list(a), list(b), list(c), list(d)

    def forward(self, buf: np.ndarray) -> None:
        self._ok(self.L.ref_forward(self.h, buf.ctypes.data))

    def backward(self, buf: np.ndarray) -> None:
        self._ok(self.L.ref_backward(self.h, buf.ctypes.data))


# ---------------------------------------------------------------------------
# Input generators
# ---------------------------------------------------------------------------
SHAPE_GAUSSIAN, SHAPE_STEP, SHAPE_RANDOM_POLY = 0, 1, 2


def _grid(N: int, D: int):
    return np.meshgrid(*([np.arange(N, dtype=np.float64)] * D), indexing="ij")


def gaussian_nd(N: int, D: int, sigma: float = 4.0) -> np.ndarray:
    """test_helpers.hpp:106-130: exp(-|x - N/2|^2 / (2 sigma^2))."""
    c = N / 2.0
    r2 = sum((g - c) ** 2 for g in _grid(N, D))
    return np.exp(-r2 / (2.0 * sigma * sigma))


def step_nd(N: int, D: int) -> np.ndarray:
    """test_helpers.hpp:136-161: 1 inside the sphere of radius N/4 at N/2."""
    c = N / 2.0
    r2 = sum((g - c) ** 2 for g in _grid(N, D))
    return (r2 <= (N / 4.0) ** 2).astype(np.float64)


def lcg_coeffs(N: int, D: int) -> np.ndarray:
    """The tests' deterministic coefficients (test_helpers.hpp:176-184)."""
    n = 1 + 3 * D
    seed = (42 + D * 7 + N * 13) & 0xFFFFFFFF
    out = np.empty(n)
    for i in range(n):
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = ((seed >> 16) & 0x7FFF) / 32768.0 - 0.5
    return out


def random_poly_nd(N: int, D: int) -> np.ndarray:
    """test_helpers.hpp:168-204: c0 + sum_d c1 x + c2 x^2 + c3 x^3, x = i/N."""
    c = lcg_coeffs(N, D)
    v = np.full((N,) * D, c[0])
    for d, g in enumerate(_grid(N, D)):
        x = g / N
        v = v + c[1 + d] * x + c[1 + D + d] * x * x + c[1 + 2 * D + d] * x ** 3
    return v


def shape_data(N: int, D: int, shape_id: int) -> np.ndarray:
    """generate_c2c_data_nd (test_helpers.hpp:209-219), real part only."""
    if shape_id == SHAPE_STEP:
        return step_nd(N, D)
    if shape_id == SHAPE_RANDOM_POLY:
        return random_poly_nd(N, D)
    return gaussian_nd(N, D)


def uniform_complex(shape, seed: int) -> np.ndarray:
    """re, im i.i.d. U[-1, 1) from numpy.random.default_rng(seed)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, shape) + 1j * rng.uniform(-1.0, 1.0, shape)


def normal_complex(shape, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def normal_real(shape, seed: int, dtype=np.float64) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape, dtype=np.float64).astype(dtype, copy=False)


def gaussian_random_field(shape, seed: int, slope: float = -3.0) -> np.ndarray:
    """Zero-mean real field with P(k) ~ k^slope: white complex noise in
    k-space scaled by sqrt(P(|k|)), k = 0 set to 0, inverse R2C in FP64."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    kc = [np.fft.fftfreq(n) * n for n in shape[:-1]] + [np.arange(shape[-1] // 2 + 1, dtype=np.float64)]
    grids = np.meshgrid(*kc, indexing="ij")
    k = np.sqrt(sum(g * g for g in grids))
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (slope / 2.0)
    noise = rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)
    field = np.fft.irfftn(noise * amp, s=shape, axes=tuple(range(len(shape))))
    return field


# ---------------------------------------------------------------------------
# metrics
# ---------------------------------------------------------------------------
def rel_l2(y, ref) -> float:
    y = np.asarray(y, dtype=np.complex128 if np.iscomplexobj(y) or np.iscomplexobj(ref) else np.float64)
    ref = np.asarray(ref, dtype=y.dtype)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((y - ref).ravel()) / (den if den > 0 else 1.0))


def max_abs(y, ref) -> float:
    return float(np.max(np.abs(np.asarray(y) - np.asarray(ref)))) if np.size(ref) else 0.0
