"""The oracle against the golden fixtures and analytic known answers (CPU).

The fixtures (tests/golden/golden_cases.npz, made by tests/golden/make_golden.py)
are forward results of the reference's own ParaFaFT_C2C / ParaFaFT_R2C
orchestration code run with an FP64 oracle backend on the reference tests'
inputs. They pin the layouts and conventions; the analytic cases pin the
arithmetic independently of any FFT implementation.
"""
import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden_cases.npz"
sys.path.insert(0, str(GOLDEN.parent))
from make_golden import CASES  # noqa: E402


def load_cases():
    z = np.load(GOLDEN)
    out = []
    for name, kind, D, N, sid in CASES:
        x = O.shape_data(N, D, sid)
        digest = hashlib.sha256(np.ascontiguousarray(x).tobytes()).digest()
        out.append({"name": name, "kind": kind, "shape": (N,) * D, "input": x,
                    "output": z[f"{name}__output"],
                    "input_ok": bytes(z[f"{name}__input_sha256"]) == digest})
    return out


@pytest.mark.parametrize("case", load_cases(), ids=lambda c: c["name"])
def test_generators_reproduce_fixture_inputs(case):
    assert case["input_ok"], "generator drifted from the one the fixtures were made with"


@pytest.mark.parametrize("impl", ["c", "scipy"])
@pytest.mark.parametrize("case", load_cases(), ids=lambda c: c["name"])
def test_oracle_matches_fixture(case, impl):
    x = case["input"]
    y = O.c2c_nd(x, -1, impl) if case["kind"] == "c2c" else O.r2c_nd(x, impl)
    assert y.shape == case["output"].shape
    # the reference tests' bound (test/c2c/test_fftw_c2c_nd.cpp:119)
    assert O.max_abs(y, case["output"]) < 1e-10
    assert O.rel_l2(y, case["output"]) < 1e-13


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 17, 30, 64, 97, 120])
def test_fast_oracle_matches_direct_dft(n):
    x = O.normal_complex(n, n)
    for sign in (-1, 1):
        assert O.rel_l2(O.fft1d(x, sign), O.dft_direct(x, sign)) < 1e-14


def test_plane_wave_known_answer():
    """exp(2 pi i k.x / N) transforms to N^D at k, zero elsewhere."""
    shape = (8, 12, 10)
    k = (3, 7, 2)
    g = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    phase = sum(kk * gg / n for kk, gg, n in zip(k, g, shape))
    x = np.exp(2j * np.pi * phase)
    y = O.c2c_nd(x)
    ref = np.zeros(shape, complex)
    ref[k] = np.prod(shape)
    assert O.max_abs(y, ref) < 1e-10


def test_delta_and_constant_known_answer():
    shape = (6, 10)
    d = np.zeros(shape)
    d[0, 0] = 1.0
    assert O.max_abs(O.r2c_nd(d), np.ones((6, 6))) < 1e-14
    c = np.full(shape, 2.0)
    ref = np.zeros((6, 6), complex)
    ref[0, 0] = 2.0 * 60
    assert O.max_abs(O.r2c_nd(c), ref) < 1e-12


def test_gaussian_matches_analytic_transform():
    """A well-resolved Gaussian (sigma 4) transforms to a sampled Gaussian."""
    N, s = 64, 4.0
    x = O.gaussian_nd(N, 1, s)
    y = O.fft1d(x.astype(complex))
    k = np.fft.fftfreq(N) * N
    ref = np.sqrt(2 * np.pi) * s * np.exp(-2 * (np.pi * s * k / N) ** 2) * np.exp(-1j * np.pi * k)
    assert O.max_abs(y, ref) < 1e-9


def test_c2r_roundtrip_and_hermitian_rules():
    x = O.normal_real((5, 7, 12), 2)
    X = O.r2c_nd(x)
    assert O.rel_l2(O.c2r_nd(X, 12) / x.size, x) < 1e-14
    X2 = X.copy()
    X2[..., 0] += 0.3j      # Im(DC) ignored by the last-axis C2R
    X2[..., 6] -= 0.7j      # Im(Nyquist) ignored
    # only the leading axes' transform of these edits survives; after the
    # last-axis C2R their imaginary parts are discarded row by row
    a = O.c2r_nd(X2, 12)
    b = O.c2r_nd(X2, 12, "scipy")
    assert O.rel_l2(a, b) < 1e-13


def test_reference_orchestrator_c2c_bug_on_non_cubic_shapes():
    """ParaFaFT_C2C sizes redistributed axes with the extent of another axis
    (parafaft_c2c.hpp:826-831 use local_n[grid_dim]); on one rank any
    non-hypercubic grid gets wrong stage shapes. ParaFaFT_R2C does not
    (parafaft_r2c.hpp:1127-1135)."""
    try:
        f = O.RefParaFaFT("c2c", (8, 6, 4, 5))
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built")
    assert f.shapes()[2] != [8, 6, 4, 5]
    g = O.RefParaFaFT("r2c", (8, 6, 10))
    assert g.shapes()[2] == [8, 6, 6]


def test_plane_oracle_matches_full_transform():
    """c2c_planes (the FP64 check of grids too large for a full FP64 copy)
    against the C oracle's full 3-D transform of the same complex64 input."""
    x = O.normal_complex((24, 16, 20), 5).astype(np.complex64)
    ks = [0, 1, 7, 12, 23]
    planes = O.c2c_planes(lambda a, b: x[a:b], 24, ks, block=5)
    full = O.c2c_nd(x.astype(np.complex128))
    assert O.rel_l2(planes, full[ks]) < 1e-14
