"""The reference orchestrators (ParaFaFT_C2C / ParaFaFT_R2C, compiled from the
reference headers) running on B200Backend: results against the FP64 oracle,
the golden fixtures, and the reference's own cuFFT backend on the same GPU.

Mirrors the reference's integration tests at np=1:
test/c2c/test_fftw_c2c_nd.cpp (1e-10 max-abs vs serial FFTW),
test/c2c/test_fftw_c2c_nd_float.cpp (1e-4 * peak),
test/c2c/test_fftw_c2c_roundtrip_nd.cpp, test/r2c/test_fftw_r2c_padded_nd.cpp,
test/r2c/test_fftw_r2c_padded_roundtrip_nd.cpp, over the matrix
N in {32 (D=2,3), 16 (D=4), 8 (D=5)} x shapes {Gaussian, step, polynomial}
(test/CMakeLists.txt:215-271).
"""
import numpy as np
import pytest

from helpers import ABS_F64, cdtype, rdtype, to_dev, to_host, tol
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

MATRIX = [(2, 32), (3, 32), (4, 16), (5, 8)]
SHAPES = [O.SHAPE_GAUSSIAN, O.SHAPE_STEP, O.SHAPE_RANDOM_POLY]


def _drivers_or_skip():
    try:
        nv.drivers()
    except ImportError as e:
        pytest.skip(str(e))


@pytest.mark.parametrize("D,N", MATRIX)
@pytest.mark.parametrize("shape_id", SHAPES)
@pytest.mark.parametrize("prec", [nv.F64, nv.F32])
def test_c2c_nd_matches_oracle(D, N, shape_id, prec):
    _drivers_or_skip()
    shape = (N,) * D
    x = O.shape_data(N, D, shape_id).astype(np.complex128)
    f = nv.ParaFaFT("c2c", shape, prec)
    s = f.shapes()
    assert s["in_shape"] == list(shape) and s["out_shape"] == list(shape)
    buf = np.zeros(f.required_size, dtype=cdtype(prec))
    buf[:x.size] = x.ravel()
    d = to_dev(buf)
    f.forward(d)
    y = to_host(d)[:x.size].reshape(shape)
    ref = O.c2c_nd(x)
    if prec == nv.F64:
        assert O.max_abs(y, ref) < ABS_F64
    else:
        assert O.max_abs(y, ref) < 1e-4 * np.max(np.abs(ref))
    assert O.rel_l2(y, ref) < tol(prec)
    f.backward(d)
    back = to_host(d)[:x.size].reshape(shape) / x.size
    assert O.rel_l2(back, x) < tol(prec)


@pytest.mark.parametrize("D,N", MATRIX)
@pytest.mark.parametrize("shape_id", SHAPES)
@pytest.mark.parametrize("prec", [nv.F64, nv.F32])
def test_r2c_padded_nd_matches_oracle(D, N, shape_id, prec):
    _drivers_or_skip()
    shape = (N,) * D
    x = O.shape_data(N, D, shape_id)
    f = nv.ParaFaFT("r2c", shape, prec)
    buf = np.zeros(f.required_size, dtype=rdtype(prec))
    p = O.pad_real(x, rdtype(prec))
    buf[:p.size] = p
    d = to_dev(buf)
    f.forward(d)
    h = to_host(d)
    nc = N // 2 + 1
    X = h[:2 * x.size // N * nc].view(cdtype(prec)).reshape(shape[:-1] + (nc,))
    ref = O.r2c_nd(x)
    if prec == nv.F64:
        assert O.max_abs(X, ref) < ABS_F64
    assert O.rel_l2(X, ref) < tol(prec)
    f.backward(d)
    back = O.unpad_real(to_host(d)[:p.size], shape) / x.size
    assert O.rel_l2(back, x) < tol(prec)


@pytest.mark.parametrize("shape", [(16, 12, 10), (8, 20, 6), (10, 6), (12, 10, 6, 4)])
@pytest.mark.parametrize("prec", [nv.F64, nv.F32])
def test_r2c_non_cubic(shape, prec):
    """ParaFaFT_R2C decomposes each axis with its own extent
    (parafaft_r2c.hpp:1127-1135), so non-cubic grids are valid there."""
    _drivers_or_skip()
    x = O.normal_real(shape, 21)
    f = nv.ParaFaFT("r2c", shape, prec)
    buf = np.zeros(f.required_size, dtype=rdtype(prec))
    p = O.pad_real(x, rdtype(prec))
    buf[:p.size] = p
    d = to_dev(buf)
    f.forward(d)
    nc = shape[-1] // 2 + 1
    X = to_host(d)[:p.size].view(cdtype(prec)).reshape(shape[:-1] + (nc,))
    assert O.rel_l2(X, O.r2c_nd(x)) < tol(prec)


@pytest.mark.parametrize("prec", [nv.F64, nv.F32])
def test_r2c_out_of_place(prec):
    """forward(real_in, complex_out) / backward(complex_in, real_out)
    (parafaft_r2c.hpp:333-339, :446-453): pad/unpad through memcpy2d."""
    _drivers_or_skip()
    shape = (12, 16, 18)
    x = O.normal_real(shape, 4).astype(rdtype(prec))
    f = nv.ParaFaFT("r2c", shape, prec)
    rin = to_dev(x.reshape(-1))
    cout = to_dev(np.zeros(f.required_size, dtype=rdtype(prec)))
    f.forward_oop(rin, cout)
    nc = shape[-1] // 2 + 1
    X = to_host(cout)[:2 * 12 * 16 * nc].view(cdtype(prec)).reshape(12, 16, nc)
    assert O.rel_l2(X, O.r2c_nd(x.astype(np.float64))) < tol(prec)
    rout = to_dev(np.zeros_like(x).reshape(-1))
    f.backward_oop(cout, rout)
    assert O.rel_l2(to_host(rout).reshape(shape) / x.size, x) < tol(prec)


@pytest.mark.parametrize("prec", [nv.F64, nv.F32])
@pytest.mark.parametrize("shape", [(12, 16, 18), (8, 10, 15), (16, 32)])
def test_fused_pad_matches_unfused(prec, shape, monkeypatch):
    """The out-of-place forward's pad (memcpy2d) fused into the R2C pass gives
    bit-for-bit the result of copy-then-transform (B200FFT_NO_DEFER), leaves
    the real input untouched, and issues no copy for odd D. Odd last axes take
    the generic kernel (input rows in real units), even ones the specialised
    one."""
    _drivers_or_skip()
    x = O.normal_real(shape, 5).astype(rdtype(prec))
    f = nv.ParaFaFT("r2c", shape, prec)
    monkeypatch.setenv("B200FFT_NO_DEFER", "1")
    g = nv.ParaFaFT("r2c", shape, prec)
    monkeypatch.delenv("B200FFT_NO_DEFER")
    outs = []
    for obj in (f, g):
        rin = to_dev(x.reshape(-1))
        cout = to_dev(np.full(obj.required_size, 7.0, dtype=rdtype(prec)))
        obj.handle().reset_stats()
        obj.forward_oop(rin, cout)
        st = obj.handle().stats()
        np.testing.assert_array_equal(to_host(rin).reshape(shape), x)
        outs.append((to_host(cout), st))
    (yf, sf), (yu, su) = outs
    n = 2 * (x.size // shape[-1]) * (shape[-1] // 2 + 1)
    np.testing.assert_array_equal(yf[:n], yu[:n])
    # For even D, forward_in_place first copies the padded output into the
    # scratch buffer (D-1 odd), so the pad is issued and that copy is fused.
    assert sf["copies_issued"] == (0 if len(shape) % 2 else 1)
    assert su["copies_issued"] >= 1
    nc = shape[-1] // 2 + 1
    X = yf[:n].view(cdtype(prec)).reshape(shape[:-1] + (nc,))
    assert O.rel_l2(X, O.r2c_nd(x.astype(np.float64))) < tol(prec)


def test_fusion_through_orchestrator():
    """ParaFaFT_R2C<3> forward+backward: 2 x (1 + N0 + 1) backend calls and
    4 exchange copies become 6 launches and no copies."""
    _drivers_or_skip()
    shape = (16, 16, 16)
    f = nv.ParaFaFT("r2c", shape, nv.F32)
    h = f.handle()
    h.reset_stats()
    d = to_dev(np.zeros(f.required_size, dtype=np.float32))
    f.forward(d)
    f.backward(d)
    st = h.stats()
    assert st["kernel_launches"] == 6
    assert st["exec_calls"] == 2 * (2 + 16)
    assert st["fused_copies"] == 4 and st["copies_issued"] == 0


@pytest.mark.parametrize("kind,shape", [("r2c", (32, 32, 32)), ("c2c", (32, 32, 32)),
                                        ("c2c", (16, 16, 16, 16))])
@pytest.mark.parametrize("prec", [nv.F32, nv.F64])
def test_matches_reference_cufft_backend(kind, shape, prec):
    """Same inputs through ParaFaFT with the reference CuFFTBackend and with
    B200Backend agree to the precision's tolerance."""
    _drivers_or_skip()
    a = nv.ParaFaFT(kind, shape, prec, backend="b200")
    b = nv.ParaFaFT(kind, shape, prec, backend="cufft")
    if kind == "c2c":
        x = O.uniform_complex(shape, 9).astype(cdtype(prec))
        buf = np.zeros(a.required_size, dtype=cdtype(prec))
        buf[:x.size] = x.ravel()
    else:
        x = O.normal_real(shape, 9)
        buf = np.zeros(a.required_size, dtype=rdtype(prec))
        p = O.pad_real(x, rdtype(prec))
        buf[:p.size] = p
    da, db = to_dev(buf), to_dev(buf)
    a.forward(da)
    b.forward(db)
    ya, yb = to_host(da), to_host(db)
    n = x.size if kind == "c2c" else 2 * (x.size // shape[-1]) * (shape[-1] // 2 + 1)
    assert O.rel_l2(ya[:n], yb[:n]) < 2 * tol(prec)


def test_golden_fixtures_on_gpu():
    """The golden fixtures (reference orchestrator + FP64 oracle) reproduced by
    ParaFaFT on B200Backend<double>."""
    _drivers_or_skip()
    from test_golden import load_cases
    for case in load_cases():
        shape = tuple(case["shape"])
        if case["kind"] == "c2c":
            f = nv.ParaFaFT("c2c", shape, nv.F64)
            buf = np.zeros(f.required_size, dtype=np.complex128)
            buf[:case["input"].size] = case["input"].ravel()
            d = to_dev(buf)
            f.forward(d)
            y = to_host(d)[:case["input"].size].reshape(case["output"].shape)
        else:
            f = nv.ParaFaFT("r2c", shape, nv.F64)
            buf = np.zeros(f.required_size, dtype=np.float64)
            p = O.pad_real(case["input"])
            buf[:p.size] = p
            d = to_dev(buf)
            f.forward(d)
            nc = shape[-1] // 2 + 1
            y = to_host(d)[:p.size].view(np.complex128).reshape(case["output"].shape)
        assert O.max_abs(y, case["output"]) < ABS_F64, case["name"]
        assert O.rel_l2(y, case["output"]) < 1e-12, case["name"]


@pytest.mark.parametrize("flag", [nv.PLAN_MEASURE, nv.PLAN_PATIENT])
def test_measured_plans(flag, tmp_path):
    """FFTPlanFlag::Measure/Patient: candidates are timed on ParaFaFT's scratch
    buffer at construction; the chosen kernels give the same results and the
    choices land in the plan cache (wisdom)."""
    _drivers_or_skip()
    nv.forget_wisdom()
    shape = (64, 96, 128)
    x = O.normal_real(shape, 31)
    f = nv.ParaFaFT("r2c", shape, nv.F32, plan_flag=flag)
    buf = np.zeros(f.required_size, np.float32)
    p = O.pad_real(x, np.float32)
    buf[:p.size] = p
    d = to_dev(buf)
    f.forward(d)
    X = to_host(d)[:p.size].view(np.complex64).reshape(64, 96, 65)
    assert O.rel_l2(X, O.r2c_nd(x)) < 2e-6
    w = tmp_path / "w.txt"
    nv.export_wisdom(w)
    entries = w.read_text().splitlines()[1:]
    assert len(entries) >= 3  # r2c, c2r and the two column stages (c2r may share)
    # a second object of the same geometry reuses the entries
    g = nv.ParaFaFT("r2c", shape, nv.F32, plan_flag=flag)
    h1, h2 = f.handle(), g.handle()
    for stage in (1, 2):
        assert h1.plan_describe(nv.KIND_C2C, stage) == h2.plan_describe(nv.KIND_C2C, stage)
