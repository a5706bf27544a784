"""The TMA-fed column passes (tile variants 8 and 9) against the FP64 oracle.

FP32 C2C columns of 256, 512 and 1024 points whose point rows are 16-byte
aligned stream their tiles into shared memory with bulk tensor copies; 256-
and 512-point columns at an odd point stride whose transforms are whole point
rows (the middle axis of a padded R2C grid) read them through a map of double
rows. Every other plan given these variants runs its default tile instead.
The launch log tells which kernel ran (family 4 = a TMA column kernel).
"""
import numpy as np
import pytest

from helpers import cdtype, to_dev, to_host, tol
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

TMA_FAMILY = 4


def _column_case(length, batch, stride, direction, seed):
    span = (length - 1) * stride + batch
    x = O.normal_complex(span, seed)
    h = nv.Handle(nv.F32, 1)
    h.set_profiling(True)
    h.plan_c2c(0, length, batch, stride, 1)
    d = to_dev(x.astype(cdtype(nv.F32)))
    h.exec_c2c(0, direction, d)
    h.sync()
    y = to_host(d)
    ref = O.c2c_batch(x, length, batch, stride, 1, -1 if direction == nv.FORWARD else +1)
    fams = {r["family"] for r in h.log()}
    h.close()
    return y, ref, fams, x


@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("length", [256, 512, 1024])
@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
def test_tma_columns(variant, length, direction, monkeypatch):
    """Whole and partial tiles (the last tile's missing columns are read as
    zeros by the tensor copy and never stored), stride wider than the batch."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    for batch, stride in ((70, 70), (4096 + 6, 4096 + 6), (150, 160)):
        y, ref, fams, x = _column_case(length, batch, stride, direction, seed=length + batch)
        assert fams == {TMA_FAMILY}, (length, batch, fams)
        assert O.rel_l2(y, ref) < tol(nv.F32), (variant, length, batch, stride)
        # the columns between batch and stride are not part of the transform
        if stride > batch:
            assert np.array_equal(y.reshape(-1)[batch:stride],
                                  x[batch:stride].astype(np.complex64))


@pytest.mark.parametrize("variant", [8, 9])
def test_tma_ineligible_plans_fall_back(variant, monkeypatch):
    """An odd stride wider than the batch (rows neither 16-byte aligned nor
    whole double rows of transforms), a non-TMA length and FP64 run the
    default tile and give the same results."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    y, ref, fams, _ = _column_case(512, 200, 257, nv.FORWARD, seed=1)
    assert fams == {0} and O.rel_l2(y, ref) < tol(nv.F32)
    y, ref, fams, _ = _column_case(128, 64, 64, nv.FORWARD, seed=2)
    assert fams == {0} and O.rel_l2(y, ref) < tol(nv.F32)
    x = O.normal_complex(511 * 64 + 64, 3)
    h = nv.Handle(nv.F64, 1)
    h.plan_c2c(0, 512, 64, 64, 1)
    d = to_dev(x.astype(cdtype(nv.F64)))
    h.exec_c2c(0, nv.FORWARD, d)
    h.sync()
    assert O.rel_l2(to_host(d), O.c2c_batch(x, 512, 64, 64, 1, -1)) < tol(nv.F64)
    h.close()


@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("shape", [(4, 512, 48), (6, 256, 40), (1024, 3, 8)])
def test_tma_through_parafaft(variant, shape, monkeypatch):
    """ParaFaFT's C2C call sequence on B200Backend<float> (the one-rank form,
    which sizes non-cubic grids correctly): the middle axis runs as coalesced
    slabs (3D tensor map, one slab per box), the first axis as one slab, both
    reading the held exchange copy's source; forward against numpy FP64 and
    the round trip."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    n = int(np.prod(shape))
    x = O.normal_complex(n, sum(shape))
    f = nv.ParaFaFT("c2c_onerank", shape, nv.F32)
    buf = np.zeros(f.required_size, np.complex64)
    buf[:n] = x
    d = to_dev(buf)
    f.handle().set_profiling(True)
    f.forward(d)
    y = to_host(d)[:n].reshape(shape)
    ref = np.fft.fftn(x.reshape(shape))
    assert O.rel_l2(y, ref) < tol(nv.F32), shape
    fams = {r["family"] for r in f.handle().log() if r["kind"] == 0}
    assert TMA_FAMILY in fams, (shape, fams)
    f.backward(d)
    z = to_host(d)[:n] / n
    assert O.rel_l2(z, x) < tol(nv.F32)
    f.close()


def test_tma_wait_timeout_reports_device_status(monkeypatch):
    """Every CTA skips the copies of its first tile (B200FFT_TMA_STALL_TEST):
    the bounded wait runs out after about a second, the CTA waits for its
    other copies and returns, sync reports B200FFT_ERR_DEVICE_STATUS, and the
    next launch on the same context is correct."""
    monkeypatch.setenv("B200FFT_VARIANT", "8")
    length, batch = 512, 64
    x = O.normal_complex((length - 1) * batch + batch, 11)
    h = nv.Handle(nv.F32, 1)
    h.plan_c2c(0, length, batch, batch, 1)
    d = to_dev(x.astype(np.complex64))
    monkeypatch.setenv("B200FFT_TMA_STALL_TEST", "1")
    h.exec_c2c(0, nv.FORWARD, d)
    with pytest.raises(nv.B200FFTError) as e:
        h.sync()
    assert e.value.code == -7
    monkeypatch.delenv("B200FFT_TMA_STALL_TEST")
    d = to_dev(x.astype(np.complex64))
    h.exec_c2c(0, nv.FORWARD, d)
    h.sync()
    assert O.rel_l2(to_host(d), O.c2c_batch(x, length, batch, batch, 1, -1)) < tol(nv.F32)
    h.close()


@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("length,widths", [(512, (257, 45, 19)), (256, (129, 97, 35))])
@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
def test_tma_odd_stride_columns(variant, length, widths, direction, monkeypatch):
    """Odd point strides W = batch: W // TB full tiles through the even- and
    odd-row boxes, and W % TB remainder columns (1, 13, 3 at TB = 16; 1, 1, 3
    at TB = 32) through plain loads."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    for w in widths:
        y, ref, fams, _ = _column_case(length, w, w, direction, seed=length + w)
        assert fams == {TMA_FAMILY}, (length, w, fams)
        assert O.rel_l2(y, ref) < tol(nv.F32), (variant, length, w)


@pytest.mark.parametrize("shape", [(24, 512, 512), (6, 256, 256), (5, 512, 36), (7, 512, 60)])
def test_tma_odd_stride_through_parafaft_r2c(shape, monkeypatch):
    """ParaFaFT_R2C on B200Backend<float> with the double-row kernel on the
    middle axis (variant 8): many slabs per launch (the slab coordinate of the
    map), the held exchange copy's source as input; forward against numpy
    FP64, round trip."""
    monkeypatch.setenv("B200FFT_VARIANT", "8")
    x = O.normal_real(shape, sum(shape))
    f = nv.ParaFaFT("r2c", shape, nv.F32)
    buf = np.zeros(f.required_size, np.float32)
    p = O.pad_real(x, np.float32)
    buf[:p.size] = p
    d = to_dev(buf)
    f.handle().set_profiling(True)
    f.forward(d)
    nc = shape[-1] // 2 + 1
    X = to_host(d)[:p.size].view(np.complex64).reshape(shape[:-1] + (nc,))
    assert O.rel_l2(X, O.r2c_nd(x)) < tol(nv.F32), shape
    fams = [r["family"] for r in f.handle().log() if r["kind"] == 0]
    assert TMA_FAMILY in fams, (shape, fams)
    f.backward(d)
    back = O.unpad_real(to_host(d)[:p.size], shape) / x.size
    assert O.rel_l2(back, x) < tol(nv.F32)
    f.close()


@pytest.mark.parametrize("variant", [8, 9])
def test_tma_odd_stride_wait_timeout_reports_device_status(variant, monkeypatch):
    """The stall hook on the double-row kernels (variant 8: one CTA per tile,
    tile 0's copies skipped; variant 9: the ring, every CTA's first tile): the
    wait runs out, sync reports B200FFT_ERR_DEVICE_STATUS, and the next launch
    on the same context is correct."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    length, w = 512, 257
    x = O.normal_complex((length - 1) * w + w, 12)
    h = nv.Handle(nv.F32, 1)
    h.plan_c2c(0, length, w, w, 1)
    d = to_dev(x.astype(np.complex64))
    monkeypatch.setenv("B200FFT_TMA_STALL_TEST", "1")
    h.exec_c2c(0, nv.FORWARD, d)
    with pytest.raises(nv.B200FFTError) as e:
        h.sync()
    assert e.value.code == -7
    monkeypatch.delenv("B200FFT_TMA_STALL_TEST")
    d = to_dev(x.astype(np.complex64))
    h.exec_c2c(0, nv.FORWARD, d)
    h.sync()
    assert O.rel_l2(to_host(d), O.c2c_batch(x, length, w, w, 1, -1)) < tol(nv.F32)
    h.close()
