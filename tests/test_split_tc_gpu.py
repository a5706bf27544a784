"""The split-precision tensor-core C2C kernels (FP32 data, FP16 hi+lo operands,
FP32 accumulation) against the FP64 oracle.

Bound: the relative L2 error of the split form stays within twice the error
of the plain FP32 kernels on the same input, and within the FP32 tolerance of
the transform tests (2e-6). Cases cover rows and columns (incl. coalesced
middle-axis slabs and tiles that straddle slab boundaries), both directions,
out-of-place fused copies, inputs whose magnitudes span many binades (the
block exponents), all-zero transforms, partial tiles, and 3D transforms
through the reference orchestrator ParaFaFT_C2C.
"""
import numpy as np
import pytest

from helpers import REL_F32, to_dev, to_host
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

LENGTHS = [256, 512, 1024]


def _run(x, length, batch, stride, dist, direction, split, slabs=None):
    h = nv.Handle(nv.F32, 1, flags=nv.FLAG_SPLIT_TC if split else 0)
    h.plan_c2c(0, length, batch, stride, dist)
    desc = h.plan_describe(nv.KIND_C2C, 0)
    d = to_dev(x.astype(np.complex64))
    if slabs is None:
        h.exec_c2c(0, direction, d)
    else:  # one call per slab, as ParaFaFT's middle-axis loop issues them
        n, step = slabs
        for i in range(n):
            h.exec_c2c(0, direction, d[i * step:])
    h.sync()
    return to_host(d), desc


def _check(x, length, batch, stride, dist, direction, slabs=None, span_ref=None):
    sign = -1 if direction == nv.FORWARD else +1
    ref = O.c2c_batch(x, length, batch, stride, dist, sign) if span_ref is None else span_ref
    y_tc, desc = _run(x, length, batch, stride, dist, direction, True, slabs)
    y_pl, desc_pl = _run(x, length, batch, stride, dist, direction, False, slabs)
    assert desc.startswith("split-tc"), desc
    assert not desc_pl.startswith("split-tc"), desc_pl
    e_tc, e_pl = O.rel_l2(y_tc, ref), O.rel_l2(y_pl, ref)
    assert e_tc < REL_F32, (length, stride, dist, e_tc)
    assert e_tc <= 2.0 * e_pl, (length, stride, dist, e_tc, e_pl)
    return e_tc, e_pl


@pytest.mark.parametrize("length", LENGTHS)
@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
def test_rows(length, direction):
    batch = 37  # not a multiple of the warps of a CTA
    x = O.normal_complex(length * batch, length)
    _check(x, length, batch, 1, length, direction)


@pytest.mark.parametrize("length", LENGTHS)
@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
def test_columns(length, direction):
    batch = 45  # columns: two full 16-column tiles and a partial one
    x = O.normal_complex(length * batch, length + 1)
    _check(x, length, batch, batch, 1, direction)


@pytest.mark.parametrize("length", LENGTHS)
def test_padded_rows_and_strided_rows(length):
    batch = 9
    dist = length + 3
    x = O.normal_complex((batch - 1) * dist + length, 7)
    _check(x, length, batch, 1, dist, nv.FORWARD)
    # stride > 1 with dist >= stride is still a row plan
    x = O.normal_complex((length - 1) * 2 + (batch - 1) * (2 * length + 1) + 1, 8)
    _check(x, length, batch, 2, 2 * length + 1, nv.BACKWARD)


@pytest.mark.parametrize("length", [256, 512])
@pytest.mark.parametrize("trailing", [21, 32])
def test_middle_axis_slabs(length, trailing):
    """ParaFaFT's middle axis: `lead` calls of (len, batch=trailing, stride=
    trailing, dist 1), coalesced into one launch. With trailing = 21 the
    16-column tiles straddle slab boundaries and rows are odd-strided (no
    16-byte pair loads); with 32 every pair load is aligned."""
    lead = 5
    x = O.normal_complex(lead * length * trailing, 11)
    ref = np.fft.fft(x.reshape(lead, length, trailing), axis=1).ravel()
    _check(x, length, trailing, trailing, 1, nv.FORWARD, slabs=(lead, length * trailing),
           span_ref=ref)


@pytest.mark.parametrize("length", LENGTHS)
@pytest.mark.parametrize("col", [False, True])
def test_wide_dynamic_range(length, col):
    """Transforms whose scales differ by 2^+-50 and entries spanning 2^+-20
    within a transform: the block exponents keep each relative error."""
    rng = np.random.default_rng(5)
    batch = 16
    x = O.normal_complex(length * batch, 3).reshape(batch, length)
    x *= 2.0 ** rng.integers(-20, 20, size=(batch, length))
    x *= 2.0 ** rng.integers(-50, 50, size=(batch, 1))
    ref = np.fft.fft(x, axis=1)
    if col:
        y, _ = _run(x.T.ravel(), length, batch, batch, 1, nv.FORWARD, True)
        y = y.reshape(length, batch).T
    else:
        y, _ = _run(x.ravel(), length, batch, 1, length, nv.FORWARD, True)
        y = y.reshape(batch, length)
    for b in range(batch):
        assert O.rel_l2(y[b], ref[b]) < REL_F32, b


def test_zeros_and_single_spike():
    length, batch = 1024, 8
    x = np.zeros(length * batch, np.complex128)
    x[3 * length + 17] = 1.0 + 2.0j  # transform 3: one spike; others all zero
    y, _ = _run(x, length, batch, 1, length, nv.FORWARD, True)
    y = y.reshape(batch, length)
    assert np.all(y[np.arange(batch) != 3] == 0)
    k = np.arange(length)
    ref = (1.0 + 2.0j) * np.exp(-2j * np.pi * 17 * k / length)
    assert O.rel_l2(y[3], ref) < REL_F32


@pytest.mark.parametrize("length", [512, 1024])
def test_fused_copy_out_of_place(length):
    """memcpy(dst <- src) then execute_stage(dst): one out-of-place pass."""
    batch = 24
    x = O.normal_complex(length * batch, 13).astype(np.complex64)
    h = nv.Handle(nv.F32, 1, flags=nv.FLAG_SPLIT_TC)
    h.plan_c2c(0, length, batch, batch, 1)
    src = to_dev(x)
    dst = to_dev(np.zeros_like(x))
    h.reset_stats()
    h.memcpy(dst, src, x.nbytes)
    h.exec_c2c(0, nv.FORWARD, dst)
    h.sync()
    st = h.stats()
    assert st["fused_copies"] == 1 and st["copies_issued"] == 0
    ref = O.c2c_batch(x.astype(np.complex128), length, batch, batch, 1, -1)
    assert O.rel_l2(to_host(dst), ref) < REL_F32
    np.testing.assert_array_equal(to_host(src), x)  # source untouched


@pytest.mark.parametrize("kind,shape", [("c2c", (256, 256, 256)),
                                        ("c2c_onerank", (512, 256, 64))])
def test_roundtrip_through_orchestrator(monkeypatch, kind, shape):
    """ParaFaFT_C2C<3> (and the one-rank orchestrator for a non-cubic grid) on
    B200Backend<float> with the split kernels (B200FFT_SPLIT_TC=1 when the
    backend is created): forward within 2x the plain error, round trip."""
    try:
        nv.drivers()
    except ImportError as e:
        pytest.skip(str(e))
    monkeypatch.setenv("B200FFT_SPLIT_TC", "1")
    f = nv.ParaFaFT(kind, shape, nv.F32)
    monkeypatch.delenv("B200FFT_SPLIT_TC")
    g = nv.ParaFaFT(kind, shape, nv.F32)
    for st in range(3):
        tc_len = shape[2 - st] in (256, 512, 1024)
        assert f.handle().plan_describe(nv.KIND_C2C, st).startswith("split-tc") == tc_len
        assert not g.handle().plan_describe(nv.KIND_C2C, st).startswith("split-tc")
    x = O.normal_complex(shape, 17)
    buf = np.zeros(f.required_size, np.complex64)
    buf[:x.size] = x.ravel()
    d, e = to_dev(buf), to_dev(buf)
    f.forward(d)
    g.forward(e)
    ref = np.fft.fftn(x)
    e_tc = O.rel_l2(to_host(d)[:x.size].reshape(shape), ref)
    e_pl = O.rel_l2(to_host(e)[:x.size].reshape(shape), ref)
    assert e_tc < REL_F32 and e_tc <= 2.0 * e_pl, (e_tc, e_pl)
    f.backward(d)
    back = to_host(d)[:x.size].reshape(shape) / x.size
    assert O.rel_l2(back, x) < REL_F32


@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
def test_rows_256_mma_sync_form(direction, monkeypatch):
    """256-point rows run on the tcgen05 kernel by default; the mma.sync form
    stays available (B200FFT_TC_FORM=mma) and meets the same bound."""
    monkeypatch.setenv("B200FFT_TC_FORM", "mma")
    x = O.normal_complex(256 * 37, 3)
    y, desc = _run(x, 256, 37, 1, 256, direction, True)
    assert desc.startswith("split-tc c2c L=256 row"), desc
    ref = O.c2c_batch(x, 256, 37, 1, 256, -1 if direction == nv.FORWARD else +1)
    assert O.rel_l2(y, ref) < REL_F32


@pytest.mark.parametrize("length,col,prefix", [(256, False, "split-tc5 "),
                                               (512, True, "split-tc5col")])
def test_tcgen05_wait_limit_reports_device_status(monkeypatch, length, col, prefix):
    """The tcgen05 kernels (256-point rows, 512-point columns) bound every wait
    for their products. With the test switch set, thread 0 issues nothing and
    waits on a barrier phase that never completes: the wait runs out (about a
    second), the CTAs free their tensor memory and return, and b200fft_sync
    reports B200FFT_ERR_DEVICE_STATUS. The context stays usable: the next
    transform is correct."""
    batch = 16
    stride, dist = (batch, 1) if col else (1, length)
    x = O.normal_complex(length * batch, 4)
    if col:  # the tcgen05 column kernel is chosen with B200FFT_TC_FORM=tc5
        monkeypatch.setenv("B200FFT_TC_FORM", "tc5")
    h = nv.Handle(nv.F32, 1, flags=nv.FLAG_SPLIT_TC)
    h.plan_c2c(0, length, batch, stride, dist)
    assert h.plan_describe(nv.KIND_C2C, 0).startswith(prefix)
    d = to_dev(x.astype(np.complex64))
    monkeypatch.setenv("B200FFT_TC5_STALL_TEST", "1")
    h.exec_c2c(0, nv.FORWARD, d)
    with pytest.raises(nv.B200FFTError) as e:
        h.sync()
    assert e.value.code == -7
    monkeypatch.delenv("B200FFT_TC5_STALL_TEST")
    d = to_dev(x.astype(np.complex64))
    h.exec_c2c(0, nv.FORWARD, d)
    h.sync()
    ref = O.c2c_batch(x, length, batch, stride, dist, -1)
    assert O.rel_l2(to_host(d), ref) < REL_F32


@pytest.mark.parametrize("direction", [nv.FORWARD, nv.BACKWARD])
@pytest.mark.parametrize("batch,slabs", [(45, None), (21, 5), (32, 3)])
def test_columns_512_tcgen05_form(direction, batch, slabs, monkeypatch):
    """512-point columns on the tcgen05 column kernel (B200FFT_TC_FORM=tc5):
    partial tiles, coalesced middle-axis slabs with tiles straddling slab
    boundaries, both directions; within 2e-6 and twice the plain error."""
    monkeypatch.setenv("B200FFT_TC_FORM", "tc5")
    if slabs is None:
        x = O.normal_complex(512 * batch, 6)
        e_tc, _ = _check(x, 512, batch, batch, 1, direction)
    else:
        x = O.normal_complex(slabs * 512 * batch, 9)
        sign = -1 if direction == nv.FORWARD else +1
        ref = (np.fft.fft if sign < 0 else lambda v, axis: np.fft.ifft(v, axis=axis) * 512)(
            x.reshape(slabs, 512, batch), axis=1).ravel()
        e_tc, _ = _check(x, 512, batch, batch, 1, direction, slabs=(slabs, 512 * batch),
                         span_ref=ref)
    _, desc = _run(x, 512, batch, batch, 1, direction, True,
                   None if slabs is None else (slabs, 512 * batch))
    assert desc.startswith("split-tc5col c2c L=512 col"), desc
