"""Parity of the B200 kernels, called through the C ABI, against the FP64 oracle.

Mirrors the backend-level tests of the reference
(test/unit/test_cufft_backend.cu:22-400, test/unit/test_fftw_backend.cpp:9-201)
and extends them over lengths, layouts, both precisions and the fusion paths.
"""
import numpy as np
import pytest

from helpers import REL_F32, REL_F64, ABS_F64, cdtype, rdtype, to_dev, to_host, tol
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

PRECS = [nv.F32, nv.F64]


def _c2c_case(prec, length, batch, stride, dist, direction, flags=0, seed=0):
    span = (length - 1) * stride + (batch - 1) * dist + 1
    x = O.normal_complex(span, seed)
    h = nv.Handle(prec, 1, flags=flags)
    h.plan_c2c(0, length, batch, stride, dist)
    d = to_dev(x.astype(cdtype(prec)))
    h.exec_c2c(0, direction, d)
    h.sync()
    y = to_host(d)
    ref = O.c2c_batch(x, length, batch, stride, dist, -1 if direction == nv.FORWARD else +1)
    return y, ref, h


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("length", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_c2c_pow2_rows_and_cols(prec, length):
    batch = max(3, 8192 // length)
    for stride, dist in ((1, length), (batch, 1)):
        for direction in (nv.FORWARD, nv.BACKWARD):
            y, ref, _ = _c2c_case(prec, length, batch, stride, dist, direction)
            assert O.rel_l2(y, ref) < tol(prec), (length, stride, dist, direction)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("length", [1, 3, 5, 6, 7, 9, 10, 12, 15, 24, 30, 40, 48, 60, 80, 96,
                                    100, 120, 160, 243, 1000, 3125, 11, 13, 31, 61])
def test_c2c_mixed_radix(prec, length):
    batch = 37
    for stride, dist in ((1, length), (batch, 1), (3, 3 * length + 1)):
        y, ref, _ = _c2c_case(prec, length, batch, stride, dist, nv.FORWARD, seed=length)
        assert O.rel_l2(y, ref) < tol(prec), (length, stride, dist)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("length", [64, 512])
def test_generic_matches_static(prec, length):
    """The runtime-generic kernel computes the same transform as the specialised one."""
    batch = 33
    a, ref, _ = _c2c_case(prec, length, batch, batch, 1, nv.FORWARD)
    b, _, _ = _c2c_case(prec, length, batch, batch, 1, nv.FORWARD, flags=nv.FLAG_GENERIC_ONLY)
    assert O.rel_l2(a, ref) < tol(prec) and O.rel_l2(b, ref) < tol(prec)


def _r2c_roundtrip(prec, n, batch, flags=0, seed=3):
    nc = n // 2 + 1
    dist = 2 * nc
    x = O.normal_real((batch, n), seed)
    buf = np.zeros((batch, dist), dtype=rdtype(prec))
    buf[:, :n] = x
    h = nv.Handle(prec, 0, flags=flags)
    h.plan_r2c(n, batch, 1, dist)
    h.plan_c2r(n, batch, 1, dist)
    d = to_dev(buf.reshape(-1))
    h.exec_r2c(d)
    h.sync()
    X = to_host(d).view(cdtype(prec)).reshape(batch, nc)
    ref = np.stack([O.r2c_nd(r) for r in x])
    h.exec_c2r(d)
    h.sync()
    back = to_host(d).reshape(batch, dist)[:, :n]
    return X, ref, back, x


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096,
                               1, 3, 5, 6, 10, 12, 15, 30, 48, 60, 96, 120, 160, 320])
def test_r2c_c2r_inplace(prec, n):
    batch = 7
    X, ref, back, x = _r2c_roundtrip(prec, n, batch)
    assert O.rel_l2(X, ref) < tol(prec), n
    assert O.rel_l2(back / n, x) < tol(prec), n


@pytest.mark.parametrize("prec", PRECS)
def test_c2r_ignores_imag_of_dc_and_nyquist(prec):
    """FFTW's c2r ignores Im(X[0]) and Im(X[N/2]) (even N)."""
    n, batch = 64, 5
    nc = n // 2 + 1
    rng = np.random.default_rng(11)
    X = rng.standard_normal((batch, nc)) + 1j * rng.standard_normal((batch, nc))
    h = nv.Handle(prec, 0)
    h.plan_c2r(n, batch, 1, 2 * nc)
    d = to_dev(X.astype(cdtype(prec)).view(rdtype(prec)).reshape(-1))
    h.exec_c2r(d)
    h.sync()
    y = to_host(d).reshape(batch, 2 * nc)[:, :n]
    ref = np.stack([O.c2r_nd(r, n) for r in X])
    assert O.rel_l2(y, ref) < tol(prec)


# ---- the reference's backend unit tests (test_cufft_backend.cu) ------------
def test_unit_contiguous_layout():
    """test_cufft_backend.cu:22-80: N=256, batch 3, Gaussian rows, roundtrip."""
    N, batch = 256, 3
    i = np.arange(N)
    row = np.exp(-((i - N / 2) / 16.0) ** 2 / 2.0).astype(np.complex128)
    x = np.tile(row, batch)
    h = nv.Handle(nv.F64, 1)
    h.plan_c2c(0, N, batch, 1, N)
    d = to_dev(x)
    h.exec_c2c(0, nv.FORWARD, d)
    h.exec_c2c(0, nv.BACKWARD, d)
    y = to_host(d) / N  # no sync(): the handle's blocking stream orders the copy
    assert np.max(np.abs(y - x)) < ABS_F64


def test_unit_strided_layout():
    """test_cufft_backend.cu:82-140: N=128, batch 4, stride=batch, dist=1."""
    N, batch = 128, 4
    b = np.arange(batch)
    x = np.tile(np.exp(2j * np.pi * b / batch), N)
    h = nv.Handle(nv.F64, 1)
    h.plan_c2c(0, N, batch, batch, 1)
    d = to_dev(x)
    h.exec_c2c(0, nv.FORWARD, d)
    h.exec_c2c(0, nv.BACKWARD, d)
    h.sync()
    assert np.max(np.abs(to_host(d) / N - x)) < ABS_F64


def test_unit_multiple_stages_reuse():
    """test_cufft_backend.cu:143-224: three stages, plans reused 3 times."""
    N = 64
    h = nv.Handle(nv.F64, 3)
    data = [np.arange(N) + 100.0 * s + 0j for s in range(3)]
    devs = [to_dev(x) for x in data]
    for s in range(3):
        h.plan_c2c(s, N, 1, 1, N)
    err = 0.0
    for _ in range(3):
        for s in range(3):
            h.exec_c2c(s, nv.FORWARD, devs[s])
            h.exec_c2c(s, nv.BACKWARD, devs[s])
            h.sync()
            y = to_host(devs[s]) / N
            err = max(err, np.max(np.abs(y - data[s])))
            devs[s].copy_(to_dev(y))
    assert err < ABS_F64


def test_unit_different_pointers():
    """test_cufft_backend.cu:227-318: one plan applied to three arrays."""
    N, batch = 64, 2
    i = np.arange(N * batch)
    xs = [i % 10 + 0j, 1j * (i % 5), np.exp(-((i - N * batch / 2) ** 2) / 200.0) + 0j]
    h = nv.Handle(nv.F64, 1)
    h.plan_c2c(0, N, batch, 1, N)
    for x in xs:
        d = to_dev(x.astype(np.complex128))
        h.exec_c2c(0, nv.FORWARD, d)
        h.exec_c2c(0, nv.BACKWARD, d)
        h.sync()
        assert np.max(np.abs(to_host(d) / N - x)) < ABS_F64


def test_unit_r2c_c2r_inplace():
    """test_cufft_backend.cu:321-400: N=128, batch 2, padded rows."""
    N, batch = 128, 2
    pd = 2 * (N // 2 + 1)
    i = np.arange(N)
    row = np.exp(-((i - N / 2) / 16.0) ** 2 / 2.0)
    buf = np.zeros((batch, pd))
    buf[:, :N] = row
    h = nv.Handle(nv.F64, 0)
    h.plan_r2c(N, batch, 1, pd)
    h.plan_c2r(N, batch, 1, pd)
    d = to_dev(buf.reshape(-1))
    h.exec_r2c(d)
    h.exec_c2r(d)
    h.sync()
    y = to_host(d).reshape(batch, pd)[:, :N] / N
    assert np.max(np.abs(y - row)) < ABS_F64


# ---- fusion ------------------------------------------------------------------
@pytest.mark.parametrize("prec", PRECS)
def test_copy_then_middle_axis_loop_fuses(prec):
    """ParaFaFT's exchange_local copy followed by the middle-axis slice loop
    (parafaft_c2c.hpp:866-897) runs as one fused launch with identical results."""
    n0, n1, n2 = 6, 32, 12
    total = n0 * n1 * n2
    x = O.normal_complex(total, 5).astype(cdtype(prec))
    outs = {}
    for flags in (0, nv.FLAG_NO_DEFER):
        h = nv.Handle(prec, 3, flags=flags)
        h.plan_c2c(0, n2, n0 * n1, 1, n2)        # last axis, full buffer
        h.plan_c2c(1, n1, n2, n2, 1)             # middle axis, one slab
        src = to_dev(x)
        dst = to_dev(np.zeros_like(x))
        h.memcpy(dst, src, x.nbytes)
        esz = x.itemsize
        for i in range(n0):
            h.exec_c2c(1, nv.FORWARD, dst.data_ptr() + i * n1 * n2 * esz)
        h.sync()
        outs[flags] = to_host(dst)
        st = h.stats()
        if flags == 0:
            assert st["kernel_launches"] == 1 and st["fused_copies"] == 1
            assert st["copies_issued"] == 0 and st["coalesced_calls"] == n0 - 1
        else:
            assert st["kernel_launches"] == n0 and st["copies_issued"] == 1
        assert np.array_equal(to_host(src), x)  # the copy's source is untouched
    full = x.astype(np.complex128).reshape(n0, n1 * n2)
    ref = np.concatenate([O.c2c_batch(full[i], n1, n2, n2, 1, -1) for i in range(n0)])
    assert O.rel_l2(outs[0], ref) < tol(prec)
    assert np.array_equal(outs[0], outs[nv.FLAG_NO_DEFER])


@pytest.mark.parametrize("prec", PRECS)
def test_partial_copy_coverage(prec):
    """A transform covering part of a held copy: the rest is still copied."""
    n, batch = 64, 10
    x = O.normal_complex(n * batch, 8).astype(cdtype(prec))
    h = nv.Handle(prec, 1)
    h.plan_c2c(0, n, 4, 1, n)  # four rows only
    src = to_dev(x)
    dst = to_dev(np.zeros_like(x))
    h.memcpy(dst, src, x.nbytes)
    off = 3 * n * x.itemsize
    h.exec_c2c(0, nv.FORWARD, dst.data_ptr() + off)
    h.sync()
    y = to_host(dst).reshape(batch, n)
    ref = x.astype(np.complex128).reshape(batch, n).copy()
    ref[3:7] = np.fft.fft(ref[3:7], axis=1)
    assert O.rel_l2(y, ref) < tol(prec)
    assert h.stats()["fused_copies"] == 1


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10])
@pytest.mark.parametrize("length", [2, 8, 64, 512, 1024, 4096])
def test_tile_variants(prec, variant, length, monkeypatch):
    """Every tile-shape candidate the planner can pick computes the same
    transform, for column and row layouts, in place and fused out of place."""
    monkeypatch.setenv("B200FFT_VARIANT", str(variant))
    batch = max(5, 40000 // length) + 3
    for stride, dist in ((batch, 1), (1, length)):
        y, ref, h = _c2c_case(prec, length, batch, stride, dist, nv.BACKWARD, seed=variant)
        assert O.rel_l2(y, ref) < tol(prec), (variant, length, stride)


@pytest.mark.parametrize("length,batch,stride", [
    (512, 257, 257),    # odd point stride: 8-byte global accesses
    (512, 258, 258),    # even stride, even batch: 16-byte global accesses
    (512, 301, 302),    # odd batch: the last pair has one transform
    (256, 255, 255),
    (256, 1024, 1024),
    (256, 96, 130),     # gaps between point rows
])
def test_pair_column_tile(length, batch, stride, monkeypatch):
    """Tile variant 10 (two neighbouring transforms per thread, FP32 columns)
    against the oracle: both directions, in place and through a fused
    out-of-place copy."""
    monkeypatch.setenv("B200FFT_VARIANT", "10")
    assert "var=10" in nv.describe(nv.F32, nv.KIND_C2C, length, batch, stride, 1)
    for direction in (nv.FORWARD, nv.BACKWARD):
        y, ref, _ = _c2c_case(nv.F32, length, batch, stride, 1, direction, seed=stride)
        assert O.rel_l2(y, ref) < tol(nv.F32), (length, batch, stride, direction)
    # out of place: a held copy folded into the pass (reads src, writes dst)
    span = (length - 1) * stride + batch
    x = O.normal_complex(span, 3).astype(np.complex64)
    src, dst = to_dev(x), to_dev(np.zeros_like(x))
    h = nv.Handle(nv.F32, 1)
    h.plan_c2c(0, length, batch, stride, 1)
    h.memcpy(dst, src, x.nbytes)
    h.exec_c2c(0, nv.FORWARD, dst)
    h.sync()
    ref = O.c2c_batch(x, length, batch, stride, 1, -1)
    assert O.rel_l2(to_host(dst), ref) < tol(nv.F32)
    assert np.array_equal(to_host(src), x)


def test_pair_column_tile_across_slabs(monkeypatch):
    """Variant 10 on a coalesced middle-axis run (the 512^3 R2C middle axis in
    miniature: slices of [512][257], odd batch, so pairs span two slabs)."""
    monkeypatch.setenv("B200FFT_VARIANT", "10")
    n, nc, slabs = 512, 257, 5
    x = O.normal_complex(slabs * n * nc, 8).astype(np.complex64)
    d = to_dev(x)
    h = nv.Handle(nv.F32, 2)
    h.plan_c2c(0, n, nc, nc, 1)             # one slice
    h.plan_c2c(1, n, slabs * nc, 1, n)      # makes the full buffer `slabs` slices
    for i in range(slabs):
        h.exec_c2c(0, nv.BACKWARD, int(d.data_ptr()) + i * n * nc * 8)
    h.sync()
    assert h.stats()["kernel_launches"] == 1
    y = to_host(d).reshape(slabs, n * nc)
    for i in range(slabs):
        ref = O.c2c_batch(x[i * n * nc:(i + 1) * n * nc], n, nc, nc, 1, +1)
        assert O.rel_l2(y[i], ref) < tol(nv.F32), i


MIXED_STATIC = [24, 30, 40, 48, 60, 80, 96, 120, 160, 192, 384, 768]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("length", MIXED_STATIC)
def test_mixed_radix_specialised_kernels(prec, length):
    """Lengths of factors 8, 4, 2, 5, 3 with a specialised kernel (flat FP64
    twiddle table, power-of-two tiles): rows, columns and strided rows against
    the oracle, and the same plans on the generic kernel."""
    batch = 37
    assert nv.describe(prec, nv.KIND_C2C, length).startswith("static")
    for stride, dist in ((1, length), (batch, 1), (3, 3 * length + 1)):
        for direction in (nv.FORWARD, nv.BACKWARD):
            y, ref, _ = _c2c_case(prec, length, batch, stride, dist, direction, seed=length)
            assert O.rel_l2(y, ref) < tol(prec), (length, stride, dist, direction)
    g, ref, _ = _c2c_case(prec, length, batch, batch, 1, nv.FORWARD, flags=nv.FLAG_GENERIC_ONLY)
    assert O.rel_l2(g, ref) < tol(prec)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("n", [48, 60, 80, 96, 120, 160, 384, 768, 1536])
def test_mixed_radix_r2c_c2r_specialised(prec, n):
    """R2C / C2R of even non-power-of-two lengths on the specialised kernels
    (half length in the mixed-radix set) against the oracle, padded rows."""
    batch = 21
    dist = 2 * (n // 2 + 1)
    assert nv.describe(prec, nv.KIND_R2C, n).startswith("static")
    x = O.normal_real((batch, n), n)
    buf = np.zeros(batch * dist, dtype=rdtype(prec))
    buf.reshape(batch, dist)[:, :n] = x
    h = nv.Handle(prec, 1)
    h.plan_r2c(n, batch, 1, dist)
    h.plan_c2r(n, batch, 1, dist)
    d = to_dev(buf)
    h.exec_r2c(d)
    h.sync()
    X = to_host(d).view(cdtype(prec)).reshape(batch, dist // 2)
    assert O.rel_l2(X, np.fft.rfft(x, axis=1)) < tol(prec)
    h.exec_c2r(d)
    h.sync()
    back = to_host(d).reshape(batch, dist)[:, :n] / n
    assert O.rel_l2(back, x) < tol(prec)
