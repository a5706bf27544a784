"""ParaFaFT_C2C / ParaFaFT_R2C on B200GridBackend<D, T> (handles_distributed:
the backend owns the grid and runs each transform as one replayed CUDA graph)
against numpy FP64, and against B200Backend<T> through the per-stage path.

The reference's distributed path (parafaft_c2c.hpp:122-149, :539-543;
parafaft_r2c.hpp:144-185, :360-364, :473-477) hands the backend the whole
transform; its tests for that path run cuFFTMp on several ranks
(test/unit/test_cufftmp_*), which has no counterpart on one GPU, so the grids
here are checked against the exact DFT directly.
"""
import numpy as np
import pytest
import torch

from helpers import cdtype, rdtype, to_dev, to_host, tol
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

PRECS = [nv.F32, nv.F64]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(16, 24), (32, 48, 40), (64, 64, 64), (8, 12, 10, 6)])
def test_grid_backend_c2c(prec, shape):
    n = int(np.prod(shape))
    f = nv.ParaFaFT("c2c", shape, prec, backend="b200grid")
    buf = f.buffer()
    assert buf is not None and buf.numel() == n
    sh = f.shapes()
    assert sh["in_shape"] == list(shape) and sh["out_shape"] == list(shape)
    assert sh["in_start"] == [0] * len(shape) and sh["out_start"] == [0] * len(shape)
    for seed in (1, 2):  # the second transform replays the same graph on new data
        x = O.normal_complex(n, seed + sum(shape))
        buf.copy_(torch.from_numpy(x.astype(cdtype(prec))))
        f.forward(None)
        y = buf.cpu().numpy().reshape(shape)
        assert O.rel_l2(y, np.fft.fftn(x.reshape(shape))) < tol(prec), (shape, seed)
        f.backward(None)
        assert O.rel_l2(buf.cpu().numpy() / n, x) < tol(prec), (shape, seed)
    f.close()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(16, 24), (32, 48, 40), (64, 64, 64), (6, 8, 10, 12)])
def test_grid_backend_r2c(prec, shape):
    n = int(np.prod(shape))
    nh = shape[-1] // 2 + 1
    f = nv.ParaFaFT("r2c", shape, prec, backend="b200grid")
    buf = f.buffer()
    rows = n // shape[-1]
    assert buf.numel() == rows * 2 * nh
    for seed in (3, 4):
        x = np.random.default_rng(seed + sum(shape)).standard_normal(shape)
        buf.copy_(torch.from_numpy(O.pad_real(x, rdtype(prec))))
        f.forward(None)
        cplx = buf.view(torch.complex128 if prec == nv.F64 else torch.complex64)
        y = cplx.cpu().numpy().reshape(shape[:-1] + (nh,))
        assert O.rel_l2(y, np.fft.rfftn(x)) < tol(prec), (shape, seed)
        f.backward(None)
        back = O.unpad_real(buf.cpu().numpy(), shape) / n
        assert O.rel_l2(back, x) < tol(prec), (shape, seed)
    f.close()


@pytest.mark.parametrize("prec", PRECS)
def test_grid_backend_matches_per_stage_backend(prec):
    """Same kernels on the same passes in the same order: the grid-owning
    backend's results are bit for bit those of B200Backend<T> through
    ParaFaFT's per-stage path (which fuses its exchange copies into the
    passes instead of running them in place)."""
    shape = (64, 64, 64)
    n = int(np.prod(shape))
    x = O.normal_complex(n, 7)
    g = nv.ParaFaFT("c2c", shape, prec, backend="b200grid")
    gb = g.buffer()
    gb.copy_(torch.from_numpy(x.astype(cdtype(prec))))
    g.forward(None)
    s = nv.ParaFaFT("c2c", shape, prec, backend="b200")
    d = np.zeros(s.required_size, cdtype(prec))
    d[:n] = x
    dd = to_dev(d)
    s.forward(dd)
    assert np.array_equal(gb.cpu().numpy(), to_host(dd)[:n])
    rshape = (32, 48, 40)
    xr = np.random.default_rng(8).standard_normal(rshape)
    p = O.pad_real(xr, rdtype(prec))
    g2 = nv.ParaFaFT("r2c", rshape, prec, backend="b200grid")
    g2.buffer().copy_(torch.from_numpy(p))
    g2.forward(None)
    s2 = nv.ParaFaFT("r2c", rshape, prec, backend="b200")
    d2 = np.zeros(s2.required_size, rdtype(prec))
    d2[:p.size] = p
    dd2 = to_dev(d2)
    s2.forward(dd2)
    assert np.array_equal(g2.buffer().cpu().numpy(), to_host(dd2)[:p.size])
    for o in (g, s, g2, s2):
        o.close()
