"""Parity at the full sizes of the measured configurations (GPU).

Each test runs one measured workload at its stated size through the reference
orchestrator on the B200 backends and checks it against an FP64 oracle on the
same seeded input:

* 64^3 complex128 through ParaFaFT_C2C<3, B200Backend<double>> (per-stage) vs
  the C oracle, rel-L2 1e-12 and the reference tests' 1e-10 max-abs
  (test/c2c/test_fftw_c2c_nd.cpp:103-119);
* 512^3 float32 R2C through ParaFaFT_R2C<3, B200Backend<float>> vs scipy FP64,
  rel-L2 2e-6 forward and round trip
  (test/r2c/test_fftw_r2c_padded_nd.cpp:117-142 for the layout);
* 1024^3 complex64 through ParaFaFT_C2C<3, B200Backend<float>>, plain and
  split-TC, on five output planes vs the FP64 plane oracle: plain 2e-6, split
  at most twice the plain error;
* 128x128x64x64 complex128 through ParaFaFT_C2C<4, B200GridBackend<4, double>>
  vs scipy FP64, rel-L2 1e-12;
* the 256 uneven float32 R2C grids (Gaussian random fields, P(k) ~ k^-3) vs
  scipy FP64 per grid, forward through each grid's own object and round trip
  through the grouped schedule replayed as a CUDA graph.
"""
import os

import numpy as np
import pytest

from helpers import REL_F32, REL_F64, ABS_F64
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

UNEVEN_SIDES = [32, 48, 60, 64, 80, 96, 120, 128, 160]


def _drivers_or_skip():
    try:
        nv.drivers()
    except ImportError as e:
        pytest.skip(str(e))


def _rel_dev(y, ref, chunk=1 << 26):
    import torch
    num = den = 0.0
    for a in range(0, ref.numel(), chunk):
        r = ref[a:a + chunk].to(torch.complex128 if ref.is_complex() else torch.float64)
        num += float(torch.linalg.vector_norm(y[a:a + chunk].to(r.dtype) - r)) ** 2
        den += float(torch.linalg.vector_norm(r)) ** 2
    return (num / den) ** 0.5


def test_c2c_64cube_fp64_per_stage():
    import torch
    _drivers_or_skip()
    shape = (64, 64, 64)
    x = O.uniform_complex(shape, 11)
    f = nv.ParaFaFT("c2c", shape, nv.F64)
    d = torch.zeros(f.required_size, dtype=torch.complex128, device="cuda")
    d[:x.size] = torch.from_numpy(x.reshape(-1)).cuda()
    f.forward(d)
    y = d[:x.size].cpu().numpy().reshape(shape)
    ref = O.c2c_nd(x)
    assert O.rel_l2(y, ref) < REL_F64
    assert O.max_abs(y, ref) < ABS_F64 * np.abs(ref).max()
    f.backward(d)
    back = d[:x.size].cpu().numpy().reshape(shape) / x.size
    assert O.rel_l2(back, x) < REL_F64
    f.close()


def test_r2c_512cube_f32():
    import torch
    _drivers_or_skip()
    shape = (512, 512, 512)
    x = O.normal_real(shape, 1234, np.float32)
    f = nv.ParaFaFT("r2c", shape, nv.F32)
    buf = O.pad_real(x, np.float32)
    assert f.required_size == buf.size
    d = torch.from_numpy(buf).cuda()
    f.forward(d)
    X = O.complex_view(d.cpu().numpy(), shape)
    err = O.rel_l2(X, O.r2c_nd(x.astype(np.float64), impl="scipy"))
    del X
    assert err < REL_F32, err
    f.backward(d)
    back = O.unpad_real(d.cpu().numpy(), shape) / x.size
    assert O.rel_l2(back, x) < REL_F32
    f.close()


def test_c2c_1024cube_f32_plain_and_split_tc_on_planes(monkeypatch):
    import torch
    _drivers_or_skip()
    shape = (1024, 1024, 1024)
    n = int(np.prod(shape))
    gen = torch.Generator(device="cuda").manual_seed(12)
    x0 = torch.complex(torch.randn(n, generator=gen, device="cuda"),
                       torch.randn(n, generator=gen, device="cuda"))
    xv = x0.view(shape)
    ks = (0, 1, 333, 512, 1023)
    ref = O.c2c_planes(lambda a, b: xv[a:b].cpu().numpy(), shape[0], ks)
    errs = {}
    for form in ("plain", "split_tc"):
        if form == "split_tc":
            monkeypatch.setenv("B200FFT_SPLIT_TC", "1")
        else:
            monkeypatch.delenv("B200FFT_SPLIT_TC", raising=False)
        f = nv.ParaFaFT("c2c", shape, nv.F32)
        d = torch.empty(f.required_size, dtype=torch.complex64, device="cuda")
        d[:n].copy_(x0)
        f.forward(d)
        yv = d[:n].view(shape)
        got = np.stack([yv[k].cpu().numpy() for k in ks])
        errs[form] = O.rel_l2(got, ref)
        f.backward(d)
        errs[form + "_rt"] = _rel_dev(d[:n] / n, x0)
        f.close()
        del d, yv
        torch.cuda.empty_cache()
    assert errs["plain"] < REL_F32, errs
    assert errs["plain_rt"] < REL_F32, errs
    assert errs["split_tc"] <= 2 * errs["plain"], errs
    assert errs["split_tc_rt"] <= 2 * max(errs["plain_rt"], 1e-7), errs


def test_c2c_4d_fp64_grid_backend():
    import torch
    _drivers_or_skip()
    shape = (128, 128, 64, 64)
    x = O.uniform_complex(shape, 13)
    g = nv.ParaFaFT("c2c", shape, nv.F64, backend="b200grid")
    buf = g.buffer()
    buf.copy_(torch.from_numpy(x.reshape(-1)).cuda())
    g.forward(None)
    y = buf.cpu().numpy().reshape(shape)
    ref = O.c2c_nd(x, -1, "scipy")
    assert O.rel_l2(y, ref) < REL_F64
    del y, ref
    g.backward(None)
    back = buf.cpu().numpy().reshape(shape) / x.size
    assert O.rel_l2(back, x) < REL_F64
    g.close()


def test_uneven_256_grids_f32():
    import torch
    _drivers_or_skip()
    rng = np.random.default_rng(2024)
    shapes = [tuple(int(s) for s in rng.choice(UNEVEN_SIDES, 3)) for _ in range(256)]
    objs, devs, hosts, xs = [], [], [], []
    for i, shp in enumerate(shapes):
        x = O.gaussian_random_field(shp, 2024 + 1 + i).astype(np.float32)
        f = nv.ParaFaFT("r2c", shp, nv.F32)
        buf = np.zeros(f.required_size, np.float32)
        p = O.pad_real(x, np.float32)
        buf[:p.size] = p
        objs.append(f)
        xs.append(x)
        hosts.append(torch.from_numpy(buf))
        devs.append(torch.from_numpy(buf).cuda())
    # forward, per grid, against the FP64 oracle
    for f, d, x, shp in zip(objs, devs, xs, shapes):
        f.forward(d)
        npad = shp[0] * shp[1] * 2 * (shp[2] // 2 + 1)
        X = O.complex_view(d.cpu().numpy()[:npad], shp)
        err = O.rel_l2(X, O.r2c_nd(x.astype(np.float64), impl="scipy"))
        assert err < REL_F32, (shp, err)
    # forward + backward of all grids as one grouped schedule in a CUDA graph
    for d, h in zip(devs, hosts):
        d.copy_(h)
    g = nv.Group([f.handle() for f in objs])
    g.begin()
    for f, d in zip(objs, devs):
        f.forward(d)
        f.backward(d)
    g.end()
    g.sync()
    g.capture()
    for d, h in zip(devs, hosts):
        d.copy_(h)
    g.replay()
    g.sync()
    for d, x, shp in zip(devs, xs, shapes):
        npad = shp[0] * shp[1] * 2 * (shp[2] // 2 + 1)
        back = O.unpad_real(d.cpu().numpy()[:npad], shp) / x.size
        assert O.rel_l2(back, x) < REL_F32, shp
    g.close()
    for f in objs:
        f.close()
