"""b200fft_c2c_noalloc, the transform entry point that allocates nothing.

It exists for callers that cannot allocate device memory where they transform
(applications that own all device memory through their own pool, loops that
must not let cudaMalloc/cudaFree synchronize the device). Its twiddle table
sits in a fixed array inside the library, so two calls in a row on one stream
must each rebuild it correctly for their own length and precision.

The results must match the ordinary handle-based entry point
(b200fft_plan_c2c + b200fft_exec_c2c) within the FP32/FP64 tolerances the other
tests use. The file name makes pytest collect it last; it also passes alone in
a fresh process.
"""
import numpy as np
import pytest

from helpers import cdtype, to_dev, to_host, tol
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu


def _with_handle(prec, direction, length, batch, stride, dist, x):
    h = nv.Handle(prec, 1)
    h.plan_c2c(0, length, batch, stride, dist)
    d = to_dev(x)
    h.exec_c2c(0, direction, d)
    h.sync()
    return to_host(d)


def _no_alloc(prec, direction, length, batch, stride, dist, x, stream=None):
    import torch
    d = to_dev(x)
    out = torch.empty_like(d)
    nv.c2c_noalloc(prec, direction, length, batch, stride, dist, d, out, stream)
    torch.cuda.synchronize()
    return to_host(out)


@pytest.mark.parametrize("prec", [nv.F32, nv.F64])
def test_no_alloc_matches_handle_path_two_calls_in_a_row(prec):
    # two consecutive calls with different lengths, layouts and directions:
    # the second must not see the first call's table
    cases = [(nv.FORWARD, 512, 257, 257, 1), (nv.BACKWARD, 64, 300, 1, 64)]
    for i, (direction, length, batch, stride, dist) in enumerate(cases):
        span = (length - 1) * stride + (batch - 1) * dist + 1
        x = O.normal_complex(span, 40 + i).astype(cdtype(prec))
        want = _with_handle(prec, direction, length, batch, stride, dist, x)
        got = _no_alloc(prec, direction, length, batch, stride, dist, x)
        assert O.rel_l2(got, want) < tol(prec), (prec, length)
        ref = O.c2c_batch(x, length, batch, stride, dist, -1 if direction == nv.FORWARD else 1)
        assert O.rel_l2(got, ref) < tol(prec), (prec, length)


def test_no_alloc_on_a_caller_stream_in_place():
    import torch
    prec, length, batch = nv.F32, 4096, 40
    x = O.normal_complex(length * batch, 7).astype(np.complex64)
    want = _with_handle(prec, nv.FORWARD, length, batch, 1, length, x)
    s = torch.cuda.Stream()
    d = to_dev(x)
    for _ in range(2):  # same input twice: each call rebuilds the table
        d.copy_(to_dev(x))
        torch.cuda.synchronize()
        nv.c2c_noalloc(prec, nv.FORWARD, length, batch, 1, length, d, d, s.cuda_stream)
        s.synchronize()
        assert O.rel_l2(to_host(d), want) < tol(prec)


def test_no_alloc_rejects_lengths_beyond_its_array():
    import torch
    d = torch.zeros(2 * 8192, dtype=torch.complex64, device="cuda")
    with pytest.raises(nv.B200FFTError) as e:
        nv.c2c_noalloc(nv.F32, nv.FORWARD, 8192, 1, 1, 8192, d, d)
    assert e.value.code == -2 and "4096" in str(e.value)
    with pytest.raises(nv.B200FFTError) as e:
        nv.c2c_noalloc(nv.F64, nv.FORWARD, 60, 1, 1, 60, d, d)
    assert e.value.code == -2


def test_no_alloc_leaves_device_memory_unchanged():
    """After first calls on the device (which may load the kernels they
    launch), further calls change neither the device's free memory nor
    PyTorch's allocations: the entry point allocates nothing."""
    import torch
    prec, length, batch = nv.F32, 1024, 64
    x = to_dev(O.normal_complex(length * batch, 12).astype(np.complex64))
    out = torch.empty_like(x)
    for direction in (nv.FORWARD, nv.BACKWARD):
        nv.c2c_noalloc(prec, direction, length, batch, 1, length, x, out)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    reserved0 = torch.cuda.memory_reserved()
    for direction in (nv.FORWARD, nv.BACKWARD, nv.FORWARD):
        nv.c2c_noalloc(prec, direction, length, batch, 1, length, x, out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
