"""Passes whose element offsets exceed 2^31: every offset in the kernels is
64-bit. A transform b holds c_b * delta(n) (c_b = b mod 7 + 1), whose DFT is
the constant c_b, checked on the device for every transform (no host copy of
the 17 GB buffers). Rows (dist 8) and columns (stride = batch) of length 8,
2^28 + 3 transforms: 2^31 + 24 complex elements."""
import pytest
import torch

from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

L = 8
BATCH = (1 << 28) + 3


def _free_gb():
    free, _ = torch.cuda.mem_get_info()
    return free / 2**30


@pytest.mark.parametrize("layout", ["rows", "cols"])
def test_offsets_beyond_2pow31(layout):
    if _free_gb() < 40:
        pytest.skip("needs about 34 GB of free device memory")
    c = (torch.arange(BATCH, device="cuda", dtype=torch.int64) % 7 + 1).to(torch.float32)
    x = torch.zeros(BATCH * L, dtype=torch.complex64, device="cuda")
    h = nv.Handle(nv.F32, 1)
    if layout == "rows":
        x.view(BATCH, L)[:, 0] = c
        h.plan_c2c(0, L, BATCH, 1, L)
    else:
        x.view(L, BATCH)[0, :] = c
        h.plan_c2c(0, L, BATCH, BATCH, 1)
    h.exec_c2c(0, nv.FORWARD, x)
    h.sync()
    torch.cuda.synchronize()
    y = x.view(BATCH, L) if layout == "rows" else x.view(L, BATCH).t()
    err = (y - c[:, None]).abs().max().item()
    assert err == 0.0, err
    del x, y, c
    torch.cuda.empty_cache()
