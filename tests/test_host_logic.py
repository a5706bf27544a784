"""Host-side logic on the CPU: the C ABI's exports, kernel selection, and the
deferral/fusion bookkeeping of the backend, run with the real ParaFaFT
orchestrators in record-only mode (plans and counts, no GPU work)."""
import ctypes as C
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

from parafaft_b200 import native as nv

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols():
    text = (ROOT / "include" / "b200fft.h").read_text()
    return sorted(set(re.findall(r"\b(b200fft_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = nv.engine()
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(nv.ENGINE_SYMBOLS) == declared


def test_version_and_no_device_refusal():
    lib = nv.engine()
    assert lib.b200fft_version() >= 100
    if lib.b200fft_device_count() == 0:
        with pytest.raises(nv.B200FFTError) as e:
            nv.Handle(nv.F32, 1)
        assert e.value.code == -6  # NO_DEVICE: no CPU fallback


def test_argument_validation():
    h = nv.Handle(nv.F32, 2, flags=nv.FLAG_RECORD_ONLY)
    with pytest.raises(nv.B200FFTError):
        h.plan_c2c(5, 64, 1, 1, 64)          # stage out of range
    with pytest.raises(nv.B200FFTError):
        h.plan_c2c(0, 0, 1, 1, 64)           # zero length
    with pytest.raises(nv.B200FFTError) as e:
        h.exec_c2c(1, nv.FORWARD, 4096)      # no plan
    assert e.value.code == -3
    with pytest.raises(nv.B200FFTError) as e:
        h.plan_c2c(0, 67 * 71, 1, 1, 67 * 71)  # prime factors above 61
    assert e.value.code == -2
    with pytest.raises(nv.B200FFTError):
        h.exec_r2c(4096)                     # no r2c plan


@pytest.mark.parametrize("kind,n,expect", [
    (nv.KIND_C2C, 512, "static c2c L=512"), (nv.KIND_C2C, 60, "static c2c L=60"),
    (nv.KIND_C2C, 100, "generic c2c L=100"), (nv.KIND_C2C, 120, "static c2c L=120 row tb=32 nt=256 radices=8x5x3"),
    (nv.KIND_R2C, 512, "static r2c L=256"), (nv.KIND_R2C, 63, "generic r2c L=63"),
    (nv.KIND_C2R, 160, "static c2r L=80"), (nv.KIND_C2R, 200, "generic c2r L=100"),
    (nv.KIND_C2C, 4096, "static c2c L=4096"), (nv.KIND_C2C, 768, "static c2c L=768"),
])
def test_kernel_selection(kind, n, expect):
    assert nv.describe(nv.F32, kind, n).startswith(expect)


def test_split_tc_selection():
    """FLAG_SPLIT_TC selects the tensor-core kernels for FP32 C2C of length
    256/512/1024 (row and column tiles) and leaves every other plan alone."""
    h = nv.Handle(nv.F32, 4, flags=nv.FLAG_RECORD_ONLY | nv.FLAG_SPLIT_TC)
    h.plan_c2c(0, 1024, 100, 1, 1024)
    h.plan_c2c(1, 512, 300, 300, 1)
    h.plan_c2c(2, 2048, 10, 1, 2048)
    h.plan_c2c(3, 256, 7, 7, 1)
    assert h.plan_describe(nv.KIND_C2C, 0).startswith(
        "split-tc c2c L=1024 row tb=4 nt=128 radices=4x16x16")
    assert h.plan_describe(nv.KIND_C2C, 1).startswith(
        "split-tc c2c L=512 col tb=16 nt=256 radices=2x16x16")
    assert h.plan_describe(nv.KIND_C2C, 2).startswith("static c2c L=2048")
    assert h.plan_describe(nv.KIND_C2C, 3).startswith(
        "split-tc c2c L=256 col tb=16 nt=256 radices=16x16")
    h.plan_r2c(512, 4, 1, 514)
    assert h.plan_describe(nv.KIND_R2C, 0).startswith("static r2c L=256")
    d = nv.Handle(nv.F64, 1, flags=nv.FLAG_RECORD_ONLY | nv.FLAG_SPLIT_TC)
    d.plan_c2c(0, 1024, 100, 1, 1024)
    assert d.plan_describe(nv.KIND_C2C, 0).startswith("static c2c L=1024")
    h.plan_c2c(1, 1024, 64, 64, 1)  # a 1024-point column tile uses 16 warps
    assert h.plan_describe(nv.KIND_C2C, 1).startswith("split-tc c2c L=1024 col tb=16 nt=512")
    h.plan_c2c(2, 256, 100, 1, 256)  # 256-point rows: the tcgen05 kernel
    assert h.plan_describe(nv.KIND_C2C, 2).startswith("split-tc5 c2c L=256 row tb=8 nt=128")


def test_supported_lengths():
    assert nv.supported(nv.F32, nv.KIND_C2C, 4096)
    assert nv.supported(nv.F64, nv.KIND_R2C, 3 * 7 * 61)
    assert not nv.supported(nv.F64, nv.KIND_R2C, 3 * 5 * 7 * 61)  # above the one-pass limit
    assert not nv.supported(nv.F32, nv.KIND_C2C, 127)  # prime above 61


def test_fastdiv_restatement():
    """The multiply-shift division used by the generic kernel (fft_common.hpp),
    restated here and checked exhaustively on the divisors the planner uses."""
    def make(d):
        if d <= 1:
            return 0, 0
        l = (d - 1).bit_length()
        return ((1 << (31 + l)) + d - 1) // d, l - 1
    import random
    rnd = random.Random(0)
    for d in list(range(1, 300)) + [4095, 4096, 4097, 65536, 2**31 - 1]:
        m, s = make(d)
        assert m < 2**32
        for n in [0, 1, d - 1, d, d + 1, 2**31 - 1] + [rnd.randrange(2**31) for _ in range(200)]:
            q = n if m == 0 else ((n * m) >> 32) >> s
            assert q == n // d, (n, d)



def test_double_row_box_geometry_restatement():
    """The tile geometry of the TMA double-row column kernels (fft_tma.cu,
    MidGeom and the box coordinates), restated and checked on every odd point
    stride W that tma_mid_ok admits up to 1025 (and 512^3's 257): a map of
    double rows {4W floats, L/2 rows}; tile c0 = k*TB takes its even point rows
    from a box of TB columns at x = c0 and its odd ones from a box of TB + 2
    columns at x = W + c0 - 1. Both boxes start on a 16-byte boundary (x * 8
    bytes), stay inside the double row, and together hold exactly the tile's
    TB columns of every point row at the offsets the kernel reads (column
    1 + t of the odd box); the W mod TB columns left over go to remainder
    tiles, so every column of every row is read by exactly one tile."""
    tile_bytes = 64 * 1024
    for L in (256, 512):
        TB = tile_bytes // (L * 8)
        half = L // 2
        even_b = TB * half * 8
        odd_w = TB + 2
        stage = even_b + odd_w * half * 8
        assert half <= 256 and stage >= tile_bytes and even_b % 128 == 0 and stage % 128 == 0
        assert 3 * stage <= 227 * 1024
        for W in [w for w in range(TB + 2, 1026) if w % 2 == 1] + [257]:
            q, rem = divmod(W, TB)
            seen = [0] * W
            for k in range(q):
                c0 = k * TB
                x_even, x_odd = c0, W + c0 - 1          # complex columns in the double row
                assert (x_even * 8) % 16 == 0 and (x_odd * 8) % 16 == 0
                assert x_even + TB <= 2 * W and x_odd + odd_w <= 2 * W
                for t in range(TB):
                    # even point row 2m: double-row column x_even + t = point column c0 + t
                    assert x_even + t == c0 + t
                    # odd point row 2m+1: double-row column W + (c0 + t) = x_odd + 1 + t
                    assert W + c0 + t == x_odd + 1 + t
                    seen[c0 + t] += 1
            for b in range(rem):                          # one slab's remainder columns
                seen[q * TB + b] += 1
            assert seen == [1] * W, (L, W)

def _run_record(script: str) -> str:
    env = dict(os.environ, B200FFT_RECORD_ONLY="1")
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True,
                       text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout



def test_geometry_beyond_32_bit_counts_without_allocating():
    """Plans and launches whose element counts pass 2^31 and 2^32 (as the
    reference's geometry unit tests check its counts without allocating,
    test/unit/test_exchange_geometry.cpp): a record-only handle never touches
    the pointers, so the addresses below are never mapped. Rows of 4096
    points over 2^20 + 3 transforms (2^32 + 12288 elements); 2^11 middle-axis
    calls of 1024 x 1024 slabs coalesced into one launch (2^31 elements); an
    R2C pass of 2^19 + 1 rows of 8192 reals."""
    h = nv.Handle(nv.F32, 2, flags=nv.FLAG_RECORD_ONLY)
    base = 1 << 40
    rows = (1 << 20) + 3
    h.plan_c2c(0, 4096, rows, 1, 4096)
    h.exec_c2c(0, nv.FORWARD, base)
    r = h.log()[-1]
    assert r["transforms"] == rows and r["slabs"] == 1
    assert r["bytes"] == 2 * 4096 * rows * 8 > 2 ** 32
    # middle axis: the last-axis plan makes the stage buffer 2^31 elements, so
    # consecutive slab calls coalesce (infer_lead) into one pass of 2048 slabs
    h.plan_c2c(0, 1024, 1 << 21, 1, 1024)
    h.plan_c2c(1, 1024, 1024, 1024, 1)
    slab_bytes = 1024 * 1024 * 8
    for k in range(2048):
        h.exec_c2c(1, nv.BACKWARD, base + k * slab_bytes)
    r = h.log()[-1]
    assert (r["stage"], r["slabs"], r["transforms"]) == (1, 2048, 1024 * 2048)
    assert r["bytes"] == 2 * (1 << 31) * 8
    st = h.stats()
    assert st["coalesced_calls"] == 2047 and st["kernel_launches"] == 2
    # R2C rows: 8192 reals each, padded to 8194
    rr = (1 << 19) + 1
    h.plan_r2c(8192, rr, 1, 8194)
    h.exec_r2c(base)
    r = h.log()[-1]
    assert r["kind"] == nv.KIND_R2C and r["transforms"] == rr
    assert r["bytes"] == rr * (8192 * 4 + 4097 * 8) > 2 ** 32
    h.close()

def _drivers_built():
    return nv.DRIVERS_PATH.exists()


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
def test_r2c_512_cube_call_sequence_fuses_to_six_launches():
    """ParaFaFT_R2C<3, B200Backend<float>> at 512^3: 2 x (1 + 512 + 1) backend
    calls plus 4 exchange copies become 6 launches moving the algorithmic
    6 463 422 464 bytes, with no copy issued."""
    out = _run_record(r'''
import ctypes as C
from parafaft_b200 import native as nv
f = nv.ParaFaFT("r2c", (512, 512, 512), nv.F32)
buf = C.c_void_p(); nv.check(nv.engine().b200fft_alloc(f.required_size * 4, C.byref(buf)))
f.forward(buf.value); f.backward(buf.value)
st = f.handle().stats(); log = f.handle().log()
print(st["kernel_launches"], st["exec_calls"], st["coalesced_calls"], st["fused_copies"],
      st["copies_issued"], st["bytes_transformed"])
print([(r["kind"], r["stage"], r["slabs"], r["fused_copy"]) for r in log])
''')
    first, second = out.strip().splitlines()
    assert first.split() == ["6", "1028", "1022", "4", "0", "6463422464"]
    assert second == ("[(1, -1, 1, 0), (0, 1, 512, 1), (0, 2, 1, 1), (0, 2, 1, 0), "
                      "(0, 1, 512, 1), (2, -1, 1, 1)]")


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
@pytest.mark.parametrize("shape,launches", [((64, 64, 64), 6), ((1024, 1024, 1024), 6),
                                           ((16, 16, 16, 16), 8), ((32, 32), 4)])
def test_c2c_call_sequences(shape, launches):
    out = _run_record(rf'''
import ctypes as C
from parafaft_b200 import native as nv
f = nv.ParaFaFT("c2c", {shape!r}, nv.F64)
buf = C.c_void_p(); nv.check(nv.engine().b200fft_alloc(f.required_size * 16, C.byref(buf)))
f.forward(buf.value); f.backward(buf.value)
st = f.handle().stats()
print(st["kernel_launches"], st["copies_issued"], st["fused_copies"], st["memcpy_calls"])
''')
    k, copies, fused, calls = map(int, out.split())
    assert k == launches and copies == 0 and fused == calls


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
def test_out_of_place_forward_fuses_the_pad():
    """ParaFaFT_R2C::forward(real, complex) pads with memcpy2d
    (parafaft_r2c.hpp:333-339, :804-822) and then runs forward_in_place: the
    pad is taken over by the R2C pass, so the forward issues 3 launches and
    no copy; backward(complex, real) keeps its unpad copy."""
    out = _run_record(r'''
import ctypes as C
from parafaft_b200 import native as nv
f = nv.ParaFaFT("r2c", (64, 64, 64), nv.F32)
lib = nv.engine()
cout = C.c_void_p(); nv.check(lib.b200fft_alloc(f.required_size * 4, C.byref(cout)))
rin = C.c_void_p(); nv.check(lib.b200fft_alloc(64 ** 3 * 4, C.byref(rin)))
h = f.handle()
h.reset_stats(); f.forward_oop(rin.value, cout.value); a = h.stats()
h.reset_stats(); f.backward_oop(cout.value, rin.value); b = h.stats()
print(a["kernel_launches"], a["copies_issued"], a["fused_copies"], a["memcpy_calls"])
print(b["kernel_launches"], b["copies_issued"], b["fused_copies"], b["memcpy_calls"])
''')
    fwd, bwd = out.strip().splitlines()
    assert fwd.split() == ["3", "0", "3", "3"]
    assert bwd.split() == ["3", "1", "2", "3"]


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
def test_no_defer_issues_every_call():
    out = _run_record(r'''
import os, ctypes as C
os.environ["B200FFT_NO_DEFER"] = "1"
from parafaft_b200 import native as nv
f = nv.ParaFaFT("r2c", (32, 32, 32), nv.F32)
buf = C.c_void_p(); nv.check(nv.engine().b200fft_alloc(f.required_size * 4, C.byref(buf)))
f.forward(buf.value)
st = f.handle().stats()
print(st["kernel_launches"], st["copies_issued"])
''')
    assert out.split() == ["34", "2"]


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
@pytest.mark.parametrize("form", ["schedule", "levels", "chains"])
def test_group_schedules_many_grids_per_depth_and_length(form, monkeypatch):
    """256 ParaFaFT_R2C<3> objects of uneven sizes, forward+backward recorded in
    one group, 256*6 passes, no copies. One chain (B200FFT_GROUP_CHAINS=1): at
    each of the 6 pass depths one grouped launch per distinct kernel length
    (every side here has a specialised kernel). Default (256 members: three
    chains of grids): the same per chain. B200FFT_GROUP_SCHEDULE=1: the
    dependency-scheduled form, one persistent launch for the whole schedule."""
    monkeypatch.delenv("B200FFT_GROUP_SCHEDULE", raising=False)
    monkeypatch.delenv("B200FFT_GROUP_CHAINS", raising=False)
    if form == "schedule":
        monkeypatch.setenv("B200FFT_GROUP_SCHEDULE", "1")
    elif form == "levels":
        monkeypatch.setenv("B200FFT_GROUP_CHAINS", "1")
    out = _run_record(r'''
import ctypes as C, numpy as np
from parafaft_b200 import native as nv
rng = np.random.default_rng(3)
sides = [32, 48, 60, 64, 80, 96, 120, 128, 160]
objs, bufs = [], []
for i in range(256):
    shape = tuple(int(x) for x in rng.choice(sides, 3))
    f = nv.ParaFaFT("r2c", shape, nv.F32)
    b = C.c_void_p(); nv.check(nv.engine().b200fft_alloc(f.required_size * 4, C.byref(b)))
    objs.append(f); bufs.append(b)
g = nv.Group([f.handle() for f in objs])
g.begin()
for f, b in zip(objs, bufs):
    f.forward(b.value)
    f.backward(b.value)
g.end()
st = g.stats()
shapes = [f.shapes()["in_shape"] for f in objs]
expect = 2 * (len({s[2] for s in shapes}) + len({s[1] for s in shapes}) + len({s[0] for s in shapes}))
print(st["kernel_launches"], st["passes_per_run"], st["copies_issued"], expect)
''')
    launches, passes, copies, expect = out.split()
    assert passes == str(256 * 6) and copies == "0"
    if form == "levels":
        assert launches == expect and int(launches) <= 6 * 9
    elif form == "chains":
        assert int(expect) < int(launches) <= 3 * int(expect)
    else:
        assert launches == "1"


@pytest.mark.skipif(not _drivers_built(), reason="ParaFaFT drivers not built")
def test_group_members_sharing_memory_keep_level_barriers(monkeypatch):
    """Two grids transformed in the same buffer are not independent: the
    group keeps one chain of per-level launches even when the dependency
    schedule or several chains are asked for (both order only each grid's
    own passes): three levels, one launch each for the two equal grids."""
    monkeypatch.setenv("B200FFT_GROUP_SCHEDULE", "1")
    monkeypatch.setenv("B200FFT_GROUP_CHAINS", "2")
    out = _run_record(r'''
import ctypes as C
from parafaft_b200 import native as nv
a = nv.ParaFaFT("r2c", (32, 48, 60), nv.F32)
b = nv.ParaFaFT("r2c", (32, 48, 60), nv.F32)
buf = C.c_void_p(); nv.check(nv.engine().b200fft_alloc(a.required_size * 4, C.byref(buf)))
g = nv.Group([a.handle(), b.handle()])
g.begin()
a.forward(buf.value)
b.forward(buf.value)
g.end()
print(g.stats()["kernel_launches"])
''')
    assert int(out.split()[0]) == 3


def test_wisdom_roundtrip_and_plan_choice(tmp_path):
    """Wisdom entries choose the kernel of later plans of the same geometry;
    export/import/forget round-trip through a text file (record-only handles,
    so nothing is timed)."""
    nv.forget_wisdom()
    w = tmp_path / "w.txt"
    # a hand-written entry: 512-point column plan, generic kernel, Patient rigor
    w.write_text("b200fft-wisdom 1\n"
                 "record-only p0 k0 n512 b131584 s131584 d1 l1 | 1 0 2 0.1\n"
                 "record-only p0 k0 n512 b257 s257 d1 l1 | 0 3 1 0.2\n"
                 "garbage line\n")
    assert nv.import_wisdom(w) == 2
    h = nv.Handle(nv.F32, 3, plan_flag=nv.PLAN_MEASURE, flags=nv.FLAG_RECORD_ONLY)
    h.plan_c2c(2, 512, 131584, 131584, 1)
    assert h.plan_describe(nv.KIND_C2C, 2).startswith("generic c2c L=512")
    h.plan_c2c(1, 512, 257, 257, 1)   # lead inferred 512 from stage 2 -> key l512: no entry
    assert "var=5" in h.plan_describe(nv.KIND_C2C, 1)  # the default tile
    e = nv.Handle(nv.F32, 3, plan_flag=nv.PLAN_ESTIMATE, flags=nv.FLAG_RECORD_ONLY)
    e.plan_c2c(2, 512, 131584, 131584, 1)  # Estimate does not consult wisdom
    assert e.plan_describe(nv.KIND_C2C, 2).startswith("static c2c L=512")
    out = tmp_path / "out.txt"
    nv.export_wisdom(out)
    lines = out.read_text().splitlines()
    assert lines[0] == "b200fft-wisdom 1" and len(lines) == 3
    nv.forget_wisdom()
    nv.export_wisdom(out)
    assert out.read_text().splitlines() == ["b200fft-wisdom 1"]
    bad = tmp_path / "bad.txt"
    bad.write_text("not wisdom\n")
    with pytest.raises(nv.B200FFTError):
        nv.import_wisdom(bad)
