"""Batches of independent uneven grids through groups (the C3 path).

Each grid is its own ParaFaFT_R2C<3, B200Backend<float>> object; their
forward+backward passes are recorded in one group and launched together, then
replayed, then replayed from a CUDA graph. Every run must equal the per-grid
result and the FP64 oracle. Every form of a group runs: the per-level launches
(default), the per-level launches of independent chains of grids
(B200FFT_GROUP_CHAINS) and the dependency-scheduled persistent launch
(B200FFT_GROUP_SCHEDULE=1).
"""
import numpy as np
import pytest

from helpers import REL_F32, to_dev, to_host
from oracle import oracle as O
from parafaft_b200 import native as nv

pytestmark = pytest.mark.gpu

SIDES = [32, 48, 60, 64, 80, 96, 120, 128, 160]


def _drivers_or_skip():
    try:
        nv.drivers()
    except ImportError as e:
        pytest.skip(str(e))


def _grids(n, seed):
    rng = np.random.default_rng(seed)
    return [tuple(int(x) for x in rng.choice(SIDES, 3)) for _ in range(n)]


def _launches_per_direction(shapes):
    """Grouped launches of one direction: per pass depth (last, middle, first
    axis) one launch per distinct length."""
    return sum(len({s[a] for s in shapes}) for a in range(3))


@pytest.fixture(params=["schedule", "levels", "chains"])
def form(request, monkeypatch):
    monkeypatch.delenv("B200FFT_GROUP_SCHEDULE", raising=False)
    monkeypatch.delenv("B200FFT_GROUP_CHAINS", raising=False)
    if request.param == "schedule":
        monkeypatch.setenv("B200FFT_GROUP_SCHEDULE", "1")
    elif request.param == "chains":
        monkeypatch.setenv("B200FFT_GROUP_CHAINS", "3")
    return request.param


def _expected_launches(form, shapes, per_direction):
    """Launches of one run: 1 for the persistent schedule; otherwise per pass
    depth one launch per distinct length, within each chain of grids."""
    if form == "schedule":
        return 1
    if form == "levels":
        return per_direction * _launches_per_direction(shapes)
    return None  # chains: at least the one-chain count (checked separately)


def test_group_forward_matches_oracle_and_per_grid(form):
    _drivers_or_skip()
    shapes = _grids(12, 5)
    objs, devs, xs = [], [], []
    for i, shp in enumerate(shapes):
        x = O.gaussian_random_field(shp, 100 + i).astype(np.float32)
        f = nv.ParaFaFT("r2c", shp, nv.F32)
        buf = np.zeros(f.required_size, np.float32)
        p = O.pad_real(x, np.float32)
        buf[:p.size] = p
        objs.append(f)
        devs.append(to_dev(buf))
        xs.append(x)
    g = nv.Group([f.handle() for f in objs])
    g.begin()
    for f, d in zip(objs, devs):
        f.forward(d)
    g.end()
    g.sync()
    # one persistent launch, or one grouped launch per pass depth and length
    want = _expected_launches(form, shapes, 1)
    got = g.stats()["kernel_launches"]
    assert got == want if want is not None else got >= _launches_per_direction(shapes)
    for shp, x, d in zip(shapes, xs, devs):
        nc = shp[-1] // 2 + 1
        X = to_host(d)[:2 * shp[0] * shp[1] * nc].view(np.complex64).reshape(shp[0], shp[1], nc)
        assert O.rel_l2(X, O.r2c_nd(x.astype(np.float64))) < REL_F32, shp


def test_group_roundtrip_replay_and_graph(form):
    _drivers_or_skip()
    shapes = _grids(20, 9)
    objs, devs, xs = [], [], []
    for i, shp in enumerate(shapes):
        x = O.normal_real(shp, i).astype(np.float32)
        f = nv.ParaFaFT("r2c", shp, nv.F32)
        buf = np.zeros(f.required_size, np.float32)
        p = O.pad_real(x, np.float32)
        buf[:p.size] = p
        objs.append(f)
        devs.append(to_dev(buf))
        xs.append(x)
    g = nv.Group([f.handle() for f in objs])
    g.begin()
    for f, d in zip(objs, devs):
        f.forward(d)
        f.backward(d)
    g.end()
    g.sync()
    scale = [float(np.prod(s)) for s in shapes]

    def check(k):
        for shp, x, d, sc in zip(shapes, xs, devs, scale):
            y = O.unpad_real(to_host(d)[:O.pad_real(x).size], shp) / sc ** k
            assert O.rel_l2(y, x) < 4 * REL_F32, (shp, k)

    check(1)
    # each run scales by N again (unnormalised forward+backward)
    for d, sc in zip(devs, scale):
        d.mul_(1.0 / sc)
    g.replay()
    g.sync()
    check(1)
    for d, sc in zip(devs, scale):
        d.mul_(1.0 / sc)
    g.capture()
    g.replay()
    g.sync()
    check(1)
    st = g.stats()
    runs = 2  # the run at end() and the replay (graph replays are not counted)
    want = _expected_launches(form, shapes, 2)
    if want is not None:
        assert st["kernel_launches"] == runs * want
    else:
        assert st["kernel_launches"] >= runs * 2 * _launches_per_direction(shapes)
    assert st["passes_per_run"] == 20 * 6
    g.close()
    # members work on their own again after the group is gone
    for f, d in zip(objs[:2], devs[:2]):
        f.forward(d)
        f.backward(d)


def test_schedule_wait_bound_reports_device_status(monkeypatch):
    """The schedule kernel's dependency waits are bounded: with the test hook
    one pass waits for a tile that never comes, the wait runs out (20 ms), the
    kernel sets its fault word and returns, and b200fft_group_sync reports
    DEVICE_STATUS. The context stays usable: a group built afterwards is
    correct."""
    _drivers_or_skip()
    monkeypatch.setenv("B200FFT_GROUP_SCHEDULE", "1")
    shapes = _grids(6, 21)

    def build():
        objs, devs, xs = [], [], []
        for i, shp in enumerate(shapes):
            x = O.normal_real(shp, 50 + i).astype(np.float32)
            f = nv.ParaFaFT("r2c", shp, nv.F32)
            buf = np.zeros(f.required_size, np.float32)
            p = O.pad_real(x, np.float32)
            buf[:p.size] = p
            objs.append(f)
            devs.append(to_dev(buf))
            xs.append(x)
        return objs, devs, xs

    objs, devs, _ = build()
    monkeypatch.setenv("B200FFT_SCHED_STALL_TEST", "1")
    g = nv.Group([f.handle() for f in objs])
    g.begin()
    for f, d in zip(objs, devs):
        f.forward(d)
    g.end()
    with pytest.raises(nv.B200FFTError) as ei:
        g.sync()
    assert ei.value.code == -7  # B200FFT_ERR_DEVICE_STATUS
    g.close()
    monkeypatch.delenv("B200FFT_SCHED_STALL_TEST")
    objs, devs, xs = build()
    g = nv.Group([f.handle() for f in objs])
    g.begin()
    for f, d in zip(objs, devs):
        f.forward(d)
    g.end()
    g.sync()
    for shp, x, d in zip(shapes, xs, devs):
        nc = shp[-1] // 2 + 1
        X = to_host(d)[:2 * shp[0] * shp[1] * nc].view(np.complex64).reshape(shp[0], shp[1], nc)
        assert O.rel_l2(X, O.r2c_nd(x.astype(np.float64))) < REL_F32, shp
    g.close()
