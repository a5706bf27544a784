"""Benchmark: 512^3 FP32 R2C forward+backward through ParaFaFT on B200Backend.

One step is ParaFaFT_R2C<3, B200Backend<float>>::forward_in_place followed by
backward_in_place (the reference's own orchestrator, parafaft_r2c.hpp:360-542)
on a padded [512][512][514] float32 buffer of N(0,1) values (seeded).

Printed JSON line (rank 0):
  value       ms per forward+backward, device-resident buffer, CUDA events on
              the backend's stream, max over ranks (N > 1 runs N independent
              replicas: the path does not shard on one rank per GPU).
  e2e         the same call with the input copied from pinned host memory and
              the result copied back inside the timed region.
  roofline    the dominant kernel's algorithmic bytes per launch over its mean
              CUDA-event duration against the measured HBM copy bandwidth.
  cpu_baseline  the oracle's CPU port (scipy.fft float32 on all host cores,
              standing in for FFTWBackend<float>, whose libfftw3f is absent).
The buffer (539 MB) exceeds the 126 MB L2, so no flush is needed between steps.

--impl reference times that CPU path alone (all host threads) on the same
workload and prints the reference arm's line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHAPE = (512, 512, 512)
SEED = 1234
METRIC = "512^3 FP32 R2C fwd+bwd ms, % HBM roofline; plain vs split-TC at rel-L2<=2e-6"
WORKLOAD = "ParaFaFT_R2C<3, float> 512x512x512 forward_in_place+backward_in_place"
# the `config` of both arms' lines (the same workload, named the same way)
CONFIG = {"workload": WORKLOAD, "shape": list(SHAPE),
          "l2": "inputs larger than L2 (539 MB buffer)"}
ALG_BYTES = 6463422464  # one read + one write per fused pass, fwd+bwd

# DRAM bytes (read + write) per launch from the last `ncu --set full` capture
# of the same kernels (profiles/r2c512_kernels_ncu_full.md).
NCU_TRAFFIC = {"r2c_fwd": 1020436736, "c2c_stage1_fwd": 1030280192,
               "c2c_stage2_fwd": 1028872448, "c2c_stage2_bwd": 1020416000,
               "c2c_stage1_bwd": 1034022144, "c2r_bwd": 1037415424}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled through NVML every few
    milliseconds while the timed region runs (nvidia-smi's 100 ms minimum
    period is longer than short timed regions)."""

    # NVML clocks-event reason bits
    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[tuple[int, int]] = []
        self._stop = threading.Event()
        self._t = None
        self.err = None

    def start(self):
        try:
            import pynvml as N
            N.nvmlInit()
            import torch
            p = torch.cuda.get_device_properties(self.gpu)
            h = None
            if hasattr(p, "pci_bus_id"):
                bus = "%08x:%02x:%02x.0" % (getattr(p, "pci_domain_id", 0), p.pci_bus_id,
                                            getattr(p, "pci_device_id", 0))
                try:
                    h = N.nvmlDeviceGetHandleByPciBusId(bus)
                except Exception:
                    h = None
            if h is None:
                vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
                idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[0].isdigit() else self.gpu
                h = N.nvmlDeviceGetHandleByIndex(idx)
            self._N, self._h = N, h
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        except Exception as e:  # clocks are reported as unavailable
            self.err = str(e)
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        N, h = self._N, self._h
        while not self._stop.is_set():
            try:
                t = time.perf_counter()
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((t, sm, rs))
            except Exception as e:
                self.err = str(e)
                return
            time.sleep(0.002)

    def mark(self, which: str):
        setattr(self, which, time.perf_counter())

    def stop(self) -> dict:
        """Samples taken between mark('t0') and mark('t1') (the timed region);
        when the region is shorter than one NVML round trip, the samples
        nearest to it on either side."""
        if self._t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "note": f"clock sampling unavailable: {self.err}"}
        self._stop.set()
        self._t.join(timeout=2)
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        inside = [x for x in self.samples if t0 <= x[0] <= t1]
        if not inside and self.samples:
            before = [x for x in self.samples if x[0] < t0][-1:]
            after = [x for x in self.samples if x[0] > t1][:1]
            inside = before + after
        sm = [x[1] for x in inside]
        reasons = sorted({n for x in inside for n, bit in self.REASONS.items() if x[2] & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(sm)}


def make_input():
    from oracle import oracle as O
    x = O.normal_real(SHAPE, SEED, np.float32)
    return O.pad_real(x, np.float32), x


def cpu_port_step(buf_real: np.ndarray, workers: int):
    """FFTWBackend<float>-equivalent forward_in_place + backward_in_place on the
    CPU: scipy.fft (pocketfft) float32, all axes, unnormalised."""
    import scipy.fft as sf
    x = buf_real.reshape(SHAPE[0], SHAPE[1], SHAPE[2] + 2)[..., :SHAPE[2]]
    X = sf.rfftn(x, workers=workers)
    return sf.irfftn(X, s=SHAPE, norm="forward", workers=workers)


def time_cpu(buf_real, budget_s: float, max_steps: int, warmup: int = 1):
    workers = os.cpu_count() or 1
    for _ in range(warmup):
        cpu_port_step(buf_real, workers)
    times = []
    t_all = time.perf_counter()
    while len(times) < max_steps and (time.perf_counter() - t_all) < budget_s:
        t0 = time.perf_counter()
        cpu_port_step(buf_real, workers)
        times.append((time.perf_counter() - t0) * 1e3)
    return float(np.mean(times)), len(times), workers


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(values, pg=None, device="cpu"):
    """Each value's maximum over all ranks (one all-reduce). Replicas time
    their own device with CUDA events; the job's time is the slowest rank."""
    if pg is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def run_reference(args):
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return 0
    buf, _ = make_input()
    # each step is one full 512^3 forward+backward on the host cores; the run
    # stops early (and says so) if K steps would exceed the time budget
    ms, n, cores = time_cpu(buf, budget_s=args.ref_budget, max_steps=args.steps,
                            warmup=min(args.warmup, 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": n, "warmup": min(args.warmup, 1),
        "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1), seed 1234",
        "config": dict(CONFIG), "method": "scipy.fft float32 on the host cores",
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "port",
                         "sample": f"{n} full 512^3 fwd+bwd steps, scipy.fft float32 "
                                   f"(FFTWBackend<float> stand-in: libfftw3f absent)"},
        "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_kernels_only(args):
    """The timed loop alone (no checks, no comparators): the command profiled
    under ncu. --config picks the workload: r2c512 (default), c2c64 / c2c1024 /
    c2c4d (forward+backward of that grid), uneven256 (the grouped schedule of
    the uneven grids captured in a CUDA graph and replayed)."""
    import torch
    from parafaft_b200 import native as nv
    torch.cuda.set_device(0)
    if args.config in C2C_CONFIGS:
        shape, prec_s, _, seed = C2C_CONFIGS[args.config]
        prec = nv.F64 if prec_s == "f64" else nv.F32
        # the 4-D grid runs through the grid-owning backend (as in the bench)
        grid = args.config == "c2c4d"
        f = nv.ParaFaFT("c2c", shape, prec, backend="b200grid" if grid else "b200")
        gen = torch.Generator(device="cuda").manual_seed(seed)
        ctype = torch.complex128 if prec == nv.F64 else torch.complex64
        data = f.buffer() if grid else torch.empty(f.required_size, dtype=ctype, device="cuda")
        data.copy_(torch.randn(data.numel(), generator=gen, device="cuda", dtype=ctype))
        arg = None if grid else data
        for _ in range(args.warmup + args.steps):
            f.forward(arg)
            f.backward(arg)
        torch.cuda.synchronize()
        print("kernels-only done", "grid backend" if grid else f.handle().stats()["kernel_launches"])
        f.close()
        return 0
    if args.config == "uneven256":
        rng = np.random.default_rng(args.seed)
        shapes = [tuple(int(s) for s in rng.choice(UNEVEN_SIDES, 3)) for _ in range(args.grids)]
        objs = [nv.ParaFaFT("r2c", shp, nv.F32) for shp in shapes]
        gen = torch.Generator(device="cuda").manual_seed(args.seed)
        devs = [torch.randn(f.required_size, generator=gen, device="cuda") for f in objs]
        g = nv.Group([f.handle() for f in objs])
        g.begin()
        for f, d in zip(objs, devs):
            f.forward(d)
            f.backward(d)
        g.end()
        g.sync()
        g.capture()
        for _ in range(args.warmup + args.steps):
            g.replay()
        g.sync()
        print("kernels-only done", g.stats()["kernel_launches"])
        return 0
    host_buf, _ = make_input()
    fft = nv.ParaFaFT("r2c", SHAPE, nv.F32)
    dev = torch.from_numpy(host_buf).cuda()
    for _ in range(args.warmup + args.steps):
        fft.forward(dev)
        fft.backward(dev)
    torch.cuda.synchronize()
    print("kernels-only done", fft.handle().stats()["kernel_launches"])
    fft.close()
    return 0


def run_single_pass(args):
    """One batched 1D pass of the engine (the command profiled under ncu for a
    single kernel): FP32 C2C rows / columns or R2C rows of the given length and
    batch, forward, repeated; prints the plan and the CUDA-event time."""
    import torch
    from parafaft_b200 import native as nv
    kind, length, layout, batch = args.single_pass.split(",")
    length, batch, col = int(length), int(batch), layout == "col"
    torch.cuda.set_device(0)
    h = nv.Handle(nv.F32, 1, flags=nv.FLAG_SPLIT_TC if args.form == "split-tc" else 0)
    h.set_stream(torch.cuda.current_stream().cuda_stream)  # the events' stream
    if kind == "c2c":
        h.plan_c2c(0, length, batch, batch if col else 1, 1 if col else length)
        d = torch.randn(2 * length * batch, device="cuda")
        run = lambda: h.exec_c2c(0, nv.FORWARD, d)
        desc = h.plan_describe(nv.KIND_C2C, 0)
    else:
        dist = 2 * (length // 2 + 1)
        h.plan_r2c(length, batch, 1, dist)
        d = torch.randn(dist * batch, device="cuda")
        run = lambda: h.exec_r2c(d)
        desc = h.plan_describe(nv.KIND_R2C, 0)
    for _ in range(args.warmup):
        run()
    h.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        run()
    h.flush()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"single_pass": args.single_pass, "form": args.form, "plan": desc,
                      "ms": round(ms, 4), "GBps": round(2 * d.numel() * 4 / ms / 1e6, 1)}))
    h.close()
    return 0


C2C_CONFIGS = {
    # name: (shape, precision, input distribution, seed)
    "c2c64": ((64, 64, 64), "f64", "uniform", 11),
    "c2c1024": ((1024, 1024, 1024), "f32", "normal", 12),
    "c2c4d": ((128, 128, 64, 64), "f64", "uniform", 13),
}
# output planes X[k0, :, :] checked against the FP64 plane oracle at 1024^3
C2_PLANES = (0, 1, 333, 512, 1023)


def _timed_steps(fn, steps, warmup, stream=None, clocks=None):
    """ms per call of fn() over `steps` calls after `warmup` untimed ones
    (CUDA events on `stream`, default: torch's current stream)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if clocks:
        clocks.mark("t0")
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    if clocks:
        clocks.mark("t1")
    return e0.elapsed_time(e1) / steps


def _rel_dev(y, ref, chunk=1 << 26):
    """rel-L2 of two device tensors of the same length, in FP64, by chunks."""
    import torch
    num = den = 0.0
    for a in range(0, ref.numel(), chunk):
        r = ref[a:a + chunk].to(torch.complex128 if ref.is_complex() else torch.float64)
        d = y[a:a + chunk].to(r.dtype) - r
        num += float(torch.linalg.vector_norm(d)) ** 2
        den += float(torch.linalg.vector_norm(r)) ** 2
    return (num / den) ** 0.5


def _env_split_tc(on: bool):
    """Context for B200FFT_SPLIT_TC (read when a backend handle is created)."""
    import contextlib

    @contextlib.contextmanager
    def cm():
        old = os.environ.get("B200FFT_SPLIT_TC")
        if on:
            os.environ["B200FFT_SPLIT_TC"] = "1"
        else:
            os.environ.pop("B200FFT_SPLIT_TC", None)
        try:
            yield
        finally:
            if old is None:
                os.environ.pop("B200FFT_SPLIT_TC", None)
            else:
                os.environ["B200FFT_SPLIT_TC"] = old
    return cm()


def measure_c2c(name, steps, warmup, gpu_index=0):
    """C2C forward+backward of one of C2C_CONFIGS through the reference
    ParaFaFT_C2C orchestrator:
      c2c64    64^3 complex128: ParaFaFT_C2C<3, B200Backend<double>> (per-stage
               backend) and ParaFaFT_C2C<3, B200GridBackend<3, double>>;
               forward checked against the C oracle (FP64, full grid).
      c2c1024  1024^3 complex64: ParaFaFT_C2C<3, B200Backend<float>>, plain and
               split-TC; forward checked on the output planes C2_PLANES against
               the FP64 plane oracle (scipy.fft on the same complex64 input).
      c2c4d    128x128x64x64 complex128: ParaFaFT_C2C<4, B200GridBackend<4,
               double>> (the reference orchestrator's own path for a grid-owning
               backend; its per-stage path mis-sizes non-hypercubic grids,
               parafaft_c2c.hpp:826-831); forward checked against scipy.fft FP64
               on the full grid.
    Returns a dict: ms, alg_bytes, hbm_frac, rel-L2 forward and round trip,
    launches per step, clocks."""
    import torch
    from parafaft_b200 import native as nv
    from oracle import oracle as O
    torch.cuda.set_device(gpu_index)
    shape, prec_s, dist, seed = C2C_CONFIGS[name]
    prec = nv.F64 if prec_s == "f64" else nv.F32
    ctype = torch.complex128 if prec == nv.F64 else torch.complex64
    n = int(np.prod(shape))
    esz = 16 if prec == nv.F64 else 8
    alg = 2 * len(shape) * 2 * n * esz  # one read + one write per pass, fwd+bwd
    peak, peak_kind = _peaks()
    out = {"workload": f"{'x'.join(map(str, shape))} C2C {'complex128' if prec == nv.F64 else 'complex64'}",
           "input": f"re, im i.i.d. {'U[-1,1)' if dist == 'uniform' else 'N(0,1)'}, seed {seed}",
           "alg_bytes": alg, "peak_gbs": peak, "peak_source": peak_kind}

    # ---- input (the oracle sees exactly the values the GPU transforms)
    if name == "c2c1024":
        gen = torch.Generator(device="cuda").manual_seed(seed)
        x0 = torch.complex(torch.randn(n, generator=gen, device="cuda"),
                           torch.randn(n, generator=gen, device="cuda"))
        x_host = None
    else:
        x_host = (O.uniform_complex(shape, seed) if dist == "uniform"
                  else O.normal_complex(shape, seed)).astype(np.complex128 if prec == nv.F64
                                                             else np.complex64)
        x0 = torch.from_numpy(x_host.reshape(-1)).cuda()

    def forms():
        if name == "c2c64":
            return [("per_stage", "c2c", "b200", False), ("grid_backend", "c2c", "b200grid", False)]
        if name == "c2c1024":
            return [("plain", "c2c", "b200", False), ("split_tc", "c2c", "b200", True)]
        return [("grid_backend", "c2c", "b200grid", False)]

    ref_full = None
    ref_planes = None
    if name == "c2c64":
        ref_full = O.c2c_nd(x_host)  # the C oracle
        out["oracle"] = "C oracle FP64 (full grid)"
    elif name == "c2c4d":
        ref_full = O.c2c_nd(x_host, -1, "scipy")
        out["oracle"] = "scipy.fft FP64 (full grid)"
    else:
        plane = shape[1] * shape[2]
        xv = x0.view(shape)
        t0 = time.perf_counter()
        ref_planes = O.c2c_planes(lambda a, b: xv[a:b].cpu().numpy(), shape[0], C2_PLANES)
        out["oracle"] = (f"scipy FP64 planes X[k0,:,:], k0 in {list(C2_PLANES)} "
                         f"({time.perf_counter() - t0:.1f} s on the host)")
        del plane
    for key, kind, backend, split in forms():
        with _env_split_tc(split):
            f = nv.ParaFaFT(kind, shape, prec, backend=backend)
        grid = backend == "b200grid"
        data = f.buffer() if grid else torch.zeros(f.required_size, dtype=ctype, device="cuda")
        arg = None if grid else data
        data[:n].copy_(x0)
        f.forward(arg)
        torch.cuda.synchronize()
        if ref_full is not None:
            rel = O.rel_l2(data[:n].cpu().numpy().reshape(shape), ref_full)
        else:
            yv = data[:n].view(shape)
            got = np.stack([yv[k].cpu().numpy() for k in C2_PLANES])
            rel = O.rel_l2(got, ref_planes)
        f.backward(arg)
        torch.cuda.synchronize()
        rt = _rel_dev(data[:n] / n, x0)
        data[:n].copy_(x0)
        h = None if grid else f.handle()
        stream = None
        if h is not None:
            stream = torch.cuda.Stream()
            h.set_stream(stream.cuda_stream)
        step = lambda: (f.forward(arg), f.backward(arg))
        k = steps * (20 if n < (1 << 20) else 1)  # tiny grid: more steps
        clocks = ClockSampler(gpu_index)
        clocks.start()
        if h is not None:
            step()
            h.reset_stats()
        ms = _timed_steps(step, k, warmup, stream, clocks)
        clk = clocks.stop()
        entry = {"backend": (f"ParaFaFT_C2C<{len(shape)}, "
                             + (f"B200GridBackend<{len(shape)}, " if grid else "B200Backend<")
                             + ("double>>" if prec == nv.F64 else "float>>")),
                 "ms": round(ms, 4), "steps": k,
                 "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peak, 4),
                 "gbps": round(alg / (ms * 1e-3) / 1e9, 1),
                 "rel_l2_fwd": rel, "rel_l2_roundtrip": rt, "clocks": clk}
        if h is not None:
            st = h.stats()
            entry["gpu_launches_per_step"] = round(st["kernel_launches"] / (k + warmup), 2)
            entry["copies_per_step"] = round(st["copies_issued"] / (k + warmup), 2)
        if split:
            desc = f.handle().plan_describe(nv.KIND_C2C, 0).split()[0]
            entry["row_kernel"] = desc
        out[key] = entry
        f.close()
        del data
        torch.cuda.empty_cache()
    if name == "c2c1024":
        out["split_tc"]["speedup_vs_plain"] = round(out["plain"]["ms"] / out["split_tc"]["ms"], 3)
        out["split_tc"]["error_vs_plain"] = round(out["split_tc"]["rel_l2_fwd"] /
                                                 out["plain"]["rel_l2_fwd"], 3)
    del x0
    torch.cuda.empty_cache()
    return out


def run_c2c_config(args):
    line = {"metric": f"{args.config} C2C fwd+bwd ms", "unit": "ms", "n_gpus": 1,
            "higher_is_better": False, "steps": args.steps, "warmup": args.warmup}
    line.update(measure_c2c(args.config, args.steps, args.warmup))
    print(json.dumps(line), flush=True)
    return 0


def time_grid_backend(kind, shape, prec, fill, steps, warmup):
    """The same forward+backward through the reference orchestrator on
    B200GridBackend<D, T> (the grid-owning backend: each transform one
    replayed CUDA graph on the backend's own buffer). `fill(buf)` writes the
    input into that buffer. Returns ms per step (CUDA events; forward and
    backward wait for their graph), the round-trip rel-L2 and launches per step."""
    import torch
    from parafaft_b200 import native as nv
    g = nv.ParaFaFT(kind, shape, prec, backend="b200grid")
    buf = g.buffer()
    fill(buf)
    x0 = buf.clone()
    n = int(np.prod(shape))
    g.forward(None)
    g.backward(None)
    if kind == "r2c":
        ref = x0.view(-1, 2 * (shape[-1] // 2 + 1))[:, :shape[-1]].double()
        got = buf.view(-1, 2 * (shape[-1] // 2 + 1))[:, :shape[-1]].double() / n
    else:
        ref, got = x0.to(torch.complex128), buf.to(torch.complex128) / n
    rt = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
    del ref, got, x0
    for _ in range(warmup):
        g.forward(None)
        g.backward(None)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        g.forward(None)
        g.backward(None)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    g.close()
    torch.cuda.empty_cache()
    return {"ms": round(ms, 4), "rel_l2_roundtrip": rt,
            "backend": f"ParaFaFT_{'R2C' if kind == 'r2c' else 'C2C'}<{len(shape)}, "
                       f"B200GridBackend<{len(shape)}, {'double' if prec == nv.F64 else 'float'}>>"}


UNEVEN_SIDES = [32, 48, 60, 64, 80, 96, 120, 128, 160]


def measure_uneven(grids, seed, steps, warmup, gpu_index=0):
    """`grids` independent R2C float32 grids of uneven sizes (each side drawn
    from UNEVEN_SIDES with numpy.random.default_rng(seed)), Gaussian random
    fields with P(k) ~ k^-3, one ParaFaFT_R2C<3, B200Backend<float>> object per
    grid. Forward+backward of all grids timed three ways:
      loop    the grids one after another (per-grid launches and syncs),
      grouped one b200fft group: each dependency level of all grids launched
              together (per-length launches side by side on several streams),
      graph   the grouped schedule captured once in a CUDA graph and replayed;
      schedule (graph) the dependency-scheduled form: one persistent launch
              walking a work list of (pass, tile) items, each grid's passes
              waiting only for that grid's previous pass.
    Every grid's forward output is checked against the FP64 oracle (scipy.fft)
    and its round trip against its input."""
    import torch
    from parafaft_b200 import native as nv
    from oracle import oracle as O
    torch.cuda.set_device(gpu_index)
    rng = np.random.default_rng(seed)
    shapes = [tuple(int(s) for s in rng.choice(UNEVEN_SIDES, 3)) for _ in range(grids)]
    objs, devs, hosts, xs = [], [], [], []
    alg = 0
    for i, shp in enumerate(shapes):
        x = O.gaussian_random_field(shp, seed + 1 + i).astype(np.float32)
        f = nv.ParaFaFT("r2c", shp, nv.F32)
        buf = np.zeros(f.required_size, np.float32)
        p = O.pad_real(x, np.float32)
        buf[:p.size] = p
        objs.append(f)
        xs.append(x)
        hosts.append(torch.from_numpy(buf))
        devs.append(torch.from_numpy(buf).cuda())
        nr = int(np.prod(shp))
        nc = shp[0] * shp[1] * (shp[2] // 2 + 1)
        alg += 2 * (4 * nr + 40 * nc)  # R2C pass + two C2C passes, each direction
    dflt = torch.cuda.default_stream()

    def loop():
        for f, d in zip(objs, devs):
            f.forward(d)
            f.backward(d)

    loop_ms = _timed_steps(loop, steps, warmup, dflt)

    def make_group(schedule):
        old = os.environ.pop("B200FFT_GROUP_SCHEDULE", None)
        if schedule:
            os.environ["B200FFT_GROUP_SCHEDULE"] = "1"
        try:
            grp = nv.Group([f.handle() for f in objs])
            grp.begin()
            for f, d in zip(objs, devs):
                f.forward(d)
                f.backward(d)
            grp.end()
            grp.sync()
        finally:
            os.environ.pop("B200FFT_GROUP_SCHEDULE", None)
            if old is not None:
                os.environ["B200FFT_GROUP_SCHEDULE"] = old
        return grp

    # the dependency-scheduled form (one persistent launch over a work list of
    # (pass, tile) items), as a CUDA graph
    gs = make_group(True)
    sched_stats = gs.stats()  # the run at group end: launches of one run
    gs.capture()
    sched_graph_ms = _timed_steps(gs.replay, steps, warmup, dflt)
    gs.close()
    # the default form: per-level launches of the specialised kernels
    g = make_group(False)
    levels_stats = g.stats()
    grouped_ms = _timed_steps(g.replay, steps, warmup, dflt)
    g.capture()
    clocks = ClockSampler(gpu_index)
    clocks.start()
    graph_ms = _timed_steps(g.replay, steps, warmup, dflt, clocks)
    clk = clocks.stop()
    # forward of every grid (per-grid objects) against the FP64 oracle
    fwd_errs = []
    for f, d, h, x, shp in zip(objs, devs, hosts, xs, shapes):
        d.copy_(h)
        f.forward(d)
        npad = shp[0] * shp[1] * 2 * (shp[2] // 2 + 1)
        X = O.complex_view(d.cpu().numpy()[:npad], shp)
        fwd_errs.append(O.rel_l2(X, O.r2c_nd(x.astype(np.float64), impl="scipy")))
    # one grouped (graph) round trip of all grids against their inputs
    for d, h in zip(devs, hosts):
        d.copy_(h)
    g.replay()
    g.sync()
    rt_errs = []
    for shp, d, x in zip(shapes, devs, xs):
        npad = shp[0] * shp[1] * 2 * (shp[2] // 2 + 1)
        y = O.unpad_real(d.cpu().numpy()[:npad], shp) / x.size
        rt_errs.append(O.rel_l2(y, x))
    stats = g.stats()
    peak, peak_kind = _peaks()
    g.close()
    for f in objs:
        f.close()
    return {
        "workload": f"{grids} independent ParaFaFT_R2C<3, float> grids, sides from {UNEVEN_SIDES}",
        "input": f"Gaussian random fields P(k)~k^-3, zero mean, seed {seed}",
        "grids": grids, "total_points": int(sum(np.prod(s) for s in shapes)),
        "loop_ms": round(loop_ms, 4), "grouped_ms": round(grouped_ms, 4),
        "graph_ms": round(graph_ms, 4), "speedup_graph_vs_loop": round(loop_ms / graph_ms, 2),
        "schedule_graph_ms": round(sched_graph_ms, 4),
        "schedule_launches_per_run": sched_stats["kernel_launches"],
        "launches_per_run": levels_stats["kernel_launches"],
        "alg_bytes": alg, "hbm_frac_graph": round(alg / (graph_ms * 1e-3) / 1e9 / peak, 4),
        "peak_gbs": peak, "peak_source": peak_kind,
        "oracle": "scipy.fft FP64 per grid",
        "max_rel_l2_fwd": max(fwd_errs), "max_rel_l2_roundtrip": max(rt_errs),
        "group": stats, "clocks": clk,
    }


def run_uneven(args):
    line = {"metric": "256 uneven R2C f32 grids fwd+bwd ms", "unit": "ms", "n_gpus": 1,
            "higher_is_better": False, "steps": args.steps, "warmup": args.warmup}
    line.update(measure_uneven(args.grids, args.seed, args.steps, args.warmup))
    line["value"] = line["graph_ms"]
    print(json.dumps(line), flush=True)
    return 0


def measure_split_tc(args, pinned, x_real, dev, stream, plain_ms):
    """The 512^3 R2C forward+backward with B200FFT_SPLIT_TC=1 (its 512-point
    column passes on the split-precision tensor-core kernels): device ms per
    step, forward rel-L2 against the FP64 reference, and plain / split."""
    import torch
    from parafaft_b200 import native as nv
    from oracle import oracle as O
    old = os.environ.get("B200FFT_SPLIT_TC")
    os.environ["B200FFT_SPLIT_TC"] = "1"
    try:
        f = nv.ParaFaFT("r2c", SHAPE, nv.F32)
    finally:
        if old is None:
            os.environ.pop("B200FFT_SPLIT_TC")
        else:
            os.environ["B200FFT_SPLIT_TC"] = old
    try:
        h = f.handle()
        h.set_stream(stream.cuda_stream)
        kinds = sorted({h.plan_describe(nv.KIND_C2C, s).split()[0] for s in (1, 2)})
        with torch.cuda.stream(stream):
            dev.copy_(pinned, non_blocking=True)
        f.forward(dev)
        X = dev.cpu().numpy().view(np.complex64).reshape(512, 512, 257)
        rel = O.rel_l2(X, O.r2c_nd(x_real.astype(np.float64), impl="scipy"))
        del X
        with torch.cuda.stream(stream):
            dev.copy_(pinned, non_blocking=True)
        for _ in range(args.warmup):
            f.forward(dev)
            f.backward(dev)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            f.forward(dev)
            f.backward(dev)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        return {"ms": round(ms, 4), "rel_l2_fwd_vs_fp64": rel, "column_kernels": kinds,
                "speedup_vs_plain": round(plain_ms / ms, 3)}
    finally:
        f.close()


def run_b200(args):
    import torch
    from parafaft_b200 import native as nv
    from oracle import oracle as O

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist

    host_buf, x_real = make_input()
    fft = nv.ParaFaFT("r2c", SHAPE, nv.F32)
    req = fft.required_size
    assert req == host_buf.size, (req, host_buf.size)
    h = fft.handle()
    stream = torch.cuda.Stream()
    h.set_stream(stream.cuda_stream)
    dev = torch.empty(req, dtype=torch.float32, device="cuda")
    pinned = torch.from_numpy(host_buf).pin_memory()
    result_host = torch.empty_like(pinned).pin_memory()

    with torch.cuda.stream(stream):
        dev.copy_(pinned, non_blocking=True)
    stream.synchronize()

    # ---- correctness of the measured configuration (outside the timed region)
    fft.forward(dev)
    X = dev.cpu().numpy().view(np.complex64).reshape(512, 512, 257)
    Xref = O.r2c_nd(x_real.astype(np.float64), impl="scipy")
    rel_fwd = O.rel_l2(X, Xref)
    del X, Xref
    fft.backward(dev)
    back = O.unpad_real(dev.cpu().numpy(), SHAPE) / np.prod(SHAPE)
    rel_rt = O.rel_l2(back, x_real)
    del back

    def step():
        fft.forward(dev)
        fft.backward(dev)

    # ---- device-resident timing
    with torch.cuda.stream(stream):
        dev.copy_(pinned, non_blocking=True)
    for _ in range(args.warmup):
        step()
    h.reset_stats()
    clocks = ClockSampler(local)
    clocks.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks.mark("t0")
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark("t1")
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    st = h.stats()
    launches = st["kernel_launches"] + st["copies_issued"]

    # ---- per-step distribution (a second pass, events between steps): the
    #      median beside the mean, as the reference's GPU benchmark reports both
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        step()
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]

    # ---- per-kernel timing (a second pass of the same steps, events around
    #      every launch on the backend's stream)
    h.set_profiling(True)
    h.reset_stats()
    for _ in range(args.steps):
        step()
    log = h.log()
    h.set_profiling(False)
    per = {}
    for r in log:
        key = ("r2c" if r["kind"] == 1 else "c2r" if r["kind"] == 2 else f"c2c_stage{r['stage']}") \
            + ("_fwd" if r["direction"] == 0 else "_bwd")
        per.setdefault(key, []).append((r["ms"], r["bytes"]))
    kernels = {k: {"ms": round(float(np.mean([m for m, _ in v])), 4),
                   "bytes": int(v[0][1]), "launches": len(v)} for k, v in per.items()}
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    peak, peak_kind = _peaks()
    ach = kernels[dom]["bytes"] / (kernels[dom]["ms"] * 1e-3) / 1e9
    for k in kernels:
        kernels[k]["GBps"] = round(kernels[k]["bytes"] / (kernels[k]["ms"] * 1e-3) / 1e9, 1)

    # ---- end to end through the same API with host buffers: every step copies
    #      its input from pinned host memory, transforms it and reads its result
    #      back; three device buffers and two copy streams let step i+1's upload,
    #      step i's transform and step i-1's download run at the same time (PCIe
    #      is full duplex), as a user streaming many fields would run it
    NBUF = 3
    bufs = (dev,) + tuple(torch.empty_like(dev) for _ in range(NBUF - 1))
    host_in = (pinned,) + tuple(torch.empty_like(pinned).pin_memory() for _ in range(NBUF - 1))
    for h_ in host_in[1:]:
        h_.copy_(pinned)
    host_out = (result_host,) + tuple(torch.empty_like(result_host).pin_memory()
                                      for _ in range(NBUF - 1))
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()
    done_down = [torch.cuda.Event() for _ in range(NBUF)]
    up_done = [torch.cuda.Event() for _ in range(NBUF)]

    # forward()/backward() return only when the transform is done (ParaFaFT
    # calls sync()), so step i+1's upload is issued before step i's transform:
    # the upload then runs during the transform and both PCIe directions stay
    # busy back to back
    def upload(i):
        k = i % NBUF
        s_up.wait_event(done_down[k])          # the buffer's previous result is out
        with torch.cuda.stream(s_up):
            bufs[k].copy_(host_in[k], non_blocking=True)
        up_done[k].record(s_up)

    def transform_and_download(i):
        k = i % NBUF
        d = bufs[k]
        stream.wait_event(up_done[k])
        fft.forward(d)
        fft.backward(d)
        comp = torch.cuda.Event()
        comp.record(stream)
        s_down.wait_event(comp)
        with torch.cuda.stream(s_down):
            host_out[k].copy_(d, non_blocking=True)
        done_down[k].record(s_down)

    def e2e_run(n):
        upload(0)
        for i in range(n):
            if i + 1 < n:
                upload(i + 1)
            transform_and_download(i)

    for k in range(NBUF):
        done_down[k].record(s_down)
    e2e_run(max(NBUF, args.warmup))
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(s_up)
    e2e_run(args.steps)
    e3.record(s_down)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3) / args.steps
    del bufs

    # ---- the split-precision tensor-core form of the same workload: the
    #      column passes (512-point C2C) on the tensor cores, FP16 hi+lo
    split = measure_split_tc(args, pinned, x_real, dev, stream, ms)

    # ---- the same step through the grid-owning backend (handles_distributed)
    grid = time_grid_backend("r2c", SHAPE, nv.F32, lambda b: b.copy_(pinned[:b.numel()]),
                             args.steps, args.warmup)
    grid["hbm_frac"] = round(ALG_BYTES / (grid["ms"] * 1e-3) / 1e9 / _peaks()[0], 4)

    # ---- the reference's cuFFT backend on the same GPU, same orchestrator
    cufft_ms = None
    try:
        ref = nv.ParaFaFT("r2c", SHAPE, nv.F32, backend="cufft")
        with torch.cuda.stream(stream):
            dev.copy_(pinned, non_blocking=True)
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            ref.forward(dev)
            ref.backward(dev)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        # CuFFTBackend uses its own blocking stream; the legacy default stream
        # orders events around it and forward/backward block on completion.
        t0.record(torch.cuda.default_stream())
        for _ in range(args.steps):
            ref.forward(dev)
            ref.backward(dev)
        t1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        cufft_ms = t0.elapsed_time(t1) / args.steps
        ref.close()
    except Exception as e:  # comparator only
        cufft_ms = f"unavailable: {e}"

    ms, e2e_ms = max_over_ranks([ms, e2e_ms], pg, "cuda")

    # ---- the other configurations, each with its own oracle check and
    #      roofline (one GPU only: at N > 1 the replicas run the headline alone)
    configs = None
    if world == 1 and not args.headline_only:
        fft.close()
        del dev, pinned, result_host
        torch.cuda.empty_cache()
        configs = {}
        for key, fn in (("c0_c2c64_f64", lambda: measure_c2c("c2c64", args.steps, args.warmup, local)),
                        ("c2_c2c1024_f32", lambda: measure_c2c("c2c1024", max(4, args.steps // 2),
                                                               args.warmup, local)),
                        ("c3_uneven256_r2c_f32", lambda: measure_uneven(args.grids, args.seed,
                                                                        args.steps, args.warmup, local)),
                        ("c4_c2c4d_f64", lambda: measure_c2c("c2c4d", args.steps, args.warmup, local))):
            t0 = time.perf_counter()
            try:
                configs[key] = fn()
            except Exception as e:  # reported, never silently dropped
                configs[key] = {"error": f"{type(e).__name__}: {e}"}
            configs[key]["wall_s"] = round(time.perf_counter() - t0, 1)
            torch.cuda.empty_cache()

    if rank == 0:
        # the CPU baseline is timed at N = 1 only (at N > 1 the other ranks
        # would wait on it at the closing barrier)
        cpu = None
        if world == 1:
            cpu_ms, cpu_n, cores = time_cpu(host_buf, budget_s=args.cpu_budget, max_steps=8)
            cpu = {"value": round(cpu_ms, 1), "unit": "ms", "cores": cores, "kind": "port",
                   "sample": f"{cpu_n} full 512^3 fwd+bwd steps, scipy.fft float32 "
                             f"(FFTWBackend<float> stand-in: libfftw3f absent)"}
        nbytes = host_buf.nbytes
        line = {
            "metric": METRIC, "value": round(ms, 4), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic N(0,1) float32, seed 1234",
            "config": dict(CONFIG), "method": "plain FP32 Stockham", "replicas": world,
            "rel_l2_fwd_vs_fp64": rel_fwd, "rel_l2_roundtrip": rel_rt,
            "step_ms_median": round(statistics.median(per_step), 4),
            "step_ms_mean_per_step_events": round(statistics.fmean(per_step), 4),
            "hbm_roofline_frac_step": round(ALG_BYTES / (ms * 1e-3) / 1e9 / peak, 4),
            # 5 N log2 N per direction (C2C-equivalent convention), and the
            # R2C convention at half of it, labelled as such
            "gflops_5nlogn": round(2 * 5 * np.prod(SHAPE) * 27 / (ms * 1e-3) / 1e9, 1),
            "gflops_r2c_half_5nlogn": round(5 * np.prod(SHAPE) * 27 / (ms * 1e-3) / 1e9, 1),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(ach / peak, 4),
                         "traffic": NCU_TRAFFIC.get(dom), "traffic_source": "ncu capture",
                         "peak_source": peak_kind},
            "kernels": kernels,
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes,
                    "pipeline": "three device buffers; step i+1's upload (issued before step i's transform), step i's transform and step i-1's download overlap"},
            "cufft_backend_ms": cufft_ms if isinstance(cufft_ms, str) else round(cufft_ms, 4),
            "split_tc": split,
            "grid_backend": grid,
            "configs": configs if configs is not None else "headline only (N > 1 replicas or --headline-only)",
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if configs is None:
        fft.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=150.0)
    ap.add_argument("--kernels-only", action="store_true",
                    help="run only the timed loop (used for ncu captures)")
    ap.add_argument("--config", default="r2c512",
                    choices=["r2c512", "uneven256", "c2c64", "c2c1024", "c2c4d"],
                    help="r2c512: the headline 512^3 R2C (default); uneven256: 256 "
                         "uneven grids; c2c64 / c2c1024 / c2c4d: the C2C configurations")
    ap.add_argument("--headline-only", action="store_true",
                    help="time the 512^3 headline alone, without the other configurations")
    ap.add_argument("--grids", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--single-pass", default=None, metavar="KIND,LENGTH,LAYOUT,BATCH",
                    help="profile one engine pass: e.g. c2c,256,row,262144 or r2c,512,row,262144 "
                         "(layout row = contiguous points, col = neighbouring transforms "
                         "adjacent); runs --warmup + --steps launches and prints the time")
    ap.add_argument("--form", default="plain", choices=["plain", "split-tc"],
                    help="split-tc: FP32 C2C passes of length 256/512/1024 use the "
                         "split-precision tensor-core kernels (FP16 hi+lo, FP32 accumulate)")
    args = ap.parse_args()
    if args.form == "split-tc":
        os.environ["B200FFT_SPLIT_TC"] = "1"  # read when each backend handle is created
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.kernels_only:
        return run_kernels_only(args)
    if args.single_pass:
        return run_single_pass(args)
    if args.config == "uneven256":
        return run_uneven(args)
    if args.config in C2C_CONFIGS:
        return run_c2c_config(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
