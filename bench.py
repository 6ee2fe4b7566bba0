"""Benchmark of the SSAM stencil path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ssam|reference]
                    [--workload NAME]

A step is one pass of the stencil over one grid.  The default workload is the
memory-bound head of the 2D box family: 9-point box (radius 1), FP32,
8192 x 8192, uniform[-1,1) input, coefficients uniform[0,1) normalised to
sum 1, zero padding, one step per call.  Inputs are seeded synthetic data.

Metric: GCells/s = cells x steps / time.  `value` is device-timed with the
grid already in HBM (CUDA events on the launching stream, max over ranks);
`e2e` is the same metric through the host-buffer C entry point
(ssam_stencil2d_host) with the host<->device copies inside the timed region.
Under torchrun every rank steps its own grid (independent shards, no
collective on the data path: weak scaling).

`--impl reference` times the reference's own CPU golden (`Convolution<T>`,
ssai-2dconv/common.h:186-216, compiled from its sources into oracle/_ref) on
the host cores for the same workload, on rank 0 only.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1000 * 1000
FALLBACK_HBM_GBS = 6650.0


def workloads():
    """name -> spec.  kind: 'box' / 'star' (ssam_stencil2d) or 'conv'."""
    w = {}
    for dt in ("f32", "f64", "bf16"):
        for r in range(1, 6):
            w[f"box{r}_{dt}_8192"] = dict(kind="box", r=r, dtype=dt, n=8192, steps=1,
                                          boundary="zero")
            w[f"box{r}_{dt}_8192_16steps"] = dict(kind="box", r=r, dtype=dt, n=8192,
                                                  steps=16, boundary="zero")
        for f in range(3, 22, 2):
            w[f"conv{f}_{dt}_8192"] = dict(kind="conv", r=f // 2, f=f, dtype=dt, n=8192,
                                           steps=1, boundary="zero")
        for r in range(1, 7):
            w[f"star{r}_{dt}_8192"] = dict(kind="star", r=r, dtype=dt, n=8192, steps=1,
                                           boundary="zero")
    w["star1_f32_4096_copy"] = dict(kind="star", r=1, dtype="f32", n=4096, steps=1,
                                    boundary="copy", coeffs=[0.2] * 5)
    # 3D, 512^3, 100 steps per call (one captured CUDA graph), fixed boundary
    for dt in ("f32", "bf16", "f64"):
        for gold, r in (("j3d7pt", 1), ("j3d13pt", 2), ("poisson", 1)):
            w[f"{gold}_{dt}_512_100steps"] = dict(kind="3d", gold=gold, r=r, dtype=dt, n=512,
                                                  steps=100, boundary="copy")
            w[f"{gold}_{dt}_512"] = dict(kind="3d", gold=gold, r=r, dtype=dt, n=512,
                                         steps=1, boundary="copy")
    # batches of 256 uneven grids (sides log-uniform in [64, 2048]), 50 steps
    for dt in ("f32", "bf16", "f64"):
        w[f"batched256_star1_{dt}_50steps"] = dict(kind="batched", shape="star", r=1, dtype=dt,
                                                   ngrids=256, steps=50, boundary="copy",
                                                   coeffs=[0.2] * 5, n=2048)
        w[f"batched256_box2_{dt}_50steps"] = dict(kind="batched", shape="box", r=2, dtype=dt,
                                                  ngrids=256, steps=50, boundary="copy", n=2048)
    # Poisson -lap(u) = f on 128^3, Dirichlet 0, 8 Gaussian-bump right-hand
    # sides, solved to 1e-5 relative residual (FP64): the plain arm (FP32
    # Jacobi sweeps inside the FP64 defect correction, from zero) and the
    # learned arm (the trained CNN + BF16 sweeps + the same FP64 loop)
    for arm in ("plain", "learned"):
        w[f"poisson128x8_{arm}"] = dict(kind="poisson", arm=arm, n=128, nb=8, tol=1e-5,
                                        dtype="f64", r=1, steps=1, boundary="zero")
    # the warm-start network's forward pass (the learned arm's tensor-core part)
    # the Poisson arms' sweep kernel alone: 100 Jacobi sweeps of 8 x 128^3
    for dt in ("f32", "bf16"):
        w[f"jacobi128x8_{dt}_100sweeps"] = dict(kind="jacobi", n=128, nb=8, dtype=dt, r=1,
                                                steps=100, boundary="zero")
    for nb in (8, 1):  # (the one-grid case is small enough for a full ncu capture)
        w[f"cnn128x{nb}_forward"] = dict(kind="cnn", n=128, nb=nb, dtype="bf16", r=1, steps=1,
                                         boundary="zero")
    return w


DEFAULT = "box1_f32_8192"

CNN_WEIGHTS = os.path.join(ROOT, "ssam_b200", "data", "poisson_cnn_n128.bin")
# sweeps between two FP64 residuals and the sweep damping of each arm
POISSON_ARMS = {
    "plain": dict(sweep_dtype="f32", sweeps_per_correction=2000, omega=1.0),
    "learned": dict(sweep_dtype="bf16", sweeps_per_correction=250, omega=0.8, cnn_smoothing=2),
}
# FP32-sweep defect-correction sweeps the plain arm needs for the 8 x 128^3
# benchmark problem to reach 1e-5 (measured on a B200; the CPU reference arm
# extrapolates its sweep rate to this count)
PLAIN_SWEEPS_128x8 = 36000


def taps(spec) -> int:
    r = spec["r"]
    if spec["kind"] == "batched":
        return 4 * r + 1 if spec["shape"] == "star" else (2 * r + 1) ** 2
    if spec["kind"] == "3d":
        return {"j3d7pt": 7, "j3d13pt": 13, "poisson": 19}[spec["gold"]]
    if spec["kind"] == "star":
        return 4 * r + 1
    if spec["kind"] == "conv":
        return spec["f"] ** 2
    return (2 * r + 1) ** 2


def cube3d(spec) -> np.ndarray:
    """The reference's own 3D coefficients (_F<z><y><x> defines, read from the
    committed tests/golden/coefficients.json), scaled so that their absolute
    values sum to 1: 100 steps stay bounded (the 19-point operator has
    coefficients of both signs)."""
    with open(os.path.join(ROOT, "tests", "golden", "coefficients.json")) as f:
        c = json.load(f)["coeffs3d"][spec["gold"]]
    r = spec["r"]
    cube = np.zeros((2 * r + 1,) * 3)
    for k, v in c.items():
        cube[int(k[0]), int(k[1]), int(k[2])] = v
    return cube / np.abs(cube).sum()


def coefficients(spec):
    """Coefficients uniform[0,1) normalised to sum 1 (seeded)."""
    if "coeffs" in spec:
        return spec["coeffs"]
    if spec["kind"] == "3d":
        return cube3d(spec)
    g = np.random.Generator(np.random.PCG64(1234 + spec["r"]))
    c = g.random(taps(spec))
    return list(c / c.sum())


def np_dtype(dt):
    return {"f32": np.float32, "f64": np.float64}.get(dt)


def elem_size(dt) -> int:
    return {"f32": 4, "f64": 8, "bf16": 2}[dt]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def load_traffic(name):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch from the
    committed ncu summary (profiles/traffic.json), if one covers the
    workload."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(name)
    except Exception:
        return None


# ----------------------------------------------------------- clock sampler --

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        time.sleep(0.15)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- CPU timing --

_CPU_PROBE: dict = {}  # per workload: (seconds per row, cached inputs)


def host_threads() -> int:
    """Threads the OpenMP loops of oracle/ and oracle/_ref run with: the
    OMP_NUM_THREADS setting, else every core this process may use."""
    env = os.environ.get("OMP_NUM_THREADS", "").split(",")[0].strip()
    if env.isdigit() and int(env) > 0:
        return int(env)
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the cpu_baseline line."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_reference_rate(spec, budget_s: float, seed: int = 7):
    """The reference's compiled Convolution<T> (or 3D gold) on the host
    cores: returns (GCells/s, sample description, cores, kind).  Runs whole
    grids until ~budget_s, or a row slab of the grid when one grid takes
    longer.  kind is "reference" when oracle/_ref was built from the
    reference's sources, else "port": the oracle's C restatement of the same
    loops (also OpenMP over rows) stands in for it."""
    import oracle
    use_ref = oracle.have_ref()
    kind = "reference" if use_ref else "port"
    if use_ref:
        conv = oracle.ref_convolution
    else:
        def conv(a, m):
            return oracle.conv2d(a, m, "zero")
    dt = np_dtype(spec["dtype"]) or np.float32
    n = spec["n"]
    g = np.random.Generator(np.random.PCG64(seed))
    cores = host_threads()
    if spec["kind"] == "3d":
        # the reference gold for this stencil (v2::j3d7pt_gold / j3d13pt_gold /
        # poisson_gold), iterated with copy-back like its IT-step check
        cur = g.random((n, n, n), dtype=np.float32).astype(dt)
        if use_ref:
            def gold(a):
                return oracle.ref_gold3d(spec["gold"], a)
        elif spec["gold"] == "poisson":
            def gold(a):
                return oracle.poisson19(a, "gold")
        else:
            cube = cube3d(spec)
            r = spec["r"]
            taps = [(z - r, y - r, x - r, float(cube[z, y, x]))
                    for z, y, x in zip(*np.nonzero(cube))]

            def gold(a):
                return oracle.taps3d(a, taps, "gold")
        t0 = time.perf_counter()
        done = 0
        while True:
            cur = gold(cur)
            done += 1
            el = time.perf_counter() - t0
            if el >= budget_s or done >= spec["steps"]:
                break
        sample = f"{done} of {spec['steps']} step(s) on the full {n}^3 grid"
        return n ** 3 * done / el / 1e9, sample, cores, kind
    c = coefficients(spec)
    if spec["kind"] == "star":
        r = spec["r"]
        m = np.zeros((2 * r + 1, 2 * r + 1))
        m[r, r] = c[0]
        for k in range(1, r + 1):
            m[r - k, r], m[r + k, r], m[r, r - k], m[r, r + k] = c[1 + 4 * (k - 1): 5 + 4 * (k - 1)]
    else:
        f = 2 * spec["r"] + 1 if spec["kind"] == "box" else spec["f"]
        m = np.array(c).reshape(f, f)
    m = m.astype(dt)
    # probe on a slab to size the sample (once per workload: the reference
    # arm calls this every step with a small budget)
    key = (id(spec), str(dt))
    if key not in _CPU_PROBE:
        rows = min(n, 256)
        slab = g.uniform(-1, 1, size=(rows, n)).astype(dt)
        t0 = time.perf_counter()
        conv(slab, m)
        _CPU_PROBE[key] = ((time.perf_counter() - t0) / rows, {})
    per_row, inputs = _CPU_PROBE[key]
    steps = spec["steps"]
    per_grid = per_row * n * steps
    if per_grid <= budget_s:
        if "grid" not in inputs:
            inputs["grid"] = g.uniform(-1, 1, size=(n, n)).astype(dt)
        src = inputs["grid"]
        reps = max(1, int(budget_s / per_grid))
        t0 = time.perf_counter()
        for _ in range(reps):
            cur = src
            for _ in range(steps):
                cur = conv(cur, m)
        el = time.perf_counter() - t0
        cells = reps * n * n * steps
        sample = f"{reps} x full {n}x{n} grid x {steps} step(s)"
    else:
        rows = max(2 * spec["r"] + 1, min(n, int(budget_s / (per_row * steps))))
        if inputs.get("slab_rows") != rows:
            inputs["slab"] = g.uniform(-1, 1, size=(rows, n)).astype(dt)
            inputs["slab_rows"] = rows
        src = inputs["slab"]
        t0 = time.perf_counter()
        cur = src
        for _ in range(steps):
            cur = conv(cur, m)
        el = time.perf_counter() - t0
        cells = rows * n * steps
        sample = f"{rows}-row slab of the {n}x{n} grid x {steps} step(s)"
    return cells / el / 1e9, sample, cores, kind


# ------------------------------------------------------------ reference arm --

def poisson_cpu_baseline(f_np, sweeps_needed, budget_s=10.0):
    """The oracle's FP64 Jacobi sweep (C, one core) on the same 8 x 128^3
    problem for a bounded number of sweeps; the time to 1e-5 is extrapolated
    from its rate and the sweep count the plain arm needed."""
    import oracle
    u = np.zeros_like(f_np)
    t0 = time.perf_counter()
    done = 0
    while time.perf_counter() - t0 < budget_s and done < 200:
        u = oracle.jacobi7(f_np, u, 4)
        done += 4
    el = time.perf_counter() - t0
    per_sweep = el / done
    return {"value": per_sweep * sweeps_needed, "unit": "s", "cores": host_threads(),
            "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{done} FP64 Jacobi sweeps of the 8 x 128^3 problem in {el:.2f} s "
                      f"({f_np.size * done / el / 1e9:.3f} GCell-updates/s), extrapolated to "
                      f"the {sweeps_needed} sweeps the plain arm needed"}


def run_reference_poisson(args, spec, name):
    from ssam_b200.workloads import gaussian_rhs
    f_np = gaussian_rhs(spec["nb"], spec["n"], 7)
    vals = []
    cb = None
    for i in range(args.steps + args.warmup):
        cb = poisson_cpu_baseline(f_np, PLAIN_SWEEPS_128x8,
                                  budget_s=max(1.0, min(10.0, 100.0 / (args.steps + args.warmup))))
        if i >= args.warmup:
            vals.append(cb["value"])
    value = statistics.median(vals)
    print(json.dumps({
        "impl": "reference", "metric": "Poisson time-to-1e-5 relative residual",
        "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (8 Gaussian-bump right-hand sides, seed 7)",
        "config": {"workload": name, "grid": f"{spec['nb']}x{spec['n']}^3", "tol": spec["tol"],
                   "arm": "plain Jacobi on the host (the reference has no Poisson solver)"},
        "cpu_baseline": dict(cb, value=value),
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference(args, spec, name):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if spec["kind"] == "poisson":
        return run_reference_poisson(args, spec, name)
    if spec["kind"] == "jacobi":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no Jacobi "
                          "sweep with a right-hand side (its 3D golds are operator sweeps)"}),
              flush=True)
        return
    if spec["kind"] == "cnn":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no network "
                          "(the warm start is new work with no reference code)"}), flush=True)
        return
    n_steps = args.steps + args.warmup
    # every step times a sample of at least 0.1 s (the whole default run of
    # 2020 steps about 3.5 minutes); the line's value is the median rate
    budget = max(0.1, min(10.0, 150.0 / max(1, n_steps)))
    rates = []
    sample = cores = cpu_kind = None
    for i in range(n_steps):
        if spec["kind"] == "batched":
            cb = batched_cpu_baseline(spec, batch_sides(spec), budget)
            rate, sample, cores, cpu_kind = cb["value"], cb["sample"], cb["cores"], cb["kind"]
        else:
            rate, sample, cores, cpu_kind = cpu_reference_rate(spec, budget, seed=i)
        if i >= args.warmup:
            rates.append(rate)
    value = statistics.median(rates) if rates else None
    nd = 3 if spec["kind"] == "3d" else 2
    cells = spec["n"] ** nd * spec["steps"]
    if spec["kind"] == "batched":
        cells = int(sum(int(h) * int(w_) for h, w_ in batch_sides(spec))) * spec["steps"]
    line = {
        "impl": "reference", "metric": "GCells/s", "value": value, "unit": "GCells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": (cells / (value * 1e9) * 1e3) if value else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": spec["dtype"], "data": "synthetic (seeded uniform[-1,1))",
        "config": dict(workload=name, grid="x".join([str(spec["n"])] * nd), kind=spec["kind"],
                       radius=spec["r"], steps_per_call=spec["steps"],
                       boundary=spec["boundary"]),
        "cpu_baseline": {"value": value, "unit": "GCells/s", "cores": cores,
                         "cpu_model": cpu_model(), "kind": cpu_kind,
                         "sample": f"per step: {sample}"},
        "e2e": {"value": value, "unit": "GCells/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm --

def batch_sides(spec, seed=256):
    g = np.random.Generator(np.random.PCG64(seed))
    return np.exp(g.uniform(np.log(64), np.log(2048), size=(spec["ngrids"], 2))).astype(int)


def run_batched(args, spec, name):
    """256 uneven grids, `steps` steps each: one persistent launch per call
    (value) against one launch chain per grid (reported beside it)."""
    import torch
    import ssam_b200 as S
    from ssam_b200 import shard
    r = shard.ranks()
    rank, world, local = r.rank, r.world, r.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shard.init("nccl", 300, dev)
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}[spec["dtype"]]
    sides = batch_sides(spec)
    gen = torch.Generator(device=dev)
    gen.manual_seed(2000 + rank)
    # pitched rows (a multiple of 128 bytes), the layout cudaMallocPitch gives
    # and the reference's conv driver uses (DevData, cudaMalloc3D)
    es_ = elem_size(spec["dtype"])
    def pitched(h, w_):
        pitch = -(-int(w_) * es_ // 128) * 128 // es_
        base = torch.empty(int(h), pitch, device=dev, dtype=tdt)
        return base[:, :int(w_)]
    srcs = []
    for h, w_ in sides:
        x = pitched(h, w_)
        x.copy_(torch.rand(int(h), int(w_), device=dev, generator=gen).to(tdt))
        srcs.append(x)
    dsts = [pitched(x.shape[0], x.shape[1]) for x in srcs]
    c = coefficients(spec)
    r = spec["r"]
    shape = S.STAR if spec["shape"] == "star" else S.BOX
    stream = torch.cuda.current_stream(dev)
    cells = int(sum(int(h) * int(w_) for h, w_ in sides))

    def call(persistent):
        S.stencil2d_batched(srcs, c, r, shape, spec["steps"], spec["boundary"], dsts=dsts,
                            persistent=persistent, stream=stream)

    def timed(persistent, k):
        for _ in range(args.warmup):
            call(persistent)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        l0 = S.lib().ssam_kernel_launches()
        a.record(stream)
        for _ in range(k):
            call(persistent)
        b.record(stream)
        l1 = S.lib().ssam_kernel_launches()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k, (l1 - l0) // k

    clocks = ClockSampler(local)
    shard.barrier()
    clocks.start()
    ms, launches = timed(True, args.steps)
    clk = clocks.stop()
    ms = shard.max_over_ranks(ms, dev)
    ms_pg, launches_pg = timed(False, max(1, min(args.steps, 3)))
    value = cells * spec["steps"] * world / (ms / 1e3) / 1e9
    es = elem_size(spec["dtype"])
    # phases of the persistent run: fused depth 4 (r=1) / 2 (r=2), rest single
    # steps; single steps throughout with a COPY or CLAMP boundary
    deep = 4 if r == 1 else (2 if r == 2 else 1)
    if spec["boundary"] in ("copy", "clamp"):
        deep = 1
    phases = spec["steps"] // deep + spec["steps"] % deep
    alg_bytes = 2 * cells * es * phases
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (ms / 1e3) / 1e9
    # end to end: every grid copied in from pinned host memory and back, per call
    hs = [torch.empty_strided(x.shape, x.stride(), dtype=x.dtype).pin_memory() for x in srcs]
    for h_, x in zip(hs, srcs):
        h_.copy_(x)
    ho = [torch.empty_strided(x.shape, x.stride(), dtype=x.dtype).pin_memory() for x in srcs]
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    k_e2e = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(k_e2e):
        for d_, h_ in zip(srcs, hs):
            d_.copy_(h_, non_blocking=True)
        call(True)
        for h_, d_ in zip(ho, dsts):
            h_.copy_(d_, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    e_ms = a.elapsed_time(b) / k_e2e
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = batched_cpu_baseline(spec, sides)
    if rank == 0:
        print(json.dumps({
            "metric": "GCells/s", "value": value, "unit": "GCells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": spec["dtype"], "data": "synthetic (seeded uniform[0,1))",
            "config": {"workload": name, "grids": spec["ngrids"], "cells": cells,
                       "sides": "log-uniform [64, 2048], seed 256; rows pitched to 128 B",
                       "kind": spec["shape"],
                       "radius": r, "steps_per_call": spec["steps"],
                       "boundary": spec["boundary"], "parallelism": f"dp{world}",
                       "l2": f"{2 * cells * es / 2**20:.0f} MiB in+out per pass vs 126 MB L2"},
            "gpu_launches": launches * args.steps,
            "per_grid_baseline": {"ms_per_step": ms_pg, "launches_per_step": launches_pg,
                                  "value": cells * spec["steps"] / (ms_pg / 1e3) / 1e9,
                                  "speedup_of_persistent": ms_pg / ms},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": load_traffic(name),
                         "algorithmic_bytes_per_launch": alg_bytes / max(1, launches)},
            "clocks": clk,
            "e2e": {"value": cells * spec["steps"] / (e_ms / 1e3) / 1e9, "unit": "GCells/s",
                    "h2d_bytes_per_step": cells * es, "d2h_bytes_per_step": cells * es,
                    "steps": k_e2e},
            "cpu_baseline": cpu,
        }), flush=True)
    shard.finish()


def batched_cpu_baseline(spec, sides, budget_s=10.0):
    """Reference Convolution<float> per grid, looped like the reference would
    run one grid per invocation, on the host cores (the oracle's restatement
    of it when oracle/_ref is not built: kind "port")."""
    import oracle
    use_ref = oracle.have_ref()
    g = np.random.Generator(np.random.PCG64(3))
    c = coefficients(spec)
    r = spec["r"]
    if spec["shape"] == "star":
        m = np.zeros((2 * r + 1, 2 * r + 1))
        m[r, r] = c[0]
        for k in range(1, r + 1):
            m[r - k, r], m[r + k, r], m[r, r - k], m[r, r + k] = c[1 + 4 * (k - 1): 5 + 4 * (k - 1)]
    else:
        m = np.array(c).reshape(2 * r + 1, 2 * r + 1)
    m = m.astype(np.float32)
    t0 = time.perf_counter()
    cells = 0
    for h, w_ in sides:
        x = g.random((int(h), int(w_)), dtype=np.float32)
        for _ in range(spec["steps"]):
            x = oracle.ref_convolution(x, m) if use_ref else oracle.conv2d(x, m, "zero")
        cells += int(h) * int(w_) * spec["steps"]
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    cores = host_threads()
    return {"value": cells / el / 1e9, "unit": "GCells/s", "cores": cores,
            "cpu_model": cpu_model(), "kind": "reference" if use_ref else "port",
            "sample": f"{cells // spec['steps']} cells of the batch x {spec['steps']} steps"}


def run_poisson(args, spec, name):
    """One step = one complete solve of the 8 right-hand sides to 1e-5
    relative residual from u = 0.  `value` is seconds per solve (device
    events around the solve; the solve itself reads FP64 residual norms on
    the host between corrections)."""
    import torch

    import ssam_b200 as S
    from ssam_b200 import shard
    from ssam_b200.workloads import gaussian_rhs_torch

    r = shard.ranks()
    rank, world, local = r.rank, r.world, r.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shard.init("nccl", 300, dev)
    n, nb, tol = spec["n"], spec["nb"], spec["tol"]
    f = gaussian_rhs_torch(nb, n, 7 + rank, dev)
    stream = torch.cuda.current_stream(dev)
    net = None
    opts = dict(POISSON_ARMS[spec["arm"]])
    if spec["arm"] == "learned":
        net = S.WarmStartCNN(n, nb)
        net.load(CNN_WEIGHTS)
        opts["cnn"] = net
    u = torch.zeros_like(f)
    # the autotuner picks the sweep kernel's tile and ring for this batch size
    # (both sweep precisions: the learned arm's line also times the plain arm)
    tuned = None
    if not args.no_autotune:
        tuned = {dt: S.autotune_jacobi3d(n, nb, dt, dev, stream) for dt in ("f32", "bf16")}

    def solve(o):
        u.zero_()
        return S.poisson_solve(f, u, tol=tol, max_sweeps=400000, stream=stream, **o)

    for _ in range(args.warmup):
        solve(opts)
    torch.cuda.synchronize()
    shard.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    times, stats = [], []
    launches0 = S.lib().ssam_kernel_launches()
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st = solve(opts)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / 1e3)
        stats.append(st)
    launches = S.lib().ssam_kernel_launches() - launches0
    clk = clocks.stop()
    sec = shard.max_over_ranks(sum(times) / len(times), dev)
    # FP64 check of the last answer by the library's residual (the tests
    # check that residual against the oracle's)
    check_gpu = max(S.poisson_residual(f, u))
    f_np = f.cpu().numpy()

    # the other arm on the same GPU and inputs, for the ratio
    other = {}
    plain_st = stats[-1]
    if spec["arm"] == "learned":
        ts = []
        for _ in range(2):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            plain_st = solve(POISSON_ARMS["plain"])
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) / 1e3)
        other = {"plain_s": min(ts), "plain_sweeps": plain_st["sweeps"],
                 "speedup_vs_plain": min(ts) / sec}
    # pure FP32 Jacobi from zero (no FP64 correction): the residual it stalls at
    plateau = None
    if spec["arm"] == "plain" and rank == 0:
        rhs32 = f.float()
        ua = torch.zeros_like(rhs32)
        ub = torch.empty_like(rhs32)
        best = 1.0
        for _ in range(30):
            S.poisson_jacobi(rhs32, ua, 2000, u_out=ub, stream=stream)
            ua, ub = ub, ua
            best = min(best, max(S.poisson_residual(f, ua.double())))
        plateau = {"sweeps": 60000, "min_rel_residual": best}

    # roofline of the dominant kernels
    peak, peak_kind = load_peaks()
    sweep_dt = opts["sweep_dtype"]
    tdt = torch.float32 if sweep_dt == "f32" else torch.bfloat16
    es = 4 if sweep_dt == "f32" else 2
    rhs_lp = f.to(tdt)
    ua = torch.zeros_like(rhs_lp)
    ub = torch.empty_like(rhs_lp)
    S.poisson_jacobi(rhs_lp, ua, 20, u_out=ub, stream=stream)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    S.poisson_jacobi(rhs_lp, ua, 200, u_out=ub, stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    sweep_ms = a.elapsed_time(b) / 200
    sweep_bytes = 3 * f.numel() * es  # u read, rhs read, u write
    roof = {"bound": "hbm", "kernel": f"Jacobi sweep ({sweep_dt} storage)",
            "achieved": sweep_bytes / (sweep_ms / 1e3) / 1e9, "peak": peak,
            "unit": "GB/s", "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": sweep_bytes, "us_per_sweep": sweep_ms * 1e3,
            "traffic": load_traffic(f"jacobi_{sweep_dt}_128x8")}
    roof["frac"] = roof["achieved"] / peak
    if net is not None:
        net.forward(f)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(10):
            net.forward(f)
        b.record(stream)
        torch.cuda.synchronize()
        fwd_ms = a.elapsed_time(b) / 10
        flops = cnn_forward_flops(n, nb)
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                tpeak, tsrc = float(json.load(fh)["bf16_tflops"]), "measured"
        except Exception:
            tpeak, tsrc = 1590.0, "fallback"
        cnn = {"bound": "tensor", "kernel": "CNN forward (13 convolutions + glue)",
               "achieved": flops / (fwd_ms / 1e3) / 1e12, "peak": tpeak,
               "unit": "TFLOP/s", "peak_source": tsrc, "ms_per_forward": fwd_ms,
               "flops_per_forward": flops}
        cnn["frac"] = cnn["achieved"] / tpeak
        roof["cnn"] = cnn

    # end to end: f from pinned host memory, the solve, u back to the host
    hf = f.cpu().pin_memory()
    hu = torch.empty_like(hf).pin_memory()
    k_e2e = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(k_e2e):
        f.copy_(hf, non_blocking=True)
        u.zero_()
        S.poisson_solve(f, u, tol=tol, max_sweeps=400000, stream=stream, **opts)
        hu.copy_(u, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_s = a.elapsed_time(b) / 1e3 / k_e2e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = poisson_cpu_baseline(f_np, plain_st["sweeps"])
    if rank == 0:
        st = stats[-1]
        print(json.dumps({
            "metric": "Poisson time-to-1e-5 relative residual", "value": sec, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": f"f64 residual/correction, {sweep_dt} sweeps"
            + (", bf16 CNN" if net is not None else ""),
            "data": "synthetic (8 Gaussian-bump right-hand sides, seed 7)",
            "config": {"workload": name, "grid": f"{nb}x{n}^3", "tol": tol, "tuned": tuned,
                       "arm": spec["arm"], **{k: v for k, v in opts.items() if k != "cnn"},
                       "weights": os.path.relpath(CNN_WEIGHTS, ROOT) if net else None,
                       "parallelism": f"dp{world} (independent right-hand sides per GPU)",
                       "l2": f"u, f, r: {3 * f.numel() * 8 / 2**20:.0f} MiB FP64 vs 126 MB L2"},
            "solve": {**st, "check_rel_residual_fp64_gpu": check_gpu,
                      "times_s": times, **other},
            "fp32_jacobi_plateau": plateau,
            "gpu_launches": launches,
            "roofline": roof,
            "clocks": clk,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": f.numel() * 8,
                    "d2h_bytes_per_step": f.numel() * 8, "steps": k_e2e},
            "cpu_baseline": cpu,
        }), flush=True)
    if net is not None:
        net.close()
    shard.finish()


def cnn_forward_flops(n, nb):
    """3x3x3 16 -> 16 convolutions of the network: 2 * 27 * 16 * 16 flop per
    voxel and source; 5 source-layers at n, 5 at n/2, 4 at n/4."""
    return 2 * 27 * 16 * 16 * (5 * n ** 3 + 5 * (n // 2) ** 3 + 4 * (n // 4) ** 3) * nb


def run_cnn(args, spec, name):
    """One step = one forward pass of the warm-start network over 8 right-hand
    sides at 128^3 (input FP64 f, output FP64 u0)."""
    import torch

    import ssam_b200 as S
    from ssam_b200 import shard
    from ssam_b200.workloads import gaussian_rhs_torch
    r = shard.ranks()
    rank, world, local = r.rank, r.world, r.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shard.init("nccl", 120, dev)
    n, nb = spec["n"], spec["nb"]
    f = gaussian_rhs_torch(nb, n, 7 + rank, dev)
    net = S.WarmStartCNN(n, nb)
    net.load(CNN_WEIGHTS)
    out = torch.empty_like(f)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        net.forward(f, out)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    l0 = S.lib().ssam_kernel_launches()
    a.record(stream)
    for _ in range(args.steps):
        net.forward(f, out)
    b.record(stream)
    launches = S.lib().ssam_kernel_launches() - l0
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = shard.max_over_ranks(a.elapsed_time(b) / args.steps, dev)
    flops = cnn_forward_flops(n, nb)
    value = flops / (ms / 1e3) / 1e12 * world
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            tpeak, tsrc = float(json.load(fh)["bf16_tflops"]), "measured"
    except Exception:
        tpeak, tsrc = 1590.0, "fallback"
    hf = f.cpu().pin_memory()
    hu = torch.empty_like(hf).pin_memory()
    k = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(k):
        f.copy_(hf, non_blocking=True)
        net.forward(f, out)
        hu.copy_(out, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    e_ms = a.elapsed_time(b) / k
    if rank == 0:
        print(json.dumps({
            "metric": "CNN forward TFLOP/s", "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (8 Gaussian-bump right-hand sides, seed 7)",
            "config": {"workload": name, "grid": f"{nb}x{n}^3", "channels": 16,
                       "weights": os.path.relpath(CNN_WEIGHTS, ROOT),
                       "l2": "activations 8 x 128^3 x 16 BF16 = 512 MiB per buffer vs 126 MB L2"},
            "gpu_launches": launches,
            "roofline": {"bound": "tensor", "achieved": value / world, "peak": tpeak,
                         "unit": "TFLOP/s", "frac": value / world / tpeak, "peak_source": tsrc,
                         "traffic": None, "flops_per_forward": flops},
            "clocks": clk,
            "e2e": {"value": flops / (e_ms / 1e3) / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": f.numel() * 8, "d2h_bytes_per_step": f.numel() * 8,
                    "steps": k},
            "cpu_baseline": None,
        }), flush=True)
    net.close()
    shard.finish()


def run_jacobi(args, spec, name):
    """One step = `steps` Jacobi sweeps of -lap(u) = f on nb x n^3 in the
    sweep storage type (the kernel both Poisson arms spend their sweeps in)."""
    import torch

    import ssam_b200 as S
    from ssam_b200 import shard
    from ssam_b200.workloads import gaussian_rhs_torch
    r = shard.ranks()
    rank, world, local = r.rank, r.world, r.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shard.init("nccl", 120, dev)
    n, nb, k = spec["n"], spec["nb"], spec["steps"]
    tdt = torch.float32 if spec["dtype"] == "f32" else torch.bfloat16
    es = 4 if spec["dtype"] == "f32" else 2
    rhs = gaussian_rhs_torch(nb, n, 7 + rank, dev).to(tdt)
    u0 = torch.zeros_like(rhs)
    out = torch.empty_like(rhs)
    stream = torch.cuda.current_stream(dev)
    tuned = None if args.no_autotune else S.autotune_jacobi3d(n, nb, spec["dtype"], dev, stream)
    for _ in range(args.warmup):
        S.poisson_jacobi(rhs, u0, k, u_out=out, stream=stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    l0 = S.lib().ssam_kernel_launches()
    a.record(stream)
    for _ in range(args.steps):
        S.poisson_jacobi(rhs, u0, k, u_out=out, stream=stream)
    b.record(stream)
    launches = S.lib().ssam_kernel_launches() - l0
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = shard.max_over_ranks(a.elapsed_time(b) / args.steps, dev)
    cells = nb * n ** 3
    peak, peak_kind = load_peaks()
    achieved = 3 * cells * es * k / (ms / 1e3) / 1e9  # u read, rhs read, u write per sweep
    if rank == 0:
        print(json.dumps({
            "metric": "GCells/s", "value": cells * k * world / (ms / 1e3) / 1e9,
            "unit": "GCells/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": spec["dtype"], "data": "synthetic (8 Gaussian-bump right-hand sides)",
            "config": {"workload": name, "grid": f"{nb}x{n}^3", "sweeps_per_step": k,
                       "tuned": tuned,
                       "l2": f"u in/out + rhs: {3 * cells * es / 2**20:.0f} MiB vs 126 MB L2"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": load_traffic(name),
                         "algorithmic_bytes_per_launch": 3 * cells * es},
            "clocks": clk, "e2e": None, "cpu_baseline": None,
        }), flush=True)
    shard.finish()


def run_ssam(args, spec, name):
    import torch

    import ssam_b200 as S
    from ssam_b200 import shard

    r = shard.ranks()
    rank, world, local = r.rank, r.world, r.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shard.init("nccl", 120, dev)

    n = spec["n"]
    kind = spec["kind"]
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}[spec["dtype"]]
    gen = torch.Generator(device=dev)
    gen.manual_seed(1000 + rank)
    dims = (n, n, n) if kind == "3d" else (n, n)
    lo = 0.0 if kind == "3d" else -1.0  # 3D: uniform[0,1); 2D: uniform[-1,1)
    # alternating inputs: enough of them that one rotation is at least twice
    # the 126 MB L2, so every step reads its input from HBM
    grid_bytes = n ** len(dims) * elem_size(spec["dtype"])
    nsrc = max(2, -(-2 * 126 * 10**6 // grid_bytes))
    srcs = [(torch.rand(*dims, device=dev, dtype=torch.float32, generator=gen) * (1 - lo)
             + lo).to(tdt) for _ in range(nsrc)]
    dst = torch.empty_like(srcs[0])
    c = coefficients(spec)
    r = spec["r"]
    shape = S.STAR if kind == "star" else S.BOX
    stream = torch.cuda.current_stream(dev)

    if kind == "conv":
        w = np.array(c).reshape(spec["f"], spec["f"])

        def step(i, s=stream):
            S.conv2d(srcs[i % nsrc], w, boundary=spec["boundary"], dst=dst, stream=s)
    elif kind == "3d":
        shape = S.POISSON19 if spec["gold"] == "poisson" else S.STAR3D

        def step(i, s=stream):
            S.stencil3d(srcs[i % nsrc], c, r, shape, steps=spec["steps"],
                        boundary=spec["boundary"], dst=dst, stream=s)
    else:
        def step(i, s=stream):
            S.stencil2d(srcs[i % nsrc], c, r, shape, steps=spec["steps"],
                        boundary=spec["boundary"], dst=dst, stream=s)

    barrier = shard.barrier

    # the project's autotuner picks P, strip width, warps and temporal depth
    # for this stencil and grid size (outside the timed region)
    tuned = None
    if not args.no_autotune and kind == "3d":
        # the 3D autotuner picks rows per warp, consumer warps and ring depth
        tuned = S.autotune_stencil3d(srcs[0], c, r, shape, boundary=spec["boundary"], dst=dst,
                                     stream=stream)
    if not args.no_autotune and kind in ("box", "star") or (kind == "conv" and spec["f"] % 2):
        coeffs_for_tune = list(np.ravel(c)) if kind != "conv" else list(w.ravel())
        tune_shape = shape if kind != "conv" else S.BOX
        if not args.no_autotune:
            tuned = S.autotune_stencil2d(srcs[0], coeffs_for_tune, r, tune_shape,
                                         steps=spec["steps"], boundary=spec["boundary"],
                                         dst=dst, stream=stream)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()

    # single-step 2D runs: the K timed calls are captured once into a CUDA
    # graph and replayed, so that host-side call overhead does not open gaps
    # between kernels of ~25-100 us (the library's own calls are what is
    # captured; the launch counter counts them at capture)
    graph = None
    if kind in ("box", "star", "conv") and spec["steps"] == 1:
        graph = torch.cuda.CUDAGraph()
        l0 = S.lib().ssam_kernel_launches()
        with torch.cuda.graph(graph):
            cs = torch.cuda.current_stream(dev)
            for i in range(args.steps):
                step(i, cs)
        graph_launches = S.lib().ssam_kernel_launches() - l0
        graph.replay()  # untimed first replay
        torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = S.lib().ssam_kernel_launches()
    t_start.record(stream)
    if graph is not None:
        graph.replay()
    else:
        for i in range(args.steps):
            ev[i][0].record(stream)
            step(i)
            ev[i][1].record(stream)
    t_end.record(stream)
    launches = S.lib().ssam_kernel_launches() - launches0
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    if graph is not None:
        launches = graph_launches
        avg_launch_ms = total_ms / max(1, launches)
    else:
        launch_ms = [a.elapsed_time(b) for a, b in ev]
        avg_launch_ms = sum(launch_ms) / len(launch_ms)
    total_ms = shard.max_over_ranks(total_ms, dev)

    cells = n ** len(dims) * spec["steps"]
    value = cells * args.steps * world / (total_ms / 1e3) / 1e9
    es = elem_size(spec["dtype"])
    # launches per call: one per chained temporal block (counted by the library)
    launches_per_step = max(1, launches // args.steps)
    peak, peak_kind = load_peaks()
    # algorithmic bytes of one call: read + write each cell once per launch
    alg_bytes = 2 * n ** len(dims) * es * launches_per_step
    achieved = alg_bytes / (avg_launch_ms / 1e3) / 1e9
    traffic = load_traffic(name)
    # the binding roof of one launch: HBM (bytes above) or the FP32 / FP64
    # FMA pipes, 2*taps-1 flop per cell and fused step; the FMA peak is the
    # nominal SM count x FMA lanes x 2 x maximum SM clock (no measured figure
    # exists for the non-tensor pipes)
    per_launch_s = avg_launch_ms / 1e3 / (1 if graph is not None else launches_per_step)
    flops_per_launch = ((2 * taps(spec) - 1) * n ** len(dims) * spec["steps"]
                        / launches_per_step)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    max_mhz = (clk or {}).get("sm_max_mhz") or 1965.0
    fma_lanes = 64 if spec["dtype"] == "f64" else 128
    fma_peak = sms * fma_lanes * 2 * max_mhz * 1e6 / 1e12  # TFLOP/s
    fma_bound = flops_per_launch / (fma_peak * 1e12) > (alg_bytes / launches_per_step) / (peak * 1e9)
    fma_achieved = flops_per_launch / per_launch_s / 1e12

    # reduced-precision runs: max / RMS error of the last call's result
    # against the same call in FP64 on the same stored inputs (the FP64
    # kernels match the CPU oracle to 1e-12 in the tests), outside the timed
    # region
    err = None
    if spec["dtype"] != "f64":
        i_last = (args.steps - 1) % nsrc
        x64 = srcs[i_last].double()
        if kind == "3d":
            ref = S.stencil3d(x64, c, r, shape, steps=spec["steps"],
                              boundary=spec["boundary"], stream=stream)
        elif kind == "conv":
            ref = S.conv2d(x64, w, boundary=spec["boundary"], stream=stream)
        else:
            ref = S.stencil2d(x64, c, r, shape, steps=spec["steps"],
                              boundary=spec["boundary"], stream=stream)
        d = dst.double() - ref
        err = {"max_abs": d.abs().max().item(), "rms": d.pow(2).mean().sqrt().item(),
               "max_rel_to_range": (d.abs().max() / ref.abs().max()).item(),
               "reference": "the same call in FP64 on the GPU on the same stored inputs "
                            "(FP64 kernels = CPU oracle to 1e-12 in tests/)"}
        del ref, d, x64

    # end to end: host buffers through ssam_stencil2d_host, copies timed
    e2e = None
    if kind != "conv":
        host_call = S.stencil3d_host if kind == "3d" else S.stencil2d_host
        k_e2e = max(3, min(args.steps, 20))
        hs = srcs[0].cpu().pin_memory()
        hd = torch.empty_like(hs).pin_memory()
        for _ in range(2):
            host_call(hs, hd, c, r, shape, spec["steps"], spec["boundary"], dev, stream)
        torch.cuda.synchronize()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k_e2e):
            host_call(hs, hd, c, r, shape, spec["steps"], spec["boundary"], dev, stream)
        b.record(stream)
        torch.cuda.synchronize()
        e_ms = shard.max_over_ranks(a.elapsed_time(b), dev)
        e2e = {"value": cells * k_e2e * world / (e_ms / 1e3) / 1e9, "unit": "GCells/s",
               "h2d_bytes_per_step": n ** len(dims) * es,
               "d2h_bytes_per_step": n ** len(dims) * es,
               "steps": k_e2e}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, sample, cores, cpu_kind = cpu_reference_rate(spec, budget_s=10.0)
            cpu = {"value": rate, "unit": "GCells/s", "cores": cores, "kind": cpu_kind,
                   "cpu_model": cpu_model(), "sample": sample}
        except Exception as exc:  # the GPU number stands without it
            cpu = {"value": None, "unit": "GCells/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": "GCells/s", "value": value, "unit": "GCells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": spec["dtype"],
            "data": "synthetic (seeded uniform[-1,1), coefficients uniform[0,1) normalised)",
            "config": {"workload": name, "grid": "x".join([str(n)] * len(dims)), "kind": kind,
                       "radius": r,
                       "taps": taps(spec), "steps_per_call": spec["steps"],
                       "boundary": spec["boundary"],
                       "l2": f"inputs rotate through {nsrc} grids of "
                             f"{n ** len(dims) * es / 2**20:.0f} MiB (>= 2x the 126 MB L2)",
                       "parallelism": f"dp{world} (independent grid per GPU)",
                       "timed_as": "one CUDA graph of the K calls" if graph is not None
                                   else "K calls",
                       "tuned": tuned},
            "gpu_launches": launches,
            "roofline": ({"bound": "fma", "achieved": fma_achieved, "peak": fma_peak,
                          "unit": "TFLOP/s", "frac": fma_achieved / fma_peak,
                          "peak_source": f"nominal: {sms} SMs x {fma_lanes} FMA lanes x 2 x "
                                         f"{max_mhz:.0f} MHz",
                          "traffic": traffic,
                          "algorithmic_flops_per_launch": flops_per_launch,
                          "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s",
                                  "frac": achieved / peak, "peak_source": peak_kind}}
                         if fma_bound else
                         {"bound": "hbm", "achieved": achieved, "peak": peak,
                          "unit": "GB/s", "frac": achieved / peak,
                          "peak_source": peak_kind,
                          "traffic": traffic,
                          "algorithmic_bytes_per_launch": alg_bytes / launches_per_step,
                          "fma": {"achieved": fma_achieved, "peak": fma_peak,
                                  "unit": "TFLOP/s", "frac": fma_achieved / fma_peak}}),
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        if err is not None:
            line["error_vs_fp64"] = err
        print(json.dumps(line), flush=True)
    shard.finish()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ssam", choices=["ssam", "reference"])
    ap.add_argument("--workload", default=DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuned", default=None, metavar="FILE",
                    help="load launch choices from a tune-cache file (ssam_autotune_save "
                         "format) instead of measuring them")
    ap.add_argument("--save-tuned", default=None, metavar="FILE",
                    help="save the launch choices this run made (to replay them with --tuned)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the built-in launch defaults instead of measuring")
    args = ap.parse_args(argv)
    if args.tuned:
        import ssam_b200 as S
        S.autotune_load(args.tuned)
        args.no_autotune = True  # replay the loaded choices, measure nothing
    wl = workloads()
    if args.workload not in wl:
        raise SystemExit(f"unknown workload {args.workload}; known: {sorted(wl)}")
    spec = wl[args.workload]
    if args.impl == "reference":
        run_reference(args, spec, args.workload)
    elif spec["kind"] == "batched":
        run_batched(args, spec, args.workload)
    elif spec["kind"] == "poisson":
        run_poisson(args, spec, args.workload)
    elif spec["kind"] == "cnn":
        run_cnn(args, spec, args.workload)
    elif spec["kind"] == "jacobi":
        run_jacobi(args, spec, args.workload)
    else:
        run_ssam(args, spec, args.workload)
    if args.save_tuned and args.impl != "reference":
        import ssam_b200 as S
        S.autotune_save(args.save_tuned)


if __name__ == "__main__":
    main()
