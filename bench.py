"""Benchmark: SHT round trips/s at T511 x 64 layers (OctahedralGaussianGrid, nlat = 768).

One step = one spherical harmonic transform round trip (spectral -> grid synthesis,
then grid -> spectral analysis) of 64 layers, inputs resident in HBM. With --gpus N
(one process per GPU under torchrun) every rank runs its own replica of the
workload (the transform does not shard; weak scaling) and the job's value is the
total round trips of all ranks divided by the slowest rank's time.

Reports the headline precision (the fastest Legendre arithmetic whose synthesis and
round trip stay within 1e-5 relative error of the FP64 oracle on every one of the 64
layers) and every variant, the
roofline of the dominant kernel, an end-to-end number through the public API with
host buffers (coefficients in page-locked host memory, copied in and out inside the
transforms, overlapped with the work over chunks of 16 layers; consecutive steps
pipelined), clocks sampled during the timed region, and the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "speedyweather.jl_b200"))

METRIC = "SHT round-trips/s at T511×64 layers, split-BF16 vs FP32 at ≤1e-5 rel err"
UNIT = "round_trips/s"
T, NLAT_HALF, LAYERS = 512, 384, 64     # T511: 1-based truncation 512, nlat = 768
ERR_BAR = 1e-5


def config(world=1):
    """The workload's description; the same dict in both arms (precision is the line's dtype)."""
    c = {"workload": "T511 OctahedralGaussianGrid nlat=768 x 64 layers, spectral->grid->spectral round trip",
         "grid": "OctahedralGaussianGrid", "truncation": "T511 (lmax=mmax=512)", "nlat": 2 * NLAT_HALF,
         "layers": LAYERS, "legendre_shortcut": "linear",
         "l2": "inputs larger than L2 (grid 154.5 MB, coefficients 67 MB, Legendre table 160 MB per pass)"}
    c["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
    return c


# ----------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # the timed region starts once the sampler has written its first line (or after 5 s)
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.05)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------------------
# multi-rank plumbing (replicas; no data-path collective)
# ----------------------------------------------------------------------------------------
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def reduce_max(value, world, device):
    """Max over ranks of a float (the slowest replica defines the job's time)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def broadcast_choice(obj, world):
    """Rank 0's value on every rank (the headline precision: all ranks time the same one)."""
    if world == 1:
        return obj
    import torch.distributed as dist
    box = [obj]
    dist.broadcast_object_list(box, src=0)
    return box[0]


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of each kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ----------------------------------------------------------------------------------------
# reference arm: the reference's CPU algorithm (C restatement) on the host cores
# ----------------------------------------------------------------------------------------
def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    from sht_cpu import CpuTransform, max_threads
    # each step: one round trip of all 64 layers (about 1 s on 16 host threads); only when
    # the K + W steps would take longer than --ref-seconds is a step cut to fewer layers
    # (a bounded sample, scaled to 64 layers), the per-step size set by a calibration trip
    cp = CpuTransform(1, NLAT_HALF, T, T, LAYERS)
    c = O.random_coeffs(O.Spectrum(T, T), LAYERS, seed=0).T.astype(np.complex64)
    g = np.empty((LAYERS, cp.npoints), np.float32)
    a = np.empty((LAYERS, cp.nlm), np.complex64)
    t0 = time.perf_counter()
    cp.synthesize(c, g)
    cp.analyze(g, a)
    per_step = time.perf_counter() - t0
    sample = LAYERS
    if per_step * (args.steps + args.warmup) > args.ref_seconds:
        sample = int(max(1, LAYERS * args.ref_seconds / ((args.steps + args.warmup) * per_step)))
        cp = CpuTransform(1, NLAT_HALF, T, T, sample)
        c, g, a = np.ascontiguousarray(c[:sample]), g[:sample], a[:sample]
    for _ in range(args.warmup):
        cp.synthesize(c, g)
        cp.analyze(g, a)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cp.synthesize(c, g)
        cp.analyze(g, a)
    dt = (time.perf_counter() - t0) / args.steps
    value = (sample / LAYERS) / dt
    cores = max_threads()
    what = ("one round trip of all 64 layers" if sample == LAYERS
            else f"one round trip of {sample} of the 64 layers, scaled to 64 layers")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": config(world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"each step: {what} at T511 (C restatement of SpeedyTransforms' CPU "
                                       f"loops, FP32, {cores} threads)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline(seconds):
    """The C restatement timed on all host threads over whole 64-layer round trips (the
    benchmark's own workload), as many as fit in `seconds` (at least two)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    from sht_cpu import CpuTransform, max_threads
    cp = CpuTransform(1, NLAT_HALF, T, T, LAYERS)
    c = O.random_coeffs(O.Spectrum(T, T), LAYERS, seed=0).T.astype(np.complex64)
    g = np.empty((LAYERS, cp.npoints), np.float32)
    a = np.empty((LAYERS, cp.nlm), np.complex64)
    cp.synthesize(c, g)
    n, t0 = 0, time.perf_counter()
    while True:
        cp.synthesize(c, g)
        cp.analyze(g, a)
        n += 1
        if n >= 2 and time.perf_counter() - t0 > seconds:
            break
    dt = (time.perf_counter() - t0) / n
    return {"value": 1.0 / dt, "unit": UNIT, "cores": max_threads(), "kind": "port",
            "sample": f"{n} round trips of all 64 layers at T511, C restatement of the reference's CPU "
                      "loops (FP32)"}


# ----------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------
def algorithmic(S):
    """Algorithmic bytes / flops per launch of each kernel at LAYERS layers."""
    sp = S.spectrum
    mt = S.mmax_truncation.astype(np.int64)
    lam_elems = int(sum(int((sp.lmax - np.arange(t + 1)).sum()) for t in mt))
    rows = int((mt + 1).sum())
    K = LAYERS
    lam_b = 4 * lam_elems
    coeff_b = sp.nlm * K * 8
    scratch_b = rows * 2 * K * 8
    grid_b = S.grid.npoints * K * 4
    return {
        "legendre_synthesis": {"bytes": lam_b + coeff_b + scratch_b, "flops": 4 * K * lam_elems},
        "fourier_synthesis": {"bytes": scratch_b + grid_b},
        "fourier_analysis": {"bytes": grid_b + scratch_b},
        "legendre_analysis": {"bytes": lam_b + scratch_b + coeff_b, "flops": 4 * K * lam_elems},
        "_lam_elems": lam_elems, "_rows": rows,
    }


def time_stages(S, lt, field, out, reps):
    """Per-kernel CUDA-event timing on the launching stream (outside the timed region)."""
    import torch
    from speedytransforms import _lib
    L = _lib.lib
    st = torch.cuda.current_stream()
    sp = st.cuda_stream
    h = S.handle
    nlm, npts = S.spectrum.nlm, S.grid.npoints
    stages = {
        "legendre_synthesis": lambda: L.sht_legendre_synthesis(h, lt.data.data_ptr(), nlm, LAYERS, sp),
        "fourier_synthesis": lambda: L.sht_fourier_synthesis(h, field.data.data_ptr(), npts, LAYERS, 0, sp),
        "fourier_analysis": lambda: L.sht_fourier_analysis(h, field.data.data_ptr(), npts, LAYERS, sp),
        "legendre_analysis": lambda: L.sht_legendre_analysis(h, out.data.data_ptr(), nlm, LAYERS, 0, sp),
    }
    res = {}
    for name, fn in stages.items():
        for _ in range(3):
            _lib.check(fn())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps
    return res


MIX = [(32, 24, 1), (64, 48, 8), (128, 96, 16), (256, 192, 64)]   # (T + 1, nlat_half, layers)


def run_mixed_batch(args):
    """The batching workload: octahedral T31 / T63 / T127 / T255 (nlat 48 / 96 / 192 / 384)
    with 1 / 8 / 16 / 64 layers, FP32, each synthesised then analysed. One step = the
    whole batch. Timed three ways with CUDA events: one sht_synthesize / sht_analyze
    call per transform (16 kernel launches), the grouped persistent launches (4), and
    their CUDA graph (1 graph launch). Prints one JSON line (not the headline metric)."""
    import torch
    import speedytransforms as st
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    device = torch.device("cuda", 0)
    entries = []
    for T_, nh, K in MIX:
        S = st.SpectralTransform(st.Spectrum(T_, T_), st.OctahedralGaussianGrid(nh), nlayers=K, precision="fp32",
                                 device=device)
        c = O.random_coeffs(O.Spectrum(T_, T_), K, seed=T_)
        lt = st.LowerTriangularArray(torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64).to(device),
                                     S.spectrum)
        f = st.Field.zeros(S.grid, K, device=device)
        a = st.LowerTriangularArray.zeros(S.spectrum, K, device=device)
        entries += [(f, lt, S), (a, f, S)]
    b = st.Batch(entries)
    bn = b.autotune()
    b.capture()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / args.steps

    t_each = timed(b.run_each)
    t_grouped = timed(b.run)
    t_graph = timed(b.launch)
    plans = [e[2] for e in entries[::2]]
    for S in plans:                          # the per-call sequence with the fused kernels
        S.fusion = S.fusion_available
    t_each_fused = timed(b.run_each)
    for S in plans:
        S.fusion = False
    line = {"metric": "mixed-batch round trips/s (octahedral T31 K1 + T63 K8 + T127 K16 + T255 K64, FP32)",
            "value": 1.0 / t_graph, "unit": "batches/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_graph * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic",
            "config": {"workload": "mixed batch of 4 round trips, one grouped launch per stage, CUDA graph",
                       "legendre_tile_columns": bn},
            "ms_per_batch": {"one_call_per_transform": t_each * 1e3, "grouped_launches": t_grouped * 1e3,
                             "grouped_graph": t_graph * 1e3,
                             "one_fused_call_per_transform": t_each_fused * 1e3},
            "gpu_launches_per_batch": {"one_call_per_transform": 16, "grouped_launches": 4, "grouped_graph": 4,
                                       "one_fused_call_per_transform": 8}}
    print(json.dumps(line))
    return 0


def run_fused(args):
    """Fused transforms (the FFT and Legendre stages in one launch per direction,
    thread-block clusters passing the Fourier rows through shared memory) beside the
    separate kernels, FP32, at T31 on the full Gaussian grid with nlat 48 x 8 layers,
    T63 octahedral nlat 96 x 8, T127 octahedral nlat 192 x 48 (8 layers x 6 fields) and
    x 8. Per case: one synthesis and one analysis call timed eagerly with CUDA events,
    and the round trip replayed from a CUDA graph of 20 round trips. Prints one JSON line
    (not the headline metric)."""
    import torch
    import speedytransforms as st
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    cases = [("T31 full nlat 48 x 8", 31, True, 24, 8), ("T63 octahedral nlat 96 x 8", 63, False, 48, 8),
             ("T127 octahedral nlat 192 x 48", 127, False, 96, 48), ("T127 octahedral nlat 192 x 8", 127, False, 96, 8),
             ("T63 full nlat 96 x 8", 63, True, 48, 8), ("T127 full nlat 192 x 8", 127, True, 96, 8),
             ("T31 full nlat 48 x 48", 31, True, 24, 48)]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, n):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(n):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / n * 1e3
    res = {}
    for name, T_, full, nh, K in cases:
        grid = st.FullGaussianGrid(nh) if full else st.OctahedralGaussianGrid(nh)
        S = st.SpectralTransform(st.Spectrum(T_ + 1, T_), grid, nlayers=K, precision="fp32")
        c = O.random_coeffs(O.Spectrum(T_ + 1, T_), K, seed=1)
        lt = st.LowerTriangularArray(torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64, device="cuda"),
                                     S.spectrum)
        f, a = st.Field.zeros(grid, K), st.LowerTriangularArray.zeros(S.spectrum, K)
        r = {"fused_available": S.fusion_available}
        for fused in ([False, True] if S.fusion_available else [False]):
            S.fusion = fused
            syn = timed(lambda: st.transform_(f, lt, S), args.steps)
            ana = timed(lambda: st.transform_(a, f, S), args.steps)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                for _ in range(3):
                    st.transform_(f, lt, S)
                    st.transform_(a, f, S)
            torch.cuda.current_stream().wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(20):
                    st.transform_(f, lt, S)
                    st.transform_(a, f, S)
            rt = timed(g.replay, max(3, args.steps // 20)) / 20
            del g
            r["fused" if fused else "separate"] = {"synthesis_us": syn, "analysis_us": ana, "graph_round_trip_us": rt}
        S.fusion = False
        assert S.device_status() == 0
        res[name] = r
    line = {"metric": "fused vs separate FFT + Legendre stages, FP32 round trip (graph-replayed), microseconds",
            "value": res["T31 full nlat 48 x 8"].get("fused", {}).get("graph_round_trip_us"), "unit": "us",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "fused transforms at the small truncations",
                       "gpu_launches_per_round_trip": {"separate": 4, "fused": 2}},
            "by_case": res}
    print(json.dumps(line))
    return 0


def run_column_emulator(args):
    """The learned-physics workload: the MLP column emulator at T63 on the octahedral grid
    with nlat = 96 (10 944 columns) and 8 sigma layers. Trains on the columns of 96 of the
    wet model's own states (the reference's initial state with seeded variations, through
    this library's transforms: speedyphysics.ModelStates, ~1e6 columns) labelled by the
    plain condensation + convection kernel, then times one grid's parameterization
    (emulator with plain fallback) against the plain kernel on fresh states and reports the
    emulator's tendency error there. Prints one JSON line (not the headline metric)."""
    import torch
    import speedyphysics as sp
    device = torch.device("cuda", 0)
    ms = sp.ModelStates(device=device)
    ncol = ms.ncol
    batch, epochs = 4096, args.train_epochs

    def rows(cols):
        T, q, u, v, ps = cols
        dT, dq = torch.empty_like(T), torch.empty_like(q)
        sp.column_physics_(dT, dq, T, q, ps)
        return sp.columns_as_rows(T, q, u, v, ps), torch.cat([dT.T, dq.T], dim=1).contiguous()

    x, y = rows(ms.columns(range(1000, 1096)))
    ntrain = x.shape[0]
    em = sp.ColumnEmulator(max(batch, ncol), seed=0, device=device)
    em.fit_normalization(x, y)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    em.train(x, y, epochs=epochs, batch=batch, lr=3e-3, schedule="cosine")
    ev[1].record()
    torch.cuda.synchronize()
    t_train = ev[0].elapsed_time(ev[1]) / 1e3
    nsteps = epochs * (ntrain // batch)
    final_loss = em.loss()
    del x, y

    def timed(fn, n):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(n):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / 1e3 / n

    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))   # noqa: E731
    errT, errq, nf = [], [], 0
    for seed in range(5000, 5008):                 # fresh states, never trained on
        T, q, u, v, ps = ms.state(seed)
        dT, dq = torch.empty_like(T), torch.empty_like(q)
        pT, pq = torch.empty_like(T), torch.empty_like(q)
        nf += em.parameterization_(dT, dq, T, q, u, v, ps)
        sp.column_physics_(pT, pq, T, q, ps)
        errT.append(rel(dT, pT))
        errq.append(rel(dq, pq))
    reps = max(args.steps, 1) * 10
    emul = lambda: em.parameterization_(dT, dq, T, q, u, v, ps, count=False)   # noqa: E731
    plain = lambda: sp.column_physics_(pT, pq, T, q, ps)                      # noqa: E731
    t_emul = timed(emul, reps)
    t_plain = timed(plain, reps)

    def graph_time(fn, per=50):
        # GPU time without the Python call overhead: `per` calls captured in one CUDA graph
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(3):
                fn()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(per):
                fn()
        t = timed(g.replay, max(args.steps, 1)) / per
        del g
        return t

    t_emul_graph, t_plain_graph = graph_time(emul), graph_time(plain)
    line = {"metric": "emulated column-physics grids/s (T63 octahedral nlat 96: 10944 columns x 8 layers)",
            "value": 1.0 / t_emul, "unit": "grids/s", "n_gpus": 1, "steps": reps, "warmup": args.warmup,
            "ms_per_step": t_emul * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16",
            "data": "the wet model's own states at T63: the reference's initial state (Jablonowski-Williamson "
                    "wind and temperature, 0.7 relative humidity) with seeded variations, through this "
                    "library's transforms; no dynamical core",
            "config": {"workload": "MLP 33-256-256-256-16 GELU (tanh form) emulator of condensation + "
                                   "convection, plain-physics fallback beyond 4 standard deviations",
                       "columns_per_grid": ncol, "train_columns": ntrain, "train_states": 96, "batch": batch,
                       "epochs": epochs, "lr_schedule": "cosine 3e-3 -> 3e-5"},
            "train_columns_per_s": epochs * (ntrain // batch) * batch / t_train,
            "train_ms_per_step": t_train / max(nsteps, 1) * 1e3, "final_train_loss": final_loss,
            "plain_physics_grids_per_s": 1.0 / t_plain, "plain_physics_ms": t_plain * 1e3,
            "emulator_vs_plain_time": t_emul / t_plain,
            "graph_replayed_ms": {"emulator": t_emul_graph * 1e3, "plain_physics": t_plain_graph * 1e3,
                                  "emulator_vs_plain_time": t_emul_graph / t_plain_graph},
            "validation": {"states": 8, "rel_l2_dtemp": sum(errT) / len(errT), "rel_l2_dhumid": sum(errq) / len(errq),
                           "rel_l2_dtemp_worst_state": max(errT), "rel_l2_dhumid_worst_state": max(errq),
                           "fallback_fraction": nf / (8 * ncol)},
            "gpu_launches_per_grid": 1}
    print(json.dumps(line))
    return 0


def run_dycore_step(args):
    """The transforms of one time step of the primitive-equation wet model at T63 on the
    octahedral grid with nlat = 96 and 8 layers, in the reference's order (transform.jl:117-191,
    tendencies.jl:161-214): gradient, UV_from_vordiv, syntheses of 2, 4L+1 and 2L layers, the
    analysis of 9L+1 layers, curl, divergences and a Laplacian; the operators fused into two
    one-launch sets (7 library calls) or as separate calls (11). Timed as eager library calls
    and as one CUDA graph replayed per step. Prints one JSON line (not the headline metric)."""
    import torch
    import speedytransforms as st
    res = {}
    for prec, fused in (("fp32", True), ("fp16x3", True), ("bf16x3", True), ("fp32", False), ("fp16x3", False)):
        step = st.DycoreStep(T=63, nlat_half=48, L=8, precision=prec, fused=fused)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

        def timed(fn):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            ev[0].record()
            for _ in range(args.steps):
                fn()
            ev[1].record()
            torch.cuda.synchronize()
            return ev[0].elapsed_time(ev[1]) / args.steps

        t_eager = timed(step)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            step()
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            step()
        t_graph = timed(graph.replay)
        res[f"{prec}{'' if fused else ' separate operator calls'}"] = {
            "eager_ms": t_eager, "graph_ms": t_graph, "library_calls": step.launches()}
        del graph
    best = min(res, key=lambda p: res[p]["graph_ms"])
    line = {"metric": "dycore-step transforms/s (T63 octahedral nlat 96, 8 layers, primitive wet model)",
            "value": 1e3 / res[best]["graph_ms"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res[best]["graph_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": best.split()[0], "data": "synthetic",
            "config": {"workload": "one time step's transforms and spectral operators, CUDA graph",
                       "library_calls_per_step": res[best]["library_calls"]},
            "ms_per_step_by_precision": res}
    print(json.dumps(line))
    return 0


def run_operators(args):
    """The spectral operators (spectral_gradients.jl) at the T511 x 64 size, one degree more
    than the order (lmax = mmax + 1, as the reference's vector operators need): curl,
    divergence, UV_from_vordiv, Laplacian, inverse Laplacian and gradient, each timed alone
    with CUDA events over `--steps` calls, three sets of 67 MB fields taken in turn so that
    consecutive calls share no data through the L2.
    Prints one JSON line (not the headline metric) with each kernel's achieved GB/s of
    algorithmic bytes (fields read + written) against the measured HBM copy bandwidth."""
    import torch
    import speedytransforms as st
    K = LAYERS
    spec = st.Spectrum(T + 1, T)
    S = st.SpectralTransform(spec, st.OctahedralGaussianGrid(NLAT_HALF), nlayers=K, precision="fp32")
    g = torch.Generator(device="cuda").manual_seed(4)

    def field():
        return st.LowerTriangularArray(torch.randn((K, spec.nlm), dtype=torch.complex64, device="cuda",
                                                   generator=g), spec)
    # three sets of (u, v, out1, out2) used in turn: consecutive calls share no data (810 MB)
    sets = [tuple(field() for _ in range(4)) for _ in range(3)]
    turn = [0]

    def nxt():
        turn[0] = (turn[0] + 1) % len(sets)
        return sets[turn[0]]
    nbytes = K * spec.nlm * 8

    def curl():
        u, v, o1, _ = nxt()
        st.curl_(o1, u, v, S, radius=6.371e6)

    def div():
        u, v, o1, _ = nxt()
        st.divergence_(o1, u, v, S, radius=6.371e6)

    def uv():
        u, v, o1, o2 = nxt()
        st.UV_from_vordiv_(o1, o2, u, v, S, radius=6.371e6)

    def lap(inverse):
        u, _, o1, _ = nxt()
        st.laplace_(o1, u, S, inverse=inverse, radius=6.371e6)

    def grad():
        u, _, o1, o2 = nxt()
        st.gradient_(o1, o2, u, S, radius=6.371e6)
    ops = {   # name: (call, fields read + written per call)
        "curl": (curl, 3),
        "divergence": (div, 3),
        "UV_from_vordiv": (uv, 4),
        "laplace": (lambda: lap(False), 2),
        "inverse_laplace": (lambda: lap(True), 2),
        "gradient": (grad, 3),
    }
    peaks, peak_src = measured_peaks()
    peak = peaks.get("hbm_gbs")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    res = {}
    for name, (fn, nf) in ops.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(args.steps):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / args.steps
        gbs = nf * nbytes / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "algorithmic_bytes": nf * nbytes, "achieved_gbs": gbs,
                     "frac_of_measured_hbm": (gbs / peak) if peak else None}
    assert S.device_status() == 0
    total = sum(r["ms"] for r in res.values())
    # CPU beside it: the six operators once each through the FP64 numpy restatement of
    # spectral_gradients.jl on the same [nlm][64] shapes (host threads as numpy uses them)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    osp = O.Spectrum(T + 1, T)
    rng = np.random.default_rng(1)
    cu = rng.standard_normal((osp.nlm, K)) + 1j * rng.standard_normal((osp.nlm, K))
    cv = rng.standard_normal((osp.nlm, K)) + 1j * rng.standard_normal((osp.nlm, K))
    t0 = time.perf_counter()
    O.curl(osp, cu, cv, radius=6.371e6)
    O.divergence(osp, cu, cv, radius=6.371e6)
    O.UV_from_vordiv(osp, cu, cv, radius=6.371e6)
    O.laplace(osp, cu, radius=6.371e6)
    O.laplace(osp, cu, inverse=True, radius=6.371e6)
    O.gradient(osp, cu, radius=6.371e6)
    cpu_s = time.perf_counter() - t0
    line = {"metric": "spectral operators at T511 x 64 layers (lmax = mmax + 1 = 513), achieved HBM GB/s",
            "value": sum(r["algorithmic_bytes"] for r in res.values()) / (total * 1e-3) / 1e9, "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "peak_hbm_gbs": peak, "peak_source": peak_src,
            "config": {"workload": "curl, divergence, UV_from_vordiv, laplace, inverse laplace, gradient "
                                   "on [64][nlm] complex FP32 fields, each call timed alone",
                       "nlm": spec.nlm, "layers": K, "field_mb": nbytes / 1e6,
                       "l2": "three sets of fields in turn, so consecutive calls share no data (810 MB)"},
            "by_operator": res,
            "cpu_baseline": {"value": sum(r["algorithmic_bytes"] for r in res.values()) / cpu_s / 1e9,
                             "unit": "GB/s", "cores": os.cpu_count(),
                             "kind": "port", "ms_all_six": cpu_s * 1e3,
                             "sample": "the six operators once each, FP64 numpy restatement (oracle), same shapes"}}
    print(json.dumps(line))
    return 0


def run_matrix(args):
    """The dense-matrix workload (MatrixSpectralTransform, matrix_transform.jl:56-260, the
    reference's GPU default at truncations <= 64): T63 on the octahedral grid with nlat 96,
    8 layers, FP32 (three TF32 products on the tensor cores), synthesis then analysis per
    step. Each matrix holds 188 MB (more than the 126 MB L2) and the two directions
    alternate, so every call streams its matrix from HBM. Prints one JSON line (not the
    headline metric) with the round trips per second, the achieved HBM GB/s of the
    matrices' bytes, the errors against the FP64 oracle, the split 16-bit forms, and the
    same round trip through the SpectralTransform for comparison."""
    import torch
    import speedytransforms as st
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    Tm, nh, K = 63, 48, 8
    spec, grid = st.Spectrum(Tm, Tm), st.OctahedralGaussianGrid(nh)
    So = O.SpectralTransform(O.Spectrum(Tm, Tm), O.Grid(O.OCTAHEDRAL_GAUSSIAN, nh))
    c_np = O.random_coeffs(So.spectrum, K, seed=5)
    lt = st.LowerTriangularArray(torch.tensor(np.ascontiguousarray(c_np.T), dtype=torch.complex64, device="cuda"), spec)
    field = st.Field.zeros(grid, K)
    out = st.LowerTriangularArray.zeros(spec, K)
    peaks, peak_src = measured_peaks()
    peak = peaks.get("hbm_gbs")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(args.steps):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / args.steps
    res = {}
    ref = So.synthesize(c_np)
    for prec in ["fp32", "fp16x3", "bf16x3"]:
        M = st.MatrixSpectralTransform(spec, grid, nlayers=K, precision=prec)

        def step():
            st.transform_(field, lt, M)
            st.transform_(out, field, M)
        ms = timed(step)
        assert M.device_status() == 0
        f = field.data.cpu().numpy().T.astype(np.float64)
        a = out.data.cpu().numpy().T.astype(np.complex128)
        matrix_bytes = 2 * grid.npoints * 2 * spec.nlm * 4      # FP32, or two 16-bit pieces
        gbs = matrix_bytes / (ms * 1e-3) / 1e9
        res[prec] = {"ms": ms, "round_trips_per_s": 1e3 / ms, "matrix_bytes": matrix_bytes, "achieved_gbs": gbs,
                     "frac_of_measured_hbm": gbs / peak if peak else None,
                     "rel_err_synthesis": float(O.rel_err(f, ref)),
                     "rel_err_roundtrip": float(O.rel_err(a, So.analyze(ref)))}
        del M
    S = st.SpectralTransform(spec, grid, nlayers=K, precision="fp32")

    def sstep():
        st.transform_(field, lt, S)
        st.transform_(out, field, S)
    res["spectral_transform_fp32"] = {"ms": timed(sstep)}
    # CPU beside it: the reference's Float32 mul! is a BLAS SGEMM; numpy's FP32 matmul (BLAS,
    # all host threads) on the same shapes, a synthesis and an analysis product per round trip
    rng = np.random.default_rng(0)
    A_ana = rng.standard_normal((2 * spec.nlm, grid.npoints), dtype=np.float32)
    A_syn = rng.standard_normal((grid.npoints, 2 * spec.nlm), dtype=np.float32)
    xs = rng.standard_normal((2 * spec.nlm, K), dtype=np.float32)
    xg = rng.standard_normal((grid.npoints, K), dtype=np.float32)
    A_syn @ xs
    A_ana @ xg
    t0 = time.perf_counter()
    ncpu = 0
    while time.perf_counter() - t0 < 3.0 or ncpu < 3:
        A_syn @ xs
        A_ana @ xg
        ncpu += 1
    cpu_rt = ncpu / (time.perf_counter() - t0)
    r = res["fp32"]
    line = {"metric": "MatrixSpectralTransform round trips per second, T63 octahedral nlat 96 x 8 layers, FP32",
            "value": r["round_trips_per_s"], "unit": "round trips/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (three tf32 products)", "data": "synthetic",
            "gpu_launches": 6 * args.steps,
            "roofline": {"bound": "hbm", "achieved": r["achieved_gbs"], "peak": peak, "unit": "GB/s",
                         "frac": r["frac_of_measured_hbm"], "traffic": None, "peak_source": peak_src,
                         "algorithmic_bytes": "both matrices once per round trip (2 x npoints x 2 nlm x 4 B)"},
            "config": {"workload": "dense-matrix synthesis + analysis, T63 OctahedralGaussianGrid nlat 96 x 8 layers",
                       "npoints": grid.npoints, "nlm": spec.nlm,
                       "l2": "each 188 MB matrix exceeds the L2; the directions alternate"},
            "by_precision": res,
            "cpu_baseline": {"value": cpu_rt, "unit": "round trips/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{ncpu} round trips: numpy FP32 matmul (BLAS) of the two dense products"}}
    print(json.dumps(line))
    return 0


def profile_run(args):
    """W + K round trips of one precision at the benchmark workload and nothing else:
    the command ncu wraps for the launch list and the per-kernel captures."""
    import torch
    import speedytransforms as st
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O
    prec = "bf16x3" if args.precision == "auto" else args.precision
    device = torch.device("cuda", 0)
    spec, grid = st.Spectrum(T, T), st.OctahedralGaussianGrid(NLAT_HALF)
    c_np = O.random_coeffs(O.Spectrum(T, T), LAYERS, seed=2)
    lt = st.LowerTriangularArray(torch.tensor(np.ascontiguousarray(c_np.T), dtype=torch.complex64).to(device), spec)
    field = st.Field.zeros(grid, LAYERS, device=device)
    out = st.LowerTriangularArray.zeros(spec, LAYERS, device=device)
    S = st.SpectralTransform(spec, grid, nlayers=LAYERS, precision=prec, device=device)
    if args.prime_stage != "direct":
        S.prime_stage = args.prime_stage
    for _ in range(args.warmup + args.steps):
        st.transform_(field, lt, S)
        st.transform_(out, field, S)
    torch.cuda.synchronize()
    print(f"profile run: {prec}, {args.warmup} + {args.steps} round trips, device status {S.device_status()}")
    return 0


def run_ours(args):
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)
    import speedytransforms as st
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sht_oracle as O

    spec = st.Spectrum(T, T)
    grid = st.OctahedralGaussianGrid(NLAT_HALF)
    c_np = O.random_coeffs(O.Spectrum(T, T), LAYERS, seed=2)
    host_c = torch.tensor(np.ascontiguousarray(c_np.T), dtype=torch.complex64).pin_memory()
    lt = st.LowerTriangularArray(host_c.to(device), spec)
    field = st.Field.zeros(grid, LAYERS, device=device)
    out = st.LowerTriangularArray.zeros(spec, LAYERS, device=device)

    precisions = [args.precision] if args.precision != "auto" else ["fp32", "bf16x3", "fp16x3", "bf16x5"]
    variants = {}
    transforms = {}
    for prec in precisions:
        try:
            S = st.SpectralTransform(spec, grid, nlayers=LAYERS, precision=prec, device=device)
        except Exception as e:            # tensor-core path not built on this revision
            variants[prec] = {"available": False, "why": str(e)[:200]}
            continue
        # the library's autotuner (tile widths; results do not depend on them), once per
        # plan before anything is timed, as a user sets a plan up
        variants.setdefault(prec, {})["tile_columns"] = list(S.autotune())
        if args.prime_stage != "direct":
            S.prime_stage = args.prime_stage
        transforms[prec] = S

    # accuracy vs the FP64 oracle on every layer (rank 0), outside any timed region: the
    # relative L2 error of each layer's synthesised grid and of each layer's round trip;
    # a variant meets the bar when its worst layer does
    ref = None
    if rank == 0:
        So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(O.OCTAHEDRAL_GAUSSIAN, NLAT_HALF))
        ref_grid = So.synthesize(c_np)
        ref_rt = So.analyze(ref_grid)
        ref = (ref_grid, ref_rt)
    for prec, S in transforms.items():
        st.transform_(field, lt, S)
        st.transform_(out, field, S)
        torch.cuda.synchronize()
        v = {"available": True, "tile_columns": variants.get(prec, {}).get("tile_columns")}
        if ref is not None:
            g = field.data.cpu().numpy().T.astype(np.float64)
            a = out.data.cpu().numpy().T.astype(np.complex128)
            v["rel_err_synthesis"] = O.rel_err(g, ref[0])
            v["rel_err_roundtrip"] = O.rel_err(a, ref[1])
            v["rel_err_synthesis_worst_layer"] = max(O.rel_err(g[:, k], ref[0][:, k]) for k in range(LAYERS))
            v["rel_err_roundtrip_worst_layer"] = max(O.rel_err(a[:, k], ref[1][:, k]) for k in range(LAYERS))
        variants[prec] = v

    def round_trip(S):
        st.transform_(field, lt, S)
        st.transform_(out, field, S)

    def timed(S, steps, warmup):
        for _ in range(warmup):
            round_trip(S)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            round_trip(S)
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        return reduce_max(e0.elapsed_time(e1) / 1e3, world, device)

    for prec, S in transforms.items():
        secs = timed(S, max(3, args.steps // 2), args.warmup)
        variants[prec]["round_trips_per_s"] = world * max(3, args.steps // 2) / secs
        variants[prec]["ms_per_round_trip"] = secs / max(3, args.steps // 2) * 1e3

    # headline: fastest variant whose worst layer is within the error bar in both the
    # synthesis and the round trip (rank 0 decides, all ranks follow)
    ok = [p for p in transforms if variants[p].get("rel_err_roundtrip_worst_layer", 0.0) <= ERR_BAR
          and variants[p].get("rel_err_synthesis_worst_layer", 0.0) <= ERR_BAR]
    ok = ok or list(transforms)
    head = max(ok, key=lambda p: variants[p].get("round_trips_per_s", 0.0))
    head = broadcast_choice(head, world)
    S = transforms[head]

    # the timed region proper
    with ClockSampler(local_rank) as clk:
        secs = timed(S, args.steps, args.warmup)
    clocks = clk.summary()
    value = world * args.steps / secs

    # outside the timed region: the distribution of single round trips (an event after each,
    # no host synchronisation between them) and the round trip replayed from a CUDA graph
    nsamp = max(3, min(200, args.steps))
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(nsamp + 1)]
    evs[0].record()
    for i in range(nsamp):
        round_trip(S)
        evs[i + 1].record()
    torch.cuda.synchronize()
    per = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(nsamp))
    per_step = {"median": per[nsamp // 2], "min": per[0], "max": per[-1], "samples": nsamp}
    side = torch.cuda.Stream(device=device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(3):
            round_trip(S)
    torch.cuda.current_stream(device).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    GRAPH_RT = 10
    with torch.cuda.graph(graph):
        for _ in range(GRAPH_RT):
            round_trip(S)
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nrep = max(3, args.steps // GRAPH_RT)
    g0.record()
    for _ in range(nrep):
        graph.replay()
    g1.record()
    torch.cuda.synchronize()
    graph_ms = g0.elapsed_time(g1) / (nrep * GRAPH_RT)
    del graph

    # end to end through the public API with host buffers: every step copies its 64 layers
    # of coefficients in from page-locked host memory and its results back into it, inside
    # the transforms (sht_synthesize_host / sht_analyze_host), one round trip per chunk of
    # 16 layers so that the copy in of the next chunk and the copy out of the previous one
    # overlap the work of the current one. Steps are pipelined like a stream of requests
    # (results alternate between two host buffers): the copies of step i + 1 overlap the
    # tail of step i, and the timed region ends after the last step's last copy to the host
    # (S.host_wait() before the end event).
    host_outs = [torch.empty((LAYERS, spec.nlm), dtype=torch.complex64).pin_memory() for _ in range(2)]
    E2E_CHUNK = 16
    S.set_host_chunk(E2E_CHUNK)
    e2e_state = {"step": 0}

    def e2e_step():
        host_out = host_outs[e2e_state["step"] % 2]
        e2e_state["step"] += 1
        for k0 in range(0, LAYERS, E2E_CHUNK):
            f = st.Field(field.data[k0:k0 + E2E_CHUNK], S.grid)
            st.transform_(f, st.LowerTriangularArray(host_c[k0:k0 + E2E_CHUNK], spec), S)
            st.transform_(st.LowerTriangularArray(host_out[k0:k0 + E2E_CHUNK], spec), f, S)

    for _ in range(args.warmup):
        e2e_step()
    S.host_wait()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    S.host_wait()
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    e2e_secs = reduce_max(e0.elapsed_time(e1) / 1e3, world, device)
    nbytes = host_c.numel() * 8
    # the host link on this box: one plain copy of the step's coefficients each way (context
    # for e2e, which the two copies bound)
    dev_c = torch.empty_like(host_c, device=device)
    dev_c2 = torch.empty_like(host_c, device=device)
    side = (torch.cuda.Stream(device=device), torch.cuda.Stream(device=device))

    def duplex():   # one copy each way at once, on two streams: the bound of a pipelined step
        cur = torch.cuda.current_stream()
        for sx in side:
            sx.wait_stream(cur)
        with torch.cuda.stream(side[0]):
            dev_c.copy_(host_c, non_blocking=True)
        with torch.cuda.stream(side[1]):
            host_outs[1].copy_(dev_c2, non_blocking=True)
        for sx in side:
            cur.wait_stream(sx)
    link = {}
    for name, fn in (("h2d_ms", lambda: dev_c.copy_(host_c, non_blocking=True)),
                     ("d2h_ms", lambda: host_outs[0].copy_(dev_c, non_blocking=True)),
                     ("both_ms", duplex)):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        link[name] = e0.elapsed_time(e1) / 3
    del dev_c, dev_c2

    # roofline of the dominant kernel (per-kernel CUDA events on the launching stream)
    stage_ms = time_stages(S, lt, field, out, reps=max(5, args.steps // 2))
    alg = algorithmic(S)
    dom = max(stage_ms, key=stage_ms.get)
    peaks, src = measured_peaks()
    achieved = alg[dom]["bytes"] / (stage_ms[dom] * 1e-3) / 1e9
    traffic = committed_traffic().get(f"{head}:{dom}")
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_source": src,
                "algorithmic_bytes": alg[dom]["bytes"],
                "stage_ms": stage_ms, "share": {k: v / sum(stage_ms.values()) for k, v in stage_ms.items()}}
    if "flops" in alg[dom]:
        mult = 3 if head in ("bf16x3", "fp16x3") else 1
        roofline["legendre_tflops"] = alg[dom]["flops"] * mult / (stage_ms[dom] * 1e-3) / 1e12
    # the whole round trip against HBM: each of Λ (both directions), the grid and the
    # coefficients read once and written once, at the measured per-GPU round-trip rate
    rt_bytes = 2 * (4 * alg["_lam_elems"] + S.grid.npoints * LAYERS * 4 + S.spectrum.nlm * LAYERS * 8)
    rt_gbs = rt_bytes * (value / world) / 1e9
    roofline["round_trip"] = {"algorithmic_bytes": rt_bytes, "achieved": rt_gbs, "unit": "GB/s",
                              "frac": rt_gbs / peaks["hbm_gbs"]}

    # this library's kernels per round trip: FFT x 2 and Legendre x 2, plus the tensor-core
    # synthesis data image (which, for fp16, also finds the data scales), plus for fp16 the
    # analysis input's max-abs pass and its scale kernel
    launches_per_rt = {"fp32": 4, "bf16x3": 5, "bf16x5": 5, "fp16x3": 7}[head]
    if args.prime_stage == "tensor":
        launches_per_rt += 2                       # the tensor-core prime stage ahead of each FFT
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": head, "data": "synthetic",
            "config": config(world),
            "e2e": {"value": world * args.steps / e2e_secs, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "plain_copy_ms": link},
            "roofline": roofline, "clocks": clocks, "gpu_launches": launches_per_rt * args.steps,
            "per_round_trip_ms": per_step,
            "graph": {"ms_per_round_trip": graph_ms, "round_trips_per_s": world * 1e3 / graph_ms,
                      "round_trips_per_replay": GRAPH_RT},
            "variants": variants}
    if args.prime_stage != "direct":
        line["prime_stage"] = args.prime_stage
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line))
    for S_ in transforms.values():
        del S_
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000, help="timed steps (default: ~1 s at T511 x 64)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp32", "bf16x3", "fp16x3", "bf16x5"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--prime-stage", default="direct", choices=["direct", "tensor"],
                    help="where the ring FFTs' prime-radix first stages run (sht_plan_set_prime_stage)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="t511",
                    choices=["t511", "mixed-batch", "column-emulator", "dycore-step", "operators", "matrix", "fused"],
                    help="t511: the headline benchmark; mixed-batch: the grouped-launch comparison; "
                         "column-emulator: the MLP parameterization at T63; dycore-step: one time step's "
                         "transforms at T63 L8, eager and as a CUDA graph; operators: the spectral "
                         "operators at T511 x 64, GB/s per kernel")
    ap.add_argument("--profile-run", action="store_true",
                    help="only W + K round trips of one precision (default bf16x3), for profilers")
    ap.add_argument("--train-epochs", type=int, default=120, help="column-emulator: training epochs")
    ap.add_argument("--ref-seconds", type=float, default=240.0,
                    help="reference arm: CPU seconds for all steps; steps of all 64 layers unless they "
                         "would take longer")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_run:
        return profile_run(args)
    if args.workload == "mixed-batch":
        return run_mixed_batch(args)
    if args.workload == "column-emulator":
        return run_column_emulator(args)
    if args.workload == "dycore-step":
        return run_dycore_step(args)
    if args.workload == "fused":
        return run_fused(args)
    if args.workload == "matrix":
        return run_matrix(args)
    if args.workload == "operators":
        return run_operators(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
