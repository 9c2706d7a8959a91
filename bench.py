"""Benchmark of the View() hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one View() frame): the displaced dispersive icosphere
configuration — 1,310,720-triangle icosphere (8 subdivisions, 3-octave value
noise), rough dispersive dielectric, diffuse ground, 64 emissive triangles —
at 1280x720, 16 spp, trace depth 8: 14,745,600 camera-path samples per step.
Metric: Msamples/s (one sample = one render() iteration of one pixel).

  value   samples / device time of the View() launches (CUDA events on the
          library's stream), scene and film resident in HBM, L2 flushed
          between steps.
  e2e     the same metric through the C ABI with host buffers: per step
          cg_view(scene, &camera) plus cg_film_read of the XYZ film into
          pinned host memory, host wall clock around synchronised steps.
  roofline the dominant kernel's algorithmic bytes per launch (from a
          counting pass of the same kernels) over its CUDA-event time.
  cpu_baseline the oracle (the reference's estimator restated in C++,
          multithreaded) on a bounded pixel sample of the same frame.
  forms   (one GPU, default workload) the batched form (256 mixed views in
          one graph-replayed wavefront) and the served form (Poisson request
          streams over four resident scenes) against the plain path.

--impl reference times that CPU implementation alone on the same workload.
Multi-GPU (torchrun): every rank renders its own frames of the workload
(weak scaling, no collective on the data path); value is the sum over ranks
of samples over the max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Msamples/s and p50/p99 latency, batched/served vs plain, 1 B200, equal RMSE"
WORKLOAD = ("displaced dispersive icosphere: 1,310,720 tris, rough dispersive dielectric + diffuse "
            "ground + 64 emissive tris, 1280x720, 16 spp, depth 8 (plain View())")
W_, H_, SPP_, DEPTH_ = 1280, 720, 16, 8
# bytes the traversal reads per unit of work (the device layout): a node
# visit reads one 128 B Bvh4Node (four float child boxes and links; 64 B
# Bvh4QNode with 8-bit boxes; 64 B BvhNode with two child boxes on the binary
# trees), a triangle test one 48 B triangle
# record, an instance entry one 64 B DevInstance; per ray the kernel reads
# 32 B of ray and writes 20 B of hit
NODE_B = {4: 128, "4q": 64, 2: 64}
TRI_B, INST_B, RAY_B = 48, 64, 52
# non-tensor FP32 peak (nominal; no measured figure exists for it)
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
# Memory traffic of the closest-hit kernel (k_extend_persistent, four-wide
# float-box trees) per extend ray, from ncu on the medium icosphere case
# (640x360, 16 spp, 16M-ray queues): DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) over the closest-hit launches of one frame divided by
# the frame's extend rays, and L2 bytes (lts__t_bytes.sum) per extend ray over
# two of those launches; with the active lanes per issued instruction
# (smsp__thread_inst_executed_per_inst_executed.ratio) of the same two.  A
# launch's traffic is taken as proportional to its rays (the trees stay
# L2-resident at both sizes).  None where no capture of the variant exists.
EXTEND_COUNTERS = {
    "dram_bytes_per_ray": 145.0,   # 2162 MB over the 14 launches of a frame of 14,915,514 rays
    "l2_bytes_per_ray": 962.3,     # L2 / DRAM bytes 6.64 on two of those launches
    "lanes_active": 10.4,          # 11.58 and 9.17 of 32 on the same two
}


def l2_copy_gbs(torch):
    """Bandwidth of a copy whose buffers stay in L2 (2 x 24 MiB, torch copy_,
    CUDA events over 200 copies, read + write bytes): the denominator of the
    closest-hit kernel's L2-side fraction."""
    a = torch.empty(24 << 20, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    for _ in range(20):
        b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(200):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize()
    return 2 * a.numel() * 200 / (e0.elapsed_time(e1) / 1e3) / 1e9


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """One process per GPU: barriers around the timed region and the max over
    ranks of each rank's device time.  No collective touches the render data
    (every rank renders its own frames).  backend "gloo" runs the same logic
    on CPU ranks."""

    def __init__(self, ws, rank, local, backend="nccl"):
        self.ws, self.rank, self.local = ws, rank, local
        self.pg = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if ws > 1:
            import datetime

            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(local)
                kw["device_id"] = torch.device("cuda", local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.pg.ReduceOp.MAX) if self.pg else x

    def sum(self, x: float) -> float:
        return self._reduce(x, self.pg.ReduceOp.SUM) if self.pg else x

    def job_rate(self, units: float, seconds: float) -> float:
        """Whole-job throughput: the units all ranks processed over the
        slowest rank's time."""
        return self.sum(units) / self.max(seconds)

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons during the timed region:
    read-only NVML queries every 20 ms from a thread (nvidia-smi at 200 ms
    where NVML is not available)."""

    NVML_PERIOD_S = 0.02

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml = pynvml
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        cmd = ["nvidia-smi", "-i", str(self.index),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _poll(self):
        n = self.nvml
        bits = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        while not self.stop.is_set():
            try:
                sm = n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)
                mx = n.nvmlDeviceGetMaxClockInfo(self.handle, n.NVML_CLOCK_SM)
                r = n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
            except Exception:
                return
            # the same row layout as the nvidia-smi query below
            row = [str(sm), str(mx), "", hex(r)] + \
                ["Active" if r & b else "Not Active" for b in bits]
            self.samples.append((time.perf_counter(), row))
            self.stop.wait(self.NVML_PERIOD_S)

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def window(self, t0, t1):
        """Keep the samples taken inside [t0, t1] (the timed region)."""
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        self.samples = inside if inside else self.samples[-1:]

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [s[1] for s in self.samples]
        sm = [float(s[0]) for s in rows if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in rows if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in rows:
            for k, n in enumerate(names):
                if len(s) > 4 + k and s[4 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


# --workload: the plain-path configurations (the icosphere frame is the default
# and the headline; the others fill the per-configuration table)
WORKLOADS = {
    "icosphere": (1280, 720, 16, 8, WORKLOAD),
    "cornell": (256, 256, 1, 2, "Cornell box: 5 wall quads, a diffuse and a specular-conductor box, "
                                "0.25x0.25 ceiling light of radiance 15; 256x256, 1 spp, depth 2 "
                                "(plain View())"),
    "instanced": (1920, 1080, 64, 12, "instanced scene: 4096 instances of 8 noise-displaced "
                                      "spheres/tori (10k-200k tris), 40/30/20/10 material mix, "
                                      "10k emissive tris; 1920x1080, 64 spp, depth 12 "
                                      "(plain View())"),
}
WORKLOAD_NAME = "icosphere"


def make_workload():
    from crystalgraphics_b200 import scenes
    if WORKLOAD_NAME == "cornell":
        return scenes.cornell(width=W_, height=H_, spp=SPP_, depth=DEPTH_)
    if WORKLOAD_NAME == "instanced":
        return scenes.instanced_scene(width=W_, height=H_, spp=SPP_, depth=DEPTH_)
    return scenes.icosphere_scene(width=W_, height=H_, spp=SPP_, depth=DEPTH_)


def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_rate(scene, budget_s=12.0, threads=0):
    """Oracle (reference estimator restated) on a bounded pixel sample of the
    workload frame: Msamples/s and a description of the sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from crystalgraphics_b200 import _abi
    native = O.use_native()  # built for this host's CPU where the compiler allows
    o = O.OracleScene(scene)
    conf = _abi.make_conf(W_, H_, SPP_, DEPTH_)
    threads = threads or cpu_threads()
    rng = np.random.default_rng(0)
    n = max(threads, 8)
    spent = 0.0
    done = 0
    film = np.zeros((H_, W_, 3), np.float32)
    seeds = np.zeros((H_, W_), np.uint32)
    while spent < budget_s:
        n = min(n, W_ * H_)
        start = int(rng.integers(0, W_ * H_ - n + 1))
        t0 = time.perf_counter()
        o.render(conf, scene.camera, film=film, seeds=seeds, rng=O.RNG_REFERENCE,
                 threads=threads, pixel_range=(start, start + n))
        dt = time.perf_counter() - t0
        spent += dt
        done += n
        if dt < budget_s / 8:
            n *= 2
    samples = done * SPP_
    return {"value": samples / spent / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "build": "g++ -O3 -march=native -ffp-contract=off" if native else
                     "g++ -O3 -march=x86-64-v2 -ffp-contract=off",
            "sample": f"{done} pixels x {SPP_} spp of the workload frame (random contiguous pixel "
                      f"runs), reference RNG order, faithful traversal, {spent:.1f} s"}


def host_packing_baseline(B):
    """The host side of the path as the reference runs it, single-threaded,
    beside this library's LoadScene: the reference rebuilds its TLAS, emissive
    buffer and alias table on the host at every View() and builds each BLAS
    once (median splits).  Timed: the reference's own AliasTable constructor
    (alias_table.h compiled unmodified, when it was built here) on the scene's
    emissive weights, and the oracle's restatement of the median-split BLAS and
    TLAS builds and of the emissive buffer; against LoadScene (binned SAH, on
    the GPU for trees of >= 16384 primitives, once per scene)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from crystalgraphics_b200 import scenes
    out = {"threads": 1,
           "per_view_host_s": "tlas + emissive + alias: what the reference redoes on the host "
                              "at every View(); LoadScene does all of it once"}
    for name, mk in (("icosphere", scenes.icosphere_scene), ("instanced", scenes.instanced_scene)):
        s = mk()
        o = O.OracleScene(s)
        ps = o.pack_seconds()
        prims, _, _ = o.emissive()
        o.close()
        w = prims["weight"].astype(np.float64)
        ref_alias = None
        if O.ref_alias_available():
            ts = []
            for _ in range(7):
                t0 = time.perf_counter()
                O.ref_alias_build(w)
                ts.append(time.perf_counter() - t0)
            ref_alias = float(np.median(ts))
        t0 = time.perf_counter()
        g = B.LoadScene(s)
        load_s = time.perf_counter() - t0
        info = g.info()
        g.close()
        alias_s = ref_alias if ref_alias is not None else ps["alias"]
        out[name] = {"emissive_entries": int(len(w)),
                     "reference_alias_table_s": ref_alias,
                     "oracle_alias_table_s": ps["alias"],
                     "oracle_blas_median_split_s": ps["blas"],
                     "oracle_tlas_median_split_s": ps["tlas"],
                     "oracle_emissive_buffer_s": ps["emissive"],
                     "per_view_host_s": ps["tlas"] + ps["emissive"] + alias_s,
                     "load_scene_s": load_s,
                     "load_scene_bvh_build_s": info.bvh_build_seconds,
                     "load_scene_bvh_device_builds": int(info.bvh_device_builds)}
    return out


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    scene = make_workload()
    rates = []
    for _ in range(args.warmup):
        cpu_rate(scene, budget_s=2.0)
    t_total = 0.0
    for _ in range(args.steps):
        r = cpu_rate(scene, budget_s=8.0)
        rates.append(r["value"])
    v = float(np.mean(rates))
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Msamples/s",
           "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": W_ * H_ * SPP_ / (v * 1e6) * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "sampled": "bounded pixel runs per step",
                      "ms_per_step": "the full frame's time at the measured rate (each step "
                                     "times a bounded pixel sample of the frame, ~8 s)"},
           "cpu_baseline": {"value": v, "unit": "Msamples/s", "cores": cpu_threads(),
                            "kind": "port", "build": r["build"], "sample": r["sample"]},
           "e2e": {"value": v, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---- batched and served forms against the plain one-view-per-View() path ----------------------
BATCH_DEPTH = 12     # the instanced scene's trace depth
SERVE_DEPTH = 12     # one conf serves all four resident scenes
SERVE_RATES = (50, 200, 2000)
SERVE_REQUESTS = 48
SERVE_REPEATS = 3


def _rel_diff(a, b):
    return float(np.abs(a - b).max()) / max(float(np.abs(b).mean()), 1e-6)


def _tuning_kwargs(t):
    return dict(queue_capacity=int(t.queue_capacity), extend_block=int(t.extend_block),
                shade_block=int(t.shade_block), use_graph=int(t.use_graph),
                bvh_width=int(t.bvh_width),
                persistent={2: False, 3: "postponed"}.get(int(t.persistent), True),
                shade_sort={1: "global", 2: "none", 3: "block"}.get(int(t.shade_sort), "global"),
                pipelines=int(t.pipelines), traversal_threads=int(t.traversal_threads))


def _plain_render(B, g, pos, d, w, h, spp, seed, depth, tuning=None, out=None):
    """One view the plain way: EnvInit for its film size, View, ReadFilm (into
    `out` when given).  Returns (film, host wall seconds, device ms of the
    View launches)."""
    t0 = time.perf_counter()
    B.EnvInit(B.PathTraceConf(render_width=w, render_height=h, sample_count=spp,
                              trace_depth=depth))
    if tuning:
        B.SetTuning(**tuning)
    B.SetSeed(seed)
    B.View(g, B.Camera(tuple(pos), tuple(d), (0.5 * w / h, 0.5)))
    film = B.ReadFilm(out=out)
    return film, time.perf_counter() - t0, B.LastStats().device_ms


def batched_form(B, torch):
    """256 views of the instanced scene (sides log-uniform 64-1024, spp in
    {1,4,16,64}, poses on an r=150 sphere) in one wavefront replayed from a
    captured CUDA graph, against 256 plain View() calls of the same views
    with the same keyed sample streams (so the same image RMSE)."""
    from crystalgraphics_b200 import scenes
    s = scenes.instanced_scene()
    views = scenes.batch_views(256)
    B.EnvInit(B.PathTraceConf(render_width=1920, render_height=1080, sample_count=64,
                              trace_depth=BATCH_DEPTH))
    g = B.LoadScene(s)
    t_tune = time.perf_counter()
    best = B.autotune_views(g, views[::32])   # 8 probe views of the batch
    t_tune = time.perf_counter() - t_tune
    tuning = _tuning_kwargs(best)
    samples = sum(w * h * spp for _, _, w, h, spp, _ in views)
    small = [v for v in views if v[2] * v[3] * v[4] <= 1 << 18]
    small_samples = sum(w * h * spp for _, _, w, h, spp, _ in small)

    def batch(vs):
        arr = B.make_views(vs)
        B.batch_render(g, arr)                     # captures the graph
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        films = B.batch_render(g, arr)             # replays it
        wall = time.perf_counter() - t0
        return films, wall, B.LastStats().device_ms

    films, b_wall, b_dev = batch(views)
    _, bs_wall, bs_dev = batch(small)
    small_ids = {id(v) for v in small}
    p_wall = p_dev = ps_wall = ps_dev = 0.0
    worst = 0.0
    for v, bf in zip(views, films):
        film, wall, dev = _plain_render(B, g, *v, BATCH_DEPTH, tuning)
        p_wall += wall
        p_dev += dev
        if id(v) in small_ids:
            ps_wall += wall
            ps_dev += dev
        worst = max(worst, _rel_diff(bf, film))
    g.close()
    B.EnvTerm()
    msps = lambda n, sec: n / sec / 1e6
    return {
        "workload": "instanced scene (4096 instances of 8 meshes, 10k emissive tris), 256 views, "
                    "side log-uniform 64-1024, spp in {1,4,16,64}, depth 12",
        "views": len(views), "samples": samples,
        "batched_msamples_per_s": msps(samples, b_dev / 1e3),
        "batched_wall_msamples_per_s": msps(samples, b_wall),
        "plain_msamples_per_s": msps(samples, p_dev / 1e3),
        "plain_wall_msamples_per_s": msps(samples, p_wall),
        "speedup_device": p_dev / b_dev, "speedup_wall": p_wall / b_wall,
        "small_views": {"views": len(small), "samples": small_samples,
                        "rule": "w*h*spp <= 262144",
                        "batched_msamples_per_s": msps(small_samples, bs_dev / 1e3),
                        "plain_msamples_per_s": msps(small_samples, ps_dev / 1e3),
                        "speedup_device": ps_dev / bs_dev, "speedup_wall": ps_wall / bs_wall},
        "max_rel_diff_vs_plain": worst,
        "tuning": tuning, "autotune_s": t_tune,
        "timing": "device: CUDA events around the launches (graph replay / View chunks); "
                  "wall: host clock incl. film readback (and EnvInit per plain view)",
    }


def served_form(B, torch):
    """Poisson request streams over four resident scenes (the icosphere and
    three instanced scenes with 4096, 2048 and 8192 instances) through the
    continuous-batching server, against the plain path serving the same
    stream live, one request at a time in arrival order (first come, first
    served) through EnvInit/View/ReadFilm.  Both write the films into the same
    per-request host buffers, allocated and touched once before timing (as a
    server reuses its output buffers; first-touch page faults of fresh
    buffers vary widely on a shared host).  Every rate runs SERVE_REPEATS
    times per form and the run with the median throughput is reported.
    Latency = finish - arrival per request; throughput = samples / (last
    finish - first arrival)."""
    from crystalgraphics_b200 import scenes
    resident = [scenes.icosphere_scene(), scenes.instanced_scene(),
                scenes.instanced_scene(instances=2048, seed=5),
                scenes.instanced_scene(instances=8192, seed=6)]
    B.EnvInit(B.PathTraceConf(render_width=1920, render_height=1080, sample_count=16,
                              trace_depth=SERVE_DEPTH))
    gs = [B.LoadScene(x) for x in resident]
    base = scenes.request_stream(SERVE_REQUESTS, 1.0)   # arrivals at 1 req/s, scaled per rate
    req_samples = [w * h * spp for _, _, _, _, w, h, spp, _ in base]
    total = sum(req_samples)
    outs = [np.ones((h, w, 3), np.float32) for _, _, _, _, w, h, _, _ in base]
    out = {"workload": "4 resident scenes, requests of {256^2, 512^2, 1280x720, 1920x1080} x "
                       "spp {1,4,16}, random poses, Poisson arrivals, depth 12",
           "requests_per_rate": SERVE_REQUESTS, "samples_per_rate": total,
           "repeats": SERVE_REPEATS, "rates": []}
    # warm both paths once
    with B.Server(gs, 32 << 30) as sv:
        _, si, p, d, w, h, spp, seed = base[0]
        sv.wait(sv.submit(si, p, d, w, h, spp, seed))
    _, si, p, d, w, h, spp, seed = base[0]
    _plain_render(B, gs[si], p, d, w, h, spp, seed, SERVE_DEPTH, out=outs[0])

    def serve_once(rate):
        with B.Server(gs, 32 << 30) as sv:
            ids = []
            t_start = time.perf_counter()
            for k, (t_arr, si, p, d, w, h, spp, seed) in enumerate(base):
                delay = t_start + t_arr / rate - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                ids.append(sv.submit(si, p, d, w, h, spp, seed, out=outs[k]))
            res = [sv.wait(i)[1] for i in ids]
            st = sv.stats()
        lat = np.array([r.finish_s - r.submit_s for r in res]) * 1e3
        span = max(r.finish_s for r in res) - min(r.submit_s for r in res)
        return {"msamples_per_s": total / span / 1e6,
                "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)),
                "peak_admitted_bytes": int(st.peak_bytes), "chunks": int(st.chunks),
                "busy_s": st.busy_s, "span_s": span, "copy_out_s": st.copy_out_s}

    def plain_once(rate):
        lat, fin = [], 0.0
        t_start = time.perf_counter()
        for k, (t_arr, si, p, d, w, h, spp, seed) in enumerate(base):
            arrival = t_start + t_arr / rate
            delay = arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            _plain_render(B, gs[si], p, d, w, h, spp, seed, SERVE_DEPTH, out=outs[k])
            fin = time.perf_counter()
            lat.append((fin - arrival) * 1e3)
        span = fin - (t_start + base[0][0] / rate)
        return {"msamples_per_s": total / span / 1e6, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "span_s": span}

    def median_run(fn, rate):
        runs = sorted((fn(rate) for _ in range(SERVE_REPEATS)), key=lambda e: e["msamples_per_s"])
        entry = runs[len(runs) // 2]
        entry["msamples_per_s_runs"] = [e["msamples_per_s"] for e in runs]
        return entry

    for rate in SERVE_RATES:
        served = median_run(serve_once, rate)
        plain = median_run(plain_once, rate)
        entry = {"rate_hz": rate, **served}
        entry["plain_msamples_per_s"] = plain["msamples_per_s"]
        entry["plain_p50_ms"] = plain["p50_ms"]
        entry["plain_p99_ms"] = plain["p99_ms"]
        entry["plain_msamples_per_s_runs"] = plain["msamples_per_s_runs"]
        out["rates"].append(entry)
    out["plain"] = ("the same arrival stream served live, one request at a time in arrival order "
                    "(first come, first served) through EnvInit/View/ReadFilm")
    out["scheduler"] = ("served: admission and dispatch shortest first (fewest samples left), "
                        "requests waiting over 1 s first (oldest first)")
    for g in gs:
        g.close()
    B.EnvTerm()
    return out


def forms_summary(forms):
    """The metric's comparison in one place: batched and served against the
    plain path (ratios > 1 favour the batched/served form)."""
    b, sv = forms["batched"], forms["served"]
    return {
        "batched_vs_plain_msamples_device": b["speedup_device"],
        "batched_vs_plain_msamples_wall": b["speedup_wall"],
        "batched_small_views_vs_plain_device": b["small_views"]["speedup_device"],
        "served_vs_plain": [{"rate_hz": e["rate_hz"],
                             "msamples": e["msamples_per_s"] / e["plain_msamples_per_s"],
                             "p50_plain_over_served": e["plain_p50_ms"] / e["p50_ms"],
                             "p99_plain_over_served": e["plain_p99_ms"] / e["p99_ms"],
                             "p50_ms": e["p50_ms"], "p99_ms": e["p99_ms"]}
                            for e in sv["rates"]],
    }


def run_ours(args):
    import torch

    from crystalgraphics_b200 import _abi
    from crystalgraphics_b200 import backend as B

    ws, rank, local = dist_env()
    d = Dist(ws, rank, local)
    torch.cuda.set_device(local)
    scene = make_workload()
    conf = B.PathTraceConf(render_width=W_, render_height=H_, sample_count=SPP_, trace_depth=DEPTH_)
    B.EnvInit(conf, device=local)
    B.SetSeed(1000 * rank)
    t_load = time.perf_counter()
    g = B.LoadScene(scene)
    t_load = time.perf_counter() - t_load
    info = g.info()
    load = {"seconds": t_load, "bvh_build_seconds": info.bvh_build_seconds,
            "bvh_device_builds": int(info.bvh_device_builds),
            "bvh_host_builds": int(info.bvh_host_builds)}
    if rank == 0 and ws == 1:
        # the same load with every tree built on the host, for comparison
        B.SetBvhBuild(_abi.CG_BVH_BUILD_HOST)
        t_h = time.perf_counter()
        gh = B.LoadScene(scene)
        load["host_build_seconds"] = time.perf_counter() - t_h
        load["host_bvh_build_seconds"] = gh.info().bvh_build_seconds
        gh.close()
        B.SetBvhBuild(_abi.CG_BVH_BUILD_AUTO)
    cam = B.Camera.from_c(scene.camera)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    samples_per_step = W_ * H_ * SPP_

    if (args.queue or args.bvh_width or args.persistent >= 0 or args.shade_sort != "default" or
            args.box_bits or args.pipelines or args.traversal_threads):
        B.SetTuning(queue_capacity=args.queue, bvh_width=args.bvh_width,
                    persistent=None if args.persistent < 0 else
                    ("postponed" if args.persistent == 3 else bool(args.persistent)),
                    shade_sort=None if args.shade_sort == "default" else args.shade_sort,
                    box_bits=args.box_bits, pipelines=args.pipelines,
                    traversal_threads=args.traversal_threads)
    if args.spectral == "hero":
        B.SetSpectral(_abi.CG_SPECTRAL_HERO)
    if args.roulette:
        B.SetRoulette(args.roulette)
    clocks = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        B.View(g, cam)
    # ---- timed region: device-resident ----
    dev_ms, launches, wall = [], 0, 0.0
    d.barrier()
    torch.cuda.synchronize()
    t_begin = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B.View(g, cam)
        wall += time.perf_counter() - t0
        st = B.LastStats()
        dev_ms.append(st.device_ms)
        launches += st.kernel_launches
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    clocks.__exit__()
    clocks.window(t_begin, t_end)
    d.barrier()
    t_dev = d.max(sum(dev_ms) / 1e3)
    value = d.job_rate(samples_per_step * args.steps, sum(dev_ms) / 1e3) / 1e6
    rays = st.extend_rays
    shadow = st.shadow_rays

    # ---- e2e through the C ABI with host buffers ----
    # the film lands in pinned host memory (one DMA per step)
    host = torch.empty((H_, W_, 3), dtype=torch.float32, pin_memory=True).numpy()
    d.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        B.View(g, cam)
        B.ReadFilm(_abi.CG_FILM_XYZ32F, out=host)
    torch.cuda.synchronize()
    e2e = d.job_rate(samples_per_step * args.steps, time.perf_counter() - t0) / 1e6

    # ---- per-kernel CUDA-event times: a separate pass of the same frames (the
    # events around every launch keep one chunk pipeline, so launches do not
    # overlap and each one's time is its own) ----
    B.SetProfiling(True)
    B.ReadProfile()
    for _ in range(args.steps):
        flush.zero_()
        B.View(g, cam)
    prof = B.ReadProfile()
    B.SetProfiling(False)

    # ---- the options beyond the reference on the same frame: Russian roulette
    # after the third bounce (as the icosphere workload's specification states
    # it) and hero-wavelength sampling (four wavelengths per sample, as the
    # Cornell workload's states it); device time of the same number of frames,
    # L2 flushed between them ----
    variants = None
    if (rank == 0 and args.spectral == "reference" and not args.roulette and
            WORKLOAD_NAME == "icosphere" and args.case == "full"):

        def frame_noise():
            """Relative variance of a pixel over independent frames (fresh
            sample streams, frame 0 each): the noise one frame leaves."""
            films = []
            for k in range(6):
                B.SetSeed(7000 + k)
                B.ViewSamples(g, cam, 0, SPP_)
                films.append(B.ReadFilm().copy())
            B.SetSeed(1000 * rank)
            f = np.stack(films).astype(np.float64)
            return float(f.var(0, ddof=1).mean() / max(f.mean() ** 2, 1e-30))

        base_ms = sum(dev_ms) / len(dev_ms)
        base_noise = frame_noise()
        variants = {"reference_frame_relative_variance": base_noise,
                    "efficiency": "time x variance of the reference sampler without roulette over "
                                  "the option's: how much sooner it reaches the same image RMSE"}
        for name, on, off in (("roulette_after_bounce_3", lambda: B.SetRoulette(3),
                               lambda: B.SetRoulette(0)),
                              ("hero_wavelengths", lambda: B.SetSpectral(_abi.CG_SPECTRAL_HERO),
                               lambda: B.SetSpectral(_abi.CG_SPECTRAL_REFERENCE))):
            on()
            for _ in range(2):
                B.View(g, cam)
            ms = 0.0
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                B.View(g, cam)
                ms += B.LastStats().device_ms
            vst = B.LastStats()
            noise = frame_noise()
            off()
            variants[name] = {"value": samples_per_step * args.steps / (ms / 1e3) / 1e6,
                              "unit": "Msamples/s", "ms_per_step": ms / args.steps,
                              "extend_rays_per_step": int(vst.extend_rays),
                              "frame_relative_variance": noise,
                              "efficiency_vs_reference": (base_ms * base_noise) /
                                                         (ms / args.steps * noise)}

    # ---- counting pass: algorithmic work of the traversal kernels ----
    B.SetCounting(True)
    B.View(g, cam)
    cst = B.LastStats()
    B.SetCounting(False)

    dominant = max(prof, key=lambda k: prof[k][0])
    ext_ms, ext_n = prof["extend"]
    sh_ms, sh_n = prof["shadow"]
    # counting pass totals cover extend + shadow; split the node/tri work by ray count
    per_frame_launch = max(ext_n // max(args.steps, 1), 1)
    tun = B.GetTuning()
    width = int(tun.bvh_width) or 4
    node_b = NODE_B["4q"] if width == 4 and int(tun.box_bits) == 8 else NODE_B[width]
    trav_bytes = (node_b * cst.node_visits + TRI_B * cst.tri_tests +
                  INST_B * cst.inst_visits)
    ext_share = cst.extend_rays / max(cst.extend_rays + cst.shadow_rays, 1)
    ext_bytes_frame = trav_bytes * ext_share + RAY_B * cst.extend_rays
    bytes_per_launch = ext_bytes_frame / per_frame_launch
    avg_launch_s = ext_ms / 1e3 / max(ext_n, 1)
    achieved = bytes_per_launch / avg_launch_s / 1e9
    # FP32 work of the same launches: 16 flops per child box tested (6 sub, 6 mul,
    # 4 min/max folded) and 40 per Moller-Trumbore test
    boxes = (width if width == 2 else 4) * cst.node_visits
    flops_per_launch = (16 * boxes + 40 * cst.tri_tests) * ext_share / per_frame_launch
    fp32_achieved = flops_per_launch / avg_launch_s / 1e12
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    # the kernel's real memory traffic, from the medium-case counters scaled by
    # this launch's rays (default kernel variant on the icosphere workload only)
    counters_apply = (WORKLOAD_NAME == "icosphere" and width == 4 and node_b == NODE_B[4] and
                      int(tun.persistent) == 1)
    rays_per_launch = cst.extend_rays / per_frame_launch
    traffic = dram_side = l2_side = None
    if counters_apply and EXTEND_COUNTERS["dram_bytes_per_ray"]:
        traffic = EXTEND_COUNTERS["dram_bytes_per_ray"] * rays_per_launch
        gbs = traffic / avg_launch_s / 1e9
        dram_side = {"bytes_per_launch": traffic, "achieved": gbs, "peak": peak, "unit": "GB/s",
                     "frac": gbs / peak}
    if counters_apply and EXTEND_COUNTERS["l2_bytes_per_ray"]:
        l2b = EXTEND_COUNTERS["l2_bytes_per_ray"] * rays_per_launch
        l2_peak = l2_copy_gbs(torch)
        gbs = l2b / avg_launch_s / 1e9
        l2_side = {"bytes_per_launch": l2b, "achieved": gbs, "peak": l2_peak, "unit": "GB/s",
                   "frac": gbs / l2_peak,
                   "peak_source": "measured here: torch copy of an L2-resident 24 MiB buffer"}

    cpu = cpu_rate(scene, budget_s=12.0) if (rank == 0 and ws == 1 and not args.no_cpu) else None
    packing = host_packing_baseline(B) if (rank == 0 and ws == 1 and not args.no_cpu and
                                           args.case == "full" and
                                           WORKLOAD_NAME == "icosphere") else None
    queue_capacity = int(B.GetTuning().queue_capacity)
    forms = None
    if rank == 0 and (args.forms == "on" or (args.forms == "auto" and ws == 1 and
                                              WORKLOAD_NAME == "icosphere" and args.case == "full")):
        del g
        g = None
        t_forms = time.perf_counter()
        forms = {"batched": batched_form(B, torch), "served": served_form(B, torch)}
        forms["seconds"] = time.perf_counter() - t_forms
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "samples_per_step": samples_per_step,
                       "spectral": args.spectral, "roulette_from_depth": args.roulette,
                       "l2": "flushed between steps (256 MiB write)",
                       "queue_capacity": queue_capacity,
                       "parallelism": f"replicas x{ws}"},
            "e2e": {"value": e2e, "unit": "Msamples/s", "h2d_bytes_per_step": 48,
                    "d2h_bytes_per_step": W_ * H_ * 12},
            "gpu_launches": launches,
            "roofline": {"kernel": "k_extend (closest-hit traversal)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src,
                         "traffic": traffic,
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                            "of k_extend_persistent per extend ray on the "
                                            "640x360 icosphere frame, times this launch's rays"
                                            if traffic else None),
                         "dram": dram_side, "l2": l2_side,
                         "lanes_active_per_instruction": EXTEND_COUNTERS["lanes_active"]
                         if counters_apply else None,
                         "bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": avg_launch_s * 1e3,
                         "fp32": {"achieved": fp32_achieved, "peak": FP32_PEAK_TFLOPS,
                                  "unit": "TFLOP/s", "frac": fp32_achieved / FP32_PEAK_TFLOPS,
                                  "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x "
                                                 "1.965 GHz (not measured)"}},
            "kernels_ms": {k: round(v[0], 3) for k, v in prof.items()},
            "kernels_note": "CUDA events around each launch in a separate pass of the same frames "
                            "(one chunk pipeline there, so launches do not overlap)",
            "kernels_launches": {k: int(v[1]) for k, v in prof.items()},
            "dominant_kernel": dominant,
            "rays_per_step": {"extend": int(rays), "shadow": int(shadow)},
            "mrays_per_s": (rays + shadow) * args.steps * ws / t_dev / 1e6,
            "traversal_counts_per_frame": {"node_visits": int(cst.node_visits),
                                           "tri_tests": int(cst.tri_tests),
                                           "inst_visits": int(cst.inst_visits)},
            "wall_ms_per_step": wall / args.steps * 1e3,
            "load_scene": load,
            "clocks": clocks.summary(),
        }
        if cpu:
            out["cpu_baseline"] = cpu
        if packing:
            out["host_packing_baseline"] = packing
        if variants:
            out["options_beyond_the_reference"] = variants
        if forms:
            out["forms_summary"] = forms_summary(forms)
            out["forms"] = forms
        print(json.dumps(out), flush=True)
    del g
    B.EnvTerm()
    d.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="icosphere", choices=sorted(WORKLOADS),
                    help="plain-path configuration (default: the icosphere frame)")
    ap.add_argument("--case", default="full", choices=["full", "medium", "small"],
                    help="small: the same scene at 320x180, 4 spp, with a 2M-ray queue; "
                         "medium: 640x360, 16 spp with a 16M-ray queue (two chunks of "
                         "1.84M samples, ~2.5 GB on the device): the cases ncu --set full "
                         "captures")
    ap.add_argument("--queue", type=int, default=0, help="ray queue capacity (0 = default)")
    ap.add_argument("--bvh-width", type=int, default=0, choices=[0, 2, 4],
                    help="node width of the traversal (0 = library default, 4)")
    ap.add_argument("--persistent", type=int, default=-1, choices=[-1, 0, 1, 3],
                    help="persistent lane-refill traversal (-1 = library default; 3 = with "
                         "postponed leaves)")
    ap.add_argument("--pipelines", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="chunk pipelines of View() (0 = library default, 2)")
    ap.add_argument("--traversal-threads", type=int, default=0,
                    help="threads per SM of the persistent traversal grids (0 = library default, "
                         "1024)")
    ap.add_argument("--box-bits", type=int, default=0, choices=[0, 8, 32],
                    help="four-wide child box precision (0 = library default, 32)")
    ap.add_argument("--forms", default="auto", choices=["auto", "on", "off"],
                    help="batched and served forms vs plain (auto: on at one GPU)")
    ap.add_argument("--spectral", default="reference", choices=["reference", "hero"],
                    help="wavelength sampling: the reference's one per sample (default) or hero "
                         "(four per sample)")
    ap.add_argument("--roulette", type=int, default=0,
                    help="Russian roulette from this hit depth on (0 = off, as the reference; 3 = "
                         "after the third bounce)")
    ap.add_argument("--shade-sort", default="default", choices=["default", "global", "block", "none"],
                    help="order of the rays the shading kernel takes (default: the library's, global)")
    args = ap.parse_args()
    global W_, H_, SPP_, DEPTH_, WORKLOAD, WORKLOAD_NAME
    WORKLOAD_NAME = args.workload
    W_, H_, SPP_, DEPTH_, WORKLOAD = WORKLOADS[args.workload]
    if args.case != "full" and args.workload != "icosphere":
        ap.error("--case applies to the icosphere workload")
    if args.case == "small":
        W_, H_, SPP_ = 320, 180, 4
        WORKLOAD = WORKLOAD.replace("1280x720, 16 spp", "320x180, 4 spp")
        args.queue = args.queue or (2 << 20)
    elif args.case == "medium":
        W_, H_ = 640, 360
        WORKLOAD = WORKLOAD.replace("1280x720", "640x360")
        args.queue = args.queue or (16 << 20)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
