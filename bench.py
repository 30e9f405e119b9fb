"""Benchmark: mixed-precision texel-FEM solve on the B200.

Workload (the icosphere configuration): icosphere subdivided 6x (81,920
triangles, vertices jittered N(0, 1e-3)), 16 latitude/longitude charts packed
with 8-texel gutters, 2048x2048 RGB texture of seeded value noise + U(-0.1, 0.1).
Operator M + 1e-3 S (screened Poisson / TextureFiltering form), right-hand side
M f + 1e-3 * 2 * S f, 3 right-hand sides solved together.

One step = one solve of all 3 right-hand sides from x = 0 to relative residual
<= 1e-6 (FP64 operator, every RHS): FP32 V-cycles inside FP64 refinement.

  value  Mtexels/s = texels x RHS / solve time / 1e6, inputs resident in HBM
         (device API gdtp_solve_device), device-timed with CUDA events.
  e2e    same through the host API with pinned host buffers: gdtp_solve_stream
         over the timed steps (H2D of b and D2H of x inside every step, on
         copy streams that overlap the neighbouring steps' solves);
         e2e.single_call is one gdtp_solve_ex per step, copies in series.
  fp64_vcycle  the plain FP64 GPU V-cycle (gdtp_solve_fp64_device) on the same
         device-resident problem, timed like value; mixed_over_fp64 = the ratio.
  cpu_baseline / oracle_error: the reference's own CPU solver (oracle/_ref/
         gdtp_ref: the reference headers compiled unmodified) run once on the
         host cores after the timed regions, FP64 V-cycles to 1e-12: its
         V-cycles to 1e-6 give the CPU rate, its converged iterate the FP64
         ground truth the device solutions are measured against.
  --impl reference: the same reference solver timed as its own arm (V-cycles
         to 1e-6), same mesh, texture, operator and tolerance.

Multi-GPU (torchrun): every rank solves its own copy (replicas, no collective on
the solve path); value = total texels x RHS of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mtexels solved/s at 1e-6 rel. residual, mixed vs FP64; p50/p99 latency"
WIDTH = 2048
LAMBDA, SHARP, TOL, K = 1e-3, 2.0, 1e-6, 3


def workload(width: int = WIDTH):
    from gradientdomaintextureprocessing_b200 import meshgen
    return meshgen.icosphere_atlas(width, width, subdiv=6, seed=0)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []   # (host time, fields)
        self.proc = None
        self.window = None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t_end = time.time() + 10.0   # the timed region starts once sampling runs
            while not self.samples and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.02)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append((time.time(), parts))

    def mark(self, t0: float, t1: float):
        """Host-time window of the timed region."""
        self.window = (t0, t1)

    def __exit__(self, *a):
        if self.proc:
            t_end = time.time() + 0.5   # let the sample that follows the region arrive
            while self.window and time.time() < t_end and not any(t > self.window[1] for t, _ in self.samples):
                time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        samples = self.samples
        if self.window and samples:
            # samples inside the timed region, widened by one sampling period on
            # each side so that a region shorter than the period still has one
            t0, t1 = self.window
            inside = [s for s in samples if t0 - 0.1 <= s[0] <= t1 + 0.1]
            samples = inside or sorted(samples, key=lambda s: min(abs(s[0] - t0), abs(s[0] - t1)))[:2]
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        f = [p for _, p in samples]
        sm = [float(p[0]) for p in f if p[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for p in f for i in range(4) if p[3 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(f[0][1]),
                "reasons": reasons, "samples": len(f)}


def max_over_ranks(ms: float, dist, device: str = "cuda") -> float:
    """The slowest rank's time: every rank's replica must finish for the job to finish."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: float, ms: float) -> float:
    """Whole-job throughput in millions of units per second: all ranks' units over the slowest time."""
    return world * units_per_rank / (ms * 1e-3) / 1e6


def gpu_local_cpus(device: int):
    """CPUs of the NUMA node the GPU hangs off (from sysfs), or None.  Pinned
    host buffers first touched from these CPUs sit in that node's memory, so
    host<->device copies do not cross the socket link."""
    try:
        import torch
        bus = torch.cuda.get_device_properties(device).pci_bus_id.lower()
        dom, rest = bus.split(":", 1)
        with open(f"/sys/bus/pci/devices/{int(dom, 16):04x}:{rest}/local_cpulist") as fh:
            cpus = set()
            for part in fh.read().strip().split(","):
                a, _, b = part.partition("-")
                cpus.update(range(int(a), int(b or a) + 1))
        return cpus & os.sched_getaffinity(0) or None
    except (OSError, ValueError, AttributeError, RuntimeError):
        return None


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local, dist


def run_reference(args, rank: int) -> dict:
    """Times the reference's CPU V-cycle loop (oracle/_ref/gdtp_ref, time mode)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref")
    cores = os.cpu_count() or 1
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "oracle/_ref/gdtp_ref not built (needs the reference sources at build time)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from gdd import read_dump
    from gradientdomaintextureprocessing_b200 import meshgen
    mesh = workload()
    with tempfile.TemporaryDirectory() as tmp:
        gdm = os.path.join(tmp, "mesh.gdm")
        meshgen.write_gdm(gdm, mesh)
        per_step, hist, counts = [], None, None
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))
        for step in range(args.warmup + args.steps):
            out = os.path.join(tmp, f"r{step}.gdd")
            subprocess.run([exe, gdm, out, "4", str(LAMBDA), str(SHARP), "60", "time", str(TOL)], check=True,
                           capture_output=True, env=env)
            d = read_dump(out)
            hist, counts = d["vcycle/history"], d["L0/counts"]
            if step >= args.warmup:
                per_step.append(float(d["time/vcycle"].sum()))
    n0 = int(counts[0])
    t = float(np.mean(per_step))
    value = n0 * K / t / 1e6
    return {"metric": METRIC, "value": value, "unit": "Mtexels/s (texels x RHS)", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "icosphere6 2048x2048 RGB, 16 charts, screened Poisson 1e-3, 3 RHS, tol 1e-6",
                       "texels": n0, "rhs": K, "levels": 4, "vcycles": len(hist) - 1,
                       "final_rel_residual": float(hist[-1]), "solver": "reference FP64 V-cycle (Vec4d), OpenMP"},
            "cpu_baseline": {"value": value, "unit": "Mtexels/s (texels x RHS)", "cores": cores, "kind": "reference",
                             "sample": "full workload: the reference V-cycles to 1e-6, set-up excluded"},
            "e2e": {"value": value, "unit": "Mtexels/s (texels x RHS)", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_leg(mesh, s, b_dev, x_dev, x_own, stream) -> dict:
    """The reference's CPU solver on this workload, run once (rank 0, N=1, after
    the timed regions): the compiled reference (oracle/_ref/gdtp_ref) builds the
    same hierarchy and operator and iterates its FP64 V-cycle to 1e-12.
    cpu_baseline: its V-cycles up to the first at <= 1e-6, timed by the reference
    run itself (set-up excluded).  oracle_error: energy-norm errors, in the
    reference's FP64 operator, of the device solve of the reference's right-hand
    side (solver error) and of this workload's own host-path solve (solver plus
    assembly and right-hand-side differences) against the reference's solution."""
    import ctypes as C
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_solution as rs
    from gradientdomaintextureprocessing_b200 import _lib
    if not rs.available():
        return {"cpu_baseline": {"unavailable": "oracle/_ref/gdtp_ref not built (needs the reference sources at build time)"}}
    ref = rs.reference_solution(mesh, 4, LAMBDA, SHARP, tol=1e-12, max_vcycles=60)
    hist, times = ref["history"], ref["vcycle_times"]
    cycles = next((i for i in range(1, len(hist)) if hist[i] <= TOL), len(hist) - 1)
    t_cpu = float(np.sum(times[:cycles]))
    n0 = int(ref["counts"][0])
    cpu = {"value": n0 * K / t_cpu / 1e6, "unit": "Mtexels/s (texels x RHS)", "cores": ref["threads"], "kind": "reference",
           "sample": "full workload: the reference FP64 V-cycles (Vec4d, OpenMP) to 1e-6, set-up excluded",
           "vcycles": cycles, "rel_residual": float(hist[cycles])}
    b_ref = torch.from_numpy(np.ascontiguousarray(ref["rhs"])).to(b_dev.device)
    x_dev.zero_()
    rep = _lib.Report()
    _lib.check(_lib.lib().gdtp_solve_device(s.handle, C.c_void_p(b_ref.data_ptr()), C.c_void_p(x_dev.data_ptr()), K, TOL, 60,
                                            C.c_void_p(stream.cuda_stream), C.byref(rep)))
    torch.cuda.synchronize()
    x_mine = x_dev.cpu().numpy()
    err = rs.energy_error(ref["A"], x_mine, ref["x"])
    err_own = rs.energy_error(ref["A"], x_own, ref["x"])
    return {"cpu_baseline": cpu,
            "oracle_error": {"energy_norm_max": float(err.max()), "energy_norm_max_own_rhs": float(err_own.max()),
                             "rel_residual_reference_operator": float(rs.relative_residual(ref["A"], ref["rhs"], x_mine).max()),
                             "reference_rel_residual": float(hist[-1]),
                             "reference": "the reference's FP64 V-cycle iterated to its residual floor on the same mesh, "
                                          "texture and operator (oracle/_ref/gdtp_ref vsolve)"}}


def serving_stream(n_requests: int, max_size: int, budget_gb: float, rate: float = 0.0) -> dict:
    """Serving stream: requests on torus / icosphere / genus-2 models at sizes
    log-uniform in [256, max_size] (sqrt(2) ladder, multiples of 8), kinds 60 %
    filtering (k = 3), 30 % geodesic (k = 1), 10 % line-integral convolution
    (k = 1, anisotropy 1e3), HBM admission budget.  Models are added and made
    resident before the stream (set-up time reported apart).  The same requests
    run three ways:
    * one at a time (each submitted after the previous one finished): the
      single-model service rate at these sizes, `single_rate`;
    * all queued at once: the server's capacity with batching and its worker
      slots, `value` (aggregate Mtexels/s) and `value_over_single`;
    * Poisson arrivals at the one-at-a-time capacity (rate 0) or at `rate` per
      second: the latencies under an offered load (`latency_ms`, `open_loop`).
    The two concurrent passes run once untimed first: a batch of a new width
    builds that width's multigrid and step graphs on first use, a one-time
    cost per model and width that is left out of the steady-state figures."""
    from gradientdomaintextureprocessing_b200 import serving
    stream = serving.request_stream(n_requests, rate_per_s=1.0, max_size=max_size, seed=0)
    server = serving.Server(budget_bytes=int(budget_gb * (1 << 30)), slots=4)
    t0 = time.time()
    models = serving.build_models(server, stream)
    setup_s = time.time() - t0
    kind_of = {v: k for k, v in serving.KIND_NAMES.items()}

    def work(r):  # texels x right-hand sides of a finished request
        return server.texels[models[(r["mesh"], r["size"], kind_of[r["kind"]])][0]] * (3 if r["kind"] == "filtering" else 1)

    queued = [(0.0,) + tuple(p[1:]) for p in stream]
    # one at a time
    t_alone, w_alone = [], []
    for p in queued:
        res, _, wall = serving.run_stream(server, [p], models)
        if res[0][1]["ok"]:
            t_alone.append(wall)
            w_alone.append(work(res[0][1]))
    single_rate = sum(w_alone) / sum(t_alone) / 1e6
    # all queued at once: once untimed (the batch widths it forms build their
    # multigrids and step graphs on first use), then timed
    serving.run_stream(server, queued, models)
    before = server.stats()
    res_q, st_q, wall_q = serving.run_stream(server, queued, models)
    ok_q = [r for _, r in res_q if r["ok"]]
    capacity = sum(work(r) for r in ok_q) / wall_q / 1e6
    batches = st_q["batches"] - before["batches"]
    batched = st_q["batched_requests"] - before["batched_requests"]
    # open loop
    if rate <= 0:
        rate = len(t_alone) / sum(t_alone)
    arrivals = serving.request_stream(n_requests, rate_per_s=rate, max_size=max_size, seed=0)
    serving.run_stream(server, arrivals, models)  # untimed: batch widths this arrival pattern forms
    results, st, wall = serving.run_stream(server, arrivals, models)
    failed = [r for _, r in results if not r["ok"]] + [r for _, r in res_q if not r["ok"]]
    results = [(x, r) for x, r in results if r["ok"]]
    lat = np.array([r["latency_ms"] for _, r in results])
    kinds = {serving.KIND_NAMES[k]: sum(1 for *_, kk in arrivals if kk == k) for k in serving.KIND_NAMES}
    return {"value": capacity, "unit": "Mtexels/s (texels x RHS, all requests queued at once)",
            "single_rate": single_rate, "value_over_single": capacity / single_rate,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "open_loop": {"arrival_rate_per_s": rate, "value": sum(work(r) for _, r in results) / wall / 1e6,
                          "note": "Poisson arrivals at the one-at-a-time capacity" if rate == len(t_alone) / sum(t_alone)
                          else "Poisson arrivals at the given rate"},
            "requests": len(arrivals), "failed": len(failed),
            "failures": [{k: r[k] for k in ("mesh", "size", "kind", "error")} for r in failed[:5]],
            "by_kind": {kn: {"p50_ms": float(np.percentile([r["latency_ms"] for _, r in results if r["kind"] == kn], 50)),
                             "p99_ms": float(np.percentile([r["latency_ms"] for _, r in results if r["kind"] == kn], 99)),
                             "max_iterations": int(max(r.get("iterations", 0) for _, r in results if r["kind"] == kn))}
                        for kn in sorted({r["kind"] for _, r in results})},
            "slowest": sorted(({k: r.get(k) for k in ("mesh", "size", "kind", "latency_ms", "iterations", "batch")}
                               for _, r in results), key=lambda d: -d["latency_ms"])[:5],
            "arrival_rate_per_s": rate, "wall_s": wall,
            "max_rel_residual": float(max(r["rel_residual_max"] for _, r in results)),
            "batches": batches, "requests_in_batches": batched,
            "evictions": st["evictions"], "resident_gb": st["resident_bytes"] / 2**30, "peak_gb": st["peak_bytes"] / 2**30,
            "budget_gb": budget_gb, "models": len(models), "setup_s": round(setup_s, 1), "kinds": kinds,
            "config": {"workload": f"torus / icosphere6 / genus-2, 256^2-{max_size}^2 log-uniform, "
                                   "60 % filtering k=3, 30 % geodesic k=1, 10 % LIC k=1", "slots": 4}}


def serve(args):
    """The serving stream as its own measurement line (--serve)."""
    import torch
    torch.cuda.set_device(0)
    from gradientdomaintextureprocessing_b200 import build as _build
    _build.build()
    out = {"metric": "serving: latency p50/p99 and aggregate Mtexels solved/s at 1e-6 rel. residual", "impl": "ours"}
    out.update(serving_stream(args.serve_requests, args.serve_max_size, args.serve_budget_gb, args.serve_rate))
    out["data"] = "synthetic"
    print(json.dumps(out), flush=True)


def timed_config(args):
    """Extra measurement lines for the geodesic and line-integral-convolution
    configurations (one JSON line each; the default run measures the filtering
    solve).  geodesics: icosphere(6) 1024^2, 64 seeded deep-texel sources as 64
    right-hand sides through the whole heat-method pipeline (host API, sources
    in, distances out).  lic: genus-2 4096^2 (32 charts), anisotropic metric of
    ratio 1e3 along a seeded tangent field, M + 1e-4 S, right-hand side M f of a
    uniform-noise texture, flexible CG around the FP32 V-cycle to 1e-6 (device
    buffers, and the host API for e2e)."""
    import torch
    import ctypes as C
    from gradientdomaintextureprocessing_b200 import build as _build
    _build.build()
    from gradientdomaintextureprocessing_b200 import _lib, meshgen
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    torch.cuda.set_device(0)
    t0 = time.time()
    if args.config == "geodesics":
        from gradientdomaintextureprocessing_b200.geodesics import DEFAULT_SMOOTHING, Geodesics, mean_texel_area
        mesh = meshgen.icosphere_atlas(1024, 1024, subdiv=6, seed=0)
        h = InitializeHierarchy(mesh, levels=4)
        t_heat = mean_texel_area(h) if args.geodesic_smoothing == "area" else DEFAULT_SMOOTHING
        G = Geodesics(h, smoothing=t_heat)
        srcs = np.random.default_rng(0).choice(h.array("deepGlobal"), size=64, replace=False)
        setup_s = time.time() - t0
        for _ in range(args.warmup):
            G.distance(srcs, tol=TOL)
        times, reps = [], []
        with ClockSampler(0) as clocks:
            th = time.time()
            for _ in range(args.steps):
                t1 = time.perf_counter()
                D, rep = G.distance(srcs, tol=TOL)
                times.append(time.perf_counter() - t1)
                reps.append(rep)
            clocks.mark(th, time.time())
        n = G.n
        t = float(np.median(times))
        out = {"metric": "heat-method geodesics: Mtexels x sources /s at 1e-6 rel. residual (both solves)", "impl": "ours",
               "value": n * 64 / t / 1e6, "unit": "Mtexels/s (texels x RHS)", "ms_per_step": t * 1e3,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32 V-cycle + f64 refinement",
               "data": "synthetic", "api": "gdtp_geodesic_distance (host sources in, host distances out, wall clock)",
               "config": {"workload": f"icosphere6 1024x1024, 16 charts, 64 sources, t = {t_heat:.4g}"
                                      f"{' (mean texel area)' if args.geodesic_smoothing == 'area' else ''}, eps = 1e-6", "texels": n,
                          "rhs": 64, "setup_s": round(setup_s, 1)},
               "rel_residual_max": float(max(r["rel_residual_max"] for r in reps)),
               "iterations": int(reps[-1]["iterations"]), "clocks": clocks.summary()}
    else:
        from gradientdomaintextureprocessing_b200.metric import InitializeAnisotropicMetric, across_for_ratio
        from gradientdomaintextureprocessing_b200.system import MASS, System, texel_signal
        mesh = meshgen.genus2_atlas(4096, 4096)
        vf = meshgen.gaussian_bump_field(mesh, bumps=8, seed=0)
        pm = InitializeAnisotropicMetric(mesh, vf, across=across_for_ratio(1e3))
        h = InitializeHierarchy(mesh, levels=4)
        s = System(h, parameter_metric=pm)
        s.update(1e-4, 1.0)
        s.set("krylov", 1)
        f = texel_signal(h, mesh["texture"])
        b = np.ascontiguousarray(s.apply(f, which=MASS).reshape(s.n, -1))
        setup_s = time.time() - t0
        L = _lib.lib()
        b_dev = torch.from_numpy(b).cuda()
        x_dev = torch.zeros_like(b_dev)
        k = b.shape[1]
        st = torch.cuda.current_stream()
        rep = _lib.Report()

        def step():
            x_dev.zero_()
            _lib.check(L.gdtp_solve_device(s.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()), k, TOL, 500,
                                           C.c_void_p(st.cuda_stream), C.byref(rep)))
            return rep.iterations, rep.rel_residual_max

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        with ClockSampler(0) as clocks:
            th = time.time()
            ev[0].record(st)
            res = [step() for _ in range(args.steps)]
            ev[1].record(st)
            torch.cuda.synchronize()
            clocks.mark(th, time.time())
        t = ev[0].elapsed_time(ev[1]) / args.steps * 1e-3
        b_pin = torch.from_numpy(b).pin_memory().numpy()
        x_pin = torch.zeros(b.shape, dtype=torch.float64).pin_memory().numpy()
        t1 = time.perf_counter()
        for _ in range(args.steps):
            _lib.check(L.gdtp_solve_ex(s.handle, b_pin.ctypes.data_as(C.c_void_p), x_pin.ctypes.data_as(C.c_void_p), k, TOL, 500, 1,
                                       C.byref(rep)))
        te = (time.perf_counter() - t1) / args.steps
        n = s.n
        out = {"metric": "line-integral convolution: Mtexels solved/s at 1e-6 rel. residual", "impl": "ours",
               "value": n * k / t / 1e6, "unit": "Mtexels/s (texels x RHS)", "ms_per_step": t * 1e3,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
               "dtype": "f32 V-cycle + f64 flexible CG", "data": "synthetic",
               "config": {"workload": "genus-2 4096x4096, 32 charts, anisotropic ratio 1e3, M + 1e-4 S, 1 RHS, tol 1e-6",
                          "texels": n, "rhs": k, "levels_used": s.levels_used, "setup_s": round(setup_s, 1)},
               "iterations": int(max(r[0] for r in res)), "rel_residual_max": float(max(r[1] for r in res)),
               "e2e": {"value": n * k / te / 1e6, "unit": "Mtexels/s (texels x RHS)", "h2d_bytes_per_step": int(b.nbytes),
                       "d2h_bytes_per_step": int(b.nbytes), "api": "gdtp_solve_ex, wall clock"},
               "clocks": clocks.summary()}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-solves", type=int, default=0,
                    help="profiling run: build the workload, run this many solves and exit (for ncu launch lists)")
    ap.add_argument("--width", type=int, default=WIDTH, help="texture resolution (profiling of smaller cases)")
    ap.add_argument("--serve", action="store_true",
                    help="serving workload instead: Poisson request stream over resident models (one JSON line)")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-max-size", type=int, default=1024,
                    help="largest texture size of the stream (4096 is the full range; host set-up then takes several minutes)")
    ap.add_argument("--serve-rate", type=float, default=0.0, help="open-loop arrivals per second (0: the one-at-a-time capacity)")
    ap.add_argument("--serve-budget-gb", type=float, default=80.0)
    ap.add_argument("--serve-requests-in-line", type=int, default=64,
                    help="requests of the compact serving stream (256^2-512^2) reported in the main line (0: none)")
    ap.add_argument("--trace-levels", action="store_true",
                    help="per-level timing of the V-cycle (events inside the captured steps), one JSON line")
    ap.add_argument("--knob", action="append", default=[], metavar="NAME=VALUE",
                    help="solver knob for --profile-solves / --trace-levels runs (e.g. tile_texels=1000000)")
    ap.add_argument("--config", choices=["filtering", "geodesics", "lic"], default="filtering",
                    help="geodesics / lic: extra measurement lines for those workloads (1 GPU)")
    ap.add_argument("--geodesic-smoothing", choices=["default", "area"], default="default",
                    help="geodesics: heat-step time t, the app's default 1e-3 or the mean texel area")
    args = ap.parse_args()
    if args.serve:
        return serve(args)
    if args.config != "filtering":
        return timed_config(args)

    rank, world, local, dist = dist_setup(args.gpus)
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank)), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    from gradientdomaintextureprocessing_b200 import build as _build
    _build.build()
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    from gradientdomaintextureprocessing_b200.system import System, texel_signal, texture_filtering_rhs
    import ctypes as C

    t0 = time.time()
    mesh = workload(args.width)
    t_mesh = time.time()
    h = InitializeHierarchy(mesh, levels=4)
    t_hier = time.time()
    s = System(h, device=local)
    s.update(LAMBDA, 1.0)
    t_sys = time.time()
    f = texel_signal(h, mesh["texture"])
    b_host = texture_filtering_rhs(s, f, LAMBDA, SHARP)
    setup_s = time.time() - t0
    setup = {"mesh_generation_s": round(t_mesh - t0, 3), "hierarchy_s": round(t_hier - t_mesh, 3),
             "assembly_and_update_s": round(t_sys - t_hier, 3), "rhs_s": round(time.time() - t_sys, 3)}
    setup["assembly_parts_ms"] = {k: round(float(v), 1) for k, v in zip(
        ("work_lists", "device_assembly", "boundary_blocks", "level0_operators", "galerkin_coarsening", "numeric_layout"),
        s.array("profile.setup")[8:14])}
    if args.knob and not (args.trace_levels or args.profile_solves):
        sys.exit("--knob applies to --profile-solves and --trace-levels runs only")
    for kv in args.knob:
        name, value = kv.split("=", 1)
        s.set(name, float(value))
    if args.trace_levels:
        s.set("trace_levels", 1)
        for _ in range(3):
            s.solve(b_host, tol=TOL)
        L = _lib.lib()
        cnt = C.c_int64()
        L.gdtp_system_array(s.handle, b"profile.reset", 0, None, C.byref(cnt))
        for _ in range(10):
            s.solve(b_host, tol=TOL)
        L.gdtp_system_array(s.handle, b"profile.levels", 0, None, C.byref(cnt))
        lv = np.zeros(cnt.value)
        L.gdtp_system_array(s.handle, b"profile.levels", 0, lv.ctypes.data_as(C.c_void_p), C.byref(cnt))
        n, nl = int(lv[0]), int(lv[1])
        stats = np.zeros(9 * nl)
        L.gdtp_system_array(s.handle, b"levelStats", 0, stats.ctypes.data_as(C.c_void_p), C.byref(cnt))
        print(json.dumps({"v_cycles_timed": n, "levels": nl,
                          "texels": [int(v) for v in stats.reshape(-1, 9)[:, 0]],
                          "boundary_texels": [int(v) for v in stats.reshape(-1, 9)[:, 2]],
                          "down_us": [round(1e3 * v / n, 1) for v in lv[2:2 + nl - 1]],
                          "coarsest_us": round(1e3 * lv[1 + nl] / n, 1),
                          "up_us": [round(1e3 * v / n, 1) for v in lv[2 + nl:2 * nl + 1]]}), flush=True)
        return
    if args.profile_solves:  # default smoother settings, no autotuner trials in the launch list
        for _ in range(args.profile_solves):
            x, r = s.solve(b_host, tol=TOL)
            print(json.dumps(r), flush=True)
        return
    t_tune = time.time()
    tuned = s.autotune(b_host, tol=TOL)
    setup["autotune_s"] = round(time.time() - t_tune, 3)
    # set-up as the reference's app does it: hierarchy, assembly and system
    # update, right-hand side, and the multigrid the first solve lays out and
    # fills (the synthetic mesh and the optional autotuner apart)
    ms_build = s.array("profile.setup")
    setup["first_multigrid_ms"] = round(float(ms_build[1] + ms_build[2] + ms_build[3]), 1)
    setup["total_with_mesh_and_autotune_s"] = round(time.time() - t0, 3)
    setup_s = (setup["hierarchy_s"] + setup["assembly_and_update_s"] + setup["rhs_s"] + setup["first_multigrid_ms"] / 1e3)
    n0 = b_host.shape[0]
    L = _lib.lib()

    # device-resident inputs
    b_dev = torch.from_numpy(b_host).to("cuda")
    x_dev = torch.zeros_like(b_dev)
    stream = torch.cuda.current_stream()
    rep = _lib.Report()

    def device_step():
        x_dev.zero_()
        code = L.gdtp_solve_device(s.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()), K, TOL, 60,
                                   C.c_void_p(stream.cuda_stream), C.byref(rep))
        if code != 0:
            _lib.check(code)
        return rep.iterations, rep.rel_residual_max

    for _ in range(args.warmup):
        device_step()
    prof_reset = C.c_int64()
    L.gdtp_system_array(s.handle, b"profile.reset", 0, None, C.byref(prof_reset))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    lat, iters, resid = [], [], []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clocks:
        t_host0 = time.time()
        ev[0].record(stream)
        for i in range(args.steps):
            it, r = device_step()
            ev[i + 1].record(stream)
            iters.append(it)
            resid.append(r)
        torch.cuda.synchronize()
        clocks.mark(t_host0, time.time())
    for i in range(args.steps):
        lat.append(ev[i].elapsed_time(ev[i + 1]))
    total_ms = ev[0].elapsed_time(ev[-1])
    total_ms = max_over_ranks(total_ms, dist)
    prof = np.zeros(6)
    cnt = C.c_int64()
    L.gdtp_system_array(s.handle, b"profile", 0, prof.ctypes.data_as(C.c_void_p), C.byref(cnt))
    value = job_rate(world, n0 * K * args.steps, total_ms)

    # end to end through the host API with pinned buffers, allocated and used
    # from the CPUs next to the GPU (their NUMA node's memory)
    all_cpus = os.sched_getaffinity(0)
    near_cpus = gpu_local_cpus(local)
    if near_cpus:
        os.sched_setaffinity(0, near_cpus)
    b_pin = torch.from_numpy(b_host).pin_memory().numpy()
    x_pin = torch.zeros(b_host.shape, dtype=torch.float64).pin_memory().numpy()

    def host_step():
        # zero initial guess: b goes host->device, x comes back device->host
        code = L.gdtp_solve_ex(s.handle, b_pin.ctypes.data_as(C.c_void_p), x_pin.ctypes.data_as(C.c_void_p), K, TOL, 60, 1,
                               C.byref(rep))
        if code != 0:
            _lib.check(code)

    host_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        host_step()
    e1.record(stream)
    torch.cuda.synchronize()
    single_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    single_value = job_rate(world, n0 * K * args.steps, single_ms)
    rel_final = float(s.residual(b_host, x_pin).max())

    # the same steps as one stream of problems (gdtp_solve_stream): every step
    # still uploads its b and downloads its x, on copy streams that overlap the
    # neighbouring steps' solves; one pinned output buffer per step
    x_pins = [torch.zeros(b_host.shape, dtype=torch.float64).pin_memory().numpy() for _ in range(max(args.steps, 2))]
    s.solve_stream([b_pin] * 2, x_pins[:2], tol=TOL)  # slot buffers and the graphs of both slots
    x_pins = x_pins[:args.steps]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    s.solve_stream([b_pin] * args.steps, x_pins, tol=TOL)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    e2e_value = job_rate(world, n0 * K * args.steps, e2e_ms)
    rel_stream = max(float(s.residual(b_host, x).max()) for x in (x_pins[0], x_pins[-1]))
    os.sched_setaffinity(0, all_cpus)  # the reference's CPU leg below uses every core

    # plain FP64 GPU V-cycle on the same problem (the comparator path), timed
    # like value: device-resident b and x, warm-up, then K solves between events
    def fp64_step():
        x_dev.zero_()
        code = L.gdtp_solve_fp64_device(s.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()), K, TOL, 60,
                                        C.c_void_p(stream.cuda_stream), C.byref(rep))
        if code != 0:
            _lib.check(code)
        return rep.vcycles, rep.rel_residual_max

    for _ in range(args.warmup):
        fp64_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    res64 = [fp64_step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    fp64_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    fp64_value = job_rate(world, n0 * K * args.steps, fp64_ms)

    # interactive re-weighting (UpdateLinearSystem with new weights): the
    # update, then the first solve, which rebuilds and factorises the multigrid;
    # the re-weighting cost is that solve less a solve on the built multigrid
    def timed_solve():
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.solve(b_host, tol=TOL)
        torch.cuda.synchronize()
        return time.perf_counter() - t
    t = time.perf_counter()
    s.update(2 * LAMBDA, 1.0)
    update_s = time.perf_counter() - t
    first_s = timed_solve()
    built_s = min(timed_solve() for _ in range(3))
    ms = s.array("profile.setup")
    setup["reweight_ms"] = round(1e3 * (update_s + first_s - built_s), 1)
    setup["reweight_parts_ms"] = {k: round(float(v), 1) for k, v in zip(
        ("update", "boundary_factorisations", "coarsest_inverse", "other_multigrid", "bs_values",
         "bs_subdomain_inverses", "bs_schur_products", "bs_schur_inverse"), ms[:8])}
    setup["device_factor"] = int(s.get("device_factor"))
    s.update(LAMBDA, 1.0)
    # dominant kernel: level-0 colour Gauss-Seidel sweep (4 colour passes), timed
    # by events recorded inside the captured refinement graph: the average of
    # the full sweeps of each V-cycle (the pre-smoothing after its zero-start
    # sweep, and the post-smoothing)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    sweep_ms = prof[1] / max(prof[0], 1)
    texels = prof[2]
    smoother = int(prof[5])  # 0 four colour passes per sweep, 1 fused tile-smoother round, 2 two row-smoother launches
    # algorithmic bytes per deep texel of one timed group (a colour sweep, or a
    # round of the fused tile smoother): 10 FP32 coefficients (40 B) + rhs
    # read, x read and x written once, k = 3 channels of 4 B (3 x 12 B) = 76 B
    sweep_bytes = texels * (40 + 3 * K * 4)
    if smoother == 1:
        kernel = "level-0 fused tile-smoother round (k_tile_smooth, one launch: every sweep of the round in 32x32 tiles)"
        # moved with the padded 4-lane vectors and the one-texel ring of a tile
        model_bytes = texels * (40 + 16 + 16 * 34 * 34 / 1024 + 16)
    elif smoother == 2:
        kernel = "level-0 4-colour Gauss-Seidel sweep (k_gs_rows x2: both colours of a row parity per launch)"
        # padded 4-lane vectors: coefficients, rhs, x written, and x of the
        # line's own row and of the rows above and below, each staged once per
        # launch (40 + 16 + 16 + 3 x 16 = 120 B)
        model_bytes = texels * (40 + 16 + 16 + 48)
    else:
        kernel = "level-0 4-colour Gauss-Seidel sweep (k_gs_colour x4)"
        # the 4-launch colour decomposition with padded 4-lane vectors:
        # coefficients, rhs, x written, and the x of the three other colours
        # read by each colour pass (40 + 16 + 16 + 3 x 16 = 120 B)
        model_bytes = texels * (40 + 16 + 16 + 48)
    achieved = sweep_bytes / (sweep_ms * 1e-3) / 1e9 if sweep_ms > 0 else None
    try:  # DRAM bytes per deep texel per timed group, from ncu captures of this workload
        traffic_per_texel = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))[
            {0: "colour", 1: "tile", 2: "rows"}[smoother]]
    except (OSError, ValueError, KeyError):
        traffic_per_texel = None
    launches = int(prof[4])  # counted by the solver: graph kernel nodes x graph launches + direct launches

    out = {"metric": METRIC, "value": value, "unit": "Mtexels/s (texels x RHS)", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 V-cycle + f64 refinement", "data": "synthetic",
           "config": {"workload": "icosphere6 2048x2048 RGB, 16 charts, screened Poisson 1e-3, 3 RHS, tol 1e-6",
                      "texels": n0, "rhs": K, "levels_used": s.levels_used, "l2": "inputs larger than L2 (>126 MB resident)",
                      "parallelism": f"replicas x{world}", "setup_s": round(setup_s, 2), "setup": setup,
                      "smoother": {k: v for k, v in tuned.items() if k != "seconds"}},
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
           "refinement_steps": {"mean": float(np.mean(iters)), "max": int(max(iters))},
           "rel_residual": {"device_path_max": float(max(resid)), "host_path_final": rel_final},
           "fp64_vcycle": {"value": fp64_value, "unit": "Mtexels/s (texels x RHS)", "ms_per_step": fp64_ms / args.steps,
                           "vcycles": int(max(r[0] for r in res64)), "rel_residual": float(max(r[1] for r in res64)),
                           "api": "gdtp_solve_fp64_device (device-resident, same warm-up, steps and events as value)"},
           "mixed_over_fp64": value / fp64_value,
           "e2e": {"value": e2e_value, "unit": "Mtexels/s (texels x RHS)", "h2d_bytes_per_step": int(b_host.nbytes),
                   "d2h_bytes_per_step": int(b_host.nbytes), "ms_per_step": e2e_ms / args.steps,
                   "api": "gdtp_solve_stream (zero initial guess, pinned host buffers, copies overlapped with the "
                          "neighbouring steps' solves)",
                   "rel_residual_max": rel_stream,
                   "single_call": {"value": single_value, "ms_per_step": single_ms / args.steps,
                                   "api": "gdtp_solve_ex per step (copies in series with the solve)"}},
           "roofline": {"bound": "hbm", "kernel": kernel,
                        "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": (achieved / peak) if achieved else None,
                        "traffic": texels * traffic_per_texel["bytes_per_deep_texel"] if traffic_per_texel and texels else None,
                        "traffic_source": traffic_per_texel["source"] if traffic_per_texel else "no ncu capture recorded",
                        "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                        "bytes_per_launch": sweep_bytes, "bytes_per_deep_texel": 40 + 3 * K * 4,
                        "bytes_moved_model": model_bytes, "ms_per_launch": sweep_ms},
           "gpu_launches": launches,
           "clocks": clocks.summary()}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        out.update(reference_leg(mesh, s, b_dev, x_dev, x_pin, stream))
    if rank == 0 and world == 1 and args.serve_requests_in_line > 0:
        # a compact serving stream after the timed regions (continuous batching,
        # admission, mixed kinds), so that every run reports serving latency
        blk = serving_stream(args.serve_requests_in_line, 512, args.serve_budget_gb)
        out["serving"] = {k: blk[k] for k in ("value", "unit", "single_rate", "value_over_single", "latency_ms", "open_loop",
                                               "requests", "failed", "max_rel_residual", "batches", "requests_in_batches",
                                               "evictions", "models", "setup_s", "by_kind", "slowest", "config")}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
