#!/usr/bin/env python
"""Benchmark of the B200 TLR approximation path.

Workload (one step): the whole TLR approximation of a 2-D square-exponential
covariance matrix (beta = 0.1, sigma = 1, no nugget) on N = 102400 points of a
320 x 320 jittered grid in Z-order, block size 1024 (10000 far-field tiles of
1024 x 1024, 1.0486e10 entries), maxrank 256, oversample 16, tol 1e-7, with
the Gaussian sketch, orthogonalisation, projection, small SVD and rank
decision of every tile, and dense near-field blocks.  Inputs are synthetic
(points from the library's own seeded generator).

Metric: Mentries/s = (sum of m*n over all blocks) / step time / 1e6, counted
only if the relative Frobenius error (FP64, every block regenerated on the
GPU) is <= tol.
  value  -- device time of starsh_b200_approximate with the factors left on
            the device (points already on the host side of the call; the
            call uploads them, 1.6 MB), CUDA events on the library's stream;
  e2e    -- the drop-in STARS-H call starsh_blrm__drsdd_b200 with host
            buffers: point upload and the copy of all factors and dense
            blocks back to host memory inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun) every rank runs an independent replica on its own GPU
(the path does not shard); value = all ranks' entries / max rank time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from ctypes import POINTER, byref, c_double, c_void_p

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "stars-h_b200"))

WORKLOAD = dict(workload="spatial-2d-sqexp-N102400-nb1024-maxrank256-os16-tol1e-7",
                kernel="sqexp", ndim=2, N=102400, nb=1024, beta=0.1, nu=0.5,
                maxrank=256, oversample=16, tol=1e-7, place=6)
# CPU baseline sample: same kernel, block size, sketch width and tol on a
# quarter of the points per side (625 tiles of the same 1024 x 1024 shape).
CPU_SAMPLE_N = 25600
CPU_STEP_N = 16384
METRIC = "TLR Mentries/s at rel-err<=tol"


# ----------------------------------------------------------- problem setup

def make_problem(lib, wl, seed=0):
    import starsh_b200 as sb
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    data = POINTER(sb.SSData)()
    assert lib.starsh_ssdata_generate(byref(data), wl["N"], wl["ndim"],
                                      wl["beta"], wl["nu"], 0.0, wl["place"],
                                      1.0) == 0
    kern = c_void_p()
    ktype = {"exp": 1, "sqexp": 2, "matern": 3}[wl["kernel"]]
    assert lib.starsh_ssdata_get_kernel(byref(kern), data, ktype) == 0
    shape = (sb.STARSH_int * 2)(wl["N"], wl["N"])
    P = POINTER(sb.Problem)()
    assert lib.starsh_problem_new(byref(P), 2, shape, b"N", b"d", data, data,
                                  kern, b"bench") == 0
    C = POINTER(sb.Cluster)()
    assert lib.starsh_cluster_new_plain(byref(C), data, wl["N"], wl["nb"]) == 0
    return dict(data=data, P=P, C=C, shape=shape)


def new_format(lib, prob):
    import starsh_b200 as sb
    F = POINTER(sb.Blrf)()
    assert lib.starsh_blrf_new_tlr(byref(F), prob["P"], b"N", prob["C"],
                                   prob["C"]) == 0
    return F


# ------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed
    region (every 200 ms)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index),
                     f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5).stdout.strip()
                f = [x.strip() for x in out.split(",")]
                self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join()

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) > 7 and s[1].replace('.', '', 1).isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 7 and s[2].replace('.', '', 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) > 7
                          for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------- CPU baseline

def cpu_reference_run(n, threads, wl):
    """Runs the reference's OpenMP RSVD path (compiled from its sources into
    oracle/_ref) on an N-point instance of the workload in a subprocess with
    OMP_NUM_THREADS=threads, OPENBLAS_NUM_THREADS=1; returns its JSON."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads),
               OPENBLAS_NUM_THREADS="1", STARSH_BACKEND="OPENMP",
               STARSH_LRENGINE="RSVD", STARSH_OVERSAMPLE=str(wl["oversample"]))
    cmd = [sys.executable, os.path.abspath(__file__), "--_cpu-run", str(n)]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True,
                         timeout=900)
    for line in out.stdout.splitlines():
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError(f"CPU reference run failed: {out.stderr[-2000:]}")


def _cpu_run(n):
    """Child process body of cpu_reference_run (reference library only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from harness import RefProblem
    wl = WORKLOAD
    ref = oracle.Ref()
    pr = RefProblem(ref, "spatial", n, wl["nb"], ndim=wl["ndim"],
                    place=wl["place"], beta=wl["beta"],
                    kernel_name=wl["kernel"])
    t0 = time.perf_counter()
    M = ref.approximate(pr.F, wl["maxrank"], wl["tol"],
                        oversample=wl["oversample"])
    dt = time.perf_counter() - t0
    err = ref.dfe(M) if n <= CPU_SAMPLE_N else None
    print(json.dumps({"seconds": dt, "entries": n * n, "rel_err": err}))


# ------------------------------------------------------------- device peak

def fp64_peak_tflops(torch):
    """FP64 tensor throughput measured in this run: torch float64 matmul
    (cuBLAS DGEMM) 4096^3, best of 5 after warm-up."""
    a = torch.randn(4096, 4096, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    return 2 * 4096 ** 3 / best / 1e12


# ------------------------------------------------------------------ main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--engine", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--n", type=int, default=WORKLOAD["N"],
                    help="points (a smaller N profiles the same kernels)")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline leg")
    ap.add_argument("--_cpu-run", type=int, default=0, dest="cpu_run")
    args = ap.parse_args()
    if args.cpu_run:
        _cpu_run(args.cpu_run)
        return

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    wl = dict(WORKLOAD)
    if args.n != wl["N"]:
        wl["N"] = args.n
        wl["workload"] = wl["workload"].replace("N102400", f"N{args.n}")
    threads = len(os.sched_getaffinity(0))

    if args.impl == "reference":
        if rank != 0:
            return
        # Reference arm: its OpenMP RSVD on the host cores, one bounded
        # sample of the workload (same tiles, sketch width, tol) per step.
        times = []
        for i in range(args.warmup + args.steps):
            r = cpu_reference_run(CPU_STEP_N, threads, wl)
            if i >= args.warmup:
                times.append(r["seconds"])
        t = statistics.mean(times)
        v = CPU_STEP_N ** 2 / t / 1e6
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v,
            "unit": "Mentries/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(workload=wl["workload"], sample_N=CPU_STEP_N,
                           engine="starsh_blrm__drsdd_omp"),
            "cpu_baseline": {"value": v, "unit": "Mentries/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"N={CPU_STEP_N} ({(CPU_STEP_N // wl['nb']) ** 2} tiles of 1024x1024)"},
            "e2e": {"value": v, "unit": "Mentries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return

    import torch
    import starsh_b200 as sb
    lib = sb.load()
    torch.cuda.set_device(local)
    assert lib.starsh_b200_set_device(local) == 0
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.ExternalStream(lib.starsh_b200_stream())
    chosen = sb.ENGINE_MIXED if args.engine == "mixed" else sb.ENGINE_FP64
    lib.starsh_set_oversample(str(wl["oversample"]).encode())
    prob = make_problem(lib, wl)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def step(engine, flags, entry=None):
        F = new_format(lib, prob)
        M = POINTER(sb.Blrm)()
        flush.zero_()          # L2 flush between steps (256 MB > 126 MB L2)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        s.record(stream)
        if entry is not None:
            info = entry(byref(M), F, wl["maxrank"], wl["tol"], 0)
        else:
            info = lib.starsh_b200_approximate(byref(M), F, wl["maxrank"],
                                               wl["tol"], 0, engine, flags)
        e.record(stream)
        e.synchronize()
        host = time.perf_counter() - t0
        assert info == 0, lib.starsh_b200_last_error()
        return M, F, s.elapsed_time(e) / 1e3, host, sb.stats(lib)

    def free(M, F):
        lib.starsh_blrm_free(M)
        lib.starsh_blrf_free(F)

    def measure(engine, clocks=None):
        """W warm-up and K timed device-resident approximations; returns the
        mean device time, the stats of the last step, its FP64 error."""
        for _ in range(args.warmup):
            M, F, *_ = step(engine, 0)
            free(M, F)
        barrier()
        times, sts = [], []
        ctx = clocks if clocks is not None else _Null()
        with ctx:
            for i in range(args.steps):
                M, F, dt, host, st = step(engine, 0)
                times.append(dt)
                sts.append(st)
                if i + 1 < args.steps:
                    free(M, F)
        barrier()
        err = lib.starsh_blrm__dfe_b200(M)
        free(M, F)
        return statistics.mean(times), sts, err

    # the chosen engine (timed region sampled for clocks), then the plain
    # FP64 form on the same GPU
    clocks = ClockSampler(local)
    t_dev, sts, err = measure(chosen, clocks)
    last = sts[-1]
    if chosen != sb.ENGINE_FP64:
        t_plain, sts_plain, err_plain = measure(sb.ENGINE_FP64)
    else:
        t_plain, sts_plain, err_plain = t_dev, sts, err
    # e2e: the drop-in call with host buffers
    entry = (lib.starsh_blrm__drsdd_b200_mp if chosen == sb.ENGINE_MIXED
             else lib.starsh_blrm__drsdd_b200)
    e2e_times, e2e_st = [], None
    barrier()
    for _ in range(args.steps):
        M, F, dt, host, st = step(chosen, 1, entry)
        e2e_times.append(host)
        e2e_st = st
        free(M, F)
    barrier()
    t_e2e = statistics.mean(e2e_times)
    entries = last.entries
    if world > 1:
        tt = torch.tensor([t_dev, t_e2e, t_plain], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_dev, t_e2e, t_plain = tt.tolist()
    value = world * entries / t_dev / 1e6
    e2e_value = world * entries / t_e2e / 1e6
    plain_value = world * entries / t_plain / 1e6

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    # roofline of the dominant kernel: the sketch GEMM (FP64 DMMA)
    per_launch_ms = last.sketch_ms / max(1, last.sketch_launches)
    flops_per_launch = last.sketch_flops / max(1, last.sketch_launches)
    achieved = flops_per_launch / (per_launch_ms / 1e3) / 1e12
    peak = fp64_peak_tflops(torch)
    accepted = bool(0 <= err <= wl["tol"])
    line = {
        "metric": METRIC, "value": value if accepted else None,
        "unit": "Mentries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded jittered grid)",
        "config": {"workload": wl["workload"],
                   "engine": "mixed (adaptive sketch, FP64 at this tol)" if chosen == sb.ENGINE_MIXED else "fp64",
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "tiles": int(last.tiles), "false_far": int(last.false_far),
                   "entries": int(entries),
                   "l2": "flushed (256 MB write) before every step",
                   "mean_rank": last.rank_sum / max(1, last.tiles - last.false_far),
                   "max_rank": last.max_rank,
                   "sketch_columns_per_tile": last.sketch_flops / max(1.0, 2.0 * entries)},
        "rel_err": err, "tol": wl["tol"], "accepted": accepted,
        "plain_fp64": {"value": plain_value, "ms_per_step": t_plain * 1e3,
                       "rel_err": err_plain,
                       "chosen_over_plain": value / plain_value},
        "e2e": {"value": e2e_value, "unit": "Mentries/s",
                "h2d_bytes_per_step": int(e2e_st.h2d_bytes),
                "d2h_bytes_per_step": int(e2e_st.d2h_bytes),
                "ms_per_step": t_e2e * 1e3},
        "gpu_launches": int(sum(s.kernel_launches for s in sts)),
        "phases_ms": {"sketch": last.sketch_ms, "project": last.project_ms,
                      "total_host": last.total_ms},
        "roofline": {"bound": "tensor", "kernel": "k_gemm_f64 (sketch Y = D Omega)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "peak_source": "measured in this run: torch float64 matmul 4096^3 (cuBLAS DGEMM); MEASURED_PEAKS.json has no FP64 figure",
                     "traffic": None},
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_cpu:
        try:
            r = cpu_reference_run(CPU_SAMPLE_N, threads, wl)
            line["cpu_baseline"] = {
                "value": r["entries"] / r["seconds"] / 1e6, "unit": "Mentries/s",
                "cores": threads, "kind": "reference",
                "sample": f"N={CPU_SAMPLE_N}: {(CPU_SAMPLE_N // wl['nb']) ** 2} tiles of 1024x1024, same kernel/maxrank/oversample/tol, starsh_blrm__drsdd_omp",
                "rel_err": r["rel_err"], "seconds": r["seconds"]}
        except Exception as exc:   # reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:300]}
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
