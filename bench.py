#!/usr/bin/env python
"""Benchmark of the B200 TLR approximation path.

Default workload (one step): the whole TLR approximation of a 2-D
square-exponential covariance matrix (beta = 0.1, sigma = 1, no nugget) on
N = 102400 points of a 320 x 320 jittered grid in Z-order, block size 1024
(10000 far-field tiles of 1024 x 1024, 1.0486e10 entries), maxrank 256,
oversample 16, tol 1e-7: per tile the Gaussian sketch, orthogonalisation,
projection, small SVD and rank decision, plus dense near-field blocks.
Other workloads (--workload): the Matérn variant of that configuration,
the 3-D Coulomb / sin(kr)/r configurations at tol 1e-5 with a TLR-by-dense
product (65536 x 64 RHS), and the reference's small 2-D exponential case.
Inputs are synthetic (the library's own seeded point generators).

Metric: Mentries/s = (sum of m*n over all blocks) / step time / 1e6, counted
only if the relative Frobenius error (FP64, every block regenerated on the
GPU) is <= tol.
  value      -- the chosen engine (mixed: adaptive sketch), device time of
                starsh_b200_approximate with the factors left on the device
                (CUDA events on the library's stream; the call uploads the
                points, 1.6 MB);
  plain_fp64 -- the same for the fixed-width all-FP64 engine;
  e2e        -- the drop-in STARS-H call (starsh_blrm__drsdd_b200_mp) with
                host buffers: point upload and the copy of all factors and
                dense blocks to host memory inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload NAME] [--engine mixed|fp64]

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
from ctypes import POINTER, byref, c_void_p

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "stars-h_b200"))

WORKLOADS = {
    "c2-sqexp": dict(kind="spatial", kernel="sqexp", ndim=2, N=102400, nb=1024,
                     beta=0.1, nu=0.5, maxrank=256, oversample=16, tol=1e-7,
                     place=6, cpu_n=25600, cpu_step_n=16384),
    "c2-matern": dict(kind="spatial", kernel="matern", ndim=2, N=102400,
                      nb=1024, beta=0.05, nu=0.7, maxrank=256, oversample=16,
                      tol=1e-7, place=6, cpu_n=None, cpu_step_n=None),
    "c3-coulomb": dict(kind="coulomb", ndim=3, N=65536, nb=512, maxrank=200,
                       oversample=10, tol=1e-5, place=1, diag=1.0,
                       cpu_n=16384, cpu_step_n=8192, dmml_nrhs=64),
    "c3-sin": dict(kind="sin", ndim=3, N=65536, nb=512, maxrank=200,
                   oversample=10, tol=1e-5, place=1, wave_k=20.0, diag=1.0,
                   cpu_n=16384, cpu_step_n=8192, dmml_nrhs=64),
    "c1-exp": dict(kind="spatial", kernel="exp", ndim=2, N=3600, nb=400,
                   beta=0.1, nu=0.5, maxrank=100, oversample=10, tol=1e-5,
                   place=6, cpu_n=3600, cpu_step_n=3600),
}
METRIC = "TLR Mentries/s at rel-err<=tol"


def workload_name(key, wl):
    if wl["kind"] == "spatial":
        head = f"spatial-{wl['ndim']}d-{wl['kernel']}"
    elif wl["kind"] == "coulomb":
        head = f"electrostatics-{wl['ndim']}d-coulomb-diag{wl['diag']:g}"
    else:
        head = f"electrodynamics-{wl['ndim']}d-sin-k{wl['wave_k']:g}"
    return (f"{head}-N{wl['N']}-nb{wl['nb']}-maxrank{wl['maxrank']}"
            f"-os{wl['oversample']}-tol{wl['tol']:g}")


# ----------------------------------------------------------- problem setup

_keep = []   # ctypes objects that must outlive the problems


def make_problem(lib, wl, seed=0):
    """The workload's problem built with the library's own host API."""
    import starsh_b200 as sb
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    kern = c_void_p()
    if wl["kind"] == "spatial":
        data = POINTER(sb.SSData)()
        assert lib.starsh_ssdata_generate(byref(data), wl["N"], wl["ndim"],
                                          wl["beta"], wl["nu"], 0.0,
                                          wl["place"], 1.0) == 0
        ktype = {"exp": 1, "sqexp": 2, "matern": 3}[wl["kernel"]]
        assert lib.starsh_ssdata_get_kernel(byref(kern), data, ktype) == 0
    elif wl["kind"] == "coulomb":
        data = POINTER(sb.Particles)()
        assert lib.starsh_particles_generate(byref(data), wl["N"], wl["ndim"],
                                             wl["place"]) == 0
        # 1/r with a regularised (unit) diagonal: a kernel handle registered
        # with the device Coulomb family and its r = 0 value
        handle = sb.KERNEL(lambda *a: None)
        _keep.append(handle)
        kern = c_void_p(ctypes.cast(handle, c_void_p).value)
        assert lib.starsh_b200_kernel_register(kern, sb.FAMILY["coulomb"],
                                               wl["diag"]) == 0
    else:
        data = POINTER(sb.EDData)()
        gen = lib.starsh_eddata_generate
        gen.restype = ctypes.c_int
        gen.argtypes = [POINTER(POINTER(sb.EDData)), sb.STARSH_int,
                        ctypes.c_int, ctypes.c_double, ctypes.c_double,
                        ctypes.c_int]
        assert gen(byref(data), wl["N"], wl["ndim"], wl["wave_k"],
                   wl["diag"], wl["place"]) == 0
        assert lib.starsh_eddata_get_kernel(byref(kern), data, sb.SIN) == 0
    shape = (sb.STARSH_int * 2)(wl["N"], wl["N"])
    P = POINTER(sb.Problem)()
    assert lib.starsh_problem_new(byref(P), 2, shape, b"N", b"d", data, data,
                                  kern, b"bench") == 0
    C = POINTER(sb.Cluster)()
    assert lib.starsh_cluster_new_plain(byref(C), data, wl["N"], wl["nb"]) == 0
    _keep.append(shape)
    return dict(data=data, P=P, C=C)


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
                self.samples.append([x.strip() for x in out.split(",")])
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
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        good = [s for s in self.samples if len(s) > 7]
        sm = [v for v in (num(s[1]) for s in good) if v is not None]
        mx = [v for v in (num(s[2]) for s in good) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for s in good for i in range(4)
                          if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


# --------------------------------------------------------- CPU baseline

def cpu_reference_run(key, n, threads):
    """The reference's OpenMP RSVD path (compiled from its sources into
    oracle/_ref) on an N-point instance of the workload, in a subprocess
    with OMP_NUM_THREADS=threads and OPENBLAS_NUM_THREADS=1."""
    wl = WORKLOADS[key]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads),
               OPENBLAS_NUM_THREADS="1", STARSH_BACKEND="OPENMP",
               STARSH_LRENGINE="RSVD", STARSH_OVERSAMPLE=str(wl["oversample"]))
    cmd = [sys.executable, os.path.abspath(__file__), "--_cpu-run", str(n),
           "--workload", key]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True,
                         timeout=900)
    for line in out.stdout.splitlines():
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError(f"CPU reference run failed: {out.stderr[-2000:]}")


def _cpu_run(key, n):
    """Child process body of cpu_reference_run (reference library only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from harness import RefProblem
    wl = WORKLOADS[key]
    ref = oracle.Ref()
    if wl["kind"] == "spatial":
        pr = RefProblem(ref, "spatial", n, wl["nb"], ndim=wl["ndim"],
                        place=wl["place"], beta=wl["beta"], nu=wl["nu"],
                        kernel_name=wl["kernel"])
    elif wl["kind"] == "coulomb":
        # the reference kernel wrapped to put 1 on the r = 0 entries
        orc = oracle.Oracle()
        ptr = ctypes.c_void_p.in_dll(orc.lib, "oracle_coulomb_ref_kernel")
        ptr.value = ref.symbol(
            f"starsh_esdata_block_coulomb_potential_kernel_{wl['ndim']}d")
        wrap = ctypes.c_void_p(ctypes.cast(orc.lib.oracle_coulomb_unit_diag,
                                           ctypes.c_void_p).value)
        pr = RefProblem(ref, "custom", n, wl["nb"],
                        data=ref.particles_data(n, wl["ndim"], wl["place"]),
                        kernel=wrap)
    else:
        pr = RefProblem(ref, "sin", n, wl["nb"], ndim=wl["ndim"],
                        place=wl["place"], wave_k=wl["wave_k"], diag=wl["diag"])
    t0 = time.perf_counter()
    M = ref.approximate(pr.F, wl["maxrank"], wl["tol"],
                        oversample=wl["oversample"])
    dt = time.perf_counter() - t0
    err = ref.dfe(M) if n <= wl.get("cpu_n") else None
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

def reference_arm(args, key, wl, threads):
    """--impl reference: the reference's OpenMP RSVD on the host cores, one
    bounded sample of the workload (same tiles, sketch width, tol) per
    step."""
    n = wl.get("cpu_step_n")
    if not n:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference kernel needs GSL, which is not installed"}))
        return
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_run(key, n, threads)
        if i >= args.warmup:
            times.append(r["seconds"])
    t = statistics.mean(times)
    v = n ** 2 / t / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v,
        "unit": "Mentries/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": dict(workload=workload_name(key, wl), sample_N=n,
                       engine="starsh_blrm__drsdd_omp"),
        "cpu_baseline": {"value": v, "unit": "Mentries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"N={n} ({(n // wl['nb']) ** 2} tiles of {wl['nb']}x{wl['nb']})"},
        "e2e": {"value": v, "unit": "Mentries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--engine", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="c2-sqexp", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=0,
                    help="points (a smaller N profiles the same kernels)")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline leg")
    ap.add_argument("--_cpu-run", type=int, default=0, dest="cpu_run")
    args = ap.parse_args()
    key = args.workload
    if args.cpu_run:
        _cpu_run(key, args.cpu_run)
        return

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    wl = dict(WORKLOADS[key])
    if args.n:
        wl["N"] = args.n
    threads = len(os.sched_getaffinity(0))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, key, wl, threads)
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

    def measure(engine, clocks=None, keep=False):
        """W warm-up and K timed device-resident approximations; mean device
        time, per-step stats, FP64 error of the last result."""
        for _ in range(args.warmup):
            M, F, *_ = step(engine, 0)
            free(M, F)
        barrier()
        times, sts = [], []
        with (clocks if clocks is not None else _Null()):
            for i in range(args.steps):
                M, F, dt, host, st = step(engine, 0)
                times.append(dt)
                sts.append(st)
                if i + 1 < args.steps:
                    free(M, F)
        barrier()
        err = lib.starsh_blrm__dfe_b200(M)
        if keep:
            return statistics.mean(times), sts, err, (M, F)
        free(M, F)
        return statistics.mean(times), sts, err, None

    clocks = ClockSampler(local)
    t_dev, sts, err, kept = measure(chosen, clocks, keep=bool(wl.get("dmml_nrhs")))
    last = sts[-1]
    if chosen != sb.ENGINE_FP64:
        t_plain, _, err_plain, _ = measure(sb.ENGINE_FP64)
    else:
        t_plain, err_plain = t_dev, err

    # TLR-by-dense product on the device-resident factors
    dmml = None
    if kept is not None:
        M, F = kept
        nrhs = wl["dmml_nrhs"]
        A = torch.randn(nrhs, wl["N"], dtype=torch.float64, device="cuda")
        B = torch.zeros(nrhs, wl["N"], dtype=torch.float64, device="cuda")
        for _ in range(2):
            assert lib.starsh_b200_blrm_dmml_device(M, nrhs, 1.0, A.data_ptr(),
                                                    wl["N"], 0.0, B.data_ptr(),
                                                    wl["N"], None) == 0
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        s.record(stream)
        for _ in range(reps):
            lib.starsh_b200_blrm_dmml_device(M, nrhs, 1.0, A.data_ptr(), wl["N"],
                                             0.0, B.data_ptr(), wl["N"], None)
        e.record(stream)
        e.synchronize()
        t = s.elapsed_time(e) / 1e3 / reps
        Mc = M.contents
        Fc = Mc.format.contents
        R = Fc.row_cluster.contents
        flops = 0.0
        byts = 2.0 * wl["N"] * nrhs * 8
        for b in range(Fc.nblocks_far):
            i, j = Fc.block_far[2 * b], Fc.block_far[2 * b + 1]
            r = Mc.far_rank[b]
            flops += 2.0 * (R.size[i] + R.size[j]) * r * nrhs
            byts += (R.size[i] + R.size[j]) * r * 8.0
        for b in range(Fc.nblocks_near):
            i, j = Fc.block_near[2 * b], Fc.block_near[2 * b + 1]
            flops += 2.0 * R.size[i] * R.size[j] * nrhs
            byts += R.size[i] * R.size[j] * 8.0
        dmml = {"nrhs": nrhs, "ms": t * 1e3, "gflops": flops / t / 1e9,
                "hbm_gbs": byts / t / 1e9,
                "bound": "fp64 tensor" if flops / byts > 5 else "hbm"}
        free(M, F)

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
    # roofline of the sketch GEMM (FP64 DMMA)
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
        "data": "synthetic (seeded point generators)",
        "config": {"workload": workload_name(key, wl),
                   "engine": ("mixed (adaptive sketch)" if chosen == sb.ENGINE_MIXED
                              else "fp64 (fixed sketch width)"),
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "tiles": int(last.tiles), "false_far": int(last.false_far),
                   "entries": int(entries),
                   "l2": "flushed (256 MB write) before every step",
                   "mean_rank": last.rank_sum / max(1, last.tiles - last.false_far),
                   "max_rank": last.max_rank,
                   "sketch_columns_per_tile": last.sketch_flops / max(1.0, 2.0 * last.tiles * wl["nb"] ** 2)},
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
    if dmml:
        line["dmml"] = dmml
    if world == 1 and not args.no_cpu:
        n = wl.get("cpu_n")
        if not n:
            line["cpu_baseline"] = {"value": None, "kind": "reference",
                                    "unavailable": "reference kernel needs GSL, which is not installed"}
        else:
            try:
                r = cpu_reference_run(key, n, threads)
                line["cpu_baseline"] = {
                    "value": r["entries"] / r["seconds"] / 1e6, "unit": "Mentries/s",
                    "cores": threads, "kind": "reference",
                    "sample": f"N={n}: {(n // wl['nb']) ** 2} tiles of {wl['nb']}x{wl['nb']}, same kernel/maxrank/oversample/tol, starsh_blrm__drsdd_omp",
                    "rel_err": r["rel_err"], "seconds": r["seconds"]}
            except Exception as exc:   # reported, not fatal
                line["cpu_baseline"] = {"value": None, "error": str(exc)[:300]}
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
