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


# ------------------------------------------- many-problem workloads (C4/C5)

C4 = dict(problems=512, nmin=1024, nmax=16384, tols=(1e-3, 1e-5, 1e-7),
          kernels=("exp", "sqexp", "matern", "coulomb", "rbf"), oversample=10)
C5 = dict(rate=200.0, seconds=60.0, median=8192, sigma_log=0.5, nmin=2048,
          nmax=65536, tols=(1e-4, 1e-6), nrhs=32, budget=120e9, oversample=10)


def tile_size(n):
    """Block size for an N-point problem (from {256, 512, 1024}): at least
    about 16 x 16 tiles for small problems, 1024 above 8192 points."""
    return 256 if n <= 2048 else 512 if n <= 8192 else 1024


def _malloc_doubles(values):
    """A libc-malloc'd copy (the library frees point arrays it owns)."""
    libc = ctypes.CDLL("libc.so.6")
    libc.malloc.restype = c_void_p
    ptr = libc.malloc(ctypes.c_size_t(8 * len(values)))
    arr = (ctypes.c_double * len(values)).from_address(ptr)
    arr[:] = list(map(float, values))
    return ctypes.cast(ptr, POINTER(ctypes.c_double))


def sphere_points(rng, n):
    """n points uniform on the surfaces of 1-8 spheres (radius U[0.05, 0.2],
    centres uniform in the unit cube)."""
    import numpy as np
    ns = int(rng.integers(1, 9))
    centres = rng.uniform(0.0, 1.0, (ns, 3))
    radii = rng.uniform(0.05, 0.2, ns)
    which = np.sort(rng.integers(0, ns, n))
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return centres[which] + radii[which, None] * v


TUNE_NB = (256, 512, 1024)


def tuned_tile_size(lib, P, tol):
    """The library autotuner's block size for problem P among TUNE_NB (each
    with maxrank min(nb / 2, 256)), measured with the mixed engine."""
    import starsh_b200 as sb
    k = len(TUNE_NB)
    cands = (ctypes.c_int * k)(*TUNE_NB)
    ranks = (ctypes.c_int * k)(*[min(nb // 2, 256) for nb in TUNE_NB])
    best = ctypes.c_int(0)
    assert lib.starsh_b200_autotune_tile(P, k, cands, ranks, tol,
                                         sb.ENGINE_MIXED, byref(best),
                                         None) == 0, lib.starsh_b200_last_error()
    return best.value


def mixed_problem(lib, seed, n, kernel, ndim, coulomb_handle, tol=None,
                  tune=False):
    """One problem of the many-problem workloads, built with the library's
    own host API: spatial kernels on a jittered grid (N rounded to a
    square / cube), 1/r (unit diagonal) on jittered particles, Gaussian RBF
    (radius 0.1) on points on spheres, all Z-sorted.  The block size comes
    from the library's autotuner when `tune`, else from tile_size()."""
    import numpy as np
    import starsh_b200 as sb
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    kern = c_void_p()
    if kernel in ("exp", "sqexp", "matern"):
        side = max(2, int(round(n ** (1.0 / ndim))))
        n = side ** ndim
        data = POINTER(sb.SSData)()
        nu = 1.5 if kernel == "matern" else 0.5
        assert lib.starsh_ssdata_generate(byref(data), n, ndim, 0.1, nu, 0.0,
                                          6, 1.0) == 0
        ktype = {"exp": 1, "sqexp": 2, "matern": 3}[kernel]
        assert lib.starsh_ssdata_get_kernel(byref(kern), data, ktype) == 0
    elif kernel == "coulomb":
        side = max(2, int(round(n ** (1.0 / ndim))))
        n = side ** ndim
        data = POINTER(sb.Particles)()
        assert lib.starsh_particles_generate(byref(data), n, ndim, 6) == 0
        kern = c_void_p(ctypes.cast(coulomb_handle, c_void_p).value)
    else:
        rng = np.random.default_rng(seed)
        pts = sphere_points(rng, n)
        part = POINTER(sb.Particles)()
        assert lib.starsh_particles_init(byref(part), n, 3,
                                         _malloc_doubles(pts.T.ravel())) == 0
        assert lib.starsh_particles_zsort_inplace(part) == 0
        soa = np.ctypeslib.as_array(part.contents.point, shape=(3 * n,))
        mesh = soa.reshape(3, n).T.ravel()          # point-major
        data = POINTER(sb.MDData)()
        assert lib.starsh_mddata_init(byref(data), n, _malloc_doubles(mesh),
                                      0, 1, 0, 0.0, 0.1, 0.0) == 0
        kern = c_void_p(sb.kernel_symbol(lib, "starsh_generate_3d_virus"))
        _keep.append(part)
    shape = (sb.STARSH_int * 2)(n, n)
    P = POINTER(sb.Problem)()
    assert lib.starsh_problem_new(byref(P), 2, shape, b"N", b"d", data, data,
                                  kern, b"mixed") == 0
    nb = tuned_tile_size(lib, P, tol) if tune else tile_size(n)
    C = POINTER(sb.Cluster)()
    assert lib.starsh_cluster_new_plain(byref(C), data, n, nb) == 0
    _keep.append(shape)
    return dict(data=data, P=P, C=C, n=n, nb=nb, maxrank=min(nb // 2, 256),
                kernel=kernel, ndim=ndim)


def c4_specs():
    """The 512 problems: N log-uniform in [1024, 16384], kernel and tol
    uniform over their sets, seed = problem index."""
    import numpy as np
    out = []
    for p in range(C4["problems"]):
        rng = np.random.default_rng(p)
        n = int(round(np.exp(rng.uniform(np.log(C4["nmin"]), np.log(C4["nmax"])))))
        kernel = C4["kernels"][int(rng.integers(len(C4["kernels"])))]
        tol = C4["tols"][int(rng.integers(len(C4["tols"])))]
        ndim = 3 if kernel in ("coulomb", "rbf") else 2
        out.append(dict(seed=p, n=n, kernel=kernel, tol=tol, ndim=ndim, t=0.0))
    return out


def c5_specs(seconds, rate, seed=12345):
    """Poisson arrivals: N lognormal (median 8192, sigma_log 0.5) clipped to
    [2048, 65536], 2-D or 3-D, kernel from the C4 set, tol in {1e-4, 1e-6}."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        n = int(np.clip(np.exp(rng.normal(np.log(C5["median"]), C5["sigma_log"])),
                        C5["nmin"], C5["nmax"]))
        kernel = C4["kernels"][int(rng.integers(len(C4["kernels"])))]
        ndim = 3 if kernel == "rbf" else int(rng.integers(2, 4))
        tol = C5["tols"][int(rng.integers(len(C5["tols"])))]
        out.append(dict(seed=len(out), n=n, kernel=kernel, tol=tol, ndim=ndim,
                        t=t))
    return out


def build_mixed(lib, specs, coulomb_handle, tune=False):
    out = []
    for sp in specs:
        pr = mixed_problem(lib, sp["seed"], sp["n"], sp["kernel"], sp["ndim"],
                           coulomb_handle, tol=sp["tol"], tune=tune)
        pr["tol"] = sp["tol"]
        pr["t"] = sp["t"]
        out.append(pr)
    return out


def reference_arm_mixed(args, key, threads):
    """--impl reference for c4-batch / c5-serve: the reference's OpenMP RSVD
    (plus its dmml with 32 right-hand sides for c5) one problem at a time on
    the host cores, over the first exp/sqexp problems of the workload (the
    reference has no Matern without GSL; its other kernels need wrappers
    this sample leaves out)."""
    specs = c4_specs() if key == "c4-batch" else c5_specs(C5["seconds"], C5["rate"])
    sample = [sp for sp in specs if sp["kernel"] in ("exp", "sqexp")][:6]
    for sp in sample:
        side = max(2, int(round(sp["n"] ** (1.0 / sp["ndim"]))))
        sp["n"] = side ** sp["ndim"]
        sp["nb"] = tile_size(sp["n"])
        sp["maxrank"] = min(sp["nb"] // 2, 256)
        sp["nrhs"] = C5["nrhs"] if key == "c5-serve" else 0
    times, entries, lat = [], 0, []
    for i in range(args.warmup + args.steps):
        env = dict(os.environ, OMP_NUM_THREADS=str(threads),
                   OPENBLAS_NUM_THREADS="1", STARSH_MIXED_SPECS=json.dumps(sample))
        out = subprocess.run([sys.executable, os.path.abspath(__file__),
                              "--_cpu-run", "1", "--workload", key], env=env,
                             capture_output=True, text=True, timeout=900)
        r = next(json.loads(x) for x in out.stdout.splitlines() if x.startswith("{"))
        if i >= args.warmup:
            times.append(r["seconds"])
            lat += r["latency_ms"]
        entries = r["entries"]
    t = statistics.mean(times)
    v = entries / t / 1e6
    import numpy as np
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mentries/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload=key, engine="starsh_blrm__drsdd_omp",
                       sample=[(sp["n"], sp["kernel"], sp["tol"]) for sp in sample]),
        "cpu_baseline": {"value": v, "unit": "Mentries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{len(sample)} exp/sqexp problems of the workload, one at a time"},
        "e2e": {"value": v, "unit": "Mentries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}
    if key == "c5-serve":
        line["latency_ms"] = {"p50": float(np.percentile(lat, 50)),
                              "p99": float(np.percentile(lat, 99)),
                              "note": "service time of one request alone, no queueing"}
    print(json.dumps(line))


def _cpu_run_mixed():
    """Child process body of reference_arm_mixed (reference library only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    import oracle
    from harness import RefProblem
    ref = oracle.Ref()
    specs = json.loads(os.environ["STARSH_MIXED_SPECS"])
    total, entries, lat = 0.0, 0, []
    for sp in specs:
        pr = RefProblem(ref, "spatial", sp["n"], sp["nb"], ndim=sp["ndim"],
                        place=6, beta=0.1, nu=0.5, kernel_name=sp["kernel"],
                        seed=sp["seed"])
        A = np.random.default_rng(1).standard_normal((sp["n"], max(1, sp["nrhs"])))
        t0 = time.perf_counter()
        M = ref.approximate(pr.F, sp["maxrank"], sp["tol"], oversample=10)
        if sp["nrhs"]:
            ref.dmml(M, A)
        dt = time.perf_counter() - t0
        total += dt
        lat.append(dt * 1e3)
        entries += sp["n"] ** 2
    print(json.dumps({"seconds": total, "entries": entries, "latency_ms": lat}))


def run_c4(args, lib, stream, clocks, torch):
    """512 independent problems in one batched call (the mixed engine),
    against the FP64 engine one problem at a time."""
    import starsh_b200 as sb
    handle = sb.KERNEL(lambda *a: None)
    _keep.append(handle)
    assert lib.starsh_b200_kernel_register(
        c_void_p(ctypes.cast(handle, c_void_p).value), sb.FAMILY["coulomb"],
        1.0) == 0
    lib.starsh_set_oversample(str(C4["oversample"]).encode())
    t_build = time.perf_counter()
    probs = build_mixed(lib, c4_specs(), handle, tune=args.tune)
    t_build = time.perf_counter() - t_build
    n = len(probs)
    ranks = (ctypes.c_int * n)(*[p["maxrank"] for p in probs])
    tols = (ctypes.c_double * n)(*[p["tol"] for p in probs])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def batched(engine):
        Fs = (POINTER(sb.Blrf) * n)(*[new_format(lib, p) for p in probs])
        Ms = (POINTER(sb.Blrm) * n)()
        flush.zero_()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        info = lib.starsh_b200_approximate_batch(n, Ms, Fs, ranks, tols, None,
                                                 engine, 0)
        e.record(stream)
        e.synchronize()
        assert info == 0, lib.starsh_b200_last_error()
        return Ms, Fs, s.elapsed_time(e) / 1e3, sb.stats(lib)

    def sequential(engine):
        total = 0.0
        for p in probs:
            F = new_format(lib, p)
            M = POINTER(sb.Blrm)()
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            assert lib.starsh_b200_approximate(byref(M), F, p["maxrank"],
                                               p["tol"], 0, engine, 0) == 0
            e.record(stream)
            e.synchronize()
            total += s.elapsed_time(e) / 1e3
            lib.starsh_blrm_free(M)
            lib.starsh_blrf_free(F)
        return total

    def free_all(Ms, Fs):
        for i in range(n):
            lib.starsh_blrm_free(Ms[i])
            lib.starsh_blrf_free(Fs[i])

    for _ in range(args.warmup):
        free_all(*batched(sb.ENGINE_MIXED)[:2])
    times, st = [], None
    with clocks:
        for i in range(args.steps):
            Ms, Fs, t, st = batched(sb.ENGINE_MIXED)
            times.append(t)
            if i + 1 < args.steps:
                free_all(Ms, Fs)
    worst = 0.0
    ok = True
    for i in range(n):
        err = lib.starsh_blrm__dfe_b200(Ms[i])
        ok &= 0 <= err <= probs[i]["tol"]
        worst = max(worst, err / probs[i]["tol"])
    free_all(Ms, Fs)
    t_dev = statistics.mean(times)
    Ms, Fs, t_fp64_batched, _ = batched(sb.ENGINE_FP64)
    free_all(Ms, Fs)
    t_seq_fp64 = sequential(sb.ENGINE_FP64)
    t_seq_mixed = sequential(sb.ENGINE_MIXED)
    entries = st.entries
    kinds = {k: sum(1 for p in probs if p["kernel"] == k) for k in C4["kernels"]}
    line = {
        "metric": METRIC, "value": entries / t_dev / 1e6 if ok else None,
        "unit": "Mentries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_dev * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded point generators)",
        "config": {"workload": "uneven-batch-512-problems-N1024-16384",
                   "engine": "mixed (adaptive sketch), one batched call",
                   "problems": n, "kernels": kinds,
                   "tols": list(C4["tols"]), "tile_sizes": list(TUNE_NB),
                   "tile_choice": ("autotuned (starsh_b200_autotune_tile)"
                                   if args.tune else "fixed rule by N"),
                   "tiles_chosen": {str(nb): sum(1 for p in probs if p["nb"] == nb)
                                    for nb in TUNE_NB},
                   "entries": int(entries), "tiles": int(st.tiles),
                   "false_far": int(st.false_far), "batches": int(st.batches),
                   "l2": "flushed (256 MB write) before every step",
                   "host_build_s": t_build,
                   "build_includes_tuning": bool(args.tune)},
        "accepted": bool(ok), "worst_err_over_tol": worst,
        "fp64_batched": {"value": entries / t_fp64_batched / 1e6,
                         "ms": t_fp64_batched * 1e3},
        "plain_fp64": {"value": entries / t_seq_fp64 / 1e6,
                       "ms_per_step": t_seq_fp64 * 1e3,
                       "what": "FP64 engine, one problem at a time",
                       "chosen_over_plain": t_seq_fp64 / t_dev},
        "mixed_one_at_a_time": {"value": entries / t_seq_mixed / 1e6,
                                "ms": t_seq_mixed * 1e3},
        "phases_ms": {"gen": st.gen_ms, "basis": st.basis_ms,
                      "project": st.project_ms, "svd": st.svd_ms,
                      "output": st.output_ms},
        "gpu_launches": int(st.kernel_launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def serve(lib, reqs, engine, max_group, A):
    """Replays the arrivals against a server; returns latencies (ms),
    entries and the wall time from the first submit to the last
    completion."""
    import numpy as np
    import starsh_b200 as sb
    srv = c_void_p()
    assert lib.starsh_b200_server_new(byref(srv), C5["budget"], engine,
                                      max_group) == 0
    fmts = [new_format(lib, r) for r in reqs]
    outs = [None] * len(reqs)
    tickets = [None] * len(reqs)
    nrhs = C5["nrhs"]
    lda = A.shape[0]

    def submitter():
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            dt = r["t"] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            outs[i] = np.empty((r["n"], nrhs), order="F")
            t = ctypes.c_longlong()
            # keep = 1: the factors stay resident after the products (the
            # caller releases them once it has the result)
            assert lib.starsh_b200_server_submit(
                srv, fmts[i], r["maxrank"], r["tol"], nrhs, A.ctypes.data, lda,
                outs[i].ctypes.data, r["n"], 1, byref(t)) == 0
            tickets[i] = t.value

    t_start = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    lat, status = [], []
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        L = ctypes.c_double()
        M = POINTER(sb.Blrm)()
        status.append(lib.starsh_b200_server_wait(srv, tickets[i], byref(M),
                                                  byref(L)))
        lat.append(L.value)
        if M:
            lib.starsh_b200_server_release(srv, M)
        outs[i] = None
    th.join()
    wall = time.perf_counter() - t_start
    st = sb.ServerStats()
    lib.starsh_b200_server_get_stats(srv, byref(st))
    lib.starsh_b200_server_free(srv)
    for F in fmts:
        lib.starsh_blrf_free(F)
    return np.array(lat), status, st, wall


def single_request_ms(lib, req, A, reps):
    """Latency of one request submitted alone to an idle server, again and
    again (each waits for the previous one); the best after the first."""
    import numpy as np
    import starsh_b200 as sb
    srv = c_void_p()
    assert lib.starsh_b200_server_new(byref(srv), C5["budget"], sb.ENGINE_MIXED,
                                      0) == 0
    nrhs = C5["nrhs"]
    lats = []
    for _ in range(reps):
        F = new_format(lib, req)
        out = np.empty((req["n"], nrhs), order="F")
        t = ctypes.c_longlong()
        assert lib.starsh_b200_server_submit(
            srv, F, req["maxrank"], req["tol"], nrhs, A.ctypes.data, A.shape[0],
            out.ctypes.data, req["n"], 0, byref(t)) == 0
        L = ctypes.c_double()
        M = POINTER(sb.Blrm)()
        assert lib.starsh_b200_server_wait(srv, t.value, byref(M), byref(L)) == 0
        lats.append(L.value)
        lib.starsh_blrf_free(F)
    lib.starsh_b200_server_free(srv)
    return float(min(lats[1:]))


def run_c5(args, lib, clocks):
    """Poisson arrivals replayed against the serving loop (mixed engine,
    continuous batching), then against the FP64 engine one request at a
    time."""
    import numpy as np
    import starsh_b200 as sb
    handle = sb.KERNEL(lambda *a: None)
    _keep.append(handle)
    assert lib.starsh_b200_kernel_register(
        c_void_p(ctypes.cast(handle, c_void_p).value), sb.FAMILY["coulomb"],
        1.0) == 0
    lib.starsh_set_oversample(str(C5["oversample"]).encode())
    seconds, rate = args.serve_seconds, args.serve_rate
    reqs = build_mixed(lib, c5_specs(seconds, rate), handle, tune=args.tune)
    A = np.asfortranarray(np.random.default_rng(1).standard_normal(
        (C5["nmax"], C5["nrhs"])))
    # warm-up on the first few requests
    serve(lib, reqs[:min(8, len(reqs))], sb.ENGINE_MIXED, 0, A)
    with clocks:
        lat, status, st, wall = serve(lib, reqs, sb.ENGINE_MIXED, 0, A)
    # the FP64 comparison over the first 10 s of arrivals (one request at
    # a time it takes far longer than the stream)
    reqs_p = [r for r in reqs if r["t"] < 10.0]
    lat_p, status_p, st_p, wall_p = serve(lib, reqs_p, sb.ENGINE_FP64, 1, A)
    ok = all(x == 0 for x in status)
    # the single-request floor: one request alone on an idle one-worker
    # server whose worker has served the same request before (2-D square
    # exponential, tol 1e-4), per N; best of three after the first
    floor = {}
    workers = os.environ.get("STARSH_B200_SERVER_WORKERS")
    os.environ["STARSH_B200_SERVER_WORKERS"] = "1"
    try:
        for nf in (4096, 16384, 65536):
            sp = [dict(seed=99, n=nf, kernel="sqexp", tol=1e-4, ndim=2, t=0.0)]
            one = build_mixed(lib, sp, handle, tune=args.tune)
            floor[str(one[0]["n"])] = single_request_ms(lib, one[0], A, reps=4)
    finally:
        if workers is None:
            del os.environ["STARSH_B200_SERVER_WORKERS"]
        else:
            os.environ["STARSH_B200_SERVER_WORKERS"] = workers

    def pct(v):
        return {"p50": float(np.percentile(v, 50)),
                "p99": float(np.percentile(v, 99)),
                "mean": float(np.mean(v)), "max": float(np.max(v))}
    big = np.array([r["n"] for r in reqs]) >= 32768
    line = {
        "metric": "served Mentries/s and request latency (submit to 32 matvecs done)",
        "value": st.entries / wall / 1e6 if ok else None, "unit": "Mentries/s",
        "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": wall * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded point generators)",
        "config": {"workload": f"serving-poisson-{rate:g}rps-{seconds:g}s",
                   "requests": len(reqs), "offered_rate_rps": rate,
                   "workers": int(os.environ.get("STARSH_B200_SERVER_WORKERS", "3")),
                   "group_entries_cap": float(os.environ.get("STARSH_B200_SERVER_GROUP_ENTRIES", "5e8")),
                   "N": "lognormal median 8192, sigma_log 0.5, clipped [2048, 65536]",
                   "tols": list(C5["tols"]), "nrhs": C5["nrhs"],
                   "hbm_budget_bytes": C5["budget"], "engine": "mixed, continuous batching"},
        "latency_ms": pct(lat),
        "latency_ms_N_ge_32768": pct(lat[big]) if big.any() else None,
        "slowest_requests": [
            {"n": int(reqs[i]["n"]), "nb": int(reqs[i]["nb"]),
             "kernel": reqs[i]["kernel"],
             "ndim": int(reqs[i]["ndim"]), "tol": reqs[i]["tol"],
             "arrival_s": float(reqs[i]["t"]), "latency_ms": float(lat[i])}
            for i in np.argsort(lat)[::-1][:8]],
        "single_request_floor_ms": floor,
        "floor_what": "one 2-D square-exponential request (tol 1e-4, 32 matvecs) alone on an idle one-worker server that served it before (best of 3 after a first), by N",
        "served_rps": len(reqs) / wall, "groups": int(st.groups),
        "server_means_ms": {
            "queue_per_request": st.queue_ms / max(1, len(reqs)),
            "approx_per_group": st.approx_ms / max(1, st.groups),
            "products_per_group": st.products_ms / max(1, st.groups),
            "requests_per_group": len(reqs) / max(1, st.groups),
            "worker_busy_frac": st.busy_ms / 1e3 / wall / max(1, int(
                os.environ.get("STARSH_B200_SERVER_WORKERS", "3")))},
        "failed": int(st.failed),
        "peak_resident_bytes": st.peak_resident_bytes,
        "plain_fp64_one_at_a_time": {
            "value": st_p.entries / wall_p / 1e6, "latency_ms": pct(lat_p),
            "served_rps": len(reqs_p) / wall_p, "wall_s": wall_p,
            "requests": len(reqs_p), "what": "the arrivals of the first 10 s"},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


# ------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed
    region: one looping `nvidia-smi -lms 200` started before it (its start-up
    is over when the first sample arrives, before any timed step) and
    stopped after it."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._start = 0
        self._proc = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])
            self._first.set()
        self._first.set()

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(10.0)
        self._start = len(self.samples)
        return self

    def __exit__(self, *a):
        if self._proc is None:
            return
        self._proc.terminate()
        try:
            self._proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self._proc.kill()
            self._proc.wait()
        self._t.join(timeout=5)

    def summary(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        # samples of the timed region (the last earlier one if it was
        # shorter than the sampling period)
        timed = self.samples[self._start:] or self.samples[-1:]
        good = [s for s in timed if len(s) > 7]
        sm = [v for v in (num(s[1]) for s in good) if v is not None]
        mx = [v for v in (num(s[2]) for s in good) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for s in good for i in range(4)
                          if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(timed)}


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


# ------------------------------------------------------------- replicas

def replica_rates(times, entries, world, device):
    """Whole-job Mentries/s of `world` independent replicas (one per rank):
    the entries of all ranks over the slowest rank's time, for each timed
    quantity in `times` (seconds).  Returns (rates, max times).  Every rank
    takes the same two all-reduce steps."""
    if world > 1:
        import torch
        import torch.distributed as dist
        tt = torch.tensor(list(times), dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ee = torch.tensor([float(entries)], dtype=torch.float64, device=device)
        dist.all_reduce(ee, op=dist.ReduceOp.SUM)
        times, total = tt.tolist(), ee.item()
    else:
        times, total = list(times), float(entries)
    return [total / t / 1e6 for t in times], times


# ---------------------------------------------------- sketch precision study

def precision_study(lib, wl, prob, torch, ntiles=64, seed=7):
    """Sketch precisions on a sample of the workload's far tiles: Y = D
    Omega with BF16, BF16x3 and TF32x3 inputs and FP32 accumulation (each
    emulated exactly: the split operands' products are exact in FP32, so an
    FP32 GEMM of them accumulates as the tensor cores' FP32 path does), the
    library's 40-bit integer slices of D (rounding as in the int8 sketch),
    and FP64; then for each the same FP64 basis (Householder QR of Y),
    projection B = Q^T D and rank rule (dsvfr tail plus the energy outside
    the basis, as the library's rank cut).  Reports per precision the share
    of tiles the rule accepts, their mean rank, and the largest energy
    outside the basis over tol^2 ||D||^2 (the sketch error the FP64 steps
    cannot repair), plus FP32-accumulate GEMM rates at the batch shape."""
    import numpy as np
    import starsh_b200 as sb
    tol, k = wl["tol"], wl["maxrank"] + wl["oversample"]
    C = prob["C"].contents
    nt = C.nblocks
    if wl["kind"] == "coulomb":
        fn = sb.kernel_symbol(lib, "starsh_esdata_block_coulomb_potential_kernel_3d")
    elif wl["kind"] == "spatial":
        name = {"exp": "exp", "sqexp": "sqrexp", "matern": "matern"}[wl["kernel"]]
        fn = sb.kernel_symbol(lib, f"starsh_ssdata_block_{name}_kernel_{wl['ndim']}d")
    else:
        fn = sb.kernel_symbol(lib, "starsh_eddata_block_sin_kernel_3d")
    gen = sb.KERNEL(fn)
    rng = np.random.default_rng(seed)
    pairs = []
    while len(pairs) < ntiles:
        i, j = (int(x) for x in rng.integers(0, nt, 2))
        if i != j:
            pairs.append((i, j))
    piv = np.ctypeslib.as_array(C.pivot, shape=(C.ndata,))
    dev = "cuda"
    f64 = torch.float64
    g = torch.Generator(device=dev).manual_seed(seed)
    n_b = int(C.size[0])
    omega = torch.randn(n_b, k, dtype=f64, device=dev, generator=g)
    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False

    def bf16(x):
        return x.to(torch.bfloat16).to(torch.float32)

    def tf32(x):
        # round-to-nearest to 10 explicit mantissa bits
        xi = x.to(torch.float32).view(torch.int32)
        xi = (xi + 0x1000) & ~0x1FFF
        return xi.view(torch.float32)

    def split3(x, rnd):
        a = rnd(x)
        r = x - a.to(f64)
        b = rnd(r)
        r = r - b.to(f64)
        return a, b, rnd(r)

    def sketch(D, how):
        if how == "fp64":
            return D @ omega
        if how == "int40":
            e = torch.ceil(torch.log2(D.abs().amax(dim=1, keepdim=True).clamp_min(1e-300)))
            s = torch.pow(2.0, 39 - e)
            q = torch.round(D * s)
            return (q @ torch.round(32 * omega).clamp(-127, 127)) / s / 32
        om = omega.to(torch.float32)
        if how == "bf16":
            return (bf16(D) @ bf16(om)).to(f64)
        parts = split3(D, bf16 if how == "bf16x3" else tf32)
        w = bf16(om) if how == "bf16x3" else tf32(om)
        acc = torch.zeros(D.shape[0], k, dtype=torch.float32, device=dev)
        for pt in parts:
            acc += pt @ w
        return acc.to(f64)

    hows = ["fp64", "int40", "tf32x3", "bf16x3", "bf16"]
    res = {h: {"accepted": 0, "ranks": [], "outside_over_budget": 0.0} for h in hows}
    for (i, j) in pairs:
        m, n = int(C.size[i]), int(C.size[j])
        ri = piv[C.start[i]:C.start[i] + m].astype(np.int64).copy()
        ci = piv[C.start[j]:C.start[j] + n].astype(np.int64).copy()
        host = np.zeros((m, n))
        gen(m, n, ri.ctypes.data_as(POINTER(sb.STARSH_int)),
            ci.ctypes.data_as(POINTER(sb.STARSH_int)), prob["data"], prob["data"],
            host.ctypes.data, m)
        D = torch.tensor(host.T.copy(), dtype=f64, device=dev).T
        nd2 = float((D * D).sum())
        for h in hows:
            Y = sketch(D, h)[:, :min(k, n)]
            Q, _ = torch.linalg.qr(Y)
            B = Q.T @ D
            sv = torch.linalg.svdvals(B)
            outside = max(0.0, nd2 - float((B * B).sum()))
            budget = tol * tol * nd2
            tail = torch.flip(torch.cumsum(torch.flip(sv * sv, [0]), 0), [0])
            ok = (tail + outside <= budget).nonzero()
            r = int(ok[0]) if len(ok) else -1
            rr = res[h]
            if r >= 0 and r <= wl["maxrank"]:
                rr["accepted"] += 1
                rr["ranks"].append(r)
            rr["outside_over_budget"] = max(rr["outside_over_budget"],
                                            outside / max(budget, 1e-300))
    out = {}
    for h in hows:
        rr = res[h]
        out[h] = {"accepted": rr["accepted"], "tiles": len(pairs),
                  "mean_rank": float(np.mean(rr["ranks"])) if rr["ranks"] else None,
                  "max_outside_over_tol2": rr["outside_over_budget"]}
    # FP32-accumulate GEMM rates at one batch's shape (tiles x m x k per n)
    bt = 512
    a32 = torch.randn(bt, n_b, n_b, device=dev, dtype=torch.float32)
    b32 = torch.randn(bt, n_b, k, device=dev, dtype=torch.float32)
    rates = {}
    for name, tf, A_, B_ in (("fp32_simt", False, a32, b32),
                             ("tf32", True, a32, b32),
                             ("bf16", False, a32.bfloat16(), b32.bfloat16())):
        torch.backends.cuda.matmul.allow_tf32 = tf
        torch.bmm(A_, B_)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            torch.bmm(A_, B_)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / 5 / 1e3
        rates[name] = 2.0 * bt * n_b * n_b * k / t / 1e12
    torch.backends.cuda.matmul.allow_tf32 = prev_tf32
    del a32, b32
    return {"what": "sketch precision on sampled far tiles (FP64 basis, projection and rank rule for every variant)",
            "tol": tol, "sketch_width": k, "results": out,
            "cublas_tflops_at_batch_shape": rates,
            "x3_cost_note": "BF16x3 / TF32x3 need 3 GEMMs per sketch"}


# ------------------------------------------------------------- device peak

# DRAM bytes (read + write) of k_sketch_i8 over its algorithmic bytes, from
# an ncu capture of a 256-tile, N = 16384 square-exponential case
SKETCH_TRAFFIC_RATIO = 1.013


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool's B200s (driver-written
    MEASURED_PEAKS.json), else the pool's earlier fallback figure."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


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


def run_single(args):
    """One approximation (or one C4 batched call) with the chosen engine;
    prints its phase times as one JSON line.  No warm-up, no comparison:
    a program for launch lists and ncu captures."""
    import starsh_b200 as sb
    lib = sb.load()
    engine = sb.ENGINE_FP64 if args.engine == "fp64" else sb.ENGINE_MIXED
    if args.workload == "c4-batch":
        handle = sb.KERNEL(lambda *a: None)
        _keep.append(handle)
        assert lib.starsh_b200_kernel_register(
            c_void_p(ctypes.cast(handle, c_void_p).value), sb.FAMILY["coulomb"],
            1.0) == 0
        lib.starsh_set_oversample(str(C4["oversample"]).encode())
        probs = build_mixed(lib, c4_specs(), handle, tune=args.tune)
        n = len(probs)
        ranks = (ctypes.c_int * n)(*[p["maxrank"] for p in probs])
        tols = (ctypes.c_double * n)(*[p["tol"] for p in probs])
        Fs = (POINTER(sb.Blrf) * n)(*[new_format(lib, p) for p in probs])
        Ms = (POINTER(sb.Blrm) * n)()
        assert lib.starsh_b200_approximate_batch(n, Ms, Fs, ranks, tols, None,
                                                 engine, 0) == 0
    else:
        wl = dict(WORKLOADS[args.workload])
        if args.n:
            wl["N"] = args.n
        lib.starsh_set_oversample(str(wl["oversample"]).encode())
        prob = make_problem(lib, wl)
        F = new_format(lib, prob)
        M = POINTER(sb.Blrm)()
        assert lib.starsh_b200_approximate(byref(M), F, wl["maxrank"], wl["tol"],
                                           0, engine, 0) == 0
        if args.products:
            # TLR products B = M A on the device, nrhs of the workload (64
            # when it names none)
            import torch
            nrhs = wl.get("dmml_nrhs", 64)
            A = torch.randn(nrhs, wl["N"], dtype=torch.float64, device="cuda")
            B = torch.zeros(nrhs, wl["N"], dtype=torch.float64, device="cuda")
            for _ in range(args.products):
                assert lib.starsh_b200_blrm_dmml_device(
                    M, nrhs, 1.0, A.data_ptr(), wl["N"], 0.0, B.data_ptr(),
                    wl["N"], None) == 0
            torch.cuda.synchronize()
    st = sb.stats(lib)
    print(json.dumps({"workload": args.workload, "engine": args.engine,
                      "total_ms": st.total_ms, "gen_ms": st.gen_ms,
                      "basis_ms": st.basis_ms, "project_ms": st.project_ms,
                      "svd_ms": st.svd_ms, "output_ms": st.output_ms,
                      "launches": int(st.kernel_launches)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--engine", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="c2-sqexp",
                    choices=sorted(WORKLOADS) + ["c4-batch", "c5-serve"])
    ap.add_argument("--serve-rate", type=float, default=C5["rate"],
                    help="c5-serve: offered requests per second")
    ap.add_argument("--serve-seconds", type=float, default=C5["seconds"],
                    help="c5-serve: length of the arrival stream")
    ap.add_argument("--n", type=int, default=0,
                    help="points (a smaller N profiles the same kernels)")
    ap.add_argument("--tune", action=argparse.BooleanOptionalAction,
                    default=True,
                    help="c4-batch / c5-serve: block sizes from the library's "
                         "autotuner (default) or the fixed rule by N")
    ap.add_argument("--precision-study", action="store_true",
                    help="c2-* / c3-*: add the sketch precision study to the line")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline leg")
    ap.add_argument("--single", action="store_true",
                    help="one approximation of the workload (c4-batch: one "
                         "batched call) and its phase times, nothing else: "
                         "the program profiles are taken on")
    ap.add_argument("--products", type=int, default=0,
                    help="--single: then this many TLR products on the device")
    ap.add_argument("--_cpu-run", type=int, default=0, dest="cpu_run")
    args = ap.parse_args()
    if args.single:
        run_single(args)
        return
    key = args.workload
    if args.cpu_run:
        if key in ("c4-batch", "c5-serve"):
            _cpu_run_mixed()
        else:
            _cpu_run(key, args.cpu_run)
        return

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if key in ("c4-batch", "c5-serve"):
        if args.impl == "reference":
            if rank == 0:
                reference_arm_mixed(args, key, len(os.sched_getaffinity(0)))
            return
        import torch
        import starsh_b200 as sb
        lib = sb.load()
        torch.cuda.set_device(local)
        assert lib.starsh_b200_set_device(local) == 0
        stream = torch.cuda.ExternalStream(lib.starsh_b200_stream())
        clocks = ClockSampler(local)
        if key == "c4-batch":
            run_c4(args, lib, stream, clocks, torch)
        else:
            run_c5(args, lib, clocks)
        return
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
            step_times.append(times)
            return statistics.mean(times), sts, err, (M, F)
        free(M, F)
        step_times.append(times)
        return statistics.mean(times), sts, err, None

    clocks = ClockSampler(local)
    step_times = []
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
        dgemm = fp64_peak_tflops(torch)
        dmml = {"nrhs": nrhs, "ms": t * 1e3, "gflops": flops / t / 1e9,
                "hbm_gbs": byts / t / 1e9,
                "bound": "fp64 tensor" if flops / byts > 5 else "hbm",
                "dgemm_tflops_in_run": dgemm,
                "frac_of_dgemm": flops / t / 1e12 / dgemm,
                "kernels": "k_prod_t (T = V^T A per input block column) + "
                           "k_prod_b (B += U T + D A per output block row)"}
        free(M, F)

    # e2e: the drop-in call with host buffers
    entry = (lib.starsh_blrm__drsdd_b200_mp if chosen == sb.ENGINE_MIXED
             else lib.starsh_blrm__drsdd_b200)
    e2e_times, e2e_st = [], None
    for _ in range(args.warmup):
        # untimed, like the device-resident warm-up (first use of the
        # library's page-locked host blocks)
        M, F, *_ = step(chosen, 1, entry)
        free(M, F)
    barrier()
    for _ in range(args.steps):
        M, F, dt, host, st = step(chosen, 1, entry)
        e2e_times.append(host)
        e2e_st = st
        free(M, F)
    barrier()
    t_e2e = statistics.mean(e2e_times)
    entries = last.entries
    (value, e2e_value, plain_value), (t_dev, t_e2e, t_plain) = replica_rates(
        [t_dev, t_e2e, t_plain], entries, world, "cuda")

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    # roofline of the sketch kernel: on the int8 tensor-core path it streams
    # D once per round from HBM (bound: HBM; algorithmic bytes = 8 m n per
    # tile and round + the Y columns written); the FP64 engine's sketch is
    # a DMMA GEMM (bound: FP64 tensor, 2 m n k flops per tile)
    per_launch_s = last.sketch_ms / 1e3 / max(1, last.sketch_launches)
    if last.fused_launches > 0:
        # the fused generation + first-round sketch: it writes D (8 m n per
        # tile) and the round's Y columns; its inputs are the points
        per_launch_s = last.fused_ms / 1e3 / last.fused_launches
        bytes_per_launch = last.fused_bytes / last.fused_launches
        achieved = bytes_per_launch / per_launch_s / 1e9
        peak, peak_src = measured_hbm_gbs()
        roof = {"bound": "hbm",
                "kernel": "k_gen_sketch_i8 (generation fused with the tcgen05 int8 sketch; D and Y written)",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "traffic": None,
                "resketch_tiles": int(last.resketch_tiles)}
    elif last.sketch_int8:
        bytes_per_launch = last.sketch_bytes / max(1, last.sketch_launches)
        achieved = bytes_per_launch / per_launch_s / 1e9
        peak, peak_src = measured_hbm_gbs()
        roof = {"bound": "hbm", "kernel": "k_sketch_i8 (tcgen05 int8 slices, Y = D Omega8)",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                # ncu on a 256-tile case: DRAM read + write
                # = 1.013x the algorithmic bytes on a 256-tile capture, so the
                # per-launch traffic is the algorithmic figure scaled by it
                "traffic": bytes_per_launch * SKETCH_TRAFFIC_RATIO,
                "traffic_source": "ncu capture of a 256-tile case, scaled by tiles"}
    else:
        flops_per_launch = last.sketch_flops / max(1, last.sketch_launches)
        achieved = flops_per_launch / per_launch_s / 1e12
        peak = fp64_peak_tflops(torch)
        roof = {"bound": "tensor", "kernel": "k_gemm_f64 (sketch Y = D Omega, FP64 DMMA)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak,
                "peak_source": "measured in this run: torch float64 matmul 4096^3 (cuBLAS DGEMM); MEASURED_PEAKS.json has no FP64 figure",
                "traffic": None}
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
        "step_ms": [round(t * 1e3, 2) for t in step_times[0]],
        "plain_fp64": {"value": plain_value, "ms_per_step": t_plain * 1e3,
                       "rel_err": err_plain,
                       "chosen_over_plain": value / plain_value},
        "e2e": {"value": e2e_value, "unit": "Mentries/s",
                "h2d_bytes_per_step": int(e2e_st.h2d_bytes),
                "d2h_bytes_per_step": int(e2e_st.d2h_bytes),
                "ms_per_step": t_e2e * 1e3,
                "last_step_host_ms": {
                    "whole_call": e2e_st.total_ms,
                    "waiting_for_batch_downloads": e2e_st.mirror_wait_ms,
                    "after_last_batch": e2e_st.finish_ms},
                "last_step_device_phases_ms": {
                    "generation": e2e_st.gen_ms, "sketch": e2e_st.sketch_ms,
                    "basis": e2e_st.basis_ms, "project": e2e_st.project_ms,
                    "svd": e2e_st.svd_ms, "output": e2e_st.output_ms}},
        "gpu_launches": int(sum(s.kernel_launches for s in sts)),
        "phases_ms": {"generation": last.gen_ms, "fused_gen_sketch": last.fused_ms,
                      "sketch": last.sketch_ms, "basis": last.basis_ms,
                      "project": last.project_ms, "svd": last.svd_ms,
                      "output": last.output_ms, "total_host": last.total_ms},
        "roofline": roof,
        "clocks": clocks.summary(),
    }
    if dmml:
        line["dmml"] = dmml
    # the other large kernels of the step, each against its own bound:
    # the generator writes D once (8 B per entry; its limit is FP64 issue),
    # the projection B = Q^T D is an FP64 DMMA contraction
    if chosen == sb.ENGINE_MIXED and last.gen_ms > 0 and last.project_ms > 0:
        dgemm = dmml["dgemm_tflops_in_run"] if dmml else fp64_peak_tflops(torch)
        hbm_peak, hbm_src = measured_hbm_gbs()
        gen_entries = float(last.entries)
        line["rooflines_other"] = {
            "generation (k_gen_tiles)": {
                "bound": "fp64 issue (an exp or Bessel evaluation per entry)",
                "entries_per_s": gen_entries / (last.gen_ms / 1e3),
                "d_write_gbs": 8.0 * gen_entries / (last.gen_ms / 1e3) / 1e9,
                "frac_of_hbm": 8.0 * gen_entries / (last.gen_ms / 1e3) / 1e9 / hbm_peak,
                "hbm_peak_source": hbm_src},
            "projection (k_gemm_f64 TN, B = Q^T D)": {
                "bound": "tensor (FP64 DMMA)",
                "achieved_tflops": last.project_flops / (last.project_ms / 1e3) / 1e12,
                "peak_tflops": dgemm,
                "frac": last.project_flops / (last.project_ms / 1e3) / 1e12 / dgemm,
                "peak_source": "cuBLAS DGEMM 4096^3 measured in this run"}}
    if args.precision_study and (key.startswith("c3") or key.startswith("c2")):
        line["precision_study"] = precision_study(lib, wl, prob, torch)
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
