#!/usr/bin/env python
"""Benchmark of the asqtad/HISQ eo-preconditioned solve on one B200 (or N
independent replicas).

Workload (one "step" = one solve): HISQ links built on the device from a
seeded gauge field U = exp(i 0.5 H) on a 32^3 x 64 lattice (t antiperiodic,
staggered signs), mass 0.01, one Gaussian source on even sites, solved with
QOP_D3_asqtad_invert (evenodd = EVEN) to |b - A x| / |b| <= 1e-10
(rsqmin = 1e-20), using the mixed-precision reliable-update solver
(16-bit fixed-point storage with per-site / per-link FP32 scales, FP32
arithmetic, FP64 reductions and reliable updates).

Reported: solves/s (device-resident inputs, CUDA events on the library
stream, max over ranks), e2e solves/s through the C ABI from pinned host
buffers, p50/p99 latency, the same solve with plain FP64 CG, Dslash GB/s
and the roofline of the dominant kernel, and the oracle's CPU time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Further workloads (one step = one QOP_D3_asqtad_invert_multi call, solved
by the batched int16 solver, compared with the same call in FP64):
  --workload multimass   HISQ 24^3x48, one source, 12 masses sqrt(logspace(-4, 0))
  --workload multisrc    asqtad 32^4 (eps 0.4), 16 sources, mass 0.005
  --workload small       F3 asqtad 8^4: the nine Dslash cases and the eo CG,
                         GPU and oracle times, Dslash parity
  --workload force       HISQ and asqtad fermion forces, 24^3x48, 8 sources
  --workload serve       the solve service (QOPB_serve_*) with HISQ 16^4,
                         24^3x48 and 32^3x64 resident, Poisson arrivals
  --workload dd          the decomposed lattice: the int16 mixed solver and
                         FP64 CG on HISQ 32^3x64; one GPU: directions
                         --dd-mask exchange halos with themselves through
                         NCCL, timed against the undecomposed solves; N GPUs
                         (torchrun): the lattice split over the GPUs
"""
import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0
# Iterations of the plain FP64 CG (the reference algorithm) on the headline
# workload (HISQ 32^3x64, eps 0.5, seed 2024, m 0.01, |r|/|b| <= 1e-10),
# measured on a B200 with QOP_D3_asqtad_invert at prec_sloppy 64: 5920.
# The CPU reference arm times a bounded number of the reference's FP64 CG
# iterations and scales by this count (a full FP64 CPU solve takes tens of
# minutes on the host cores); the device arm reports its own FP64 iteration
# count beside it.
FP64_ITERS_HEADLINE = 5920


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--lattice", default=None, help="default: 32,32,32,64 (single) or the workload's own")
    ap.add_argument("--mass", type=float, default=0.01)
    ap.add_argument("--tol", type=float, default=1e-10, help="|r|/|b| target")
    ap.add_argument("--eps", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--prec", type=int, default=16, choices=[16, 32, 64], help="sloppy precision")
    ap.add_argument("--ru-delta", type=float, default=0.3, help="reliable-update threshold on |r|")
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--cpu-iters", type=int, default=12, help="CG iterations timed on the host")
    ap.add_argument("--ref-iters", type=int, default=None,
                    help="FP64 CG iterations of one solve, for the reference arm's solves/s (default: the "
                         "measured count of the headline workload)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--prof-every", type=int, default=7,
                    help="headline solve: bracket every n-th launch of each kernel class with CUDA events (odd n: "
                         "the samples rotate over the positions in a 16-iteration chunk, so the first launch "
                         "after each host check is not over-represented)")
    ap.add_argument("--quick", action="store_true", help="skip FP64 baseline and e2e (development)")
    ap.add_argument("--other-configs", default="multimass,multisrc",
                    help="headline run on one GPU: batched workloads also run (own processes, after the timed "
                         "region) and summarised in its line; empty to skip")
    ap.add_argument("--dd-mask", type=int, default=15, help="dd workload on one GPU: self-split directions")
    ap.add_argument("--dd-runs", default="u16,u64,d16,d64",
                    help="dd workload runs: u/d (undecomposed / decomposed) x 16/64 (sloppy precision)")
    ap.add_argument("--dd-max-iter", type=int, default=200000, help="dd workload: iteration limit of each solve")
    ap.add_argument("--hop-kernel", type=int, default=None, help="int16 hop variant (library default if unset)")
    ap.add_argument("--batch-kernel", type=int, default=None, help="batched hop variant (chosen by batch size if unset)")
    ap.add_argument("--ms-stop", type=float, default=None,
                    help="multi-shift phase: stop target of the shifted systems (relative |r|^2; library default if unset)")
    ap.add_argument("--ab", default=None, help="A/B of a 0/1 solver option (e.g. fuse_update) on the headline solve: "
                                               "--steps pairs of solves interleaved in one process, clocks sampled")
    ap.add_argument("--workload", default="single",
                    choices=["single", "multimass", "multisrc", "serve", "small", "force", "dd"],
                    help="single: the headline solve; multimass / multisrc: batched invert_multi workloads; "
                         "serve: the solve service under Poisson load")
    ap.add_argument("--serve-burst", type=int, default=12, help="requests of the peak-throughput burst")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="arrival window per load level")
    ap.add_argument("--serve-policy", type=int, default=0, choices=[0, 1],
                    help="0: step every engine in turn; 1: only the engine holding the oldest request")
    return ap.parse_args()


def kernel_opts(a):
    """Kernel-variant options given on the command line (else library defaults)."""
    o = {}
    if a.hop_kernel is not None:
        o["hop_kernel"] = a.hop_kernel
    if a.batch_kernel is not None:
        o["batch_kernel"] = a.batch_kernel
    if a.ms_stop is not None:
        o["ms_stop"] = a.ms_stop
    return o


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def workload_name(a, L):
    return "hisq_%s_m%g_tol%g_eps%g_seed%d" % ("x".join(map(str, L)), a.mass, a.tol, a.eps, a.seed)


def headline_config(a, L, world):
    """The `config` of the headline line, identical in both arms."""
    V = int(np.prod(L))
    return {"workload": workload_name(a, L), "lattice": list(L), "mass": a.mass, "tol": a.tol, "eps": a.eps,
            "parallelism": "replicas x%d" % world,
            "l2": ("inputs larger than L2 (links %.2f GB FP64)" if V * 16 * 18 * 8 > 126e6 else
                   "L2-resident inputs (links %.2f GB FP64)") % (V * 16 * 18 * 8 / 1e9)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return PEAK_FALLBACK_GBS, "fallback"


def ncu_traffic(kernel_class, L):
    """DRAM bytes per launch from the committed ncu summary of this kernel
    class (captured on a smaller lattice and scaled by the sites one launch
    processes; traffic per site is volume independent once the fields exceed
    L2), or None when no capture is committed."""
    import glob
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "ncu_%s_*.md" % kernel_class))):
        m = re.search(r"dram_bytes_per_site:\s*([0-9.eE+]+)", open(p).read())
        if m:
            return float(m.group(1)) * int(np.prod(L)) // 2
    return None


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.samples, self.stop, self.t = gpu, [], False, None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self.stop:
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            time.sleep(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *exc):
        self.stop = True
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if "Active" in s[3 + k]
                          and not s[3 + k].startswith("Not")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------- replicas
def reduce_max(x, dist, device):
    """Max of a per-rank scalar over all ranks (the job is as slow as its
    slowest replica); identity without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(steps, world, max_ms):
    """Solves/s of the whole job: every replica solves `steps` systems; the
    elapsed time is the slowest rank's."""
    return steps * world / (max_ms / 1e3)


# ---------------------------------------------------------------- reference arm
def cpu_iteration_time(fat, lng, L, src, mass, iters, threads):
    """Seconds per FP64 CG iteration of the reference algorithm on the host
    cores, from a bounded EVEN solve of `iters` iterations (max_restarts 0,
    an unreachable rsqmin): the reference's own compiled path
    (oracle/_ref/libqopref.so: QOP_D3_asqtad_invert_qdp over its QDP/C
    stand-in, OpenMP site loops) where it was built, else the oracle's C
    restatement.  Returns (s/iter, iterations, threads, kind, what)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import refqop as R
    ia = O.InvertArg(1e9, iters, iters, 0, 0)
    ra = O.ResidArg(1e-30, 0, 0, 0, 0, 0)
    if R.available():
        th = R.set_threads(L, threads)
        fo = R.RefFla(L, fat, lng, R.D3)
        kind, what = "reference", "QOP_D3_asqtad_invert (the reference's own lib/asqtad_invert_p.c, compiled by oracle/ref)"
    else:
        O.set_threads(threads)
        th = O.get_threads()
        fo = O.Fla(O.Lattice(L), fat, lng)
        kind, what = "port", "the oracle (the reference algorithm restated in C, OpenMP)"
    t0 = time.perf_counter()
    fo.invert(mass, src, ia, ra)
    dt = time.perf_counter() - t0
    del fo
    return dt / max(ra.final_iter, 1), ra.final_iter, th, kind, what


def oracle_true_rsq(fat, lng, L, src, out, mass, threads):
    """|b - A x|^2 / |b|^2 on the even sites for the solve output out = m A^-1 b
    (A = m^2 - D_eo D_oe), computed by the oracle in FP64 as the reference's
    check_resids does (examples/asqtad_test.c:84-130)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    fo = O.Fla(O.Lattice(L), fat, lng)
    V = int(np.prod(L))
    t = fo.dslash(mass, out, O.EVENODD, O.EVEN)
    chk = fo.dslash(-mass, t, O.EVEN, O.EVENODD)
    b = src[: V // 2]
    r = chk[: V // 2] / mass + b
    return float((r ** 2).sum() / (b ** 2).sum())


class _StdoutToStderr:
    """Sends what C code prints to stdout (the reference's own progress and
    SVD messages) to stderr, so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def run_reference(a):
    """The reference's own CPU implementation of the path, on the host cores:
    HISQ links built by its QOP_hisq_create_L_from_G, then bounded FP64 CG
    iterations of its QOP_D3_asqtad_invert (its default path: mixed_rsq
    1e9 keeps every iteration in FP64) per step, extrapolated to the FP64
    iteration count of the workload.  Without oracle/_ref (the reference
    sources were absent when the tree was built) the oracle's restatement
    stands in and the line says kind "port"."""
    rank, _, world = rank_info()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import refqop as R
    from qopqdp_b200 import lattice as LT
    L = tuple(int(x) for x in (a.lattice or "32,32,32,64").split(","))
    threads = os.cpu_count() or 1
    U = LT.random_gauge(L, a.eps, a.seed, device="cpu")
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    quiet = _StdoutToStderr()
    quiet.__enter__()
    if R.available():
        R.set_threads(L, threads)
        U = R.rephase_G(L, U, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
        sets, _, _ = R.hisq_links(L, hc, U)
        fat, lng = sets[0]
        del sets
    else:
        O.set_threads(threads)
        lat = O.Lattice(L)
        U = lat.rephase_G(U, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
        fat, lng, _, _ = lat.hisq_links(hc, U)
    del U
    src = LT.gaussian_vector(L, a.seed)
    n_solve = a.ref_iters or (FP64_ITERS_HEADLINE if workload_name(a, L) == workload_name(a, (32, 32, 32, 64))
                              and (a.mass, a.tol, a.eps, a.seed) == (0.01, 1e-10, 0.5, 2024) else None)
    per = []
    for k in range(a.warmup + a.steps):
        s, it, th, kind, what = cpu_iteration_time(fat, lng, L, src, a.mass, a.cpu_iters, threads)
        if k >= a.warmup:
            per.append(s)
    quiet.__exit__()
    s_it = float(np.median(per))
    if n_solve:
        value = 1.0 / (s_it * n_solve)
        sample = ("%d FP64 CG iterations of %s per step on %d host threads, %.4f s per iteration (median of %d "
                  "steps); solves/s extrapolated to %d iterations, the FP64 CG iteration count of this workload"
                  % (it, what, th, s_it, a.steps, n_solve))
    else:
        value = None
        sample = "%d CG iterations per step; no FP64 iteration count for this workload (--ref-iters)" % a.cpu_iters
    line = {"metric": "mixed-prec CG solves/s @1e-10 (HISQ eo solve)", "value": value, "unit": "solves/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 / value if value else None, "ms_per_step_kind": "extrapolated",
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(a, L, world),
            "impl": "reference",
            "measured": {"sec_per_iter": s_it, "iters_per_step": it, "fp64_iters_per_solve": n_solve},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": th, "kind": kind, "sample": sample,
                             "sec_per_iter": s_it},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- device arm
def other_configs(a):
    """The batched workloads in their own processes after the headline's
    timed region (one warm-up call and one timed call each; multisrc without
    its 16-solve FP64 comparison), summarised for the headline line."""
    out = {}
    for wl in a.other_configs.split(","):
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", wl, "--steps", "1", "--warmup", "1",
               "--seed", str(a.seed), "--tol", str(a.tol)]
        if wl == "multisrc":
            cmd.append("--quick")
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
            d = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
            keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "final_rsq_max", "config",
                    "speedup_vs_fp64", "gpu_launches", "clocks")
            o = {k: d.get(k) for k in keep}
            roof = d.get("roofline") or {}
            o["roofline"] = {k: roof.get(k) for k in ("kernel", "avg_us", "achieved", "frac", "peak")}
            if d.get("fp64"):
                o["fp64_solves_per_s"] = d["fp64"]["solves_per_s"]
            if d.get("batched_mode"):
                o["batched_mode_solves_per_s"] = d["batched_mode"]["solves_per_s"]
            o["command"] = " ".join(["python bench.py"] + cmd[2:])
            out[wl] = o
        except Exception as e:   # recorded, never fatal to the headline line
            out[wl] = {"error": "%s: %s" % (type(e).__name__, str(e)[:200])}
    return out


def run_b200(a):
    rank, local, world = rank_info()
    import torch
    import ctypes as C
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import (Qop, QOP_invert_arg_t, QOP_resid_arg_t, QOP_info_t, QOP_EVEN, load_library)
    lib = load_library()
    lib.QOPB_stream.restype = C.c_void_p

    class KStat(C.Structure):
        _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("total_ms", C.c_double),
                    ("bytes_per_launch", C.c_double)]

    lib.QOPB_prof_end.argtypes = [C.POINTER(KStat), C.c_int]
    lib.QOPB_launch_count.restype = C.c_ulonglong

    def prof_end():
        buf = (KStat * 32)()
        n = lib.QOPB_prof_end(buf, 32)
        return {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms, buf[i].bytes_per_launch)
                for i in range(min(n, 32))}

    L = tuple(int(x) for x in (a.lattice or "32,32,32,64").split(","))
    V = int(np.prod(L))
    q = Qop("D")
    assert q.init(L) == 0
    t_setup = time.perf_counter()
    U = LT.random_gauge(L, a.eps, a.seed, device="cuda")
    G = q.create_G(U)
    del U
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    q.set_hisq_opts(want_aux=0)
    info = QOP_info_t()
    H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G, info)
    q.destroy_G(G)
    fla = q.hisq_asqtad_links(H, 0)
    src = LT.gaussian_vector(L, a.seed)
    t_setup = time.perf_counter() - t_setup
    stream = torch.cuda.ExternalStream(lib.QOPB_stream())
    rsq = a.tol * a.tol
    big = 1 << 30

    def solve(hout, hin, prec):
        q.set_opts(prec_sloppy=prec, half_format=0, ru_delta=a.ru_delta, **kernel_opts(a))
        q.dslash(fla, 0.0, hout, hout, QOP_EVEN, QOP_EVEN)          # zero initial guess
        ia = QOP_invert_arg_t(1e9, 200000, 200000, 10, QOP_EVEN)
        ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
        inf = q.invert(fla, a.mass, hout, hin, ia, ra)
        return ra, inf

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, dist, "cuda")

    hin = q.create_V(src, QOP_EVEN)
    hout = q.create_V(np.zeros_like(src))
    for _ in range(a.warmup):
        ra, _ = solve(hout, hin, a.prec)
    # ---------------- timed region (device-resident inputs)
    lat_ms, iters, rsqs = [], [], []
    lib.QOPB_prof_every(a.prof_every)       # events around a sample of the launches
    lib.QOPB_prof_begin()
    barrier()
    n_launch0 = lib.QOPB_launch_count()
    with Clocks(local) as clk:
        e0 = ev()
        for _ in range(a.steps):
            s0 = ev()
            ra, _ = solve(hout, hin, a.prec)
            s1 = ev()
            s1.synchronize()
            lat_ms.append(s0.elapsed_time(s1))
            iters.append(ra.final_iter)
            rsqs.append(ra.final_rsq)
        e1 = ev()
        barrier()
    n_launch = lib.QOPB_launch_count() - n_launch0
    kst = prof_end()
    lib.QOPB_prof_every(1)
    total_ms = max_over_ranks(e0.elapsed_time(e1))
    value = job_throughput(a.steps, world, total_ms)
    # independent FP64 check of the last solution's residual (not timed)
    sol = q.extract_V(hout, V)
    # ---------------- plain FP64 GPU CG (the reference algorithm in FP64)
    fp64 = {}
    if not a.quick and a.fp64_steps > 0:
        t64, it64 = [], []
        lib.QOPB_prof_begin()
        for _ in range(a.fp64_steps):
            s0 = ev()
            r64, _ = solve(hout, hin, 64)
            s1 = ev()
            s1.synchronize()
            t64.append(s0.elapsed_time(s1))
            it64.append(r64.final_iter)
        k64 = prof_end()
        fp64 = {"solves_per_s": 1e3 / float(np.mean(t64)), "ms_per_solve": float(np.mean(t64)),
                "iters": int(np.median(it64)), "final_rsq": r64.final_rsq}
        h = k64.get("hop_f64")
        if h and h[1] > 0:
            fp64["hop_f64_gbs"] = h[0] * h[2] / (h[1] * 1e-3) / 1e9
    # ---------------- e2e through the C ABI from pinned host buffers
    e2e = None
    if not a.quick:
        src_pin = torch.empty(src.shape, dtype=torch.float64, pin_memory=True).numpy()
        src_pin[...] = src
        dst_pin = torch.empty(src.shape, dtype=torch.float64, pin_memory=True).numpy()
        barrier()
        t0 = time.perf_counter()
        e0 = ev()                                                   # whole loop, like `value`
        for _ in range(a.steps):
            h_in = q.create_V(src_pin, QOP_EVEN)                   # H2D: even half
            solve(hout, h_in, a.prec)
            q.extract_V(hout, V, QOP_EVEN, into=dst_pin)           # D2H: even half
            q.destroy_V(h_in)
        e1 = ev()
        e1.synchronize()
        barrier()
        e_tot = max_over_ranks(e0.elapsed_time(e1))
        half = (V // 2) * 3 * 2 * 8
        e2e = {"value": job_throughput(a.steps, world, e_tot), "unit": "solves/s", "h2d_bytes_per_step": half,
               "d2h_bytes_per_step": half, "wall_s": time.perf_counter() - t0}
    # ---------------- roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    dom = max(kst.items(), key=lambda kv: kv[1][1]) if kst else None
    roof = None
    kernels = {}
    for name, (n, ms, b) in kst.items():
        kernels[name] = {"timed_launches": n, "total_ms": ms, "avg_us": 1e3 * ms / max(n, 1),
                         "gbs": n * b / (ms * 1e-3) / 1e9 if ms > 0 else None, "bytes_per_launch": b}
    if dom:
        name, (n, ms, b) = dom
        ach = n * b / (ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_kind": peak_kind, "kernel": name, "traffic": ncu_traffic(name, L),
                "bytes_per_launch": b, "sampled_every": a.prof_every}
    # ---------------- oracle checks and CPU baseline on rank 0 (not timed)
    cpu = None
    oracle_rsq = None
    n_fp64 = fp64.get("iters")
    if rank == 0 and not a.no_cpu:
        fat, lng = q.extract_L(fla, V)
        threads = os.cpu_count() or 1
        # the FP64 true residual |b - A x|^2 / |b|^2 of the headline solution,
        # recomputed by the oracle from the device's links
        oracle_rsq = oracle_true_rsq(fat, lng, L, src, sol, a.mass, threads)
        if world == 1:
            with _StdoutToStderr():
                s_it, nit, th, kind, what = cpu_iteration_time(fat, lng, L, src, a.mass, a.cpu_iters, threads)
            n_ref = n_fp64 or FP64_ITERS_HEADLINE
            cpu = {"value": 1.0 / (s_it * n_ref), "unit": "solves/s", "cores": th, "kind": kind,
                   "sample": "%d FP64 CG iterations of %s on %d host threads, %.4f s/iteration, extrapolated "
                             "to the %d iterations of the FP64 solve" % (nit, what, th, s_it, n_ref),
                   "sec_per_iter": s_it}
        del fat, lng
    if rank == 0:
        lat_sorted = np.sort(lat_ms)
        line = {
            "metric": "mixed-prec CG solves/s @1e-10 (HISQ eo solve)",
            "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if a.prec < 64 else "f64",
            "data": "synthetic",
            "config": headline_config(a, L, world),
            "precision": ("int16 fixed-point" if a.prec == 16 else "FP%d" % a.prec) + " storage, FP32 arithmetic, FP64 reductions and reliable updates (delta %g)" % a.ru_delta,
            "p50_ms": float(np.percentile(lat_sorted, 50)), "p99_ms": float(np.percentile(lat_sorted, 99)),
            "iters": int(np.median(iters)), "final_rsq": float(max(rsqs)), "oracle_rsq": oracle_rsq,
            "fp64_cg": fp64,
            "speedup_vs_fp64": (value / world) / fp64["solves_per_s"] if fp64 else None,
            "roofline": roof, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(n_launch),
            "clocks": clk.summary(), "setup_s": t_setup,
        }
        # device time x SM clock of the dominant kernel: constant if the
        # kernel is bound by instruction issue, falling with the clock if
        # it is bound by HBM
        mhz = line["clocks"].get("sm_mhz")
        if roof and mhz:
            roof["avg_us_x_sm_mhz"] = kernels[roof["kernel"]]["avg_us"] * mhz
        if world == 1 and not a.quick and a.other_configs:
            line["other_configs"] = other_configs(a)
        print(json.dumps(line), flush=True)
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.hisq_destroy_L(H)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched workloads
MULTI = {
    # HISQ 24^3x48, one source, 12 masses m_i = sqrt(sigma_i), sigma log-spaced 1e-4..1
    "multimass": {"lattice": (24, 24, 24, 48), "eps": 0.5, "kind": "hisq", "nsrc": 1,
                  "masses": [float(x) for x in np.sqrt(np.logspace(-4, 0, 12))]},
    # asqtad 32^4 (eps 0.4), 16 sources, mass 0.005
    "multisrc": {"lattice": (32, 32, 32, 32), "eps": 0.4, "kind": "asqtad", "nsrc": 16, "masses": [0.005]},
}


def run_multi(a):
    """One step = one QOP_D3_asqtad_invert_multi call on the EVEN parity:
    `multimass` solves one source at 12 masses, `multisrc` 16 sources at
    one mass, every solve to |r|/|b| <= tol.  The int16 path runs the masses
    of one source as an int16 multi-shift CG and then refines every solve in
    one batched reliable-update CG sharing each hop's links (multisrc: the
    batched CG alone).
    Compared with the same call in FP64 (the reference algorithm: CGMS +
    refine for multimass; for multisrc one FP64 single-source solve times 16,
    which bounds the reference's sequential restarts from below)."""
    rank, local, world = rank_info()
    import torch
    import ctypes as C
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, QOP_invert_arg_t, QOP_resid_arg_t, QOP_EVEN, load_library
    w = MULTI[a.workload]
    L = tuple(int(x) for x in a.lattice.split(",")) if a.lattice else w["lattice"]
    lib = load_library()
    lib.QOPB_stream.restype = C.c_void_p
    lib.QOPB_launch_count.restype = C.c_ulonglong

    class KStat(C.Structure):
        _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("total_ms", C.c_double),
                    ("bytes_per_launch", C.c_double)]

    lib.QOPB_prof_end.argtypes = [C.POINTER(KStat), C.c_int]
    q = Qop("D")
    assert q.init(L) == 0
    U = LT.random_gauge(L, w["eps"], a.seed, device="cuda")
    G = q.create_G(U)
    del U
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    H = None
    if w["kind"] == "hisq":
        q.set_hisq_opts(want_aux=0)
        H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G)
        fla = q.hisq_asqtad_links(H, 0)
    else:
        fla = q.create_L_from_G(LT.ASQTAD_BENCH_COEFFS, G)
    q.destroy_G(G)
    srcs = [LT.gaussian_vector(L, a.seed + s) for s in range(w["nsrc"])]
    hins = [q.create_V(s, QOP_EVEN) for s in srcs]
    masses = [list(w["masses"]) for _ in range(w["nsrc"])]
    nsolve = sum(len(m) for m in masses)
    stream = torch.cuda.ExternalStream(lib.QOPB_stream())
    rsq = a.tol * a.tol

    def step(prec, ms=masses, ins=hins, multi_shift=1):
        q.set_opts(prec_sloppy=prec, half_format=0, ru_delta=a.ru_delta, multi_shift=multi_shift, **kernel_opts(a))
        outs = [[q.create_V(np.zeros_like(srcs[0])) for _ in m] for m in ms]
        ras = [[QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0) for _ in m] for m in ms]
        ia = QOP_invert_arg_t(1e9, 200000, 200000, 50, QOP_EVEN)
        q.invert_multi(fla, ms, outs, ins, ia, ras)
        for row in outs:
            for h in row:
                q.destroy_V(h)
        return [r for row in ras for r in row]

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(a.warmup):
        step(a.prec)
    lib.QOPB_prof_begin()
    barrier()
    n0 = lib.QOPB_launch_count()
    rsqs, lat = [], []
    with Clocks(local) as clk:
        e0 = ev()
        for _ in range(a.steps):
            s0 = ev()
            ras = step(a.prec)
            s1 = ev()
            s1.synchronize()
            lat.append(s0.elapsed_time(s1))
            rsqs += [r.final_rsq for r in ras]
        e1 = ev()
        barrier()
    n_launch = lib.QOPB_launch_count() - n0
    buf = (KStat * 32)()
    nk = lib.QOPB_prof_end(buf, 32)
    kst = {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms, buf[i].bytes_per_launch) for i in range(nk)}
    total_ms = reduce_max(e0.elapsed_time(e1), dist, "cuda")
    value = nsolve * a.steps * world / (total_ms / 1e3)
    # FP64 reference algorithm for comparison (not timed into value)
    fp64 = None
    if not a.quick and a.fp64_steps > 0:
        torch.cuda.synchronize()
        s0 = ev()
        if a.workload == "multisrc":
            r64 = step(64, [masses[0]], [hins[0]])
            mult = nsolve
        else:
            r64 = step(64)
            mult = 1
        s1 = ev()
        s1.synchronize()
        ms64 = s0.elapsed_time(s1) * mult
        fp64 = {"ms_per_step": ms64, "solves_per_s": nsolve / (ms64 / 1e3),
                "max_final_rsq": max(r.final_rsq for r in r64),
                "how": "one FP64 single-source solve x %d" % nsolve if mult > 1 else "the same call in FP64"}
    # the other int16 multi-mass mode (option multi_shift = 0: every mass a
    # system of the batched solver from the start; not timed into value)
    mshift = None
    if not a.quick and a.workload == "multimass" and a.prec == 16:
        step(16, multi_shift=0)
        torch.cuda.synchronize()
        s0 = ev()
        rms = step(16, multi_shift=0)
        s1 = ev()
        s1.synchronize()
        msm = s0.elapsed_time(s1)
        mshift = {"ms_per_step": msm, "solves_per_s": nsolve / (msm / 1e3),
                  "max_final_rsq": max(r.final_rsq for r in rms), "iters_max": max(r.final_iter for r in rms),
                  "how": "option multi_shift = 0: the batched solver alone, every mass from zero"}
        q.set_opts(multi_shift=1)
    peak, peak_kind = measured_peak()
    dom = max(kst.items(), key=lambda kv: kv[1][1]) if kst else None
    roof = None
    if dom:
        name, (n, ms, b) = dom
        ach = n * b / (ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_kind": peak_kind, "kernel": name, "avg_us": 1e3 * ms / max(n, 1), "bytes_per_launch": b,
                "traffic": None}
    if rank == 0:
        line = {"metric": "mixed-prec solves/s @%g (%s)" % (a.tol, a.workload), "value": value, "unit": "solves/s",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if a.prec < 64 else "f64", "data": "synthetic",
                "config": {"workload": a.workload, "lattice": L, "kind": w["kind"], "eps": w["eps"],
                           "masses": w["masses"], "sources": w["nsrc"], "tol": a.tol,
                           "parallelism": "replicas x%d" % world},
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "final_rsq_max": float(max(rsqs)), "fp64": fp64, "batched_mode": mshift,
                "speedup_vs_fp64": (value / world) / fp64["solves_per_s"] if fp64 else None,
                "roofline": roof, "kernels": {k: {"launches": v[0], "avg_us": 1e3 * v[1] / max(v[0], 1)}
                                              for k, v in kst.items()},
                "gpu_launches": int(n_launch), "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    for h in hins:
        q.destroy_V(h)
    if H is not None:
        q.hisq_destroy_L(H)
    else:
        q.destroy_L(fla)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_small(a):
    """Plain asqtad in single precision (QOP_F3_*) on 8^4 (eps 0.3), m = 0.1:
    the nine (eo_out, eo_in) Dslash cases and the eo-preconditioned CG to
    |r|/|b| <= 1e-5 (rsqmin 1e-10), timed on the GPU (CUDA events, mean over
    --steps repetitions after --warmup) and with the reference's own F3 code
    (oracle/_ref; the oracle where it was not built) on the host;
    each Dslash checked against the oracle (F3 tolerance 2e-6 per site).
    The whole problem is cache-resident: not an HBM measurement."""
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, QOP_invert_arg_t, QOP_resid_arg_t, QOP_EVEN, load_library
    L = (8, 8, 8, 8)
    V = int(np.prod(L))
    lat = O.Lattice(L)
    U = lat.rephase_G(LT.random_gauge(L, 0.3, a.seed, device="cpu"), LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    fat, lng = lat.make_imp_links(LT.ASQTAD_BENCH_COEFFS, list(U), naik=True)
    fat = [np.asarray(x, np.float32) for x in fat]
    lng = [np.asarray(x, np.float32) for x in lng]
    fo = O.Fla(lat, [x.astype(np.float64) for x in fat], [x.astype(np.float64) for x in lng])
    q = Qop("F")
    assert q.init(L) == 0
    lib = load_library()
    lib.QOPB_stream.restype = __import__("ctypes").c_void_p
    stream = torch.cuda.ExternalStream(lib.QOPB_stream())
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, a.seed).astype(np.float32)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    mass = 0.1
    m32 = float(np.float32(mass))

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    cases, worst = {}, 0.0
    for eo_out in (0, 1, 2):
        for eo_in in (0, 1, 2):
            for _ in range(a.warmup):
                q.dslash(fla, mass, hout, hin, eo_out, eo_in)
            e0 = ev()
            for _ in range(a.steps):
                q.dslash(fla, mass, hout, hin, eo_out, eo_in)
            e1 = ev()
            e1.synchronize()
            got = q.extract_V(hout, V).astype(np.float64)
            ref = fo.dslash(m32, src.astype(np.float64), eo_out, eo_in)
            num = np.sqrt(((got - ref) ** 2).reshape(V, -1).sum(1))
            den = np.sqrt((ref ** 2).reshape(V, -1).sum(1))
            err = float(np.max(num[den > 0] / den[den > 0])) if (den > 0).any() else 0.0
            worst = max(worst, err)
            cases["%d,%d" % (eo_out, eo_in)] = {"us": 1e3 * e0.elapsed_time(e1) / a.steps, "max_site_rel_err": err}
    # eo CG (reference algorithm, F3)
    q.set_opts(prec_sloppy=64)
    cg_ms, iters = [], 0
    for k in range(a.warmup + a.steps):
        q.dslash(fla, 0.0, hout, hout, QOP_EVEN, QOP_EVEN)
        ia = QOP_invert_arg_t(1e9, 2000, 2000, 5, QOP_EVEN)
        ra = QOP_resid_arg_t(1e-10, 0, 0, 0, 0, 0)
        e0 = ev()
        q.invert(fla, mass, hout, hin, ia, ra)
        e1 = ev()
        e1.synchronize()
        if k >= a.warmup:
            cg_ms.append(e0.elapsed_time(e1))
            iters = ra.final_iter
    # on the host: the reference's own F3 build (oracle/_ref) where it was
    # built, else the oracle: one Dslash (EVENODD) and the same CG
    import refqop as R
    kind = "reference" if R.available() else "port"
    threads = os.cpu_count() or 1
    if kind == "reference":
        cores = R.set_threads(L, threads)
        cpu = R.RefFla(L, [x.astype(np.float64) for x in fat], [x.astype(np.float64) for x in lng], R.F3)
    else:
        O.set_threads(threads)
        cores = O.get_threads()
        cpu = fo
    src64 = src.astype(np.float64).reshape(V, 6)
    with _StdoutToStderr():
        cpu.dslash(m32, src64, 2, 2)
        t0 = time.perf_counter()
        for _ in range(20):
            cpu.dslash(m32, src64, 2, 2)
        cpu_dslash_us = (time.perf_counter() - t0) / 20 * 1e6
        t0 = time.perf_counter()
        ora = O.ResidArg(1e-10, 0, 0, 0, 0, 0)
        cpu.invert(m32, src64, O.InvertArg(1e9, 2000, 2000, 5, 0), ora)
        cpu_cg_ms = (time.perf_counter() - t0) * 1e3
    line = {"metric": "F3 asqtad 8^4: Dslash us and eo CG ms", "value": float(np.mean(cg_ms)), "unit": "ms per CG solve",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": float(np.mean(cg_ms)),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "small", "lattice": L, "mass": mass, "rsqmin": 1e-10, "eps": 0.3,
                       "note": "cache-resident, not an HBM measurement"},
            "dslash": cases, "dslash_max_site_rel_err": worst, "cg_iters": iters, "cpu_cg_iters": ora.final_iter,
            "cpu_baseline": {"dslash_us": cpu_dslash_us, "cg_ms": cpu_cg_ms, "kind": kind, "cores": cores,
                             "sample": "one EVENODD Dslash (mean of 20) and the same eo CG, %s" %
                                       ("the reference's QOP_F3 build (oracle/_ref)" if kind == "reference"
                                        else "the oracle (FP64)")}}
    print(json.dumps(line), flush=True)
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)


def run_force(a):
    """Fermion forces (QOP_D3_hisq_force_multi and QOP_D3_asqtad_force_multi)
    on HISQ / asqtad links of a 24^3x48 gauge field (eps 0.5) with 8 sources
    (one Naik group), FP64: device time per call (CUDA events, mean of
    --steps after --warmup) and the oracle's time for the same call on a
    12^4 lattice scaled by the volume ratio (the work is local per site)."""
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, load_library
    L = tuple(int(x) for x in a.lattice.split(",")) if a.lattice else (24, 24, 24, 48)
    V = int(np.prod(L))
    nsrc = 8
    q = Qop("D")
    assert q.init(L) == 0
    lib = load_library()
    lib.QOPB_stream.restype = __import__("ctypes").c_void_p
    stream = torch.cuda.ExternalStream(lib.QOPB_stream())
    U = LT.random_gauge(L, a.eps, a.seed, device="cuda")
    G = q.create_G(U)
    del U
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    q.set_hisq_opts(want_aux=1)
    hc = LT.hisq_bench_coeffs()
    H = q.hisq_create_L_from_G(hc, G)
    F = q.create_F([np.zeros((V, 3, 3, 2)) for _ in range(4)])
    hv = [q.create_V(LT.gaussian_vector(L, a.seed + i)) for i in range(nsrc)]
    res = [0.1 * (i + 1) for i in range(nsrc)]
    acoef = LT.ASQTAD_BENCH_COEFFS

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    out = {}
    for name, call in (("hisq", lambda: q.hisq_force(H, F, hc, res, hv, [nsrc])),
                       ("asqtad", lambda: q.asqtad_force(G, F, acoef, res, hv))):
        for _ in range(a.warmup):
            assert call().status == 0
        e0 = ev()
        for _ in range(a.steps):
            call()
        e1 = ev()
        e1.synchronize()
        out[name] = {"ms": e0.elapsed_time(e1) / a.steps}
    # the reference's own force code (oracle/_ref) on a 12^4 lattice, scaled
    # by volume; the oracle's restatement where the reference was not built
    import refqop as R
    Lc = (12, 12, 12, 12)
    Vc = int(np.prod(Lc))
    lat = O.Lattice(Lc)
    Uc = lat.rephase_G(LT.random_gauge(Lc, a.eps, a.seed, device="cpu"), LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    xs = [LT.gaussian_vector(Lc, a.seed + i).reshape(Vc, 6) for i in range(nsrc)]
    kind = "reference" if R.available() else "port"
    threads = os.cpu_count() or 1
    if kind == "reference":
        cores = R.set_threads(Lc, threads)
        hisq_cpu = lambda: R.hisq_force(Lc, LT.hisq_coeff_vector(hc), Uc, [0.0], res, xs, [nsrc])
        asq_cpu = lambda: R.asqtad_force(Lc, acoef, Uc, res, xs)
        what = "QOP_D3_hisq_force_multi_qdp / QOP_D3_asqtad_force_multi_qdp (the reference's own code, oracle/_ref)"
    else:
        O.set_threads(threads)
        cores = O.get_threads()
        hisq_cpu = lambda: lat.hisq_force(LT.hisq_coeff_vector(hc), Uc, [0.0], res, xs, [nsrc])
        asq_cpu = lambda: lat.asqtad_force(acoef, Uc, res, xs)
        what = "the oracle's restatement"
    with _StdoutToStderr():
        t0 = time.perf_counter()
        hisq_cpu()
        out["hisq"]["cpu_ms"] = (time.perf_counter() - t0) * 1e3 * V / Vc
        t0 = time.perf_counter()
        asq_cpu()
        out["asqtad"]["cpu_ms"] = (time.perf_counter() - t0) * 1e3 * V / Vc
    for k in out:
        out[k]["speedup_vs_cpu"] = out[k]["cpu_ms"] / out[k]["ms"]
    line = {"metric": "fermion force ms per call (8 sources, FP64)", "value": out["hisq"]["ms"], "unit": "ms",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": out["hisq"]["ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "force", "lattice": L, "sources": nsrc, "eps": a.eps},
            "forces": out,
            "cpu_baseline": {"kind": kind, "cores": cores,
                             "sample": "one call of %s on 12^4 with %d host threads, scaled by the volume ratio"
                                       % (what, cores)}}
    print(json.dumps(line), flush=True)
    for h in hv:
        q.destroy_V(h)
    q.destroy_F(F)
    q.hisq_destroy_L(H)
    q.destroy_G(G)


def run_ab(a):
    """Interleaved A/B of a 0/1 option of QOP_asqtad_invert_set_opts on the
    headline solve (the single workload's lattice, links, source and
    target): --steps rounds, each timing two solves with the option 0 and
    two with 1 (order alternating between rounds), CUDA events on the
    library stream, SM clock and power sampled during each pair."""
    import ctypes as C
    import torch
    torch.cuda.set_device(0)
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, QOP_invert_arg_t, QOP_resid_arg_t, QOP_EVEN, load_library
    L = tuple(int(x) for x in (a.lattice or "32,32,32,64").split(","))
    q = Qop("D")
    assert q.init(L) == 0
    lib = load_library()
    lib.QOPB_stream.restype = C.c_void_p
    U = LT.random_gauge(L, a.eps, a.seed, device="cuda")
    G = q.create_G(U)
    del U
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    q.set_hisq_opts(want_aux=0)
    H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G)
    q.destroy_G(G)
    fla = q.hisq_asqtad_links(H, 0)
    src = LT.gaussian_vector(L, a.seed)
    hin, hout = q.create_V(src, QOP_EVEN), q.create_V(np.zeros_like(src))
    stream = torch.cuda.ExternalStream(lib.QOPB_stream())

    def solve(v):
        q.set_opts(prec_sloppy=a.prec, **{a.ab: v})
        q.dslash(fla, 0.0, hout, hout, QOP_EVEN, QOP_EVEN)
        ra = QOP_resid_arg_t(a.tol * a.tol, 0, 0, 0, 0, 0)
        assert q.invert(fla, a.mass, hout, hin, QOP_invert_arg_t(1e9, 200000, 200000, 10, QOP_EVEN), ra).status == 0
        return ra.final_iter

    for v in (0, 1):
        solve(v)
    res = {0: [], 1: []}
    for rnd in range(a.steps):
        for v in ((0, 1) if rnd % 2 == 0 else (1, 0)):
            with Clocks(0) as clk:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                its = [solve(v) for _ in range(2)]
                e1.record(stream)
                e1.synchronize()
            c = clk.summary()
            res[v].append({"ms_per_solve": e0.elapsed_time(e1) / 2, "iters": its[0], "sm_mhz": c.get("sm_mhz")})
    out = {}
    for v in (0, 1):
        ms = [r["ms_per_solve"] for r in res[v]]
        out[str(v)] = {"ms_per_solve_mean": float(np.mean(ms)), "ms_per_solve": ms, "iters": res[v][0]["iters"],
                       "sm_mhz": [r["sm_mhz"] for r in res[v]]}
    print(json.dumps({"ab": a.ab, "workload": workload_name(a, L), "rounds": a.steps, "results": out}), flush=True)


def run_dd(a):
    """Decomposed lattice.  Links: HISQ smeared on each process's block
    (periodic within the block: synthetic links of the production form),
    made on the undecomposed block lattice and passed node-local to the
    decomposed one.  One step = one solve (QOP_D3_asqtad_invert, EVEN
    source) to |r|/|b| <= --tol, with the int16 mixed solver (the value) and
    with FP64 CG (the reference algorithm).  On one GPU the
    directions of --dd-mask are decomposed with the process as its own
    neighbour (every hop packs, exchanges through NCCL and reads halos) and
    the same solve is timed on the undecomposed lattice; with N processes
    the lattice is split as the reference's layout splits it.  Device time
    on the library stream, max over ranks."""
    import ctypes as C
    import datetime
    import torch
    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, QOP_invert_arg_t, QOP_resid_arg_t, QOP_EVEN, load_library, layout_hyper
    lib = load_library()
    lib.QOPB_stream.restype = C.c_void_p

    class KStat(C.Structure):
        _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("total_ms", C.c_double),
                    ("bytes_per_launch", C.c_double)]

    lib.QOPB_prof_end.argtypes = [C.POINTER(KStat), C.c_int]
    L = tuple(int(x) for x in (a.lattice or "32,32,32,64").split(","))
    P = layout_hyper(L, world) if world > 1 else (1, 1, 1, 1)
    B = tuple(L[i] // P[i] for i in range(4))
    Vb = int(np.prod(B))
    q = Qop("D")
    # links of this block, smeared on the block lattice
    assert q.init(B) == 0
    U = LT.random_gauge(B, a.eps, a.seed + rank, device="cuda")
    G = q.create_G(U)
    del U
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    q.set_hisq_opts(want_aux=0)
    H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G)
    q.destroy_G(G)
    fat, lng = q.extract_L(q.hisq_asqtad_links(H, 0), Vb)
    q.hisq_destroy_L(H)
    q.finalize()
    src = LT.gaussian_vector(B, a.seed + 100 + rank)
    src[Vb // 2:] = 0
    rsq = a.tol * a.tol

    def measure(label, prec):
        stream = torch.cuda.ExternalStream(lib.QOPB_stream())
        fla = q.create_L_from_raw(fat, lng)
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        q.set_opts(prec_sloppy=prec, cg=0)

        def solve():
            q.dslash(fla, 0.0, hout, hout, QOP_EVEN, QOP_EVEN)   # zero initial guess
            ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
            inf = q.invert(fla, a.mass, hout, hin, QOP_invert_arg_t(1e9, a.dd_max_iter, a.dd_max_iter, 10, QOP_EVEN),
                           ra)
            assert inf.status == 0
            return ra

        for _ in range(a.warmup):
            solve()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        lib.QOPB_prof_begin()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        its = [solve().final_iter for _ in range(a.steps)]
        e1.record(stream)
        e1.synchronize()
        buf = (KStat * 32)()
        n = lib.QOPB_prof_end(buf, 32)
        kst = {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms) for i in range(min(n, 32))}
        ms = reduce_max(e0.elapsed_time(e1) / a.steps, dist, "cuda")
        q.destroy_V(hin)
        q.destroy_V(hout)
        q.destroy_L(fla)
        hop = {k: {"launches": v[0], "us_per_launch": 1e3 * v[1] / max(v[0], 1)} for k, v in kst.items()
               if k.startswith("hop_")}
        return {"label": label, "prec_sloppy": prec, "ms_per_solve": ms, "iters": int(np.median(its)), "hop": hop}

    want = set(a.dd_runs.split(","))
    if not want & {"d16", "d64"}:
        raise SystemExit("--dd-runs needs d16 or d64")
    runs = []
    if world == 1:
        assert q.init(L) == 0
        for prec in (16, 64):
            if "u%d" % prec in want:
                runs.append(measure("undecomposed", prec))
        q.finalize()
        uid = q.comm_unique_id()
    else:
        uid = q.comm_unique_id() if rank == 0 else None
        obj = [uid]
        dist.broadcast_object_list(obj, src=0)
        uid = obj[0]
    assert q.comm_init(uid, world, rank) == 0
    if world == 1:
        assert q.dd_self_split(a.dd_mask) == 0
        assert q.init(L) == 0
    else:
        assert q.init(L, machsize=P) == 0
    info = q.dd_info()
    for prec in (16, 64):
        if "d%d" % prec in want:
            runs.append(measure("decomposed", prec))
    q.finalize()
    q.dd_self_split(0)
    q.comm_finalize()
    dd = next(r for r in runs if r["label"] == "decomposed")
    value = world * 1e3 / dd["ms_per_solve"] if world > 1 else 1e3 / dd["ms_per_solve"]
    if rank == 0:
        line = {"metric": "mixed-prec CG solves/s @%g, decomposed lattice" % a.tol, "value": value, "unit": "solves/s",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": dd["ms_per_solve"],
                "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": "dd", "lattice": L, "grid": P, "block": B, "mask": info["mask"],
                           "mass": a.mass, "tol": a.tol, "eps": a.eps},
                "runs": runs}
        if world == 1:
            ms = {(r["label"][0], r["prec_sloppy"]): r["ms_per_solve"] for r in runs}
            line["overhead_vs_undecomposed"] = {k: ms[("d", p)] / ms[("u", p)] for k, p in (("int16", 16), ("fp64", 64))
                                                if ("d", p) in ms and ("u", p) in ms}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


SERVE_LATTICES = [(16, 16, 16, 16), (24, 24, 24, 48), (32, 32, 32, 64)]


def run_serve(a):
    """Solve service under load: HISQ links resident on 16^4, 24^3x48 and
    32^3x64 (one process, three lattices); requests pick a lattice uniformly,
    a mass log-uniform in [0.005, 0.1], |r|/|b| in {1e-8, 1e-10} and 1-8
    sources (seeded).  Peak throughput is measured on a burst of requests
    submitted at once; then Poisson arrivals at 50 / 80 / 95 % of that peak
    for --serve-seconds each give p50 / p99 latency (submit -> result in the
    caller's buffer) and the throughput achieved."""
    rank, local, world = rank_info()
    import torch
    import threading as th
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    from qopqdp_b200 import lattice as LT
    from qopqdp_b200.qop import Qop, QOP_EVEN
    q = Qop("D")
    assert q.init(SERVE_LATTICES[0]) == 0
    lats, links, pools = [], [], []
    q.set_hisq_opts(want_aux=0)
    for k, L in enumerate(SERVE_LATTICES):
        lat = 0 if k == 0 else q.lattice_create(L)
        assert q.lattice_use(lat) == 0
        U = LT.random_gauge(L, a.eps, a.seed + k, device="cuda")
        G = q.create_G(U)
        del U
        q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
        H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G)
        q.destroy_G(G)
        lats.append(lat)
        links.append((H, q.hisq_asqtad_links(H, 0)))
        srcs = [LT.gaussian_vector(L, a.seed + 100 * k + s) for s in range(8)]
        pools.append((srcs, [np.zeros_like(s) for s in srcs]))
    rng = np.random.default_rng(a.seed + 7 * rank)

    def request():
        k = int(rng.integers(0, len(SERVE_LATTICES)))
        mass = float(np.exp(rng.uniform(np.log(0.005), np.log(0.1))))
        tol = 1e-8 if rng.random() < 0.5 else 1e-10
        return k, mass, tol * tol, int(rng.integers(1, 9))

    def submit(k, mass, rsq, nrhs):
        srcs, dsts = pools[k]
        return q.serve_submit(links[k][1], lats[k], QOP_EVEN, mass, rsq, srcs[:nrhs], dsts[:nrhs])

    def collect(tickets):
        out = []
        for t, nrhs, rsq in tickets:
            rc, res = q.serve_wait(t, 3600.0)
            out.append((rc, res.status, res.total_ms, res.final_rsq_max / rsq, nrhs, res.batch_systems))
        return out

    assert q.set_opts(serve_policy=a.serve_policy) == 0
    assert q.serve_start() == 0
    # warm-up: one request per lattice (builds the int16 link copies)
    collect([(submit(k, 0.05, 1e-16, 1), 1, 1e-16) for k in range(len(SERVE_LATTICES))])
    # peak: a burst submitted at once
    burst = [request() for _ in range(a.serve_burst)]
    t0 = time.perf_counter()
    done = collect([(submit(*r), r[3], r[2]) for r in burst])
    t_peak = time.perf_counter() - t0
    peak = sum(d[4] for d in done) / t_peak
    loads = []
    for frac in (0.5, 0.8, 0.95):
        rate = frac * peak / 4.5                       # requests/s (mean 4.5 sources per request)
        reqs = []
        t_arr = 0.0
        while t_arr < a.serve_seconds:
            t_arr += rng.exponential(1.0 / rate)
            reqs.append((t_arr, request()))
        tickets = []

        def feeder():
            s0 = time.perf_counter()
            for t_at, r in reqs:
                dt = t_at - (time.perf_counter() - s0)
                if dt > 0:
                    time.sleep(dt)
                tickets.append((submit(*r), r[3], r[2]))

        s0 = time.perf_counter()
        f = th.Thread(target=feeder)
        f.start()
        f.join()
        res = collect(tickets)
        wall = time.perf_counter() - s0
        lat = np.array([r[2] for r in res])
        ok = all(r[0] == 0 and r[1] == 0 for r in res)
        loads.append({"load": frac, "requests": len(res), "solves": int(sum(r[4] for r in res)),
                      "offered_solves_per_s": frac * peak, "solves_per_s": sum(r[4] for r in res) / wall,
                      "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                      "mean_batch": float(np.mean([r[5] for r in res])),
                      "max_final_rsq_over_target": max(r[3] for r in res) if res else None, "all_ok": ok})
    q.serve_stop()
    p99 = reduce_max(max(l["p99_ms"] for l in loads), dist, "cuda")
    if rank == 0:
        line = {"metric": "solve service p99 latency and solves/s (3 resident HISQ lattices)",
                "value": peak * world, "unit": "solves/s", "n_gpus": world, "steps": a.serve_burst,
                "warmup": len(SERVE_LATTICES), "ms_per_step": 1e3 * t_peak / a.serve_burst,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": "serve", "lattices": SERVE_LATTICES, "mass": "log-uniform [0.005, 0.1]",
                           "tol": [1e-8, 1e-10], "sources_per_request": "1-8", "burst": a.serve_burst,
                           "seconds_per_load": a.serve_seconds, "policy": a.serve_policy,
                           "parallelism": "replicas x%d" % world},
                "peak_solves_per_s": peak, "loads": loads, "p99_ms_max_over_ranks": p99}
        print(json.dumps(line), flush=True)
    for lat, (H, _) in zip(lats, links):
        q.lattice_use(lat)
        q.hisq_destroy_L(H)
    q.lattice_use(0)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        if a.workload != "single":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm covers the single-solve "
                              "workload only"}), flush=True)
            return
        run_reference(a)
    elif a.workload == "serve":
        run_serve(a)
    elif a.workload == "small":
        run_small(a)
    elif a.workload == "force":
        run_force(a)
    elif a.ab:
        run_ab(a)
    elif a.workload == "dd":
        run_dd(a)
    elif a.workload != "single":
        run_multi(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
