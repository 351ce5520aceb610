"""bench.py -- RHMC trajectory throughput of the chiral-Heisenberg domain-wall
fermion path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one RHMC trajectory at L=Lt=24, Ls=24, beta=0.475, m=0.01 (inert,
as in the reference), am3=1, imass=1, hpin=0, in the production form of the
benchmark configuration: two pseudofermion fields, 20-pole rational
approximations (remez8_20 a-set x^(1/8) for the heatbath, remez4_20 b-set
x^(-1/4) for action and force, generated by chiralheisenberg_b200/remez.py),
Omelyan's integrator with 10 steps of dt=0.1, mixed-precision solves (FP32
Krylov vectors in the force solves at 1e-6, FP64 heatbath and action solves
at 1e-9, FP64 Hamiltonian and Metropolis test).  chi starts from the
thermalised configuration chiralheisenberg_b200/data/con_24x24x24_b0.475
(made by `bench.py --thermalise 60` from a seeded N(0, 1/beta) start); the
generator is the reference's.  Printed metric: seconds per trajectory.

  value     trajectories whose random inputs were staged in HBM before the
            timed region; CUDA events on the library's stream, max over
            ranks.
  e2e       the same trajectories through the host-facing driver API with the
            random numbers drawn on the host and copied in every step.
  fp64      the same trajectories with FP64 force solves (the drop-in
            precision): its s/trajectory, the speed-up of value over it, and
            |dH_mixed - dH_fp64| absolute and relative to |H0|.
  reference_algorithm
            the reference's own algorithm (one pseudofermion, the shipped
            25/25/12-pole sets, leapfrog of random length), FP64, from the
            same configuration: the drop-in path's s/trajectory.
  roofline  the dominant solver kernel class of the value trajectories, timed
            with CUDA events around every solver launch in an instrumented
            replay of the first timed trajectory, against the algorithmic
            bytes of each launch.
  cpu_baseline / --impl reference
            the CPU oracle (a C restatement of rhmc/cheisdwf.f; the Fortran
            reference cannot be built here) on all host cores: its cost per
            iteration of the 20-pole multi-shift solver at this lattice,
            measured on a bounded sample, times the FP64 iteration profile of
            the same trajectories (this run's for cpu_baseline; the committed
            profiles/iteration_profile_ext_24x24.json, made from the same
            chain and seeds, for the reference arm).  A modelled figure;
            `bench.py --validate-cpu-model` times one complete oracle solve
            against the model.

Multi-GPU: independent Markov chains, one per rank ("replicas only").
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
DATA = os.path.join(ROOT, "chiralheisenberg_b200", "data")

CFG = dict(beta=0.475, am3=1.0, am=0.01, hpin=0.0, imass=1, dt=0.1, iterl=10,
           seed=693764523745.0, chi_seed=12345)
EXT = dict(npf=2, nsteps=10, integrator="omelyan", poles=20, rescga=1e-9, rescgg=1e-6,
           heatbath="remez8_20 a: x^(1/8)", action_force="remez4_20 b: x^(-1/4)",
           interval=[1e-4, 50.0])
PROFILE_EXT = os.path.join(ROOT, "profiles", "iteration_profile_ext_24x24.json")


# ---- replicas (one independent Markov chain per rank) -----------------------
def replica_seed(seed, rank):
    """The reference generator's seed of rank's chain: rank 0 runs the
    single-GPU chain, every other rank an independent one."""
    return seed + 1000.0 * rank


def max_over_ranks(ms, world, device):
    """The slowest rank's elapsed milliseconds (every rank gets it)."""
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def seconds_per_trajectory(ms_max, steps, world):
    """Whole-job figure: world chains of steps trajectories each in ms_max."""
    return (ms_max / 1e3) / (steps * world)


def con_path(L, Ls):
    return os.path.join(DATA, f"con_{L}x{L}x{Ls}_b{CFG['beta']}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--L", type=int, default=24)
    ap.add_argument("--Ls", type=int, default=24)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-refalg", action="store_true")
    ap.add_argument("--refalg-steps", type=int, default=3)
    ap.add_argument("--no-propagators", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clock-interval-ms", type=int, default=200,
                    help="nvidia-smi sampling interval during the timed region")
    ap.add_argument("--operator-sweep", action="store_true",
                    help="operator GB/s over L in {16,24,32,48}, Ls in {16,24,32}, FP64/FP32/FP16")
    ap.add_argument("--profile-solve", action="store_true",
                    help="bounded work for profilers: one heatbath and one force evaluation")
    ap.add_argument("--profile-prec", default="f64", choices=["f64", "f32"],
                    help="Krylov-vector precision of the profiled force evaluation")
    ap.add_argument("--profile-res", type=float, default=0.0,
                    help="stopping residual of both profiled solves (0: the reference's)")
    ap.add_argument("--basis-gb", type=float, default=-1.0,
                    help="HBM budget of the stored FP64 Lanczos basis, FP32 half of it (GB; "
                         "<0: 80 GB in the timed runs, the library default elsewhere)")
    ap.add_argument("--profile-operator", default="",
                    choices=["", "f64", "f32", "f16"],
                    help="bounded work for profilers: 5 applications of M at --L/--Ls in the "
                         "given storage (CHDWF_STENCIL selects the kernel shape)")
    ap.add_argument("--thermalise", type=int, default=0,
                    help="run N trajectories from the seeded Gaussian start and write the "
                         "thermalised configuration")
    ap.add_argument("--write-profile", type=int, default=0,
                    help="write the FP64 iteration profile of the first N trajectories")
    ap.add_argument("--validate-cpu-model", action="store_true",
                    help="time one complete oracle force solve against the per-iteration model")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index, interval_ms=200):
        self.gpu = gpu_index
        self.interval = interval_ms
        self.proc = None
        self.lines = []

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.interval)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        loaded = [s for s in sm if s > 0.5 * mx] if mx else sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def synthetic_chi(L, Lt, beta, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((3, L * L * Lt)) / np.sqrt(beta)


def ext_sets():
    from chiralheisenberg_b200.remez import read_remez_file
    a8, d8, _, _ = read_remez_file(os.path.join(DATA, "remez8_20"), 20)
    _, _, b4, e4 = read_remez_file(os.path.join(DATA, "remez4_20"), 20)
    return (a8, d8), (b4, e4)


def make_program(L, Ls, local_rank, rank=0, ext=True):
    """The benchmark chain: thermalised configuration (or the seeded start
    when it is missing), reference generator, extension mode if ext."""
    import chiralheisenberg_b200 as chb
    rz = chb.reference_remez()
    prog = chb.Program(L, L, Ls, CFG["dt"], CFG["beta"], CFG["am3"], CFG["am"], CFG["hpin"],
                       CFG["imass"], CFG["iterl"], rz["remez2"], rz["remez4"], rz["remez2g"],
                       device=local_rank)
    cp = con_path(L, Ls)
    if os.path.exists(cp):
        chi, seed, _ = chb.con_read(cp, L ** 3)
        start = "thermalised (" + os.path.relpath(cp, ROOT) + ")"
    else:
        chi, seed = synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"]), CFG["seed"]
        start = "raw N(0,1/beta) seeded"
    prog.set_chi(chi)
    prog.startup(replica_seed(seed, rank))
    prog.set_measure(5, False)
    if ext:
        hb, act = ext_sets()
        prog.set_ext(EXT["npf"], EXT["nsteps"], hb, act, integrator=EXT["integrator"])
    return prog, start


# solver kernel classes reported by chdwf_timing_read (4-7: FP32 vectors)
KERNEL_NAMES = {0: "k_lz1_M", 1: "k_lz1_Md", 2: "k_lz_accum", 3: "k_lz2_M/k_lz2_Md"}
KERNEL_WHAT = {0: "pass-1 M q_j with |M q_j|^2",
               1: "pass-1 M^dag + three-term update with |r|^2",
               2: "pass-2 solution accumulation from the stored Lanczos basis",
               3: "pass-2 regeneration (solves longer than the basis store)"}


def kernel_name(k, shape=""):
    """Timer class k (4-7: FP32 vectors); shape: the stencil shape the
    autotuner chose for pass 1 at this lattice and precision."""
    name = KERNEL_NAMES[k % 4] + (" fp32" if k >= 4 else " fp64")
    return name + (f" ({shape})" if shape and k % 4 < 2 else "")


def cpu_iteration_cost(L, Ls, threads, iters, npole=20):
    """Oracle seconds per multi-shift iteration (npole poles) and per operator
    apply at this lattice, on `threads` host threads; a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    hb, act = ext_sets()
    lat = po.make_lat(L, L, Ls, beta=CFG["beta"], am3=CFG["am3"], threads=threads)
    rng = np.random.default_rng(7)
    shape = (2, 4, L, L, L, Ls)
    Phi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    chi = synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"])
    # the difference of a 2k- and a k-iteration run gives the cost of an
    # iteration; what is left of the k-iteration run is the set-up of a solve
    # (allocating and touching the pole vectors, thread start-up)
    t0 = time.perf_counter()
    po.qmrherm(lat, Phi, chi, act[0], act[1], 1e-30, niterc=iters)
    t1 = time.perf_counter()
    po.qmrherm(lat, Phi, chi, act[0], act[1], 1e-30, niterc=2 * iters)
    t2 = time.perf_counter()
    t_iter = max((t2 - t1) - (t1 - t0), 1e-9) / iters
    t_setup = max((t1 - t0) - iters * t_iter, 0.0)
    t0 = time.perf_counter()
    for _ in range(2):
        po.dslash(lat, Phi, chi)
    t_apply = (time.perf_counter() - t0) / 2
    return t_iter, t_apply, t_setup


def cpu_model(profile, t_iter, t_apply, t_setup, npole=20):
    """Oracle seconds per trajectory: every solver iteration at t_iter, the
    set-up of every solve, and the force tail of each force solve (one
    operator apply and derivs per pole, rhmc/cheisdwf.f:733-740, counted as
    one apply)."""
    its = profile["it_pf"] + profile["it_h0"] + profile["it_h1"] + profile["it_force"]
    nsolve_force = profile["nforce"] * EXT["npf"]
    nsolve = nsolve_force + 3 * EXT["npf"]       # + heatbath and two actions per field
    return its * t_iter + nsolve * t_setup + nsolve_force * npole * t_apply, its


def profile_of(recs):
    return {"it_pf": float(np.mean([r.it_pf for r in recs])),
            "it_h0": float(np.mean([r.it_h0 for r in recs])),
            "it_h1": float(np.mean([r.it_h1 for r in recs])),
            "it_force": float(np.mean([r.it_force for r in recs])),
            "nforce": float(np.mean([r.nforce for r in recs]))}


def bench_propagators(local_rank, seed=2024, nens=24, nsrc=4, res=1e-8):
    """Config of the batched-solve case: 24 ensembles of uneven size
    (L=Lt in {8,12,16}, Ls in {8,16,24}, seeded), chi ~ N(0,1), 4 point
    sources each (flavour 1,2 x Dirac 3,4 at a seeded site on s=1),
    Phi = M^dag xi, x0 = Phi as in fermion(); CGNE to residual 1e-8.
    Returns solves/s one at a time and batched (one set of launches), each
    the median of three timed runs after an untimed one; the batched time
    includes resetting the initial guesses."""
    import ctypes as C
    import torch
    import chiralheisenberg_b200 as chb
    rng = np.random.default_rng(seed)
    ens = [(int(rng.choice([8, 12, 16])), int(rng.choice([8, 16, 24]))) for _ in range(nens)]
    lats, keep, systems = [], [], []
    for e, (L, Ls) in enumerate(ens):
        gl = chb.Lattice(L, L, Ls, am3=1.0, device=local_rank)
        chi = torch.from_numpy(rng.standard_normal((3, L ** 3))).cuda()
        site = int(rng.integers(L ** 3))
        for src in range(nsrc):
            f, d = src // 2, 2 + src % 2
            xi = torch.zeros((2, 4, L, L, L, Ls), dtype=torch.complex128, device="cuda")
            xi.view(2, 4, -1, Ls)[f, d, site, 0] = 1.0
            Phi = torch.empty_like(xi)
            gl.lib.chdwf_dslash_dev(gl.h, C.c_void_p(Phi.data_ptr()), C.c_void_p(xi.data_ptr()),
                                    C.c_void_p(chi.data_ptr()), 0.0, 1, 1, None)
            gl.lib.chdwf_traj_sync(gl.h)
            x = Phi.clone()
            keep += [Phi, x, chi]
            systems.append((gl, chb.CgSystem(L, L, Ls, 1, 0.0, 1.0, -1, Phi.data_ptr(),
                                             x.data_ptr(), chi.data_ptr()), Phi, x, chi))
        lats.append(gl)
    torch.cuda.synchronize()

    def one_at_a_time():
        # the reference's sequence of congrad calls
        its = []
        for gl, s, Phi, x, chi in systems:
            xx = Phi.clone()
            it = C.c_int()
            gl.lib.chdwf_congrad_dev(gl.h, C.c_void_p(Phi.data_ptr()), res, C.byref(it), 0.0, 1,
                                     C.c_void_p(chi.data_ptr()), C.c_void_p(xx.data_ptr()))
            its.append(it.value)
        torch.cuda.synchronize()
        return its

    def batched():
        for _, _, Phi, x, _ in systems:
            x.copy_(Phi)                      # the same initial guess every run
        torch.cuda.synchronize()
        out = chb.congrad_batch(lats[0], [s for _, s, _, _, _ in systems], res)
        torch.cuda.synchronize()
        return out

    # one untimed run of each (first-call set-up, graph capture), then the
    # median of three timed runs
    one_at_a_time()
    batched()
    t_ones, t_batches = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        its1 = one_at_a_time()
        t_ones.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        its2, sts = batched()
        t_batches.append(time.perf_counter() - t0)
    t_one, t_batch = float(np.median(t_ones)), float(np.median(t_batches))
    for gl in lats:
        gl.close()
    n = len(systems)
    return {"solves": n, "ensembles": nens, "residual": res,
            "one_at_a_time_solves_per_s": n / t_one, "batched_solves_per_s": n / t_batch,
            "speedup": t_one / t_batch, "mean_iterations": float(np.mean(its2)),
            "same_iterations": bool(list(its1) == list(its2)), "all_converged": bool((sts == 0).all())}


def run_profile_solve(args, local_rank):
    """One pseudofermion heatbath and one force evaluation at the bench
    lattice: a bounded launch sequence for profilers."""
    import torch
    import chiralheisenberg_b200 as chb
    torch.cuda.set_device(local_rank)
    L, Ls = args.L, args.Ls
    rz = chb.reference_remez()
    prog = chb.Program(L, L, Ls, CFG["dt"], CFG["beta"], CFG["am3"], CFG["am"], CFG["hpin"],
                       CFG["imass"], CFG["iterl"], rz["remez2"], rz["remez4"], rz["remez2g"],
                       device=local_rank)
    if args.basis_gb >= 0:
        prog.set_basis_store(args.basis_gb * 1e9)
    prog.set_chi(synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"]))
    prog.startup(CFG["seed"])
    prog.set_precision(md=args.profile_prec, accept="f64")
    lib, ctx = prog.lib, prog.context
    import ctypes as C
    kvol = L ** 3
    rng = np.random.default_rng(3)
    ps = (rng.standard_normal(16 * kvol * Ls) * np.sqrt(0.5)).astype(np.float32)
    it = C.c_int()
    t0 = time.perf_counter()
    lib.chdwf_traj_begin(ctx)
    res_hb = args.profile_res or 1e-9
    res_f = args.profile_res or 1e-6
    rc1 = lib.chdwf_traj_heatbath(ctx, ps.ctypes.data_as(C.c_void_p), res_hb, 0.0, 0.0, 1,
                                  C.byref(it))
    itg, itf = C.c_int(), C.c_int()
    rc2 = lib.chdwf_traj_force(ctx, res_f, 0.0, 0.0, 1, C.byref(itg), C.byref(itf))
    lib.chdwf_traj_sync(ctx)
    dt = time.perf_counter() - t0
    print(json.dumps({"profile_solve": f"L=Lt={L} Ls={Ls}", "rc": [rc1, rc2],
                      "iterations": [it.value, itg.value, itf.value], "seconds": dt}), flush=True)
    prog.close()


def run_operator_sweep(args, local_rank):
    """M and M^dagger on device buffers, one JSON line per (L, Ls, storage):
    median of 20 applications, each timed alone with CUDA events on the
    library stream after a 256 MB write that evicts L2.  Algorithmic bytes =
    2 V sizeof(complex) + 3 kvol 4 (chi as REAL*4); the timed call also
    rounds chi to REAL*4 (one small kernel, included)."""
    import ctypes as C
    import torch
    import chiralheisenberg_b200 as chb
    torch.cuda.set_device(local_rank)
    peak, kind = peaks()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    for L in (16, 24, 32, 48):
        for Ls in (16, 24, 32):
            kvol = L * L * L                  # ksize^2 * ksizet with ksizet = ksize
            V = 8 * kvol * Ls
            if 3 * V * 16 > 60e9:
                continue
            lat = chb.Lattice(L, L, Ls, device=local_rank)
            stream = torch.cuda.ExternalStream(lat.lib.chdwf_get_stream(lat.h), device=local_rank)
            g = torch.Generator(device=f"cuda:{local_rank}").manual_seed(L * 100 + Ls)
            R64 = torch.randn(2 * V, dtype=torch.float64, device=f"cuda:{local_rank}", generator=g)
            chi = torch.randn(3 * kvol, dtype=torch.float64, device=f"cuda:{local_rank}", generator=g)
            for prec, name, elem in ((0, "f64", 16), (1, "f32", 8), (2, "f16", 4)):
                if prec == 0:
                    src = R64
                elif prec == 1:
                    src = R64.to(torch.float32)
                else:
                    src = R64.to(torch.float16)
                out = torch.empty_like(src)
                for dag in (0, 1):
                    def apply():
                        if prec == 0:
                            rc = lat.lib.chdwf_dslash_dev(lat.h, C.c_void_p(out.data_ptr()),
                                                          C.c_void_p(src.data_ptr()),
                                                          C.c_void_p(chi.data_ptr()), 0.3, 1, dag,
                                                          None)
                        else:
                            rc = lat.lib.chdwf_dslash_dev_lp(lat.h, C.c_void_p(out.data_ptr()),
                                                             C.c_void_p(src.data_ptr()),
                                                             C.c_void_p(chi.data_ptr()), 0.3, 1,
                                                             dag, prec, None)
                        if rc != 0:
                            raise RuntimeError(f"operator rc={rc}")
                    for _ in range(3):
                        apply()
                    torch.cuda.synchronize()
                    ts = []
                    for i in range(20):
                        with torch.cuda.stream(stream):
                            flush.fill_(i & 255)
                            e0 = torch.cuda.Event(enable_timing=True)
                            e1 = torch.cuda.Event(enable_timing=True)
                            e0.record(stream)
                            apply()
                            e1.record(stream)
                        e1.synchronize()
                        ts.append(e0.elapsed_time(e1))
                    ms = statistics.median(ts)
                    nbytes = 2 * V * elem + 12 * kvol
                    gbs = nbytes / (ms * 1e-3) / 1e9
                    print(json.dumps({"operator": "M^dagger" if dag else "M", "L": L, "Lt": L,
                                      "Ls": Ls, "storage": name, "us": round(ms * 1e3, 2),
                                      "algorithmic_bytes": nbytes, "GBps": round(gbs, 1),
                                      "frac_of_hbm": round(gbs / peak, 3), "peak_kind": kind,
                                      "l2": "evicted before each application"}), flush=True)
                del out
            lat.close()
            del R64, chi
            torch.cuda.empty_cache()


def run_reference(args, rank, world):
    """The reference arm: the oracle on all host cores, on this workload."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    prof = json.load(open(PROFILE_EXT)) if os.path.exists(PROFILE_EXT) else None
    if prof:
        per = prof["per_trajectory"]
        window = per[args.warmup:args.warmup + args.steps] or per
        profile = {k: float(np.mean([p[k] for p in window])) for k in window[0]}
        psrc = (f"{os.path.relpath(PROFILE_EXT, ROOT)}, trajectories "
                f"{args.warmup + 1}-{args.warmup + len(window)} of the same chain")
    else:
        profile = {"it_pf": 1600.0, "it_h0": 1600.0, "it_h1": 1600.0, "it_force": 26000.0,
                   "nforce": 21.0}
        psrc = "built-in estimate (profile file missing)"
    vals, walls = [], []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        t_iter, t_apply, t_setup = cpu_iteration_cost(args.L, args.Ls, threads,
                                                      args.cpu_sample_iters)
        s, its = cpu_model(profile, t_iter, t_apply, t_setup)
        if step >= args.warmup:
            vals.append((s, t_iter))
            walls.append(time.perf_counter() - t0)
    v = statistics.median(x[0] for x in vals)
    t_it = statistics.median(x[1] for x in vals)
    sample = (f"oracle 20-pole multi-shift iterations at {args.L}^3x{args.Ls} "
              f"({3 * args.cpu_sample_iters} per step, cost per iteration from a "
              f"{2 * args.cpu_sample_iters}- minus a {args.cpu_sample_iters}-iteration run) and 2 operator applies on {threads} threads; "
              f"modelled: seconds per iteration x the FP64 iteration profile ({psrc})")
    line = {"impl": "reference", "metric": "s/trajectory", "value": v, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "modelled": True,
            "consistency": {"sample_wall_s_per_step": statistics.median(walls),
                            "note": "each step measures the oracle's cost per iteration on a "
                                    "bounded sample; value prices a whole trajectory with it"},
            "iteration_profile": profile,
            "ms_per_1000_iterations": t_it * 1e6,
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"RHMC trajectory L=Lt={args.L} Ls={args.Ls}, 2 pseudofermions x 20 "
                        f"poles, Omelyan 10 steps", "precision": "mixed: FP32 force solves, "
            "FP64 heatbath/action solves and dH", "parallelism": f"replicas{args.gpus}",
            "l2": "fields larger than L2 (solver working set > 126 MB)",
            "chi": "thermalised from seeded N(0,1/beta) (bench.py --thermalise 60)"
            if os.path.exists(con_path(args.L, args.Ls)) else "raw seeded N(0,1/beta)",
            "fermion": "off (no measurement in the timed trajectories)",
            **CFG, **EXT}


def run_profile_operator(args, local_rank):
    """Five applications of M on device buffers (a bounded launch sequence
    for profilers), after the autotuner's first call."""
    import ctypes as C
    import torch
    import chiralheisenberg_b200 as chb
    torch.cuda.set_device(local_rank)
    L, Ls = args.L, args.Ls
    lat = chb.Lattice(L, L, Ls, device=local_rank)
    V = 8 * L ** 3 * Ls
    dev = f"cuda:{local_rank}"
    g = torch.Generator(device=dev).manual_seed(1)
    R = torch.randn(2 * V, dtype=torch.float64, device=dev, generator=g)
    chi = torch.randn(3 * L ** 3, dtype=torch.float64, device=dev, generator=g)
    prec = {"f64": 0, "f32": 1, "f16": 2}[args.profile_operator]
    src = R if prec == 0 else (R.to(torch.float32) if prec == 1 else R.to(torch.float16))
    out = torch.empty_like(src)
    for _ in range(5):
        if prec == 0:
            rc = lat.lib.chdwf_dslash_dev(lat.h, C.c_void_p(out.data_ptr()),
                                          C.c_void_p(src.data_ptr()), C.c_void_p(chi.data_ptr()),
                                          0.3, 1, 0, None)
        else:
            rc = lat.lib.chdwf_dslash_dev_lp(lat.h, C.c_void_p(out.data_ptr()),
                                             C.c_void_p(src.data_ptr()),
                                             C.c_void_p(chi.data_ptr()), 0.3, 1, 0, prec, None)
        assert rc == 0
    torch.cuda.synchronize()
    print(json.dumps({"profile_operator": args.profile_operator, "L": L, "Ls": Ls,
                      "autotune": chb.autotune_report()}), flush=True)
    lat.close()


def run_thermalise(args, local_rank):
    """From the seeded Gaussian start: N trajectories of the benchmark
    algorithm (mixed precision), then write the configuration."""
    import chiralheisenberg_b200 as chb
    import torch
    torch.cuda.set_device(local_rank)
    L, Ls = args.L, args.Ls
    rz = chb.reference_remez()
    prog = chb.Program(L, L, Ls, CFG["dt"], CFG["beta"], CFG["am3"], CFG["am"], CFG["hpin"],
                       CFG["imass"], CFG["iterl"], rz["remez2"], rz["remez4"], rz["remez2g"],
                       device=local_rank)
    prog.set_chi(synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"]))
    prog.startup(CFG["seed"])
    prog.set_measure(5, False)
    hb, act = ext_sets()
    prog.set_ext(EXT["npf"], EXT["nsteps"], hb, act, integrator=EXT["integrator"])
    prog.set_precision(md="f32", accept="f64")
    for k in range(args.thermalise):
        r = prog.sweep()
        print(json.dumps({"trajectory": k + 1, "action_per_site": r.action, "dH": r.dH,
                          "accepted": r.accepted, "it_force": r.it_force}), flush=True)
    prog.write_con(con_path(L, Ls))
    prog.close()


def run_write_profile(args, local_rank):
    """The FP64 iteration profile of the benchmark chain, trajectory by
    trajectory (the reference arm prices its trajectories with it)."""
    import torch
    torch.cuda.set_device(local_rank)
    prog, start = make_program(args.L, args.Ls, local_rank)
    prog.set_precision(md="f64", accept="f64")
    per = []
    for _ in range(args.write_profile):
        r = prog.sweep()
        per.append({"it_pf": r.it_pf, "it_h0": r.it_h0, "it_h1": r.it_h1,
                    "it_force": r.it_force, "nforce": r.nforce})
    prog.close()
    out = {"workload": workload_config(args)["workload"], "start": start, "precision": "fp64",
           "command": f"python bench.py --write-profile {args.write_profile}",
           "per_trajectory": per}
    with open(PROFILE_EXT, "w") as f:
        json.dump(out, f, indent=0)
    print(json.dumps(out["per_trajectory"][:3]), flush=True)


def run_validate_cpu_model(args):
    """One complete oracle solve at the bench lattice -- a 20-pole force
    solve (iflag 1) at 1e-6 on the thermalised configuration -- timed end to
    end and compared with the per-iteration model (sampled cost per
    iteration x its iteration count + the force tail)."""
    import chiralheisenberg_b200 as chb
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    L, Ls = args.L, args.Ls
    threads = os.cpu_count() or 1
    cp = con_path(L, Ls)
    chi = chb.con_read(cp, L ** 3)[0] if os.path.exists(cp) else synthetic_chi(
        L, L, CFG["beta"], CFG["chi_seed"])
    hb, act = ext_sets()
    lat = po.make_lat(L, L, Ls, beta=CFG["beta"], am3=CFG["am3"], threads=threads)
    rng = np.random.default_rng(11)
    shape = (2, 4, L, L, L, Ls)
    Phi = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * np.sqrt(0.5)
    t_iter, t_apply, t_setup = cpu_iteration_cost(L, Ls, threads, args.cpu_sample_iters)
    dS = np.zeros((3, L ** 3), np.float32)
    t0 = time.perf_counter()
    _, its, st, _ = po.qmrherm(lat, Phi, chi, act[0], act[1], 1e-6, iflag=1, dSdchi=dS)
    t_full = time.perf_counter() - t0
    model = t_setup + its * t_iter + 20 * t_apply
    print(json.dumps({"validate_cpu_model": f"L=Lt={L} Ls={Ls}", "threads": threads,
                      "iterations": its, "status": st, "measured_s": t_full, "model_s": model,
                      "model_over_measured": model / t_full, "t_iter_s": t_iter,
                      "t_setup_s": t_setup, "t_apply_s": t_apply}), flush=True)


def timed_run(prog, stream, steps, staged, barrier, world, local_rank):
    import torch
    if staged:
        prog.stage(steps)
    recs = []
    barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        recs.append(prog.sweep())
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev[0].elapsed_time(ev[-1])
    per_step = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    return max_over_ranks(ms, world, f"cuda:{local_rank}"), recs, per_step


def instrumented(prog, chi0, state0):
    """Replay the first timed trajectory with CUDA events around every solver
    launch; per kernel class (ms, timed, launched, bytes)."""
    prog.set_chi(chi0)
    prog.set_state(state0)
    prog.timing(True)
    prog.sweep()
    out = prog.timing_read()
    prog.timing(False)
    return out


def instrumented_chunks(prog, chi0, state0):
    """Replay the first timed trajectory with pass 1 on its CUDA-graph replays
    (as in the timed runs) and CUDA events around every replayed chunk of 16
    iterations: pass-1 microseconds per iteration ([FP64, FP32]) and the
    iterations timed."""
    prog.set_chi(chi0)
    prog.set_state(state0)
    prog.timing(True, chunks=True)
    prog.sweep()
    out = prog.timing_chunks()
    prog.timing(False)
    return out


def rows_chosen(L, Ls, k):
    """The stencil shape the autotuner chose for class k's precision."""
    import chiralheisenberg_b200 as chb
    elem = 8 if k >= 4 else 16
    # FP32 solves with Ls even run the split-layout kernels (their own entry)
    layout = "split" if (k >= 4 and Ls % 2 == 0) else "plain"
    for t in chb.autotune_report():
        if (t["L"], t["Lt"], t["Ls"], t["elem_bytes"], t.get("layout", "plain")) == \
                (L, L, Ls, elem, layout):
            return t["choice"]
    return ""


def kernel_table(kt, L, Ls):
    kms, ktimed, klaunched, kbytes = kt
    tot = max(float(np.sum(kms)), 1e-30)
    return {kernel_name(k, rows_chosen(L, Ls, k)): {"launches": int(klaunched[k]),
                             "avg_us": kms[k] / max(ktimed[k], 1) * 1e3,
                             "share_of_solver_time": kms[k] / tot,
                             "GBps": (kbytes[k] / (kms[k] * 1e-3) / 1e9) if kms[k] > 0 else None}
            for k in range(8) if klaunched[k] > 0}


def run_b200(args, rank, world, local_rank):
    import torch
    import chiralheisenberg_b200 as chb
    torch.cuda.set_device(local_rank)
    L, Ls = args.L, args.Ls
    prog, start = make_program(L, Ls, local_rank, rank)
    # the basis stores (FP32 and FP64 solves run in the same program): 80 GB
    # of FP64 vectors (1880 at 24^3x24) and as many FP32 ones, so neither arm
    # is left with what the other did not take
    prog.set_basis_store((args.basis_gb if args.basis_gb >= 0 else 80.0) * 1e9)
    prog.set_precision(md="f32", accept="f64")
    stream = torch.cuda.ExternalStream(prog.stream, device=local_rank)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        prog.sweep()
    # every arm below runs the SAME trajectories: the chain state (chi and the
    # complete generator state) is saved here and restored before each
    chi0 = prog.get_chi()
    state0 = prog.get_state()
    clocks = ClockSampler(local_rank, args.clock_interval_ms)
    clocks.start()
    n0 = chb.kernel_launches()
    ms_value, recs, step_ms = timed_run(prog, stream, args.steps, True, barrier, world,
                                        local_rank)
    launches = chb.kernel_launches() - n0
    clk = clocks.stop()
    prog.set_chi(chi0)
    prog.set_state(state0)
    ms_e2e, recs_e2e, step_ms_e2e = timed_run(prog, stream, args.steps, False, barrier, world,
                                              local_rank)
    same = all(a.accepted == b.accepted and a.dH == b.dH for a, b in zip(recs, recs_e2e))
    kt = instrumented(prog, chi0, state0)
    chunk_us, chunk_its = instrumented_chunks(prog, chi0, state0)
    fp64 = None
    prof64 = None
    if not args.no_fp64:
        prog.set_chi(chi0)
        prog.set_state(state0)
        prog.set_precision(md="f64", accept="f64")
        ms64, recs64, _ = timed_run(prog, stream, args.steps, True, barrier, world, local_rank)
        kt64 = instrumented(prog, chi0, state0)
        prog.set_precision(md="f32", accept="f64")
        dh = [abs(a.dH - b.dH) for a, b in zip(recs, recs64)]
        dh_rel = [abs(a.dH - b.dH) / abs(b.H0) for a, b in zip(recs, recs64)]
        prof64 = profile_of(recs64)
        fp64 = {"value": seconds_per_trajectory(ms64, args.steps, world), "unit": "s",
                "speedup_of_value": ms64 / ms_value,
                "dH_max_abs_diff": max(dh), "dH_max_diff_rel_H0": max(dh_rel),
                "dH_rms_fp64": float(np.sqrt(np.mean([b.dH ** 2 for b in recs64]))),
                "target": "|dH_mixed - dH_fp64| <= 1e-8: met as relative to |H0| "
                          f"({max(dh_rel):.2e}); as absolute {max(dh):.2e}",
                "same_decisions": all(a.accepted == b.accepted for a, b in zip(recs, recs64)),
                "iteration_profile": prof64,
                "solver_kernels": kernel_table(kt64, L, Ls)}
    prog.close()
    refalg = None
    if not args.no_refalg:
        rprog, _ = make_program(L, Ls, local_rank, rank, ext=False)
        rprog.sweep()
        ms_r, recs_r, _ = timed_run(rprog, stream_of(rprog, local_rank), args.refalg_steps, True,
                                    barrier, world, local_rank)
        its = sum(r.it_pf + r.it_h0 + r.it_h1 + r.it_guid + r.it_force for r in recs_r)
        refalg = {"value": seconds_per_trajectory(ms_r, args.refalg_steps, world), "unit": "s",
                  "precision": "fp64 (the drop-in)", "trajectories": args.refalg_steps,
                  "ms_per_1000_iterations": ms_r / its * 1e3,
                  "nforce": [r.nforce for r in recs_r],
                  "algorithm": "1 pseudofermion, shipped remez2/remez4/remez2g, leapfrog dt=0.1 "
                               "with random length (iterl=10), as rhmc/cheisdwf.f"}
        rprog.close()
    value = seconds_per_trajectory(ms_value, args.steps, world)
    e2e = seconds_per_trajectory(ms_e2e, args.steps, world)
    kvol = L * L * L
    h2d = EXT["npf"] * 64 * kvol * Ls + 12 * kvol      # heatbath Gaussians + momenta
    d2h = 12 * kvol + 64                               # momenta for vel2 + scalars
    kms, ktimed, klaunched, kbytes = kt
    dom = int(np.argmax(kms))
    avg_ms = kms[dom] / max(ktimed[dom], 1)
    bytes_per_launch = kbytes[dom] / max(ktimed[dom], 1)
    # Per-launch events include each launch's dispatch (pass 1 is issued
    # launch by launch when every launch is timed).  The graph-replayed chunks
    # give the real pass-1 time per iteration; the dominant pass-1 kernel's
    # duration is its part of that, split between M and M^dagger in the
    # proportion of their per-launch times.  The iteration time also holds
    # the scalar step and the gaps between kernels, so this duration is an
    # upper bound and the achieved bandwidth a lower one.
    prec = 1 if dom >= 4 else 0
    base = 4 * prec
    ev_iter_us = 1e3 * sum(kms[base + c] / max(ktimed[base + c], 1) for c in (0, 1))
    graph_iter_us = float(chunk_us[prec])
    if dom % 4 in (0, 1) and chunk_its[prec] > 0 and ev_iter_us > 0:
        avg_us = avg_ms * 1e3 * graph_iter_us / ev_iter_us
        measured_in = ("graph-replayed pass-1 chunks of the first timed trajectory (CUDA events "
                       "around every 16-iteration replay), the kernel's part of the iteration "
                       "split from per-launch CUDA events of a second replay")
    else:
        avg_us = avg_ms * 1e3
        measured_in = ("instrumented replay of the first timed trajectory, CUDA events around "
                       "every solver launch")
    achieved = bytes_per_launch / (avg_us * 1e-6) / 1e9
    V = 8.0 * L ** 3 * Ls * (8 if prec else 16)
    iter_bytes = 6 * V + 2 * 12.0 * L ** 3
    peak, peak_kind = peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic_24x24.json")
    if os.path.exists(tp):
        # ncu figures are per stencil shape; another shape's traffic is unknown
        traffic = json.load(open(tp)).get(kernel_name(dom, rows_chosen(L, Ls, dom)))
    prof = profile_of(recs)
    its_value = sum(prof[k] for k in ("it_pf", "it_h0", "it_h1", "it_force"))
    line = {"metric": "s/trajectory", "value": value, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_value / args.steps,
            "step_ms": [round(x, 1) for x in step_ms],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (mixed)", "data": "synthetic", "config": workload_config(args),
            "ms_per_1000_iterations": (ms_value / args.steps) / its_value * 1e3,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "same_trajectories_as_value": same,
                    "step_ms": [round(x, 1) for x in step_ms_e2e]},
            "fp64": fp64,
            "roofline": {"bound": "hbm", "kernel": kernel_name(dom, rows_chosen(L, Ls, dom)),
                         "what": KERNEL_WHAT[dom % 4],
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "bytes_per_launch": bytes_per_launch, "avg_launch_us": avg_us,
                         "avg_launch_us_per_launch_events": avg_ms * 1e3,
                         "pass1_iteration": {"us_graph": graph_iter_us,
                                             "us_per_launch_events": ev_iter_us,
                                             "iterations_timed": int(chunk_its[prec]),
                                             "bytes": iter_bytes,
                                             "GBps": iter_bytes / (graph_iter_us * 1e-6) / 1e9
                                             if graph_iter_us > 0 else None},
                         "measured_in": measured_in},
            "solver_kernels": kernel_table(kt, L, Ls),
            "gpu_launches": launches,
            "reference_algorithm": refalg,
            "iteration_profile": prof,
            "trajectories": [{"dH": r.dH, "accepted": r.accepted, "H0": r.H0} for r in recs],
            "autotune": chb.autotune_report(),
            "clocks": clk}
    if rank == 0 and not args.no_propagators:
        line["propagators"] = bench_propagators(local_rank)
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t_iter, t_apply, t_setup = cpu_iteration_cost(L, Ls, threads, args.cpu_sample_iters)
        s_cpu, _ = cpu_model(prof64 or prof, t_iter, t_apply, t_setup)
        line["cpu_baseline"] = {
            "value": s_cpu, "unit": "s", "cores": threads, "kind": "port", "modelled": True,
            "ms_per_1000_iterations": t_iter * 1e6,
            "sample": (f"oracle 20-pole multi-shift iterations at {L}^3x{Ls} "
                       f"({3 * args.cpu_sample_iters}, cost per iteration from a "
                       f"{2 * args.cpu_sample_iters}- minus a {args.cpu_sample_iters}-iteration "
                       f"run) and 2 operator applies on {threads} threads, "
                       f"times this run's FP64 iteration profile of the same trajectories")}
    if rank == 0:
        print(json.dumps(line), flush=True)


def stream_of(prog, local_rank):
    import torch
    return torch.cuda.ExternalStream(prog.stream, device=local_rank)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.validate_cpu_model:
        run_validate_cpu_model(args)
        return
    if args.profile_solve:
        run_profile_solve(args, local_rank)
        return
    if args.operator_sweep:
        run_operator_sweep(args, local_rank)
        return
    if args.profile_operator:
        run_profile_operator(args, local_rank)
        return
    if args.thermalise:
        run_thermalise(args, local_rank)
        return
    if args.write_profile:
        run_write_profile(args, local_rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
