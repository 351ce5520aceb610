"""bench.py -- RHMC trajectory throughput of the chiral-Heisenberg domain-wall
path on B200, in the reference's own algorithm (1 pseudofermion, the shipped
25/25/12-pole Remez sets, leapfrog with random trajectory length).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--L 24] [--Ls 24]

A step is one RHMC trajectory (heatbath, H0, molecular dynamics with a force
evaluation per step, H1, Metropolis) at L=Lt=24, Ls=24 on synthetic fields:
chi drawn from a seeded N(0, 1/beta), the reference's random-number generator
from its default seed.  Measurements (fermion()) are off.  Printed metric:
seconds per trajectory (lower is better).

  value     trajectories whose random inputs were staged in HBM before the
            timed region (chdwf_prog_stage); CUDA events on the library's
            stream, max over ranks.
  e2e       the same trajectories through the host-facing driver API with the
            random numbers drawn on the host and copied in every step.
  roofline  the dominant solver kernel class, timed with CUDA events around
            every solver launch in an instrumented replay of the first timed
            trajectory, against the algorithmic bytes the library reports for
            each launch.
  cpu_baseline / --impl reference
            the CPU oracle (a C restatement of rhmc/cheisdwf.f; the Fortran
            reference cannot be built here) on the host cores: per-iteration
            cost of each solve type sampled at the same lattice, times the
            trajectory's iteration profile.

Multi-GPU: independent Markov chains, one per rank ("replicas only"); value
is trajectories of all ranks per unit time expressed as seconds per
trajectory of the whole job.
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

# Workload (the configuration the metric is quoted on): L=Lt=24, Ls=24,
# beta=0.475, m=0.01 (accepted and unused, as in the reference), am3=1,
# imass=1, hpin=0; dt=0.1 with mean trajectory length dt*iterl = 1.
CFG = dict(beta=0.475, am3=1.0, am=0.01, hpin=0.0, imass=1, dt=0.1, iterl=10,
           seed=693764523745.0, chi_seed=12345)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-propagators", action="store_true")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--L", type=int, default=24)
    ap.add_argument("--Ls", type=int, default=24)
    ap.add_argument("--cpu-sample-iters", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clock-interval-ms", type=int, default=200,
                    help="nvidia-smi sampling interval during the timed region")
    ap.add_argument("--operator-sweep", action="store_true",
                    help="operator GB/s over L in {16,24,32,48}, Ls in {16,24,32}, FP64/FP32/FP16")
    ap.add_argument("--profile-solve", action="store_true",
                    help="bounded work for profilers: one heatbath and one force evaluation")
    ap.add_argument("--profile-res", type=float, default=0.0,
                    help="stopping residual of both profiled solves (0: the reference's)")
    ap.add_argument("--basis-gb", type=float, default=-1.0,
                    help="HBM budget of the stored Lanczos basis (GB; <0 library default)")
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


# solver kernel classes reported by chdwf_timing_read
KERNEL_NAMES = {0: "k_lz1_M", 1: "k_lz1_Md", 2: "k_lz_accum", 3: "k_lz2_M/k_lz2_Md"}
KERNEL_WHAT = {0: "pass-1 M q_j with |M q_j|^2",
               1: "pass-1 M^dag + three-term update with |r|^2",
               2: "pass-2 solution accumulation from the stored Lanczos basis",
               3: "pass-2 regeneration (solves longer than the basis store)"}


def cpu_sample(L, Ls, threads, iters, profile):
    """Oracle cost per solver iteration for each solve type at this lattice,
    combined with a trajectory's iteration profile into seconds/trajectory."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    import chiralheisenberg_b200 as chb
    rz = chb.reference_remez()
    lat = po.make_lat(L, L, Ls, beta=CFG["beta"], am3=CFG["am3"], threads=threads)
    rng = np.random.default_rng(7)
    shape = (2, 4, L, L, L, Ls)
    Phi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    chi = synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"])
    t_iter = {}
    t0all = time.perf_counter()
    for name, n in (("remez2", 25), ("remez2g", 12)):
        r = rz[name]
        t0 = time.perf_counter()
        po.qmrherm(lat, Phi, chi, r["bnum"], r["bden"], 1e-30, niterc=iters)
        t_iter[n] = (time.perf_counter() - t0) / iters
    # force tail: one M apply + derivs per guidance pole (rhmc/cheisdwf.f:733-740)
    t0 = time.perf_counter()
    for _ in range(2):
        po.dslash(lat, Phi, chi)
    t_apply = (time.perf_counter() - t0) / 2
    sampled = time.perf_counter() - t0all
    it25 = profile["it_pf"] + profile["it_h0"] + profile["it_h1"]
    it12 = profile["it_guid"] + profile["it_force"]
    s_traj = it25 * t_iter[25] + it12 * t_iter[12] + profile["nforce"] * 12 * t_apply
    sample = (f"oracle qmrherm at {L}^3x{Ls}: {iters} iterations each of the 25- and 12-pole "
              f"solves + 2 operator applies ({sampled:.1f} s), scaled by the iteration profile "
              f"of one trajectory ({it25:.0f} 25-pole + {it12:.0f} 12-pole iterations, "
              f"{profile['nforce']:.1f} force calls)")
    return s_traj, sample, {"t_iter_25": t_iter[25], "t_iter_12": t_iter[12], "t_apply": t_apply}


def default_profile():
    p = os.path.join(ROOT, "profiles", "iteration_profile_24x24.json")
    if os.path.exists(p):
        return json.load(open(p))
    # iteration counts of a trajectory at 24^3x24 on this workload, from the
    # GPU arm (same algorithm and stopping rule)
    return {"it_pf": 530, "it_h0": 530, "it_h1": 530, "it_guid": 5000.0, "it_force": 5000.0,
            "nforce": 11.0}


def bench_propagators(local_rank, seed=2024, nens=24, nsrc=4, res=1e-8):
    """Config of the batched-solve case: 24 ensembles of uneven size
    (L=Lt in {8,12,16}, Ls in {8,16,24}, seeded), chi ~ N(0,1), 4 point
    sources each (flavour 1,2 x Dirac 3,4 at a seeded site on s=1),
    Phi = M^dag xi, x0 = Phi as in fermion(); CGNE to residual 1e-8.
    Returns solves/s one at a time and batched (one set of launches)."""
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
    # one at a time (the reference's sequence of congrad calls)
    t0 = time.perf_counter()
    its1 = []
    for gl, s, Phi, x, chi in systems:
        xx = Phi.clone()
        it = C.c_int()
        gl.lib.chdwf_congrad_dev(gl.h, C.c_void_p(Phi.data_ptr()), res, C.byref(it), 0.0, 1,
                                 C.c_void_p(chi.data_ptr()), C.c_void_p(xx.data_ptr()))
        its1.append(it.value)
    torch.cuda.synchronize()
    t_one = time.perf_counter() - t0
    # batched
    t0 = time.perf_counter()
    its2, sts = chb.congrad_batch(lats[0], [s for _, s, _, _, _ in systems], res)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    for gl in lats:
        gl.close()
    n = len(systems)
    return {"solves": n, "ensembles": nens, "residual": res,
            "one_at_a_time_solves_per_s": n / t_one, "batched_solves_per_s": n / t_batch,
            "speedup": t_one / t_batch, "mean_iterations": float(np.mean(its2)),
            "same_iterations": bool(list(its1) == list(its2)), "all_converged": bool((sts == 0).all())}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    profile = default_profile()
    vals = []
    sample = ""
    for step in range(args.warmup + args.steps):
        s_traj, sample, _ = cpu_sample(args.L, args.Ls, threads, args.cpu_sample_iters, profile)
        if step >= args.warmup:
            vals.append(s_traj)
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "s/trajectory", "value": v, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"RHMC trajectory L=Lt={args.L} Ls={args.Ls}", **CFG},
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


def run_b200(args, rank, world, local_rank):
    import torch
    import chiralheisenberg_b200 as chb
    torch.cuda.set_device(local_rank)
    L, Ls = args.L, args.Ls
    rz = chb.reference_remez()
    prog = chb.Program(L, L, Ls, CFG["dt"], CFG["beta"], CFG["am3"], CFG["am"], CFG["hpin"],
                       CFG["imass"], CFG["iterl"], rz["remez2"], rz["remez4"], rz["remez2g"],
                       device=local_rank)
    prog.set_chi(synthetic_chi(L, L, CFG["beta"], CFG["chi_seed"] + rank))
    prog.startup(CFG["seed"] + 1000.0 * rank)
    prog.set_measure(5, False)
    stream = torch.cuda.ExternalStream(prog.stream, device=local_rank)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        prog.sweep()

    def timed(staged):
        if staged:
            prog.stage(args.steps)
        recs = []
        barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev[0].record(stream)
        for k in range(args.steps):
            recs.append(prog.sweep())
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = ev[0].elapsed_time(ev[-1])
        timed.per_step = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
        t = torch.tensor([ms], device=f"cuda:{local_rank}", dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item()), recs

    # value and e2e run the SAME trajectories: the chain state (chi and the
    # complete generator state) is saved before the first and restored
    # before the second
    chi0 = prog.get_chi()
    state0 = prog.get_state()
    clocks = ClockSampler(local_rank, args.clock_interval_ms)
    clocks.start()
    n0 = chb.kernel_launches()
    ms_value, recs = timed(staged=True)
    step_ms_value = list(timed.per_step)
    launches = chb.kernel_launches() - n0
    clk = clocks.stop()
    prog.set_chi(chi0)
    prog.set_state(state0)
    ms_e2e, recs_e2e = timed(staged=False)
    step_ms_e2e = list(timed.per_step)
    same = all(a.nsteps == b.nsteps and a.accepted == b.accepted and a.dH == b.dH
               for a, b in zip(recs, recs_e2e))
    mixed = None
    if not args.no_mixed:
        # the same trajectories with FP32 Krylov vectors in the force solves
        prog.set_chi(chi0)
        prog.set_state(state0)
        prog.set_precision(md="f32", accept="f64")
        ms_mix, recs_mix = timed(staged=True)
        prog.set_precision(md="f64", accept="f64")
        dh = [abs(a.dH - b.dH) for a, b in zip(recs, recs_mix)]
        dh_rel = [abs(a.dH - b.dH) / abs(a.H0) for a, b in zip(recs, recs_mix)]
        mixed = {"value": (ms_mix / 1e3) / (args.steps * world), "unit": "s",
                 "precision": "FP32 Krylov vectors in the force solves, FP64 heatbath/hamilton",
                 "speedup_vs_fp64": ms_value / ms_mix,
                 "dH_max_abs_diff_vs_fp64": max(dh), "dH_max_diff_rel_H": max(dh_rel),
                 "same_decisions": all(a.accepted == b.accepted and a.nsteps == b.nsteps
                                       for a, b in zip(recs, recs_mix))}

    # Per-kernel timing: the first timed trajectory again, instrumented --
    # CUDA events around every solver launch on the library's stream (the
    # instrumented replay issues launches one by one, so it is not part of
    # the timed value above)
    prog.set_chi(chi0)
    prog.set_state(state0)
    prog.timing(True)
    prog.sweep()
    kms, ktimed, klaunched, kbytes = prog.timing_read()
    prog.timing(False)

    # whole job: steps*world trajectories in the slowest rank's time
    ntraj = args.steps * world
    value = (ms_value / 1e3) / ntraj
    e2e = (ms_e2e / 1e3) / ntraj
    kvol = L * L * L
    h2d = 64 * kvol * Ls + 12 * kvol          # heatbath Gaussians + momenta
    d2h = 12 * kvol + 64                      # momenta for vel2 + scalars
    dom = int(np.argmax(kms))
    avg_ms = kms[dom] / max(ktimed[dom], 1)
    achieved = kbytes[dom] / (kms[dom] * 1e-3) / 1e9
    bytes_per_launch = kbytes[dom] / max(ktimed[dom], 1)
    peak, peak_kind = peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic_24x24.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(KERNEL_NAMES[dom])
    prof = {"it_pf": float(np.mean([r.it_pf for r in recs])),
            "it_h0": float(np.mean([r.it_h0 for r in recs])),
            "it_h1": float(np.mean([r.it_h1 for r in recs])),
            "it_guid": float(np.mean([r.it_guid for r in recs])),
            "it_force": float(np.mean([r.it_force for r in recs])),
            "nforce": float(np.mean([r.nforce for r in recs]))}
    line = {"metric": "s/trajectory", "value": value, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_value / args.steps,
            "step_ms": [round(x, 1) for x in step_ms_value],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"RHMC trajectory L=Lt={L} Ls={Ls}", "precision": "fp64",
                       "parallelism": f"replicas{world}", "l2": "fields larger than L2 "
                       "(solver working set > 126 MB)", **CFG},
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "same_trajectories_as_value": same,
                    "step_ms": [round(x, 1) for x in step_ms_e2e]},
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "what": KERNEL_WHAT[dom],
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "bytes_per_launch": bytes_per_launch, "avg_launch_us": avg_ms * 1e3,
                         "measured_in": "instrumented replay of the first timed trajectory, "
                                        "CUDA events around every solver launch"},
            "solver_kernels": {KERNEL_NAMES[k]: {
                "launches": int(klaunched[k]), "avg_us": kms[k] / max(ktimed[k], 1) * 1e3,
                "share_of_solver_time": kms[k] / max(sum(kms), 1e-30),
                "GBps": (kbytes[k] / (kms[k] * 1e-3) / 1e9) if kms[k] > 0 else None}
                for k in range(4)},
            "gpu_launches": launches,
            "mixed": mixed,
            "iteration_profile": prof,
            "trajectories": [{"dH": r.dH, "accepted": r.accepted, "nsteps": r.nsteps}
                             for r in recs],
            "clocks": clk}
    if rank == 0 and not args.no_propagators:
        line["propagators"] = bench_propagators(local_rank)
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s_cpu, sample, _ = cpu_sample(L, Ls, threads, args.cpu_sample_iters, prof)
        line["cpu_baseline"] = {"value": s_cpu, "unit": "s", "cores": threads, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    prog.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile_solve:
        run_profile_solve(args, local_rank)
        return
    if args.operator_sweep:
        run_operator_sweep(args, int(os.environ.get("LOCAL_RANK", "0")))
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
