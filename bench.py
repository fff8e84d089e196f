"""Benchmark: HDG Newton solves/s on the 3D convection-diffusion workload.

Workload (one GPU): HDG p=4 on a 16^3 hexahedral mesh of the unit cube (4096 elements,
125 nodes each, 326,400 trace unknowns), velocity (1, 0.5, 0.25), kappa = 0.01,
Gaussian source at the centre (sigma 0.1), u = 0 on the boundary, DIRK(3,3) with
dt = 0.01.  One step = one DIRK-stage Newton solve to a residual ratio of 1e-8: source
update, assembly with static condensation, block-Jacobi GMRES(50), Newton update and
residual check.  The headline value is the mixed-precision form (3xTF32 tensor-core element
elimination into FP32 blocks, FP64 residual refinement); the plain FP64 form of the same
solves is timed in the same run and reported beside it.  Two more legs follow on one GPU:
the 3D Euler isentropic-vortex configuration at its full 32^3 size in both forms (`euler3d`,
where the elimination is compute-bound), the served stream of 2D convection-diffusion
requests (`served`), and the LDG discretisation with its pseudo-transient solver on the Euler
vortex (`ldg`: 8^3 beside the reference's own CPU solve of the same stage, and 32^3).  Inputs are seeded synthetic data with the configurations' shapes.  With --gpus N (torchrun) every rank solves its own
replica: the path has no data-path collective, so scaling is weak.

Prints one JSON line.  `--impl reference` times the reference's own CPU solver
(cput2cEXASIM, built from the reference tree into oracle/_ref by oracle/build_ref_full.py)
on the same full workload, one process per usable host core; `cpu_baseline` in the GPU line
is one such process timed on one stage solve beside the GPU legs.
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "HDG Newton solves/s, p50/p99 latency vs plain FP64 on B200 at ||r||/||r0||<=1e-8"
CFG_N, CFG_P = 16, 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=CFG_N, help="elements per cube edge")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="both", choices=["both", "mixed", "plain", "served", "euler", "ldg"],
                    help="time both forms (default) or one; one form prints a partial line, for profiling")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests per configuration of the served-stream leg (0 skips it)")
    ap.add_argument("--serve-slots", type=int, default=16)
    ap.add_argument("--serve-rates", default="100,1000",
                    help="Poisson arrival rates (1/s) of the served leg; the configuration sweeps 10,30,100,300,1000")
    ap.add_argument("--euler-n", type=int, default=32, help="elements per cube edge of the 3D Euler leg")
    ap.add_argument("--euler-steps", type=int, default=4, help="timed stage solves per form of the 3D Euler leg (0 skips it)")
    ap.add_argument("--ldg-n", type=int, default=32, help="elements per cube edge of the LDG leg's large case (0 skips the leg)")
    return ap.parse_args()


def config(n):
    return {"workload": f"3D convection-diffusion HDG p={CFG_P}, {n}^3 hexahedra ({n ** 3} elements), "
                        "DIRK(3,3) dt=0.01, block-Jacobi GMRES(50) to 1e-8",
            "elements": n ** 3, "porder": CFG_P, "ndofuhat": 25 * (3 * n * n * (n + 1)),
            "step": "one DIRK-stage Newton solve",
            "l2": "inputs larger than L2 (condensed blocks H 737 MB, D^-1 F 614 MB per solve at 16^3)",
            "parallelism": "replicas (one independent solve per GPU)"}


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def make_case(tmp, n):
    from exasim_b200 import cases
    d = os.path.join(tmp, "datain")
    # 20 DIRK steps of dt = 0.01 (the configuration); stages beyond them wrap around
    cases.convdiff3d_hex(d, n=n, porder=CFG_P, nsteps=20, dt=0.01)
    return d


def _oracle_case(tmp, n):
    from oracle.hdg import HDGOracle
    from oracle.models import MODELS
    from exasim_b200 import cases
    d = os.path.join(tmp, f"cpu_datain_{n}")
    cases.convdiff3d_hex(d, n=n, porder=CFG_P, nsteps=20, dt=0.01)
    return HDGOracle(d, MODELS["convdiff3d"]())


def _oracle_stage_times(o, nsolves):
    """Wall time of each DIRK-stage Newton solve of the oracle (stages of successive steps)."""
    times = []

    def hook(istep, j, _o):
        times.append(time.perf_counter())

    t0 = time.perf_counter()
    times.append(t0)
    o.dirk_solve(nsteps=(nsolves + 2) // 3, on_stage=hook)
    d = np.diff(times)
    return list(d[:nsolves])


SAMPLE_N = 4


def cpu_baseline_sample(tmp, full_n):
    """Oracle (numpy + LAPACK, all host threads) on a 4^3 sub-problem of the same physics:
    DIRK(3,3) stage Newton solves; solves/s scaled by element count to the full mesh."""
    o = _oracle_case(tmp, SAMPLE_N)
    per = _oracle_stage_times(o, 3)
    per_solve = statistics.median(per)
    scale = (SAMPLE_N ** 3) / float(full_n ** 3)
    return {"value": scale / per_solve, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle/hdg.py (numpy + LAPACK, {os.cpu_count()} host threads): DIRK(3,3) stage "
                      f"Newton solves on the {SAMPLE_N}^3 sub-mesh ({SAMPLE_N ** 3} of {full_n ** 3} elements), "
                      f"{per_solve:.2f} s per solve, scaled by element count"}


def max_over_ranks(ms, world, dist, torch, device):
    """The slowest rank's time: whole-job throughput of independent replicas is the units of all
    ranks over the time of the slowest (one all-reduce of one number)."""
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(steps_per_rank, world, total_ms):
    """Whole-job solves/s of `world` replicas that each made `steps_per_rank` solves."""
    return world * steps_per_rank / (total_ms / 1000.0)


REF_MODEL = "convdiff3d"
REF_MODEL_EULER = "euler3d"


def reference_processes(n):
    """Concurrent reference processes this host can take: one per usable core, each needing
    about 8 GB of host memory at 16^3 (7.3 GB resident measured), with a fifth of the free
    memory left over."""
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    avail = None
    try:
        with open("/proc/meminfo") as fh:
            for ln in fh:
                if ln.startswith("MemAvailable:"):
                    avail = int(ln.split()[1]) * 1024
    except OSError:
        pass
    per = 8e9 * (n / 16.0) ** 3
    by_mem = int(0.8 * avail / per) if avail else cores
    return max(1, min(cores, by_mem, 64)), cores, avail


def _reference_case(tmp, n, nsteps):
    from exasim_b200 import cases
    d = os.path.join(tmp, f"ref_datain_{n}_{nsteps}")
    cases.convdiff3d_hex(d, n=n, porder=CFG_P, nsteps=nsteps, dt=0.01)
    return d


def run_reference(args):
    """The reference's own CPU solver (cput2cEXASIM from oracle/_ref, built from the reference
    tree by oracle/build_ref_full.py with its flags -O3 -ffast-math, Kokkos serial, OpenBLAS with
    one thread) on the full workload: P concurrent processes, one per usable host core (bounded
    by host memory), each solving one DIRK(3,3) step (three stage Newton solves) of the 16^3 p=4
    mesh.  Each process's first stage is its warm-up; its second and third are timed from the
    stage's header line to the last Newton line of its solve.  value = timed solves / (last timed
    end - first timed start) over all processes."""
    from oracle import refsolver as R
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not R.available(REF_MODEL):
        print(json.dumps({"impl": "reference", "unavailable": "the reference solver is not built "
                          "(oracle/build_ref_full.py needs the reference tree)"}), flush=True)
        return 0
    P, cores, avail = reference_processes(args.n)
    with tempfile.TemporaryDirectory() as tmp:
        d = _reference_case(tmp, args.n, 1)
        runs = R.run_many(d, REF_MODEL, [os.path.join(tmp, f"p{i}") for i in range(P)], threads=1,
                          timeout=3000)
    bad = [r for r in runs if r.returncode != 0 or len(r.solves) < 3]
    if bad:
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed (rc {bad[0].returncode}): "
                          + bad[0].stdout[-300:].replace(chr(10), " ")}), flush=True)
        return 0
    timed, per = [], []
    for r in runs:
        for (_, _, t0), sv in list(zip(r.stage_starts, r.solves))[1:3]:
            timed.append((t0, sv[3]))
            per.append(sv[3] - t0)
    span = max(e for _, e in timed) - min(s0 for s0, _ in timed)
    v = len(timed) / span
    asm = [a for r in runs for a in r.assembly_ms]
    gm = [g for r in runs for g in r.gmres_ms]
    its = [sv[1] for r in runs for sv in r.solves]
    sample = (f"cput2cEXASIM (the reference's CPU solver, -O3 -ffast-math, Kokkos serial, OpenBLAS 1 thread): "
              f"{P} concurrent processes on {cores} usable host cores, each one DIRK(3,3) step of the full "
              f"{args.n}^3 p={CFG_P} mesh; {len(timed)} timed stage solves (stages 2 and 3 of each process)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": len(timed), "warmup": P, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh and source of the configuration's shape)", "config": config(args.n),
            "latency_ms": {"p50": float(np.percentile(per, 50)) * 1000.0,
                           "p99": float(np.percentile(per, 99)) * 1000.0},
            "processes": P, "host_cores": cores, "host_mem_available_bytes": avail,
            "reference_timers_ms": {"assembly_per_newton": float(np.mean(asm)), "gmres_per_newton": float(np.mean(gm))},
            "gmres_iters_per_solve": float(np.mean(its)),
            "newton_steps_per_solve": float(np.mean([sv[0] for r in runs for sv in r.solves])),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": P, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


class ReferenceBaseline:
    """The cpu_baseline of the GPU arm: one cput2cEXASIM process (one thread) on the same full
    workload, started before the GPU legs and stopped after its first DIRK-stage Newton solve,
    so it runs beside the GPU work on a host core of its own."""

    def __init__(self, tmp, n):
        self.n = n
        self.res = None
        self.err = None
        self.t = None
        from oracle import refsolver as R
        if not R.available(REF_MODEL):
            return
        d = _reference_case(tmp, n, 1)

        def go():
            try:
                self.res = R.run_many(d, REF_MODEL, [os.path.join(tmp, "cpu_baseline")], threads=1,
                                      timeout=1800, stop_after_stages=1)[0]
            except Exception as e:  # noqa: BLE001 - reported in the line instead
                self.err = repr(e)

        self.t = threading.Thread(target=go, daemon=True)
        self.t.start()

    def result(self):
        from oracle import refsolver as R
        if self.t is None:
            return None
        self.t.join()
        if self.err or self.res is None or not R.stage_times(self.res):
            return {"unavailable": self.err or "reference run gave no stage time"}
        sec = R.stage_times(self.res)[0]
        return {"value": 1.0 / sec, "unit": "solves/s", "cores": 1, "kind": "reference",
                "sample": f"cput2cEXASIM (the reference's CPU solver, -O3 -ffast-math, one thread), one process: "
                          f"the first DIRK(3,3) stage Newton solve of the full {self.n}^3 p={CFG_P} mesh, "
                          f"{sec:.1f} s (assembly {self.res.assembly_ms[0] / 1000:.1f} s, GMRES "
                          f"{self.res.gmres_ms[0] / 1000:.2f} s, {self.res.solves[0][1]} iterations)",
                "seconds_per_solve": sec}


# mixed-precision form of the timed solve: each refinement step solves the FP32 system to
# 1e-4 and the FP64 residual must fall by 1e-8 (the plain form's GMRES tolerance)
MIXED = {"inner_tol": 1e-4, "rtol": 1e-8}
# the served stream's small 2D solves: a looser inner GMRES tolerance per refinement step
# takes fewer iterations in all (restarts lose less of the Krylov space)
MIXED_SERVED = {"inner_tol": 1e-3, "rtol": 1e-8}
# 3D Euler is nonlinear: the refinement steps reuse one assembly (a chord iteration), whose rate
# and not the inner tolerance bounds each step, so a loose inner solve saves Krylov iterations
MIXED_EULER = {"inner_tol": 1e-2, "rtol": 1e-8}


def run_form(s, lib, torch, local, args, world, dist, ndt=20, S=3, steps=None, warmup=None, prof_steps=5):
    """W warm-up and K timed DIRK-stage solves of one solver on its own stream, through ndt
    time steps of S stages (wrapping around).  The per-phase profile comes from prof_steps
    further solves after the timed region: its events between kernels, and the plain launches
    it needs in place of the captured GMRES steps, stay out of the timed solves."""
    stream = torch.cuda.ExternalStream(s.stream(), device=local)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    k = [0]

    def stage():
        istep, j = divmod(k[0], S)
        its, _ = s.DIRKStage(istep % ndt, j)
        k[0] += 1
        return its

    for _ in range(warmup):
        stage()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    gmres, newton, ratios = [], [], []
    l0 = lib.exa_launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        torch.cuda.profiler.start()  # a profiler started with --profile-from-start off sees the timed region only
        ev[0].record(stream)
        for i in range(steps):
            newton.append(stage())
            gmres.append(s.stats()["gmres_total"])
            r0, r1 = s.last_residual()
            ratios.append(r1 / r0 if r0 > 0 else 0.0)
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    launches = lib.exa_launch_count() - l0
    s.profile(True)  # per-phase CUDA events on the solver's stream
    for _ in range(prof_steps):
        stage()
    s.profile(False)
    prof = s.profile_read()
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    total = max_over_ranks(ev[0].elapsed_time(ev[steps]), world, dist, torch, f"cuda:{local}")
    return {"total_ms": total, "per": per, "gmres": gmres, "newton": newton, "ratios": ratios,
            "launches": launches, "prof": prof, "prof_steps": prof_steps, "clocks": clk.summary(), "stream": stream,
            "stage": stage}


def phases_of(prof, steps):
    out = {}
    for k, (ms, cnt, fl) in prof.items():
        if cnt == 0:
            continue
        d = {"ms_per_solve": ms / steps, "regions": cnt}
        if fl > 0:
            d["tflops"] = fl / (ms * 1e-3) / 1e12
        out[k] = d
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from exasim_b200 import HDGSolver, load_library, build as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    if rank == 0:
        B.build(["convdiff3d"])
    if world > 1:
        dist.barrier()
    lib = load_library("convdiff3d")
    with tempfile.TemporaryDirectory() as tmp:
        cpu_ref = ReferenceBaseline(tmp, args.n) if (rank == 0 and world == 1 and not args.no_cpu_baseline
                                                     and args.form == "both") else None
        d = make_case(tmp, args.n)
        s64 = HDGSolver(d, "convdiff3d", device=local)
        s32 = HDGSolver(d, "convdiff3d", device=local)
        s32.set_precision(1, **MIXED)
        if args.form in ("euler", "ldg"):
            s64.close()
            s32.close()
            if rank == 0 and args.form == "euler":
                print(json.dumps({"metric": METRIC, "form": "euler", "euler3d": run_euler(args, local, tmp)}), flush=True)
            if rank == 0 and args.form == "ldg":
                print(json.dumps({"metric": METRIC, "form": "ldg",
                                  "ldg": run_ldg(args, local, tmp, with_cpu=not args.no_cpu_baseline)}), flush=True)
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
            return 0
        if args.form == "served":
            served = run_served(args, local)
            if rank == 0:
                print(json.dumps({"metric": METRIC, "form": "served", "served": served}), flush=True)
            s64.close()
            s32.close()
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
            return 0
        if args.form != "both":
            run_one_form(s32 if args.form == "mixed" else s64, lib, torch, local, args, world, dist, rank)
            s64.close()
            s32.close()
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
            return 0
        plain = run_form(s64, lib, torch, local, args, world, dist)
        mixed = run_form(s32, lib, torch, local, args, world, dist)
        value = replicas_value(args.steps, world, mixed["total_ms"])
        plain_value = replicas_value(args.steps, world, plain["total_ms"])

        # end-to-end: one more stage solve through the C ABI (exa_solve) from pinned host
        # buffers: its start state (saved before an untimed run of the stage) and its source
        nu, nh, ns = s32.field_size("udg"), s32.field_size("uh"), s32.field_size("sdg")
        h_udg = torch.from_numpy(s32.get("udg")).pin_memory().numpy()
        h_uh = torch.from_numpy(s32.get("uh")).pin_memory().numpy()
        mixed["stage"]()
        h_sdg = torch.from_numpy(s32.get("sdg")).pin_memory().numpy()
        o_udg = torch.empty(nu, dtype=torch.float64).pin_memory().numpy()
        o_uh = torch.empty(nh, dtype=torch.float64).pin_memory().numpy()
        ne2e = args.e2e_steps or max(3, min(args.steps, 10))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            s32.set("sdg", h_sdg)
            s32.solve(h_udg, h_uh, o_udg, o_uh)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        e2e_ms = max_over_ranks(e2e_s * 1000.0, world, dist, torch, f"cuda:{local}")
        e2e = {"value": replicas_value(ne2e, world, e2e_ms), "unit": "solves/s", "steps": ne2e,
               "h2d_bytes_per_step": 8 * (nu + nh + ns), "d2h_bytes_per_step": 8 * (nu + nh)}

        roof = kernel_rooflines(s32, s64, mixed, plain, torch, args.steps)
        out = None
        if rank == 0:
            out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                   "warmup": args.warmup, "ms_per_step": mixed["total_ms"] / args.steps, "higher_is_better": True,
                   "scaling": "weak", "vs_baseline": None,
                   "dtype": "3xtf32/f32 element elimination + f64 residual, Newton and GMRES",
                   "data": "synthetic (seeded mesh and source of the configuration's shape)",
                   "config": config(args.n),
                   "latency_ms": {"p50": float(np.percentile(mixed["per"], 50)),
                                  "p99": float(np.percentile(mixed["per"], 99))},
                   "residual_ratio_max": max(mixed["ratios"]),
                   "newton_steps_per_solve": float(np.mean(mixed["newton"])),
                   "gmres_iters_per_solve": float(np.mean(mixed["gmres"])),
                   "gpu_launches": int(mixed["launches"]), "clocks": mixed["clocks"], "e2e": e2e,
                   "speedup_vs_plain_fp64": value / plain_value,
                   "plain_fp64": {"value": plain_value, "unit": "solves/s",
                                  "ms_per_step": plain["total_ms"] / args.steps,
                                  "latency_ms": {"p50": float(np.percentile(plain["per"], 50)),
                                                 "p99": float(np.percentile(plain["per"], 99))},
                                  "residual_ratio_max": max(plain["ratios"]),
                                  "gmres_iters_per_solve": float(np.mean(plain["gmres"])),
                                  "gpu_launches": int(plain["launches"]), "clocks": plain["clocks"],
                                  "phases": phases_of(plain["prof"], plain["prof_steps"]),
                                  "roofline": roof.pop("plain_roofline")},
                   "phases": phases_of(mixed["prof"], mixed["prof_steps"])}
            out["autotuned"] = autotuned(s32)
            out.update(roof)
            if args.serve_requests > 0 and world == 1:
                out["served"] = run_served(args, local)
            if args.euler_steps > 0 and world == 1:
                out["euler3d"] = run_euler(args, local, tmp)
            if args.ldg_n > 0 and world == 1:
                out["ldg"] = run_ldg(args, local, tmp, with_cpu=rank == 0 and not args.no_cpu_baseline)
            if cpu_ref is not None:
                cb = cpu_ref.result()
                if cb is None or "unavailable" in cb:
                    # the reference solver is not built here: the oracle port on a sub-mesh
                    cb = dict(cpu_baseline_sample(tmp, args.n), reference=cb)
                out["cpu_baseline"] = cb
            print(json.dumps(out), flush=True)
        s64.close()
        s32.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_one_form(s, lib, torch, local, args, world, dist, rank):
    """One form alone (--form mixed|plain): a partial line without the comparison, for profiling."""
    r = run_form(s, lib, torch, local, args, world, dist)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "form": args.form, "value": replicas_value(args.steps, world, r["total_ms"]),
                          "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": r["total_ms"] / args.steps, "config": config(args.n),
                          "gmres_iters_per_solve": float(np.mean(r["gmres"])),
                          "residual_ratio_max": max(r["ratios"]), "gpu_launches": int(r["launches"]),
                          "clocks": r["clocks"], "phases": phases_of(r["prof"], r["prof_steps"])}), flush=True)


def run_euler(args, local, tmp):
    """The 3D Euler leg: the isentropic-vortex configuration (p = 3 hexahedra of a periodic
    cube, 5 conserved variables, strength 5, Mach 0.5, DIRK(2,2) dt = 0.05) on args.euler_n^3
    elements.  Its element blocks are 320 x 320 and its condensed blocks 480 x 480, and there is
    no q, so the elimination is the block inverse and the Schur products: compute-bound, where
    the plain form runs FP64 DMMA and the mixed form 3xTF32 tcgen05.  Both forms solve the same
    stages from the same start (W warm-up, then the timed ones); the mixed solution is compared
    with the FP64 one after the last stage."""
    import torch
    from exasim_b200 import HDGSolver, load_library, build as B, cases
    B.build(["euler3d"])
    lib = load_library("euler3d")
    n = args.euler_n
    d = os.path.join(tmp, "euler_datain")
    cases.euler3d_vortex_hex(d, n=n, porder=3, nsteps=5, dt=0.05)
    forms = {}
    sol = {}
    for name, prec in (("plain_fp64", 0), ("mixed", 1)):
        s = HDGSolver(d, "euler3d", device=local)
        if prec:
            s.set_precision(1, **MIXED_EULER)
        r = run_form(s, lib, torch, local, args, 1, None, ndt=5, S=2, steps=args.euler_steps, prof_steps=2)
        st = args.euler_steps
        forms[name] = {"value": st / (r["total_ms"] * 1e-3), "unit": "solves/s", "ms_per_step": r["total_ms"] / st,
                       "latency_ms": {"p50": float(np.percentile(r["per"], 50)),
                                      "p99": float(np.percentile(r["per"], 99))},
                       "newton_steps_per_solve": float(np.mean(r["newton"])),
                       "gmres_iters_per_solve": float(np.mean(r["gmres"])),
                       "residual_ratio_max": max(r["ratios"]), "gpu_launches": int(r["launches"]),
                       "clocks": r["clocks"], "phases": phases_of(r["prof"], r["prof_steps"])}
        sol[name] = s.get("udg")
        s.close()
    u, ref = sol["mixed"], sol["plain_fp64"]
    return {"workload": f"3D Euler HDG p=3, periodic {n}^3 hexahedra ({n ** 3} elements, 320 x 320 element "
                        "blocks), isentropic vortex strength 5, Mach 0.5, DIRK(2,2) dt=0.05, block-Jacobi GMRES",
            "elements": n ** 3, "steps": args.euler_steps, "warmup": args.warmup,
            "mixed": forms["mixed"], "plain_fp64": forms["plain_fp64"],
            "speedup_vs_plain_fp64": forms["mixed"]["value"] / forms["plain_fp64"]["value"],
            "mixed_vs_fp64_rel_l2": float(np.linalg.norm(u - ref) / np.linalg.norm(ref))}


LDG_SMALL_N = 8


def ldg_residual_bytes(sz, nge, ngf):
    """Algorithmic bytes of one LDG residual evaluation: the states and the stage source read
    once, the element geometry (Gauss-point coordinates, Xx, jacobian) and the face geometry
    (coordinates, normal, jacobian) read once, the residual written once."""
    ne, nf, npe, ncu, nd = sz["ne"], sz["nf"], sz["npe"], sz["ncu"], sz["nd"]
    return 8 * (3 * npe * ncu * ne + nge * (nd + nd * nd + 1) * ne + ngf * (nd + nd + 1) * nf)


def run_ldg(args, local, tmp, with_cpu):
    """The LDG leg: the reference's other discretisation (problem[0] = 0) on the 3D Euler
    isentropic vortex, p = 3 hexahedra of a periodic cube, the first DIRK(2,2) stage solved by
    the pseudo-transient solver (GMRES(50) on finite-difference Jacobian products, identity
    preconditioner, PTC to 1e-8).  Each timed solve starts from the same initial state.  On
    LDG_SMALL_N^3 elements the reference's own CPU solver runs the same stage solve (one
    process, one thread, beside the GPU work); on args.ldg_n^3 the residual evaluation, the
    products' building block, is timed with CUDA events on the context's stream against its
    algorithmic bytes."""
    import torch
    from exasim_b200 import HDGSolver, build as B, cases
    from oracle import refsolver as R
    B.build(["euler3d"])
    peaks, src = measured_peaks()
    ref_res, ref_err, th = {}, {}, None
    ds = os.path.join(tmp, "ldg_small")
    cases.euler3d_vortex_hex(ds, n=LDG_SMALL_N, porder=3, nsteps=1, hybrid=0)
    if with_cpu and R.available(REF_MODEL_EULER):
        def go():
            try:
                ref_res["r"] = R.run_many(ds, REF_MODEL_EULER, [os.path.join(tmp, "ldg_ref")], threads=1, timeout=900,
                                          stop_after_stages=1)[0]
            except Exception as e:  # noqa: BLE001 - reported in the line instead
                ref_err["e"] = repr(e)
        th = threading.Thread(target=go, daemon=True)
        th.start()
    out = {"workload": "3D Euler LDG p=3, periodic n^3 hexahedra, isentropic vortex strength 5, Mach 0.5, first "
                       "DIRK(2,2) stage (dt 0.05) by pseudo-transient continuation to |R| < 1e-8: GMRES(50) to 1e-8 "
                       "on finite-difference Jacobian products (step 1e-3), identity preconditioner"}
    for name, n, W, K in (("small", LDG_SMALL_N, 2, 5), ("large", args.ldg_n, 1, 3)):
        d = ds if name == "small" else os.path.join(tmp, f"ldg_{n}")
        if name != "small":
            cases.euler3d_vortex_hex(d, n=n, porder=3, nsteps=1, hybrid=0)
        s = HDGSolver(d, "euler3d", device=local)
        stream = torch.cuda.ExternalStream(s.stream())
        u0 = s.get("udg")
        ms, its = [], []
        for k in range(W + K):
            s.set("udg", u0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            it, _ = s.DIRKStage(0, 0)
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= W:
                ms.append(e0.elapsed_time(e1))
                its.append((it, s.stats()["gmres_total"]))
        r = {"elements": n ** 3, "unknowns": int(s.sizes["npe"] * s.sizes["ncu"] * s.sizes["ne"]),
             "ms_per_stage_solve": float(np.mean(ms)), "stage_solves_per_s": 1000.0 / float(np.mean(ms)),
             "ptc_steps": its[-1][0], "gmres_iters": its[-1][1]}
        if name == "large":
            # residual evaluations alone at the stage's time and source
            s.set("udg", u0)
            s.DIRKStage(0, 0)
            for _ in range(3):
                s.evalResidual()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 20
            # the profiler range (cudaProfilerStart/Stop) holds exactly these evaluations
            torch.cuda.profiler.start()
            e0.record(stream)
            for _ in range(reps):
                s.evalResidual()
            e1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            rms = e0.elapsed_time(e1) / reps
            nge = s.sizes["nge"]
            ngf = s.sizes["ngf"]
            ab = ldg_residual_bytes(s.sizes, nge, ngf)
            achieved = ab / (rms * 1e-3) / 1e9
            r["residual_ms"] = rms
            r["residual_roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                      "frac": achieved / peaks["hbm_gbs"], "peak_source": src,
                                      "algorithmic_bytes": ab,
                                      "note": "one residual evaluation with its norm; its kernels pass the "
                                              "Gauss-point values and face residuals through HBM, so DRAM "
                                              "traffic exceeds these bytes"}
            s.profile(True)
            s.set("udg", u0)
            s.DIRKStage(0, 0)
            torch.cuda.synchronize()
            r["phases"] = phases_of(s.profile_read(), 1)
            s.profile(False)
        s.close()
        out[name] = r
    if th is not None:
        th.join()
        rr = ref_res.get("r")
        if rr is not None and R.stage_times(rr):
            sec = R.stage_times(rr)[0]
            out["small"]["reference_cpu"] = {
                "ms_per_stage_solve": sec * 1000.0, "cores": 1, "kind": "reference",
                "sample": f"cput2cEXASIM (-O3 -ffast-math, one thread) with problem[0] = 0 on the same "
                          f"{LDG_SMALL_N}^3 input, the same first-stage PTC solve ({len(rr.ptc[0]) - 1} PTC steps, "
                          f"{rr.solves[0][1]} GMRES iterations)"}
            out["small"]["speedup_vs_reference_cpu"] = sec * 1000.0 / out["small"]["ms_per_stage_solve"]
        else:
            out["small"]["reference_cpu"] = {"unavailable": ref_err.get("e", "reference run gave no stage time")}
    return out


SERVED_WORKLOAD = ("served stream of 2D convection-diffusion HDG solves: kappa log-uniform [1e-3, 1], unit "
                   "velocity of uniform direction, p uniform in {2, 3, 4}, n x n quadrilaterals with n uniform in "
                   "{8..64}, source sin(a pi x) sin(b pi y); plain form: one Newton step, block-Jacobi GMRES(50) "
                   "to 1e-11; mixed form: FP64 refinement to ||r||/||r0|| <= 1e-8")


SERVE_BATCH = 64  # job slots of the batched Krylov steps (exa_server_set_batching)


def run_served(args, device):
    """The served-stream leg: the same seeded requests solved (a) one at a time in plain FP64,
    (b) by the server with `slots` overlapping solves in plain FP64 and (c) in the mixed form,
    then (d, e) both forms with batched Krylov steps, each after a warm-up pass that creates the
    resident context of every (mesh, order) pair once; then the batched servers of both forms
    under Poisson arrivals at the rates of --serve-rates for p50/p99 latency.  Times are host
    wall-clock from submit to result."""
    from exasim_b200 import build as B
    from exasim_b200.serve import CaseCache, Server, stream_requests, with_params
    B.build(["cdsin2d"])
    R = args.serve_requests
    cache = CaseCache()
    reqs = stream_requests(R, 0.0, seed=2024)
    blobs = [[with_params(cache.get(n, p)[0], prm)] + cache.get(n, p)[1:] for _, n, p, prm in reqs]
    budget = 48 << 30

    def saturated(srv, precision, which=None):
        t0 = time.perf_counter()
        sel = blobs if which is None else [blobs[i] for i in which]
        ids = [srv.submit(b, precision=precision, **(MIXED_SERVED if precision else {})) for b in sel]
        res = [srv.wait(i) for i in ids]
        return time.perf_counter() - t0, res

    # the warm-up pass: one request of each (mesh, order) pair, so that every resident context the
    # stream can reuse exists (as far as the memory budget holds them) before anything is timed
    first = {}
    for i, (_, n, p, _) in enumerate(reqs):
        first.setdefault((n, p), i)
    warm = sorted(first.values())

    out = {"workload": SERVED_WORKLOAD, "requests": R, "slots": args.serve_slots, "hbm_budget_bytes": budget,
           "batch_slots": SERVE_BATCH}
    lines = {}
    for name, slots, precision, batch in (("plain_fp64_one_at_a_time", 1, 0, 0),
                                          ("served_plain_fp64", args.serve_slots, 0, 0),
                                          ("served_mixed", args.serve_slots, 1, 0),
                                          ("served_batched_plain_fp64", args.serve_slots, 0, SERVE_BATCH),
                                          ("served_batched_mixed", args.serve_slots, 1, SERVE_BATCH)):
        with Server("cdsin2d", device=device, hbm_budget=budget, slots=slots, batch=batch) as srv:
            saturated(srv, precision, warm)      # warm: every (n, p) context created once
            b0 = srv.batch_stats()
            wall, res = saturated(srv, precision)
            st = srv.stats()
            b1 = srv.batch_stats()
        dofs = [r.uh.size for r in res]
        lat = [r.latency_ms for r in res]
        ratio = max((r.residual / r.residual0) if r.residual0 > 0 else 0.0 for r in res)
        lines[name] = {"solves_per_s": R / wall, "dofs_per_s": sum(dofs) / wall,
                       "mean_run_ms": float(np.mean([r.run_ms for r in res])),
                       "gmres_iters_per_solve": float(np.mean([r.gmres for r in res])),
                       "residual_ratio_max": ratio, "contexts_reused": st["contexts_reused"],
                       "peak_bytes_held": st["peak_bytes_held"],
                       "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))}}
        if batch:
            steps = b1["steps"] - b0["steps"]
            lines[name]["batched"] = {"steps": steps, "launches": b1["launches"] - b0["launches"],
                                      "gmres_iters_per_step": sum(r.gmres for r in res) / max(steps, 1),
                                      "matvec_elements_per_warp": b1["matvec_elements_per_warp"]}
    base = lines["plain_fp64_one_at_a_time"]["solves_per_s"]
    for v in lines.values():
        v["speedup_vs_plain_fp64_one_at_a_time"] = v["solves_per_s"] / base
    out.update(lines)
    # the like-for-like ratios: both forms served the same way, each request brought to a true
    # FP64 residual ratio <= 1e-8 (residual_ratio_max above)
    out["mixed_vs_plain_fp64_same_slots"] = lines["served_mixed"]["solves_per_s"] / lines["served_plain_fp64"]["solves_per_s"]
    out["mixed_vs_plain_fp64_batched"] = (lines["served_batched_mixed"]["solves_per_s"] /
                                          lines["served_batched_plain_fp64"]["solves_per_s"])
    rates_list = [float(r) for r in str(args.serve_rates).split(",") if r.strip()]
    for name, precision in (("poisson_arrivals_batched_mixed", 1), ("poisson_arrivals_batched_plain_fp64", 0)):
        rates = {}
        with Server("cdsin2d", device=device, hbm_budget=budget, slots=args.serve_slots, batch=SERVE_BATCH) as srv:
            saturated(srv, precision, warm)
            for rate in rates_list:
                arr = stream_requests(R, rate, seed=7)
                t0 = time.perf_counter()
                ids = []
                for (ta, n, p, prm), b in zip(arr, blobs):
                    dt = t0 + ta - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                    ids.append(srv.submit(b, precision=precision, **(MIXED_SERVED if precision else {})))
                res = [srv.wait(i) for i in ids]
                wall = time.perf_counter() - t0
                lat = [r.latency_ms for r in res]
                dofs = sum(r.uh.size for r in res)
                rates[f"{rate:g}/s"] = {"solves_per_s": R / wall, "dofs_per_s": dofs / wall,
                                        "latency_ms": {"p50": float(np.percentile(lat, 50)),
                                                       "p99": float(np.percentile(lat, 99))}}
        out[name] = rates
    return out


# DRAM traffic of the four q-elimination GEMM launches of one FP64 assembly, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) on the 10^3-element mesh of this
# workload: 4.458 GB for 1000 elements; it scales with the element count (each element's
# blocks are read once), so per launch and element it is 4.458e9 / 1000 / 4 bytes.
QELIM_TRAFFIC_PER_ELEMENT_LAUNCH = 4.458e9 / 1000 / 4
# The same for the mixed form's four 3xTF32 q-elimination launches (umma3_kernel, FP32
# operands split on chip), one ncu capture on the 10^3 mesh: 0.564, 0.642, 0.709 and 0.721 GB
# read + written, mean 0.659 GB per launch for 1000 elements (the algorithmic 0.658).
QELIM_MIXED_TRAFFIC_PER_ELEMENT_LAUNCH = 0.6590e9 / 1000


def fp64_gemm_peak(torch):
    """cuBLAS DGEMM at 8192^3 on this GPU, in TFLOP/s (the FP64 tensor-core reference)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(4):
        a @ b
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 4
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms * 1e-3) / 1e12


def pack_floats(R, K):
    """Floats of one operand packed for the tensor cores (8-row groups x 16-k chunks)."""
    return ((R + 7) // 8) * ((K + 15) // 16) * 128


def qelim_mixed_bytes(sz):
    """Algorithmic bytes of the four q-elimination products of one assembly, per element
    D += B MinvC, F -= B MinvE, K += G MinvC and H -= G MinvE (K = npe nd per trace component):
    every product reads its FP32 operands once (A: M x K, B: K x N, unpadded), reads its FP64
    Cin and writes its FP32 results: D and H plain, F packed (the B operand of D^-1 F), K plain
    and packed (the A operand of K D^-1 F)."""
    npe, nd, ne, ncu = sz["npe"], sz["nd"], sz["ne"], sz.get("ncu", 1)
    ndf = sz["npf"] * sz["nfe"]
    n, m, kq = npe * ncu, ndf * ncu, npe * nd
    d = 4 * ncu * n * kq + 4 * kq * npe + 8 * n * npe * ncu + 4 * n * npe * ncu
    f = 4 * ncu * n * kq + 4 * kq * ndf + 8 * n * ndf * ncu + 4 * n * ndf * ncu
    k = 4 * ncu * m * kq + 4 * kq * npe + 8 * m * npe * ncu + 8 * m * npe * ncu
    h = 4 * ncu * m * kq + 4 * kq * ndf + 8 * m * ndf * ncu + 4 * m * ndf * ncu
    return (d + f + k + h) * ne


def autotuned(s):
    """The shapes the project's autotuners chose for this workload (timed on scratch blocks
    when the contexts were created): the element inverse of order n in FP32 and FP64 (shape
    0-3 of the column-by-warp Gauss-Jordan) and the FP64 DMMA tile of each q-elimination and
    Schur product (exa_dgemm_tune's index into its tiles)."""
    import ctypes
    L, sz = s.lib, s.sizes
    n, m, npe, ndf, nd = sz["n"], sz["m"], sz["npe"], sz["npf"] * sz["nfe"], sz["nd"]
    out = {}
    for fp64 in (0, 1):
        v = ctypes.c_int(-1)
        L.exa_inverse_autotune(n, fp64, sz["ne"], None, ctypes.byref(v))
        out[f"inverse_n{n}_{'fp64' if fp64 else 'fp32'}_shape"] = v.value
    for M, N, K in ((n, npe, npe * nd), (n, ndf, npe * nd), (m, npe, npe * nd), (m, ndf, npe * nd), (n, m, n),
                    (m, m, n)):
        t = ctypes.c_int(-1)
        L.exa_dgemm_tune(M, N, K, min(sz["ne"], 512), None, ctypes.byref(t))
        out[f"dgemm_{M}x{N}x{K}_tile"] = t.value
    return out


def kernel_rooflines(s32, s64, mixed, plain, torch, steps):
    """roofline: the q-elimination GEMMs of the mixed solve, umma3_kernel on the TF32 tensor
    cores, HBM-bound, from the phase timers (CUDA events on the solver's stream around each
    q-elimination region) of the profiled solves that follow the timed ones.  The plain form's
    FP64 q-elimination (dmma_gemm_kernel) is reported beside it against cuBLAS DGEMM, and the
    FP32 condensed matvec is timed alone on the solver's stream."""
    peaks, src = measured_peaks()
    sz = s32.sizes
    ne, m, N = sz["ne"], sz["m"], sz["ndofuhat"]
    q_ms, q_regions, _ = mixed["prof"]["qelim"]
    launches = 4 * q_regions
    qbytes = qelim_mixed_bytes(sz)
    ms_launch = q_ms / max(launches, 1)
    achieved = qbytes / 4 / (ms_launch * 1e-3) / 1e9 if q_ms > 0 else 0.0
    roofline = {"kernel": "umma3_kernel (q-elimination GEMMs D += B MinvC, F -= B MinvE, K += G MinvC, "
                          "H -= G MinvE; 3xTF32 on tcgen05: FP32 operands by cp.async.bulk, split into TF32 "
                          "hi and lo parts in shared memory)",
                "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": src,
                "algorithmic_bytes_per_launch": qbytes / 4, "ms_per_launch": ms_launch, "launches": launches,
                "traffic": QELIM_MIXED_TRAFFIC_PER_ELEMENT_LAUNCH * ne,
                "traffic_source": "ncu dram bytes of the four launches on a 10^3 mesh, mean per launch, scaled by "
                                  "element count"}
    p_ms, p_regions, p_flops = plain["prof"]["qelim"]
    peak64 = fp64_gemm_peak(torch)
    pl = 4 * p_regions
    p_ach = p_flops / (p_ms * 1e-3) / 1e12 if p_ms > 0 else 0.0
    plain_roof = {"kernel": "dmma_gemm_kernel (FP64 q-elimination GEMMs on the DMMA tensor cores)", "bound": "tensor",
                  "achieved": p_ach, "peak": peak64, "unit": "TFLOP/s", "frac": p_ach / peak64,
                  "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                  "algorithmic_flops_per_launch": p_flops / max(pl, 1), "ms_per_launch": p_ms / max(pl, 1),
                  "launches": pl, "traffic": QELIM_TRAFFIC_PER_ELEMENT_LAUNCH * ne,
                  "traffic_source": "ncu dram bytes of the same launches on a 10^3 mesh, scaled by element count"}
    def matvec_roof(s, stream, hbytes, what):
        """The condensed matvec timed alone on the solver's stream: H read once (hbytes per
        entry), the gathered input and element output (16 m ne) and the face vector (16 N)."""
        v = torch.randn(N, dtype=torch.float64, device=f"cuda:{torch.cuda.current_device()}")
        w = torch.empty_like(v)
        torch.cuda.synchronize()
        for _ in range(3):
            s.evalMatVec(v.data_ptr(), w.data_ptr())
        reps = 20
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            s.evalMatVec(v.data_ptr(), w.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        nbytes = hbytes * m * m * ne + 16 * (m * ne + N)
        ach = nbytes / (ms * 1e-3) / 1e9
        return {"kernel": f"condensed matvec, {what} blocks (bgemv_kernel + scatter_kernel)", "bound": "hbm",
                "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                "peak_source": src, "algorithmic_bytes_per_launch": nbytes, "ms_per_launch": ms}

    plain_roof["matvec_roofline"] = matvec_roof(s64, plain["stream"], 8, "FP64")
    return {"roofline": roofline, "plain_roofline": plain_roof,
            "matvec_roofline": matvec_roof(s32, mixed["stream"], 4, "FP32")}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
