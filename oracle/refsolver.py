"""Run the reference's own CPU solver on a datain/ folder.

Test infrastructure: tests/, tests/golden/ and bench.py's reference arm use it as the checker
and as the CPU baseline; the product never imports it.  The solver is cput2cEXASIM, built from
the reference tree by oracle/build_ref_full.py into oracle/_ref/ (backend/Main/main.cpp with
-D_TEXT2CODE: it reads the datain/ folder named by a pdeapp.txt, exasim.hpp:281-298, and
writes dataout/out*.bin).  The model library (libpdemodelserial.so, generated by the
reference's text2code) is chosen per run through LD_LIBRARY_PATH.

With debugmode = 1 in app.bin (flag 3, readbinaryfiles.cpp) the reference writes the
intermediate arrays of its first Newton step (uequation.cpp:182-202, 542-556, 683-693,
764-774; qequation.cpp:155-167, 474-483; matvec.cpp:114-116, 185-187, 235-237, 385-387;
solution.cpp:140-184) and stops there with status 1, as designed ("stop for debugging").
"""
from __future__ import annotations

import os
import re
import select
import subprocess
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")

# pdeapp.txt keys the reader requires (readpdeapp.cpp); the solver itself takes only the
# data paths from this file, everything else comes from datain/app.bin
_PDEAPP = """model = "ModelD";
modelfile = "pdemodel.txt";
meshfile = "grid.bin";
discretization = "hdg";
platform = "cpu";
mpiprocs = 1;
porder = 1;
pgauss = 2;
physicsparam = [1];
tau = [1];
boundaryconditions = [1];
boundaryexpressions = ["x > -1e9"];
datapath = "{datapath}";
exasimpath = "{exasimpath}";
"""


def solver_path(strict: bool = False) -> str:
    return os.path.join(REF, "cput2cEXASIM_strict" if strict else "cput2cEXASIM")


def model_dir(model: str) -> str:
    return os.path.join(REF, "models", model)


def available(model: str, strict: bool = False) -> bool:
    return os.path.exists(solver_path(strict)) and os.path.exists(os.path.join(model_dir(model), "libpdemodelserial.so"))


def set_app_flag(datain: str, index: int, value: float, part: int = 2) -> None:
    """Set entry `index` of part `part` of datain/app.bin (part 2 = flag: 3 debugmode,
    part 3 = problem: 13 NewtonIter, 14 GMRESiter, 15 GMRESrestart, 16 RBdim;
    part 8 = solversparam: 0 NewtonTol, 1 GMREStol), the layout of readpdeapp.cpp:820-918."""
    fn = os.path.join(datain, "app.bin")
    a = np.fromfile(fn, dtype=np.float64)
    ls = int(a[0])
    ns = a[1:1 + ls].astype(np.int64)
    off = 1 + ls + int(ns[:part - 1].sum())
    assert index < ns[part - 1], (index, ns[part - 1])
    a[off + index] = value
    a.tofile(fn)


@dataclass
class RefRun:
    returncode: int
    stdout: str
    lines: List[Tuple[float, str]]        # (host clock when read, line)
    wall_s: float
    dataout: str
    newton: List[Tuple[int, float, float, float]] = field(default_factory=list)  # it, alpha, nrm0, nrm
    gmres_iters: List[int] = field(default_factory=list)
    assembly_ms: List[float] = field(default_factory=list)
    gmres_ms: List[float] = field(default_factory=list)
    stage_starts: List[Tuple[int, int, float]] = field(default_factory=list)   # step, stage, clock
    # per Newton solve (one per steady solve or DIRK stage): [Newton steps, GMRES iterations,
    # host clock at its first residual line, at its last Newton line]
    solves: List[List[float]] = field(default_factory=list)
    # LDG runs (PTC solver, ptcsolver.cpp:255-330): per solve, the residual norms it prints (the
    # initial one, then one per PTC step)
    ptc: List[List[float]] = field(default_factory=list)

    def dump(self, name: str) -> np.ndarray:
        """An intermediate array of a debugmode run, e.g. 'uEquationElemSchur_H' (raw FP64)."""
        return np.fromfile(os.path.join(self.dataout, f"out{name}.bin"), dtype=np.float64)

    def dumps(self) -> List[str]:
        return sorted(f[3:-4] for f in os.listdir(self.dataout)
                      if f.startswith("out") and f.endswith(".bin") and "_np" not in f)

    def uhat(self) -> np.ndarray:
        """outuhat_np0.bin: (ncu, npf, nf) header then the snapshots (solution.h:45-117)."""
        return np.fromfile(os.path.join(self.dataout, "outuhat_np0.bin"), dtype=np.float64)

    def udg(self) -> np.ndarray:
        return np.fromfile(os.path.join(self.dataout, "outudg_np0.bin"), dtype=np.float64)


_RE_NEWTON = re.compile(r"Newton Iteration: (\d+), Alpha: ([-+0-9.eE]+), Original Norm: ([-+0-9.eEnaif]+),\s+Updated Norm: ([-+0-9.eEnaif]+)")
_RE_GMRES = re.compile(r"GMRES\(\d+\) converges to the tolerance \S+ within\s+(\d+) iterations")
_RE_GMRES_NC = re.compile(r"GMRES\(\d+\) does not converge to the tolerance \S+ within\s+(\d+) iterations")
_RE_ASM = re.compile(r"hdgAssembleLinearSystem time: ([0-9.eE+-]+) miliseconds")
_RE_GT = re.compile(r"^GMRES time: ([0-9.eE+-]+) miliseconds")
_RE_STAGE = re.compile(r"Timestep :\s+(\d+),\s+Timestage :\s+(\d+)")
_RE_SOLVE = re.compile(r"Newton Iteration: 0,\s+Residual Norm")
_RE_PTC0 = re.compile(r"PTC Iteration: 0,\s+Solution Norm")
_RE_PTC = re.compile(r"PTC Iteration: (\d+),\s+Residual Norm: ([-+0-9.eEnaif]+)")
_RE_LGMRES = re.compile(r"^GMRES converges to the tolerance \S+ within\s+(\d+) iterations")


def _start(datain: str, model: str, workdir: str, strict: bool, threads: int) -> subprocess.Popen:
    if not available(model, strict):
        raise FileNotFoundError(f"reference solver or model {model} not built (oracle/build_ref_full.py)")
    workdir = os.path.abspath(workdir)
    os.makedirs(os.path.join(workdir, "dataout"), exist_ok=True)
    link = os.path.join(workdir, "datain")
    if os.path.abspath(datain) != link:
        if os.path.islink(link):
            os.unlink(link)
        os.symlink(os.path.abspath(datain), link)
    with open(os.path.join(workdir, "run.txt"), "w") as fh:
        fh.write(_PDEAPP.format(datapath=workdir, exasimpath=os.path.join(REF, "Exasim")))
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = model_dir(model) + (":" + env["LD_LIBRARY_PATH"] if env.get("LD_LIBRARY_PATH") else "")
    for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS"):
        env[k] = str(threads)
    cmd = ["stdbuf", "-oL", "-eL", solver_path(strict), "run.txt"]
    return subprocess.Popen(cmd, cwd=workdir, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, bufsize=0)


def _parse(res: RefRun) -> RefRun:
    for t, ln in res.lines:
        if _RE_PTC0.search(ln):
            res.ptc.append([])
            res.solves.append([0, 0, t, t])
            continue
        if (m := _RE_PTC.search(ln)):
            if res.ptc:
                res.ptc[-1].append(float(m.group(2)))
                if len(res.ptc[-1]) > 1:
                    res.solves[-1][0] += 1
                    res.solves[-1][3] = t
            continue
        if (m := _RE_LGMRES.search(ln.strip())):
            res.gmres_iters.append(int(m.group(1)))
            if res.solves:
                res.solves[-1][1] += int(m.group(1))
            continue
        if _RE_SOLVE.search(ln):
            res.solves.append([0, 0, t, t])
        elif (m := _RE_NEWTON.search(ln)):
            res.newton.append((int(m.group(1)), float(m.group(2)), float(m.group(3)), float(m.group(4))))
            if res.solves:
                res.solves[-1][0] += 1
                res.solves[-1][3] = t
        elif (m := _RE_GMRES.search(ln)) or (m := _RE_GMRES_NC.search(ln)):
            res.gmres_iters.append(int(m.group(1)))
            if res.solves:
                res.solves[-1][1] += int(m.group(1))
        elif (m := _RE_ASM.search(ln)):
            res.assembly_ms.append(float(m.group(1)))
        elif (m := _RE_GT.search(ln.strip())):
            res.gmres_ms.append(float(m.group(1)))
        elif (m := _RE_STAGE.search(ln)):
            res.stage_starts.append((int(m.group(1)), int(m.group(2)), t))
    return res


def run_many(datain: str, model: str, workdirs: List[str], strict: bool = False, timeout: Optional[float] = None,
             threads: int = 1, stop_after_stages: Optional[int] = None) -> List[RefRun]:
    """Run one reference process per work folder on the same datain/, concurrently.

    Lines are read as the solvers print them (stdout made line-buffered through stdbuf), each
    stamped with the host clock, so stage and Newton times can be read off without changing the
    solver.  With stop_after_stages = k a process is stopped once its (k+1)-th DIRK stage
    begins, or after its k-th Newton solve has finished its last step when it prints no
    further stage (the run then counts as complete)."""
    t0 = time.perf_counter()
    procs = [_start(datain, model, w, strict, threads) for w in workdirs]
    lines: List[List[Tuple[float, str]]] = [[] for _ in procs]
    bufs = [b""] * len(procs)
    open_fds = {p.stdout.fileno(): i for i, p in enumerate(procs)}
    stopped = [False] * len(procs)
    try:
        while open_fds:
            if timeout is not None and time.perf_counter() - t0 > timeout:
                raise TimeoutError(f"reference solver exceeded {timeout} s")
            r, _, _ = select.select(list(open_fds), [], [], 0.5)
            for fd in r:
                i = open_fds[fd]
                chunk = os.read(fd, 65536)
                if not chunk:
                    del open_fds[fd]
                    continue
                now = time.perf_counter()
                bufs[i] += chunk
                *done, bufs[i] = bufs[i].split(b"\n")
                lines[i] += [(now, ln.decode(errors="replace")) for ln in done]
                if stop_after_stages is not None and not stopped[i]:
                    nst = sum(1 for _, ln in lines[i] if _RE_STAGE.search(ln))
                    if nst > stop_after_stages:
                        procs[i].kill()
                        stopped[i] = True
            if not r:
                for fd, i in list(open_fds.items()):
                    if procs[i].poll() is not None:
                        del open_fds[fd]
    finally:
        for p in procs:
            if p.poll() is None and timeout is not None and time.perf_counter() - t0 > timeout:
                p.kill()
    out = []
    for i, p in enumerate(procs):
        rc = p.wait()
        if bufs[i]:
            lines[i].append((time.perf_counter(), bufs[i].decode(errors="replace")))
        res = RefRun(0 if stopped[i] else rc, "\n".join(l for _, l in lines[i]), lines[i],
                     time.perf_counter() - t0, os.path.join(os.path.abspath(workdirs[i]), "dataout"))
        out.append(_parse(res))
    return out


def run(datain: str, model: str, workdir: str, strict: bool = False, timeout: Optional[float] = None,
        threads: int = 1) -> RefRun:
    """Run the reference solver on `datain` with model `model`; outputs go to workdir/dataout."""
    return run_many(datain, model, [workdir], strict, timeout, threads)[0]


def stage_times(res: RefRun) -> List[float]:
    """Seconds per DIRK-stage Newton solve: from the stage's header line (exasim.hpp:440-441) to
    the last Newton step line of the solve that follows it (solution.cpp:216, 235)."""
    out = []
    for (_, _, t0), sv in zip(res.stage_starts, res.solves):
        if sv[0] > 0:
            out.append(sv[3] - t0)
    return out
