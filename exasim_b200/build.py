"""Build the CUDA solver libraries in-tree: exasim_b200/lib/libexasim_b200_<model>.so.

For each model source folder under exasim_b200/models/ (Exasim-generated format) the
model is turned into device functions (exasim_b200.modelc) and compiled together with
the model-independent kernels for sm_100a.  Any other folder of text2code output (the
backend/Model/*.cpp files text2code writes for a pdemodel.txt) builds the same way, as is:
    python -m exasim_b200.build [model ...] [--source NAME=FOLDER ...]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from typing import List, Optional

from . import modelc

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
MODELS = os.path.join(PKG, "models")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
COMMON = ["exa_linalg.cu", "exa_umma.cu", "exa_volmat_tc.cu", "exa_kernels.cu", "exa_drivers.cu", "exa_api.cu", "exa_conn.cpp", "exa_bilu0.cpp", "exa_bilu0_dev.cu", "exa_server.cpp", "exa_batch.cu", "exa_poly.cpp", "exa_ldg.cu"]


def available_models() -> List[str]:
    return sorted(d for d in os.listdir(MODELS) if os.path.isdir(os.path.join(MODELS, d))
                  and any(f.endswith(".cpp") for f in os.listdir(os.path.join(MODELS, d))))


def lib_path(model: str) -> str:
    return os.path.join(LIB, f"libexasim_b200_{model}.so")


def exe_path(model: str) -> str:
    """The model's executable (csrc/exa_main.cpp): datain/ in, the reference's output files out."""
    return os.path.join(BIN, f"exasim_b200_{model}")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def _newer(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> List[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(PKG, "..", "include", "exasim_b200.h")]


def _compile(src: str, obj: str, extra: Optional[List[str]] = None, deps: Optional[List[str]] = None):
    deps = [src] + _headers() + (deps or [])
    if not _newer(obj, deps):
        return obj
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    cmd = [NVCC] + ARCH + FLAGS + (extra or []) + ["-I", CSRC, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + FLAGS + ["-x", "cu"] + ARCH + (extra or []) + ["-I", CSRC, "-c", src, "-o", obj]
    _run(cmd)
    return obj


def build(models: Optional[List[str]] = None, jobs: int = 8, sources: Optional[dict] = None) -> List[str]:
    """Build the libraries (and executables) of `models` (default: every folder under
    exasim_b200/models/).  `sources` maps further model names to folders of generated model
    sources, which are compiled unchanged; those names are built too."""
    sources = dict(sources or {})
    models = list(models or ([] if sources else available_models()))
    models += [m for m in sources if m not in models]
    os.makedirs(LIB, exist_ok=True)
    common_objs = [os.path.join(BUILD, "common", os.path.splitext(f)[0] + ".o") for f in COMMON]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, os.path.join(CSRC, f), o) for f, o in zip(COMMON, common_objs)]
        mfuts = {}
        for mname in models:
            mdir = os.path.join(BUILD, mname)
            os.makedirs(mdir, exist_ok=True)
            hdr = os.path.join(mdir, f"model_{mname}.cuh")
            sdir = sources.get(mname, os.path.join(MODELS, mname))
            srcs = [os.path.join(sdir, f) for f in os.listdir(sdir) if f.endswith(".cpp")]
            if _newer(hdr, srcs + [modelc.__file__]):
                with open(hdr, "w") as fh:
                    fh.write(modelc.generate(sdir, mname))
            obj = os.path.join(mdir, "exa_model.o")
            extra = [f'-DEXA_MODEL_HEADER="{hdr}"', f"-DEXA_MODEL_NS=exa_model_{mname}"]
            mfuts[mname] = ex.submit(_compile, os.path.join(CSRC, "exa_model.cu"), obj, extra, [hdr])
        for f in futs:
            f.result()
        outs = []
        for mname, f in mfuts.items():
            obj = f.result()
            so = lib_path(mname)
            if _newer(so, common_objs + [obj]):
                _run([NVCC] + ARCH + ["-shared", "-o", so] + common_objs + [obj])
            outs.append(so)
            exe, main = exe_path(mname), os.path.join(CSRC, "exa_main.cpp")
            if _newer(exe, [so, main] + _headers()):
                os.makedirs(BIN, exist_ok=True)
                _run(["g++", "-O2", "-std=c++17", main, "-o", exe, "-L", LIB, f"-l:libexasim_b200_{mname}.so",
                      "-Wl,-rpath,$ORIGIN/../lib"])
    return outs


if __name__ == "__main__":
    names = [a for a in sys.argv[1:] if not a.startswith("--source")]
    srcs = {}
    for a in sys.argv[1:]:
        if a.startswith("--source="):
            k, v = a[len("--source="):].split("=", 1)
            srcs[k] = os.path.abspath(v)
    for p in build(names or None, sources=srcs):
        print(p)
