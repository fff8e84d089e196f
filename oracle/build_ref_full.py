"""Build the reference's own CPU solver and its model libraries from the reference tree.

Test infrastructure only: the products are the parity source of tests/golden and of the
reference-backed GPU tests, and the CPU arm of bench.py.  Nothing in exasim_b200/ loads them.
Nothing is fetched over a network; every input is in the reference tree or in this image.

Steps (each skipped when its output exists):
 1. Kokkos (vendored kokkos/, serial backend, shared libraries) -> oracle/_ref/kokkos
 2. The BLAS/LAPACK names of backend/Common/common.h:116-150 forwarded to scipy's bundled
    OpenBLAS (oracle/ref_blas_shim.c) -> oracle/_ref/libexa_refblas.so
 3. SymEngine (vendored text2code/symengine, INTEGER_CLASS=boostmp, its vendored boost headers)
    -> oracle/_ref_build/symengine
 4. text2code (text2code/text2code/text2code.cpp) -> oracle/_ref_build/text2code
 5. Per model: a writable copy of backend/ and text2code/text2code/ under a path whose last
    component named Exasim is the copy (text2code derives exasimpath from it).  text2code runs
    on the model's pdemodel.txt and writes the generated sources into the copy's backend/Model/
    (Code2Cpp + SymEngine, text2code/text2code/CodeCompiler.cpp:236-283).  They are kept in
    oracle/_ref/models/<model>/gen and compiled with the reference's backend/Model/libpdemodel.cpp
    into oracle/_ref/models/<model>/libpdemodelserial.so (the command of
    CodeCompiler.cpp:327-361, against the shared Kokkos of step 1).
 6. backend/Main/main.cpp with -D_TEXT2CODE -DASSUME_GENERATOR, linked to libpdemodelserial by
    name (the model is chosen at run time by LD_LIBRARY_PATH): oracle/_ref/cput2cEXASIM with the
    reference's flags (-O3 -ffast-math) and oracle/_ref/cput2cEXASIM_strict (-O3, IEEE).
 7. oracle/_ref/Exasim/: the solver's exasimpath, with the master-node table its VTU writer reads.

Models: poisson2d and poisson3d use the reference's own examples/Poisson/poisson{2,3}d
pdemodel.txt; poisson3d_builtin takes the reference's shipped generated sources
(backend/Main/BuiltIn/Poisson3D) as they are; the others use oracle/ref_models/<model>/pdemodel.txt,
this project's descriptions of the benchmark models in text2code's input language.

Usage:  python oracle/build_ref_full.py [--ref DIR] [--models m1,m2]   (DIR defaults to $EXASIM_REF)
Build folders go to oracle/_ref_build/ (not shipped); products to oracle/_ref/ (not committed).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
WORK = os.path.join(HERE, "_ref_build")
KOKKOS = os.path.join(OUT, "kokkos")
SYMENGINE = os.path.join(WORK, "symengine")
TEXT2CODE = os.path.join(WORK, "text2code")

# model -> (nd, ncu, model kind, elemtype); pdemodel.txt from oracle/ref_models unless noted
MODELS = {
    "poisson2d": (2, 1, "ModelD", 1),
    "poisson3d": (3, 1, "ModelD", 1),
    "convdiff2d": (2, 1, "ModelD", 1),
    "convdiff3d": (3, 1, "ModelD", 1),
    "cdsin2d": (2, 1, "ModelD", 1),
    "ns2d": (2, 4, "ModelD", 1),
    "euler3d": (3, 5, "ModelC", 1),
}
EXAMPLE_MODELS = {"poisson2d": "examples/Poisson/poisson2d", "poisson3d": "examples/Poisson/poisson3d"}


def _run(cmd, log, cwd=None, env=None):
    with open(log, "w") as fh:
        r = subprocess.run(cmd, cwd=cwd, env=env, stdout=fh, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        with open(log) as fh:
            tail = fh.read()[-3000:]
        raise RuntimeError(f"failed ({r.returncode}): {' '.join(cmd)}\n{tail}")


def _openblas_dir():
    import scipy
    return os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))


def build_kokkos(ref):
    if os.path.exists(os.path.join(KOKKOS, "lib", "libkokkoscore.so")):
        return
    b = os.path.join(WORK, "kbuild")
    _run(["cmake", "-S", os.path.join(ref, "kokkos"), "-B", b, "-DCMAKE_BUILD_TYPE=Release",
          "-DBUILD_SHARED_LIBS=ON", "-DCMAKE_POSITION_INDEPENDENT_CODE=ON", "-DKokkos_ENABLE_SERIAL=ON",
          "-DCMAKE_CXX_STANDARD=17", f"-DCMAKE_INSTALL_PREFIX={KOKKOS}"], os.path.join(WORK, "kcfg.log"))
    _run(["cmake", "--build", b, f"-j{os.cpu_count()}"], os.path.join(WORK, "kbuild.log"))
    _run(["cmake", "--install", b], os.path.join(WORK, "kinst.log"))


def build_blas_shim():
    so = os.path.join(OUT, "libexa_refblas.so")
    src = os.path.join(HERE, "ref_blas_shim.c")
    if os.path.exists(so) and os.path.getmtime(so) > os.path.getmtime(src):
        return
    ob = _openblas_dir()
    lib = [f for f in os.listdir(ob) if f.startswith("libscipy_openblas")][0]
    _run(["gcc", "-O2", "-fPIC", "-shared", src, "-o", so, f"-L{ob}", f"-l:{lib}", f"-Wl,-rpath,{ob}"],
         os.path.join(WORK, "blas.log"))


def build_symengine(ref):
    if os.path.exists(os.path.join(SYMENGINE, "lib", "libsymengine.a")):
        return
    src = os.path.join(ref, "text2code", "symengine")
    b = os.path.join(WORK, "sbuild")
    _run(["cmake", "-S", src, "-B", b, "-DCMAKE_BUILD_TYPE=Release", "-DINTEGER_CLASS=boostmp",
          f"-DBoost_INCLUDE_DIR={src}", "-DBUILD_TESTS=OFF", "-DBUILD_BENCHMARKS=OFF",
          f"-DCMAKE_INSTALL_PREFIX={SYMENGINE}"], os.path.join(WORK, "scfg.log"))
    _run(["cmake", "--build", b, f"-j{os.cpu_count()}"], os.path.join(WORK, "sbuild.log"))
    _run(["cmake", "--install", b], os.path.join(WORK, "sinst.log"))


def build_text2code(ref):
    if os.path.exists(TEXT2CODE):
        return
    _run(["g++", "-O2", "-std=c++17", "-w", os.path.join(ref, "text2code", "text2code", "text2code.cpp"),
          "-o", TEXT2CODE, f"-L{OUT}", "-lexa_refblas", f"-Wl,-rpath,{OUT}"], os.path.join(WORK, "t2c_build.log"))


def _symengine_tree(ref):
    """text2code compiles its Code2Cpp.cpp with -I<exasim>/text2code/symengine{,/include} and
    links <exasim>/text2code/symengine/lib/libsymengine.a; boost comes from the first path."""
    t = os.path.join(WORK, "symengine_tree")
    if not os.path.exists(t):
        os.makedirs(t)
        os.symlink(os.path.join(SYMENGINE, "include"), os.path.join(t, "include"))
        os.symlink(os.path.join(SYMENGINE, "lib"), os.path.join(t, "lib"))
        os.symlink(os.path.join(ref, "text2code", "symengine", "boost"), os.path.join(t, "boost"))
    return t


def write_grid_bin(fn, nd):
    """A 2 x 2 (x 2) grid of quadrilaterals or hexahedra in the grid.bin layout of
    text2code/text2code/readmesh.cpp:83-98 (only the model is generated from it)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from exasim_b200 import inputs as I
    g = I.square_quad_grid(2) if nd == 2 else I.cube_hex_grid(2)
    hdr = np.array([nd, g.p.shape[1], g.t.shape[0], g.t.shape[1]], dtype=np.float64)
    np.concatenate([hdr, g.p.ravel(order="F"), (g.t + 1).ravel(order="F").astype(np.float64)]).tofile(fn)


def _pdeapp(model, nd, ncu, kind, exasim):
    bc = "[1]"
    return "\n".join([
        f'model = "{kind}";', 'modelfile = "pdemodel.txt";', 'meshfile = "grid.bin";',
        'discretization = "hdg";', 'platform = "cpu";', "mpiprocs = 1;", "debugmode = 0;",
        "runmode = 0;", "modelnumber = 0;", "porder = 1;", "pgauss = 2;", "torder = 1;", "nstage = 1;",
        f"ncu = {ncu};", "ncw = 0;", "neb = 4096;", "nfb = 8192;", "time = 0;", "tau = [1];", "dt = [0];",
        "physicsparam = [" + ", ".join(["1"] * 8) + "];", "externalparam = [0, 0];",
        f"boundaryconditions = {bc};", 'boundaryexpressions = ["x > -1e9"];',
        'curvedboundaries = [0];', 'curvedboundaryexprs = [""];', f'exasimpath = "{exasim}";', ""])


def generate_model(ref, model):
    """Runs text2code's code generation for one model and builds its libpdemodelserial.so."""
    dst = os.path.join(OUT, "models", model)
    so = os.path.join(dst, "libpdemodelserial.so")
    if os.path.exists(so):
        return so
    gen = os.path.join(dst, "gen")
    if model == "poisson3d_builtin":
        os.makedirs(dst, exist_ok=True)
        shutil.copytree(os.path.join(ref, "backend", "Main", "BuiltIn", "Poisson3D"), gen)
    else:
        nd, ncu, kind, _ = MODELS[model]
        exasim = os.path.join(WORK, "rw", model, "Exasim")
        if os.path.exists(os.path.join(WORK, "rw", model)):
            shutil.rmtree(os.path.join(WORK, "rw", model))
        os.makedirs(os.path.join(exasim, "text2code"))
        shutil.copytree(os.path.join(ref, "backend"), os.path.join(exasim, "backend"))
        shutil.copytree(os.path.join(ref, "text2code", "text2code"), os.path.join(exasim, "text2code", "text2code"))
        os.symlink(_symengine_tree(ref), os.path.join(exasim, "text2code", "symengine"))
        case = os.path.join(exasim, "case")
        os.makedirs(case)
        src = (os.path.join(ref, EXAMPLE_MODELS[model], "pdemodel.txt") if model in EXAMPLE_MODELS
               else os.path.join(HERE, "ref_models", model, "pdemodel.txt"))
        shutil.copy(src, os.path.join(case, "pdemodel.txt"))
        write_grid_bin(os.path.join(case, "grid.bin"), nd)
        with open(os.path.join(case, "pdeapp.txt"), "w") as fh:
            fh.write(_pdeapp(model, nd, ncu, kind, exasim))
        _run([TEXT2CODE, "pdeapp.txt"], os.path.join(case, "t2c.log"), cwd=case)
        mdir = os.path.join(exasim, "backend", "Model")
        os.makedirs(dst, exist_ok=True)
        os.makedirs(gen)
        # the generated sources: every .cpp that libpdemodel.cpp includes, as text2code left them
        with open(os.path.join(ref, "backend", "Model", "libpdemodel.cpp")) as fh:
            incs = [ln.split('"')[1] for ln in fh if ln.startswith("#include \"")]
        for f in incs:
            if os.path.exists(os.path.join(mdir, f)):
                shutil.copy(os.path.join(mdir, f), os.path.join(gen, f))
    # libpdemodel.cpp from the reference tree, compiled against the generated sources
    lib_src = os.path.join(ref, "backend", "Model", "libpdemodel.cpp")
    shutil.copy(lib_src, os.path.join(dst, "libpdemodel.cpp"))
    for f in ("libpdemodel.hpp",):
        shutil.copy(os.path.join(ref, "backend", "Model", f), os.path.join(dst, f))
    _run(["g++", "-shared", "-std=c++17", "-fPIC", "-O3", "-ffast-math", "-w", f"-I{gen}",
          f"-I{os.path.join(KOKKOS, 'include')}", os.path.join(dst, "libpdemodel.cpp"),
          f"-L{os.path.join(KOKKOS, 'lib')}", "-lkokkoscore", "-lkokkoscontainers",
          f"-Wl,-rpath,{os.path.join(KOKKOS, 'lib')}", "-o", so], os.path.join(dst, "build.log"))
    return so


def build_solver(ref, strict=False):
    exe = os.path.join(OUT, "cput2cEXASIM_strict" if strict else "cput2cEXASIM")
    if os.path.exists(exe):
        return exe
    # any generated model library satisfies the link; the run picks one by LD_LIBRARY_PATH
    mlib = os.path.join(OUT, "models", "poisson2d")
    flags = ["-O3"] if strict else ["-O3", "-ffast-math"]
    _run(["g++", "-std=c++17"] + flags + ["-DNDEBUG", "-D_TEXT2CODE", "-DASSUME_GENERATOR", "-w",
          f"-I{os.path.join(KOKKOS, 'include')}", os.path.join(ref, "backend", "Main", "main.cpp"), "-o", exe,
          f"-L{mlib}", "-lpdemodelserial", f"-L{os.path.join(KOKKOS, 'lib')}", "-lkokkoscore",
          "-lkokkoscontainers", f"-L{OUT}", "-lexa_refblas", "-ldl",
          f"-Wl,-rpath,{os.path.join(KOKKOS, 'lib')}", f"-Wl,-rpath,{OUT}"],
         os.path.join(WORK, "main_strict.log" if strict else "main.log"))
    return exe


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("EXASIM_REF"))
    ap.add_argument("--models", default=",".join(list(MODELS) + ["poisson3d_builtin"]))
    a = ap.parse_args(argv)
    if not a.ref or not os.path.isdir(os.path.join(a.ref, "backend")):
        sys.exit("set --ref or EXASIM_REF to the reference tree (with backend/, kokkos/, text2code/)")
    ref = os.path.abspath(a.ref)
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(WORK, exist_ok=True)
    build_kokkos(ref)
    build_blas_shim()
    build_symengine(ref)
    build_text2code(ref)
    for m in a.models.split(","):
        print("model", m, generate_model(ref, m), flush=True)
    for strict in (False, True):
        print("solver", build_solver(ref, strict), flush=True)
    # the solver's exasimpath: a folder named Exasim (exasim.hpp:351, readpdeapp.cpp:787-795)
    # holding the master-node table its VTU writer reads (visualization.cpp:89)
    t = os.path.join(OUT, "Exasim", "text2code", "text2code")
    os.makedirs(t, exist_ok=True)
    shutil.copy(os.path.join(ref, "text2code", "text2code", "masternodes.bin"), t)


if __name__ == "__main__":
    main()
