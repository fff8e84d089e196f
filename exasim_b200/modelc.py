"""Turn Exasim's generated pointwise model sources into CUDA device functions.

Exasim's text2code emits one C++ file per model function (``HdgFlux.cpp``,
``HdgSource.cpp``, ``HdgFbou.cpp`` + ``HdgFbou1.cpp``..., ``KokkosFlux.cpp``, ...;
generator ``backend/Model/SymbolicScalarsVectors.cpp:374-440``, names
``backend/Model/Code2Cpp.cpp:13-44``, declared in ``backend/Model/libpdemodel.hpp:3-41``).
Each file defines ``void F(params) { Kokkos::parallel_for("tag", N,
KOKKOS_LAMBDA(const size_t i) { BODY }); }`` where BODY reads point ``i`` of
structure-of-arrays inputs (``uq[k*N+i]``) and writes outputs the same way.
Boundary functions add a dispatcher (``HdgFbou``) that calls ``HdgFbou<ib>``.

This module rewrites every such function into
``__device__ void F_pt(const size_t i, params) { BODY }`` with the parameter list
unchanged, so the HDG kernels evaluate the model at one quadrature point per thread
on shared-memory tiles (N = points in the tile) inside the fused assembly kernels.
Dispatchers become device functions that call the ``_pt`` forms.  Host-side
initialisers (``cpuInitu`` ...) are plain loops and are kept as host code.

Usage:  python -m exasim_b200.modelc <model source dir> <out header>
"""
from __future__ import annotations

import os
import re
import sys
from typing import Dict, List, Tuple

_FUNC = re.compile(r"\bvoid\s+(\w+)\s*\(([^{};]*?)\)\s*\{", re.S)
_LAMBDA = re.compile(r"Kokkos::parallel_for\s*\(\s*\"[^\"]*\"\s*,\s*\w+\s*,\s*KOKKOS_LAMBDA\s*\(\s*const\s+size_t\s+(\w+)\s*\)\s*\{", re.S)


def _match_brace(s: str, open_idx: int) -> int:
    """Index of the '}' matching the '{' at open_idx."""
    depth = 0
    for k in range(open_idx, len(s)):
        c = s[k]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return k
    raise ValueError("unbalanced braces in model source")


def _functions(src: str) -> List[Tuple[str, str, str]]:
    out = []
    pos = 0
    while True:
        m = _FUNC.search(src, pos)
        if not m:
            return out
        ob = m.end() - 1
        cb = _match_brace(src, ob)
        out.append((m.group(1), " ".join(m.group(2).split()), src[ob + 1:cb]))
        pos = cb + 1


def parse_dir(srcdir: str) -> Dict[str, Tuple[str, str, str]]:
    """name -> (params, kind, body) for every function in every *.cpp of srcdir."""
    funcs = {}
    for fn in sorted(os.listdir(srcdir)):
        if not fn.endswith(".cpp") or fn[:-4] not in MODEL_FILES:
            continue
        with open(os.path.join(srcdir, fn)) as f:
            src = f.read()
        for name, params, body in _functions(src):
            lm = _LAMBDA.search(body)
            if lm:
                lb = lm.end() - 1
                le = _match_brace(body, lb)
                idx = lm.group(1)
                inner = body[lb + 1:le]
                if idx != "i":
                    inner = re.sub(rf"\b{idx}\b", "i", inner)
                funcs[name] = (params, "point", inner)
            elif name.startswith("cpu"):
                funcs[name] = (params, "host", body)
            else:
                funcs[name] = (params, "dispatch", body)
    return funcs


# One generated file per model function, as the generated model.hpp includes them
# (names of backend/Model/libpdemodel.hpp:3-41); numbered siblings such as HdgFlux1.cpp
# belong to other model numbers and are not part of this model.
MODEL_FILES = {
    "KokkosFlux", "KokkosSource", "KokkosTdfunc", "KokkosUbou", "KokkosFbou", "KokkosFhat",
    "KokkosUhat", "KokkosStab", "KokkosSourcew", "KokkosOutput", "KokkosMonitor", "KokkosAvfield",
    "KokkosEoS", "KokkosEoSdu", "KokkosEoSdw", "KokkosVisScalars", "KokkosVisVectors",
    "KokkosVisTensors", "KokkosQoIvolume", "KokkosQoIboundary", "KokkosInitu", "KokkosInitq",
    "KokkosInitudg", "KokkosInitwdg", "KokkosInitodg", "HdgFlux", "HdgSource", "HdgFbou",
    "HdgFbouonly", "HdgFint", "HdgFintonly", "HdgSourcew", "HdgSourcewonly", "HdgEoS",
    "cpuInitu", "cpuInitq", "cpuInitudg", "cpuInitwdg", "cpuInitodg",
}

OPTIONAL_BOUNDARY = ("KokkosUbou", "KokkosFbou")
BOUNDARY_PARAMS = ("dstype* f, const dstype* xdg, const dstype* udg, const dstype* odg, const dstype* wdg, "
                   "const dstype* uhg, const dstype* nlg, const dstype* tau, const dstype* uinf, "
                   "const dstype* param, const dstype time, const int modelnumber, const int ib, const int ng, "
                   "const int nc, const int ncu, const int nd, const int ncx, const int nco, const int ncw")

REQUIRED = ("HdgFlux", "HdgSource", "HdgFbou", "HdgFbouonly", "KokkosFlux", "KokkosSource",
            "KokkosTdfunc", "cpuInitu")


def generate(srcdir: str, model_name: str) -> str:
    funcs = parse_dir(srcdir)
    missing = [r for r in REQUIRED if r not in funcs]
    if missing:
        raise ValueError(f"model {model_name}: missing generated functions {missing}")
    dev = [n for n, (_, k, _) in funcs.items() if k in ("point", "dispatch")]
    lines = [f"// Generated by exasim_b200.modelc from {os.path.basename(os.path.abspath(srcdir))}; do not edit.",
             "#pragma once", "#include <cmath>", f"namespace exa_model_{model_name} {{",
             "typedef double dstype;", "using std::pow; using std::sqrt; using std::exp; using std::log;",
             "using std::sin; using std::cos; using std::tan; using std::atan; using std::atan2;",
             "using std::acos; using std::asin; using std::tanh; using std::fabs; using std::abs;"]
    call = re.compile(r"\b(" + "|".join(re.escape(n) for n in dev) + r")\s*\(")
    # emit callees before callers (point functions first, dispatchers after their targets)
    done, order = set(), []

    def visit(n, stack=()):
        if n in done:
            return
        if n in stack:
            raise ValueError(f"recursive dispatch in model function {n}")
        if funcs[n][1] == "dispatch":
            for c in call.findall(funcs[n][2]):
                if c != n:
                    visit(c, stack + (n,))
        done.add(n)
        order.append(n)

    for n in dev:
        visit(n)
    for n in order:
        params, kind, body = funcs[n]
        if kind == "dispatch":
            body = call.sub(lambda m: f"{m.group(1)}_pt(i, ", body)
        lines.append(f"__device__ __forceinline__ void {n}_pt(const size_t i, {params})\n{{{body}}}")
    # the LDG boundary functions are optional: a model without them gets empty stand-ins and
    # a false has_ flag, and the solver refuses LDG on meshes with boundary faces
    for n in OPTIONAL_BOUNDARY:
        present = n in funcs and funcs[n][1] == "dispatch"
        if not present:
            lines.append(f"__device__ __forceinline__ void {n}_pt(const size_t i, {BOUNDARY_PARAMS}) {{}}")
        lines.append(f"constexpr bool has_{n} = {'true' if present else 'false'};")
    for n, (params, kind, body) in funcs.items():
        if kind == "host":
            lines.append(f"inline void {n}({params})\n{{{body}}}")
    lines.append(f"}}  // namespace exa_model_{model_name}")
    return "\n".join(lines) + "\n"


def main(argv):
    srcdir, out = argv[1], argv[2]
    name = argv[3] if len(argv) > 3 else os.path.basename(os.path.abspath(srcdir))
    text = generate(srcdir, name)
    with open(out, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main(sys.argv)
