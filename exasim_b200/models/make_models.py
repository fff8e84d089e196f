"""Write the generated-format model sources used by the benchmark and test cases.

Exasim's text2code turns a pdemodel.txt into one C++ file per model function
(generator backend/Model/SymbolicScalarsVectors.cpp:374-440).  SymEngine is not
available here, so the pointwise expressions of each case are written out by this
script in that same file format; exasim_b200.modelc then turns them into device
functions exactly as it does for text2code's output.

Cases (Jacobian entries follow Exasim's ordering J[out + nout*in]):
  poisson2d / poisson3d  flux mu0*q, source d*pi^2*prod sin(pi x_k), FbouHdg tau*(0-uhat)
                         (examples/Poisson/poisson{2,3}d/pdemodel.txt)
  convdiff2d / convdiff3d  flux mu0*q + c*u with c = mu[1..nd], source exp(-|x-x0|^2/(2 s^2))
                         with x0 = mu[nd+1..2nd], s = mu[2nd+1]; FbouHdg tau*(0-uhat)
Usage:  python make_models.py   (rewrites the case folders next to this file)
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))

PT = ("dstype* f, {J}const dstype* x, const dstype* uq, const dstype* v, const dstype* w, "
      "const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, "
      "const int szx, const int szuq, const int szv, const int szw, const int szeta, const int szmu")
PTB = ("dstype* f, {J}const dstype* x, const dstype* uq, const dstype* v, const dstype* w, "
       "const dstype* uhat, const dstype* n, const dstype* tau, const dstype* eta, const dstype* mu, "
       "const dstype t, const int modelnumber, const int N, const int szx, const int szuq, "
       "const int szv, const int szw, const int szuhat, const int szn, const int sztau, "
       "const int szeta, const int szmu")
DISPATCH = ("dstype* f, {J}const dstype* xdg, const dstype* udg, const dstype* odg, const dstype* wdg, "
            "const dstype* uhg, const dstype* nlg, const dstype* tau, const dstype* uinf, "
            "const dstype* param, const dstype time, const int modelnumber, const int ib, const int ng, "
            "const int nc, const int ncu, const int nd, const int ncx, const int nco, const int ncw")


def fn(name, sig, tag, loads, stores):
    body = "\n".join(f"    dstype {a} = {b};" for a, b in loads)
    st = "\n".join(f"    {a} = {b};" for a, b in stores)
    return (f"void {name}({sig})\n{{\n\n  Kokkos::parallel_for(\"{tag}\", N, KOKKOS_LAMBDA(const size_t i) {{\n"
            f"{body}\n\n{st}\n  }});\n}}\n")


def flux_terms(nd, conv):
    nc = nd + 1
    loads = [(f"uq{k}", f"uq[{k}*N+i]") for k in range(nc)] + [("mu0", "mu[0]")]
    if conv:
        loads += [(f"mu{1 + d}", f"mu[{1 + d}]") for d in range(nd)]
    f, J = [], []
    for d in range(nd):
        e = f"uq{1 + d}*mu0"
        if conv:
            e = f"uq0*mu{1 + d} + uq{1 + d}*mu0"
        f.append((f"f[{d} * N + i]", e))
    for c in range(nc):
        for d in range(nd):
            v = "0"
            if c == 1 + d:
                v = "mu0"
            elif c == 0 and conv:
                v = f"mu{1 + d}"
            J.append((f"J1[{d + nd * c} * N + i]", v))
    return loads, f, J


def source_terms(nd, conv):
    loads = [(f"x{k}", f"x[{k}*N+i]") for k in range(nd)]
    if not conv:
        c = "1.973920880217872E+1" if nd == 2 else "2.960881320326807E+1"
        e = "*".join(f"sin(x{k}*3.141592653589793)" for k in range(nd)) + "*" + c
    else:
        loads += [(f"mu{nd + 1 + k}", f"mu[{nd + 1 + k}]") for k in range(nd)] + [("s", f"mu[{2 * nd + 1}]")]
        r2 = "+".join(f"(x{k}-mu{nd + 1 + k})*(x{k}-mu{nd + 1 + k})" for k in range(nd))
        e = f"exp(-({r2})/(2*s*s))"
    return loads, e


def write_case(name, nd, conv):
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    nc = nd + 1
    fl, ff, fj = flux_terms(nd, conv)
    sl, se = source_terms(nd, conv)
    files = {
        "KokkosFlux": fn("KokkosFlux", PT.format(J=""), "Flux", fl, ff),
        "HdgFlux": fn("HdgFlux", PT.format(J="dstype* J1, dstype* J2, "), "Flux", fl, ff + fj),
        "KokkosSource": fn("KokkosSource", PT.format(J=""), "Source", sl, [("f[0 * N + i]", se)]),
        "HdgSource": fn("HdgSource", PT.format(J="dstype* J1, dstype* J2, "), "Source", sl,
                        [("f[0 * N + i]", se)] + [(f"J1[{c} * N + i]", "0") for c in range(nc)]),
        "KokkosTdfunc": fn("KokkosTdfunc", PT.format(J=""), "Tdfunc", [], [("f[0 * N + i]", "1")]),
    }
    fb1 = fn("HdgFbou1", PTB.format(J="dstype* J1, dstype* J2, dstype* J3, "), "FbouHdg",
             [("uhat0", "uhat[0*N+i]"), ("tau0", "tau[0]")],
             [("f[0 * N + i]", "-tau0*uhat0")] + [(f"J1[{c} * N + i]", "0") for c in range(nc)]
             + [("J3[0 * N + i]", "-tau0")])
    fb1o = fn("HdgFbouonly1", PTB.format(J=""), "FbouHdg",
              [("uhat0", "uhat[0*N+i]"), ("tau0", "tau[0]")], [("f[0 * N + i]", "-tau0*uhat0")])
    args = "xdg, udg, odg, wdg, uhg, nlg, tau, uinf, param, time, modelnumber, ng, nc, ncu, nd, ncx, nco, ncw, nc, ncu, nd"
    files["HdgFbou"] = fb1 + (f"\nvoid HdgFbou({DISPATCH.format(J='dstype* f_udg, dstype* f_wdg, dstype* f_uhg, ')}) {{\n"
                              f"    if (ib == 1 )\n        HdgFbou1(f, f_udg, f_wdg, f_uhg, {args});\n}}\n")
    files["HdgFbouonly"] = fb1o + (f"\nvoid HdgFbouonly({DISPATCH.format(J='')}) {{\n"
                                   f"    if (ib == 1 )\n        HdgFbouonly1(f, {args});\n}}\n")
    files["cpuInitu"] = ("void cpuInitu(dstype* f, const dstype* x, const dstype* eta, const dstype* mu, "
                         "const int modelnumber, const int N, const int ncx, const int nce, const int npe, "
                         "const int ne)\n{\n\n  for (int i = 0; i < N; ++i) {\n    int p = i%npe; \n"
                         "    int e = i/npe; \n\n\n    f[p+npe*0 +npe*nce*e] = 0.0;\n  }\n}\n")
    for k, v in files.items():
        with open(os.path.join(d, k + ".cpp"), "w") as fh:
            fh.write(v)


if __name__ == "__main__":
    write_case("poisson2d", 2, False)
    write_case("poisson3d", 3, False)
    write_case("convdiff2d", 2, True)
    write_case("convdiff3d", 3, True)
