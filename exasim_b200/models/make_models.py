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
  ns2d       2D compressible Navier-Stokes, q = -grad u, 4 conserved variables, mu = [gamma, Re,
             Pr, Minf]; Taylor-Green initial state (examples/NavierStokes/TaylorGreenVortex)
  euler3d    3D compressible Euler (ModelC, no q), mu = [gamma, Minf]; isentropic vortex initial
             state (examples/Euler/EulerVortex, extended to 3D)
  cdsin2d    2D convection-diffusion, flux kappa q + c u, source sin(a pi x) sin(b pi y), mu =
             [kappa, c_x, c_y, a, b]; FbouHdg tau*(0-uhat)
The symbolic cases take their Jacobians from sympy, as text2code takes them from SymEngine.
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


# ------------------------------------------------------------------------------------
# Models written symbolically: the pointwise expressions (and their exact derivatives,
# as text2code takes them with SymEngine) come from sympy here, printed in the generated
# file format above.

def _printer():
    import sympy as sp
    from sympy.printing.c import C99CodePrinter

    class Printer(C99CodePrinter):
        def _print_Pow(self, e):
            b, x = e.base, e.exp
            if x.is_Integer and 1 <= abs(int(x)) <= 4:
                prod = "*".join([self.parenthesize(b, 100)] * abs(int(x)))
                return f"({prod})" if int(x) > 0 else f"(1.0/({prod}))"
            if x == sp.Rational(1, 2):
                return f"sqrt({self._print(b)})"
            return f"pow({self._print(b)}, {self._print(x)})"

    return Printer()


def _emit(outs):
    """C statements for [(lhs, sympy expr)], common subexpressions hoisted."""
    import sympy as sp
    pr = _printer()
    exprs = [sp.sympify(e) for _, e in outs]
    reps, red = sp.cse(exprs, symbols=sp.numbered_symbols("t"), optimizations="basic")
    lines = [f"    dstype {sym} = {pr.doprint(v)};" for sym, v in reps]
    lines += [f"    {lhs} = {pr.doprint(e)};" for (lhs, _), e in zip(outs, red)]
    return "\n".join(lines)


def _fn_sym(name, sig, tag, loads, outs):
    body = "\n".join(f"    dstype {a} = {b};" for a, b in loads)
    return (f"void {name}({sig})\n{{\n\n  Kokkos::parallel_for(\"{tag}\", N, KOKKOS_LAMBDA(const size_t i) {{\n"
            f"{body}\n\n{_emit(outs)}\n  }});\n}}\n")


def write_symbolic_case(name, nd, ncu, modelD, nparam, flux, source, fbou, initu, ubou=None):
    """One case folder from sympy callables.

    flux(uq, x, mu) -> [[f(m, d) for d] for m]; source(uq, x, mu) -> [s_m]; fbou(uq, x, mu,
    uhat, n, tau) -> [fb_m] (boundary code 1); initu(x, mu) -> [u_m]; ubou (optional, same
    arguments as fbou) -> [uhat_m], with which the LDG boundary files are written too.  uq holds u then, for
    ModelD, q with entry ncu + m + ncu*d = the d-th derivative component of u_m."""
    import sympy as sp
    nc = ncu * (nd + 1) if modelD else ncu
    uq = sp.symbols(f"uq0:{nc}")
    x = sp.symbols(f"x0:{nd}")
    mu = sp.symbols(f"mu0:{nparam}")
    uh = sp.symbols(f"uhat0:{ncu}")
    nl = sp.symbols(f"n0:{nd}")
    tau0 = sp.Symbol("tau0")
    lu = [(f"uq{k}", f"uq[{k}*N+i]") for k in range(nc)]
    lx = [(f"x{k}", f"x[{k}*N+i]") for k in range(nd)]
    lm = [(f"mu{k}", f"mu[{k}]") for k in range(nparam)]
    lh = [(f"uhat{k}", f"uhat[{k}*N+i]") for k in range(ncu)]
    ln = [(f"n{k}", f"n[{k}*N+i]") for k in range(nd)]
    F = flux(uq, x, mu)
    fo = [(f"f[{m + ncu * d} * N + i]", F[m][d]) for d in range(nd) for m in range(ncu)]
    fj = [(f"J1[{m + ncu * d + ncu * nd * c} * N + i]", sp.diff(F[m][d], uq[c]))
          for c in range(nc) for d in range(nd) for m in range(ncu)]
    S = source(uq, x, mu)
    so = [(f"f[{m} * N + i]", S[m]) for m in range(ncu)]
    sj = [(f"J1[{m + ncu * c} * N + i]", sp.diff(S[m], uq[c])) for c in range(nc) for m in range(ncu)]
    FB = fbou(uq, x, mu, uh, nl, tau0)
    bo = [(f"f[{m} * N + i]", FB[m]) for m in range(ncu)]
    bj1 = [(f"J1[{m + ncu * c} * N + i]", sp.diff(FB[m], uq[c])) for c in range(nc) for m in range(ncu)]
    bj3 = [(f"J3[{m + ncu * c} * N + i]", sp.diff(FB[m], uh[c])) for c in range(ncu) for m in range(ncu)]
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    J = "dstype* J1, dstype* J2, "
    files = {
        "KokkosFlux": _fn_sym("KokkosFlux", PT.format(J=""), "Flux", lx + lu + lm, fo),
        "HdgFlux": _fn_sym("HdgFlux", PT.format(J=J), "Flux", lx + lu + lm, fo + fj),
        "KokkosSource": _fn_sym("KokkosSource", PT.format(J=""), "Source", lx + lu + lm, so),
        "HdgSource": _fn_sym("HdgSource", PT.format(J=J), "Source", lx + lu + lm, so + sj),
        "KokkosTdfunc": _fn_sym("KokkosTdfunc", PT.format(J=""), "Tdfunc", [],
                                [(f"f[{m} * N + i]", 1) for m in range(ncu)]),
    }
    lb = lx + lu + lh + ln + [("tau0", "tau[0]")] + lm
    fb1 = _fn_sym("HdgFbou1", PTB.format(J="dstype* J1, dstype* J2, dstype* J3, "), "FbouHdg", lb, bo + bj1 + bj3)
    fb1o = _fn_sym("HdgFbouonly1", PTB.format(J=""), "FbouHdg", lb, bo)
    args = "xdg, udg, odg, wdg, uhg, nlg, tau, uinf, param, time, modelnumber, ng, nc, ncu, nd, ncx, nco, ncw, nc, ncu, nd"
    files["HdgFbou"] = fb1 + (f"\nvoid HdgFbou({DISPATCH.format(J='dstype* f_udg, dstype* f_wdg, dstype* f_uhg, ')}) {{\n"
                              f"    if (ib == 1 )\n        HdgFbou1(f, f_udg, f_wdg, f_uhg, {args});\n}}\n")
    files["HdgFbouonly"] = fb1o + (f"\nvoid HdgFbouonly({DISPATCH.format(J='')}) {{\n"
                                   f"    if (ib == 1 )\n        HdgFbouonly1(f, {args});\n}}\n")
    if ubou is not None:
        # the LDG boundary functions: uhat at the boundary face nodes (Ubou) and the boundary
        # flux (Fbou), boundary code 1
        lu_b = ubou(uq, x, mu, uh, nl, tau0)
        files["KokkosUbou"] = (_fn_sym("KokkosUbou1", PTB.format(J=""), "Ubou", lb,
                                       [(f"f[{m} * N + i]", lu_b[m]) for m in range(ncu)])
                               + f"\nvoid KokkosUbou({DISPATCH.format(J='')}) {{\n"
                               f"    if (ib == 1 )\n        KokkosUbou1(f, {args});\n}}\n")
        files["KokkosFbou"] = (_fn_sym("KokkosFbou1", PTB.format(J=""), "Fbou", lb, bo)
                               + f"\nvoid KokkosFbou({DISPATCH.format(J='')}) {{\n"
                               f"    if (ib == 1 )\n        KokkosFbou1(f, {args});\n}}\n")
    U0 = initu(x, mu)
    init_loads = "\n".join(f"    dstype x{k} = x[p+npe*{k}+npe*ncx*e];" for k in range(nd))
    init_loads += "\n" + "\n".join(f"    dstype mu{k} = mu[{k}];" for k in range(nparam))
    init_body = _emit([(f"f[p+npe*{m} +npe*nce*e]", U0[m]) for m in range(ncu)])
    files["cpuInitu"] = ("void cpuInitu(dstype* f, const dstype* x, const dstype* eta, const dstype* mu, "
                         "const int modelnumber, const int N, const int ncx, const int nce, const int npe, "
                         "const int ne)\n{\n\n  for (int i = 0; i < N; ++i) {\n    int p = i%npe; \n"
                         f"    int e = i/npe; \n{init_loads}\n\n{init_body}\n  }}\n}}\n")
    for k, v in files.items():
        with open(os.path.join(d, k + ".cpp"), "w") as fh:
            fh.write(v)


def _tau_fbou(F, uq, uh, nl, tau0, ncu, nd):
    """FbouHdg = f(u, q) . n + tau (u - uhat) (examples' fbouhdg)."""
    return [sum(F[m][d] * nl[d] for d in range(nd)) + tau0 * (uq[m] - uh[m]) for m in range(ncu)]


def ns2d_flux(uq, x, mu):
    """Compressible Navier-Stokes flux, inviscid + viscous, q = -grad(u) convention
    (examples/NavierStokes/TaylorGreenVortex/pdemodel.m reduced to two dimensions);
    mu = [gamma, Re, Pr, Minf]."""
    import sympy as sp
    gam, Re, Pr, Minf = mu[0], mu[1], mu[2], mu[3]
    gam1 = gam - 1
    Re1 = 1 / Re
    M2 = Minf * Minf
    c23 = sp.Rational(2, 3)
    fc = 1 / (gam1 * M2 * Re * Pr)
    r, ru, rv, rE = uq[0:4]
    rx, rux, rvx, rEx, ry, ruy, rvy, rEy = uq[4:12]
    r1 = 1 / r
    uv, vv = ru * r1, rv * r1
    E = rE * r1
    ke = (uv * uv + vv * vv) / 2
    p = gam1 * (rE - r * ke)
    h = E + p * r1
    ux, vx = (rux - rx * uv) * r1, (rvx - rx * vv) * r1
    kex = uv * ux + vv * vx
    px = gam1 * (rEx - rx * ke - r * kex)
    Tx = gam * M2 * (px * r - p * rx) * r1 * r1
    uy, vy = (ruy - ry * uv) * r1, (rvy - ry * vv) * r1
    key = uv * uy + vv * vy
    py = gam1 * (rEy - ry * ke - r * key)
    Ty = gam * M2 * (py * r - p * ry) * r1 * r1
    txx = Re1 * c23 * (2 * ux - vy)
    txy = Re1 * (uy + vx)
    tyy = Re1 * c23 * (2 * vy - ux)
    fx = [ru, ru * uv + p + txx, rv * uv + txy, ru * h + uv * txx + vv * txy + fc * Tx]
    fy = [rv, ru * vv + txy, rv * vv + p + tyy, rv * h + uv * txy + vv * tyy + fc * Ty]
    return [[fx[m], fy[m]] for m in range(4)]


def tgv2d_initu(x, mu):
    """2D Taylor-Green vortex on [0, 2 pi]^2: rho = 1, u = sin x cos y, v = -cos x sin y,
    p = 1/(gamma Minf^2) + (cos 2x + cos 2y)/4."""
    import sympy as sp
    gam, Minf = mu[0], mu[3]
    u = sp.sin(x[0]) * sp.cos(x[1])
    v = -sp.cos(x[0]) * sp.sin(x[1])
    p = 1 / (gam * Minf * Minf) + (sp.cos(2 * x[0]) + sp.cos(2 * x[1])) / 4
    return [sp.Integer(1), u, v, p / (gam - 1) + (u * u + v * v) / 2]


def euler3d_flux(uq, x, mu):
    """Compressible Euler flux (examples/Euler/EulerVortex/pdemodel.py in three dimensions);
    mu = [gamma, Minf]."""
    gam1 = mu[0] - 1
    r, ru, rv, rw, rE = uq[0:5]
    r1 = 1 / r
    uv, vv, wv = ru * r1, rv * r1, rw * r1
    p = gam1 * (rE - r * (uv * uv + vv * vv + wv * wv) / 2)
    h = rE * r1 + p * r1
    return [[ru, rv, rw], [ru * uv + p, ru * vv, ru * wv], [rv * uv, rv * vv + p, rv * wv],
            [rw * uv, rw * vv, rw * wv + p], [ru * h, rv * h, rw * h]]


def vortex3d_initu(x, mu):
    """Isentropic vortex of strength 5 about the z axis (examples/Euler/EulerVortex/pdemodel.py
    at t = 0), uniform in z, no z velocity."""
    import sympy as sp
    gam, M = mu[0], mu[1]
    phi = 5
    r2 = x[0] * x[0] + x[1] * x[1]
    rho = (1 - ((gam - 1) / (16 * sp.pi ** 2)) * phi ** 2 * sp.exp(2 * (1 - r2))) ** (1 / (gam - 1))
    ru = rho * (1 - phi * sp.exp(1 - r2) * x[1] / (2 * sp.pi * M))
    rv = rho * phi * sp.exp(1 - r2) * x[0] / (2 * sp.pi * M)
    p = rho ** gam / (gam * M * M)
    return [rho, ru, rv, sp.Integer(0), p / (gam - 1) + (ru * ru + rv * rv) / (2 * rho)]


def cdsin2d_flux(uq, x, mu):
    """kappa q + c u, mu = [kappa, c_x, c_y, a, b]."""
    return [[uq[1] * mu[0] + uq[0] * mu[1], uq[2] * mu[0] + uq[0] * mu[2]]]


def cdsin2d_source(uq, x, mu):
    """sin(a pi x) sin(b pi y)."""
    import sympy as sp
    return [sp.sin(mu[3] * sp.pi * x[0]) * sp.sin(mu[4] * sp.pi * x[1])]


def write_symbolic_cases():
    import sympy as sp
    zero = lambda ncu: (lambda uq, x, mu: [sp.Integer(0)] * ncu)
    write_symbolic_case(
        "ns2d", 2, 4, True, 4, ns2d_flux, zero(4),
        lambda uq, x, mu, uh, nl, t0: _tau_fbou(ns2d_flux(uq, x, mu), uq, uh, nl, t0, 4, 2), tgv2d_initu)
    write_symbolic_case(
        "euler3d", 3, 5, False, 2, euler3d_flux, zero(5),
        lambda uq, x, mu, uh, nl, t0: _tau_fbou(euler3d_flux(uq, x, mu), uq, uh, nl, t0, 5, 3), vortex3d_initu,
        ubou=lambda uq, x, mu, uh, nl, t0: [uq[m] for m in range(5)])
    write_symbolic_case(
        "cdsin2d", 2, 1, True, 5, cdsin2d_flux, cdsin2d_source,
        lambda uq, x, mu, uh, nl, t0: [t0 * (0 - uh[0])], lambda x, mu: [sp.Integer(0)])


if __name__ == "__main__":
    write_case("poisson2d", 2, False)
    write_case("poisson3d", 3, False)
    write_case("convdiff2d", 2, True)
    write_case("convdiff3d", 3, True)
    write_symbolic_cases()
