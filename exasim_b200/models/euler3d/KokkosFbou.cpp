void KokkosFbou1(dstype* f, const dstype* x, const dstype* uq, const dstype* v, const dstype* w, const dstype* uhat, const dstype* n, const dstype* tau, const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, const int szx, const int szuq, const int szv, const int szw, const int szuhat, const int szn, const int sztau, const int szeta, const int szmu)
{

  Kokkos::parallel_for("Fbou", N, KOKKOS_LAMBDA(const size_t i) {
    dstype x0 = x[0*N+i];
    dstype x1 = x[1*N+i];
    dstype x2 = x[2*N+i];
    dstype uq0 = uq[0*N+i];
    dstype uq1 = uq[1*N+i];
    dstype uq2 = uq[2*N+i];
    dstype uq3 = uq[3*N+i];
    dstype uq4 = uq[4*N+i];
    dstype uhat0 = uhat[0*N+i];
    dstype uhat1 = uhat[1*N+i];
    dstype uhat2 = uhat[2*N+i];
    dstype uhat3 = uhat[3*N+i];
    dstype uhat4 = uhat[4*N+i];
    dstype n0 = n[0*N+i];
    dstype n1 = n[1*N+i];
    dstype n2 = n[2*N+i];
    dstype tau0 = tau[0];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];

    dstype t0 = n0*uq1;
    dstype t1 = n1*uq2;
    dstype t2 = n2*uq3;
    dstype t3 = (1.0/(uq0));
    dstype t4 = (uq1*uq1);
    dstype t5 = 2*t3;
    dstype t6 = 2*uq4;
    dstype t7 = (uq2*uq2);
    dstype t8 = (uq3*uq3);
    dstype t9 = (mu0 - 1)*(t3*(t4 + t7 + t8) - t6);
    dstype t10 = t3*uq2;
    dstype t11 = t3*uq3;
    dstype t12 = (1.0/2.0)*t3*(t6 - t9);
    f[0 * N + i] = t0 + t1 + t2 - tau0*(uhat0 - uq0);
    f[1 * N + i] = -1.0/2.0*n0*(-t4*t5 + t9) + n1*t3*uq1*uq2 + n2*t3*uq1*uq3 - tau0*(uhat1 - uq1);
    f[2 * N + i] = -1.0/2.0*n1*(-t5*t7 + t9) + t0*t10 + t10*t2 - tau0*(uhat2 - uq2);
    f[3 * N + i] = -1.0/2.0*n2*(-t5*t8 + t9) + t0*t11 + t1*t11 - tau0*(uhat3 - uq3);
    f[4 * N + i] = t0*t12 + t1*t12 + t12*t2 - tau0*(uhat4 - uq4);
  });
}

void KokkosFbou(dstype* f, const dstype* xdg, const dstype* udg, const dstype* odg, const dstype* wdg, const dstype* uhg, const dstype* nlg, const dstype* tau, const dstype* uinf, const dstype* param, const dstype time, const int modelnumber, const int ib, const int ng, const int nc, const int ncu, const int nd, const int ncx, const int nco, const int ncw) {
    if (ib == 1 )
        KokkosFbou1(f, xdg, udg, odg, wdg, uhg, nlg, tau, uinf, param, time, modelnumber, ng, nc, ncu, nd, ncx, nco, ncw, nc, ncu, nd);
}
