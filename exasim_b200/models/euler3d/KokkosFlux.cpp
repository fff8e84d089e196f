void KokkosFlux(dstype* f, const dstype* x, const dstype* uq, const dstype* v, const dstype* w, const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, const int szx, const int szuq, const int szv, const int szw, const int szeta, const int szmu)
{

  Kokkos::parallel_for("Flux", N, KOKKOS_LAMBDA(const size_t i) {
    dstype x0 = x[0*N+i];
    dstype x1 = x[1*N+i];
    dstype x2 = x[2*N+i];
    dstype uq0 = uq[0*N+i];
    dstype uq1 = uq[1*N+i];
    dstype uq2 = uq[2*N+i];
    dstype uq3 = uq[3*N+i];
    dstype uq4 = uq[4*N+i];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];

    dstype t0 = (1.0/(uq0));
    dstype t1 = (uq1*uq1);
    dstype t2 = (uq2*uq2);
    dstype t3 = (uq3*uq3);
    dstype t4 = (1.0/2.0)*(mu0 - 1)*(t0*(t1 + t2 + t3) - 2*uq4);
    dstype t5 = t0*uq1;
    dstype t6 = t5*uq2;
    dstype t7 = t5*uq3;
    dstype t8 = -t4 + uq4;
    dstype t9 = t0*uq2;
    dstype t10 = t9*uq3;
    f[0 * N + i] = uq1;
    f[1 * N + i] = t0*t1 - t4;
    f[2 * N + i] = t6;
    f[3 * N + i] = t7;
    f[4 * N + i] = t5*t8;
    f[5 * N + i] = uq2;
    f[6 * N + i] = t6;
    f[7 * N + i] = t0*t2 - t4;
    f[8 * N + i] = t10;
    f[9 * N + i] = t8*t9;
    f[10 * N + i] = uq3;
    f[11 * N + i] = t7;
    f[12 * N + i] = t10;
    f[13 * N + i] = t0*t3 - t4;
    f[14 * N + i] = t0*t8*uq3;
  });
}
