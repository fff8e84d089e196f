void KokkosFlux(dstype* f, const dstype* x, const dstype* uq, const dstype* v, const dstype* w, const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, const int szx, const int szuq, const int szv, const int szw, const int szeta, const int szmu)
{

  Kokkos::parallel_for("Flux", N, KOKKOS_LAMBDA(const size_t i) {
    dstype x0 = x[0*N+i];
    dstype x1 = x[1*N+i];
    dstype uq0 = uq[0*N+i];
    dstype uq1 = uq[1*N+i];
    dstype uq2 = uq[2*N+i];
    dstype uq3 = uq[3*N+i];
    dstype uq4 = uq[4*N+i];
    dstype uq5 = uq[5*N+i];
    dstype uq6 = uq[6*N+i];
    dstype uq7 = uq[7*N+i];
    dstype uq8 = uq[8*N+i];
    dstype uq9 = uq[9*N+i];
    dstype uq10 = uq[10*N+i];
    dstype uq11 = uq[11*N+i];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];
    dstype mu2 = mu[2];
    dstype mu3 = mu[3];

    dstype t0 = (1.0/(uq0));
    dstype t1 = (uq1*uq1);
    dstype t2 = 2*uq3;
    dstype t3 = (uq2*uq2);
    dstype t4 = t1 + t3;
    dstype t5 = t0*t4 - t2;
    dstype t6 = t5*(mu0 - 1);
    dstype t7 = (1.0/2.0)*t6;
    dstype t8 = t0*uq4;
    dstype t9 = t8*uq1;
    dstype t10 = t0*uq8;
    dstype t11 = t10*uq2;
    dstype t12 = -t11 + uq10;
    dstype t13 = (1.0/(mu1));
    dstype t14 = t0*t13;
    dstype t15 = (2.0/3.0)*t14;
    dstype t16 = t15*(t12 + 2*t9 - 2*uq5);
    dstype t17 = -t8*uq2 + uq6;
    dstype t18 = -t10*uq1 + uq9;
    dstype t19 = t17 + t18;
    dstype t20 = t13*t19;
    dstype t21 = t0*(t20 + uq1*uq2);
    dstype t22 = t2 - t6;
    dstype t23 = t4/(uq0*uq0);
    dstype t24 = 2*t0;
    dstype t25 = (1.0/2.0)*mu0*t14/mu2;
    dstype t26 = t15*(-2*t11 + t9 + 2*uq10 - uq5);
    f[0 * N + i] = uq1;
    f[1 * N + i] = t0*t1 - t16 - t7;
    f[2 * N + i] = t21;
    f[3 * N + i] = t0*(t0*t13*t19*uq2 - t16*uq1 + (1.0/2.0)*t22*uq1 - t25*(-t5*uq4 + uq0*(t23*uq4 + t24*(t17*uq2 + uq1*(-t9 + uq5)) - 2*uq7)));
    f[4 * N + i] = uq2;
    f[5 * N + i] = t21;
    f[6 * N + i] = t0*t3 + t26 - t7;
    f[7 * N + i] = t0*(t0*t20*uq1 + (1.0/2.0)*t22*uq2 - t25*(-t5*uq8 + uq0*(t23*uq8 + t24*(t12*uq2 + t18*uq1) - 2*uq11)) + t26*uq2);
  });
}
