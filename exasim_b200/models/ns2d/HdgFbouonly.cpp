void HdgFbouonly1(dstype* f, const dstype* x, const dstype* uq, const dstype* v, const dstype* w, const dstype* uhat, const dstype* n, const dstype* tau, const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, const int szx, const int szuq, const int szv, const int szw, const int szuhat, const int szn, const int sztau, const int szeta, const int szmu)
{

  Kokkos::parallel_for("FbouHdg", N, KOKKOS_LAMBDA(const size_t i) {
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
    dstype uhat0 = uhat[0*N+i];
    dstype uhat1 = uhat[1*N+i];
    dstype uhat2 = uhat[2*N+i];
    dstype uhat3 = uhat[3*N+i];
    dstype n0 = n[0*N+i];
    dstype n1 = n[1*N+i];
    dstype tau0 = tau[0];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];
    dstype mu2 = mu[2];
    dstype mu3 = mu[3];

    dstype t0 = (1.0/(uq0));
    dstype t1 = (1.0/(mu1));
    dstype t2 = t0*uq4;
    dstype t3 = -t2*uq2 + uq6;
    dstype t4 = t0*uq8;
    dstype t5 = -t4*uq1 + uq9;
    dstype t6 = t3 + t5;
    dstype t7 = t1*t6;
    dstype t8 = t7 + uq1*uq2;
    dstype t9 = (uq1*uq1);
    dstype t10 = 6*t0;
    dstype t11 = 2*uq3;
    dstype t12 = (uq2*uq2);
    dstype t13 = t12 + t9;
    dstype t14 = t0*t13 - t11;
    dstype t15 = t14*(mu0 - 1);
    dstype t16 = 3*t15;
    dstype t17 = t2*uq1;
    dstype t18 = t4*uq2;
    dstype t19 = -t18 + uq10;
    dstype t20 = t0*t1;
    dstype t21 = 4*t20;
    dstype t22 = t21*(2*t17 + t19 - 2*uq5);
    dstype t23 = (1.0/6.0)*n0;
    dstype t24 = t21*(t17 - 2*t18 + 2*uq10 - uq5);
    dstype t25 = (1.0/6.0)*n1;
    dstype t26 = t11 - t15;
    dstype t27 = t13/(uq0*uq0);
    dstype t28 = 2*t0;
    dstype t29 = 3*mu0*t20/mu2;
    f[0 * N + i] = n0*uq1 + n1*uq2 - tau0*(uhat0 - uq0);
    f[1 * N + i] = n1*t0*t8 - t23*(-t10*t9 + t16 + t22) - tau0*(uhat1 - uq1);
    f[2 * N + i] = n0*t0*t8 + t25*(t10*t12 - t16 + t24) - tau0*(uhat2 - uq2);
    f[3 * N + i] = t0*t23*(6*t0*t1*t6*uq2 - t22*uq1 + 3*t26*uq1 - t29*(-t14*uq4 + uq0*(t27*uq4 + t28*(t3*uq2 + uq1*(-t17 + uq5)) - 2*uq7))) + t0*t25*(t10*t7*uq1 + t24*uq2 + 3*t26*uq2 - t29*(-t14*uq8 + uq0*(t27*uq8 + t28*(t19*uq2 + t5*uq1) - 2*uq11))) - tau0*(uhat3 - uq3);
  });
}

void HdgFbouonly(dstype* f, const dstype* xdg, const dstype* udg, const dstype* odg, const dstype* wdg, const dstype* uhg, const dstype* nlg, const dstype* tau, const dstype* uinf, const dstype* param, const dstype time, const int modelnumber, const int ib, const int ng, const int nc, const int ncu, const int nd, const int ncx, const int nco, const int ncw) {
    if (ib == 1 )
        HdgFbouonly1(f, xdg, udg, odg, wdg, uhg, nlg, tau, uinf, param, time, modelnumber, ng, nc, ncu, nd, ncx, nco, ncw, nc, ncu, nd);
}
