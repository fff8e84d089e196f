void cpuInitu(dstype* f, const dstype* x, const dstype* eta, const dstype* mu, const int modelnumber, const int N, const int ncx, const int nce, const int npe, const int ne)
{

  for (int i = 0; i < N; ++i) {
    int p = i%npe; 
    int e = i/npe; 
    dstype x0 = x[p+npe*0+npe*ncx*e];
    dstype x1 = x[p+npe*1+npe*ncx*e];
    dstype x2 = x[p+npe*2+npe*ncx*e];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];

    dstype t0 = mu0 - 1;
    dstype t1 = (x0*x0);
    dstype t2 = (x1*x1);
    dstype t3 = exp(-2*t1 - 2*t2 + 2)/(M_PI*M_PI);
    dstype t4 = (1.0/(t0));
    dstype t5 = pow(-25.0/16.0*t0*t3 + 1, t4);
    dstype t6 = (1.0/(M_PI));
    dstype t7 = (1.0/(mu1));
    dstype t8 = exp(-t1 - t2 + 1);
    dstype t9 = t6*t7*t8*x1;
    dstype t10 = (1.0/(mu1*mu1));
    f[p+npe*0 +npe*nce*e] = t5;
    f[p+npe*1 +npe*nce*e] = t5*(1 - 5.0/2.0*t9);
    f[p+npe*2 +npe*nce*e] = (5.0/2.0)*t5*t6*t7*t8*x0;
    f[p+npe*3 +npe*nce*e] = 0;
    f[p+npe*4 +npe*nce*e] = (1.0/8.0)*t5*(25*t1*t10*t3 + ((2 - 5*t9)*(2 - 5*t9))) + t10*t4*pow(t5, mu0)/mu0;
  }
}
