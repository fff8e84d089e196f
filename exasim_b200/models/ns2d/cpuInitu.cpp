void cpuInitu(dstype* f, const dstype* x, const dstype* eta, const dstype* mu, const int modelnumber, const int N, const int ncx, const int nce, const int npe, const int ne)
{

  for (int i = 0; i < N; ++i) {
    int p = i%npe; 
    int e = i/npe; 
    dstype x0 = x[p+npe*0+npe*ncx*e];
    dstype x1 = x[p+npe*1+npe*ncx*e];
    dstype mu0 = mu[0];
    dstype mu1 = mu[1];
    dstype mu2 = mu[2];
    dstype mu3 = mu[3];

    dstype t0 = sin(x0);
    dstype t1 = cos(x1);
    dstype t2 = sin(x1);
    dstype t3 = cos(x0);
    f[p+npe*0 +npe*nce*e] = 1;
    f[p+npe*1 +npe*nce*e] = t0*t1;
    f[p+npe*2 +npe*nce*e] = -t2*t3;
    f[p+npe*3 +npe*nce*e] = (1.0/2.0)*(t0*t0)*(t1*t1) + (1.0/2.0)*(t2*t2)*(t3*t3) + (1.0/4.0)*(cos(2*x0) + cos(2*x1) + 4/(mu0*(mu3*mu3)))/(mu0 - 1);
  }
}
