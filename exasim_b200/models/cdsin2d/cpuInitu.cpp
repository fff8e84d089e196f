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
    dstype mu4 = mu[4];

    f[p+npe*0 +npe*nce*e] = 0;
  }
}
