void KokkosSource(dstype* f, const dstype* x, const dstype* uq, const dstype* v, const dstype* w, const dstype* eta, const dstype* mu, const dstype t, const int modelnumber, const int N, const int szx, const int szuq, const int szv, const int szw, const int szeta, const int szmu)
{

  Kokkos::parallel_for("Source", N, KOKKOS_LAMBDA(const size_t i) {
    dstype x0 = x[0*N+i];
    dstype x1 = x[1*N+i];
    dstype x2 = x[2*N+i];

    f[0 * N + i] = sin(x0*3.141592653589793)*sin(x1*3.141592653589793)*sin(x2*3.141592653589793)*2.960881320326807E+1;
  });
}
