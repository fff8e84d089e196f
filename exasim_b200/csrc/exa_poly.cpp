// Host part of the polynomial preconditioner (getPoly, backend/Solver/getpoly.cpp:150-247, and
// the Ritz-value post-processing of GMRES, backend/Solver/gmres.cpp:385-398): from the
// Hessenberg matrix of m Arnoldi steps of the preconditioned operator, the harmonic Ritz values
// in Leja order, the roots of the polynomial that ApplyPoly (gmres.cpp:319-357) applies.
//
//   eigH (getpoly.cpp:111-124): Hm + beta^2 (Hm^-T e_m) e_m^T, with Hm the leading m x m block
//     and beta = H(m, m-1), the subdiagonal entry below it;
//   its eigenvalues (the reference calls LAPACK dgeev; here the Francis double-shift QR
//     iteration on the upper Hessenberg matrix, Golub & Van Loan, Matrix Computations, 7.5);
//   LejaSort (getpoly.cpp:130-173): the largest in modulus first, then each next point
//     maximising the sum of log-distances to those chosen, complex pairs kept together;
//   when every value is real, m points spread over [lmin, lmax] by
//     lmin + (lmax - lmin) (1/2 - cos((2i-1) pi / (2m)) / (2 cos(pi / (2m)))), Leja-ordered again.
#include <cmath>
#include <vector>

#include "exa_common.cuh"

namespace {

// eigenvalues of an upper Hessenberg n x n matrix a (column-major, changed in place)
bool hessenberg_eigenvalues(std::vector<double>& a, int n, std::vector<double>& wr, std::vector<double>& wi) {
  auto A = [&](int i, int j) -> double& { return a[(size_t)i + (size_t)n * j]; };
  wr.assign(n, 0.0);
  wi.assign(n, 0.0);
  double anorm = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = (i > 0 ? i - 1 : 0); j < n; ++j) anorm += std::fabs(A(i, j));
  int hi = n - 1;      // last row of the active block
  double shift = 0.0;  // exceptional shifts accumulated
  int its = 0;
  while (hi >= 0) {
    // the active block's first row: the subdiagonal entry above it is negligible
    int lo = hi;
    for (; lo >= 1; --lo) {
      double s = std::fabs(A(lo - 1, lo - 1)) + std::fabs(A(lo, lo));
      if (s == 0.0) s = anorm;
      if (std::fabs(A(lo, lo - 1)) + s == s) {
        A(lo, lo - 1) = 0.0;
        break;
      }
    }
    double x = A(hi, hi);
    if (lo == hi) {  // a 1 x 1 block: one real eigenvalue
      wr[hi] = x + shift;
      wi[hi] = 0.0;
      --hi;
      its = 0;
      continue;
    }
    double y = A(hi - 1, hi - 1), w = A(hi, hi - 1) * A(hi - 1, hi);
    if (lo == hi - 1) {  // a 2 x 2 block: a real pair or a complex-conjugate pair
      const double p = 0.5 * (y - x), q = p * p + w;
      double z = std::sqrt(std::fabs(q));
      x += shift;
      if (q >= 0.0) {
        z = p + (p >= 0.0 ? z : -z);
        wr[hi - 1] = wr[hi] = x + z;
        if (z != 0.0) wr[hi] = x - w / z;
        wi[hi - 1] = wi[hi] = 0.0;
      } else {
        // a conjugate pair with the positive imaginary part first, as LAPACK returns them
        wr[hi - 1] = wr[hi] = x + p;
        wi[hi - 1] = z;
        wi[hi] = -z;
      }
      hi -= 2;
      its = 0;
      continue;
    }
    if (its == 60) return false;
    if (its == 10 || its == 20) {  // exceptional shift
      shift += x;
      for (int i = 0; i <= hi; ++i) A(i, i) -= x;
      const double s = std::fabs(A(hi, hi - 1)) + std::fabs(A(hi - 1, hi - 2));
      y = x = 0.75 * s;
      w = -0.4375 * s * s;
    }
    ++its;
    // first column of (H - s1 I)(H - s2 I) from the trailing 2 x 2 block's eigenvalues,
    // starting at the lowest row m where the bulge does not interact with the block above
    int m = hi - 2;
    double p = 0.0, q = 0.0, r = 0.0, z = 0.0;
    for (; m >= lo; --m) {
      z = A(m, m);
      const double rr = x - z, ss = y - z;
      p = (rr * ss - w) / A(m + 1, m) + A(m, m + 1);
      q = A(m + 1, m + 1) - z - rr - ss;
      r = A(m + 2, m + 1);
      const double sc = std::fabs(p) + std::fabs(q) + std::fabs(r);
      p /= sc;
      q /= sc;
      r /= sc;
      if (m == lo) break;
      const double u = std::fabs(A(m, m - 1)) * (std::fabs(q) + std::fabs(r));
      const double v = std::fabs(p) * (std::fabs(A(m - 1, m - 1)) + std::fabs(z) + std::fabs(A(m + 1, m + 1)));
      if (u + v == v) break;
    }
    for (int i = m + 2; i <= hi; ++i) {
      A(i, i - 2) = 0.0;
      if (i != m + 2) A(i, i - 3) = 0.0;
    }
    // chase the bulge with 3-element Householder reflections
    for (int k = m; k <= hi - 1; ++k) {
      if (k != m) {
        p = A(k, k - 1);
        q = A(k + 1, k - 1);
        r = (k != hi - 1) ? A(k + 2, k - 1) : 0.0;
        x = std::fabs(p) + std::fabs(q) + std::fabs(r);
        if (x != 0.0) {
          p /= x;
          q /= x;
          r /= x;
        }
      }
      const double nrm = std::sqrt(p * p + q * q + r * r);
      const double s = p >= 0.0 ? nrm : -nrm;
      if (s == 0.0) continue;
      if (k == m) {
        if (lo != m) A(k, k - 1) = -A(k, k - 1);
      } else {
        A(k, k - 1) = -s * x;
      }
      p += s;
      x = p / s;
      y = q / s;
      z = r / s;
      q /= p;
      r /= p;
      for (int j = k; j <= hi; ++j) {  // rows k .. k + 2
        double t = A(k, j) + q * A(k + 1, j);
        if (k != hi - 1) {
          t += r * A(k + 2, j);
          A(k + 2, j) -= t * z;
        }
        A(k + 1, j) -= t * y;
        A(k, j) -= t * x;
      }
      const int imax = hi < k + 3 ? hi : k + 3;
      for (int i = lo; i <= imax; ++i) {  // columns k .. k + 2
        double t = x * A(i, k) + y * A(i, k + 1);
        if (k != hi - 1) {
          t += z * A(i, k + 2);
          A(i, k + 2) -= t * r;
        }
        A(i, k + 1) -= t * q;
        A(i, k) -= t;
      }
    }
  }
  return true;
}

// LejaSort (getpoly.cpp:130-173): lr, li in; sr, si out (n values)
void leja_sort(const std::vector<double>& lr, const std::vector<double>& li, std::vector<double>& sr,
               std::vector<double>& si, int n) {
  sr.assign(n, 0.0);
  si.assign(n, 0.0);
  auto cabs = [](double a, double b) { return std::sqrt(a * a + b * b); };
  sr[0] = lr[0];
  si[0] = li[0];
  for (int i = 1; i < n; ++i)
    if (cabs(lr[i], li[i]) > cabs(sr[0], si[0])) {
      sr[0] = lr[i];
      si[0] = li[i];
    }
  int j = 1;
  if (std::fabs(si[0]) > 1e-10) {
    if (n > 1) {
      sr[1] = sr[0];
      si[1] = -si[0];
    }
    j = 2;
  } else {
    si[0] = 0.0;
  }
  std::vector<double> prod(n);
  while (j < n) {
    for (int i = 0; i < n; ++i) {
      prod[i] = 1.0;
      for (int k = 0; k < j; ++k) prod[i] += std::log(cabs(lr[i] - sr[k], li[i] - si[k]));
    }
    sr[j] = lr[0];
    si[j] = li[0];
    double best = prod[0];
    for (int i = 1; i < n; ++i)
      if (prod[i] > best) {
        sr[j] = lr[i];
        si[j] = li[i];
        best = prod[i];
      }
    if (std::fabs(si[j]) > 1e-10) {
      if (j + 1 < n) {
        sr[j + 1] = sr[j];
        si[j + 1] = -si[j];
      }
      j += 1;
    } else {
      si[j] = 0.0;
    }
    j += 1;
  }
}

// in-place inverse of an m x m matrix by Gauss-Jordan with partial pivoting (the reference
// uses LAPACK getrf + getri, cpuimpl.h cpuComputeInverse); false if singular
bool small_inverse(std::vector<double>& a, int m) {
  std::vector<int> piv(m);
  std::vector<double> inv((size_t)m * m, 0.0);
  std::vector<double> w(a);
  for (int i = 0; i < m; ++i) inv[(size_t)i + (size_t)m * i] = 1.0;
  for (int k = 0; k < m; ++k) {
    int p = k;
    for (int r = k + 1; r < m; ++r)
      if (std::fabs(w[(size_t)r + (size_t)m * k]) > std::fabs(w[(size_t)p + (size_t)m * k])) p = r;
    if (w[(size_t)p + (size_t)m * k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < m; ++j) {
        std::swap(w[(size_t)p + (size_t)m * j], w[(size_t)k + (size_t)m * j]);
        std::swap(inv[(size_t)p + (size_t)m * j], inv[(size_t)k + (size_t)m * j]);
      }
    const double d = 1.0 / w[(size_t)k + (size_t)m * k];
    for (int j = 0; j < m; ++j) {
      w[(size_t)k + (size_t)m * j] *= d;
      inv[(size_t)k + (size_t)m * j] *= d;
    }
    for (int r = 0; r < m; ++r) {
      if (r == k) continue;
      const double f = w[(size_t)r + (size_t)m * k];
      if (f == 0.0) continue;
      for (int j = 0; j < m; ++j) {
        w[(size_t)r + (size_t)m * j] -= f * w[(size_t)k + (size_t)m * j];
        inv[(size_t)r + (size_t)m * j] -= f * inv[(size_t)k + (size_t)m * j];
      }
    }
  }
  a.swap(inv);
  return true;
}

}  // namespace

extern "C" int exa_poly_ritz(const double* H, int m, double* sr_out, double* si_out) {
  if (!H || !sr_out || !si_out || m < 2 || m > 64) {
    exa_set_error("poly ritz: need H [(m+1) x m], outputs and 2 <= m <= 64 (m = %d)", m);
    return EXA_ERR_ARG;
  }
  const int m1 = m + 1;
  // eigH: Hm^T, its inverse, work = Hm^-T e_m, then Hm + beta^2 work e_m^T
  std::vector<double> HT((size_t)m * m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) HT[(size_t)j + (size_t)m * i] = H[(size_t)i + (size_t)m1 * j];
  if (!small_inverse(HT, m)) {
    exa_set_error("poly ritz: the Hessenberg block is singular");
    return EXA_ERR_SINGULAR;
  }
  std::vector<double> work(m);
  for (int i = 0; i < m; ++i) work[i] = HT[(size_t)i + (size_t)m * (m - 1)];
  const double beta2 = H[(size_t)m1 * m - 1] * H[(size_t)m1 * m - 1];
  std::vector<double> A((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i)
      A[(size_t)i + (size_t)m * j] = H[(size_t)i + (size_t)m1 * j] + (j == m - 1 ? beta2 * work[i] : 0.0);
  std::vector<double> wr, wi, sr, si;
  if (!hessenberg_eigenvalues(A, m, wr, wi)) {
    exa_set_error("poly ritz: the QR iteration did not converge");
    return EXA_ERR_NOTCONV;
  }
  leja_sort(wr, wi, sr, si, m);
  double lmin = 1.0e10, lmax = -1.0e10, smax = 0.0;
  for (int i = 0; i < m; ++i) {
    lmax = sr[i] > lmax ? sr[i] : lmax;
    lmin = sr[i] < lmin ? sr[i] : lmin;
    smax = std::fabs(si[i]) > smax ? std::fabs(si[i]) : smax;
  }
  if (smax == 0.0) {
    const double pi = 3.14159265358979323846;
    std::vector<double> lam(m), zero(m, 0.0);
    for (int i = 1; i <= m; ++i)
      lam[i - 1] = lmin + (lmax - lmin) * (0.5 - 0.5 * std::cos((2 * i - 1) * pi / (2 * m)) / std::cos(pi / (2 * m)));
    leja_sort(lam, zero, sr, si, m);
  }
  for (int i = 0; i < m; ++i) {
    sr_out[i] = sr[i];
    si_out[i] = si[i];
  }
  return EXA_OK;
}
