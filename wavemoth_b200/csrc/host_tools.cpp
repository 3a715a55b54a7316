// Host-side numerical tools of the plan-file writer (the precompute step that
// produces rev1 resource files):
//   - normalised associated Legendre matrices (legendre.cuh),
//   - the even/odd recurrence coefficients,
//   - a precision-controlled interpolative decomposition (ID).
//
// The ID follows the semantics of the ID library routine iddp_id that the
// reference's compressor calls (wavemoth/interpolative_decomposition.pyx:
// 42-107, libidlight/idd_qrpiv.f:391-...): Householder QR with greedy column
// pivoting that stops as soon as the largest remaining column norm satisfies
// ||a_j||^2 <= eps^2 * max_j ||a_j(input)||^2 (or the rank reaches
// min(rows, cols)); then T = R11^{-1} R12, so that
//     A[:, ipol] ~= A[:, iden] @ T.
// Column norms are recomputed from the trailing block at every step instead
// of being downdated; this costs the same order as the reflection itself and
// has no cancellation problem.
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>
#include <algorithm>

#include "legendre.cuh"

extern "C" {

// out is (ntheta, lmax - m + 1) row-major; returns 0 or a negative error.
int wm_host_legendre(int m, const double *theta, int ntheta, int lmax, double eps,
                     double *out) {
  if (m < 0 || lmax < m || ntheta < 0) return -1;
  const int nl = lmax - m + 1;
  for (int i = 0; i < ntheta; ++i) {
    if (!(theta[i] >= 0.0 && theta[i] <= 3.14159265358979323846)) return -2;
    wm::legendre_column(m, theta[i], lmax, eps, out + (size_t)i * nl);
  }
  return 0;
}

// aux[3*(k-2) + {0,1,2}] = (alpha_k, beta_k, gamma_k) for k = 2..nk-1.
void wm_host_recurrence_coefficients(int64_t m, int64_t lmin, int64_t nk, double *aux) {
  for (int64_t k = 2; k < nk; ++k)
    wm::rec_abg(m, lmin, k, aux + 3 * (k - 2), aux + 3 * (k - 2) + 1, aux + 3 * (k - 2) + 2);
}

// A: (m x n) column-major, destroyed.  On return:
//   *krank = numerical rank,
//   perm[0..n) = column permutation; perm[0..krank) are the skeleton columns,
//   proj (krank x (n-krank), column-major) with A[:, perm[krank+j]] ~=
//        sum_i A[:, perm[i]] proj[i + j*krank].
// Returns 0.
int wm_host_interp_decomp(double *A, int m, int n, double eps, int *krank_out, int *perm,
                          double *proj) {
  for (int j = 0; j < n; ++j) perm[j] = j;
  *krank_out = 0;
  if (m <= 0 || n <= 0) return 0;
  std::vector<double> ss(n), v(m);
  auto col = [&](int j) { return A + (size_t)j * m; };
  double ssmaxin = 0.0;
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    const double *c = col(j);
    for (int i = 0; i < m; ++i) s += c[i] * c[i];
    ss[j] = s;
    ssmaxin = std::max(ssmaxin, s);
  }
  const double thresh = eps * eps * ssmaxin;
  const int kmax = std::min(m, n);
  int k = 0;
  for (;;) {
    if (k >= kmax) break;
    int kpiv = k;
    double ssmax = ss[k];
    for (int j = k + 1; j < n; ++j)
      if (ss[j] > ssmax) { ssmax = ss[j]; kpiv = j; }
    if (!(ssmax > thresh)) break;
    if (kpiv != k) {
      std::swap(perm[k], perm[kpiv]);
      std::swap(ss[k], ss[kpiv]);
      double *a = col(k), *b = col(kpiv);
      for (int i = 0; i < m; ++i) std::swap(a[i], b[i]);
    }
    // Householder reflection zeroing A[k+1:, k]
    double *ck = col(k);
    double norm2 = 0.0;
    for (int i = k; i < m; ++i) norm2 += ck[i] * ck[i];
    double nrm = sqrt(norm2);
    double alpha = (ck[k] > 0) ? -nrm : nrm;
    double vtv = 0.0;
    for (int i = k; i < m; ++i) v[i] = ck[i];
    v[k] -= alpha;
    for (int i = k; i < m; ++i) vtv += v[i] * v[i];
    ck[k] = alpha;
    for (int i = k + 1; i < m; ++i) ck[i] = 0.0;
    if (vtv > 0.0) {
      const double inv = 2.0 / vtv;
      for (int j = k + 1; j < n; ++j) {
        double *cj = col(j);
        double d = 0.0;
        for (int i = k; i < m; ++i) d += v[i] * cj[i];
        d *= inv;
        for (int i = k; i < m; ++i) cj[i] -= d * v[i];
      }
    }
    ++k;
    for (int j = k; j < n; ++j) {
      const double *cj = col(j);
      double s = 0.0;
      for (int i = k; i < m; ++i) s += cj[i] * cj[i];
      ss[j] = s;
    }
  }
  const int krank = k;
  *krank_out = krank;
  // proj = R11^{-1} R12 by back substitution, column by column
  for (int j = 0; j < n - krank; ++j) {
    const double *r = col(krank + j);
    double *t = proj + (size_t)j * krank;
    for (int i = krank - 1; i >= 0; --i) {
      double s = r[i];
      for (int p = i + 1; p < krank; ++p) s -= col(p)[i] * t[p];
      t[i] = s / col(i)[i];
    }
  }
  return 0;
}

// Row nk - 1 of the three-term recurrence P_k = (x2 + alpha_k) beta_k P_{k-1}
// + gamma_k P_{k-2} started from P0, P1 (aux: (alpha, beta, gamma) for k =
// 2 .. nk - 1), for nx columns; the plan writer's stability check.
void wm_host_recurrence_last_row(const double *x2, const double *P0, const double *P1, const double *aux,
                                 int64_t nx, int64_t nk, double *out) {
  for (int64_t j = 0; j < nx; ++j) {
    double pp = P0[j], p = P1[j];
    if (nk <= 1) {
      out[j] = pp;
      continue;
    }
    for (int64_t k = 2; k < nk; ++k) {
      const double *a = aux + 3 * (k - 2);
      const double nv = (x2[j] + a[0]) * a[1] * p + a[2] * pp;
      pp = p;
      p = nv;
    }
    out[j] = p;
  }
}

}  // extern "C"
