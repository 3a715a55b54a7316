// Normalised associated Legendre values lambda_lm(theta) in FP64, shared by
// host code (the plan-file writer) and device code (seed values for
// recomputed residual blocks).
//
// Algorithm (libpsht's Ylmgen, libpshtlight/ylmgen_c.c:643-732, as used by
// wavemoth/legendre.pyx:24-57): start from
//     lambda_mm = (-1)^m sqrt(1/4pi) prod_{k=1..m} sqrt((2k+1)/(2k)) sin^m(theta)
// evaluated in the log2 domain, split into a mantissa and an exponent that is
// a multiple of 90, and run the step-1 recurrence in l
//     lambda_{l+1} = cos(theta) r0(l) lambda_l - r1(l) lambda_{l-1},
//     r0(l) = sqrt((4(l+1)^2 - 1) / ((l+m+1)(l-m+1))), r1(l) = r0(l)/r0(l-1),
// renormalising by 2^-90 whenever the scaled value exceeds 2^90 until the
// exponent reaches zero.  Values before the first l with |lambda| > eps are
// returned as 0.
#pragma once
#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define WM_HD __host__ __device__ __forceinline__
#else
#define WM_HD inline
#endif

namespace wm {

constexpr int kExpStep = 90;      // log2 of the rescaling factor
constexpr int kMinScale = -4;     // lowest exponent bucket (2^-360)

// log2 of sqrt(1/4pi) * prod_{k=1..m} sqrt((2k+1)/2k)
WM_HD double log2_pmm_prefactor(int m) {
  double f = 1.0;
  for (int k = 1; k <= m; ++k) f *= sqrt((2.0 * k + 1.0) / (2.0 * k));
  return log2(0.28209479177387814347 * f);
}

WM_HD double rec_r0(int l, int m) {
  return sqrt(4.0 * (l + 1) * (l + 1) - 1.0) / sqrt((double)(l + m + 1) * (double)(l - m + 1));
}

// Walks lambda_lm(theta) for l = m..lmax and calls visit(l, value) for every
// l from the first with |value| > eps on (the values before it are zero);
// stops early when visit returns false.  theta in [0, pi].  Returns that
// first l (lmax + 1 if all values are zero).
template <class Visit>
WM_HD int legendre_walk(int m, double theta, int lmax, double eps, Visit &&visit) {
  const double pi = 3.14159265358979323846;
  if (theta == 0.0) theta = 1e-16;
  if (fabs(theta - pi) < 1e-15) theta = pi - 1e-15;
  double cth = cos(theta), sth = sin(theta);
  if (m > 0 && sth == 0.0) return lmax + 1;

  double lg = log2_pmm_prefactor(m);
  if (m > 0) lg += m * log2(sth);
  int scale = (int)(lg / kExpStep) - kMinScale;      // bucket index, >= 0 means representable
  double prev = 0.0;
  double cur = exp2(lg - (double)((scale + kMinScale) * kExpStep));
  if (m & 1) cur = -cur;
  const double big = 0x1p90, small = 0x1p-90;

  int l = m;
  double r1_prev = 1.0;  // r0(l-1) for r1 = r0(l)/r0(l-1)
  // advance one step: (prev, cur) at l -> at l+1
  auto step = [&](int lcur) {
    double r0 = rec_r0(lcur, m);
    double r1 = (lcur == m) ? 0.0 : r0 / r1_prev;
    double nxt = cth * cur * r0 - prev * r1;
    r1_prev = r0;
    prev = cur;
    cur = nxt;
  };
  // scaled phase: values carry an implicit factor 2^((scale + kMinScale) * 90)
  while (scale < 0) {
    if (l + 1 > lmax) return lmax + 1;
    step(l);
    ++l;
    if (fabs(cur) > big) {
      while (fabs(cur) > big) { prev *= small; cur *= small; ++scale; }
    }
  }
  {
    // remaining implicit factor; 2^0 for the bucket that needs no scaling
    double f = exp2((double)((scale + kMinScale) * kExpStep));
    prev *= f;
    cur *= f;
  }
  // skip values below eps
  while (fabs(cur) <= eps) {
    if (l + 1 > lmax) return lmax + 1;
    step(l);
    ++l;
  }
  int first = l;
  if (!visit(l, cur)) return first;
  while (l + 1 <= lmax) {
    step(l);
    ++l;
    if (!visit(l, cur)) break;
  }
  return first;
}

// Fills out[l - m] for l = m..lmax (zero before the first |value| > eps).
// Returns the first l with a value stored (lmax + 1 if all zero).
WM_HD int legendre_column(int m, double theta, int lmax, double eps, double *out) {
  for (int l = m; l <= lmax; ++l) out[l - m] = 0.0;
  return legendre_walk(m, theta, lmax, eps, [&](int l, double v) {
    out[l - m] = v;
    return true;
  });
}

// Recurrence coefficients of the even/odd (step-2) three-term recurrence
//   P_k = (x^2 + alpha_k) beta_k P_{k-1} + gamma_k P_{k-2},  l_k = lmin + 2k
// with c_l = sqrt((l-m+1)(l-m+2)(l+m+1)(l+m+2) / ((2l+1)(2l+3)^2(2l+5))),
//      d_l = (2l(l+1) - 2m^2 - 1) / ((2l-1)(2l+3)),
//      alpha_k = -d_{l_k-2}, beta_k = 1/c_{l_k-2}, gamma_k = -c_{l_k-4}/c_{l_k-2}
// (src/legendre_transform.c.in:723-747).
WM_HD double rec_c(int64_t l, int64_t m) {
  double num = (double)((l - m + 1) * (l - m + 2) * (l + m + 1) * (l + m + 2));
  double den = (double)((2 * l + 1) * (2 * l + 3) * (2 * l + 3) * (2 * l + 5));
  return sqrt(num / den);
}
WM_HD double rec_d(int64_t l, int64_t m) {
  return (double)(2 * l * (l + 1) - 2 * m * m - 1) / (double)((2 * l - 1) * (2 * l + 3));
}
WM_HD void rec_abg(int64_t m, int64_t lmin, int64_t k, double *alpha, double *beta,
                   double *gamma) {
  int64_t l1 = lmin + 2 * (k - 1), l2 = lmin + 2 * (k - 2);
  double c1 = rec_c(l1, m);
  *alpha = -rec_d(l1, m);
  *beta = 1.0 / c1;
  *gamma = -rec_c(l2, m) / c1;
}

}  // namespace wm
