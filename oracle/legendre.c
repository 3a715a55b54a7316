/*
 * ORACLE (test infrastructure only; never linked into the product).
 *
 * CPU restatement, in plain C, of the scalar pieces of the reference's
 * Legendre machinery.  Each function cites the reference code it follows.
 * Compiled with -ffp-contract=off so that every product/sum is rounded
 * separately, as in the reference's SSE2 build (no FMA contraction).
 *
 *  - or_normalized_legendre: normalised associated Legendre values
 *      lambda_lm(theta) for one m and many thetas, following libpsht's
 *      Ylmgen (libpshtlight/ylmgen_c.c:419-504 init, :548-585 set_theta,
 *      :604-619 recurrence factors, :643-732 Ylmgen_recalc_Ylm) as driven by
 *      wavemoth/legendre.pyx:24-57 (one generator per call, thetas in order,
 *      so the "all below epsilon" shortcut state m_crit/cth_crit carries over
 *      from one theta to the next exactly as in the reference).
 *  - or_legendre_auxdata: the (alpha, beta, gamma) coefficients of the
 *      even/odd three-term recurrence (src/legendre_transform.c.in:723-747).
 *  - or_legendre_transform: the scalar residual-strip transform
 *      y = P^T a (src/legendre_transform.c.in:680-716).
 *  - or_legendre_transform_T: its adjoint a += P y, the analysis direction
 *      (wavemoth/cuda/legendre_transform.cu.in:643-679 computes this for
 *      dense Lambda).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define OR_BIG_EXP2 90   /* rescaling step, 2^90 (ylmgen_c.c:37) */
#define OR_MINSCALE (-4)
#define OR_MAXSCALE 11

int or_normalized_legendre(int m, const double *theta_in, int ntheta, int lmax,
                           double eps, double *out /* ntheta x (lmax-m+1) */) {
  const double ln2 = 0.6931471805599453094172321214581766;
  const double inv_ln2 = 1.4426950408889634073599246810018921;
  const double inv_sqrt4pi = 0.2820947917738781434740397257803862929220;
  const double pi = 3.141592653589793238462643383279502884197;
  int nl = lmax - m + 1;
  if (m < 0 || lmax < m || ntheta < 0) return -1;

  /* scale table: cf[s] = 2^((s + minscale) * 90) */
  double cf[OR_MAXSCALE - OR_MINSCALE + 1];
  for (int s = 0; s <= OR_MAXSCALE - OR_MINSCALE; ++s)
    cf[s] = ldexp(1.0, (s + OR_MINSCALE) * OR_BIG_EXP2);
  const double fsmall = ldexp(1.0, -OR_BIG_EXP2), fbig = ldexp(1.0, OR_BIG_EXP2);

  /* log2 of the P_mm prefactor sqrt(1/4pi) * prod_k sqrt((2k+1)/2k) */
  double mfac_lin = 1.0;
  for (int k = 1; k <= m; ++k) mfac_lin = mfac_lin * sqrt((2 * k + 1.) / (2 * k));
  double log2_pmm = inv_ln2 * log(inv_sqrt4pi * mfac_lin);

  /* two-term recurrence factors in l (step 1) */
  double *rf0 = malloc(sizeof(double) * (lmax + 1));
  double *rf1 = malloc(sizeof(double) * (lmax + 1));
  if (!rf0 || !rf1) { free(rf0); free(rf1); return -2; }
  double f_old = 1.0;
  for (int l = m; l <= lmax; ++l) {
    double t1 = sqrt(4. * (l + 1) * (l + 1) - 1.);
    double t2a = 1. / sqrt((l + m) + 1.);
    double t2b = 1. / sqrt((l - m) + 1.);
    rf0[l] = t1 * t2a * t2b;
    rf1[l] = rf0[l] / f_old;
    f_old = rf0[l];
  }

  int m_crit = lmax + 1;       /* Ylmgen_init: m_crit = mmax + 1 with mmax = lmax */
  double cth_crit = 2.0;

  for (int it = 0; it < ntheta; ++it) {
    double *row = out + (size_t)it * nl;
    double th = theta_in[it];
    if (!(th >= 0. && th <= pi)) { free(rf0); free(rf1); return -3; }
    if (th == 0.) th = 1e-16;
    if (fabs(th - pi) < 1e-15) th = pi - 1e-15;
    double cth = cos(th), sth = sin(th);
    double logsth = inv_ln2 * log(sth);

    int firstl;
    if ((m >= m_crit && fabs(cth) >= cth_crit) || (m > 0 && sth == 0)) {
      firstl = lmax + 1;
    } else {
      double logval = log2_pmm;
      if (m > 0) logval += m * logsth;
      int scale = (int)(logval / OR_BIG_EXP2) - OR_MINSCALE;
      double corfac = (scale < 0) ? 0. : cf[scale];
      double lam_1 = 0;
      double lam_2 = exp(ln2 * (logval - (scale + OR_MINSCALE) * OR_BIG_EXP2));
      if (m & 1) lam_2 = -lam_2;
      int l = m;
      if (scale < 0) {
        for (;;) {
          if (++l > lmax) break;
          lam_1 = cth * lam_2 * rf0[l - 1] - lam_1 * rf1[l - 1];
          if (++l > lmax) break;
          lam_2 = cth * lam_1 * rf0[l - 1] - lam_2 * rf1[l - 1];
          if (fabs(lam_2) > fbig) {
            while (fabs(lam_2) > fbig) { lam_1 *= fsmall; lam_2 *= fsmall; ++scale; }
            corfac = (scale < 0) ? 0. : cf[scale];
            if (scale >= 0) break;
          }
        }
      }
      lam_1 *= corfac;
      lam_2 *= corfac;
      if (l <= lmax) {
        for (;;) {
          if (fabs(lam_2) > eps) break;
          if (++l > lmax) break;
          lam_1 = cth * lam_2 * rf0[l - 1] - lam_1 * rf1[l - 1];
          if (fabs(lam_1) > eps) { double t = lam_1; lam_1 = lam_2; lam_2 = t; break; }
          if (++l > lmax) break;
          lam_2 = cth * lam_1 * rf0[l - 1] - lam_2 * rf1[l - 1];
        }
      }
      firstl = l;
      if (l > lmax) {
        m_crit = m;
        cth_crit = fabs(cth);
      } else {
        for (;;) {
          row[l - m] = lam_2;
          if (++l > lmax) break;
          lam_1 = cth * lam_2 * rf0[l - 1] - lam_1 * rf1[l - 1];
          row[l - m] = lam_1;
          if (++l > lmax) break;
          lam_2 = cth * lam_1 * rf0[l - 1] - lam_2 * rf1[l - 1];
        }
      }
    }
    int zstop = firstl < lmax + 1 ? firstl : lmax + 1;
    for (int l = m; l < zstop; ++l) row[l - m] = 0.0;
  }
  free(rf0);
  free(rf1);
  return 0;
}

/* (alpha, beta, gamma) for rows k >= 2 of the step-2 recurrence starting at
   l = lmin; 3*(nk-2) values. */
void or_legendre_auxdata(int64_t m, int64_t lmin, int64_t nk, double *aux) {
  double cp = 0, cpp = 0, dp = 0;
  for (int64_t k = 0, l = lmin; k < nk; ++k, l += 2) {
    double cnum = (double)((l - m + 1) * (l - m + 2) * (l + m + 1) * (l + m + 2));
    double cden = (double)((2 * l + 1) * (2 * l + 3) * (2 * l + 3) * (2 * l + 5));
    double c = sqrt(cnum / cden);
    double d = (double)(2 * l * (l + 1) - 2 * m * m - 1) / (double)((2 * l - 1) * (2 * l + 3));
    if (k >= 2) {
      aux[3 * (k - 2) + 0] = -dp;
      aux[3 * (k - 2) + 1] = 1 / cp;
      aux[3 * (k - 2) + 2] = -cpp / cp;
    }
    dp = d;
    cpp = cp;
    cp = c;
  }
}

/* y[i, j] = sum_k P_k(x_i) a[k*a_stride + j]; P_0 = P0[i], P_1 = P1[i],
   P_k = (x_i^2 + alpha_k) beta_k P_{k-1} + gamma_k P_{k-2}. */
void or_legendre_transform(int64_t nx, int64_t nk, int64_t nvecs, const double *a,
                           int64_t a_stride, double *y, const double *x2,
                           const double *aux, const double *P0, const double *P1) {
  for (int64_t i = 0; i < nx; ++i) {
    double pp = P0[i], p = P1[i];
    for (int64_t j = 0; j < nvecs; ++j) y[i * nvecs + j] = pp * a[j];
    if (nk > 1)
      for (int64_t j = 0; j < nvecs; ++j) y[i * nvecs + j] += p * a[a_stride + j];
    for (int64_t k = 2; k < nk; ++k) {
      const double *ak = aux + 3 * (k - 2);
      double v = (x2[i] + ak[0]) * ak[1] * p + ak[2] * pp;
      pp = p;
      p = v;
      for (int64_t j = 0; j < nvecs; ++j) y[i * nvecs + j] += v * a[k * a_stride + j];
    }
  }
}

/* Adjoint of or_legendre_transform: a[k*a_stride + j] += sum_i P_k(x_i) y[i, j]. */
void or_legendre_transform_T(int64_t nx, int64_t nk, int64_t nvecs, double *a,
                             int64_t a_stride, const double *y, const double *x2,
                             const double *aux, const double *P0, const double *P1) {
  for (int64_t i = 0; i < nx; ++i) {
    double pp = P0[i], p = P1[i];
    for (int64_t j = 0; j < nvecs; ++j) a[j] += pp * y[i * nvecs + j];
    if (nk > 1)
      for (int64_t j = 0; j < nvecs; ++j) a[a_stride + j] += p * y[i * nvecs + j];
    for (int64_t k = 2; k < nk; ++k) {
      const double *ak = aux + 3 * (k - 2);
      double v = (x2[i] + ak[0]) * ak[1] * p + ak[2] * pp;
      pp = p;
      p = v;
      for (int64_t j = 0; j < nvecs; ++j) a[k * a_stride + j] += v * y[i * nvecs + j];
    }
  }
}
