/*
 * pair_bound.h -- CPU restatement of the library's analytic screening bound
 * (test infrastructure: the oracle's and the reference arm's copy; the product
 * computes the same bound on the device).
 *
 * For a primitive pair (exponents x0, x1 on centres A, B, zeta = x0 + x1, P the
 * product centre, rho = |r - P|) every Cartesian component of the product is
 * bounded pointwise by K (rho + |PA|)^l0 (rho + |PB|)^l1 exp(-zeta rho^2) with
 * K = |c0 c1| exp(-x0 x1 |AB|^2 / zeta).  The Coulomb norm is monotone for
 * positive functions and subadditive, and ||rho^n exp(-zeta rho^2)|| =
 * N_n zeta^-(2n+5)/4 (N_n^2 the Coulomb self-energy of r^n exp(-r^2)), so
 *   Q_prim = K sum_n N_n zeta^-(2n+5)/4 [t^n] (|PA| + t)^l0 (|PB| + t)^l1,
 * times the spherical transform's largest coefficient sum per shell.  A
 * contracted pair sums Q_prim over its primitive pairs (triangle inequality),
 * and |(ab|cd)| <= Q_ab Q_cd element by element (Cauchy-Schwarz in the Coulomb
 * metric).  Each stage is widened by a factor 1 + 1e-6 for its own rounding,
 * as the device code does.  The reference has no screening; this bound is the
 * library's.
 */
#ifndef ORACLE_PAIR_BOUND_H
#define ORACLE_PAIR_BOUND_H
#include <math.h>

static const double pb_rn_norm[13] = {4.9738746919472297, 5.1652368552576019, 6.4612527577002005,
                                      9.2648431767816622, 14.794795287711256, 25.818805439099522,
                                      48.591021989124202, 97.655519373091779, 208.00183355514711,
                                      466.71786414003641, 1097.8288726985819, 2696.1716819638506,
                                      6889.8632213814936};
static const double pb_sph_colsum[7] = {1.0, 1.0, 2.0, 4.0, 8.9442719099991597, 20.493901531919201,
                                        47.096974425115671};

/* Coulomb-norm bound of the contracted pair (shells s0, s1). */
static double pb_pair(int l0, int l1, int k0, int k1, const double *x0, const double *c0, const double *x1,
                      const double *c1, const double *A, const double *B, int spherical) {
  if (l0 < 0 || l0 > 6 || l1 < 0 || l1 > 6) return INFINITY;
  const double r2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  const double R = sqrt(r2);
  const double f = spherical ? pb_sph_colsum[l0] * pb_sph_colsum[l1] : 1.0;
  double Q = 0.0;
  for (int i = 0; i < k0; ++i)
    for (int j = 0; j < k1; ++j) {
      const double z = x0[i] + x1[j];
      const double K = fabs(c0[i] * c1[j]) * exp(-x0[i] * x1[j] / z * r2);
      if (K == 0.0) continue;
      const double pa = x1[j] / z * R, pbv = x0[i] / z * R;
      double c[13] = {1.0};
      int deg = 0;
      for (int r = 0; r < l0 + l1; ++r) {
        const double p = r < l0 ? pa : pbv;
        c[deg + 1] = c[deg];
        for (int n = deg; n > 0; --n) c[n] = c[n] * p + c[n - 1];
        c[0] *= p;
        ++deg;
      }
      const double s = 1.0 / sqrt(z);
      double poly = 0.0, sn = 1.0;
      for (int n = 0; n <= deg; ++n) {
        poly += c[n] * pb_rn_norm[n] * sn;
        sn *= s;
      }
      Q += 1.000001 * f * K * s * s * sqrt(s) * poly;
    }
  return Q * 1.000001;
}

/* bound of quartet (s[0] s[1] | s[2] s[3]) */
static double pb_quartet(const int *s, const int *shell_l, const int *shell_k, const int *shell_ptr,
                         const double *shell_xyz, const double *prim_exp, const double *prim_coef, int spherical) {
  double q[2];
  for (int side = 0; side < 2; ++side) {
    const int a = s[2 * side], b = s[2 * side + 1];
    q[side] = pb_pair(shell_l[a], shell_l[b], shell_k[a], shell_k[b], prim_exp + shell_ptr[a],
                      prim_coef + shell_ptr[a], prim_exp + shell_ptr[b], prim_coef + shell_ptr[b],
                      shell_xyz + 3 * a, shell_xyz + 3 * b, spherical);
  }
  return q[0] * q[1] * 1.000001;
}
#endif
