/*
 * eri_oracle.c -- CPU restatement of the reference's contracted-ERI path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke check
 * and bench.py's cpu_baseline leg may call it; the product (intception_b200)
 * never links or calls it.
 *
 * It restates, in plain C, what the C99 emitted by the reference generator for
 * the ERI input script (oracle/eri_input.py) computes, function by function:
 *   oracle_boys ........ generator/callables/generator_boys_function.py:98-205
 *   base [00|00]^(m) ... generator/callables/integral_wrapper_base_function.py:84-162
 *   VRR a, c, d ........ generator/callables/main_source_algorithms/contracted_general.py:720-1082
 *                        (recurrence terms: the input script's vrra/vrrc/vrrd)
 *   contraction ........ generator/callables/generator_contract_function.py:69-125,
 *                        driven by contracted_general.py:1083-1417 (a truncated to
 *                        [la, la+lb], c and d to exactly lc and ld)
 *   HRR a -> b ......... generator/callables/generator_hrr_function.py:265-436,
 *                        driver contracted_general.py:1574-1807; the HGP form of
 *                        dsl_extensions.py:903-950, (a,b+1i) = (a+1i,b) + AB_i (a,b)
 *   sph transform ...... generator/callables/generator_sph_trans_function.py:69-125
 *                        out[pre + isph*n_pre] = sum_cart in[pre + cart*skip] T[cart + isph*ncart]
 *   output copy ........ contracted_general.py:1808-1876 (caller strides)
 *   work-array size .... contracted_general.py:240-502 (integer formula, bit-exact)
 *
 * Component order inside one angular-momentum level: x-descending, then
 * y-descending (dsl.py:988-1001); index within the level
 * mz + (my+mz)(my+mz+1)/2, cumulative offset (l)(l+1)(l+2)/6 (dsl.py:1029-1041).
 *
 * The Boys tables are regenerated with mpmath by oracle/gen_boys_tables.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "boys_tables.h"
#include "pair_bound.h"

/* Arithmetic of the recurrences, contraction, HRR and transform: double (the
 * default, the restatement proper), or with -DORACLE_QUAD binary128 with an
 * accurate binary128 Boys function (oracle/_gen/liberi_oracle_quad.so): an
 * exact evaluation of the same integrals for quartets on which every double
 * scheme loses digits (contractions that mix tight and diffuse exponents). */
#ifdef ORACLE_QUAD
#include <quadmath.h>
typedef __float128 oreal;
#define OR_EXP expq
#define OR_SQRT sqrtq
#define OR_POW powq
#define OR_PI M_PIq
#else
typedef double oreal;
#define OR_EXP exp
#define OR_SQRT sqrt
#define OR_POW pow
#define OR_PI 3.14159265358979323846
#endif

#define OR_LMAX 8

static const double oracle_oof[7] = {1.0, 1.0, 1.0 / 2.0, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0};

static int nc_l(int l) { return (l + 1) * (l + 2) / 2; }
static int ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }
static int cidx(int mx, int my, int mz) {
  int l = mx + my + mz;
  return ncum(l - 1) + mz + (my + mz) * (my + mz + 1) / 2;
}

/* Cartesian exponents of every cumulative component index up to OR_LMAX*2 */
#define OR_NCUM_MAX 1771 /* ncum(20) */
static int comp_tab[OR_NCUM_MAX][3];
static int comp_tab_ready = 0;
static void init_comp_tab(void) {
  if (comp_tab_ready) return;
  int n = 0;
  for (int l = 0; l <= 20; ++l)
    for (int mx = l; mx >= 0; --mx)
      for (int my = l - mx; my >= 0; --my) {
        comp_tab[n][0] = mx;
        comp_tab[n][1] = my;
        comp_tab[n][2] = l - mx - my;
        ++n;
      }
  comp_tab_ready = 1;
}

/* Off (the default): the reference's Boys function below.  On: an accurate
 * one, for checking the recurrences apart from the reference's Boys error.
 * The reference's 7-term Taylor steps on a 0.1 grid truncate at about 1e-13
 * relative (2.7e-14 measured at m = 0 against 30-digit mpmath values) and its
 * x >= 35 branch drops exp(-x) (3.8e-6 relative at m = 12, x = 35); the VRR's
 * cancellations carry such errors into the f-shell classes' integrals at up to
 * 1e-9 relative.  Accurate mode: below x = 50 the series
 *   F_n(x) = exp(-x) sum_k (2x)^k / ((2n+1)(2n+3)...(2n+2k+1))
 * (positive terms, summed until they stop changing the sum) for F_nmax, then
 * downward recursion; from x = 50 the asymptotic F_0 and the exact upward
 * recursion F_{m+1} = ((m+1/2) F_m - exp(-x)/2) / x. */
static int oracle_boys_exact_mode = 0;
void oracle_set_boys_exact(int on) { oracle_boys_exact_mode = on; }

static void oracle_boys_accurate(double *f, int ifskip, int nmin, int nmax, double x) {
  double ex = exp(-x);
  if (x < 50.0) {
    double term = 1.0 / (2.0 * nmax + 1.0), sum = term;
    for (int k = 1; k < 2000; ++k) {
      term *= 2.0 * x / (2.0 * nmax + 2.0 * k + 1.0);
      double next = sum + term;
      if (next == sum) break;
      sum = next;
    }
    f[nmax * ifskip] = ex * sum;
    for (int m = nmax - 1; m >= nmin; --m)
      f[m * ifskip] = (2.0 * x * f[(m + 1) * ifskip] + ex) / (2.0 * m + 1.0);
  } else {
    double oox = 1.0 / x, g = 0.5 * sqrt(3.141592653589793 * oox);
    for (int m = 0; m <= nmax; ++m) {
      if (m >= nmin) f[m * ifskip] = g;
      g = ((double)m + 0.5) * oox * g - 0.5 * ex * oox;
    }
  }
}

/* generator_boys_function.py:98-205: small x (<=15) 7-term Taylor about the
 * nearest 0.1 grid point then downward recursion; 15<x<35 F_0 Taylor then upward
 * recursion; x>=35 asymptotic F_0 and upward recursion without exp(-x). */
void oracle_boys(double *f, int ifskip, int nmin, int nmax, double x) {
  if (oracle_boys_exact_mode) {
    oracle_boys_accurate(f, ifskip, nmin, nmax, x);
    return;
  }
  if (x <= 15.0) {
    int i = (int)round(x * 10.0);
    double dx = (double)i * 0.1 - x;
    double xn = 1.0;
    f[nmax * ifskip] = oracle_boys_smallx[i][nmax];
    for (int k = 1; k < 7; ++k) {
      xn *= dx;
      f[nmax * ifskip] += oracle_boys_smallx[i][nmax + k] * xn * oracle_oof[k];
    }
    double ex = exp(-x);
    for (int m = nmax - 1; m >= nmin; --m)
      f[m * ifskip] = (2.0 * x * f[(m + 1) * ifskip] + ex) / (2.0 * (double)m + 1.0);
  } else if (x < 35.0) {
    int i = (int)round(x * 10.0);
    double dx = (double)i * 0.1 - x;
    i -= 150;
    double oox = 1.0 / x, xn = 1.0;
    f[0] = oracle_boys_mediumx[i][0];
    for (int k = 1; k < 7; ++k) {
      xn *= dx;
      f[0] += oracle_boys_mediumx[i][k] * xn * oracle_oof[k];
    }
    double ex = exp(-x);
    for (int m = 0; m < nmax; ++m)
      f[(m + 1) * ifskip] = ((double)m + 0.5) * oox * f[m * ifskip] - ex * 0.5 * oox;
  } else {
    double oox = 1.0 / x;
    f[0] = 0.5 * sqrt(3.141592653589793 * oox);
    for (int m = 0; m < nmax; ++m)
      f[(m + 1) * ifskip] = ((double)m + 0.5) * oox * f[m * ifskip];
  }
}

/* contracted_general.py:240-502 (emitted as <class>_work_array_size) */
static int hrr_layer_size(int lb, int la) {
  /* generator.py:1112-1157: the largest HRR layer, max over l_b' = 0..lb of
   * ncart-sum of the a range [la, la+lb-lb'] times ncart(lb') */
  int best = 0;
  for (int j = 0; j <= lb; ++j) {
    int na = ncum(la + lb - j) - ncum(la - 1);
    int v = na * nc_l(j);
    if (v > best) best = v;
  }
  return best;
}

int oracle_eri_work_array_size(int la, int lb, int lc, int ld, int na_prim, int nb_prim, int nc_prim,
                               int nd_prim, int na_cont, int nb_cont, int nc_cont, int nd_cont) {
  int nw = ncum(la + lb) * ncum(lc) * ncum(ld);
  int n1 = na_prim * nb_prim * nd_prim * nc_prim;
  int mem1 = 2 * (nw * n1 + ld + lc + la + lb + 1);
  int n2 = na_cont * nb_prim * nd_prim * nc_prim;
  if (n1 < n2) n1 = n2;
  n2 = na_cont * nb_cont * nd_prim * nc_prim;
  if (n1 < n2) n1 = n2;
  n2 = na_cont * nb_cont * nd_cont * nc_prim;
  if (n1 < n2) n1 = n2;
  n2 = na_cont * nb_cont * nd_cont * nc_cont;
  if (n1 < n2) n1 = n2;
  int mem2 = 2 * nw * n1;
  if (mem2 > mem1) mem1 = mem2;
  n1 = na_cont * nb_cont * nd_cont * nc_cont;
  mem2 = 2 * hrr_layer_size(lb, la) * nc_l(lc) * nc_l(ld) * n1;
  if (mem2 > mem1) mem1 = mem2;
  mem2 = 2 * nc_l(lc) * nc_l(ld) * nc_l(lb) * nc_l(la) * n1;
  if (mem2 > mem1) mem1 = mem2;
  return mem1;
}

/* F_0..F_nmax(x) in the recurrences' arithmetic: the reference's Boys function
 * for double; for binary128 the series below x = 60 (positive terms, downward
 * recursion) and erf-based F_0 with upward recursion from there. */
#ifdef ORACLE_QUAD
static void oracle_boys_real(oreal *f, int nmax, oreal x) {
  oreal ex = expq(-x);
  if (x < 60) {
    oreal term = 1 / (oreal)(2 * nmax + 1), sum = term;
    for (int k = 1; k < 100000; ++k) {
      term *= 2 * x / (oreal)(2 * nmax + 2 * k + 1);
      oreal next = sum + term;
      if (next == sum) break;
      sum = next;
    }
    f[nmax] = ex * sum;
    for (int m = nmax - 1; m >= 0; --m) f[m] = (2 * x * f[m + 1] + ex) / (oreal)(2 * m + 1);
  } else {
    oreal g = 0.5Q * sqrtq(M_PIq / x) * erfq(sqrtq(x));
    for (int m = 0; m <= nmax; ++m) {
      f[m] = g;
      g = ((oreal)m + 0.5Q) / x * g - 0.5Q * ex / x;
    }
  }
}
#else
static void oracle_boys_real(oreal *f, int nmax, oreal x) { oracle_boys(f, 1, 0, nmax, x); }
#endif

/* One primitive quartet: V[m][a][c][d] over cumulative component indices, with
 * a <= la+lb, c <= lc, d <= ld and m + |a| + |c| + |d| <= L.  Recurrences are the
 * input script's vrra / vrrc / vrrd (Obara-Saika with the auxiliary index m). */
typedef struct {
  int L, na, nc, nd; /* cumulative counts */
  oreal *v;
} vtab;
#define V(t, m, a, c, d) ((t)->v[(((size_t)(m) * (t)->na + (a)) * (t)->nc + (c)) * (t)->nd + (d)])

static int first_dir(const int *e) { return e[0] > 0 ? 0 : (e[1] > 0 ? 1 : 2); }

static void prim_vrr(vtab *t, int lab, int lc, int ld, const oreal *base, const oreal PA[3],
                     const oreal WP[3], const oreal QC[3], const oreal QD[3], const oreal WQ[3],
                     oreal o2z, oreal roz, oreal o2e, oreal roe, oreal o2zpe) {
  int L = t->L;
  for (int m = 0; m <= L; ++m) V(t, m, 0, 0, 0) = base[m];
  /* vrra: [a+1i| = PA_i [a| + WP_i [a|^(m+1) + a_i/(2zeta) ([a-1i| - rho/zeta [a-1i|^(m+1)) */
  for (int ia = 1; ia < ncum(lab); ++ia) {
    const int *e = comp_tab[ia];
    int la_ = e[0] + e[1] + e[2];
    int i = first_dir(e);
    int em[3] = {e[0], e[1], e[2]};
    em[i] -= 1;
    int a1 = cidx(em[0], em[1], em[2]);
    int n2 = em[i];
    int a2 = -1;
    if (n2 > 0) {
      int e2[3] = {em[0], em[1], em[2]};
      e2[i] -= 1;
      a2 = cidx(e2[0], e2[1], e2[2]);
    }
    for (int m = 0; m + la_ <= L; ++m) {
      oreal v = PA[i] * V(t, m, a1, 0, 0) + WP[i] * V(t, m + 1, a1, 0, 0);
      if (a2 >= 0) v += o2z * n2 * (V(t, m, a2, 0, 0) - roz * V(t, m + 1, a2, 0, 0));
      V(t, m, ia, 0, 0) = v;
    }
  }
  /* vrrc: [a|c+1i] = QC_i [a|c] + WQ_i [a|c]^(m+1) + c_i/(2eta)([a|c-1i] - rho/eta [..]^(m+1))
   *                  + a_i/(2(zeta+eta)) [a-1i|c]^(m+1) */
  for (int ic = 1; ic < ncum(lc); ++ic) {
    const int *f = comp_tab[ic];
    int lf = f[0] + f[1] + f[2];
    int i = first_dir(f);
    int fm[3] = {f[0], f[1], f[2]};
    fm[i] -= 1;
    int c1 = cidx(fm[0], fm[1], fm[2]);
    int n2 = fm[i];
    int c2 = -1;
    if (n2 > 0) {
      int f2[3] = {fm[0], fm[1], fm[2]};
      f2[i] -= 1;
      c2 = cidx(f2[0], f2[1], f2[2]);
    }
    for (int ia = 0; ia < ncum(lab); ++ia) {
      const int *e = comp_tab[ia];
      int le = e[0] + e[1] + e[2];
      int na_i = e[i], a1 = -1;
      if (na_i > 0) {
        int em[3] = {e[0], e[1], e[2]};
        em[i] -= 1;
        a1 = cidx(em[0], em[1], em[2]);
      }
      for (int m = 0; m + le + lf <= L; ++m) {
        oreal v = QC[i] * V(t, m, ia, c1, 0) + WQ[i] * V(t, m + 1, ia, c1, 0);
        if (c2 >= 0) v += o2e * n2 * (V(t, m, ia, c2, 0) - roe * V(t, m + 1, ia, c2, 0));
        if (a1 >= 0) v += o2zpe * na_i * V(t, m + 1, a1, c1, 0);
        V(t, m, ia, ic, 0) = v;
      }
    }
  }
  /* vrrd: [a|c,d+1i] = QD_i [..] + WQ_i [..]^(m+1) + d_i/(2eta)([..d-1i] - rho/eta [..]^(m+1))
   *        + c_i/(2eta)([a|c-1i,d] - rho/eta [..]^(m+1)) + a_i/(2(zeta+eta)) [a-1i|c,d]^(m+1) */
  for (int id = 1; id < ncum(ld); ++id) {
    const int *g = comp_tab[id];
    int lg = g[0] + g[1] + g[2];
    int i = first_dir(g);
    int gm[3] = {g[0], g[1], g[2]};
    gm[i] -= 1;
    int d1 = cidx(gm[0], gm[1], gm[2]);
    int n2 = gm[i];
    int d2 = -1;
    if (n2 > 0) {
      int g2[3] = {gm[0], gm[1], gm[2]};
      g2[i] -= 1;
      d2 = cidx(g2[0], g2[1], g2[2]);
    }
    for (int ia = 0; ia < ncum(lab); ++ia) {
      const int *e = comp_tab[ia];
      int le = e[0] + e[1] + e[2];
      int na_i = e[i], a1 = -1;
      if (na_i > 0) {
        int em[3] = {e[0], e[1], e[2]};
        em[i] -= 1;
        a1 = cidx(em[0], em[1], em[2]);
      }
      for (int ic = 0; ic < ncum(lc); ++ic) {
        const int *f = comp_tab[ic];
        int lf = f[0] + f[1] + f[2];
        int nc_i = f[i], c1 = -1;
        if (nc_i > 0) {
          int fm[3] = {f[0], f[1], f[2]};
          fm[i] -= 1;
          c1 = cidx(fm[0], fm[1], fm[2]);
        }
        for (int m = 0; m + le + lf + lg <= L; ++m) {
          oreal v = QD[i] * V(t, m, ia, ic, d1) + WQ[i] * V(t, m + 1, ia, ic, d1);
          if (d2 >= 0) v += o2e * n2 * (V(t, m, ia, ic, d2) - roe * V(t, m + 1, ia, ic, d2));
          if (c1 >= 0) v += o2e * nc_i * (V(t, m, ia, c1, d1) - roe * V(t, m + 1, ia, c1, d1));
          if (a1 >= 0) v += o2zpe * na_i * V(t, m + 1, a1, ic, d1);
          V(t, m, ia, ic, id) = v;
        }
      }
    }
  }
}

/* Full contracted quartet.  T* are the caller's Cartesian->spherical matrices
 * (T[icart + isph*ncart]) or NULL for Cartesian output. */
static void oracle_eri_cont(const double *xa, const double *cA, int la, int na, int iskipa, int na_prim,
                            int na_cont, int iskipa_cont, const double *ca, const double *Ta,
                            const double *xb, const double *cB, int lb, int nb, int iskipb, int nb_prim,
                            int nb_cont, int iskipb_cont, const double *cb, const double *Tb,
                            const double *xc, const double *cC, int lc, int nc, int iskipc, int nc_prim,
                            int nc_cont, int iskipc_cont, const double *cc, const double *Tc,
                            const double *xd, const double *cD, int ld, int nd, int iskipd, int nd_prim,
                            int nd_cont, int iskipd_cont, const double *cd, const double *Td,
                            double *out) {
  init_comp_tab();
  const oreal two_pi52 = 2.0 * OR_POW(OR_PI, 2.5);
  int lab = la + lb, L = la + lb + lc + ld;
  int ne = ncum(lab) - ncum(la - 1); /* a range [la, la+lb] */
  int e0 = ncum(la - 1);
  int ncc = nc_l(lc), ncd = nc_l(ld);
  int c0 = ncum(lc - 1), d0 = ncum(ld - 1);
  int ncont = na_cont * nb_cont * nc_cont * nd_cont;
  /* contracted [e0|cd]: index ((((ka*nbk+kb)*nck+kc)*ndk+kd)*ne + e)*ncc + c)*ncd + d */
  size_t nblk = (size_t)ne * ncc * ncd;
  oreal *acc = calloc(nblk * ncont, sizeof(oreal));
  vtab t;
  t.L = L;
  t.na = ncum(lab);
  t.nc = ncum(lc);
  t.nd = ncum(ld);
  t.v = calloc((size_t)(L + 1) * t.na * t.nc * t.nd, sizeof(oreal));
  oreal F[4 * OR_LMAX + 1];
  oreal AB[3], CD[3];
  for (int i = 0; i < 3; ++i) {
    AB[i] = (oreal)cA[i] - cB[i];
    CD[i] = (oreal)cC[i] - cD[i];
  }
  oreal RAB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  oreal RCD2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
  for (int pc = 0; pc < nc_prim; ++pc)
    for (int pd = 0; pd < nd_prim; ++pd) {
      oreal eta = (oreal)xc[pc] + xd[pd], oeta = 1.0 / eta;
      oreal Q[3], QC[3], QD[3];
      for (int i = 0; i < 3; ++i) {
        Q[i] = ((oreal)xc[pc] * cC[i] + (oreal)xd[pd] * cD[i]) * oeta;
        QC[i] = Q[i] - cC[i];
        QD[i] = Q[i] - cD[i];
      }
      oreal xi_cd = (oreal)xc[pc] * xd[pd] * oeta;
      for (int pb = 0; pb < nb_prim; ++pb)
        for (int pa = 0; pa < na_prim; ++pa) {
          oreal zeta = (oreal)xa[pa] + xb[pb], ozeta = 1.0 / zeta;
          oreal P[3], PA[3], W[3], WP[3], WQ[3], PQ[3];
          for (int i = 0; i < 3; ++i) {
            P[i] = ((oreal)xa[pa] * cA[i] + (oreal)xb[pb] * cB[i]) * ozeta;
            PA[i] = P[i] - cA[i];
          }
          oreal xi_ab = (oreal)xa[pa] * xb[pb] * ozeta;
          oreal ozpe = 1.0 / (zeta + eta);
          oreal rho = zeta * eta * ozpe;
          for (int i = 0; i < 3; ++i) {
            PQ[i] = P[i] - Q[i];
            W[i] = (zeta * P[i] + eta * Q[i]) * ozpe;
            WP[i] = W[i] - P[i];
            WQ[i] = W[i] - Q[i];
          }
          oreal RPQ2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
          /* base: 2 pi^{5/2} / (zeta eta sqrt(zeta+eta)) exp(-xi_ab RAB2 - xi_cd RCD2) F_m(rho RPQ2) */
          oracle_boys_real(F, L, rho * RPQ2);
          oreal pref = two_pi52 * ozeta * oeta * OR_SQRT(ozpe) * OR_EXP(-xi_ab * RAB2 - xi_cd * RCD2);
          for (int m = 0; m <= L; ++m) F[m] *= pref;
          prim_vrr(&t, lab, lc, ld, F, PA, WP, QC, QD, WQ, 0.5 * ozeta, rho * ozeta, 0.5 * oeta, rho * oeta,
                   0.5 * ozpe);
          for (int ka = 0; ka < na_cont; ++ka)
            for (int kb = 0; kb < nb_cont; ++kb)
              for (int kc = 0; kc < nc_cont; ++kc)
                for (int kd = 0; kd < nd_cont; ++kd) {
                  oreal w = (oreal)ca[pa + ka * na_prim] * cb[pb + kb * nb_prim] * cc[pc + kc * nc_prim] *
                             cd[pd + kd * nd_prim];
                  oreal *blk = acc + ((((size_t)ka * nb_cont + kb) * nc_cont + kc) * nd_cont + kd) * nblk;
                  for (int e = 0; e < ne; ++e)
                    for (int c = 0; c < ncc; ++c)
                      for (int d = 0; d < ncd; ++d)
                        blk[((size_t)e * ncc + c) * ncd + d] += w * V(&t, 0, e0 + e, c0 + c, d0 + d);
                }
        }
    }
  free(t.v);

  /* HRR a -> b on contracted data, layer by layer in l_b (generator_hrr_function.py:265-436):
   * direction = x if b_x>0, else y if b_y>0, else z. */
  int nca = nc_l(la), ncb = nc_l(lb);
  size_t nout_cart = (size_t)nca * ncb * ncc * ncd;
  oreal *cart = malloc(sizeof(oreal) * nout_cart * ncont); /* index (((a*ncb+b)*ncc+c)*ncd+d) */
  for (int k = 0; k < ncont; ++k) {
    const oreal *blk = acc + (size_t)k * nblk;
    /* layer j holds (e, b) for |b| = j, e in [la, la+lb-j] (cumulative index offset e0) */
    oreal *prev = malloc(sizeof(oreal) * nblk);
    memcpy(prev, blk, sizeof(oreal) * nblk);
    int prev_ne = ne;
    for (int j = 1; j <= lb; ++j) {
      int cur_ne = ncum(lab - j) - ncum(la - 1);
      int nbj = nc_l(j), nbp = nc_l(j - 1);
      size_t cur_sz = (size_t)cur_ne * nbj * ncc * ncd;
      oreal *cur = malloc(sizeof(oreal) * cur_sz);
      for (int ib = 0; ib < nbj; ++ib) {
        const int *bb = comp_tab[ncum(j - 1) + ib];
        int i = first_dir(bb);
        int bm[3] = {bb[0], bb[1], bb[2]};
        bm[i] -= 1;
        int ibm = cidx(bm[0], bm[1], bm[2]) - ncum(j - 2);
        for (int ie = 0; ie < cur_ne; ++ie) {
          const int *e = comp_tab[e0 + ie];
          int ep[3] = {e[0], e[1], e[2]};
          ep[i] += 1;
          int iep = cidx(ep[0], ep[1], ep[2]) - e0;
          for (int cdx = 0; cdx < ncc * ncd; ++cdx)
            cur[((size_t)ie * nbj + ib) * ncc * ncd + cdx] =
                prev[((size_t)iep * nbp + ibm) * ncc * ncd + cdx] +
                AB[i] * prev[((size_t)ie * nbp + ibm) * ncc * ncd + cdx];
        }
      }
      free(prev);
      prev = cur;
      prev_ne = cur_ne;
    }
    (void)prev_ne;
    /* prev now holds (a, b) with a in level la only (cur_ne == nca) */
    memcpy(cart + (size_t)k * nout_cart, prev, sizeof(oreal) * nout_cart);
    free(prev);
  }
  free(acc);

  /* spherical transform of each index with the caller's matrices, then output copy */
  /* the emitted copy loop runs over the caller's n? components (contracted_general.py:1808-1876) */
  int oa = na, ob = nb, oc = nc, od = nd;
  for (int ka = 0; ka < na_cont; ++ka)
    for (int kb = 0; kb < nb_cont; ++kb)
      for (int kc = 0; kc < nc_cont; ++kc)
        for (int kd = 0; kd < nd_cont; ++kd) {
          int k = ((ka * nb_cont + kb) * nc_cont + kc) * nd_cont + kd;
          const oreal *X = cart + (size_t)k * nout_cart;
          for (int sa = 0; sa < oa; ++sa)
            for (int sb = 0; sb < ob; ++sb)
              for (int sc = 0; sc < oc; ++sc)
                for (int sd = 0; sd < od; ++sd) {
                  oreal s = 0.0;
                  for (int a = 0; a < nca; ++a) {
                    oreal wa = Ta ? Ta[a + sa * nca] : (a == sa);
                    if (wa == 0.0) continue;
                    for (int b = 0; b < ncb; ++b) {
                      oreal wb = Tb ? Tb[b + sb * ncb] : (b == sb);
                      if (wb == 0.0) continue;
                      for (int c = 0; c < ncc; ++c) {
                        oreal wc = Tc ? Tc[c + sc * ncc] : (c == sc);
                        if (wc == 0.0) continue;
                        for (int d = 0; d < ncd; ++d) {
                          oreal wd = Td ? Td[d + sd * ncd] : (d == sd);
                          if (wd == 0.0) continue;
                          s += wa * wb * wc * wd * X[(((size_t)a * ncb + b) * ncc + c) * ncd + d];
                        }
                      }
                    }
                  }
                  out[(size_t)sa * iskipa + (size_t)ka * iskipa_cont + (size_t)sb * iskipb +
                      (size_t)kb * iskipb_cont + (size_t)sc * iskipc + (size_t)kc * iskipc_cont +
                      (size_t)sd * iskipd + (size_t)kd * iskipd_cont] = s;
                }
        }
  free(cart);
}

/* Same argument list as the emitted intception_integral_eri_abcd_m_cont_cart_main */
void oracle_eri_cont_cart_main(const double *xa, const double cA[3], int la, int na, int iskipa, int na_prim,
                               int na_cont, int iskipa_cont, const double *ca, const double *xb,
                               const double cB[3], int lb, int nb, int iskipb, int nb_prim, int nb_cont,
                               int iskipb_cont, const double *cb, const double *xc, const double cC[3], int lc,
                               int nc, int iskipc, int nc_prim, int nc_cont, int iskipc_cont, const double *cc,
                               const double *xd, const double cD[3], int ld, int nd, int iskipd, int nd_prim,
                               int nd_cont, int iskipd_cont, const double *cd, double *work, double *out) {
  (void)work;
  oracle_eri_cont(xa, cA, la, na, iskipa, na_prim, na_cont, iskipa_cont, ca, NULL, xb, cB, lb, nb, iskipb,
                  nb_prim, nb_cont, iskipb_cont, cb, NULL, xc, cC, lc, nc, iskipc, nc_prim, nc_cont,
                  iskipc_cont, cc, NULL, xd, cD, ld, nd, iskipd, nd_prim, nd_cont, iskipd_cont, cd, NULL, out);
}

/* Same argument list as the emitted intception_integral_eri_abcd_m_cont_sph_main */
void oracle_eri_cont_sph_main(const double *xa, const double cA[3], int la, int na, int iskipa, int na_prim,
                              int na_cont, int iskipa_cont, const double *ca, const double *Ta,
                              const double *xb, const double cB[3], int lb, int nb, int iskipb, int nb_prim,
                              int nb_cont, int iskipb_cont, const double *cb, const double *Tb,
                              const double *xc, const double cC[3], int lc, int nc, int iskipc, int nc_prim,
                              int nc_cont, int iskipc_cont, const double *cc, const double *Tc,
                              const double *xd, const double cD[3], int ld, int nd, int iskipd, int nd_prim,
                              int nd_cont, int iskipd_cont, const double *cd, const double *Td, double *work,
                              double *out) {
  (void)work;
  oracle_eri_cont(xa, cA, la, na, iskipa, na_prim, na_cont, iskipa_cont, ca, Ta, xb, cB, lb, nb, iskipb,
                  nb_prim, nb_cont, iskipb_cont, cb, Tb, xc, cC, lc, nc, iskipc, nc_prim, nc_cont, iskipc_cont,
                  cc, Tc, xd, cD, ld, nd, iskipd, nd_prim, nd_cont, iskipd_cont, cd, Td, out);
}

/* Batch driver over a shell table (segmented contraction, n_cont = 1).  Each
 * quartet's block is written at out + out_off[q] with a fastest:
 * index = ia + na*(ib + nb*(ic + nc*id)).  sphT[l] is the ncart x nsph matrix
 * for angular momentum l, or sphT == NULL for Cartesian output. */
void oracle_eri_batch(int nq, const int *quartets, const int *shell_l, const int *shell_k,
                      const int *shell_ptr, const double *shell_xyz, const double *prim_exp,
                      const double *prim_coef, const double *const *sphT, const long long *out_off,
                      double *out) {
  for (int q = 0; q < nq; ++q) {
    const int *s = quartets + 4 * q;
    int l[4], n[4];
    for (int i = 0; i < 4; ++i) {
      l[i] = shell_l[s[i]];
      n[i] = sphT ? 2 * l[i] + 1 : nc_l(l[i]);
    }
    int sk[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
    const double *T[4] = {NULL, NULL, NULL, NULL};
    if (sphT)
      for (int i = 0; i < 4; ++i) T[i] = sphT[l[i]];
    const double *x[4], *c[4], *r[4];
    for (int i = 0; i < 4; ++i) {
      x[i] = prim_exp + shell_ptr[s[i]];
      c[i] = prim_coef + shell_ptr[s[i]];
      r[i] = shell_xyz + 3 * s[i];
    }
    oracle_eri_cont(x[0], r[0], l[0], n[0], sk[0], shell_k[s[0]], 1, 0, c[0], T[0], x[1], r[1], l[1], n[1],
                    sk[1], shell_k[s[1]], 1, 0, c[1], T[1], x[2], r[2], l[2], n[2], sk[2], shell_k[s[2]], 1, 0,
                    c[2], T[2], x[3], r[3], l[3], n[3], sk[3], shell_k[s[3]], 1, 0, c[3], T[3],
                    out + out_off[q]);
  }
}

/* ---------------------------------------------------------------------------
 * Two-index classes of the reference's example script (examples/example_input.py:58-110),
 * primitive Cartesian: overlap_2idx (base sqrt(pi^3/p^3) exp(-xi R_AB^2), vrr1 on a,
 * vrr2 on b) and nuclear_2idx (base 2 pi/p exp(-xi R_AB^2) F_m(p R_PC^2), vrr1 on b,
 * vrr2 on a, both with the auxiliary m).  Tables over cumulative components.
 * ------------------------------------------------------------------------- */
static void oracle_2idx(int kind, double xa, const double *A, int la, int na, int iskipa, double xb,
                        const double *B, int lb, int nb, int iskipb, const double *Cn, double *out) {
  init_comp_tab();
  const double p = xa + xb, op = 1.0 / p, o2p = 0.5 * op, xi = xa * xb * op;
  double PA[3], PB[3], PC[3], AB2 = 0.0, PC2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double P = (xa * A[i] + xb * B[i]) * op;
    PA[i] = P - A[i];
    PB[i] = P - B[i];
    PC[i] = kind ? P - Cn[i] : 0.0;
    AB2 += (A[i] - B[i]) * (A[i] - B[i]);
    PC2 += PC[i] * PC[i];
  }
  const int L = kind ? la + lb : 0;
  const int nA = ncum(la), nB = ncum(lb);
  double *V = calloc((size_t)(L + 2) * nA * nB, sizeof(double));
#define V2(m, a, b) V[((size_t)(m) * nA + (a)) * nB + (b)]
  double F[4 * OR_LMAX + 2];
  if (kind == 0) {
    V2(0, 0, 0) = sqrt(31.006276680299816 * op * op * op) * exp(-xi * AB2);
    /* vrr1: [a+1i|0] = PA_i [a|0] + a_i/2p [a-1i|0] */
    for (int ia = 1; ia < nA; ++ia) {
      const int *e = comp_tab[ia];
      const int i = first_dir(e);
      int em[3] = {e[0], e[1], e[2]};
      em[i] -= 1;
      double v = PA[i] * V2(0, cidx(em[0], em[1], em[2]), 0);
      if (em[i] > 0) {
        int e2[3] = {em[0], em[1], em[2]};
        e2[i] -= 1;
        v += o2p * em[i] * V2(0, cidx(e2[0], e2[1], e2[2]), 0);
      }
      V2(0, ia, 0) = v;
    }
    /* vrr2: [a|b+1i] = PB_i [a|b] + b_i/2p [a|b-1i] + a_i/2p [a-1i|b] */
    for (int ib = 1; ib < nB; ++ib) {
      const int *f = comp_tab[ib];
      const int i = first_dir(f);
      int fm[3] = {f[0], f[1], f[2]};
      fm[i] -= 1;
      const int b1 = cidx(fm[0], fm[1], fm[2]);
      int b2 = -1;
      if (fm[i] > 0) {
        int f2[3] = {fm[0], fm[1], fm[2]};
        f2[i] -= 1;
        b2 = cidx(f2[0], f2[1], f2[2]);
      }
      for (int ia = 0; ia < nA; ++ia) {
        const int *e = comp_tab[ia];
        double v = PB[i] * V2(0, ia, b1);
        if (b2 >= 0) v += o2p * fm[i] * V2(0, ia, b2);
        if (e[i] > 0) {
          int em[3] = {e[0], e[1], e[2]};
          em[i] -= 1;
          v += o2p * e[i] * V2(0, cidx(em[0], em[1], em[2]), b1);
        }
        V2(0, ia, ib) = v;
      }
    }
  } else {
    oracle_boys(F, 1, 0, L, p * PC2);
    const double pref = 2.0 * 3.141592653589793 * op * exp(-xi * AB2);
    for (int m = 0; m <= L; ++m) V2(m, 0, 0) = pref * F[m];
    /* vrr1 on b: [0|b+1i]^(m) = PB_i [..]^(m) - PC_i [..]^(m+1) + b_i/2p ([b-1i]^(m) - [b-1i]^(m+1)) */
    for (int ib = 1; ib < nB; ++ib) {
      const int *f = comp_tab[ib];
      const int lf = f[0] + f[1] + f[2];
      const int i = first_dir(f);
      int fm[3] = {f[0], f[1], f[2]};
      fm[i] -= 1;
      const int b1 = cidx(fm[0], fm[1], fm[2]);
      int b2 = -1;
      if (fm[i] > 0) {
        int f2[3] = {fm[0], fm[1], fm[2]};
        f2[i] -= 1;
        b2 = cidx(f2[0], f2[1], f2[2]);
      }
      for (int m = 0; m + lf <= L; ++m) {
        double v = PB[i] * V2(m, 0, b1) - PC[i] * V2(m + 1, 0, b1);
        if (b2 >= 0) v += o2p * fm[i] * (V2(m, 0, b2) - V2(m + 1, 0, b2));
        V2(m, 0, ib) = v;
      }
    }
    /* vrr2 on a: [a+1i|b]^(m) = PA_i [a|b]^(m) - PC_i [a|b]^(m+1) + b_i/2p ([a|b-1i] - ..^(m+1))
     *                          + a_i/2p ([a-1i|b] - ..^(m+1)) */
    for (int ia = 1; ia < nA; ++ia) {
      const int *e = comp_tab[ia];
      const int le = e[0] + e[1] + e[2];
      const int i = first_dir(e);
      int em[3] = {e[0], e[1], e[2]};
      em[i] -= 1;
      const int a1 = cidx(em[0], em[1], em[2]);
      int a2 = -1;
      if (em[i] > 0) {
        int e2[3] = {em[0], em[1], em[2]};
        e2[i] -= 1;
        a2 = cidx(e2[0], e2[1], e2[2]);
      }
      for (int ib = 0; ib < nB; ++ib) {
        const int *f = comp_tab[ib];
        const int lf = f[0] + f[1] + f[2];
        int b1 = -1;
        if (f[i] > 0) {
          int fm[3] = {f[0], f[1], f[2]};
          fm[i] -= 1;
          b1 = cidx(fm[0], fm[1], fm[2]);
        }
        for (int m = 0; m + le + lf <= L; ++m) {
          double v = PA[i] * V2(m, a1, ib) - PC[i] * V2(m + 1, a1, ib);
          if (b1 >= 0) v += o2p * f[i] * (V2(m, a1, b1) - V2(m + 1, a1, b1));
          if (a2 >= 0) v += o2p * em[i] * (V2(m, a2, ib) - V2(m + 1, a2, ib));
          V2(m, ia, ib) = v;
        }
      }
    }
  }
  const int a0 = ncum(la - 1), b0 = ncum(lb - 1);
  for (int ib = 0; ib < nb; ++ib)
    for (int ia = 0; ia < na; ++ia) out[(size_t)ia * iskipa + (size_t)ib * iskipb] = V2(0, a0 + ia, b0 + ib);
#undef V2
  free(V);
}

/* Same argument lists as the emitted example functions */
void oracle_overlap_2idx_ab_prim_cart_main(double xa, const double cA[3], int la, int na, int iskipa, double xb,
                                           const double cB[3], int lb, int nb, int iskipb, double *work, double *out) {
  (void)work;
  oracle_2idx(0, xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, NULL, out);
}

void oracle_nuclear_2idx_ab_m_cC_prim_cart_main(double xa, const double cA[3], int la, int na, int iskipa, double xb,
                                                const double cB[3], int lb, int nb, int iskipb, const double cC[3],
                                                double *work, double *out) {
  (void)work;
  oracle_2idx(1, xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, cC, out);
}

/* work-array sizes as emitted (examples/example_input.py classes) */
int oracle_2idx_work_array_size(int kind, int la, int lb) {
  return kind == 0 ? ncum(la) * ncum(lb) : 2 * (ncum(lb) * ncum(la) + la + lb + 1);
}

void oracle_2idx_batch(int kind, int n, const double *xa, const double *ca, const int *la, const double *xb,
                       const double *cb, const int *lb, const double *cc, const long long *off, double *out) {
  for (int p = 0; p < n; ++p) {
    const int na = nc_l(la[p]), nb = nc_l(lb[p]);
    oracle_2idx(kind, xa[p], ca + 3 * p, la[p], na, 1, xb[p], cb + 3 * p, lb[p], nb, na, kind ? cc + 3 * p : NULL,
                out + off[p]);
  }
}

/* The library's analytic screening bound of every quartet (pair_bound.h). */
void oracle_quartet_bounds(int nq, const int *quartets, const int *shell_l, const int *shell_k, const int *shell_ptr,
                           const double *shell_xyz, const double *prim_exp, const double *prim_coef, int spherical,
                           double *bounds) {
  for (int q = 0; q < nq; ++q)
    bounds[q] = pb_quartet(quartets + 4 * q, shell_l, shell_k, shell_ptr, shell_xyz, prim_exp, prim_coef, spherical);
}
