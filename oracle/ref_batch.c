/*
 * ref_batch.c -- batch driver around the reference-emitted C99 (test infrastructure).
 *
 * Compiled by oracle/gen_ref.py into oracle/_ref/libref_eri_{cart,sph}.so together
 * with the C99 the reference generator emitted for oracle/eri_input.py.  It calls
 * the emitted per-quartet function once per shell quartet, exactly as a host
 * program using the reference would, with one work array per OpenMP thread.
 *
 * Layout contract (shared with the oracle and the CUDA batch path): shells are
 * segmented (n_cont = 1); quartet q writes its block at out + out_off[q] with a
 * fastest, index = ia + na*(ib + nb*(ic + nc*id)).
 */
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "pair_bound.h"

#if defined(REF_VARIANT_SPH)
#include "intception_integral_eri_abcd_m_cont_sph.h"
#define REF_MAIN intception_integral_eri_abcd_m_cont_sph_main
#define REF_WSIZE intception_integral_eri_abcd_m_cont_sph_work_array_size
#else
#include "intception_integral_eri_abcd_m_cont_cart.h"
#define REF_MAIN intception_integral_eri_abcd_m_cont_cart_main
#define REF_WSIZE intception_integral_eri_abcd_m_cont_cart_work_array_size
#endif

static int rb_ncart(int l) { return (l + 1) * (l + 2) / 2; }

int ref_work_array_size(int la, int lb, int lc, int ld, int ka, int kb, int kc, int kd, int ca, int cb,
                        int cc, int cd) {
  return REF_WSIZE(la, lb, lc, ld, ka, kb, kc, kd, ca, cb, cc, cd);
}

/* Returns the number of quartets evaluated.  nthreads <= 0 uses all cores. */
int ref_eri_batch(int nq, const int *quartets, const int *shell_l, const int *shell_k, const int *shell_ptr,
                  const double *shell_xyz, const double *prim_exp, const double *prim_coef,
                  const double *const *sphT, const long long *out_off, double *out, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_num_procs();
#pragma omp parallel num_threads(nthreads)
  {
    size_t wcap = 0;
    double *work = NULL;
#pragma omp for schedule(dynamic, 64)
    for (int q = 0; q < nq; ++q) {
      const int *s = quartets + 4 * q;
      int l[4], n[4], k[4];
      for (int i = 0; i < 4; ++i) {
        l[i] = shell_l[s[i]];
        k[i] = shell_k[s[i]];
#if defined(REF_VARIANT_SPH)
        n[i] = 2 * l[i] + 1;
#else
        n[i] = rb_ncart(l[i]);
#endif
      }
      size_t need = (size_t)REF_WSIZE(l[0], l[1], l[2], l[3], k[0], k[1], k[2], k[3], 1, 1, 1, 1);
      if (need > wcap) {
        free(work);
        wcap = need;
        work = (double *)malloc(sizeof(double) * wcap);
      }
      int sk[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
      const double *x[4], *c[4], *r[4];
      for (int i = 0; i < 4; ++i) {
        x[i] = prim_exp + shell_ptr[s[i]];
        c[i] = prim_coef + shell_ptr[s[i]];
        r[i] = shell_xyz + 3 * s[i];
      }
#if defined(REF_VARIANT_SPH)
      REF_MAIN(x[0], r[0], l[0], n[0], sk[0], k[0], 1, 0, c[0], sphT[l[0]], x[1], r[1], l[1], n[1], sk[1], k[1], 1,
               0, c[1], sphT[l[1]], x[2], r[2], l[2], n[2], sk[2], k[2], 1, 0, c[2], sphT[l[2]], x[3], r[3], l[3],
               n[3], sk[3], k[3], 1, 0, c[3], sphT[l[3]], work, out + out_off[q]);
#else
      (void)sphT;
      REF_MAIN(x[0], r[0], l[0], n[0], sk[0], k[0], 1, 0, c[0], x[1], r[1], l[1], n[1], sk[1], k[1], 1, 0, c[1],
               x[2], r[2], l[2], n[2], sk[2], k[2], 1, 0, c[2], x[3], r[3], l[3], n[3], sk[3], k[3], 1, 0, c[3],
               work, out + out_off[q]);
#endif
    }
    free(work);
  }
  return nq;
}

/* The same batch with the library's screening in front of the reference's
 * function: quartets whose analytic bound (pair_bound.h) is below skip_below
 * get a zero block, the rest are evaluated by the emitted function, exactly as
 * ref_eri_batch does.  Returns the number evaluated. */
int ref_eri_batch_screened(int nq, const int *quartets, const int *shell_l, const int *shell_k, const int *shell_ptr,
                           const double *shell_xyz, const double *prim_exp, const double *prim_coef,
                           const double *const *sphT, const long long *out_off, double *out, int nthreads,
                           double skip_below) {
  if (nthreads <= 0) nthreads = omp_get_num_procs();
#if defined(REF_VARIANT_SPH)
  const int sph = 1;
#else
  const int sph = 0;
#endif
  int *keep = (int *)malloc(sizeof(int) * (size_t)(nq > 0 ? nq : 1));
  int nkeep = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
  for (int q = 0; q < nq; ++q) {
    const int *s = quartets + 4 * q;
    const double bnd = pb_quartet(s, shell_l, shell_k, shell_ptr, shell_xyz, prim_exp, prim_coef, sph);
    if (bnd < skip_below) {
      int tot = 1;
      for (int i = 0; i < 4; ++i) tot *= sph ? 2 * shell_l[s[i]] + 1 : rb_ncart(shell_l[s[i]]);
      memset(out + out_off[q], 0, sizeof(double) * (size_t)tot);
      keep[q] = 0;
    } else {
      keep[q] = 1;
    }
  }
  int *kq = (int *)malloc(sizeof(int) * 4 * (size_t)(nq > 0 ? nq : 1));
  long long *ko = (long long *)malloc(sizeof(long long) * (size_t)(nq > 0 ? nq : 1));
  for (int q = 0; q < nq; ++q)
    if (keep[q]) {
      for (int i = 0; i < 4; ++i) kq[4 * nkeep + i] = quartets[4 * q + i];
      ko[nkeep++] = out_off[q];
    }
  ref_eri_batch(nkeep, kq, shell_l, shell_k, shell_ptr, shell_xyz, prim_exp, prim_coef, sphT, ko, out, nthreads);
  free(keep);
  free(kq);
  free(ko);
  return nkeep;
}
