/*
 * ref_batch_2idx.c -- batch driver around the reference-emitted C99 of the
 * reference's own example script (examples/example_input.py): primitive
 * Cartesian 2-index overlap and nuclear attraction.  Test infrastructure.
 * Pair p writes its block at out + off[p], a fastest (ia + na*ib).
 */
#include <stdlib.h>

#include "intception_integral_nuclear_2idx_ab_m_cC_prim_cart.h"
#include "intception_integral_overlap_2idx_ab_prim_cart.h"

static int rb2_ncart(int l) { return (l + 1) * (l + 2) / 2; }

/* kind 0: overlap, 1: nuclear attraction to the point cC[3*p]; OpenMP over pairs */
void ref_2idx_batch(int kind, int n, const double *xa, const double *ca, const int *la, const double *xb,
                    const double *cb, const int *lb, const double *cc, const long long *off, double *out) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int p = 0; p < n; ++p) {
    int na = rb2_ncart(la[p]), nb = rb2_ncart(lb[p]);
    int nw = kind == 0 ? intception_integral_overlap_2idx_ab_prim_cart_work_array_size(la[p], lb[p])
                       : intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size(la[p], lb[p]);
    double *work = (double *)malloc(sizeof(double) * (nw + 8));
    if (kind == 0)
      intception_integral_overlap_2idx_ab_prim_cart_main(xa[p], ca + 3 * p, la[p], na, 1, xb[p], cb + 3 * p, lb[p], nb,
                                                         na, work, out + off[p]);
    else
      intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main(xa[p], ca + 3 * p, la[p], na, 1, xb[p], cb + 3 * p,
                                                              lb[p], nb, na, cc + 3 * p, work, out + off[p]);
    free(work);
  }
}

int ref_2idx_work_array_size(int kind, int la, int lb) {
  return kind == 0 ? intception_integral_overlap_2idx_ab_prim_cart_work_array_size(la, lb)
                   : intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size(la, lb);
}
