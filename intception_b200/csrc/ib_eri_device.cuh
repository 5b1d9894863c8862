// ib_eri_device.cuh -- device-side building blocks shared by every ERI kernel.
//
// Data model (HBM, structure of arrays):
//   shell_l/k/ptr [nshell] int32, shell_xyz [3*nshell] f64,
//   prim_exp/prim_coef [nprim] f64 (coefficients already normalised, as the
//   reference's contract_array_?; contracted_general.py:42-68),
//   items [n] IbItem: the four shells of one quartet after canonical permutation
//   and the output strides that undo it.
// Boys: F_L(T) by 7-term Taylor about the nearest point of a 1/16 grid (the
// seven columns L..L+6 of the table row, read through the read-only cache),
// downward recursion to F_0; T >= 36 uses the asymptotic F_0 and upward
// recursion (the scheme of generator_boys_function.py:98-205 on a finer grid).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "_gen/boys_table.h"

#ifndef IB_BLOCK
#define IB_BLOCK 128
#endif

#define IB_LMAX 6
#define IB_NPAIR ((IB_LMAX + 1) * (IB_LMAX + 2) / 2)
// pair ids: la >= lb canonical (0 .. IB_NPAIR-1), and the reversed pair (2,3)
// -- the d shell built on, the f shell reached by the HRR -- as IB_NPAIR
#define IB_NPAIR_EXT (IB_NPAIR + 1)
#define IB_NCLASS (IB_NPAIR_EXT * (IB_NPAIR_EXT + 1) / 2)
#define IB_BOYS_TAYLOR 7

struct IbItem {
  int s[4];         // shells (a, b, c, d) in canonical order
  int st[4];        // output strides of the canonical indices (>= 1; st[0] == 0 marks a quartet
                    // with an l out of range, which the generic kernel evaluates as (ss|ss))
  long long off;    // block offset into the output
};

struct IbLaunch {
  const IbItem* items;
  const int* ranges;  // [2*IB_NCLASS] begin/end of each class id in items
  const int* shell_l;
  const int* shell_k;
  const int* shell_ptr;
  const double* shell_xyz;
  const double* prim_exp;
  const double* prim_coef;
  const double* boys_tab;  // [IB_BOYS_NPTS * IB_BOYS_NCOL]
  const double* sph;       // library Cartesian->spherical matrices, packed per l
  double* out;
  int* status;             // device error word (0 = ok)
  int* flags;              // per sorted item: bit 0 = FP32 result rejected (recompute in FP64),
                           // bit 1 = on the redo list
  int* redo;               // sorted items the generic kernel recomputes (HRR check): [0] heavy count,
                           // [1] light count, then redo_cap slots, heavy items from the front,
                           // light ones from the back
  int redo_cap;            // slots of the redo list (the batch's item count)
  int split_min;           // primitive quartets from which a generic quartet is heavy (ib_generic_split_min)
  double hrr_tol;          // class kernels: largest accepted HRR rounding-error estimate (0: no check)
  int recheck;             // FP64 kernels: evaluate only items with flag bit 0
  double mixed_tol;        // FP32 kernels: largest accepted error bound per quartet
  int max_slices;          // class kernels: cap on lane groups sharing one quartet (0: lane groups per block)
  int slice_boost;         // class kernels: choose slices as if the grid had this many times its lane groups (>= 1)
  int* counter;            // class kernels: next quartet of the range (zero before the launch; one per launch)
  double prim_tol;         // class kernels: skip primitive quartets whose bound is below this (0: exact zeros only)
};

// Rounding-error estimate of a class kernel's horizontal recurrences.  The
// HRRs map the contracted [e0|f0] table linearly onto the block; an element at
// levels (la + k, lc + j) enters every output with a coefficient of at most
// C(lb,k) |AB|^(lb-k) C(ld,j) |CD|^(ld-j), and its rounding error (from the
// vertical recurrences, the contraction and the HRR steps) with it.  The
// kernels take the largest |element| x coefficient over the table and
// multiply by IB_HRR_ERR_COEF.  Measured against binary128 evaluations of the
// same scheme (l <= 4, K <= 8, exponents in [0.02, 1e5]; 162 quartets with an
// error above 1e-16), the error stayed below 21.7 x 2^-53 x that maximum, so
// with 32 units a quartet that passes a tolerance t is within about 0.7 t.
#define IB_HRR_ERR_COEF (32.0 * 1.1102230246251565e-16)

// The generic kernel splits a quartet of at least split_min primitive quartets
// ("heavy") over the blocks of a thread-block cluster (2 or 4, the launch's
// IbGenWork::split); split_min is IB_GEN_SPLIT_MIN unless
// INTCEPTION_B200_GENERIC_SPLIT_MIN sets another (ib_generic_split_min).
// 512: on the l <= 4 workload's classes, 2 000 quartets each, 3-10 % faster
// than 128 per live primitive quartet ((gg|ff) with the HRR check 291 against
// 323 ns), 1 024 no better
#define IB_GEN_SPLIT_MIN 512
int ib_generic_split_min();

// Puts sorted item p on the generic kernel's redo list once (flag bit 1):
// heavy quartets at the front of the list, light ones at the back.
__device__ __forceinline__ void ib_redo_push(const IbLaunch& a, int p) {
  if (atomicOr(a.flags + p, 2) & 2) return;
  const int* s = a.items[p].s;
  const int np = a.shell_k[s[0]] * a.shell_k[s[1]] * a.shell_k[s[2]] * a.shell_k[s[3]];
  if (np >= a.split_min)
    a.redo[2 + atomicAdd(a.redo, 1)] = p;
  else
    a.redo[2 + a.redo_cap - 1 - atomicAdd(a.redo + 1, 1)] = p;
}

// Items of one generic-kernel launch.  Range form (redo 0): heavy items
// ranges[heavy_slot] .. ranges[heavy_slot + 1] (heavy_slot < 0: none), light
// ones ranges[light_slot] .. ranges[light_slot + 1].  List form (redo 1): the
// launch's redo list (IbLaunch::redo).  tickets: two counters (heavy, light)
// zeroed before the launch; the blocks take items in list order from them.
// Null tickets: every item on one block, block b taking items b, b + grid, ...
// split: with tickets, heavy items go to clusters of this many blocks (2 or 4;
// 0: one block each as well).
struct IbGenWork {
  int heavy_slot, light_slot, redo;
  int* tickets;
  int split;
};

// Which generic launches split heavy quartets over clusters:
// INTCEPTION_B200_GENERIC_SPLIT = 0 none, 1 the redo lists, 2 the redo lists
// and the batch's generic range (the default).
int ib_generic_split();

// The generic kernel (eri_generic.cu): blocks per SM it runs with, and its
// launch.  With tickets and wk.split, heavy items go to clusters of wk.split
// blocks (the grid is rounded down to whole clusters that fit the GPU at once).
int ib_generic_bps();
cudaError_t ib_generic_launch(int grid, cudaStream_t s, const IbLaunch& a, const IbGenWork& wk, int sph,
                              double* scratch, long long slice);

// Smallest primitive exponent of shell s.
__device__ __forceinline__ double ib_min_exp(const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                                             const double* __restrict__ prim_exp, int s) {
  const int k = __ldg(shell_k + s), p0 = __ldg(shell_ptr + s);
  double m = __ldg(prim_exp + p0);
  for (int i = 1; i < k; ++i) m = fmin(m, __ldg(prim_exp + p0 + i));
  return m;
}

// Within a pair of equal l, the shell the vertical recurrence builds on comes
// first: the more compact one (larger smallest exponent).  The product centre
// then lies near it, the [e0| and |f0] intermediates stay small, and the
// horizontal recurrence cancels fewer digits (measured: intermediates of 2e3
// for a block of 1e-2 with the diffuse shell first, 6e-2 with the compact one).
__device__ __forceinline__ void ib_compact_first(const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                                                 const double* __restrict__ prim_exp, int* s, const int* l, int* st) {
  for (int i = 0; i < 4; i += 2) {
    if (l[i] != l[i + 1] || s[i] == s[i + 1]) continue;
    if (ib_min_exp(shell_k, shell_ptr, prim_exp, s[i]) < ib_min_exp(shell_k, shell_ptr, prim_exp, s[i + 1])) {
      int t = s[i]; s[i] = s[i + 1]; s[i + 1] = t;
      t = st[i]; st[i] = st[i + 1]; st[i + 1] = t;
    }
  }
}

// Conditioning of a pair's horizontal recurrence.  The vertical recurrence
// builds the pair on shell 0 (exponents x0[k0]) and the HRR moves l1 levels to
// shell 1 (x1[k1], R apart): it combines intermediates of size
// ~(sig + |PA| + R)^l1 into a result of size ~(sig + |PB|)^l1 (sig = zeta^-1/2,
// P the product centre, A shell 0's centre, B shell 1's), so rounding errors
// grow by up to kappa = max over the primitive pairs of
// ((sig + |PA| + R) / (sig + |PB|))^l1.  Large when shell 0 is diffuse and
// shell 1 tight and far: P then sits near B, far from A.  Plain loads, so
// the host (drop-ins) and the device share it.
__host__ __device__ inline double ib_hrr_kappa(int l1, int k0, int k1, const double* x0, const double* x1, double R) {
  float kmax = 1.0f;
  const float Rf = (float)R;
  for (int i = 0; i < k0; ++i)
    for (int j = 0; j < k1; ++j) {
      const float a = (float)x0[i], b = (float)x1[j];
      const float z = a + b, oz = 1.0f / z, sig = 1.0f / sqrtf(z);
      const float r = (sig + b * oz * Rf + Rf) / (sig + a * oz * Rf);
      float k = 1.0f;
      for (int n = 0; n < l1; ++n) k *= r;
      kmax = k > kmax ? k : kmax;
    }
  return (double)kmax;
}

// A pair built on its higher-l shell (l0 > l1 >= 1) whose HRR kappa exceeds
// IB_KAPPA_ROUTE, where building on the other shell lowers it by at least
// IB_KAPPA_GAIN, is evaluated the other way round by the generic kernel (any
// shell order); the unrolled class kernels only build on the higher-l shell.
#define IB_KAPPA_ROUTE 1.0e4
#define IB_KAPPA_GAIN 100.0
__host__ __device__ inline bool ib_pair_reverse(int l0, int l1, int k0, int k1, const double* x0, const double* x1,
                                                double R) {
  if (!(l0 > l1 && l1 >= 1)) return false;
  const double kc = ib_hrr_kappa(l1, k0, k1, x0, x1, R);
  if (!(kc > IB_KAPPA_ROUTE)) return false;
  return ib_hrr_kappa(l0, k1, k0, x1, x0, R) * IB_KAPPA_GAIN < kc;
}

// The generic kernel's shell order for a canonical quartet (s, l, st permuted
// alike): pairs that ib_pair_reverse picks are swapped.  Returns whether any was.
__device__ __forceinline__ bool ib_orient_generic(const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                                                  const double* __restrict__ prim_exp,
                                                  const double* __restrict__ shell_xyz, int* s, int* l, int* st) {
  bool any = false;
  for (int i = 0; i < 4; i += 2) {
    if (!(l[i] > l[i + 1] && l[i + 1] >= 1)) continue;
    double R2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double u = shell_xyz[3 * s[i] + d] - shell_xyz[3 * s[i + 1] + d];
      R2 += u * u;
    }
    if (ib_pair_reverse(l[i], l[i + 1], shell_k[s[i]], shell_k[s[i + 1]], prim_exp + shell_ptr[s[i]],
                        prim_exp + shell_ptr[s[i + 1]], sqrt(R2))) {
      int t = s[i]; s[i] = s[i + 1]; s[i + 1] = t;
      t = l[i]; l[i] = l[i + 1]; l[i + 1] = t;
      t = st[i]; st[i] = st[i + 1]; st[i + 1] = t;
      any = true;
    }
  }
  return any;
}

// Pair id of an ordered pair: la >= lb canonical; (2,3) the reversed pair.
__host__ __device__ inline int ib_pair_ext(int la, int lb) {
  return la >= lb ? la * (la + 1) / 2 + lb : IB_NPAIR;
}

// Reversal for the class kernels of a canonical quartet (s, l, st permuted
// alike).  0: no pair needs it (ib_pair_reverse); 1: every pair that does is an
// (f d) pair and all four l <= 3, so the quartet is reordered here for the
// (d f| class kernels (the pair reversed, then the pair with the larger
// ib_pair_ext id first); 2: the generic kernel is needed (left unchanged).
// fd_only (the HRR check is on, and it covers every other pair): only the
// (f d) pairs of l <= 3 quartets are tested, so the result is 0 or 1.
__device__ __forceinline__ int ib_reverse_for_classes(const int* __restrict__ shell_k,
                                                      const int* __restrict__ shell_ptr,
                                                      const double* __restrict__ prim_exp,
                                                      const double* __restrict__ shell_xyz, int* s, int* l, int* st,
                                                      bool fd_only = false) {
  if (fd_only && max(max(l[0], l[1]), max(l[2], l[3])) > 3) return 0;
  bool rev[2] = {false, false};
  for (int i = 0; i < 4; i += 2) {
    if (!(l[i] > l[i + 1] && l[i + 1] >= 1)) continue;
    if (fd_only && !(l[i] == 3 && l[i + 1] == 2)) continue;
    double R2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double u = shell_xyz[3 * s[i] + d] - shell_xyz[3 * s[i + 1] + d];
      R2 += u * u;
    }
    rev[i / 2] = ib_pair_reverse(l[i], l[i + 1], shell_k[s[i]], shell_k[s[i + 1]], prim_exp + shell_ptr[s[i]],
                                 prim_exp + shell_ptr[s[i + 1]], sqrt(R2));
  }
  if (!rev[0] && !rev[1]) return 0;
  const int lm = max(max(l[0], l[1]), max(l[2], l[3]));
  for (int h = 0; h < 2; ++h)
    if (rev[h] && !(l[2 * h] == 3 && l[2 * h + 1] == 2)) return 2;
  if (lm > 3) return 2;
  for (int h = 0; h < 2; ++h) {
    if (!rev[h]) continue;
    const int i = 2 * h;
    int t = s[i]; s[i] = s[i + 1]; s[i + 1] = t;
    t = l[i]; l[i] = l[i + 1]; l[i + 1] = t;
    t = st[i]; st[i] = st[i + 1]; st[i + 1] = t;
  }
  if (ib_pair_ext(l[0], l[1]) < ib_pair_ext(l[2], l[3])) {
    for (int k = 0; k < 2; ++k) {
      int t = s[k]; s[k] = s[k + 2]; s[k + 2] = t;
      t = l[k]; l[k] = l[k + 2]; l[k + 2] = t;
      t = st[k]; st[k] = st[k + 2]; st[k + 2] = t;
    }
  }
  return 1;
}

// Per-lane constants of a lane-group kernel.  steps: the lane's base-chain
// path, 5 bits per step (direction 0..2, or 3 for an identity step that pads
// shorter paths at the front; then the exponent before the step); misc: the
// lane's Cartesian component (3 bits per axis) and the lanes owning
// component - 1x, - 1y, - 1z inside the group (7 bits each).
struct IbLaneCode {
  unsigned steps;
  unsigned misc;
};

// An opaque register copy: the compiler keeps the value in a register (or
// spills it) instead of re-loading it where it is used.
__device__ __forceinline__ unsigned ib_pin(unsigned x) {
  unsigned y;
  asm volatile("mov.b32 %0, %1;" : "=r"(y) : "r"(x));
  return y;
}

// Barrier over the n threads (64 or 128) of multi-warp lane group g of the
// block (named barrier g+1).
__device__ __forceinline__ void ib_group_bar(int g, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(n) : "memory");
}

// Slices per quartet of a class kernel: the largest power of two W <= gpb
// (and <= cap when cap > 0) with n * W <= boost x the grid's lane groups, so
// that a class with fewer quartets than lane groups spreads each quartet's
// primitive quartets over W groups.  Uniform over the grid (n, gridDim, cap,
// boost are).
__device__ __forceinline__ int ib_slices(int n, int gpb, int cap, int boost = 1) {
  const int wmax = cap > 0 ? min(cap, gpb) : gpb;
  const long long groups = (long long)gridDim.x * gpb * max(boost, 1);
  int w = 1;
  while (2 * w <= wmax && (long long)n * (2 * w) <= groups) w *= 2;
  return w;
}

// Slices for kernels with three lane groups per warp: 3 (one warp per
// quartet) when the class's quartets fill at most a third of the grid's groups
// and the cap allows it, else 1.
__device__ __forceinline__ int ib_slices_in_threes(int n, int gpb, int cap, int boost = 1) {
  const long long groups = (long long)gridDim.x * gpb * max(boost, 1);
  return ((cap == 0 || cap >= 3) && (long long)n * 3 <= groups) ? 3 : 1;
}

// Barrier over the sg-th quartet slot of the block (SG lanes): a warp-level
// sync inside a warp, named barrier sg+1 for two warps, the block barrier for
// the whole block.  Every lane of the slot calls it the same number of times.
__device__ __forceinline__ void ib_sg_sync(int SG, int sg, unsigned mask) {
  if (SG <= 32) {
    __syncwarp(mask);
  } else if (SG < IB_BLOCK) {
    asm volatile("bar.sync %0, %1;" ::"r"(sg + 1), "r"(SG) : "memory");
  } else {
    __syncthreads();
  }
}

// Register budgets of the class kernels: variant v4 + 4 * mi is launched with
// __launch_bounds__(IB_BLOCK, IB_MINB_VALUES[mi]) (minimum resident blocks per
// SM; 1 = no register cap).  The autotuner picks mi per class and variant.
#define IB_NMINB 4
__host__ __device__ inline constexpr int ib_minb_value(int mi) { return mi == 0 ? 1 : mi + 2; }  // 1, 3, 4, 5

// The next quartet for the sg-th quartet slot of the block (SG lanes, r = this
// lane's rank, lane0 = the warp lane of rank 0 when SG <= 32): one atomic per
// quartet, broadcast to the slot, so that slots that finish early take the
// remaining quartets (the range is sorted longest first).  slot: an int of
// shared memory owned by the quartet slot (used when it spans warps).
__device__ __forceinline__ int ib_grab(int* ctr, int beg, int r, int SG, int sg, unsigned sgmask, int lane0,
                                       int* slot) {
  if (SG <= 32) {
    int v = 0;
    if (r == 0) v = atomicAdd(ctr, 1);
    return beg + __shfl_sync(sgmask, v, lane0);
  }
  ib_sg_sync(SG, sg, sgmask);  // every lane has read the previous value
  if (r == 0) *slot = atomicAdd(ctr, 1);
  ib_sg_sync(SG, sg, sgmask);
  return beg + *slot;
}

typedef void (*IbLaunchFn)(int variant, int grid, cudaStream_t s, const IbLaunch& a);
typedef int (*IbOccFn)(int variant);
struct IbClassEntry {
  int cid;
  IbLaunchFn launch;    // null: no unrolled kernel (the generic kernel serves the class)
  IbOccFn occupancy;
  int kind;             // 1: FP64 variants only, 2: FP64 and FP32 variants
};

__host__ __device__ inline constexpr double ib_two_pi52() { return 34.98683665524972497; }  // 2 pi^(5/2)

// F_m(T), m = 0..L, into F[] (compile-time L so the recursion unrolls), from
// the global table (rows of IB_BOYS_NCOL values F_n(T_i); the seven columns
// L..L+6 of one row are read through the read-only cache, which keeps the
// class's 578 x 7 working set resident next to the kernel's shared memory).
template <int L>
__device__ __forceinline__ void ib_boys(double T, const double* __restrict__ tab, double* F) {
  if (T < IB_BOYS_TMAX) {
    const int i = __double2int_rn(T * (double)IB_BOYS_H_INV);
    const double dx = (double)i * (1.0 / IB_BOYS_H_INV) - T;
    const double* r = tab + i * IB_BOYS_NCOL + L;
    double f = __ldg(r + 6) * (1.0 / 720.0);
    f = fma(f, dx, __ldg(r + 5) * (1.0 / 120.0));
    f = fma(f, dx, __ldg(r + 4) * (1.0 / 24.0));
    f = fma(f, dx, __ldg(r + 3) * (1.0 / 6.0));
    f = fma(f, dx, __ldg(r + 2) * 0.5);
    f = fma(f, dx, __ldg(r + 1));
    f = fma(f, dx, __ldg(r));
    F[L] = f;
    if (L > 0) {
      const double e = exp(-T), t2 = T + T;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * (1.0 / (2 * m + 1));
    }
  } else {
    const double oT = 1.0 / T;
    F[0] = sqrt(0.78539816339744830962 * oT);  // (1/2) sqrt(pi/T)
    if (L > 0) {
      const double he = 0.5 * exp(-T);
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = fma((double)m + 0.5, F[m], -he) * oT;
    }
  }
}

// FP32 Boys for the FP32 tier's setup: the same scheme, the table values
// rounded to float, the arithmetic in float (T and the grid offset in FP64).
// Relative error of every F_m <= IB_F32_SETUP_ROUNDINGS x 2^-24 (7 Taylor
// roundings and the table's, 3 per recursion step, 2 ulp of expf).
template <int L>
__device__ __forceinline__ void ib_boys_f32(double T, const double* __restrict__ tab, double* F) {
  float f32[L + 1];
  if (T < IB_BOYS_TMAX) {
    const int i = __double2int_rn(T * (double)IB_BOYS_H_INV);
    const float dx = (float)((double)i * (1.0 / IB_BOYS_H_INV) - T);
    const double* r = tab + i * IB_BOYS_NCOL + L;
    float f = (float)__ldg(r + 6) * (1.0f / 720.0f);
    f = fmaf(f, dx, (float)__ldg(r + 5) * (1.0f / 120.0f));
    f = fmaf(f, dx, (float)__ldg(r + 4) * (1.0f / 24.0f));
    f = fmaf(f, dx, (float)__ldg(r + 3) * (1.0f / 6.0f));
    f = fmaf(f, dx, (float)__ldg(r + 2) * 0.5f);
    f = fmaf(f, dx, (float)__ldg(r + 1));
    f = fmaf(f, dx, (float)__ldg(r));
    f32[L] = f;
    if (L > 0) {
      const float e = expf((float)-T), t2 = (float)(T + T);
#pragma unroll
      for (int m = L - 1; m >= 0; --m) f32[m] = fmaf(t2, f32[m + 1], e) * (1.0f / (2 * m + 1));
    }
  } else {
    const float oT = 1.0f / (float)T;
    f32[0] = sqrtf(0.78539816339744830962f * oT);
    if (L > 0) {
      const float he = 0.5f * expf((float)-T);
#pragma unroll
      for (int m = 0; m < L; ++m) f32[m + 1] = fmaf((float)m + 0.5f, f32[m], -he) * oT;
    }
  }
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] = (double)f32[m];
}
// Extra roundings of unit 2^-24 in the FP32 setup's scaled Boys values (Boys in
// float <= 7 + 1 + 3 L + 2 for L <= 16, the float prefactor exponentials and
// square root 5), counted into the FP32 tier's error bound.
#define IB_F32_SETUP_ROUNDINGS 72

// 1/x: a float reciprocal refined by one FP64 Newton step (relative error
// ~2^-46, far below the FP32 tier's rounding unit), for the FP32 setup.
__device__ __forceinline__ double ib_rcp_refined(double x) {
  double r = (double)(1.0f / (float)x);
  return r * fma(-x, r, 2.0);
}

// Pair prefactor for the FP32 setup: expf where its result stays a normal
// float (the argument above -80), the FP64 exp below, so that the prefactor is
// zero exactly where the FP64 one is and primitive quartets are culled alike.
__device__ __forceinline__ double ib_pair_factor_f32(double xa, double ca, double xb, double cb, double oz, double r2) {
  const double arg = -xa * xb * oz * r2;
  return ca * cb * (arg > -80.0 ? (double)expf((float)arg) : exp(arg));
}

// Runtime-L variant reading the global table directly (one thread, no staging).
__device__ inline void ib_boys_rt(double T, int L, const double* __restrict__ tab, double* F) {
  if (T < IB_BOYS_TMAX) {
    const int i = __double2int_rn(T * (double)IB_BOYS_H_INV);
    const double dx = (double)i * (1.0 / IB_BOYS_H_INV) - T;
    const double* r = tab + i * IB_BOYS_NCOL + L;
    double f = r[6] * (1.0 / 720.0);
    f = fma(f, dx, r[5] * (1.0 / 120.0));
    f = fma(f, dx, r[4] * (1.0 / 24.0));
    f = fma(f, dx, r[3] * (1.0 / 6.0));
    f = fma(f, dx, r[2] * 0.5);
    f = fma(f, dx, r[1]);
    f = fma(f, dx, r[0]);
    F[L] = f;
    const double e = exp(-T), t2 = T + T;
    for (int m = L - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) / (double)(2 * m + 1);
  } else {
    const double oT = 1.0 / T;
    F[0] = sqrt(0.78539816339744830962 * oT);
    const double he = 0.5 * exp(-T);
    for (int m = 0; m < L; ++m) F[m + 1] = fma((double)m + 0.5, F[m], -he) * oT;
  }
}

// First-order bound on the rounding error of an FP32 evaluation of the VRR of
// one primitive quartet, for every target [s|c]^(0) (lane side s up to level
// S, chain side c up to level C).  The absolute-value recurrence is bounded by
// |s0| g^S h^C with g^2 >= aS g + bS (base chain: aS = |X|+|W|, bS =
// S (1+r)/2x) and h^2 >= (aC + tC/g) h + bC (chain side with the transfer
// term tC = S/2(zeta+eta)); each value passes through at most 4(S+C)+2
// roundings of unit 2^-24, plus `extra` for inputs that carry rounding errors
// of their own.  g and h are found in float (a few ulp each); the factor
// 1.0001 covers their rounding through the powers (S + C <= 16).
__device__ __forceinline__ double ib_fp32_err(double s0, double aS, double bS, int S, double aC, double bC,
                                              double tC, int C, int extra = 0) {
  const float as = (float)aS, bs = (float)bS;
  const float g = fmaxf(0.5f * (as + sqrtf(as * as + 4.0f * bs)), 1.0f);
  const float a2 = (float)aC + (float)tC / g;
  const float h = fmaxf(0.5f * (a2 + sqrtf(a2 * a2 + 4.0f * (float)bC)), 1.0f);
  float gh = 1.0001f;
  for (int i = 0; i < S; ++i) gh *= g;
  for (int i = 0; i < C; ++i) gh *= h;
  return (4.0 * (S + C) + 2.0 + extra) * 5.9604644775390625e-08 * fabs(s0) * (double)gh;
}

__device__ __forceinline__ double ib_amax3(double x, double y, double z) { return fmax(fabs(x), fmax(fabs(y), fabs(z))); }

struct IbQuartet {
  double A[3], B[3], C[3], D[3];
  double AB[3], CD[3];
  double RAB2, RCD2;
  int k[4], ptr[4], st[4];
  long long off;
};

__device__ __forceinline__ void ib_load_quartet(const IbLaunch& a, int p, IbQuartet& g) {
  const IbItem it = a.items[p];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int s = it.s[i];
    g.k[i] = __ldg(a.shell_k + s);
    g.ptr[i] = __ldg(a.shell_ptr + s);
    g.st[i] = it.st[i];
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g.A[d] = __ldg(a.shell_xyz + 3 * it.s[0] + d);
    g.B[d] = __ldg(a.shell_xyz + 3 * it.s[1] + d);
    g.C[d] = __ldg(a.shell_xyz + 3 * it.s[2] + d);
    g.D[d] = __ldg(a.shell_xyz + 3 * it.s[3] + d);
  }
  g.off = it.off;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g.AB[d] = g.A[d] - g.B[d];
    g.CD[d] = g.C[d] - g.D[d];
  }
  g.RAB2 = g.AB[0] * g.AB[0] + g.AB[1] * g.AB[1] + g.AB[2] * g.AB[2];
  g.RCD2 = g.CD[0] * g.CD[0] + g.CD[1] * g.CD[1] + g.CD[2] * g.CD[2];
}

struct IbBraPair {
  double zeta, oz, K;
  double P[3], PA[3];
};

// Prefactor c_a c_b exp(-xa xb/(xa+xb) R^2) of a primitive pair: the one
// expression every pair evaluation uses, so that a pair culled for a zero
// prefactor is exactly a pair whose primitive quartets would all be zero.
__device__ __forceinline__ double ib_pair_factor(double xa, double ca, double xb, double cb, double oz, double r2) {
  return ca * cb * exp(-xa * xb * oz * r2);
}

// Bra pair of primitives ia, ib.  F32SETUP (the FP32 tier): the reciprocal by
// ib_rcp_refined and the prefactor by ib_pair_factor_f32.
template <bool F32SETUP = false>
__device__ __forceinline__ void ib_bra_pair(const IbLaunch& a, const IbQuartet& g, int ia, int ib, IbBraPair& bp) {
  const double xa = __ldg(a.prim_exp + g.ptr[0] + ia), ca = __ldg(a.prim_coef + g.ptr[0] + ia);
  const double xb = __ldg(a.prim_exp + g.ptr[1] + ib), cb = __ldg(a.prim_coef + g.ptr[1] + ib);
  bp.zeta = xa + xb;
  bp.oz = F32SETUP ? ib_rcp_refined(bp.zeta) : 1.0 / bp.zeta;
  bp.K = F32SETUP ? ib_pair_factor_f32(xa, ca, xb, cb, bp.oz, g.RAB2) : ib_pair_factor(xa, ca, xb, cb, bp.oz, g.RAB2);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    bp.P[d] = (xa * g.A[d] + xb * g.B[d]) * bp.oz;
    bp.PA[d] = bp.P[d] - g.A[d];
  }
}

// Live primitive pairs of one side of the quartet (side 0: shells a, b; 1: c, d)
// within the tile of pair indices [p0, p0 + n), n <= 64: the offsets t (pair
// p0 + t, pair index = i0 * K1 + i1) whose prefactor is not zero, in
// increasing order, into lst[]; returns their number.  Run by nb <= 32
// builder lanes of one warp (b = this lane's rank, bmask their lanes, bbase
// the lane of rank 0); every builder returns the same count.
__device__ __forceinline__ int ib_live_pairs(const IbLaunch& a, const IbQuartet& g, int side, int p0, int n,
                                             unsigned char* __restrict__ lst, int b, int nb, unsigned bmask,
                                             int bbase) {
  const int ptr0 = g.ptr[2 * side], ptr1 = g.ptr[2 * side + 1], k1 = g.k[2 * side + 1];
  const double r2 = side ? g.RCD2 : g.RAB2;
  int cnt = 0;
  for (int t0 = 0; t0 < n; t0 += nb) {
    const int t = t0 + b;
    bool live = false;
    if (t < n) {
      const int p = p0 + t, i0 = p / k1, i1 = p - i0 * k1;
      const double x0 = __ldg(a.prim_exp + ptr0 + i0), c0 = __ldg(a.prim_coef + ptr0 + i0);
      const double x1 = __ldg(a.prim_exp + ptr1 + i1), c1 = __ldg(a.prim_coef + ptr1 + i1);
      live = ib_pair_factor(x0, c0, x1, c1, 1.0 / (x0 + x1), r2) != 0.0;
    }
    const unsigned bal = __ballot_sync(bmask, live) >> bbase;
    if (live) lst[cnt + __popc(bal & ((1u << b) - 1u))] = (unsigned char)t;
    cnt += __popc(bal);
  }
  return cnt;
}

// ---- Primitive screening.  For a primitive pair (exponents x0, x1 on
// centres A, B; P the product centre, zeta = x0 + x1) every Cartesian
// component of the product is bounded pointwise,
//   |c0 c1 (x-A_x)^i .. (x-B_x)^j ..| exp(-x0|r-A|^2 - x1|r-B|^2)
//     <= K (rho + |PA|)^l0 (rho + |PB|)^l1 exp(-zeta rho^2),   rho = |r - P|,
// K = |c0 c1| exp(-x0 x1 |AB|^2 / zeta).  The Coulomb norm ||f|| = (f|f)^1/2
// is monotone for positive f and obeys the triangle inequality, and
// ||rho^n exp(-zeta rho^2)|| = N_n zeta^-(2n+5)/4 with N_n^2 the self-energy of
// r^n exp(-r^2) (N_0^2 = sqrt(2) pi^5/2; the others by quadrature, 30
// digits).  So the primitive pair's charge distributions have Coulomb norm
//   Q <= K sum_ij C(l0,i) C(l1,j) |PA|^(l0-i) |PB|^(l1-j) N_(i+j) zeta^-(2(i+j)+5)/4,
// times, for spherical output, the largest sum of |coefficients| of a
// spherical function over Cartesians (per shell).  By Cauchy-Schwarz a
// primitive quartet changes no element of its block by more than
// Q_ab Q_cd: skipping those below a tolerance t moves an element by at most
// (number skipped) x t.
__host__ __device__ inline constexpr double ib_rn_norm(int n) {
  return n == 0 ? 4.9738746919472297 : n == 1 ? 5.1652368552576019 : n == 2 ? 6.4612527577002005
       : n == 3 ? 9.2648431767816622 : n == 4 ? 14.794795287711256 : n == 5 ? 25.818805439099522
       : n == 6 ? 48.591021989124202 : n == 7 ? 97.655519373091779 : n == 8 ? 208.00183355514711
       : n == 9 ? 466.71786414003641 : n == 10 ? 1097.8288726985819 : n == 11 ? 2696.1716819638506
       : 6889.8632213814936;
}
__host__ __device__ inline constexpr double ib_binom(int n, int k) {
  return k == 0 || k == n ? 1.0 : ib_binom(n - 1, k - 1) + ib_binom(n - 1, k);
}
// largest sum of |Cartesian coefficients| of one spherical function of the
// library's transformation matrices, l = 0..6 (rounded up)
__host__ __device__ inline constexpr double ib_sph_colsum(int l) {
  return l <= 1 ? 1.0 : l == 2 ? 2.0 : l == 3 ? 4.0 : l == 4 ? 8.9442719099991597 : l == 5 ? 20.493901531919201
       : 47.096974425115671;
}

template <int L0, int L1, bool SPH>
__device__ __forceinline__ double ib_pair_bound(double K, double zeta, double pa, double pb) {
  const double s = 1.0 / sqrt(zeta);  // zeta^-1/2
  double poly = 0.0;
#pragma unroll
  for (int i = 0; i <= L0; ++i) {
#pragma unroll
    for (int j = 0; j <= L1; ++j) {
      double t = ib_binom(L0, i) * ib_binom(L1, j) * ib_rn_norm(i + j);
#pragma unroll
      for (int k = 0; k < L0 - i; ++k) t *= pa;
#pragma unroll
      for (int k = 0; k < L1 - j; ++k) t *= pb;
#pragma unroll
      for (int k = 0; k < i + j; ++k) t *= s;
      poly += t;
    }
  }
  // zeta^-5/4; the factor 1 + 1e-6 covers the rounding of the bound itself
  const double sph = SPH ? ib_sph_colsum(L0) * ib_sph_colsum(L1) : 1.0;
  return 1.000001 * sph * K * s * s * sqrt(s) * poly;
}

// ib_pair_bound for angular momenta known only at run time (l0, l1 <= 6), in
// float: the sum over i, j of C(l0,i) C(l1,j) |PA|^(l0-i) |PB|^(l1-j)
// N_(i+j) s^(i+j), regrouped by n = i + j as the coefficients of
// (pa + t)^l0 (pb + t)^l1 (loops unrolled to the largest degree so the
// coefficients stay in registers).  Every operand is positive, so the float
// result is within a few hundred ulp (< 1e-4 relative) of the exact one; the
// factor 1.001 makes it an upper bound.  The Gaussian factor exp(-x0 x1 R^2 /
// zeta): float above exp(-80); down to exp(-708) a float 2^frac scaled by an
// exact power of two (FP64 range, float accuracy); in the subnormal band FP64
// exp; zero below exp(-745.2), where FP64 exp is zero too.
template <int MAXDEG>
__device__ __forceinline__ double ib_pair_bound_rt(int l0, int l1, bool sph, double cc, double x0, double x1,
                                                   double R) {
  const float z = (float)(x0 + x1), oz = 1.0f / z;
  // the Gaussian's argument in float: ~4e-7 relative, so under 3e-4 of the
  // factor at the exp(-708) end, inside the 1.001 margin with the polynomial's error
  const float arg = -((float)x0 * (float)x1 * oz) * (float)(R * R);
  if (arg < -745.2f) return 0.0;  // exp underflows to zero in FP64 there (a NaN goes on)
  double e;
  if (arg > -80.0f) {
    e = (double)__expf(arg);
  } else if (arg > -708.0f) {
    // 2^t, t = arg log2(e): float 2^frac times an exact normal power of two (5e-5 relative)
    const float t = arg * 1.44269504f, n = floorf(t);
    e = (double)exp2f(t - n) * __longlong_as_double((long long)(1023 + (int)n) << 52);
  } else {
    e = exp((double)arg);  // the subnormal band, where a scaled float would round differently
  }
  const float pa = (float)x1 * oz * (float)R, pb = (float)x0 * oz * (float)R;
  const int deg = l0 + l1;
  float c[MAXDEG + 1];  // MAXDEG >= l0 + l1: the batch's 2 lmax, so the unrolled loops stay short
#pragma unroll
  for (int n = 0; n <= MAXDEG; ++n) c[n] = n == 0 ? 1.0f : 0.0f;
#pragma unroll
  for (int r = 0; r < MAXDEG; ++r) {
    if (r < deg) {
      const float p = r < l0 ? pa : pb;
#pragma unroll
      for (int n = r + 1; n > 0; --n) c[n] = fmaf(c[n], p, c[n - 1]);
      c[0] *= p;
    }
  }
  const float s = rsqrtf(z);
  float poly = 0.0f, sn = 1.0f;
#pragma unroll
  for (int n = 0; n <= MAXDEG; ++n) {
    if (n <= deg) poly = fmaf(c[n] * (float)ib_rn_norm(n), sn, poly);
    sn *= s;
  }
  const float f = sph ? (float)(ib_sph_colsum(l0) * ib_sph_colsum(l1)) : 1.0f;
  return 1.001 * fabs(cc) * e * (double)(f * s * s * sqrtf(s) * poly);
}

// Bound Q of primitive pair i0 * k1 + i1 of two shells (exponent/coefficient
// runs at ptr0, ptr1; squared centre distance r2).
template <int L0, int L1, bool SPH>
__device__ __forceinline__ double ib_pair_q(const double* __restrict__ pe, const double* __restrict__ pc, int ptr0,
                                            int ptr1, int k1, double r2, int p) {
  const int i0 = p / k1, i1 = p - i0 * k1;
  const double x0 = __ldg(pe + ptr0 + i0), c0 = __ldg(pc + ptr0 + i0);
  const double x1 = __ldg(pe + ptr1 + i1), c1 = __ldg(pc + ptr1 + i1);
  const double z = x0 + x1, oz = 1.0 / z, R = sqrt(r2);
  const double K = fabs(ib_pair_factor(x0, c0, x1, c1, oz, r2));
  return ib_pair_bound<L0, L1, SPH>(K, z, x1 * oz * R, x0 * oz * R);
}

// Power-of-two exponent e with Q <= 2^e (Q >= 0), clamped to [-127, 127];
// 127 stands for "not small": Q >= 2^126, infinite or NaN (never for
// normalised shells; a primitive quartet with it is never skipped, so a NaN
// input still reaches the result as on the exact path).
__device__ __forceinline__ signed char ib_q_exp(double q) {
  if (q == 0.0) return -127;
  if (!(q < 0x1p126)) return 127;
  const int e = ilogb(q) + 1;  // q < 2^(ilogb(q) + 1)
  return (signed char)max(-127, min(e, 127));
}

// A primitive quartet of the screened lists (list positions qa, qc) whose
// bound Q_ab Q_cd <= 2^(e_ab + e_cd) is below tol.
__device__ __forceinline__ bool ib_quartet_negligible(const unsigned char* __restrict__ lst, int qa, int qc,
                                                      double tol) {
  const int ea = (signed char)lst[128 + qa], ec = (signed char)lst[192 + qc];
  return ea < 127 && ec < 127 && ldexp(1.0, ea + ec) < tol;
}

// Live-pair lists of one 64 x 64 pair tile with primitive screening (tol > 0):
// pair ab (tile offset t, pair p0 + t of shells a, b) stays if Q_ab times the
// largest Q_cd of the tile reaches tol, and likewise for cd; every primitive
// quartet dropped this way has Q_ab Q_cd < tol.  Beside each list entry
// (lst[128 + pos] side 0, lst[192 + pos] side 1) goes the exponent of its
// pair's bound, for ib_quartet_negligible.  Run by the nb builder lanes of one
// warp as ib_live_pairs (lane rank b, lanes bmask starting at bbase); the
// largest bounds are reduced over those lanes as floats rounded up.  The class
// kernels call it before their accumulators are live.  Returns (n0, n1).
template <int LA, int LB, int LC, int LD, bool SPH>
__device__ __forceinline__ int2 ib_live_pairs_screened(const double* __restrict__ pe, const double* __restrict__ pc,
                                                    int pa, int pb, int kb, int pcs, int pd, int kd, double rab2,
                                                    double rcd2, int p0, int m0, int p1, int m1,
                                                    unsigned char* __restrict__ lst, int b, int nb, unsigned bmask,
                                                    int bbase, double tol) {
  double q0 = 0.0, q1 = 0.0;
  for (int t = b; t < m0; t += nb) q0 = fmax(q0, ib_pair_q<LA, LB, SPH>(pe, pc, pa, pb, kb, rab2, p0 + t));
  for (int t = b; t < m1; t += nb) q1 = fmax(q1, ib_pair_q<LC, LD, SPH>(pe, pc, pcs, pd, kd, rcd2, p1 + t));
  const double M0 = (double)__uint_as_float(__reduce_max_sync(bmask, __float_as_uint(__double2float_ru(q0))));
  const double M1 = (double)__uint_as_float(__reduce_max_sync(bmask, __float_as_uint(__double2float_ru(q1))));
  int n[2];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int p = side ? p1 : p0, m = side ? m1 : m0;
    const double other = side ? M0 : M1;
    unsigned char* __restrict__ l = lst + 64 * side;
    int cnt = 0;
    for (int t0 = 0; t0 < m; t0 += nb) {
      const int t = t0 + b;
      bool live = false;
      double q = 0.0;
      if (t < m) {
        q = side ? ib_pair_q<LC, LD, SPH>(pe, pc, pcs, pd, kd, rcd2, p + t)
                 : ib_pair_q<LA, LB, SPH>(pe, pc, pa, pb, kb, rab2, p + t);
        live = !(q == 0.0 || q * other < tol);  // dropped only when provably small (NaN stays)
      }
      const unsigned bal = __ballot_sync(bmask, live) >> bbase;
      if (live) {
        const int pos = cnt + __popc(bal & ((1u << b) - 1u));
        l[pos] = (unsigned char)t;
        l[128 + pos] = (unsigned char)ib_q_exp(q);
      }
      cnt += __popc(bal);
    }
    n[side] = cnt;
  }
  return make_int2(n[0], n[1]);
}

template <typename R>
struct IbPrimQuartet {
  R PA[3], WP[3], QC[3], WQ[3];
  R o2z, roz, o2e, roe, o2zpe;
};

// Ket pair, quartet geometry and the scaled Boys values F[m] = pref * F_m(T).
// Returns false (and computes nothing else) when the pair prefactors multiply
// to exactly zero: every value of that primitive quartet would be +-0, so
// skipping it leaves the contracted sums bit-identical.
template <typename R, int L>
__device__ __forceinline__ bool ib_prim_quartet(const IbLaunch& a, const IbQuartet& g, const IbBraPair& bp, int ic,
                                                int id, const double* __restrict__ boys_tab, double* F,
                                                IbPrimQuartet<R>& pq) {
  const double xc = __ldg(a.prim_exp + g.ptr[2] + ic), cc = __ldg(a.prim_coef + g.ptr[2] + ic);
  const double xd = __ldg(a.prim_exp + g.ptr[3] + id), cd = __ldg(a.prim_coef + g.ptr[3] + id);
  // the FP32 tier (R = float) computes the reciprocals, exponentials, square
  // root and Boys values in float (reciprocals refined in FP64); its error
  // bound counts IB_F32_SETUP_ROUNDINGS more roundings for the scaled F_m
  constexpr bool F32 = sizeof(R) == 4;
  const double eta = xc + xd, oe = F32 ? ib_rcp_refined(eta) : 1.0 / eta;
  const double Kcd = F32 ? ib_pair_factor_f32(xc, cc, xd, cd, oe, g.RCD2) : ib_pair_factor(xc, cc, xd, cd, oe, g.RCD2);
  if (bp.K * Kcd == 0.0) return false;
  const double ozpe = F32 ? ib_rcp_refined(bp.zeta + eta) : 1.0 / (bp.zeta + eta);
  const double rho = bp.zeta * eta * ozpe;
  double Q[3], PQ[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    Q[d] = (xc * g.C[d] + xd * g.D[d]) * oe;
    PQ[d] = bp.P[d] - Q[d];
  }
  const double RPQ2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
  if (F32)
    ib_boys_f32<L>(rho * RPQ2, boys_tab, F);
  else
    ib_boys<L>(rho * RPQ2, boys_tab, F);
  const double pref = ib_two_pi52() * bp.oz * oe * (F32 ? (double)sqrtf((float)ozpe) : sqrt(ozpe)) * bp.K * Kcd;
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] *= pref;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double W = (bp.zeta * bp.P[d] + eta * Q[d]) * ozpe;
    pq.PA[d] = (R)bp.PA[d];
    pq.WP[d] = (R)(W - bp.P[d]);
    pq.QC[d] = (R)(Q[d] - g.C[d]);
    pq.WQ[d] = (R)(W - Q[d]);
  }
  pq.o2z = (R)(0.5 * bp.oz);
  pq.roz = (R)(rho * bp.oz);
  pq.o2e = (R)(0.5 * oe);
  pq.roe = (R)(rho * oe);
  pq.o2zpe = (R)(0.5 * ozpe);
  return true;
}
