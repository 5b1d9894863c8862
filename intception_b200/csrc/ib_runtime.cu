// ib_runtime.cu -- host runtime and C ABI of the B200 ERI backend.
//
// Batch pipeline (all on the device, stream-ordered, no host round trip):
//   1. ib_classify   : per quartet, canonical class id (la>=lb, lc>=ld,
//                      bra pair >= ket pair), screening and precision bits,
//                      log2 of the primitive quartet count -> 16-bit sort key
//   2. CUB radix sort: quartets grouped by (screening, precision, class), the
//                      longest first within a class
//   3. ib_build_items: permuted shells + output strides per sorted quartet, and
//                      the [begin,end) range of every (precision, class)
//   4. per-class persistent kernels (unrolled, emitted) fanned out over side
//      streams, plus the generic block-per-quartet kernel for the rest.
// The drop-ins build the same items on the host for one quartet (all
// contraction combinations) and reuse the class kernels.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/intception_b200.h"
#include "_gen/boys_table_data.h"
#include "ib_eri_device.cuh"
#include "ib_generic.cuh"

void ib_register_emitted_classes(IbClassEntry* table);
// Real solid harmonics in the library convention (m = -l..l, each scaled to the
// norm of x^l); computed once on the host and kept on the device.
void build_sph_host(std::vector<double>& out);
extern const int ib_n_emitted_classes;
extern const int ib_lmax_emitted;
extern const int ib_tuned_minb[IB_NCLASS][4];
extern const int ib_tuned_slice_cap[IB_NCLASS];
extern const int ib_tuned_fp32[IB_NCLASS];

namespace {

constexpr int kNSideMax = 64;                   // side streams for concurrent class kernels (upper limit)
constexpr int kSlotFp32 = 2 * IB_NCLASS;        // ranges offset of the FP32 copies
constexpr int kSlotGenHeavy = 4 * IB_NCLASS;    // [begin, end) of the generic kernel's heavy quartets
constexpr int kSlotSkip = 4 * IB_NCLASS + 2;    // [begin, end) of the screened-out quartets
constexpr int kSlotGenLight = 4 * IB_NCLASS + 4;  // [begin, end) of the generic kernel's light quartets
constexpr int kNRanges = 4 * IB_NCLASS + 6;
constexpr int kNCounters = 3 * IB_NCLASS;      // quartet counters: FP64 pass, FP32 pass, FP64 recheck pass
// sort key: skip(1) generic(1) fp32(1) class(9) work(4), two radix passes; a
// generic quartet's class and work bits hold light(1) and its cost code (8)
constexpr int kKeyBits = 16;
constexpr size_t kScratchCap = size_t(4) << 30;  // bytes of generic-kernel scratch at most
constexpr int kRedoGroups = 4;  // redo lists of an l >= 3 batch (dispatch)
constexpr int kTickets = 2 * (1 + kRedoGroups);  // generic-kernel ticket pairs: the range launch, each redo list
// blocks per cluster sharing a heavy generic quartet: a redo list is short and
// its end waits for its heaviest quartets, so 4; a batch's generic range keeps
// every block busy, and rank 0's HRRs idle fewer ranks with 2 (l <= 4 sample,
// 2 000 quartets of one class: (gg|gg) 878 against 1 038 ns per live primitive
// quartet with 2 and 4, the redo-heavy (gg|ff) 387 against 325)
constexpr int kSplitRedo = 4, kSplitRange = 2;

thread_local int tl_status = IB_OK;
thread_local std::string tl_msg;
thread_local int tl_launches = 0;

int set_status(int st, const std::string& msg) {
  tl_status = st;
  tl_msg = msg;
  return st;
}

#define IB_CUDA(call)                                                                             \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return set_status(IB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)

int ncart_h(int l) { return (l + 1) * (l + 2) / 2; }
int pair_index_h(int la, int lb) { return la * (la + 1) / 2 + lb; }

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, cap + cap / 2);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(bytes, size_t(1) << 16);
    cudaError_t e = cudaMallocHost(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
};

struct Context {
  int device = -1;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  int nside = 40;  // INTCEPTION_B200_STREAMS, 1..64: enough for every class kernel to run concurrently
  int slice_cap[IB_NCLASS] = {};  // per class: cap on lane groups per quartet (0: no cap; INTCEPTION_B200_MAX_SLICES)
  // INTCEPTION_B200_SLICE_BOOST: slices chosen as if the grid had this many
  // times its lane groups.  The class kernels of a batch run concurrently and
  // their quartets differ widely in length; measured on the l <= 2 workload,
  // 4 shortens the last, thinly occupied waves (screened step -17 %, full
  // FP64 step -5 %) and 8 is slower again.
  int slice_boost = 4;
  double prim_tol = 0.0;  // batch entries: primitive-quartet screening tolerance (0: exact zeros only)
  // class kernels: quartets whose HRR rounding-error estimate (IB_HRR_ERR_COEF
  // x the largest weighted contracted element) exceeds this are recomputed by
  // the generic kernel (0: no check)
  double hrr_tol = 1e-13;
  cudaStream_t side[kNSideMax] = {};
  cudaEvent_t fork = nullptr, join[kNSideMax] = {};
  DevBuf boys_tab, sph, keys, vals, keys2, vals2, items, ranges, status, cub_tmp, scratch;
  DevBuf counters;  // per class kernel launch of a batch: the next quartet (FP64, FP32, FP64 recheck passes)
  DevBuf sw_quartets, sw_sizes, sw_off, sw_tmp, sw_blocks;  // Schwarz-bound work buffers
  DevBuf flags;    // per sorted item of the last batch: FP32 rejection (bit 0), on the redo list (bit 1)
  int flags_nq = 0;  // its quartet count (flags beyond it are stale)
  DevBuf redo;     // the last batch's redo lists (redo_groups of them, redo_stride ints apart; IbLaunch::redo)
  int redo_groups = 1, redo_stride = 2;
  DevBuf tickets;  // kTickets ints: the generic kernel's ticket pairs (zeroed by every dispatch)
  DevBuf kind;                                              // per class: 0 generic, 1 FP64, 2 FP64+FP32
  int kind_h[IB_NCLASS] = {};  // host copy of kind: 2 where the class has FP32 kernels and the FP32 tier uses them
  DevBuf d_stage, d_cart, d_res;
  HostBuf h_stage, h_res;
  IbClassEntry table[IB_NCLASS] = {};
  int occ[IB_NCLASS][4 * IB_NMINB] = {};
  int minb_idx[IB_NCLASS][4] = {};  // register budget chosen per class and variant (autotuned defaults)
  std::mutex mu;
};

Context* g_ctx[64] = {};
std::mutex g_ctx_mu;

// ---------------------------------------------------------------- kernels

__device__ __forceinline__ int ib_ncart_d(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int ib_pair_d(int la, int lb) { return la * (la + 1) / 2 + lb; }

// canonical order: (a,b) with la>=lb, (c,d) with lc>=ld, bra pair index >= ket pair index
__device__ __forceinline__ void ib_canon(int* s, int* l, int* st) {
  if (l[0] < l[1]) {
    int t = s[0]; s[0] = s[1]; s[1] = t;
    t = l[0]; l[0] = l[1]; l[1] = t;
    t = st[0]; st[0] = st[1]; st[1] = t;
  }
  if (l[2] < l[3]) {
    int t = s[2]; s[2] = s[3]; s[3] = t;
    t = l[2]; l[2] = l[3]; l[3] = t;
    t = st[2]; st[2] = st[3]; st[3] = t;
  }
  if (ib_pair_d(l[0], l[1]) < ib_pair_d(l[2], l[3])) {
    for (int k = 0; k < 2; ++k) {
      int t = s[k]; s[k] = s[k + 2]; s[k + 2] = t;
      t = l[k]; l[k] = l[k + 2]; l[k + 2] = t;
      t = st[k]; st[k] = st[k + 2]; st[k + 2] = t;
    }
  }
}

// ib_reverse_for_classes out of line: classify runs it for every evaluated
// quartet but it rarely does anything, and inlined its registers would lower
// the occupancy of the whole (gather-latency-bound) kernel.
__device__ __noinline__ int ib_reverse_noinline(const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                                                const double* __restrict__ prim_exp,
                                                const double* __restrict__ shell_xyz, int* s, int* l, int* st,
                                                bool fd_only) {
  return ib_reverse_for_classes(shell_k, shell_ptr, prim_exp, shell_xyz, s, l, st, fd_only);
}

__global__ void ib_classify(const int* __restrict__ quartets, const int* __restrict__ shell_l,
                            const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                            const double* __restrict__ prim_exp, const double* __restrict__ shell_xyz, int nq,
                            int lmax, const double* __restrict__ bounds, double skip_below, double thr, int mixed,
                            const int* __restrict__ kind, int route_rev, int split_min,
                            unsigned* __restrict__ keys, int* __restrict__ vals, int* status) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    int s[4], l[4], st[4] = {0, 0, 0, 0};
    bool bad = false;
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      l[i] = shell_l[s[i]];
      bad |= (l[i] < 0) | (l[i] > lmax) | (l[i] > IB_LMAX);
    }
    if (bad) {
      atomicExch(status, IB_ERR_ARG);
      for (int i = 0; i < 4; ++i) l[i] = 0;
    }
    ib_canon(s, l, st);
    const int skip = (bounds && bounds[q] < skip_below) ? 1 : 0;
    // a class kernel builds every pair on its higher-l shell; a pair whose
    // horizontal recurrence would lose too many digits that way is built on
    // the other shell by the (d f| class kernels for an (f d) pair of an
    // l <= 3 quartet (ib_reverse_for_classes).  Any other such quartet stays
    // with its class kernel while the HRR check is on (route_rev 0: the check
    // hands it to the generic kernel if its estimate is over the tolerance),
    // else goes to the generic kernel
    const int rv =
        (!skip && !bad) ? ib_reverse_noinline(shell_k, shell_ptr, prim_exp, shell_xyz, s, l, st, !route_rev) : 0;
    const int pb = ib_pair_ext(l[0], l[1]), pk = ib_pair_ext(l[2], l[3]);
    const int cid = pb * (pb + 1) / 2 + pk;
    const int nprim = shell_k[s[0]] * shell_k[s[1]] * shell_k[s[2]] * shell_k[s[3]];
    const int work = min(15, 31 - __clz(max(nprim, 1)));  // floor(log2) of the primitive quartet count
    const int k = kind[cid];
    const int gen = (!skip && (k == 0 || rv == 2)) ? 1 : 0;  // rv 2 only when route_rev
    const int fp32 = (!gen && !skip && mixed && k == 2 && bounds[q] < thr) ? 1 : 0;
    // primitive quartet counts (powers of two) descending inside a class: the
    // longest quartets start first.  The generic kernel's quartets: heavy ones
    // (split over a cluster) first, then light ones, each by a cost estimate
    // descending (primitive quartets x (contracted [e0|f0] elements + 64), in
    // quarter powers of two), whatever their class
    unsigned low = (unsigned(cid) << 4) | unsigned(15 - work);
    if (gen) {
      const long long ne = ib_ncum(l[0] + l[1]) - ib_ncum(l[0] - 1), nf = ib_ncum(l[2] + l[3]) - ib_ncum(l[2] - 1);
      const unsigned long long cost = (unsigned long long)max(nprim, 1) * (unsigned long long)(ne * nf + 64);
      const int e2 = 63 - __clzll((long long)cost);  // >= 6
      const int qc = min(255, 4 * e2 + (int)((cost >> (e2 - 2)) & 3));
      low = (unsigned(nprim < split_min) << 12) | (unsigned(255 - qc) << 4);
    }
    keys[q] = (unsigned(skip) << 15) | (unsigned(gen) << 14) | (unsigned(fp32) << 13) | low;
    vals[q] = q;
  }
}

__global__ void ib_build_items(const unsigned* __restrict__ keys, const int* __restrict__ order, int nq,
                               const int* __restrict__ quartets, const int* __restrict__ shell_l,
                               const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                               const double* __restrict__ prim_exp, const double* __restrict__ shell_xyz,
                               const long long* __restrict__ out_off, int spherical, int route_rev,
                               IbItem* __restrict__ items, int* __restrict__ ranges) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nq; p += gridDim.x * blockDim.x) {
    const int q = order[p];
    int s[4], l[4], n[4];
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      l[i] = min(max(shell_l[s[i]], 0), IB_LMAX);
      n[i] = spherical ? 2 * l[i] + 1 : ib_ncart_d(l[i]);
    }
    int st[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
    ib_canon(s, l, st);
    const unsigned key = keys[p];
    const int slot = (int)(key >> 4);  // skip*2048 + generic*1024 + fp32*512 + cid
    // the (d f| classes: the reordering classify chose (the same decision)
    if (((slot >> 10) & 3) == 0 && (slot & 511) >= IB_NPAIR * (IB_NPAIR + 1) / 2)
      ib_reverse_for_classes(shell_k, shell_ptr, prim_exp, shell_xyz, s, l, st, !route_rev);
    if (!(slot >> 11)) ib_compact_first(shell_k, shell_ptr, prim_exp, s, l, st);  // evaluated quartets only
    if (((slot >> 10) & 3) == 1) ib_orient_generic(shell_k, shell_ptr, prim_exp, shell_xyz, s, l, st);
    IbItem it;
    for (int i = 0; i < 4; ++i) {
      it.s[i] = s[i];
      it.st[i] = st[i];
    }
    it.off = out_off[q];
    items[p] = it;
    const int prev = p > 0 ? (int)(keys[p - 1] >> 4) : -1;
    const int next = p + 1 < nq ? (int)(keys[p + 1] >> 4) : -1;
    if (slot >> 11) {  // screened out: one range for all of them, sorted last
      if (prev < 0 || !(prev >> 11)) ranges[kSlotSkip] = p;
      if (next < 0) ranges[kSlotSkip + 1] = p + 1;
      continue;
    }
    if ((slot >> 10) & 1) {  // the generic kernel's quartets: a heavy range, then a light one
      // 0: not the generic kernel's, 1: heavy, 2: light
      auto state = [](int sl) { return (sl < 0 || (sl >> 10) != 1) ? 0 : 1 + ((sl >> 8) & 1); };
      const int st_p = state(slot), rs = st_p == 1 ? kSlotGenHeavy : kSlotGenLight;
      if (state(prev) != st_p) ranges[rs] = p;
      if (state(next) != st_p) ranges[rs + 1] = p + 1;
      continue;
    }
    const int cid = slot & 511, fp32 = (slot >> 9) & 1;
    const int rs = 2 * (cid + fp32 * IB_NCLASS);
    if (prev != slot) ranges[rs] = p;
    if (next != slot) ranges[rs + 1] = p + 1;
  }
}

// Screened-out quartets (bound below the skip threshold, so |(ab|cd)| <= bound):
// their blocks are written as zeros.  The kernel walks the quartets in the
// caller's order (the classify keys, unsorted, carry the skip bit), so that
// consecutive blocks usually lie next to each other in memory and the stores
// of one warp fill whole sectors.  Each lane fetches one quartet's offset and
// size (0 when it is evaluated); the warp then writes the 32 blocks.
__global__ void ib_zero_screened(const unsigned* __restrict__ keys, int nq, const int* __restrict__ quartets,
                                 const int* __restrict__ shell_l, const long long* __restrict__ out_off,
                                 int spherical, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int base = wg * 32; base < nq; base += nw * 32) {  // warp-uniform
    const int q = base + lane;
    long long off = 0;
    int tot = 0;
    if (q < nq && (keys[q] >> 15)) {
      tot = 1;
      for (int i = 0; i < 4; ++i) {
        const int l = min(max(shell_l[quartets[4 * q + i]], 0), IB_LMAX);
        tot *= spherical ? 2 * l + 1 : ib_ncart_d(l);
      }
      off = out_off[q];
    }
    unsigned any = __ballot_sync(0xffffffffu, tot > 0);
    while (any) {
      const int k = __ffs(any) - 1;
      any &= any - 1;
      const long long o = __shfl_sync(0xffffffffu, off, k);
      const int n = __shfl_sync(0xffffffffu, tot, k);
      double* __restrict__ d = out + o;
      for (int e = lane; e < n; e += 32) d[e] = 0.0;
    }
  }
}

// Analytic screening bound of every quartet: bounds[q] = Q_ab Q_cd >=
// |(ab|cd)| of every element (Cauchy-Schwarz in the Coulomb metric), Q of a
// pair the sum of the Coulomb-norm bounds of its primitive pairs
// (ib_pair_bound_rt; the triangle inequality over the contraction).  An l
// outside [0, 6] gives +inf (never screened; the batch reports it).
//
// One warp takes 16 quartets, 32 pairs (lane 2i the bra of quartet i, lane
// 2i+1 its ket).  Their primitive pairs (1 to K^2 each) form one list in pair
// order; the lanes evaluate it strided, 256 entries at a time, into shared
// memory, and each lane then adds its own pair's entries in order.  Pairs of
// different lengths no longer hold the warp to the longest one, and each Q is
// the same ordered sum as a lane looping over its own primitive pairs.
#define IB_QB_CHUNK 256
template <int MAXDEG>
__global__ void __launch_bounds__(256) ib_quartet_bounds(const int* __restrict__ quartets, int nq,
                                  const int* __restrict__ shell_l, const int* __restrict__ shell_k,
                                  const int* __restrict__ shell_ptr, const double* __restrict__ shell_xyz,
                                  const double* __restrict__ prim_exp, const double* __restrict__ prim_coef,
                                  int spherical, double* __restrict__ bounds) {
  __shared__ double val[8][IB_QB_CHUNK];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* __restrict__ v = val[wib];
  const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 16; q0 < nq; q0 += nwarp * 16) {
    const long long q = q0 + (lane >> 1);
    const int side = lane & 1;
    int n = 0, l0 = 0, l1 = 0, k1 = 1, p0 = 0, p1 = 0;
    double R = 0.0, Q = 0.0;
    if (q < nq) {
      const int s0 = __ldg(quartets + 4 * q + 2 * side), s1 = __ldg(quartets + 4 * q + 2 * side + 1);
      l0 = __ldg(shell_l + s0);
      l1 = __ldg(shell_l + s1);
      if (l0 < 0 || l1 < 0 || l0 > IB_LMAX || l1 > IB_LMAX || l0 + l1 > MAXDEG) {  // l above lmax: never screened
        Q = __longlong_as_double(0x7ff0000000000000LL);
      } else {
        k1 = __ldg(shell_k + s1);
        n = __ldg(shell_k + s0) * k1;
        p0 = __ldg(shell_ptr + s0);
        p1 = __ldg(shell_ptr + s1);
        double r2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double u = __ldg(shell_xyz + 3 * s0 + d) - __ldg(shell_xyz + 3 * s1 + d);
          r2 += u * u;
        }
        R = sqrt(r2);
      }
    }
    // this pair's first entry in the warp's list, and the list's length
    int start = n;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, start, o);
      if (lane >= o) start += t;
    }
    const int total = __shfl_sync(0xffffffffu, start, 31);
    start -= n;
    for (int c0 = 0; c0 < total; c0 += IB_QB_CHUNK) {
      for (int t = c0 + lane; t < c0 + IB_QB_CHUNK; t += 32) {
        // the pair holding entry t: the last lane whose start is <= t (binary search)
        int j = 0;
        for (int step = 16; step > 0; step >>= 1) {
          const int st = __shfl_sync(0xffffffffu, start, j + step);
          if (st <= t) j += step;
        }
        const int sj = __shfl_sync(0xffffffffu, start, j), nj = __shfl_sync(0xffffffffu, n, j);
        const int k1j = __shfl_sync(0xffffffffu, k1, j), p0j = __shfl_sync(0xffffffffu, p0, j);
        const int p1j = __shfl_sync(0xffffffffu, p1, j);
        const int l0j = __shfl_sync(0xffffffffu, l0, j), l1j = __shfl_sync(0xffffffffu, l1, j);
        const double Rj = __shfl_sync(0xffffffffu, R, j);
        if (t < total && t - sj < nj) {
          const int u = t - sj, i0 = u / k1j, i1 = u - i0 * k1j;
          const double x0 = __ldg(prim_exp + p0j + i0), c0v = __ldg(prim_coef + p0j + i0);
          const double x1 = __ldg(prim_exp + p1j + i1), c1v = __ldg(prim_coef + p1j + i1);
          v[t - c0] = ib_pair_bound_rt<MAXDEG>(l0j, l1j, spherical != 0, c0v * c1v, x0, x1, Rj);
        }
      }
      __syncwarp();
      const int a = max(start, c0), e = min(start + n, c0 + IB_QB_CHUNK);
      for (int t = a; t < e; ++t) Q += v[t - c0];
      __syncwarp();
    }
    if (n > 0) Q *= 1.000001;  // the rounding of the sum
    const double other = __shfl_xor_sync(0xffffffffu, Q, 1);
    if (q < nq && side == 0) bounds[q] = Q * other * 1.000001;
  }
}

struct ZeroFill {  // the caller's quartets whose blocks the screened path writes as zeros
  const unsigned* keys;
  int nq;
  const int* quartets;
  const int* shell_l;
  const long long* out_off;
};

// Diagonal quartets (a,b|a,b) of a chunk of shell pairs, their block sizes, and
// afterwards sqrt(max |(ij|ij)|) over the diagonal of each block.
__global__ void ib_diag_quartets(const int* __restrict__ pairs, int n, const int* __restrict__ shell_l, int spherical,
                                 int* __restrict__ quartets, long long* __restrict__ sizes) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int a = pairs[2 * p], b = pairs[2 * p + 1];
    quartets[4 * p] = a;
    quartets[4 * p + 1] = b;
    quartets[4 * p + 2] = a;
    quartets[4 * p + 3] = b;
    const int la = shell_l[a], lb = shell_l[b];
    const long long na = spherical ? 2 * la + 1 : ib_ncart_d(la), nb = spherical ? 2 * lb + 1 : ib_ncart_d(lb);
    sizes[p] = na * na * nb * nb;
  }
}

__global__ void ib_diag_max(const int* __restrict__ pairs, int n, const int* __restrict__ shell_l, int spherical,
                            const long long* __restrict__ off, const double* __restrict__ blocks, double* __restrict__ q) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int la = shell_l[pairs[2 * p]], lb = shell_l[pairs[2 * p + 1]];
    const int na = spherical ? 2 * la + 1 : ib_ncart_d(la), nb = spherical ? 2 * lb + 1 : ib_ncart_d(lb);
    const double* blk = blocks + off[p];
    double m = 0.0;
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < nb; ++j) m = fmax(m, fabs(blk[i + na * (j + nb * (i + na * j))]));
    // a diagonal below the normal range may have underflowed to 0 while
    // (ab|cd) does not: flooring it at DBL_MIN keeps q an upper bound
    q[p] = sqrt(fmax(m, 2.2250738585072014e-308)) * (1.0 + 1e-12);
  }
}

// Apply 4 spherical (or truncating) transforms index by index and emit the
// caller-ordered compact block: res[blk][ia + na*(ib + nb*(ic + nc*id))].
// One block per contraction combination; T[i] == nullptr keeps the first n[i]
// Cartesian components.
struct IbXform {
  const double* T[4];
  int l[4], n[4];
  int nblk, cart_block, res_block;
};

__global__ void ib_transform_blocks(const IbXform x, const double* __restrict__ cart, double* __restrict__ res,
                                    double* __restrict__ tmp) {
  const int blk = blockIdx.x;
  if (blk >= x.nblk) return;
  int dims[4];
  for (int i = 0; i < 4; ++i) dims[i] = ib_ncart_d(x.l[i]);
  const double* src = cart + (size_t)blk * x.cart_block;
  double* bufs[2] = {tmp + (size_t)blk * 2 * x.cart_block, tmp + (size_t)blk * 2 * x.cart_block + x.cart_block};
  int which = 0;
  // layout of src: a fastest (index ia + na*(ib + nb*(ic + nc*id)))
  for (int axis = 0; axis < 4; ++axis) {
    const int nin = dims[axis], nout = x.n[axis];
    int inner = 1, outer = 1;
    for (int k = 0; k < axis; ++k) inner *= dims[k];
    for (int k = axis + 1; k < 4; ++k) outer *= dims[k];
    double* dst = (axis == 3) ? res + (size_t)blk * x.res_block : bufs[which];
    const int total = inner * nout * outer;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int in = idx % inner, rest = idx / inner;
      const int s = rest % nout, o = rest / nout;
      double v;
      if (x.T[axis]) {
        v = 0.0;
        for (int c = 0; c < nin; ++c) v += x.T[axis][c + s * nin] * src[((size_t)o * nin + c) * inner + in];
      } else {
        v = src[((size_t)o * nin + s) * inner + in];
      }
      dst[idx] = v;
    }
    __syncthreads();
    dims[axis] = nout;
    src = dst;
    which ^= 1;
  }
}

__global__ void ib_boys_kernel(const double* __restrict__ x, int n, int nmax, const double* __restrict__ tab,
                               double* __restrict__ f) {
  double F[4 * IB_LMAX + 8];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    ib_boys_rt(x[i], nmax, tab, F);
    for (int m = 0; m <= nmax; ++m) f[(size_t)i * (nmax + 1) + m] = F[m];
  }
}

// ---------------------------------------------------------------- context

int packed_sph_size() {
  int n = 0;
  for (int l = 0; l <= IB_LMAX; ++l) n += ncart_h(l) * (2 * l + 1);
  return n;
}

int get_context(Context** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_status(IB_ERR_NODEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return set_status(IB_ERR_NODEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (!g_ctx[dev]) {
    Context* c = new Context();
    c->device = dev;
    IB_CUDA(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev));
    IB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    if (const char* env = std::getenv("INTCEPTION_B200_STREAMS")) c->nside = std::max(1, std::min(kNSideMax, std::atoi(env)));
    for (int i = 0; i < c->nside; ++i) {
      IB_CUDA(cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking));
      IB_CUDA(cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming));
    }
    IB_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    IB_CUDA(c->boys_tab.ensure(sizeof(ib_boys_host_table)));
    IB_CUDA(cudaMemcpy(c->boys_tab.p, ib_boys_host_table, sizeof(ib_boys_host_table), cudaMemcpyHostToDevice));
    std::vector<double> sph;
    build_sph_host(sph);
    IB_CUDA(c->sph.ensure(sph.size() * sizeof(double)));
    IB_CUDA(cudaMemcpy(c->sph.p, sph.data(), sph.size() * sizeof(double), cudaMemcpyHostToDevice));
    IB_CUDA(c->ranges.ensure(kNRanges * sizeof(int)));
    IB_CUDA(c->counters.ensure((kNCounters + 1) * sizeof(int)));  // + the drop-in's own
    IB_CUDA(c->status.ensure(sizeof(int)));
    IB_CUDA(cudaMemset(c->status.p, 0, sizeof(int)));
    ib_register_emitted_classes(c->table);
    std::vector<int> kind(IB_NCLASS, 0);
    for (int cid = 0; cid < IB_NCLASS; ++cid) {
      if (!c->table[cid].launch) continue;
      kind[cid] = (c->table[cid].kind == 2 && ib_tuned_fp32[cid]) ? 2 : 1;
      c->kind_h[cid] = kind[cid];
      for (int v = 0; v < 4 * IB_NMINB; ++v) c->occ[cid][v] = std::max(1, c->table[cid].occupancy(v));
      for (int v = 0; v < 4; ++v) c->minb_idx[cid][v] = std::min(std::max(ib_tuned_minb[cid][v], 0), IB_NMINB - 1);
      c->slice_cap[cid] = ib_tuned_slice_cap[cid];
    }
    if (const char* env = std::getenv("INTCEPTION_B200_SLICE_BOOST")) c->slice_boost = std::max(1, std::atoi(env));
    if (const char* env = std::getenv("INTCEPTION_B200_MAX_SLICES"))
      for (int cid = 0; cid < IB_NCLASS; ++cid) c->slice_cap[cid] = std::max(0, std::atoi(env));
    IB_CUDA(c->kind.ensure(IB_NCLASS * sizeof(int)));
    IB_CUDA(cudaMemcpy(c->kind.p, kind.data(), IB_NCLASS * sizeof(int), cudaMemcpyHostToDevice));
    IB_CUDA(cudaGetLastError());
    g_ctx[dev] = c;
  }
  *out = g_ctx[dev];
  return IB_OK;
}

IbLaunch base_launch(Context* c) {
  IbLaunch a;
  std::memset(&a, 0, sizeof(a));
  a.boys_tab = c->boys_tab.as<double>();
  a.sph = c->sph.as<double>();
  a.status = c->status.as<int>();
  a.slice_boost = c->slice_boost;
  a.split_min = ib_generic_split_min();
  return a;
}

// Scratch doubles per block of the generic kernel, for shells up to lmax.
long long generic_slice(int lmax) {
  long long best = 0;
  for (int a = 0; a <= lmax; ++a)  // every shell order: the generic kernel may build a pair on either shell
    for (int b = 0; b <= lmax; ++b)
      for (int cc = 0; cc <= lmax; ++cc)
        for (int d = 0; d <= lmax; ++d) {
          IbGenericDims g = ib_generic_dims(a, b, cc, d);
          best = std::max(best, g.total);
        }
  return (best + 31) / 32 * 32;
}

// Largest l of class cid (pair ids pb >= pk, ib_pair_ext; IB_NPAIR is (2,3)).
int class_lmax(int cid) {
  int pb = 0;
  while ((pb + 1) * (pb + 2) / 2 <= cid) ++pb;
  const int pk = cid - pb * (pb + 1) / 2;
  auto pair_lmax = [](int p) {
    if (p == IB_NPAIR) return 3;
    int la = 0;
    while ((la + 1) * (la + 2) / 2 <= p) ++la;
    return la;
  };
  return std::max(pair_lmax(pb), pair_lmax(pk));
}

// The generic kernel over the redo list of a (on stream s, after the class
// kernels that fill it); tickets: a zeroed pair (null: fixed order, no cluster).
cudaError_t redo_launch(Context* c, cudaStream_t s, const IbLaunch& a, bool sph, int lmax, int* tickets) {
  const long long slice = generic_slice(lmax);
  long long nblk = std::min<long long>((long long)ib_generic_bps() * c->nsm,
                                      (long long)(kScratchCap / (slice * sizeof(double))));
  nblk = std::max<long long>(nblk, 1);
  cudaError_t e = c->scratch.ensure((size_t)nblk * slice * sizeof(double));
  if (e != cudaSuccess) return e;
  const IbGenWork wk{-1, 0, 1, tickets, ib_generic_split() >= 1 ? kSplitRedo : 0};
  return ib_generic_launch((int)nblk, s, a, wk, sph ? 1 : 0, c->scratch.as<double>(), slice);
}

// Launch the emitted kernels for the given variants and the generic kernel;
// items/ranges already on the device.  Returns the number of kernels launched.
int dispatch(Context* c, cudaStream_t s, const IbLaunch& a, bool fp64_present, bool fp32_present, bool sph,
             int lmax, int* nlaunch, const ZeroFill* zf = nullptr) {
  // the generic kernel's tickets: pair 0 for its range launch, pair 1 + g for redo list g
  IB_CUDA(c->tickets.ensure(kTickets * sizeof(int)));
  IB_CUDA(cudaMemsetAsync(c->tickets.p, 0, kTickets * sizeof(int), s));
  int* const tk = c->tickets.as<int>();
  IB_CUDA(cudaEventRecord(c->fork, s));
  for (int i = 0; i < c->nside; ++i) IB_CUDA(cudaStreamWaitEvent(c->side[i], c->fork, 0));
  int k = 0;
  // redo lists: one per group of side streams when the batch has several
  // (the class kernels of side stream j fill list j mod G; each group's redo
  // launch follows its own class kernels and overlaps the others')
  const bool redo_on = a.redo && a.hrr_tol > 0.0;
  const int G = redo_on ? std::min(c->redo_groups, c->nside) : 1;
  // generic-kernel scratch: the range launch's region, then one per grouped redo launch
  const long long gslice = generic_slice(lmax);
  const long long gfull = std::max<long long>(
      1, std::min<long long>((long long)ib_generic_bps() * c->nsm, (long long)(kScratchCap / (gslice * sizeof(double)))));
  const long long ggroup = gfull;  // each group's redo may take the whole GPU once the others are done
  if (G > 1) IB_CUDA(c->scratch.ensure((size_t)(gfull + G * ggroup) * gslice * sizeof(double)));
  // screened quartets: zero blocks, concurrent with the class kernels (launched
  // first with 4 blocks per SM: measured no slower than 1 or 2 blocks per SM, or
  // than launching it after the class kernels)
  if (zf) {
    ib_zero_screened<<<c->nsm * 4, 256, 0, c->side[c->nside - 1]>>>(zf->keys, zf->nq, zf->quartets, zf->shell_l,
                                                                     zf->out_off, sph ? 1 : 0, a.out);
    ++*nlaunch;
  }
  // the generic kernel serves the classes without an unrolled kernel and, for
  // lmax >= 2 with the HRR check off, the quartets classify routes to it (an
  // empty range returns at once).  From lmax 3 its range is the longest job
  // of a batch, so it starts first; below, after the class kernels.
  auto launch_generic = [&]() -> cudaError_t {
    cudaError_t e = c->scratch.ensure((size_t)(gfull + (G > 1 ? G * ggroup : 0)) * gslice * sizeof(double));
    if (e != cudaSuccess) return e;
    // heavy quartets of the range over clusters too (INTCEPTION_B200_GENERIC_SPLIT 2)
    e = ib_generic_launch((int)gfull, c->side[k % c->nside], a,
                          IbGenWork{kSlotGenHeavy, kSlotGenLight, 0, tk, ib_generic_split() >= 2 ? kSplitRange : 0},
                          sph ? 1 : 0, c->scratch.as<double>(), gslice);
    ++k;
    return e;
  };
  const bool generic = (lmax > ib_lmax_emitted || lmax >= 2) && fp64_present;
  if (generic && lmax >= 3) IB_CUDA(launch_generic());
  for (int prec = 0; prec < 2; ++prec) {
    if ((prec == 0 && !fp64_present) || (prec == 1 && !fp32_present)) continue;
    IbLaunch ap = a;
    if (prec == 1) ap.ranges = a.ranges + kSlotFp32;
    const int variant = prec * 2 + (sph ? 1 : 0);
    // heaviest classes first so they start early on their streams
    for (int cid = IB_NCLASS - 1; cid >= 0; --cid) {
      if (!c->table[cid].launch || class_lmax(cid) > lmax) continue;  // no quartet of the batch has this class
      if (prec == 1 && c->kind_h[cid] != 2) continue;
      const int vt = variant + 4 * c->minb_idx[cid][variant];
      const int grid = c->nsm * c->occ[cid][vt];
      cudaStream_t ss = c->side[k % c->nside];
      if (G > 1) ap.redo = a.redo + (size_t)((k % c->nside) % G) * c->redo_stride;
      ap.max_slices = c->slice_cap[cid];
      ap.counter = c->counters.as<int>() + prec * IB_NCLASS + cid;
      c->table[cid].launch(vt, grid, ss, ap);
      ++k;
      if (prec == 1) {
        // FP64 pass over the same items: recomputes the quartets the FP32
        // kernel rejected (same stream, so it sees their flags)
        IbLaunch ar = ap;
        ar.recheck = 1;
        ar.counter = c->counters.as<int>() + 2 * IB_NCLASS + cid;
        const int v64 = sph ? 1 : 0;
        const int vt64 = v64 + 4 * c->minb_idx[cid][v64];
        c->table[cid].launch(vt64, c->nsm * c->occ[cid][vt64], ss, ar);
        ++k;
      }
    }
  }
  if (generic && lmax < 3) IB_CUDA(launch_generic());
  IB_CUDA(cudaGetLastError());
  if (G > 1) {
    // group g's redo on side stream g, after every class kernel of its streams
    for (int j = 0; j < c->nside; ++j) IB_CUDA(cudaEventRecord(c->join[j], c->side[j]));
    for (int g = 0; g < G; ++g) {
      for (int j = g; j < c->nside; j += G)
        if (j != g) IB_CUDA(cudaStreamWaitEvent(c->side[g], c->join[j], 0));
      IbLaunch ag = a;
      ag.redo = a.redo + (size_t)g * c->redo_stride;
      const IbGenWork wk{-1, 0, 1, tk + 2 * (1 + g), ib_generic_split() >= 1 ? kSplitRedo : 0};
      IB_CUDA(ib_generic_launch((int)ggroup, c->side[g], ag, wk, sph ? 1 : 0,
                                c->scratch.as<double>() + (size_t)(gfull + g * ggroup) * gslice, gslice));
      ++k;
    }
  }
  for (int i = 0; i < c->nside; ++i) {
    IB_CUDA(cudaEventRecord(c->join[i], c->side[i]));
    IB_CUDA(cudaStreamWaitEvent(s, c->join[i], 0));
  }
  // one redo list: after every class kernel (an empty list returns at once)
  if (redo_on && G == 1) {
    IB_CUDA(redo_launch(c, s, a, sph, lmax, tk + 2));
    ++k;
  }
  *nlaunch += k;
  return IB_OK;
}

// ---------------------------------------------------------------- drop-in

struct DropShell {
  const double* x;
  const double* cen;
  int l, n, iskip, nprim, ncont, iskip_cont;
  const double* coef;
  const double* T;
};

int dropin(DropShell* sh, bool sph, double* output_array) {
  for (int i = 0; i < 4; ++i) {
    const DropShell& s = sh[i];
    if (s.l < 0 || s.l > IB_LMAX)
      return set_status(IB_ERR_ARG, "angular momentum outside [0, " + std::to_string(IB_LMAX) + "]");
    const int natural = sph ? 2 * s.l + 1 : ncart_h(s.l);
    if (s.n != natural)
      return set_status(IB_ERR_ARG, "n? must equal the component count of l? ((l+1)(l+2)/2 Cartesian, 2l+1 spherical)");
    if (s.nprim < 1 || s.ncont < 1 || s.nprim > 64) return set_status(IB_ERR_ARG, "need 1 <= n?_prim <= 64, n?_cont >= 1");
    if (!s.x || !s.cen || !s.coef || (sph && !s.T)) return set_status(IB_ERR_ARG, "null input pointer");
  }
  if (!output_array) return set_status(IB_ERR_ARG, "null output_array");
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  IB_CUDA(cudaSetDevice(c->device));
  // virtual shells: one per (index, contracted function)
  int nshell = 0, nprim = 0;
  int shell0[4];
  for (int i = 0; i < 4; ++i) {
    shell0[i] = nshell;
    nshell += sh[i].ncont;
    nprim += sh[i].ncont * sh[i].nprim;
  }
  const int nblk = sh[0].ncont * sh[1].ncont * sh[2].ncont * sh[3].ncont;
  int nc[4];
  for (int i = 0; i < 4; ++i) nc[i] = ncart_h(sh[i].l);
  const int cart_block = nc[0] * nc[1] * nc[2] * nc[3];
  const int res_block = sh[0].n * sh[1].n * sh[2].n * sh[3].n;
  int tsize[4] = {0, 0, 0, 0};
  if (sph)
    for (int i = 0; i < 4; ++i) tsize[i] = nc[i] * (2 * sh[i].l + 1);
  // host staging layout
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  size_t o_l = 0;
  size_t o_k = al(o_l + nshell * sizeof(int));
  size_t o_p = al(o_k + nshell * sizeof(int));
  size_t o_xyz = al(o_p + nshell * sizeof(int));
  size_t o_e = al(o_xyz + 3 * nshell * sizeof(double));
  size_t o_c = al(o_e + nprim * sizeof(double));
  size_t o_it = al(o_c + nprim * sizeof(double));
  size_t o_rg = al(o_it + nblk * sizeof(IbItem));
  size_t o_T[4];
  size_t cur = al(o_rg + kNRanges * sizeof(int));
  for (int i = 0; i < 4; ++i) {
    o_T[i] = cur;
    cur = al(cur + tsize[i] * sizeof(double));
  }
  const size_t total = cur;
  IB_CUDA(c->h_stage.ensure(total));
  IB_CUDA(c->d_stage.ensure(total));
  char* h = static_cast<char*>(c->h_stage.p);
  int* hl = reinterpret_cast<int*>(h + o_l);
  int* hk = reinterpret_cast<int*>(h + o_k);
  int* hp = reinterpret_cast<int*>(h + o_p);
  double* hxyz = reinterpret_cast<double*>(h + o_xyz);
  double* he = reinterpret_cast<double*>(h + o_e);
  double* hc = reinterpret_cast<double*>(h + o_c);
  IbItem* hit = reinterpret_cast<IbItem*>(h + o_it);
  int* hrg = reinterpret_cast<int*>(h + o_rg);
  int ps = 0;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < sh[i].ncont; ++k) {
      const int s = shell0[i] + k;
      hl[s] = sh[i].l;
      hk[s] = sh[i].nprim;
      hp[s] = ps;
      for (int d = 0; d < 3; ++d) hxyz[3 * s + d] = sh[i].cen[d];
      for (int p = 0; p < sh[i].nprim; ++p) {
        he[ps + p] = sh[i].x[p];
        hc[ps + p] = sh[i].coef[p + k * sh[i].nprim];
      }
      ps += sh[i].nprim;
    }
  // canonical permutation, shared by every combination
  int lperm[4] = {sh[0].l, sh[1].l, sh[2].l, sh[3].l};
  int sperm[4] = {0, 1, 2, 3};
  int stperm[4] = {1, nc[0], nc[0] * nc[1], nc[0] * nc[1] * nc[2]};
  auto swp = [&](int i, int j) {
    std::swap(lperm[i], lperm[j]);
    std::swap(sperm[i], sperm[j]);
    std::swap(stperm[i], stperm[j]);
  };
  if (lperm[0] < lperm[1]) swp(0, 1);
  if (lperm[2] < lperm[3]) swp(2, 3);
  if (pair_index_h(lperm[0], lperm[1]) < pair_index_h(lperm[2], lperm[3])) {
    swp(0, 2);
    swp(1, 3);
  }
  // within a pair of equal l the more compact shell first (as the batch entries do)
  auto min_exp = [&](int i) { return *std::min_element(sh[i].x, sh[i].x + sh[i].nprim); };
  for (int i = 0; i < 4; i += 2)
    if (lperm[i] == lperm[i + 1] && min_exp(sperm[i]) < min_exp(sperm[i + 1])) swp(i, i + 1);
  const int pb = pair_index_h(lperm[0], lperm[1]), pk = pair_index_h(lperm[2], lperm[3]);
  const int cid = pb * (pb + 1) / 2 + pk;
  // pairs whose horizontal recurrence is ill-conditioned when built on the
  // higher-l shell are built on the other one, by the generic kernel (as the
  // batch entries route them)
  bool rev[2] = {false, false};
  for (int i = 0; i < 4; i += 2) {
    const DropShell& s0 = sh[sperm[i]];
    const DropShell& s1 = sh[sperm[i + 1]];
    double R2 = 0.0;
    for (int d = 0; d < 3; ++d) R2 += (s0.cen[d] - s1.cen[d]) * (s0.cen[d] - s1.cen[d]);
    rev[i / 2] = ib_pair_reverse(lperm[i], lperm[i + 1], s0.nprim, s1.nprim, s0.x, s1.x, std::sqrt(R2));
  }
  // (f d) pairs of an l <= 3 quartet: the (d f| class kernels; any other: generic
  bool route = false, to_class = rev[0] || rev[1];
  for (int h = 0; h < 2; ++h)
    if (rev[h] && !(lperm[2 * h] == 3 && lperm[2 * h + 1] == 2)) to_class = false;
  if (std::max(std::max(lperm[0], lperm[1]), std::max(lperm[2], lperm[3])) > 3) to_class = false;
  // with the HRR check on, a reversed pair that no (d f| kernel serves stays
  // with the class kernel in its canonical order (the check redoes it if needed)
  if (!to_class && (rev[0] || rev[1])) route = !(c->hrr_tol > 0.0);
  if (to_class || route)
    for (int h = 0; h < 2; ++h)
      if (rev[h]) swp(2 * h, 2 * h + 1);
  if (to_class && ib_pair_ext(lperm[0], lperm[1]) < ib_pair_ext(lperm[2], lperm[3])) {
    swp(0, 2);
    swp(1, 3);
  }
  const int pbx = ib_pair_ext(lperm[0], lperm[1]), pkx = ib_pair_ext(lperm[2], lperm[3]);
  const int cidx = to_class ? pbx * (pbx + 1) / 2 + pkx : cid;
  int b = 0;
  for (int ka = 0; ka < sh[0].ncont; ++ka)
    for (int kb = 0; kb < sh[1].ncont; ++kb)
      for (int kc = 0; kc < sh[2].ncont; ++kc)
        for (int kd = 0; kd < sh[3].ncont; ++kd, ++b) {
          const int orig[4] = {shell0[0] + ka, shell0[1] + kb, shell0[2] + kc, shell0[3] + kd};
          IbItem it;
          for (int i = 0; i < 4; ++i) {
            it.s[i] = orig[sperm[i]];
            it.st[i] = stperm[i];
          }
          it.off = (long long)b * cart_block;
          hit[b] = it;
        }
  std::memset(hrg, 0, kNRanges * sizeof(int));
  const bool emitted = c->table[cidx].launch != nullptr && !route;
  if (emitted) {
    hrg[2 * cidx] = 0;
    hrg[2 * cidx + 1] = nblk;
  } else {
    hrg[kSlotGenLight] = 0;  // one block per item (no cluster split in the drop-in)
    hrg[kSlotGenLight + 1] = nblk;
  }
  for (int i = 0; i < 4; ++i)
    if (sph) std::memcpy(h + o_T[i], sh[i].T, tsize[i] * sizeof(double));
  IB_CUDA(c->d_cart.ensure((size_t)nblk * cart_block * sizeof(double)));
  IB_CUDA(c->d_res.ensure((size_t)nblk * (res_block + 2 * cart_block) * sizeof(double)));
  IB_CUDA(c->h_res.ensure((size_t)nblk * res_block * sizeof(double)));
  cudaStream_t s = c->stream;
  char* d = static_cast<char*>(c->d_stage.p);
  IB_CUDA(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, s));
  IbLaunch a = base_launch(c);
  a.items = reinterpret_cast<const IbItem*>(d + o_it);
  a.ranges = reinterpret_cast<const int*>(d + o_rg);
  a.shell_l = reinterpret_cast<const int*>(d + o_l);
  a.shell_k = reinterpret_cast<const int*>(d + o_k);
  a.shell_ptr = reinterpret_cast<const int*>(d + o_p);
  a.shell_xyz = reinterpret_cast<const double*>(d + o_xyz);
  a.prim_exp = reinterpret_cast<const double*>(d + o_e);
  a.prim_coef = reinterpret_cast<const double*>(d + o_c);
  a.out = c->d_cart.as<double>();
  IB_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(int), s));
  if (emitted) {
    const int vt = 4 * c->minb_idx[cidx][0];
    const int grid = std::max(1, std::min(c->nsm * c->occ[cidx][vt], (nblk + IB_BLOCK - 1) / IB_BLOCK));
    a.counter = c->counters.as<int>() + kNCounters;  // never used by a batch that may still run
    IB_CUDA(cudaMemsetAsync(a.counter, 0, sizeof(int), s));
    IB_CUDA(c->flags.ensure((size_t)nblk * sizeof(int)));
    IB_CUDA(cudaMemsetAsync(c->flags.p, 0, (size_t)nblk * sizeof(int), s));
    IB_CUDA(c->redo.ensure((size_t)(nblk + 2) * sizeof(int)));
    IB_CUDA(cudaMemsetAsync(c->redo.p, 0, 2 * sizeof(int), s));
    c->redo_groups = 1;
    c->redo_stride = nblk + 2;
    c->flags_nq = nblk;
    a.flags = c->flags.as<int>();
    a.redo = c->redo.as<int>();
    a.redo_cap = nblk;
    a.hrr_tol = c->hrr_tol;
    c->table[cidx].launch(vt, grid, s, a);
    if (a.hrr_tol > 0.0)
      IB_CUDA(redo_launch(c, s, a, false, std::max(std::max(sh[0].l, sh[1].l), std::max(sh[2].l, sh[3].l)),
                          nullptr));
  } else {
    const long long slice = generic_slice(std::max(std::max(sh[0].l, sh[1].l), std::max(sh[2].l, sh[3].l)));
    long long nb = std::min<long long>({(long long)nblk, (long long)ib_generic_bps() * c->nsm,
                                        (long long)(kScratchCap / (slice * sizeof(double)))});
    nb = std::max<long long>(nb, 1);
    IB_CUDA(c->scratch.ensure((size_t)nb * slice * sizeof(double)));
    IB_CUDA(ib_generic_launch((int)nb, s, a, IbGenWork{-1, kSlotGenLight, 0, nullptr}, 0, c->scratch.as<double>(),
                              slice));
  }
  IB_CUDA(cudaGetLastError());
  IbXform x;
  for (int i = 0; i < 4; ++i) {
    x.T[i] = sph ? reinterpret_cast<const double*>(d + o_T[i]) : nullptr;
    x.l[i] = sh[i].l;
    x.n[i] = sh[i].n;
  }
  x.nblk = nblk;
  x.cart_block = cart_block;
  x.res_block = res_block;
  double* dres = c->d_res.as<double>();
  ib_transform_blocks<<<nblk, 128, 0, s>>>(x, c->d_cart.as<double>(), dres, dres + (size_t)nblk * res_block);
  IB_CUDA(cudaGetLastError());
  int hstatus = 0;
  IB_CUDA(cudaMemcpyAsync(c->h_res.p, dres, (size_t)nblk * res_block * sizeof(double), cudaMemcpyDeviceToHost, s));
  IB_CUDA(cudaMemcpyAsync(&hstatus, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  IB_CUDA(cudaStreamSynchronize(s));
  if (hstatus) return set_status(hstatus, "device kernel reported status " + std::to_string(hstatus));
  // place the compact result at the caller's strides (the emitted code's final
  // copy loop, contracted_general.py:1808-1876)
  const double* r = static_cast<const double*>(c->h_res.p);
  b = 0;
  for (int ka = 0; ka < sh[0].ncont; ++ka)
    for (int kb = 0; kb < sh[1].ncont; ++kb)
      for (int kc = 0; kc < sh[2].ncont; ++kc)
        for (int kd = 0; kd < sh[3].ncont; ++kd, ++b) {
          const long long base = (long long)ka * sh[0].iskip_cont + (long long)kb * sh[1].iskip_cont +
                                 (long long)kc * sh[2].iskip_cont + (long long)kd * sh[3].iskip_cont;
          const double* rb = r + (size_t)b * res_block;
          int e = 0;
          for (int id = 0; id < sh[3].n; ++id)
            for (int ic = 0; ic < sh[2].n; ++ic)
              for (int ib = 0; ib < sh[1].n; ++ib)
                for (int ia = 0; ia < sh[0].n; ++ia, ++e)
                  output_array[base + (long long)ia * sh[0].iskip + (long long)ib * sh[1].iskip +
                               (long long)ic * sh[2].iskip + (long long)id * sh[3].iskip] = rb[e];
        }
  return set_status(IB_OK, "");
}

// contracted_general.py:240-502, integer formula emitted as <class>_work_array_size
int ncum_h(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }
int work_array_size(int la, int lb, int lc, int ld, int ka, int kb, int kc, int kd, int ca, int cb, int cc, int cd) {
  const int nw = ncum_h(la + lb) * ncum_h(lc) * ncum_h(ld);
  int n1 = ka * kb * kd * kc;
  int mem1 = 2 * (nw * n1 + ld + lc + la + lb + 1);
  int n2 = ca * kb * kd * kc;
  if (n1 < n2) n1 = n2;
  n2 = ca * cb * kd * kc;
  if (n1 < n2) n1 = n2;
  n2 = ca * cb * cd * kc;
  if (n1 < n2) n1 = n2;
  n2 = ca * cb * cd * cc;
  if (n1 < n2) n1 = n2;
  int mem2 = 2 * nw * n1;
  if (mem2 > mem1) mem1 = mem2;
  n1 = ca * cb * cd * cc;
  int layer = 0;  // generator.py:1112-1157 hrr_layer[lb][la]
  for (int j = 0; j <= lb; ++j) layer = std::max(layer, (ncum_h(la + lb - j) - ncum_h(la - 1)) * ncart_h(j));
  mem2 = 2 * layer * ncart_h(lc) * ncart_h(ld) * n1;
  if (mem2 > mem1) mem1 = mem2;
  mem2 = 2 * ncart_h(lc) * ncart_h(ld) * ncart_h(lb) * ncart_h(la) * n1;
  if (mem2 > mem1) mem1 = mem2;
  return mem1;
}

// ---------------------------------------------------------------- sph matrices
double dfact(int n) {
  double r = 1.0;
  while (n > 1) {
    r *= n;
    n -= 2;
  }
  return r;
}
double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

void sph_matrix_host(int l, double* T) {
  const int nc = ncart_h(l), ns = 2 * l + 1;
  std::vector<int> cx, cy, cz;
  for (int mx = l; mx >= 0; --mx)
    for (int my = l - mx; my >= 0; --my) {
      cx.push_back(mx);
      cy.push_back(my);
      cz.push_back(l - mx - my);
    }
  auto idx = [&](int i, int j, int k) {
    for (int c = 0; c < nc; ++c)
      if (cx[c] == i && cy[c] == j && cz[c] == k) return c;
    return -1;
  };
  for (int c = 0; c < nc * ns; ++c) T[c] = 0.0;
  for (int col = 0; col < ns; ++col) {
    const int m = col - l, am = std::abs(m);
    const double vm = m < 0 ? 0.5 : 0.0;
    for (int t = 0; t <= (l - am) / 2; ++t)
      for (int u = 0; u <= t; ++u)
        for (double v = vm; v <= std::floor(am / 2.0 - vm) + vm + 1e-9; v += 1.0) {
          const int two_v = (int)std::lround(2 * v);
          const double sign = ((int)std::lround(t + v - vm) % 2) ? -1.0 : 1.0;
          const double coef = sign * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) * binom(t, u) *
                              binom(am, two_v);
          const int i = 2 * t + am - 2 * u - two_v, j = 2 * u + two_v, k = l - 2 * t - am;
          const int c = idx(i, j, k);
          if (c >= 0 && coef != 0.0) T[c + col * nc] += coef;
        }
    // scale to the norm of x^l (monomial overlaps up to an l-only factor)
    double nrm = 0.0;
    for (int p = 0; p < nc; ++p)
      for (int q = 0; q < nc; ++q) {
        const int a = cx[p] + cx[q], bq = cy[p] + cy[q], cq = cz[p] + cz[q];
        if ((a | bq | cq) & 1) continue;
        nrm += T[p + col * nc] * T[q + col * nc] * dfact(a - 1) * dfact(bq - 1) * dfact(cq - 1);
      }
    const double sc = std::sqrt(dfact(2 * l - 1) / nrm);
    for (int p = 0; p < nc; ++p) T[p + col * nc] *= sc;
  }
}

}  // namespace

void build_sph_host(std::vector<double>& out) {
  out.assign(packed_sph_size(), 0.0);
  for (int l = 0; l <= IB_LMAX; ++l) sph_matrix_host(l, out.data() + ib_sph_offset(l));
}

// Sets the calling thread's status word (intception_b200_last_status/_last_error)
// for entry points defined in other translation units.
int ib_runtime_set_status(int st, const char* msg) { return set_status(st, msg ? msg : ""); }

namespace {
// The caller's stream; NULL is the legacy default stream (CUDA's convention).
int resolve_stream(Context* c, void* stream, cudaStream_t* s) {
  (void)c;
  *s = static_cast<cudaStream_t>(stream);
  return IB_OK;
}

// The batch pipeline on stream s; the caller holds the context lock.
int batch_impl(Context* c, const intception_b200_basis* basis, const int* quartets, const long long* out_off, int nq,
               int spherical, int precision, const double* bounds, double skip_below, double fp32_below,
               double mixed_tol, double* out, cudaStream_t s, int* nl, bool screen_prims = true) {
  if (!basis || nq < 0 || (nq > 0 && (!quartets || !out_off || !out)))
    return set_status(IB_ERR_ARG, "eri_batch: null argument");
  if (basis->lmax < 0 || basis->lmax > IB_LMAX) return set_status(IB_ERR_ARG, "eri_batch: basis lmax out of range");
  if (precision != IB_PREC_FP64 && precision != IB_PREC_MIXED) return set_status(IB_ERR_ARG, "eri_batch: precision");
  if ((precision == IB_PREC_MIXED || skip_below > 0.0) && !bounds)
    return set_status(IB_ERR_ARG, "eri_batch: mixed precision and screening need bounds");
  if (nq == 0) return set_status(IB_OK, "");
  IB_CUDA(c->keys.ensure((size_t)nq * sizeof(unsigned)));
  IB_CUDA(c->keys2.ensure((size_t)nq * sizeof(unsigned)));
  IB_CUDA(c->vals.ensure((size_t)nq * sizeof(int)));
  IB_CUDA(c->vals2.ensure((size_t)nq * sizeof(int)));
  IB_CUDA(c->items.ensure((size_t)nq * sizeof(IbItem)));
  size_t tmp_bytes = 0;
  IB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, c->keys.as<unsigned>(), c->keys2.as<unsigned>(),
                                          c->vals.as<int>(), c->vals2.as<int>(), nq, 0, kKeyBits, s));
  IB_CUDA(c->cub_tmp.ensure(tmp_bytes));
  IB_CUDA(cudaMemsetAsync(c->ranges.p, 0, kNRanges * sizeof(int), s));
  IB_CUDA(cudaMemsetAsync(c->counters.p, 0, kNCounters * sizeof(int), s));
  IB_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(int), s));
  const int grid = std::min((nq + 255) / 256, c->nsm * 16);
  const bool use_bounds = bounds != nullptr && (precision == IB_PREC_MIXED || skip_below > 0.0);
  ib_classify<<<grid, 256, 0, s>>>(quartets, basis->shell_l, basis->shell_k, basis->shell_ptr, basis->prim_exp,
                                   basis->shell_xyz, nq, basis->lmax,
                                   use_bounds ? bounds : nullptr, skip_below, fp32_below,
                                   precision == IB_PREC_MIXED ? 1 : 0, c->kind.as<int>(), c->hrr_tol > 0.0 ? 0 : 1,
                                   ib_generic_split_min(), c->keys.as<unsigned>(),
                                   c->vals.as<int>(), c->status.as<int>());
  ++*nl;
  IB_CUDA(cudaGetLastError());
  IB_CUDA(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp_bytes, c->keys.as<unsigned>(), c->keys2.as<unsigned>(),
                                          c->vals.as<int>(), c->vals2.as<int>(), nq, 0, kKeyBits, s));
  ib_build_items<<<grid, 256, 0, s>>>(c->keys2.as<unsigned>(), c->vals2.as<int>(), nq, quartets, basis->shell_l,
                                      basis->shell_k, basis->shell_ptr, basis->prim_exp, basis->shell_xyz, out_off,
                                      spherical ? 1 : 0, c->hrr_tol > 0.0 ? 0 : 1, c->items.as<IbItem>(),
                                      c->ranges.as<int>());
  ++*nl;
  IB_CUDA(cudaGetLastError());
  IbLaunch a = base_launch(c);
  a.items = c->items.as<IbItem>();
  a.ranges = c->ranges.as<int>();
  a.shell_l = basis->shell_l;
  a.shell_k = basis->shell_k;
  a.shell_ptr = basis->shell_ptr;
  a.shell_xyz = basis->shell_xyz;
  a.prim_exp = basis->prim_exp;
  a.prim_coef = basis->prim_coef;
  a.out = out;
  a.prim_tol = screen_prims ? c->prim_tol : 0.0;
  IB_CUDA(c->flags.ensure((size_t)nq * sizeof(int)));
  IB_CUDA(cudaMemsetAsync(c->flags.p, 0, (size_t)nq * sizeof(int), s));
  // l >= 3 batches: four redo lists, one per group of side streams (dispatch)
  c->redo_groups = (basis->lmax >= 3 && c->hrr_tol > 0.0) ? kRedoGroups : 1;
  c->redo_stride = nq + 2;
  IB_CUDA(c->redo.ensure((size_t)c->redo_groups * (nq + 2) * sizeof(int)));
  for (int g = 0; g < c->redo_groups; ++g)
    IB_CUDA(cudaMemsetAsync(c->redo.as<int>() + (size_t)g * (nq + 2), 0, 2 * sizeof(int), s));
  c->flags_nq = nq;
  a.flags = c->flags.as<int>();
  a.redo = c->redo.as<int>();
  a.redo_cap = nq;
  a.hrr_tol = c->hrr_tol;
  if (precision == IB_PREC_MIXED) a.mixed_tol = mixed_tol;
  const ZeroFill zf = {c->keys.as<unsigned>(), nq, quartets, basis->shell_l, out_off};
  return dispatch(c, s, a, true, precision == IB_PREC_MIXED, spherical != 0, basis->lmax, nl,
                  use_bounds && skip_below > 0.0 ? &zf : nullptr);
}
}  // namespace

// ================================================================ C ABI
extern "C" {

void intception_integral_eri_abcd_m_cont_cart_main(
    const double* xa, const double cA[3], const int la, const int na, const int iskipa, const int na_prim,
    const int na_cont, const int iskipa_cont, const double* contract_array_a, const double* xb, const double cB[3],
    const int lb, const int nb, const int iskipb, const int nb_prim, const int nb_cont, const int iskipb_cont,
    const double* contract_array_b, const double* xc, const double cC[3], const int lc, const int nc,
    const int iskipc, const int nc_prim, const int nc_cont, const int iskipc_cont, const double* contract_array_c,
    const double* xd, const double cD[3], const int ld, const int nd, const int iskipd, const int nd_prim,
    const int nd_cont, const int iskipd_cont, const double* contract_array_d, double* work_array,
    double* output_array) {
  (void)work_array;
  DropShell sh[4] = {{xa, cA, la, na, iskipa, na_prim, na_cont, iskipa_cont, contract_array_a, nullptr},
                     {xb, cB, lb, nb, iskipb, nb_prim, nb_cont, iskipb_cont, contract_array_b, nullptr},
                     {xc, cC, lc, nc, iskipc, nc_prim, nc_cont, iskipc_cont, contract_array_c, nullptr},
                     {xd, cD, ld, nd, iskipd, nd_prim, nd_cont, iskipd_cont, contract_array_d, nullptr}};
  dropin(sh, false, output_array);
}

int intception_integral_eri_abcd_m_cont_cart_work_array_size(const int la, const int lb, const int lc,
                                                              const int ld, const int na_prim, const int nb_prim,
                                                              const int nc_prim, const int nd_prim,
                                                              const int na_cont, const int nb_cont,
                                                              const int nc_cont, const int nd_cont) {
  return work_array_size(la, lb, lc, ld, na_prim, nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont);
}

void intception_integral_eri_abcd_m_cont_sph_main(
    const double* xa, const double cA[3], const int la, const int na, const int iskipa, const int na_prim,
    const int na_cont, const int iskipa_cont, const double* contract_array_a, const double* sph_trans_array_a,
    const double* xb, const double cB[3], const int lb, const int nb, const int iskipb, const int nb_prim,
    const int nb_cont, const int iskipb_cont, const double* contract_array_b, const double* sph_trans_array_b,
    const double* xc, const double cC[3], const int lc, const int nc, const int iskipc, const int nc_prim,
    const int nc_cont, const int iskipc_cont, const double* contract_array_c, const double* sph_trans_array_c,
    const double* xd, const double cD[3], const int ld, const int nd, const int iskipd, const int nd_prim,
    const int nd_cont, const int iskipd_cont, const double* contract_array_d, const double* sph_trans_array_d,
    double* work_array, double* output_array) {
  (void)work_array;
  DropShell sh[4] = {{xa, cA, la, na, iskipa, na_prim, na_cont, iskipa_cont, contract_array_a, sph_trans_array_a},
                     {xb, cB, lb, nb, iskipb, nb_prim, nb_cont, iskipb_cont, contract_array_b, sph_trans_array_b},
                     {xc, cC, lc, nc, iskipc, nc_prim, nc_cont, iskipc_cont, contract_array_c, sph_trans_array_c},
                     {xd, cD, ld, nd, iskipd, nd_prim, nd_cont, iskipd_cont, contract_array_d, sph_trans_array_d}};
  dropin(sh, true, output_array);
}

int intception_integral_eri_abcd_m_cont_sph_work_array_size(const int la, const int lb, const int lc,
                                                             const int ld, const int na_prim, const int nb_prim,
                                                             const int nc_prim, const int nd_prim,
                                                             const int na_cont, const int nb_cont,
                                                             const int nc_cont, const int nd_cont) {
  return work_array_size(la, lb, lc, ld, na_prim, nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont);
}

int intception_b200_last_status(void) { return tl_status; }
const char* intception_b200_last_error(void) { return tl_msg.c_str(); }
int intception_b200_lmax(void) { return IB_LMAX; }
int intception_b200_last_launch_count(void) { return tl_launches; }

int intception_b200_sph_matrix(int l, double* T) {
  if (l < 0 || l > IB_LMAX || !T) return set_status(IB_ERR_ARG, "l out of range or null T");
  sph_matrix_host(l, T);
  return set_status(IB_OK, "");
}

int intception_b200_boys_batch(const double* x, int n, int nmax, double* f, void* stream) {
  if (n < 0 || nmax < 0 || nmax > 4 * IB_LMAX || (n > 0 && (!x || !f)))
    return set_status(IB_ERR_ARG, "boys_batch: bad arguments");
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  if (n == 0) return set_status(IB_OK, "");
  cudaStream_t s;
  resolve_stream(c, stream, &s);
  const int grid = std::min((n + 255) / 256, c->nsm * 8);
  ib_boys_kernel<<<grid, 256, 0, s>>>(x, n, nmax, c->boys_tab.as<double>(), f);
  IB_CUDA(cudaGetLastError());
  return set_status(IB_OK, "");
}

void intception_boys(double* f, const int ifskip, const int nmin, const int nmax, const double x) {
  if (!f || nmin < 0 || nmax < nmin || nmax > 4 * IB_LMAX || !(x >= 0.0)) {
    set_status(IB_ERR_ARG, "intception_boys: bad arguments");
    return;
  }
  Context* c = nullptr;
  if (get_context(&c)) return;
  std::lock_guard<std::mutex> lk(c->mu);
  if (c->h_stage.ensure(64 * sizeof(double)) != cudaSuccess || c->d_stage.ensure(64 * sizeof(double)) != cudaSuccess) {
    set_status(IB_ERR_CUDA, "intception_boys: allocation failed");
    return;
  }
  double* h = static_cast<double*>(c->h_stage.p);
  double* d = c->d_stage.as<double>();
  h[0] = x;
  cudaStream_t s = c->stream;
  cudaMemcpyAsync(d, h, sizeof(double), cudaMemcpyHostToDevice, s);
  ib_boys_kernel<<<1, 32, 0, s>>>(d, 1, nmax, c->boys_tab.as<double>(), d + 8);
  cudaMemcpyAsync(h + 8, d + 8, (nmax + 1) * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_status(IB_ERR_CUDA, std::string("intception_boys: ") + cudaGetErrorString(e));
    return;
  }
  for (int m = nmin; m <= nmax; ++m) f[m * ifskip] = h[8 + m];
  set_status(IB_OK, "");
}

int intception_b200_synchronize(void) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  IB_CUDA(cudaStreamSynchronize(c->stream));
  return set_status(IB_OK, "");
}

int intception_b200_eri_batch(const intception_b200_basis* basis, const int* quartets, const long long* out_off,
                              int nq, int spherical, int precision, const double* bounds, double skip_below,
                              double fp32_below, double mixed_tol, double* out, void* stream) {
  tl_launches = 0;
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t s;
  resolve_stream(c, stream, &s);
  int nl = 0;
  st = batch_impl(c, basis, quartets, out_off, nq, spherical, precision, bounds, skip_below, fp32_below, mixed_tol,
                  out, s, &nl);
  tl_launches = nl;
  if (st) return st;
  return set_status(IB_OK, "");
}

int intception_b200_schwarz(const intception_b200_basis* basis, const int* pairs, int npairs, int spherical,
                            double* q, void* stream) {
  if (!basis || npairs < 0 || (npairs > 0 && (!pairs || !q))) return set_status(IB_ERR_ARG, "schwarz: null argument");
  if (npairs == 0) return set_status(IB_OK, "");
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t s;
  resolve_stream(c, stream, &s);
  const int chunk = 1 << 17;
  IB_CUDA(c->sw_quartets.ensure((size_t)chunk * 4 * sizeof(int)));
  IB_CUDA(c->sw_sizes.ensure((size_t)(chunk + 1) * sizeof(long long)));
  IB_CUDA(c->sw_off.ensure((size_t)(chunk + 1) * sizeof(long long)));
  size_t tmp = 0;
  IB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, c->sw_sizes.as<long long>(), c->sw_off.as<long long>(),
                                        chunk + 1, s));
  IB_CUDA(c->sw_tmp.ensure(tmp));
  for (int p0 = 0; p0 < npairs; p0 += chunk) {
    const int n = std::min(chunk, npairs - p0);
    const int grid = std::min((n + 255) / 256, c->nsm * 8);
    IB_CUDA(cudaMemsetAsync(c->sw_sizes.as<long long>() + n, 0, sizeof(long long), s));
    ib_diag_quartets<<<grid, 256, 0, s>>>(pairs + 2 * (size_t)p0, n, basis->shell_l, spherical ? 1 : 0,
                                          c->sw_quartets.as<int>(), c->sw_sizes.as<long long>());
    IB_CUDA(cudaGetLastError());
    IB_CUDA(cub::DeviceScan::ExclusiveSum(c->sw_tmp.p, tmp, c->sw_sizes.as<long long>(), c->sw_off.as<long long>(),
                                          n + 1, s));
    long long total = 0;
    IB_CUDA(cudaMemcpyAsync(&total, c->sw_off.as<long long>() + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
    IB_CUDA(cudaStreamSynchronize(s));
    IB_CUDA(c->sw_blocks.ensure((size_t)total * sizeof(double)));
    int nl = 0;
    st = batch_impl(c, basis, c->sw_quartets.as<int>(), c->sw_off.as<long long>(), n, spherical, IB_PREC_FP64,
                    nullptr, 0.0, 0.0, 0.0, c->sw_blocks.as<double>(), s, &nl,
                    false);
    if (st) return st;
    ib_diag_max<<<grid, 256, 0, s>>>(pairs + 2 * (size_t)p0, n, basis->shell_l, spherical ? 1 : 0,
                                     c->sw_off.as<long long>(), c->sw_blocks.as<double>(), q + p0);
    IB_CUDA(cudaGetLastError());
  }
  return set_status(IB_OK, "");
}

int intception_b200_quartet_bounds(const intception_b200_basis* basis, const int* quartets, int nq, int spherical,
                                   double* bounds, void* stream) {
  if (!basis || nq < 0 || (nq > 0 && (!quartets || !bounds)))
    return set_status(IB_ERR_ARG, "quartet_bounds: null argument");
  if (nq == 0) return set_status(IB_OK, "");
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  cudaStream_t s;
  resolve_stream(c, stream, &s);
  const long long warps = (nq + 15) / 16;  // 16 quartets per warp, 8 warps per block
  const int grid = (int)std::min<long long>((warps + 7) / 8, (long long)c->nsm * 16);
  if (basis->lmax < 0 || basis->lmax > IB_LMAX) return set_status(IB_ERR_ARG, "quartet_bounds: basis lmax out of range");
#define IB_QB(D)                                                                                                 \
  ib_quartet_bounds<D><<<grid, 256, 0, s>>>(quartets, nq, basis->shell_l, basis->shell_k, basis->shell_ptr,      \
                                            basis->shell_xyz, basis->prim_exp, basis->prim_coef, spherical ? 1 : 0, \
                                            bounds)
  switch (basis->lmax) {  // the polynomial degree is at most 2 lmax
    case 0: IB_QB(0); break;
    case 1: IB_QB(2); break;
    case 2: IB_QB(4); break;
    case 3: IB_QB(6); break;
    case 4: IB_QB(8); break;
    case 5: IB_QB(10); break;
    default: IB_QB(12); break;
  }
#undef IB_QB
  IB_CUDA(cudaGetLastError());
  return set_status(IB_OK, "");
}

// ---------------------------------------------------------------- CUDA graphs
struct IbGraph {
  Context* ctx;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int launches;
};

int intception_b200_eri_graph_create(const intception_b200_basis* basis, const int* quartets, const long long* out_off,
                                     int nq, int spherical, int precision, const double* bounds, double skip_below,
                                     double fp32_below, double mixed_tol, double* out, void** handle) {
  if (!handle) return set_status(IB_ERR_ARG, "graph_create: null handle");
  *handle = nullptr;
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t s = nullptr;
  IB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  // eager pass: sizes every work buffer, so the captured pass allocates nothing
  int nl = 0;
  st = batch_impl(c, basis, quartets, out_off, nq, spherical, precision, bounds, skip_below, fp32_below, mixed_tol,
                  out, s, &nl);
  if (st) {
    cudaStreamDestroy(s);
    return st;
  }
  IB_CUDA(cudaStreamSynchronize(s));
  IbGraph* g = new IbGraph{c, nullptr, nullptr, 0};
  IB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  nl = 0;
  st = batch_impl(c, basis, quartets, out_off, nq, spherical, precision, bounds, skip_below, fp32_below, mixed_tol,
                  out, s, &nl);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s, &graph);
  cudaStreamDestroy(s);
  if (st || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    delete g;
    return st ? st : set_status(IB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
  }
  g->graph = graph;
  g->launches = nl;
  const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
  if (ei != cudaSuccess) {
    cudaGraphDestroy(graph);
    delete g;
    return set_status(IB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
  }
  *handle = g;
  return set_status(IB_OK, "");
}

int intception_b200_eri_graph_launch(void* handle, void* stream) {
  IbGraph* g = static_cast<IbGraph*>(handle);
  if (!g) return set_status(IB_ERR_ARG, "graph_launch: null handle");
  tl_launches = g->launches;
  IB_CUDA(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
  return set_status(IB_OK, "");
}

int intception_b200_eri_graph_destroy(void* handle) {
  IbGraph* g = static_cast<IbGraph*>(handle);
  if (!g) return set_status(IB_OK, "");
  cudaGraphExecDestroy(g->exec);
  cudaGraphDestroy(g->graph);
  delete g;
  return set_status(IB_OK, "");
}

// Number of quartets of the last batch whose FP32 result was rejected and
// recomputed in FP64 (0 unless it was a mixed batch; synchronous).
int intception_b200_last_fp32_rejections(void) {
  Context* c = nullptr;
  if (get_context(&c)) return -1;
  if (!c->flags.p || c->flags_nq <= 0) return 0;
  IB_CUDA(cudaDeviceSynchronize());
  // only the last batch's flags: the buffer keeps stale entries past them
  const size_t n = std::min((size_t)c->flags_nq, c->flags.cap / sizeof(int));
  std::vector<int> h(n);
  IB_CUDA(cudaMemcpy(h.data(), c->flags.p, n * sizeof(int), cudaMemcpyDeviceToHost));
  int k = 0;
  for (int v : h) k += v & 1;
  return k;
}

// Number of quartets of the last batch (or drop-in call) that the class
// kernels put on the redo list (HRR rounding-error estimate over the
// tolerance) and the generic kernel recomputed (synchronous).
int intception_b200_last_hrr_redo(void) {
  Context* c = nullptr;
  if (get_context(&c)) return -1;
  if (!c->redo.p) return 0;
  IB_CUDA(cudaDeviceSynchronize());
  int total = 0;
  for (int g = 0; g < c->redo_groups; ++g) {
    int h[2] = {0, 0};  // heavy and light counts
    IB_CUDA(cudaMemcpy(h, c->redo.as<int>() + (size_t)g * c->redo_stride, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    total += h[0] + h[1];
  }
  return total;
}

// Tolerance of the class kernels' HRR rounding-error estimate, in the output's
// units (0 switches the check off).
int intception_b200_set_hrr_tol(double tol) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  if (!(tol >= 0.0) || tol > 1e-6) return set_status(IB_ERR_ARG, "set_hrr_tol: tolerance outside [0, 1e-6]");
  std::lock_guard<std::mutex> lk(c->mu);
  c->hrr_tol = tol;
  return set_status(IB_OK, "");
}

// Cap on the lane groups that share one quartet in the class kernels, per
// canonical class id (cid < 0: every class); 0 removes the cap.
int intception_b200_set_slice_cap(int cid, int cap) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  if (cid >= IB_NCLASS || cap < 0) return set_status(IB_ERR_ARG, "set_slice_cap: class id or cap out of range");
  for (int k = 0; k < IB_NCLASS; ++k)
    if (cid < 0 || k == cid) c->slice_cap[k] = cap;
  return set_status(IB_OK, "");
}

// Primitive screening in the batch entries' class kernels: a primitive
// quartet whose Coulomb-norm bound Q_ab Q_cd is below tol is skipped, which
// moves no element of its block by more than tol (0 restores exact-zero
// culling only; the drop-in functions never screen).
int intception_b200_set_prim_tol(double tol) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  if (!(tol >= 0.0) || tol > 1e-6) return set_status(IB_ERR_ARG, "set_prim_tol: tolerance outside [0, 1e-6]");
  c->prim_tol = tol;
  return set_status(IB_OK, "");
}

// Register budget of the kernel of canonical class cid for variant v4
// (0 FP64 Cartesian, 1 FP64 spherical, 2 FP32 Cartesian, 3 FP32 spherical):
// minb = minimum resident blocks per SM it was compiled for (1, 3, 4, 5);
// 0 restores the built-in (autotuned) default.
int intception_b200_set_class_minb(int cid, int v4, int minb) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  int mi = -1;
  for (int k = 0; k < IB_NMINB; ++k)
    if (ib_minb_value(k) == minb) mi = k;
  if (minb == 0 && cid >= 0 && cid < IB_NCLASS && v4 >= 0 && v4 <= 3)
    mi = std::min(std::max(ib_tuned_minb[cid][v4], 0), IB_NMINB - 1);  // back to the built-in default
  if (cid < 0 || cid >= IB_NCLASS || v4 < 0 || v4 > 3 || mi < 0 || !c->table[cid].launch)
    return set_status(IB_ERR_ARG, "set_class_minb: class, variant or budget not available");
  c->minb_idx[cid][v4] = mi;
  return set_status(IB_OK, "");
}

// Whether the FP32 tier runs the FP32 kernel of canonical class cid (cid < 0:
// every class): on = 1 where the class has one, 0 never (its FP32-tier
// quartets run in FP64), -1 the built-in (autotuned) default.  Waits for the
// device first: the classify kernel of a batch in flight reads the table.
int intception_b200_set_class_fp32(int cid, int on) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  if (cid >= IB_NCLASS || on < -1 || on > 1) return set_status(IB_ERR_ARG, "set_class_fp32: class id or value");
  for (int k = 0; k < IB_NCLASS; ++k) {
    if ((cid >= 0 && k != cid) || !c->table[k].launch) continue;
    const int want = on < 0 ? ib_tuned_fp32[k] : on;
    c->kind_h[k] = (c->table[k].kind == 2 && want) ? 2 : 1;
  }
  IB_CUDA(cudaDeviceSynchronize());
  IB_CUDA(cudaMemcpy(c->kind.p, c->kind_h, IB_NCLASS * sizeof(int), cudaMemcpyHostToDevice));
  return set_status(IB_OK, "");
}

// Device status word of the last batch (reads it synchronously).
int intception_b200_batch_status(void) {
  Context* c = nullptr;
  int st = get_context(&c);
  if (st) return st;
  int h = 0;
  IB_CUDA(cudaDeviceSynchronize());
  IB_CUDA(cudaMemcpy(&h, c->status.p, sizeof(int), cudaMemcpyDeviceToHost));
  return h;
}

}  // extern "C"
