// ib_twoidx.cu -- primitive Cartesian two-index integrals: the overlap and the
// nuclear-attraction classes of the reference's example input script
// (examples/example_input.py:83-107), generated there as
// intception_integral_overlap_2idx_ab_prim_cart and
// intception_integral_nuclear_2idx_ab_m_cC_prim_cart (contracted = False).
//
//   overlap:  (a|b) = sqrt(pi^3/p^3) exp(-xi R_AB^2) * OS recurrences on a, b
//   nuclear:  (a|C|b)^(m), base 2 pi/p exp(-xi R_AB^2) F_m(p R_PC^2), OS
//             recurrences with the auxiliary index m
// with p = alpha_a + alpha_b, xi = alpha_a alpha_b / p, P the Gaussian product
// centre.  Results are primitive (no normalisation, no coefficients), as the
// emitted functions return them.
//
// Device layout: one lane group (G lanes of a warp) per pair; the group's
// tables live in shared memory.
//   overlap: the integral factorises over x, y, z: three lanes build the 1D
//     tables S_d[i][j] (i <= la, j <= lb) with the 1D form of the two
//     recurrences, then every output is a product of three table entries.
//   nuclear: the larger side carries the recurrence (the integral is symmetric
//     under a <-> b): VRR on e = 0..la+lb with all needed m (the electron-free
//     form of the reference's vrr2 with b = 0), then HRR
//     (e|f+1i) = (e+1i|f) + (A-B)_i (e|f) moves angular momentum to b.  Table
//     sizes are at most 1820 (VRR) + 1640 (HRR) doubles per group for
//     la = lb = 6.
// The Boys function is the library's own (7-term Taylor about a 1/16 grid,
// downward recursion; asymptotic form with upward recursion for T >= 36).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/intception_b200.h"
#include "_gen/boys_table_data.h"
#include "ib_eri_device.cuh"

int ib_runtime_set_status(int st, const char* msg);

#define IB2_LMAX 6
#define IB2_NCOMP 455  // Cartesian components of levels 0..2*IB2_LMAX
#define IB2_BLOCK 128

namespace {

static __device__ __align__(256) double ib2_boys[IB_BOYS_NPTS * IB_BOYS_NCOL];

struct Ib2Args {
  int n;
  int lmax;
  const double* xa;
  const double* ca;
  const int* la;
  const double* xb;
  const double* cb;
  const int* lb;
  const double* cc;
  const long long* off;
  double* out;
  const double* boys;
  int* status;
};

__host__ __device__ __forceinline__ int ib2_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ __forceinline__ int ib2_ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }  // ncum(-1) = 0
__device__ __forceinline__ int ib2_cidx(int y, int z) { return z + (y + z) * (y + z + 1) / 2; }

// Offset of level n in the VRR table of total L: sum_{n'<n} ncart(n') (L - n' + 1).
__host__ __device__ __forceinline__ int ib2_vrr_off(int n, int L) {
  return (L + 1) * n * (n + 1) * (n + 2) / 6 - (n - 1) * n * (n + 1) * (n + 2) / 8;
}

// (x, y, z) of every component of levels 0..12 in the reference's order
// (cumulative index ncum(n-1) + k; within a level z + (y+z)(y+z+1)/2 = k).
__device__ __forceinline__ void ib2_stage_comps(uchar4* comp) {
  for (int t = threadIdx.x; t < IB2_NCOMP; t += blockDim.x) {
    int n = 0;
    while (ib2_ncum(n) <= t) ++n;
    const int k = t - ib2_ncum(n - 1);
    int s = 0;
    while ((s + 1) * (s + 2) / 2 <= k) ++s;
    const int z = k - s * (s + 1) / 2;
    comp[t] = make_uchar4((unsigned char)(n - s), (unsigned char)(s - z), (unsigned char)z, (unsigned char)n);
  }
}

__device__ __forceinline__ double ib2_sel(int i, double v0, double v1, double v2) {
  return i == 0 ? v0 : (i == 1 ? v1 : v2);
}

template <int G>
__device__ __forceinline__ unsigned ib2_mask() {
  if (G == 32) return 0xffffffffu;
  return ((1u << G) - 1u) << ((threadIdx.x & 31) / G * G);
}

// A pair the kernels refuse: l outside [0, lmax], or an exponent that is not
// positive (p <= 0 would index the Boys table below its first point).
__device__ __forceinline__ bool ib2_bad(int la, int lb, int lmax, double xa, double xb) {
  return la < 0 || la > lmax || lb < 0 || lb > lmax || !(xa > 0.0) || !(xb > 0.0);
}

// ---------------------------------------------------------------------------
// overlap: smem per group 3 * 49 doubles
template <int G>
__global__ void __launch_bounds__(IB2_BLOCK) ib2_overlap_kernel(const Ib2Args a) {
  extern __shared__ double sm2[];
  constexpr int kGroups = IB2_BLOCK / G;
  constexpr int kPer = 3 * (IB2_LMAX + 1) * (IB2_LMAX + 1);
  uchar4* comp = reinterpret_cast<uchar4*>(sm2 + kGroups * kPer);
  ib2_stage_comps(comp);
  __syncthreads();
  const int gib = threadIdx.x / G, lane = threadIdx.x % G;
  const unsigned mask = ib2_mask<G>();
  double* S = sm2 + gib * kPer;
  for (int p = blockIdx.x * kGroups + gib; p < a.n; p += gridDim.x * kGroups) {
    const int la = __ldg(a.la + p), lb = __ldg(a.lb + p);
    const double xa = __ldg(a.xa + p), xb = __ldg(a.xb + p);
    if (ib2_bad(la, lb, a.lmax, xa, xb)) {
      if (lane == 0 && a.status) atomicExch(a.status, IB_ERR_ARG);
      continue;
    }
    const double op = 1.0 / (xa + xb), o2p = 0.5 * op, xi = xa * xb * op;
    const int nj = lb + 1;
    if (lane < 3) {
      const double A = __ldg(a.ca + 3 * p + lane), B = __ldg(a.cb + 3 * p + lane);
      const double AB = A - B, PA = -xb * op * AB, PB = xa * op * AB;
      double* s = S + lane * (IB2_LMAX + 1) * (IB2_LMAX + 1);
      s[0] = 1.0;
      for (int i = 1; i <= la; ++i) {
        double v = PA * s[(i - 1) * nj];
        if (i >= 2) v = fma((double)(i - 1) * o2p, s[(i - 2) * nj], v);
        s[i * nj] = v;
      }
      for (int j = 1; j <= lb; ++j)
        for (int i = 0; i <= la; ++i) {
          double v = PB * s[i * nj + j - 1];
          if (j >= 2) v = fma((double)(j - 1) * o2p, s[i * nj + j - 2], v);
          if (i >= 1) v = fma((double)i * o2p, s[(i - 1) * nj + j - 1], v);
          s[i * nj + j] = v;
        }
    }
    __syncwarp(mask);
    double ab2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double t = __ldg(a.ca + 3 * p + d) - __ldg(a.cb + 3 * p + d);
      ab2 = fma(t, t, ab2);
    }
    const double pref = sqrt(31.006276680299820175 * op * op * op) * exp(-xi * ab2);  // pi^3 / p^3
    const int na = ib2_ncart(la), nb = ib2_ncart(lb), tot = na * nb;
    const uchar4* ca_ = comp + ib2_ncum(la - 1);
    const uchar4* cb_ = comp + ib2_ncum(lb - 1);
    constexpr int kDir = (IB2_LMAX + 1) * (IB2_LMAX + 1);
    double* o = a.out + __ldg(a.off + p);
    for (int t = lane; t < tot; t += G) {
      const int ia = t % na, ib = t / na;
      const uchar4 e = ca_[ia], f = cb_[ib];
      o[t] = pref * S[e.x * nj + f.x] * S[kDir + e.y * nj + f.y] * S[2 * kDir + e.z * nj + f.z];
    }
    __syncwarp(mask);
  }
}

// ---------------------------------------------------------------------------
// nuclear attraction: smem per group rv + rb doubles (VRR region, HRR region)
template <int G>
__global__ void __launch_bounds__(IB2_BLOCK) ib2_nuclear_kernel(const Ib2Args a, int rv, int rb) {
  extern __shared__ double sm2[];
  constexpr int kGroups = IB2_BLOCK / G;
  const int per = rv + rb;
  uchar4* comp = reinterpret_cast<uchar4*>(sm2 + kGroups * per);
  ib2_stage_comps(comp);
  __syncthreads();
  const int gib = threadIdx.x / G, lane = threadIdx.x % G;
  const unsigned mask = ib2_mask<G>();
  double* V = sm2 + gib * per;
  double* H = V + rv;
  for (int p = blockIdx.x * kGroups + gib; p < a.n; p += gridDim.x * kGroups) {
    const int la0 = __ldg(a.la + p), lb0 = __ldg(a.lb + p);
    if (ib2_bad(la0, lb0, a.lmax, __ldg(a.xa + p), __ldg(a.xb + p))) {
      if (lane == 0 && a.status) atomicExch(a.status, IB_ERR_ARG);
      continue;
    }
    const bool swap = la0 < lb0;  // recur on the larger side
    const int la = swap ? lb0 : la0, lb = swap ? la0 : lb0, L = la + lb;
    const double* pa = swap ? a.cb + 3 * p : a.ca + 3 * p;
    const double* pb = swap ? a.ca + 3 * p : a.cb + 3 * p;
    const double xa = __ldg(swap ? a.xb + p : a.xa + p), xb = __ldg(swap ? a.xa + p : a.xb + p);
    const double op = 1.0 / (xa + xb), o2p = 0.5 * op, xi = xa * xb * op;
    double AB[3], PA[3], PC[3], ab2 = 0.0, pc2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double A = __ldg(pa + d), B = __ldg(pb + d), C = __ldg(a.cc + 3 * p + d);
      AB[d] = A - B;
      PA[d] = -xb * op * AB[d];
      PC[d] = (xa * (A - C) + xb * (B - C)) * op;
      ab2 = fma(AB[d], AB[d], ab2);
      pc2 = fma(PC[d], PC[d], pc2);
    }
    if (lane == 0) {
      ib_boys_rt((xa + xb) * pc2, L, a.boys, V);
      const double pref = 6.283185307179586477 * op * exp(-xi * ab2);
      for (int m = 0; m <= L; ++m) V[m] *= pref;
    }
    __syncwarp(mask);
    // VRR: [e]^(m) = PA_i [e-1i]^(m) - PC_i [e-1i]^(m+1) + (e_i-1)/2p ([e-2i]^(m) - [e-2i]^(m+1))
    for (int n = 1; n <= L; ++n) {
      const int M = L - n + 1, tot = ib2_ncart(n) * M;
      const int o0 = ib2_vrr_off(n, L), o1 = ib2_vrr_off(n - 1, L), o2 = n >= 2 ? ib2_vrr_off(n - 2, L) : 0;
      const uchar4* cn = comp + ib2_ncum(n - 1);
      for (int t = lane; t < tot; t += G) {
        const int k = t / M, m = t - k * M;
        const uchar4 e = cn[k];
        const int i = e.x ? 0 : (e.y ? 1 : 2);
        const int ei = i == 0 ? e.x : (i == 1 ? e.y : e.z);
        const int y1 = e.y - (i == 1), z1 = e.z - (i == 2);
        const double* r1 = V + o1 + ib2_cidx(y1, z1) * (M + 1) + m;
        double v = ib2_sel(i, PA[0], PA[1], PA[2]) * r1[0] - ib2_sel(i, PC[0], PC[1], PC[2]) * r1[1];
        if (ei >= 2) {
          const double* r2 = V + o2 + ib2_cidx(y1 - (i == 1), z1 - (i == 2)) * (M + 2) + m;
          v = fma((double)(ei - 1) * o2p, r2[0] - r2[1], v);
        }
        V[o0 + t] = v;
      }
      __syncwarp(mask);
    }
    // HRR over b levels j = 1..lb: H_j[(e - first e of level la)][f]; odd j in H, even j in V
    const int base = ib2_ncum(la - 1);
    for (int j = 1; j <= lb; ++j) {
      double* Hn = (j & 1) ? H : V;
      const double* Hp = (j & 1) ? V : H;
      const int nf = ib2_ncart(j), nfp = ib2_ncart(j - 1);
      const int tot = (ib2_ncum(L - j) - base) * nf;
      const uchar4* cf = comp + ib2_ncum(j - 1);
      for (int t = lane; t < tot; t += G) {
        const int ec = t / nf, fk = t - ec * nf;
        const uchar4 e = comp[base + ec], f = cf[fk];
        const int i = f.x ? 0 : (f.y ? 1 : 2);
        const int fkp = ib2_cidx(f.y - (i == 1), f.z - (i == 2));
        const int n = e.w;
        const int k0 = ib2_cidx(e.y, e.z), k1 = ib2_cidx(e.y + (i == 1), e.z + (i == 2));
        double h0, h1;
        if (j == 1) {  // previous level is the VRR table at m = 0
          h0 = V[ib2_vrr_off(n, L) + k0 * (L - n + 1)];
          h1 = V[ib2_vrr_off(n + 1, L) + k1 * (L - n)];
        } else {
          h0 = Hp[(ib2_ncum(n - 1) - base + k0) * nfp + fkp];
          h1 = Hp[(ib2_ncum(n) - base + k1) * nfp + fkp];
        }
        Hn[t] = fma(ib2_sel(i, AB[0], AB[1], AB[2]), h0, h1);
      }
      __syncwarp(mask);
    }
    const int na0 = ib2_ncart(la0), nb0 = ib2_ncart(lb0), tot = na0 * nb0, nbs = ib2_ncart(lb);
    const double* R = (lb & 1) ? H : V;
    const int vo = ib2_vrr_off(la, L);
    double* o = a.out + __ldg(a.off + p);
    for (int t = lane; t < tot; t += G) {
      const int ia = t % na0, ib = t / na0;
      const int k = swap ? ib : ia, fk = swap ? ia : ib;
      o[t] = lb == 0 ? V[vo + k * (L - la + 1)] : R[k * nbs + fk];
    }
    __syncwarp(mask);
  }
}

// ---------------------------------------------------------------------------
// host side

// Shared-memory regions (doubles per group) of the nuclear kernel for l <= lmax.
void nuclear_regions(int lmax, int* rv, int* rb) {
  int v = 1, b = 0;
  for (int la = 0; la <= lmax; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      const int L = la + lb;
      v = std::max(v, ib2_vrr_off(L + 1, L));
      for (int j = 1; j <= lb; ++j) {
        const int h = (ib2_ncum(L - j) - ib2_ncum(la - 1)) * ib2_ncart(j);
        if (j & 1)
          b = std::max(b, h);
        else
          v = std::max(v, h);
      }
    }
  *rv = v;
  *rb = b;
}

int pick_group(int kind, int lmax) {
  if (kind == 0) return lmax <= 1 ? 4 : (lmax <= 3 ? 8 : 16);
  return lmax == 0 ? 4 : (lmax == 1 ? 8 : (lmax == 2 ? 16 : 32));
}

size_t smem_bytes(int kind, int G, int lmax) {
  const int groups = IB2_BLOCK / G;
  size_t per;
  if (kind == 0) {
    per = 3 * (IB2_LMAX + 1) * (IB2_LMAX + 1);
  } else {
    int rv, rb;
    nuclear_regions(lmax, &rv, &rb);
    per = (size_t)(rv + rb);
  }
  return groups * per * sizeof(double) + IB2_NCOMP * sizeof(uchar4);
}

struct Single {
  double d[12];  // xa, A[3], xb, B[3], C[3], pad
  int l[2];
  long long off;
};

struct TwoIdxDevice {
  bool ready = false;
  int nsm = 0;
  double* boys = nullptr;
  Single* single = nullptr;
  double* single_out = nullptr;
  int* single_status = nullptr;
  cudaStream_t stream = nullptr;
  std::mutex mu;  // serialises the single-pair entry points on this device
};

static __device__ __align__(256) Single ib2_single;
static __device__ __align__(256) double ib2_single_out[28 * 28];
static __device__ __align__(256) int ib2_single_status;

TwoIdxDevice g_dev2[64];
std::mutex g_mu2;

template <class K>
cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Once per device, with that device current: the Boys table, the large-shared-memory
// opt-in of every kernel instantiation, the single-pair staging symbols, a stream.
int twoidx_setup(TwoIdxDevice** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return ib_runtime_set_status(IB_ERR_NODEVICE, "two-index: no CUDA device");
  std::lock_guard<std::mutex> lk(g_mu2);
  TwoIdxDevice& d = g_dev2[dev];
  if (!d.ready) {
    bool ok = cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
    ok = ok && cudaMemcpyToSymbol(ib2_boys, ib_boys_host_table, sizeof(ib_boys_host_table)) == cudaSuccess;
    ok = ok && cudaGetSymbolAddress((void**)&d.boys, ib2_boys) == cudaSuccess;
    ok = ok && cudaGetSymbolAddress((void**)&d.single, ib2_single) == cudaSuccess;
    ok = ok && cudaGetSymbolAddress((void**)&d.single_out, ib2_single_out) == cudaSuccess;
    ok = ok && cudaGetSymbolAddress((void**)&d.single_status, ib2_single_status) == cudaSuccess;
    // each group size serves the lmax values pick_group maps to it
    ok = ok && allow_smem(ib2_nuclear_kernel<32>, smem_bytes(1, 32, IB2_LMAX)) == cudaSuccess;
    ok = ok && allow_smem(ib2_nuclear_kernel<16>, smem_bytes(1, 16, 2)) == cudaSuccess;
    ok = ok && allow_smem(ib2_nuclear_kernel<8>, smem_bytes(1, 8, 1)) == cudaSuccess;
    ok = ok && allow_smem(ib2_nuclear_kernel<4>, smem_bytes(1, 4, 0)) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) return ib_runtime_set_status(IB_ERR_CUDA, "two-index: device setup failed");
    d.ready = true;
  }
  *out = &d;
  return IB_OK;
}

template <class K>
int grid_for(K kernel, size_t smem, int n, int groups, int nsm) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, IB2_BLOCK, smem);
  per_sm = std::max(per_sm, 1);
  const long long need = ((long long)n + groups - 1) / groups;
  return (int)std::max(1LL, std::min<long long>(need, (long long)per_sm * nsm));
}

int launch(int kind, const Ib2Args& a, int nsm, cudaStream_t s) {
  const int G = pick_group(kind, a.lmax);
  const size_t smem = smem_bytes(kind, G, a.lmax);
  const int groups = IB2_BLOCK / G;
  if (kind == 0) {
#define IB2_OV(g)                                                        \
  case g: {                                                              \
    const int grid = grid_for(ib2_overlap_kernel<g>, smem, a.n, groups, nsm); \
    ib2_overlap_kernel<g><<<grid, IB2_BLOCK, smem, s>>>(a);              \
    break;                                                               \
  }
    switch (G) {
      IB2_OV(4)
      IB2_OV(8)
      IB2_OV(16)
      default:
        return IB_ERR_ARG;
    }
#undef IB2_OV
  } else {
    int rv, rb;
    nuclear_regions(a.lmax, &rv, &rb);
#define IB2_NU(g)                                                        \
  case g: {                                                              \
    const int grid = grid_for(ib2_nuclear_kernel<g>, smem, a.n, groups, nsm); \
    ib2_nuclear_kernel<g><<<grid, IB2_BLOCK, smem, s>>>(a, rv, rb);      \
    break;                                                               \
  }
    switch (G) {
      IB2_NU(4)
      IB2_NU(8)
      IB2_NU(16)
      IB2_NU(32)
      default:
        return IB_ERR_ARG;
    }
#undef IB2_NU
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? IB_OK : IB_ERR_CUDA;
}

// One pair from host memory (the emitted functions' calling convention): stage,
// evaluate, copy back, scatter with the caller's strides.
void single_pair(int kind, double xa, const double* cA, int la, int na, int iskipa, double xb, const double* cB,
                 int lb, int nb, int iskipb, const double* cC, double* out) {
  if (la < 0 || la > IB2_LMAX || lb < 0 || lb > IB2_LMAX) {
    ib_runtime_set_status(IB_ERR_ARG, "two-index: angular momentum outside [0, 6]");
    return;
  }
  if (na != ib2_ncart(la) || nb != ib2_ncart(lb)) {
    ib_runtime_set_status(IB_ERR_ARG, "two-index: n? must equal (l?+1)(l?+2)/2");
    return;
  }
  if (!cA || !cB || (kind == 1 && !cC) || !out) {
    ib_runtime_set_status(IB_ERR_ARG, "two-index: null pointer");
    return;
  }
  TwoIdxDevice* d = nullptr;
  if (twoidx_setup(&d)) return;
  std::lock_guard<std::mutex> lk(d->mu);
  Single h = {};
  h.d[0] = xa;
  h.d[4] = xb;
  for (int i = 0; i < 3; ++i) {
    h.d[1 + i] = cA[i];
    h.d[5 + i] = cB[i];
    h.d[8 + i] = kind == 1 ? cC[i] : 0.0;
  }
  h.l[0] = la;
  h.l[1] = lb;
  h.off = 0;
  Ib2Args a;
  a.n = 1;
  a.lmax = std::max(la, lb);
  a.xa = d->single->d;
  a.ca = d->single->d + 1;
  a.xb = d->single->d + 4;
  a.cb = d->single->d + 5;
  a.cc = d->single->d + 8;
  a.la = d->single->l;
  a.lb = d->single->l + 1;
  a.off = &d->single->off;
  a.out = d->single_out;
  a.boys = d->boys;
  a.status = d->single_status;
  const int tot = na * nb;
  double res[28 * 28];
  int dst = 0;
  cudaStream_t s = d->stream;
  if (cudaMemcpyAsync(d->single, &h, sizeof(h), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(d->single_status, 0, sizeof(int), s) != cudaSuccess) {
    ib_runtime_set_status(IB_ERR_CUDA, "two-index: staging copy failed");
    return;
  }
  int st = launch(kind, a, d->nsm, s);
  if (st) {
    ib_runtime_set_status(st, "two-index: launch failed");
    return;
  }
  if (cudaMemcpyAsync(res, d->single_out, tot * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&dst, d->single_status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    ib_runtime_set_status(IB_ERR_CUDA, "two-index: result copy failed");
    return;
  }
  if (dst) {
    ib_runtime_set_status(dst, "two-index: device reported an invalid pair");
    return;
  }
  for (int ib = 0; ib < nb; ++ib)
    for (int ia = 0; ia < na; ++ia) out[(long long)ia * iskipa + (long long)ib * iskipb] = res[ia + na * ib];
  ib_runtime_set_status(IB_OK, "");
}

}  // namespace

extern "C" {

void intception_integral_overlap_2idx_ab_prim_cart_main(const double xa, const double cA[3], const int la,
                                                         const int na, const int iskipa, const double xb,
                                                         const double cB[3], const int lb, const int nb,
                                                         const int iskipb, double* work_array,
                                                         double* output_array) {
  (void)work_array;
  single_pair(0, xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, nullptr, output_array);
}

int intception_integral_overlap_2idx_ab_prim_cart_work_array_size(const int la, const int lb) {
  return ib2_ncum(la) * ib2_ncum(lb);
}

void intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main(const double xa, const double cA[3], const int la,
                                                              const int na, const int iskipa, const double xb,
                                                              const double cB[3], const int lb, const int nb,
                                                              const int iskipb, const double cC[3],
                                                              double* work_array, double* output_array) {
  (void)work_array;
  single_pair(1, xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, cC, output_array);
}

int intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size(const int la, const int lb) {
  return 2 * (ib2_ncum(lb) * ib2_ncum(la) + la + lb + 1);
}

int intception_b200_twoidx_batch(int kind, int n, int lmax, const double* xa, const double* ca, const int* la,
                                 const double* xb, const double* cb, const int* lb, const double* cc,
                                 const long long* off, double* out, int* status, void* stream) {
  if (kind != IB_TWOIDX_OVERLAP && kind != IB_TWOIDX_NUCLEAR)
    return ib_runtime_set_status(IB_ERR_ARG, "twoidx_batch: kind must be 0 (overlap) or 1 (nuclear)");
  if (n < 0 || lmax < 0 || lmax > IB2_LMAX) return ib_runtime_set_status(IB_ERR_ARG, "twoidx_batch: n or lmax");
  if (n > 0 && (!xa || !ca || !la || !xb || !cb || !lb || !off || !out || (kind == IB_TWOIDX_NUCLEAR && !cc)))
    return ib_runtime_set_status(IB_ERR_ARG, "twoidx_batch: null pointer");
  if (n == 0) return ib_runtime_set_status(IB_OK, "");
  TwoIdxDevice* d = nullptr;
  int st = twoidx_setup(&d);
  if (st) return st;
  Ib2Args a;
  a.n = n;
  a.lmax = lmax;
  a.xa = xa;
  a.ca = ca;
  a.la = la;
  a.xb = xb;
  a.cb = cb;
  a.lb = lb;
  a.cc = cc;
  a.off = off;
  a.out = out;
  a.boys = d->boys;
  a.status = status;
  st = launch(kind, a, d->nsm, static_cast<cudaStream_t>(stream));
  if (st) return ib_runtime_set_status(st, "twoidx_batch: launch failed");
  return ib_runtime_set_status(IB_OK, "");
}

}  // extern "C"
