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
#include <atomic>
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
  int lthr;  // lane-group kernels: pairs with max(la, lb) <= lthr belong to the thread-per-pair kernels
  int bulk_ok;  // thread-per-pair kernel: every input array 16-byte aligned (complete chunks by bulk copy)
  long long stall_chunk;  // testing: this chunk's barrier is armed but its copies are not issued (-1: none)
  int wait_iters;         // iterations of a bounded wait for a chunk's copies (1 << 22: about 0.4 s)
};

__host__ __device__ __forceinline__ int ib2_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ __forceinline__ int ib2_ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }  // ncum(-1) = 0
__device__ __forceinline__ int ib2_cidx(int y, int z) { return z + (y + z) * (y + z + 1) / 2; }

// Offset of level n in the VRR table of total L: sum_{n'<n} ncart(n') (L - n' + 1).
__host__ __device__ constexpr int ib2_vrr_off(int n, int L) {
  return (L + 1) * n * (n + 1) * (n + 2) / 6 - (n - 1) * n * (n + 1) * (n + 2) / 8;
}
__host__ __device__ constexpr int ib2_ncart_c(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int ib2_ncum_c(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
__host__ __device__ constexpr int ib2_cidx_c(int y, int z) { return z + (y + z) * (y + z + 1) / 2; }

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
    if (max(la, lb) <= a.lthr) continue;  // done by the thread-per-pair kernel
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
    if (max(la0, lb0) <= a.lthr) continue;  // done by the thread-per-pair kernel
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
// Thread-per-pair kernels for max(la, lb) <= IB2_LT: the recurrences of one
// class fully unrolled at compile time (every table index a constant, the
// tables in registers); the class is picked per thread by a switch.
#define IB2_LT 2

// Largest HRR level table, (ncum(L-j) - ncum(LA-1)) ncart(j) over j = 1..LB.
__host__ __device__ constexpr int ib2_hrr_max(int LA, int LB) {
  int h = 1;
  for (int j = 1; j <= LB; ++j) {
    const int t = (ib2_ncum_c(LA + LB - j) - ib2_ncum_c(LA - 1)) * ib2_ncart_c(j);
    h = t > h ? t : h;
  }
  return h;
}

// F_m(T), m = 0..L, reading the global table (no staging; L is a constant).
template <int L>
__device__ __forceinline__ void ib2_boys_f(double T, const double* __restrict__ tab, double* F) {
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
    F[L] = fma(f, dx, __ldg(r));
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

// Nuclear attraction of one pair, LA >= LB; element (k of LA, f of LB) to o[k*sa + f*sb].
template <int LA, int LB>
__device__ __forceinline__ void ib2_nuclear_pair(double xa, const double* __restrict__ pa, double xb,
                                                 const double* __restrict__ pb, const double* __restrict__ pc,
                                                 const double* __restrict__ boys, double* __restrict__ o, int sa,
                                                 int sb) {
  constexpr int L = LA + LB;
  const double op = 1.0 / (xa + xb), o2p = 0.5 * op, xi = xa * xb * op;
  double AB[3], PA[3], PC[3], ab2 = 0.0, pc2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double A = pa[d], B = pb[d], C = pc[d];
    AB[d] = A - B;
    PA[d] = -xb * op * AB[d];
    PC[d] = (xa * (A - C) + xb * (B - C)) * op;
    ab2 = fma(AB[d], AB[d], ab2);
    pc2 = fma(PC[d], PC[d], pc2);
  }
  double V[ib2_vrr_off(L + 1, L)];
  ib2_boys_f<L>((xa + xb) * pc2, boys, V);
  const double pref = 6.283185307179586477 * op * exp(-xi * ab2);
#pragma unroll
  for (int m = 0; m <= L; ++m) V[m] *= pref;
  // VRR: [e]^(m) = PA_i [e-1i]^(m) - PC_i [e-1i]^(m+1) + (e_i-1)/2p ([e-2i]^(m) - [e-2i]^(m+1))
#pragma unroll
  for (int n = 1; n <= L; ++n) {
    const int M = L - n + 1;
#pragma unroll
    for (int s = 0; s <= n; ++s)
#pragma unroll
      for (int z = 0; z <= s; ++z) {
        const int y = s - z, x = n - s, k = z + s * (s + 1) / 2;
        const int i = x ? 0 : (y ? 1 : 2);
        const int ei = i == 0 ? x : (i == 1 ? y : z);
        const int y1 = y - (i == 1), z1 = z - (i == 2);
        const int r1 = ib2_vrr_off(n - 1, L) + ib2_cidx_c(y1, z1) * (M + 1);
        const int r2 = n >= 2 ? ib2_vrr_off(n - 2, L) + ib2_cidx_c(y1 - (i == 1), z1 - (i == 2)) * (M + 2) : 0;
#pragma unroll
        for (int m = 0; m < M; ++m) {
          double v = PA[i] * V[r1 + m] - PC[i] * V[r1 + m + 1];
          if (ei >= 2) v = fma((double)(ei - 1) * o2p, V[r2 + m] - V[r2 + m + 1], v);
          V[ib2_vrr_off(n, L) + k * M + m] = v;
        }
      }
  }
  if (LB == 0) {
#pragma unroll
    for (int k = 0; k < ib2_ncart_c(LA); ++k) o[k * sa] = V[ib2_vrr_off(LA, L) + k * (L - LA + 1)];
    return;
  }
  // HRR: (e|f+1i) = (e+1i|f) + AB_i (e|f); H[(e - first e of level LA)*ncart(j) + f]
  constexpr int base = ib2_ncum_c(LA - 1);
  constexpr int NH = ib2_hrr_max(LA, LB);
  double H[2][NH];  // level j in H[j & 1]
#pragma unroll
  for (int j = 1; j <= LB; ++j) {
    double* Hn = H[j & 1];
    const double* Hp = H[(j - 1) & 1];
    const int nf = ib2_ncart_c(j), nfp = ib2_ncart_c(j - 1);
#pragma unroll
    for (int n = LA; n <= L - j; ++n)
#pragma unroll
      for (int s = 0; s <= n; ++s)
#pragma unroll
        for (int z = 0; z <= s; ++z) {
          const int y = s - z, k0 = z + s * (s + 1) / 2;
#pragma unroll
          for (int fs = 0; fs <= j; ++fs)
#pragma unroll
            for (int fz = 0; fz <= fs; ++fz) {
              const int fy = fs - fz, fx = j - fs, fk = fz + fs * (fs + 1) / 2;
              const int i = fx ? 0 : (fy ? 1 : 2);
              const int fkp = ib2_cidx_c(fy - (i == 1), fz - (i == 2));
              const int k1 = ib2_cidx_c(y + (i == 1), z + (i == 2));
              double h0, h1;
              if (j == 1) {
                h0 = V[ib2_vrr_off(n, L) + k0 * (L - n + 1)];
                h1 = V[ib2_vrr_off(n + 1, L) + k1 * (L - n)];
              } else {
                h0 = Hp[(ib2_ncum_c(n - 1) - base + k0) * nfp + fkp];
                h1 = Hp[(ib2_ncum_c(n) - base + k1) * nfp + fkp];
              }
              Hn[(ib2_ncum_c(n - 1) - base + k0) * nf + fk] = fma(AB[i], h0, h1);
            }
        }
  }
#pragma unroll
  for (int k = 0; k < ib2_ncart_c(LA); ++k)
#pragma unroll
    for (int f = 0; f < ib2_ncart_c(LB); ++f) o[k * sa + f * sb] = H[LB & 1][k * ib2_ncart_c(LB) + f];
}

template <int LA, int LB>
__device__ __forceinline__ void ib2_overlap_pair(double xa, const double* __restrict__ pa, double xb,
                                                 const double* __restrict__ pb, double* __restrict__ o) {
  const double op = 1.0 / (xa + xb), o2p = 0.5 * op, xi = xa * xb * op;
  double S[3][LA + 1][LB + 1];
  double ab2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double AB = pa[d] - pb[d], PA = -xb * op * AB, PB = xa * op * AB;
    ab2 = fma(AB, AB, ab2);
    S[d][0][0] = 1.0;
#pragma unroll
    for (int i = 1; i <= LA; ++i) {
      double v = PA * S[d][i - 1][0];
      if (i >= 2) v = fma((double)(i - 1) * o2p, S[d][i - 2][0], v);
      S[d][i][0] = v;
    }
#pragma unroll
    for (int j = 1; j <= LB; ++j)
#pragma unroll
      for (int i = 0; i <= LA; ++i) {
        double v = PB * S[d][i][j - 1];
        if (j >= 2) v = fma((double)(j - 1) * o2p, S[d][i][j - 2], v);
        if (i >= 1) v = fma((double)i * o2p, S[d][i - 1][j - 1], v);
        S[d][i][j] = v;
      }
  }
  const double pref = sqrt(31.006276680299820175 * op * op * op) * exp(-xi * ab2);  // pi^3 / p^3
#pragma unroll
  for (int fs = 0; fs <= LB; ++fs)
#pragma unroll
    for (int fz = 0; fz <= fs; ++fz)
#pragma unroll
      for (int es = 0; es <= LA; ++es)
#pragma unroll
        for (int ez = 0; ez <= es; ++ez) {
          const int ex = LA - es, ey = es - ez, fx = LB - fs, fy = fs - fz;
          const int ia = ez + es * (es + 1) / 2, ib = fz + fs * (fs + 1) / 2;
          o[ia + ib2_ncart_c(LA) * ib] = pref * S[0][ex][fx] * S[1][ey][fy] * S[2][ez][fz];
        }
}

// Block-cooperative chunks: a block stages IB2_CHUNK pairs' inputs in shared
// memory (coalesced, each input byte read once), counting-sorts them by class
// there, and its warps run the sorted list, so the 32 lanes of a warp execute
// the same unrolled class code.  Pairs of the lane-group kernel and refused
// pairs are left out of the list.
//
// The inputs of a complete chunk are contiguous byte ranges of the caller's
// arrays; they are fetched by bulk copies (TMA, cp.async.bulk) into one of two
// chunk buffers while the block evaluates the other, with completion counted
// on an mbarrier per buffer.  The last (partial) chunk, and callers whose
// arrays are not 16-byte aligned, take plain loads.
#define IB2_CHUNK 512
#define IB2_TPB 256

// One chunk's inputs; every member is a whole number of 16-byte units.
template <int KIND>
struct Ib2Buf {
  double xa[IB2_CHUNK], xb[IB2_CHUNK];
  double ca[3 * IB2_CHUNK], cb[3 * IB2_CHUNK];
  double cc[KIND == 1 ? 3 * IB2_CHUNK : 2];
  long long off[IB2_CHUNK];
  int la[IB2_CHUNK], lb[IB2_CHUNK];
};

template <int KIND>
struct Ib2Stage {
  Ib2Buf<KIND> buf[2];
  unsigned long long full[2];  // mbarrier of each buffer: complete when its bulk copies have landed
  short order[IB2_CHUNK];     // chunk-local pair index, sorted by class
  unsigned char cls[IB2_CHUNK];
  unsigned char swp[IB2_CHUNK];
  int count[16], start[16];
};

__device__ __forceinline__ unsigned ib2_smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Thread 0: fetch complete chunk ch into bf; the buffer's mbarrier completes
// when every byte has arrived.  The block has finished reading bf (a block
// barrier precedes the call); the proxy fence orders those reads before the
// copies' writes.
template <int KIND>
__device__ __forceinline__ void ib2_issue(const Ib2Args& a, Ib2Buf<KIND>& bf, long long ch, unsigned mb) {
  const long long p0 = ch * IB2_CHUNK;
  const unsigned n8 = IB2_CHUNK * 8, n24 = 3 * IB2_CHUNK * 8, n4 = IB2_CHUNK * 4;
  const unsigned bytes = 3 * n8 + 2 * n4 + 2 * n24 + (KIND == 1 ? n24 : 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
  if (ch == a.stall_chunk) return;  // testing: bytes announced that no copy delivers; the wait gives up
#define IB2_BULK(dst, src, nb)                                                                                  \
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"( \
                   ib2_smem_addr(dst)),                                                                         \
               "l"(src), "r"(nb), "r"(mb)                                                                       \
               : "memory")
  IB2_BULK(bf.xa, a.xa + p0, n8);
  IB2_BULK(bf.xb, a.xb + p0, n8);
  IB2_BULK(bf.off, a.off + p0, n8);
  IB2_BULK(bf.la, a.la + p0, n4);
  IB2_BULK(bf.lb, a.lb + p0, n4);
  IB2_BULK(bf.ca, a.ca + 3 * p0, n24);
  IB2_BULK(bf.cb, a.cb + 3 * p0, n24);
  if (KIND == 1) IB2_BULK(bf.cc, a.cc + 3 * p0, n24);
#undef IB2_BULK
}

// Bounded wait for phase `parity` of the mbarrier at mb: false after `iters`
// polls without completion (1 << 22 of them, about 0.4 s: a copy that never
// lands), so that the block can report the error and return instead of
// spinning on.
__device__ __forceinline__ bool ib2_wait(unsigned mb, unsigned parity, int iters) {
  for (int it = 0; it < iters; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(mb), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(100);
  }
  return false;
}

template <int KIND>
__device__ __forceinline__ void ib2_thread_pair(const Ib2Buf<KIND>& st, const unsigned char* swp, int c, int j,
                                                const double* boys, double* out) {
  if (KIND == 0) {
    const double* pa = st.ca + 3 * j;
    const double* pb = st.cb + 3 * j;
    double* o = out + st.off[j];
    const double xa = st.xa[j], xb = st.xb[j];
    switch (c) {
      case 0: ib2_overlap_pair<0, 0>(xa, pa, xb, pb, o); break;
      case 1: ib2_overlap_pair<0, 1>(xa, pa, xb, pb, o); break;
      case 2: ib2_overlap_pair<0, 2>(xa, pa, xb, pb, o); break;
      case 3: ib2_overlap_pair<1, 0>(xa, pa, xb, pb, o); break;
      case 4: ib2_overlap_pair<1, 1>(xa, pa, xb, pb, o); break;
      case 5: ib2_overlap_pair<1, 2>(xa, pa, xb, pb, o); break;
      case 6: ib2_overlap_pair<2, 0>(xa, pa, xb, pb, o); break;
      case 7: ib2_overlap_pair<2, 1>(xa, pa, xb, pb, o); break;
      default: ib2_overlap_pair<2, 2>(xa, pa, xb, pb, o); break;
    }
  } else {
    const bool swap = swp[j];
    const double* pa = swap ? st.cb + 3 * j : st.ca + 3 * j;
    const double* pb = swap ? st.ca + 3 * j : st.cb + 3 * j;
    const double xa = swap ? st.xb[j] : st.xa[j], xb = swap ? st.xa[j] : st.xb[j];
    double* o = out + st.off[j];
    const double* pc = st.cc + 3 * j;
#define IB2_NU(A_, B_)                                                                                      \
  ib2_nuclear_pair<A_, B_>(xa, pa, xb, pb, pc, boys, o, swap ? ib2_ncart_c(B_) : 1, swap ? 1 : ib2_ncart_c(A_)); \
  break;
    switch (c) {
      case 0: IB2_NU(0, 0)
      case 1: IB2_NU(1, 0)
      case 2: IB2_NU(1, 1)
      case 3: IB2_NU(2, 0)
      case 4: IB2_NU(2, 1)
      default: IB2_NU(2, 2)
    }
#undef IB2_NU
  }
}

template <int KIND>
__global__ void __launch_bounds__(IB2_TPB, 2) ib2_thread_kernel(const Ib2Args a) {
  constexpr int kClasses = KIND == 0 ? (IB2_LT + 1) * (IB2_LT + 1) : (IB2_LT + 1) * (IB2_LT + 2) / 2;
  extern __shared__ __align__(16) unsigned char ib2_raw[];
  Ib2Stage<KIND>& st = *reinterpret_cast<Ib2Stage<KIND>*>(ib2_raw);
  const long long nchunk = ((long long)a.n + IB2_CHUNK - 1) / IB2_CHUNK;
  const long long nfull = a.bulk_ok ? (long long)a.n / IB2_CHUNK : 0;  // chunks fetched by bulk copies
  const unsigned mb0 = ib2_smem_addr(&st.full[0]), mb1 = ib2_smem_addr(&st.full[1]);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if ((long long)blockIdx.x < nfull) ib2_issue<KIND>(a, st.buf[0], blockIdx.x, mb0);
  }
  __syncthreads();
  int k = 0;
  for (long long ch = blockIdx.x; ch < nchunk; ch += gridDim.x, ++k) {
    const int b = k & 1;
    Ib2Buf<KIND>& bf = st.buf[b];
    const unsigned mb_this = b ? mb1 : mb0, mb_next = b ? mb0 : mb1;
    const long long nxt = ch + gridDim.x;
    // prefetch the next chunk into the other buffer (read by the previous
    // iteration, which ended with a block barrier)
    if (threadIdx.x == 0 && nxt < nfull) ib2_issue<KIND>(a, st.buf[b ^ 1], nxt, mb_next);
    const int p0 = (int)(ch * IB2_CHUNK);
    const int np = min(IB2_CHUNK, a.n - p0);
    if (ch < nfull) {
      const bool ok = ib2_wait(mb_this, (k >> 1) & 1, a.wait_iters);
      if (__syncthreads_or(!ok)) {  // uniform: report, drain the copies still in flight, stop
        if (threadIdx.x == 0) {
          if (a.status) atomicExch(a.status, IB_ERR_TIMEOUT);
          ib2_wait(mb_this, (k >> 1) & 1, a.wait_iters);
          if (nxt < nfull) ib2_wait(mb_next, ((k + 1) >> 1) & 1, a.wait_iters);
        }
        return;
      }
    } else {
      for (int t = threadIdx.x; t < np; t += IB2_TPB) {
        bf.xa[t] = __ldg(a.xa + p0 + t);
        bf.xb[t] = __ldg(a.xb + p0 + t);
        bf.off[t] = __ldg(a.off + p0 + t);
        bf.la[t] = __ldg(a.la + p0 + t);
        bf.lb[t] = __ldg(a.lb + p0 + t);
      }
      for (int t = threadIdx.x; t < 3 * np; t += IB2_TPB) {
        bf.ca[t] = __ldg(a.ca + 3LL * p0 + t);
        bf.cb[t] = __ldg(a.cb + 3LL * p0 + t);
        if (KIND == 1) bf.cc[t] = __ldg(a.cc + 3LL * p0 + t);
      }
    }
    if (threadIdx.x < 16) st.count[threadIdx.x] = 0;
    __syncthreads();
    // class of every staged pair; per-class counts
    for (int t = threadIdx.x; t < np; t += IB2_TPB) {
      const int la = bf.la[t], lb = bf.lb[t];
      int c = 255;
      if (ib2_bad(la, lb, a.lmax, bf.xa[t], bf.xb[t])) {
        if (a.status) atomicExch(a.status, IB_ERR_ARG);
      } else if (KIND == 0) {
        if (la <= IB2_LT && lb <= IB2_LT) c = la * (IB2_LT + 1) + lb;
      } else {
        const int hi = max(la, lb), lo = min(la, lb);
        if (hi <= IB2_LT) c = hi * (hi + 1) / 2 + lo;
        st.swp[t] = la < lb;
      }
      st.cls[t] = (unsigned char)c;
      if (c != 255) atomicAdd(&st.count[c], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int c = 0; c < kClasses; ++c) {
        st.start[c] = acc;
        acc += st.count[c];
      }
      st.start[kClasses] = acc;
      for (int c = 0; c < kClasses; ++c) st.count[c] = st.start[c];  // running insert positions
    }
    __syncthreads();
    for (int t = threadIdx.x; t < np; t += IB2_TPB) {
      const int c = st.cls[t];
      if (c != 255) st.order[atomicAdd(&st.count[c], 1)] = (short)t;
    }
    __syncthreads();
    const int total = st.start[kClasses];
    for (int i = threadIdx.x; i < total; i += IB2_TPB) {
      const int j = st.order[i];
      ib2_thread_pair<KIND>(bf, st.swp, st.cls[j], j, a.boys, a.out);
    }
    __syncthreads();  // this buffer and the sort arrays are reused
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
    ok = ok && allow_smem(ib2_thread_kernel<0>, sizeof(Ib2Stage<0>)) == cudaSuccess;
    ok = ok && allow_smem(ib2_thread_kernel<1>, sizeof(Ib2Stage<1>)) == cudaSuccess;
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

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Testing knob for the bounded waits (intception_b200_twoidx_test_stall): the
// next intception_b200_twoidx_batch call leaves one chunk's copies unissued
// and waits `iters` polls for them.  Read and cleared by that call.
std::atomic<long long> g_stall_chunk{-1};
std::atomic<int> g_stall_iters{0};
constexpr int kWaitIters = 1 << 22;

int launch(int kind, const Ib2Args& a0, int nsm, cudaStream_t s) {
  // every pair passes the thread-per-pair kernel (which also flags invalid
  // pairs); pairs with max(la, lb) > IB2_LT then take the lane-group kernel
  {
    Ib2Args at = a0;
    at.bulk_ok = aligned16(a0.xa) && aligned16(a0.xb) && aligned16(a0.ca) && aligned16(a0.cb) &&
                 aligned16(a0.off) && aligned16(a0.la) && aligned16(a0.lb) && (kind == 0 || aligned16(a0.cc));
    const long long chunks = ((long long)a0.n + IB2_CHUNK - 1) / IB2_CHUNK;
    const int grid = (int)std::max(1LL, std::min<long long>(chunks, 2LL * nsm));
    if (kind == 0)
      ib2_thread_kernel<0><<<grid, IB2_TPB, sizeof(Ib2Stage<0>), s>>>(at);
    else
      ib2_thread_kernel<1><<<grid, IB2_TPB, sizeof(Ib2Stage<1>), s>>>(at);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return IB_ERR_CUDA;
  }
  if (a0.lmax <= IB2_LT) return IB_OK;
  Ib2Args a = a0;
  a.lthr = IB2_LT;
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
  Ib2Args a = {};
  a.stall_chunk = -1;
  a.wait_iters = kWaitIters;
  a.lthr = -1;
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
  Ib2Args a = {};
  a.stall_chunk = g_stall_chunk.exchange(-1);
  a.wait_iters = g_stall_iters.exchange(0);
  if (a.wait_iters <= 0) a.wait_iters = kWaitIters;
  a.lthr = -1;
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

// Testing the bounded waits: see the header.
int intception_b200_twoidx_test_stall(long long chunk, int wait_iters) {
  if (chunk < 0 || wait_iters < 1 || wait_iters > kWaitIters)
    return ib_runtime_set_status(IB_ERR_ARG, "twoidx_test_stall: chunk >= 0, 1 <= wait_iters <= 1 << 22");
  g_stall_iters.store(wait_iters);
  g_stall_chunk.store(chunk);
  return ib_runtime_set_status(IB_OK, "");
}

}  // extern "C"
