// ib_jk.cu -- density digestion of ERI blocks: J/K energies and their nuclear
// gradient (the adjoint of the integral evaluation with respect to centres).
//
// Quartets are unique shell quartets (a>=b, c>=d, pair(ab)>=pair(cd) in the
// caller's ordering), each standing for its 8-fold permutation family with
// degeneracy deg = (a!=b ? 2:1)(c!=d ? 2:1)(ab!=cd ? 2:1).  With a real
// symmetric density P (Cartesian basis):
//   E_J = 1/2 sum_ijkl P_ij P_kl (ij|kl),   E_K = -1/4 sum_ijkl P_ik P_jl (ij|kl)
// so the symmetrised weight of one element is
//   D_ijkl = 1/2 P_ij P_kl - 1/8 (P_ik P_jl + P_il P_jk).
// Gradient: d/dA_x of a primitive x^ax y^ay z^az exp(-alpha r_A^2) is
//   2 alpha [a+1x] - ax [a-1x],
// so dE/dA_x = sum deg D (a~+1x b|cd) - ax D (a-1x b|cd), with a~ the shell with
// coefficients 2 alpha c and l+1.  The caller evaluates those auxiliary
// blocks with the ERI kernels; these kernels map every auxiliary element back
// to the component it differentiates and accumulate the atom's force, and
// the opposite contribution on centre D (translational invariance).
#include <cuda_runtime.h>

#include "../../include/intception_b200.h"
#include "ib_generic.cuh"

namespace {

__device__ __forceinline__ void jk_comp(int l, int k, int& x, int& y, int& z) {
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= k) ++s;
  z = k - s * (s + 1) / 2;
  y = s - z;
  x = l - s;
}

__device__ __forceinline__ int jk_index(int x, int y, int z) { return z + (y + z) * (y + z + 1) / 2; }

__device__ __forceinline__ double jk_weight(const double* __restrict__ P, int n, int i, int j, int k, int l) {
  const double pij = __ldg(P + (size_t)i * n + j), pkl = __ldg(P + (size_t)k * n + l);
  const double pik = __ldg(P + (size_t)i * n + k), pjl = __ldg(P + (size_t)j * n + l);
  const double pil = __ldg(P + (size_t)i * n + l), pjk = __ldg(P + (size_t)j * n + k);
  return 0.5 * pij * pkl - 0.125 * (pik * pjl + pil * pjk);
}

__device__ __forceinline__ double jk_deg(const int* s) {
  return (s[0] != s[1] ? 2.0 : 1.0) * (s[2] != s[3] ? 2.0 : 1.0) * ((s[0] != s[2] || s[1] != s[3]) ? 2.0 : 1.0);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Compensated (double-double) sums: the energy of a large system is a sum of
// ~1e8 quartet terms, and a plain sum in an order that changes with the
// quartet list (atomics, a geometry's screening) moves it by ~1e-13
// relative -- enough to swamp a central difference with h = 1e-4.
// Block partials of the energy kernel (4 doubles per block), one array per
// device: calls on one device run in stream order (JKSystem uses one stream).
#define JK_MAX_PART_BLOCKS 4096
__device__ double ib_jk_part[4 * JK_MAX_PART_BLOCKS];

struct JkDD {
  double hi, lo;
};
__device__ __forceinline__ JkDD jk_dd_add(JkDD a, double b) {  // Knuth's TwoSum
  const double s = a.hi + b, bb = s - a.hi, e = (a.hi - (s - bb)) + (b - bb);
  return {s, a.lo + e};
}
__device__ __forceinline__ JkDD jk_dd_add(JkDD a, JkDD b) {
  JkDD r = jk_dd_add(a, b.hi);
  r.lo += b.lo;
  return r;
}

// One warp per quartet.  Each lane sums its shares in plain double (a few
// hundred terms, a fixed order), the warp, block and grid sums are
// double-double: block k writes its (E_J, E_K) partials to part[4k .. 4k+3]
// and ib_jk_energy_finish adds them in block order into e_out.  The result
// does not depend on scheduling.
__global__ void ib_jk_energy_kernel(const int* __restrict__ quartets, const long long* __restrict__ out_off, int nq,
                                    const int* __restrict__ shell_l, const int* __restrict__ fofs,
                                    const double* __restrict__ P, int nbf, const double* __restrict__ blocks,
                                    double* __restrict__ part) {
  __shared__ JkDD red[2][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
  double sj = 0.0, sk = 0.0;  // this lane's plain sums: a few hundred terms in a fixed order
  for (int q = warp; q < nq; q += nwarp) {
    int s[4], n[4], f[4];
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      n[i] = ib_ncart(shell_l[s[i]]);
      f[i] = fofs[s[i]];
    }
    const double deg = jk_deg(s);
    const double* blk = blocks + out_off[q];
    const int tot = n[0] * n[1] * n[2] * n[3];
    double pj = 0.0, pk = 0.0;
    for (int e = lane; e < tot; e += 32) {
      const int ia = e % n[0], r1 = e / n[0];
      const int ib = r1 % n[1], r2 = r1 / n[1];
      const int ic = r2 % n[2], id = r2 / n[2];
      const int i = f[0] + ia, j = f[1] + ib, k = f[2] + ic, l = f[3] + id;
      const double v = blk[e];
      pj += __ldg(P + (size_t)i * nbf + j) * __ldg(P + (size_t)k * nbf + l) * v;
      pk += (__ldg(P + (size_t)i * nbf + k) * __ldg(P + (size_t)j * nbf + l) +
             __ldg(P + (size_t)i * nbf + l) * __ldg(P + (size_t)j * nbf + k)) * v;
    }
    sj += 0.5 * deg * pj;
    sk -= 0.125 * deg * pk;
  }
  // the lanes' sums over the warp in double-double, in a fixed shuffle order
  JkDD ej = {sj, 0.0}, ek = {sk, 0.0};
  for (int o = 16; o > 0; o >>= 1) {
    ej = jk_dd_add(ej, JkDD{__shfl_xor_sync(0xffffffffu, ej.hi, o), __shfl_xor_sync(0xffffffffu, ej.lo, o)});
    ek = jk_dd_add(ek, JkDD{__shfl_xor_sync(0xffffffffu, ek.hi, o), __shfl_xor_sync(0xffffffffu, ek.lo, o)});
  }
  if (lane == 0) {
    red[0][wib] = ej;
    red[1][wib] = ek;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    JkDD a = {0.0, 0.0}, b = {0.0, 0.0};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = jk_dd_add(a, red[0][w]);
      b = jk_dd_add(b, red[1][w]);
    }
    part[4 * blockIdx.x + 0] = a.hi;
    part[4 * blockIdx.x + 1] = a.lo;
    part[4 * blockIdx.x + 2] = b.hi;
    part[4 * blockIdx.x + 3] = b.lo;
  }
}

// One warp: e_out[0..1] += the partials of nb blocks (lane t takes blocks t,
// t + 32, ..., then the lanes' sums meet in a fixed shuffle order).
__global__ void ib_jk_energy_finish(const double* __restrict__ part, int nb, double* __restrict__ e_out) {
  const int lane = threadIdx.x;
  JkDD a = {0.0, 0.0}, b = {0.0, 0.0};
  for (int k = lane; k < nb; k += 32) {
    a = jk_dd_add(a, JkDD{part[4 * k], part[4 * k + 1]});
    b = jk_dd_add(b, JkDD{part[4 * k + 2], part[4 * k + 3]});
  }
  for (int o = 16; o > 0; o >>= 1) {
    a = jk_dd_add(a, JkDD{__shfl_xor_sync(0xffffffffu, a.hi, o), __shfl_xor_sync(0xffffffffu, a.lo, o)});
    b = jk_dd_add(b, JkDD{__shfl_xor_sync(0xffffffffu, b.hi, o), __shfl_xor_sync(0xffffffffu, b.lo, o)});
  }
  if (lane == 0) {
    e_out[0] += a.hi + a.lo;
    e_out[1] += b.hi + b.lo;
  }
}

// Gradient contribution of one auxiliary batch: centre `pos` (0..2) of each
// listed quartet carries level l+1 (sign > 0, shell coefficients 2 alpha c)
// or l-1 (sign < 0).  aux_off[k] locates the auxiliary block of quartet
// qidx[k] of the unique quartet list.  Forces accumulate in shared memory per
// atom and are flushed once per block.
//
// One warp per quartet.  When every shell has l <= JK_STAGE_L and the block has
// at least 128 elements, the six density
// blocks the quartet's weights read (P over the shell pairs ab, cd, ac, bd, ad,
// bc) are first copied to the warp's slice of shared memory with coalesced
// row loads, and every weight then reads shared memory: an element of the
// auxiliary block needs up to 3 weights of 6 density values each, which as
// global gathers dominated the kernel.
#define JK_STAGE_L 3
#define JK_STAGE_N 10  // ncart(JK_STAGE_L)
#define JK_WARPS 8

__device__ __forceinline__ void jk_stage(const double* __restrict__ P, int nbf, int r0, int nr, int c0, int nc,
                                         double* __restrict__ dst, int lane) {
  for (int e = lane; e < nr * nc; e += 32) {
    const int i = e / nc, j = e - i * nc;
    dst[i * JK_STAGE_N + j] = __ldg(P + (size_t)(r0 + i) * nbf + c0 + j);
  }
}

__global__ void ib_jk_force_kernel(const int* __restrict__ quartets, const int* __restrict__ qidx,
                                   const long long* __restrict__ aux_off, int naux, int pos, int sign,
                                   const int* __restrict__ shell_l, const int* __restrict__ fofs,
                                   const int* __restrict__ shell_atom, const double* __restrict__ P, int nbf,
                                   int natom, const double* __restrict__ blocks, double* __restrict__ force) {
  extern __shared__ double fs[];
  // [3 natom] force sums, then per warp 6 staged density blocks of JK_STAGE_N^2
  double* stage = fs + ((3 * natom + 1) & ~1);
  for (int i = threadIdx.x; i < 3 * natom; i += blockDim.x) fs[i] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* __restrict__ st = stage + (size_t)wib * 6 * JK_STAGE_N * JK_STAGE_N;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < naux; k += nwarp) {
    const int q = qidx[k];
    int s[4], l[4], n[4], f[4];
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      l[i] = shell_l[s[i]];
      f[i] = fofs[s[i]];
      n[i] = ib_ncart(l[i]);
    }
    const int lx = l[pos] + (sign > 0 ? 1 : -1);
    int na[4] = {n[0], n[1], n[2], n[3]};
    na[pos] = ib_ncart(lx);
    const double deg = jk_deg(s);
    const double* blk = blocks + aux_off[k];
    const int tot = na[0] * na[1] * na[2] * na[3];
    // staged blocks: 0 ab, 1 cd, 2 ac, 3 bd, 4 ad, 5 bc (rows of the first shell)
    // staging pays for large blocks only: a block of a few elements needs fewer
    // gathers than the six density blocks hold (measured: staging every quartet
    // made the 60-atom gradient's digestion 1.69 -> 2.04 s)
    const bool staged = max(max(l[0], l[1]), max(l[2], l[3])) <= JK_STAGE_L && tot >= 128;
    const int SS = JK_STAGE_N * JK_STAGE_N;
    if (staged) {
      __syncwarp();
      jk_stage(P, nbf, f[0], n[0], f[1], n[1], st + 0 * SS, lane);
      jk_stage(P, nbf, f[2], n[2], f[3], n[3], st + 1 * SS, lane);
      jk_stage(P, nbf, f[0], n[0], f[2], n[2], st + 2 * SS, lane);
      jk_stage(P, nbf, f[1], n[1], f[3], n[3], st + 3 * SS, lane);
      jk_stage(P, nbf, f[0], n[0], f[3], n[3], st + 4 * SS, lane);
      jk_stage(P, nbf, f[1], n[1], f[2], n[2], st + 5 * SS, lane);
      __syncwarp();
    }
    double g[3] = {0.0, 0.0, 0.0};
    for (int e = lane; e < tot; e += 32) {
      int idx[4];
      int r = e;
      for (int i = 0; i < 4; ++i) {
        idx[i] = r % na[i];
        r /= na[i];
      }
      const double v = deg * blk[e];
      int cx, cy, cz;
      jk_comp(lx, idx[pos], cx, cy, cz);
      int c[3] = {cx, cy, cz};
      for (int d = 0; d < 3; ++d) {
        int o[3] = {c[0], c[1], c[2]};
        double coef;
        if (sign > 0) {
          if (o[d] == 0) continue;
          o[d] -= 1;
          coef = 1.0;
        } else {
          o[d] += 1;
          coef = -(double)o[d];
        }
        int li[4] = {idx[0], idx[1], idx[2], idx[3]};  // component indices within each shell
        li[pos] = jk_index(o[0], o[1], o[2]);
        double w;
        if (staged) {
          const int N = JK_STAGE_N;
          w = 0.5 * st[0 * SS + li[0] * N + li[1]] * st[1 * SS + li[2] * N + li[3]] -
              0.125 * (st[2 * SS + li[0] * N + li[2]] * st[3 * SS + li[1] * N + li[3]] +
                       st[4 * SS + li[0] * N + li[3]] * st[5 * SS + li[1] * N + li[2]]);
        } else {
          w = jk_weight(P, nbf, f[0] + li[0], f[1] + li[1], f[2] + li[2], f[3] + li[3]);
        }
        g[d] += coef * v * w;
      }
    }
    for (int d = 0; d < 3; ++d) g[d] = warp_sum(g[d]);
    if (lane == 0) {
      const int ax = shell_atom[s[pos]], ad = shell_atom[s[3]];
      for (int d = 0; d < 3; ++d) {
        atomicAdd(&fs[3 * ax + d], g[d]);
        atomicAdd(&fs[3 * ad + d], -g[d]);  // translational invariance: d/dD = -(d/dA + d/dB + d/dC)
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * natom; i += blockDim.x)
    if (fs[i] != 0.0) atomicAdd(force + i, fs[i]);
}

// All six auxiliary batches of a quartet list at once.  aux.off[b][q] locates
// quartet q's block in aux.blk[b] (b = 2 pos + (sign < 0); -1: the quartet has
// no block there, an l = 0 shell at pos for sign < 0).  The loop runs over the
// quartet's ORIGINAL elements o: its density weight W(o) is formed once, and
// for each centre pos and direction x
//   dE/dA_pos,x += deg W(o) [(o + 1x | raised at pos) - o_x (o - 1x | lowered at pos)],
// the adjoint of the derivative rule above; centre D takes the opposite sum.
struct JkAux {
  const long long* off[6];
  const double* blk[6];
};

__global__ void ib_jk_force_all_kernel(const int* __restrict__ quartets, int nq, const JkAux aux,
                                       const int* __restrict__ shell_l, const int* __restrict__ fofs,
                                       const int* __restrict__ shell_atom, const double* __restrict__ P, int nbf,
                                       int natom, double* __restrict__ force) {
  extern __shared__ double fs[];
  double* stage = fs + ((3 * natom + 1) & ~1);
  for (int i = threadIdx.x; i < 3 * natom; i += blockDim.x) fs[i] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* __restrict__ st = stage + (size_t)wib * 6 * JK_STAGE_N * JK_STAGE_N;
  const int SS = JK_STAGE_N * JK_STAGE_N;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int q = warp; q < nq; q += nwarp) {
    int s[4], l[4], n[4], f[4];
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      l[i] = shell_l[s[i]];
      f[i] = fofs[s[i]];
      n[i] = ib_ncart(l[i]);
    }
    long long off[6];
    for (int b = 0; b < 6; ++b) off[b] = __ldg(aux.off[b] + q);
    const double deg = jk_deg(s);
    const int tot = n[0] * n[1] * n[2] * n[3];
    const bool staged = max(max(l[0], l[1]), max(l[2], l[3])) <= JK_STAGE_L && tot >= 128;
    if (staged) {
      __syncwarp();
      jk_stage(P, nbf, f[0], n[0], f[1], n[1], st + 0 * SS, lane);
      jk_stage(P, nbf, f[2], n[2], f[3], n[3], st + 1 * SS, lane);
      jk_stage(P, nbf, f[0], n[0], f[2], n[2], st + 2 * SS, lane);
      jk_stage(P, nbf, f[1], n[1], f[3], n[3], st + 3 * SS, lane);
      jk_stage(P, nbf, f[0], n[0], f[3], n[3], st + 4 * SS, lane);
      jk_stage(P, nbf, f[1], n[1], f[2], n[2], st + 5 * SS, lane);
      __syncwarp();
    }
    double g[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // [pos][x]
    for (int e = lane; e < tot; e += 32) {
      int idx[4];
      int r = e;
      for (int i = 0; i < 4; ++i) {
        idx[i] = r % n[i];
        r /= n[i];
      }
      double w;
      if (staged) {
        const int N = JK_STAGE_N;
        w = 0.5 * st[0 * SS + idx[0] * N + idx[1]] * st[1 * SS + idx[2] * N + idx[3]] -
            0.125 * (st[2 * SS + idx[0] * N + idx[2]] * st[3 * SS + idx[1] * N + idx[3]] +
                     st[4 * SS + idx[0] * N + idx[3]] * st[5 * SS + idx[1] * N + idx[2]]);
      } else {
        w = jk_weight(P, nbf, f[0] + idx[0], f[1] + idx[1], f[2] + idx[2], f[3] + idx[3]);
      }
      w *= deg;
      for (int pos = 0; pos < 3; ++pos) {
        int cx, cy, cz;
        jk_comp(l[pos], idx[pos], cx, cy, cz);
        const int c[3] = {cx, cy, cz};
        // flat index of the block with component k at pos and extent m there
        int lo = 0, stride = 1;  // contribution of the indices before pos, stride of pos
        for (int i = 0; i < pos; ++i) {
          lo += idx[i] * stride;
          stride *= n[i];
        }
        int hi = 0, hs = 1;  // indices after pos, in units of the stride after pos
        for (int i = pos + 1; i < 4; ++i) {
          hi += idx[i] * hs;
          hs *= n[i];
        }
        const int np1 = ib_ncart(l[pos] + 1), nm1 = ib_ncart(l[pos] - 1);
        const double* bp = aux.blk[2 * pos] + off[2 * pos];
        const double* bm = off[2 * pos + 1] >= 0 ? aux.blk[2 * pos + 1] + off[2 * pos + 1] : nullptr;
        for (int x = 0; x < 3; ++x) {
          int o[3] = {c[0], c[1], c[2]};
          o[x] += 1;
          double v = __ldg(bp + lo + stride * (jk_index(o[0], o[1], o[2]) + np1 * hi));
          if (c[x] > 0 && bm) {
            o[x] -= 2;
            v -= (double)c[x] * __ldg(bm + lo + stride * (jk_index(o[0], o[1], o[2]) + nm1 * hi));
          }
          g[3 * pos + x] += w * v;
        }
      }
    }
    for (int k = 0; k < 9; ++k) g[k] = warp_sum(g[k]);
    if (lane == 0) {
      const int ad = shell_atom[s[3]];
      for (int pos = 0; pos < 3; ++pos) {
        const int ax = shell_atom[s[pos]];
        for (int x = 0; x < 3; ++x) {
          atomicAdd(&fs[3 * ax + x], g[3 * pos + x]);
          atomicAdd(&fs[3 * ad + x], -g[3 * pos + x]);
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * natom; i += blockDim.x)
    if (fs[i] != 0.0) atomicAdd(force + i, fs[i]);
}

}  // namespace

extern "C" int intception_b200_jk_energy(const int* quartets, const long long* out_off, int nq, const int* shell_l,
                                         const int* fofs, const double* P, int nbf, const double* blocks,
                                         double* e_out, void* stream) {
  if (nq < 0 || (nq > 0 && (!quartets || !out_off || !shell_l || !fofs || !P || !blocks || !e_out)))
    return IB_ERR_ARG;
  if (nq == 0) return IB_OK;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IB_ERR_NODEVICE;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, wpb = threads / 32;
  int blocks_n = (nq + wpb - 1) / wpb;
  if (blocks_n > nsm * 16) blocks_n = nsm * 16;
  if (blocks_n > JK_MAX_PART_BLOCKS) blocks_n = JK_MAX_PART_BLOCKS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = nullptr;  // this device's copy of the file-scope partials array
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&part), ib_jk_part) != cudaSuccess) return IB_ERR_CUDA;
  ib_jk_energy_kernel<<<blocks_n, threads, 0, s>>>(quartets, out_off, nq, shell_l, fofs, P, nbf, blocks, part);
  ib_jk_energy_finish<<<1, 32, 0, s>>>(part, blocks_n, e_out);
  return cudaGetLastError() == cudaSuccess ? IB_OK : IB_ERR_CUDA;
}

extern "C" int intception_b200_jk_force(const int* quartets, const int* qidx, const long long* aux_off, int naux,
                                        int pos, int sign, const int* shell_l, const int* fofs,
                                        const int* shell_atom, const double* P, int nbf, int natom,
                                        const double* blocks, double* force, void* stream) {
  if (naux < 0 || pos < 0 || pos > 2 || (sign != 1 && sign != -1) || natom < 1 || natom > 4096) return IB_ERR_ARG;
  if (naux == 0) return IB_OK;
  if (!quartets || !qidx || !aux_off || !shell_l || !fofs || !shell_atom || !P || !blocks || !force)
    return IB_ERR_ARG;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IB_ERR_NODEVICE;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem =
      sizeof(double) * (((3 * (size_t)natom + 1) & ~(size_t)1) + (size_t)JK_WARPS * 6 * JK_STAGE_N * JK_STAGE_N);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(ib_jk_force_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return IB_ERR_CUDA;
  const int threads = 32 * JK_WARPS, wpb = JK_WARPS;
  int blocks_n = (naux + wpb - 1) / wpb;
  if (blocks_n > nsm * 8) blocks_n = nsm * 8;
  ib_jk_force_kernel<<<blocks_n, threads, smem, static_cast<cudaStream_t>(stream)>>>(
      quartets, qidx, aux_off, naux, pos, sign, shell_l, fofs, shell_atom, P, nbf, natom, blocks, force);
  return cudaGetLastError() == cudaSuccess ? IB_OK : IB_ERR_CUDA;
}

extern "C" int intception_b200_jk_force_all(const int* quartets, int nq, const long long* const* aux_off,
                                            const double* const* aux_blocks, const int* shell_l, const int* fofs,
                                            const int* shell_atom, const double* P, int nbf, int natom,
                                            double* force, void* stream) {
  if (nq < 0 || natom < 1 || natom > 4096) return IB_ERR_ARG;
  if (nq == 0) return IB_OK;
  if (!quartets || !aux_off || !aux_blocks || !shell_l || !fofs || !shell_atom || !P || !force) return IB_ERR_ARG;
  JkAux aux;
  for (int b = 0; b < 6; ++b) {
    if (!aux_off[b] || !aux_blocks[b]) return IB_ERR_ARG;
    aux.off[b] = aux_off[b];
    aux.blk[b] = aux_blocks[b];
  }
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IB_ERR_NODEVICE;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem =
      sizeof(double) * (((3 * (size_t)natom + 1) & ~(size_t)1) + (size_t)JK_WARPS * 6 * JK_STAGE_N * JK_STAGE_N);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(ib_jk_force_all_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return IB_ERR_CUDA;
  const int threads = 32 * JK_WARPS, wpb = JK_WARPS;
  int blocks_n = (nq + wpb - 1) / wpb;
  if (blocks_n > nsm * 8) blocks_n = nsm * 8;
  ib_jk_force_all_kernel<<<blocks_n, threads, smem, static_cast<cudaStream_t>(stream)>>>(
      quartets, nq, aux, shell_l, fofs, shell_atom, P, nbf, natom, force);
  return cudaGetLastError() == cudaSuccess ? IB_OK : IB_ERR_CUDA;
}
