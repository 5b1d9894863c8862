// eri_generic.cu -- one thread block per contracted quartet, any l <= IB_LMAX.
//
// Used for the classes that have no unrolled kernel (some l > the emitted
// maximum), for quartets whose pairs are best built on their lower-l shell,
// and for the quartets the class kernels put on the redo list (HRR rounding
// estimate over the tolerance).  Same schedule as the emitted kernels (HGP:
// bra VRR, ket VRR with the electron-transfer term, contraction, bra HRR, ket
// HRR, spherical transform), but every stage is a loop over the elements of
// one recurrence level, spread over the block's threads, with the levels in
// global scratch (one slice per resident block).  FP64 throughout.
//
// Each primitive pair is built on the shell that conditions its HRR
// (ib_gen_orient): a contraction that mixes tight and diffuse exponents on
// both shells of a pair has no single good orientation (whichever shell the
// recurrences build on, some primitive pairs put the product centre far from
// it and the HRR then cancels many digits), so the quartet is evaluated in up
// to four passes, one per (bra orientation, ket orientation) that some
// primitive quartet uses, each over those primitive quartets only; the first
// pass stores the block and the others add to it.
//
// One block walks a quartet's primitive quartets one after the other, so a
// quartet of K = 8 shells alone would outlast a whole batch.  Heavy quartets
// (IB_GEN_SPLIT_MIN primitive quartets or more) therefore go to a cluster of
// CS blocks (2 or 4, chosen per launch): each pass numbers its live primitive
// quartets in order and block r of the cluster adds those numbered r, r + CS,
// ... into its own contracted table; after a cluster barrier the blocks sum the tables
// in rank order (each a share of the elements) into rank 0's, which then runs
// the HRRs and stores the block.  The sum order is fixed, so the results do
// not depend on the timing.  Clusters take heavy quartets from a ticket
// counter in list order (heaviest first in a range), then every block takes
// light quartets alone from a second one.
//
// Scratch slice layout (doubles), sizes from ib_generic_dims():
//   acc  [nf * ne]                 contracted [e0|f0] stored [f][e], e in [la,la+lb], f in [lc,lc+ld]
//   bra  [(L+2) * ncumE]           [e0|00]^(m) over every e <= la+lb
//   ket  3 * klev                  [e0|f0]^(m) of the ket levels f >= 1, level f in slot f mod 3
//   h0,h1 [hmax] ping-pong buffers for HRR and the spherical transform
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>

#include "ib_eri_device.cuh"
#include "ib_generic.cuh"

namespace cg = cooperative_groups;

namespace {

// Cartesian exponents of every cumulative component index below ncum(12)
// (every index the kernel decodes: levels up to 2 IB_LMAX), 5 bits each,
// filled once per block: the level loops read them instead of decoding.
#define IB_GEN_NCT 455
// primitive quartets tested at once (IB_GEN_CHUNK / IB_GEN_BLOCK per thread)
#define IB_GEN_CHUNK 1024
static_assert(IB_GEN_NCT == (2 * IB_LMAX + 1) * (2 * IB_LMAX + 2) * (2 * IB_LMAX + 3) / 6, "component table size");
__device__ __forceinline__ void ib_ct_get(const unsigned short* ct, int cum, int& x, int& y, int& z) {
  const unsigned v = ct[cum];
  x = v & 31;
  y = (v >> 5) & 31;
  z = v >> 10;
}

__device__ __forceinline__ void ib_comp_of(int cum, int& x, int& y, int& z) {
  // level l with ncum(l-1) <= cum < ncum(l), then the in-level index k
  int l = 0;
  while (ib_ncum(l) <= cum) ++l;
  int k = cum - ib_ncum(l - 1);
  // k = mz + (my+mz)(my+mz+1)/2 ; s = my + mz
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= k) ++s;
  z = k - s * (s + 1) / 2;
  y = s - z;
  x = l - s;
}

// Orientation of one primitive pair (exponents x0 on the pair's first shell,
// l0, and x1 on its second, l1, R apart): 0 builds it on the first shell and
// moves l1 quanta to the second by the HRR, 1 the other way round; the one
// with the smaller growth bound ((sig + |PA| + R) / (sig + |PB|))^l_moved
// (ib_hrr_kappa's per-pair term; ties: 0).  Every thread evaluates it alike.
__device__ __forceinline__ int ib_gen_orient(int l0, int l1, double x0, double x1, float R) {
  if (l1 == 0) return 0;
  if (l0 == 0) return 1;
  const float a = (float)x0, b = (float)x1, z = a + b, oz = 1.0f / z, sig = rsqrtf(z);
  const float pa = b * oz * R, pb = a * oz * R;
  const float g0 = (float)l1 * __logf((sig + pa + R) / (sig + pb));
  const float g1 = (float)l0 * __logf((sig + pb + R) / (sig + pa));
  return g1 < g0 ? 1 : 0;
}

struct IbGenShared {
  IbGenericDims d;
  double A[3], B[3], C[3], D[3], AB[3], CD[3];  // this pass's shell order
  double PA[3], WP[3], QC[3], WQ[3];
  double o2z, roz, o2e, roe, o2zpe;
  double F[4 * IB_LMAX + 1];
  int k[4], ptr[4], st[4];     // this pass's shell order
  int s0[4], l0[4], st0[4];    // the item's shell order
  int use[2];                  // per pair: bit o set when some primitive pair has orientation o
  float R[2];                  // |AB|, |CD| of the item
  long long off;
  unsigned short live[IB_GEN_CHUNK];  // this rank's live primitive quartets of the chunk (offsets)
  int wcnt[IB_GEN_BLOCK / 32];        // per warp: live primitive quartets of one round
};

// ct[cum]: the Cartesian exponents of every cumulative component index;
// em[i][e]: the index of e - 1_i (low 9 bits) and the exponent of e along i
// (above them; 0: no such component); eu[i][e]: the index of e + 1_i (0 for
// the top level, whose e + 1_i no recurrence reads).  The recurrences look
// their neighbours up here: decoding them into small arrays indexed by i put
// those arrays in local memory, written and read for every element.
__device__ __forceinline__ void ib_gen_tables(unsigned short* ct, unsigned short* em, unsigned short* eu) {
  for (int t = threadIdx.x; t < IB_GEN_NCT; t += blockDim.x) {
    int x, y, z;
    ib_comp_of(t, x, y, z);
    ct[t] = (unsigned short)(x | (y << 5) | (z << 10));
    const bool top = x + y + z == 2 * IB_LMAX;
    em[t] = x ? (unsigned short)(ib_cidx(x - 1, y, z) | (x << 9)) : 0;
    em[IB_GEN_NCT + t] = y ? (unsigned short)(ib_cidx(x, y - 1, z) | (y << 9)) : 0;
    em[2 * IB_GEN_NCT + t] = z ? (unsigned short)(ib_cidx(x, y, z - 1) | (z << 9)) : 0;
    eu[t] = top ? 0 : (unsigned short)ib_cidx(x + 1, y, z);
    eu[IB_GEN_NCT + t] = top ? 0 : (unsigned short)ib_cidx(x, y + 1, z);
    eu[2 * IB_GEN_NCT + t] = top ? 0 : (unsigned short)ib_cidx(x, y, z + 1);
  }
}

// Direction of the recurrence that builds component (x, y, z): the first
// nonzero exponent.
__device__ __forceinline__ int ib_gen_dir(int x, int y) { return x > 0 ? 0 : (y > 0 ? 1 : 2); }

// One contracted quartet, sorted item p, in the block's scratch slice w.
// CS > 1: this block is rank crank of the CS blocks of a cluster that evaluate
// the quartet together (every rank calls this with the same p); wc is rank 0's
// slice, the ranks' slices follow it slice doubles apart.
template <int CS>
__device__ __forceinline__ void ib_gen_item(const IbLaunch& a, int p, int sph, double* __restrict__ w,
                                            double* __restrict__ wc, long long slice, int crank, IbGenShared& sh,
                                            const unsigned short* __restrict__ ct,
                                            const unsigned short* __restrict__ em,
                                            const unsigned short* __restrict__ eu) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
      const IbItem it = a.items[p];
      const bool bad = it.st[0] == 0;  // an l out of range: evaluated as (ss|ss), the status already says so
      for (int i = 0; i < 4; ++i) {
        sh.s0[i] = it.s[i];
        sh.l0[i] = bad ? 0 : a.shell_l[it.s[i]];
        sh.st0[i] = it.st[i];
      }
      sh.off = it.off;
      for (int h = 0; h < 2; ++h) {
        const int s0 = it.s[2 * h], s1 = it.s[2 * h + 1];
        double R2 = 0.0;
        for (int c = 0; c < 3; ++c) {
          const double u = a.shell_xyz[3 * s0 + c] - a.shell_xyz[3 * s1 + c];
          R2 += u * u;
        }
        sh.R[h] = (float)sqrt(R2);
        const int k0 = a.shell_k[s0], k1 = a.shell_k[s1], p0 = a.shell_ptr[s0], p1 = a.shell_ptr[s1];
        int use = 0;
        for (int i = 0; i < k0 && use != 3; ++i)
          for (int j = 0; j < k1 && use != 3; ++j)
            use |= 1 << ib_gen_orient(sh.l0[2 * h], sh.l0[2 * h + 1], a.prim_exp[p0 + i], a.prim_exp[p1 + j], sh.R[h]);
        sh.use[h] = use;
      }
    }
    __syncthreads();
    bool first = true;
    for (int pass = 0; pass < 4; ++pass) {
    const int ob = pass >> 1, ok = pass & 1;
    if (!((sh.use[0] >> ob) & 1) || !((sh.use[1] >> ok) & 1)) continue;  // uniform: shared
    const bool split_b = sh.use[0] == 3, split_k = sh.use[1] == 3;
    __syncthreads();  // the previous pass is done with sh
    if (tid == 0) {
      const int ord[4] = {ob, 1 - ob, 2 + ok, 3 - ok};
      int l[4];
      for (int i = 0; i < 4; ++i) {
        const int s = sh.s0[ord[i]];
        l[i] = sh.l0[ord[i]];
        sh.k[i] = a.shell_k[s];
        sh.ptr[i] = a.shell_ptr[s];
        sh.st[i] = sh.st0[ord[i]];
        double* R = i == 0 ? sh.A : (i == 1 ? sh.B : (i == 2 ? sh.C : sh.D));
        for (int c = 0; c < 3; ++c) R[c] = a.shell_xyz[3 * s + c];
      }
      for (int c = 0; c < 3; ++c) {
        sh.AB[c] = sh.A[c] - sh.B[c];
        sh.CD[c] = sh.C[c] - sh.D[c];
      }
      sh.d = ib_generic_dims(l[0], l[1], l[2], l[3]);
    }
    __syncthreads();
    const IbGenericDims d = sh.d;
    if ((long long)d.total > slice) {
      if (tid == 0) atomicExch(a.status, 3);  // scratch slice too small for this class
      break;
    }
    double* acc = w + d.o_acc;
    double* bra = w + d.o_bra;
    double* ket = w + d.o_ket;
    for (int i = tid; i < d.ne * d.nf; i += nt) acc[i] = 0.0;
    const double RAB2 = sh.AB[0] * sh.AB[0] + sh.AB[1] * sh.AB[1] + sh.AB[2] * sh.AB[2];
    const double RCD2 = sh.CD[0] * sh.CD[0] + sh.CD[1] * sh.CD[1] + sh.CD[2] * sh.CD[2];
    const int nprim = sh.k[0] * sh.k[1] * sh.k[2] * sh.k[3];
    // The pass's live primitive quartets (not exactly zero, and of this pass's
    // orientations) are numbered in order; live quartet j belongs to rank
    // j % CS, so the ranks get equal shares of the work.  A chunk of
    // IB_GEN_CHUNK is tested in parallel, one quartet per thread and round (a
    // block prefix of warp ballots numbers them), and this rank's live ones are
    // listed in order in sh.live.  One block (CS 1) thus adds its live
    // primitive quartets in ascending order.
    int base = 0;  // live primitive quartets of the pass before the current round
    auto ranks_below = [&](int n) { return n > crank ? (n - crank + CS - 1) / CS : 0; };  // this rank's, of the first n
    for (int c0 = 0; c0 < nprim; c0 += IB_GEN_CHUNK) {
      const int mine0 = ranks_below(base);
      for (int k0 = 0; k0 < IB_GEN_CHUNK; k0 += IB_GEN_BLOCK) {
        const int pq = c0 + k0 + tid;
        bool live = false;
        if (pq < nprim) {
          int r = pq;
          const int id = r % sh.k[3]; r /= sh.k[3];
          const int ic = r % sh.k[2]; r /= sh.k[2];
          const int ib = r % sh.k[1]; r /= sh.k[1];
          const int ia = r;
          const double xa = a.prim_exp[sh.ptr[0] + ia], xb = a.prim_exp[sh.ptr[1] + ib];
          const double xc = a.prim_exp[sh.ptr[2] + ic], xd = a.prim_exp[sh.ptr[3] + id];
          // the prefactor's Gaussian exactly as below: zero means the primitive quartet adds exact zeros
          live = exp(-xa * xb * (1.0 / (xa + xb)) * RAB2 - xc * xd * (1.0 / (xc + xd)) * RCD2) != 0.0;
          // exponents in the item's order of each pair
          if (live && split_b) live = ib_gen_orient(sh.l0[0], sh.l0[1], ob ? xb : xa, ob ? xa : xb, sh.R[0]) == ob;
          if (live && split_k) live = ib_gen_orient(sh.l0[2], sh.l0[3], ok ? xd : xc, ok ? xc : xd, sh.R[1]) == ok;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, live);
        if (lane == 0) sh.wcnt[warp] = __popc(bal);
        __syncthreads();
        int before = __popc(bal & ((1u << lane) - 1u)), total = 0;
        for (int w2 = 0; w2 < nwarp; ++w2) {
          const int cnt = sh.wcnt[w2];
          before += w2 < warp ? cnt : 0;
          total += cnt;
        }
        const int j = base + before;  // the live ordinal of pq
        if (live && j % CS == crank) sh.live[(j - crank) / CS - mine0] = (unsigned short)(pq - c0);
        base += total;
        __syncthreads();  // sh.wcnt is rewritten by the next round
      }
      const int nmine = ranks_below(base) - mine0;
    for (int li = 0; li < nmine; ++li) {
      const int pq = c0 + sh.live[li];
      __syncthreads();
      if (tid == 0) {
        int r = pq;
        const int id = r % sh.k[3]; r /= sh.k[3];
        const int ic = r % sh.k[2]; r /= sh.k[2];
        const int ib = r % sh.k[1]; r /= sh.k[1];
        const int ia = r;
        const double xa = a.prim_exp[sh.ptr[0] + ia], ca = a.prim_coef[sh.ptr[0] + ia];
        const double xb = a.prim_exp[sh.ptr[1] + ib], cb = a.prim_coef[sh.ptr[1] + ib];
        const double xc = a.prim_exp[sh.ptr[2] + ic], cc = a.prim_coef[sh.ptr[2] + ic];
        const double xd = a.prim_exp[sh.ptr[3] + id], cd = a.prim_coef[sh.ptr[3] + id];
        const double zeta = xa + xb, oz = 1.0 / zeta, eta = xc + xd, oe = 1.0 / eta;
        const double ozpe = 1.0 / (zeta + eta), rho = zeta * eta * ozpe;
        double P[3], Q[3], PQ[3];
        for (int c = 0; c < 3; ++c) {
          P[c] = (xa * sh.A[c] + xb * sh.B[c]) * oz;
          Q[c] = (xc * sh.C[c] + xd * sh.D[c]) * oe;
          PQ[c] = P[c] - Q[c];
          const double W = (zeta * P[c] + eta * Q[c]) * ozpe;
          sh.PA[c] = P[c] - sh.A[c];
          sh.WP[c] = W - P[c];
          sh.QC[c] = Q[c] - sh.C[c];
          sh.WQ[c] = W - Q[c];
        }
        sh.o2z = 0.5 * oz;
        sh.roz = rho * oz;
        sh.o2e = 0.5 * oe;
        sh.roe = rho * oe;
        sh.o2zpe = 0.5 * ozpe;
        const double RPQ2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
        ib_boys_rt(rho * RPQ2, d.L, a.boys_tab, sh.F);
        const double pref = ib_two_pi52() * oz * oe * sqrt(ozpe) * ca * cb * cc * cd *
                            exp(-xa * xb * oz * RAB2 - xc * xd * oe * RCD2);
        for (int m = 0; m <= d.L; ++m) sh.F[m] *= pref;
      }
      __syncthreads();
      // ---- bra VRR, level by level: bra[m*ncumE + e]
      for (int m = tid; m <= d.L; m += nt) {
        bra[m * d.ncumE] = sh.F[m];
        if (m == 0 && d.lc == 0 && d.la == 0) acc[0] += sh.F[0];
      }
      for (int le = 1; le <= d.E; ++le) {
        __syncthreads();
        const int nce = ib_ncart(le), nm = d.L - le + 1;
        for (int idx = tid; idx < nce * nm; idx += nt) {
          const int m = idx / nce, e = ib_ncum(le - 1) + idx % nce;
          int ex, ey, ez;
          ib_ct_get(ct, e, ex, ey, ez);
          const int i = ib_gen_dir(ex, ey);
          const unsigned t1 = em[i * IB_GEN_NCT + e];
          const int e1 = t1 & 511, n = (int)(t1 >> 9) - 1;  // e - 1_i, its exponent along i
          double v = sh.PA[i] * bra[m * d.ncumE + e1] + sh.WP[i] * bra[(m + 1) * d.ncumE + e1];
          if (n > 0) {
            const int e2 = em[i * IB_GEN_NCT + e1] & 511;  // e - 2_i
            v += n * sh.o2z * (bra[m * d.ncumE + e2] - sh.roz * bra[(m + 1) * d.ncumE + e2]);
          }
          bra[m * d.ncumE + e] = v;
          if (m == 0 && d.lc == 0 && e >= d.e0) acc[e - d.e0] += v;  // f = 0 column of [f][e]
        }
      }
      // ---- ket VRR: level f stored at ket + koff(f) as [m][fcomp][e].  One warp per
      // row (m, fcomp): the f-side indices once per row; its lanes run over e, with
      // e - 1_i and the exponent of e along i from the table em
      for (int lf = 1; lf <= d.F; ++lf) {
        __syncthreads();
        const int ncf = ib_ncart(lf), nm = d.F - lf + 1, E_ = d.ncumE;
        double* dst = ket + ib_koff(d, lf);
        const double* s1 = lf == 1 ? bra : ket + ib_koff(d, lf - 1);
        const double* s2 = lf <= 2 ? bra : ket + ib_koff(d, lf - 2);  // read only when lf >= 2
        const int nc1 = ib_ncart(lf - 1), nc2 = ib_ncart(lf - 2);
        for (int row = warp; row < nm * ncf; row += nwarp) {
          const int m = row / ncf, fc = row - m * ncf;
          int fx, fy, fz;
          ib_ct_get(ct, ib_ncum(lf - 1) + fc, fx, fy, fz);
          const int i = ib_gen_dir(fx, fy);
          const unsigned tf = em[i * IB_GEN_NCT + ib_ncum(lf - 1) + fc];
          const int nn = (int)(tf >> 9) - 1;              // exponent of f - 1_i along i
          const int f1 = (int)(tf & 511) - ib_ncum(lf - 2);  // in-level index of f - 1_i at lf-1
          int f2 = 0;
          if (nn > 0) f2 = (int)(em[i * IB_GEN_NCT + (tf & 511)] & 511) - ib_ncum(lf - 3);  // f - 2_i
          const double qc = sh.QC[i], wq = sh.WQ[i], t2 = nn * sh.o2e, roe = sh.roe, o2zpe = sh.o2zpe;
          const double* __restrict__ r10 = s1 + ((size_t)m * nc1 + f1) * E_;
          const double* __restrict__ r11 = s1 + ((size_t)(m + 1) * nc1 + f1) * E_;
          const double* __restrict__ r20 = s2 + ((size_t)m * nc2 + f2) * E_;
          const double* __restrict__ r21 = s2 + ((size_t)(m + 1) * nc2 + f2) * E_;
          double* __restrict__ out = dst + ((size_t)m * ncf + fc) * E_;
          const unsigned short* emi = em + i * IB_GEN_NCT;
          const bool to_acc = m == 0 && lf >= d.lc;
          double* accc = acc + (size_t)(ib_ncum(lf - 1) + fc - d.f0) * d.ne;  // this f's row of [f][e]
#pragma unroll 4
          for (int e = lane; e < E_; e += 32) {  // unrolled: the lanes' loads of several e issue together
            double v = qc * r10[e] + wq * r11[e];
            if (nn > 0) v += t2 * (r20[e] - roe * r21[e]);
            const unsigned t = emi[e];
            if (t >> 9) v += (double)(t >> 9) * o2zpe * r11[t & 511];
            out[e] = v;
            if (to_acc && e >= d.e0) accc[e - d.e0] += v;
          }
        }
      }
    }  // this rank's live primitive quartets of the chunk
    }  // chunk
    __syncthreads();
    if (CS > 1) {
      // the ranks' contracted tables are complete: each rank sums its share of
      // the elements over the ranks, in rank order, into rank 0's table (reads
      // from L2, __ldcg: a rank's L1 may hold lines another rank has written)
      __threadfence();
      cg::this_cluster().sync();
      const int nacc = d.ne * d.nf, per = (nacc + CS - 1) / CS;
      const int x1 = min(nacc, (crank + 1) * per);
      double* __restrict__ acc0 = wc + d.o_acc;
      for (int x = crank * per + tid; x < x1; x += nt) {
        double v = __ldcg(acc0 + x);
        for (int k = 1; k < CS; ++k) v += __ldcg(acc0 + (size_t)k * slice + x);
        acc0[x] = v;
      }
      __threadfence();
      cg::this_cluster().sync();
      if (crank != 0) continue;  // rank 0 runs the HRRs and stores the block
    }
    // ---- bra HRR: [e][b][f] layers, (a, b+1i) = (a+1i, b) + AB_i (a, b)
    // the contracted table was accumulated as [f][e] (the lanes' e contiguous);
    // the HRRs read [e][f]: transpose it into h1 (the bra HRR's first layer
    // writes h0, every later stage alternates)
    double* h0 = w + d.o_h0;
    double* h1 = w + d.o_h1;
    for (int x = tid; x < d.ne * d.nf; x += nt) {
      const int e = x / d.nf, f = x - e * d.nf;
      h1[x] = CS > 1 ? __ldcg(acc + (size_t)f * d.ne + e) : acc[(size_t)f * d.ne + e];
    }
    __syncthreads();
    double* src = h1;
    for (int j = 1; j <= d.lb; ++j) {
      double* dst = (j & 1) ? h0 : h1;
      const int ne_j = ib_ncum(d.E - j) - d.e0, ne_p = ib_ncum(d.E - j + 1) - d.e0;
      const int ncb = ib_ncart(j), ncp = ib_ncart(j - 1);
      (void)ne_p;
      const int n = ne_j * ncb * d.nf;
      for (int idx = tid; idx < n; idx += nt) {
        const int f = idx % d.nf, rest = idx / d.nf;
        const int b = rest % ncb, e = rest / ncb;
        int bx, by, bz;
        ib_ct_get(ct, ib_ncum(j - 1) + b, bx, by, bz);
        const int i = ib_gen_dir(bx, by);
        const int bm = (int)(em[i * IB_GEN_NCT + ib_ncum(j - 1) + b] & 511) - ib_ncum(j - 2);  // b - 1_i
        const int ep = (int)eu[i * IB_GEN_NCT + d.e0 + e] - d.e0;                             // e + 1_i
        dst[idx] = src[((size_t)ep * ncp + bm) * d.nf + f] + sh.AB[i] * src[((size_t)e * ncp + bm) * d.nf + f];
      }
      __syncthreads();
      src = dst;
    }
    // src: [a][b][f] = [ab][f], nab = ncart(la)*ncart(lb)
    const int nab = ib_ncart(d.la) * ib_ncart(d.lb);
    for (int j = 1; j <= d.ld; ++j) {
      double* dst = (src == h0) ? h1 : h0;
      const int nc_j = ib_ncum(d.F - j) - d.f0, nc_p = ib_ncum(d.F - j + 1) - d.f0;
      const int ndj = ib_ncart(j), ndp = ib_ncart(j - 1);
      const int n = nab * nc_j * ndj;
      for (int idx = tid; idx < n; idx += nt) {
        const int dd = idx % ndj, rest = idx / ndj;
        const int c = rest % nc_j, ab = rest / nc_j;
        int dx, dy, dz;
        ib_ct_get(ct, ib_ncum(j - 1) + dd, dx, dy, dz);
        const int i = ib_gen_dir(dx, dy);
        const int dm = (int)(em[i * IB_GEN_NCT + ib_ncum(j - 1) + dd] & 511) - ib_ncum(j - 2);  // d - 1_i
        const int cp = (int)eu[i * IB_GEN_NCT + d.f0 + c] - d.f0;                              // c + 1_i
        dst[idx] = src[((size_t)ab * nc_p + cp) * ndp + dm] + sh.CD[i] * src[((size_t)ab * nc_p + c) * ndp + dm];
      }
      __syncthreads();
      src = dst;
    }
    // src: [a][b][c][d] Cartesian block
    int dims[4] = {ib_ncart(d.la), ib_ncart(d.lb), ib_ncart(d.lc), ib_ncart(d.ld)};
    const int ls[4] = {d.la, d.lb, d.lc, d.ld};
    if (sph) {
#pragma unroll  // constant axis: dims, nd and ls stay in registers
      for (int axis = 3; axis >= 0; --axis) {
        double* dst = (src == h0) ? h1 : h0;
        const int l = ls[axis], ncs = ib_ncart(l), ns = 2 * l + 1;
        const double* T = a.sph + ib_sph_offset(l);
        int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
        nd[axis] = ns;
        const int n = nd[0] * nd[1] * nd[2] * nd[3];
        int inner = 1;
        for (int k = axis + 1; k < 4; ++k) inner *= dims[k];
        for (int idx = tid; idx < n; idx += nt) {
          const int in = idx % inner, rest = idx / inner;
          const int s = rest % ns, outer = rest / ns;
          double v = 0.0;
          for (int c = 0; c < ncs; ++c) v += T[c + s * ncs] * src[((size_t)outer * ncs + c) * inner + in];
          dst[idx] = v;
        }
        __syncthreads();
        dims[axis] = ns;
        src = dst;
      }
    }
    double* o = a.out + sh.off;
    // the block's extents and strides in registers (dims is indexed by axis above)
    const int n1 = dims[1], n2 = dims[2], n3 = dims[3], n = dims[0] * n1 * n2 * n3;
    const long long st0 = sh.st[0], st1 = sh.st[1], st2 = sh.st[2], st3 = sh.st[3];
    for (int idx = tid; idx < n; idx += nt) {
      const int i3 = idx % n3, r3 = idx / n3;
      const int i2 = r3 % n2, r2 = r3 / n2;
      const int i1 = r2 % n1, i0 = r2 / n1;
      double* dst = o + i0 * st0 + i1 * st1 + i2 * st2 + i3 * st3;
      // each element once per pass; an earlier pass's stores are visible after its closing barrier
      *dst = first ? src[idx] : *dst + src[idx];
    }
    first = false;
    __syncthreads();
    }  // pass
    __syncthreads();
}

}  // namespace

// CS > 1: launched in clusters of CS blocks (ib_generic_launch); the heavy
// items are shared by a cluster, the light ones taken by single blocks.
template <int MINB, int CS>
__global__ void __launch_bounds__(IB_GEN_BLOCK, MINB) ib_eri_generic(const IbLaunch a, const IbGenWork wk, int sph,
                                                                     double* __restrict__ scratch, long long slice) {
  __shared__ IbGenShared sh;
  __shared__ unsigned short ct[IB_GEN_NCT];
  __shared__ unsigned short em[3 * IB_GEN_NCT];
  __shared__ unsigned short eu[3 * IB_GEN_NCT];
  __shared__ int ticket;
  ib_gen_tables(ct, em, eu);
  __syncthreads();
  const int tid = threadIdx.x;
  int crank = 0;
  if constexpr (CS > 1) crank = (int)cg::this_cluster().block_rank();
  double* __restrict__ w = scratch + (size_t)blockIdx.x * (size_t)slice;
  double* __restrict__ wc = w - (size_t)crank * (size_t)slice;  // rank 0's slice (ranks are consecutive blocks)
  int hb = 0, nh = 0, lb = 0, nl = 0;
  if (wk.redo) {
    nh = a.redo[0];
    nl = a.redo[1];
  } else {
    if (wk.heavy_slot >= 0) {
      hb = a.ranges[wk.heavy_slot];
      nh = a.ranges[wk.heavy_slot + 1] - hb;
    }
    lb = a.ranges[wk.light_slot];
    nl = a.ranges[wk.light_slot + 1] - lb;
  }
  // item t of the heavy list (t < nh), then of the light list
  auto item = [&](int t) -> int {
    if (t < nh) return wk.redo ? a.redo[2 + t] : hb + t;
    t -= nh;
    return wk.redo ? a.redo[2 + a.redo_cap - 1 - t] : lb + t;
  };
  if (!wk.tickets) {  // fixed order, one block per item
    for (int t = blockIdx.x; t < nh + nl; t += gridDim.x) ib_gen_item<1>(a, item(t), sph, w, w, slice, 0, sh, ct, em, eu);
    return;
  }
  if constexpr (CS > 1) {
    cg::cluster_group cl = cg::this_cluster();
    for (;;) {  // every rank takes the same sequence of items and barriers
      if (crank == 0 && tid == 0) ticket = atomicAdd(wk.tickets, 1);
      cl.sync();
      const int t = *cl.map_shared_rank(&ticket, 0);
      cl.sync();  // read by every rank before rank 0 takes the next ticket
      if (t >= nh) break;
      ib_gen_item<CS>(a, item(t), sph, w, wc, slice, crank, sh, ct, em, eu);
    }
  } else {
    for (;;) {
      if (tid == 0) ticket = atomicAdd(wk.tickets, 1);
      __syncthreads();
      const int t = ticket;
      __syncthreads();
      if (t >= nh) break;
      ib_gen_item<1>(a, item(t), sph, w, w, slice, 0, sh, ct, em, eu);
    }
  }
  for (;;) {
    if (tid == 0) ticket = atomicAdd(wk.tickets + 1, 1);
    __syncthreads();
    const int t = ticket;
    __syncthreads();
    if (t >= nl) break;
    ib_gen_item<1>(a, item(nh + t), sph, w, w, slice, 0, sh, ct, em, eu);
  }
}

// Resident blocks per SM the generic kernel is compiled for and launched
// with: INTCEPTION_B200_GENERIC_BPS = 2 (the default), 3 or 4.  More blocks
// hide more of the scratch latency but hold fewer registers per thread and
// more scratch in flight.
int ib_generic_bps() {
  static const int v = [] {
    const char* e = getenv("INTCEPTION_B200_GENERIC_BPS");
    const int x = e ? atoi(e) : 2;
    return (x == 3 || x == 4) ? x : 2;
  }();
  return v;
}

int ib_generic_split() {
  static const int v = [] {
    const char* e = getenv("INTCEPTION_B200_GENERIC_SPLIT");
    const int x = e ? atoi(e) : 2;
    return (x == 0 || x == 1) ? x : 2;
  }();
  return v;
}

int ib_generic_split_min() {
  static const int v = [] {
    const char* e = getenv("INTCEPTION_B200_GENERIC_SPLIT_MIN");
    const int x = e ? atoi(e) : IB_GEN_SPLIT_MIN;
    return x >= 1 ? x : IB_GEN_SPLIT_MIN;
  }();
  return v;
}

namespace {

// Clusters of CS blocks of the split kernel resident at once on the current
// device (cached per device; 0 when the device cannot hold one).
template <int MINB, int CS>
int split_clusters_resident() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  int v = cache[dev].load();
  if (v) return v - 1;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(CS);
  cfg.blockDim = dim3(IB_GEN_BLOCK);
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, ib_eri_generic<MINB, CS>, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;  // this launch without clusters; asked again next time
  }
  cache[dev].store(n + 1);
  return n;
}

// The launch with clusters of CS blocks (as many as fit the grid and the GPU
// at once); without clusters when none fits.
template <int MINB, int CS>
cudaError_t launch_split(int grid, cudaStream_t s, const IbLaunch& a, const IbGenWork& wk, int sph,
                         double* scratch, long long slice) {
  const int clusters = std::min(grid / CS, split_clusters_resident<MINB, CS>());
  if (clusters > 0) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(clusters * CS);
    cfg.blockDim = dim3(IB_GEN_BLOCK);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, ib_eri_generic<MINB, CS>, a, wk, sph, scratch, slice);
  }
  ib_eri_generic<MINB, 1><<<grid, IB_GEN_BLOCK, 0, s>>>(a, wk, sph, scratch, slice);
  return cudaGetLastError();
}

template <int MINB>
cudaError_t launch_bps(int grid, cudaStream_t s, const IbLaunch& a, const IbGenWork& wk, int sph, double* scratch,
                       long long slice) {
  if (wk.tickets && wk.split >= 4) return launch_split<MINB, 4>(grid, s, a, wk, sph, scratch, slice);
  if (wk.tickets && wk.split >= 2) return launch_split<MINB, 2>(grid, s, a, wk, sph, scratch, slice);
  ib_eri_generic<MINB, 1><<<grid, IB_GEN_BLOCK, 0, s>>>(a, wk, sph, scratch, slice);
  return cudaGetLastError();
}

}  // namespace

cudaError_t ib_generic_launch(int grid, cudaStream_t s, const IbLaunch& a, const IbGenWork& wk, int sph,
                              double* scratch, long long slice) {
  switch (ib_generic_bps()) {
    case 3: return launch_bps<3>(grid, s, a, wk, sph, scratch, slice);
    case 4: return launch_bps<4>(grid, s, a, wk, sph, scratch, slice);
    default: return launch_bps<2>(grid, s, a, wk, sph, scratch, slice);
  }
}

namespace {
template <int MINB>
int grid_of(int cs, int grid) {
  if (cs == 2) return 2 * std::min(grid / 2, split_clusters_resident<MINB, 2>());
  if (cs == 4) return 4 * std::min(grid / 4, split_clusters_resident<MINB, 4>());
  return grid;
}
}  // namespace

extern "C" int intception_b200_generic_grid(int cluster_size) {
  if (cluster_size != 1 && cluster_size != 2 && cluster_size != 4) return -1;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return -1;
  }
  const int grid = ib_generic_bps() * nsm;
  switch (ib_generic_bps()) {
    case 3: return grid_of<3>(cluster_size, grid);
    case 4: return grid_of<4>(cluster_size, grid);
    default: return grid_of<2>(cluster_size, grid);
  }
}
