// ib_generic.cuh -- index helpers and scratch sizing shared by host and device.
#pragma once

#define IB_GEN_BLOCK 256

__host__ __device__ inline int ib_ncart(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) / 2; }
__host__ __device__ inline int ib_ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }
__host__ __device__ inline int ib_cidx(int x, int y, int z) {
  const int l = x + y + z;
  return ib_ncum(l - 1) + z + (y + z) * (y + z + 1) / 2;
}
__host__ __device__ inline int ib_sph_offset(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += ib_ncart(k) * (2 * k + 1);
  return o;
}

struct IbGenericDims {
  int la, lb, lc, ld, L, E, F;
  int ncumE, e0, ne, f0, nf;
  long long klev;  // doubles of the largest ket level; the ket levels roll through 3 slots of this size
  long long o_acc, o_bra, o_ket, o_h0, o_h1, total;
};

__host__ __device__ inline long long ib_koff_raw(int F, int ncumE, int lf) {
  long long o = 0;
  for (int f = 1; f < lf; ++f) o += (long long)(F - f + 1) * ib_ncart(f) * ncumE;
  return o;
}

// Ket level lf (>= 1) is built from levels lf-1 and lf-2 only, and the
// contracted table takes its elements as it is built, so three slots suffice.
__host__ __device__ inline long long ib_koff(const IbGenericDims& d, int lf) { return (long long)(lf % 3) * d.klev; }

__host__ __device__ inline IbGenericDims ib_generic_dims(int la, int lb, int lc, int ld) {
  IbGenericDims d;
  d.la = la; d.lb = lb; d.lc = lc; d.ld = ld;
  d.L = la + lb + lc + ld;
  d.E = la + lb;
  d.F = lc + ld;
  d.ncumE = ib_ncum(d.E);
  d.e0 = ib_ncum(la - 1);
  d.ne = d.ncumE - d.e0;
  d.f0 = ib_ncum(lc - 1);
  d.nf = ib_ncum(d.F) - d.f0;
  // HRR / transform buffer: the largest bra layer, ket layer, or 4-index block
  long long hmax = 0;
  for (int j = 0; j <= lb; ++j) {
    long long v = (long long)(ib_ncum(d.E - j) - d.e0) * ib_ncart(j) * d.nf;
    if (v > hmax) hmax = v;
  }
  const long long nab = (long long)ib_ncart(la) * ib_ncart(lb);
  for (int j = 0; j <= ld; ++j) {
    long long v = nab * (ib_ncum(d.F - j) - d.f0) * ib_ncart(j);
    if (v > hmax) hmax = v;
  }
  // spherical stages never exceed the Cartesian block
  d.klev = 0;
  for (int lf = 1; lf <= d.F; ++lf) {
    const long long v = (long long)(d.F - lf + 1) * ib_ncart(lf) * d.ncumE;
    if (v > d.klev) d.klev = v;
  }
  d.o_acc = 0;
  d.o_bra = d.o_acc + (long long)d.ne * d.nf;
  d.o_ket = d.o_bra + (long long)(d.L + 2) * d.ncumE;
  d.o_h0 = d.o_ket + 3 * d.klev;
  d.o_h1 = d.o_h0 + hmax;
  d.total = d.o_h1 + hmax;
  return d;
}
