// ib_noalloc.cu -- ERI batch entry point that allocates no device memory.
//
// For callers that cannot call cudaMalloc: a host framework that owns the whole
// device memory through its own pool allocator, or code that must not incur
// the implicit device synchronisation of cudaMalloc/cudaFree in the middle of
// its work.  Everything this path needs besides the caller's inputs and
// outputs lives in file-scope __device__ arrays of fixed size, which every GPU
// that loads the library holds until the process exits:
//   scratch  IB_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB) for the block-per-
//            quartet kernel's recurrence levels,
//   items    IB_NOALLOC_MAX_QUARTETS quartet descriptors (the per-call limit),
//   ranges, a status word, and copies of the Boys table and the spherical
//            matrices.
// The quartets are evaluated by the same block-per-quartet kernel the batch
// path uses for classes without an unrolled kernel (ib_eri_generic), FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/intception_b200.h"
#include "_gen/boys_table_data.h"
#include "ib_eri_device.cuh"
#include "ib_generic.cuh"

void build_sph_host(std::vector<double>& out);

#define IB_NOALLOC_SCRATCH_DOUBLES (size_t(4) << 20)  // 32 MiB
#define IB_NOALLOC_MAX_QUARTETS 65536

namespace {

constexpr int kNoallocSlot = 4 * IB_NCLASS;  // same generic range slot as the batch path
constexpr int kNoallocRanges = 4 * IB_NCLASS + 2;
constexpr int kSphDoubles = 28 * 13 + 21 * 11 + 15 * 9 + 10 * 7 + 6 * 5 + 3 * 3 + 1;  // l = 0..6

static __device__ __align__(256) double ib_noalloc_scratch[IB_NOALLOC_SCRATCH_DOUBLES];
static __device__ __align__(256) IbItem ib_noalloc_items[IB_NOALLOC_MAX_QUARTETS];
static __device__ __align__(256) int ib_noalloc_ranges[kNoallocRanges];
static __device__ __align__(256) int ib_noalloc_status;
static __device__ __align__(256) double ib_noalloc_boys[IB_BOYS_NPTS * IB_BOYS_NCOL];
static __device__ __align__(256) double ib_noalloc_sph[kSphDoubles];

struct NoallocDevice {
  bool ready = false;
  int nsm = 0;
  double* scratch = nullptr;
  IbItem* items = nullptr;
  int* ranges = nullptr;
  int* status = nullptr;
  double* boys = nullptr;
  double* sph = nullptr;
};
NoallocDevice g_dev[64];
std::mutex g_mu;

// Once per device, with that device current: host-side addresses of the
// arrays above (the array names in host code are only stand-ins) and the
// table contents.  cudaMemcpyToSymbol copies into existing storage.
int noalloc_setup(int dev, NoallocDevice** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  NoallocDevice& d = g_dev[dev];
  if (!d.ready) {
    if (cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.scratch, ib_noalloc_scratch) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.items, ib_noalloc_items) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.ranges, ib_noalloc_ranges) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.status, ib_noalloc_status) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.boys, ib_noalloc_boys) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.sph, ib_noalloc_sph) != cudaSuccess) return IB_ERR_CUDA;
    if (cudaMemcpyToSymbol(ib_noalloc_boys, ib_boys_host_table, sizeof(ib_boys_host_table)) != cudaSuccess)
      return IB_ERR_CUDA;
    std::vector<double> sph;
    build_sph_host(sph);
    if (sph.size() != (size_t)kSphDoubles) return IB_ERR_ARG;
    if (cudaMemcpyToSymbol(ib_noalloc_sph, sph.data(), sph.size() * sizeof(double)) != cudaSuccess)
      return IB_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return IB_OK;
}

__device__ __forceinline__ int na_pair(int la, int lb) { return la * (la + 1) / 2 + lb; }

// One descriptor per quartet, in the caller's order, with the canonical shell
// permutation (la >= lb, lc >= ld, bra pair >= ket pair; within a pair of
// equal l the more compact shell first, and a pair whose horizontal
// recurrence is ill-conditioned built on its lower-l shell, as the batch path
// orders its generic quartets) and the
// output strides that undo it; the generic range covers all of them.  A
// quartet with an l outside [0, lmax] sets IB_ERR_ARG and is marked
// (st[0] = 0): the generic kernel then writes the (ss|ss) value of its shells
// into the first element of its block, as the batch path does.
__global__ void ib_noalloc_items_kernel(const int* __restrict__ quartets, const int* __restrict__ shell_l,
                                        const int* __restrict__ shell_k, const int* __restrict__ shell_ptr,
                                        const double* __restrict__ prim_exp, const double* __restrict__ shell_xyz,
                                        const long long* __restrict__ out_off,
                                        int nq, int spherical, int lmax, IbItem* __restrict__ items,
                                        int* __restrict__ ranges, int* status) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    int s[4], l[4], n[4];
    bool bad = false;
    for (int i = 0; i < 4; ++i) {
      s[i] = quartets[4 * q + i];
      l[i] = shell_l[s[i]];
      bad |= (l[i] < 0) | (l[i] > lmax);
    }
    if (bad) {
      atomicExch(status, IB_ERR_ARG);
      for (int i = 0; i < 4; ++i) l[i] = 0;
    }
    for (int i = 0; i < 4; ++i) n[i] = spherical ? 2 * l[i] + 1 : (l[i] + 1) * (l[i] + 2) / 2;
    int st[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
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
    if (na_pair(l[0], l[1]) < na_pair(l[2], l[3])) {
      for (int k = 0; k < 2; ++k) {
        int t = s[k]; s[k] = s[k + 2]; s[k + 2] = t;
        t = l[k]; l[k] = l[k + 2]; l[k + 2] = t;
        t = st[k]; st[k] = st[k + 2]; st[k + 2] = t;
      }
    }
    if (!bad) {
      ib_compact_first(shell_k, shell_ptr, prim_exp, s, l, st);
      ib_orient_generic(shell_k, shell_ptr, prim_exp, shell_xyz, s, l, st);  // as the batch path's generic quartets
    }
    IbItem it;
    for (int i = 0; i < 4; ++i) {
      it.s[i] = s[i];
      it.st[i] = st[i];
    }
    if (bad) it.st[0] = 0;
    it.off = out_off[q];
    items[q] = it;
    if (q == 0) {
      ranges[kNoallocSlot] = 0;
      ranges[kNoallocSlot + 1] = nq;
    }
  }
}

long long noalloc_slice(int lmax) {
  long long best = 0;
  for (int a = 0; a <= lmax; ++a)  // every shell order (ib_orient_generic may build a pair on either shell)
    for (int b = 0; b <= lmax; ++b)
      for (int c = 0; c <= lmax; ++c)
        for (int d = 0; d <= lmax; ++d) best = std::max(best, ib_generic_dims(a, b, c, d).total);
  return (best + 31) / 32 * 32;
}

}  // namespace

int ib_runtime_set_status(int st, const char* msg);

extern "C" int intception_b200_eri_batch_noalloc(const intception_b200_basis* basis, const int* quartets,
                                                 const long long* out_off, int nq, int spherical, double* out,
                                                 void* stream) {
  if (!basis || nq < 0 || (nq > 0 && (!quartets || !out_off || !out)))
    return ib_runtime_set_status(IB_ERR_ARG, "eri_batch_noalloc: null argument");
  if (nq > IB_NOALLOC_MAX_QUARTETS)  // more quartets than the static descriptor array holds
    return ib_runtime_set_status(IB_ERR_ARG, "eri_batch_noalloc: more than 65536 quartets");
  if (basis->lmax < 0 || basis->lmax > IB_LMAX)
    return ib_runtime_set_status(IB_ERR_ARG, "eri_batch_noalloc: basis lmax out of range");
  if (nq == 0) return ib_runtime_set_status(IB_OK, "");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return ib_runtime_set_status(IB_ERR_NODEVICE, "eri_batch_noalloc: no CUDA device");
  NoallocDevice* d = nullptr;
  int st = noalloc_setup(dev, &d);
  if (st) return ib_runtime_set_status(st, "eri_batch_noalloc: set-up of the static arrays failed");
  const long long slice = noalloc_slice(basis->lmax);
  const long long fit = (long long)(IB_NOALLOC_SCRATCH_DOUBLES / (size_t)slice);
  if (fit < 1)  // one quartet's recurrence levels exceed the static scratch
    return ib_runtime_set_status(IB_ERR_SCRATCH, "eri_batch_noalloc: one quartet needs more than 32 MiB");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(d->status, 0, sizeof(int), s) != cudaSuccess)
    return ib_runtime_set_status(IB_ERR_CUDA, "eri_batch_noalloc: clearing the status word failed");
  const int tb = 256, nb = std::min((nq + tb - 1) / tb, 4 * d->nsm);
  ib_noalloc_items_kernel<<<nb, tb, 0, s>>>(quartets, basis->shell_l, basis->shell_k, basis->shell_ptr,
                                            basis->prim_exp, basis->shell_xyz, out_off, nq, spherical ? 1 : 0,
                                            basis->lmax, d->items,
                                            d->ranges, d->status);
  IbLaunch a;
  memset(&a, 0, sizeof(a));
  a.items = d->items;
  a.ranges = d->ranges;
  a.shell_l = basis->shell_l;
  a.shell_k = basis->shell_k;
  a.shell_ptr = basis->shell_ptr;
  a.shell_xyz = basis->shell_xyz;
  a.prim_exp = basis->prim_exp;
  a.prim_coef = basis->prim_coef;
  a.boys_tab = d->boys;
  a.sph = d->sph;
  a.out = out;
  a.status = d->status;
  a.slice_boost = 1;
  a.split_min = IB_GEN_SPLIT_MIN;  // unused here: one block per quartet, no redo list
  const long long grid = std::min<long long>({(long long)nq, (long long)ib_generic_bps() * d->nsm, fit});
  // one block per quartet in a fixed order (no tickets: nothing to zero, no cluster)
  const cudaError_t e =
      ib_generic_launch((int)grid, s, a, IbGenWork{-1, kNoallocSlot, 0, nullptr}, spherical ? 1 : 0, d->scratch, slice);
  if (e != cudaSuccess)
    return ib_runtime_set_status(IB_ERR_CUDA, (std::string("eri_batch_noalloc: ") + cudaGetErrorString(e)).c_str());
  return ib_runtime_set_status(IB_OK, "");
}

// Device status word of the allocation-free entry on the current device: waits
// for stream, then reads it (IB_OK, IB_ERR_ARG for an l out of range,
// IB_ERR_SCRATCH).  Allocates nothing.
extern "C" int intception_b200_noalloc_status(void* stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return ib_runtime_set_status(IB_ERR_NODEVICE, "noalloc_status: no CUDA device");
  NoallocDevice* d = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev[dev].ready) return ib_runtime_set_status(IB_OK, "");  // no call on this device yet
    d = &g_dev[dev];
  }
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d->status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess)
    return ib_runtime_set_status(IB_ERR_CUDA, (std::string("noalloc_status: ") + cudaGetErrorString(e)).c_str());
  ib_runtime_set_status(IB_OK, "");
  return h;
}
