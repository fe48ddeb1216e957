// Saddle detection between hop groups; replaces dev_compute_saddle_list
// (f90:2433-2813) of the reference.
//
// For every member p1 of group g1 and each of its first nhop neighbours p2 in
// another group g2 > 0, the link (g1 -> g2) has value min(rho(p1), rho(p2));
// the directed saddle is the maximum over links (f90:2590-2610).  Links are
// emitted as 64-bit (g1, g2) keys, radix-sorted and max-reduced by key
// (a segmented max; no atomics, so the result is deterministic).  A pair is
// kept only if both directions exist and takes the smaller of the two values
// (f90:2650-2688).  Each group's row is then ordered by decreasing saddle
// density (f90:2762-2773).  Rows are returned as a CSR over groups 1..ngroups.
// The reference's row order among exactly equal saddle values follows its
// unstable quicksort; nothing downstream depends on that order (the colouring
// uses the row only up to the first value <= the threshold).
#include <climits>
#include <string>
#include <cub/cub.cuh>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

// Cross-group links per particle; the 64-bit total guards the 32-bit offsets.
__global__ void link_count_kernel(const int32_t* __restrict__ group, const int32_t* __restrict__ nei, int nstore,
                                  int nhop, int64_t n, int32_t* __restrict__ cnt,
                                  unsigned long long* __restrict__ total) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int c = 0;
  if (s < n) {
    const int32_t g1 = group[s];
    if (g1 > 0) {
      for (int i = 0; i < nhop; ++i) {
        const int32_t g2 = group[nei[s * nstore + i]];
        c += (g2 > 0 && g2 != g1);
      }
    }
    cnt[s] = c;
  }
  const unsigned w = __reduce_add_sync(0xffffffffu, (unsigned)c);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(total, (unsigned long long)w);
}

__global__ void link_emit_kernel(const int32_t* __restrict__ group, const int32_t* __restrict__ nei, int nstore,
                                 int nhop, const double* __restrict__ dens, int64_t n,
                                 const int32_t* __restrict__ off, unsigned long long* __restrict__ key,
                                 double* __restrict__ val) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t g1 = group[s];
  if (g1 <= 0) return;
  int32_t o = off[s];
  double d1 = dens[s];
  for (int i = 0; i < nhop; ++i) {
    int32_t t = nei[s * nstore + i];
    int32_t g2 = group[t];
    if (g2 > 0 && g2 != g1) {
      key[o] = ((unsigned long long)(uint32_t)g1 << 32) | (uint32_t)g2;
      val[o] = fmin(d1, dens[t]);
      ++o;
    }
  }
}

struct MaxOp {
  __device__ __forceinline__ double operator()(double a, double b) const { return a > b ? a : b; }
};

// keep mutual pairs; value = min of the two directions
__global__ void symmetrize_kernel(const unsigned long long* __restrict__ ukey, const double* __restrict__ uval,
                                  int32_t nu, int32_t* __restrict__ keep, double* __restrict__ sval,
                                  int32_t* __restrict__ rowcnt) {
  int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nu) return;
  unsigned long long k = ukey[i];
  uint32_t g1 = (uint32_t)(k >> 32), g2 = (uint32_t)(k & 0xffffffffu);
  unsigned long long rk = ((unsigned long long)g2 << 32) | g1;
  int32_t lo = 0, hi = nu - 1, f = -1;
  while (lo <= hi) {
    int32_t mid = (lo + hi) >> 1;
    unsigned long long mk = ukey[mid];
    if (mk == rk) { f = mid; break; }
    if (mk < rk) lo = mid + 1; else hi = mid - 1;
  }
  if (f >= 0) {
    keep[i] = 1;
    sval[i] = fmin(uval[i], uval[f]);
    atomicAdd(&rowcnt[g1], 1);
  } else {
    keep[i] = 0;
    sval[i] = 0.0;
  }
}

__global__ void compact_kernel(const unsigned long long* __restrict__ ukey, const double* __restrict__ sval,
                               const int32_t* __restrict__ keep, const int32_t* __restrict__ kpos, int32_t nu,
                               int32_t* __restrict__ isad, double* __restrict__ rho) {
  int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nu || !keep[i]) return;
  int32_t p = kpos[i];
  isad[p] = (int32_t)(ukey[i] & 0xffffffffu);
  rho[p] = sval[i];
}

int stage_saddles(Engine& E) {
  const int64_t n = E.n;
  const Params& P = E.prm;
  cudaStream_t st = E.stream;
  const int T = 256;
  const unsigned grid = (unsigned)((n + T - 1) / T);
  const int32_t ng = E.ngroups;
  // per-particle link counts and offsets
  AHOP_CUDA_TRY(E.d_idx2.ensure((n + 1) * 4));
  AHOP_CUDA_TRY(E.d_idx.ensure((n + 1) * 4));
  int32_t* cnt = E.d_idx2.as<int32_t>();
  int32_t* off = E.d_idx.as<int32_t>();
  AHOP_CUDA_TRY(E.d_flags.ensure(512));
  unsigned long long* d_total = reinterpret_cast<unsigned long long*>(E.d_flags.as<char>() + 448);
  AHOP_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, st));
  E.launches++;
  link_count_kernel<<<grid, T, 0, st>>>(E.d_group.as<int32_t>(), E.d_nei.as<int32_t>(), E.nstore, P.nhop, n, cnt,
                                        d_total);
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemsetAsync(cnt + n, 0, 4, st));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, off, (int)(n + 1), st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, cnt, off, (int)(n + 1), st));
  int32_t nlink = 0;
  unsigned long long total = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&nlink, off + n, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(&total, d_total, 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (total > (unsigned long long)INT32_MAX) {
    set_error("saddles: " + std::to_string(total) + " cross-group links exceed 32-bit offsets");
    return AHOP_ELIMIT;
  }
  const size_t nl = (size_t)(nlink > 0 ? nlink : 1);
  AHOP_CUDA_TRY(E.d_sad_key.ensure(nl * 8));
  AHOP_CUDA_TRY(E.d_sad_key2.ensure(nl * 8));
  AHOP_CUDA_TRY(E.d_sad_val.ensure(nl * 8));
  AHOP_CUDA_TRY(E.d_sad_val2.ensure(nl * 8));
  AHOP_CUDA_TRY(E.d_soff.ensure((size_t)(ng + 2) * 4));
  E.nconn = 0;
  if (nlink == 0) {
    AHOP_CUDA_TRY(cudaMemsetAsync(E.d_soff.p, 0, (size_t)(ng + 2) * 4, st));
    AHOP_CUDA_TRY(E.d_sisad.ensure(4));
    AHOP_CUDA_TRY(E.d_srho.ensure(8));
    return AHOP_OK;
  }
  E.launches++;
  link_emit_kernel<<<grid, T, 0, st>>>(E.d_group.as<int32_t>(), E.d_nei.as<int32_t>(), E.nstore, P.nhop,
                                       E.d_dens.as<double>(), n, off, E.d_sad_key.as<unsigned long long>(),
                                       E.d_sad_val.as<double>());
  AHOP_CUDA_TRY(cudaGetLastError());
  // sort links by (g1, g2)
  int gb = 1;
  while ((1LL << gb) <= (int64_t)ng + 1) ++gb;
  tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, E.d_sad_key.as<unsigned long long>(),
                                  E.d_sad_key2.as<unsigned long long>(), E.d_sad_val.as<double>(),
                                  E.d_sad_val2.as<double>(), nlink, 0, 32 + gb, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, E.d_sad_key.as<unsigned long long>(),
                                                E.d_sad_key2.as<unsigned long long>(), E.d_sad_val.as<double>(),
                                                E.d_sad_val2.as<double>(), nlink, 0, 32 + gb, st));
  // segmented max over equal keys -> unique directed saddles (ukey in d_sad_key, uval in d_sad_val)
  AHOP_CUDA_TRY(E.d_sad_keep.ensure((size_t)(nlink + 1) * 4));
  AHOP_CUDA_TRY(E.d_sad_kpos.ensure((size_t)(nlink + 2) * 4));
  int32_t* d_nu = E.d_sad_kpos.as<int32_t>() + nlink + 1;
  tmp = 0;
  cub::DeviceReduce::ReduceByKey(nullptr, tmp, E.d_sad_key2.as<unsigned long long>(),
                                 E.d_sad_key.as<unsigned long long>(), E.d_sad_val2.as<double>(),
                                 E.d_sad_val.as<double>(), d_nu, MaxOp(), nlink, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceReduce::ReduceByKey(E.d_cub.p, tmp, E.d_sad_key2.as<unsigned long long>(),
                                               E.d_sad_key.as<unsigned long long>(), E.d_sad_val2.as<double>(),
                                               E.d_sad_val.as<double>(), d_nu, MaxOp(), nlink, st));
  int32_t nu = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&nu, d_nu, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  // mutual pairs and per-row counts
  int32_t* keep = E.d_sad_keep.as<int32_t>();            // [nu+1]
  int32_t* kpos = E.d_sad_kpos.as<int32_t>();            // [nu+1]
  double* sval = E.d_sad_val2.as<double>();               // [nu]
  AHOP_CUDA_TRY(E.d_sad_cnt.ensure((size_t)(ng + 2) * 4));
  int32_t* rowcnt = E.d_sad_cnt.as<int32_t>();
  AHOP_CUDA_TRY(cudaMemsetAsync(rowcnt, 0, (size_t)(ng + 2) * 4, st));
  const unsigned gu = (unsigned)((nu + T - 1) / T);
  E.launches++;
  symmetrize_kernel<<<gu, T, 0, st>>>(E.d_sad_key.as<unsigned long long>(), E.d_sad_val.as<double>(), nu, keep,
                                      sval, rowcnt);
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemsetAsync(keep + nu, 0, 4, st));
  tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, keep, kpos, nu + 1, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, keep, kpos, nu + 1, st));
  int32_t nc = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&nc, kpos + nu, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  E.nconn = nc;
  const size_t ncs = (size_t)(nc > 0 ? nc : 1);
  AHOP_CUDA_TRY(E.d_sisad.ensure(ncs * 4));
  AHOP_CUDA_TRY(E.d_srho.ensure(ncs * 8));
  // row offsets over groups: soff[g-1] .. soff[g] for group g (rowcnt index g)
  tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, rowcnt + 1, E.d_soff.as<int32_t>(), ng + 1, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, rowcnt + 1, E.d_soff.as<int32_t>(), ng + 1, st));
  if (nc == 0) return AHOP_OK;
  // compacted (g1, g2) order == row order by g1; scatter then sort each row by decreasing saddle
  E.launches++;
  compact_kernel<<<gu, T, 0, st>>>(E.d_sad_key.as<unsigned long long>(), sval, keep, kpos, nu,
                                   E.d_sisad.as<int32_t>(), E.d_sad_val.as<double>());
  AHOP_CUDA_TRY(cudaGetLastError());
  // segmented sort by value descending within each row (payload: neighbour id)
  AHOP_CUDA_TRY(E.d_sad_key2.ensure(ncs * 8));
  int32_t* isad_sorted = reinterpret_cast<int32_t*>(E.d_sad_key2.p);
  tmp = 0;
  cub::DeviceSegmentedSort::StableSortPairsDescending(nullptr, tmp, E.d_sad_val.as<double>(), E.d_srho.as<double>(),
                                                      E.d_sisad.as<int32_t>(), isad_sorted, nc, ng,
                                                      E.d_soff.as<int32_t>(), E.d_soff.as<int32_t>() + 1, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairsDescending(
      E.d_cub.p, tmp, E.d_sad_val.as<double>(), E.d_srho.as<double>(), E.d_sisad.as<int32_t>(), isad_sorted, nc,
      ng, E.d_soff.as<int32_t>(), E.d_soff.as<int32_t>() + 1, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_sisad.p, isad_sorted, (size_t)nc * 4, cudaMemcpyDeviceToDevice, st));
  return AHOP_OK;
}

}  // namespace ahop
