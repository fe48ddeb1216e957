// Hop linking and group construction; replaces find_local_maxima
// (f90:748-881) of the reference.
//
//  * hop target: the densest of {self} and the first nhop neighbours, equal
//    densities resolved to the smallest particle index (f90:777-793);
//  * pointer jumping to the terminal peak instead of the Fortran's serial
//    chain walk (f90:819-845) -- the terminal peak of a chain is unique;
//  * peaks numbered 1..ngroups in increasing particle index (f90:797-803);
//  * members of each group in DEcreasing particle index, the order of the
//    Fortran linked lists (f90:853-861), stored as a CSR (goff, gmem);
//  * a second view of each group's members in decreasing density with
//    running density sums, used by the structure-tree stage to count and sum
//    the members above a threshold without rescanning them.
#include <cub/cub.cuh>
#include <climits>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

__global__ void hop_kernel(const double* __restrict__ dens, const int32_t* __restrict__ nei, int nstore,
                           int nhop, const int32_t* __restrict__ orig, int64_t n, double rhot,
                           int32_t* __restrict__ hop) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  double ds = dens[s];
  if (!(ds > rhot)) { hop[s] = -1; return; }
  int32_t best = (int32_t)s;
  double bd = ds;
  int32_t bo = orig[s];
  for (int i = 0; i < nhop; ++i) {
    int32_t t = nei[s * nstore + i];
    double dt = dens[t];
    int32_t ot = orig[t];
    if (dt > bd || (dt == bd && ot < bo)) { best = t; bd = dt; bo = ot; }
  }
  hop[s] = best;
}

// One pointer-doubling pass: root[s] <- root[root[s]]; flags a change.
__global__ void jump_kernel(int32_t* __restrict__ root, int64_t n, int* __restrict__ changed) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t r = root[s];
  if (r < 0) return;
  int32_t rr = root[r];
  if (rr != r) {
    root[s] = rr;
    *changed = 1;
  }
}

__global__ void peak_flag_kernel(const int32_t* __restrict__ hop, const int32_t* __restrict__ orig, int64_t n,
                                 int32_t* __restrict__ flag_orig) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  flag_orig[orig[s]] = (hop[s] == (int32_t)s) ? 1 : 0;
}

// group[s] = 1 + exclusive-scan(peak flags in particle order)[orig(root(s))]
__global__ void group_kernel(const int32_t* __restrict__ root, const int32_t* __restrict__ orig,
                             const int32_t* __restrict__ peakscan, const double* __restrict__ dens, int64_t n,
                             int32_t* __restrict__ group, double* __restrict__ densg, int32_t* __restrict__ gpeak,
                             int32_t* __restrict__ gcount) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t r = root[s];
  if (r < 0) { group[s] = 0; return; }
  int32_t g = peakscan[orig[r]] + 1;
  group[s] = g;
  atomicAdd(&gcount[g], 1);
  if (r == (int32_t)s) { densg[g] = dens[s]; gpeak[g] = (int32_t)s; }
}

// sort key: (group ascending, particle index descending); inactive particles
// last.  The index takes ob bits (2^ob > n), the group the bits above.
__global__ void member_keys_kernel(const int32_t* __restrict__ group, const int32_t* __restrict__ orig,
                                   int64_t n, int32_t ngroups, int ob, unsigned long long* __restrict__ key,
                                   int32_t* __restrict__ val) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t g = group[s];
  unsigned long long gg = (unsigned long long)(g > 0 ? g : ngroups + 1);
  key[s] = (gg << ob) | (((1ull << ob) - 1ull) - (unsigned long long)(uint32_t)orig[s]);
  val[s] = (int32_t)s;
}

__global__ void gather_rho_kernel(const int32_t* __restrict__ slots, const double* __restrict__ dens, int64_t m,
                                  double* __restrict__ rho) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  rho[i] = dens[slots[i]];
}

static int bits_for(int64_t v) {
  int b = 1;
  while ((1LL << b) <= v) ++b;
  return b;
}

int stage_hop_groups(Engine& E) {
  const int64_t n = E.n;
  const Params& P = E.prm;
  cudaStream_t st = E.stream;
  const int T = 256;
  const unsigned grid = (unsigned)((n + T - 1) / T);
  AHOP_CUDA_TRY(E.d_hop.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_root.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_group.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_peakflag.ensure((n + 1) * 4));
  int32_t* hop = E.d_hop.as<int32_t>();
  int32_t* root = E.d_root.as<int32_t>();
  E.launches++;
  hop_kernel<<<grid, T, 0, st>>>(E.d_dens.as<double>(), E.d_nei.as<int32_t>(), E.nstore, P.nhop,
                                 E.d_orig.as<int32_t>(), n, P.rho_threshold, hop);
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemcpyAsync(root, hop, n * 4, cudaMemcpyDeviceToDevice, st));
  // pointer jumping: chains strictly increase (density, -index), so they end
  // at a self-pointing peak; doubling converges in ceil(log2(chain)) passes.
  int* d_changed = reinterpret_cast<int*>(E.d_peakflag.p);  // reuse as flag before peak flags
  int* h_changed = reinterpret_cast<int*>(E.h_scalars);
  bool converged = false;
  for (int it = 0; it < 64; ++it) {
    AHOP_CUDA_TRY(cudaMemsetAsync(d_changed, 0, 4, st));
    E.launches++;
    jump_kernel<<<grid, T, 0, st>>>(root, n, d_changed);
    AHOP_CUDA_TRY(cudaGetLastError());
    AHOP_CUDA_TRY(cudaMemcpyAsync(h_changed, d_changed, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    E.hop_passes = it + 1;
    if (*h_changed == 0) { converged = true; break; }
  }
  if (!converged) { set_error("hop pointer jumping did not converge in 64 passes"); return AHOP_ELIMIT; }
  // peaks numbered in increasing particle index
  int32_t* flag = E.d_peakflag.as<int32_t>();
  E.launches++;
  peak_flag_kernel<<<grid, T, 0, st>>>(hop, E.d_orig.as<int32_t>(), n, flag);
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemsetAsync(flag + n, 0, 4, st));
  AHOP_CUDA_TRY(E.d_idx.ensure((n + 1) * 4));
  int32_t* scan = E.d_idx.as<int32_t>();  // sort scratch no longer needed
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag, scan, (int)(n + 1), st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, flag, scan, (int)(n + 1), st));
  int32_t ng = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&ng, scan + n, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  E.ngroups = ng;
  AHOP_CUDA_TRY(E.d_densg.ensure((size_t)(ng + 2) * 8));
  AHOP_CUDA_TRY(E.d_gpeak.ensure((size_t)(ng + 2) * 4));
  AHOP_CUDA_TRY(E.d_goff.ensure((size_t)(ng + 2) * 4));
  AHOP_CUDA_TRY(E.d_sad_cnt.ensure((size_t)(ng + 2) * 4));
  int32_t* gcount = E.d_sad_cnt.as<int32_t>();  // gcount[g], g = 1..ng; gcount[0] = gcount[ng+1] = 0
  AHOP_CUDA_TRY(cudaMemsetAsync(gcount, 0, (size_t)(ng + 2) * 4, st));
  E.launches++;
  group_kernel<<<grid, T, 0, st>>>(root, E.d_orig.as<int32_t>(), scan, E.d_dens.as<double>(), n,
                                   E.d_group.as<int32_t>(), E.d_densg.as<double>(), E.d_gpeak.as<int32_t>(),
                                   gcount);
  AHOP_CUDA_TRY(cudaGetLastError());
  // goff[g] = sum_{h<g} gcount[h]: group g's members occupy [goff[g], goff[g+1]); goff[ng+1] = nactive
  {
    size_t t2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t2, gcount, E.d_goff.as<int32_t>(), ng + 2, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(t2));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, t2, gcount, E.d_goff.as<int32_t>(), ng + 2, st));
  }
  // member CSR in (group asc, particle index desc)
  AHOP_CUDA_TRY(E.d_key.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_key2.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_idx2.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_gmem.ensure(n * 4));
  E.launches++;
  const int ob = bits_for(n);  // 2^ob > n > every particle index
  member_keys_kernel<<<grid, T, 0, st>>>(E.d_group.as<int32_t>(), E.d_orig.as<int32_t>(), n, ng, ob,
                                         E.d_key.as<unsigned long long>(), E.d_idx2.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  int end_bit = ob + bits_for((int64_t)ng + 2);
  if (end_bit > 64) end_bit = 64;
  tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, E.d_key.as<unsigned long long>(),
                                  E.d_key2.as<unsigned long long>(), E.d_idx2.as<int32_t>(),
                                  E.d_gmem.as<int32_t>(), (int)n, 0, end_bit, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, E.d_key.as<unsigned long long>(),
                                                E.d_key2.as<unsigned long long>(), E.d_idx2.as<int32_t>(),
                                                E.d_gmem.as<int32_t>(), (int)n, 0, end_bit, st));
  int32_t nact = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&nact, E.d_goff.as<int32_t>() + ng + 1, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  E.nactive = nact;
  return AHOP_OK;
}

}  // namespace ahop
