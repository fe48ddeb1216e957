// Maximum spanning forest of the saddle graph, for the structure tree.
//
// The structure tree (create_group_tree / dev_do_colorize_local,
// f90:885-983, 1188-1242) colours, at each threshold rhot, the connected
// components of the groups linked by saddles > rhot.  Those components are
// exactly the components of a maximum spanning forest's edges > rhot: if two
// groups were joined by saddles > rhot but not by forest edges > rhot, the
// forest path between them would hold an edge <= rhot that a heavier saddle
// could replace, so the forest would not be maximum.  A forest has at most
// ngroups - 1 edges, against every saddle pair in the full graph, so the
// tree stage links (and watches for threshold crossings) only forest edges.
//
// Boruvka on the GPU.  Edges are ordered strictly by (saddle desc, lower
// group id, higher group id), so every component's heaviest outgoing edge is
// unique and the only cycles of the hook graph are mutual pairs.  A round:
//   best   a warp per group finds its heaviest edge to another component
//          (rows are sorted by decreasing saddle; a per-group cursor skips
//          the leading entries already inside the component for good);
//   key    the component's heaviest weight, then the smallest key at it;
//   pick   the group owning that edge names the component across it;
//   hook   a component hooks under that one (the smaller of a mutual pair
//          stays a root) and records the edge;
//   jump   pointer jumping to the roots; relabel every group.
// The forest comes back as a CSR over groups with rows sorted by decreasing
// saddle, the layout of the full saddle rows.
#include <cub/cub.cuh>

#include "engine.h"

namespace ahop {

namespace {

struct ForestArgs {
  int32_t ng;
  const int32_t* soff;     // [ng+1] saddle rows
  const int32_t* sisad;    // partner group ids (1-based)
  const double* srho;      // saddle densities, each row decreasing
  int32_t* comp;           // [ng+1] component (root group id) of each group
  int32_t* cur;            // [ng+1] row prefix known to lie inside the component
  int32_t* gbest;          // [ng+1] group's heaviest outgoing entry, -1 if none
  int32_t* parent;         // [ng+1] hook target of each component root
  int32_t* bto;            // [ng+1] component across the component's best edge
  unsigned long long* bw;  // [ng+1] component's best weight (bits; 0 = none)
  unsigned long long* bk;  // [ng+1] smallest edge key at that weight
  unsigned long long* fkey;  // [ng] forest edges: lower id << 32 | higher id
  double* fw;                // [ng] forest edge saddles
  int32_t* ctr;            // [0] forest edges, [1] hooks this round, [2] jump not finished
};

__device__ __forceinline__ unsigned long long edge_key(int32_t g, int32_t h) {
  const int32_t lo = g < h ? g : h, hi = g < h ? h : g;
  return ((unsigned long long)(unsigned)lo << 32) | (unsigned)hi;
}

__global__ void forest_init_kernel(ForestArgs F) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > F.ng) return;
  F.comp[g] = g;
  F.cur[g] = 0;
  F.gbest[g] = -1;
  F.parent[g] = g;
  F.bw[g] = 0ULL;
  F.bk[g] = ~0ULL;
  if (g < 3) F.ctr[g] = 0;
}

// a warp per group: heaviest entry of the row leading to another component
__global__ void forest_best_kernel(ForestArgs F) {
  const int32_t g = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) + 1;
  const int lane = threadIdx.x & 31;
  if (g > F.ng) return;
  const int32_t c = F.comp[g];
  const int32_t base = F.soff[g - 1], e1 = F.soff[g];
  int32_t first = -1;
  for (int32_t e = base + F.cur[g]; e < e1; e += 32) {
    const int32_t ee = e + lane;
    const bool cross = ee < e1 && F.comp[F.sisad[ee]] != c;
    const unsigned m = __ballot_sync(0xffffffffu, cross);
    if (m) {
      first = e + __ffs(m) - 1;
      break;
    }
  }
  if (lane == 0) F.cur[g] = (first < 0 ? e1 : first) - base;  // entries before `first` stay inside
  if (first < 0) {
    if (lane == 0) F.gbest[g] = -1;
    return;
  }
  // among the entries of the same saddle, the smallest key
  const double w = F.srho[first];
  unsigned long long bkey = ~0ULL;
  int32_t be = -1;
  for (int32_t e = first; e < e1; e += 32) {
    const int32_t ee = e + lane;
    const bool in = ee < e1 && F.srho[ee] == w;
    if (in) {
      const int32_t h = F.sisad[ee];
      if (F.comp[h] != c) {
        const unsigned long long k = edge_key(g, h);
        if (k < bkey) { bkey = k; be = ee; }
      }
    }
    if (!__all_sync(0xffffffffu, in)) break;  // past the run of equal saddles
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ok = __shfl_xor_sync(0xffffffffu, bkey, o);
    const int32_t oe = __shfl_xor_sync(0xffffffffu, be, o);
    if (ok < bkey) { bkey = ok; be = oe; }
  }
  if (lane == 0) {
    F.gbest[g] = be;
    atomicMax(&F.bw[c], (unsigned long long)__double_as_longlong(w));  // positive doubles order as bits
  }
}

__global__ void forest_key_kernel(ForestArgs F) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > F.ng) return;
  const int32_t be = F.gbest[g];
  if (be < 0) return;
  const int32_t c = F.comp[g];
  if ((unsigned long long)__double_as_longlong(F.srho[be]) != F.bw[c]) return;
  atomicMin(&F.bk[c], edge_key(g, F.sisad[be]));
}

__global__ void forest_pick_kernel(ForestArgs F) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > F.ng) return;
  const int32_t be = F.gbest[g];
  if (be < 0) return;
  const int32_t c = F.comp[g], h = F.sisad[be];
  if ((unsigned long long)__double_as_longlong(F.srho[be]) == F.bw[c] && edge_key(g, h) == F.bk[c])
    F.bto[c] = F.comp[h];  // the edge's key is unique, so one group per component gets here
}

__global__ void forest_hook_kernel(ForestArgs F) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (c > F.ng || F.comp[c] != c) return;
  if (F.bw[c] == 0ULL) {
    F.parent[c] = c;
    return;
  }
  const int32_t t = F.bto[c];
  const bool mutual = F.bw[t] == F.bw[c] && F.bk[t] == F.bk[c];
  if (mutual && c < t) {
    F.parent[c] = c;
    return;
  }
  F.parent[c] = t;
  const int32_t slot = atomicAdd(&F.ctr[0], 1);
  if (slot < F.ng) {
    F.fkey[slot] = F.bk[c];
    F.fw[slot] = __longlong_as_double((long long)F.bw[c]);
  }
  atomicAdd(&F.ctr[1], 1);
}

// pointer jumping over the component roots (bounded per launch; the host
// relaunches while some chain is not finished)
__global__ void forest_jump_kernel(ForestArgs F) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (c > F.ng || F.comp[c] != c) return;
  for (int it = 0; it < 32; ++it) {
    const int32_t p = F.parent[c];
    const int32_t pp = F.parent[p];
    if (pp == p) return;
    F.parent[c] = pp;
  }
  F.ctr[2] = 1;
}

__global__ void forest_relabel_kernel(ForestArgs F) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > F.ng) return;
  F.comp[g] = F.parent[F.comp[g]];
}

__global__ void forest_reset_kernel(ForestArgs F) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > F.ng) return;
  F.bw[g] = 0ULL;
  F.bk[g] = ~0ULL;
  if (g == 1) { F.ctr[1] = 0; F.ctr[2] = 0; }
}

// forest CSR: per-row counts, then both directions of every edge
__global__ void forest_count_kernel(const unsigned long long* __restrict__ fkey, int32_t nfe, int32_t* cnt) {
  const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfe) return;
  atomicAdd(&cnt[(int32_t)(fkey[f] >> 32) - 1], 1);
  atomicAdd(&cnt[(int32_t)(fkey[f] & 0xffffffffu) - 1], 1);
}

__global__ void forest_scatter_kernel(const unsigned long long* __restrict__ fkey, const double* __restrict__ fw,
                                      int32_t nfe, const int32_t* __restrict__ moff, int32_t* fill,
                                      int32_t* __restrict__ isad, double* __restrict__ rho) {
  const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfe) return;
  const int32_t lo = (int32_t)(fkey[f] >> 32), hi = (int32_t)(fkey[f] & 0xffffffffu);
  const double w = fw[f];
  int32_t p = moff[lo - 1] + atomicAdd(&fill[lo - 1], 1);
  isad[p] = hi;
  rho[p] = w;
  p = moff[hi - 1] + atomicAdd(&fill[hi - 1], 1);
  isad[p] = lo;
  rho[p] = w;
}

}  // namespace

int build_saddle_forest(Engine& E) {
  const int32_t ng = E.ngroups;
  cudaStream_t st = E.stream;
  const int T = 256;
  const size_t G = (size_t)ng + 1;
  auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t need = r256(G * 4) * 6 + r256(G * 8) * 4 + r256(64);
  AHOP_CUDA_TRY(E.d_forest.ensure(need));
  char* p = static_cast<char*>(E.d_forest.p);
  auto take = [&](size_t b) { char* q = p; p += r256(b); return q; };
  ForestArgs F;
  F.ng = ng;
  F.soff = E.d_soff.as<int32_t>();
  F.sisad = E.d_sisad.as<int32_t>();
  F.srho = E.d_srho.as<double>();
  F.comp = reinterpret_cast<int32_t*>(take(G * 4));
  F.cur = reinterpret_cast<int32_t*>(take(G * 4));
  F.gbest = reinterpret_cast<int32_t*>(take(G * 4));
  F.parent = reinterpret_cast<int32_t*>(take(G * 4));
  F.bto = reinterpret_cast<int32_t*>(take(G * 4));
  int32_t* cnt = reinterpret_cast<int32_t*>(take(G * 4));  // row counts, then fill cursors
  F.bw = reinterpret_cast<unsigned long long*>(take(G * 8));
  F.bk = reinterpret_cast<unsigned long long*>(take(G * 8));
  F.fkey = reinterpret_cast<unsigned long long*>(take(G * 8));
  F.fw = reinterpret_cast<double*>(take(G * 8));
  F.ctr = reinterpret_cast<int32_t*>(take(64));
  int32_t* h = reinterpret_cast<int32_t*>(E.h_scalars);
  const unsigned gb = (unsigned)((G + T - 1) / T);
  const unsigned wb = (unsigned)(((int64_t)ng * 32 + T - 1) / T);
  E.launches++;
  forest_init_kernel<<<gb, T, 0, st>>>(F);
  AHOP_CUDA_TRY(cudaGetLastError());
  // every round at least halves the number of components that still have an
  // outgoing edge, so 40 rounds cover any int32 group count
  int round = 0;
  for (;; ++round) {
    if (round > 40) { set_error("saddle forest: too many rounds"); return AHOP_ELIMIT; }
    E.launches += 4;
    forest_best_kernel<<<wb, T, 0, st>>>(F);
    forest_key_kernel<<<gb, T, 0, st>>>(F);
    forest_pick_kernel<<<gb, T, 0, st>>>(F);
    forest_hook_kernel<<<gb, T, 0, st>>>(F);
    AHOP_CUDA_TRY(cudaGetLastError());
    AHOP_CUDA_TRY(cudaMemcpyAsync(h, F.ctr, 8, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[1] == 0) break;
    for (int pass = 0;; ++pass) {
      if (pass > 64) { set_error("saddle forest: pointer jumping did not finish"); return AHOP_ELIMIT; }
      AHOP_CUDA_TRY(cudaMemsetAsync(F.ctr + 2, 0, 4, st));
      E.launches++;
      forest_jump_kernel<<<gb, T, 0, st>>>(F);
      AHOP_CUDA_TRY(cudaMemcpyAsync(h + 2, F.ctr + 2, 4, cudaMemcpyDeviceToHost, st));
      AHOP_CUDA_TRY(cudaStreamSynchronize(st));
      if (h[2] == 0) break;
    }
    E.launches += 2;
    forest_relabel_kernel<<<gb, T, 0, st>>>(F);
    forest_reset_kernel<<<gb, T, 0, st>>>(F);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  E.forest_rounds = round;
  const int32_t nfe = h[0];
  if (nfe >= ng && ng > 0) { set_error("saddle forest: more edges than groups - 1"); return AHOP_EINVARIANT; }
  E.forest_edges = nfe;
  // CSR, rows by decreasing saddle
  AHOP_CUDA_TRY(E.d_moff.ensure(G * 4));
  AHOP_CUDA_TRY(E.d_misad.ensure((size_t)(2 * nfe + 1) * 4 * 2));
  AHOP_CUDA_TRY(E.d_mrho.ensure((size_t)(2 * nfe + 1) * 8 * 2));
  int32_t* moff = E.d_moff.as<int32_t>();
  int32_t* isad0 = E.d_misad.as<int32_t>();
  int32_t* isad1 = isad0 + (2 * nfe + 1);
  double* rho0 = E.d_mrho.as<double>();
  double* rho1 = rho0 + (2 * nfe + 1);
  AHOP_CUDA_TRY(cudaMemsetAsync(cnt, 0, G * 4, st));
  if (nfe > 0) {
    E.launches++;
    forest_count_kernel<<<(unsigned)((nfe + T - 1) / T), T, 0, st>>>(F.fkey, nfe, cnt);
  }
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, moff, ng + 1, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, cnt, moff, ng + 1, st));
  E.m_isad = isad0;
  E.m_rho = rho0;
  if (nfe == 0) return AHOP_OK;
  AHOP_CUDA_TRY(cudaMemsetAsync(cnt, 0, G * 4, st));
  E.launches++;
  forest_scatter_kernel<<<(unsigned)((nfe + T - 1) / T), T, 0, st>>>(F.fkey, F.fw, nfe, moff, cnt, isad1, rho1);
  AHOP_CUDA_TRY(cudaGetLastError());
  tmp = 0;
  cub::DeviceSegmentedSort::SortPairsDescending(nullptr, tmp, rho1, rho0, isad1, isad0, 2 * nfe, ng, moff,
                                                moff + 1, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceSegmentedSort::SortPairsDescending(E.d_cub.p, tmp, rho1, rho0, isad1, isad0, 2 * nfe,
                                                              ng, moff, moff + 1, st));
  return AHOP_OK;
}

}  // namespace ahop
