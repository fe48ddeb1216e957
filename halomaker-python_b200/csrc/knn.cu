// Morton-bucketed tree build and warp-per-query periodic kNN fused with the
// SPH cubic-spline density.
//
// Replaces create_tree_structure/create_KDtree (f90:2967-3221),
// omp_find_nearest_parts/walk_tree2 (f90:2841-2962) and omp_compute_density
// (f90:2816-2838) of the reference.
//
// Layout: particles are radix-sorted by a 63-bit Morton key; leaf j holds the
// 32 consecutive sorted particles [32j, 32j+32); each internal level groups 32
// consecutive nodes of the level below.  Every node stores its padded
// axis-aligned box as centre + half-width (6 doubles).  The kNN result of a
// query is the set of its nvoisins nearest particles under the reference's
// periodic distance, ordered by (distance, particle index); distances and the
// density use the reference's exact expression order in explicitly rounded
// FP64 (no FMA), so the density matches the reference bit for bit whenever the
// neighbour order does.
#include <algorithm>
#include <cub/cub.cuh>
#include <cfloat>
#include <climits>
#include <math_constants.h>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

// ---------------------------------------------------------------- Morton keys
__device__ __forceinline__ unsigned long long spread21(unsigned int v) {
  unsigned long long x = v & 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

__device__ __forceinline__ unsigned int quant21(double v, double half, double L) {
  double u = (v + half) / L;  // [0,1) for v in [-L/2, L/2)
  double q = u * 2097152.0;
  if (!(q >= 0.0)) q = 0.0;
  if (q > 2097151.0) q = 2097151.0;
  return (unsigned int)q;
}

__global__ void morton_kernel(const double* __restrict__ pos, int64_t n, double Lx, double Ly, double Lz,
                              unsigned long long* __restrict__ key, int32_t* __restrict__ idx) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = pos[3 * i + 0], y = pos[3 * i + 1], z = pos[3 * i + 2];
  unsigned int qx = quant21(x, 0.5 * Lx, Lx), qy = quant21(y, 0.5 * Ly, Ly), qz = quant21(z, 0.5 * Lz, Lz);
  key[i] = (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz);
  idx[i] = (int32_t)i;
}

__global__ void gather_sorted_kernel(const double* __restrict__ pos, const double* __restrict__ mass,
                                     const int32_t* __restrict__ idx, int64_t n, double* __restrict__ x,
                                     double* __restrict__ y, double* __restrict__ z, double* __restrict__ m,
                                     int32_t* __restrict__ orig, int32_t* __restrict__ rank) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t o = idx[s];
  x[s] = pos[3 * (int64_t)o + 0];
  y[s] = pos[3 * (int64_t)o + 1];
  z[s] = pos[3 * (int64_t)o + 2];
  m[s] = mass[o];
  orig[s] = o;
  rank[o] = (int32_t)s;
}

// Box storage: 6 doubles per node: cx, cy, cz, wx, wy, wz (centre, padded half-width).
__device__ __forceinline__ void warp_minmax(double& lo, double& hi) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
}

// Leaf boxes: one warp per leaf.
__global__ void leaf_box_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                const double* __restrict__ z, int64_t n, int64_t nleaf, double pad,
                                double* __restrict__ box) {
  int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= nleaf) return;
  int64_t p = w * kLeaf + lane;
  bool v = p < n;
  double lx = v ? x[p] : DBL_MAX, hx = v ? x[p] : -DBL_MAX;
  double ly = v ? y[p] : DBL_MAX, hy = v ? y[p] : -DBL_MAX;
  double lz = v ? z[p] : DBL_MAX, hz = v ? z[p] : -DBL_MAX;
  warp_minmax(lx, hx);
  warp_minmax(ly, hy);
  warp_minmax(lz, hz);
  if (lane == 0) {
    double* b = box + 6 * w;
    b[0] = 0.5 * (lx + hx); b[1] = 0.5 * (ly + hy); b[2] = 0.5 * (lz + hz);
    b[3] = 0.5 * (hx - lx) + pad; b[4] = 0.5 * (hy - ly) + pad; b[5] = 0.5 * (hz - lz) + pad;
  }
}

// Internal boxes: one warp per node over its (<= 32) child boxes.
__global__ void node_box_kernel(const double* __restrict__ child, int64_t nchild, int64_t nnode,
                                double* __restrict__ box) {
  int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= nnode) return;
  int64_t c = w * kFan + lane;
  bool v = c < nchild;
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = v ? child[6 * c + k] - child[6 * c + 3 + k] : DBL_MAX;
    hi[k] = v ? child[6 * c + k] + child[6 * c + 3 + k] : -DBL_MAX;
    warp_minmax(lo[k], hi[k]);
  }
  if (lane == 0) {
    double* b = box + 6 * w;
    for (int k = 0; k < 3; ++k) {
      b[k] = 0.5 * (lo[k] + hi[k]);
      b[3 + k] = 0.5 * (hi[k] - lo[k]) * (1.0 + 1e-12) + 1e-300;
    }
  }
}

int stage_sort_and_tree(Engine& E, const double* d_pos, const double* d_mass) {
  const int64_t n = E.n;
  const Params& P = E.prm;
  cudaStream_t st = E.stream;
  AHOP_CUDA_TRY(E.d_key.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_key2.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_idx.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_idx2.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_x.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_y.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_z.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_m.ensure(n * 8));
  AHOP_CUDA_TRY(E.d_orig.ensure(n * 4));
  AHOP_CUDA_TRY(E.d_rank.ensure(n * 4));
  const int T = 256;
  unsigned grid = (unsigned)((n + T - 1) / T);
  E.launches++;
  morton_kernel<<<grid, T, 0, st>>>(d_pos, n, P.xlong, P.ylong, P.zlong, E.d_key.as<unsigned long long>(),
                                    E.d_idx.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, E.d_key.as<unsigned long long>(),
                                  E.d_key2.as<unsigned long long>(), E.d_idx.as<int32_t>(),
                                  E.d_idx2.as<int32_t>(), (int)n, 0, 63, st);
  AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
  E.cub_calls++;
  AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, E.d_key.as<unsigned long long>(),
                                                E.d_key2.as<unsigned long long>(), E.d_idx.as<int32_t>(),
                                                E.d_idx2.as<int32_t>(), (int)n, 0, 63, st));
  E.launches++;
  if (E.mass_pending) {  // host path: the masses were uploaded on the copy stream
    AHOP_CUDA_TRY(cudaStreamWaitEvent(st, E.ev_mass, 0));
    E.mass_pending = false;
  }
  gather_sorted_kernel<<<grid, T, 0, st>>>(d_pos, d_mass, E.d_idx2.as<int32_t>(), n, E.d_x.as<double>(),
                                           E.d_y.as<double>(), E.d_z.as<double>(), E.d_m.as<double>(),
                                           E.d_orig.as<int32_t>(), E.d_rank.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  // levels
  int64_t cnt = (n + kLeaf - 1) / kLeaf;
  int nlev = 0;
  int64_t off = 0;
  for (;;) {
    if (nlev >= kMaxLevels) { set_error("too many tree levels"); return AHOP_EINVAL; }
    E.lev_off[nlev] = off;
    E.lev_cnt[nlev] = cnt;
    off += cnt;
    nlev++;
    if (cnt == 1) break;
    cnt = (cnt + kFan - 1) / kFan;
  }
  E.lev_off[nlev] = off;
  E.nlev = nlev;
  AHOP_CUDA_TRY(E.d_box.ensure(off * 6 * 8));
  double* box = E.d_box.as<double>();
  double pad = 1e-12 * fmax(P.xlong, fmax(P.ylong, P.zlong));
  {
    int64_t threads = E.lev_cnt[0] * 32;
    E.launches++;
    leaf_box_kernel<<<(unsigned)((threads + T - 1) / T), T, 0, st>>>(E.d_x.as<double>(), E.d_y.as<double>(),
                                                                     E.d_z.as<double>(), n, E.lev_cnt[0], pad,
                                                                     box);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  for (int l = 1; l < nlev; ++l) {
    int64_t threads = E.lev_cnt[l] * 32;
    E.launches++;
    node_box_kernel<<<(unsigned)((threads + T - 1) / T), T, 0, st>>>(
        box + 6 * E.lev_off[l - 1], E.lev_cnt[l - 1], E.lev_cnt[l], box + 6 * E.lev_off[l]);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  return AHOP_OK;
}

// ------------------------------------------------------------------ kNN kernel
struct KnnArgs {
  const double *x, *y, *z, *m;
  const int32_t* orig;
  const double* box;
  int64_t lev_off[kMaxLevels];
  int64_t lev_cnt[kMaxLevels];
  int nlev;
  int64_t n;
  int32_t n32;  // n as int32 (n < 2^31 is checked at the boundary)
  double Lx, Ly, Lz, xyzlong;
  int nv;       // nvoisins (<= 32)
  int nstore;   // neighbours written per particle
  int32_t* nei; // [n][nstore] sorted-slot ids
  double* dens; // [n]
  int* err;     // error flag (stack overflow)
  unsigned long long* kstats;  // [0] query leaves [1] candidate leaves [2] leaf visits [3] insertions [4] overflows
  unsigned* kspill;             // per-warp candidate spill buffers [grid warps][2 * kMaxCandSpill], or null
  const float4* box32;          // boxes of every level in FP32, widened (leaf_box32_kernel)
                // profiled instances also count [5] leaves within the final radius, [6]/[7] cycles of
                // overflow/other leaves, [24..28] phase cycles of the other leaves (bound, candidates +
                // sort, seed lists, scan, density)
};

constexpr int kWarpsPerBlock = 8;
constexpr int kStack = 256;

__device__ __forceinline__ double box_dist2(const double* __restrict__ b, double qx, double qy, double qz,
                                            double Lx, double Ly, double Lz) {
  double dx = fabs(b[0] - qx); dx = fmin(dx, Lx - dx); dx = fmax(0.0, dx - b[3]);
  double dy = fabs(b[1] - qy); dy = fmin(dy, Ly - dy); dy = fmax(0.0, dy - b[4]);
  double dz = fabs(b[2] - qz); dz = fmin(dz, Lz - dz); dz = fmax(0.0, dz - b[5]);
  return dx * dx + dy * dy + dz * dz;
}

// Squared distance from the query to particle p; wrap = false (uniform over
// the warp) when every particle the caller passes lies within half a period
// of the query on each axis (same bits, fewer operations: dist2_near).
__device__ __forceinline__ double qdist2(const KnnArgs& A, bool wrap, double qx, double qy, double qz, int64_t p) {
  return wrap ? pdist2(qx, qy, qz, A.x[p], A.y[p], A.z[p], A.Lx, A.Ly, A.Lz)
              : dist2_near(qx, qy, qz, A.x[p], A.y[p], A.z[p]);
}

// The warp's running neighbour list: lane i holds the i-th nearest (ld, ls, lo):
// squared distance, sorted slot, original index; empty slots hold +inf.
struct WarpList {
  double ld;
  int32_t ls;
  double r2;   // acceptance bound: the smaller of the nv-th entry and cap
  double cap;  // an upper bound of the query's final nv-th distance known in advance (+inf: none)
};

// Insert the particles of one leaf that belong in the list.  Candidates at
// exactly the nv-th distance are taken in too: an exact distance tie is
// settled by particle index, so one that does not precede the last entry
// lands at position nv and drops out.  Particle indices are only read for
// such ties.
template <int C>
__device__ __forceinline__ void leaf_insert(const KnnArgs& A, WarpList& L, int32_t leaf, int64_t self, double qx,
                                            double qy, double qz, int lane, unsigned& nvis, unsigned& nins,
                                            bool wrap = true) {
  const int nvv = C ? C : A.nv;
  ++nvis;
  const int32_t p = leaf * kLeaf + lane;
  const bool v = (p < A.n32) && (p != (int32_t)self);
  double d = CUDART_INF;
  if (v) d = qdist2(A, wrap, qx, qy, qz, p);
  unsigned mask = __ballot_sync(0xffffffffu, v && d <= L.r2);
  if (!mask) return;
  while (mask) {
    ++nins;
    const int src = __ffs(mask) - 1;
    const double cd = __shfl_sync(0xffffffffu, d, src);
    const int32_t cs = leaf * kLeaf + src;
    bool prec = (lane < nvv) && (L.ld < cd);
    const bool tie = (lane < nvv) && (L.ld == cd);
    if (__any_sync(0xffffffffu, tie)) {
      const int32_t co = A.orig[cs];
      if (tie) prec = A.orig[L.ls] < co;
    }
    const int pos = __popc(__ballot_sync(0xffffffffu, prec));
    const double ud = __shfl_up_sync(0xffffffffu, L.ld, 1);
    const int32_t us = __shfl_up_sync(0xffffffffu, L.ls, 1);
    if (lane > pos) { L.ld = ud; L.ls = us; }
    if (lane == pos) { L.ld = cd; L.ls = cs; }
    if (lane >= nvv) { L.ld = CUDART_INF; L.ls = -1; }
    // the bound is refreshed once per leaf: a candidate that an earlier one
    // of this leaf pushed beyond the list finds every entry ahead of it
    // (pos = nv) and changes nothing
    mask &= ~(1u << src);
  }
  L.r2 = fmin(__shfl_sync(0xffffffffu, L.ld, nvv - 1), L.cap);
}

__device__ __forceinline__ bool key_less(double da, int32_t oa, double db, int32_t ob) {
  return da < db || (da == db && oa < ob);
}

// A query's 64 seed candidates: lane l holds element l (own leaf jl, lane l)
// and element 32 + l (adjacent leaf jn, lane l).  Empty ones are
// (+inf, INT_MAX) and order last.
__device__ __forceinline__ void seed_candidate(const KnnArgs& A, int64_t jl, int64_t jn, int64_t self, double qx,
                                               double qy, double qz, int e, double& d, int32_t& o, bool wrap) {
  const int64_t p = (e < 32) ? jl * kLeaf + e : jn * kLeaf + (e - 32);
  d = CUDART_INF;
  o = INT_MAX;
  if ((e < 32 || (jn >= 0 && jn != jl)) && p < A.n && p != self) {
    d = qdist2(A, wrap, qx, qy, qz, p);
    o = A.orig[p];
  }
}

// Sort a query's 64 seed candidates by (distance, index) with a warp bitonic
// network (two per lane, element 2*lane + slot), write the element numbers of
// the first 32 in order to list[0..31], and return the nv-th smallest
// distance (+inf when fewer than nv exist) to every lane.
template <int C>
__device__ __forceinline__ double seed_sort(const KnnArgs& A, int64_t jl, int64_t jn, int64_t self, double qx,
                                           double qy, double qz, int lane, unsigned char* list, bool wrap) {
  const int nvv = C ? C : A.nv;
  double d0, d1;
  int32_t o0, o1, s0 = lane, s1 = 32 + lane;
  seed_candidate(A, jl, jn, self, qx, qy, qz, lane, d0, o0, wrap);
  seed_candidate(A, jl, jn, self, qx, qy, qz, 32 + lane, d1, o1, wrap);
#pragma unroll
  for (int size = 2; size <= 64; size <<= 1) {
    const bool asc = ((2 * lane) & size) == 0;  // same for both elements of the lane
#pragma unroll
    for (int stride = size >> 1; stride >= 1; stride >>= 1) {
      if (stride == 1) {
        const bool sw = asc ? key_less(d1, o1, d0, o0) : key_less(d0, o0, d1, o1);
        if (sw) {
          const double td = d0; d0 = d1; d1 = td;
          const int32_t to = o0; o0 = o1; o1 = to;
          const int32_t ts = s0; s0 = s1; s1 = ts;
        }
      } else {
        const int ls = stride >> 1;  // partner lane distance
        const double pd0 = __shfl_xor_sync(0xffffffffu, d0, ls), pd1 = __shfl_xor_sync(0xffffffffu, d1, ls);
        const int32_t po0 = __shfl_xor_sync(0xffffffffu, o0, ls), po1 = __shfl_xor_sync(0xffffffffu, o1, ls);
        const int32_t ps0 = __shfl_xor_sync(0xffffffffu, s0, ls), ps1 = __shfl_xor_sync(0xffffffffu, s1, ls);
        const bool kmin = (((lane & ls) == 0) == asc);  // this lane keeps the smaller of the pair
        if (kmin ? key_less(pd0, po0, d0, o0) : key_less(d0, o0, pd0, po0)) { d0 = pd0; o0 = po0; s0 = ps0; }
        if (kmin ? key_less(pd1, po1, d1, o1) : key_less(d1, o1, pd1, po1)) { d1 = pd1; o1 = po1; s1 = ps1; }
      }
    }
  }
  // sorted element 2*lane + slot; the first 32 are in lanes 0..15
  if (lane < 16) {
    list[2 * lane] = (unsigned char)s0;
    list[2 * lane + 1] = (unsigned char)s1;
  }
  const int e = nvv - 1;
  const double a = __shfl_sync(0xffffffffu, d0, e >> 1), b = __shfl_sync(0xffffffffu, d1, e >> 1);
  return (e & 1) ? b : a;
}

// The same sort on distances alone: a squared distance is non-negative, so
// its bit pattern orders like its value.  seed_key gives those bits for
// element e of a query's 64 seed candidates (+inf for none).
__device__ __forceinline__ unsigned long long seed_key(const KnnArgs& A, int64_t jl, int64_t jn, int64_t self,
                                                       double qx, double qy, double qz, int e, bool wrap) {
  const int64_t p = (e < 32) ? jl * kLeaf + e : jn * kLeaf + (e - 32);
  double d = CUDART_INF;
  if ((e < 32 || (jn >= 0 && jn != jl)) && p < A.n && p != self)
    d = qdist2(A, wrap, qx, qy, qz, p);
  return (unsigned long long)__double_as_longlong(d);
}

// The same sort on 32-bit keys: the squared distance rounded up to float
// (rounding is monotone and non-negative floats order like their bits), its
// 6 lowest bits replaced by the element number, so one 32-bit value moves
// through the network.  The order is exact between keys whose upper 26 bits
// differ; the list needs the first 33 elements in exact (distance, index)
// order, so when two neighbours among them share those bits (distances
// within about 2^-17 relative, or exact ties) the function returns false and
// the caller sorts again exactly with the particle indices (seed_sort).
// Empty candidates (+inf) may share them: they are never list entries.
template <int C>
__device__ __forceinline__ bool seed_sort_keys(const KnnArgs& A, int64_t jl, int64_t jn, int64_t self, double qx,
                                               double qy, double qz, int lane, unsigned char* list, double& kth,
                                               bool wrap) {
  const int nvv = C ? C : A.nv;
  const unsigned kInfHi = 0x7F800000u >> 6;
  auto key32 = [&](int e) {
    const double d = __longlong_as_double((long long)seed_key(A, jl, jn, self, qx, qy, qz, e, wrap));
    return (__float_as_uint(__double2float_ru(d)) & ~63u) | (unsigned)e;
  };
  unsigned k0 = key32(lane), k1 = key32(32 + lane);
#pragma unroll
  for (int size = 2; size <= 64; size <<= 1) {
    const bool asc = ((2 * lane) & size) == 0;
#pragma unroll
    for (int stride = size >> 1; stride >= 1; stride >>= 1) {
      if (stride == 1) {
        if (asc ? (k1 < k0) : (k0 < k1)) {
          const unsigned tk = k0; k0 = k1; k1 = tk;
        }
      } else {
        const int ls = stride >> 1;
        const unsigned pk0 = __shfl_xor_sync(0xffffffffu, k0, ls), pk1 = __shfl_xor_sync(0xffffffffu, k1, ls);
        const bool kmin = (((lane & ls) == 0) == asc);
        if (kmin ? (pk0 < k0) : (k0 < pk0)) k0 = pk0;
        if (kmin ? (pk1 < k1) : (k1 < pk1)) k1 = pk1;
      }
    }
  }
  // sorted element 2*lane + slot: neighbours (e, e + 1), e < 32, sharing the upper bits
  const unsigned h0 = k0 >> 6, h1 = k1 >> 6;
  const unsigned nx = __shfl_down_sync(0xffffffffu, h0, 1);
  const bool tie = lane < 16 && ((h0 == h1 && h0 != kInfHi) || (h1 == nx && h1 != kInfHi));
  if (__any_sync(0xffffffffu, tie)) return false;
  if (lane < 16) {
    list[2 * lane] = (unsigned char)(k0 & 63u);
    list[2 * lane + 1] = (unsigned char)(k1 & 63u);
  }
  // the nv-th distance, rounded up (a bound for the candidate search), +inf
  // when fewer than nv candidates exist
  const int e = nvv - 1;
  const unsigned a = __shfl_sync(0xffffffffu, k0, e >> 1), b = __shfl_sync(0xffffffffu, k1, e >> 1);
  const unsigned kk = (e & 1) ? b : a;
  kth = (kk >> 6) == kInfHi ? CUDART_INF : (double)__uint_as_float(kk | 63u);
  return true;
}

// A query's first list: the nv smallest (distance, index) pairs of its 64
// seed candidates, rebuilt from the order seed_sort recorded (one distance
// per lane, the same expression, so the same bits).
template <int C>
__device__ __forceinline__ void seed_list(const KnnArgs& A, WarpList& L, int64_t jl, int64_t jn, int64_t self,
                                          double qx, double qy, double qz, int lane, const unsigned char* list,
                                          unsigned& nvis, bool wrap) {
  const int nvv = C ? C : A.nv;
  const int e = list[lane];
  const double d = __longlong_as_double((long long)seed_key(A, jl, jn, self, qx, qy, qz, e, wrap));
  const int64_t p = (e < 32) ? jl * kLeaf + e : jn * kLeaf + (e - 32);
  L.ld = d;
  L.ls = (d < CUDART_INF) ? (int32_t)p : -1;
  if (lane >= nvv) { L.ld = CUDART_INF; L.ls = -1; }
  L.r2 = fmin(__shfl_sync(0xffffffffu, L.ld, nvv - 1), L.cap);
  nvis += (jn >= 0 && jn != jl) ? 2 : 1;
}

// Per-query depth-first traversal from the root, nearest child first (used
// when a query leaf's candidate list overflows).  Leaves skip0/skip1 were
// already scanned.
template <int C>
__device__ void query_dfs(const KnnArgs& A, WarpList& L, int64_t s, double qx, double qy, double qz, int lane,
                          int32_t* s_node, double* s_bd, int64_t skip0, int64_t skip1, unsigned& nvis, unsigned& nins) {
  const int top = A.nlev - 1;
  int sp = 0;
  if (lane == 0) { s_node[0] = (top << 27) | 0; s_bd[0] = 0.0; }
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    --sp;
    const int32_t ent = s_node[sp];
    const double bd = s_bd[sp];
    __syncwarp();
    if (!(bd < L.r2)) continue;
    const int lvl = ent >> 27;
    const int64_t j = ent & ((1 << 27) - 1);
    if (lvl == 0) {
      if (j == skip0 || j == skip1) continue;
      leaf_insert<C>(A, L, j, s, qx, qy, qz, lane, nvis, nins);
      continue;
    }
    const int64_t c = j * kFan + lane;
    const bool valid = c < A.lev_cnt[lvl - 1];
    double bdc = CUDART_INF;
    if (valid) bdc = box_dist2(A.box + 6 * (A.lev_off[lvl - 1] + c), qx, qy, qz, A.Lx, A.Ly, A.Lz);
    const bool cand = valid && bdc < L.r2;
    const unsigned mask = __ballot_sync(0xffffffffu, cand);
    if (!mask) continue;
    const int cnt = __popc(mask);
    if (sp + cnt > kStack) {  // cannot happen for <= 7 levels; guard anyway
      if (lane == 0) atomicExch(A.err, 1);
      break;
    }
    double best = cand ? bdc : CUDART_INF;
    int bl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int ol = __shfl_xor_sync(0xffffffffu, bl, o);
      if (ob < best || (ob == best && ol < bl)) { best = ob; bl = ol; }
    }
    if (cand) {
      int r = __popc(mask & ((1u << lane) - 1));
      int slot;
      if (lane == bl) slot = sp + cnt - 1;
      else {
        int rb = __popc(mask & ((1u << bl) - 1));
        slot = sp + (r < rb ? r : r - 1);
      }
      s_node[slot] = ((lvl - 1) << 27) | (int32_t)c;
      s_bd[slot] = bdc;
    }
    sp += cnt;
    __syncwarp();
  }
}

// SPH density (f90:2816-2838) in the exact evaluation order, and the stored
// neighbour slots.  The nv - 1 terms are summed in list order by lane 0 from
// the warp's scratch st (32 doubles of shared memory), not with a shuffle per
// term.
template <int C>
__device__ __forceinline__ void finish_query(const KnnArgs& A, const WarpList& L, int64_t s, int lane, double* st) {
  const int nv = C ? C : A.nv;
  const double dlast = __shfl_sync(0xffffffffu, L.ld, nv - 1);
  const double r = xmul(xsqrt(dlast), 0.5);
  const double r3 = xmul(xmul(r, r), r);
  const double unsr = xdiv(1.0, r);
  double term = 0.0;
  if (lane < nv - 1) term = xmul(A.m[L.ls], spline(xmul(xsqrt(L.ld), unsr)));
  st[lane] = term;
  __syncwarp();
  if (lane == 0) {
    double contrib = 0.0;
    for (int i = 0; i < nv - 1; ++i) contrib = xadd(contrib, st[i]);
    const double pi_f = (double)3.141592654f;  // f90:58 single-precision literal
    A.dens[s] = xdiv(xmul(A.xyzlong, xadd(contrib, A.m[s])), xmul(pi_f, r3));
  }
  if (lane < A.nstore) A.nei[s * A.nstore + lane] = L.ls;
  __syncwarp();  // st is the fallback search stack of the next query
}

// Boxes in FP32 for the candidate tests: centre rounded to
// float, half width widened to cover that rounding plus every rounding of the
// FP32 test below (2^-21 L), so the FP32 distance is never above the exact
// point-to-box distance: a pruning bound, looser by a negligible margin.
__global__ void leaf_box32_kernel(const double* __restrict__ box, int64_t nleaf, double Lmax,
                                  float4* __restrict__ out) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nleaf) return;
  const double* b = box + 6 * j;
  const double pad = Lmax * 0x1p-21;
  float c[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c[k] = (float)b[k];
    w[k] = __double2float_ru(b[3 + k] + fabs(b[k] - (double)c[k]) + pad);
  }
  out[2 * j] = make_float4(c[0], c[1], c[2], 0.f);
  out[2 * j + 1] = make_float4(w[0], w[1], w[2], 0.f);
}

// Lower bound of the squared periodic distance from (qx, qy, qz) (as floats)
// to a leaf's FP32 box, rounded down at every step.
__device__ __forceinline__ float box_dist2_lb(const float4* __restrict__ b, float qx, float qy, float qz, float Lx,
                                              float Ly, float Lz) {
  const float4 c = b[0], w = b[1];
  float dx = fabsf(c.x - qx); dx = fminf(dx, Lx - dx); dx = fmaxf(0.f, __fsub_rd(dx, w.x));
  float dy = fabsf(c.y - qy); dy = fminf(dy, Ly - dy); dy = fmaxf(0.f, __fsub_rd(dy, w.y));
  float dz = fabsf(c.z - qz); dz = fminf(dz, Lz - dz); dz = fmaxf(0.f, __fsub_rd(dz, w.z));
  return __fadd_rd(__fadd_rd(__fmul_rd(dx, dx), __fmul_rd(dy, dy)), __fmul_rd(dz, dz));
}

// True when every particle of the leaf with FP32 box b (which contains the
// leaf's exact box) lies within half a period of the query on each axis, so
// that dist2_near applies.  Evaluated in FP64 (float operands are exact
// there) with a margin of 2^-30 L for its own roundings.
__device__ __forceinline__ bool near_box(const float4* __restrict__ b, double qx, double qy, double qz, double Lx,
                                         double Ly, double Lz) {
  const float4 c = b[0], w = b[1];
  return fabs((double)c.x - qx) + (double)w.x <= Lx * (0.5 - 0x1p-30) &&
         fabs((double)c.y - qy) + (double)w.y <= Ly * (0.5 - 0x1p-30) &&
         fabs((double)c.z - qz) + (double)w.z <= Lz * (0.5 - 0x1p-30);
}

// near_box in FP32 for a query (qx, qy, qz) rounded to float (|q - qf| <=
// 2^-25 L for |q| <= L/2): |c - qf| rounded up, plus w rounded up, against
// lim = L (1/2 - 2^-22) rounded down, a margin far above those roundings.
// False more often than near_box only within that margin (the periodic path
// is then taken, which is exact too).
__device__ __forceinline__ bool near_box32(const float4* __restrict__ b, float qx, float qy, float qz, float limx,
                                           float limy, float limz) {
  const float4 c = b[0], w = b[1];
  const float ux = __fadd_ru(__fsub_ru(fmaxf(c.x, qx), fminf(c.x, qx)), w.x);
  const float uy = __fadd_ru(__fsub_ru(fmaxf(c.y, qy), fminf(c.y, qy)), w.y);
  const float uz = __fadd_ru(__fsub_ru(fmaxf(c.z, qz), fminf(c.z, qz)), w.z);
  return ux <= limx && uy <= limy && uz <= limz;
}

// Periodic squared distance between two padded boxes (centre, half width).
// Lower bound of the squared periodic distance between two widened FP32 boxes.
__device__ __forceinline__ float boxbox_dist2_lb(const float4* __restrict__ a, const float4* __restrict__ b,
                                                 float Lx, float Ly, float Lz) {
  const float4 ca = a[0], wa = a[1], cb = b[0], wb = b[1];
  float dx = fabsf(ca.x - cb.x); dx = fminf(dx, Lx - dx); dx = fmaxf(0.f, __fsub_rd(__fsub_rd(dx, wa.x), wb.x));
  float dy = fabsf(ca.y - cb.y); dy = fminf(dy, Ly - dy); dy = fmaxf(0.f, __fsub_rd(__fsub_rd(dy, wa.y), wb.y));
  float dz = fabsf(ca.z - cb.z); dz = fminf(dz, Lz - dz); dz = fmaxf(0.f, __fsub_rd(__fsub_rd(dz, wa.z), wb.z));
  return __fadd_rd(__fadd_rd(__fmul_rd(dx, dx), __fmul_rd(dy, dy)), __fmul_rd(dz, dz));
}

__device__ __forceinline__ double boxbox_dist2(const double* __restrict__ a, const double* __restrict__ b,
                                               double Lx, double Ly, double Lz) {
  double dx = fabs(a[0] - b[0]); dx = fmin(dx, Lx - dx); dx = fmax(0.0, dx - a[3] - b[3]);
  double dy = fabs(a[1] - b[1]); dy = fmin(dy, Ly - dy); dy = fmax(0.0, dy - a[4] - b[4]);
  double dz = fabs(a[2] - b[2]); dz = fmin(dz, Lz - dz); dz = fmax(0.0, dz - a[5] - b[5]);
  return dx * dx + dy * dy + dz * dz;
}

constexpr int kMaxCand = 512;        // candidate leaves per query leaf held in shared memory
constexpr int kMaxCandSpill = 4096;  // ... in the warp's global spill buffer (else per-query DFS)
// the candidate sort pads a list to the next power of two inside its buffer
static_assert((kMaxCand & (kMaxCand - 1)) == 0 && (kMaxCandSpill & (kMaxCandSpill - 1)) == 0,
              "candidate capacities must be powers of two");

// Ascending bitonic sort of the 32 * E keys at kb by one warp in registers:
// lane l holds keys [l * E, l * E + E); strides below E are exchanges inside
// a lane, larger ones shuffles with lane l ^ (stride / E).  The keys are
// distinct (slot numbers in their low bits), so the order is the same as any
// other sort's.
template <int E>
__device__ __forceinline__ void warp_sort_regs(unsigned* kb, int lane) {
  constexpr int N = 32 * E;
  unsigned v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) v[r] = kb[lane * E + r];
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= E) {
        const int lj = j / E, lk = k / E;
        const bool keep_min = ((lane & lj) == 0) == ((lane & lk) == 0);
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const unsigned p = __shfl_xor_sync(0xffffffffu, v[r], lj);
          v[r] = keep_min ? min(v[r], p) : max(v[r], p);
        }
      } else {
#pragma unroll
        for (int r = 0; r < E; ++r) {
          if ((r & j) == 0) {
            const bool asc = ((lane * E + r) & k) == 0;
            const unsigned a = v[r], b = v[r | j];
            const unsigned lo = min(a, b), hi = max(a, b);
            v[r] = asc ? lo : hi;
            v[r | j] = asc ? hi : lo;
          }
        }
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < E; ++r) kb[lane * E + r] = v[r];
  __syncwarp();
}

// One warp per query leaf (its 32 Morton-consecutive particles).
//  A. every query sorts the 64 particles of its own and the adjacent leaf
//     (the order is kept, 32 bytes per query); their nv-th distance bounds
//     its final kNN radius r_q; R = max_q r_q;
//  B. one traversal collects every leaf whose box lies within R of this
//     leaf's box, then sorts them by that box-to-box distance;
//  C. each query starts from its seed order and scans the candidates
//     nearest-first, skipping leaves farther than its current nv-th
//     distance and stopping at the first whose box-to-box distance exceeds it.
// The candidate leaves are shared by the 32 queries, so the traversal is
// paid once per leaf and the leaf data mostly comes from L1.
// kProf: the counters and cycle stamps of the profiling API (off in the
// production instances, so they cost nothing there).
template <int C, bool kProf>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4) knn_leaf_kernel(KnnArgs A) {
  __shared__ __align__(16) int32_t s_node[kWarpsPerBlock][kStack];
  __shared__ double s_bd[kWarpsPerBlock][kStack];
  __shared__ int32_t s_cand[kWarpsPerBlock][kMaxCand];
  __shared__ unsigned char s_list[kWarpsPerBlock][kLeaf][32];  // each query's seed order
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
  const int64_t nleaf = A.lev_cnt[0];
  const int top = A.nlev - 1;
  const float Lxf = (float)A.Lx, Lyf = (float)A.Ly, Lzf = (float)A.Lz;
  const float hlx = __double2float_rd(A.Lx * (0.5 - 0x1p-22)), hly = __double2float_rd(A.Ly * (0.5 - 0x1p-22)),
              hlz = __double2float_rd(A.Lz * (0.5 - 0x1p-22));
  // candidate sort keys; s_bd is only used by the per-query fallback, which
  // runs exactly when there is no candidate list
  unsigned* s_key = reinterpret_cast<unsigned*>(s_bd[wib]);
  static_assert(kStack * 2 >= kMaxCand, "sort keys must fit the fallback stack");
  for (int64_t jl = (int64_t)blockIdx.x * kWarpsPerBlock + wib; jl < nleaf; jl += nwarps) {
    const long long t_leaf = kProf ? clock64() : 0;
    const int64_t jn = (jl + 1 < nleaf) ? jl + 1 : jl - 1;  // adjacent leaf (jn >= 0 when nleaf >= 2)
    const int64_t s0 = jl * kLeaf;
    const int nq = (int)((A.n - s0) < kLeaf ? (A.n - s0) : (int64_t)kLeaf);
    // ---- A: per-query bound from the two leaves
    double Rq = 0.0;
    bool ok = true;
    unsigned wrapmask = 0u;  // bit q: query q needs the periodic fold for its two seed leaves
    for (int q = 0; q < nq; ++q) {
      const int64_t s = s0 + q;
      const double qx = A.x[s], qy = A.y[s], qz = A.z[s];
      const bool wrap = !(near_box(A.box32 + 2 * jl, qx, qy, qz, A.Lx, A.Ly, A.Lz) &&
                          near_box(A.box32 + 2 * jn, qx, qy, qz, A.Lx, A.Ly, A.Lz));
      if (wrap) wrapmask |= 1u << q;
      double kth;
      if (!seed_sort_keys<C>(A, jl, jn, s, qx, qy, qz, lane, s_list[wib][q], kth, wrap))
        kth = seed_sort<C>(A, jl, jn, s, qx, qy, qz, lane, s_list[wib][q], wrap);
      if (!(kth < CUDART_INF)) ok = false;  // fewer than nv others in the two leaves
      if (lane == q) Rq = kth;
    }
    __syncwarp();
    double R2 = ok ? Rq : CUDART_INF;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) R2 = fmax(R2, __shfl_xor_sync(0xffffffffu, R2, o));
    if (!ok) R2 = CUDART_INF;
    const long long t_a = kProf ? clock64() : 0;
    // ---- B: candidate leaves within R of this leaf's box; the list lives in
    // shared memory and moves to the warp's global spill buffer past kMaxCand
    const float4* myb32 = A.box32 + 2 * jl;
    int ncand = 0;
    unsigned* kb = s_key;
    int32_t* cb = s_cand[wib];
    int cap = kMaxCand;
    bool overflow = !(R2 < CUDART_INF);
    if (!overflow) {
      const double lim = R2 * (1.0 + 1e-12);
      int sp = 0;
      if (lane == 0) { s_node[wib][0] = (top << 27) | 0; }
      sp = 1;
      __syncwarp();
      while (sp > 0 && !overflow) {
        --sp;
        const int32_t ent = s_node[wib][sp];
        __syncwarp();
        const int lvl = ent >> 27;
        const int64_t j = ent & ((1 << 27) - 1);
        const int64_t c = j * kFan + lane;
        const bool valid = c < A.lev_cnt[lvl - 1];
        bool cand = false;
        double bbd = CUDART_INF;
        if (valid) {
          bbd = (double)boxbox_dist2_lb(myb32, A.box32 + 2 * (A.lev_off[lvl - 1] + c), Lxf, Lyf, Lzf);
          cand = bbd <= lim;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, cand);
        const int cnt = __popc(mask);
        if (!cnt) continue;
        const int r = __popc(mask & ((1u << lane) - 1));
        if (lvl - 1 == 0) {
          if (ncand + cnt > cap) {
            if (cap == kMaxCand && A.kspill) {
              unsigned* gk = A.kspill + (size_t)(blockIdx.x * kWarpsPerBlock + wib) * (2 * kMaxCandSpill);
              int32_t* gc = reinterpret_cast<int32_t*>(gk + kMaxCandSpill);
              for (int i = lane; i < ncand; i += 32) { gk[i] = kb[i]; gc[i] = cb[i]; }
              __syncwarp();
              kb = gk;
              cb = gc;
              cap = kMaxCandSpill;
            }
            if (ncand + cnt > cap) { overflow = true; break; }
          }
          if (cand) {
            // sort key: the leaf-to-leaf distance rounded down to 20 bits, then the slot
            const unsigned fb = __float_as_uint(__double2float_rd(bbd));
            kb[ncand + r] = ((fb >> 11) << 12) | (unsigned)(ncand + r);
            cb[ncand + r] = (int32_t)c;
          }
          ncand += cnt;
        } else {
          if (sp + cnt > kStack) { overflow = true; break; }
          if (cand) s_node[wib][sp + r] = ((lvl - 1) << 27) | (int32_t)c;
          sp += cnt;
        }
        __syncwarp();
      }
      __syncwarp();
    }
    if (!overflow) {
      // candidates nearest-first: warp bitonic sort of the keys, in
      // registers up to kMaxCand keys, else in the spill buffer
      int N = 32;
      while (N < ncand) N <<= 1;
      for (int i = ncand + lane; i < N; i += 32) kb[i] = 0xffffffffu;
      __syncwarp();
      switch (N) {
        case 32: warp_sort_regs<1>(kb, lane); break;
        case 64: warp_sort_regs<2>(kb, lane); break;
        case 128: warp_sort_regs<4>(kb, lane); break;
        case 256: warp_sort_regs<8>(kb, lane); break;
        case 512: warp_sort_regs<16>(kb, lane); break;
        default: break;
      }
      for (int k = 2; k <= (N > kMaxCand ? N : 1); k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int t = lane; t < (N >> 1); t += 32) {
            const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
            const unsigned a = kb[i], b = kb[i + j];
            if ((a > b) == ((i & k) == 0)) { kb[i] = b; kb[i + j] = a; }
          }
          __syncwarp();
        }
      }
    }
    const long long t_b = kProf ? clock64() : 0;
    long long c_init = 0, c_scan = 0, c_fin = 0;
    // ---- C: per-query kNN over the candidates
    unsigned nvis = 0, nins = 0, nideal = 0, nchunk = 0, nbits = 0;
    unsigned visbits = 0;  // profiling: lane l holds candidates [32 l, 32 l + 32) visited by any query
    int32_t prev_ls = -1;  // lane's entry of the previous query's final list
    for (int q = 0; q < nq; ++q) {
      const int64_t s = s0 + q;
      const double qx = A.x[s], qy = A.y[s], qz = A.z[s];
      const float qxf = (float)qx, qyf = (float)qy, qzf = (float)qz;
      WarpList L;
      const long long tq0 = kProf ? clock64() : 0;
      // A bound for this query from its predecessor in the leaf (a close
      // particle): the previous query's nv neighbours, with this query
      // replaced by the previous query itself, are nv distinct other
      // particles, so the largest of their exact distances from this query
      // bounds its nv-th distance.  It tightens the acceptance bound from the
      // start (fewer visits and fewer insertions that later drop out).
      L.cap = CUDART_INF;
      if (q > 0) {
        const int nvv = C ? C : A.nv;
        int32_t ps = prev_ls;
        if (ps == (int32_t)s) ps = (int32_t)s - 1;
        // Only an upper bound is needed: the distance without the periodic fold
        // is at least the folded one (equal bits within half a period), and
        // the warp maximum is taken over the high words rounded up (one
        // reduction; non-negative doubles order like their bits).
        unsigned hk = 0u;
        if (lane < nvv)
          hk = ps >= 0 ? (unsigned)(__double_as_longlong(dist2_near(qx, qy, qz, A.x[ps], A.y[ps], A.z[ps])) >> 32) + 1u
                       : 0x7FF00000u;  // +inf
        hk = __reduce_max_sync(0xffffffffu, hk);
        L.cap = __longlong_as_double((long long)((unsigned long long)hk << 32));
      }
      const bool swrap = (wrapmask >> q) & 1u;
      seed_list<C>(A, L, jl, jn, s, qx, qy, qz, lane, s_list[wib][q], nvis, swrap);
      const long long tq1 = kProf ? clock64() : 0;
      if (overflow) {
        query_dfs<C>(A, L, s, qx, qy, qz, lane, s_node[wib], s_bd[wib], jl, jn, nvis, nins);
      } else {
        for (int c0 = 0; c0 < ncand; c0 += 32) {
          // every query lies in this leaf's box, so a candidate whose box is at
          // least the current radius from that box (and all after it) is out
          const double lb = (double)__uint_as_float((kb[c0] >> 12) << 11);
          if (lb * (1.0 - 1e-9) >= L.r2) break;
          if (kProf) ++nchunk;
          const int ci = c0 + lane;
          // candidate leaf with bit 30 set when its particles need the periodic
          // fold (leaf ids are below 2^26)
          int32_t leafw = -1;
          float bd = CUDART_INF_F;
          if (ci < ncand) {
            const int32_t leaf = cb[kb[ci] & 4095u];
            leafw = leaf;
            if (leaf != jl && leaf != jn) {
              bd = box_dist2_lb(A.box32 + 2 * (int64_t)leaf, qxf, qyf, qzf, Lxf, Lyf, Lzf);
              if (!near_box32(A.box32 + 2 * (int64_t)leaf, qxf, qyf, qzf, hlx, hly, hlz)) leafw |= 1 << 30;
            }
          }
          // visit test in FP32 against the bound rounded up: a superset of the
          // leaves whose lower bound is below the bound, so nothing is lost.
          // The chunk's leaves are visited nearest-first by that lower bound
          // (its bits with the lane in the 5 lowest: non-negative floats order
          // like their bits, and clearing bits rounds the bound down), so the
          // list tightens sooner and the visits stop at the first leaf at or
          // beyond the bound.
          float r2f = __double2float_ru(L.r2);
          unsigned key = (bd < r2f) ? ((__float_as_uint(bd) & ~31u) | (unsigned)lane) : 0xffffffffu;
          for (;;) {
            const unsigned m = __reduce_min_sync(0xffffffffu, key);
            if (!(__uint_as_float(m & ~31u) < r2f)) break;  // none left, or all at or beyond the bound
            const int src = (int)(m & 31u);
            if (lane == src) key = 0xffffffffu;
            if (kProf) ++nbits;
            const int32_t slw = __shfl_sync(0xffffffffu, leafw, src);
            if (kProf && lane == ((c0 + src) >> 5)) visbits |= 1u << ((c0 + src) & 31);
            leaf_insert<C>(A, L, slw & ~(1 << 30), s, qx, qy, qz, lane, nvis, nins, (slw >> 30) & 1);
            r2f = __double2float_ru(L.r2);
          }
        }
      }
      const long long tq2 = kProf ? clock64() : 0;
      c_init += tq1 - tq0;
      c_scan += tq2 - tq1;
      if (kProf && !overflow) {
        // leaves that any search with these boxes must visit: box within the final radius
        for (int c0 = 0; c0 < ncand; c0 += 32) {
          const int ci = c0 + lane;
          bool in = false;
          if (ci < ncand) in = box_dist2(A.box + 6 * (int64_t)cb[ci], qx, qy, qz, A.Lx, A.Ly, A.Lz) < L.r2;
          nideal += __popc(__ballot_sync(0xffffffffu, in));
        }
      }
      const long long tq3 = kProf ? clock64() : 0;
      prev_ls = L.ls;
      // the traversal stack is free once the query's search is done
      finish_query<C>(A, L, s, lane, reinterpret_cast<double*>(s_node[wib]));
      __syncwarp();
      if (kProf) c_fin += clock64() - tq3;
    }
    if (kProf && lane == 0) {
      unsigned long long* ph = A.kstats + 24;  // phase cycles of non-overflow leaves
      if (!overflow) {
        atomicAdd(&ph[0], (unsigned long long)(t_a - t_leaf));
        atomicAdd(&ph[1], (unsigned long long)(t_b - t_a));
        atomicAdd(&ph[2], (unsigned long long)c_init);
        atomicAdd(&ph[3], (unsigned long long)c_scan);
        atomicAdd(&ph[4], (unsigned long long)c_fin);
      }
      atomicAdd(&A.kstats[5], (unsigned long long)nideal);
      atomicAdd(&A.kstats[overflow ? 6 : 7], (unsigned long long)(clock64() - t_leaf));
    }
    if (kProf) {
      unsigned u = (!overflow && cap == kMaxCand) ? __popc(visbits) : 0u;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
      if (lane == 0) {
        atomicAdd(&A.kstats[8], (unsigned long long)nchunk);
        atomicAdd(&A.kstats[9], (unsigned long long)nbits);
        atomicAdd(&A.kstats[10], (unsigned long long)u);
        if (!overflow && cap == kMaxCand) atomicAdd(&A.kstats[11], 1ULL);
      }
    }
    if (kProf && lane == 0) {
      atomicAdd(&A.kstats[0], 1ULL);
      atomicAdd(&A.kstats[1], (unsigned long long)ncand);
      atomicAdd(&A.kstats[2], (unsigned long long)nvis);
      atomicAdd(&A.kstats[3], (unsigned long long)nins);
      if (overflow) atomicAdd(&A.kstats[4], 1ULL);
    }
  }
}

int stage_knn_density(Engine& E) {
  const int64_t n = E.n;
  const Params& P = E.prm;
  E.nstore = E.req_store > 0 ? E.req_store : P.nhop;
  if (E.nstore < P.nhop) E.nstore = P.nhop;
  if (E.nstore > P.nvoisins) E.nstore = P.nvoisins;
  AHOP_CUDA_TRY(E.d_nei.ensure((size_t)n * E.nstore * 4));
  AHOP_CUDA_TRY(E.d_dens.ensure(n * 8));
  KnnArgs A;
  A.x = E.d_x.as<double>(); A.y = E.d_y.as<double>(); A.z = E.d_z.as<double>(); A.m = E.d_m.as<double>();
  A.orig = E.d_orig.as<int32_t>();
  A.box = E.d_box.as<double>();
  const int64_t nbox = E.lev_off[E.nlev];  // boxes of every level
  AHOP_CUDA_TRY(E.d_box32.ensure((size_t)nbox * 32 + 32));
  A.box32 = E.d_box32.as<float4>();
  E.launches++;
  leaf_box32_kernel<<<(unsigned)((nbox + 255) / 256), 256, 0, E.stream>>>(
      A.box, nbox, std::max(P.xlong, std::max(P.ylong, P.zlong)), E.d_box32.as<float4>());
  AHOP_CUDA_TRY(cudaGetLastError());
  for (int l = 0; l < kMaxLevels; ++l) { A.lev_off[l] = E.lev_off[l]; A.lev_cnt[l] = E.lev_cnt[l]; }
  A.nlev = E.nlev;
  A.n = n;
  A.n32 = (int32_t)n;
  A.Lx = P.xlong; A.Ly = P.ylong; A.Lz = P.zlong; A.xyzlong = P.xyzlong;
  A.nv = P.nvoisins;
  A.nstore = E.nstore;
  A.nei = E.d_nei.as<int32_t>();
  A.dens = E.d_dens.as<double>();
  AHOP_CUDA_TRY(E.d_flags.ensure(512));
  AHOP_CUDA_TRY(cudaMemsetAsync(E.d_flags.p, 0, 512, E.stream));
  A.err = E.d_flags.as<int>();
  A.kstats = reinterpret_cast<unsigned long long*>(E.d_flags.as<char>() + 64);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, E.device);
  // the default nvoisins = 32 (one list entry per lane) has its own build with
  // the count fixed at compile time
  const bool nv32 = P.nvoisins == 32;
  int per_sm = 0;
  const bool prof = E.task_profile;
  const void* kfn = nv32 ? (prof ? (const void*)knn_leaf_kernel<32, true> : (const void*)knn_leaf_kernel<32, false>)
                         : (prof ? (const void*)knn_leaf_kernel<0, true> : (const void*)knn_leaf_kernel<0, false>);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  int64_t want = (E.lev_cnt[0] + kWarpsPerBlock - 1) / kWarpsPerBlock;
  int64_t grid = (int64_t)nsm * per_sm * 2;
  if (grid > want) grid = want;
  AHOP_CUDA_TRY(E.d_kspill.ensure((size_t)grid * kWarpsPerBlock * 2 * kMaxCandSpill * 4));
  A.kspill = E.d_kspill.as<unsigned>();
  E.launches++;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[9], E.stream));
  if (nv32 && prof) knn_leaf_kernel<32, true><<<(unsigned)grid, kWarpsPerBlock * 32, 0, E.stream>>>(A);
  else if (nv32) knn_leaf_kernel<32, false><<<(unsigned)grid, kWarpsPerBlock * 32, 0, E.stream>>>(A);
  else if (prof) knn_leaf_kernel<0, true><<<(unsigned)grid, kWarpsPerBlock * 32, 0, E.stream>>>(A);
  else knn_leaf_kernel<0, false><<<(unsigned)grid, kWarpsPerBlock * 32, 0, E.stream>>>(A);
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[10], E.stream));
  AHOP_CUDA_TRY(cudaGetLastError());
  int herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, E.d_flags.p, 4, cudaMemcpyDeviceToHost, E.stream));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.knn_stats, E.d_flags.as<char>() + 64, 12 * 8, cudaMemcpyDeviceToHost, E.stream));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.knn_phase, E.d_flags.as<char>() + 64 + 24 * 8, 5 * 8, cudaMemcpyDeviceToHost,
                                E.stream));
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  if (herr) { set_error("kNN traversal stack overflow"); return AHOP_ELIMIT; }
  return AHOP_OK;
}

}  // namespace ahop
