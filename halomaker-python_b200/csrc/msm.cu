// Halo/subhalo selection by the Most-massive Sub Method and member grouping;
// replaces select_with_MS_method_1319 (src/compute_neiKDtree_mod.py:260-464)
// and the argsort/unique grouping of compute_adaptahop_131 (NEI:107-119).
//
// Runs on the finder's device outputs (renumbered node tables, membership):
//  1. own mass: each node minus its children, subtracted along the sister
//     chain from firstchild (NEI:266-281), from the unmodified values;
//  2. most massive sub, bottom-up one level at a time: strict '>' on truemass
//     along the sister chain, first wins (NEI:296-316); the node then adds the
//     chosen child's accumulated mass and truemass.  Nodes are numbered by
//     level (node_precedes), so each level is a contiguous index range;
//  3. structure ids: halos (mother <= 0) and non-most-massive children start
//     a structure, numbered in node order; every node points to its mother if
//     it is the most massive child, and pointer jumping resolves the chains
//     (NEI:318-343);
//  4. membership rewritten to structure ids (NEI:380-383);
//  5. the structure tree: halos chained in order, daughters of a structure in
//     order of their starting node, level = mother's level + 1 (NEI:399-425);
//  6. members grouped by structure id (stable radix sort; the reference's
//     np.argsort is not stable, so only the per-structure member sets are
//     specified) with run-length offsets and counts.
#include <cub/cub.cuh>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

struct MsmArgs {
  int32_t nn;
  const double* rt;   // [nn][8]
  const int32_t* it;  // [nn][6]
  int32_t* m1; double* t1;   // own mass (1-based)
  int32_t* m2; double* t2;   // accumulated
  int32_t* most;             // most massive child, -1 if none
  int32_t* lvstart;          // first node of each level (1-based levels)
  int32_t* flag;             // starters
  int32_t* sid;              // structure id of starters (scan)
  int32_t* par;              // pointer-jumping parents
  int32_t* n2s;              // node -> structure
  int32_t* err;
};

#define IT(i, f) A.it[6 * (size_t)((i) - 1) + (f)]
#define RT(i, f) A.rt[8 * (size_t)((i) - 1) + (f)]

__global__ void msm_own_kernel(MsmArgs A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > A.nn) return;
  int32_t m = IT(i, 0);
  double t = RT(i, 4);
  int32_t c = IT(i, 3);
  const bool has = c > 0;
  int guard = 0;
  while (c > 0 && guard++ < A.nn) {
    m -= IT(c, 0);
    t -= RT(c, 4);
    c = IT(c, 5);
  }
  if (has && (m <= 0 || !(t > 0.0))) atomicCAS(A.err, 0, i);  // NEI:282-284
  A.m1[i] = m; A.t1[i] = t;
  A.m2[i] = m; A.t2[i] = t;
  A.most[i] = -1;
  const int32_t L = IT(i, 1);
  if (i == 1 || IT(i - 1, 1) != L) A.lvstart[L] = i;
}

__global__ void msm_most_kernel(MsmArgs A, int32_t i0, int32_t i1) {
  const int32_t i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i1) return;
  int32_t c = IT(i, 3);
  if (c <= 0) return;
  int32_t best = c;
  double mx = A.t2[c];
  c = IT(c, 5);
  int guard = 0;
  while (c > 0 && guard++ < A.nn) {
    if (A.t2[c] > mx) { best = c; mx = A.t2[c]; }
    c = IT(c, 5);
  }
  A.most[i] = best;
  A.m2[i] = A.m1[i] + A.m2[best];
  A.t2[i] = xadd(A.t1[i], A.t2[best]);
}

__global__ void msm_starter_kernel(MsmArgs A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > A.nn + 1) return;
  if (i == A.nn + 1) { A.flag[i - 1] = 0; return; }
  const int32_t mo = IT(i, 2);
  const bool halo = mo <= 0;
  const bool mostc = !halo && A.most[mo] == i;
  A.flag[i - 1] = (halo || !mostc) ? 1 : 0;
  A.par[i] = mostc ? mo : i;
}

__global__ void msm_jump_kernel(MsmArgs A, int* changed) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > A.nn) return;
  const int32_t p = A.par[i], pp = A.par[p];
  if (pp != p) { A.par[i] = pp; *changed = 1; }
}

__global__ void msm_n2s_kernel(MsmArgs A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > A.nn) return;
  A.n2s[i] = A.sid[A.par[i] - 1] + 1;  // inclusive id of the chain's starter
}

__global__ void msm_members_kernel(const int32_t* __restrict__ liste, int64_t n, const int32_t* __restrict__ n2s,
                                   int32_t* __restrict__ wp, uint32_t* __restrict__ key, int32_t* __restrict__ val) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t v = liste[p];
  const int32_t s = v > 0 ? n2s[v] : 0;
  wp[p] = s;
  key[p] = (uint32_t)s;
  val[p] = (int32_t)p;
}

// per structure: mother structure; struct level filled level by level
__global__ void msm_struct_kernel(MsmArgs A, int32_t i0, int32_t i1, int32_t* mother_s, int32_t* level_s,
                                  uint32_t* skey, int32_t* sval) {
  const int32_t i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i1 || !A.flag[i - 1]) return;
  const int32_t k = A.sid[i - 1] + 1;
  const int32_t mo = IT(i, 2);
  int32_t ms = 0, lv = 1;
  if (mo > 0) {
    ms = A.n2s[mo];
    lv = level_s[ms - 1] + 1;
  }
  mother_s[k - 1] = ms;
  level_s[k - 1] = lv;
  skey[k - 1] = (uint32_t)ms;
  sval[k - 1] = k;
}

__global__ void msm_links_kernel(int32_t ns, const uint32_t* __restrict__ key, const int32_t* __restrict__ val,
                                 int32_t* first_sister, int32_t* first_daughter) {
  const int32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ns) return;
  if (p + 1 < ns && key[p + 1] == key[p]) first_sister[val[p] - 1] = val[p + 1];
  if ((p == 0 || key[p - 1] != key[p]) && key[p] > 0) first_daughter[key[p] - 1] = val[p];
}

__global__ void fill_kernel(int32_t* a, int64_t n, int32_t v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

}  // namespace ahop

using namespace ahop;

namespace {
struct MsmState {
  DevBuf d_scr, d_wp, d_key, d_key2, d_val, d_val2, d_struct, d_runs;
  HostBuf h_wp, h_struct, h_sorted, h_runs;
  AhopStructs out{};
  bool have = false;       // a selection is held (device grouping below)
  int32_t nruns = 0;       // runs of the sorted structure ids (id 0 first when present)
  int32_t skip = 0;        // runs of id 0 (unassigned particles): 0 or 1
  int64_t nmembers = 0;    // particles in structures (id >= 1)
  int64_t n = 0;
  int32_t ns = 0;          // structures of the selection (sizes the run arrays)
  bool particle_views = true;  // copy whereIam_parts / pids_groupsorted to the host
};

// Gather of the members of every structure (id >= 1) into structure order:
// member k of the grouping is particle src = sorted[first + k]; per-structure
// offsets from the run offsets.
__global__ void gather_members_kernel(const int32_t* __restrict__ sorted, int64_t first, int64_t nmem,
                                      const double* __restrict__ pos, const double* __restrict__ vel,
                                      const double* __restrict__ mass, const double* __restrict__ dens,
                                      double* __restrict__ gpos, double* __restrict__ gvel,
                                      double* __restrict__ gmass, double* __restrict__ gdens) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nmem) return;
  const int64_t i = sorted[first + k];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    gpos[3 * k + c] = pos[3 * i + c];
    if (gvel) gvel[3 * k + c] = vel[3 * i + c];
  }
  gmass[k] = mass[i];
  if (gdens) gdens[k] = dens[i];
}

__global__ void member_offsets_kernel(const int32_t* __restrict__ idxs, int32_t skip, int32_t nr1, int64_t n,
                                      int64_t* __restrict__ off, int32_t* __restrict__ ids,
                                      const uint32_t* __restrict__ uids) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > nr1) return;
  const int64_t base = idxs[skip];
  off[r] = (r < nr1 ? (int64_t)idxs[skip + r] : n) - base;
  if (r < nr1 && ids) ids[r] = (int32_t)uids[skip + r];
}
MsmState& msm_state() {
  static MsmState* s = new MsmState();
  return *s;
}
}  // namespace

extern "C" int ahop_select_msm(AhopStructs* out) {
  Engine& E = engine();
  if (!out) { set_error("null out"); return AHOP_EINVAL; }
  if (!E.have_result) { set_error("no finder result (call compute first)"); return AHOP_ESTATE; }
  MsmState& S = msm_state();
  cudaStream_t st = E.stream;
  const int32_t nn = E.nnodes;
  const int64_t n = E.prm.nusedpart > 0 ? std::min<int64_t>(E.prm.nusedpart, E.n) : E.n;
  const int T = 256;
  // scratch: 10 int/double arrays of nn+2
  const size_t G = (size_t)nn + 2;
  AHOP_CUDA_TRY(S.d_scr.ensure(G * (4 * 9 + 8 * 2) + 64 * 4 + 4096));
  char* p = static_cast<char*>(S.d_scr.p);
  auto take = [&](size_t b) { char* q = p; p += (b + 255) & ~size_t(255); return q; };
  MsmArgs A;
  A.nn = nn;
  A.rt = E.d_rtab.as<double>();
  A.it = E.d_itab.as<int32_t>();
  A.m1 = reinterpret_cast<int32_t*>(take(G * 4));
  A.m2 = reinterpret_cast<int32_t*>(take(G * 4));
  A.t1 = reinterpret_cast<double*>(take(G * 8));
  A.t2 = reinterpret_cast<double*>(take(G * 8));
  A.most = reinterpret_cast<int32_t*>(take(G * 4));
  A.lvstart = reinterpret_cast<int32_t*>(take(64 * 4));
  A.flag = reinterpret_cast<int32_t*>(take(G * 4));
  A.sid = reinterpret_cast<int32_t*>(take(G * 4));
  A.par = reinterpret_cast<int32_t*>(take(G * 4));
  A.n2s = reinterpret_cast<int32_t*>(take(G * 4));
  A.err = reinterpret_cast<int32_t*>(take(16));
  int32_t* h = reinterpret_cast<int32_t*>(E.h_scalars);
  int32_t ns = 0, nhalo = 0;
  AHOP_CUDA_TRY(S.d_wp.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.d_key.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.d_key2.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.d_val.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.d_val2.ensure(n * 4 + 4));
  std::vector<int32_t> lv(64, 0);
  int maxlev = 0;
  if (nn > 0) {
    AHOP_CUDA_TRY(cudaMemsetAsync(A.err, 0, 16, st));
    AHOP_CUDA_TRY(cudaMemsetAsync(A.lvstart, 0, 64 * 4, st));
    msm_own_kernel<<<(nn + T - 1) / T, T, 0, st>>>(A);
    AHOP_CUDA_TRY(cudaGetLastError());
    AHOP_CUDA_TRY(cudaMemcpyAsync(lv.data(), A.lvstart, 64 * 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h, A.err, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[0] != 0) { set_error("MSM: node " + std::to_string(h[0]) + " has non-positive own mass"); return AHOP_EINVARIANT; }
    for (int L = 1; L < 63; ++L) if (lv[L] > 0) maxlev = L;
    if (maxlev >= 62) { set_error("MSM: too many levels"); return AHOP_EINVAL; }
    auto lv_end = [&](int L) { return (L + 1 <= maxlev && lv[L + 1] > 0) ? lv[L + 1] : nn + 1; };
    for (int L = maxlev; L >= 1; --L) {
      if (lv[L] <= 0) continue;
      const int32_t i0 = lv[L], i1 = lv_end(L);
      msm_most_kernel<<<(i1 - i0 + T - 1) / T, T, 0, st>>>(A, i0, i1);
    }
    AHOP_CUDA_TRY(cudaGetLastError());
    msm_starter_kernel<<<(nn + 1 + T - 1) / T, T, 0, st>>>(A);
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, A.flag, A.sid, nn + 1, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, A.flag, A.sid, nn + 1, st));
    int* changed = A.err + 1;
    bool conv = false;
    for (int it = 0; it < 64; ++it) {
      AHOP_CUDA_TRY(cudaMemsetAsync(changed, 0, 4, st));
      msm_jump_kernel<<<(nn + T - 1) / T, T, 0, st>>>(A, changed);
      AHOP_CUDA_TRY(cudaMemcpyAsync(h, changed, 4, cudaMemcpyDeviceToHost, st));
      AHOP_CUDA_TRY(cudaStreamSynchronize(st));
      if (h[0] == 0) { conv = true; break; }
    }
    if (!conv) { set_error("MSM pointer jumping did not converge"); return AHOP_ELIMIT; }
    msm_n2s_kernel<<<(nn + T - 1) / T, T, 0, st>>>(A);
    AHOP_CUDA_TRY(cudaGetLastError());
    AHOP_CUDA_TRY(cudaMemcpyAsync(h, A.sid + nn, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    ns = h[0];
    // the level-1 nodes are the halos
    nhalo = (lv[1] > 0) ? (lv_end(1) - lv[1]) : 0;
  }
  // structure arrays: mother, first_sister, first_daughter, level (+ sort keys)
  const size_t S4 = (size_t)(ns > 0 ? ns : 1) * 4;
  AHOP_CUDA_TRY(S.d_struct.ensure(S4 * 8));
  int32_t* mother_s = S.d_struct.as<int32_t>();
  int32_t* fsis = mother_s + (ns > 0 ? ns : 1);
  int32_t* fdau = fsis + (ns > 0 ? ns : 1);
  int32_t* lvl_s = fdau + (ns > 0 ? ns : 1);
  uint32_t* skey = reinterpret_cast<uint32_t*>(lvl_s + (ns > 0 ? ns : 1));
  uint32_t* skey2 = skey + (ns > 0 ? ns : 1);
  int32_t* sval = reinterpret_cast<int32_t*>(skey2 + (ns > 0 ? ns : 1));
  int32_t* sval2 = sval + (ns > 0 ? ns : 1);
  if (ns > 0) {
    fill_kernel<<<(ns + T - 1) / T, T, 0, st>>>(fsis, ns, -1);
    fill_kernel<<<(ns + T - 1) / T, T, 0, st>>>(fdau, ns, -1);
    auto lv_end = [&](int L) { return (L + 1 <= maxlev && lv[L + 1] > 0) ? lv[L + 1] : nn + 1; };
    for (int L = 1; L <= maxlev; ++L) {
      if (lv[L] <= 0) continue;
      const int32_t i0 = lv[L], i1 = lv_end(L);
      msm_struct_kernel<<<(i1 - i0 + T - 1) / T, T, 0, st>>>(A, i0, i1, mother_s, lvl_s, skey, sval);
    }
    AHOP_CUDA_TRY(cudaGetLastError());
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, skey, skey2, sval, sval2, ns, 0, 32, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, skey, skey2, sval, sval2, ns, 0, 32, st));
    msm_links_kernel<<<(ns + T - 1) / T, T, 0, st>>>(ns, skey2, sval2, fsis, fdau);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  // membership and grouping
  msm_members_kernel<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(E.d_liste.as<int32_t>(), n, A.n2s,
                                                                S.d_wp.as<int32_t>(), S.d_key.as<uint32_t>(),
                                                                S.d_val.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  {
    int kb = 1;
    while ((1LL << kb) <= (int64_t)ns) ++kb;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, S.d_key.as<uint32_t>(), S.d_key2.as<uint32_t>(),
                                    S.d_val.as<int32_t>(), S.d_val2.as<int32_t>(), (int)n, 0, kb, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, S.d_key.as<uint32_t>(), S.d_key2.as<uint32_t>(),
                                                  S.d_val.as<int32_t>(), S.d_val2.as<int32_t>(), (int)n, 0, kb,
                                                  st));
  }
  // run-length encode the sorted structure ids: unique ids, counts, offsets
  AHOP_CUDA_TRY(S.d_runs.ensure((size_t)(ns + 2) * 4 * 3 + 16));
  uint32_t* uids = S.d_runs.as<uint32_t>();
  int32_t* cnts = reinterpret_cast<int32_t*>(uids + ns + 2);
  int32_t* idxs = cnts + ns + 2;
  int32_t* nruns = idxs + ns + 2;
  {
    size_t tmp = 0;
    cub::DeviceRunLengthEncode::Encode(nullptr, tmp, S.d_key2.as<uint32_t>(), uids, cnts, nruns, (int)n, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    AHOP_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(E.d_cub.p, tmp, S.d_key2.as<uint32_t>(), uids, cnts, nruns,
                                                     (int)n, st));
  }
  AHOP_CUDA_TRY(cudaMemcpyAsync(h, nruns, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  const int32_t nr = h[0];
  {
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnts, idxs, nr, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, tmp, cnts, idxs, nr, st));
  }
  // first run of a structure (id 0 = unassigned particles sorts first)
  {
    uint32_t first_id = 1;
    if (nr > 0) AHOP_CUDA_TRY(cudaMemcpyAsync(&first_id, uids, 4, cudaMemcpyDeviceToHost, st));
    int32_t first_idx = 0;
    if (nr > 1) AHOP_CUDA_TRY(cudaMemcpyAsync(&first_idx, idxs + 1, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    S.nruns = nr;
    S.skip = (nr > 0 && first_id == 0) ? 1 : 0;
    S.nmembers = S.skip ? (nr > 1 ? n - first_idx : 0) : n;
    S.n = n;
    S.ns = ns;
  }
  // host copies
  AHOP_CUDA_TRY(S.h_wp.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.h_sorted.ensure(n * 4 + 4));
  AHOP_CUDA_TRY(S.h_struct.ensure(S4 * 4));
  AHOP_CUDA_TRY(S.h_runs.ensure((size_t)(nr + 1) * 4 * 3));
  if (S.particle_views) {
    AHOP_CUDA_TRY(cudaMemcpyAsync(S.h_wp.p, S.d_wp.p, n * 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(S.h_sorted.p, S.d_val2.p, n * 4, cudaMemcpyDeviceToHost, st));
  }
  if (ns > 0) AHOP_CUDA_TRY(cudaMemcpyAsync(S.h_struct.p, mother_s, S4 * 4, cudaMemcpyDeviceToHost, st));
  int32_t* hr = S.h_runs.as<int32_t>();
  AHOP_CUDA_TRY(cudaMemcpyAsync(hr, uids, (size_t)nr * 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(hr + nr, idxs, (size_t)nr * 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(hr + 2 * nr, cnts, (size_t)nr * 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  const int32_t* hs = S.h_struct.as<int32_t>();
  const size_t sw = (size_t)(ns > 0 ? ns : 1);
  out->nstruct = ns;
  out->nb_of_halos = nhalo;
  out->nb_of_subhalos = ns - nhalo;
  out->nusedpart = n;
  out->whereIam_parts = S.particle_views ? S.h_wp.as<int32_t>() : nullptr;
  out->mother = hs;
  out->first_sister = hs + sw;
  out->first_daughter = hs + 2 * sw;
  out->level = hs + 3 * sw;
  out->pids_groupsorted = S.particle_views ? S.h_sorted.as<int32_t>() : nullptr;
  out->ngroupruns = nr;
  out->run_ids = hr;
  out->run_idxs = hr + nr;
  out->run_counts = hr + 2 * nr;
  S.have = true;
  return AHOP_OK;
}

extern "C" int ahop_msm_set_particle_views(int32_t on) {
  msm_state().particle_views = on != 0;
  return AHOP_OK;
}

extern "C" int ahop_structure_members(int32_t* nstructs, int64_t* nmembers) {
  MsmState& S = msm_state();
  if (!nstructs || !nmembers) { set_error("null out"); return AHOP_EINVAL; }
  if (!S.have) { set_error("no selection (call ahop_select_msm first)"); return AHOP_ESTATE; }
  *nstructs = S.nruns - S.skip;
  *nmembers = S.nmembers;
  return AHOP_OK;
}

extern "C" int ahop_gather_member_index_device(int32_t* d_index, void* stream) {
  Engine& E = engine();
  MsmState& S = msm_state();
  if (!S.have || !E.have_result) { set_error("no selection (call ahop_select_msm first)"); return AHOP_ESTATE; }
  if (!d_index && S.nmembers > 0) { set_error("null device buffer"); return AHOP_EINVAL; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  if (S.nmembers > 0)
    AHOP_CUDA_TRY(cudaMemcpyAsync(d_index, S.d_val2.as<int32_t>() + (S.n - S.nmembers),
                                  (size_t)S.nmembers * 4, cudaMemcpyDeviceToDevice, st));
  return AHOP_OK;
}

extern "C" int ahop_gather_members_device(const double* d_pos, const double* d_vel, const double* d_mass,
                                          int64_t* d_off, int32_t* d_ids, double* d_gpos, double* d_gvel,
                                          double* d_gmass, double* d_gdens, void* stream) {
  Engine& E = engine();
  MsmState& S = msm_state();
  if (!S.have || !E.have_result) { set_error("no selection (call ahop_select_msm first)"); return AHOP_ESTATE; }
  if (!d_pos || !d_mass || !d_off || !d_gpos || !d_gmass) { set_error("null device buffer"); return AHOP_EINVAL; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the selection's arrays were written on the engine stream
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  const int32_t nr1 = S.nruns - S.skip;
  const int T = 256;
  uint32_t* uids = S.d_runs.as<uint32_t>();
  const int32_t ns2 = S.ns + 2;  // run arrays: uids, counts, offsets, each ns + 2 long
  const int32_t* idxs = reinterpret_cast<const int32_t*>(uids + ns2) + ns2;
  if (nr1 > 0) {
    member_offsets_kernel<<<(nr1 + 1 + T - 1) / T, T, 0, st>>>(idxs, S.skip, nr1, S.n, d_off, d_ids, uids);
    AHOP_CUDA_TRY(cudaGetLastError());
  } else {
    AHOP_CUDA_TRY(cudaMemsetAsync(d_off, 0, 8, st));
  }
  if (S.nmembers > 0) {
    const int64_t first = S.n - S.nmembers;
    gather_members_kernel<<<(unsigned)((S.nmembers + T - 1) / T), T, 0, st>>>(
        S.d_val2.as<int32_t>(), first, S.nmembers, d_pos, d_vel, d_mass, E.d_dens_orig.as<double>(), d_gpos,
        (d_vel && d_gvel) ? d_gvel : nullptr, d_gmass, d_gdens);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  return AHOP_OK;
}
