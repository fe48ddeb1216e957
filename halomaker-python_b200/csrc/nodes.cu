// Structure tree of hop groups ("create nodes"); replaces create_group_tree,
// omp_dev_create_nodes_task, dev_do_colorize_local, treat_particles and
// reorder_nodes_deterministic (f90:885-1131, 1188-1628, 2317-2429).
//
// Execution model.  A task is (node, threshold rhot, contiguous range of the
// group list GL).  Tasks run one CUDA block each, in waves: a block runs the
// Fortran task loop for its task -- percolate the groups above rhot through
// saddles > rhot, measure every component, test significance -- until the
// task branches (nsisters > 1: child nodes are created and their tasks queued
// for the next wave) or ends.  The nsisters == 1 chain, which the reference
// runs serially level after level, stays inside the block.
//
// Order.  GL keeps the reference's igr order (f90:1337-1367): components are
// contiguous, ordered by their smallest position before the level, and keep
// their previous relative order inside.  Components are found with a
// block-level union-find over saddle edges > rhot linking to the smaller
// position, then reordered by a chunked stable radix sort on the root.  The
// structure can only change when rhot crosses a saddle value or a group peak
// density of the task, so this pass is skipped at levels below the next such
// value.
//
// Sums.  The significance tests (f90:1459-1463) need, per component, the
// number of member particles above rhot (exact integer), the maximum group
// peak density (exact) and density/position sums that the reference
// accumulates sequentially.  Per level they are taken from running sums over
// each group's members sorted by decreasing density (an O(log n) lookup per
// group instead of the reference's rescan of every member) and carry a
// rigorous rounding bound; a test whose outcome lies within that bound, and
// every node that is actually created, is recomputed in the reference's exact
// order: members in decreasing particle index, groups in GL order, posref and
// periodic unwrapping as in treat_particles (f90:2337-2386).  Node outputs
// are therefore the reference's sums bit for bit.
//
// Membership.  A child task paints the members of its groups that lie above
// its creation threshold (f90:1297-1306); later (deeper) paints win.  The
// final node of a particle is therefore the deepest node containing its group
// whose rho_saddle is below the particle density; it is computed per particle
// after the waves.
#include <cooperative_groups.h>
#include <cub/cub.cuh>
#include <cfloat>
#include <climits>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

constexpr int kNT = 256;        // threads per task block (grid-wide root kernels, small tasks)
constexpr int kNTBig = 1024;    // threads per block for tasks of more than Engine::big_task groups
constexpr int kTermWarps = 8;   // warps that sum large groups in an exact pass
constexpr int kSmallComp = 4;   // components of at most this many groups are decided by one thread
constexpr int kIPT = 4;         // items per thread in the reorder sort (2 for 1024-thread blocks)
__host__ __device__ constexpr int ipt_for(int nt) { return nt >= 1024 ? 2 : kIPT; }
// most groups whose union-find parents a task block keeps in shared memory
// (a 1024-thread launch sizes its array to its largest task, up to this)
__host__ __device__ constexpr int par_cap(int nt) { return nt >= 1024 ? 32768 : 1024; }
constexpr int kBigGroup = 96;   // groups larger than this are summed by a warp
constexpr int kRowWarp = 8;     // saddle-row prefixes longer than this are linked by a warp
constexpr int kMaxBigRows = 512;
constexpr long long kMaxTaskLevels = 4000000LL;  // cap on one task's threshold levels (error, never a hang)
// A wide task runs on a thread-block cluster of this many CTAs: the leader
// runs the task, the followers take slices of its position-parallel phases.
constexpr int kClusterCtas = 4;
constexpr int32_t kPhUnion = 1, kPhFind = 2, kPhTerms = 3, kPhExit = 4, kPhDecide = 5, kPhReorder = 6;
constexpr int32_t kClusterReorderChunks = 8;  // reorders of at least this many chunks use the cluster
constexpr int kProfPhases = 16;  // phase cycle counters per task (structural 0..7, 12; statistics 8..11)

struct Task {
  double rhot;
  int32_t inode, a, b, level;
};

struct TreeArgs {
  // particles (sorted order)
  const double *x, *y, *z, *m, *dens;
  const int32_t* orig;
  // groups (1-based ids)
  int32_t ngroups;
  const double* densg;
  const int32_t* gpeak;
  const int32_t* goff;    // [ng+2] member offsets
  const int32_t* gmem;    // members, decreasing particle index
  const double* rdesc;    // member densities, decreasing density (same offsets)
  const double* pref;     // [nact][6] running sums in decreasing-density order:
                          // rho, m, m*dx, m*dy, m*dz, m*|d|^2 (d relative to the group peak)
  // saddle forest (maximum spanning forest of the saddle rows)
  const int32_t* soff;    // [ng+1] row g at [soff[g-1], soff[g])
  const int32_t* sisad;
  const double* srho;
  // parameters
  double Lx, Ly, Lz, hx, hy, hz;  // box and half box (xlongs2...)
  double fudge, alphap, epsilon;
  int32_t nmembthresh;
  // tree state
  int32_t* GL;            // [ng] group list
  int32_t* GL2;           // [ng] reorder target
  int32_t* pos_of;        // [ng+1] position of each group in GL
  int32_t* par;           // [ng] union-find parent (absolute positions)
  int32_t* cnt;           // [ng] component sizes by root / running ranks
  int32_t* run;           // [ng]
  int32_t* cstart;        // [ng] component k of a task starts at cstart[a+k]
  int32_t* compidx;       // [ng] component index of each position
  int32_t* gn;            // [ng] per-position member count above rhot
  double* gs;             // [ng][8] per-position scratch sums
  double* cs;             // [ng][12] per-component scratch
  int32_t* deepnode;      // [ng+1]
  int32_t* gcur;          // [ng+1] members above the group's last threshold
  int32_t* ecur;          // [ng+1] saddle-row entries above the group's last threshold
  NodeRec* node;          // [nnodesmax+1]
  int32_t nnodesmax;
  int32_t* nnodes;        // counter
  Task* next;             // next wave's tasks of at most big_task groups
  int32_t* nnext;
  Task* next_big;         // next wave's tasks of more than big_task groups (kNTBig-thread blocks)
  int32_t big_task;
  int32_t* nnext_big;
  int32_t* max_big;       // largest task pushed to next_big (bounds every task a wide launch runs)
  int32_t* rcnt;          // [kClusterCtas][ng+1] roots counted per CTA in a cluster reorder, by position
  int32_t* rrun;          // [kClusterCtas][ng+1] running ranks per CTA in a cluster reorder, by position
  int32_t par_cap_big;    // union-find parents in shared memory for wide tasks of at most this many groups
  // a slot of next / next_big is readable once its flag is set; ntaken /
  // ntaken_big count the slots that blocks of the current wave took over
  int32_t* qready;
  int32_t* qready_big;
  int32_t* ntaken;
  int32_t* ntaken_big;
  int32_t* err;           // [0] code, [1] detail
  unsigned long long* stats;  // [11] counters (see the end of tree_wave_kernel; [8..10] undecided tests)
  long long* tprof;       // [nnodesmax+1][kProfRow] per-task profile row by node id, or null
};

__device__ __forceinline__ void set_err(const TreeArgs& A, int code, int detail) {
  if (atomicCAS(A.err, 0, code) == 0) A.err[1] = detail;
}

__device__ __forceinline__ void push_task(const TreeArgs& A, const Task& t) {
  const bool big = t.b - t.a > A.big_task;
  if (big) atomicMax(A.max_big, t.b - t.a);
  const int32_t s = atomicAdd(big ? A.nnext_big : A.nnext, 1);
  (big ? A.next_big : A.next)[s] = t;
  __threadfence();
  atomicExch((big ? A.qready_big : A.qready) + s, 1);
}

constexpr long long kTakeSpin = 1LL << 22;  // waits for a claimed slot's record (bounded; an error past it)

// Take a queued task of the next wave, if one is there (one thread).  A slot
// is claimed by advancing the taken counter past it while it is below the
// pushed count; its record was claimed by a pusher that writes it at once,
// so the wait for its flag is short.  Returns false when the queue is empty.
__device__ bool take_task(const TreeArgs& A, bool big, Task& out) {
  int32_t* taken = big ? A.ntaken_big : A.ntaken;
  const int32_t* pushed = big ? A.nnext_big : A.nnext;
  for (;;) {
    const int32_t t = atomicAdd(taken, 0);
    const int32_t n = atomicAdd(const_cast<int32_t*>(pushed), 0);
    if (t >= n) return false;
    if (atomicCAS(taken, t, t + 1) != t) continue;
    int32_t* ready = (big ? A.qready_big : A.qready) + t;
    long long it = 0;
    while (atomicAdd(ready, 0) == 0) {
      if (++it > kTakeSpin) { set_err(A, 18, t); return false; }
      __nanosleep(64);
    }
    __threadfence();
    // another SM wrote the record in this launch: read it past L1
    const Task* r = (big ? A.next_big : A.next) + t;
    out.rhot = __ldcg(&r->rhot);
    out.inode = __ldcg(&r->inode);
    out.a = __ldcg(&r->a);
    out.b = __ldcg(&r->b);
    out.level = __ldcg(&r->level);
    return true;
  }
}


__device__ __forceinline__ double wrapd(double d, double L, double h) {
  // f90:2359-2373 / 1516-1532
  if (d >= h) return xsub(d, L);
  if (d < -h) return xadd(d, L);
  return d;
}

// number of members of group g with density > rhot (members sorted by
// decreasing density).  A group's threshold only rises (a task's rhot grows
// and children start above their parent), so the count is searched downward
// from the group's previous count hi (members [0, hi) were above the group's
// previous threshold; rlast = the density of member hi - 1, off = goff[g]):
// a galloping step then a binary search.
__device__ __forceinline__ int32_t count_above_at(const TreeArgs& A, int32_t g, int32_t off, int32_t hi, double rlast,
                                                  double rhot) {
  if (hi == 0 || rlast > rhot) return hi;
  const double* r = A.rdesc + off;
  // r[j] <= rhot; gallop down until an index above rhot (or 0) brackets the answer
  int32_t j = hi - 1, lo = 0, step = 1;
  while (true) {
    const int32_t k = j - step;
    if (k < 0) { lo = 0; break; }
    if (r[k] > rhot) { lo = k + 1; break; }
    j = k;
    step <<= 1;
  }
  int32_t a2 = lo, b2 = j;  // first index with r <= rhot lies in [lo, j]
  while (a2 < b2) {
    const int32_t mid = (a2 + b2) >> 1;
    if (r[mid] > rhot) a2 = mid + 1; else b2 = mid;
  }
  A.gcur[g] = a2;
  return a2;
}

__device__ __forceinline__ int32_t count_above(const TreeArgs& A, int32_t g, double rhot) {
  const int32_t off = A.goff[g], hi = A.gcur[g];
  return count_above_at(A, g, off, hi, hi > 0 ? A.rdesc[off + hi - 1] : 0.0, rhot);
}

// number of saddle-row entries of group g above rhot (the row is sorted by
// decreasing saddle), searched downward from the previous count hi like
// count_above (e0 = the row's start, rlast = the saddle of entry hi - 1).
__device__ __forceinline__ int32_t edges_above_at(const TreeArgs& A, int32_t g, int32_t e0, int32_t hi, double rlast,
                                                  double rhot) {
  if (hi == 0 || rlast > rhot) return hi;
  const double* r = A.srho + e0;
  int32_t j = hi - 1, lo = 0, step = 1;
  while (true) {
    const int32_t k = j - step;
    if (k < 0) { lo = 0; break; }
    if (r[k] > rhot) { lo = k + 1; break; }
    j = k;
    step <<= 1;
  }
  int32_t a2 = lo, b2 = j;
  while (a2 < b2) {
    const int32_t mid = (a2 + b2) >> 1;
    if (r[mid] > rhot) a2 = mid + 1; else b2 = mid;
  }
  A.ecur[g] = a2;
  return a2;
}

__device__ int32_t uf_find(int32_t* par, int32_t i) {
  // path halving; every chain ends at a self-parent
  for (int it = 0; it < (1 << 26); ++it) {
    int32_t p = par[i];
    if (p == i) return i;
    int32_t gp = par[p];
    if (gp != p) atomicCAS(&par[i], p, gp);
    i = gp;
  }
  return i;
}

__device__ void uf_union(int32_t* par, int32_t i, int32_t j) {
  for (int it = 0; it < (1 << 26); ++it) {
    i = uf_find(par, i);
    j = uf_find(par, j);
    if (i == j) return;
    if (i < j) { int32_t t = i; i = j; j = t; }  // link the larger root under the smaller
    if (atomicCAS(&par[i], i, j) == i) return;
  }
}

__device__ __forceinline__ double atomic_min_pos(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long nv = __double_as_longlong(v);
  unsigned long long old = atomicMin(a, nv);
  return __longlong_as_double(old);
}

// -------------------------------------------------------------------------
// Structural pass at rhot over positions [a, b): drop groups with peak
// density <= rhot, percolate through saddles > rhot, reorder components.
// Returns (in shared) new b, ncomp, and the next threshold at which the
// structure can change.
struct SharedTask {
  double rhot;
  double next_event;
  int32_t inode, a, b, level, ncomp, nsurv, nsisters, done, nexact, inode1, kk;
  int32_t flag, nbig;
  long long iters;
  // the task the block runs next (a child it continues), and its size at start
  unsigned long long best;
  Task cont;
  int32_t has_cont, groups0;
  // groups dropped from the range as below the member threshold for good:
  // how many, and the bits of their largest peak density (0: none)
  int32_t npruned;
  unsigned long long pruned_max_bits;
  // cluster phases of a wide task: the phase the leader hands its followers,
  // whether the union-find array is the leader's shared memory, and each
  // follower's smallest next event of a union phase
  int32_t phase, plocal;
  double ev_part[kClusterCtas];
  int32_t fold_n;  // large components whose partial sums a decide phase folds
};

namespace cg = cooperative_groups;

// CTAs of the launch's cluster (1 outside a cluster launch)
__device__ __forceinline__ int cluster_ctas() { return (int)cg::this_cluster().num_blocks(); }

// The leader hands phase `code` to its followers: a cluster-wide barrier that
// every thread of every CTA of the cluster takes; the phase ends with a second
// one (cg::this_cluster().sync()) once each CTA has done its slice.
__device__ __forceinline__ void lead_phase(SharedTask& T, int32_t code, bool local) {
  if (threadIdx.x == 0) { T.phase = code; T.plocal = local ? 1 : 0; }
  cg::this_cluster().sync();
}

// ---- position-parallel phases of a structural pass, over the positions
// [a, b) that fall to cluster-wide thread gt (stride gs): one block runs them
// with gt = threadIdx.x, gs = NT; a wide task's cluster splits them over its
// CTAs (see tree_wave_kernel).  par is the union-find array (entries relative
// to poff), in the leader CTA's shared memory or in global memory.
//
// Union over saddle edges above rhot (a prefix of each row, rows sorted by
// decreasing saddle).  Each undirected edge is linked once, from the row of
// its smaller group id; rows with more than kRowWarp such edges go to the
// block's list s_big (count *nbig) for union_long_rows.  The next event is the
// smallest peak density or saddle still above rhot (the last edge of each
// prefix): the block's minimum lands in *ev_min.
template <int NT>
__device__ void union_short_rows(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, double rhot, int32_t* par,
                                 int32_t* s_big, int32_t* nbig, double* ev_min, int32_t gt, int32_t gs) {
  double ev = DBL_MAX;
  for (int32_t i = a + gt; i < b; i += gs) {
    const int32_t g = A.GL[i];
    const double dg = A.densg[g];
    if (!(dg > rhot)) continue;
    ev = fmin(ev, dg);
    const int32_t e0 = A.soff[g - 1];
    const int32_t c = A.ecur[g];
    const int32_t ne = edges_above_at(A, g, e0, c, c > 0 ? A.srho[e0 + c - 1] : 0.0, rhot);
    if (ne == 0) continue;
    ev = fmin(ev, A.srho[e0 + ne - 1]);
    if (ne > kRowWarp) {
      const int32_t slot = atomicAdd(nbig, 1);
      if (slot < kMaxBigRows) { s_big[slot] = i; continue; }
    }
    for (int32_t e = e0; e < e0 + ne; ++e) {
      const int32_t h = A.sisad[e];
      const int32_t j = A.pos_of[h];
      if (j < a || j >= b) { set_err(A, 11, g); continue; }  // f90:1229-1233
      if (h > g) uf_union(par, i - poff, j - poff);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ev = fmin(ev, __shfl_xor_sync(0xffffffffu, ev, o));
  if ((threadIdx.x & 31) == 0 && ev < DBL_MAX) atomic_min_pos(ev_min, ev);
}

// the block's long rows (s_big), a warp each
template <int NT>
__device__ void union_long_rows(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, int32_t* par,
                                const int32_t* s_big, int32_t nbig) {
  const int tid = threadIdx.x, lane = tid & 31;
  nbig = min(nbig, kMaxBigRows);
  for (int32_t bi = tid >> 5; bi < nbig; bi += NT / 32) {
    const int32_t i = s_big[bi];
    const int32_t g = A.GL[i];
    const int32_t e0 = A.soff[g - 1], e1 = e0 + A.ecur[g];
    for (int32_t e = e0 + lane; e < e1; e += 32) {
      const int32_t h = A.sisad[e];
      const int32_t j = A.pos_of[h];
      if (j < a || j >= b) { set_err(A, 11, g); continue; }
      if (h > g) uf_union(par, i - poff, j - poff);
    }
  }
}

// roots of the surviving positions, component sizes by root in cnt; dropped
// groups get -1
__device__ __forceinline__ void find_roots(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, double rhot,
                                           int32_t* par, int32_t gt, int32_t gs) {
  for (int32_t i = a + gt; i < b; i += gs) {
    const int32_t g = A.GL[i];
    if (A.densg[g] > rhot) {
      const int32_t r = uf_find(par, i - poff);
      par[i - poff] = r;
      atomicAdd(&A.cnt[r + poff], 1);
    } else {
      par[i - poff] = -1;
    }
  }
}

// Stable reorder by root of positions [c_begin, c_end) (whole chunks of
// NT * IPT positions from a, or the task's end) into GL2: inside a chunk a
// stable block radix sort groups equal roots; a run's rank is its offset from
// the run head (block max-scan of head indices); run[] carries each root's
// rank across the chunks (entry r - a for root position r).
template <int NT, class SortT, class MaxScanT>
__device__ void reorder_chunks(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, const int32_t* par,
                               int32_t* run, int32_t c_begin, int32_t c_end,
                               typename SortT::TempStorage& sort_tmp,
                               typename MaxScanT::TempStorage& maxscan_tmp, int32_t* s_keys) {
  constexpr int IPT = ipt_for(NT);
  const int tid = threadIdx.x;
  const int32_t sent = b - a;  // key of dropped groups, above every root offset
  const int kbits = 32 - __clz(sent);
  for (int32_t c0 = c_begin; c0 < c_end; c0 += (NT * IPT)) {
    int32_t keys[IPT], vals[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      int32_t i = c0 + tid * IPT + k;
      int32_t r = (i < c_end) ? par[i - poff] : -1;
      keys[k] = (r >= 0) ? (r + poff - a) : sent;
      vals[k] = i;
    }
    SortT(sort_tmp).Sort(keys, vals, 0, kbits);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < IPT; ++k) s_keys[tid * IPT + k] = keys[k];
    __syncthreads();
    int32_t headq[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      int q = tid * IPT + k;
      headq[k] = (q == 0 || s_keys[q - 1] != keys[k]) ? q : 0;
    }
    MaxScanT(maxscan_tmp).InclusiveScan(headq, headq, cub::Max());
    bool tail[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      int q = tid * IPT + k;
      tail[k] = (q == (NT * IPT) - 1) || (s_keys[q + 1] != keys[k]);
      if (keys[k] == sent) continue;
      int32_t np = a + A.cnt[keys[k] + a] + run[keys[k]] + (q - headq[k]);
      if (np < a || np >= b) { set_err(A, 17, np); continue; }
      A.GL2[np] = A.GL[vals[k]];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      int q = tid * IPT + k;
      if (tail[k] && keys[k] != sent) run[keys[k]] += q - headq[k] + 1;
    }
    __syncthreads();
  }
}

// chunk range [ch0, ch1) of the cluster's CTA `rank` (of K) over positions [a, b)
template <int NT>
__device__ __forceinline__ void reorder_range_of(int32_t a, int32_t b, int rank, int K, int32_t& p0, int32_t& p1) {
  constexpr int32_t CH = NT * ipt_for(NT);
  const int32_t nch = (b - a + CH - 1) / CH, per = (nch + K - 1) / K;
  const int32_t ch0 = min(nch, rank * per), ch1 = min(nch, ch0 + per);
  p0 = a + ch0 * CH;
  p1 = min(b, a + ch1 * CH);
}

// a cluster reorder, step 1: CTA rank counts the roots of its chunk range in
// its own row of A.rcnt, at the root's absolute position (the positions of
// tasks that run at the same time on other clusters are disjoint)
template <int NT>
__device__ void reorder_count(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, const int32_t* par, int rank,
                              int K) {
  const int tid = threadIdx.x;
  int32_t* cnt = A.rcnt + (size_t)rank * (A.ngroups + 1) + a;  // entry r - a
  for (int32_t j = tid; j < b - a; j += NT) cnt[j] = 0;
  __syncthreads();
  int32_t p0, p1;
  reorder_range_of<NT>(a, b, rank, K, p0, p1);
  for (int32_t i = p0 + tid; i < p1; i += NT) {
    const int32_t r = par[i - poff];
    if (r >= 0) atomicAdd(&cnt[r + poff - a], 1);
  }
}

// step 2 (after every CTA's count): ranks start after the counts of the
// ranges before this one, then the range is reordered
template <int NT, class SortT, class MaxScanT>
__device__ void reorder_range(const TreeArgs& A, int32_t a, int32_t b, int32_t poff, const int32_t* par, int rank,
                              int K, typename SortT::TempStorage& sort_tmp,
                              typename MaxScanT::TempStorage& maxscan_tmp, int32_t* s_keys) {
  const int tid = threadIdx.x;
  const size_t G = (size_t)A.ngroups + 1;
  int32_t* run = A.rrun + (size_t)rank * G + a;  // entry r - a
  for (int32_t j = tid; j < b - a; j += NT) {
    int32_t v = 0;
    for (int r = 0; r < rank; ++r) v += A.rcnt[(size_t)r * G + a + j];
    run[j] = v;
  }
  __syncthreads();
  int32_t p0, p1;
  reorder_range_of<NT>(a, b, rank, K, p0, p1);
  reorder_chunks<NT, SortT, MaxScanT>(A, a, b, poff, par, run, p0, p1, sort_tmp, maxscan_tmp, s_keys);
}

template <int NT, class SortT, class ScanT, class MaxScanT>
__device__ void structural_pass(const TreeArgs& A, SharedTask& T, typename SortT::TempStorage& sort_tmp,
                                typename ScanT::TempStorage& scan_tmp, typename MaxScanT::TempStorage& maxscan_tmp,
                                int32_t* s_keys, int32_t* s_big, int32_t* s_par, long long* ph) {
  constexpr int IPT = ipt_for(NT);
  const int tid = threadIdx.x;
  const int32_t a = T.a, b = T.b;
  // union-find parents: in shared memory when the task fits (entries relative
  // to a), else the global array (absolute positions)
  const bool local = (b - a) <= (NT >= 1024 ? A.par_cap_big : par_cap(NT));
  int32_t* par = local ? s_par : A.par;
  const int32_t poff = local ? a : 0;
  const double rhot = T.rhot;
  long long tl = clock64();
  // thread 0 charges the cycles since the last mark to phase k
  auto mark = [&](int k) {
    if (tid == 0) { const long long t = clock64(); ph[k] += t - tl; tl = t; }
  };
  if (tid == 0) { T.next_event = DBL_MAX; T.nbig = 0; }
  for (int32_t i = a + tid; i < b; i += NT) {
    par[i - poff] = i - poff;
    A.cnt[i] = 0;
    A.run[i] = 0;
  }
  __syncthreads();
  mark(0);
  const int K = NT >= 1024 ? cluster_ctas() : 1;
  if (K > 1) lead_phase(T, kPhUnion, local);
  union_short_rows<NT>(A, a, b, poff, rhot, par, s_big, &T.nbig, &T.next_event, tid, K * NT);
  __syncthreads();
  mark(12);
  union_long_rows<NT>(A, a, b, poff, par, s_big, T.nbig);
  if (K > 1) {
    cg::this_cluster().sync();  // the followers' unions and next events are in
    if (tid == 0)
      for (int r = 1; r < K; ++r) T.next_event = fmin(T.next_event, T.ev_part[r]);
  }
  __syncthreads();
  mark(1);
  if (K > 1) lead_phase(T, kPhFind, local);
  find_roots(A, a, b, poff, rhot, par, tid, K * NT);
  if (K > 1) cg::this_cluster().sync();
  __syncthreads();
  mark(2);
  // exclusive scan of component sizes over root positions -> component offsets (in cnt)
  int32_t carry = 0;
  for (int32_t c0 = a; c0 < b; c0 += NT) {
    int32_t i = c0 + tid;
    int32_t v = (i < b) ? A.cnt[i] : 0;
    int32_t ex, tot;
    ScanT(scan_tmp).ExclusiveSum(v, ex, tot);
    __syncthreads();
    if (i < b) A.cnt[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  const int32_t nsurv = carry;
  mark(3);
  // stable reorder by root, chunk by chunk: inside a chunk a stable block
  // radix sort groups equal roots; a run's rank is its offset from the run
  // head (block max-scan of head indices); run[] carries ranks across chunks
  if (K > 1 && b - a > (kClusterReorderChunks - 1) * NT * IPT) {
    // the cluster's CTAs take contiguous ranges of chunks: each counts the
    // roots of its range, then starts its ranks after the counts of the
    // ranges before it (worth its three barriers and the rank set-up only
    // for long tasks)
    lead_phase(T, kPhReorder, local);
    reorder_count<NT>(A, a, b, poff, par, 0, K);
    cg::this_cluster().sync();
    reorder_range<NT, SortT, MaxScanT>(A, a, b, poff, par, 0, K, sort_tmp, maxscan_tmp, s_keys);
    cg::this_cluster().sync();
  } else {
    reorder_chunks<NT, SortT, MaxScanT>(A, a, b, poff, par, A.run + a, a, b, sort_tmp, maxscan_tmp, s_keys);
  }
  mark(4);
  // copy back, positions, component starts
  for (int32_t i = a + tid; i < a + nsurv; i += NT) {
    int32_t g = A.GL2[i];
    A.GL[i] = g;
    A.pos_of[g] = i;
  }
  __syncthreads();
  mark(5);
  // component starts: root positions r (par[r] == r before reorder) map to start a + cnt[r]
  // collect them in order with a scan over root flags
  carry = 0;
  for (int32_t c0 = a; c0 < b; c0 += NT) {
    int32_t i = c0 + tid;
    int32_t isroot = (i < b && par[i - poff] == i - poff) ? 1 : 0;
    int32_t ex, tot;
    ScanT(scan_tmp).ExclusiveSum(isroot, ex, tot);
    __syncthreads();
    if (isroot) A.cstart[a + carry + ex] = a + A.cnt[i];
    carry += tot;
    __syncthreads();
  }
  const int32_t ncomp = carry;
  mark(6);
  if (tid == 0) {
    T.ncomp = ncomp;
    T.nsurv = nsurv;
    T.b = a + nsurv;
  }
  // component index of every surviving position: inclusive scan of the
  // component-start flags (run[] is free after the reorder)
  for (int32_t i = a + tid; i < a + nsurv; i += NT) A.run[i] = 0;
  __syncthreads();
  for (int32_t k = tid; k < ncomp; k += NT) A.run[A.cstart[a + k]] = 1;
  __syncthreads();
  carry = 0;
  for (int32_t c0 = a; c0 < a + nsurv; c0 += NT) {
    const int32_t i = c0 + tid;
    const int32_t v = (i < a + nsurv) ? A.run[i] : 0;
    int32_t inc, tot;
    ScanT(scan_tmp).InclusiveSum(v, inc, tot);
    __syncthreads();
    if (i < a + nsurv) A.compidx[i] = carry + inc - 1;
    carry += tot;
  }
  __syncthreads();
  mark(7);
}

__device__ __forceinline__ int32_t comp_end(const TreeArgs& A, const SharedTask& T, int32_t k) {
  return (k + 1 < T.ncomp) ? A.cstart[T.a + k + 1] : T.b;
}

// -------------------------------------------------------------------------
// Per-component quantities.  cs row (12 doubles) for component k at index a+k:
//  0 mass_loc  1 mass_comp  2 densmax  3 sum rho  4 M  5 Sx 6 Sy 7 Sz 8 Q
//  9 decision (0 false, 1 true, 2 unknown)  10 exact flag  11 posref
// (9..11 hold the component's anchor while its groups' terms are formed).
// An exact recomputation overwrites 0..9 (colour_fold).

// Three-state outcomes as bit sets: bit 0 "can be true", bit 1 "can be
// false" -- kTrue = 1, kFalse = 2, kUnknown = 3.  Branch-free.
constexpr int kTrue = 1, kFalse = 2, kUnknown = 3;
__device__ __forceinline__ int tri_and(int p, int q) { return (p & q & 1) | ((p | q) & 2); }
__device__ __forceinline__ int tri_or(int p, int q) { return ((p | q) & 1) | (p & q & 2); }
// v > t with v known to +-e (NaN: unknown)
__device__ __forceinline__ int tri_gt(double v, double t, double e) {
  const bool can_true = !(v + e <= t), can_false = !(v - e > t);
  return (can_true ? 1 : 0) | (can_false ? 2 : 0);
}

// Approximate terms of the group at position i for its component's anchor
// (a: x, y, z of the peak of the component's first group).  gs row:
// 0 densg, 1 sum rho, 2 mass, 3..5 first moments about the anchor, 6 second
// moment, 7 tri-state test "mean density of the group above rhot";
// gn[i] = members above rhot (exact).
__device__ __forceinline__ void store_terms(const TreeArgs& A, int32_t i, int32_t ng, double dg, const double* P,
                                            double dx, double dy, double dz, double rhot) {
  const double u = 1.1102230246251565e-16;
  double* G = A.gs + 8 * (size_t)i;
  A.gn[i] = ng;
  double t[7] = {0, 0, 0, 0, 0, 0, (double)kFalse};
  if (ng > 0) {
    const double sg = P[0], mg = P[1];
    t[0] = sg;
    t[1] = mg;
    t[2] = P[2] + mg * dx;
    t[3] = P[3] + mg * dy;
    t[4] = P[4] + mg * dz;
    t[5] = P[5] + 2.0 * (dx * P[2] + dy * P[3] + dz * P[4]) + mg * (dx * dx + dy * dy + dz * dz);
    const double dn = (double)ng;
    const double vg = (sg / dn) / (1.0 + A.fudge / sqrt(dn));
    t[6] = (double)tri_gt(vg, rhot, (2.0 * dn + 8.0) * u * fabs(vg) * 1.01);
  }
  G[0] = dg;
#pragma unroll
  for (int c = 0; c < 7; ++c) G[1 + c] = t[c];
}

__device__ __forceinline__ void position_terms(const TreeArgs& A, int32_t i, double rhot, const double* a) {
  const int32_t g = A.GL[i];
  const int32_t ng = count_above(A, g, rhot);
  double P[6] = {0, 0, 0, 0, 0, 0};
  double dx = 0, dy = 0, dz = 0;
  if (ng > 0) {
    const double* Pp = A.pref + 6 * (size_t)(A.goff[g] + ng - 1);
#pragma unroll
    for (int c = 0; c < 6; ++c) P[c] = Pp[c];
    const int32_t pg = A.gpeak[g];
    dx = wrapd(A.x[pg] - a[0], A.Lx, A.hx);
    dy = wrapd(A.y[pg] - a[1], A.Ly, A.hy);
    dz = wrapd(A.z[pg] - a[2], A.Lz, A.hz);
  }
  store_terms(A, i, ng, A.densg[g], P, dx, dy, dz, rhot);
}

// Sum the gs rows of positions [c0, c1) over one warp and decide the
// significance test (f90:1459-1463) in three states from the rigorous
// rounding bounds; lane 0 writes cs row C.
// The three-state significance test (f90:1459-1463) from a component's
// approximate sums; writes cs row C.
__device__ void decide_from_sums(const TreeArgs& A, double rhot, long long nl, int32_t nmax, double dmax, double S,
                                 double M, double Sx, double Sy, double Sz, double Q, int triB, double* C) {
  const double u = 1.1102230246251565e-16;
  const double n = (double)nl;
  C[0] = n; C[1] = (double)nmax; C[2] = dmax; C[3] = S;
  C[4] = M; C[5] = Sx; C[6] = Sy; C[7] = Sz; C[8] = Q;
  int dec;
  if (nl < A.nmembthresh) {
    dec = 0;
  } else {
    const double dm = S / n;
    const double edm = (2.0 * n + 8.0) * u * dm * 1.01;
    const double thrA = xmul(rhot, xadd(1.0, xdiv(A.fudge, xsqrt(n))));
    const int tA = tri_gt(dm, thrA, edm);
    // dmax >= alphap * densmoy, densmoy known to +-edm
    const double tiny = 8.0 * u * fabs(A.alphap * dm);
    const bool c_true = dmax >= A.alphap * (dm + edm) + tiny, c_false = dmax < A.alphap * (dm - edm) - tiny;
    const int tC = (c_false ? 0 : 1) | (c_true ? 0 : 2);
    // radius test r >= epsilon.  The reference forms r^2 from absolute
    // coordinates (|u| <= L after the unwrap about posref), so its own value
    // carries up to ~(18n+48)u L^2 of cancellation error; these sums carry up
    // to ~3(2n+8)u * 3L^2 * 2 more.  Decide only outside both.
    const double r2 = Q / M - (Sx * Sx + Sy * Sy + Sz * Sz) / (M * M);
    const double Lm = fmax(A.Lx, fmax(A.Ly, A.Lz));
    const double er2 = ((18.0 * n + 48.0) + 18.0 * (2.0 * n + 8.0)) * u * Lm * Lm * 1.01;
    const double e2 = A.epsilon * A.epsilon;
    const bool d_true = r2 - er2 >= e2 * (1.0 + 16.0 * u), d_false = r2 + er2 < e2 * (1.0 - 16.0 * u);
    const int tD = (d_false ? 0 : 1) | (d_true ? 0 : 2);
    const int t = tri_and(tri_and(tri_or(tA, triB), tC), tD);
    dec = (t == kTrue) ? 1 : (t == kFalse ? 0 : 2);
    if (dec == 2) {
      if (tA == kUnknown) atomicAdd(&A.stats[8], 1ULL);
      if (triB == kUnknown) atomicAdd(&A.stats[9], 1ULL);
      if (tC == kUnknown || tD == kUnknown) atomicAdd(&A.stats[10], 1ULL);
    }
  }
  C[9] = (double)dec;
  C[10] = (dec == 2) ? 1.0 : 0.0;  // undecided: recompute exactly
}

// component_decide for a small component on one thread (no shuffles)
__device__ void component_decide_thread(const TreeArgs& A, int32_t c0, int32_t c1, double rhot, double* C) {
  long long nl = 0;
  int32_t nmax = 0;
  double dmax = -1.0, S = 0, M = 0, Sx = 0, Sy = 0, Sz = 0, Q = 0;
  int triB = kFalse;
  for (int32_t i = c0; i < c1; ++i) {
    const double* G = A.gs + 8 * (size_t)i;
    const int32_t ng = A.gn[i];
    nl += ng;
    nmax = max(nmax, ng);
    dmax = fmax(dmax, G[0]);
    S += G[1];
    M += G[2];
    Sx += G[3];
    Sy += G[4];
    Sz += G[5];
    Q += G[6];
    triB = tri_or(triB, (int)G[7]);
  }
  decide_from_sums(A, rhot, nl, nmax, dmax, S, M, Sx, Sy, Sz, Q, triB, C);
}

__device__ void component_decide(const TreeArgs& A, int32_t c0, int32_t c1, double rhot, double* C, int lane) {
  long long nl = 0;
  int32_t nmax = 0;
  double dmax = -1.0, S = 0, M = 0, Sx = 0, Sy = 0, Sz = 0, Q = 0;
  int triB = kFalse;  // densmoy_comp_max > rhot
#pragma unroll 4
  for (int32_t i = c0 + lane; i < c1; i += 32) {
    const double* G = A.gs + 8 * (size_t)i;
    const int32_t ng = A.gn[i];
    nl += ng;
    nmax = max(nmax, ng);
    dmax = fmax(dmax, G[0]);
    S += G[1];
    M += G[2];
    Sx += G[3];
    Sy += G[4];
    Sz += G[5];
    Q += G[6];
    triB = tri_or(triB, (int)G[7]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nl += __shfl_xor_sync(0xffffffffu, nl, o);
    nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    S += __shfl_xor_sync(0xffffffffu, S, o);
    M += __shfl_xor_sync(0xffffffffu, M, o);
    Sx += __shfl_xor_sync(0xffffffffu, Sx, o);
    Sy += __shfl_xor_sync(0xffffffffu, Sy, o);
    Sz += __shfl_xor_sync(0xffffffffu, Sz, o);
    Q += __shfl_xor_sync(0xffffffffu, Q, o);
    triB = tri_or(triB, __shfl_xor_sync(0xffffffffu, triB, o));
  }
  if (lane != 0) return;
  decide_from_sums(A, rhot, nl, nmax, dmax, S, M, Sx, Sy, Sz, Q, triB, C);
}

// component_decide for a large component on the whole block: every thread
// sums a strided share of its rows, warps fold their lanes, warp 0 folds the
// warps.  (The three-state test's bounds hold for any summation order.)
struct CompSums {
  long long nl;
  int32_t nmax, triB;
  double dmax, S, M, Sx, Sy, Sz, Q;
};

template <int NT>
__device__ CompSums block_partial_sums(const TreeArgs& A, int32_t c0, int32_t c1, int32_t gt, int32_t gs,
                                       CompSums* red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  CompSums s{0, 0, kFalse, -1.0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int32_t i = c0 + gt; i < c1; i += gs) {
    const double* G = A.gs + 8 * (size_t)i;
    const int32_t ng = A.gn[i];
    s.nl += ng;
    s.nmax = max(s.nmax, ng);
    s.dmax = fmax(s.dmax, G[0]);
    s.S += G[1];
    s.M += G[2];
    s.Sx += G[3];
    s.Sy += G[4];
    s.Sz += G[5];
    s.Q += G[6];
    s.triB = tri_or(s.triB, (int)G[7]);
  }
  auto fold = [&](CompSums& v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v.nl += __shfl_xor_sync(0xffffffffu, v.nl, o);
      v.nmax = max(v.nmax, __shfl_xor_sync(0xffffffffu, v.nmax, o));
      v.dmax = fmax(v.dmax, __shfl_xor_sync(0xffffffffu, v.dmax, o));
      v.S += __shfl_xor_sync(0xffffffffu, v.S, o);
      v.M += __shfl_xor_sync(0xffffffffu, v.M, o);
      v.Sx += __shfl_xor_sync(0xffffffffu, v.Sx, o);
      v.Sy += __shfl_xor_sync(0xffffffffu, v.Sy, o);
      v.Sz += __shfl_xor_sync(0xffffffffu, v.Sz, o);
      v.Q += __shfl_xor_sync(0xffffffffu, v.Q, o);
      v.triB = tri_or(v.triB, __shfl_xor_sync(0xffffffffu, v.triB, o));
    }
  };
  fold(s);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  CompSums w{0, 0, kFalse, -1.0, 0, 0, 0, 0, 0, 0};
  if (warp == 0) {
    if (lane < NT / 32) w = red[lane];
    fold(w);
  }
  __syncthreads();  // red is reused by the next call
  return w;
}

// two partial sums folded (any order: the test's bounds do not depend on it)
__device__ __forceinline__ CompSums add_sums(CompSums x, const CompSums& y) {
  x.nl += y.nl;
  x.nmax = max(x.nmax, y.nmax);
  x.dmax = fmax(x.dmax, y.dmax);
  x.S += y.S;
  x.M += y.M;
  x.Sx += y.Sx;
  x.Sy += y.Sy;
  x.Sz += y.Sz;
  x.Q += y.Q;
  x.triB = tri_or(x.triB, y.triB);
  return x;
}

template <int NT>
__device__ void component_decide_block(const TreeArgs& A, int32_t c0, int32_t c1, double rhot, double* C,
                                       CompSums* red) {
  const CompSums w = block_partial_sums<NT>(A, c0, c1, threadIdx.x, NT, red);
  if (threadIdx.x == 0) decide_from_sums(A, rhot, w.nl, w.nmax, w.dmax, w.S, w.M, w.Sx, w.Sy, w.Sz, w.Q, w.triB, C);
}

// components of more groups than this are summed by the whole block
__host__ __device__ constexpr int block_comp_for(int nt) { return nt >= 1024 ? 512 : 1024; }
constexpr int kMaxBlockComps = 32;
// large components a cluster's decide phase takes at once (their per-CTA
// partial sums sit after the block fold's scratch, over the reorder keys)
constexpr int kFoldBatch = 8;
static_assert((kNTBig / 32 + kFoldBatch * kClusterCtas) * (int)sizeof(CompSums) <= kNTBig * 2 * 4,
              "cluster partial sums must fit the reorder keys");

// The decide phase of a wide task's cluster: warp w of CTA rank decides the
// mid-sized components k = rank * NT / 32 + w (stride K * NT / 32); then for
// each of the nbc large components listed in bc the CTA's partial sums over
// its slice of rows go to parts[j * kClusterCtas + rank] (the leader's shared
// memory), which the leader folds and decides.
template <int NT>
__device__ void decide_slice(const TreeArgs& A, int32_t a, int32_t b, int32_t ncomp, double rhot, int rank, int K,
                             const int32_t* bc, int32_t nbc, CompSums* red, CompSums* parts) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int32_t k = rank * (NT / 32) + warp; k < ncomp; k += K * (NT / 32)) {
    const int32_t c0 = A.cstart[a + k], c1 = k + 1 < ncomp ? A.cstart[a + k + 1] : b;
    if (c1 - c0 > kSmallComp && c1 - c0 <= block_comp_for(NT))
      component_decide(A, c0, c1, rhot, A.cs + 12 * (size_t)(a + k), lane);
  }
  for (int32_t j = 0; j < nbc; ++j) {
    const int32_t k = bc[j];
    const int32_t c0 = A.cstart[a + k], c1 = k + 1 < ncomp ? A.cstart[a + k + 1] : b;
    const CompSums p = block_partial_sums<NT>(A, c0, c1, rank * NT + tid, K * NT, red);
    if (tid == 0) parts[j * kClusterCtas + rank] = p;
  }
}

// Approximate statistics of every component of the task: anchors, then the
// groups' terms position-parallel over the whole block, then a thread per
// small component, a warp per mid-sized one and the whole block per large
// one sums them and decides.
// s_bc (kMaxBlockComps entries) and s_red (NT / 32) are scratch that the
// block's other phases own (no extra shared memory: that would shrink L1);
// T.nbig counts the large components here.
template <int NT>
__device__ void approx_stats(const TreeArgs& A, SharedTask& T, long long* ph, int32_t* s_bc, CompSums* s_red) {
  int32_t& s_nbc = T.nbig;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double rhot = T.rhot;
  const int32_t a = T.a, b = T.b, ncomp = T.ncomp;
  long long tl = clock64();
  auto mark = [&](int k) {
    if (tid == 0) { const long long t = clock64(); ph[k] += t - tl; tl = t; }
  };
  if (tid == 0) s_nbc = 0;
  for (int32_t k = tid; k < ncomp; k += NT) {
    const int32_t p0 = A.gpeak[A.GL[A.cstart[a + k]]];
    double* C = A.cs + 12 * (size_t)(a + k);
    C[9] = A.x[p0];
    C[10] = A.y[p0];
    C[11] = A.z[p0];
  }
  __syncthreads();
  mark(8);
  {
    const int K = NT >= 1024 ? cluster_ctas() : 1;
    if (K > 1) lead_phase(T, kPhTerms, false);
    for (int32_t i = a + tid; i < b; i += K * NT)
      position_terms(A, i, rhot, A.cs + 12 * (size_t)(a + A.compidx[i]) + 9);
    if (K > 1) cg::this_cluster().sync();
  }
  __syncthreads();
  mark(9);
  for (int32_t k = tid; k < ncomp; k += NT) {
    const int32_t c0 = A.cstart[a + k], c1 = comp_end(A, T, k);
    if (c1 - c0 <= kSmallComp) {
      component_decide_thread(A, c0, c1, rhot, A.cs + 12 * (size_t)(a + k));
    } else if (c1 - c0 > block_comp_for(NT)) {
      const int32_t slot = atomicAdd(&s_nbc, 1);
      if (slot < kMaxBlockComps) s_bc[slot] = k;
    }
  }
  __syncthreads();
  mark(10);
  // more large components than the list holds: warps take all of them
  const int32_t nbc = s_nbc;
  const bool by_block = nbc <= kMaxBlockComps;
  const int K = NT >= 1024 ? cluster_ctas() : 1;
  if (K > 1 && by_block && nbc <= kFoldBatch) {
    CompSums* s_parts = s_red + NT / 32;
    if (tid == 0) T.fold_n = nbc;
    lead_phase(T, kPhDecide, false);
    decide_slice<NT>(A, a, b, ncomp, rhot, 0, K, s_bc, nbc, s_red, s_parts);
    cg::this_cluster().sync();  // every CTA's decisions and partial sums are in
    if (tid == 0)
      for (int32_t j = 0; j < nbc; ++j) {
        CompSums w = s_parts[j * kClusterCtas];
        for (int r = 1; r < K; ++r) w = add_sums(w, s_parts[j * kClusterCtas + r]);
        decide_from_sums(A, rhot, w.nl, w.nmax, w.dmax, w.S, w.M, w.Sx, w.Sy, w.Sz, w.Q, w.triB,
                         A.cs + 12 * (size_t)(a + s_bc[j]));
      }
    __syncthreads();
    mark(11);
    return;
  }
  for (int32_t k = warp; k < ncomp; k += NT / 32) {
    const int32_t c0 = A.cstart[a + k], c1 = comp_end(A, T, k);
    if (c1 - c0 > kSmallComp && !(by_block && c1 - c0 > block_comp_for(NT)))
      component_decide(A, c0, c1, rhot, A.cs + 12 * (size_t)(a + k), lane);
  }
  if (by_block) {
    for (int32_t j = 0; j < nbc; ++j) {
      const int32_t k = s_bc[j];
      component_decide_block<NT>(A, A.cstart[a + k], comp_end(A, T, k), rhot, A.cs + 12 * (size_t)(a + k), s_red);
    }
  }
  __syncthreads();
  mark(11);
}

// Exact per-group sums in the reference order (treat_particles f90:2317-2401):
// members in decreasing particle index, only those above rhot, positions
// unwrapped about posref then shifted back.  G[0..6] = imass, truemass,
// posg(3), rsquare, densmoy.
__device__ void group_sums_thread(const TreeArgs& A, int32_t g, double rhot, double rx, double ry, double rz,
                                  double* G) {
  int32_t imass = 0;
  double tm = 0, px = 0, py = 0, pz = 0, rs = 0, dm = 0;
  for (int32_t q = A.goff[g]; q < A.goff[g + 1]; ++q) {
    const int32_t s = A.gmem[q];
    const double d = A.dens[s];
    if (!(d > rhot)) continue;
    imass += 1;
    const double xm = A.m[s];
    tm = xadd(tm, xm);
    double ux = wrapd(xsub(A.x[s], rx), A.Lx, A.hx);
    double uy = wrapd(xsub(A.y[s], ry), A.Ly, A.hy);
    double uz = wrapd(xsub(A.z[s], rz), A.Lz, A.hz);
    ux = xadd(ux, rx);
    uy = xadd(uy, ry);
    uz = xadd(uz, rz);
    px = xadd(px, xmul(ux, xm));
    py = xadd(py, xmul(uy, xm));
    pz = xadd(pz, xmul(uz, xm));
    rs = xadd(rs, xmul(xm, xadd(xadd(xmul(ux, ux), xmul(uy, uy)), xmul(uz, uz))));
    dm = xadd(dm, d);
  }
  G[0] = (double)imass; G[1] = tm; G[2] = px; G[3] = py; G[4] = pz; G[5] = rs; G[6] = dm;
}

// Same sums for a large group by one warp: each lane computes the terms of
// one member (explicitly rounded, so each term has the reference's bits); the
// terms of the members above rhot are packed in member order and lanes 0..5
// each run one of the six sequential sums over them -- the same sequence of
// roundings as the Fortran loop, without one dependent global load per
// member on one thread.  st: 32*6 doubles of warp-private shared memory.
__device__ void group_sums_warp(const TreeArgs& A, int32_t g, double rhot, double rx, double ry, double rz,
                                double* G, double* st, int lane) {
  const int32_t q0 = A.goff[g], q1 = A.goff[g + 1];
  int32_t imass = 0;
  double acc = 0.0;  // lane c < 6 carries sum c: truemass, posg(3), rsquare, densmoy
  for (int32_t base = q0; base < q1; base += 32) {
    const int32_t q = base + lane;
    bool ok = false;
    double t[6];
    if (q < q1) {
      const int32_t s = A.gmem[q];
      const double d = A.dens[s];
      if (d > rhot) {
        ok = true;
        const double xm = A.m[s];
        const double ux = xadd(wrapd(xsub(A.x[s], rx), A.Lx, A.hx), rx);
        const double uy = xadd(wrapd(xsub(A.y[s], ry), A.Ly, A.hy), ry);
        const double uz = xadd(wrapd(xsub(A.z[s], rz), A.Lz, A.hz), rz);
        t[0] = xm;
        t[1] = xmul(ux, xm);
        t[2] = xmul(uy, xm);
        t[3] = xmul(uz, xm);
        t[4] = xmul(xm, xadd(xadd(xmul(ux, ux), xmul(uy, uy)), xmul(uz, uz)));
        t[5] = d;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    const int cnt = __popc(m);
    if (ok) {
      const int slot = __popc(m & ((1u << lane) - 1));
#pragma unroll
      for (int c = 0; c < 6; ++c) st[slot * 6 + c] = t[c];
    }
    __syncwarp();
    if (lane < 6) {
#pragma unroll 8
      for (int l = 0; l < cnt; ++l) acc = xadd(acc, st[l * 6 + lane]);
    }
    imass += cnt;
    __syncwarp();
  }
  const double tm = __shfl_sync(0xffffffffu, acc, 0);
  const double px = __shfl_sync(0xffffffffu, acc, 1);
  const double py = __shfl_sync(0xffffffffu, acc, 2);
  const double pz = __shfl_sync(0xffffffffu, acc, 3);
  const double rs = __shfl_sync(0xffffffffu, acc, 4);
  const double dm = __shfl_sync(0xffffffffu, acc, 5);
  if (lane == 0) { G[0] = (double)imass; G[1] = tm; G[2] = px; G[3] = py; G[4] = pz; G[5] = rs; G[6] = dm; }
}

// posref of a colour: first particle above rhot of its first group (f90:2340-2344).
__device__ int32_t colour_posref(const TreeArgs& A, int32_t g0, double rhot) {
  for (int32_t q = A.goff[g0]; q < A.goff[g0 + 1]; ++q) {
    const int32_t s = A.gmem[q];
    if (A.dens[s] > rhot) return s;
  }
  set_err(A, 18, g0);  // cannot happen: the peak is above rhot
  return A.gpeak[g0];
}

// Fold a colour's group sums in GL order and apply the significance test
// (f90:1407-1466).  Exact record: C[0] mass_loc, C[1] mass_comp, C[2] densmax,
// C[3] densmoy, C[4] truemass, C[5..7] posg, C[8] radius, C[9] decision.
__device__ void colour_fold(const TreeArgs& A, int32_t c0, int32_t c1, double rhot, double* C) {
  double posg0 = 0, posg1 = 0, posg2 = 0, tm = 0, rsg = 0, dmg = 0, dmax = -1.0, dcm = -1.0;
  int32_t ml = 0, mc = 0;
  for (int32_t i = c0; i < c1; ++i) {
    const double* G = A.gs + 8 * (size_t)i;
    const int32_t g = A.GL[i];
    dmax = fmax(dmax, A.densg[g]);
    const int32_t mt = (int32_t)G[0];
    posg0 = xadd(posg0, G[2]);
    posg1 = xadd(posg1, G[3]);
    posg2 = xadd(posg2, G[4]);
    rsg = xadd(rsg, G[5]);
    ml += mt;
    tm = xadd(tm, G[1]);
    dmg = xadd(dmg, G[6]);
    mc = max(mc, mt);
    if (mt > 0) {
      const double dmt = xdiv(G[6], (double)mt);
      dcm = fmax(dcm, xdiv(dmt, xadd(1.0, xdiv(A.fudge, xsqrt((double)mt)))));
    }
  }
  const double p2 = xadd(xadd(xmul(posg0, posg0), xmul(posg1, posg1)), xmul(posg2, posg2));
  const double rsq = xsqrt(fabs(xdiv(xsub(xmul(tm, rsg), p2), xmul(tm, tm))));
  const double densmoy = xdiv(dmg, (double)ml);
  const bool ok = ml >= A.nmembthresh &&
                  (densmoy > xmul(rhot, xadd(1.0, xdiv(A.fudge, xsqrt((double)ml)))) || dcm > rhot) &&
                  dmax >= xmul(A.alphap, densmoy) && rsq >= A.epsilon;
  C[0] = (double)ml; C[1] = (double)mc; C[2] = dmax; C[3] = densmoy; C[4] = tm;
  C[5] = posg0; C[6] = posg1; C[7] = posg2; C[8] = rsq; C[9] = ok ? 1.0 : 0.0;
}

// Exact sums in the reference order for the colours flagged in cs[..][10].
template <int NT>
__device__ void exact_stats(const TreeArgs& A, SharedTask& T, double* s_terms) {
  const int tid = threadIdx.x;
  const double rhot = T.rhot;
  for (int32_t k = tid; k < T.ncomp; k += NT) {
    double* C = A.cs + 12 * (size_t)(T.a + k);
    if (C[10] == 0.0) continue;
    C[11] = (double)colour_posref(A, A.GL[A.cstart[T.a + k]], rhot);
  }
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  for (int32_t i = T.a + warp; warp < kTermWarps && i < T.b; i += kTermWarps) {  // large groups: a warp each
    const double* C = A.cs + 12 * (size_t)(T.a + A.compidx[i]);
    if (C[10] == 0.0) continue;
    const int32_t g = A.GL[i];
    if (A.goff[g + 1] - A.goff[g] <= kBigGroup) continue;
    const int32_t ref = (int32_t)C[11];
    group_sums_warp(A, g, rhot, A.x[ref], A.y[ref], A.z[ref], A.gs + 8 * (size_t)i, s_terms + warp * 32 * 6, lane);
  }
  for (int32_t i = T.a + tid; i < T.b; i += NT) {  // small groups: a thread each
    const double* C = A.cs + 12 * (size_t)(T.a + A.compidx[i]);
    if (C[10] == 0.0) continue;
    const int32_t g = A.GL[i];
    if (A.goff[g + 1] - A.goff[g] > kBigGroup) continue;
    const int32_t ref = (int32_t)C[11];
    group_sums_thread(A, g, rhot, A.x[ref], A.y[ref], A.z[ref], A.gs + 8 * (size_t)i);
  }
  __syncthreads();
  for (int32_t k = tid; k < T.ncomp; k += NT) {
    double* C = A.cs + 12 * (size_t)(T.a + k);
    if (C[10] == 0.0) continue;
    colour_fold(A, A.cstart[T.a + k], comp_end(A, T, k), rhot, C);
  }
  __syncthreads();
}

// ------------------------------------------------ root level on the whole grid
// The first iteration of the root task (rhot = rho_threshold over every group,
// f90:930-958) colours all groups at once; it runs here as grid-wide kernels
// instead of one block.  Colours are connected components of the saddle graph
// (every saddle exceeds rho_threshold), ordered by their smallest group id,
// groups inside a colour by id -- the reference's idgroup order.
// a warp per group: its lanes link the row's edges above rhot (the row's
// prefix), each undirected edge from its smaller group id
__global__ void root_union_kernel(const TreeArgs A, double rhot) {
  const int32_t g = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) + 1;
  const int lane = threadIdx.x & 31;
  if (g > A.ngroups) return;
  const int32_t e1 = A.soff[g];
  for (int32_t e = A.soff[g - 1] + lane; e < e1; e += 32) {
    if (!(A.srho[e] > rhot)) break;
    const int32_t h = A.sisad[e];
    if (h > g) uf_union(A.par, g - 1, h - 1);
  }
}

__global__ void root_roots_kernel(const TreeArgs A, int32_t* keys, int32_t* vals) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.ngroups) return;
  keys[i] = uf_find(A.par, i);
  vals[i] = i + 1;
}

// heads of colour runs (keys sorted) -> cstart via an exclusive scan of flags
__global__ void root_heads_kernel(const TreeArgs A, const int32_t* keys, int32_t* flag) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > A.ngroups) return;
  flag[i] = (i < A.ngroups && (i == 0 || keys[i] != keys[i - 1])) ? 1 : 0;
  if (i < A.ngroups) A.pos_of[A.GL[i]] = i;
}

__global__ void root_cstart_kernel(const TreeArgs A, const int32_t* flag, const int32_t* scan) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.ngroups) return;
  if (flag[i]) A.cstart[scan[i]] = i;
  A.compidx[i] = scan[i] + flag[i] - 1;
}

// anchor of every colour (peak of its first group) in cs[k][9..11]
__global__ void root_anchor_kernel(const TreeArgs A, int32_t ncomp) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncomp) return;
  const int32_t p0 = A.gpeak[A.GL[A.cstart[k]]];
  double* C = A.cs + 12 * (size_t)k;
  C[9] = A.x[p0];
  C[10] = A.y[p0];
  C[11] = A.z[p0];
}

__global__ void root_terms_kernel(const TreeArgs A, double rhot) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.ngroups) return;
  position_terms(A, i, rhot, A.cs + 12 * (size_t)A.compidx[i] + 9);
}

// a warp per colour: approximate sums and the three-state test
// (colours of more than kRootBig groups are left to root_decide_big_kernel)
constexpr int32_t kRootBig = 2048;
__global__ void root_decide_kernel(const TreeArgs A, int32_t ncomp, double rhot) {
  const int32_t k = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (k >= ncomp) return;
  const int32_t c1 = (k + 1 < ncomp) ? A.cstart[k + 1] : A.ngroups;
  if (c1 - A.cstart[k] > kRootBig) return;
  component_decide(A, A.cstart[k], c1, rhot, A.cs + 12 * (size_t)k, threadIdx.x & 31);
}

// a block per colour of more than kRootBig groups (blocks stride over the
// colours): the block folds the sums (the test's bounds hold for any order)
__global__ void __launch_bounds__(kNT) root_decide_big_kernel(const TreeArgs A, int32_t ncomp, double rhot) {
  __shared__ CompSums red[kNT / 32];
  for (int32_t k = blockIdx.x; k < ncomp; k += gridDim.x) {
    const int32_t c0 = A.cstart[k], c1 = (k + 1 < ncomp) ? A.cstart[k + 1] : A.ngroups;
    if (c1 - c0 <= kRootBig) continue;  // the same for every thread of the block
    const CompSums w = block_partial_sums<kNT>(A, c0, c1, threadIdx.x, kNT, red);
    if (threadIdx.x == 0)
      decide_from_sums(A, rhot, w.nl, w.nmax, w.dmax, w.S, w.M, w.Sx, w.Sy, w.Sz, w.Q, w.triB,
                       A.cs + 12 * (size_t)k);
  }
}

// one block per undecided colour: exact sums and the significance test
__global__ void __launch_bounds__(kNT) root_colour_kernel(const TreeArgs A, int32_t ncomp, double rhot) {
  __shared__ double s_terms[kNT / 32 * 32 * 6];
  __shared__ int32_t s_ref;
  const int32_t k = blockIdx.x;
  if (A.cs[12 * (size_t)k + 10] == 0.0) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t c0 = A.cstart[k], c1 = (k + 1 < ncomp) ? A.cstart[k + 1] : A.ngroups;
  if (tid == 0) s_ref = colour_posref(A, A.GL[c0], rhot);
  __syncthreads();
  const int32_t ref = s_ref;
  const double rx = A.x[ref], ry = A.y[ref], rz = A.z[ref];
  for (int32_t i = c0 + warp; i < c1; i += kNT / 32) {
    const int32_t g = A.GL[i];
    if (A.goff[g + 1] - A.goff[g] > kBigGroup)
      group_sums_warp(A, g, rhot, rx, ry, rz, A.gs + 8 * (size_t)i, s_terms + warp * 32 * 6, lane);
  }
  for (int32_t i = c0 + tid; i < c1; i += kNT) {
    const int32_t g = A.GL[i];
    if (A.goff[g + 1] - A.goff[g] <= kBigGroup) group_sums_thread(A, g, rhot, rx, ry, rz, A.gs + 8 * (size_t)i);
  }
  __syncthreads();
  if (tid == 0) colour_fold(A, c0, c1, rhot, A.cs + 12 * (size_t)k);
}

__global__ void root_okflag_kernel(const TreeArgs A, int32_t ncomp, int32_t* flag) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > ncomp) return;
  flag[k] = (k < ncomp && A.cs[12 * (size_t)k + 9] == 1.0) ? 1 : 0;
}

// level-1 nodes in colour order (reserve_nodes_block gives 1..nsisters),
// child tasks (f90:1484-1571), deepest node per group
__global__ void root_nodes_kernel(const TreeArgs A, int32_t ncomp, const int32_t* flag, const int32_t* rank,
                                  int32_t nsisters, double rhot) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncomp || !flag[k]) return;
  const double* C = A.cs + 12 * (size_t)k;
  const int32_t is = rank[k];
  const int32_t io = 1 + is;
  NodeRec& nd = A.node[io];
  nd.mother = 0;
  nd.densmax = C[2];
  nd.sister = is > 0 ? io - 1 : 0;
  nd.nsisters = nsisters;
  nd.mass = (int32_t)C[0];
  nd.rho_saddle = rhot;
  nd.level = 1;
  nd.firstchild = 0;
  if (nd.mass == 0) set_err(A, 15, io);
  const int32_t c0 = A.cstart[k], c1 = (k + 1 < ncomp) ? A.cstart[k + 1] : A.ngroups;
  push_task(A, Task{xmul(rhot, xadd(1.0, xdiv(A.fudge, xsqrt(C[1])))), io, c0, c1, 1});
  if (is == nsisters - 1) A.node[0].firstchild = io;  // f90:1540
}

__global__ void root_deepnode_kernel(const TreeArgs A, const int32_t* flag, const int32_t* rank) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.ngroups) return;
  const int32_t k = A.compidx[i];
  if (flag[k]) A.deepnode[A.GL[i]] = 1 + rank[k];
}

// order a wave's small tasks by decreasing size (long tasks start first, so
// the wave does not end on one late long task)
__global__ void task_keys_kernel(const Task* __restrict__ t, int32_t n, uint32_t* keys, int32_t* vals) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ~(uint32_t)(t[i].b - t[i].a);
  vals[i] = i;
}

__global__ void task_gather_kernel(const Task* __restrict__ in, const int32_t* __restrict__ idx, int32_t n,
                                   Task* __restrict__ out) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[idx[i]];
}

// Dynamic shared memory of a task block: reorder keys, warp-linked row
// positions (also approx_stats' list of large components) and the union-find
// parents of tasks of at most pcap groups, all scratch of a structural pass;
// the exact-sum staging (kTermWarps warps; also approx_stats' block fold),
// used only after the pass, lies over the same bytes.  What the block does
// not take stays L1, which the per-group loads of every level hit.
__host__ __device__ constexpr size_t wave_dyn_smem(int nt, int pcap) {
  const size_t pass = (size_t)nt * ipt_for(nt) * 4 + (size_t)kMaxBigRows * 4 + (size_t)pcap * 4;
  const size_t terms = (size_t)kTermWarps * 32 * 6 * 8;
  return pass > terms ? pass : terms;
}
// the block fold (over the reorder keys) must end before the large-component list
static_assert(kNT * kIPT * 4 >= (kNT / 32) * (int)sizeof(CompSums) &&
              kNTBig * 2 * 4 >= (kNTBig / 32) * (int)sizeof(CompSums) && kMaxBigRows >= kMaxBlockComps,
              "approx_stats scratch must fit the regions it borrows");

// Components whose member count above the threshold is below nmembthresh
// fail the mass test (f90:1459) at this level and at every later one: the
// count only falls as the threshold rises, and a later sub-component holds
// fewer members still.  They make no node, and they never rejoin another
// component (components only split as the threshold rises), so a task that
// continues drops them from its range at a level where a structural pass
// follows anyway.  The kept groups keep their relative order, hence the
// reference's colour order; the dropped groups keep the task's node as their
// deepest node, which is what the reference gives them.  Their largest peak
// density is kept for the continuation test, which counts every surviving
// group.  Worth it only when a good share of the range goes.
constexpr int32_t kMinPrune = 64;

template <int NT, class ScanT>
__device__ void prune_low_components(const TreeArgs& A, SharedTask& T, typename ScanT::TempStorage& scan_tmp) {
  const int tid = threadIdx.x;
  const int32_t a = T.a, b = T.b, ncomp = T.ncomp;
  const double thr = (double)A.nmembthresh;
  // new start of every kept component (cnt is free until the next pass)
  int32_t carry = 0;
  for (int32_t k0 = 0; k0 < ncomp; k0 += NT) {
    const int32_t k = k0 + tid;
    int32_t v = 0;
    if (k < ncomp && !(A.cs[12 * (size_t)(a + k)] < thr)) v = comp_end(A, T, k) - A.cstart[a + k];
    int32_t ex, tot;
    ScanT(scan_tmp).ExclusiveSum(v, ex, tot);
    __syncthreads();
    if (k < ncomp) A.cnt[a + k] = carry + ex;
    carry += tot;
  }
  const int32_t nkeep = carry, ndrop = b - a - carry;  // the same in every thread
  if (ndrop < kMinPrune || ndrop < (b - a) / 16) return;
  __syncthreads();
  unsigned long long mx = 0ull;  // peak densities are positive: their bits order like them
  for (int32_t i = a + tid; i < b; i += NT) {
    const int32_t k = A.compidx[i];
    const int32_t g = A.GL[i];
    if (A.cs[12 * (size_t)(a + k)] < thr)
      mx = max(mx, (unsigned long long)__double_as_longlong(A.densg[g]));
    else
      A.GL2[a + A.cnt[a + k] + (i - A.cstart[a + k])] = g;
  }
  if (mx) atomicMax(&T.pruned_max_bits, mx);
  __syncthreads();
  for (int32_t i = a + tid; i < a + nkeep; i += NT) {
    const int32_t g = A.GL2[i];
    A.GL[i] = g;
    A.pos_of[g] = i;
  }
  __syncthreads();
  if (tid == 0) {
    T.b = a + nkeep;
    T.nsurv = nkeep;
    T.npruned += ndrop;
    T.next_event = -DBL_MAX;  // components, starts and indices are rebuilt by the pass
  }
  __syncthreads();
}

// A follower CTA of a wide task's cluster: it waits for the leader's phases
// and runs its slice of each (positions a + rank * NT + tid, stride K * NT),
// reading the leader's task state and, when the task fits, its union-find
// array through distributed shared memory.  Each phase is a pair of cluster
// barriers, the pair the leader takes around its own slice; kPhExit ends the
// loop, and one last barrier tells the leader that its shared memory is read
// no more.
template <int NT, class SortT, class MaxScanT>
__device__ void follow_phases(const TreeArgs& A, SharedTask& T, int32_t* s_big, int32_t* s_par, CompSums* s_red,
                              int32_t* s_keys, typename SortT::TempStorage& sort_tmp,
                              typename MaxScanT::TempStorage& maxscan_tmp) {
  cg::cluster_group cl = cg::this_cluster();
  const int K = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x;
  SharedTask* LT = cl.map_shared_rank(&T, 0);
  int32_t* lpar = cl.map_shared_rank(s_par, 0);
  const int32_t gt = rank * NT + tid, gs = K * NT;
  for (;;) {
    cl.sync();  // a phase starts
    const int32_t code = LT->phase;
    if (code == kPhExit) break;
    const int32_t a = LT->a, b = LT->b;
    const double rhot = LT->rhot;
    const bool local = LT->plocal != 0;
    int32_t* par = local ? lpar : A.par;
    const int32_t poff = local ? a : 0;
    if (code == kPhUnion) {
      if (tid == 0) { T.nbig = 0; T.next_event = DBL_MAX; }
      __syncthreads();
      union_short_rows<NT>(A, a, b, poff, rhot, par, s_big, &T.nbig, &T.next_event, gt, gs);
      __syncthreads();
      union_long_rows<NT>(A, a, b, poff, par, s_big, T.nbig);
      if (tid == 0) LT->ev_part[rank] = T.next_event;
    } else if (code == kPhFind) {
      find_roots(A, a, b, poff, rhot, par, gt, gs);
    } else if (code == kPhTerms) {
      for (int32_t i = a + gt; i < b; i += gs)
        position_terms(A, i, rhot, A.cs + 12 * (size_t)(a + A.compidx[i]) + 9);
    } else if (code == kPhReorder) {
      reorder_count<NT>(A, a, b, poff, par, rank, K);
      cl.sync();  // every CTA's count is in (the leader takes this barrier too)
      reorder_range<NT, SortT, MaxScanT>(A, a, b, poff, par, rank, K, sort_tmp, maxscan_tmp, s_keys);
    } else if (code == kPhDecide) {
      decide_slice<NT>(A, a, b, LT->ncomp, rhot, rank, K, cl.map_shared_rank(s_big, 0), LT->fold_n, s_red,
                       cl.map_shared_rank(s_red + NT / 32, 0));
    }
    cl.sync();  // the phase ends
  }
  cl.sync();
}

template <int NT>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 4) tree_wave_kernel(TreeArgs A, const Task* __restrict__ tasks) {
  using SortT = cub::BlockRadixSort<int32_t, NT, ipt_for(NT), int32_t>;
  using ScanT = cub::BlockScan<int32_t, NT>;
  using MaxScanT = cub::BlockScan<int32_t, NT>;
  __shared__ typename SortT::TempStorage sort_tmp;
  __shared__ typename ScanT::TempStorage scan_tmp;
  __shared__ typename MaxScanT::TempStorage maxscan_tmp;
  extern __shared__ __align__(16) unsigned char wave_dyn[];
  double* s_terms = reinterpret_cast<double*>(wave_dyn);  // over s_keys, s_big, s_par
  int32_t* s_keys = reinterpret_cast<int32_t*>(wave_dyn);
  int32_t* s_big = s_keys + NT * ipt_for(NT);
  int32_t* s_par = s_big + kMaxBigRows;
  __shared__ SharedTask T;
  __shared__ long long s_clk[6];  // structural, approx, exact cycles; levels; structural passes; max ncomp
  __shared__ long long s_ph[kProfPhases];  // cycles per phase of the structural passes and statistics
  const int tid = threadIdx.x;
  // wide tasks: CTA 0 of each cluster leads, the others serve its phases
  int K = 1;
  if (NT >= 1024) {
    K = cluster_ctas();
    if (cg::this_cluster().block_rank() != 0) {
      follow_phases<NT, SortT, MaxScanT>(A, T, s_big, s_par, reinterpret_cast<CompSums*>(s_terms), s_keys, sort_tmp,
                                         maxscan_tmp);
      return;
    }
  }
  if (tid == 0) T.cont = tasks[blockIdx.x / K];
  // A block runs its task and then, when the task branches, one of the new
  // children itself (the one with the most groups) instead of leaving it to
  // the next wave: the longest chains of the tree no longer wait at every
  // wave boundary.  The children's work is independent, so this changes
  // only the schedule, not the nodes (their ids are renumbered at the end).
  for (;;) {
  long long t_start = clock64();
  if (tid < 6) s_clk[tid] = 0;
  if (tid < kProfPhases) s_ph[tid] = 0;
  if (tid == 0) {
    const Task t = T.cont;
    T.rhot = t.rhot; T.inode = t.inode; T.a = t.a; T.b = t.b; T.level = t.level;
    T.groups0 = t.b - t.a;
    T.next_event = -DBL_MAX;  // force a structural pass first
    T.nsurv = 0;
    T.ncomp = 0;
    T.done = 0;
    T.iters = 0;
    T.has_cont = 0;
    T.npruned = 0;
    T.pruned_max_bits = 0ull;
  }
  __syncthreads();
  while (true) {
    // every thread must take the same branch: snapshot the test before thread 0
    // rewrites next_event inside the pass
    const bool restructure = T.rhot >= T.next_event;
    __syncthreads();
    long long c0 = clock64();
    if (restructure) {
      structural_pass<NT, SortT, ScanT, MaxScanT>(A, T, sort_tmp, scan_tmp, maxscan_tmp, s_keys, s_big, s_par, s_ph);
      if (tid == 0) { atomicAdd(&A.stats[7], 1ULL); s_clk[4] += 1; }
    }
    long long c1 = clock64();
    if (tid == 0) { s_clk[0] += c1 - c0; s_clk[3] += 1; s_clk[5] = max(s_clk[5], (long long)T.ncomp); }
    if (T.nsurv == 0) {  // all groups below the threshold (f90:1348-1351 prints, then ends with no colour)
      if (tid == 0) A.node[T.inode].firstchild = 0;
      break;
    }
    approx_stats<NT>(A, T, s_ph, s_big, reinterpret_cast<CompSums*>(s_terms));
    if (tid == 0) {
      s_clk[1] += clock64() - c1;
      T.nexact = 0;
      T.nsisters = 0;
      T.kk = -1;
    }
    __syncthreads();
    for (int32_t k = tid; k < T.ncomp; k += NT)
      if (A.cs[12 * (size_t)(T.a + k) + 10] != 0.0) atomicAdd(&T.nexact, 1);
    __syncthreads();
    if (T.nexact > 0) {  // undecided tests: exact sums in the reference order
      long long c2 = clock64();
      exact_stats<NT>(A, T, s_terms);
      if (tid == 0) { s_clk[2] += clock64() - c2; atomicAdd(&A.stats[4], 1ULL); }
    }
    for (int32_t k = tid; k < T.ncomp; k += NT) {
      if (A.cs[12 * (size_t)(T.a + k) + 9] == 1.0) {
        atomicAdd(&T.nsisters, 1);
        T.kk = k;  // the significant component when there is exactly one
      }
    }
    __syncthreads();
    const int32_t ns = T.nsisters;
    if (ns == 0) {
      if (tid == 0) A.node[T.inode].firstchild = 0;
      break;
    }
    if (ns == 1) {
      if (tid == 0) {
        const double mc = A.cs[12 * (size_t)(T.a + T.kk) + 1];
        const double rnew = xmul(T.rhot, xadd(1.0, xdiv(A.fudge, xsqrt(mc))));
        // more than one surviving group (f90:1595), those pruned from the range included
        if (T.nsurv > 1 || __longlong_as_double((long long)T.pruned_max_bits) > T.rhot) {
          T.rhot = rnew;
          T.done = 0;
        } else {
          A.node[T.inode].firstchild = 0;
          T.done = 1;
        }
        T.iters += 1;
        if (T.iters > kMaxTaskLevels) { set_err(A, 12, T.inode); T.done = 1; }
      }
      __syncthreads();
      if (T.done) break;
      // the next level restructures anyway: drop what can never be a node
      if (T.rhot >= T.next_event) prune_low_components<NT, ScanT>(A, T, scan_tmp);
      continue;
    }
    // ---- branching (f90:1484-1571): one node per significant component in
    // colour order.  Counts, densmax and the child thresholds are exact here;
    // truemass, position, radius and mean density are formed after the
    // waves (node_sums), in the reference's summation order.
    if (tid == 0) {
      const int32_t first = atomicAdd(A.nnodes, ns) + 1;
      if (first + ns - 1 > A.nnodesmax) set_err(A, 14, first);
      T.inode1 = first;
      T.done = (first + ns - 1 > A.nnodesmax);
    }
    __syncthreads();
    if (T.done) break;
    // the child this block continues: the significant component with the
    // most groups (ties: the first), packed as (groups, ~index) for atomicMax
    if (tid == 0) T.best = 0ull;
    __syncthreads();
    for (int32_t k = tid; k < T.ncomp; k += NT) {
      if (A.cs[12 * (size_t)(T.a + k) + 9] == 1.0) {
        const unsigned long long ng_k = (unsigned long long)(comp_end(A, T, k) - A.cstart[T.a + k]);
        atomicMax(&T.best, (ng_k << 32) | (unsigned long long)(0xffffffffu - (unsigned)k));
      }
    }
    __syncthreads();
    const int32_t kc = (int32_t)(0xffffffffu - (unsigned)(T.best & 0xffffffffull));
    {
      int32_t carry = 0;
      for (int32_t k0 = 0; k0 < T.ncomp; k0 += NT) {
        const int32_t k = k0 + tid;
        const double* C = A.cs + 12 * (size_t)(T.a + k);
        const int sig = (k < T.ncomp && C[9] == 1.0) ? 1 : 0;
        int32_t ex, tot;
        ScanT(scan_tmp).ExclusiveSum(sig, ex, tot);
        __syncthreads();
        if (k < T.ncomp) A.cnt[T.a + k] = sig ? T.inode1 + carry + ex : 0;  // node of component k
        if (sig) {
          const int32_t is = carry + ex;
          const int32_t io = T.inode1 + is;
          NodeRec& nd = A.node[io];
          nd.mother = T.inode;
          nd.densmax = C[2];
          nd.sister = is > 0 ? io - 1 : 0;
          nd.nsisters = ns;
          nd.mass = (int32_t)C[0];
          nd.rho_saddle = T.rhot;
          nd.level = T.level + 1;
          nd.firstchild = 0;
          if (nd.mass == 0) set_err(A, 15, io);  // f90:1506-1510
          // child task (f90:1543-1556)
          const double rc = xmul(T.rhot, xadd(1.0, xdiv(A.fudge, xsqrt(C[1]))));
          const Task child{rc, io, A.cstart[T.a + k], comp_end(A, T, k), T.level + 1};
          if (k == kc) {
            T.cont = child;
            T.has_cont = 1;
          } else {
            // queued only after this task's last reads of its range (below):
            // a queued child may start at once in another block
            double* Cw = A.cs + 12 * (size_t)(T.a + k);
            Cw[3] = child.rhot;
            Cw[4] = (double)child.inode;
            Cw[5] = (double)child.a;
            Cw[6] = (double)child.b;
            Cw[7] = (double)child.level;
          }
        }
        carry += tot;
      }
    }
    if (tid == 0) A.node[T.inode].firstchild = T.inode1 + ns - 1;  // f90:1540
    __syncthreads();
    // deepest node per group
    for (int32_t i = T.a + tid; i < T.b; i += NT) {
      const int32_t io = A.cnt[T.a + A.compidx[i]];
      if (io > 0) A.deepnode[A.GL[i]] = io;
    }
    __syncthreads();
    for (int32_t k = tid; k < T.ncomp; k += NT) {
      const double* C = A.cs + 12 * (size_t)(T.a + k);
      if (C[9] == 1.0 && k != kc)
        push_task(A, Task{C[3], (int32_t)C[4], (int32_t)C[5], (int32_t)C[6], (int32_t)C[7]});
    }
    break;
  }
  if (tid == 0) {
    // [0..2] cycles structural/approx/exact, [3] levels, [4] undecided-test
    // exact passes, [5] max levels of one task, [6] max cycles of one task
    atomicAdd(&A.stats[0], (unsigned long long)s_clk[0]);
    atomicAdd(&A.stats[1], (unsigned long long)s_clk[1]);
    atomicAdd(&A.stats[2], (unsigned long long)s_clk[2]);
    atomicAdd(&A.stats[3], (unsigned long long)s_clk[3]);
    atomicMax(&A.stats[5], (unsigned long long)s_clk[3]);
    atomicMax(&A.stats[6], (unsigned long long)(s_clk[0] + s_clk[1] + s_clk[2]));
    if (A.tprof) {
      long long* r = A.tprof + kProfRow * (size_t)T.inode;
      r[0] = T.groups0;       // groups in the task's range
      r[1] = s_clk[3];        // levels
      r[2] = s_clk[4];        // structural passes
      r[3] = s_clk[0];        // cycles: structural
      r[4] = s_clk[1];        // cycles: approximate statistics
      r[5] = s_clk[2];        // cycles: exact sums
      r[6] = clock64() - t_start;  // cycles: whole task
      r[7] = s_clk[5];        // largest component count at one level
      for (int k = 0; k < kProfPhases; ++k) r[8 + k] = s_ph[k];  // phases
      r[24] = A.node[T.inode].mother;  // creation-time node id of the mother
      r[25] = T.npruned;               // groups dropped below the member threshold
    }
  }
  // no child to continue: take a task that another block queued for the next
  // wave (wide blocks take wide tasks first, then narrow ones)
  if (tid == 0 && !T.has_cont) {
    Task t;
    if ((NT >= kNTBig && take_task(A, true, t)) || take_task(A, false, t)) {
      T.cont = t;
      T.has_cont = 1;
    }
  }
  __syncthreads();
  const bool more = T.has_cont != 0;
  __syncthreads();  // thread 0 rewrites T for the next task
  if (!more) break;
  }
  if (K > 1) {  // release the followers, then wait until they no longer read T
    if (tid == 0) T.phase = kPhExit;
    cg::this_cluster().sync();
    cg::this_cluster().sync();
  }
}

// ------------------------------------------------------------- node sums
// truemass, position, radius and mean density of every created node, in the
// reference's order: treat_particles (f90:2317-2401) per group at the node's
// creation threshold, posref from the first group, then the fold over the
// colour's groups in colour order (f90:1407-1432), which is ascending group
// id (a colour's groups keep their relative order through every reorder).
// A node's groups are the groups whose deepest node lies in its subtree, so
// every (node, group) pair is independent: all of them are summed at once
// after the waves instead of inside the task that created the node.

// pairs per group: the depth of its deepest node; cnt[ng] = 0 closes the scan
__global__ void pair_count_kernel(const TreeArgs A, int32_t nn, int32_t* cnt) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > A.ngroups + 1) return;
  if (g == A.ngroups + 1) { cnt[A.ngroups] = 0; return; }
  int32_t d = 0, N = A.deepnode[g];
  while (N > 0 && d <= nn) {
    ++d;
    N = A.node[N].mother;
  }
  if (d > nn) { set_err(A, 19, g); d = 0; }  // a cycle in the mother links
  cnt[g - 1] = d;
}

__global__ void pair_emit_kernel(const TreeArgs A, const int32_t* __restrict__ off,
                                 unsigned long long* __restrict__ keys) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (g > A.ngroups) return;
  int32_t p = off[g - 1];
  const int32_t p1 = off[g];
  for (int32_t N = A.deepnode[g]; N > 0 && p < p1; N = A.node[N].mother)
    keys[p++] = ((unsigned long long)N << 32) | (unsigned)g;
}

// pair range [nstart[N], nend[N]) of every node in the sorted pair keys
__global__ void node_range_kernel(const unsigned long long* __restrict__ keys, int64_t np, int32_t* nstart,
                                  int32_t* nend) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int32_t N = (int32_t)(keys[p] >> 32);
  if (p == 0 || (int32_t)(keys[p - 1] >> 32) != N) nstart[N] = (int32_t)p;
  if (p == np - 1 || (int32_t)(keys[p + 1] >> 32) != N) nend[N] = (int32_t)(p + 1);
}

// posref of every node (f90:2340-2344): the first member, in list order, of
// its first group above its threshold; a warp per node
__global__ void node_posref_kernel(const TreeArgs A, int32_t nn, const unsigned long long* __restrict__ keys,
                                   const int32_t* __restrict__ nstart, const int32_t* __restrict__ nend,
                                   int32_t* __restrict__ posref) {
  const int32_t N = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) + 1;
  const int lane = threadIdx.x & 31;
  if (N > nn) return;
  if (nstart[N] >= nend[N]) {
    if (lane == 0) { set_err(A, 20, N); posref[N] = 0; }
    return;
  }
  const int32_t g0 = (int32_t)(keys[nstart[N]] & 0xffffffffu);
  const double rhot = A.node[N].rho_saddle;
  const int32_t q1 = A.goff[g0 + 1];
  for (int32_t base = A.goff[g0]; base < q1; base += 32) {
    const int32_t q = base + lane;
    const int32_t s = (q < q1) ? A.gmem[q] : -1;
    const bool ok = (s >= 0) && A.dens[s] > rhot;
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (m) {
      if (lane == __ffs(m) - 1) posref[N] = s;
      return;
    }
  }
  if (lane == 0) { set_err(A, 18, g0); posref[N] = A.gpeak[g0]; }  // cannot happen: the peak is above
}

// per (node, group) pair sums, a thread per pair of a small group
__global__ void pair_sums_kernel(const TreeArgs A, const unsigned long long* __restrict__ keys, int64_t np,
                                 const int32_t* __restrict__ posref, double* __restrict__ ps) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int32_t N = (int32_t)(keys[p] >> 32), g = (int32_t)(keys[p] & 0xffffffffu);
  if (A.goff[g + 1] - A.goff[g] > kBigGroup) return;
  const int32_t ref = posref[N];
  group_sums_thread(A, g, A.node[N].rho_saddle, A.x[ref], A.y[ref], A.z[ref], ps + 8 * p);
}

// the same for pairs of large groups, a warp per pair
__global__ void __launch_bounds__(256) pair_sums_warp_kernel(const TreeArgs A,
                                                             const unsigned long long* __restrict__ keys,
                                                             int64_t np, const int32_t* __restrict__ posref,
                                                             double* __restrict__ ps) {
  __shared__ double st[8][32 * 6];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * 8;
  for (int64_t p = (int64_t)blockIdx.x * 8 + wib; p < np; p += nw) {
    const int32_t N = (int32_t)(keys[p] >> 32), g = (int32_t)(keys[p] & 0xffffffffu);
    if (A.goff[g + 1] - A.goff[g] <= kBigGroup) continue;
    const int32_t ref = posref[N];
    group_sums_warp(A, g, A.node[N].rho_saddle, A.x[ref], A.y[ref], A.z[ref], ps + 8 * p, st[wib], lane);
  }
}

// fold every node's pair sums in ascending group id and write its fields
// (f90:1407-1432, 1511-1538).  A warp per node: the lanes stage 32 pairs at
// a time in shared memory and lanes 0..5 each run one of the six sequential
// sums (lane 6 the member count) -- the fold's additions in the fold's order.
__global__ void __launch_bounds__(256) node_fold_kernel(const TreeArgs A, int32_t nn,
                                                        const int32_t* __restrict__ nstart,
                                                        const int32_t* __restrict__ nend,
                                                        const double* __restrict__ ps) {
  __shared__ double st[8][32 * 7];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int32_t N = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) + 1;
  if (N > nn) return;
  // pair-sum columns of the six chains: posg(3), rsquare, truemass, densmoy
  const int col = (lane == 0) ? 2 : (lane == 1) ? 3 : (lane == 2) ? 4 : (lane == 3) ? 5 : (lane == 4) ? 1 : 6;
  double acc = 0.0;
  int32_t ml = 0;
  const int32_t p0 = nstart[N], p1 = nend[N];
  // the next chunk's pair sums are loaded into registers while the current
  // chunk is folded (the folds are sequential: their order is the reference's)
  double nx[7];
  if (p0 + lane < p1) {
    const double* G = ps + 8 * (size_t)(p0 + lane);
#pragma unroll
    for (int c = 0; c < 7; ++c) nx[c] = G[c];
  }
  for (int32_t base = p0; base < p1; base += 32) {
    if (base + lane < p1) {
#pragma unroll
      for (int c = 0; c < 7; ++c) st[wib][lane * 7 + c] = nx[c];
    }
    __syncwarp();
    const int32_t pn = base + 32 + lane;
    if (pn < p1) {
      const double* G = ps + 8 * (size_t)pn;
#pragma unroll
      for (int c = 0; c < 7; ++c) nx[c] = G[c];
    }
    const int cnt = min(32, p1 - base);
    if (lane < 6) {
#pragma unroll 8
      for (int l = 0; l < cnt; ++l) acc = xadd(acc, st[wib][l * 7 + col]);
    } else if (lane == 6) {
      for (int l = 0; l < cnt; ++l) ml += (int32_t)st[wib][l * 7];
    }
    __syncwarp();
  }
  const double posg0 = __shfl_sync(0xffffffffu, acc, 0);
  const double posg1 = __shfl_sync(0xffffffffu, acc, 1);
  const double posg2 = __shfl_sync(0xffffffffu, acc, 2);
  const double rsg = __shfl_sync(0xffffffffu, acc, 3);
  const double tm = __shfl_sync(0xffffffffu, acc, 4);
  const double dmg = __shfl_sync(0xffffffffu, acc, 5);
  ml = __shfl_sync(0xffffffffu, ml, 6);
  if (lane != 0) return;
  NodeRec& nd = A.node[N];
  if (ml != nd.mass) set_err(A, 21, N);
  const double p2 = xadd(xadd(xmul(posg0, posg0), xmul(posg1, posg1)), xmul(posg2, posg2));
  nd.radius = xsqrt(fabs(xdiv(xsub(xmul(tm, rsg), p2), xmul(tm, tm))));
  nd.density = xdiv(dmg, (double)ml);
  nd.truemass = tm;
  double pf0 = xdiv(posg0, tm), pf1 = xdiv(posg1, tm), pf2 = xdiv(posg2, tm);
  if (pf0 >= A.hx) pf0 = xsub(pf0, A.Lx); else if (pf0 < -A.hx) pf0 = xadd(pf0, A.Lx);
  if (pf1 >= A.hy) pf1 = xsub(pf1, A.Ly); else if (pf1 < -A.hy) pf1 = xadd(pf1, A.Ly);
  if (pf2 >= A.hz) pf2 = xsub(pf2, A.Lz); else if (pf2 < -A.hz) pf2 = xadd(pf2, A.Lz);
  nd.pos[0] = pf0;
  nd.pos[1] = pf1;
  nd.pos[2] = pf2;
}

// ------------------------------------------------------- setup / membership / order
__global__ void init_groups_kernel(const TreeArgs A) {
  const int32_t ng = A.ngroups;
  int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) {
    A.GL[i] = i + 1;
    A.pos_of[i + 1] = i;
    A.gcur[i + 1] = A.goff[i + 2] - A.goff[i + 1];
    A.ecur[i + 1] = A.soff[i + 1] - A.soff[i];
  }
  if (i <= ng) A.deepnode[i] = 0;
}

// per-group members in decreasing density: gather keys for the segmented sort
__global__ void gather_member_rho(const int32_t* __restrict__ gmem, const double* __restrict__ dens, int64_t m,
                                  double* __restrict__ rho) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) rho[i] = dens[gmem[i]];
}

// Members by decreasing density inside each group with one radix sort of all
// members: key = group (ascending: the groups' member ranges stay where they
// are), then the density rounded down to float, decreasing (rounding is
// monotone, and non-negative floats order like their bits).  Members whose
// keys are equal (densities within a float step) are then put in exact order
// by member_fix_runs_kernel.  Exactly equal densities may end in any order:
// counts above a threshold and the bounded running sums do not depend on it.
__global__ void member_rho_keys_kernel(const int32_t* __restrict__ gmem, const int32_t* __restrict__ group,
                                       const double* __restrict__ dens, int64_t m,
                                       unsigned long long* __restrict__ key) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int32_t s = gmem[i];
  key[i] = ((unsigned long long)(uint32_t)group[s] << 32) |
           (unsigned long long)(0xffffffffu - __float_as_uint(__double2float_rd(dens[s])));
}

constexpr int kMaxKeyRun = 64;  // longer runs of equal keys (contrived inputs): the segmented sort instead

// a thread per run of equal keys (of at most kMaxKeyRun members): insertion
// sort by exact density, decreasing; a longer run raises *flag
__global__ void member_fix_runs_kernel(const unsigned long long* __restrict__ key, int64_t m, int32_t* __restrict__ mem,
                                       double* __restrict__ rho, int32_t* __restrict__ flag) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i + 1 >= m || key[i + 1] != key[i] || (i > 0 && key[i - 1] == key[i])) return;
  int64_t e = i + 2;
  while (e < m && key[e] == key[i]) {
    if (e - i >= kMaxKeyRun) { atomicExch(flag, 1); return; }
    ++e;
  }
  for (int64_t j = i + 1; j < e; ++j) {
    const double r = rho[j];
    const int32_t v = mem[j];
    int64_t k = j;
    while (k > i && rho[k - 1] < r) {
      rho[k] = rho[k - 1];
      mem[k] = mem[k - 1];
      --k;
    }
    rho[k] = r;
    mem[k] = v;
  }
}

// running sums per group (one warp per group) in decreasing-density order
__global__ void prefix_moments_kernel(const int32_t* __restrict__ goff, int32_t ng,
                                      const int32_t* __restrict__ mem_rho_order, const double* __restrict__ rdesc,
                                      const int32_t* __restrict__ gpeak, const double* __restrict__ x,
                                      const double* __restrict__ y, const double* __restrict__ z,
                                      const double* __restrict__ mm, double Lx, double Ly, double Lz,
                                      double hx, double hy, double hz, double* __restrict__ pref) {
  const int lane = threadIdx.x & 31;
  const int32_t g = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) + 1;
  if (g > ng) return;
  const int32_t p = gpeak[g];
  const double ax = x[p], ay = y[p], az = z[p];
  double c[6] = {0, 0, 0, 0, 0, 0};
  for (int32_t base = goff[g]; base < goff[g + 1]; base += 32) {
    const int32_t q = base + lane;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (q < goff[g + 1]) {
      const int32_t s = mem_rho_order[q];
      const double w = mm[s];
      double dx = wrapd(x[s] - ax, Lx, hx), dy = wrapd(y[s] - ay, Ly, hy), dz = wrapd(z[s] - az, Lz, hz);
      v[0] = rdesc[q]; v[1] = w; v[2] = w * dx; v[3] = w * dy; v[4] = w * dz;
      v[5] = w * (dx * dx + dy * dy + dz * dz);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        double up = __shfl_up_sync(0xffffffffu, v[t], o);
        if (lane >= o) v[t] += up;
      }
    }
    if (q < goff[g + 1]) {
#pragma unroll
      for (int t = 0; t < 6; ++t) pref[6 * (size_t)q + t] = c[t] + v[t];
    }
#pragma unroll
    for (int t = 0; t < 6; ++t) c[t] += __shfl_sync(0xffffffffu, v[t], 31);
  }
}

__global__ void membership_kernel(const int32_t* __restrict__ group, const double* __restrict__ dens,
                                  const int32_t* __restrict__ orig, const int32_t* __restrict__ deepnode,
                                  const NodeRec* __restrict__ node, int64_t n, int32_t* __restrict__ liste,
                                  int32_t* err) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t g = group[s];
  int32_t nd = 0;
  if (g > 0) {
    nd = deepnode[g];
    const double d = dens[s];
    int guard = 0;
    while (nd > 0 && !(d > node[nd].rho_saddle)) {
      nd = node[nd].mother;
      if (++guard > 100000) { atomicExch(err, 16); nd = 0; break; }
    }
  }
  liste[orig[s]] = nd;
}

struct NodeLess {
  const NodeRec* node;
  __device__ bool operator()(int32_t ia, int32_t ib) const {
    // node_precedes (f90:1083-1131)
    const NodeRec& a = node[ia];
    const NodeRec& b = node[ib];
    if (a.level != b.level) return a.level < b.level;
    if (a.truemass != b.truemass) return a.truemass > b.truemass;
    if (a.mass != b.mass) return a.mass > b.mass;
    if (a.densmax != b.densmax) return a.densmax > b.densmax;
    if (a.density != b.density) return a.density > b.density;
    if (a.rho_saddle != b.rho_saddle) return a.rho_saddle > b.rho_saddle;
    for (int k = 0; k < 3; ++k)
      if (a.pos[k] != b.pos[k]) return a.pos[k] < b.pos[k];
    return ia < ib;
  }
};

__global__ void iota_kernel(int32_t* v, int32_t n, int32_t base) {
  int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i + base;
}

__global__ void old_to_new_kernel(const int32_t* __restrict__ new_to_old, int32_t nn, int32_t* __restrict__ o2n) {
  int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nn) o2n[new_to_old[k]] = k + 1;
  if (k == 0) o2n[0] = 0;
}

__global__ void tables_kernel(const NodeRec* __restrict__ node, const int32_t* __restrict__ new_to_old,
                              const int32_t* __restrict__ o2n, int32_t nn, double* __restrict__ rt,
                              int32_t* __restrict__ it) {
  int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nn) return;
  const NodeRec& d = node[new_to_old[k]];
  double* r = rt + 8 * (size_t)k;
  r[0] = d.rho_saddle; r[1] = d.density; r[2] = d.densmax; r[3] = d.radius; r[4] = d.truemass;
  r[5] = d.pos[0]; r[6] = d.pos[1]; r[7] = d.pos[2];
  int32_t* t = it + 6 * (size_t)k;
  t[0] = d.mass; t[1] = d.level;
  t[2] = d.mother > 0 ? o2n[d.mother] : d.mother;
  t[3] = d.firstchild > 0 ? o2n[d.firstchild] : d.firstchild;
  t[4] = d.nsisters;
  t[5] = d.sister > 0 ? o2n[d.sister] : d.sister;
}

__global__ void remap_liste_kernel(int32_t* __restrict__ liste, int64_t n, const int32_t* __restrict__ o2n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t v = liste[i];
  if (v > 0) liste[i] = o2n[v];
}

int stage_nodes(Engine& E) {
  const int64_t n = E.n;
  const Params& P = E.prm;
  cudaStream_t st = E.stream;
  const int32_t ng = E.ngroups;
  const int T = 256;
  AHOP_CUDA_TRY(E.d_liste.ensure(n * 4));
  E.nnodes = 0;
  for (int k = 11; k <= 13; ++k) AHOP_CUDA_TRY(cudaEventRecord(E.ev[k], st));
  if (ng == 0) {
    AHOP_CUDA_TRY(cudaMemsetAsync(E.d_liste.p, 0, n * 4, st));
    return AHOP_OK;
  }
  const int64_t nact = E.nactive;
  const int32_t nnodesmax = 2 * ng;  // f90:906
  // ---- per-group members by decreasing density + running sums
  AHOP_CUDA_TRY(E.d_gmem_rho.ensure(nact * 8 * 2 + 8));
  AHOP_CUDA_TRY(E.d_gmem_rho_pref.ensure(nact * 8 * 6 + 8));
  AHOP_CUDA_TRY(E.d_sad_val2.ensure((size_t)nact * 4 + 8));  // member order by density
  double* rho_idx = E.d_gmem_rho.as<double>();        // densities in particle-index order
  double* rdesc = E.d_gmem_rho.as<double>() + nact;   // sorted decreasing
  int32_t* mem_rho = reinterpret_cast<int32_t*>(E.d_sad_val2.p);
  bool sorted = false;
  if (nact > 0) {
    // one radix sort of (group, density rounded to float), then exact order
    // inside runs of equal keys (member_rho_keys_kernel)
    AHOP_CUDA_TRY(E.d_key.ensure((size_t)nact * 8));
    AHOP_CUDA_TRY(E.d_key2.ensure((size_t)nact * 8));
    unsigned long long* k0 = E.d_key.as<unsigned long long>();
    unsigned long long* k1 = E.d_key2.as<unsigned long long>();
    const unsigned gm = (unsigned)((nact + T - 1) / T);
    E.launches++;
    member_rho_keys_kernel<<<gm, T, 0, st>>>(E.d_gmem.as<int32_t>(), E.d_group.as<int32_t>(), E.d_dens.as<double>(),
                                             nact, k0);
    AHOP_CUDA_TRY(cudaGetLastError());
    int end_bit = 32;
    while (end_bit < 64 && (1LL << (end_bit - 32)) <= (int64_t)ng) ++end_bit;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, k0, k1, E.d_gmem.as<int32_t>(), mem_rho, (int)nact, 0, end_bit, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, tmp, k0, k1, E.d_gmem.as<int32_t>(), mem_rho,
                                                  (int)nact, 0, end_bit, st));
    E.launches += 2;
    gather_member_rho<<<gm, T, 0, st>>>(mem_rho, E.d_dens.as<double>(), nact, rdesc);
    int32_t* fl = reinterpret_cast<int32_t*>(k0);  // the unsorted keys are no longer needed
    AHOP_CUDA_TRY(cudaMemsetAsync(fl, 0, 4, st));
    member_fix_runs_kernel<<<gm, T, 0, st>>>(k1, nact, mem_rho, rdesc, fl);
    AHOP_CUDA_TRY(cudaGetLastError());
    int32_t* hf = reinterpret_cast<int32_t*>(E.h_scalars);
    AHOP_CUDA_TRY(cudaMemcpyAsync(hf, fl, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    sorted = hf[0] == 0;
  }
  if (!sorted && nact > 0) {  // a run of more than kMaxKeyRun equal keys: sort the groups' members exactly
    E.launches++;
    gather_member_rho<<<(unsigned)((nact + T - 1) / T), T, 0, st>>>(E.d_gmem.as<int32_t>(), E.d_dens.as<double>(),
                                                                    nact, rho_idx);
    AHOP_CUDA_TRY(cudaGetLastError());
    size_t tmp = 0;
    cub::DeviceSegmentedSort::SortPairsDescending(nullptr, tmp, rho_idx, rdesc, E.d_gmem.as<int32_t>(), mem_rho,
                                                  (int)nact, ng, E.d_goff.as<int32_t>() + 1,
                                                  E.d_goff.as<int32_t>() + 2, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceSegmentedSort::SortPairsDescending(E.d_cub.p, tmp, rho_idx, rdesc,
                                                                E.d_gmem.as<int32_t>(), mem_rho, (int)nact, ng,
                                                                E.d_goff.as<int32_t>() + 1,
                                                                E.d_goff.as<int32_t>() + 2, st));
  }
  {
    int64_t threads = (int64_t)ng * 32;
    E.launches++;
    prefix_moments_kernel<<<(unsigned)((threads + T - 1) / T), T, 0, st>>>(
        E.d_goff.as<int32_t>(), ng, mem_rho, rdesc, E.d_gpeak.as<int32_t>(), E.d_x.as<double>(),
        E.d_y.as<double>(), E.d_z.as<double>(), E.d_m.as<double>(), P.xlong, P.ylong, P.zlong, P.xlongs2,
        P.ylongs2, P.zlongs2, E.d_gmem_rho_pref.as<double>());
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  // ---- maximum spanning forest of the saddle graph: the colours at every
  // threshold are its components, so the tree links only its edges
  {
    const int rc = build_saddle_forest(E);
    if (rc) return rc;
  }
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[11], st));
  // ---- tree scratch
  const size_t G = (size_t)ng + 1;
  const size_t bytes_i = G * 4;
  // every sub-array starts on a 256-byte boundary: size the buffer with the rounding
  auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t need = r256(bytes_i) * 12 + r256(bytes_i * kClusterCtas) * 2 + r256(G * 8 * 8) + r256(G * 12 * 8) +
                      r256((size_t)(nnodesmax + 1) * sizeof(Task)) * 4 + r256((size_t)(nnodesmax + 1) * 4) * 4;
  AHOP_CUDA_TRY(E.d_tree_scratch.ensure(need));
  char* p = static_cast<char*>(E.d_tree_scratch.p);
  auto take = [&](size_t b) { char* q = p; p += (b + 255) & ~size_t(255); return q; };
  TreeArgs A;
  A.GL = reinterpret_cast<int32_t*>(take(bytes_i));
  A.GL2 = reinterpret_cast<int32_t*>(take(bytes_i));
  A.pos_of = reinterpret_cast<int32_t*>(take(bytes_i));
  A.par = reinterpret_cast<int32_t*>(take(bytes_i));
  A.cnt = reinterpret_cast<int32_t*>(take(bytes_i));
  A.run = reinterpret_cast<int32_t*>(take(bytes_i));
  A.cstart = reinterpret_cast<int32_t*>(take(bytes_i));
  A.compidx = reinterpret_cast<int32_t*>(take(bytes_i));
  A.gn = reinterpret_cast<int32_t*>(take(bytes_i));
  A.deepnode = reinterpret_cast<int32_t*>(take(bytes_i));
  A.gcur = reinterpret_cast<int32_t*>(take(bytes_i));
  A.ecur = reinterpret_cast<int32_t*>(take(bytes_i));
  A.rcnt = reinterpret_cast<int32_t*>(take(bytes_i * kClusterCtas));
  A.rrun = reinterpret_cast<int32_t*>(take(bytes_i * kClusterCtas));
  A.gs = reinterpret_cast<double*>(take(G * 8 * 8));
  A.cs = reinterpret_cast<double*>(take(G * 12 * 8));
  A.big_task = E.big_task;
  Task* tasks[2];   // tasks of at most big_task groups, by wave parity
  Task* tasksB[2];  // larger tasks
  tasks[0] = reinterpret_cast<Task*>(take((size_t)(nnodesmax + 1) * sizeof(Task)));
  tasks[1] = reinterpret_cast<Task*>(take((size_t)(nnodesmax + 1) * sizeof(Task)));
  tasksB[0] = reinterpret_cast<Task*>(take((size_t)(nnodesmax + 1) * sizeof(Task)));
  tasksB[1] = reinterpret_cast<Task*>(take((size_t)(nnodesmax + 1) * sizeof(Task)));
  int32_t* ready[2];   // slot flags of tasks[k]
  int32_t* readyB[2];  // ... of tasksB[k]
  for (int k = 0; k < 2; ++k) {
    ready[k] = reinterpret_cast<int32_t*>(take((size_t)(nnodesmax + 1) * 4));
    readyB[k] = reinterpret_cast<int32_t*>(take((size_t)(nnodesmax + 1) * 4));
  }
  const size_t ready_bytes = (size_t)(nnodesmax + 1) * 4;
  AHOP_CUDA_TRY(E.d_nodes.ensure((size_t)(nnodesmax + 1) * sizeof(NodeRec)));
  AHOP_CUDA_TRY(cudaMemsetAsync(E.d_nodes.p, 0, (size_t)(nnodesmax + 1) * sizeof(NodeRec), st));
  AHOP_CUDA_TRY(E.d_flags.ensure(512));
  AHOP_CUDA_TRY(cudaMemsetAsync(E.d_flags.p, 0, 256, st));
  // [0..1] err, [2] nnodes, [3] nnext, [4] nnext_big, [5] ntaken, [6] ntaken_big, [7] max_big
  int32_t* flags = E.d_flags.as<int32_t>();
  A.stats = reinterpret_cast<unsigned long long*>(E.d_flags.as<char>() + 128);
  A.tprof = nullptr;
  if (E.task_profile) {
    AHOP_CUDA_TRY(E.d_tprof.ensure((size_t)(nnodesmax + 1) * kProfRow * 8));
    AHOP_CUDA_TRY(cudaMemsetAsync(E.d_tprof.p, 0, (size_t)(nnodesmax + 1) * kProfRow * 8, st));
    A.tprof = E.d_tprof.as<long long>();
  }
  A.err = flags;
  A.nnodes = flags + 2;
  A.nnext = flags + 3;
  A.nnext_big = flags + 4;
  A.ntaken = flags + 5;
  A.ntaken_big = flags + 6;
  A.max_big = flags + 7;
  A.par_cap_big = par_cap(kNTBig);
  A.x = E.d_x.as<double>(); A.y = E.d_y.as<double>(); A.z = E.d_z.as<double>(); A.m = E.d_m.as<double>();
  A.dens = E.d_dens.as<double>();
  A.orig = E.d_orig.as<int32_t>();
  A.ngroups = ng;
  A.densg = E.d_densg.as<double>();
  A.gpeak = E.d_gpeak.as<int32_t>();
  A.goff = E.d_goff.as<int32_t>();
  A.gmem = E.d_gmem.as<int32_t>();
  A.rdesc = rdesc - 0;  // indexed with goff (which starts group 1 at 0)
  A.pref = E.d_gmem_rho_pref.as<double>();
  A.soff = E.d_moff.as<int32_t>();  // forest rows (same layout as the saddle rows)
  A.sisad = E.m_isad;
  A.srho = E.m_rho;
  A.Lx = P.xlong; A.Ly = P.ylong; A.Lz = P.zlong; A.hx = P.xlongs2; A.hy = P.ylongs2; A.hz = P.zlongs2;
  A.fudge = P.fudge; A.alphap = P.alphap; A.epsilon = P.epsilon; A.nmembthresh = P.nmembthresh;
  A.node = E.d_nodes.as<NodeRec>();
  A.nnodesmax = nnodesmax;
  E.launches++;
  init_groups_kernel<<<(unsigned)((ng + 1 + T - 1) / T), T, 0, st>>>(A);
  AHOP_CUDA_TRY(cudaGetLastError());
  // root node 0 (f90:934-943): mass and truemass stay 0, densmax = max peak density
  int32_t nsmall = 0, nbig = 0;
  int32_t max_big = ng;  // largest task of the next wide launch (every task its blocks take is smaller)
  int32_t off_s = 0, off_b = 0;  // first task of the launch lists not taken by blocks of the previous wave
  {
    const Task root{P.rho_threshold, 0, 0, ng, 0};
    const bool big = ng > A.big_task;
    AHOP_CUDA_TRY(cudaMemcpyAsync(big ? tasksB[0] : tasks[0], &root, sizeof(Task), cudaMemcpyHostToDevice, st));
    (big ? nbig : nsmall) = 1;
  }
  int cur = 0;
  int32_t* h = reinterpret_cast<int32_t*>(E.h_scalars);
  // ---- root level on the whole grid
  {
    const double rhot = P.rho_threshold;
    const unsigned gb = (unsigned)((ng + T - 1) / T);
    E.launches++;
    iota_kernel<<<gb, T, 0, st>>>(A.par, ng, 0);
    E.launches++;
    root_union_kernel<<<(unsigned)(((int64_t)ng * 32 + T - 1) / T), T, 0, st>>>(A, rhot);
    E.launches++;
    root_roots_kernel<<<gb, T, 0, st>>>(A, A.cnt, A.run);
    AHOP_CUDA_TRY(cudaGetLastError());
    int kb = 1;
    while ((1LL << kb) <= (int64_t)ng) ++kb;
    size_t t1 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, A.cnt, A.par, A.run, A.GL, ng, 0, kb, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(t1));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, t1, A.cnt, A.par, A.run, A.GL, ng, 0, kb, st));
    E.launches++;
    root_heads_kernel<<<(unsigned)((ng + 1 + T - 1) / T), T, 0, st>>>(A, A.par, A.cnt);
    t1 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t1, A.cnt, A.run, ng + 1, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(t1));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, t1, A.cnt, A.run, ng + 1, st));
    E.launches++;
    root_cstart_kernel<<<gb, T, 0, st>>>(A, A.cnt, A.run);
    AHOP_CUDA_TRY(cudaMemcpyAsync(h + 4, A.run + ng, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    const int32_t ncomp = h[4];
    E.launches += 5;
    root_anchor_kernel<<<(unsigned)((ncomp + T - 1) / T), T, 0, st>>>(A, ncomp);
    root_terms_kernel<<<gb, T, 0, st>>>(A, rhot);
    root_decide_kernel<<<(unsigned)(((int64_t)ncomp * 32 + T - 1) / T), T, 0, st>>>(A, ncomp, rhot);
    root_decide_big_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(ncomp, 296)), kNT, 0, st>>>(A, ncomp, rhot);
    root_colour_kernel<<<ncomp, kNT, 0, st>>>(A, ncomp, rhot);
    E.launches++;
    root_okflag_kernel<<<(unsigned)((ncomp + 1 + T - 1) / T), T, 0, st>>>(A, ncomp, A.cnt);
    t1 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t1, A.cnt, A.run, ncomp + 1, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(t1));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, t1, A.cnt, A.run, ncomp + 1, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h + 4, A.run + ncomp, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h, flags, 8, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[0] != 0) {
      set_error("structure tree invariant failed at the root level (code " + std::to_string(h[0]) + ")");
      return AHOP_EINVARIANT;
    }
    const int32_t nsis = h[4];
    if (nsis >= 2) {
      // the root branches at once (the usual case): level-1 nodes 1..nsis
      A.next = tasks[1];
      A.next_big = tasksB[1];
      A.qready = ready[1];
      A.qready_big = readyB[1];
      AHOP_CUDA_TRY(cudaMemsetAsync(A.nnext, 0, 20, st));
      E.launches++;
      root_nodes_kernel<<<(unsigned)((ncomp + T - 1) / T), T, 0, st>>>(A, ncomp, A.cnt, A.run, nsis, rhot);
      E.launches++;
      root_deepnode_kernel<<<gb, T, 0, st>>>(A, A.cnt, A.run);
      AHOP_CUDA_TRY(cudaGetLastError());
      h[5] = nsis;
      AHOP_CUDA_TRY(cudaMemcpyAsync(A.nnodes, h + 5, 4, cudaMemcpyHostToDevice, st));
      AHOP_CUDA_TRY(cudaMemcpyAsync(h, flags, 32, cudaMemcpyDeviceToHost, st));
      AHOP_CUDA_TRY(cudaStreamSynchronize(st));
      nsmall = h[3];
      nbig = h[4];
      max_big = h[7];
      cur = 1;
    } else {
      // zero or one significant colour: the root task continues (f90:1577-1626)
      // on the general path from the initial group order
      E.launches++;
      init_groups_kernel<<<(unsigned)((ng + 1 + T - 1) / T), T, 0, st>>>(A);
      AHOP_CUDA_TRY(cudaGetLastError());
    }
  }
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[12], st));
  // Waves: small tasks on the compute stream, large ones (the critical path)
  // in wider blocks on a second stream at the same time.
  if (!E.stream2) {
    AHOP_CUDA_TRY(cudaFuncSetAttribute(tree_wave_kernel<kNTBig>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)wave_dyn_smem(kNTBig, par_cap(kNTBig))));
    AHOP_CUDA_TRY(cudaFuncSetAttribute(tree_wave_kernel<kNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)wave_dyn_smem(kNT, par_cap(kNT))));
    // the wide blocks run the largest tasks, the tree's critical path: their
    // stream has the highest priority, so their blocks are scheduled first
    // when SMs free up
    int prio_lo = 0, prio_hi = 0;
    AHOP_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    AHOP_CUDA_TRY(cudaStreamCreateWithPriority(&E.stream2, cudaStreamNonBlocking, prio_hi));
    AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_join, cudaEventDisableTiming));
  }
  if (E.tree_cluster_for != E.tree_cluster_req) {
    // wide tasks on clusters of kClusterCtas CTAs when the device can hold one
    // at the largest shared-memory size; else one CTA per wide task
    int ncl = 0;
    if (E.tree_cluster_req > 1) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(kClusterCtas);
      cfg.blockDim = dim3(kNTBig);
      cfg.dynamicSmemBytes = wave_dyn_smem(kNTBig, par_cap(kNTBig));
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = kClusterCtas;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      if (cudaOccupancyMaxActiveClusters(&ncl, tree_wave_kernel<kNTBig>, &cfg) != cudaSuccess) {
        cudaGetLastError();  // not supported here: no clusters
        ncl = 0;
      }
    }
    E.tree_cluster = ncl > 0 ? kClusterCtas : 1;
    E.tree_cluster_for = E.tree_cluster_req;
  }
  for (int wave = 0; nsmall + nbig > 0; ++wave) {
    if (wave > 100000) { set_error("structure tree: too many waves"); return AHOP_ELIMIT; }
    A.next = tasks[cur ^ 1];
    A.next_big = tasksB[cur ^ 1];
    A.qready = ready[cur ^ 1];
    A.qready_big = readyB[cur ^ 1];
    AHOP_CUDA_TRY(cudaMemsetAsync(ready[cur ^ 1], 0, ready_bytes, st));
    AHOP_CUDA_TRY(cudaMemsetAsync(readyB[cur ^ 1], 0, ready_bytes, st));
    AHOP_CUDA_TRY(cudaMemsetAsync(A.nnext, 0, 20, st));
    Task* list_s = tasks[cur] + off_s;
    Task* list_b = tasksB[cur] + off_b;
    if (nsmall > 2048) {
      const size_t nb = (size_t)nsmall;
      AHOP_CUDA_TRY(E.d_task_sort.ensure(nb * 16 + nb * sizeof(Task) + 256));
      uint32_t* k0 = E.d_task_sort.as<uint32_t>();
      uint32_t* k1 = k0 + nb;
      int32_t* v0 = reinterpret_cast<int32_t*>(k1 + nb);
      int32_t* v1 = v0 + nb;
      Task* tmp = reinterpret_cast<Task*>(reinterpret_cast<char*>(E.d_task_sort.p) + ((nb * 16 + 255) & ~size_t(255)));
      E.launches += 2;
      task_keys_kernel<<<(unsigned)((nb + T - 1) / T), T, 0, st>>>(list_s, nsmall, k0, v0);
      cub::DoubleBuffer<uint32_t> kb(k0, k1);
      cub::DoubleBuffer<int32_t> vb(v0, v1);
      size_t t1 = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, t1, kb, vb, nsmall, 0, 32, st);
      AHOP_CUDA_TRY(E.d_cub.ensure(t1));
      E.cub_calls++;
      AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(E.d_cub.p, t1, kb, vb, nsmall, 0, 32, st));
      task_gather_kernel<<<(unsigned)((nb + T - 1) / T), T, 0, st>>>(list_s, vb.Current(), nsmall, tmp);
      AHOP_CUDA_TRY(cudaMemcpyAsync(list_s, tmp, nb * sizeof(Task), cudaMemcpyDeviceToDevice, st));
      AHOP_CUDA_TRY(cudaGetLastError());
    }
    const bool prof = E.task_profile && wave < kMaxProfiledWaves;
    if (prof && !E.wave_ev[0]) {
      for (auto& e : E.wave_ev) AHOP_CUDA_TRY(cudaEventCreate(&e));
    }
    if (nbig > 0) {
      AHOP_CUDA_TRY(cudaEventRecord(E.ev_fork, st));
      AHOP_CUDA_TRY(cudaStreamWaitEvent(E.stream2, E.ev_fork, 0));
      if (prof) AHOP_CUDA_TRY(cudaEventRecord(E.wave_ev[2], E.stream2));
      E.launches++;
      // union-find parents sized to the launch's largest task: the rest of the
      // shared-memory carveout stays L1
      A.par_cap_big = std::min(par_cap(kNTBig), std::max(max_big, 1));
      if (E.tree_par_cap > 0) A.par_cap_big = std::min(A.par_cap_big, E.tree_par_cap);  // larger tasks: global array
      if (E.tree_cluster > 1) {
        // a cluster per wide task: CTA 0 runs the task, the others take slices
        // of its position-parallel phases (tree_wave_kernel, follow_phases)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)nbig * (unsigned)E.tree_cluster);
        cfg.blockDim = dim3(kNTBig);
        cfg.dynamicSmemBytes = wave_dyn_smem(kNTBig, A.par_cap_big);
        cfg.stream = E.stream2;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)E.tree_cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        AHOP_CUDA_TRY(cudaLaunchKernelEx(&cfg, tree_wave_kernel<kNTBig>, A, (const Task*)list_b));
      } else {
        tree_wave_kernel<kNTBig><<<nbig, kNTBig, wave_dyn_smem(kNTBig, A.par_cap_big), E.stream2>>>(A, list_b);
      }
      AHOP_CUDA_TRY(cudaGetLastError());
      if (prof) AHOP_CUDA_TRY(cudaEventRecord(E.wave_ev[3], E.stream2));
      AHOP_CUDA_TRY(cudaEventRecord(E.ev_join, E.stream2));
    }
    if (prof) AHOP_CUDA_TRY(cudaEventRecord(E.wave_ev[0], st));
    if (nsmall > 0) {
      E.launches++;
      tree_wave_kernel<kNT><<<nsmall, kNT, wave_dyn_smem(kNT, par_cap(kNT)), st>>>(A, list_s);
      AHOP_CUDA_TRY(cudaGetLastError());
    }
    if (prof) AHOP_CUDA_TRY(cudaEventRecord(E.wave_ev[1], st));
    if (nbig > 0) AHOP_CUDA_TRY(cudaStreamWaitEvent(st, E.ev_join, 0));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h, flags, 32, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    if (prof) {
      float ms_s = 0.f, ms_b = 0.f;
      cudaEventElapsedTime(&ms_s, E.wave_ev[0], E.wave_ev[1]);
      if (nbig > 0) cudaEventElapsedTime(&ms_b, E.wave_ev[2], E.wave_ev[3]);
      float* r = E.wave_prof + 4 * wave;
      r[0] = (float)nsmall; r[1] = ms_s; r[2] = (float)nbig; r[3] = ms_b;
      E.nwave_prof = wave + 1;
    }
    if (h[0] != 0) {
      set_error("structure tree invariant failed (code " + std::to_string(h[0]) + ", detail " +
                std::to_string(h[1]) + ")");
      return (h[0] == 12 || h[0] == 18) ? AHOP_ELIMIT : AHOP_EINVARIANT;
    }
    // tasks queued in this wave that no block took run in the next one
    nsmall = h[3] - h[5];
    nbig = h[4] - h[6];
    off_s = h[5];
    off_b = h[6];
    max_big = h[7];
    cur ^= 1;
    E.waves = wave + 1;
  }
  const int32_t nn = h[2];
  E.nnodes = nn;
  // ---- node sums in the reference order (deferred from the waves)
  if (nn > 0) {
    const unsigned gb1 = (unsigned)((ng + 1 + T - 1) / T);
    E.launches++;
    pair_count_kernel<<<gb1, T, 0, st>>>(A, nn, A.cnt);
    AHOP_CUDA_TRY(cudaGetLastError());
    size_t t1 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t1, A.cnt, A.run, ng + 1, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(t1));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(E.d_cub.p, t1, A.cnt, A.run, ng + 1, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h + 4, A.run + ng, 4, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t np = h[4];
    if (np > 0) {
      AHOP_CUDA_TRY(E.d_pairs.ensure((size_t)np * 16));
      AHOP_CUDA_TRY(E.d_pair_sums.ensure((size_t)np * 64));
      AHOP_CUDA_TRY(E.d_node_aux.ensure((size_t)(nn + 1) * 12));
      unsigned long long* k0 = E.d_pairs.as<unsigned long long>();
      unsigned long long* k1 = k0 + np;
      int32_t* nstart = E.d_node_aux.as<int32_t>();
      int32_t* nend = nstart + (nn + 1);
      int32_t* posref = nend + (nn + 1);
      E.launches++;
      pair_emit_kernel<<<gb1, T, 0, st>>>(A, A.run, k0);
      AHOP_CUDA_TRY(cudaGetLastError());
      int nb = 1;
      while ((1LL << nb) <= (int64_t)nn) ++nb;
      cub::DoubleBuffer<unsigned long long> kb(k0, k1);
      t1 = 0;
      cub::DeviceRadixSort::SortKeys(nullptr, t1, kb, (int)np, 0, 32 + nb, st);
      AHOP_CUDA_TRY(E.d_cub.ensure(t1));
      E.cub_calls++;
      AHOP_CUDA_TRY(cub::DeviceRadixSort::SortKeys(E.d_cub.p, t1, kb, (int)np, 0, 32 + nb, st));
      const unsigned long long* keys = kb.Current();
      AHOP_CUDA_TRY(cudaMemsetAsync(nstart, 0, (size_t)(nn + 1) * 8, st));
      const unsigned pb = (unsigned)((np + T - 1) / T);
      E.launches++;
      node_range_kernel<<<pb, T, 0, st>>>(keys, np, nstart, nend);
      E.launches++;
      node_posref_kernel<<<(unsigned)(((int64_t)nn * 32 + T - 1) / T), T, 0, st>>>(A, nn, keys, nstart, nend,
                                                                                    posref);
      E.launches++;
      pair_sums_kernel<<<pb, T, 0, st>>>(A, keys, np, posref, E.d_pair_sums.as<double>());
      int nsm = 148;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, E.device);
      int64_t wblocks = (np + 7) / 8;
      if (wblocks > (int64_t)nsm * 8) wblocks = (int64_t)nsm * 8;
      E.launches++;
      pair_sums_warp_kernel<<<(unsigned)wblocks, 256, 0, st>>>(A, keys, np, posref, E.d_pair_sums.as<double>());
      E.launches++;
      node_fold_kernel<<<(unsigned)(((int64_t)nn * 32 + T - 1) / T), T, 0, st>>>(A, nn, nstart, nend,
                                                                    E.d_pair_sums.as<double>());
      AHOP_CUDA_TRY(cudaGetLastError());
    }
  }
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[13], st));
  // ---- membership (f90:1297-1306 paint order => deepest node above rho_saddle)
  E.launches++;
  membership_kernel<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(E.d_group.as<int32_t>(), E.d_dens.as<double>(),
                                                              E.d_orig.as<int32_t>(), A.deepnode, A.node, n,
                                                              E.d_liste.as<int32_t>(), flags);
  AHOP_CUDA_TRY(cudaGetLastError());
  // ---- deterministic renumbering (f90:987-1041)
  AHOP_CUDA_TRY(E.d_rtab.ensure((size_t)(nn > 0 ? nn : 1) * 64));
  AHOP_CUDA_TRY(E.d_itab.ensure((size_t)(nn > 0 ? nn : 1) * 24));
  if (nn > 0) {
    AHOP_CUDA_TRY(E.d_idx2.ensure((size_t)(nn + 1) * 4 * 2));
    int32_t* new_to_old = E.d_idx2.as<int32_t>();
    int32_t* o2n = new_to_old + nn + 1;
    E.launches++;
    iota_kernel<<<(unsigned)((nn + T - 1) / T), T, 0, st>>>(new_to_old, nn, 1);
    AHOP_CUDA_TRY(cudaGetLastError());
    size_t tmp = 0;
    NodeLess less{A.node};
    cub::DeviceMergeSort::SortKeys(nullptr, tmp, new_to_old, nn, less, st);
    AHOP_CUDA_TRY(E.d_cub.ensure(tmp));
    E.cub_calls++;
    AHOP_CUDA_TRY(cub::DeviceMergeSort::SortKeys(E.d_cub.p, tmp, new_to_old, nn, less, st));
    E.launches++;
    old_to_new_kernel<<<(unsigned)((nn + T - 1) / T), T, 0, st>>>(new_to_old, nn, o2n);
    AHOP_CUDA_TRY(cudaGetLastError());
    E.launches++;
    tables_kernel<<<(unsigned)((nn + T - 1) / T), T, 0, st>>>(A.node, new_to_old, o2n, nn, E.d_rtab.as<double>(),
                                                              E.d_itab.as<int32_t>());
    AHOP_CUDA_TRY(cudaGetLastError());
    E.launches++;
    remap_liste_kernel<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(E.d_liste.as<int32_t>(), n, o2n);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaMemcpyAsync(h, flags, 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.tree_stats, E.d_flags.as<char>() + 128, 11 * 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[0] != 0) {
    set_error("membership walk exceeded its bound");
    return AHOP_ELIMIT;
  }
  return AHOP_OK;
}

}  // namespace ahop
