// Internal state of the AdaptaHOP engine (one per process, like the Fortran
// module neiKDtree).  All particle arrays live in HBM in Morton-sorted order
// ("s" index); orig[s] maps back to the caller's 0-based particle index.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "ahop_b200.h"

namespace ahop {

// Growable device buffer; never shrinks until close().
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, need ? need : 16);
    if (e == cudaSuccess) bytes = need ? need : 16;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Growable pinned host buffer (module outputs live here; fast D2H).
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, need ? need : 16);
    if (e == cudaSuccess) bytes = need ? need : 16;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct Params {
  int64_t npart = 0;
  int32_t nusedpart = 0;
  int32_t nvoisins = 32, nhop = 16, nlevelmax = 30, nmembthresh = 20, nMembers = 20, nbPes = 1;
  double rho_threshold = 80.0, fudge = 4.0, alphap = 1.0, epsilon = 0.0, fudgepsilon = 1e-5;
  double massp = 0, boxsize = 1, boxsize2 = 1, Lf = 1;
  double xlong = 1, ylong = 1, zlong = 1, xlongs2 = 0.5, ylongs2 = 0.5, zlongs2 = 0.5, xyzlong = 1;
  bool verbose = false, megaverbose = false, optimize_nodes = false;
  std::string method = "MSM";
  AhopInit init{};
};

// Node record on the device; same fields as the Fortran `supernode`
// (f90:160-174).
struct NodeRec {
  double rho_saddle, density, densmax, radius, truemass, pos[3];
  int32_t mass, level, mother, firstchild, nsisters, sister;
};

constexpr int kLeaf = 32;         // particles per leaf bucket
constexpr int kFan = 32;          // children per internal node
constexpr int kMaxLevels = 8;
constexpr int kMaxProfiledWaves = 64;
constexpr int kProfRow = 32;  // int64 entries per structure-tree task-profile row

struct Engine {
  Params prm;
  int device = -1;
  cudaStream_t stream = nullptr;  // stream of the current call
  cudaStream_t stream2 = nullptr; // structure tree: large tasks run here beside the small ones
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int tree_cluster = 1;           // CTAs per wide structure-tree task in use (1: no clusters)
  int tree_cluster_req = 4;       // CTAs asked for (debug API: 4 or 1)
  int tree_cluster_for = 0;       // the request tree_cluster was chosen for (0: none yet)
  int tree_par_cap = 0;           // cap on the wide tasks' shared union-find array (0: none; debug API)
  cudaStream_t stream_copy = nullptr;   // host path: density copy-out during the later stages
  cudaEvent_t ev_dens = nullptr, ev_copied = nullptr;
  cudaEvent_t ev_mass = nullptr;        // host path: masses uploaded on the copy stream
  cudaEvent_t ev_posup = nullptr;       // host path: positions uploaded (the masses follow)
  bool mass_pending = false;            // ... and not yet waited for by the compute stream
  cudaEvent_t wave_ev[4] = {};          // per-wave timing (task profile only)
  float wave_prof[4 * 64] = {};         // per wave: small tasks, ms, large tasks, ms
  int32_t nwave_prof = 0;
  int32_t big_task = 512;               // structure-tree tasks above this many groups use wide blocks
  cudaEvent_t ev[16] = {};
  int32_t launches = 0, cub_calls = 0, waves = 0, hop_passes = 0;  // counters of the current compute
  int32_t forest_rounds = 0, forest_edges = 0;                        // saddle forest of the current compute
  unsigned long long tree_stats[11] = {};                             // structure-tree kernel counters
  unsigned long long knn_stats[12] = {};
  unsigned long long knn_phase[5] = {};                              // kNN kernel counters
  bool events_ready = false;
  AhopTimings timings{};

  int64_t n = 0;          // particles in the current run
  int32_t nstore = 16;    // neighbours stored per particle
  int32_t req_store = 0;  // requested via debug API (0 = nhop)
  bool task_profile = false;  // per-task structure-tree profile (debug API)
  bool have_result = false;

  // inputs / sorted particle arrays
  DevBuf d_pos_in, d_mass_in;            // staging for host inputs
  DevBuf d_key, d_key2, d_idx, d_idx2;   // Morton keys + permutation
  DevBuf d_x, d_y, d_z, d_m;             // sorted SoA
  DevBuf d_orig;                         // orig index (0-based) per sorted slot
  DevBuf d_rank;                         // sorted slot per orig index
  DevBuf d_box;                          // AABBs of all levels (6 doubles each)
  DevBuf d_box32;                        // AABBs of all levels in FP32, widened (2 float4 each)
  int32_t nlev = 0;
  int64_t lev_off[kMaxLevels + 1] = {};
  int64_t lev_cnt[kMaxLevels] = {};
  DevBuf d_cub;                          // CUB scratch

  // kNN / density
  DevBuf d_nei;                          // [n][nstore] sorted-slot neighbour ids
  DevBuf d_kspill;                       // kNN candidate spill buffers (per resident warp)
  DevBuf d_dens;                         // density in sorted order
  // hop / groups
  DevBuf d_hop, d_root, d_group;         // per sorted slot
  DevBuf d_peakflag;                     // per orig index
  int32_t ngroups = 0;
  DevBuf d_densg;                        // [ngroups+1] peak density per group
  DevBuf d_gpeak;                        // [ngroups+1] sorted slot of peak
  DevBuf d_goff;                         // [ngroups+2] member CSR offsets (desc orig order)
  DevBuf d_gmem;                         // [nactive] sorted slots
  DevBuf d_gmem_rho;                     // [nactive] member density in desc-density order
  DevBuf d_gmem_rho_pref;                // [nactive] prefix sums of density (desc density order)
  int64_t nactive = 0;
  // saddles
  DevBuf d_sad_key, d_sad_key2, d_sad_val, d_sad_val2, d_sad_cnt, d_sad_keep, d_sad_kpos;
  DevBuf d_flags;                        // small device error/status flags
  DevBuf d_soff, d_sisad, d_srho;        // final CSR
  int32_t nconn = 0;
  // nodes
  DevBuf d_nodes;                        // NodeRec[nnodesmax+1]
  DevBuf d_tree_scratch;
  DevBuf d_task_sort;                    // wave task ordering scratch
  DevBuf d_tprof;                        // per-task profile rows (debug)
  DevBuf d_forest;                       // saddle-forest scratch
  DevBuf d_moff, d_misad, d_mrho;        // saddle forest CSR (rows by decreasing saddle)
  int32_t* m_isad = nullptr;             // sorted forest rows inside d_misad / d_mrho
  double* m_rho = nullptr;
  DevBuf d_pairs;                        // (node, group) pair keys, sort double buffer
  DevBuf d_pair_sums;                    // [npairs][8] per-pair sums
  DevBuf d_node_aux;                     // per node: pair range, posref
  int32_t nnodes = 0;
  DevBuf d_liste;                        // [n] node id per ORIG particle (1-based), 0 none
  DevBuf d_dens_orig;                    // [n] density in ORIG order
  DevBuf d_rtab, d_itab;                 // exported tables

  // host copies (module outputs), pinned
  HostBuf h_liste, h_itab, h_dens, h_rtab;
  int64_t h_n = 0, h_nused = 0;

  // small pinned host scalars
  int64_t* h_scalars = nullptr;
};

Engine& engine();
void set_error(const std::string& s);

// Stage entry points (return AHOP_* codes).
int stage_sort_and_tree(Engine& E, const double* d_pos_aos, const double* d_mass);
int stage_knn_density(Engine& E);
int stage_hop_groups(Engine& E);
int stage_saddles(Engine& E);
int stage_nodes(Engine& E);
int build_saddle_forest(Engine& E);  // maximum spanning forest of the saddle rows (forest.cu)

}  // namespace ahop

#define AHOP_CUDA_TRY(expr)                                                                      \
  do {                                                                                            \
    cudaError_t _e = (expr);                                                                      \
    if (_e != cudaSuccess) {                                                                      \
      ::ahop::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) + " at " + __FILE__ + \
                        ":" + std::to_string(__LINE__));                                          \
      return (_e == cudaErrorMemoryAllocation) ? AHOP_ENOMEM : AHOP_ECUDA;                        \
    }                                                                                             \
  } while (0)
