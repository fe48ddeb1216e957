// C ABI of the AdaptaHOP engine (declared in include/ahop_b200.h).
//
// Mirrors the f2py surface of the reference module neiKDtree
// (fortran/compute_adaptahop.pyf): three parameter setters, compute, the
// module output arrays and close.  Errors are returned, never fatal.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"

namespace ahop {

static Engine* g_engine = nullptr;
static thread_local std::string g_error;

Engine& engine() {
  if (!g_engine) g_engine = new Engine();
  return *g_engine;
}

void set_error(const std::string& s) { g_error = s; }

// Copy outputs to caller order: density (orig order) and the node tables.
__global__ void dens_to_orig_kernel(const double* __restrict__ dens, const int32_t* __restrict__ orig, int64_t n,
                                    double* __restrict__ out) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  out[orig[s]] = dens[s];
}

static int ensure_device(Engine& E) {
  if (E.device < 0) {
    int dev = 0;
    AHOP_CUDA_TRY(cudaGetDevice(&dev));
    E.device = dev;
  } else {
    AHOP_CUDA_TRY(cudaSetDevice(E.device));
  }
  if (!E.events_ready) {
    for (auto& e : E.ev) AHOP_CUDA_TRY(cudaEventCreate(&e));
    AHOP_CUDA_TRY(cudaMallocHost(&E.h_scalars, 64));
    E.events_ready = true;
  }
  return AHOP_OK;
}

static int validate(const Engine& E, int64_t n) {
  const Params& P = E.prm;
  if (n <= 0) { set_error("npart must be positive"); return AHOP_EINVAL; }
  if (n > 2000000000LL) { set_error("npart exceeds int32 particle ids"); return AHOP_EINVAL; }
  if (P.nvoisins < 2 || P.nvoisins > 32) { set_error("nvoisins must be in [2, 32]"); return AHOP_EINVAL; }
  if (P.nhop < 1 || P.nhop > P.nvoisins) { set_error("nhop must be in [1, nvoisins]"); return AHOP_EINVAL; }
  if (n <= P.nvoisins) { set_error("npart must exceed nvoisins"); return AHOP_EINVAL; }
  if (!(P.xlong > 0 && P.ylong > 0 && P.zlong > 0)) { set_error("box lengths must be positive"); return AHOP_EINVAL; }
  if (!(P.fudge > 0)) {
    // with fudge <= 0 the threshold never rises in the nsisters == 1 chain and
    // the reference's create-nodes loop (f90:1577-1603) does not terminate
    set_error("fudge must be positive");
    return AHOP_EINVAL;
  }
  if (P.optimize_nodes) {
    // the opt-in moment path of the reference (f90:1149-2314) is not
    // reproduced; its classic path (the default) is
    set_error("optimize_nodes=.true. is not supported (classic create_nodes path only)");
    return AHOP_EINVAL;
  }
  return AHOP_OK;
}

// h_dens_early: pinned host buffer that receives the density (caller order)
// on a copy stream while the later stages run, or null.
static int run_pipeline(Engine& E, const double* d_pos, const double* d_mass, int last_stage = 99,
                        double* h_dens_early = nullptr) {
  int rc;
  E.launches = E.cub_calls = E.waves = E.hop_passes = 0;
  cudaStream_t st = E.stream;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[1], st));
  if ((rc = stage_sort_and_tree(E, d_pos, d_mass))) return rc;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[2], st));
  if (last_stage < 2) return AHOP_OK;
  if ((rc = stage_knn_density(E))) return rc;
  // the density is final here: back to caller order now
  AHOP_CUDA_TRY(E.d_dens_orig.ensure(E.n * 8));
  E.launches++;
  dens_to_orig_kernel<<<(unsigned)((E.n + 255) / 256), 256, 0, st>>>(E.d_dens.as<double>(),
                                                                     E.d_orig.as<int32_t>(), E.n,
                                                                     E.d_dens_orig.as<double>());
  AHOP_CUDA_TRY(cudaGetLastError());
  if (h_dens_early) {
    if (!E.stream_copy) {
      AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream_copy, cudaStreamNonBlocking));
      AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_dens, cudaEventDisableTiming));
      AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_copied, cudaEventDisableTiming));
    }
    AHOP_CUDA_TRY(cudaEventRecord(E.ev_dens, st));
    AHOP_CUDA_TRY(cudaStreamWaitEvent(E.stream_copy, E.ev_dens, 0));
    AHOP_CUDA_TRY(cudaMemcpyAsync(h_dens_early, E.d_dens_orig.p, E.n * 8, cudaMemcpyDeviceToHost, E.stream_copy));
    AHOP_CUDA_TRY(cudaEventRecord(E.ev_copied, E.stream_copy));
  }
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[3], st));
  if (last_stage < 3) return AHOP_OK;
  if ((rc = stage_hop_groups(E))) return rc;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[4], st));
  if (last_stage < 4) return AHOP_OK;
  if ((rc = stage_saddles(E))) return rc;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[5], st));
  if (last_stage < 5) return AHOP_OK;
  if ((rc = stage_nodes(E))) return rc;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[6], st));
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[7], st));
  return AHOP_OK;
}

static void fill_timings(Engine& E, bool host) {
  auto el = [&](int a, int b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, E.ev[a], E.ev[b]);
    return ms;
  };
  AhopTimings& t = E.timings;
  t.upload = host ? el(0, 1) : 0.f;
  t.tree = el(1, 2);
  t.knn_density = el(2, 3);
  t.hop_groups = el(3, 4);
  t.saddles = el(4, 5);
  t.nodes = el(5, 6);
  t.membership = el(6, 7);
  t.download = host ? el(7, 8) : 0.f;
  t.total = host ? el(0, 8) : el(1, 7);
  t.knn_kernel = el(9, 10);
  t.nodes_prep = el(5, 11);
  t.nodes_root = el(11, 12);
  t.nodes_waves = el(12, 13);
  t.nodes_order = el(13, 6);
  t.kernel_launches = E.launches;
  t.cub_calls = E.cub_calls;
  t.tree_waves = E.waves;
  t.hop_passes = E.hop_passes;
}

}  // namespace ahop

using namespace ahop;

extern "C" {

const char* ahop_last_error(void) { return g_error.c_str(); }

int ahop_sync_from_init_adaptahop(const AhopInit* init) {
  if (!init) { set_error("null init"); return AHOP_EINVAL; }
  Params& P = engine().prm;
  P.init = *init;
  P.npart = init->npart;
  P.nmembthresh = init->nmembthresh;
  P.nMembers = init->nMembers;
  P.boxsize2 = init->boxsize2;
  P.Lf = init->Lf;
  P.xlong = init->xlong; P.ylong = init->ylong; P.zlong = init->zlong;
  P.xyzlong = P.xlong * P.ylong * P.zlong;  // f90:632
  P.xlongs2 = init->xlongs2; P.ylongs2 = init->ylongs2; P.zlongs2 = init->zlongs2;
  return AHOP_OK;
}

int ahop_sync_from_change_pos(int64_t npart, int32_t nusedpart, double epsilon, double fudgepsilon, double xlong,
                              double boxsize2) {
  Params& P = engine().prm;
  P.npart = npart;
  P.nusedpart = nusedpart;
  P.epsilon = epsilon;
  P.fudgepsilon = fudgepsilon;
  P.xlong = xlong;
  P.boxsize2 = boxsize2;
  return AHOP_OK;
}

int ahop_sync_others(const AhopOthers* o) {
  if (!o) { set_error("null others"); return AHOP_EINVAL; }
  Params& P = engine().prm;
  P.verbose = o->verbose != 0;
  P.megaverbose = o->megaverbose != 0;
  P.npart = o->npart;
  P.nbPes = o->nbPes;
  P.rho_threshold = o->rho_threshold;
  P.massp = o->massp;
  P.boxsize = o->boxsize;
  P.nhop = o->nhop;
  P.nvoisins = o->nvoisins;
  P.fudge = o->fudge;
  P.alphap = o->alphap;
  char m[9] = {0};
  std::memcpy(m, o->method, 8);
  P.method = m;
  P.nlevelmax = o->nlevelmax;
  P.optimize_nodes = o->optimize_nodes != 0;
  return AHOP_OK;
}

int ahop_compute_adaptahop_device(const double* d_pos, const double* d_mass, int64_t npart, void* stream) {
  Engine& E = engine();
  int rc;
  if ((rc = ensure_device(E))) return rc;
  if ((rc = validate(E, npart))) return rc;
  E.have_result = false;
  E.n = npart;
  E.stream = static_cast<cudaStream_t>(stream);
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[0], E.stream));
  E.mass_pending = false;  // the caller's device inputs are ready on its stream
  if ((rc = run_pipeline(E, d_pos, d_mass))) return rc;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[8], E.stream));
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  fill_timings(E, false);
  E.have_result = true;
  return AHOP_OK;
}

int ahop_compute_adaptahop(const double* pos_in, const double* mass_in, int64_t npart) {
  Engine& E = engine();
  int rc;
  if (!pos_in || !mass_in) { set_error("null input"); return AHOP_EINVAL; }
  if ((rc = ensure_device(E))) return rc;
  if ((rc = validate(E, npart))) return rc;
  E.have_result = false;
  E.n = npart;
  if (!E.stream) AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
  cudaStream_t st = E.stream;
  AHOP_CUDA_TRY(E.d_pos_in.ensure(npart * 24));
  AHOP_CUDA_TRY(E.d_mass_in.ensure(npart * 8));
  AHOP_CUDA_TRY(E.h_dens.ensure(npart * 8));
  if (!E.stream_copy) {
    AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream_copy, cudaStreamNonBlocking));
    AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_dens, cudaEventDisableTiming));
    AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_copied, cudaEventDisableTiming));
  }
  if (!E.ev_mass) AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_mass, cudaEventDisableTiming));
  if (!E.ev_posup) AHOP_CUDA_TRY(cudaEventCreateWithFlags(&E.ev_posup, cudaEventDisableTiming));
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[0], st));
  // positions first on the compute stream (the Morton keys and the sort need
  // only them); the masses follow on the copy stream once the positions are
  // in (two uploads at once would share the link and delay the positions),
  // overlapping the Morton sort, and are waited for just before the sorted
  // gather
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_pos_in.p, pos_in, npart * 24, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaEventRecord(E.ev_posup, st));
  AHOP_CUDA_TRY(cudaStreamWaitEvent(E.stream_copy, E.ev_posup, 0));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_mass_in.p, mass_in, npart * 8, cudaMemcpyHostToDevice, E.stream_copy));
  AHOP_CUDA_TRY(cudaEventRecord(E.ev_mass, E.stream_copy));
  E.mass_pending = true;
  // the density goes back to the host on a copy stream during the later stages
  if ((rc = run_pipeline(E, E.d_pos_in.as<double>(), E.d_mass_in.as<double>(), 99, E.h_dens.as<double>())))
    return rc;
  // module outputs to host (pinned, reused across calls)
  const int64_t nused = E.prm.nusedpart > 0 ? std::min<int64_t>(E.prm.nusedpart, npart) : npart;
  AHOP_CUDA_TRY(E.h_liste.ensure(nused * 4));
  AHOP_CUDA_TRY(E.h_rtab.ensure((size_t)(E.nnodes > 0 ? E.nnodes : 1) * 64));
  AHOP_CUDA_TRY(E.h_itab.ensure((size_t)(E.nnodes > 0 ? E.nnodes : 1) * 24));
  AHOP_CUDA_TRY(cudaStreamWaitEvent(st, E.ev_copied, 0));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.h_liste.p, E.d_liste.p, nused * 4, cudaMemcpyDeviceToHost, st));
  if (E.nnodes > 0) {
    AHOP_CUDA_TRY(cudaMemcpyAsync(E.h_rtab.p, E.d_rtab.p, (size_t)E.nnodes * 64, cudaMemcpyDeviceToHost, st));
    AHOP_CUDA_TRY(cudaMemcpyAsync(E.h_itab.p, E.d_itab.p, (size_t)E.nnodes * 24, cudaMemcpyDeviceToHost, st));
  }
  E.h_n = npart;
  E.h_nused = nused;
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[8], st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  fill_timings(E, true);
  E.have_result = true;
  return AHOP_OK;
}

int ahop_get_outputs(AhopOutputs* out) {
  Engine& E = engine();
  if (!out) { set_error("null out"); return AHOP_EINVAL; }
  if (!E.have_result || E.h_n != E.n) { set_error("no host outputs (call ahop_compute_adaptahop)"); return AHOP_ESTATE; }
  out->npart = E.n;
  out->nusedpart = E.h_nused;
  out->nnodes = E.nnodes;
  out->ngroups = E.ngroups;
  out->liste_parts = E.h_liste.as<int32_t>();
  out->density = E.h_dens.as<double>();
  out->real_table = E.h_rtab.as<double>();
  out->integer_table = E.h_itab.as<int32_t>();
  return AHOP_OK;
}

int ahop_get_device_outputs(AhopOutputs* out) {
  Engine& E = engine();
  if (!out) { set_error("null out"); return AHOP_EINVAL; }
  if (!E.have_result) { set_error("no outputs (call compute first)"); return AHOP_ESTATE; }
  out->npart = E.n;
  out->nusedpart = E.n;
  out->nnodes = E.nnodes;
  out->ngroups = E.ngroups;
  out->liste_parts = E.d_liste.as<int32_t>();
  out->density = E.d_dens_orig.as<double>();
  out->real_table = E.d_rtab.as<double>();
  out->integer_table = E.d_itab.as<int32_t>();
  return AHOP_OK;
}

int ahop_get_timings(AhopTimings* t) {
  Engine& E = engine();
  if (!t) return AHOP_EINVAL;
  *t = E.timings;
  return AHOP_OK;
}

static void release_device(Engine& E) {
  DevBuf* bufs[] = {&E.d_pos_in, &E.d_mass_in, &E.d_key, &E.d_key2, &E.d_idx, &E.d_idx2, &E.d_x, &E.d_y,
                    &E.d_z, &E.d_m, &E.d_orig, &E.d_rank, &E.d_box, &E.d_box32, &E.d_cub, &E.d_nei, &E.d_dens,
                    &E.d_hop, &E.d_root, &E.d_group, &E.d_peakflag, &E.d_densg, &E.d_gpeak, &E.d_goff,
                    &E.d_gmem, &E.d_gmem_rho, &E.d_gmem_rho_pref, &E.d_sad_key, &E.d_sad_key2, &E.d_sad_val,
                    &E.d_sad_val2, &E.d_sad_cnt, &E.d_sad_keep, &E.d_sad_kpos, &E.d_flags, &E.d_soff,
                    &E.d_sisad, &E.d_srho, &E.d_nodes, &E.d_tree_scratch, &E.d_liste, &E.d_dens_orig,
                    &E.d_rtab, &E.d_itab, &E.d_tprof, &E.d_pairs, &E.d_pair_sums, &E.d_node_aux,
                    &E.d_forest, &E.d_moff, &E.d_misad, &E.d_mrho, &E.d_kspill, &E.d_task_sort};
  if (E.device >= 0) cudaSetDevice(E.device);
  for (DevBuf* b : bufs) b->release();
  E.h_liste.release(); E.h_dens.release(); E.h_rtab.release(); E.h_itab.release();
}

// close (f90:3227-3264) deallocates the module's arrays.  Here the module
// outputs are dropped; device buffers stay cached for the next compute (a
// pool, like torch's caching allocator) -- the reference calls close() after
// every snapshot (NEI:64), and re-allocating gigabytes per snapshot would
// dominate the run.  ahop_release_device_memory() returns them.
int ahop_close(void) {
  if (!g_engine) return AHOP_OK;
  Engine& E = *g_engine;
  E.h_n = 0;
  E.h_nused = 0;
  E.have_result = false;
  E.nnodes = 0;
  E.ngroups = 0;
  E.n = 0;
  return AHOP_OK;
}

int ahop_release_device_memory(void) {
  if (!g_engine) return AHOP_OK;
  ahop_close();
  release_device(*g_engine);
  return AHOP_OK;
}

// ---------------------------------------------------------------- debug views
int ahop_debug_compute_stages(const double* pos_in, const double* mass_in, int64_t npart, int32_t last_stage) {
  Engine& E = engine();
  int rc;
  if (!pos_in || !mass_in) { set_error("null input"); return AHOP_EINVAL; }
  if ((rc = ensure_device(E))) return rc;
  if ((rc = validate(E, npart))) return rc;
  E.have_result = false;
  E.n = npart;
  if (!E.stream) AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
  AHOP_CUDA_TRY(E.d_pos_in.ensure(npart * 24));
  AHOP_CUDA_TRY(E.d_mass_in.ensure(npart * 8));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_pos_in.p, pos_in, npart * 24, cudaMemcpyHostToDevice, E.stream));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_mass_in.p, mass_in, npart * 8, cudaMemcpyHostToDevice, E.stream));
  E.mass_pending = false;  // both inputs on the compute stream here
  rc = run_pipeline(E, E.d_pos_in.as<double>(), E.d_mass_in.as<double>(), last_stage);
  if (rc) return rc;
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  return AHOP_OK;
}

int ahop_debug_tree_stats(int64_t* out, int32_t n) {
  Engine& E = engine();
  for (int i = 0; i < n && i < 8; ++i) out[i] = (int64_t)E.tree_stats[i];
  for (int i = 8; i < n && i < 13; ++i) out[i] = (int64_t)E.knn_stats[i - 8];
  for (int i = 13; i < n && i < 16; ++i) out[i] = (int64_t)E.tree_stats[i - 5];
  if (n > 16) out[16] = E.forest_rounds;
  if (n > 17) out[17] = E.forest_edges;
  for (int i = 18; i < n && i < 21; ++i) out[i] = (int64_t)E.knn_stats[i - 13];
  for (int i = 21; i < n && i < 26; ++i) out[i] = (int64_t)E.knn_phase[i - 21];
  for (int i = 26; i < n && i < 30; ++i) out[i] = (int64_t)E.knn_stats[i - 18];
  return AHOP_OK;
}

int ahop_debug_set_task_profile(int32_t on) {
  engine().task_profile = on != 0;
  return AHOP_OK;
}

int ahop_debug_task_profile(int64_t* out, int32_t maxrows) {
  Engine& E = engine();
  if (!E.task_profile || !E.d_tprof.p) { set_error("task profile not enabled"); return AHOP_ESTATE; }
  const int64_t rows = std::min<int64_t>((int64_t)maxrows, (int64_t)2 * E.ngroups + 1);
  if (rows <= 0) return AHOP_OK;
  AHOP_CUDA_TRY(cudaMemcpy(out, E.d_tprof.p, (size_t)rows * kProfRow * 8, cudaMemcpyDeviceToHost));
  return AHOP_OK;
}

int ahop_debug_set_tree_cluster(int32_t ctas) {
  if (ctas != 1 && ctas != 4) { set_error("tree cluster size must be 1 or 4"); return AHOP_EINVAL; }
  engine().tree_cluster_req = ctas;
  return AHOP_OK;
}

int ahop_debug_get_tree_cluster(void) { return engine().tree_cluster; }

int ahop_debug_set_tree_par_cap(int32_t groups) {
  if (groups < 0) { set_error("tree union-find cap must be >= 0"); return AHOP_EINVAL; }
  engine().tree_par_cap = groups;
  return AHOP_OK;
}

int ahop_debug_set_big_task(int32_t groups) {
  if (groups < 1) { set_error("big-task threshold must be positive"); return AHOP_EINVAL; }
  engine().big_task = groups;
  return AHOP_OK;
}

int ahop_debug_wave_profile(float* out, int32_t maxwaves) {
  Engine& E = engine();
  const int32_t n = std::min(maxwaves, E.nwave_prof);
  for (int32_t i = 0; i < 4 * n; ++i) out[i] = E.wave_prof[i];
  return n;
}

int ahop_debug_set_store_neighbours(int32_t k) {
  engine().req_store = k;
  return AHOP_OK;
}

__global__ void nei_to_orig_kernel(const int32_t* __restrict__ nei, int nstore, int k,
                                   const int32_t* __restrict__ orig, int64_t n, int32_t* __restrict__ out) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int64_t o = orig[s];
  for (int i = 0; i < k; ++i) out[o * k + i] = orig[nei[s * nstore + i]] + 1;
}

int ahop_debug_neighbours(int32_t* out, int32_t k) {
  Engine& E = engine();
  if (!E.have_result && E.n == 0) { set_error("no result"); return AHOP_ESTATE; }
  if (k < 1 || k > E.nstore) { set_error("k exceeds stored neighbours"); return AHOP_EINVAL; }
  DevBuf tmp;
  AHOP_CUDA_TRY(tmp.ensure((size_t)E.n * k * 4));
  E.launches++;
  nei_to_orig_kernel<<<(unsigned)((E.n + 255) / 256), 256, 0, E.stream>>>(E.d_nei.as<int32_t>(), E.nstore, k,
                                                                          E.d_orig.as<int32_t>(), E.n,
                                                                          tmp.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemcpyAsync(out, tmp.p, (size_t)E.n * k * 4, cudaMemcpyDeviceToHost, E.stream));
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  tmp.release();
  return AHOP_OK;
}

int ahop_debug_density(double* out) {
  Engine& E = engine();
  if (E.n == 0 || !out) { set_error("no result"); return AHOP_ESTATE; }
  AHOP_CUDA_TRY(E.d_dens_orig.ensure(E.n * 8));
  E.launches++;
  dens_to_orig_kernel<<<(unsigned)((E.n + 255) / 256), 256, 0, E.stream>>>(E.d_dens.as<double>(),
                                                                          E.d_orig.as<int32_t>(), E.n,
                                                                          E.d_dens_orig.as<double>());
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaMemcpyAsync(out, E.d_dens_orig.p, E.n * 8, cudaMemcpyDeviceToHost, E.stream));
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  return AHOP_OK;
}

__global__ void groups_to_orig_kernel(const int32_t* __restrict__ hop, const int32_t* __restrict__ group,
                                      const int32_t* __restrict__ orig, int64_t n, int32_t* __restrict__ hop_out,
                                      int32_t* __restrict__ grp_out) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int32_t o = orig[s];
  int32_t h = hop[s];
  hop_out[o] = h >= 0 ? orig[h] + 1 : 0;
  grp_out[o] = group[s];
}

int ahop_debug_groups(int32_t* hop_target, int32_t* group_id, int32_t* ngroups) {
  Engine& E = engine();
  if (E.n == 0) { set_error("no result"); return AHOP_ESTATE; }
  if (ngroups) *ngroups = E.ngroups;
  if (!hop_target && !group_id) return AHOP_OK;
  DevBuf tmp;
  AHOP_CUDA_TRY(tmp.ensure((size_t)E.n * 8));
  int32_t* h = tmp.as<int32_t>();
  E.launches++;
  groups_to_orig_kernel<<<(unsigned)((E.n + 255) / 256), 256, 0, E.stream>>>(
      E.d_hop.as<int32_t>(), E.d_group.as<int32_t>(), E.d_orig.as<int32_t>(), E.n, h, h + E.n);
  AHOP_CUDA_TRY(cudaGetLastError());
  if (hop_target) AHOP_CUDA_TRY(cudaMemcpyAsync(hop_target, h, E.n * 4, cudaMemcpyDeviceToHost, E.stream));
  if (group_id) AHOP_CUDA_TRY(cudaMemcpyAsync(group_id, h + E.n, E.n * 4, cudaMemcpyDeviceToHost, E.stream));
  AHOP_CUDA_TRY(cudaStreamSynchronize(E.stream));
  tmp.release();
  return AHOP_OK;
}

int ahop_debug_saddles(int32_t* nconn, int32_t* offsets, int32_t* isad, double* rho) {
  Engine& E = engine();
  if (E.n == 0) { set_error("no result"); return AHOP_ESTATE; }
  if (nconn) *nconn = E.nconn;
  cudaStream_t st = E.stream;
  if (offsets) AHOP_CUDA_TRY(cudaMemcpyAsync(offsets, E.d_soff.p, (size_t)(E.ngroups + 1) * 4, cudaMemcpyDeviceToHost, st));
  if (isad && E.nconn) AHOP_CUDA_TRY(cudaMemcpyAsync(isad, E.d_sisad.p, (size_t)E.nconn * 4, cudaMemcpyDeviceToHost, st));
  if (rho && E.nconn) AHOP_CUDA_TRY(cudaMemcpyAsync(rho, E.d_srho.p, (size_t)E.nconn * 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  return AHOP_OK;
}

}  // extern "C"
