/* ahop_b200 — B200-native AdaptaHOP halo finder, C ABI.
 *
 * Drop-in for the f2py module `compute_adaptahop.neikdtree` that the reference
 * builds from fortran/compute_adaptahop.pyf + fortran/compute_adaptahop.f90 and
 * calls from src/compute_neiKDtree_mod.py.  Plain pointers and sizes only.
 *
 * Conventions
 *  - Every entry point returns 0 on success and a nonzero AHOP_E* code on
 *    failure; ahop_last_error() gives a one-line reason.  Nothing aborts the
 *    process (the Fortran STOPs; this library reports instead).
 *  - State is module-global like the Fortran module: one finder per process,
 *    not re-entrant, one CUDA device (the current device at the first call).
 *  - Particle positions are in [-L/2, L/2) per axis with L = xlong (=boxsize2),
 *    laid out like the Fortran pos(3,npart): x0,y0,z0,x1,y1,z1,...
 *  - Particle, group and node ids at this boundary are 1-based like the
 *    Fortran; 0 means "none".
 */
#ifndef AHOP_B200_H
#define AHOP_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  AHOP_OK = 0,
  AHOP_EINVAL = 1,     /* bad argument or parameter */
  AHOP_ECUDA = 2,      /* CUDA runtime error */
  AHOP_ENOMEM = 3,     /* device allocation failed */
  AHOP_ESTATE = 4,     /* called out of order (e.g. outputs before compute) */
  AHOP_EINVARIANT = 5, /* an internal consistency check failed (Fortran would STOP) */
  AHOP_ELIMIT = 6,     /* a bounded device loop hit its iteration cap */
  AHOP_EDATA = 7,      /* input data rejected (malformed file, ids outside the dense layout) */
  AHOP_EIO = 8         /* a file could not be opened or read */
};

/* Arguments of sync_from_init_adaptahop (fortran/compute_adaptahop.pyf:25-48,
 * f90:591-641; called once per run from src/compute_neiKDtree_mod.py:183-197). */
typedef struct {
  int64_t npart;
  int32_t nmembthresh, nMembers;
  double omegaL, omega_lambda_f, omega0, omega_f, aexp_max, af, hubble, H_f;
  double boxsize2, Lf, xlong, ylong, zlong, xlongs2, ylongs2, zlongs2, Hub_pt, aexp;
  double pos_shift[3];
} AhopInit;

/* Arguments of sync_others (pyf:50-65, f90:643-678; NEI:738-747). */
typedef struct {
  int32_t verbose, megaverbose;
  int32_t npart, nbPes;
  double rho_threshold, massp, boxsize;
  int32_t nhop, nvoisins;
  double fudge, alphap;
  char method[8];
  int32_t nlevelmax, optimize_nodes;
} AhopOthers;

/* Borrowed views of the module outputs after compute (f90:485-490, node2table
 * f90:550-573).  real_table is [nnodes][8] = rho_saddle, density, densmax,
 * radius, truemass, x, y, z; integer_table is [nnodes][6] = mass, level,
 * mother, firstchild, nsisters, sister.  Row k is node k+1.  Valid until the
 * next compute or close. */
typedef struct {
  int64_t npart, nusedpart;
  int32_t nnodes, ngroups;
  const int32_t* liste_parts; /* [nusedpart] node id per particle, 0 = none */
  const double* density;      /* [npart] */
  const double* real_table;   /* [nnodes][8] */
  const int32_t* integer_table; /* [nnodes][6] */
} AhopOutputs;

/* Per-stage device timings of the last compute, milliseconds (CUDA events on
 * the compute stream), plus launch counts of the last compute: kernels of this
 * library, and CUB device-wide primitives it invoked. */
typedef struct {
  float upload, tree, knn_density, hop_groups, saddles, nodes, membership, download, total;
  float knn_kernel; /* the fused kNN + density kernel alone */
  /* parts of `nodes`: per-group density-sorted members and running sums,
   * root level, task waves, membership + renumbering + tables */
  float nodes_prep, nodes_root, nodes_waves, nodes_order;
  int32_t kernel_launches, cub_calls, tree_waves, hop_passes;
} AhopTimings;

const char* ahop_last_error(void);

/* replaces sync_from_init_adaptahop (pyf:25-48, f90:591) */
int ahop_sync_from_init_adaptahop(const AhopInit* init);
/* replaces sync_from_change_pos (pyf:16-23, f90:576) */
int ahop_sync_from_change_pos(int64_t npart, int32_t nusedpart, double epsilon, double fudgepsilon,
                              double xlong, double boxsize2);
/* replaces sync_others (pyf:50-65, f90:643) */
int ahop_sync_others(const AhopOthers* others);
/* replaces compute_adaptahop(pos_in, mass_in) (pyf:9-12, f90:495): host
 * buffers pos_in[npart][3], mass_in[npart]; copies in, runs every stage on the
 * GPU, copies the module outputs back to host memory owned by the library. */
int ahop_compute_adaptahop(const double* pos_in, const double* mass_in, int64_t npart);
/* The same pipeline on device-resident inputs (pos_in[npart][3] and
 * mass_in[npart] in device memory, read on `stream`, a cudaStream_t or NULL).
 * Outputs stay on the device; ahop_get_device_outputs exposes them. */
int ahop_compute_adaptahop_device(const double* d_pos_in, const double* d_mass_in, int64_t npart,
                                  void* stream);
/* replaces the module arrays liste_parts/density/nnodes/real_table/
 * integer_table read by src/compute_neiKDtree_mod.py:53-60 (host copies). */
int ahop_get_outputs(AhopOutputs* out);
/* Device-pointer view of the same outputs after either compute call. */
int ahop_get_device_outputs(AhopOutputs* out);
int ahop_get_timings(AhopTimings* t);
/* replaces close (pyf:67, f90:3227): drops the module outputs.  Device
 * buffers stay cached for the next compute; ahop_release_device_memory()
 * frees them. */
int ahop_close(void);
/* Frees every device buffer of the finder (no reference counterpart: the
 * Fortran module has no device memory). */
int ahop_release_device_memory(void);

/* ---- stage views for parity tests (host copies of device intermediates) ---- */
/* First k (<= stored count) neighbours of every particle, 1-based ids, sorted by
 * (distance, particle id); the kNN of omp_find_nearest_parts (f90:2841). */
int ahop_debug_neighbours(int32_t* out, int32_t k);
/* SPH density (omp_compute_density f90:2816-2838) of every particle, caller order. */
int ahop_debug_density(double* out);
/* Hop target (densest of the first nhop neighbours, f90:774-795), 1-based, 0
 * for particles at or below rho_threshold; and group id per particle after
 * find_local_maxima (f90:819-845), 0 for none. */
int ahop_debug_groups(int32_t* hop_target, int32_t* group_id, int32_t* ngroups);
/* Saddle CSR (dev_compute_saddle_list f90:2433-2813) before the tree build:
 * offsets[ngroups+1] (0-based), neighbour group ids (1-based) and saddle
 * densities, rows in decreasing saddle density.  Pass NULLs to get nconn. */
int ahop_debug_saddles(int32_t* nconn, int32_t* offsets, int32_t* isad, double* rho);
/* Run the pipeline on host inputs up to stage last_stage (2 = kNN + density,
 * 3 = hop + groups, 4 = saddles, 5 = everything) for stage-wise parity tests;
 * the stage views above then describe that partial run. */
int ahop_debug_compute_stages(const double* pos_in, const double* mass_in, int64_t npart, int32_t last_stage);
/* Kernel counters of the last compute: [0..7] structure tree -- cycles in
 * structural passes, in per-level statistics and in exact recomputation
 * (summed over blocks), threshold levels, exact passes for undecided tests,
 * the largest number of levels of one task, the largest cycle count of one
 * task, structural passes; [8..12] kNN -- query leaves, candidate leaves,
 * leaf visits, list insertions, leaves that fell back to per-query search;
 * [13..15] significance tests left undecided by the approximate sums, by
 * part: mean density, largest group mean density, densmax or radius;
 * [16..17] saddle forest: Boruvka rounds, forest edges; [18..20] kNN, only
 * while the task profile is on: candidate leaves within each query's final
 * radius, cycles spent in leaves that fell back to per-query search and in
 * the other leaves (summed over warps), then [21..25] the cycles of those
 * other leaves by phase: radius bound, candidate list and its sort, seed
 * lists, candidate scan, density; [26..29] kNN, task profile on: candidate
 * chunks examined, candidate leaves passing a query's box test at its ballot,
 * candidate leaves visited by at least one query of their leaf (leaves whose
 * list stayed in shared memory), and the number of such leaves.  The
 * counters [8..12] and [18..29] come from the profiling instance of the kNN
 * kernel, which runs only while the task profile is on. */
int ahop_debug_tree_stats(int64_t* out, int32_t n);
/* Per-task structure-tree profile (off by default; turning it on costs one
 * store per task).  Row k (32 int64) describes the task of node k (node ids
 * as created, before the final renumbering): [0] groups in its range, [1]
 * levels, [2] structural passes, cycles [3] in structural passes, [4] in
 * approximate statistics, [5] in exact sums, [6] in the whole task, [7] the
 * largest component count at one level, then phase cycles: [8..15] structural
 * (reset, union of long saddle rows, find, offsets, reorder, copy, starts,
 * component index), [16..19] statistics (anchors, group terms, small
 * components, large components), [20] structural union of short rows, [24]
 * the mother's node id as created, [25] groups the task dropped from its
 * range as below the member threshold for good.  Rows of nodes without a
 * task stay 0. */
int ahop_debug_set_task_profile(int32_t on);
/* Structure-tree waves of the last compute while the task profile is on (at
 * most 64): per wave the number of small tasks, their launch's milliseconds,
 * the number of large tasks and theirs.  Returns the number of waves. */
int ahop_debug_wave_profile(float* out, int32_t maxwaves);
/* Tuning: structure-tree tasks of more than `groups` groups run in
 * 1024-thread blocks on a second stream (default 512). */
int ahop_debug_set_big_task(int32_t groups);
/* Tuning: CTAs per wide structure-tree task: 4 (default; a thread-block
 * cluster whose leader runs the task and whose other CTAs take slices of its
 * union, root-finding and group-term passes, used when the device can hold
 * such a cluster) or 1 (one CTA per task).  get returns the size the last
 * compute used (1 before any). */
int ahop_debug_set_tree_cluster(int32_t ctas);
int ahop_debug_get_tree_cluster(void);
/* Testing: wide tasks of more than `groups` groups keep their union-find
 * parents in global memory instead of shared memory (0: no cap, the default;
 * the shared array then holds up to 32,768 groups). */
int ahop_debug_set_tree_par_cap(int32_t groups);
int ahop_debug_task_profile(int64_t* out, int32_t maxrows);
/* Ask compute to keep the first k neighbours per particle (default nhop). */
int ahop_debug_set_store_neighbours(int32_t k);

/* ---- halo/subhalo selection (MSM) and member grouping --------------------------
 * Replaces select_with_MS_method_1319 (src/compute_neiKDtree_mod.py:260-464)
 * and the member grouping of compute_adaptahop_131 (NEI:107-119), on the
 * device outputs of the last compute.  Structure ids are 1-based; particles in
 * no node get 0.  mother/first_sister/first_daughter/level are the
 * reference's mother_1319/first_sister_1319/first_daughter_1319/level_1319
 * (-1 = none, 0 = no mother).  pids_groupsorted lists 0-based particle
 * indices grouped by structure id (ascending), members in increasing index;
 * run_ids/run_idxs/run_counts are np.unique(..., return_index=True,
 * return_counts=True) of the sorted ids.  Host views, valid until the next
 * call. */
typedef struct {
  int32_t nstruct, nb_of_halos, nb_of_subhalos, ngroupruns;
  int64_t nusedpart;
  const int32_t* whereIam_parts;
  const int32_t *mother, *first_sister, *first_daughter, *level;
  const int32_t* pids_groupsorted;
  const int32_t *run_ids, *run_idxs, *run_counts;
} AhopStructs;
int ahop_select_msm(AhopStructs* out);
/* on = 0: later selections skip the host copies of the two per-particle arrays
 * (whereIam_parts and pids_groupsorted come back NULL); for callers that use
 * the device gather below (default on). */
int ahop_msm_set_particle_views(int32_t on);
/* The per-halo member gather of the reference's property loop (CHP:497-506:
 * members of structure s are pids0_groupsorted[whereIam_idxs[s] ...]) on the
 * device, after ahop_select_msm.  nstructs = structures with at least one
 * member (ascending id), nmembers = particles in them.  The gather writes, in
 * structure order: d_off[nstructs+1] member offsets, d_ids[nstructs] structure
 * ids (may be NULL), and each member's d_pos/d_vel ((n,3), caller's particle
 * order; d_vel/d_gvel may be NULL), d_mass and finder density (d_gdens may be
 * NULL), on `stream`. */
int ahop_structure_members(int32_t* nstructs, int64_t* nmembers);
int ahop_gather_members_device(const double* d_pos, const double* d_vel, const double* d_mass, int64_t* d_off,
                               int32_t* d_ids, double* d_gpos, double* d_gvel, double* d_gmass, double* d_gdens,
                               void* stream);
/* The particle index (0-based, caller's order; the reference's indexps) of
 * every gathered member, in the same structure order, into d_index[nmembers]
 * on `stream`: with ahop_halo_props' index/ndm it splits dark matter from
 * stars (CHP:766, 962). */
int ahop_gather_member_index_device(int32_t* d_index, void* stream);

/* ---- RAMSES particle reader --------------------------------------------------
 * Replaces _read_ramses_new_1010 (src/input_output.py:624-760) and the
 * count/load passes of read_ramses_new_101 (input_output.py:856-989) with the
 * stellar payload off: the part files' records are decoded on the device into
 * the dense arrays the finder reads (pos_10 = x - 0.5, vel_10 = v * scale_l /
 * scale_t * 1e-5, mass_10; source_pid_10 = |id| for a single family), in the
 * reference's layout (ind = |id| - 1, stars after the ndm dark-matter rows
 * when family = all).  open reads every file once (paths in cpu order) and
 * counts the families; decode fills caller device arrays of nselected rows
 * (d_source_pid may be NULL; it is written for family dm/star only).  Errors
 * as the reference raises them: AHOP_EDATA for record-length mismatches,
 * selected ids outside [1, nselected] or repeated within a file, unwritten
 * rows of a single family, no particle selected; AHOP_EIO for unreadable
 * files. */
typedef struct {
  int32_t version;  /* 3 (Ra3: families from birth time and id sign) or 4 (Ra4: family record) */
  int32_t family;   /* H.family: 0 all, 1 dm, 2 star */
  double scale_l, scale_t; /* info file units (unit_l, unit_t) */
} AhopRamsesParams;
typedef struct {
  int64_t total, ndm, nstar, nselected;
  int32_t nfiles, ndim;
} AhopRamsesCounts;
int ahop_ramses_open(const char* const* paths, int32_t nfiles, const AhopRamsesParams* p, AhopRamsesCounts* out);
int ahop_ramses_decode_device(double* d_pos, double* d_vel, double* d_mass, int64_t* d_source_pid, void* stream);
int ahop_ramses_close(void);

/* ---- batched halo properties ------------------------------------------------
 * Replaces the per-halo reductions of src/compute_halo_props.py run by
 * _compute_halo_props (CHP:270-301): det_mass_17 (with the dark-matter /
 * star split of mode 'full', CHP:766-780), det_center_18 (densest member, or
 * with cdm the member closest to the centre of mass, CHP:917-936; sigma_dm and
 * sigma* of CHP:962-966), compute_ang_mom_19, r_halos_1a,
 * det_inertial_tensor_1b20 + det_main_axis_1b2, det_halo_energies_1b3 (E_kin
 * with Hubble flow; E_pot as the direct pair sum for every halo size) and
 * compute_spin_parameter_1c.  Members of halo h are rows [off[h], off[h+1]).
 * Each halo gets AHOP_HALO_NFIELDS doubles, indexed by the HP_* constants
 * (counts as doubles). */
enum {
  HP_M = 0, HP_PX, HP_PY, HP_PZ, HP_VX, HP_VY, HP_VZ, HP_LX, HP_LY, HP_LZ, HP_R,
  HP_IXX, HP_IXY, HP_IXZ, HP_IYY, HP_IYZ, HP_IZZ, HP_EK, HP_EP64, HP_EP32C, HP_SIGMA,
  HP_SHA, HP_SHB, HP_SHC, HP_SPIN64, HP_SPIN32C, HP_ICENTER,
  HP_NDM, HP_NSTAR, HP_MDM, HP_MSTAR, HP_MCONTAM, HP_SIGMA_DM, HP_SIGMA_STAR, AHOP_HALO_NFIELDS
};

typedef struct {
  double Lbox;      /* period (H.Lbox_pt), same unit as positions */
  double Hub_pt;    /* Hubble constant used for the Hubble flow in E_kin */
  double gravconst; /* G (H.gravconst = 430.1) */
  int32_t periodic; /* H.FlagPeriod != 0 */
  int32_t epot;     /* bit 0: FP64 direct sum, bit 1: FP32-compensated direct sum */
  int32_t sc;       /* H.SC: shrinking-sphere centre (refine_centers_1b, CHP:1555-1596), off by default */
  int32_t pad;
  double dcell_min; /* H.dcell_min: smallest sphere radius */
  double eps_sc;    /* H.eps_SC: radius shrink factor per step, in (0, 1) when sc is on */
  int32_t cdm;      /* H.cdm: centre = member closest to the centre of mass instead of the densest one */
  int32_t pad2;
  int64_t ndm;      /* H.ndm: a member whose particle index is below ndm is dark matter (CHP:766, 962) */
  double massp;     /* H.massp: dark-matter members heavier than massp * 1.00001 are contamination (CHP:768) */
  const int32_t* index; /* particle index of every member (the reference's indexps), in the same memory as
                           the call's other arrays (host for ahop_halo_props, device otherwise); NULL: every
                           member is dark matter */
} AhopHaloParams;

typedef struct {
  float moments, epot64, epot32c, finalize, total; /* ms, CUDA events */
  double pairs;                                    /* sum over halos of n(n-1)/2 */
  int32_t items, kernel_launches;
  float tune_ms;          /* host wall time of the tile autotuner in this call (0 when it did not run) */
  int32_t graph_replays;  /* replays of the captured launch graph since its capture (-1: graphs off) */
} AhopHaloTimings;

/* Host buffers: off[nhalo+1], pos[n][3], vel[n][3], mass[n], density[n];
 * out[nhalo][AHOP_HALO_NFIELDS] (host). */
int ahop_halo_props(const AhopHaloParams* p, const int64_t* off, int64_t nhalo, const double* pos,
                    const double* vel, const double* mass, const double* density, double* out);
/* Same on device buffers (all pointers device memory), on `stream`. */
int ahop_halo_props_device(const AhopHaloParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                           const double* d_vel, const double* d_mass, const double* d_density, double* d_out,
                           void* stream);
int ahop_halo_get_timings(AhopHaloTimings* t);
/* Tile shapes of the FP32-compensated pair kernel, one per halo-size bucket
 * (members n < 512, < 4096, < 32768, < 262144, >= 262144): 128, 256 or 512
 * rows per work item (1, 2 or 4 rows per thread).  Unless pinned, a bucket's
 * shape is picked by timing the three shapes on the first call that holds
 * halos of that bucket (about 3e9 pairs of that call's own halos per shape),
 * and kept for the process.  The shape changes the FP32 summation groups, so
 * ep32c may differ between shapes by its rounding error (well below 1e-6
 * relative); pin the shapes for bit-reproducible FP32 results across
 * processes.  get: rows[AHOP_HALO_BUCKETS] in use (0 = not tuned yet),
 * ms[AHOP_HALO_BUCKETS * 3] the autotuner's times per shape (may be null).
 * set: rows[b] in {128, 256, 512} pins bucket b, 0 lets the autotuner pick;
 * rows == NULL forgets every pin and every tuned shape. */
#define AHOP_HALO_BUCKETS 5
int ahop_halo_get_tiles(int32_t* rows, float* ms);
int ahop_halo_set_tiles(const int32_t* rows);
/* The launch sequence of ahop_halo_props(_device) is captured once as a CUDA
 * graph and replayed while the call's device pointers, halo count and work
 * list sizes stay the same (on = 1, the default); on = 0 launches directly. */
int ahop_halo_set_graph(int32_t on);
/* Allocation-free variant of ahop_halo_props_device (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- code running while
 * another part of the process captures a CUDA graph, frameworks that own all
 * device memory through their own pool, callers with a fixed memory budget.
 * It allocates nothing: its scratch is a file-scope device array of about
 * 10 MB (held on every GPU that loads the library until exit), limiting one
 * call to 65,536 halos and 262,144 work items (one item per 256 members of a
 * halo); larger calls are rejected with AHOP_EINVAL.  The caller passes device
 * inputs and the device output [nhalo][AHOP_HALO_NFIELDS].  Every call shares
 * that array, so calls that overlap on the GPU (other streams, other host
 * threads) race; serialise them.  The first call on a device looks up the
 * array's address and should come before any stream capture.  Each call
 * blocks the host twice (it reads the work-item count, then the error flag,
 * back from the device), so it must not be called on a stream that is being
 * captured (it returns AHOP_EINVAL there).  Next to another thread's capture,
 * pass a non-blocking stream (cudaStreamNonBlocking): the legacy default
 * stream synchronises implicitly with blocking streams and would join it. */
int ahop_halo_props_noalloc(const AhopHaloParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                            const double* d_vel, const double* d_mass, const double* d_density, double* d_out,
                            void* stream);

/* ---- virial properties ------------------------------------------------------
 * Replaces det_vir_1b (CHP:1248-1262): det_main_axis_1b2 (principal axes with
 * eigenvectors), tab_props_inside_1b40 (nshell concentric ellipsoids: mass and
 * kinetic energy with Hubble flow), potential_profile_1b40 under the
 * reference's default policies (shell integration, exact shell self-pair
 * counting; halos of fewer than direct_limit members rescaled to their direct
 * E_pot, larger ones take the profile's outer value as E_pot) and
 * det_vir_props_1b4 (virial theorem to 20 %, else the overdensity
 * vir_overdens * rho_mean), with the TSIS profile (rho_0, r_c).  Inputs are
 * the members (as for ahop_halo_props) and that call's output rows; each halo
 * gets AHOP_VIR_NFIELDS doubles indexed by VIR_*.  Halos whose axes degenerate
 * (or that find no virial region) get NaN virial fields, as the reference. */
enum {
  VIR_RVIR = 0, VIR_MVIR, VIR_CVEL, VIR_TVIR, VIR_RHO0, VIR_RC, VIR_EP, VIR_ET, VIR_AMAX, VIR_BMAX, VIR_CMAX,
  AHOP_VIR_NFIELDS
};

typedef struct {
  double Lbox, Hub_pt, gravconst; /* as AhopHaloParams */
  double vir_overdens, rho_mean;  /* H.vir_overdens, H.rho_mean (CHP:1330-1331) */
  int32_t periodic;
  int32_t nshell;       /* ttab, 1000 in the reference; at most 1024 */
  int32_t direct_limit; /* full_PE / virial_direct_pe_nmax, 1000 in the reference */
  int32_t ep_field;     /* HP_EP64 or HP_EP32C: which direct E_pot to rescale to */
} AhopVirialParams;

/* Host buffers: off[nhalo+1], pos[n][3], vel[n][3], mass[n],
 * props[nhalo][AHOP_HALO_NFIELDS] (ahop_halo_props output); out[nhalo][AHOP_VIR_NFIELDS]. */
int ahop_halo_virial(const AhopVirialParams* p, const int64_t* off, int64_t nhalo, const double* pos,
                     const double* vel, const double* mass, const double* props, double* out);
/* Same on device buffers, on `stream`. */
int ahop_halo_virial_device(const AhopVirialParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                            const double* d_vel, const double* d_mass, const double* d_props, double* d_out,
                            void* stream);
/* Milliseconds of the last virial launch (CUDA events). */
float ahop_halo_virial_last_ms(void);

/* ---- differentiation -----------------------------------------------------------
 * SPH density with FIXED neighbour lists (nei[n][nvoisins], 0-based particle
 * indices sorted by distance at the lists' reference configuration) and its
 * adjoint with respect to positions; the gradient of each halo's direct-sum
 * potential.  The density forward is omp_compute_density (f90:2816-2838)
 * with the same rounding, so with the finder's own lists it reproduces the
 * finder's densities bit for bit; the potential is det_halo_energies_1b3's
 * direct sum (CHP:1413-1427).  All pointers are device memory; gpos is
 * accumulated into (zero it first). */
typedef struct {
  int32_t nvoisins, pad;
  double xlong, ylong, zlong;
} AhopAdjParams;
int ahop_density_fixed(const AhopAdjParams* p, const double* d_pos, const double* d_mass, const int32_t* d_nei,
                       int64_t n, double* d_dens, void* stream);
int ahop_density_adjoint(const AhopAdjParams* p, const double* d_pos, const double* d_mass, const int32_t* d_nei,
                         int64_t n, const double* d_gdens, double* d_gpos, void* stream);
/* dE_h/dx scaled by gh[h], accumulated into gpos; centre[h] = index (within
 * the halo) of the densest member, the origin of the min-image separations;
 * h_off is the host copy of d_off. */
int ahop_epot_grad(const AhopHaloParams* p, const int64_t* d_off, const int64_t* h_off, int64_t nhalo,
                   const double* d_pos, const double* d_mass, const int32_t* d_centre, const double* d_gh,
                   double* d_gpos, void* stream);

#ifdef __cplusplus
}
#endif
#endif
