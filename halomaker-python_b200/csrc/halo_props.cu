// Batched per-halo properties; replaces the per-halo NumPy reductions of
// src/compute_halo_props.py that _compute_halo_props (CHP:270-301) runs for
// every halo in a multiprocessing pool:
//   det_mass_17 (CHP:754-780)          m
//   det_center_18 (CHP:901-966)        centre = densest member (cdm=False),
//                                      bulk velocity, sigma
//   compute_ang_mom_19 (CHP:783-824)   L about the centre, min-image
//   r_halos_1a (CHP:828-851)           r = max |dr|
//   det_inertial_tensor_1b20 (CHP:1932-1951) + det_main_axis_1b2 (1954-1967)
//                                      I_ab, sha/shb/shc = sqrt(eig(I)/m)
//   det_halo_energies_1b3 (CHP:1400-1444) E_kin with Hubble flow and the
//                                      direct-sum E_pot for every halo size
//   compute_spin_parameter_1c (CHP:1599-1602)
//
// Layout: members of halo h are rows [off[h], off[h+1]) of pos/vel (n,3),
// mass (n) and density (n), FP64 in HBM.  The O(n) quantities come from two
// passes over the members in chunks of 8,192 (a block per chunk, partials
// folded per halo in chunk order, so results are deterministic).  The O(n^2)
// potential runs as persistent launches over a work list of (halo, row tile,
// partner chunk) items sorted by decreasing cost; each item sums m_j / r_ij
// for its rows over its partners j > i.  Two forms share the schedule:
//   * FP64: relative positions, 1/r from the double reciprocal square root;
//   * FP32-compensated: positions relative to the halo centre split into
//     hi = float(r) and lo = float(r - hi) (packed pairs in shared memory);
//     a pair separation is (hi_j - hi_i) + (lo_j - lo_i) in FP32 (packed
//     f32x2 arithmetic), 1/r from the approximate reciprocal square root,
//     partial sums Kahan-compensated in FP32 and folded into FP64 per item.
// Per-item partials are reduced per halo in item order (deterministic); the
// launch sequence is captured once as a CUDA graph and replayed.  The
// allocation-free entry point at the end of the file keeps the single-block
// moment kernel and one 256-row list.
#include <cuda_runtime.h>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <cub/cub.cuh>

#include "ahop_halo.h"
#include "engine.h"

namespace ahop {

constexpr int kPB = 256;  // threads per block (and i-tile size of the pair kernel)
constexpr long long kMaxShrinkSteps = 1000000;  // shrinking-sphere steps per halo (error past this)

__device__ __forceinline__ double wrap_chp(double d, double L, double h, int periodic) {
  // correct_for_periodicity_1d (CHP:854-863): strict comparisons
  if (!periodic) return d;
  if (d > h) d -= L;
  if (d < -h) d += L;
  return d;
}

// det_mass_17's dmmask (CHP:766): particle index below ndm
__device__ __forceinline__ bool member_is_dm(const HaloArgs& A, int64_t i) {
  return A.index == nullptr || (int64_t)A.index[i] < A.ndm;
}

// correct_for_periodicity on an absolute coordinate (CHP:880-885)
__device__ __forceinline__ double wrap_abs(double x, double L, double h, int periodic) {
  return wrap_chp(x, L, h, periodic);
}

template <class T, int NT = kPB>
__device__ __forceinline__ T block_sum(T v, T* sh) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  T r = 0;
  if (tid < 32) {
    r = (tid < NT / 32) ? sh[tid] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  if (tid == 0) sh[0] = r;
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}

// Shrinking-sphere centre (refine_centers_1b with SC, CHP:1555-1596 ->
// det_halo_center_sphere_1b1, 1498-1541): from the densest member and the
// radius of the farthest member, repeatedly take the centre of mass of the
// members within r (min-image offsets) and shrink r by (1 - eps_SC), while
// r > dcell_min and the sphere holds mass; the centre becomes the member
// closest to the last centre of mass (first such member).  s_c[0..2] and
// s_c[6] (centre and its member index) are updated in place.
__device__ void shrink_sphere_centre(const HaloArgs& A, int64_t b0, int64_t b1, double* s_c, double* sh,
                                     double* s_best_d, long long* s_best_i) {
  __shared__ double s_sc[5];  // x0, y0, z0, r0, continue
  const int tid = threadIdx.x;
  double x0 = s_c[0], y0 = s_c[1], z0 = s_c[2];
  auto dist2 = [&](int64_t i, double ax, double ay, double az, double& dx, double& dy, double& dz) {
    dx = wrap_chp(A.pos[3 * i] - ax, A.L, A.h, A.periodic);
    dy = wrap_chp(A.pos[3 * i + 1] - ay, A.L, A.h, A.periodic);
    dz = wrap_chp(A.pos[3 * i + 2] - az, A.L, A.h, A.periodic);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  };
  // r0: farthest member from the densest one (_radius_from_center)
  double r2 = 0.0;
  for (int64_t i = b0 + tid; i < b1; i += kPB) {
    double dx, dy, dz;
    r2 = fmax(r2, dist2(i, x0, y0, z0, dx, dy, dz));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
  if ((tid & 31) == 0) s_best_d[tid >> 5] = r2;
  __syncthreads();
  double r0 = s_best_d[0];
  for (int w = 1; w < kPB / 32; ++w) r0 = fmax(r0, s_best_d[w]);
  r0 = sqrt(r0);
  __syncthreads();
  if (!(r0 > 0.0) || !isfinite(r0)) return;
  double xc = x0, yc = y0, zc = z0;
  for (long long it = 0;; ++it) {
    const double r02 = r0 * r0;
    double pcx = 0, pcy = 0, pcz = 0, mt = 0;
    for (int64_t i = b0 + tid; i < b1; i += kPB) {
      double dx, dy, dz;
      if (dist2(i, x0, y0, z0, dx, dy, dz) <= r02) {
        const double w = A.mass[i];
        pcx += w * dx; pcy += w * dy; pcz += w * dz; mt += w;
      }
    }
    pcx = block_sum(pcx, sh); pcy = block_sum(pcy, sh); pcz = block_sum(pcz, sh); mt = block_sum(mt, sh);
    if (tid == 0) {
      if (mt > 0) { xc = pcx / mt + x0; yc = pcy / mt + y0; zc = pcz / mt + z0; }
      else { xc = x0; yc = y0; zc = z0; }
      bool cont = r0 > A.dcell_min && mt > 0;
      if (cont && it >= kMaxShrinkSteps) { atomicExch(A.err, 1); cont = false; }
      s_sc[0] = xc; s_sc[1] = yc; s_sc[2] = zc; s_sc[3] = (1.0 - A.eps_sc) * r0; s_sc[4] = cont ? 1.0 : 0.0;
    }
    __syncthreads();
    xc = s_sc[0]; yc = s_sc[1]; zc = s_sc[2];
    const bool cont = s_sc[4] != 0.0;
    r0 = s_sc[3];
    __syncthreads();
    if (!cont) break;
    x0 = xc; y0 = yc; z0 = zc;
  }
  // the member closest to the last centre of mass (np.argmin: first minimum)
  double bd = DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t i = b0 + tid; i < b1; i += kPB) {
    double dx, dy, dz;
    const double d = dist2(i, xc, yc, zc, dx, dy, dz);
    if (d < bd || (d == bd && i < bi)) { bd = d; bi = i; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bd, o);
    const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (od < bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
  }
  if ((tid & 31) == 0) { s_best_d[tid >> 5] = bd; s_best_i[tid >> 5] = bi; }
  __syncthreads();
  if (tid == 0) {
    double d = s_best_d[0];
    long long ii = s_best_i[0];
    for (int w = 1; w < kPB / 32; ++w)
      if (s_best_d[w] < d || (s_best_d[w] == d && s_best_i[w] < ii)) { d = s_best_d[w]; ii = s_best_i[w]; }
    s_c[0] = A.pos[3 * ii]; s_c[1] = A.pos[3 * ii + 1]; s_c[2] = A.pos[3 * ii + 2];
    s_c[6] = (double)(ii - b0);
  }
  __syncthreads();
}

// One block per halo: pass 1 (mass, momentum, densest member), pass 2
// (L, r, inertia, E_kin, sigma) about the densest member and bulk velocity.
__global__ void __launch_bounds__(kPB) halo_moments_kernel(HaloArgs A) {
  __shared__ double sh[kPB / 32];
  __shared__ double s_best_d[kPB / 32];
  __shared__ long long s_best_i[kPB / 32];
  __shared__ double s_c[7];
  const int tid = threadIdx.x;
  const int64_t h = blockIdx.x;
  const int64_t b0 = A.off[h], b1 = A.off[h + 1];
  // pass 1
  double m = 0, mvx = 0, mvy = 0, mvz = 0, bd = -DBL_MAX;
  double mdm = 0, mst = 0, ndm = 0, nst = 0, mcon = 0, cmx = 0, cmy = 0, cmz = 0;
  long long bi = LLONG_MAX;
  const double fx = b1 > b0 ? A.pos[3 * b0] : 0.0, fy = b1 > b0 ? A.pos[3 * b0 + 1] : 0.0,
               fz = b1 > b0 ? A.pos[3 * b0 + 2] : 0.0;
  for (int64_t i = b0 + tid; i < b1; i += kPB) {
    const double w = A.mass[i];
    m += w;
    mvx += w * A.vel[3 * i];
    mvy += w * A.vel[3 * i + 1];
    mvz += w * A.vel[3 * i + 2];
    if (member_is_dm(A, i)) {
      mdm += w; ndm += 1.0;
      if (w > A.massp * 1.00001) mcon += w;
    } else {
      mst += w; nst += 1.0;
    }
    if (A.cdm) {
      cmx += w * wrap_chp(A.pos[3 * i] - fx, A.L, A.h, A.periodic);
      cmy += w * wrap_chp(A.pos[3 * i + 1] - fy, A.L, A.h, A.periodic);
      cmz += w * wrap_chp(A.pos[3 * i + 2] - fz, A.L, A.h, A.periodic);
    }
    const double d = A.dens[i];
    if (d > bd || (d == bd && i < bi)) { bd = d; bi = i; }  // np.argmax: first maximum
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double od = __shfl_xor_sync(0xffffffffu, bd, o);
    long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (od > bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
  }
  if ((tid & 31) == 0) { s_best_d[tid >> 5] = bd; s_best_i[tid >> 5] = bi; }
  m = block_sum(m, sh);
  mvx = block_sum(mvx, sh);
  mvy = block_sum(mvy, sh);
  mvz = block_sum(mvz, sh);
  mdm = block_sum(mdm, sh); mst = block_sum(mst, sh); ndm = block_sum(ndm, sh); nst = block_sum(nst, sh);
  mcon = block_sum(mcon, sh);
  if (A.cdm) { cmx = block_sum(cmx, sh); cmy = block_sum(cmy, sh); cmz = block_sum(cmz, sh); }
  if (tid == 0) {
    double d = s_best_d[0];
    long long ii = s_best_i[0];
    for (int w = 1; w < kPB / 32; ++w)
      if (s_best_d[w] > d || (s_best_d[w] == d && s_best_i[w] < ii)) { d = s_best_d[w]; ii = s_best_i[w]; }
    if (ii != LLONG_MAX) {
      s_c[0] = A.pos[3 * ii]; s_c[1] = A.pos[3 * ii + 1]; s_c[2] = A.pos[3 * ii + 2];
    } else {  // a halo without members
      s_c[0] = s_c[1] = s_c[2] = 0.0;
      ii = b0;
    }
    s_c[3] = mvx / m; s_c[4] = mvy / m; s_c[5] = mvz / m;
    s_c[6] = (double)(ii - b0);
  }
  __syncthreads();
  if (A.cdm && b1 > b0) {
    // the member closest to the centre of mass (CHP:917-934)
    const double px = wrap_abs(cmx / m + fx, A.L, A.h, A.periodic);
    const double py = wrap_abs(cmy / m + fy, A.L, A.h, A.periodic);
    const double pz = wrap_abs(cmz / m + fz, A.L, A.h, A.periodic);
    double bdd = DBL_MAX;
    long long bii = LLONG_MAX;
    for (int64_t i = b0 + tid; i < b1; i += kPB) {
      const double dx = wrap_chp(A.pos[3 * i] - px, A.L, A.h, A.periodic);
      const double dy = wrap_chp(A.pos[3 * i + 1] - py, A.L, A.h, A.periodic);
      const double dz = wrap_chp(A.pos[3 * i + 2] - pz, A.L, A.h, A.periodic);
      const double dd = dx * dx + dy * dy + dz * dz;
      if (dd < bdd || (dd == bdd && i < bii)) { bdd = dd; bii = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double od = __shfl_xor_sync(0xffffffffu, bdd, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, bii, o);
      if (od < bdd || (od == bdd && oi < bii)) { bdd = od; bii = oi; }
    }
    if ((tid & 31) == 0) { s_best_d[tid >> 5] = bdd; s_best_i[tid >> 5] = bii; }
    __syncthreads();
    if (tid == 0) {
      double d = s_best_d[0];
      long long ii = s_best_i[0];
      for (int w = 1; w < kPB / 32; ++w)
        if (s_best_d[w] < d || (s_best_d[w] == d && s_best_i[w] < ii)) { d = s_best_d[w]; ii = s_best_i[w]; }
      s_c[0] = A.pos[3 * ii]; s_c[1] = A.pos[3 * ii + 1]; s_c[2] = A.pos[3 * ii + 2];
      s_c[6] = (double)(ii - b0);
    }
    __syncthreads();
  }
  if (A.sc) shrink_sphere_centre(A, b0, b1, s_c, sh, s_best_d, s_best_i);
  const double cx = s_c[0], cy = s_c[1], cz = s_c[2], vx = s_c[3], vy = s_c[4], vz = s_c[5];
  // pass 2
  double Lx = 0, Ly = 0, Lz = 0, r2max = 0, Ixx = 0, Ixy = 0, Ixz = 0, Iyy = 0, Iyz = 0, Izz = 0, ek = 0, sg = 0;
  double sgd = 0, sgs = 0;
  for (int64_t i = b0 + tid; i < b1; i += kPB) {
    const double w = A.mass[i];
    const double dx = wrap_chp(A.pos[3 * i] - cx, A.L, A.h, A.periodic);
    const double dy = wrap_chp(A.pos[3 * i + 1] - cy, A.L, A.h, A.periodic);
    const double dz = wrap_chp(A.pos[3 * i + 2] - cz, A.L, A.h, A.periodic);
    const double ux = A.vel[3 * i] - vx, uy = A.vel[3 * i + 1] - vy, uz = A.vel[3 * i + 2] - vz;
    const double px = w * ux, py = w * uy, pz = w * uz;
    Lx += dy * pz - dz * py;
    Ly += dz * px - dx * pz;
    Lz += dx * py - dy * px;
    r2max = fmax(r2max, dx * dx + dy * dy + dz * dz);
    Ixx += w * dx * dx; Ixy += w * dx * dy; Ixz += w * dx * dz;
    Iyy += w * dy * dy; Iyz += w * dy * dz; Izz += w * dz * dz;
    const double tx = ux + dx * A.hub, ty = uy + dy * A.hub, tz = uz + dz * A.hub;
    ek += w * (tx * tx + ty * ty + tz * tz);
    const double dv2 = w * (ux * ux + uy * uy + uz * uz);
    sg += dv2;
    if (member_is_dm(A, i)) sgd += dv2;
    else sgs += dv2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2max = fmax(r2max, __shfl_xor_sync(0xffffffffu, r2max, o));
  if ((tid & 31) == 0) s_best_d[tid >> 5] = r2max;
  Lx = block_sum(Lx, sh); Ly = block_sum(Ly, sh); Lz = block_sum(Lz, sh);
  Ixx = block_sum(Ixx, sh); Ixy = block_sum(Ixy, sh); Ixz = block_sum(Ixz, sh);
  Iyy = block_sum(Iyy, sh); Iyz = block_sum(Iyz, sh); Izz = block_sum(Izz, sh);
  ek = block_sum(ek, sh);
  sg = block_sum(sg, sh);
  sgd = block_sum(sgd, sh);
  sgs = block_sum(sgs, sh);
  if (tid == 0) {
    double rm = s_best_d[0];
    for (int w = 1; w < kPB / 32; ++w) rm = fmax(rm, s_best_d[w]);
    double* o = A.out + (size_t)kHaloFields * h;
    o[HP_M] = m;
    o[HP_PX] = cx; o[HP_PY] = cy; o[HP_PZ] = cz;
    o[HP_VX] = vx; o[HP_VY] = vy; o[HP_VZ] = vz;
    o[HP_LX] = Lx; o[HP_LY] = Ly; o[HP_LZ] = Lz;
    o[HP_R] = sqrt(rm);
    o[HP_IXX] = Ixx; o[HP_IXY] = Ixy; o[HP_IXZ] = Ixz; o[HP_IYY] = Iyy; o[HP_IYZ] = Iyz; o[HP_IZZ] = Izz;
    o[HP_EK] = 0.5 * ek;
    o[HP_SIGMA] = sqrt(sg / m);
    o[HP_ICENTER] = s_c[6];
    o[HP_MDM] = mdm; o[HP_MSTAR] = mst; o[HP_NDM] = ndm; o[HP_NSTAR] = nst; o[HP_MCONTAM] = mcon;
    o[HP_SIGMA_DM] = mdm > 0 ? sqrt(sgd / mdm) : 0.0;
    o[HP_SIGMA_STAR] = mst > 0 ? sqrt(sgs / mst) : 0.0;
  }
}

// ------------------------------------------------- chunked moment passes
// The same two passes as halo_moments_kernel with every halo cut into chunks
// of kMomChunk members, one block per chunk, so a halo of a million members
// no longer runs on one block.  Chunk partials are folded per halo in chunk
// order (deterministic); the densest member is an exact argmax, so the centre
// is the one the single-block kernel finds.
constexpr int64_t kMomChunk = 8192;

struct MomChunk {
  int32_t h, pad;
  int64_t b0, b1;
};
// pass 1 sums: mass, momentum, the dark-matter / star split of det_mass_17
// (CHP:766-780) and the mass-weighted offsets from the halo's first member
// that det_center_18's centre of mass starts from (CHP:920-926)
constexpr int kP1 = 12;  // m mvx mvy mvz mdm mstar ndm nstar mcontam cmx cmy cmz
struct MomP1 {
  double v[kP1];
  double bd;
  long long bi;
};
constexpr int kP2 = 13;  // Lx Ly Lz Ixx Ixy Ixz Iyy Iyz Izz ek sg sg_dm sg_star
struct MomP2 {
  double v[kP2];
  double r2max;
};
struct MomCentre {
  double c[6];  // centre x, y, z, bulk velocity x, y, z
  long long ic; // centre member (absolute index)
  double cm[3]; // centre of mass (cdm)
};
struct MomArg {  // chunk argmin of the distance to the centre of mass (cdm)
  double d;
  long long i;
};

// Sums of N values over the block (warp shuffles, then warp 0 over the
// warps in order); the totals land in every thread's v.
template <int N>
__device__ __forceinline__ void block_sum_n(double (&v)[N], double* sh) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane == 0) sh[k * (kPB / 32) + w] = v[k];
  }
  __syncthreads();
  if (tid < N) {
    double s = sh[tid * (kPB / 32)];
    for (int j = 1; j < kPB / 32; ++j) s += sh[tid * (kPB / 32) + j];
    sh[N * (kPB / 32) + tid] = s;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = sh[N * (kPB / 32) + k];
  __syncthreads();
}

__global__ void __launch_bounds__(kPB) mom_pass1_kernel(HaloArgs A, const MomChunk* __restrict__ ch,
                                                        MomP1* __restrict__ P) {
  __shared__ double sh[(kP1 + 1) * (kPB / 32) + 16];
  __shared__ double s_bd[kPB / 32];
  __shared__ long long s_bi[kPB / 32];
  const int tid = threadIdx.x;
  const MomChunk c = ch[blockIdx.x];
  double v[kP1] = {}, bd = -DBL_MAX;
  long long bi = LLONG_MAX;
  const int64_t first = A.off[c.h];
  const double fx = A.pos[3 * first], fy = A.pos[3 * first + 1], fz = A.pos[3 * first + 2];
  const double heavy = A.massp * 1.00001;
  for (int64_t i = c.b0 + tid; i < c.b1; i += kPB) {
    const double w = A.mass[i];
    v[0] += w;
    v[1] += w * A.vel[3 * i];
    v[2] += w * A.vel[3 * i + 1];
    v[3] += w * A.vel[3 * i + 2];
    if (member_is_dm(A, i)) {
      v[4] += w;
      v[6] += 1.0;
      if (w > heavy) v[8] += w;
    } else {
      v[5] += w;
      v[7] += 1.0;
    }
    if (A.cdm) {
      v[9] += w * wrap_chp(A.pos[3 * i] - fx, A.L, A.h, A.periodic);
      v[10] += w * wrap_chp(A.pos[3 * i + 1] - fy, A.L, A.h, A.periodic);
      v[11] += w * wrap_chp(A.pos[3 * i + 2] - fz, A.L, A.h, A.periodic);
    }
    const double d = A.dens[i];
    if (d > bd || (d == bd && i < bi)) { bd = d; bi = i; }  // np.argmax: first maximum
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bd, o);
    const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (od > bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
  }
  if ((tid & 31) == 0) { s_bd[tid >> 5] = bd; s_bi[tid >> 5] = bi; }
  block_sum_n<kP1>(v, sh);
  if (tid == 0) {
    bd = s_bd[0]; bi = s_bi[0];
    for (int w = 1; w < kPB / 32; ++w)
      if (s_bd[w] > bd || (s_bd[w] == bd && s_bi[w] < bi)) { bd = s_bd[w]; bi = s_bi[w]; }
    MomP1 r;
#pragma unroll
    for (int k = 0; k < kP1; ++k) r.v[k] = v[k];
    r.bd = bd;
    r.bi = bi;
    P[blockIdx.x] = r;
  }
}

// per halo: chunk partials in order -> mass, bulk velocity, densest member
__global__ void mom_fold1_kernel(HaloArgs A, const int64_t* __restrict__ hcoff, const MomP1* __restrict__ P,
                                 MomCentre* __restrict__ C, int64_t nhalo) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  double v[kP1] = {}, bd = -DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t k = hcoff[h]; k < hcoff[h + 1]; ++k) {
    const MomP1& p = P[k];
#pragma unroll
    for (int j = 0; j < kP1; ++j) v[j] += p.v[j];
    if (p.bd > bd || (p.bd == bd && p.bi < bi)) { bd = p.bd; bi = p.bi; }
  }
  const double m = v[0];
  MomCentre c;
  if (bi != LLONG_MAX) {
    c.c[0] = A.pos[3 * bi]; c.c[1] = A.pos[3 * bi + 1]; c.c[2] = A.pos[3 * bi + 2];
  } else {
    c.c[0] = c.c[1] = c.c[2] = 0.0;
  }
  c.c[3] = v[1] / m; c.c[4] = v[2] / m; c.c[5] = v[3] / m;
  c.ic = bi;
  c.cm[0] = c.cm[1] = c.cm[2] = 0.0;
  const int64_t first = A.off[h];
  if (A.cdm && A.off[h + 1] > first) {
    // centre of mass about the first member, then wrapped (CHP:920-927)
    c.cm[0] = wrap_abs(v[9] / m + A.pos[3 * first], A.L, A.h, A.periodic);
    c.cm[1] = wrap_abs(v[10] / m + A.pos[3 * first + 1], A.L, A.h, A.periodic);
    c.cm[2] = wrap_abs(v[11] / m + A.pos[3 * first + 2], A.L, A.h, A.periodic);
  }
  C[h] = c;
  double* o = A.out + (size_t)kHaloFields * h;
  o[HP_M] = m;
  o[HP_MDM] = v[4]; o[HP_MSTAR] = v[5]; o[HP_NDM] = v[6]; o[HP_NSTAR] = v[7]; o[HP_MCONTAM] = v[8];
}

// cdm: per chunk, the member closest to the halo's centre of mass
// (np.argmin: first minimum, CHP:929-934)
__global__ void __launch_bounds__(kPB) mom_cdm_kernel(HaloArgs A, const MomChunk* __restrict__ ch,
                                                      const MomCentre* __restrict__ C, MomArg* __restrict__ P) {
  __shared__ double s_bd[kPB / 32];
  __shared__ long long s_bi[kPB / 32];
  const int tid = threadIdx.x;
  const MomChunk k = ch[blockIdx.x];
  const double* cm = C[k.h].cm;
  double bd = DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t i = k.b0 + tid; i < k.b1; i += kPB) {
    const double dx = wrap_chp(A.pos[3 * i] - cm[0], A.L, A.h, A.periodic);
    const double dy = wrap_chp(A.pos[3 * i + 1] - cm[1], A.L, A.h, A.periodic);
    const double dz = wrap_chp(A.pos[3 * i + 2] - cm[2], A.L, A.h, A.periodic);
    const double d = dx * dx + dy * dy + dz * dz;
    if (d < bd || (d == bd && i < bi)) { bd = d; bi = i; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bd, o);
    const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (od < bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
  }
  if ((tid & 31) == 0) { s_bd[tid >> 5] = bd; s_bi[tid >> 5] = bi; }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < kPB / 32; ++w)
      if (s_bd[w] < s_bd[0] || (s_bd[w] == s_bd[0] && s_bi[w] < s_bi[0])) { s_bd[0] = s_bd[w]; s_bi[0] = s_bi[w]; }
    P[blockIdx.x] = MomArg{s_bd[0], s_bi[0]};
  }
}

__global__ void mom_cdm_fold_kernel(HaloArgs A, const int64_t* __restrict__ hcoff, const MomArg* __restrict__ P,
                                    MomCentre* __restrict__ C, int64_t nhalo) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  double bd = DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t k = hcoff[h]; k < hcoff[h + 1]; ++k)
    if (P[k].d < bd || (P[k].d == bd && P[k].i < bi)) { bd = P[k].d; bi = P[k].i; }
  if (bi == LLONG_MAX) return;
  C[h].c[0] = A.pos[3 * bi]; C[h].c[1] = A.pos[3 * bi + 1]; C[h].c[2] = A.pos[3 * bi + 2];
  C[h].ic = bi;
}

// shrinking-sphere refinement (SC on): one block per halo, as in the
// single-block kernel
__global__ void __launch_bounds__(kPB) mom_sc_kernel(HaloArgs A, MomCentre* __restrict__ C) {
  __shared__ double sh[kPB / 32];
  __shared__ double s_best_d[kPB / 32];
  __shared__ long long s_best_i[kPB / 32];
  __shared__ double s_c[7];
  const int64_t h = blockIdx.x;
  const int64_t b0 = A.off[h], b1 = A.off[h + 1];
  if (b1 <= b0) return;
  if (threadIdx.x < 6) s_c[threadIdx.x] = C[h].c[threadIdx.x];
  if (threadIdx.x == 6) s_c[6] = (double)(C[h].ic - b0);
  __syncthreads();
  shrink_sphere_centre(A, b0, b1, s_c, sh, s_best_d, s_best_i);
  if (threadIdx.x < 3) C[h].c[threadIdx.x] = s_c[threadIdx.x];
  if (threadIdx.x == 0) C[h].ic = b0 + (long long)s_c[6];
}

__global__ void __launch_bounds__(kPB) mom_pass2_kernel(HaloArgs A, const MomChunk* __restrict__ ch,
                                                        const MomCentre* __restrict__ C, MomP2* __restrict__ P) {
  __shared__ double sh[(kP2 + 1) * (kPB / 32) + 16];
  __shared__ double s_r[kPB / 32];
  const int tid = threadIdx.x;
  const MomChunk k = ch[blockIdx.x];
  const MomCentre c = C[k.h];
  const double cx = c.c[0], cy = c.c[1], cz = c.c[2], vx = c.c[3], vy = c.c[4], vz = c.c[5];
  double v[kP2] = {};
  double r2max = 0;
  for (int64_t i = k.b0 + tid; i < k.b1; i += kPB) {
    const double w = A.mass[i];
    const double dx = wrap_chp(A.pos[3 * i] - cx, A.L, A.h, A.periodic);
    const double dy = wrap_chp(A.pos[3 * i + 1] - cy, A.L, A.h, A.periodic);
    const double dz = wrap_chp(A.pos[3 * i + 2] - cz, A.L, A.h, A.periodic);
    const double ux = A.vel[3 * i] - vx, uy = A.vel[3 * i + 1] - vy, uz = A.vel[3 * i + 2] - vz;
    const double px = w * ux, py = w * uy, pz = w * uz;
    v[0] += dy * pz - dz * py;
    v[1] += dz * px - dx * pz;
    v[2] += dx * py - dy * px;
    r2max = fmax(r2max, dx * dx + dy * dy + dz * dz);
    v[3] += w * dx * dx; v[4] += w * dx * dy; v[5] += w * dx * dz;
    v[6] += w * dy * dy; v[7] += w * dy * dz; v[8] += w * dz * dz;
    const double tx = ux + dx * A.hub, ty = uy + dy * A.hub, tz = uz + dz * A.hub;
    v[9] += w * (tx * tx + ty * ty + tz * tz);
    const double dv2 = w * (ux * ux + uy * uy + uz * uz);
    v[10] += dv2;
    v[member_is_dm(A, i) ? 11 : 12] += dv2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2max = fmax(r2max, __shfl_xor_sync(0xffffffffu, r2max, o));
  if ((tid & 31) == 0) s_r[tid >> 5] = r2max;
  block_sum_n<kP2>(v, sh);
  if (tid == 0) {
    double rm = s_r[0];
    for (int w = 1; w < kPB / 32; ++w) rm = fmax(rm, s_r[w]);
    MomP2 p;
#pragma unroll
    for (int j = 0; j < kP2; ++j) p.v[j] = v[j];
    p.r2max = rm;
    P[blockIdx.x] = p;
  }
}

__global__ void mom_fold2_kernel(HaloArgs A, const int64_t* __restrict__ hcoff, const MomP2* __restrict__ P,
                                 const MomCentre* __restrict__ C, int64_t nhalo) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  double v[kP2] = {};
  double rm = 0;
  for (int64_t k = hcoff[h]; k < hcoff[h + 1]; ++k) {
#pragma unroll
    for (int j = 0; j < kP2; ++j) v[j] += P[k].v[j];
    rm = fmax(rm, P[k].r2max);
  }
  const MomCentre c = C[h];
  double* o = A.out + (size_t)kHaloFields * h;
  const double m = o[HP_M];
  o[HP_PX] = c.c[0]; o[HP_PY] = c.c[1]; o[HP_PZ] = c.c[2];
  o[HP_VX] = c.c[3]; o[HP_VY] = c.c[4]; o[HP_VZ] = c.c[5];
  o[HP_LX] = v[0]; o[HP_LY] = v[1]; o[HP_LZ] = v[2];
  o[HP_R] = sqrt(rm);
  o[HP_IXX] = v[3]; o[HP_IXY] = v[4]; o[HP_IXZ] = v[5]; o[HP_IYY] = v[6]; o[HP_IYZ] = v[7]; o[HP_IZZ] = v[8];
  o[HP_EK] = 0.5 * v[9];
  o[HP_SIGMA] = sqrt(v[10] / m);
  o[HP_ICENTER] = (double)(c.ic - A.off[h]);
  // det_center_18, mode 'full' (CHP:962-966)
  o[HP_SIGMA_DM] = o[HP_MDM] > 0 ? sqrt(v[11] / o[HP_MDM]) : 0.0;
  o[HP_SIGMA_STAR] = o[HP_MSTAR] > 0 ? sqrt(v[12] / o[HP_MSTAR]) : 0.0;
}

// ---------------------------------------------------------------- pair sums
// Work item: member rows [i0, i0 + rows) of halo h against partners
// j in [j0, j1), j > i.  j0 is either i0 (the item holds the diagonal tile) or
// i0 plus a multiple of the row count, so partner tiles line up with the row
// tile.  A halo's items cover every pair once; item partials are folded per
// halo in halo order by epot_finalize_kernel, so the result does not depend on
// the schedule.
struct PairItem {
  int32_t h, i0, j0, j1;
};

constexpr int kT64 = 256;  // FP64 form: rows per item = threads per block = partner tile

__device__ __forceinline__ void rel_pos(const HaloArgs& A, int64_t k, double cx, double cy, double cz,
                                        double& rx, double& ry, double& rz) {
  rx = wrap_chp(A.pos[3 * k] - cx, A.L, A.h, A.periodic);
  ry = wrap_chp(A.pos[3 * k + 1] - cy, A.L, A.h, A.periodic);
  rz = wrap_chp(A.pos[3 * k + 2] - cz, A.L, A.h, A.periodic);
}

// Plain FP64 form: relative positions, 1/r from the double reciprocal square
// root, one row per thread, partner tiles of 256 in shared memory.
__global__ void __launch_bounds__(kT64) epot64_kernel(HaloArgs A, const PairItem* __restrict__ items,
                                                      int32_t nitems, int32_t* __restrict__ counter,
                                                      double* __restrict__ part) {
  __shared__ double s_dx[kT64], s_dy[kT64], s_dz[kT64], s_dm[kT64];
  __shared__ double sh[kT64 / 32];
  __shared__ int32_t s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int32_t w = s_item;
    __syncthreads();
    if (w >= nitems) break;
    const PairItem it = items[w];
    const int64_t base = A.off[it.h];
    const int32_t n = (int32_t)(A.off[it.h + 1] - base);
    const double* c = A.out + (size_t)kHaloFields * it.h;
    const double cx = c[HP_PX], cy = c[HP_PY], cz = c[HP_PZ];
    const int32_t i = it.i0 + tid;
    const bool vi = i < n;
    double rxi = 0, ryi = 0, rzi = 0;
    if (vi) rel_pos(A, base + i, cx, cy, cz, rxi, ryi, rzi);
    double ds = 0.0;
    for (int32_t j0 = it.j0; j0 < it.j1; j0 += kT64) {
      const int32_t j = j0 + tid;
      if (j < it.j1) {
        double rx, ry, rz;
        rel_pos(A, base + j, cx, cy, cz, rx, ry, rz);
        s_dx[tid] = rx; s_dy[tid] = ry; s_dz[tid] = rz; s_dm[tid] = A.mass[base + j];
      } else {
        s_dm[tid] = 0.0; s_dx[tid] = s_dy[tid] = s_dz[tid] = 3.0e30;
      }
      __syncthreads();
      if (vi) {
        const int jstart = (j0 == it.i0) ? tid + 1 : 0;  // j > i on the diagonal tile
        const int jend = min(kT64, it.j1 - j0);
#pragma unroll 4
        for (int jj = jstart; jj < jend; ++jj) {
          const double dx = s_dx[jj] - rxi, dy = s_dy[jj] - ryi, dz = s_dz[jj] - rzi;
          const double r2 = dx * dx + dy * dy + dz * dz;
          if (r2 > 0.0) ds += s_dm[jj] * rsqrt(r2);
        }
      }
      __syncthreads();
    }
    const double tot = block_sum(vi ? A.mass[base + i] * ds : 0.0, sh);
    if (tid == 0) part[w] = tot;
  }
}

// FP32-compensated form on packed FP32 pairs (the sm_100 f32x2 add/sub/mul/fma
// instructions: two lanes per 64-bit register, one instruction).
//
// Members are read in the Morton order of their position about the halo
// centre (sort32_* kernels below), so a run of consecutive members is a
// compact region.  Every item takes an origin o, the centre of its rows' box,
// and expresses rows and partners relative to it, split into hi = float(b)
// and lo = float(b - hi).  Two pair forms:
//   * near: separation (hi_j - hi_i) + (lo_j - lo_i) per axis (9 operations
//     per pair for the three axes);
//   * far: separation hi_j - hi_i (3 operations).  Its error per axis is at
//     most 2^-24 (|a_i| + |b_j| + |d|) (the roundings of both hi values and of
//     the difference), so relative to the separation d it is at most
//     2^-24 (K + 1) with K = (|a_i| + |b_j|) / |d|.  A warp takes the far form
//     for a group of 32 partners when K <= kFarK = 4 holds for every pair of
//     its rows with that group, from boxes: K <= (rho_w + beta_g) / dist,
//     rho_w = the largest |a_i| of the warp's rows, beta_g = the largest |b_j|
//     of the group, dist = the distance between the rows' box and the group's
//     box.  The far form thus adds at most 5 * 2^-24 = 3.0e-7 relative error
//     to a pair's 1/r; every term of the sum is positive, so the halo's sum
//     keeps that bound.
// The two lanes of every packed register hold two partners j, 2q and 2q+1, of
// the same row i, so a row's own coordinates are loop-invariant (hi_i, hi_i)
// pairs.  Each thread owns R rows; the warp's rows are 32 R consecutive
// members.  Partner tiles are 128 R wide, shared memory holds them as packed
// pairs.  For every row, sixteen partner pairs (32 terms) are accumulated by a
// fused multiply-add chain per lane, then enter a Kahan-compensated FP32 sum;
// rows fold into FP64 per item.  Separations of exactly zero (coincident
// members) are excluded like in the FP64 form: the fast loops do not test for
// them -- rsqrt(0) = inf makes the row's sum non-finite, and the block then
// recomputes the item with a per-pair test.  The tile shape (R = 1, 2 or 4
// rows per thread) is chosen per halo-size bucket by the host-side autotuner
// and read per item.
typedef unsigned long long f2_t;

__device__ __forceinline__ f2_t f2_pack(float a, float b) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2_t v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
  f2_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
  f2_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
  f2_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
  f2_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr int kB32 = 128;              // threads per block of the FP32 form
constexpr int kMaxR32 = 4;             // rows per thread, largest shape
constexpr int kMaxT32 = kB32 * kMaxR32;
constexpr int kGroup32 = 16;           // partner pairs per compensated fold (= one bound group of 32 partners)
constexpr int kChunkJ = 32768;         // partners per item at most (a multiple of every tile width)
constexpr float kFar = 1.0e18f;        // padding position: its terms vanish (mass 0, finite r)
// far form when (rho_w + beta_g)^2 <= kFarK^2 dist^2; the factor below 16
// covers the FP32 roundings of that test (a few 2^-24 relative)
constexpr float kFarK2 = 16.0f * (1.0f - 1.0e-4f);

struct Tile32 {
  float4 a[kMaxT32 / 2];  // hi x(2q), x(2q+1), y(2q), y(2q+1)
  float4 b[kMaxT32 / 2];  // hi z(2q), z(2q+1), mass(2q), mass(2q+1)
  float4 c[kMaxT32 / 2];  // lo x, x, y, y
  float2 d[kMaxT32 / 2];  // lo z, z
  float4 glo[kMaxT32 / 32];  // per group of 32 partners: box low corner (x, y, z), largest |b| (w)
  float4 ghi[kMaxT32 / 32];  // box high corner
};

__device__ __forceinline__ void split_hilo(double r, float& hi, float& lo) {
  hi = (float)r;
  lo = (float)(r - (double)hi);
}

// Member k relative to the halo centre, and its mass: from the Morton-sorted
// copy when there is one, else from the caller's arrays.
__device__ __forceinline__ void member_rel(const HaloArgs& A, int64_t k, double cx, double cy, double cz, double& rx,
                                           double& ry, double& rz, double& m) {
  if (A.srel) {
    const double4 v = A.srel[k];
    rx = v.x; ry = v.y; rz = v.z; m = v.w;
  } else {
    rel_pos(A, k, cx, cy, cz, rx, ry, rz);
    m = A.mass[k];
  }
}

// |v| rounded up to float (the double norm's own rounding is covered by the
// 1e-12 widening).
__device__ __forceinline__ float norm_ru(double x, double y, double z) {
  return __double2float_ru(sqrt(x * x + y * y + z * z) * (1.0 + 1e-12));
}

// Stage partners [j0, j0 + T) (T = 128 R) of one item relative to the origin
// o, with the box and radius bound of every group of 32; slots past j1 get the
// padding (mass 0, far away) and stay out of the bounds.
template <int R>
__device__ __forceinline__ void stage_tile32(Tile32& S, const HaloArgs& A, int64_t base, int32_t j0, int32_t j1,
                                             double cx, double cy, double cz, double ox, double oy, double oz) {
  constexpr int P = kB32 * R / 2;  // a multiple of 32: a warp is in or out of an iteration as a whole
  for (int q = threadIdx.x; q < P; q += kB32) {
    float hx[2], hy[2], hz[2], m[2], lx[2], ly[2], lz[2];
    float blx = FLT_MAX, bly = FLT_MAX, blz = FLT_MAX, bhx = -FLT_MAX, bhy = -FLT_MAX, bhz = -FLT_MAX, bm = 0.f;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const int32_t j = j0 + 2 * q + l;
      if (j < j1) {
        double rx, ry, rz, mm;
        member_rel(A, base + j, cx, cy, cz, rx, ry, rz, mm);
        const double bx = rx - ox, by = ry - oy, bz = rz - oz;
        split_hilo(bx, hx[l], lx[l]);
        split_hilo(by, hy[l], ly[l]);
        split_hilo(bz, hz[l], lz[l]);
        m[l] = (float)mm;
        blx = fminf(blx, __double2float_rd(bx)); bhx = fmaxf(bhx, __double2float_ru(bx));
        bly = fminf(bly, __double2float_rd(by)); bhy = fmaxf(bhy, __double2float_ru(by));
        blz = fminf(blz, __double2float_rd(bz)); bhz = fmaxf(bhz, __double2float_ru(bz));
        bm = fmaxf(bm, norm_ru(bx, by, bz));
      } else {
        hx[l] = hy[l] = hz[l] = kFar;
        lx[l] = ly[l] = lz[l] = 0.f;
        m[l] = 0.f;
      }
    }
    S.a[q] = make_float4(hx[0], hx[1], hy[0], hy[1]);
    S.b[q] = make_float4(hz[0], hz[1], m[0], m[1]);
    S.c[q] = make_float4(lx[0], lx[1], ly[0], ly[1]);
    S.d[q] = make_float2(lz[0], lz[1]);
    // the 16 lanes of a half warp stage one group of 32 partners
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      blx = fminf(blx, __shfl_xor_sync(0xffffffffu, blx, o));
      bly = fminf(bly, __shfl_xor_sync(0xffffffffu, bly, o));
      blz = fminf(blz, __shfl_xor_sync(0xffffffffu, blz, o));
      bhx = fmaxf(bhx, __shfl_xor_sync(0xffffffffu, bhx, o));
      bhy = fmaxf(bhy, __shfl_xor_sync(0xffffffffu, bhy, o));
      bhz = fmaxf(bhz, __shfl_xor_sync(0xffffffffu, bhz, o));
      bm = fmaxf(bm, __shfl_xor_sync(0xffffffffu, bm, o));
    }
    if ((q & 15) == 0) {
      S.glo[q >> 4] = make_float4(blx, bly, blz, bm);
      S.ghi[q >> 4] = make_float4(bhx, bhy, bhz, 0.f);
    }
  }
}

__device__ __forceinline__ void kahan_add(float t, float& ks, float& kc) {
  const float y = t - kc;
  const float s2 = ks + y;
  kc = (s2 - ks) - y;
  ks = s2;
}

// One partner (tile slot jj) of one row with the zero-separation test; the
// per-pair path of the diagonal tile and of the recomputation.
__device__ __forceinline__ void pair_checked(const Tile32& S, int jj, float hx, float hy, float hz, float lx,
                                             float ly, float lz, float& ks, float& kc) {
  const int q = jj >> 1, l = jj & 1;
  const float* a = reinterpret_cast<const float*>(&S.a[q]);
  const float* b = reinterpret_cast<const float*>(&S.b[q]);
  const float* c = reinterpret_cast<const float*>(&S.c[q]);
  const float* d = reinterpret_cast<const float*>(&S.d[q]);
  const float dx = (a[l] - hx) + (c[l] - lx);
  const float dy = (a[2 + l] - hy) + (c[2 + l] - ly);
  const float dz = (b[l] - hz) + (d[l] - lz);
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  if (r2 > 0.f) kahan_add(b[2 + l] * rsqrtf(r2), ks, kc);
}

__device__ __forceinline__ void warp_minmax_f(float& lo, float& hi) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
}

// sred: 6 * (kB32 / 32) doubles of shared scratch for the origin.
template <int R>
__device__ double epot32_item(Tile32& S, double* sh, double* sred, const HaloArgs& A, const PairItem& it,
                              bool checked) {
  constexpr int T = kB32 * R;
  constexpr int NW = kB32 / 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int64_t base = A.off[it.h];
  const int32_t n = (int32_t)(A.off[it.h + 1] - base);
  const double* cen = A.out + (size_t)kHaloFields * it.h;
  const double cx = cen[HP_PX], cy = cen[HP_PY], cz = cen[HP_PZ];
  // rows: warp w owns the 32 R consecutive rows [32 R w, 32 R (w + 1)) of the
  // item; they are read twice (for the origin, then relative to it) rather
  // than held in registers across the block reduction
  bool vi[R];
  double lo3[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi3[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int32_t i = it.i0 + 32 * R * wid + lane + 32 * r;
    vi[r] = i < n;
    if (vi[r]) {
      double rx, ry, rz, mm;
      member_rel(A, base + i, cx, cy, cz, rx, ry, rz, mm);
      lo3[0] = fmin(lo3[0], rx); hi3[0] = fmax(hi3[0], rx);
      lo3[1] = fmin(lo3[1], ry); hi3[1] = fmax(hi3[1], ry);
      lo3[2] = fmin(lo3[2], rz); hi3[2] = fmax(hi3[2], rz);
    }
  }
  // origin: centre of the box of the item's rows
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo3[k] = fmin(lo3[k], __shfl_xor_sync(0xffffffffu, lo3[k], o));
      hi3[k] = fmax(hi3[k], __shfl_xor_sync(0xffffffffu, hi3[k], o));
    }
    if (lane == 0) { sred[k * NW + wid] = lo3[k]; sred[(3 + k) * NW + wid] = hi3[k]; }
  }
  __syncthreads();
  double o3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double l = sred[k * NW], h = sred[(3 + k) * NW];
    for (int w = 1; w < NW; ++w) { l = fmin(l, sred[k * NW + w]); h = fmax(h, sred[(3 + k) * NW + w]); }
    o3[k] = 0.5 * (l + h);
  }
  const double ox = o3[0], oy = o3[1], oz = o3[2];
  f2_t HX[R], HY[R], HZ[R], LX[R], LY[R], LZ[R], ks[R], kc[R];
  float ksd[R], kcd[R];  // per-pair path sums
  // the warp's rows: box and radius bound about o (rounded outwards)
  float wlx = FLT_MAX, wly = FLT_MAX, wlz = FLT_MAX, whx = -FLT_MAX, why = -FLT_MAX, whz = -FLT_MAX, wrho = 0.f;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float hx, hy, hz, lx, ly, lz;
    if (vi[r]) {
      double rx, ry, rz, mm;
      member_rel(A, base + it.i0 + 32 * R * wid + lane + 32 * r, cx, cy, cz, rx, ry, rz, mm);
      const double bx = rx - ox, by = ry - oy, bz = rz - oz;
      split_hilo(bx, hx, lx);
      split_hilo(by, hy, ly);
      split_hilo(bz, hz, lz);
      wlx = fminf(wlx, __double2float_rd(bx)); whx = fmaxf(whx, __double2float_ru(bx));
      wly = fminf(wly, __double2float_rd(by)); why = fmaxf(why, __double2float_ru(by));
      wlz = fminf(wlz, __double2float_rd(bz)); whz = fmaxf(whz, __double2float_ru(bz));
      wrho = fmaxf(wrho, norm_ru(bx, by, bz));
    } else {
      // far on the other side from the padding: every separation stays finite
      hx = hy = hz = -kFar;
      lx = ly = lz = 0.f;
    }
    HX[r] = f2_pack(hx, hx); HY[r] = f2_pack(hy, hy); HZ[r] = f2_pack(hz, hz);
    LX[r] = f2_pack(lx, lx); LY[r] = f2_pack(ly, ly); LZ[r] = f2_pack(lz, lz);
    ks[r] = kc[r] = 0ull;
    ksd[r] = kcd[r] = 0.f;
  }
  warp_minmax_f(wlx, whx);
  warp_minmax_f(wly, why);
  warp_minmax_f(wlz, whz);
  float dummy = 0.f;
  warp_minmax_f(dummy, wrho);
  // a warp without rows takes the far form: its sums are discarded
  const bool wvalid = whx >= wlx;
  for (int32_t j0 = it.j0; j0 < it.j1; j0 += T) {
    stage_tile32<R>(S, A, base, j0, it.j1, cx, cy, cz, ox, oy, oz);
    __syncthreads();
    const int jend = min(T, it.j1 - j0);
    if (j0 == it.i0 || checked) {
      // per-pair path: j > i on the diagonal tile, every pair when recomputing
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!vi[r]) continue;
        const int jstart = (j0 == it.i0) ? 32 * R * wid + lane + 32 * r + 1 : 0;
        float hx, hy, hz, lx, ly, lz, t;
        f2_unpack(HX[r], hx, t); f2_unpack(HY[r], hy, t); f2_unpack(HZ[r], hz, t);
        f2_unpack(LX[r], lx, t); f2_unpack(LY[r], ly, t); f2_unpack(LZ[r], lz, t);
        for (int jj = jstart; jj < jend; ++jj) pair_checked(S, jj, hx, hy, hz, lx, ly, lz, ksd[r], kcd[r]);
      }
    } else {
      const int np = ((jend + 2 * kGroup32 - 1) / (2 * kGroup32)) * kGroup32;  // partner pairs, padded
      const ulonglong2* Sa = reinterpret_cast<const ulonglong2*>(S.a);
      const ulonglong2* Sb = reinterpret_cast<const ulonglong2*>(S.b);
      const ulonglong2* Sc = reinterpret_cast<const ulonglong2*>(S.c);
      const f2_t* Sd = reinterpret_cast<const f2_t*>(S.d);
      for (int q0 = 0; q0 < np; q0 += kGroup32) {
        const float4 gl = S.glo[q0 / kGroup32], gh = S.ghi[q0 / kGroup32];
        const float gx = fmaxf(0.f, fmaxf(gl.x - whx, wlx - gh.x));
        const float gy = fmaxf(0.f, fmaxf(gl.y - why, wly - gh.y));
        const float gz = fmaxf(0.f, fmaxf(gl.z - whz, wlz - gh.z));
        const float dist2 = gx * gx + gy * gy + gz * gz;
        const float num = wrho + gl.w;
        const bool far = !wvalid || (dist2 > 0.f && num * num <= kFarK2 * dist2);
        f2_t acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0ull;
        if (far) {
#pragma unroll
          for (int g = 0; g < kGroup32; ++g) {
            const ulonglong2 pa = Sa[q0 + g], pb = Sb[q0 + g];
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const f2_t dx = f2_sub(pa.x, HX[r]);
              const f2_t dy = f2_sub(pa.y, HY[r]);
              const f2_t dz = f2_sub(pb.x, HZ[r]);
              const f2_t r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
              float u, v;
              f2_unpack(r2, u, v);
              acc[r] = f2_fma(pb.y, f2_pack(rsqrt_ftz(u), rsqrt_ftz(v)), acc[r]);
            }
          }
        } else {
#pragma unroll
          for (int g = 0; g < kGroup32; ++g) {
            const ulonglong2 pa = Sa[q0 + g], pb = Sb[q0 + g], pc = Sc[q0 + g];
            const f2_t pd = Sd[q0 + g];
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const f2_t dx = f2_add(f2_sub(pa.x, HX[r]), f2_sub(pc.x, LX[r]));
              const f2_t dy = f2_add(f2_sub(pa.y, HY[r]), f2_sub(pc.y, LY[r]));
              const f2_t dz = f2_add(f2_sub(pb.x, HZ[r]), f2_sub(pd, LZ[r]));
              const f2_t r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
              float u, v;
              f2_unpack(r2, u, v);
              acc[r] = f2_fma(pb.y, f2_pack(rsqrt_ftz(u), rsqrt_ftz(v)), acc[r]);
            }
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const f2_t y = f2_sub(acc[r], kc[r]);
          const f2_t s2 = f2_add(ks[r], y);
          kc[r] = f2_sub(f2_sub(s2, ks[r]), y);
          ks[r] = s2;
        }
      }
    }
    __syncthreads();
  }
  double mine = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (!vi[r]) continue;
    float s0, s1, c0, c1;
    f2_unpack(ks[r], s0, s1);
    f2_unpack(kc[r], c0, c1);
    const double row = (((double)s0 - (double)c0) + ((double)s1 - (double)c1)) + ((double)ksd[r] - (double)kcd[r]);
    double rx, ry, rz, mm;
    member_rel(A, base + it.i0 + 32 * R * wid + lane + 32 * r, cx, cy, cz, rx, ry, rz, mm);
    mine += mm * row;
  }
  return block_sum<double, kB32>(mine, sh);
}

// Persistent FP32-compensated pair kernel: items taken from a counter in list
// order; the shape of an item is hshape[h] (code 0, 1, 2 = 1, 2, 4 rows per
// thread), or fixed_code for every item when hshape is null.
__global__ void __launch_bounds__(kB32, 4) epot32_kernel(HaloArgs A, const PairItem* __restrict__ items,
                                                         const int8_t* __restrict__ hshape, int fixed_code,
                                                         int32_t nitems, int32_t* __restrict__ counter,
                                                         double* __restrict__ part) {
  __shared__ Tile32 S;
  __shared__ double sh[kB32 / 32];
  __shared__ double sred[6 * (kB32 / 32)];
  __shared__ int32_t s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int32_t w = s_item;
    __syncthreads();
    if (w >= nitems) break;
    const PairItem it = items[w];
    const int code = hshape ? (int)hshape[it.h] : fixed_code;
    double tot;
    if (code == 2) tot = epot32_item<4>(S, sh, sred, A, it, false);
    else if (code == 1) tot = epot32_item<2>(S, sh, sred, A, it, false);
    else tot = epot32_item<1>(S, sh, sred, A, it, false);
    // a zero separation in the fast path shows as a non-finite sum: recompute
    // the item with the per-pair test (block-uniform decision)
    if (__syncthreads_or(tid == 0 && !isfinite(tot))) {
      if (code == 2) tot = epot32_item<4>(S, sh, sred, A, it, true);
      else if (code == 1) tot = epot32_item<2>(S, sh, sred, A, it, true);
      else tot = epot32_item<1>(S, sh, sred, A, it, true);
    }
    if (tid == 0) part[w] = tot;
  }
}

// ---- Morton-sorted member copy for the FP32-compensated form
// Members of every halo ordered by the Morton key of their position about the
// halo centre (10 bits per axis over the halo's largest radius), stored as
// (x, y, z relative to the centre, mass).  The key's high bits are the halo,
// so a halo's members stay in its own range [off[h], off[h+1]).
__device__ __forceinline__ unsigned spread10(unsigned v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x30000ffu;
  v = (v | (v << 8)) & 0x300f00fu;
  v = (v | (v << 4)) & 0x30c30c3u;
  v = (v | (v << 2)) & 0x9249249u;
  return v;
}

__device__ __forceinline__ unsigned quant10(double r, double inv) {
  const double u = fmin(fmax((r * inv + 1.0) * 512.0, 0.0), 1023.0);
  return (unsigned)u;
}

__global__ void __launch_bounds__(kPB) sort32_keys_kernel(HaloArgs A, const MomChunk* __restrict__ ch,
                                                          unsigned long long* __restrict__ key,
                                                          int32_t* __restrict__ val) {
  const MomChunk c = ch[blockIdx.x];
  const double* o = A.out + (size_t)kHaloFields * c.h;
  const double cx = o[HP_PX], cy = o[HP_PY], cz = o[HP_PZ], rr = o[HP_R];
  const double inv = rr > 0.0 ? 1.0 / (rr * (1.0 + 1e-9)) : 0.0;
  for (int64_t k = c.b0 + threadIdx.x; k < c.b1; k += kPB) {
    double rx, ry, rz;
    rel_pos(A, k, cx, cy, cz, rx, ry, rz);
    const unsigned m =
        (spread10(quant10(rx, inv)) << 2) | (spread10(quant10(ry, inv)) << 1) | spread10(quant10(rz, inv));
    key[k] = ((unsigned long long)c.h << 30) | m;
    val[k] = (int32_t)k;
  }
}

__global__ void __launch_bounds__(kPB) sort32_gather_kernel(HaloArgs A, const MomChunk* __restrict__ ch,
                                                            const int32_t* __restrict__ val,
                                                            double4* __restrict__ srel) {
  const MomChunk c = ch[blockIdx.x];
  const double* o = A.out + (size_t)kHaloFields * c.h;
  const double cx = o[HP_PX], cy = o[HP_PY], cz = o[HP_PZ];
  for (int64_t q = c.b0 + threadIdx.x; q < c.b1; q += kPB) {
    const int64_t k = val[q];
    double rx, ry, rz;
    rel_pos(A, k, cx, cy, cz, rx, ry, rz);
    srel[q] = make_double4(rx, ry, rz, A.mass[k]);
  }
}

// Rows per item of shape code c.
__host__ __device__ constexpr int rows32_of(int code) { return kB32 << code; }

// Item partials of one work list, folded per halo in halo order: the items
// of halo h are entries [hoff[h], hoff[h+1]) of the halo-ordered list, and
// order[k] is where entry k ran in the schedule.
struct ItemFold {
  const int64_t* hoff;
  const int32_t* order;
  const double* part;  // null: this form was not computed
};

// One warp per halo: lane l sums entries l, l + 32, ... in order, then a
// butterfly over the lanes (every lane ends with the same bits), so the fold
// is deterministic and a halo with many items does not serialise on one thread.
__device__ __forceinline__ double fold_items(const ItemFold& F, int64_t h, int lane) {
  double s = 0.0;
  if (!F.part) return s;
  for (int64_t k = F.hoff[h] + lane; k < F.hoff[h + 1]; k += 32) s += F.part[F.order[k]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

constexpr int kFinBlock = 128;  // four halos per block

static inline unsigned finalize_blocks(int64_t nhalo) {
  return (unsigned)((nhalo * 32 + kFinBlock - 1) / kFinBlock);
}

// per-halo reduction of item partials, then E_pot, totals and spin
__global__ void __launch_bounds__(kFinBlock) epot_finalize_kernel(HaloArgs A, ItemFold f64, ItemFold f32,
                                                                  int64_t nhalo) {
  const int64_t h = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;  // uniform per warp
  const int lane = threadIdx.x & 31;
  if (h >= nhalo) return;
  const double s64 = fold_items(f64, h, lane), s32 = fold_items(f32, h, lane);
  if (lane != 0) return;
  double* o = A.out + (size_t)kHaloFields * h;
  o[HP_EP64] = -A.G * s64;
  o[HP_EP32C] = -A.G * s32;
  const double m = o[HP_M];
  const double hl = sqrt(o[HP_LX] * o[HP_LX] + o[HP_LY] * o[HP_LY] + o[HP_LZ] * o[HP_LZ]);
  // compute_spin_parameter_1c: |L| sqrt(|E|) / m^2.5 / G with E = ek + ep
  o[HP_SPIN64] = hl * sqrt(fabs(o[HP_EK] + o[HP_EP64])) / pow(m, 2.5) / A.G;
  o[HP_SPIN32C] = hl * sqrt(fabs(o[HP_EK] + o[HP_EP32C])) / pow(m, 2.5) / A.G;
  // principal axes: Jacobi eigenvalues of the symmetric inertia tensor
  double a[3][3] = {{o[HP_IXX], o[HP_IXY], o[HP_IXZ]}, {o[HP_IXY], o[HP_IYY], o[HP_IYZ]},
                    {o[HP_IXZ], o[HP_IYZ], o[HP_IZZ]}};
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-34 * dia || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < 3; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = cs * akp - sn * akq;
          a[k][q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = cs * apk - sn * aqk;
          a[q][k] = sn * apk + cs * aqk;
        }
      }
  }
  double e0 = a[0][0], e1 = a[1][1], e2 = a[2][2], t;
  if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
  if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
  if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
  o[HP_SHA] = sqrt(e0 / m);
  o[HP_SHB] = sqrt(e1 / m);
  o[HP_SHC] = sqrt(e2 / m);
}

}  // namespace ahop

// ------------------------------------------------------------------ host side
namespace ahop {

// Halo-size buckets of the FP32-compensated pair kernel's tile shape:
// n < 512, < 4096, < 32768, < 262144, >= 262144 members.
constexpr int kBuckets = AHOP_HALO_BUCKETS;
constexpr int kShapes = 3;                       // 1, 2 or 4 rows per thread (128, 256, 512 rows per item)
constexpr int kDefaultShape = 1;
constexpr double kTunePairs = 3.0e9;             // pairs timed per bucket and shape by the autotuner, at least
constexpr int kTuneWaves = 4;                    // ... and at least this many items per resident block, largest shape

static int bucket_of(int64_t n) {
  return n < 512 ? 0 : n < 4096 ? 1 : n < 32768 ? 2 : n < 262144 ? 3 : 4;
}

// One work list in halo order plus its schedule (items by decreasing cost).
struct ItemList {
  std::vector<PairItem> items;   // halo order
  std::vector<int64_t> cost;
  std::vector<int64_t> hoff;     // [nhalo+1]
  std::vector<PairItem> sched;   // run order
  std::vector<int32_t> order;    // halo-order entry k ran as sched[order[k]]
  void clear() { items.clear(); cost.clear(); hoff.clear(); }
};

// Items of halo h (n members) with `rows` rows per item over rows [0, row_limit),
// partners in chunks of kChunkJ.
static void add_halo_items(ItemList& L, int32_t h, int64_t n, int rows, int64_t row_limit) {
  const int64_t rl = std::min(n, row_limit);
  for (int64_t i0 = 0; i0 < rl; i0 += rows) {
    const int64_t r = std::min<int64_t>(rows, n - i0);
    for (int64_t j0 = i0; j0 < n; j0 += kChunkJ) {
      const int64_t j1 = std::min<int64_t>(n, j0 + kChunkJ);
      L.items.push_back(PairItem{h, (int32_t)i0, (int32_t)j0, (int32_t)j1});
      L.cost.push_back(j0 == i0 ? r * (j1 - j0) - r * r / 2 : r * (j1 - j0));
    }
  }
}

static void schedule(ItemList& L) {
  const int32_t ni = (int32_t)L.items.size();
  std::vector<int32_t> idx(ni);
  for (int32_t k = 0; k < ni; ++k) idx[k] = k;
  std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return L.cost[a] > L.cost[b]; });
  L.sched.resize(ni);
  L.order.resize(ni);
  for (int32_t k = 0; k < ni; ++k) {
    L.sched[k] = L.items[idx[k]];
    L.order[idx[k]] = k;
  }
}

struct ListBufs {
  DevBuf items, order, hoff, part;
  int32_t n = 0;
};

struct GraphSig {
  HaloArgs A;
  const void* ptr[21];
  int64_t nch, nmem;
  size_t scub_bytes;
  int32_t sort_end_bit, pad2;
  int64_t nhalo;
  int32_t n64, n32, grid64, grid32, epot, pad;
};

struct HaloEngine {
  DevBuf d_off, d_pos, d_vel, d_mass, d_dens, d_out;  // staging for host inputs
  ListBufs l64, l32, tune;
  DevBuf d_hshape, d_counter, d_err;
  DevBuf d_mch, d_mcoff, d_mp1, d_mp2, d_mcen, d_marg;  // chunked moment passes
  DevBuf d_index;                                        // staging of the host entry point's member indices
  int64_t nch = 0;
  // Morton-sorted member copy of the FP32-compensated form
  DevBuf d_skey, d_skey2, d_sval, d_sval2, d_srel, d_scub;
  size_t scub_bytes = 0;
  int64_t nmem = 0;
  int sort_end_bit = 31;
  cudaEvent_t ev[5] = {};
  cudaEvent_t ev_in = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
  bool ready = false;
  cudaStream_t own = nullptr;  // host-buffer entry point
  cudaStream_t gs = nullptr;   // launches and graph replays
  AhopHaloTimings t{};
  std::vector<int64_t> h_off;
  ItemList L64, L32;
  // autotuner: tuned shape per bucket (-1 = not yet), pinned shapes, timings
  int8_t code[kBuckets] = {-1, -1, -1, -1, -1};
  int8_t pinned[kBuckets] = {-1, -1, -1, -1, -1};
  float tune_ms[kBuckets][kShapes] = {};
  double tune_pairs[kBuckets] = {};
  // CUDA graph of the launch sequence, replayed while its arguments match
  bool use_graph = true;
  cudaGraphExec_t gexec = nullptr;
  GraphSig gsig{};
  int32_t graph_replays = 0;
};

static HaloEngine& halo_engine() {
  static HaloEngine* e = new HaloEngine();
  return *e;
}

template <class T>
static int upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  AHOP_CUDA_TRY(b.ensure(std::max<size_t>(v.size() * sizeof(T), 16)));
  if (!v.empty()) AHOP_CUDA_TRY(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return AHOP_OK;
}

static int upload_list(ListBufs& B, const ItemList& L, cudaStream_t st) {
  int rc;
  if ((rc = upload(B.items, L.sched, st))) return rc;
  if ((rc = upload(B.order, L.order, st))) return rc;
  if ((rc = upload(B.hoff, L.hoff, st))) return rc;
  AHOP_CUDA_TRY(B.part.ensure(std::max<size_t>(L.sched.size() * 8, 16)));
  B.n = (int32_t)L.sched.size();
  return AHOP_OK;
}

static int grid_for(const void* fn, int threads) {
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0);
  return nsm * (per > 0 ? per : 1);
}

// Autotuner: for every bucket present in this call whose shape is neither
// tuned nor pinned, time each shape on the same sample of that bucket's pairs
// and keep the fastest.  The sample takes the bucket's halos in order, in
// slabs of 512 rows (a multiple of every shape's rows, so every shape sees the
// same pairs), until it holds kTunePairs pairs and enough items of the
// largest shape to keep every resident block busy for kTuneWaves items (or
// the whole bucket): a sample that leaves blocks idle would favour the small
// shapes.  Needs the halo centres (moments) in A.out.
static int tune_buckets(HaloEngine& H, const HaloArgs& A, const int64_t* h_off, int64_t nhalo, cudaStream_t st) {
  bool need[kBuckets] = {};
  bool any = false;
  for (int64_t h = 0; h < nhalo; ++h) {
    const int b = bucket_of(h_off[h + 1] - h_off[h]);
    if (H.code[b] < 0 && H.pinned[b] < 0 && h_off[h + 1] - h_off[h] > 1) need[b] = any = true;
  }
  if (!any) return AHOP_OK;
  if (!H.ev_t0) {
    AHOP_CUDA_TRY(cudaEventCreate(&H.ev_t0));
    AHOP_CUDA_TRY(cudaEventCreate(&H.ev_t1));
  }
  const int grid = grid_for((const void*)epot32_kernel, kB32);
  for (int b = 0; b < kBuckets; ++b) {
    if (!need[b]) continue;
    std::vector<std::pair<int32_t, int64_t>> sample;  // (halo, row limit)
    double acc = 0;
    int64_t items_big = 0;
    const int64_t want_items = (int64_t)kTuneWaves * grid;
    auto enough = [&] { return acc >= kTunePairs && items_big >= want_items; };
    for (int64_t h = 0; h < nhalo && !enough(); ++h) {
      const int64_t n = h_off[h + 1] - h_off[h];
      if (bucket_of(n) != b || n < 2) continue;
      int64_t rl = 0;
      while (rl < n && !enough()) {  // one slab of kMaxT32 rows = one item row of the largest shape
        const int64_t r = std::min<int64_t>(kMaxT32, n - rl);
        acc += (double)r * (double)(n - rl) - 0.5 * (double)r * (double)(r + 1);
        items_big += (n - rl + kChunkJ - 1) / kChunkJ;
        rl += r;
      }
      sample.emplace_back((int32_t)h, rl);
    }
    H.tune_pairs[b] = acc;
    float best = 0.f;
    int best_c = kDefaultShape;
    for (int c = 0; c < kShapes; ++c) {
      ItemList L;
      for (auto& s : sample) add_halo_items(L, s.first, h_off[s.first + 1] - h_off[s.first], rows32_of(c), s.second);
      schedule(L);
      int rc;
      if ((rc = upload(H.tune.items, L.sched, st))) return rc;
      AHOP_CUDA_TRY(H.tune.part.ensure(std::max<size_t>(L.sched.size() * 8, 16)));
      float ms = 0.f;
      for (int rep = (c == 0 ? 0 : 1); rep < 2; ++rep) {  // the bucket's first run warms up
        AHOP_CUDA_TRY(cudaMemsetAsync(H.d_counter.as<int32_t>() + 2, 0, 4, st));
        AHOP_CUDA_TRY(cudaEventRecord(H.ev_t0, st));
        epot32_kernel<<<grid, kB32, 0, st>>>(A, H.tune.items.as<PairItem>(), nullptr, c, (int32_t)L.sched.size(),
                                             H.d_counter.as<int32_t>() + 2, H.tune.part.as<double>());
        AHOP_CUDA_TRY(cudaGetLastError());
        AHOP_CUDA_TRY(cudaEventRecord(H.ev_t1, st));
      }
      AHOP_CUDA_TRY(cudaEventSynchronize(H.ev_t1));
      AHOP_CUDA_TRY(cudaEventElapsedTime(&ms, H.ev_t0, H.ev_t1));
      H.tune_ms[b][c] = ms;
      if (c == 0 || ms < best) { best = ms; best_c = c; }
    }
    H.code[b] = (int8_t)best_c;
  }
  return AHOP_OK;
}

// Buffers of the Morton-sorted member copy (keys, values, CUB scratch, the
// copy itself) for nmem members of nhalo halos.
static int ensure_sort32(HaloEngine& H, int64_t nhalo, int64_t nmem, cudaStream_t st) {
  if (nmem > INT32_MAX) { set_error("more than 2^31 - 1 members in one call"); return AHOP_EINVAL; }
  H.nmem = nmem;
  int hb = 1;
  while ((int64_t(1) << hb) < nhalo) ++hb;
  H.sort_end_bit = 30 + hb;
  const size_t m = (size_t)std::max<int64_t>(nmem, 1);
  AHOP_CUDA_TRY(H.d_skey.ensure(m * 8));
  AHOP_CUDA_TRY(H.d_skey2.ensure(m * 8));
  AHOP_CUDA_TRY(H.d_sval.ensure(m * 4));
  AHOP_CUDA_TRY(H.d_sval2.ensure(m * 4));
  AHOP_CUDA_TRY(H.d_srel.ensure(m * 32));
  size_t tmp = 0;
  AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, H.d_skey.as<unsigned long long>(),
                                                H.d_skey2.as<unsigned long long>(), H.d_sval.as<int32_t>(),
                                                H.d_sval2.as<int32_t>(), (int)m, 0, H.sort_end_bit, st));
  AHOP_CUDA_TRY(H.d_scub.ensure(std::max<size_t>(tmp, 16)));
  H.scub_bytes = tmp;
  return AHOP_OK;
}

// Morton keys about each halo centre (needs the centres and radii in A.out),
// one radix sort, then the sorted copy A.srel.
static int enqueue_sort32(HaloEngine& H, const HaloArgs& A, cudaStream_t s, int* launches) {
  if (H.nch == 0 || H.nmem == 0) return AHOP_OK;
  sort32_keys_kernel<<<(unsigned)H.nch, kPB, 0, s>>>(A, H.d_mch.as<MomChunk>(), H.d_skey.as<unsigned long long>(),
                                                     H.d_sval.as<int32_t>());
  AHOP_CUDA_TRY(cudaGetLastError());
  size_t tmp = H.scub_bytes;
  AHOP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(H.d_scub.p, tmp, H.d_skey.as<unsigned long long>(),
                                                H.d_skey2.as<unsigned long long>(), H.d_sval.as<int32_t>(),
                                                H.d_sval2.as<int32_t>(), (int)H.nmem, 0, H.sort_end_bit, s));
  sort32_gather_kernel<<<(unsigned)H.nch, kPB, 0, s>>>(A, H.d_mch.as<MomChunk>(), H.d_sval2.as<int32_t>(),
                                                       H.d_srel.as<double4>());
  AHOP_CUDA_TRY(cudaGetLastError());
  if (launches) *launches += 3;
  return AHOP_OK;
}

// The device work of one call, in stream order; `capture` marks the timing
// events as graph nodes.
static int enqueue_props(HaloEngine& H, const HaloArgs& A, int64_t nhalo, int epot, int grid64, int grid32,
                         cudaStream_t s, bool capture, int* launches) {
  const unsigned flags = capture ? cudaEventRecordExternal : 0u;
  AHOP_CUDA_TRY(cudaMemsetAsync(H.d_counter.p, 0, 8, s));
  AHOP_CUDA_TRY(cudaMemsetAsync(H.d_err.p, 0, 4, s));
  AHOP_CUDA_TRY(cudaEventRecordWithFlags(H.ev[0], s, flags));
  *launches = 0;
  if (nhalo > 0) {
    const unsigned hb = (unsigned)((nhalo + 127) / 128);
    if (H.nch > 0) {
      mom_pass1_kernel<<<(unsigned)H.nch, kPB, 0, s>>>(A, H.d_mch.as<MomChunk>(), H.d_mp1.as<MomP1>());
      ++*launches;
    }
    mom_fold1_kernel<<<hb, 128, 0, s>>>(A, H.d_mcoff.as<int64_t>(), H.d_mp1.as<MomP1>(), H.d_mcen.as<MomCentre>(),
                                        nhalo);
    ++*launches;
    if (A.cdm && H.nch > 0) {
      mom_cdm_kernel<<<(unsigned)H.nch, kPB, 0, s>>>(A, H.d_mch.as<MomChunk>(), H.d_mcen.as<MomCentre>(),
                                                     H.d_marg.as<MomArg>());
      mom_cdm_fold_kernel<<<hb, 128, 0, s>>>(A, H.d_mcoff.as<int64_t>(), H.d_marg.as<MomArg>(),
                                             H.d_mcen.as<MomCentre>(), nhalo);
      *launches += 2;
    }
    if (A.sc) {
      mom_sc_kernel<<<(unsigned)nhalo, kPB, 0, s>>>(A, H.d_mcen.as<MomCentre>());
      ++*launches;
    }
    if (H.nch > 0) {
      mom_pass2_kernel<<<(unsigned)H.nch, kPB, 0, s>>>(A, H.d_mch.as<MomChunk>(), H.d_mcen.as<MomCentre>(),
                                                       H.d_mp2.as<MomP2>());
      ++*launches;
    }
    mom_fold2_kernel<<<hb, 128, 0, s>>>(A, H.d_mcoff.as<int64_t>(), H.d_mp2.as<MomP2>(), H.d_mcen.as<MomCentre>(),
                                        nhalo);
    ++*launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecordWithFlags(H.ev[1], s, flags));
  if ((epot & 1) && H.l64.n > 0) {
    epot64_kernel<<<grid64, kT64, 0, s>>>(A, H.l64.items.as<PairItem>(), H.l64.n, H.d_counter.as<int32_t>(),
                                          H.l64.part.as<double>());
    ++*launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecordWithFlags(H.ev[2], s, flags));
  if ((epot & 2) && H.l32.n > 0) {
    // the sort belongs to the FP32-compensated form and is timed with it
    int rc;
    if ((rc = enqueue_sort32(H, A, s, launches))) return rc;
    epot32_kernel<<<grid32, kB32, 0, s>>>(A, H.l32.items.as<PairItem>(), H.d_hshape.as<int8_t>(), kDefaultShape,
                                          H.l32.n, H.d_counter.as<int32_t>() + 1, H.l32.part.as<double>());
    ++*launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecordWithFlags(H.ev[3], s, flags));
  if (nhalo > 0) {
    const ItemFold f64{H.l64.hoff.as<int64_t>(), H.l64.order.as<int32_t>(),
                       (epot & 1) ? H.l64.part.as<double>() : nullptr};
    const ItemFold f32{H.l32.hoff.as<int64_t>(), H.l32.order.as<int32_t>(),
                       (epot & 2) ? H.l32.part.as<double>() : nullptr};
    epot_finalize_kernel<<<finalize_blocks(nhalo), kFinBlock, 0, s>>>(A, f64, f32, nhalo);
    ++*launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecordWithFlags(H.ev[4], s, flags));
  return AHOP_OK;
}

static int halo_run(HaloEngine& H, const AhopHaloParams* p, const int64_t* d_off, const int64_t* h_off,
                    int64_t nhalo, const double* d_pos, const double* d_vel, const double* d_mass,
                    const double* d_dens, double* d_out, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  AHOP_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("the stream is being captured; this entry point synchronises with the host and cannot run inside a stream capture");
    return AHOP_EINVAL;
  }
  if (!H.ready) {
    for (auto& e : H.ev) AHOP_CUDA_TRY(cudaEventCreate(&e));
    AHOP_CUDA_TRY(cudaEventCreateWithFlags(&H.ev_in, cudaEventDisableTiming));
    AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&H.gs, cudaStreamNonBlocking));
    H.ready = true;
  }
  double pairs = 0;
  for (int64_t h = 0; h < nhalo; ++h) {
    const int64_t n = h_off[h + 1] - h_off[h];
    if (n < 0 || n > INT32_MAX - kChunkJ) { set_error("halo member count out of range"); return AHOP_EINVAL; }
    pairs += 0.5 * (double)n * (double)(n - 1);
  }
  HaloArgs A;
  memset(&A, 0, sizeof A);  // compared bytewise for graph reuse
  A.off = d_off; A.pos = d_pos; A.vel = d_vel; A.mass = d_mass; A.dens = d_dens; A.out = d_out;
  A.L = p->Lbox; A.h = 0.5 * p->Lbox; A.hub = p->Hub_pt; A.G = p->gravconst; A.periodic = p->periodic != 0;
  A.sc = p->sc != 0; A.dcell_min = p->dcell_min; A.eps_sc = p->eps_sc;
  A.cdm = p->cdm != 0; A.ndm = p->ndm; A.massp = p->massp; A.index = p->index;
  AHOP_CUDA_TRY(H.d_err.ensure(16));
  AHOP_CUDA_TRY(H.d_counter.ensure(16));
  A.err = H.d_err.as<int>();
  const int epot = p->epot & 3;
  int rc;
  // chunks of the moment passes (also the blocks of the member sort)
  std::vector<MomChunk> mch;
  std::vector<int64_t> mcoff(nhalo + 1, 0);
  for (int64_t h = 0; h < nhalo; ++h) {
    mcoff[h] = (int64_t)mch.size();
    for (int64_t b = h_off[h]; b < h_off[h + 1]; b += kMomChunk)
      mch.push_back(MomChunk{(int32_t)h, 0, b, std::min<int64_t>(h_off[h + 1], b + kMomChunk)});
  }
  mcoff[nhalo] = (int64_t)mch.size();
  H.nch = (int64_t)mch.size();
  if ((rc = upload(H.d_mch, mch, st))) return rc;
  if ((rc = upload(H.d_mcoff, mcoff, st))) return rc;
  if (epot & 2) {
    if ((rc = ensure_sort32(H, nhalo, nhalo > 0 ? h_off[nhalo] - h_off[0] : 0, st))) return rc;
    A.srel = H.d_srel.as<double4>();
  }
  float tune_total = 0.f;
  if (epot & 2) {
    // shapes for this call's buckets; the tuner needs the centres first
    bool need = false;
    for (int64_t h = 0; h < nhalo && !need; ++h) {
      const int b = bucket_of(h_off[h + 1] - h_off[h]);
      need = H.code[b] < 0 && H.pinned[b] < 0 && h_off[h + 1] - h_off[h] > 1;
    }
    if (need) {
      auto t0 = std::chrono::steady_clock::now();
      AHOP_CUDA_TRY(cudaMemsetAsync(H.d_err.p, 0, 4, st));
      halo_moments_kernel<<<(unsigned)nhalo, kPB, 0, st>>>(A);
      AHOP_CUDA_TRY(cudaGetLastError());
      if ((rc = enqueue_sort32(H, A, st, nullptr))) return rc;
      if ((rc = tune_buckets(H, A, h_off, nhalo, st))) return rc;
      tune_total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  // work lists (halo order), schedules, per-halo shape codes
  std::vector<int8_t> hshape;
  H.L64.clear();
  H.L32.clear();
  H.L64.hoff.assign(nhalo + 1, 0);
  H.L32.hoff.assign(nhalo + 1, 0);
  if (epot & 2) hshape.resize(nhalo > 0 ? nhalo : 1, (int8_t)kDefaultShape);
  for (int64_t h = 0; h < nhalo; ++h) {
    const int64_t n = h_off[h + 1] - h_off[h];
    H.L64.hoff[h] = (int64_t)H.L64.items.size();
    H.L32.hoff[h] = (int64_t)H.L32.items.size();
    if (epot & 1) add_halo_items(H.L64, (int32_t)h, n, kT64, n);
    if (epot & 2) {
      const int b = bucket_of(n);
      const int c = H.pinned[b] >= 0 ? H.pinned[b] : H.code[b] >= 0 ? H.code[b] : kDefaultShape;
      hshape[h] = (int8_t)c;
      add_halo_items(H.L32, (int32_t)h, n, rows32_of(c), n);
    }
  }
  H.L64.hoff[nhalo] = (int64_t)H.L64.items.size();
  H.L32.hoff[nhalo] = (int64_t)H.L32.items.size();
  schedule(H.L64);
  schedule(H.L32);
  AHOP_CUDA_TRY(H.d_mp1.ensure(std::max<size_t>(mch.size() * sizeof(MomP1), 16)));
  AHOP_CUDA_TRY(H.d_mp2.ensure(std::max<size_t>(mch.size() * sizeof(MomP2), 16)));
  AHOP_CUDA_TRY(H.d_marg.ensure(std::max<size_t>(mch.size() * sizeof(MomArg), 16)));
  AHOP_CUDA_TRY(H.d_mcen.ensure(std::max<size_t>((size_t)nhalo * sizeof(MomCentre), 16)));
  if ((rc = upload_list(H.l64, H.L64, st))) return rc;
  if ((rc = upload_list(H.l32, H.L32, st))) return rc;
  if ((rc = upload(H.d_hshape, hshape, st))) return rc;
  const int grid64 = grid_for((const void*)epot64_kernel, kT64);
  const int grid32 = grid_for((const void*)epot32_kernel, kB32);
  // the launches run on the engine's stream after everything queued on st
  AHOP_CUDA_TRY(cudaEventRecord(H.ev_in, st));
  AHOP_CUDA_TRY(cudaStreamWaitEvent(H.gs, H.ev_in, 0));
  int launches = 0;
  if (H.use_graph) {
    GraphSig sig;
    memset(&sig, 0, sizeof sig);
    sig.A = A;
    const void* ptrs[21] = {H.l64.items.p, H.l64.order.p, H.l64.hoff.p, H.l64.part.p, H.l32.items.p,
                            H.l32.order.p, H.l32.hoff.p, H.l32.part.p, H.d_hshape.p, H.d_counter.p,
                            H.d_mch.p,     H.d_mcoff.p,   H.d_mp1.p,    H.d_mp2.p,    H.d_mcen.p,
                            H.d_skey.p,    H.d_skey2.p,   H.d_sval.p,   H.d_sval2.p,  H.d_scub.p,
                            H.d_marg.p};
    memcpy(sig.ptr, ptrs, sizeof ptrs);
    sig.nch = H.nch;
    sig.nmem = H.nmem;
    sig.scub_bytes = H.scub_bytes;
    sig.sort_end_bit = H.sort_end_bit;
    sig.nhalo = nhalo; sig.n64 = H.l64.n; sig.n32 = H.l32.n; sig.grid64 = grid64; sig.grid32 = grid32;
    sig.epot = epot;
    if (!H.gexec || memcmp(&sig, &H.gsig, sizeof sig) != 0) {
      if (H.gexec) { cudaGraphExecDestroy(H.gexec); H.gexec = nullptr; }
      cudaGraph_t g = nullptr;
      AHOP_CUDA_TRY(cudaStreamBeginCapture(H.gs, cudaStreamCaptureModeThreadLocal));
      rc = enqueue_props(H, A, nhalo, epot, grid64, grid32, H.gs, true, &launches);
      const cudaError_t ec = cudaStreamEndCapture(H.gs, &g);
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      AHOP_CUDA_TRY(ec);
      const cudaError_t ei = cudaGraphInstantiate(&H.gexec, g, 0);
      cudaGraphDestroy(g);
      AHOP_CUDA_TRY(ei);
      H.gsig = sig;
      H.graph_replays = 0;
    } else {
      ++H.graph_replays;
      launches = H.t.kernel_launches;
    }
    AHOP_CUDA_TRY(cudaGraphLaunch(H.gexec, H.gs));
  } else {
    if ((rc = enqueue_props(H, A, nhalo, epot, grid64, grid32, H.gs, false, &launches))) return rc;
  }
  int herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, H.d_err.p, 4, cudaMemcpyDeviceToHost, H.gs));
  AHOP_CUDA_TRY(cudaStreamSynchronize(H.gs));
  if (herr) { set_error("shrinking-sphere centre: step limit reached"); return AHOP_ELIMIT; }
  auto el = [&](int a, int b) { float ms = 0; cudaEventElapsedTime(&ms, H.ev[a], H.ev[b]); return ms; };
  H.t.moments = el(0, 1);
  H.t.epot64 = el(1, 2);
  H.t.epot32c = el(2, 3);
  H.t.finalize = el(3, 4);
  H.t.total = el(0, 4);
  H.t.pairs = pairs;
  H.t.items = H.l64.n + H.l32.n;
  H.t.kernel_launches = launches;
  H.t.tune_ms = tune_total;
  H.t.graph_replays = H.use_graph ? H.graph_replays : -1;
  return AHOP_OK;
}

static int halo_validate(const AhopHaloParams* p, int64_t nhalo) {
  if (!p) { set_error("null params"); return AHOP_EINVAL; }
  if (nhalo < 0) { set_error("nhalo must be >= 0"); return AHOP_EINVAL; }
  if (p->periodic && !(p->Lbox > 0)) { set_error("Lbox must be positive for periodic boxes"); return AHOP_EINVAL; }
  if (p->sc && !(p->eps_sc > 0.0 && p->eps_sc < 1.0)) {
    // the reference's recursion never ends with eps_SC <= 0
    set_error("eps_SC must be in (0, 1) when the shrinking-sphere centre is on");
    return AHOP_EINVAL;
  }
  return AHOP_OK;
}

}  // namespace ahop

using namespace ahop;

extern "C" {

int ahop_halo_props_device(const AhopHaloParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                           const double* d_vel, const double* d_mass, const double* d_density, double* d_out,
                           void* stream) {
  int rc;
  if ((rc = halo_validate(p, nhalo))) return rc;
  HaloEngine& H = halo_engine();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  H.h_off.resize(nhalo + 1);
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.h_off.data(), d_off, (nhalo + 1) * 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  return halo_run(H, p, d_off, H.h_off.data(), nhalo, d_pos, d_vel, d_mass, d_density, d_out, st);
}

int ahop_halo_props(const AhopHaloParams* p, const int64_t* off, int64_t nhalo, const double* pos,
                    const double* vel, const double* mass, const double* density, double* out) {
  int rc;
  if ((rc = halo_validate(p, nhalo))) return rc;
  if (!off || (nhalo > 0 && (!pos || !vel || !mass || !density || !out))) { set_error("null input"); return AHOP_EINVAL; }
  HaloEngine& H = halo_engine();
  if (!H.own) AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&H.own, cudaStreamNonBlocking));
  cudaStream_t st = H.own;
  const int64_t n = off[nhalo];
  AHOP_CUDA_TRY(H.d_off.ensure((nhalo + 1) * 8));
  AHOP_CUDA_TRY(H.d_pos.ensure(n * 24 + 8));
  AHOP_CUDA_TRY(H.d_vel.ensure(n * 24 + 8));
  AHOP_CUDA_TRY(H.d_mass.ensure(n * 8 + 8));
  AHOP_CUDA_TRY(H.d_dens.ensure(n * 8 + 8));
  AHOP_CUDA_TRY(H.d_out.ensure((size_t)nhalo * kHaloFields * 8 + 8));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_off.p, off, (nhalo + 1) * 8, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_pos.p, pos, n * 24, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_vel.p, vel, n * 24, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_mass.p, mass, n * 8, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_dens.p, density, n * 8, cudaMemcpyHostToDevice, st));
  AhopHaloParams pd = *p;  // the member indices move to the device with the other inputs
  if (p->index) {
    AHOP_CUDA_TRY(H.d_index.ensure(n * 4 + 8));
    AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_index.p, p->index, n * 4, cudaMemcpyHostToDevice, st));
    pd.index = H.d_index.as<int32_t>();
  }
  if ((rc = halo_run(H, &pd, H.d_off.as<int64_t>(), off, nhalo, H.d_pos.as<double>(), H.d_vel.as<double>(),
                     H.d_mass.as<double>(), H.d_dens.as<double>(), H.d_out.as<double>(), st)))
    return rc;
  AHOP_CUDA_TRY(cudaMemcpyAsync(out, H.d_out.p, (size_t)nhalo * kHaloFields * 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  return AHOP_OK;
}

int ahop_halo_get_timings(AhopHaloTimings* t) {
  if (!t) return AHOP_EINVAL;
  *t = halo_engine().t;
  return AHOP_OK;
}

int ahop_halo_get_tiles(int32_t* rows, float* ms) {
  if (!rows) { set_error("null rows"); return AHOP_EINVAL; }
  HaloEngine& H = halo_engine();
  for (int b = 0; b < kBuckets; ++b) {
    const int c = H.pinned[b] >= 0 ? H.pinned[b] : H.code[b];
    rows[b] = c >= 0 ? rows32_of(c) : 0;
    if (ms)
      for (int k = 0; k < kShapes; ++k) ms[b * kShapes + k] = H.tune_ms[b][k];
  }
  return AHOP_OK;
}

int ahop_halo_set_tiles(const int32_t* rows) {
  HaloEngine& H = halo_engine();
  if (!rows) {
    for (int b = 0; b < kBuckets; ++b) {
      H.pinned[b] = H.code[b] = -1;
      for (int k = 0; k < kShapes; ++k) H.tune_ms[b][k] = 0.f;
    }
    return AHOP_OK;
  }
  int8_t c[kBuckets];
  for (int b = 0; b < kBuckets; ++b) {
    if (rows[b] == 0) c[b] = -1;
    else if (rows[b] == rows32_of(0)) c[b] = 0;
    else if (rows[b] == rows32_of(1)) c[b] = 1;
    else if (rows[b] == rows32_of(2)) c[b] = 2;
    else { set_error("tile rows must be 0, 128, 256 or 512"); return AHOP_EINVAL; }
  }
  for (int b = 0; b < kBuckets; ++b) H.pinned[b] = c[b];
  return AHOP_OK;
}

int ahop_halo_set_graph(int32_t on) {
  HaloEngine& H = halo_engine();
  H.use_graph = on != 0;
  if (!H.use_graph && H.gexec) {
    cudaGraphExecDestroy(H.gexec);
    H.gexec = nullptr;
  }
  return AHOP_OK;
}

}  // extern "C"

// --------------------------------------------------- allocation-free variant
// For callers that cannot allocate device memory -- code running while a CUDA
// graph is being captured elsewhere in the process, host frameworks that own
// every device allocation through their own pool, or embedded callers whose
// memory budget is fixed up front -- ahop_halo_props_noalloc computes the same
// fields with all of its scratch (the (halo, tile) work list, per-item partial
// sums, per-halo item offsets and the work counters) in this file-scope device
// array.  Every GPU that loads the library holds it until the process exits.
namespace ahop {

constexpr int64_t kNoAllocMaxHalos = 65536;         // halos per call
constexpr int64_t kNoAllocMaxItems = 262144;        // (halo, 256-member tile) items per call

struct NoAllocScratch {
  PairItem items[kNoAllocMaxItems];
  int32_t order[kNoAllocMaxItems];
  double part64[kNoAllocMaxItems];
  double part32[kNoAllocMaxItems];
  int64_t hoff[kNoAllocMaxHalos + 1];
  int32_t counter[4];  // [0],[1]: work counters of the two pair kernels; [2]: item total; [3]: error
};

// ~10 MB; in host code this name is only a host-side stand-in, the device
// address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Per-halo tile counts and offsets in one block (nhalo <= kNoAllocMaxHalos).
__global__ void __launch_bounds__(1024) noalloc_offsets_kernel(const int64_t* __restrict__ off, int64_t nhalo,
                                                               NoAllocScratch* S) {
  using Scan = cub::BlockScan<int64_t, 1024>;
  __shared__ typename Scan::TempStorage tmp;
  int64_t carry = 0;
  for (int64_t base = 0; base < nhalo; base += 1024) {
    const int64_t h = base + threadIdx.x;
    int64_t nit = 0;
    if (h < nhalo) {
      const int64_t n = off[h + 1] - off[h];
      nit = n > 0 ? (n + kT64 - 1) / kT64 : 0;
    }
    int64_t ex, tot;
    Scan(tmp).ExclusiveSum(nit, ex, tot);
    __syncthreads();
    if (h < nhalo) S->hoff[h] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    S->hoff[nhalo] = carry;
    S->counter[2] = carry > kNoAllocMaxItems ? -1 : (int32_t)carry;
  }
}

// Work items in halo order, one per 256 rows of a halo with all of its
// partners (no cost sort, no partner chunks).  The FP64 form and the FP32
// form (at 2 rows per thread, also 256 rows per item) share the list.  The
// FP64 rows equal the allocating entry point's to rounding; the
// FP32-compensated ones are summed in other groups (that entry point chunks
// partners and picks tile shapes per halo size) and agree to its error.
__global__ void noalloc_items_kernel(const int64_t* __restrict__ off, int64_t nhalo, NoAllocScratch* S) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  const int64_t n = off[h + 1] - off[h];
  int64_t k = S->hoff[h];
  for (int64_t i0 = 0; i0 < n; i0 += kT64, ++k) {
    S->items[k] = PairItem{(int32_t)h, (int32_t)i0, (int32_t)i0, (int32_t)n};
    S->order[k] = (int32_t)k;
  }
}

static NoAllocScratch* g_noalloc_ptr[128] = {};

// First call on a device (with that device current) looks up the array's
// device address; do it before any stream capture.
static int noalloc_setup(NoAllocScratch** out) {
  int dev = 0;
  AHOP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) { set_error("device ordinal out of range"); return AHOP_EINVAL; }
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") + cudaGetErrorString(e));
      return AHOP_ECUDA;
    }
    g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return AHOP_OK;
}

}  // namespace ahop

extern "C" int ahop_halo_props_noalloc(const AhopHaloParams* p, const int64_t* d_off, int64_t nhalo,
                                       const double* d_pos, const double* d_vel, const double* d_mass,
                                       const double* d_density, double* d_out, void* stream) {
  using namespace ahop;
  int rc;
  if ((rc = halo_validate(p, nhalo))) return rc;
  if (nhalo > kNoAllocMaxHalos) {
    set_error("ahop_halo_props_noalloc: nhalo " + std::to_string(nhalo) + " exceeds the maximum of " +
              std::to_string(kNoAllocMaxHalos));
    return AHOP_EINVAL;
  }
  if (nhalo == 0) return AHOP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the call reads the item count and the error flag back to the host, so it
  // cannot be recorded into a graph: refuse a capturing stream before any
  // work is enqueued (enqueueing would invalidate the caller's capture)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  AHOP_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("the stream is being captured; ahop_halo_props_noalloc synchronises with the host and cannot run "
              "inside a stream capture");
    return AHOP_EINVAL;
  }
  NoAllocScratch* S = nullptr;
  if ((rc = noalloc_setup(&S))) return rc;
  noalloc_offsets_kernel<<<1, 1024, 0, st>>>(d_off, nhalo, S);
  AHOP_CUDA_TRY(cudaGetLastError());
  int32_t total = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&total, &S->counter[2], 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (total < 0) {
    set_error("ahop_halo_props_noalloc: more than " + std::to_string(kNoAllocMaxItems) +
              " (halo, 256-member tile) work items; split the call");
    return AHOP_EINVAL;
  }
  noalloc_items_kernel<<<(unsigned)((nhalo + 255) / 256), 256, 0, st>>>(d_off, nhalo, S);
  AHOP_CUDA_TRY(cudaGetLastError());
  // the work counters and the error flag must start at zero: the array keeps
  // the last call's contents
  AHOP_CUDA_TRY(cudaMemsetAsync(S->counter, 0, 2 * sizeof(int32_t), st));
  AHOP_CUDA_TRY(cudaMemsetAsync(&S->counter[3], 0, sizeof(int32_t), st));
  HaloArgs A;
  memset(&A, 0, sizeof A);
  A.off = d_off; A.pos = d_pos; A.vel = d_vel; A.mass = d_mass; A.dens = d_density; A.out = d_out;
  A.L = p->Lbox; A.h = 0.5 * p->Lbox; A.hub = p->Hub_pt; A.G = p->gravconst; A.periodic = p->periodic != 0;
  A.sc = p->sc != 0; A.dcell_min = p->dcell_min; A.eps_sc = p->eps_sc;
  A.cdm = p->cdm != 0; A.ndm = p->ndm; A.massp = p->massp; A.index = p->index;
  A.err = &S->counter[3];
  halo_moments_kernel<<<(unsigned)nhalo, kPB, 0, st>>>(A);
  AHOP_CUDA_TRY(cudaGetLastError());
  if ((p->epot & 1) && total > 0) {
    epot64_kernel<<<grid_for((const void*)epot64_kernel, kT64), kT64, 0, st>>>(A, S->items, total, &S->counter[0],
                                                                               S->part64);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  if ((p->epot & 2) && total > 0) {
    static_assert(rows32_of(1) == kT64, "the FP32 form shares the 256-row list");
    epot32_kernel<<<grid_for((const void*)epot32_kernel, kB32), kB32, 0, st>>>(A, S->items, nullptr, 1, total,
                                                                               &S->counter[1], S->part32);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  const ItemFold f64{S->hoff, S->order, (p->epot & 1) ? S->part64 : nullptr};
  const ItemFold f32{S->hoff, S->order, (p->epot & 2) ? S->part32 : nullptr};
  epot_finalize_kernel<<<finalize_blocks(nhalo), kFinBlock, 0, st>>>(A, f64, f32, nhalo);
  AHOP_CUDA_TRY(cudaGetLastError());
  int32_t herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, &S->counter[3], 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) { set_error("shrinking-sphere centre: step limit reached"); return AHOP_ELIMIT; }
  return AHOP_OK;
}
