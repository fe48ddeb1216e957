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
  long long bi = LLONG_MAX;
  for (int64_t i = b0 + tid; i < b1; i += kPB) {
    const double w = A.mass[i];
    m += w;
    mvx += w * A.vel[3 * i];
    mvy += w * A.vel[3 * i + 1];
    mvz += w * A.vel[3 * i + 2];
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
  if (A.sc) shrink_sphere_centre(A, b0, b1, s_c, sh, s_best_d, s_best_i);
  const double cx = s_c[0], cy = s_c[1], cz = s_c[2], vx = s_c[3], vy = s_c[4], vz = s_c[5];
  // pass 2
  double Lx = 0, Ly = 0, Lz = 0, r2max = 0, Ixx = 0, Ixy = 0, Ixz = 0, Iyy = 0, Iyz = 0, Izz = 0, ek = 0, sg = 0;
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
    sg += w * (ux * ux + uy * uy + uz * uz);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2max = fmax(r2max, __shfl_xor_sync(0xffffffffu, r2max, o));
  if ((tid & 31) == 0) s_best_d[tid >> 5] = r2max;
  Lx = block_sum(Lx, sh); Ly = block_sum(Ly, sh); Lz = block_sum(Lz, sh);
  Ixx = block_sum(Ixx, sh); Ixy = block_sum(Ixy, sh); Ixz = block_sum(Ixz, sh);
  Iyy = block_sum(Iyy, sh); Iyz = block_sum(Iyz, sh); Izz = block_sum(Izz, sh);
  ek = block_sum(ek, sh);
  sg = block_sum(sg, sh);
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
struct MomP1 {
  double m, mvx, mvy, mvz, bd;
  long long bi;
};
constexpr int kP2 = 11;  // Lx Ly Lz Ixx Ixy Ixz Iyy Iyz Izz ek sg
struct MomP2 {
  double v[kP2];
  double r2max;
};
struct MomCentre {
  double c[6];  // centre x, y, z, bulk velocity x, y, z
  long long ic; // centre member (absolute index)
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
  __shared__ double sh[5 * (kPB / 32) + 8];
  __shared__ double s_bd[kPB / 32];
  __shared__ long long s_bi[kPB / 32];
  const int tid = threadIdx.x;
  const MomChunk c = ch[blockIdx.x];
  double v[4] = {0, 0, 0, 0}, bd = -DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t i = c.b0 + tid; i < c.b1; i += kPB) {
    const double w = A.mass[i];
    v[0] += w;
    v[1] += w * A.vel[3 * i];
    v[2] += w * A.vel[3 * i + 1];
    v[3] += w * A.vel[3 * i + 2];
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
  block_sum_n<4>(v, sh);
  if (tid == 0) {
    bd = s_bd[0]; bi = s_bi[0];
    for (int w = 1; w < kPB / 32; ++w)
      if (s_bd[w] > bd || (s_bd[w] == bd && s_bi[w] < bi)) { bd = s_bd[w]; bi = s_bi[w]; }
    P[blockIdx.x] = MomP1{v[0], v[1], v[2], v[3], bd, bi};
  }
}

// per halo: chunk partials in order -> mass, bulk velocity, densest member
__global__ void mom_fold1_kernel(HaloArgs A, const int64_t* __restrict__ hcoff, const MomP1* __restrict__ P,
                                 MomCentre* __restrict__ C, int64_t nhalo) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  double m = 0, mvx = 0, mvy = 0, mvz = 0, bd = -DBL_MAX;
  long long bi = LLONG_MAX;
  for (int64_t k = hcoff[h]; k < hcoff[h + 1]; ++k) {
    const MomP1 p = P[k];
    m += p.m; mvx += p.mvx; mvy += p.mvy; mvz += p.mvz;
    if (p.bd > bd || (p.bd == bd && p.bi < bi)) { bd = p.bd; bi = p.bi; }
  }
  MomCentre c;
  if (bi != LLONG_MAX) {
    c.c[0] = A.pos[3 * bi]; c.c[1] = A.pos[3 * bi + 1]; c.c[2] = A.pos[3 * bi + 2];
  } else {
    c.c[0] = c.c[1] = c.c[2] = 0.0;
  }
  c.c[3] = mvx / m; c.c[4] = mvy / m; c.c[5] = mvz / m;
  c.ic = bi;
  C[h] = c;
  A.out[(size_t)kHaloFields * h + HP_M] = m;
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
    v[10] += w * (ux * ux + uy * uy + uz * uz);
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
// instructions: two lanes per 64-bit register, one instruction).  Positions
// relative to the halo centre are split into hi = float(r) and
// lo = float(r - hi); a separation is (hi_j - hi_i) + (lo_j - lo_i).  The two
// lanes of every packed register hold two partners j, 2q and 2q+1, of the same
// row i, so a row's own coordinates are loop-invariant (hi_i, hi_i) pairs.
// Each thread owns R rows (rows tid + 128 r); partner tiles are 128 * R
// wide, shared memory holds them as packed pairs.  For every row, sixteen
// partner pairs (32 terms) are accumulated by a fused multiply-add chain per
// lane, then enter a Kahan-compensated FP32 sum; rows fold into FP64 per item.
// Separations of exactly zero (coincident members) are excluded like in the
// FP64 form: the fast path does not test for them -- rsqrt(0) = inf makes the
// row's sum non-finite, and the block then recomputes the item with a
// per-pair test.  The tile shape (R = 1, 2 or 4 rows per thread) is chosen
// per halo-size bucket by the host-side autotuner and read per item.
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
constexpr int kGroup32 = 16;           // partner pairs per compensated fold
constexpr int kChunkJ = 32768;         // partners per item at most (a multiple of every tile width)
constexpr float kFar = 1.0e18f;        // padding position: its terms vanish (mass 0, finite r)

struct Tile32 {
  float4 a[kMaxT32 / 2];  // hi x(2q), x(2q+1), y(2q), y(2q+1)
  float4 b[kMaxT32 / 2];  // hi z(2q), z(2q+1), mass(2q), mass(2q+1)
  float4 c[kMaxT32 / 2];  // lo x, x, y, y
  float2 d[kMaxT32 / 2];  // lo z, z
};

__device__ __forceinline__ void split_hilo(double r, float& hi, float& lo) {
  hi = (float)r;
  lo = (float)(r - (double)hi);
}

// Stage partners [j0, j0 + T) (T = 128 R) of one item; slots past j1 get the
// padding (mass 0, far away).
template <int R>
__device__ __forceinline__ void stage_tile32(Tile32& S, const HaloArgs& A, int64_t base, int32_t j0, int32_t j1,
                                             double cx, double cy, double cz) {
  constexpr int P = kB32 * R / 2;
  for (int q = threadIdx.x; q < P; q += kB32) {
    float hx[2], hy[2], hz[2], m[2], lx[2], ly[2], lz[2];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const int32_t j = j0 + 2 * q + l;
      if (j < j1) {
        double rx, ry, rz;
        rel_pos(A, base + j, cx, cy, cz, rx, ry, rz);
        split_hilo(rx, hx[l], lx[l]);
        split_hilo(ry, hy[l], ly[l]);
        split_hilo(rz, hz[l], lz[l]);
        m[l] = (float)A.mass[base + j];
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

template <int R>
__device__ double epot32_item(Tile32& S, double* sh, const HaloArgs& A, const PairItem& it, bool checked) {
  constexpr int T = kB32 * R;
  const int tid = threadIdx.x;
  const int64_t base = A.off[it.h];
  const int32_t n = (int32_t)(A.off[it.h + 1] - base);
  const double* cen = A.out + (size_t)kHaloFields * it.h;
  const double cx = cen[HP_PX], cy = cen[HP_PY], cz = cen[HP_PZ];
  float hx[R], hy[R], hz[R], lx[R], ly[R], lz[R];
  f2_t HX[R], HY[R], HZ[R], LX[R], LY[R], LZ[R], ks[R], kc[R];
  float ksd[R], kcd[R];  // per-pair path sums
  bool vi[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int32_t i = it.i0 + tid + kB32 * r;
    vi[r] = i < n;
    if (vi[r]) {
      double rx, ry, rz;
      rel_pos(A, base + i, cx, cy, cz, rx, ry, rz);
      split_hilo(rx, hx[r], lx[r]);
      split_hilo(ry, hy[r], ly[r]);
      split_hilo(rz, hz[r], lz[r]);
    } else {
      // far on the other side from the padding: every separation stays finite
      hx[r] = hy[r] = hz[r] = -kFar;
      lx[r] = ly[r] = lz[r] = 0.f;
    }
    HX[r] = f2_pack(hx[r], hx[r]); HY[r] = f2_pack(hy[r], hy[r]); HZ[r] = f2_pack(hz[r], hz[r]);
    LX[r] = f2_pack(lx[r], lx[r]); LY[r] = f2_pack(ly[r], ly[r]); LZ[r] = f2_pack(lz[r], lz[r]);
    ks[r] = kc[r] = 0ull;
    ksd[r] = kcd[r] = 0.f;
  }
  for (int32_t j0 = it.j0; j0 < it.j1; j0 += T) {
    stage_tile32<R>(S, A, base, j0, it.j1, cx, cy, cz);
    __syncthreads();
    const int jend = min(T, it.j1 - j0);
    if (j0 == it.i0 || checked) {
      // per-pair path: j > i on the diagonal tile, every pair when recomputing
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!vi[r]) continue;
        const int jstart = (j0 == it.i0) ? tid + kB32 * r + 1 : 0;
        for (int jj = jstart; jj < jend; ++jj)
          pair_checked(S, jj, hx[r], hy[r], hz[r], lx[r], ly[r], lz[r], ksd[r], kcd[r]);
      }
    } else {
      const int np = ((jend + 2 * kGroup32 - 1) / (2 * kGroup32)) * kGroup32;  // partner pairs, padded
      const ulonglong2* Sa = reinterpret_cast<const ulonglong2*>(S.a);
      const ulonglong2* Sb = reinterpret_cast<const ulonglong2*>(S.b);
      const ulonglong2* Sc = reinterpret_cast<const ulonglong2*>(S.c);
      const f2_t* Sd = reinterpret_cast<const f2_t*>(S.d);
      for (int q0 = 0; q0 < np; q0 += kGroup32) {
        f2_t acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0ull;
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
    mine += A.mass[base + it.i0 + tid + kB32 * r] * row;
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
    if (code == 2) tot = epot32_item<4>(S, sh, A, it, false);
    else if (code == 1) tot = epot32_item<2>(S, sh, A, it, false);
    else tot = epot32_item<1>(S, sh, A, it, false);
    // a zero separation in the fast path shows as a non-finite sum: recompute
    // the item with the per-pair test (block-uniform decision)
    if (__syncthreads_or(tid == 0 && !isfinite(tot))) {
      if (code == 2) tot = epot32_item<4>(S, sh, A, it, true);
      else if (code == 1) tot = epot32_item<2>(S, sh, A, it, true);
      else tot = epot32_item<1>(S, sh, A, it, true);
    }
    if (tid == 0) part[w] = tot;
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
  const void* ptr[15];
  int64_t nch;
  int64_t nhalo;
  int32_t n64, n32, grid64, grid32, epot, pad;
};

struct HaloEngine {
  DevBuf d_off, d_pos, d_vel, d_mass, d_dens, d_out;  // staging for host inputs
  ListBufs l64, l32, tune;
  DevBuf d_hshape, d_counter, d_err;
  DevBuf d_mch, d_mcoff, d_mp1, d_mp2, d_mcen;  // chunked moment passes
  int64_t nch = 0;
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
  AHOP_CUDA_TRY(H.d_err.ensure(16));
  AHOP_CUDA_TRY(H.d_counter.ensure(16));
  A.err = H.d_err.as<int>();
  const int epot = p->epot & 3;
  int rc;
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
  // chunks of the moment passes
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
  AHOP_CUDA_TRY(H.d_mp1.ensure(std::max<size_t>(mch.size() * sizeof(MomP1), 16)));
  AHOP_CUDA_TRY(H.d_mp2.ensure(std::max<size_t>(mch.size() * sizeof(MomP2), 16)));
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
    const void* ptrs[15] = {H.l64.items.p, H.l64.order.p, H.l64.hoff.p, H.l64.part.p, H.l32.items.p,
                            H.l32.order.p, H.l32.hoff.p, H.l32.part.p, H.d_hshape.p, H.d_counter.p,
                            H.d_mch.p,     H.d_mcoff.p,   H.d_mp1.p,    H.d_mp2.p,    H.d_mcen.p};
    memcpy(sig.ptr, ptrs, sizeof ptrs);
    sig.nch = H.nch;
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
  if ((rc = halo_run(H, p, H.d_off.as<int64_t>(), off, nhalo, H.d_pos.as<double>(), H.d_vel.as<double>(),
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
