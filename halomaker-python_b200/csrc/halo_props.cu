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
// mass (n) and density (n), FP64 in HBM.  One block per halo computes the
// O(n) quantities (two passes over the members, fixed-order block
// reductions, so results are deterministic).  The O(n^2) potential runs as
// one persistent launch over a work list of (halo, i-tile) items sorted by
// decreasing cost; each item sums m_j / r_ij for its 256 i-particles over all
// j > i.  Two forms share the schedule:
//   * FP64: relative positions, 1/r from the double reciprocal square root;
//   * FP32-compensated: positions relative to the halo centre split into
//     hi = float(r) and lo = float(r - hi) (float4 tiles in shared memory);
//     a pair separation is (hi_j - hi_i) + (lo_j - lo_i) in FP32, 1/r from
//     rsqrtf, partial sums Kahan-compensated in FP32 and folded into FP64 per
//     item.
// Per-item partials are reduced per halo in item order (deterministic).
#include <cuda_runtime.h>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>
#include <algorithm>
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

template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  T r = 0;
  if (tid < 32) {
    r = (tid < kPB / 32) ? sh[tid] : T(0);
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
    s_c[0] = A.pos[3 * ii]; s_c[1] = A.pos[3 * ii + 1]; s_c[2] = A.pos[3 * ii + 2];
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

// Potential pair sums.  Work item w: halo item_h[w], i-tile start item_i[w].
template <bool FP32C>
__global__ void __launch_bounds__(kPB) epot_pairs_kernel(HaloArgs A, const int32_t* __restrict__ item_h,
                                                         const int32_t* __restrict__ item_i, int32_t nitems,
                                                         int32_t* __restrict__ counter, double* __restrict__ part) {
  __shared__ float4 s_h[kPB], s_l[kPB];  // FP32 form: (hi x, hi y, hi z, mass), (lo x, lo y, lo z, -)
  __shared__ double s_dx[kPB], s_dy[kPB], s_dz[kPB], s_dm[kPB];
  __shared__ double sh[kPB / 32];
  __shared__ int32_t s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int32_t w = s_item;
    __syncthreads();
    if (w >= nitems) break;
    const int32_t h = item_h[w];
    const int64_t base = A.off[h];
    const int32_t n = (int32_t)(A.off[h + 1] - base);
    const int32_t i0 = item_i[w];
    const double* c = A.out + (size_t)kHaloFields * h;
    const double cx = c[HP_PX], cy = c[HP_PY], cz = c[HP_PZ];
    const int32_t i = i0 + tid;
    const bool vi = i < n;
    double rxi = 0, ryi = 0, rzi = 0;
    if (vi) {
      rxi = wrap_chp(A.pos[3 * (base + i)] - cx, A.L, A.h, A.periodic);
      ryi = wrap_chp(A.pos[3 * (base + i) + 1] - cy, A.L, A.h, A.periodic);
      rzi = wrap_chp(A.pos[3 * (base + i) + 2] - cz, A.L, A.h, A.periodic);
    }
    const float hxi = (float)rxi, hyi = (float)ryi, hzi = (float)rzi;
    const float lxi = (float)(rxi - (double)hxi), lyi = (float)(ryi - (double)hyi), lzi = (float)(rzi - (double)hzi);
    float ks = 0.f, kc = 0.f;  // Kahan sum / compensation (FP32 form)
    double ds = 0.0;           // FP64 form
    for (int32_t j0 = i0; j0 < n; j0 += kPB) {
      const int32_t j = j0 + tid;
      if (j < n) {
        const double rx = wrap_chp(A.pos[3 * (base + j)] - cx, A.L, A.h, A.periodic);
        const double ry = wrap_chp(A.pos[3 * (base + j) + 1] - cy, A.L, A.h, A.periodic);
        const double rz = wrap_chp(A.pos[3 * (base + j) + 2] - cz, A.L, A.h, A.periodic);
        if (FP32C) {
          const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
          s_h[tid] = make_float4(hx, hy, hz, (float)A.mass[base + j]);
          s_l[tid] = make_float4((float)(rx - (double)hx), (float)(ry - (double)hy), (float)(rz - (double)hz), 0.f);
        } else {
          s_dx[tid] = rx; s_dy[tid] = ry; s_dz[tid] = rz; s_dm[tid] = A.mass[base + j];
        }
      } else {
        if (FP32C) { s_h[tid] = make_float4(3.0e30f, 3.0e30f, 3.0e30f, 0.f); s_l[tid] = make_float4(0.f, 0.f, 0.f, 0.f); }
        else { s_dm[tid] = 0.0; s_dx[tid] = s_dy[tid] = s_dz[tid] = 3.0e30; }
      }
      __syncthreads();
      if (vi) {
        const int jstart = (j0 == i0) ? tid + 1 : 0;  // j > i on the diagonal tile
        const int jend = min(kPB, n - j0);
        if (FP32C) {
#pragma unroll 8
          for (int jj = jstart; jj < jend; ++jj) {
            const float4 hj = s_h[jj], lj = s_l[jj];
            const float dx = (hj.x - hxi) + (lj.x - lxi);
            const float dy = (hj.y - hyi) + (lj.y - lyi);
            const float dz = (hj.z - hzi) + (lj.z - lzi);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            // hardware reciprocal square root (a few ulp): per-halo sums stay
            // within the 1e-6 bound of the FP64 form (checked by the tests)
            const float t = (r2 > 0.f) ? hj.w * rsqrtf(r2) : 0.f;
            const float y = t - kc;
            const float s2 = ks + y;
            kc = (s2 - ks) - y;
            ks = s2;
          }
        } else {
#pragma unroll 4
          for (int jj = jstart; jj < jend; ++jj) {
            const double dx = s_dx[jj] - rxi, dy = s_dy[jj] - ryi, dz = s_dz[jj] - rzi;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0.0) ds += s_dm[jj] * rsqrt(r2);
          }
        }
      }
      __syncthreads();
    }
    double mine = 0.0;
    if (vi) {
      const double mi = A.mass[base + i];
      mine = FP32C ? mi * ((double)ks - (double)kc) : mi * ds;
    }
    const double tot = block_sum(mine, sh);
    if (tid == 0) part[w] = tot;
  }
}

// FP32-compensated pair sums with two i-rows per thread: 128 threads cover
// an item's 256 rows (rows tid and tid + 128), so every float4 pair of
// shared-memory loads serves two pairs.  Same schedule, same per-item partial
// and the same arithmetic per pair as epot_pairs_kernel<true>.
constexpr int kPB2 = kPB / 2;

__device__ __forceinline__ float pair_term(const float4& hj, const float4& lj, float hx, float hy, float hz,
                                           float lx, float ly, float lz) {
  const float dx = (hj.x - hx) + (lj.x - lx);
  const float dy = (hj.y - hy) + (lj.y - ly);
  const float dz = (hj.z - hz) + (lj.z - lz);
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  return (r2 > 0.f) ? hj.w * rsqrtf(r2) : 0.f;
}

__device__ __forceinline__ void kahan_add(float t, float& ks, float& kc) {
  const float y = t - kc;
  const float s2 = ks + y;
  kc = (s2 - ks) - y;
  ks = s2;
}

__device__ __forceinline__ void kahan_pair(const float4& hj, const float4& lj, float hx, float hy, float hz,
                                           float lx, float ly, float lz, float& ks, float& kc) {
  kahan_add(pair_term(hj, lj, hx, hy, hz, lx, ly, lz), ks, kc);
}

__global__ void __launch_bounds__(kPB2) epot_pairs32_kernel(HaloArgs A, const int32_t* __restrict__ item_h,
                                                            const int32_t* __restrict__ item_i, int32_t nitems,
                                                            int32_t* __restrict__ counter,
                                                            double* __restrict__ part) {
  __shared__ float4 s_h[kPB], s_l[kPB];
  __shared__ double sh[kPB2 / 32];
  __shared__ int32_t s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int32_t w = s_item;
    __syncthreads();
    if (w >= nitems) break;
    const int32_t h = item_h[w];
    const int64_t base = A.off[h];
    const int32_t n = (int32_t)(A.off[h + 1] - base);
    const int32_t i0 = item_i[w];
    const double* c = A.out + (size_t)kHaloFields * h;
    const double cx = c[HP_PX], cy = c[HP_PY], cz = c[HP_PZ];
    float hx[2], hy[2], hz[2], lx[2], ly[2], lz[2], ks[2] = {0.f, 0.f}, kc[2] = {0.f, 0.f};
    bool vi[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int32_t i = i0 + tid + r * kPB2;
      vi[r] = i < n;
      double rx = 0, ry = 0, rz = 0;
      if (vi[r]) {
        rx = wrap_chp(A.pos[3 * (base + i)] - cx, A.L, A.h, A.periodic);
        ry = wrap_chp(A.pos[3 * (base + i) + 1] - cy, A.L, A.h, A.periodic);
        rz = wrap_chp(A.pos[3 * (base + i) + 2] - cz, A.L, A.h, A.periodic);
      }
      hx[r] = (float)rx; hy[r] = (float)ry; hz[r] = (float)rz;
      lx[r] = (float)(rx - (double)hx[r]); ly[r] = (float)(ry - (double)hy[r]); lz[r] = (float)(rz - (double)hz[r]);
    }
    for (int32_t j0 = i0; j0 < n; j0 += kPB) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int32_t t = tid + r * kPB2;
        const int32_t j = j0 + t;
        if (j < n) {
          const double rx = wrap_chp(A.pos[3 * (base + j)] - cx, A.L, A.h, A.periodic);
          const double ry = wrap_chp(A.pos[3 * (base + j) + 1] - cy, A.L, A.h, A.periodic);
          const double rz = wrap_chp(A.pos[3 * (base + j) + 2] - cz, A.L, A.h, A.periodic);
          const float fx = (float)rx, fy = (float)ry, fz = (float)rz;
          s_h[t] = make_float4(fx, fy, fz, (float)A.mass[base + j]);
          s_l[t] = make_float4((float)(rx - (double)fx), (float)(ry - (double)fy), (float)(rz - (double)fz), 0.f);
        } else {
          s_h[t] = make_float4(3.0e30f, 3.0e30f, 3.0e30f, 0.f);
          s_l[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      __syncthreads();
      const int jend = min(kPB, n - j0);
      if (j0 == i0) {
        // diagonal tile: j > i for each row (row 0 is tile row tid, row 1 is tid + kPB2)
        for (int jj = tid + 1; jj < jend; ++jj) {
          const float4 hj = s_h[jj], lj = s_l[jj];
          if (vi[0]) kahan_pair(hj, lj, hx[0], hy[0], hz[0], lx[0], ly[0], lz[0], ks[0], kc[0]);
          if (vi[1] && jj > tid + kPB2) kahan_pair(hj, lj, hx[1], hy[1], hz[1], lx[1], ly[1], lz[1], ks[1], kc[1]);
        }
      } else if (vi[0]) {
        // groups of four partners: the four terms of a row are added as a
        // small tree (independent work), then the group enters the
        // compensated sum once -- one dependent chain per four pairs
        int jj = 0;
        for (; jj + 4 <= jend; jj += 4) {
          float g[2];
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const float t0 = pair_term(s_h[jj], s_l[jj], hx[r], hy[r], hz[r], lx[r], ly[r], lz[r]);
            const float t1 = pair_term(s_h[jj + 1], s_l[jj + 1], hx[r], hy[r], hz[r], lx[r], ly[r], lz[r]);
            const float t2 = pair_term(s_h[jj + 2], s_l[jj + 2], hx[r], hy[r], hz[r], lx[r], ly[r], lz[r]);
            const float t3 = pair_term(s_h[jj + 3], s_l[jj + 3], hx[r], hy[r], hz[r], lx[r], ly[r], lz[r]);
            g[r] = (t0 + t1) + (t2 + t3);
          }
          kahan_add(g[0], ks[0], kc[0]);
          kahan_add(g[1], ks[1], kc[1]);
        }
        for (; jj < jend; ++jj) {
          const float4 hj = s_h[jj], lj = s_l[jj];
          kahan_pair(hj, lj, hx[0], hy[0], hz[0], lx[0], ly[0], lz[0], ks[0], kc[0]);
          kahan_pair(hj, lj, hx[1], hy[1], hz[1], lx[1], ly[1], lz[1], ks[1], kc[1]);
        }
      }
      __syncthreads();
    }
    double mine = 0.0;
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (vi[r]) mine += A.mass[base + i0 + tid + r * kPB2] * ((double)ks[r] - (double)kc[r]);
    // block sum over kPB2 threads
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((tid & 31) == 0) sh[tid >> 5] = mine;
    __syncthreads();
    if (tid == 0) {
      double tot = 0.0;
      for (int k = 0; k < kPB2 / 32; ++k) tot += sh[k];
      part[w] = tot;
    }
    __syncthreads();
  }
}

// per-halo reduction of item partials (items of a halo are contiguous in the
// halo-ordered list hitem_off), then E_pot, totals and spin
__global__ void epot_finalize_kernel(HaloArgs A, const int64_t* __restrict__ hitem_off,
                                     const int32_t* __restrict__ order, const double* __restrict__ part64,
                                     const double* __restrict__ part32, int64_t nhalo) {
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  double s64 = 0, s32 = 0;
  for (int64_t k = hitem_off[h]; k < hitem_off[h + 1]; ++k) {
    const int32_t w = order[k];
    if (part64) s64 += part64[w];
    if (part32) s32 += part32[w];
  }
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

struct HaloEngine {
  DevBuf d_off, d_pos, d_vel, d_mass, d_dens, d_out;  // staging for host inputs
  DevBuf d_item_h, d_item_i, d_part64, d_part32, d_counter, d_hoff, d_order, d_err;
  cudaEvent_t ev[5] = {};
  bool ready = false;
  cudaStream_t own = nullptr;
  AhopHaloTimings t{};
  std::vector<int64_t> h_off;
};

static HaloEngine& halo_engine() {
  static HaloEngine* e = new HaloEngine();
  return *e;
}

static int halo_run(HaloEngine& H, const AhopHaloParams* p, const int64_t* d_off, const int64_t* h_off,
                    int64_t nhalo, const double* d_pos, const double* d_vel, const double* d_mass,
                    const double* d_dens, double* d_out, cudaStream_t st) {
  if (!H.ready) {
    for (auto& e : H.ev) AHOP_CUDA_TRY(cudaEventCreate(&e));
    H.ready = true;
  }
  // work list: (halo, i-tile) items sorted by decreasing pair cost
  std::vector<int64_t> cost;
  std::vector<int32_t> ih, ii;
  std::vector<int64_t> hoff(nhalo + 1, 0);
  double pairs = 0;
  for (int64_t h = 0; h < nhalo; ++h) {
    const int64_t n = h_off[h + 1] - h_off[h];
    if (n < 0 || n > INT32_MAX) { set_error("halo member count out of range"); return AHOP_EINVAL; }
    pairs += 0.5 * (double)n * (double)(n - 1);
    hoff[h] = (int64_t)ih.size();
    for (int64_t i0 = 0; i0 < n; i0 += kPB) {
      ih.push_back((int32_t)h);
      ii.push_back((int32_t)i0);
      cost.push_back((n - i0) * (int64_t)kPB);
    }
  }
  hoff[nhalo] = (int64_t)ih.size();
  const int32_t nitems = (int32_t)ih.size();
  std::vector<int32_t> sorted(nitems);
  for (int32_t k = 0; k < nitems; ++k) sorted[k] = k;
  std::stable_sort(sorted.begin(), sorted.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
  std::vector<int32_t> sh(nitems), si(nitems), order(nitems);
  for (int32_t k = 0; k < nitems; ++k) {
    sh[k] = ih[sorted[k]];
    si[k] = ii[sorted[k]];
    order[sorted[k]] = k;  // halo-ordered item k runs as scheduled item order[k]
  }
  const size_t ni = (size_t)(nitems > 0 ? nitems : 1);
  AHOP_CUDA_TRY(H.d_item_h.ensure(ni * 4));
  AHOP_CUDA_TRY(H.d_item_i.ensure(ni * 4));
  AHOP_CUDA_TRY(H.d_order.ensure(ni * 4));
  AHOP_CUDA_TRY(H.d_part64.ensure(ni * 8));
  AHOP_CUDA_TRY(H.d_part32.ensure(ni * 8));
  AHOP_CUDA_TRY(H.d_counter.ensure(16));
  AHOP_CUDA_TRY(H.d_hoff.ensure((size_t)(nhalo + 1) * 8));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_item_h.p, sh.data(), nitems * 4, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_item_i.p, si.data(), nitems * 4, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_order.p, order.data(), nitems * 4, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(H.d_hoff.p, hoff.data(), (nhalo + 1) * 8, cudaMemcpyHostToDevice, st));
  HaloArgs A;
  A.off = d_off; A.pos = d_pos; A.vel = d_vel; A.mass = d_mass; A.dens = d_dens; A.out = d_out;
  A.L = p->Lbox; A.h = 0.5 * p->Lbox; A.hub = p->Hub_pt; A.G = p->gravconst; A.periodic = p->periodic != 0;
  A.sc = p->sc != 0; A.dcell_min = p->dcell_min; A.eps_sc = p->eps_sc;
  AHOP_CUDA_TRY(H.d_err.ensure(16));
  AHOP_CUDA_TRY(cudaMemsetAsync(H.d_err.p, 0, 4, st));
  A.err = H.d_err.as<int>();
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int launches = 0;
  AHOP_CUDA_TRY(cudaEventRecord(H.ev[0], st));
  if (nhalo > 0) {
    halo_moments_kernel<<<(unsigned)nhalo, kPB, 0, st>>>(A);
    ++launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecord(H.ev[1], st));
  if ((p->epot & 1) && nitems > 0) {
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, epot_pairs_kernel<false>, kPB, 0);
    AHOP_CUDA_TRY(cudaMemsetAsync(H.d_counter.p, 0, 4, st));
    epot_pairs_kernel<false><<<nsm * (per > 0 ? per : 1), kPB, 0, st>>>(
        A, H.d_item_h.as<int32_t>(), H.d_item_i.as<int32_t>(), nitems, H.d_counter.as<int32_t>(),
        H.d_part64.as<double>());
    ++launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecord(H.ev[2], st));
  if ((p->epot & 2) && nitems > 0) {
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, epot_pairs32_kernel, kPB2, 0);
    AHOP_CUDA_TRY(cudaMemsetAsync(H.d_counter.as<int32_t>() + 1, 0, 4, st));
    epot_pairs32_kernel<<<nsm * (per > 0 ? per : 1), kPB2, 0, st>>>(
        A, H.d_item_h.as<int32_t>(), H.d_item_i.as<int32_t>(), nitems, H.d_counter.as<int32_t>() + 1,
        H.d_part32.as<double>());
    ++launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecord(H.ev[3], st));
  if (nhalo > 0) {
    epot_finalize_kernel<<<(unsigned)((nhalo + 127) / 128), 128, 0, st>>>(
        A, H.d_hoff.as<int64_t>(), H.d_order.as<int32_t>(), (p->epot & 1) ? H.d_part64.as<double>() : nullptr,
        (p->epot & 2) ? H.d_part32.as<double>() : nullptr, nhalo);
    ++launches;
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecord(H.ev[4], st));
  int herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, H.d_err.p, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) { set_error("shrinking-sphere centre: step limit reached"); return AHOP_ELIMIT; }
  auto el = [&](int a, int b) { float ms = 0; cudaEventElapsedTime(&ms, H.ev[a], H.ev[b]); return ms; };
  H.t.moments = el(0, 1);
  H.t.epot64 = el(1, 2);
  H.t.epot32c = el(2, 3);
  H.t.finalize = el(3, 4);
  H.t.total = el(0, 4);
  H.t.pairs = pairs;
  H.t.items = nitems;
  H.t.kernel_launches = launches;
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
  int32_t item_h[kNoAllocMaxItems];
  int32_t item_i[kNoAllocMaxItems];
  int32_t order[kNoAllocMaxItems];
  double part64[kNoAllocMaxItems];
  double part32[kNoAllocMaxItems];
  int64_t hoff[kNoAllocMaxHalos + 1];
  int32_t counter[4];  // [0],[1]: work counters of the two pair kernels; [2]: item total; [3]: error
};

// ~7.9 MB; in host code this name is only a host-side stand-in, the device
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
      nit = n > 0 ? (n + kPB - 1) / kPB : 0;
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

// Work items in halo order (no cost sort: per-item partials and the per-halo
// fold order do not depend on the schedule, so results match the allocating
// entry point bit for bit).
__global__ void noalloc_items_kernel(const int64_t* __restrict__ off, int64_t nhalo, NoAllocScratch* S) {
  const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhalo) return;
  const int64_t n = off[h + 1] - off[h];
  int64_t k = S->hoff[h];
  for (int64_t i0 = 0; i0 < n; i0 += kPB, ++k) {
    S->item_h[k] = (int32_t)h;
    S->item_i[k] = (int32_t)i0;
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
  NoAllocScratch* S = nullptr;
  if ((rc = noalloc_setup(&S))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
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
  A.off = d_off; A.pos = d_pos; A.vel = d_vel; A.mass = d_mass; A.dens = d_density; A.out = d_out;
  A.L = p->Lbox; A.h = 0.5 * p->Lbox; A.hub = p->Hub_pt; A.G = p->gravconst; A.periodic = p->periodic != 0;
  A.sc = p->sc != 0; A.dcell_min = p->dcell_min; A.eps_sc = p->eps_sc;
  A.err = &S->counter[3];
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  halo_moments_kernel<<<(unsigned)nhalo, kPB, 0, st>>>(A);
  AHOP_CUDA_TRY(cudaGetLastError());
  if ((p->epot & 1) && total > 0) {
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, epot_pairs_kernel<false>, kPB, 0);
    epot_pairs_kernel<false><<<nsm * (per > 0 ? per : 1), kPB, 0, st>>>(A, S->item_h, S->item_i, total,
                                                                        &S->counter[0], S->part64);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  if ((p->epot & 2) && total > 0) {
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, epot_pairs32_kernel, kPB2, 0);
    epot_pairs32_kernel<<<nsm * (per > 0 ? per : 1), kPB2, 0, st>>>(A, S->item_h, S->item_i, total,
                                                                       &S->counter[1], S->part32);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  epot_finalize_kernel<<<(unsigned)((nhalo + 127) / 128), 128, 0, st>>>(
      A, S->hoff, S->order, (p->epot & 1) ? S->part64 : nullptr, (p->epot & 2) ? S->part32 : nullptr, nhalo);
  AHOP_CUDA_TRY(cudaGetLastError());
  int32_t herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, &S->counter[3], 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) { set_error("shrinking-sphere centre: step limit reached"); return AHOP_ELIMIT; }
  return AHOP_OK;
}
