// Differentiable pieces: the SPH density with fixed neighbour lists and its
// adjoint, and the gradient of the direct-sum halo potential.
//
// Density (omp_compute_density, f90:2816-2838) for particle i with its list of
// nv neighbours n_0..n_{nv-1} sorted by distance at the list's reference
// configuration:
//   r = d_{nv-1} / 2,  u_k = d_k / r,
//   rho_i = C (sum_{k<nv-1} m_{n_k} W(u_k) + m_i) / r^3,  C = xyzlong / pi_f,
// with the reference's periodic distance.  The forward uses the same
// explicitly rounded arithmetic as the finder, so with the finder's own lists
// it reproduces the finder's densities bit for bit.
// Adjoint: with upstream g_i = dL/drho_i and e_k the unit separation
// (min-image, pointing from i to n_k),
//   drho_i/dd_k     = C m_{n_k} W'(u_k) / r^4                       (k < nv-1)
//   drho_i/dd_{nv-1} = (C/2) [ -sum_k m_{n_k} W'(u_k) d_k / r^5 - 3 S / r^4 ]
//   dL/dx_{n_k} += g_i drho_i/dd_k e_k,   dL/dx_i -= g_i drho_i/dd_k e_k.
// The weights are recomputed from positions (nothing is stored between the
// passes); contributions are scattered with FP64 atomics.
//
// Potential gradient (det_halo_energies_1b3 CHP:1413-1427 direct sum,
// E_h = -G sum_{i<j} m_i m_j / r_ij):
//   dE_h/dx_i = G m_i sum_{j != i} m_j (x_i - x_j) / r_ij^3  = -F_i,
// evaluated per halo over all member pairs, positions taken relative to the
// halo's densest member with the reference's strict min-image rule; scaled by
// an upstream weight per halo.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"
#include "exact.cuh"

namespace ahop {

__device__ __forceinline__ double spline_deriv(double x) {
  // d/dx of the cubic spline of f90:3270-3287
  if (x <= 1.0) return -3.0 * x + 2.25 * x * x;
  if (x <= 2.0) {
    const double y = 2.0 - x;
    return -0.75 * y * y;
  }
  return 0.0;
}

// signed min-image separation b - a along one axis (|.| as in the reference)
__device__ __forceinline__ double pdelta(double a, double b, double L) {
  double d = b - a;
  if (d > 0.5 * L) d -= L;
  else if (d < -0.5 * L) d += L;
  return d;
}

struct AdjArgs {
  const double* pos;   // [n][3]
  const double* mass;  // [n]
  const int32_t* nei;  // [n][nv], 0-based
  int64_t n;
  int nv;
  double Lx, Ly, Lz, xyzlong;
};

__global__ void density_fixed_kernel(AdjArgs A, double* __restrict__ dens) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const double* pi = A.pos + 3 * i;
  const int32_t* nb = A.nei + (size_t)A.nv * i;
  const int64_t jl = nb[A.nv - 1];
  const double dl = pdist2(pi[0], pi[1], pi[2], A.pos[3 * jl], A.pos[3 * jl + 1], A.pos[3 * jl + 2], A.Lx, A.Ly, A.Lz);
  const double r = xmul(xsqrt(dl), 0.5);
  const double r3 = xmul(xmul(r, r), r);
  const double unsr = xdiv(1.0, r);
  double contrib = 0.0;
  for (int k = 0; k < A.nv - 1; ++k) {
    const int64_t j = nb[k];
    const double d2 = pdist2(pi[0], pi[1], pi[2], A.pos[3 * j], A.pos[3 * j + 1], A.pos[3 * j + 2], A.Lx, A.Ly, A.Lz);
    contrib = xadd(contrib, xmul(A.mass[j], spline(xmul(xsqrt(d2), unsr))));
  }
  const double pi_f = (double)3.141592654f;
  dens[i] = xdiv(xmul(A.xyzlong, xadd(contrib, A.mass[i])), xmul(pi_f, r3));
}

__global__ void density_adjoint_kernel(AdjArgs A, const double* __restrict__ gdens, double* __restrict__ gpos) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const double g = gdens[i];
  if (g == 0.0) return;
  const double* pi = A.pos + 3 * i;
  const int32_t* nb = A.nei + (size_t)A.nv * i;
  const double C = A.xyzlong / (double)3.141592654f;
  const int64_t jl = nb[A.nv - 1];
  const double lx = pdelta(pi[0], A.pos[3 * jl], A.Lx), ly = pdelta(pi[1], A.pos[3 * jl + 1], A.Ly),
               lz = pdelta(pi[2], A.pos[3 * jl + 2], A.Lz);
  const double dlast = sqrt(lx * lx + ly * ly + lz * lz);
  const double r = 0.5 * dlast;
  double S = A.mass[i], T = 0.0;  // T = sum m W'(u) d
  double gi0 = 0, gi1 = 0, gi2 = 0;
  const double r4 = r * r * r * r;
  for (int k = 0; k < A.nv - 1; ++k) {
    const int64_t j = nb[k];
    const double dx = pdelta(pi[0], A.pos[3 * j], A.Lx), dy = pdelta(pi[1], A.pos[3 * j + 1], A.Ly),
                 dz = pdelta(pi[2], A.pos[3 * j + 2], A.Lz);
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    const double u = d / r;
    const double mj = A.mass[j];
    S += mj * spline(u);
    const double wp = spline_deriv(u);
    T += mj * wp * d;
    if (d > 0.0) {
      const double a = g * C * mj * wp / r4 / d;  // times the separation vector = times e_k
      atomicAdd(&gpos[3 * j], a * dx);
      atomicAdd(&gpos[3 * j + 1], a * dy);
      atomicAdd(&gpos[3 * j + 2], a * dz);
      gi0 -= a * dx; gi1 -= a * dy; gi2 -= a * dz;
    }
  }
  // through r = d_last / 2
  const double drho_dr = C * (-T / (r4 * r) - 3.0 * S / r4);  // d rho / d r = C [-T/r^5 - 3 S/r^4]
  if (dlast > 0.0) {
    const double a = g * 0.5 * drho_dr / dlast;
    atomicAdd(&gpos[3 * jl], a * lx);
    atomicAdd(&gpos[3 * jl + 1], a * ly);
    atomicAdd(&gpos[3 * jl + 2], a * lz);
    gi0 -= a * lx; gi1 -= a * ly; gi2 -= a * lz;
  }
  atomicAdd(&gpos[3 * i], gi0);
  atomicAdd(&gpos[3 * i + 1], gi1);
  atomicAdd(&gpos[3 * i + 2], gi2);
}

// dE/dx for every member: one block per (halo, 256-member tile); each thread
// sums over all members of its halo.  Positions relative to the member at
// centre_index (the densest member) with the strict min-image rule.
__global__ void __launch_bounds__(256) epot_grad_kernel(const int64_t* __restrict__ off,
                                                       const int32_t* __restrict__ item_h,
                                                       const int32_t* __restrict__ item_i, int32_t nitems,
                                                       const double* __restrict__ pos, const double* __restrict__ mass,
                                                       const int32_t* __restrict__ centre, const double* __restrict__ gh,
                                                       double L, int periodic, double G, double* __restrict__ gpos) {
  __shared__ double sx[256], sy[256], sz[256], sm[256];
  const int32_t w = blockIdx.x;
  if (w >= nitems) return;
  const int32_t h = item_h[w];
  const int64_t base = off[h];
  const int32_t n = (int32_t)(off[h + 1] - base);
  const int64_t c = base + centre[h];
  const double cx = pos[3 * c], cy = pos[3 * c + 1], cz = pos[3 * c + 2];
  auto rel = [&](double v, double cc) {
    double d = v - cc;
    if (periodic) {
      if (d > 0.5 * L) d -= L;
      if (d < -0.5 * L) d += L;
    }
    return d;
  };
  const int32_t i = item_i[w] + threadIdx.x;
  const bool vi = i < n;
  double xi = 0, yi = 0, zi = 0;
  if (vi) { xi = rel(pos[3 * (base + i)], cx); yi = rel(pos[3 * (base + i) + 1], cy); zi = rel(pos[3 * (base + i) + 2], cz); }
  double ax = 0, ay = 0, az = 0;
  for (int32_t j0 = 0; j0 < n; j0 += 256) {
    const int32_t j = j0 + threadIdx.x;
    if (j < n) {
      sx[threadIdx.x] = rel(pos[3 * (base + j)], cx);
      sy[threadIdx.x] = rel(pos[3 * (base + j) + 1], cy);
      sz[threadIdx.x] = rel(pos[3 * (base + j) + 2], cz);
      sm[threadIdx.x] = mass[base + j];
    }
    __syncthreads();
    if (vi) {
      const int jend = min(256, n - j0);
      // the member itself (r2 = 0) and coincident members drop out, as in
      // the forward sum; one double reciprocal square root per pair
#pragma unroll 4
      for (int jj = 0; jj < jend; ++jj) {
        const double dx = xi - sx[jj], dy = yi - sy[jj], dz = zi - sz[jj];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0.0) {
          const double inv = rsqrt(r2);
          const double f = sm[jj] * (inv * inv * inv);
          ax += f * dx; ay += f * dy; az += f * dz;
        }
      }
    }
    __syncthreads();
  }
  if (vi) {
    const double s = gh[h] * G * mass[base + i];
    gpos[3 * (base + i)] += s * ax;
    gpos[3 * (base + i) + 1] += s * ay;
    gpos[3 * (base + i) + 2] += s * az;
  }
}

}  // namespace ahop

using namespace ahop;

extern "C" {

int ahop_density_fixed(const AhopAdjParams* p, const double* d_pos, const double* d_mass, const int32_t* d_nei,
                       int64_t n, double* d_dens, void* stream) {
  if (!p || p->nvoisins < 2 || n <= 0) { set_error("bad density_fixed arguments"); return AHOP_EINVAL; }
  AdjArgs A{d_pos, d_mass, d_nei, n, p->nvoisins, p->xlong, p->ylong, p->zlong, p->xlong * p->ylong * p->zlong};
  density_fixed_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(A, d_dens);
  AHOP_CUDA_TRY(cudaGetLastError());
  return AHOP_OK;
}

int ahop_density_adjoint(const AhopAdjParams* p, const double* d_pos, const double* d_mass, const int32_t* d_nei,
                         int64_t n, const double* d_gdens, double* d_gpos, void* stream) {
  if (!p || p->nvoisins < 2 || n <= 0) { set_error("bad density_adjoint arguments"); return AHOP_EINVAL; }
  AdjArgs A{d_pos, d_mass, d_nei, n, p->nvoisins, p->xlong, p->ylong, p->zlong, p->xlong * p->ylong * p->zlong};
  density_adjoint_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(A, d_gdens,
                                                                                                   d_gpos);
  AHOP_CUDA_TRY(cudaGetLastError());
  return AHOP_OK;
}

int ahop_epot_grad(const AhopHaloParams* p, const int64_t* d_off, const int64_t* h_off, int64_t nhalo,
                   const double* d_pos, const double* d_mass, const int32_t* d_centre, const double* d_gh,
                   double* d_gpos, void* stream) {
  if (!p || nhalo < 0 || !h_off) { set_error("bad epot_grad arguments"); return AHOP_EINVAL; }
  std::vector<int32_t> ih, ii;
  for (int64_t h = 0; h < nhalo; ++h)
    for (int64_t i0 = 0; i0 < h_off[h + 1] - h_off[h]; i0 += 256) { ih.push_back((int32_t)h); ii.push_back((int32_t)i0); }
  if (ih.empty()) return AHOP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DevBuf items;
  AHOP_CUDA_TRY(items.ensure(ih.size() * 8));
  int32_t* d_ih = items.as<int32_t>();
  int32_t* d_ii = d_ih + ih.size();
  AHOP_CUDA_TRY(cudaMemcpyAsync(d_ih, ih.data(), ih.size() * 4, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(d_ii, ii.data(), ii.size() * 4, cudaMemcpyHostToDevice, st));
  epot_grad_kernel<<<(unsigned)ih.size(), 256, 0, st>>>(d_off, d_ih, d_ii, (int32_t)ih.size(), d_pos, d_mass,
                                                        d_centre, d_gh, p->Lbox, p->periodic, p->gravconst, d_gpos);
  AHOP_CUDA_TRY(cudaGetLastError());
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  items.release();
  return AHOP_OK;
}

}  // extern "C"
