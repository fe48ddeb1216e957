// Virial properties of every halo; replaces det_vir_1b (CHP:1248-1262) of
// the reference's per-halo chain:
//   det_main_axis_1b2 (CHP:1954-1967)   principal axes: eigenpairs of the
//                                        inertia tensor, sha <= shb <= shc
//   tab_props_inside_1b40 (CHP:969-1032) nshell concentric ellipsoids along
//                                        those axes; cumulative mass and
//                                        kinetic energy (Hubble flow) per shell
//   potential_profile_1b40 (CHP:1065-1123) under the reference's default
//                                        policies: shell integration with exact
//                                        self-pair counting; halos below the
//                                        direct-sum limit are rescaled to their
//                                        direct E_pot, larger ones take the
//                                        profile's outer value as E_pot
//   det_vir_props_1b4 (CHP:1127-1229)   outermost shell meeting the virial
//                                        theorem to 20 %, else the
//                                        overdensity criterion; TSIS profile
//                                        (compute_halo_profile_1b41, 1232-1239)
//
// One block per halo.  The members are binned into shared-memory shell
// tables with atomics (the reference adds them in member order; sums agree
// to rounding); the cumulative tables, the potential profile and the scans
// of det_vir_props_1b4 then run on one thread in the reference's order.
// Centre, bulk velocity, r, E_kin, the inertia tensor and the direct E_pot
// come from the batched property kernels (ahop_halo_props*).
#include <cuda_runtime.h>
#include <cfloat>
#include <math_constants.h>

#include "ahop_halo.h"
#include "engine.h"

namespace ahop {

constexpr int kVB = 256;            // threads per halo block
constexpr int kMaxShells = 1024;    // shell-table capacity (the reference uses 1000)

struct VirArgs {
  const int64_t* off;
  const double* pos;
  const double* vel;
  const double* mass;
  const double* props;  // [nhalo][AHOP_HALO_NFIELDS]
  double* out;          // [nhalo][AHOP_VIR_NFIELDS]
  double L, h, hub, G, vir_overdens, rho_mean;
  int periodic, nshell, direct_limit, ep_field;
  int* err;
};

__device__ __forceinline__ double vwrap(double d, double L, double h, int periodic) {
  // correct_for_periodicity_1d (CHP:854-863): strict comparisons
  if (!periodic) return d;
  if (d > h) d -= L;
  if (d < -h) d += L;
  return d;
}

// Eigenpairs of the symmetric 3x3 matrix a (cyclic Jacobi); eigenvalues
// ascending in w, eigenvector k in column k of v.
__device__ void sym3_eigen(double a[3][3], double w[3], double v[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) v[i][j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off == 0.0 || off <= 1e-36 * dia) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int idx[3] = {0, 1, 2};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2 - i; ++j)
      if (a[idx[j]][idx[j]] > a[idx[j + 1]][idx[j + 1]]) { const int t = idx[j]; idx[j] = idx[j + 1]; idx[j + 1] = t; }
  double vv[3][3];
  for (int k = 0; k < 3; ++k) {
    w[k] = a[idx[k]][idx[k]];
    for (int i = 0; i < 3; ++i) vv[i][k] = v[i][idx[k]];
  }
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) v[i][k] = vv[i][k];
}

__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = sh[0];
  for (int w = 1; w < kVB / 32; ++w) r = fmax(r, sh[w]);
  __syncthreads();
  return r;
}

// projections of dr on the principal axes, in numpy's order (no contraction)
__device__ __forceinline__ void project(const double* g, double dx, double dy, double dz, double& pa, double& pb,
                                        double& pc) {
  pa = __dadd_rn(__dadd_rn(__dmul_rn(dx, g[0]), __dmul_rn(dy, g[3])), __dmul_rn(dz, g[6]));
  pb = __dadd_rn(__dadd_rn(__dmul_rn(dx, g[1]), __dmul_rn(dy, g[4])), __dmul_rn(dz, g[7]));
  pc = __dadd_rn(__dadd_rn(__dmul_rn(dx, g[2]), __dmul_rn(dy, g[5])), __dmul_rn(dz, g[8]));
}

__device__ __forceinline__ double ell_radius(double pa, double pb, double pc, double a, double b, double c) {
  const double x = __ddiv_rn(pa, a), y = __ddiv_rn(pb, b), z = __ddiv_rn(pc, c);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

__global__ void __launch_bounds__(kVB) halo_virial_kernel(VirArgs V) {
  __shared__ double s_m[kMaxShells], s_k[kMaxShells], s_p[kMaxShells];
  __shared__ int s_n[kMaxShells];
  __shared__ double s_g[16];  // eigenvector matrix (row-major, column k = axis k), sha, shb, shc, ok
  __shared__ double sh[kVB / 32];
  __shared__ int s_lost;
  const int tid = threadIdx.x;
  const int64_t h = blockIdx.x;
  const int64_t b0 = V.off[h], b1 = V.off[h + 1];
  const int nr = V.nshell;
  const double* P = V.props + (size_t)AHOP_HALO_NFIELDS * h;
  double* o = V.out + (size_t)AHOP_VIR_NFIELDS * h;
  const double m = P[HP_M];
  if (tid == 0) {
    double a[3][3] = {{P[HP_IXX], P[HP_IXY], P[HP_IXZ]}, {P[HP_IXY], P[HP_IYY], P[HP_IYZ]},
                      {P[HP_IXZ], P[HP_IYZ], P[HP_IZZ]}};
    double w[3], v[3][3];
    sym3_eigen(a, w, v);
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) s_g[3 * i + k] = v[i][k];
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
      s_g[9 + k] = sqrt(w[k] / m);  // det_main_axis_1b2: d = sqrt(eig / m)
      ok = ok && (s_g[9 + k] > 0.0) && isfinite(s_g[9 + k]);
    }
    s_g[12] = ok ? 1.0 : 0.0;
    s_lost = 0;
  }
  for (int i = tid; i < nr; i += kVB) { s_m[i] = 0.0; s_k[i] = 0.0; s_n[i] = 0; }
  __syncthreads();
  const double cx = P[HP_PX], cy = P[HP_PY], cz = P[HP_PZ];
  const double vx = P[HP_VX], vy = P[HP_VY], vz = P[HP_VZ];
  const int64_t count = b1 - b0;
  const double ek = P[HP_EK];
  double ep = P[V.ep_field];
  if (s_g[12] == 0.0) {  // degenerate axes: no shells (the reference cannot bin this halo)
    if (tid == 0) {
      for (int f = 0; f < AHOP_VIR_NFIELDS; ++f) o[f] = CUDART_NAN;
      o[VIR_EP] = ep;
      o[VIR_ET] = ek + ep;
    }
    return;
  }
  const double sha = s_g[9], shb = s_g[10], shc = s_g[11];
  // tab_props_inside_1b40: the ellipsoid through the farthest member
  double rmax = 0.0;
  for (int64_t i = b0 + tid; i < b1; i += kVB) {
    const double dx = vwrap(V.pos[3 * i] - cx, V.L, V.h, V.periodic);
    const double dy = vwrap(V.pos[3 * i + 1] - cy, V.L, V.h, V.periodic);
    const double dz = vwrap(V.pos[3 * i + 2] - cz, V.L, V.h, V.periodic);
    double pa, pb, pc;
    project(s_g, dx, dy, dz, pa, pb, pc);
    rmax = fmax(rmax, ell_radius(pa, pb, pc, sha, shb, shc));
  }
  rmax = block_max(rmax, sh);
  const double eps = 1e-2;
  const double amax = rmax * sha * (1.0 + eps), bmax = rmax * shb * (1.0 + eps), cmax = rmax * shc * (1.0 + eps);
  for (int64_t i = b0 + tid; i < b1; i += kVB) {
    const double dx = vwrap(V.pos[3 * i] - cx, V.L, V.h, V.periodic);
    const double dy = vwrap(V.pos[3 * i + 1] - cy, V.L, V.h, V.periodic);
    const double dz = vwrap(V.pos[3 * i + 2] - cz, V.L, V.h, V.periodic);
    double pa, pb, pc;
    project(s_g, dx, dy, dz, pa, pb, pc);
    const double re = ell_radius(pa, pb, pc, amax, bmax, cmax);
    const int ib = (int)__dmul_rn(re, (double)nr);
    const double tx = V.vel[3 * i] - vx + dx * V.hub;
    const double ty = V.vel[3 * i + 1] - vy + dy * V.hub;
    const double tz = V.vel[3 * i + 2] - vz + dz * V.hub;
    const double w = V.mass[i];
    if (ib >= 0 && ib < nr) {
      atomicAdd(&s_m[ib], w);
      atomicAdd(&s_k[ib], 0.5 * w * (tx * tx + ty * ty + tz * tz));
      atomicAdd(&s_n[ib], 1);
    } else {
      atomicAdd(&s_lost, 1);
    }
  }
  __syncthreads();
  if (tid != 0) return;
  if (s_lost) atomicExch(V.err, 1);  // the reference raises ValueError here
  // cumulative tables, then potential_profile_1b40 (shell / count / profile
  // outer for large) as the reference's cumulative sum
  for (int i = 1; i < nr; ++i) { s_m[i] += s_m[i - 1]; s_k[i] += s_k[i - 1]; }
  const double reff0 = pow(amax * bmax * cmax, 1.0 / 3.0);
  double acc = 0.0;
  for (int i = 0; i < nr; ++i) {
    const double dm = s_m[i] - (i > 0 ? s_m[i - 1] : 0.0);
    const double before = s_m[i] - dm;
    const double nn = (double)s_n[i];
    const double self = (s_n[i] > 0) ? 0.5 * (nn - 1.0) / nn : 0.0;
    const double scale = (i == 0) ? 0.5 / (double)(nr - 1) : (double)i / (double)(nr - 1);
    acc += (before + self * dm) * dm / (scale * reff0);
    s_p[i] = -V.G * acc;
  }
  const double outer = s_p[nr - 1];
  const bool rescale = count < V.direct_limit && ep != outer && outer != 0.0;
  if (count >= V.direct_limit) ep = outer;
  const double et = ek + ep;
  // det_vir_props_1b4
  const int ttab = nr;
  double mvir = s_m[ttab - 1];
  int i1;
  for (i1 = ttab - 1; i1 >= 1; --i1)
    if (s_m[i1 - 1] < s_m[i1]) break;
  if (i1 < 1) i1 = 1;  // the reference's loop variable ends at 1
  double avir = (double)i1 / (double)(ttab - 1) * amax;
  double bvir = (double)i1 / (double)(ttab - 1) * bmax;
  double cvir = (double)i1 / (double)(ttab - 1) * cmax;
  double rvir = pow(avir * bvir * cvir, 1.0 / 3.0);
  double virth_old = 1.0, virth = 100.0;
  for (int i0 = ttab - 1; i0 >= 0; --i0) {
    const double tp = rescale ? s_p[i0] / outer * ep : s_p[i0];
    const double tk = s_k[i0];
    if (tk + tp >= 0.0) continue;  // unbound: cannot be virialised
    virth = fabs((2.0 * tk + tp) / (tk + tp));
    if (virth < virth_old) {
      mvir = s_m[i0];
      avir = fmin(avir, (double)i0 / (double)(ttab - 1) * amax);
      bvir = fmin(bvir, (double)i0 / (double)(ttab - 1) * bmax);
      cvir = fmin(cvir, (double)i0 / (double)(ttab - 1) * cmax);
      rvir = pow(avir * bvir * cvir, 1.0 / 3.0);
      virth_old = virth;
      if (virth <= 0.20) break;
    }
  }
  const double pi = CUDART_PI;
  const double volmin = 4. / 3. * pi * (amax / (ttab - 1)) * (bmax / (ttab - 1)) * (cmax / (ttab - 1));
  if (virth > 0.20 || mvir < V.vir_overdens * V.rho_mean * 4. / 3. * pi * avir * bvir * cvir) {
    int ii1;
    for (ii1 = ttab - 1; ii1 >= 1; --ii1) {
      const double mv = V.vir_overdens * V.rho_mean * volmin * (double)ii1 * (double)ii1 * (double)ii1;
      if (s_m[ii1] >= mv && s_m[ii1 - 1] < s_m[ttab - 1]) break;
    }
    if (ii1 < 1) ii1 = 1;
    mvir = s_m[ii1];
    avir = (double)ii1 / (double)(ttab - 1) * amax;
    bvir = (double)ii1 / (double)(ttab - 1) * bmax;
    cvir = (double)ii1 / (double)(ttab - 1) * cmax;
    rvir = pow(avir * bvir * cvir, 1.0 / 3.0);
  }
  o[VIR_EP] = ep;
  o[VIR_ET] = et;
  o[VIR_AMAX] = amax;
  o[VIR_BMAX] = bmax;
  o[VIR_CMAX] = cmax;
  if (mvir > 0.0 && rvir > 0.0) {
    const double rv = fmin(rvir, P[HP_R]);
    o[VIR_RVIR] = rv;
    o[VIR_MVIR] = mvir;
    o[VIR_CVEL] = sqrt(V.G * mvir / rv);
    o[VIR_TVIR] = 35.9 * V.G * mvir / rv;
    o[VIR_RHO0] = mvir / (4.0 * pi * rv * rv * rv);
    o[VIR_RC] = rv;
  } else {
    o[VIR_RVIR] = o[VIR_MVIR] = o[VIR_CVEL] = o[VIR_TVIR] = o[VIR_RHO0] = o[VIR_RC] = CUDART_NAN;
  }
}

}  // namespace ahop

// ------------------------------------------------------------------ host side
namespace ahop {

struct VirEngine {
  DevBuf d_off, d_pos, d_vel, d_mass, d_props, d_out, d_err;
  cudaStream_t own = nullptr;
  cudaEvent_t ev[2] = {};
  float ms = 0.f;
};

static VirEngine& vir_engine() {
  static VirEngine* e = new VirEngine();
  return *e;
}

static int vir_validate(const AhopVirialParams* p, int64_t nhalo) {
  if (!p) { set_error("null params"); return AHOP_EINVAL; }
  if (nhalo < 0) { set_error("nhalo must be >= 0"); return AHOP_EINVAL; }
  if (p->nshell < 2 || p->nshell > kMaxShells) {
    set_error("nshell must be in [2, " + std::to_string(kMaxShells) + "]");
    return AHOP_EINVAL;
  }
  if (p->ep_field != HP_EP64 && p->ep_field != HP_EP32C) { set_error("ep_field must be HP_EP64 or HP_EP32C"); return AHOP_EINVAL; }
  if (p->periodic && !(p->Lbox > 0)) { set_error("Lbox must be positive for periodic boxes"); return AHOP_EINVAL; }
  return AHOP_OK;
}

static int vir_run(VirEngine& E, const AhopVirialParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                   const double* d_vel, const double* d_mass, const double* d_props, double* d_out, cudaStream_t st) {
  if (!E.ev[0]) {
    for (auto& e : E.ev) AHOP_CUDA_TRY(cudaEventCreate(&e));
  }
  AHOP_CUDA_TRY(E.d_err.ensure(16));
  AHOP_CUDA_TRY(cudaMemsetAsync(E.d_err.p, 0, 4, st));
  VirArgs V;
  V.off = d_off; V.pos = d_pos; V.vel = d_vel; V.mass = d_mass; V.props = d_props; V.out = d_out;
  V.L = p->Lbox; V.h = 0.5 * p->Lbox; V.hub = p->Hub_pt; V.G = p->gravconst;
  V.vir_overdens = p->vir_overdens; V.rho_mean = p->rho_mean;
  V.periodic = p->periodic != 0; V.nshell = p->nshell; V.direct_limit = p->direct_limit; V.ep_field = p->ep_field;
  V.err = E.d_err.as<int>();
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[0], st));
  if (nhalo > 0) {
    halo_virial_kernel<<<(unsigned)nhalo, kVB, 0, st>>>(V);
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  AHOP_CUDA_TRY(cudaEventRecord(E.ev[1], st));
  int herr = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(&herr, E.d_err.p, 4, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  cudaEventElapsedTime(&E.ms, E.ev[0], E.ev[1]);
  if (herr) {
    set_error("virial shells: a member fell outside the outermost ellipsoid");
    return AHOP_EINVARIANT;
  }
  return AHOP_OK;
}

}  // namespace ahop

using namespace ahop;

extern "C" {

int ahop_halo_virial_device(const AhopVirialParams* p, const int64_t* d_off, int64_t nhalo, const double* d_pos,
                            const double* d_vel, const double* d_mass, const double* d_props, double* d_out,
                            void* stream) {
  int rc;
  if ((rc = vir_validate(p, nhalo))) return rc;
  return vir_run(vir_engine(), p, d_off, nhalo, d_pos, d_vel, d_mass, d_props, d_out,
                 static_cast<cudaStream_t>(stream));
}

int ahop_halo_virial(const AhopVirialParams* p, const int64_t* off, int64_t nhalo, const double* pos,
                     const double* vel, const double* mass, const double* props, double* out) {
  int rc;
  if ((rc = vir_validate(p, nhalo))) return rc;
  if (!off || (nhalo > 0 && (!pos || !vel || !mass || !props || !out))) { set_error("null input"); return AHOP_EINVAL; }
  VirEngine& E = vir_engine();
  if (!E.own) AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&E.own, cudaStreamNonBlocking));
  cudaStream_t st = E.own;
  const int64_t n = off[nhalo];
  AHOP_CUDA_TRY(E.d_off.ensure((nhalo + 1) * 8));
  AHOP_CUDA_TRY(E.d_pos.ensure(n * 24 + 8));
  AHOP_CUDA_TRY(E.d_vel.ensure(n * 24 + 8));
  AHOP_CUDA_TRY(E.d_mass.ensure(n * 8 + 8));
  AHOP_CUDA_TRY(E.d_props.ensure((size_t)nhalo * AHOP_HALO_NFIELDS * 8 + 8));
  AHOP_CUDA_TRY(E.d_out.ensure((size_t)nhalo * AHOP_VIR_NFIELDS * 8 + 8));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_off.p, off, (nhalo + 1) * 8, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_pos.p, pos, n * 24, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_vel.p, vel, n * 24, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_mass.p, mass, n * 8, cudaMemcpyHostToDevice, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(E.d_props.p, props, (size_t)nhalo * AHOP_HALO_NFIELDS * 8, cudaMemcpyHostToDevice, st));
  if ((rc = vir_run(E, p, E.d_off.as<int64_t>(), nhalo, E.d_pos.as<double>(), E.d_vel.as<double>(),
                    E.d_mass.as<double>(), E.d_props.as<double>(), E.d_out.as<double>(), st)))
    return rc;
  AHOP_CUDA_TRY(cudaMemcpyAsync(out, E.d_out.p, (size_t)nhalo * AHOP_VIR_NFIELDS * 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  return AHOP_OK;
}

float ahop_halo_virial_last_ms(void) { return vir_engine().ms; }

}  // extern "C"
