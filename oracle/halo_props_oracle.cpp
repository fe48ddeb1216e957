// FP64 direct-sum potential oracle for the batched halo properties -- TEST
// INFRASTRUCTURE ONLY (checker and CPU baseline), never used by the library.
//
// For each halo: S = sum_{i<j} m_i m_j / |x_j - x_i|, the pair difference
// wrapped to the nearest image with the strict comparisons of
// det_halo_energies_1b3 (src/compute_halo_props.py:1419-1427); E_pot = -G S.
// The reference only sums pairs below 1000 members; this oracle sums them for
// every size so the GPU's FP64 and FP32-compensated forms can be checked.
#include <cmath>
#include <cstdint>
#include <omp.h>

extern "C" int halo_oracle_epot(const int64_t* off, int64_t nhalo, const double* pos, const double* mass,
                                double L, int periodic, int nthreads, double* out_sum) {
  const double h = 0.5 * L;
  for (int64_t k = 0; k < nhalo; ++k) {
    const int64_t a = off[k], b = off[k + 1];
    double total = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t i = a; i < b; ++i) {
      double s = 0.0;
      const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
      for (int64_t j = i + 1; j < b; ++j) {
        double dx = pos[3 * j] - xi, dy = pos[3 * j + 1] - yi, dz = pos[3 * j + 2] - zi;
        if (periodic) {
          if (dx > h) dx -= L;
          if (dx < -h) dx += L;
          if (dy > h) dy -= L;
          if (dy < -h) dy += L;
          if (dz > h) dz -= L;
          if (dz < -h) dz += L;
        }
        const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (r > 0.0) s += mass[j] / r;
      }
      total += mass[i] * s;
    }
    out_sum[k] = total;
  }
  return 0;
}
