// Internal arguments of the batched halo-property kernels.
#pragma once
#include <cstdint>

#include "ahop_b200.h"

namespace ahop {

constexpr int kHaloFields = AHOP_HALO_NFIELDS;

struct HaloArgs {
  const int64_t* off;     // [nhalo+1] member offsets
  const double* pos;      // [n][3]
  const double* vel;      // [n][3]
  const double* mass;     // [n]
  const double* dens;     // [n]
  double* out;            // [nhalo][kHaloFields]
  double L, h, hub, G;    // period, half period, Hubble constant, gravitational constant
  int periodic;
  int sc;                 // shrinking-sphere centre (H.SC)
  double dcell_min, eps_sc;
  int* err;               // set when a bounded device loop hits its cap
};

}  // namespace ahop
