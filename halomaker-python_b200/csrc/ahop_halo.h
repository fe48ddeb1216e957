// Internal arguments of the batched halo-property kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

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
  int cdm;                // centre = member closest to the centre of mass (H.cdm)
  int64_t ndm;            // members with particle index < ndm are dark matter (H.ndm)
  double massp;           // dark-matter members heavier than massp * 1.00001 are contamination
  const int32_t* index;   // [n] particle index per member (indexps), or null: every member is dark matter
  // members in Morton order about their halo centre: (x, y, z relative to the
  // centre, mass) per member; null: the FP32-compensated form reads pos/mass
  const double4* srel;
};

}  // namespace ahop
