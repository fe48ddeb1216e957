// AdaptaHOP CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// A C++17/OpenMP restatement of the reference's native finder
// (fortran/compute_adaptahop.f90), routine by routine and in the same
// floating-point evaluation order, so that its outputs can serve as the
// checker for the CUDA path and as the timed CPU baseline.  It must never be
// linked into, called by, or used as a fallback for the product library.
//
// Arrays are 1-based (index 0 unused) exactly like the Fortran, to keep the
// restatement auditable line by line.  Build with -O3 -fopenmp
// -ffp-contract=off and no -march flags: gfortran's default x86-64 build of
// the reference has no FMA, so every product and sum rounds separately.
//
// Parity status: the reference Fortran cannot be compiled in this container
// (no Fortran compiler); the restatement is pinned against fixtures produced
// by the reference's own Python finder (tests/golden/), see tests.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "ahop_oracle.h"

namespace {

// f90:58  pi is a default-kind (single precision) literal promoted to real(8).
const double kPi = (double)3.141592654f;
// f90:91
const int kNpartpercell = 100;
// f90:94
const double kBignum = 1.0e30;

thread_local std::string g_err;

struct Oracle {
  // parameters (f90:135-152)
  int64_t npart = 0;
  int nvoisins = 32, nhop = 16, nlevelmax = 30, nmembthresh = 20, nbPes = 1;
  double rho_threshold = 80, fudge = 4, alphap = 1, epsilon = 0;
  double xlong = 1, ylong = 1, zlong = 1, xlongs2 = 0.5, ylongs2 = 0.5, zlongs2 = 0.5, xyzlong = 1;

  // particle data, 1-based
  std::vector<double> pos;   // pos[3*i + k], k = 0..2
  std::vector<double> mass;
  std::vector<double> density;
  std::vector<int32_t> liste_parts;

  // octree (f90:102-109), 1-based cells
  std::vector<int32_t> mass_cell, sister, firstchild, idpart, idpart_tmp, icidpart_tmp;
  std::vector<double> size_cell, pos_cell;  // pos_cell[3*c + k]
  int32_t ncell = 0;

  // hop / groups
  std::vector<int32_t> idpart_adapt, firstpart;
  std::vector<double> densityg;
  int32_t ngroups = 0;

  // saddle CSR (f90:155-158), 1-based
  std::vector<int32_t> grp_nhnei, grp_offset, isad_all;
  std::vector<double> rho_saddle_all;
  bool keep_saddles = false;
  std::vector<int32_t> snap_offset, snap_isad;   // CSR copy before colorize truncation
  std::vector<double> snap_rho;

  // node tree
  struct Node {
    int32_t mass = 0, level = 0, mother = 0, firstchild = 0, nsisters = 0, sister = 0;
    double rho_saddle = 0, density = 0, densmax = 0, radius = 0, truemass = 0;
    double position[3] = {0, 0, 0};
  };
  std::vector<Node> node;
  int32_t nnodes = 0, nnodesmax = 0;
  std::vector<int32_t> idgroup, idgroup_tmp, igroupid, color;

  // optional stage captures for tests
  int32_t* cap_nei = nullptr; int cap_nei_k = 0;   // 0-based particle ids, [N][k]
  int32_t* cap_hop = nullptr;                       // hop target (0-based) or -1 inactive
  int32_t* cap_group = nullptr;                     // group id per particle after maxima

  // -------------------------------------------------------------------
  // f90:3033-3221 create_KDtree (recursive octree, leaf <= npartpercell)
  void create_KDtree(int nlevel, const double pos_this_node[3], int32_t npart_this_node,
                     int32_t npart_pos_this_node, int32_t idmother, double size_my) {
    if (npart_this_node <= 0) return;
    ncell += 1;
    const int32_t inccell = ncell;
    if ((size_t)inccell >= mass_cell.size()) {
      size_t nsz = mass_cell.size() * 2 + 16;
      mass_cell.resize(nsz); sister.resize(nsz); firstchild.resize(nsz);
      size_cell.resize(nsz); pos_cell.resize(3 * nsz);
    }
    for (int k = 0; k < 3; ++k) pos_cell[3 * inccell + k] = pos_this_node[k];
    mass_cell[inccell] = npart_this_node;
    size_cell[inccell] = size_my;
    sister[inccell] = 0;
    firstchild[inccell] = 0;
    if (idmother > 0) {            // f90:3154-3157  prepend to the mother's child list
      sister[inccell] = firstchild[idmother];
      firstchild[idmother] = inccell;
    }
    if (npart_this_node <= kNpartpercell || nlevel == nlevelmax) {
      firstchild[inccell] = -(npart_pos_this_node + 1);
      return;
    }
    int32_t incsubcell[8] = {0}, nsubcell[8] = {0};
    for (int32_t ipar = npart_pos_this_node + 1; ipar <= npart_pos_this_node + npart_this_node; ++ipar) {
      int32_t ipid = idpart[ipar];
      int icid = 0;
      if (pos[3 * ipid + 0] >= pos_this_node[0]) icid += 1;
      if (pos[3 * ipid + 1] >= pos_this_node[1]) icid += 2;
      if (pos[3 * ipid + 2] >= pos_this_node[2]) icid += 4;
      icidpart_tmp[ipar] = icid;
      incsubcell[icid] += 1;
    }
    nsubcell[0] = 0;
    for (int j = 1; j < 8; ++j) nsubcell[j] = nsubcell[j - 1] + incsubcell[j - 1];
    for (int j = 0; j < 8; ++j) incsubcell[j] = 0;
    for (int32_t ipar = npart_pos_this_node + 1; ipar <= npart_pos_this_node + npart_this_node; ++ipar) {
      int icid = icidpart_tmp[ipar];
      incsubcell[icid] += 1;
      idpart_tmp[incsubcell[icid] + nsubcell[icid] + npart_pos_this_node] = idpart[ipar];
    }
    for (int32_t ipar = npart_pos_this_node + 1; ipar <= npart_pos_this_node + npart_this_node; ++ipar)
      idpart[ipar] = idpart_tmp[ipar];
    const double size_child = size_my * 0.5;
    static const double ref[8][3] = {{-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
                                     {-1, -1, 1},  {1, -1, 1},  {-1, 1, 1},  {1, 1, 1}};
    for (int j = 0; j < 8; ++j) {
      if (incsubcell[j] <= 0) continue;
      double pout[3];
      for (int k = 0; k < 3; ++k) pout[k] = pos_this_node[k] + size_child * ref[j][k];
      create_KDtree(nlevel + 1, pout, incsubcell[j], npart_pos_this_node + nsubcell[j], inccell, size_child);
    }
  }

  // f90:2967-3029
  void create_tree_structure() {
    const int32_t n = (int32_t)npart;
    idpart.assign(n + 1, 0);
    idpart_tmp.assign(n + 1, 0);
    icidpart_tmp.assign(n + 1, 0);
    size_t cap = (size_t)std::max<int64_t>(16, npart / 20);
    mass_cell.assign(cap, 0); sister.assign(cap, 0); firstchild.assign(cap, 0);
    size_cell.assign(cap, 0); pos_cell.assign(3 * cap, 0);
    for (int32_t i = 1; i <= n; ++i) idpart[i] = i;
    ncell = 0;
    double p0[3] = {0, 0, 0};
    double sizeroot = std::max(xlong, std::max(ylong, zlong));
    create_KDtree(0, p0, n, 0, 0, sizeroot * 0.5);
    std::vector<int32_t>().swap(idpart_tmp);
    std::vector<int32_t>().swap(icidpart_tmp);
  }

  // f90:2924-2956 (leaf part of walk_tree2): insertion into the sorted list
  void scan_leaf(int32_t icellid_out, const double poshere[3], double* dist2, int32_t iparid,
                 int32_t* iparnei) const {
    double r2max = dist2[nvoisins];
    int32_t base = -firstchild[icellid_out] - 1;
    for (int32_t i = base + 1; i <= base + mass_cell[icellid_out]; ++i) {
      int32_t iparcell = idpart[i];
      if (iparcell == iparid) continue;
      double dx = std::fabs(pos[3 * iparcell + 0] - poshere[0]);
      dx = std::max(0.0, std::min(dx, xlong - dx));
      double d2p = dx * dx;
      if (d2p >= r2max) continue;
      double dy = std::fabs(pos[3 * iparcell + 1] - poshere[1]);
      dy = std::max(0.0, std::min(dy, ylong - dy));
      d2p = d2p + dy * dy;
      if (d2p >= r2max) continue;
      double dz = std::fabs(pos[3 * iparcell + 2] - poshere[2]);
      dz = std::max(0.0, std::min(dz, zlong - dz));
      d2p = d2p + dz * dz;
      if (d2p < r2max) {
        int idist = nvoisins - 1;
        while (dist2[idist] > d2p) {
          dist2[idist + 1] = dist2[idist];
          iparnei[idist + 1] = iparnei[idist];
          idist -= 1;
        }
        dist2[idist + 1] = d2p;
        iparnei[idist + 1] = iparcell;
        r2max = dist2[nvoisins];
      }
    }
  }

  // f90:2867-2962 walk_tree2
  void walk_tree2(int32_t icellidin, const double poshere[3], double* dist2, int32_t iparid,
                  int32_t* iparnei) const {
    int32_t icid[9];
    double discell2[9];
    int32_t icell = firstchild[icellidin];
    int inc = 1;
    double r2max = dist2[nvoisins];
    discell2[0] = 0;
    for (int i = 1; i <= 8; ++i) discell2[i] = 1.0e30;
    while (icell != 0) {
      double sizec = size_cell[icell];
      double dx = std::fabs(pos_cell[3 * icell + 0] - poshere[0]);
      double dy = std::fabs(pos_cell[3 * icell + 1] - poshere[1]);
      double dz = std::fabs(pos_cell[3 * icell + 2] - poshere[2]);
      dx = std::max(0.0, std::min(dx, xlong - dx) - sizec);
      dy = std::max(0.0, std::min(dy, ylong - dy) - sizec);
      dz = std::max(0.0, std::min(dz, zlong - dz) - sizec);
      double distance2 = dx * dx + dy * dy + dz * dz;
      if (distance2 < r2max) {
        int idist = inc - 1;
        while (discell2[idist] > distance2) {
          discell2[idist + 1] = discell2[idist];
          icid[idist + 1] = icid[idist];
          idist -= 1;
        }
        discell2[idist + 1] = distance2;
        icid[idist + 1] = icell;
        inc += 1;
      }
      icell = sister[icell];
    }
    for (int ic = 1; ic <= inc - 1; ++ic) {
      int32_t icellid_out = icid[ic];
      if (firstchild[icellid_out] < 0) {
        if (discell2[ic] < r2max) {
          scan_leaf(icellid_out, poshere, dist2, iparid, iparnei);
          r2max = dist2[nvoisins];
        }
      } else if (discell2[ic] < r2max) {
        walk_tree2(icellid_out, poshere, dist2, iparid, iparnei);
        r2max = dist2[nvoisins];
      }
    }
  }

  // f90:2841-2862  dist2[0..nvoisins], iparnei[1..nvoisins]
  void find_nearest_parts(int32_t ipar, double* dist2, int32_t* iparnei) const {
    double poshere[3] = {pos[3 * ipar + 0], pos[3 * ipar + 1], pos[3 * ipar + 2]};
    dist2[0] = 0.0;
    for (int i = 1; i <= nvoisins; ++i) dist2[i] = kBignum;
    for (int i = 1; i <= nvoisins; ++i) iparnei[i] = 0;
    if (firstchild[1] < 0) {
      // Root cell is a leaf (npart <= npartpercell).  The Fortran would index
      // its cell arrays with the negative leaf marker here; the oracle scans
      // the root leaf directly, which is the kNN the walk intends.
      scan_leaf(1, poshere, dist2, ipar, iparnei);
      return;
    }
    walk_tree2(1, poshere, dist2, ipar, iparnei);
  }

  // f90:3270-3287
  static double spline(double x) {
    if (x <= 1.0) {
      double x2 = x * x;
      double x3 = x2 * x;
      return 1.0 - 1.5 * x2 + 0.75 * x3;
    } else if (x <= 2.0) {
      double x2 = (2.0 - x);
      double x3 = x2 * x2 * x2;
      return 0.25 * x3;
    }
    return 0.0;
  }

  // f90:2816-2838
  void compute_density_one(int32_t ipar, const double* dist2, const int32_t* iparnei) {
    double r = std::sqrt(dist2[nvoisins]) * 0.5;
    double r3 = r * r * r;
    double unsr = 1.0 / r;
    double contrib = 0.0;
    for (int idist = 1; idist <= nvoisins - 1; ++idist)
      contrib = contrib + mass[iparnei[idist]] * spline(std::sqrt(dist2[idist]) * unsr);
    density[ipar] = xyzlong * (contrib + mass[ipar]) / (kPi * r3);
  }

  // f90:682-744
  void compute_mean_density_and_np() {
    const int32_t n = (int32_t)npart;
    density.assign(n + 1, 0.0);
#pragma omp parallel num_threads(nbPes)
    {
      std::vector<double> dist2(nvoisins + 1);
      std::vector<int32_t> iparnei(nvoisins + 1);
#pragma omp for schedule(static)
      for (int32_t ipar = 1; ipar <= n; ++ipar) {
        find_nearest_parts(ipar, dist2.data(), iparnei.data());
        compute_density_one(ipar, dist2.data(), iparnei.data());
        if (cap_nei) {
          for (int k = 0; k < cap_nei_k; ++k)
            cap_nei[(int64_t)(ipar - 1) * cap_nei_k + k] = iparnei[k + 1] - 1;
        }
      }
    }
  }

  // f90:748-881
  void find_local_maxima() {
    const int32_t n = (int32_t)npart;
    liste_parts.assign(n + 1, 0);
    idpart_adapt.assign(n + 1, 0);
    ngroups = 0;
#pragma omp parallel num_threads(nbPes)
    {
      std::vector<double> dist2(nvoisins + 1);
      std::vector<int32_t> iparnei(nvoisins + 1);
#pragma omp for schedule(guided, 256)
      for (int32_t ipar = 1; ipar <= n; ++ipar) {
        if (density[ipar] <= rho_threshold) continue;
        find_nearest_parts(ipar, dist2.data(), iparnei.data());
        double densest = density[ipar];
        int32_t iparsel = ipar;
        for (int idist = 1; idist <= nhop; ++idist) {
          int32_t iparid = iparnei[idist];
          if (density[iparid] > densest) {
            iparsel = iparid;
            densest = density[iparid];
          } else if (density[iparid] == densest) {
            iparsel = std::min(iparsel, iparid);
          }
        }
        idpart_adapt[ipar] = iparsel;
      }
    }
    if (cap_hop) {
      for (int32_t i = 1; i <= n; ++i)
        cap_hop[i - 1] = (density[i] <= rho_threshold) ? -1 : idpart_adapt[i] - 1;
    }
    for (int32_t ipar = 1; ipar <= n; ++ipar) {
      if (density[ipar] <= rho_threshold) continue;
      if (idpart_adapt[ipar] == ipar) {
        ngroups += 1;
        idpart_adapt[ipar] = -ngroups;
      }
    }
    densityg.assign(ngroups + 1, 0.0);
    firstpart.assign(ngroups + 1, 0);
    for (int32_t ipar = 1; ipar <= n; ++ipar) {
      if (density[ipar] <= rho_threshold) continue;
      int32_t iparid = idpart_adapt[ipar];
      if (iparid < 0) {
        int32_t groupid = -iparid;
        densityg[groupid] = density[ipar];
        liste_parts[ipar] = groupid;
      } else {
        int32_t groupid = 0;
        while (iparid > 0) {
          if (liste_parts[iparid] > 0) { groupid = liste_parts[iparid]; break; }
          iparid = idpart_adapt[iparid];
        }
        if (iparid < 0) groupid = -iparid;
        liste_parts[ipar] = groupid;
      }
    }
    for (int32_t ipar = 1; ipar <= n; ++ipar) {
      if (density[ipar] <= rho_threshold) continue;
      int32_t igroup = liste_parts[ipar];
      if (igroup > 0) {
        idpart_adapt[ipar] = firstpart[igroup];
        firstpart[igroup] = ipar;
      }
    }
    if (cap_group) for (int32_t i = 1; i <= n; ++i) cap_group[i - 1] = liste_parts[i];
  }

  // f90:220-303  Numerical Recipes indexx (1-based arr/indx)
  static bool indexx(int n, const double* arr, int* indx) {
    const int M = 7, NSTACK = 50;
    int istack[NSTACK + 1];
    for (int j = 1; j <= n; ++j) indx[j] = j;
    int jstack = 0, l = 1, ir = n;
    for (;;) {
      if (ir - l < M) {
        for (int j = l + 1; j <= ir; ++j) {
          int indxt = indx[j];
          double a = arr[indxt];
          int i;
          for (i = j - 1; i >= 1; --i) {
            if (arr[indx[i]] <= a) break;
            indx[i + 1] = indx[i];
          }
          indx[i + 1] = indxt;
        }
        if (jstack == 0) return true;
        ir = istack[jstack];
        l = istack[jstack - 1];
        jstack -= 2;
      } else {
        int k = (l + ir) / 2;
        std::swap(indx[k], indx[l + 1]);
        if (arr[indx[l + 1]] > arr[indx[ir]]) std::swap(indx[l + 1], indx[ir]);
        if (arr[indx[l]] > arr[indx[ir]]) std::swap(indx[l], indx[ir]);
        if (arr[indx[l + 1]] > arr[indx[l]]) std::swap(indx[l + 1], indx[l]);
        int i = l + 1, j = ir;
        int indxt = indx[l];
        double a = arr[indxt];
        for (;;) {
          do { i++; } while (arr[indx[i]] < a);
          do { j--; } while (arr[indx[j]] > a);
          if (j < i) break;
          std::swap(indx[i], indx[j]);
        }
        indx[l] = indx[j];
        indx[j] = indxt;
        jstack += 2;
        if (jstack > NSTACK) return false;
        if (ir - i + 1 >= j - l) {
          istack[jstack] = ir;
          istack[jstack - 1] = i;
          ir = j - 1;
        } else {
          istack[jstack] = j - 1;
          istack[jstack - 1] = l;
          l = i;
        }
      }
    }
  }

  // f90:2433-2813
  bool compute_saddle_list() {
    const int32_t ng = ngroups;
    grp_nhnei.assign(ng + 1, 0);
    grp_offset.assign(ng + 2, 0);
    int max_neig = 0;
    // first pass: count distinct neighbouring groups (f90:2495-2531)
#pragma omp parallel num_threads(nbPes) reduction(max : max_neig)
    {
      std::vector<char> touch(ng + 1, 0);
      std::vector<int32_t> listg(ng + 1, 0);
      std::vector<double> dist2(nvoisins + 1);
      std::vector<int32_t> iparnei(nvoisins + 1);
#pragma omp for schedule(dynamic, 8)
      for (int32_t igroup1 = 1; igroup1 <= ng; ++igroup1) {
        int ineig = 0;
        int32_t ipar1 = firstpart[igroup1];
        while (ipar1 > 0) {
          find_nearest_parts(ipar1, dist2.data(), iparnei.data());
          for (int idist = 1; idist <= nhop; ++idist) {
            int32_t ipar2 = iparnei[idist];
            int32_t igroup2 = liste_parts[ipar2];
            if (igroup2 > 0 && igroup2 != igroup1 && !touch[igroup2]) {
              ineig += 1;
              touch[igroup2] = 1;
              listg[ineig] = igroup2;
            }
          }
          ipar1 = idpart_adapt[ipar1];
        }
        for (int in1 = 1; in1 <= ineig; ++in1) touch[listg[in1]] = 0;
        grp_nhnei[igroup1] = ineig;
        max_neig = std::max(max_neig, ineig);
      }
    }
    grp_offset[1] = 1;
    for (int32_t g = 1; g <= ng; ++g) grp_offset[g + 1] = grp_offset[g] + grp_nhnei[g];
    int32_t total_conn = grp_offset[ng + 1] - 1;
    isad_all.assign(std::max(total_conn, 1) + 1, 0);
    rho_saddle_all.assign(std::max(total_conn, 1) + 1, 0.0);
    bool ok = true;
    // second pass: fill rows in first-encounter order (f90:2573-2632)
#pragma omp parallel num_threads(nbPes)
    {
      std::vector<char> touch(ng + 1, 0);
      std::vector<int32_t> listg(ng + 1, 0);
      std::vector<double> rho_sad_thr(std::max(max_neig, 1) + 1, 0.0);
      std::vector<double> dist2(nvoisins + 1);
      std::vector<int32_t> iparnei(nvoisins + 1);
#pragma omp for schedule(dynamic, 8)
      for (int32_t igroup1 = 1; igroup1 <= ng; ++igroup1) {
        int neig = grp_nhnei[igroup1];
        if (neig <= 0) continue;
        int ineig = 0;
        int32_t ipar1 = firstpart[igroup1];
        int32_t base = grp_offset[igroup1];
        while (ipar1 > 0) {
          find_nearest_parts(ipar1, dist2.data(), iparnei.data());
          double density1 = density[ipar1];
          for (int idist = 1; idist <= nhop; ++idist) {
            int32_t ipar2 = iparnei[idist];
            int32_t igroup2 = liste_parts[ipar2];
            if (igroup2 > 0 && igroup2 != igroup1) {
              double density2 = density[ipar2];
              double rho_sad12 = std::min(density1, density2);
              if (!touch[igroup2]) {
                ineig += 1;
                touch[igroup2] = 1;
                listg[igroup2] = ineig;
                rho_sad_thr[ineig] = rho_sad12;
                isad_all[base + ineig - 1] = igroup2;
              } else {
                int ineig2 = listg[igroup2];
                rho_sad_thr[ineig2] = std::max(rho_sad_thr[ineig2], rho_sad12);
              }
            }
          }
          ipar1 = idpart_adapt[ipar1];
        }
        if (ineig != neig) {
#pragma omp critical
          { ok = false; g_err = "saddle neighbour count mismatch"; }
        }
        for (int k = 1; k <= ineig; ++k) rho_saddle_all[base + k - 1] = rho_sad_thr[k];
        for (int in1 = 1; in1 <= ineig; ++in1) touch[isad_all[base + in1 - 1]] = 0;
      }
    }
    if (!ok) return false;
    // symmetry (f90:2647-2688)
    for (int32_t g1 = 1; g1 <= ng; ++g1) {
      int neig = grp_nhnei[g1];
      if (neig <= 0) continue;
      int32_t base = grp_offset[g1];
      for (int in1 = 1; in1 <= neig; ++in1) {
        int32_t idx1 = base + in1 - 1;
        bool exist = false;
        int32_t g2 = isad_all[idx1];
        if (g2 > 0) {
          int32_t base2 = grp_offset[g2];
          for (int in2 = 1; in2 <= grp_nhnei[g2]; ++in2) {
            int32_t idx2 = base2 + in2 - 1;
            if (isad_all[idx2] == g1) {
              exist = true;
              double r12 = std::min(rho_saddle_all[idx2], rho_saddle_all[idx1]);
              rho_saddle_all[idx2] = r12;
              rho_saddle_all[idx1] = r12;
              break;
            }
          }
        }
        if (!exist) isad_all[idx1] = 0;
      }
    }
    // compact + sort rows by decreasing saddle (f90:2702-2776)
    std::vector<int32_t> new_nhnei(ng + 1, 0), new_offset(ng + 2, 0);
    for (int32_t g1 = 1; g1 <= ng; ++g1) {
      int32_t base = grp_offset[g1];
      for (int in1 = 1; in1 <= grp_nhnei[g1]; ++in1)
        if (isad_all[base + in1 - 1] > 0) new_nhnei[g1] += 1;
    }
    new_offset[1] = 1;
    for (int32_t g1 = 1; g1 <= ng; ++g1) new_offset[g1 + 1] = new_offset[g1] + new_nhnei[g1];
    int32_t new_total = new_offset[ng + 1] - 1;
    std::vector<int32_t> new_isad(std::max(new_total, 1) + 1, 0);
    std::vector<double> new_rho(std::max(new_total, 1) + 1, 0.0);
    std::vector<double> rho_sad(std::max(max_neig, 1) + 1);
    std::vector<int32_t> isad(std::max(max_neig, 1) + 1), indx(std::max(max_neig, 1) + 1);
    for (int32_t g1 = 1; g1 <= ng; ++g1) {
      int neig = grp_nhnei[g1];
      if (neig <= 0) continue;
      int32_t base = grp_offset[g1];
      int ineig = 0;
      for (int in1 = 1; in1 <= neig; ++in1) {
        int32_t idx1 = base + in1 - 1;
        int32_t g2 = isad_all[idx1];
        if (g2 > 0) {
          ineig += 1;
          rho_sad[ineig] = rho_saddle_all[idx1];
          isad[ineig] = g2;
        }
      }
      if (ineig > 0) {
        if (!indexx(ineig, rho_sad.data(), indx.data())) { g_err = "nstack too small in indexx"; return false; }
        int32_t outbase = new_offset[g1];
        for (int i = 1; i <= ineig; ++i) {
          int i2 = indx[i];
          new_isad[outbase + ineig - i] = isad[i2];
          new_rho[outbase + ineig - i] = rho_sad[i2];
        }
      }
    }
    grp_nhnei.swap(new_nhnei);
    grp_offset.swap(new_offset);
    isad_all.swap(new_isad);
    rho_saddle_all.swap(new_rho);
    if (keep_saddles) { snap_offset = grp_offset; snap_isad = isad_all; snap_rho = rho_saddle_all; }
    // the octree is no longer needed (f90:2799-2810)
    std::vector<int32_t>().swap(mass_cell); std::vector<int32_t>().swap(sister);
    std::vector<int32_t>().swap(firstchild); std::vector<int32_t>().swap(idpart);
    std::vector<double>().swap(size_cell); std::vector<double>().swap(pos_cell);
    return true;
  }

  // f90:2404-2429
  void treat_particles_linkonly(int32_t igroup, double rhot) {
    int32_t ipar = firstpart[igroup], iparold = 0;
    bool first_good = false;
    while (ipar > 0) {
      if (density[ipar] > rhot) {
        if (!first_good) { first_good = true; firstpart[igroup] = ipar; }
        else idpart_adapt[iparold] = ipar;
        iparold = ipar;
      }
      ipar = idpart_adapt[ipar];
    }
    if (!first_good) firstpart[igroup] = 0;
  }

  // f90:2317-2401
  bool treat_particles(int32_t igroup, double rhot, double posg[3], int32_t& imass, int32_t& igroupref,
                       double posref[3], double& rsquare, double& densmoy, double& truemass) {
    imass = 0; truemass = 0.0; rsquare = 0.0; densmoy = 0.0;
    posg[0] = posg[1] = posg[2] = 0.0;
    int32_t ipar = firstpart[igroup], iparold = 0;
    bool first_good = false;
    double densmax = 0, densmin = 0;
    while (ipar > 0) {
      double density_ipar = density[ipar];
      if (density_ipar > rhot) {
        if (!first_good) {
          if (igroupref == 0) {
            posref[0] = pos[3 * ipar + 0]; posref[1] = pos[3 * ipar + 1]; posref[2] = pos[3 * ipar + 2];
            igroupref = igroup;
          }
          first_good = true;
          firstpart[igroup] = ipar;
          densmin = density_ipar;
          densmax = densmin;
        } else {
          idpart_adapt[iparold] = ipar;
        }
        iparold = ipar;
        imass += 1;
        double xm = mass[ipar];
        truemass = truemass + xm;
        double px = pos[3 * ipar + 0] - posref[0];
        double py = pos[3 * ipar + 1] - posref[1];
        double pz = pos[3 * ipar + 2] - posref[2];
        if (px >= xlongs2) px = px - xlong; else if (px < -xlongs2) px = px + xlong;
        if (py >= ylongs2) py = py - ylong; else if (py < -ylongs2) py = py + ylong;
        if (pz >= zlongs2) pz = pz - zlong; else if (pz < -zlongs2) pz = pz + zlong;
        px = px + posref[0];
        py = py + posref[1];
        pz = pz + posref[2];
        posg[0] = posg[0] + px * xm;
        posg[1] = posg[1] + py * xm;
        posg[2] = posg[2] + pz * xm;
        rsquare = rsquare + xm * (px * px + py * py + pz * pz);
        densmoy = densmoy + density_ipar;
        densmax = std::max(densmax, density_ipar);
        densmin = std::min(densmin, density_ipar);
      }
      ipar = idpart_adapt[ipar];
    }
    if (first_good) idpart_adapt[iparold] = 0;
    else firstpart[igroup] = 0;
    if (densmin <= rhot || densmax != densityg[igroup]) {
      char buf[256];
      snprintf(buf, sizeof buf, "treat_particles invariant failed: igroup=%d densmax=%.17g rhot=%.17g", igroup,
               densityg[igroup], rhot);
      g_err = buf;
      return false;
    }
    return true;
  }

  // f90:1188-1242
  bool do_colorize_local(int32_t igroup, int32_t igr, double rhot, std::vector<int32_t>& queue, int32_t color_id) {
    queue[1] = igroup;
    int32_t front = 1, back = 2;
    color[igr] = color_id;
    while (front < back) {
      int32_t g = queue[front];
      front += 1;
      int neig = grp_nhnei[g];
      int32_t base = grp_offset[g];
      for (int ineig = 1; ineig <= neig; ++ineig) {
        int32_t idx = base + ineig - 1;
        if (rho_saddle_all[idx] > rhot) {
          int32_t g2 = isad_all[idx];
          int32_t igr2 = igroupid[g2];
          if (color[igr2] == 0) {
            color[igr2] = color_id;
            if (back > (int32_t)queue.size() - 1) { g_err = "colorize queue overflow"; return false; }
            queue[back] = g2;
            back += 1;
          } else if (color[igr2] != color_id) {
            g_err = "colorize: connections are not symmetric";
            return false;
          }
        } else {
          grp_nhnei[g] = ineig - 1;
          break;
        }
      }
    }
    return true;
  }

  // f90:1169-1185
  bool reserve_nodes_block(int32_t nnew, int32_t& inode_first) {
    inode_first = nnodes + 1;
    nnodes += nnew;
    if (nnodes > nnodesmax) { g_err = "nnodes > nnodesmax"; return false; }
    return true;
  }

  // f90:1245-1628 (OpenMP tasks replaced by serial depth-first recursion; node
  // ids are canonicalised afterwards by reorder_nodes_deterministic)
  bool create_nodes_task(double rhot0, int32_t inode0, int32_t igr1_0, int32_t igr2_0, bool do_paint) {
    double rhot = rhot0;
    const int32_t inode = inode0;
    int32_t igr1 = igr1_0, igr2 = igr2_0;
    if (do_paint) {
      for (int32_t igr = igr1; igr <= igr2; ++igr) {
        int32_t igroup = idgroup[igr];
        int32_t ipar = firstpart[igroup];
        while (ipar > 0) { liste_parts[ipar] = inode; ipar = idpart_adapt[ipar]; }
      }
    }
    for (;;) {
      std::vector<int32_t> queue_local(std::max(igr2 - igr1 + 1, 1) + 1);
      for (int32_t igr = igr1; igr <= igr2; ++igr) color[igr] = 0;
      int32_t ncolors = 0;
      for (int32_t igr = igr1; igr <= igr2; ++igr) {
        int32_t igroup = idgroup[igr];
        if (color[igr] == 0) {
          ncolors += 1;
          if (!do_colorize_local(igroup, igr, rhot, queue_local, ncolors)) return false;
        }
      }
      std::vector<int32_t> igrpos(ncolors + 1, 0), igrinc(ncolors + 1, 0);
      igrpos[0] = igr1 - 1;
      for (int32_t igr = igr1; igr <= igr2; ++igr) {
        int32_t ic = color[igr];
        if (densityg[idgroup[igr]] > rhot) igrpos[ic] += 1;
      }
      for (int32_t ic = 1; ic <= ncolors; ++ic) igrpos[ic] = igrpos[ic - 1] + igrpos[ic];
      for (int32_t igr = igr1; igr <= igr2; ++igr) {
        int32_t ic = color[igr];
        int32_t igroup = idgroup[igr];
        if (densityg[igroup] > rhot) {
          igrinc[ic] += 1;
          int32_t igr_eff = igrinc[ic] + igrpos[ic - 1];
          idgroup_tmp[igr_eff] = igroup;
          igroupid[igroup] = igr_eff;
        }
      }
      igr2 = igrpos[ncolors];
      for (int32_t igr = igr1; igr <= igr2; ++igr) idgroup[igr] = idgroup_tmp[igr];
      int32_t inc_color_tot = 0;
      for (int32_t ic = 1; ic <= ncolors; ++ic) if (igrinc[ic] > 0) inc_color_tot += 1;
      std::vector<int32_t> igrposnew(inc_color_tot + 1);
      igrposnew[0] = igrpos[0];
      inc_color_tot = 0;
      for (int32_t ic = 1; ic <= ncolors; ++ic)
        if (igrinc[ic] > 0) { inc_color_tot += 1; igrposnew[inc_color_tot] = igrpos[ic]; }

      const int32_t nc = inc_color_tot;
      std::vector<double> posgg(3 * (nc + 1)), truemassg(nc + 1), densmaxg(nc + 1), rsq(nc + 1), densmoy(nc + 1);
      std::vector<int32_t> massg(nc + 1), mass_compg(nc + 1), ok_color(nc + 1);
      std::vector<char> ifok(nc + 1, 0);
      for (int32_t ic = 1; ic <= nc; ++ic) {
        double posg[3] = {0, 0, 0}, posref[3] = {0, 0, 0};
        int32_t mass_loc = 0, mass_comp = 0, igroupref = 0;
        double truemass = 0, rsquareg = 0, densmoyg = 0, densmaxgroup = -1.0, densmoy_comp_max = -1.0;
        int32_t a = igrposnew[ic - 1] + 1, b = igrposnew[ic];
        for (int32_t igr = a; igr <= b; ++igr) {
          int32_t igroup = idgroup[igr];
          densmaxgroup = std::max(densmaxgroup, densityg[igroup]);
          double posgtmp[3], rsqtmp, dmtmp, tmtmp;
          int32_t masstmp;
          if (!treat_particles(igroup, rhot, posgtmp, masstmp, igroupref, posref, rsqtmp, dmtmp, tmtmp)) return false;
          posg[0] = posg[0] + posgtmp[0];
          posg[1] = posg[1] + posgtmp[1];
          posg[2] = posg[2] + posgtmp[2];
          rsquareg = rsquareg + rsqtmp;
          mass_loc = mass_loc + masstmp;
          truemass = truemass + tmtmp;
          densmoyg = densmoyg + dmtmp;
          mass_comp = std::max(mass_comp, masstmp);
          if (masstmp > 0) {
            dmtmp = dmtmp / (double)masstmp;
            densmoy_comp_max = std::max(densmoy_comp_max, dmtmp / (1.0 + fudge / std::sqrt((double)masstmp)));
          }
        }
        massg[ic] = mass_loc;
        truemassg[ic] = truemass;
        posgg[3 * ic + 0] = posg[0]; posgg[3 * ic + 1] = posg[1]; posgg[3 * ic + 2] = posg[2];
        densmaxg[ic] = densmaxgroup;
        mass_compg[ic] = mass_comp;
        double p2 = posg[0] * posg[0] + posg[1] * posg[1] + posg[2] * posg[2];
        rsq[ic] = std::sqrt(std::fabs((truemass * rsquareg - p2) / (truemass * truemass)));
        densmoy[ic] = densmoyg / (double)mass_loc;
        ifok[ic] = mass_loc >= nmembthresh &&
                   (densmoy[ic] > rhot * (1.0 + fudge / std::sqrt((double)mass_loc)) || densmoy_comp_max > rhot) &&
                   densmaxg[ic] >= alphap * densmoy[ic] && rsq[ic] >= epsilon;
      }
      int32_t nsisters = 0, icolor_ref = 0;
      for (int32_t ic = 1; ic <= nc; ++ic)
        if (ifok[ic]) { nsisters += 1; ok_color[nsisters] = ic; icolor_ref = ic; }

      if (nsisters > 1) {
        int32_t inode1;
        if (!reserve_nodes_block(nsisters, inode1)) return false;
        for (int32_t is = 1; is <= nsisters; ++is) {
          int32_t ic = ok_color[is];
          int32_t io = inode1 + is - 1;
          Node& nd = node[io];
          nd.mother = inode;
          nd.densmax = densmaxg[ic];
          nd.sister = (is > 1) ? io - 1 : 0;
          nd.nsisters = nsisters;
          nd.mass = massg[ic];
          nd.truemass = truemassg[ic];
          if (massg[ic] == 0) { g_err = "NULL mass node"; return false; }
          double pf[3] = {posgg[3 * ic + 0] / truemassg[ic], posgg[3 * ic + 1] / truemassg[ic],
                          posgg[3 * ic + 2] / truemassg[ic]};
          nd.radius = rsq[ic];
          nd.density = densmoy[ic];
          if (pf[0] >= xlongs2) pf[0] = pf[0] - xlong; else if (pf[0] < -xlongs2) pf[0] = pf[0] + xlong;
          if (pf[1] >= ylongs2) pf[1] = pf[1] - ylong; else if (pf[1] < -ylongs2) pf[1] = pf[1] + ylong;
          if (pf[2] >= zlongs2) pf[2] = pf[2] - zlong; else if (pf[2] < -zlongs2) pf[2] = pf[2] + zlong;
          nd.position[0] = pf[0]; nd.position[1] = pf[1]; nd.position[2] = pf[2];
          nd.rho_saddle = rhot;
          nd.level = node[inode].level + 1;
        }
        node[inode].firstchild = inode1 + nsisters - 1;
        for (int32_t is = 1; is <= nsisters; ++is) {
          int32_t ic = ok_color[is];
          double rc = rhot * (1.0 + fudge / std::sqrt((double)mass_compg[ic]));
          if (!create_nodes_task(rc, inode1 + is - 1, igrposnew[ic - 1] + 1, igrposnew[ic], true)) return false;
        }
        return true;
      } else if (nsisters == 1) {
        int32_t ic = icolor_ref;
        double rhotout = rhot * (1.0 + fudge / std::sqrt((double)mass_compg[ic]));
        int32_t a = igrposnew[0] + 1, b = igrposnew[nc];
        if (b != a) { rhot = rhotout; igr1 = a; igr2 = b; continue; }
        node[inode].firstchild = 0;
        return true;
      } else {
        node[inode].firstchild = 0;
        return true;
      }
    }
  }

  // f90:1083-1131
  bool node_precedes(int32_t ia, int32_t ib) const {
    const Node &a = node[ia], &b = node[ib];
    if (a.level != b.level) return a.level < b.level;
    if (a.truemass != b.truemass) return a.truemass > b.truemass;
    if (a.mass != b.mass) return a.mass > b.mass;
    if (a.densmax != b.densmax) return a.densmax > b.densmax;
    if (a.density != b.density) return a.density > b.density;
    if (a.rho_saddle != b.rho_saddle) return a.rho_saddle > b.rho_saddle;
    for (int k = 0; k < 3; ++k)
      if (a.position[k] != b.position[k]) return a.position[k] < b.position[k];
    return ia < ib;
  }

  // f90:987-1041 (the comparator is a strict total order, so any correct sort
  // yields the permutation of sort_node_ids f90:1044-1080)
  void reorder_nodes_deterministic() {
    if (nnodes <= 1) return;
    std::vector<int32_t> new_to_old(nnodes);
    for (int32_t i = 0; i < nnodes; ++i) new_to_old[i] = i + 1;
    std::sort(new_to_old.begin(), new_to_old.end(), [this](int32_t a, int32_t b) { return node_precedes(a, b); });
    std::vector<int32_t> old_to_new(nnodes + 1, 0);
    for (int32_t k = 0; k < nnodes; ++k) old_to_new[new_to_old[k]] = k + 1;
    std::vector<Node> sorted(nnodes + 1);
    sorted[0] = node[0];
    for (int32_t k = 1; k <= nnodes; ++k) {
      sorted[k] = node[new_to_old[k - 1]];
      if (sorted[k].mother > 0) sorted[k].mother = old_to_new[sorted[k].mother];
      if (sorted[k].firstchild > 0) sorted[k].firstchild = old_to_new[sorted[k].firstchild];
      if (sorted[k].sister > 0) sorted[k].sister = old_to_new[sorted[k].sister];
    }
    for (int64_t i = 1; i <= npart; ++i) {
      int32_t o = liste_parts[i];
      if (o > 0) liste_parts[i] = old_to_new[o];
    }
    for (int32_t k = 0; k <= nnodes; ++k) node[k] = sorted[k];
  }

  // f90:885-983
  bool create_group_tree() {
    if (!compute_saddle_list()) return false;
    nnodesmax = 2 * ngroups;
    node.assign(nnodesmax + 1, Node());
    idgroup.assign(ngroups + 1, 0);
    color.assign(ngroups + 1, 0);
    igroupid.assign(ngroups + 1, 0);
    idgroup_tmp.assign(ngroups + 1, 0);
    std::fill(liste_parts.begin(), liste_parts.end(), 0);
    nnodes = 0;
    double rhot = rho_threshold;
    for (int32_t g = 1; g <= ngroups; ++g) treat_particles_linkonly(g, rhot);
    node[0].mother = 0;
    node[0].mass = 0;
    node[0].truemass = 0.0;
    double dmax = -HUGE_VAL;
    for (int32_t g = 1; g <= ngroups; ++g) dmax = std::max(dmax, densityg[g]);
    node[0].densmax = dmax;
    node[0].level = 0;
    for (int32_t g = 1; g <= ngroups; ++g) { idgroup[g] = g; igroupid[g] = g; }
    if (ngroups > 0 && !create_nodes_task(rhot, 0, 1, ngroups, false)) return false;
    reorder_nodes_deterministic();
    return true;
  }
};

Oracle* g_last = nullptr;

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_adaptahop(const OracleParams* p, const double* pos3n, const double* mass_in, OracleResult* out,
                     const OracleCapture* cap) {
  g_err.clear();
  if (!p || !pos3n || !mass_in || !out) { g_err = "null argument"; return 1; }
  if (p->npart <= p->nvoisins) { g_err = "npart must exceed nvoisins"; return 2; }
  if (p->nhop > p->nvoisins || p->nhop < 1) { g_err = "need 1 <= nhop <= nvoisins"; return 2; }
  if (p->npart > 2000000000LL) { g_err = "npart too large for int32 particle ids"; return 2; }
  delete g_last;
  g_last = new Oracle();
  Oracle& o = *g_last;
  o.npart = p->npart;
  o.nvoisins = p->nvoisins; o.nhop = p->nhop; o.nlevelmax = p->nlevelmax; o.nmembthresh = p->nmembthresh;
  o.nbPes = p->nthreads > 0 ? p->nthreads : 1;
  o.rho_threshold = p->rho_threshold; o.fudge = p->fudge; o.alphap = p->alphap; o.epsilon = p->epsilon;
  o.xlong = p->xlong; o.ylong = p->ylong; o.zlong = p->zlong;
  o.xlongs2 = p->xlongs2; o.ylongs2 = p->ylongs2; o.zlongs2 = p->zlongs2;
  o.xyzlong = o.xlong * o.ylong * o.zlong;  // f90:632
  const int64_t n = p->npart;
  o.pos.assign(3 * (n + 1), 0.0);
  std::memcpy(o.pos.data() + 3, pos3n, sizeof(double) * 3 * n);
  o.mass.assign(n + 1, 0.0);
  std::memcpy(o.mass.data() + 1, mass_in, sizeof(double) * n);
  if (cap) {
    o.cap_nei = cap->neighbours; o.cap_nei_k = cap->neighbours_k;
    o.cap_hop = cap->hop_target; o.cap_group = cap->group_id;
    o.keep_saddles = cap->keep_saddles != 0;
  }
  double t0 = omp_get_wtime();
  o.create_tree_structure();
  double t1 = omp_get_wtime();
  o.compute_mean_density_and_np();
  double t2 = omp_get_wtime();
  o.find_local_maxima();
  double t3 = omp_get_wtime();
  if (!o.create_group_tree()) return 3;
  double t4 = omp_get_wtime();
  out->stage_seconds[0] = t1 - t0;
  out->stage_seconds[1] = t2 - t1;
  out->stage_seconds[2] = t3 - t2;
  out->stage_seconds[3] = t4 - t3;
  out->ngroups = o.ngroups;
  out->nnodes = o.nnodes;
  out->ncells = o.ncell;
  return 0;
}

int oracle_copy_outputs(double* density, int32_t* liste_parts, double* real_table, int32_t* integer_table) {
  if (!g_last) { g_err = "no result"; return 1; }
  Oracle& o = *g_last;
  const int64_t n = o.npart;
  if (density) std::memcpy(density, o.density.data() + 1, sizeof(double) * n);
  if (liste_parts) std::memcpy(liste_parts, o.liste_parts.data() + 1, sizeof(int32_t) * n);
  for (int32_t k = 1; k <= o.nnodes; ++k) {
    const auto& nd = o.node[k];
    if (real_table) {
      double* r = real_table + 8 * (int64_t)(k - 1);
      r[0] = nd.rho_saddle; r[1] = nd.density; r[2] = nd.densmax; r[3] = nd.radius; r[4] = nd.truemass;
      r[5] = nd.position[0]; r[6] = nd.position[1]; r[7] = nd.position[2];
    }
    if (integer_table) {
      int32_t* t = integer_table + 6 * (int64_t)(k - 1);
      t[0] = nd.mass; t[1] = nd.level; t[2] = nd.mother; t[3] = nd.firstchild; t[4] = nd.nsisters; t[5] = nd.sister;
    }
  }
  return 0;
}

// Saddle CSR of the last run (captured before the tree build truncates rows):
// row g (1-based group id) spans [offsets[g-1], offsets[g]) with 0-based
// offsets; neighbour ids are 1-based group ids; rows sorted by decreasing
// saddle density exactly as f90:2762-2773 leaves them.
int oracle_saddles(int32_t* nconn_out, int32_t* offsets, int32_t* isad, double* rho) {
  if (!g_last || g_last->snap_offset.empty()) { g_err = "no saddle snapshot (set keep_saddles)"; return 1; }
  Oracle& o = *g_last;
  int32_t ng = o.ngroups;
  int32_t tot = o.snap_offset[ng + 1] - 1;
  if (nconn_out) *nconn_out = tot;
  if (offsets) for (int32_t g = 1; g <= ng + 1; ++g) offsets[g - 1] = o.snap_offset[g] - 1;
  if (isad) for (int32_t i = 1; i <= tot; ++i) isad[i - 1] = o.snap_isad[i];
  if (rho) for (int32_t i = 1; i <= tot; ++i) rho[i - 1] = o.snap_rho[i];
  return 0;
}

void oracle_release(void) { delete g_last; g_last = nullptr; }

}  // extern "C"
