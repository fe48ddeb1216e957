/* AdaptaHOP CPU oracle — TEST INFRASTRUCTURE ONLY (checker and CPU baseline).
 * Restates fortran/compute_adaptahop.f90 of the reference; never part of the
 * product library. */
#ifndef AHOP_ORACLE_H
#define AHOP_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t npart;
  int32_t nvoisins, nhop, nlevelmax, nmembthresh, nthreads;
  double rho_threshold, fudge, alphap, epsilon;
  double xlong, ylong, zlong, xlongs2, ylongs2, zlongs2;
} OracleParams;

typedef struct {
  int32_t ngroups, nnodes, ncells, pad;
  double stage_seconds[4]; /* tree, kNN+density, local maxima, group tree */
} OracleResult;

typedef struct {
  int32_t* neighbours;  /* [npart][neighbours_k] 0-based ids, sorted by distance */
  int32_t neighbours_k;
  int32_t* hop_target;  /* [npart] 0-based densest-of-nhop target, -1 if inactive */
  int32_t* group_id;    /* [npart] peak group id after find_local_maxima, 0 if none */
  int32_t keep_saddles; /* nonzero: keep a copy of the saddle CSR for oracle_saddles */
} OracleCapture;

const char* oracle_last_error(void);
int oracle_adaptahop(const OracleParams* p, const double* pos3n, const double* mass, OracleResult* out,
                     const OracleCapture* cap);
int oracle_copy_outputs(double* density, int32_t* liste_parts, double* real_table, int32_t* integer_table);
int oracle_saddles(int32_t* nconn, int32_t* offsets, int32_t* isad, double* rho);
void oracle_release(void);

#ifdef __cplusplus
}
#endif
#endif
