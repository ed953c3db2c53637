/*
 * cgx_ops.h -- the reference solver's discrete operators built on the GPU
 * from a compact mesh (C ABI, exported by libcgx.so).
 *
 * Input: what a mesher hands over for a triply periodic box -- owned cells
 * (volume, centroid), compact faces (cells, area vector, centroid) and the
 * level-1 periodic ghosts those faces reach.  Output: the same
 * cgx_meshgen_out (include/cgx_meshgen.h) that the host generator fills,
 * array for array and in the same order, ready for cgx_mesh_create():
 *
 *   cvocv_i / cvocv_v      buildCvocv, src/core/common/StaticSolver.cpp:6659-6726
 *   cvocv_grad_coeff       calcCvGradCoeff, StaticSolver.cpp:5598-5765
 *   cvoef / n_ef / c_ef    StripedMesh::buildExtendedFaces with EF_OPS DEFAULT,
 *                          src/core/common/StripedMesh.hpp:5269-6960 (operator
 *                          rows :6014-6130, transpose and face assembly
 *                          :6589-6866), level-2 ghosts appended in order of
 *                          first use
 *   area_over_delta_fa     StaticSolver.cpp:4447-4459
 *   cmag_cv, dcmag_hat_cv  src/charles/FlowSolver.hpp:702-760
 *   sa_to_vol_ratio        src/charles/FlowSolver.hpp:859-878
 *
 * The device evaluates every floating-point expression in the host
 * generator's order without multiply-add contraction, so the two builds agree
 * bit for bit.  This replaces the host preprocessing between mesher and solver
 * for a served mesh.
 */
#ifndef CGX_OPS_H
#define CGX_OPS_H

#include "cgx_meshgen.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cgx_compact_desc {
  int ncv;                  /* owned cells */
  int ncv_g;                /* owned cells + level-1 ghosts */
  int nfa, nfa_i;           /* compact faces; [0, nfa_i) internal */
  double L[3];              /* periodic box lengths */
  double h;                 /* lattice spacing, passed through */
  const int*    cvofa;      /* [nfa][2]: internal c0 < c1 < ncv, faces ordered by c0;
                               periodic c0 owned, c1 a ghost in [ncv, ncv_g) */
  const double* n_fa;       /* [nfa][3] area vector c0 -> c1 */
  const double* x_fa;       /* [nfa][3] face centroid, frame of c0 */
  const double* vol_cv;     /* [ncv] */
  const double* x_cv;       /* [ncv][3] owned-cell centroids */
  const double* x_vv;       /* [ncv][3] Voronoi seeds, passed through, or NULL */
  const int*    icv_owner_g;/* [ncv_g-ncv] owner of each level-1 ghost */
  const int*    shift_g;    /* [ncv_g-ncv][3] its periodic shift, in box lengths, |s| <= 1 */
  /* boundary faces (0 for a triply periodic box).  Gij_bf enters the
   * gradient coefficients (calcCvGradCoeff's boundary term,
   * StaticSolver.cpp:5642-5650), each cell's faces in increasing index; the
   * rest is passed through to the output. */
  int nbf, nbf_zones;
  const int*    cvobf;              /* [nbf] */
  const int*    zone_bf;            /* [nbf] or NULL */
  const double* n_bf;               /* [nbf][3] or NULL */
  const double* x_bf;               /* [nbf][3] or NULL */
  const double* area_bf;            /* [nbf] or NULL */
  const double* area_over_delta_bf; /* [nbf] or NULL */
  const double* Gij_bf;             /* [nbf][3][3] */
} cgx_compact_desc;

/*
 * Build the operators on device `device`.  *out is allocated here and
 * released with cgx_operators_free().  device_ms (may be NULL) receives the
 * device time from the end of the upload to the start of the download.
 * Returns 0, CGX_E_ARG for an inconsistent mesh, a box too thin for the
 * extended stencil (a cell reaching its own image) or an operator row longer
 * than 384 entries (the host generator's limit), CGX_E_OOM or CGX_E_CUDA;
 * cgx_last_error() says which.
 */
int cgx_operators_build(const cgx_compact_desc* in, double interp_factor, double sigma_thresh,
                        int device, cgx_meshgen_out** out, float* device_ms);

void cgx_operators_free(cgx_meshgen_out* m);

#ifdef __cplusplus
}
#endif
#endif
