/*
 * cgx_mles.h -- reader for the mesher's .mles files (C ABI, exported by
 * libcgx_meshgen.so).
 *
 * Restates StripedMesh::read_mles (src/core/common/StripedMesh.hpp:1336-2380)
 * for a single process: the UGP record stream (magic 123581321, io version
 * 5), each record a 256-byte header (name[52], id, skip, idata[16],
 * rdata[12], ui8data[4]; Defs.hpp:228-247) followed by its data, 64-bit
 * counts stored as (lsw, msw) int pairs (ByteSwap.hpp:117-132).  The records
 * read are the ones Stitch writes for the solver:
 *
 *   counts            no_fa_bf_cv_counts (nno, nbf, nfa, ncv, nno_p, nno_pb,
 *                     27 face-zone counts)
 *   nodes             x_no
 *   internal faces    cvofa (int8 pairs), noofa (counts + int8 nodes), n_fa,
 *                     x_fa
 *   boundary faces    bf zone headers, cvobf, noobf, n_bf, x_bf, area_bf,
 *                     area_over_delta_bf, Gij_bf
 *   cells             cv zone headers, vol_cv, r_vv, x_vv, x_cv
 *
 * Timestamps, parameters, hash ids, surface and bounding-box records are
 * skipped, as the reference's solver-side read skips them.  Periodic meshes
 * (periodic faces or nodes, periodic transforms) and byte-swapped files are
 * rejected with CGX_MLES_E_UNSUPPORTED.  Extended faces are not stored in the
 * file (the solver builds them: include/cgx_ops.h).
 */
#ifndef CGX_MLES_H
#define CGX_MLES_H

#ifdef __cplusplus
extern "C" {
#endif

#define CGX_MLES_OK                0
#define CGX_MLES_E_IO             -1   /* cannot open or read the file */
#define CGX_MLES_E_FORMAT         -2   /* not a UGP record stream, or inconsistent records */
#define CGX_MLES_E_UNSUPPORTED    -3   /* io version, byte order or periodicity not handled */
#define CGX_MLES_E_OOM            -4

typedef struct cgx_mles_bf_zone {
  char   name[52];
  long long nbf, ibf_f;           /* faces [ibf_f, ibf_f + nbf) of the boundary arrays */
  double area, area_over_delta;   /* zone totals from the header */
  double n[3], x[3];
} cgx_mles_bf_zone;

typedef struct cgx_mles {
  int io_version;
  long long nno, nbf, nfa, ncv;   /* nodes, boundary faces, internal faces, cells */
  long long nno_p, nno_pb, nfa_p; /* periodic nodes, periodic+boundary nodes, periodic faces */
  long long nfa_zone[27];         /* 0..25 periodic flavours, 26 internal */
  double (*x_no)[3];              /* [nno] */
  int    (*cvofa)[2];             /* [nfa] */
  int     *noofa_i;               /* [nfa+1] CSR into noofa_v */
  int     *noofa_v;               /* node indices */
  double (*n_fa)[3], (*x_fa)[3];  /* [nfa] area vector cvofa0 -> cvofa1, centroid */
  int     *cvobf;                 /* [nbf] */
  int     *noobf_i, *noobf_v;     /* [nbf+1], node indices */
  double (*n_bf)[3], (*x_bf)[3];  /* [nbf] outward area vector, centroid */
  double  *area_bf, *area_over_delta_bf;  /* [nbf] */
  double (*Gij_bf)[3][3];         /* [nbf] */
  double  *vol_cv, *r_vv;         /* [ncv] */
  double (*x_vv)[3], (*x_cv)[3];  /* [ncv] */
  int nbf_zones;
  cgx_mles_bf_zone* bf_zones;     /* [nbf_zones] in file order */
  int ncv_zones;
  long long cv_zone_ncv[16];      /* cells per fluid zone (first 16 zones) */
} cgx_mles;

/* Read `path`.  *out is allocated here and released with cgx_mles_free().
 * Arrays absent from the file are NULL. */
int cgx_mles_read(const char* path, cgx_mles** out);
void cgx_mles_free(cgx_mles* m);

/*
 * Result files (.sles), as StaticSolver::writeSles -> writeData writes them
 * (src/core/common/StaticSolver.hpp:2311-2321, StaticSolver.cpp:7560-7640):
 * the UGP record stream with magic 123581322 (the restart magic + 1) and io
 * version 5, then
 *   UGP_IO_HASHIDS  two 20-byte hash ids (written as zeros: this library
 *                   keeps no mesh hash)
 *   UGP_IO_PARAMS   the caller's parameter text (may be empty)
 *   the registered data in name order, as CtiData::writeData lays them out
 *   (src/core/common/CtiRegister.cpp:412-610): CV_D1 "rho", CV_D1 "rhoE",
 *   I0 "step", D0 "time", CV_D2 "u" -- cell values in the mesh's global cell
 *   order, counts as (lsw, msw) int pairs
 *   EOF
 * cgx_sles_read reads those five records back (any order, other records
 * skipped) for a mesh of ncv cells; rho, u, rhoE may be NULL.
 */
int cgx_sles_write(const char* path, long long ncv, int step, double time, const double* rho,
                   const double* u, const double* rhoE, const char* params);
int cgx_sles_read(const char* path, long long ncv, int* step, double* time, double* rho, double* u,
                  double* rhoE);

/* Error text for the last failing call on this thread. */
const char* cgx_mles_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
