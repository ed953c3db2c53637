// cgx_kernels.cuh -- device-side records of the B200 compressible-LES
// right-hand side.
//
// Data layout in HBM (cells renumbered on a space-filling curve, "new" order):
//   state    rho[N], u0[N], u1[N], u2[N], rhoE[N]          (SoA, FP64)
//   rhs      rhs[stage][5][N]                              (SoA, FP64)
//   LRec[N]  {u0,u1,u2, 1/rho, p, h, rho, sos}  64 B       neighbour gathers
//   PRec[N]  {mu_total, loc_total, a_sgs, fgr, symh, symp, -, -}  64 B (per step)
//   GRec[N]  dudx[3][3] + pad                   80 B
//   QRec[N]  {log(p/p_ref), p, 1/rho, 1/(R T)}  32 B (Gibbs sensor)
//   extended faces: one 48 B record {n[3], c[3] (halved)} per face;
//   compact faces (ids [0, n_cf) of the same numbering) one 48 B record
//   {unit_n[3], area, area_over_delta, area/area_over_delta}.
//   Per-cell face lists (CSR over cells): entries {nbr cell, face id |
//   0x80000000 when the cell is the face's second cell}; a cell's compact
//   faces come first.  The lists are walked by a group of G lanes per cell.
//   Gradient coefficients per directed compact entry in a second CSR.
#ifndef CGX_KERNELS_CUH
#define CGX_KERNELS_CUH

#include <cstdint>

namespace cgx {

constexpr int kRevBit = 0x80000000;
constexpr int kFidMask = 0x7fffffff;

struct alignas(16) LRec {
  double u[3];
  double sp_vol;
  double p;
  double h;
  double rho;
  double sos;
};

struct alignas(16) PRec {
  double mu_total;
  double loc_total;
  double a_sgs;
  double fgr;
  double symh;
  double symp;
  double pad0, pad1;
};

struct alignas(16) GRec {
  double g[9];  // dudx[i][j] at 3*i+j
  double pad;
};

struct alignas(16) QRec {
  double logp;
  double p;
  double iv;  // 1/rho
  double ib;  // 1/(R T)
};

struct alignas(16) EFRec {
  double n[3];
  double c[3];  // already halved
};

struct alignas(16) CFRec {
  double un[3];  // unit normal along the extended face's orientation
  double area;
  double aod;    // area_over_delta
  double delta;  // area / area_over_delta
};

// Mixed-precision records (FP32).  Pressure and enthalpy are stored as
// perturbations about p_ref and h_ref = R gamma/(gamma-1) T_ref so that their
// differences keep FP32's relative precision at low Mach.
struct alignas(16) LRecF {
  float u[3];
  float sp_vol;
  float pp;  // p - p_ref
  float hh;  // h - h_ref
  float rho;
  float sos;
};

struct alignas(16) PRecF {
  float mu_total, loc_total, a_sgs, fgr, symh, symp, pad0, pad1;
};

struct alignas(16) GRecF {
  float g[9];
  float pad[3];
};

struct alignas(16) QRecF {
  float logp, pp, iv, ib;
};

struct alignas(16) EFRecF {
  float n[3];
  float c[3];
  float pad[2];
};

struct alignas(16) CFRecF {
  float un[3];
  float area;
  float aod;
  float delta;
  float pad[2];
};

struct Phys {
  double gamma, R, p_ref, T_ref, mu_ref, mu_power_law, Pr_lam;
  int sgs_model;
  double vreman_coeff, a_sgs_coeff, a_sgs_coeff2, lambda_dil_coeff, Pr_t;
  double coeff_p, coeff_h, gr_nrm;
  int diss_mode;
  int dt_mode;
  double dt_max;  // CFL_DT
  double h_ref;   // R gamma/(gamma-1) T_ref (mixed-precision offsets)
};

// Device-resident control block (one per solver).
struct Ctl {
  double dt;         // dt of the next step (read by the RK kernels)
  double dt_last;    // dt of the last completed step (the reference's `dt`)
  double time;
  double dt_data0;   // DT value or CFL target
  double cfl_max;    // last calcCfl(NULL, 1.0)
  int step;
  int nan;           // NaN seen in rho, p or T since last reset
  unsigned int blocks_done;
  int pad;
};

struct MeshDev {
  int N;                        // owned cells
  const long long* off;         // [N+1] extended-face CSR
  const int* ncomp;             // [N] compact faces at the head of each list
  const int* nbr;               // [E_dir]
  const int* fid;               // [E_dir]
  const long long* coff;        // [N+1] gradient CSR (cvocv without the diagonal)
  const int* cnbr;              // [C_dir]
  const double* gcx;            // [C_dir]
  const double* gcy;
  const double* gcz;
  const EFRec* ef;
  const CFRec* cf;
  const double* vol;
  const double* inv_vol;
  const double4* cc;            // {pow(vol,1/3), pow(vol,2/3), dcmag_hat, sa_to_vol}
  // FP32 copies for the mixed-precision form (null until a mixed solver exists)
  const EFRecF* ef32;
  const CFRecF* cf32;
  const float* gcx32;
  const float* gcy32;
  const float* gcz32;
};

struct StateDev {
  double* rho;
  double* u0;
  double* u1;
  double* u2;
  double* rhoE;
  double* rhs;  // [3][5][N]
  LRec* L;
  PRec* P;
  GRec* G;
  QRec* Q;
  // mixed-precision records (null for FP64 solvers)
  LRecF* LF;
  PRecF* PF;
  GRecF* GF;
  QRecF* QF;
  Ctl* ctl;
  double* red;  // per-block partials: [nblocks] cfl max, [nblocks] nan
};

// One resident case: its mesh, its state and its parameters.  The step
// kernels take a table of these and a work list of items.
struct CaseDev {
  MeshDev m;
  StateDev s;
  Phys ph;
  int nitems;  // work items of this case (partials of the per-step reduction)
  int pad;
};

// A work item: up to kItemCells consecutive cells of one case.
constexpr int kItemCells = 256;
struct Item {
  int c;      // case slot in the table
  int cell0;  // first cell
  int ncell;  // cells in this item (<= kItemCells)
  int idx;    // item index within its case
};

}  // namespace cgx

#endif
