// cgx_kernels.cuh -- device side of the B200 compressible-LES right-hand side.
//
// Data layout in HBM (cells renumbered on a space-filling curve, "new" order):
//   state    rho[N], u0[N], u1[N], u2[N], rhoE[N]          (SoA, FP64)
//   rhs      rhs[stage][5][N]                              (SoA, FP64)
//   Lrec[N]  {u0,u1,u2, 1/rho, p, h, rho, sos}  64 B       neighbour gathers
//   Prec[N]  {mu_total, loc_total, a_sgs, fgr, symh, symp, -, -}  64 B (per step)
//   Grec[N]  dudx[3][3] + pad                   80 B
//   Qrec[N]  {log(p/p_ref), p, 1/rho, 1/(R T)}  32 B (Gibbs sensor)
//   extended faces: per face one 64 B record {n[3], c[3] (halved), -, -};
//   compact faces (ids [0, n_cf) of the same numbering) one 64 B record
//   {unit_n[3], area, area_over_delta, n_fa[3]}.
//   Per-cell face lists in SELL-32: slot (slice s, k, lane) at
//   slice_off[s] + 32 k + lane, entries {nbr cell, face id | 0x80000000 when
//   the cell is the face's second cell}; a cell's compact faces come first.
//   Gradient coefficients per directed compact entry in a second SELL-32.
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
  double iv;   // 1/rho
  double ib;   // 1/(R T)
};

struct alignas(16) EFRec {
  double n[3];
  double c[3];  // already halved
  double pad0, pad1;
};

struct alignas(16) CFRec {
  double un[3];  // unit normal along the extended face's orientation
  double area;
  double aod;    // area_over_delta
  double nfa[3]; // n_fa along the same orientation
};

struct Phys {
  double gamma, R, p_ref, T_ref, mu_ref, mu_power_law, Pr_lam;
  int sgs_model;
  double vreman_coeff, a_sgs_coeff, a_sgs_coeff2, lambda_dil_coeff, Pr_t;
  double coeff_p, coeff_h, gr_nrm;
  int diss_mode;
  int dt_mode;
  double dt_max;  // CFL_DT
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
  int N;                     // owned cells
  int nslices;
  const long long* slice_off;   // [nslices+1] extended SELL
  const int* slice_w;           // [nslices]
  const long long* cslice_off;  // [nslices+1] compact SELL (gradient coeffs)
  const int* meta;              // [N] deg | ncomp << 16
  const int* nbr;               // [slots]
  const int* fid;               // [slots]
  const double* gcx;            // [cslots]
  const double* gcy;
  const double* gcz;
  const EFRec* ef;
  const CFRec* cf;
  const double* vol;
  const double* inv_vol;
  const double4* cc;            // {pow(vol,1/3), pow(vol,2/3), dcmag_hat, sa_to_vol}
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
  Ctl* ctl;
  double* red;  // per-block partials: [nblocks] cfl max, [nblocks] nan
};

}  // namespace cgx

#endif
