// cgx_kernels.cuh -- device-side records of the B200 compressible-LES
// right-hand side.
//
// Data layout in HBM (cells renumbered on a space-filling curve, "new" order):
//   state    rho[N], u0[N], u1[N], u2[N], rhoE[N]          (SoA, FP64)
//   rhs      rhs[stage][5][N]                              (SoA, FP64)
//   LRec[N]  {u0,u1,u2, 1/rho, p, h, rho, sos}  64 B       neighbour gathers
//   VRec[N]  {mu_total, loc_total, a_sgs, fgr, symh, symp, dudx[9], -}
//            128 B: lagged properties (per step) and the velocity gradient
//            (per stage), one 128 B line per neighbour gather
//   QRec[N]  {log(p/p_ref), p, 1/rho, 1/(R T)}  32 B (Gibbs sensor)
//   Work items: runs of at most kItemCells consecutive cells.  For each item
//   the mesh lists its halo, the cells outside the item that its cells'
//   extended faces reach (hcell) and, separately, those their compact faces
//   reach (chcell), ascending.  The face-flux kernels copy the packed records
//   of an item's cells and halo into shared memory once, then every face reads
//   its neighbour there through a 16-bit local index (the item's own cells
//   first, then the halo in list order).
//   Extended-face entries: a CSR over cells (off[N+1]) of directed entries,
//   one per (cell, face) pair, a cell's compact faces first.  Per entry: the
//   local index lidx[k], the global neighbour nbr[k] and six FP64 planes
//   en[d*E + k] {normal along the entry (n[3], negated for the face's second
//   cell), the halved c vector (c[3])}, streamed contiguously by the cell's G
//   lanes.
//   Compact-face entries: the first ncomp(i) = qoff[i+1]-qoff[i] extended
//   entries of each cell; their local indices in the compact union clidx[q]
//   and six FP64 planes qg[d*Q + q] {unit normal along the entry (3), area,
//   area_over_delta, area/area_over_delta} at q = qoff[i] + t.
//   Gradient coefficients per directed compact entry in a second CSR (coff,
//   the reference's cvocv order).
#ifndef CGX_KERNELS_CUH
#define CGX_KERNELS_CUH

#include <cstdint>

namespace cgx {

constexpr int kRevBit = 0x80000000;
constexpr int kMaxScalars = 8;  // transport scalars per cell
constexpr int kFidMask = 0x7fffffff;

struct alignas(32) LRec {
  double u[3];
  double sp_vol;
  double p;
  double h;
  double rho;
  double sos;
};

// per-cell viscous record: lagged properties then dudx[i][j] at g[3*i+j];
// mu_lam (the laminar viscosity of the wall boundary flux) in the last slot
struct alignas(128) VRec {
  double mu_total;
  double loc_total;
  double a_sgs;
  double fgr;
  double symh;
  double symp;
  double g[9];
  double mu_lam;
};

struct alignas(32) QRec {
  double logp;
  double p;
  double iv;  // 1/rho
  double ib;  // 1/(R T)
};

// geometry of one face as built on the host (expanded into the per-entry
// planes on the device)
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
struct alignas(32) LRecF {
  float u[3];
  float sp_vol;
  float pp;  // p - p_ref
  float hh;  // h - h_ref
  float rho;
  float sos;
};

struct alignas(64) VRecF {
  float mu_total, loc_total, a_sgs, fgr, symh, symp;
  float g[9];
  float mu_lam;
};

struct alignas(16) QRecF {
  float logp, pp, iv, ib;
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
  int limit_asgs; // LIMIT_ASGS
  double invgm1;  // 1/(gamma-1)
};

// Device-resident control block (one per solver).
// A boundary zone's condition: its kind (CGX_BC_*, 0 until set) and its
// parameters.  Walls: a[0..2] the wall velocity, a[3] T_bc (isothermal).
// CBC zones: the boundary state of each face, velocity a[0..2] + a[3] n/|n|,
// p = a[4], sp_vol = a[5], h = a[6], as the reference's initData fills its
// bf_state from the zone's parameters.
struct BcZone {
  int kind;
  int pad;
  double a[7];
};

struct Ctl {
  double dt;         // dt of the next step (read by the RK kernels)
  double dt_last;    // dt of the last completed step (the reference's `dt`)
  double time;
  double dt_data0;   // DT value or CFL target
  double cfl_max;    // last calcCfl(NULL, 1.0)
  double dt_sgs;     // the reference's `dt` for properties computed outside a
                     // step: 0 until a step runs, then the last step's dt (kept
                     // through a restore, as restoreData keeps it)
  int step;
  int nan;           // NaN seen in rho, p or T since last reset
  unsigned int blocks_done;
  int pad;
};

// A work item: up to kItemCells consecutive cells of one case and where its
// halo lists start.
constexpr int kItemCells = 128;
struct alignas(32) Item {
  int c;      // case slot in the table (0 in a mesh's own table)
  int cell0;  // first cell
  int ncell;  // cells in this item (<= kItemCells)
  int idx;    // item index within its case
  int hoff;   // extended-face halo: hcell[hoff, hoff + nh)
  int nh;
  int choff;  // compact-face halo: chcell[choff, choff + nch)
  int nch;
};

struct MeshDev {
  int N;                        // owned cells
  int nitems;                   // work items (mesh order)
  long long E;                  // directed extended entries
  long long Q;                  // directed compact entries
  const Item* items;            // [nitems]
  const int* hcell;             // extended-face halos
  const int* chcell;            // compact-face halos
  const long long* off;         // [N+1] extended-entry CSR
  const long long* qoff;        // [N+1] compact-entry CSR
  const int* nbr;               // [E] neighbour (new numbering, ghosts -> owner)
  const unsigned short* lidx;   // [E] neighbour in the item's extended union
  const unsigned short* clidx;  // [Q] neighbour in the item's compact union
  const double* en;             // [6][E] n (along the entry), c/2
  const double* qg;             // [6][Q] unit normal, area, aod, delta
  const long long* coff;        // [N+1] gradient CSR (cvocv without the diagonal)
  const int* cnbr;              // [C_dir]
  const unsigned short* cglidx; // [C_dir] neighbour in the item's compact union
  const double* gcx;            // [C_dir]
  const double* gcy;
  const double* gcz;
  const double* vol;
  const double* inv_vol;
  const double4* cc;            // {pow(vol,1/3), pow(vol,2/3), dcmag_hat, sa_to_vol}
  // boundary faces, ordered by cell (none: nbf = 0, pointers null)
  int nbf;
  int nzones;  // boundary zones
  int nbc;                      // cells with boundary faces
  const int* bfc;               // [N+1] each cell's faces in the bf arrays
  const int* bcell;             // [nbc] the cells with boundary faces, ascending
  const double* bf_n;           // [3][nbf] outward area vector
  const double* bf_aod;         // [nbf] area_over_delta_bf
  const int* bf_zone;           // [nbf]
  // FP32 copies for the mixed-precision form (null until a mixed solver exists)
  const float* en32;            // [6][E]
  const float* qg32;            // [6][Q]
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
  VRec* V;
  QRec* Q;
  // mixed-precision records (null for FP64 solvers)
  LRecF* LF;
  VRecF* VF;
  QRecF* QF;
  Ctl* ctl;
  double* red;  // per-block partials: [nblocks] cfl max, [nblocks] nan
  // transport scalars (calcRhsScalars / advanceScalars), FP64 solvers only
  int nsc;         // scalars per cell (0: none; the pointers below are null)
  double* sc;      // [nsc][N]
  double* rhs_sc;  // [3][nsc][N]
  double* mf;      // [E] mass flux of each extended entry, entry direction
  // boundary conditions per boundary zone
  const struct BcZone* bc;
  // per boundary face: the boundary state of zones whose state follows the
  // flow ([6][nbf]: u[3], sp_vol, p, h) and CBC_TOTAL_PT's normal speed
  // ([nbf]); bc_dyn: such zones exist (1 extrapolated, 2 total p/T)
  double* bfs;
  double* un_bc;
  // NSCBC zones, per boundary face ([20][nbf]): rho_bc, p_bc, u_bc[3], then
  // the characteristic rhs of stages 1..3 (5 each); wall-model faces keep
  // tau_wall and q_wall in rows 0 and 1 (stored and restored with rows 0-4)
  double* nsb;
  // per zone [8]: the zone sums of this stage (0..3) and the zone's own
  // state (4: CBC_TOTAL_PT USE_AVG's relaxed mean normal speed)
  double* zst;
  // a sponge zone: each cell's sponge state [4][N] (T, u), and the cells of
  // the layer with their strength ((s - L_max + length)/length)^2 times the
  // zone's strength
  double* spg;
  const int* spc;
  const double* spw;
  int nsp;
  double sp_p, sp_relax;  // the sponge's pressure and relaxation time
  int bc_dyn;  // 1 extrapolated, 2 total p/T, 4 NSCBC zones, 8 zone sums, 16 a sponge, 32 wall models
  double frame_om[3];  // the rotating frame's rate in radians per unit time (0: none)
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

}  // namespace cgx

#endif
