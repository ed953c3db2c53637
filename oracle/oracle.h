/*
 * oracle.h -- CPU restatement of the reference's compressible-LES hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the GPU path
 * (libcgx.so) is compared against, and the timed CPU baseline.  No product
 * code links or calls it.
 *
 * The solver mirrors IdealGasSolver (src/charles/ideal_gas/) on one or more
 * "ranks": nparts contiguous cell ranges that each run the reference's face
 * loops on their own faces, with faces between ranges handled from each side
 * as the reference handles inter-processor faces (calcRhsBase ranges
 * [n_cc_i, n_cc_b), IdealGasSolver.cpp:416-533).  nparts = 1 is the
 * reference's single-rank order.  Ghosts are explicit copies of their owners,
 * refreshed where the reference calls updateCv2ClassStart/Finish.
 */
#ifndef CGX_ORACLE_H
#define CGX_ORACLE_H

#include "../include/cgx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_solver orc_solver;

orc_solver* orc_create(const cgx_mesh_desc* mesh, const cgx_params* p, int nparts);
void orc_destroy(orc_solver* o);

void orc_set_state(orc_solver* o, const double* rho, const double* u, const double* rhoE);
void orc_set_state_primitive(orc_solver* o, const double* rho, const double* u, const double* p);
void orc_get_state(const orc_solver* o, double* rho, double* u, double* rhoE);

void orc_init_complete(orc_solver* o);
void orc_update_primitive(orc_solver* o);
void orc_calc_sgs_props(orc_solver* o);
/* zero rhs[stage-1], run calcRhsBase into it; copy to rhs_out[ncv][5] if
 * non-NULL; scale_out[ncv][5] (optional) = sum over the cell's faces of
 * |face flux| per component, the conditioning scale of the face sum. */
void orc_calc_rhs(orc_solver* o, int rk_stage, double* rhs_out, double* scale_out);
void orc_rk3_step(orc_solver* o, const double w[3], double dt, int rk_stage);
/* Transport scalars (calcRhsScalars / advanceScalars): nsc per cell,
 * sc[icv*nsc + isc] over the ncv owned cells (ghosts are copies).  Once set,
 * orc_calc_rhs and the steps also form and apply rhs_sc.  0, or -1 on a bad
 * argument. */
int orc_set_scalars(orc_solver* o, int nsc, const double* sc);
void orc_get_scalars(const orc_solver* o, double* sc);
/* rhs_sc[ncv][nsc] of stage rk_stage as the last orc_calc_rhs / step left it;
 * scale_out (optional) = sum of |face flux| per cell and scalar (filled by an
 * orc_calc_rhs called with a scale_out). */
void orc_get_rhs_sc(const orc_solver* o, int rk_stage, double* rhs_sc, double* scale_out);
double orc_calc_cfl(const orc_solver* o, double dt, double* cfl);
/* setDt per dt_mode; returns dt */
double orc_set_dt(orc_solver* o);
/* advanceSolution with the current dt: 0, or -1 on NaN (state restored) */
int orc_advance_solution(orc_solver* o);
/* nsteps of {setDt; advanceSolution; report}; 0 or -1 */
int orc_step(orc_solver* o, int nsteps);
void orc_totals(const orc_solver* o, double out[5]);
void orc_get_time(const orc_solver* o, double* time, double* dt, int* step);

void orc_get_primitive(const orc_solver* o, double* p, double* T, double* sos);
void orc_get_grad(const orc_solver* o, double* dudx);
void orc_get_aux(const orc_solver* o, double* aux);
/* Source terms added by calc_rhs after the face sums, where the reference's
 * calcRhs calls addSourceHook (IdealGasSolver.hpp:697-705): per cell
 * f = vol rho (A u + g) into rhs.rhou and f.u into rhs.rhoE (the body and
 * relaxation forces of the reference's example hooks,
 * quiver/charles/charles.sphere.cpp:166-173), plus field[ncv][5] if non-NULL.
 * A = 0, g = 0 and field = NULL remove them. */
void orc_set_source(orc_solver* o, double A, const double g[3], const double* field);
/* Boundary condition of boundary zone `zone` (the mesh's zone_bf), as
 * registerBoundaryConditions sets one per zone (IdealGasSolver.hpp:170-231):
 * CGX_BC_SLIP or CGX_BC_WALL_ADIABATIC with the wall velocity u_wall (NULL:
 * zero).  0, or -1 on a bad argument. */
int orc_set_bc(orc_solver* o, int zone, int kind, const double u_wall[3]);
/* Boundary condition with the reference's zone parameters (the kinds and
 * parameter lists of cgx_set_bc_params): WALL_ISOTHERMAL T, CBC_UPT u p T,
 * CBC_RUNP rho un p, CBC_MPT mdot p T, CBC_EXTRAPOLATE, CBC_TOTAL_PT p_total
 * T_total t_relax [use_avg], NSCBC_MT mdot T (T < 0: total temperature -T),
 * NSCBC_OUTLET_P p_ref sigma L_ref, NSCBC_OUTLET_MDOT mdot t_relax; SLIP and
 * WALL_ADIABATIC as orc_set_bc.  0, or -1 on a bad argument. */
int orc_set_bc_params(orc_solver* o, int zone, int kind, const double* params, int nparams);
/* write a NaN into rho[icv] (host-side fault injection for the NaN path) */
void orc_poison(orc_solver* o, int icv);

/* 1 if this build evaluates the face fluxes with the reference's own
 * IdealGasSolverFlux.hpp compiled in place, 0 for the restatement. */
int orc_uses_reference_flux(void);
/* The algebraic wall model's tau_wall and wall heat flux on their own. */
double orc_wm_solve_tau(double u1, double y1, double rho, double mu, double ut_guess);
double orc_wm_q_wall(double T1, double Tw, double tau, double rho, double mu, double locp, double cp, double y1);
double orc_wm_r_approx(double tau, double rho, double mu, double locp, double cp, double y1);
/* CBC_PROFILE: the zone's faces (in face order) take bf_state[nz][6] = u[3], sp_vol, p, h. */
int orc_set_bc_profile(orc_solver* o, int zone, const double* bf_state, int nz);
/* ROTATING_REFERENCE_FRAME (revolutions per unit time); needs the mesh's x_cv. */
int orc_set_frame_rotation(orc_solver* o, const double rev[3]);
/* A velocity face by face, u[nz][3] in face order: an adiabatic wall's u_bc or
 * CBC_TOTAL_PT's frame velocity. */
int orc_set_bc_face_velocity(orc_solver* o, int zone, const double* u, int nz);
/* A WM_EXCHANGE zone's exchange points: cells cv[nz] (-1: not located), points x[nz][3]. */
int orc_set_bc_exchange(orc_solver* o, int zone, const int* cv, const double* x, int nz);
/* The equilibrium wall model's solve: tqT = {tau_w, q_w, T_w} in and out. */
int orc_wm_eq_solve(double* tqT, double u1, double T1, double rho1, double y1, double mu1, double Pr_lam, double cp,
                    double relax, double y_plus0, double tol);

#ifdef __cplusplus
}
#endif
#endif
