// cgx_mixed.cuh -- mixed-precision form of the face-flux, gradient and
// once-per-step kernels (included by cgx.cu).
//
// Reconstruction, fluxes, gradients and the SGS/property/sensor arithmetic
// run in FP32 on the FP32 records (cgx_kernels.cuh); every cell's face sums
// are accumulated in FP64.  The conserved state, the RK3 update, the pressure
// recovery p = (gamma-1)(rhoE - rho|u|^2/2), dt and the totals stay FP64.
//
// Pressure and enthalpy enter the FP32 flux arithmetic as perturbations
// p' = p - p_ref, h' = h - h_ref.  This is exact algebra on the reference's
// flux functions (src/charles/ideal_gas/IdealGasSolverFlux.hpp:9-215):
//  * every enthalpy term of the energy flux multiplies a mass-flux term
//    (skew mdot h_f, symmetric h_f dmdot, closure -ap_dp h_f and
//    -lf_drho (h_f - pv_m)), so F_E = h_ref F_rho + F_E(h'); the h_ref F_rho
//    part is added per cell in FP64 from the FP64 mass-flux sum;
//  * the constant pressure enters the momentum flux only as p_ref n, whose
//    sum over a cell's faces is p_ref times the extended-face GCL defect
//    (sum n = 0, FlowSolver.hpp:1596-1630), and is dropped.
#ifndef CGX_MIXED_CUH
#define CGX_MIXED_CUH

// (included inside cgx.cu's anonymous namespace)

struct FluxF {
  float rho, ru[3], rE;
};

// FP32 records in the swizzled shared arrays
__device__ __forceinline__ void smem_LF(const int4* sm, int j, LRecF& r) {
  const float4* p = reinterpret_cast<const float4*>(sm);
  const float4 a = p[swz<2>(j, 0)], b = p[swz<2>(j, 1)];
  r.u[0] = a.x; r.u[1] = a.y; r.u[2] = a.z; r.sp_vol = a.w;
  r.pp = b.x; r.hh = b.y; r.rho = b.z; r.sos = b.w;
}

__device__ __forceinline__ void smem_VF_sum(const int4* sm, int a, int b, VRecF& r) {
  const float4* p = reinterpret_cast<const float4*>(sm);
  float4 x = p[swz<4>(a, 0)], y = p[swz<4>(b, 0)];
  r.mu_total = x.x + y.x; r.loc_total = x.y + y.y; r.a_sgs = x.z + y.z; r.fgr = x.w + y.w;
  x = p[swz<4>(a, 1)]; y = p[swz<4>(b, 1)];
  r.symh = x.x + y.x; r.symp = x.y + y.y; r.g[0] = x.z + y.z; r.g[1] = x.w + y.w;
  x = p[swz<4>(a, 2)]; y = p[swz<4>(b, 2)];
  r.g[2] = x.x + y.x; r.g[3] = x.y + y.y; r.g[4] = x.z + y.z; r.g[5] = x.w + y.w;
  x = p[swz<4>(a, 3)]; y = p[swz<4>(b, 3)];
  r.g[6] = x.x + y.x; r.g[7] = x.y + y.y; r.g[8] = x.z + y.z;
}

// the once-per-step kernel's streams, mixed form
__device__ __forceinline__ void prefetch_end_f(const MeshDev& m, const Item& it, int sub, int cpr) {
  const int a = min(sub * cpr, it.ncell), b = min((sub + 1) * cpr, it.ncell);
  const int t = threadIdx.x;
  if (a >= b || t >= 6) return;
  if (t == 0) {
    const long long k0 = __ldg(m.off + it.cell0 + a), k1 = __ldg(m.off + it.cell0 + b);
    prefetch_l2(m.lidx + k0, (k1 - k0) * 2);
    return;
  }
  const long long q0 = __ldg(m.qoff + it.cell0 + a), q1 = __ldg(m.qoff + it.cell0 + b);
  if (t == 5)
    prefetch_l2(m.clidx + q0, (q1 - q0) * 2);
  else
    prefetch_l2(m.qg32 + (t - 1) * m.Q + q0, (q1 - q0) * 4);
}

// ext_flux (cgx.cu) on the FP32 perturbation variables; F[4] excludes the
// h_ref F[0] part, and p_ref n (summing to p_ref times the GCL defect) is
// dropped.
__device__ __forceinline__ void ext_flux_f(float F[5], const float n[3], const float c[3], const LRecF& a,
                                           const LRecF& b) {
  const float rho_f = __fdividef(2.0f, a.sp_vol + b.sp_vol);
  float uf[3], du[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    uf[d] = 0.5f * (a.u[d] + b.u[d]);
    du[d] = b.u[d] - a.u[d];
  }
  const float un = uf[0] * n[0] + uf[1] * n[1] + uf[2] * n[2];
  const float uc = uf[0] * c[0] + uf[1] * c[1] + uf[2] * c[2];
  const float duc = du[0] * c[0] + du[1] * c[1] + du[2] * c[2];
  const float uaub = a.u[0] * b.u[0] + a.u[1] * b.u[1] + a.u[2] * b.u[2];
  const float ufdu = uf[0] * du[0] + uf[1] * du[1] + uf[2] * du[2];
  const float mdot = un * rho_f;
  const float dmdot = uc * (b.rho - a.rho) + rho_f * duc;
  const float mdot_c = uc * rho_f;
  const float M = mdot + dmdot;
  const float p_f = 0.5f * (a.pp + b.pp);
  const float dp = b.pp - a.pp;
  const float h_f = 0.5f * ((a.hh + b.hh) + uaub);
  const float dH = (b.hh - a.hh) + ufdu;
  F[0] = M;
#pragma unroll
  for (int d = 0; d < 3; ++d) F[1 + d] = p_f * n[d] + dp * c[d] + M * uf[d] + mdot_c * du[d];
  F[4] = M * h_f + mdot_c * dH;
}

__device__ __forceinline__ void compact_flux_add_f(FluxF& F, const float un_[3], float area, float aod,
                                                   float delta, const LRecF& a, const LRecF& b,
                                                   const VRecF& vs, const float uf[3], float h_f,
                                                   float p_ref) {
  const float half_aod = 0.5f * aod;
  const float mu_area = 0.5f * vs.mu_total * area;
  const float mu_aod = vs.mu_total * half_aod;
  const float k_aod = vs.loc_total * half_aod;
  const float hua = 0.5f * (a.u[0] * a.u[0] + a.u[1] * a.u[1] + a.u[2] * a.u[2]);
  const float hub = 0.5f * (b.u[0] * b.u[0] + b.u[1] * b.u[1] + b.u[2] * b.u[2]);
  const float d_half_usq = hub - hua;
  const float dh = b.hh - a.hh;
  float una = 0.0f, unb = 0.0f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    una += a.u[d] * un_[d];
    unb += b.u[d] * un_[d];
  }
  const float dun = unb - una;
  const float dun_3 = dun * (1.0f / 3.0f);
  const float dun2_6 = (unb * unb - una * una) * (1.0f / 6.0f);
  const float dp = b.pp - a.pp;
  const float fgr_f = 0.5f * vs.fgr;
  const float rho_m = 0.5f * (b.rho + a.rho);
  const float un_m = 0.5f * (una + unb);
  const float c_m = 0.5f * (a.sos + b.sos);
  const float mach_n = __fdividef(fabsf(un_m), c_m);
  const float drho = b.rho - a.rho;
  const float lf = fminf(fgr_f * mach_n, 0.5f) * (c_m + fabsf(un_m)) * area;
  const float lf_drho = lf * drho;
  const float lf_rho = lf * rho_m;
  float ap = 0.5f * vs.a_sgs * delta * area;
  ap += vs.symp * half_aod;
  const float ap_dp = ap * dp;
  F.rho -= lf_drho + ap_dp;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    F.ru[d] -= mu_aod * (b.u[d] - a.u[d] + dun_3 * un_[d]);
    F.ru[d] -= lf_drho * uf[d];
    F.ru[d] -= lf_rho * dun * un_[d];
    F.ru[d] -= uf[d] * ap_dp;
  }
  F.rE -= mu_aod * (d_half_usq + dun2_6);
  float hs = vs.symh * rho_m * fabsf(un_m) * half_aod;
  hs = fmaxf(hs - k_aod, 0.0f);
  F.rE -= (k_aod + hs) * dh;
  F.rE -= ap_dp * h_f;
  // p v with the full pressure (a value, no cancellation) and its difference
  // in perturbation form
  const float pv_m = 0.5f * ((a.pp * a.sp_vol + b.pp * b.sp_vol) + p_ref * (a.sp_vol + b.sp_vol));
  const float dpv = (b.pp * b.sp_vol - a.pp * a.sp_vol) + p_ref * (b.sp_vol - a.sp_vol);
  const float de = dh - dpv;
  F.rE -= lf_drho * (h_f - pv_m);
  F.rE -= lf_rho * de;
  F.rE -= lf_rho * un_m * dun;
  float gn[3];
  float gnn_3 = 0.0f, div_23 = 0.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    gn[k] = 0.5f * (vs.g[k] * un_[0] + vs.g[3 + k] * un_[1] + vs.g[6 + k] * un_[2]);
    gnn_3 += gn[k] * un_[k];
    div_23 += vs.g[4 * k];
  }
  div_23 *= (1.0f / 3.0f);
  gnn_3 *= (1.0f / 3.0f);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float t = (gn[d] - un_[d] * (gnn_3 + div_23)) * mu_area;
    F.ru[d] -= t;
    F.rE -= uf[d] * t;
  }
}

template <int G, bool DIRECT>
__global__ void __launch_bounds__(256, 4) k_rhs_ext_f(CASE_ARGS, int stage) {
  extern __shared__ int4 smem[];
#define PF_EXTF(it, mm, r) prefetch_round<false>(mm, mm.en32, it, r, 256 / G)
  STAGED_LOOP_BEGIN(PF_EXTF)
  stage_records<2>(smem, s.LF, it_, m.hcell + it_.hoff, it_.nh);
  stage_wait();
  const long long E = m.E;
  const double h_ref = CASE_PH.h_ref;
  STAGED_ROUNDS_BEGIN(G, PF_EXTF)
  long long b = 0, e = 0;
  LRecF Li;
  if (valid) {
    b = m.off[i];
    e = m.off[i + 1];
    smem_LF(smem, loc_, Li);
  }
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long k = b + lane; k < e; k += G) {
    const int jl = __ldg(m.lidx + k);
    const float* g = m.en32 + k;
    const float n[3] = {__ldg(g), __ldg(g + E), __ldg(g + 2 * E)};
    const float c[3] = {__ldg(g + 3 * E), __ldg(g + 4 * E), __ldg(g + 5 * E)};
    LRecF Lj;
    smem_LF(smem, jl, Lj);
    float F[5];
    ext_flux_f(F, n, c, Li, Lj);
    if (s.mf) s.mf[k] = double(F[0]);  // mass flux for calcRhsScalars
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] -= double(F[q]);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = group_sum<G>(acc[c]);
  acc[4] += h_ref * acc[0];
  if (valid) {
    double* r = s.rhs + size_t(stage) * 5 * m.N;
#pragma unroll
    for (int c = 0; c < 5; ++c)
      if (c % G == lane) r[size_t(c) * m.N + i] = acc[c];
  }
  STAGED_ROUNDS_END
  STAGED_LOOP_END
#undef PF_EXTF
}

template <int G, bool DIRECT>
__global__ void __launch_bounds__(256, 3) k_rhs_comp_f(CASE_ARGS, int stage) {
  extern __shared__ int4 smem[];
#define PF_COMPF(it, mm, r) prefetch_round<true>(mm, mm.qg32, it, r, 256 / G)
  STAGED_LOOP_BEGIN(PF_COMPF)
  const int nu = it_.ncell + it_.nch;
  int4* sV = smem + swz_chunks<2>(nu);
  stage_records<2>(smem, s.LF, it_, m.chcell + it_.choff, it_.nch);
  stage_records<4>(sV, s.VF, it_, m.chcell + it_.choff, it_.nch);
  stage_wait();
  const long long Q = m.Q;
  const double h_ref = CASE_PH.h_ref;
  const float p_ref = float(CASE_PH.p_ref);
  STAGED_ROUNDS_BEGIN(G, PF_COMPF)
  long long q0 = 0, q1 = 0;
  LRecF Li;
  if (valid) {
    q0 = m.qoff[i];
    q1 = m.qoff[i + 1];
    smem_LF(smem, loc_, Li);
  }
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long q = q0 + lane; q < q1; q += G) {
    const int jl = __ldg(m.clidx + q);
    const float* h = m.qg32 + q;
    const float un[3] = {__ldg(h), __ldg(h + Q), __ldg(h + 2 * Q)};
    const float area = __ldg(h + 3 * Q), aod = __ldg(h + 4 * Q), delta = __ldg(h + 5 * Q);
    LRecF Lj;
    smem_LF(smem, jl, Lj);
    VRecF Vs;
    smem_VF_sum(sV, loc_, jl, Vs);
    float uf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) uf[d] = 0.5f * (Li.u[d] + Lj.u[d]);
    const float uaub = Li.u[0] * Lj.u[0] + Li.u[1] * Lj.u[1] + Li.u[2] * Lj.u[2];
    const float h_f = 0.5f * ((Lj.hh + Li.hh) + uaub);
    FluxF F;
    F.rho = 0.0f; F.ru[0] = F.ru[1] = F.ru[2] = 0.0f; F.rE = 0.0f;
    compact_flux_add_f(F, un, area, aod, delta, Li, Lj, Vs, uf, h_f, p_ref);
    if (s.mf) s.mf[m.off[i] + (q - q0)] += double(F.rho);  // the closure's mass flux
    acc[0] -= double(F.rho);
    acc[1] -= double(F.ru[0]);
    acc[2] -= double(F.ru[1]);
    acc[3] -= double(F.ru[2]);
    acc[4] -= double(F.rE);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = group_sum<G>(acc[c]);
  acc[4] += h_ref * acc[0];
  if (valid && q1 > q0) {
    double* r = s.rhs + size_t(stage) * 5 * m.N;
#pragma unroll
    for (int c = 0; c < 5; ++c)
      if (c % G == lane) r[size_t(c) * m.N + i] += acc[c];
  }
  STAGED_ROUNDS_END
  STAGED_LOOP_END
#undef PF_COMPF
}

template <int G, bool DIRECT>
__global__ void __launch_bounds__(256) k_grad_f(CASE_ARGS) {
  extern __shared__ int4 smem[];
#define PF_GRADF(it, mm, r) prefetch_grad(mm, mm.gcx32, mm.gcy32, mm.gcz32, it, r, 256 / G)
  STAGED_LOOP_BEGIN(PF_GRADF)
  stage_records<1, 2>(smem, s.LF, it_, m.chcell + it_.choff, it_.nch);
  stage_wait();
  const float4* su = reinterpret_cast<const float4*>(smem);
  STAGED_ROUNDS_BEGIN(G, PF_GRADF)
  long long b = 0, e = 0;
  float ui[3] = {0.0f, 0.0f, 0.0f};
  if (valid) {
    b = m.coff[i];
    e = m.coff[i + 1];
    const float4 a = su[loc_];
    ui[0] = a.x; ui[1] = a.y; ui[2] = a.z;
  }
  float g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long k = b + lane; k < e; k += G) {
    const int jl = __ldg(m.cglidx + k);
    const float cx = __ldg(m.gcx32 + k), cy = __ldg(m.gcy32 + k), cz = __ldg(m.gcz32 + k);
    const float4 ja = su[jl];
    const float du[3] = {ja.x - ui[0], ja.y - ui[1], ja.z - ui[2]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      g[3 * d + 0] += cx * du[d];
      g[3 * d + 1] += cy * du[d];
      g[3 * d + 2] += cz * du[d];
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) g[c] += __shfl_xor_sync(0xffffffffu, g[c], o);
  }
  if (valid) {
#pragma unroll
    for (int c = 0; c < 9; ++c)
      if (c % G == lane) s.VF[i].g[c] = g[c];
  }
  STAGED_ROUNDS_END
  STAGED_LOOP_END
#undef PF_GRADF
}

// cell_props in FP32 (SGS, properties and the sensor function; dt the
// solver's dt for limitAsgs); returns whether rho, p or T is NaN.
__device__ __forceinline__ int cell_props_f(const Phys& ph, const MeshDev& m, const StateDev& s, int i,
                                            const LRecF& Li, float vv2, double dt) {
  float g[9];
  {
    const float* vg = s.VF[i].g;
#pragma unroll
    for (int c = 0; c < 9; ++c) g[c] = __ldg(vg + c);
  }
  const double2 cc01 = __ldg(reinterpret_cast<const double2*>(m.cc + i));
  const double2 cc23 = __ldg(reinterpret_cast<const double2*>(m.cc + i) + 1);
  const float rho = Li.rho, sos = Li.sos;
  const float p = float(ph.p_ref) + Li.pp;
  const float T = p / (rho * float(ph.R));
  float mu_sgs = 0.0f, a_sgs = 0.0f, loc_sgs = 0.0f;
  if (ph.sgs_model == CGX_SGS_VREMAN) {
    const float dx = float(cc01.x);
    const float dx2 = dx * dx;
    const float a11 = g[0], a12 = g[1], a13 = g[2];
    const float a21 = g[3], a22 = g[4], a23 = g[5];
    const float a31 = g[6], a32 = g[7], a33 = g[8];
    const float a11s = a11 * a11, a22s = a22 * a22, a33s = a33 * a33;
    const float a12s = a12 * a12, a13s = a13 * a13, a23s = a23 * a23;
    const float a21s = a21 * a21, a31s = a31 * a31, a32s = a32 * a32;
    const float b11 = dx2 * (a11s + a21s + a31s);
    const float b22 = dx2 * (a12s + a22s + a32s);
    const float b33 = dx2 * (a13s + a23s + a33s);
    const float b12 = dx2 * (a11 * a12 + a21 * a22 + a31 * a32);
    const float b13 = dx2 * (a11 * a13 + a21 * a23 + a31 * a33);
    const float b23 = dx2 * (a12 * a13 + a22 * a23 + a32 * a33);
    float B = (b11 * b22 - b12 * b12) + (b11 * b33 - b13 * b13) + (b22 * b33 - b23 * b23);
    B = (B + fabsf(B)) * 0.5f;
    const float alal = ((a11s + a22s) + (a33s + a12s)) + ((a13s + a23s) + (a21s + a31s)) + a32s;
    const float s_mag = sqrtf(B / (alal + 1.0E-20f));
    mu_sgs = rho * float(ph.vreman_coeff) * s_mag;
    const float inv_sos2 = 1.0f / (sos * sos);
    a_sgs = float(ph.a_sgs_coeff) * s_mag / dx2;
    const float dil = g[0] + g[4] + g[8];
    const float tt = fabsf(dil) * dx / sos;
    if (tt > 0.01f) {
      const float Masq = (Li.u[0] * Li.u[0] + Li.u[1] * Li.u[1] + Li.u[2] * Li.u[2]) * inv_sos2;
      a_sgs += float(ph.a_sgs_coeff2) * float(cc23.y) * fminf(Masq, 10.0f) * sos;
    }
    a_sgs *= inv_sos2;
    // limitAsgs (IdealGasSolverSgs.cpp:4-48)
    if (ph.limit_asgs && dt > 0.0) {
      const float usq = Li.u[0] * Li.u[0] + Li.u[1] * Li.u[1] + Li.u[2] * Li.u[2];
      const float fax = float(ph.invgm1) + 0.5f * usq * inv_sos2;
      const float ceil_a = 1.0f / (float(dt) * fax * 4.0f) * inv_sos2;
      if (a_sgs > ceil_a) a_sgs = ceil_a;
    }
    loc_sgs = float(ph.lambda_dil_coeff) * rho * fabsf(dil) * dx2;
    loc_sgs += mu_sgs * float(1.0 / ph.Pr_t);
  }
  const float mu_lam =
      float(ph.mu_ref) * (1.0f + expm1f(float(ph.mu_power_law) * logf(T * float(1.0 / ph.T_ref))));
  const float loc_lam = mu_lam * float(1.0 / ph.Pr_lam);
  const float sos2 = float(ph.gamma) * p / rho;
  const float lambda = sqrtf(Li.u[0] * Li.u[0] + Li.u[1] * Li.u[1] + Li.u[2] * Li.u[2]) + sqrtf(sos2);
  const float symp = fmaxf(float(ph.coeff_p) * float(cc23.x) * lambda / sos2 - float(cc01.y) * a_sgs, 0.0f);
  const float symh = float(ph.coeff_h) * float(cc23.x);
  float fgr = 0.5f / (1.0f + expf(-2.0f * (vv2 - float(ph.gr_nrm)) / 5.0e-03f));
  if (ph.diss_mode == CGX_DISS_NONE) fgr = 0.0f;
  if (ph.diss_mode == CGX_DISS_ALL) fgr = 0.5f;
  float* P = reinterpret_cast<float*>(s.VF + i);
  reinterpret_cast<float4*>(P)[0] = make_float4(mu_lam + mu_sgs, loc_lam + loc_sgs, a_sgs, fgr);
  reinterpret_cast<float2*>(P)[2] = make_float2(symh, symp);
  P[15] = mu_lam;
  return (rho != rho) || (p != p) || (T != T);
}

// once per step, mixed form: FP32 SGS/properties/sensor, FP64 CFL sums and
// reductions (same structure as k_step_end)
template <int G, bool DIRECT>
__global__ void __launch_bounds__(256, 3) k_step_end_f(CASE_ARGS, int mode) {
  extern __shared__ int4 smem[];
  __shared__ double sh_cfl[256];
  __shared__ int sh_nan[256];
  __shared__ bool am_last;
#define PF_ENDF(it, mm, r) prefetch_end_f(mm, it, r, 256 / G)
  STAGED_LOOP_BEGIN(PF_ENDF)
  const Phys& ph = CASE_PH;
  const int nu = it_.ncell + it_.nh;
  int4* sL = smem + swz_chunks<1>(nu);
  stage_records<1>(smem, s.QF, it_, m.hcell + it_.hoff, it_.nh);
  stage_records<2>(sL, s.LF, it_, m.chcell + it_.choff, it_.nch);
  stage_wait();
  const long long Q = m.Q;
  // limitAsgs's dt: this step's, or outside a step the control block's
  const double dt_sgs = (mode & 1) ? s.ctl->dt : s.ctl->dt_sgs;
  double cmax = 0.0;
  int anynan = 0;
  STAGED_ROUNDS_BEGIN(G, PF_ENDF)
  long long b = 0, e = 0, q0 = 0, q1 = 0;
  LRecF Li;
  float4 qi = make_float4(0.f, 0.f, 0.f, 0.f);
  if (valid) {
    b = m.off[i];
    e = m.off[i + 1];
    q0 = m.qoff[i];
    q1 = m.qoff[i + 1];
    smem_LF(sL, loc_, Li);
    qi = reinterpret_cast<const float4*>(smem)[loc_];
  }
  float vv2 = 0.0f;
  double cfl = 0.0;
  for (long long k = b + lane; k < e; k += G) {
    const float4 qj = reinterpret_cast<const float4*>(smem)[__ldg(m.lidx + k)];
    const float dp = qj.y - qi.y;
    const float v_avg = 0.5f * (qi.z + qj.z);
    const float beta = 0.5f * (qi.w + qj.w);
    const float gr = qj.x - qi.x - v_avg * dp * beta;
    vv2 = fmaxf(vv2, fabsf(gr));
  }
  for (long long q = q0 + lane; q < q1; q += G) {
    const int jl = __ldg(m.clidx + q);
    const float* h = m.qg32 + q;
    const float un[3] = {__ldg(h), __ldg(h + Q), __ldg(h + 2 * Q)};
    const float area = __ldg(h + 3 * Q);
    LRecF Lj;
    smem_LF(sL, jl, Lj);
    const float undA = 0.5f * area * ((Li.u[0] * un[0] + Li.u[1] * un[1] + Li.u[2] * un[2]) +
                                      (Lj.u[0] * un[0] + Lj.u[1] * un[1] + Lj.u[2] * un[2]));
    cfl += double(fabsf(undA)) + double(area) * (0.5 * (double(Li.sos) + double(Lj.sos)));
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) vv2 = fmaxf(vv2, __shfl_xor_sync(0xffffffffu, vv2, o));
  cfl = group_sum<G>(cfl);
  if (valid && lane == 0) {
    anynan |= cell_props_f(ph, m, s, i, Li, vv2, dt_sgs);
    cfl += cfl_bf(m, i, double(Li.u[0]), double(Li.u[1]), double(Li.u[2]), double(Li.sos));
    cmax = fmax(cmax, cfl * (0.5 * 1.0 * __ldg(m.inv_vol + i)));
  }
  STAGED_ROUNDS_END
  sh_cfl[threadIdx.x] = cmax;
  sh_nan[threadIdx.x] = anynan;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) {
      sh_cfl[threadIdx.x] = fmax(sh_cfl[threadIdx.x], sh_cfl[threadIdx.x + w]);
      sh_nan[threadIdx.x] |= sh_nan[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int np = CASE_NITEMS;
    s.red[it_.idx] = sh_cfl[0];
    s.red[np + it_.idx] = double(sh_nan[0]);
    __threadfence();
    const unsigned int done = atomicAdd(&s.ctl->blocks_done, 1u);
    am_last = (done == unsigned(np) - 1u);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    finalize_ctl(s.ctl, s.red, ph.dt_mode, ph.dt_max, mode, CASE_NITEMS);
  }
  STAGED_LOOP_END
#undef PF_ENDF
}

#endif
