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

__device__ __forceinline__ void load_LF(const LRecF* base, int j, LRecF& r) {
  const float4* p = reinterpret_cast<const float4*>(base + j);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  r.u[0] = a.x; r.u[1] = a.y; r.u[2] = a.z; r.sp_vol = a.w;
  r.pp = b.x; r.hh = b.y; r.rho = b.z; r.sos = b.w;
}

__device__ __forceinline__ void load_PF(const PRecF* base, int j, PRecF& r) {
  const float4* p = reinterpret_cast<const float4*>(base + j);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  r.mu_total = a.x; r.loc_total = a.y; r.a_sgs = a.z; r.fgr = a.w; r.symh = b.x; r.symp = b.y;
}

__device__ __forceinline__ void load_GF(const GRecF* base, int j, float g[9]) {
  const float4* p = reinterpret_cast<const float4*>(base + j);
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w;
  g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w; g[8] = c.x;
}

// skew-symmetric central flux on perturbation variables (F.rE excludes h_ref F.rho)
__device__ __forceinline__ void skew_flux_f(FluxF& F, const float n[3], const LRecF& a, const LRecF& b,
                                            float uf[3], float& rho_f, float& h_f) {
  rho_f = 2.0f / (a.sp_vol + b.sp_vol);
  const float p_f = 0.5f * (b.pp + a.pp);
  float un = 0.0f, uaub = 0.0f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float um = 0.5f * (a.u[d] + b.u[d]);
    un += um * n[d];
    uaub += a.u[d] * b.u[d];
    uf[d] = um;
    F.ru[d] = p_f * n[d];
  }
  const float mdot = un * rho_f;
  F.rho = mdot;
#pragma unroll
  for (int d = 0; d < 3; ++d) F.ru[d] += mdot * uf[d];
  h_f = 0.5f * ((b.hh + a.hh) + uaub);
  F.rE = mdot * h_f;
}

__device__ __forceinline__ void sym_flux_add_f(FluxF& F, const float c[3], const LRecF& a, const LRecF& b,
                                               const float uf[3], float rho_f, float h_f) {
  float du[3];
  float du_c = 0.0f, uf_c = 0.0f;
  const float dp = b.pp - a.pp;
  float dH = b.hh - a.hh;
  const float drho = b.rho - a.rho;
  float Gp[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float dd = b.u[d] - a.u[d];
    du[d] = dd;
    du_c += dd * c[d];
    uf_c += uf[d] * c[d];
    dH += uf[d] * dd;
    Gp[d] = dp * c[d];
  }
  const float dmdot = uf_c * drho + rho_f * du_c;
  const float mdot_c = uf_c * rho_f;
  F.rho += dmdot;
#pragma unroll
  for (int d = 0; d < 3; ++d) F.ru[d] += Gp[d] + (mdot_c * du[d] + uf[d] * dmdot);
  F.rE += h_f * dmdot + mdot_c * dH;
}

__device__ __forceinline__ void compact_flux_add_f(FluxF& F, const float un_[3], float area, float aod,
                                                   float delta, const LRecF& a, const LRecF& b,
                                                   const PRecF& ax, const PRecF& bx, const float uf[3],
                                                   float h_f, const float ga[9], const float gb[9],
                                                   float p_ref) {
  const float half_aod = 0.5f * aod;
  const float mu_area = 0.5f * (ax.mu_total + bx.mu_total) * area;
  const float mu_aod = (ax.mu_total + bx.mu_total) * half_aod;
  const float k_aod = (ax.loc_total + bx.loc_total) * half_aod;
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
  const float fgr_f = 0.5f * (bx.fgr + ax.fgr);
  const float rho_m = 0.5f * (b.rho + a.rho);
  const float un_m = 0.5f * (una + unb);
  const float c_m = 0.5f * (a.sos + b.sos);
  const float mach_n = fabsf(un_m) / c_m;
  const float drho = b.rho - a.rho;
  const float lf = fminf(fgr_f * mach_n, 0.5f) * (c_m + fabsf(un_m)) * area;
  const float lf_drho = lf * drho;
  const float lf_rho = lf * rho_m;
  float ap = 0.5f * (ax.a_sgs + bx.a_sgs) * delta * area;
  ap += (ax.symp + bx.symp) * half_aod;
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
  float hs = (ax.symh + bx.symh) * rho_m * fabsf(un_m) * half_aod;
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
    gn[k] = 0.5f * ((ga[k] + gb[k]) * un_[0] + (ga[3 + k] + gb[3 + k]) * un_[1] +
                    (ga[6 + k] + gb[6 + k]) * un_[2]);
    gnn_3 += gn[k] * un_[k];
    div_23 += ga[4 * k] + gb[4 * k];
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
  ITEM_LOOP_BEGIN(G)
  long long b = 0, e = 0;
  LRecF Li;
  if (valid) {
    b = m.off[i];
    e = m.off[i + 1];
    load_LF(s.LF, i, Li);
  }
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long k = b + lane; k < e; k += G) {
    const int j = __ldg(m.nbr + k);
    const int f = __ldg(m.fid + k);
    const float sg = (f < 0) ? -1.0f : 1.0f;
    const float4* ge = reinterpret_cast<const float4*>(m.ef32 + (f & kFidMask));
    const float4 g0 = __ldg(ge), g1 = __ldg(ge + 1);
    const float n[3] = {sg * g0.x, sg * g0.y, sg * g0.z};
    const float c[3] = {g0.w, g1.x, g1.y};
    LRecF Lj;
    load_LF(s.LF, j, Lj);
    FluxF F;
    float uf[3], rho_f, h_f;
    skew_flux_f(F, n, Li, Lj, uf, rho_f, h_f);
    FluxF C;
    C.rho = 0.0f; C.ru[0] = C.ru[1] = C.ru[2] = 0.0f; C.rE = 0.0f;
    sym_flux_add_f(C, c, Li, Lj, uf, rho_f, h_f);
    acc[0] -= double(F.rho) + double(C.rho);
    acc[1] -= double(F.ru[0]) + double(C.ru[0]);
    acc[2] -= double(F.ru[1]) + double(C.ru[1]);
    acc[3] -= double(F.ru[2]) + double(C.ru[2]);
    acc[4] -= double(F.rE) + double(C.rE);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = group_sum<G>(acc[c]);
  acc[4] += CASE_PH.h_ref * acc[0];
  if (valid) {
    double* r = s.rhs + size_t(stage) * 5 * m.N;
#pragma unroll
    for (int c = 0; c < 5; ++c)
      if (c % G == lane) r[size_t(c) * m.N + i] = acc[c];
  }
  ITEM_LOOP_END
}

template <int G, bool DIRECT>
__global__ void __launch_bounds__(256, 2) k_rhs_comp_f(CASE_ARGS, int stage) {
  ITEM_LOOP_BEGIN(G)
  long long b = 0, e = 0;
  LRecF Li;
  PRecF Pi;
  float gi[9];
  if (valid) {
    b = m.off[i];
    e = b + __ldg(m.ncomp + i);
    if (e > b + lane) {
      load_LF(s.LF, i, Li);
      load_PF(s.PF, i, Pi);
      load_GF(s.GF, i, gi);
    }
  }
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long k = b + lane; k < e; k += G) {
    const int j = __ldg(m.nbr + k);
    const int f = __ldg(m.fid + k);
    const float sg = (f < 0) ? -1.0f : 1.0f;
    const float4* gc = reinterpret_cast<const float4*>(m.cf32 + (f & kFidMask));
    const float4 h0 = __ldg(gc), h1 = __ldg(gc + 1);
    const float un[3] = {sg * h0.x, sg * h0.y, sg * h0.z};
    LRecF Lj;
    load_LF(s.LF, j, Lj);
    PRecF Pj;
    load_PF(s.PF, j, Pj);
    float gj[9];
    load_GF(s.GF, j, gj);
    float uf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) uf[d] = 0.5f * (Li.u[d] + Lj.u[d]);
    const float uaub = Li.u[0] * Lj.u[0] + Li.u[1] * Lj.u[1] + Li.u[2] * Lj.u[2];
    const float h_f = 0.5f * ((Lj.hh + Li.hh) + uaub);
    FluxF F;
    F.rho = 0.0f; F.ru[0] = F.ru[1] = F.ru[2] = 0.0f; F.rE = 0.0f;
    compact_flux_add_f(F, un, h0.w, h1.x, h1.y, Li, Lj, Pi, Pj, uf, h_f, gi, gj,
                       float(CASE_PH.p_ref));
    acc[0] -= double(F.rho);
    acc[1] -= double(F.ru[0]);
    acc[2] -= double(F.ru[1]);
    acc[3] -= double(F.ru[2]);
    acc[4] -= double(F.rE);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = group_sum<G>(acc[c]);
  acc[4] += CASE_PH.h_ref * acc[0];
  if (valid && e > b) {
    double* r = s.rhs + size_t(stage) * 5 * m.N;
#pragma unroll
    for (int c = 0; c < 5; ++c)
      if (c % G == lane) r[size_t(c) * m.N + i] += acc[c];
  }
  ITEM_LOOP_END
}

template <int G, bool DIRECT>
__global__ void __launch_bounds__(256) k_grad_f(CASE_ARGS) {
  ITEM_LOOP_BEGIN(G)
  long long b = 0, e = 0;
  float ui[3] = {0.0f, 0.0f, 0.0f};
  if (valid) {
    b = m.coff[i];
    e = m.coff[i + 1];
    const float4 a = __ldg(reinterpret_cast<const float4*>(s.LF + i));
    ui[0] = a.x; ui[1] = a.y; ui[2] = a.z;
  }
  float g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long k = b + lane; k < e; k += G) {
    const int j = __ldg(m.cnbr + k);
    const float cx = __ldg(m.gcx32 + k), cy = __ldg(m.gcy32 + k), cz = __ldg(m.gcz32 + k);
    const float4 ja = __ldg(reinterpret_cast<const float4*>(s.LF + j));
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
      if (c % G == lane) s.GF[i].g[c] = g[c];
  }
  ITEM_LOOP_END
}

// once per step, mixed form: FP32 SGS/properties/sensor, FP64 CFL sums and
// reductions (same structure as k_step_end)
template <int G, bool DIRECT>
__global__ void __launch_bounds__(256) k_step_end_f(CASE_ARGS, int mode) {
  constexpr int kCells = 256 / G;
  __shared__ double sh_cfl[kCells];
  __shared__ int sh_nan[kCells];
  __shared__ bool am_last;
  const int cl = threadIdx.x / G;
  ITEM_LOOP_BEGIN(G)
  const Phys& ph = CASE_PH;
  long long b = 0, e = 0, ec = 0;
  LRecF Li;
  float4 qi = make_float4(0.f, 0.f, 0.f, 0.f);
  if (valid) {
    b = m.off[i];
    e = m.off[i + 1];
    ec = b + __ldg(m.ncomp + i);
    load_LF(s.LF, i, Li);
    qi = __ldg(reinterpret_cast<const float4*>(s.QF + i));
  }
  float vv2 = 0.0f;
  double cfl = 0.0;
  for (long long k = b + lane; k < e; k += G) {
    const int j = __ldg(m.nbr + k);
    const float4 qj = __ldg(reinterpret_cast<const float4*>(s.QF + j));
    const float dp = qj.y - qi.y;
    const float v_avg = 0.5f * (qi.z + qj.z);
    const float beta = 0.5f * (qi.w + qj.w);
    const float gr = qj.x - qi.x - v_avg * dp * beta;
    vv2 = fmaxf(vv2, fabsf(gr));
    if (k < ec) {
      const int f = __ldg(m.fid + k);
      const float sg = (f < 0) ? -1.0f : 1.0f;
      const float4 h0 = __ldg(reinterpret_cast<const float4*>(m.cf32 + (f & kFidMask)));
      const float un[3] = {sg * h0.x, sg * h0.y, sg * h0.z};
      const float area = h0.w;
      LRecF Lj;
      load_LF(s.LF, j, Lj);
      const float undA = 0.5f * area * ((Li.u[0] * un[0] + Li.u[1] * un[1] + Li.u[2] * un[2]) +
                                        (Lj.u[0] * un[0] + Lj.u[1] * un[1] + Lj.u[2] * un[2]));
      cfl += double(fabsf(undA)) + double(area) * (0.5 * (double(Li.sos) + double(Lj.sos)));
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) vv2 = fmaxf(vv2, __shfl_xor_sync(0xffffffffu, vv2, o));
  cfl = group_sum<G>(cfl);
  int nan = 0;
  if (valid && lane == 0) {
    float g[9];
    load_GF(s.GF, i, g);
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
    float4* P = reinterpret_cast<float4*>(s.PF + i);
    P[0] = make_float4(mu_lam + mu_sgs, loc_lam + loc_sgs, a_sgs, fgr);
    P[1] = make_float4(symh, symp, 0.0f, 0.0f);
    nan = (rho != rho) || (p != p) || (T != T);
    cfl *= 0.5 * 1.0 * __ldg(m.inv_vol + i);
  }
  if (lane == 0) {
    sh_cfl[cl] = valid ? cfl : 0.0;
    sh_nan[cl] = valid ? nan : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    int an = 0;
    for (int c = 0; c < kCells; ++c) {
      mx = fmax(mx, sh_cfl[c]);
      an |= sh_nan[c];
    }
    const int np = CASE_NITEMS * G;
    const int part = it_.idx * G + sub_;
    s.red[part] = mx;
    s.red[np + part] = double(an);
    __threadfence();
    const unsigned int done = atomicAdd(&s.ctl->blocks_done, 1u);
    am_last = (done == unsigned(np) - 1u);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    finalize_ctl(s, ph, mode, CASE_NITEMS * G);
  }
  __syncthreads();
  ITEM_LOOP_END
}

#endif
