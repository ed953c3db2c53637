// cgx_ops.cu -- the reference solver's discrete operators built on the GPU
// from a compact periodic mesh (include/cgx_ops.h).
//
// Reference semantics (src/ paths relative to the reference), restated in the
// same operation order as the host generator (csrc/meshgen.cpp) so that both
// give the same bits; this file is compiled with -fmad=false for that reason:
//   buildCvocv                src/core/common/StaticSolver.cpp:6659-6726
//   calcCvGradCoeff           src/core/common/StaticSolver.cpp:5598-5765
//   EF_OPS DEFAULT operator   src/core/common/StripedMesh.hpp:6014-6130
//   transpose + ef assembly   src/core/common/StripedMesh.hpp:6589-6866
//   area_over_delta_fa        src/core/common/StaticSolver.cpp:4447-4459
//   cmag/dcmag_hat            src/charles/FlowSolver.hpp:702-760
//   sa_to_vol_ratio           src/charles/FlowSolver.hpp:859-878
//
// Layout of the work (one stream, every step deterministic):
//   1. local faces of each cell (faocv), ifa ascending; cvocv            thread/face, thread/cell
//   2. gradient coefficients (3x3 SVD pseudo-inverse per cell)           thread/cell
//   3. operator rows D(r, image): the row's distinct images collected in a
//      shared-memory hash set and bitonic-sorted by one warp; then the row's
//      terms, 32 at a time in the host's term order, are added to per-image
//      shared-memory accumulators in rounds that keep that order per image
//      (no floating-point atomics, so sums are order-exact)               warp/row
//   4. extended faces: n = D_ij - D_ji, c = D_ij + D_ji per canonical pair,
//      bucketed by the smaller cell, ordered by (cell, image); periodic
//      pairs split into one side per owner; level-2 ghosts numbered by
//      first use                                                          warp/row, thread/cell
//   5. area_over_delta, cmag, dcmag_hat, sa_to_vol                        thread/face, thread/cell
// Positions taken with atomics are always re-sorted by a unique key before
// anything is written out, so the result does not depend on scheduling.

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cgx.h"
#include "../../include/cgx_ops.h"
#include "host_staging.h"
#include "svd33.h"

namespace cgx {
void set_last_error(const std::string& s);
}

namespace {

typedef long long i64;

constexpr int kRowMax = 384;  // distinct entries of one operator row (the host generator's limit)
constexpr int kHash = 512;    // hash slots per row (power of two above kRowMax)
constexpr int kRowWarps = 4;  // rows (warps) per block of the row kernels
constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

enum { ERR_INPUT = 0, ERR_ROW = 1, ERR_THIN = 2, ERR_INTERNAL = 3, ERR_SLOTS = 4 };

__device__ __forceinline__ i64 img_key(int cell, int sx, int sy, int sz) {
  return i64(cell) * 343 + (sx + 3) * 49 + (sy + 3) * 7 + (sz + 3);
}
__device__ __forceinline__ void img_unkey(i64 k, int& cell, int& sx, int& sy, int& sz) {
  cell = int(k / 343);
  int r = int(k % 343);
  sx = r / 49 - 3;
  r %= 49;
  sy = r / 7 - 3;
  sz = r % 7 - 3;
}
__device__ __forceinline__ bool key_is_local(i64 k) { return k % 343 == 171; }  // shift (0,0,0)

struct Mesh {
  int ncv, ncv_g, nfa, nfa_i;
  double L0, L1, L2, f_int;
  const int* cvofa;
  const double* n_fa;
  const double* x_fa;
  const double* vol;
  const double* xcv;      // [ncv][3]
  const int* g_owner;     // level-1 ghosts
  const int* g_shift;
  const int* faocv_i;     // [ncv+1]
  const int* loc;         // local faces (compact face ids), ifa ascending per cell
  const int* cvocv_i;
  const int* cvocv_v;
  const double* gc;       // [ncoc][3]
  const int* bfocv_i;     // [ncv+1] boundary faces of each cell
  const int* bfocv_v;     // boundary face ids, ascending per cell
  const double* Gij;      // [nbf][3][3]
  int* err;
};

__device__ __forceinline__ void nbr_image(const Mesh& M, int idx, int& cell, int& sx, int& sy, int& sz) {
  if (idx < M.ncv) {
    cell = idx;
    sx = sy = sz = 0;
  } else {
    const int g = idx - M.ncv;
    cell = M.g_owner[g];
    sx = M.g_shift[3 * g];
    sy = M.g_shift[3 * g + 1];
    sz = M.g_shift[3 * g + 2];
  }
}

// A local face of cell a: outward normal, centroid in a's frame, neighbour.
struct LF {
  double n[3], xf[3];
  int nbr_idx, cell, sx, sy, sz;
};
__device__ __forceinline__ void local_face(const Mesh& M, int a, int foc, LF& f) {
  const int ifa = M.loc[foc];
  const int c0 = M.cvofa[2 * ifa], c1 = M.cvofa[2 * ifa + 1];
  const bool own = (c0 == a);
  f.nbr_idx = own ? c1 : c0;
  for (int d = 0; d < 3; ++d) {
    const double nv = M.n_fa[3 * size_t(ifa) + d];
    f.n[d] = own ? nv : -nv;
    f.xf[d] = M.x_fa[3 * size_t(ifa) + d];
  }
  nbr_image(M, f.nbr_idx, f.cell, f.sx, f.sy, f.sz);
}
__device__ __forceinline__ void image_pos(const Mesh& M, int cell, int sx, int sy, int sz, double x[3]) {
  x[0] = M.xcv[3 * size_t(cell)] + sx * M.L0;
  x[1] = M.xcv[3 * size_t(cell) + 1] + sy * M.L1;
  x[2] = M.xcv[3 * size_t(cell) + 2] + sz * M.L2;
}

// ---------------------------------------------------------------------------
// 1. local faces and cvocv
// ---------------------------------------------------------------------------
__global__ void k_check_ghosts(int ncv, int ng, const int* owner, const int* shift, int* err) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const int o = owner[g];
    bool bad = o < 0 || o >= ncv;
    for (int d = 0; d < 3; ++d) bad |= shift[3 * g + d] < -1 || shift[3 * g + d] > 1;
    bad |= shift[3 * g] == 0 && shift[3 * g + 1] == 0 && shift[3 * g + 2] == 0;
    if (bad) atomicExch(&err[ERR_INPUT], 1);
  }
}

__global__ void k_face_count(Mesh M, int* cnt) {
  for (int ifa = blockIdx.x * blockDim.x + threadIdx.x; ifa < M.nfa; ifa += gridDim.x * blockDim.x) {
    const int c0 = M.cvofa[2 * ifa], c1 = M.cvofa[2 * ifa + 1];
    if (c0 < 0 || c0 >= M.ncv) {
      atomicExch(&M.err[ERR_INPUT], 1);
      continue;
    }
    if (ifa < M.nfa_i) {
      if (c1 <= c0 || c1 >= M.ncv) {
        atomicExch(&M.err[ERR_INPUT], 1);
        continue;
      }
      atomicAdd(&cnt[c1], 1);
    } else {
      if (c1 < M.ncv || c1 >= M.ncv_g) {
        atomicExch(&M.err[ERR_INPUT], 1);
        continue;
      }
      if (M.g_owner[c1 - M.ncv] == c0) atomicExch(&M.err[ERR_THIN], 1);  // cell touches its own image
    }
    atomicAdd(&cnt[c0], 1);
  }
}

__global__ void k_face_fill(Mesh M, int* fill, int* loc) {
  for (int ifa = blockIdx.x * blockDim.x + threadIdx.x; ifa < M.nfa; ifa += gridDim.x * blockDim.x) {
    const int c0 = M.cvofa[2 * ifa], c1 = M.cvofa[2 * ifa + 1];
    loc[atomicAdd(&fill[c0], 1)] = ifa;
    if (ifa < M.nfa_i) loc[atomicAdd(&fill[c1], 1)] = ifa;
  }
}

// order each cell's faces by compact face id and write cvocv (diagonal first)
__global__ void k_cell_faces(Mesh M, int* loc, int* cvocv_i, int* cvocv_v) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < M.ncv; a += gridDim.x * blockDim.x) {
    const int b = M.faocv_i[a], e = M.faocv_i[a + 1];
    for (int i = b + 1; i < e; ++i) {
      const int v = loc[i];
      int j = i - 1;
      while (j >= b && loc[j] > v) {
        loc[j + 1] = loc[j];
        --j;
      }
      loc[j + 1] = v;
    }
    const int coc0 = b + a;
    cvocv_i[a] = coc0;
    if (a == M.ncv - 1) cvocv_i[M.ncv] = e + M.ncv;
    cvocv_v[coc0] = a;
    for (int foc = b; foc < e; ++foc) {
      const int ifa = loc[foc];
      const int c0 = M.cvofa[2 * ifa], c1 = M.cvofa[2 * ifa + 1];
      cvocv_v[coc0 + 1 + (foc - b)] = (c0 == a) ? c1 : c0;
    }
  }
}

// ---------------------------------------------------------------------------
// 2. gradient coefficients (StaticSolver.cpp:5598-5765)
// ---------------------------------------------------------------------------
__global__ void k_grad_coeff(Mesh M, double sigma_thresh, double* gc, int* n_threshold) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < M.ncv; a += gridDim.x * blockDim.x) {
    const int coc_f = M.cvocv_i[a];
    const int coc_l = M.cvocv_i[a + 1] - 1;
    double A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 3; ++i) A[i * 3 + i] = M.vol[a];
    // boundary faces first, as the reference loops them
    for (int boc = M.bfocv_i[a]; boc < M.bfocv_i[a + 1]; ++boc) {
      const double* G = M.Gij + 9 * size_t(M.bfocv_v[boc]);
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) A[j * 3 + i] += G[3 * i + j];
    }
    double g0[3] = {0.0, 0.0, 0.0};
    const double xc[3] = {M.xcv[3 * size_t(a)], M.xcv[3 * size_t(a) + 1], M.xcv[3 * size_t(a) + 2]};
    const int fb = M.faocv_i[a], fe = M.faocv_i[a + 1];
    for (int foc = fb; foc < fe; ++foc) {
      LF lf;
      local_face(M, a, foc, lf);
      const int coc = coc_f + foc - fb + 1;
      double xnb[3];
      image_pos(M, lf.cell, lf.sx, lf.sy, lf.sz, xnb);
      double r[3];
      for (int i = 0; i < 3; ++i) r[i] = lf.xf[i] - 0.5 * (xc[i] + xnb[i]);
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) A[j * 3 + i] -= r[j] * lf.n[i];
      for (int i = 0; i < 3; ++i) {
        gc[3 * size_t(coc) + i] = 0.0 + 0.5 * lf.n[i];
        g0[i] -= 0.5 * lf.n[i];
      }
    }
    for (int i = 0; i < 3; ++i) gc[3 * size_t(coc_f) + i] = g0[i];
    const double inv_vol = 1.0 / M.vol[a];
    for (int k = 0; k < 9; ++k) A[k] *= inv_vol;
    double U[9], V[9], sigma[3];
    svd33(A, U, V, sigma);
    double sigma_inv[3];
    bool thr = false;
    for (int i = 0; i < 3; ++i) {
      if (sigma[i] < sigma_thresh) {
        sigma_inv[i] = 0.0;
        thr = true;
      } else {
        sigma_inv[i] = 1.0 / sigma[i];
      }
    }
    if (thr) atomicAdd(n_threshold, 1);
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) V[j * 3 + i] *= sigma_inv[j];
    for (int coc = coc_f; coc <= coc_l; ++coc) {
      double g[3];
      for (int i = 0; i < 3; ++i) g[i] = gc[3 * size_t(coc) + i] * inv_vol;
      double b_tmp[3];
      for (int i = 0; i < 3; ++i) {
        b_tmp[i] = 0.0;
        for (int j = 0; j < 3; ++j) b_tmp[i] += A[j * 3 + i] * g[j];
      }
      double tmp[3];
      for (int i = 0; i < 3; ++i)
        tmp[i] = U[i * 3 + 0] * (g[0] - b_tmp[0]) + U[i * 3 + 1] * (g[1] - b_tmp[1]) +
                 U[i * 3 + 2] * (g[2] - b_tmp[2]);
      for (int i = 0; i < 3; ++i)
        gc[3 * size_t(coc) + i] = g[i] + (V[0 * 3 + i] * tmp[0] + V[1 * 3 + i] * tmp[1] + V[2 * 3 + i] * tmp[2]);
    }
  }
}

// ---------------------------------------------------------------------------
// 3. operator rows (StripedMesh.hpp:6014-6130)
// Row r of D gathers (i) the terms r adds for each of its compact faces and
// (ii) the terms each compact neighbour k adds to row r, with k's periodic
// shift moved onto the column.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned hash_slot(i64 k) {
  unsigned long long z = (unsigned long long)k + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return unsigned(z ^ (z >> 31)) & (kHash - 1);
}

// Insert key into the warp's set; true if it was new.
__device__ __forceinline__ bool set_insert(i64* hs, i64 key, bool& full) {
  unsigned h = hash_slot(key);
  for (int probe = 0; probe < kHash; ++probe) {
    const i64 prev = (i64)atomicCAS(reinterpret_cast<unsigned long long*>(&hs[h]),
                                    (unsigned long long)(-1LL), (unsigned long long)key);
    if (prev == -1) return true;
    if (prev == key) return false;
    h = (h + 1) & (kHash - 1);
  }
  full = true;
  return false;
}

// First local face of k (in face order) whose neighbour is image (r, -s);
// -1 if none.  Warp-uniform result.
__device__ __forceinline__ int back_face(const Mesh& M, int k, int r, int sx, int sy, int sz, int lane) {
  const int fb = M.faocv_i[k], fe = M.faocv_i[k + 1];
  for (int base = fb; base < fe; base += 32) {
    const int foc = base + lane;
    bool hit = false;
    if (foc < fe) {
      const int ifa = M.loc[foc];
      const int c0 = M.cvofa[2 * ifa], c1 = M.cvofa[2 * ifa + 1];
      int cell, qx, qy, qz;
      nbr_image(M, c0 == k ? c1 : c0, cell, qx, qy, qz);
      hit = cell == r && qx == -sx && qy == -sy && qz == -sz;
    }
    const unsigned b = __ballot_sync(kFull, hit);
    if (b) return base + __ffs(b) - 1;
  }
  return -1;
}

// The sorted distinct images of row r into sk[0..n); returns n, or -1 when
// the row is longer than kRowMax (err set).  Whole warp.
__device__ int row_images(const Mesh& M, int r, i64* hs, i64* sk, int lane) {
  for (int s = lane; s < kHash; s += 32) hs[s] = -1;
  __syncwarp();
  int n = 0;
  bool full = false, thin = false;
  const int fb = M.faocv_i[r], fe = M.faocv_i[r + 1];
  for (int foc = fb; foc < fe; ++foc) {
    LF lf;
    local_face(M, r, foc, lf);
    bool ins = false;
    if (lane == 0) ins = set_insert(hs, img_key(lf.cell, lf.sx, lf.sy, lf.sz), full);
    n += __popc(__ballot_sync(kFull, ins));
    if (back_face(M, lf.cell, r, lf.sx, lf.sy, lf.sz, lane) < 0) continue;
    const int cb = M.cvocv_i[lf.cell], ce = M.cvocv_i[lf.cell + 1];
    for (int base = cb; base < ce; base += 32) {
      const int coc = base + lane;
      bool ins2 = false;
      if (coc < ce) {
        int c2, s2x, s2y, s2z;
        nbr_image(M, M.cvocv_v[coc], c2, s2x, s2y, s2z);
        if (!(c2 == r && s2x == -lf.sx && s2y == -lf.sy && s2z == -lf.sz)) {
          thin |= (c2 == r);
          ins2 = set_insert(hs, img_key(c2, s2x + lf.sx, s2y + lf.sy, s2z + lf.sz), full);
        }
      }
      n += __popc(__ballot_sync(kFull, ins2));
    }
  }
  __syncwarp();
  if (__any_sync(kFull, thin) && lane == 0) atomicExch(&M.err[ERR_THIN], 1);
  if (__any_sync(kFull, full) || n > kRowMax) {
    if (lane == 0) atomicExch(&M.err[ERR_ROW], 1);
    return -1;
  }
  int base = 0;
  for (int t = 0; t < kHash; t += 32) {
    const i64 v = hs[t + lane];
    const bool occ = v != -1;
    const unsigned b = __ballot_sync(kFull, occ);
    if (occ) sk[base + __popc(b & ((1u << lane) - 1))] = v;
    base += __popc(b);
  }
  int P = 32;
  while (P < n) P <<= 1;
  for (int i = n + lane; i < P; i += 32) sk[i] = LLONG_MAX;
  __syncwarp();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const i64 x = sk[i], y = sk[ixj];
          const bool up = (i & k) == 0;
          if ((x > y) == up) {
            sk[i] = y;
            sk[ixj] = x;
          }
        }
      }
      __syncwarp();
    }
  }
  return n;
}

__global__ void __launch_bounds__(kRowWarps * 32) k_row_count(Mesh M, i64* rcnt) {
  extern __shared__ i64 smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  i64* hs = smem + size_t(w) * 2 * kHash;
  i64* sk = hs + kHash;
  for (int r = blockIdx.x * kRowWarps + w; r < M.ncv; r += gridDim.x * kRowWarps) {
    const int n = row_images(M, r, hs, sk, lane);
    if (lane == 0) rcnt[r] = n < 0 ? 0 : n;
    __syncwarp();
  }
}

// Row values, one lane per image: each lane walks the row's whole term list
// and adds the terms that hit its image.  Used for rows too long for the
// shared-memory accumulators of row_values_by_term.
__device__ void row_values_by_image(const Mesh& M, int r, const i64* sk, int n, double* dv, int lane) {
  const double f = M.f_int;
  const i64 self = img_key(r, 0, 0, 0);
  const double xr[3] = {M.xcv[3 * size_t(r)], M.xcv[3 * size_t(r) + 1], M.xcv[3 * size_t(r) + 2]};
  const int fb = M.faocv_i[r], fe = M.faocv_i[r + 1];
  const int rb = M.cvocv_i[r], re = M.cvocv_i[r + 1];
  for (int kb = 0; kb < n; kb += 32) {
    const int e = kb + lane;
    const i64 K = e < n ? sk[e] : -2;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int foc = fb; foc < fe; ++foc) {
      LF lf;
      local_face(M, r, foc, lf);
      // (i) own terms
      if (K == img_key(lf.cell, lf.sx, lf.sy, lf.sz)) {
        acc0 += 0.5 * lf.n[0];
        acc1 += 0.5 * lf.n[1];
        acc2 += 0.5 * lf.n[2];
      }
      double xk[3];
      image_pos(M, lf.cell, lf.sx, lf.sy, lf.sz, xk);
      double dx[3];
      for (int i = 0; i < 3; ++i) dx[i] = 0.5 * lf.xf[i] - (0.5 - 0.25 * f) * xr[i] - 0.25 * f * xk[i];
      for (int coc = rb; coc < re; ++coc) {
        int c2, s2x, s2y, s2z;
        nbr_image(M, M.cvocv_v[coc], c2, s2x, s2y, s2z);
        const i64 k2 = img_key(c2, s2x, s2y, s2z);
        if (k2 != self && K == k2) {
          const double* g = &M.gc[3 * size_t(coc)];
          const double dp = g[0] * dx[0] + g[1] * dx[1] + g[2] * dx[2];
          acc0 += dp * lf.n[0];
          acc1 += dp * lf.n[1];
          acc2 += dp * lf.n[2];
        }
      }
      // (ii) terms the neighbour k adds to row r
      const int k = lf.cell;
      const int bf = back_face(M, k, r, lf.sx, lf.sy, lf.sz, lane);
      if (bf < 0) continue;
      LF bk;
      local_face(M, k, bf, bk);
      const double xkk[3] = {M.xcv[3 * size_t(k)], M.xcv[3 * size_t(k) + 1], M.xcv[3 * size_t(k) + 2]};
      double xri[3];
      image_pos(M, r, -lf.sx, -lf.sy, -lf.sz, xri);
      double dxb[3];
      for (int i = 0; i < 3; ++i) dxb[i] = 0.5 * bk.xf[i] - (0.5 - 0.25 * f) * xkk[i] - 0.25 * f * xri[i];
      const int cb = M.cvocv_i[k], ce = M.cvocv_i[k + 1];
      for (int coc = cb; coc < ce; ++coc) {
        int c2, s2x, s2y, s2z;
        nbr_image(M, M.cvocv_v[coc], c2, s2x, s2y, s2z);
        if (c2 == r && s2x == -lf.sx && s2y == -lf.sy && s2z == -lf.sz) continue;
        if (K == img_key(c2, s2x + lf.sx, s2y + lf.sy, s2z + lf.sz)) {
          const double* g = &M.gc[3 * size_t(coc)];
          const double dp = g[0] * dxb[0] + g[1] * dxb[1] + g[2] * dxb[2];
          acc0 -= dp * bk.n[0];
          acc1 -= dp * bk.n[1];
          acc2 -= dp * bk.n[2];
        }
      }
    }
    if (e < n) {
      dv[3 * size_t(e)] = acc0;
      dv[3 * size_t(e) + 1] = acc1;
      dv[3 * size_t(e) + 2] = acc2;
    }
  }
}

// Add one chunk of up to 32 consecutive terms (lane order = term order) into
// the shared accumulators acc[3 * image].  Terms that hit the same image are
// added in rounds, lowest lane first, so each image receives its terms in
// term order, exactly as a sequential loop would add them.
__device__ __forceinline__ void add_terms(const Mesh& M, const i64* sk, int n, double* acc, bool active, i64 key,
                                          double v0, double v1, double v2, int lane) {
  int idx = -1;
  if (active) {
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (sk[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    if (lo < n && sk[lo] == key) idx = lo;
    else atomicExch(&M.err[ERR_INTERNAL], 1);
  }
  const unsigned grp = __match_any_sync(kFull, idx);
  const int rank = __popc(grp & ((1u << lane) - 1));
  const int rounds = __reduce_max_sync(kFull, idx >= 0 ? unsigned(__popc(grp)) : 0u);
  for (int t = 0; t < rounds; ++t) {
    if (idx >= 0 && rank == t) {
      acc[3 * idx] += v0;
      acc[3 * idx + 1] += v1;
      acc[3 * idx + 2] += v2;
    }
    __syncwarp();
  }
}

// Row values, lanes over terms: each chunk of 32 consecutive terms is
// evaluated in parallel and added by add_terms.  acc holds 3 * n doubles.
__device__ void row_values_by_term(const Mesh& M, int r, const i64* sk, int n, double* acc, int lane) {
  const double f = M.f_int;
  const i64 self = img_key(r, 0, 0, 0);
  for (int i = lane; i < 3 * n; i += 32) acc[i] = 0.0;
  __syncwarp();
  const double xr[3] = {M.xcv[3 * size_t(r)], M.xcv[3 * size_t(r) + 1], M.xcv[3 * size_t(r) + 2]};
  const int fb = M.faocv_i[r], fe = M.faocv_i[r + 1];
  const int rb = M.cvocv_i[r], re = M.cvocv_i[r + 1];
  for (int foc = fb; foc < fe; ++foc) {
    LF lf;
    local_face(M, r, foc, lf);
    // (i) own terms: the face's half normal, then the gradient correction
    add_terms(M, sk, n, acc, lane == 0, img_key(lf.cell, lf.sx, lf.sy, lf.sz), 0.5 * lf.n[0], 0.5 * lf.n[1],
              0.5 * lf.n[2], lane);
    double xk[3];
    image_pos(M, lf.cell, lf.sx, lf.sy, lf.sz, xk);
    double dx[3];
    for (int i = 0; i < 3; ++i) dx[i] = 0.5 * lf.xf[i] - (0.5 - 0.25 * f) * xr[i] - 0.25 * f * xk[i];
    for (int base = rb; base < re; base += 32) {
      const int coc = base + lane;
      bool act = coc < re;
      i64 k2 = -3;
      double dp = 0.0;
      if (act) {
        int c2, s2x, s2y, s2z;
        nbr_image(M, M.cvocv_v[coc], c2, s2x, s2y, s2z);
        k2 = img_key(c2, s2x, s2y, s2z);
        act = k2 != self;
        const double* g = &M.gc[3 * size_t(coc)];
        dp = g[0] * dx[0] + g[1] * dx[1] + g[2] * dx[2];
      }
      add_terms(M, sk, n, acc, act, k2, dp * lf.n[0], dp * lf.n[1], dp * lf.n[2], lane);
    }
    // (ii) terms the neighbour k adds to row r (subtracted: added negated)
    const int k = lf.cell;
    const int bf = back_face(M, k, r, lf.sx, lf.sy, lf.sz, lane);
    if (bf < 0) continue;
    LF bk;
    local_face(M, k, bf, bk);
    const double xkk[3] = {M.xcv[3 * size_t(k)], M.xcv[3 * size_t(k) + 1], M.xcv[3 * size_t(k) + 2]};
    double xri[3];
    image_pos(M, r, -lf.sx, -lf.sy, -lf.sz, xri);
    double dxb[3];
    for (int i = 0; i < 3; ++i) dxb[i] = 0.5 * bk.xf[i] - (0.5 - 0.25 * f) * xkk[i] - 0.25 * f * xri[i];
    const int cb = M.cvocv_i[k], ce = M.cvocv_i[k + 1];
    for (int base = cb; base < ce; base += 32) {
      const int coc = base + lane;
      bool act = coc < ce;
      i64 key = -3;
      double dp = 0.0;
      if (act) {
        int c2, s2x, s2y, s2z;
        nbr_image(M, M.cvocv_v[coc], c2, s2x, s2y, s2z);
        act = !(c2 == r && s2x == -lf.sx && s2y == -lf.sy && s2z == -lf.sz);
        key = img_key(c2, s2x + lf.sx, s2y + lf.sy, s2z + lf.sz);
        const double* g = &M.gc[3 * size_t(coc)];
        dp = g[0] * dxb[0] + g[1] * dxb[1] + g[2] * dxb[2];
      }
      add_terms(M, sk, n, acc, act, key, -(dp * bk.n[0]), -(dp * bk.n[1]), -(dp * bk.n[2]), lane);
    }
  }
}

__global__ void __launch_bounds__(kRowWarps * 32) k_row_fill(Mesh M, const i64* drow_i, i64* dkey, double* dval) {
  extern __shared__ i64 smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  i64* hs = smem + size_t(w) * 2 * kHash;
  i64* sk = hs + kHash;
  double* acc = reinterpret_cast<double*>(hs);  // the hash set is done with once sk is sorted
  for (int r = blockIdx.x * kRowWarps + w; r < M.ncv; r += gridDim.x * kRowWarps) {
    const int n = row_images(M, r, hs, sk, lane);
    if (n >= 0) {
      const i64 off = drow_i[r];
      for (int i = lane; i < n; i += 32) dkey[off + i] = sk[i];
      if (3 * n <= kHash) {
        row_values_by_term(M, r, sk, n, acc, lane);
        for (int i = lane; i < 3 * n; i += 32) dval[3 * size_t(off) + i] = acc[i];
      } else {
        row_values_by_image(M, r, sk, n, dval + 3 * size_t(off), lane);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// 4. extended faces (StripedMesh.hpp:6589-6866)
// canonical pair (a, b, s) with a < b: n = D(a,(b,s)) - D(b,(a,-s)),
//                                      c = D(a,(b,s)) + D(b,(a,-s)).
// ---------------------------------------------------------------------------
__device__ __forceinline__ i64 row_find(const i64* drow_i, const i64* dkey, int row, i64 key) {
  i64 lo = drow_i[row], hi = drow_i[row + 1];
  while (lo < hi) {
    const i64 mid = (lo + hi) >> 1;
    if (dkey[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return (lo < drow_i[row + 1] && dkey[lo] == key) ? lo : -1;
}

// pass 0 counts faces per bucket (smaller cell), pass 1 writes them
__global__ void k_ef_emit(int ncv, const i64* drow_i, const i64* dkey, const double* dval, int pass,
                          int* bcnt, const i64* boff, i64* fkey, double* fn, double* fc) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < ncv; r += gridDim.x * wpb) {
    for (i64 e = drow_i[r] + lane; e < drow_i[r + 1]; e += 32) {
      int j, sx, sy, sz;
      img_unkey(dkey[e], j, sx, sy, sz);
      if (j == r) continue;  // a cell's own image: the build fails (ERR_THIN)
      const i64 t = row_find(drow_i, dkey, j, img_key(r, -sx, -sy, -sz));
      int bucket;
      if (j > r) bucket = r;
      else if (t < 0) bucket = j;
      else continue;  // emitted from row j
      const int pos = atomicAdd(&bcnt[bucket], 1);
      if (pass == 0) continue;
      const i64 o = boff[bucket] + pos;
      const double* v = &dval[3 * size_t(e)];
      if (j > r) {
        fkey[o] = img_key(j, sx, sy, sz);
        for (int i = 0; i < 3; ++i) {
          const double dij = v[i], dji = t >= 0 ? dval[3 * size_t(t) + i] : 0.0;
          fn[3 * size_t(o) + i] = dij - dji;
          fc[3 * size_t(o) + i] = dij + dji;
        }
      } else {
        fkey[o] = img_key(r, -sx, -sy, -sz);
        for (int i = 0; i < 3; ++i) {
          fn[3 * size_t(o) + i] = 0.0 - v[i];
          fc[3 * size_t(o) + i] = v[i];
        }
      }
    }
  }
}

// Order each bucket by image key (keys are unique within a bucket); count
// its internal faces and the periodic sides of both owners.
__global__ void k_ef_bucket_sort(int ncv, const i64* boff, const i64* fkey, const double* fn, const double* fc,
                                 i64* skey, double* sn, double* sc, int* ni, int* np) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < ncv; a += gridDim.x * blockDim.x) {
    const i64 b = boff[a], e = boff[a + 1];
    int nint = 0;
    for (i64 p = b; p < e; ++p) {
      const i64 k = fkey[p];
      i64 rank = 0;
      for (i64 q = b; q < e; ++q) rank += fkey[q] < k;
      const i64 o = b + rank;
      skey[o] = k;
      for (int i = 0; i < 3; ++i) {
        sn[3 * size_t(o) + i] = fn[3 * size_t(p) + i];
        sc[3 * size_t(o) + i] = fc[3 * size_t(p) + i];
      }
      if (key_is_local(k)) {
        ++nint;
      } else {
        atomicAdd(&np[a], 1);
        atomicAdd(&np[int(k / 343)], 1);
      }
    }
    ni[a] = nint;
  }
}

// internal faces in (a, b) order; periodic sides to both owners (unordered)
__global__ void k_ef_split(int ncv, const i64* boff, const i64* skey, const double* sn, const double* sc,
                           const int* ioff, int* cvoef, double* n_ef, double* c_ef,
                           const i64* poff, int* pfill, i64* pkey, double* pn, double* pc) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < ncv; a += gridDim.x * blockDim.x) {
    int ii = ioff[a];
    for (i64 p = boff[a]; p < boff[a + 1]; ++p) {
      const i64 k = skey[p];
      int b, sx, sy, sz;
      img_unkey(k, b, sx, sy, sz);
      if (key_is_local(k)) {
        cvoef[2 * size_t(ii)] = a;
        cvoef[2 * size_t(ii) + 1] = b;
        for (int i = 0; i < 3; ++i) {
          n_ef[3 * size_t(ii) + i] = sn[3 * size_t(p) + i];
          c_ef[3 * size_t(ii) + i] = sc[3 * size_t(p) + i];
        }
        ++ii;
      } else {
        const i64 o0 = poff[a] + atomicAdd(&pfill[a], 1);
        pkey[o0] = k;
        for (int i = 0; i < 3; ++i) {
          pn[3 * size_t(o0) + i] = sn[3 * size_t(p) + i];
          pc[3 * size_t(o0) + i] = sc[3 * size_t(p) + i];
        }
        const i64 o1 = poff[b] + atomicAdd(&pfill[b], 1);
        pkey[o1] = img_key(a, -sx, -sy, -sz);
        for (int i = 0; i < 3; ++i) {
          pn[3 * size_t(o1) + i] = -sn[3 * size_t(p) + i];
          pc[3 * size_t(o1) + i] = sc[3 * size_t(p) + i];
        }
      }
    }
  }
}

// order each owner's periodic sides by image key; write cvoef[.][0], n, c
__global__ void k_ef_periodic_sort(int ncv, i64 nef_i, const i64* poff, const i64* pkey, const double* pn,
                                   const double* pc, i64* pkey_sorted, int* cvoef, double* n_ef, double* c_ef) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < ncv; a += gridDim.x * blockDim.x) {
    const i64 b = poff[a], e = poff[a + 1];
    for (i64 p = b; p < e; ++p) {
      const i64 k = pkey[p];
      i64 rank = 0;
      for (i64 q = b; q < e; ++q) rank += pkey[q] < k;
      const i64 o = b + rank;
      pkey_sorted[o] = k;
      const size_t ii = size_t(nef_i + o);
      cvoef[2 * ii] = a;
      for (int i = 0; i < 3; ++i) {
        n_ef[3 * ii + i] = pn[3 * size_t(p) + i];
        c_ef[3 * ii + i] = pc[3 * size_t(p) + i];
      }
    }
  }
}

// level-1 ghost keys (for lookup)
__global__ void k_ghost_keys(int ng, const int* owner, const int* shift, i64* gkey, int* gid) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    gkey[g] = img_key(owner[g], shift[3 * g], shift[3 * g + 1], shift[3 * g + 2]);
    gid[g] = g;
  }
}

// each periodic side: its level-1 ghost, or -1 when its image is not one
__global__ void k_ghost_lookup(i64 nper, const i64* pkey, int ng, const i64* gkey_sorted, const int* gid_sorted,
                               int ncv, int* gcomp, i64* seq) {
  for (i64 k = blockIdx.x * i64(blockDim.x) + threadIdx.x; k < nper; k += i64(gridDim.x) * blockDim.x) {
    const i64 key = pkey[k];
    int lo = 0, hi = ng;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (gkey_sorted[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    gcomp[k] = (lo < ng && gkey_sorted[lo] == key) ? ncv + gid_sorted[lo] : -1;
    seq[k] = k;
  }
}

// first use of each new image (sorted by key; equal keys keep side order)
__global__ void k_ghost_heads(i64 nper, const i64* skey, const i64* sval, const int* gcomp, int* isnew) {
  for (i64 p = blockIdx.x * i64(blockDim.x) + threadIdx.x; p < nper; p += i64(gridDim.x) * blockDim.x) {
    const bool head = p == 0 || skey[p] != skey[p - 1];
    if (head && gcomp[sval[p]] < 0) isnew[sval[p]] = 1;
  }
}

__global__ void k_ghost_assign(i64 nper, i64 nef_i, int ncv, int ncv_g, int ng1, const i64* skey, const i64* sval,
                               const int* gcomp, const int* newrank, int* cvoef, int* g_owner, int* g_shift) {
  for (i64 p = blockIdx.x * i64(blockDim.x) + threadIdx.x; p < nper; p += i64(gridDim.x) * blockDim.x) {
    const i64 k = sval[p];
    int id = gcomp[k];
    if (id < 0) {
      i64 h = p;
      while (h > 0 && skey[h - 1] == skey[p]) --h;
      const int r = newrank[sval[h]];
      id = ncv_g + r;
      if (h == p) {
        int b, sx, sy, sz;
        img_unkey(skey[p], b, sx, sy, sz);
        g_owner[ng1 + r] = b;
        g_shift[3 * size_t(ng1 + r)] = sx;
        g_shift[3 * size_t(ng1 + r) + 1] = sy;
        g_shift[3 * size_t(ng1 + r) + 2] = sz;
      }
    }
    cvoef[2 * size_t(nef_i + k) + 1] = id;
  }
}

__global__ void k_ghost_copy(int ng1, const int* owner, const int* shift, int* g_owner, int* g_shift) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng1; g += gridDim.x * blockDim.x) {
    g_owner[g] = owner[g];
    for (int d = 0; d < 3; ++d) g_shift[3 * g + d] = shift[3 * g + d];
  }
}

__global__ void k_x_cv(int ncv, int ncv_g2, double L0, double L1, double L2, const double* xcv,
                       const int* g_owner, const int* g_shift, double* x_cv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv_g2; i += gridDim.x * blockDim.x) {
    if (i < ncv) {
      for (int d = 0; d < 3; ++d) x_cv[3 * size_t(i) + d] = xcv[3 * size_t(i) + d];
    } else {
      const int g = i - ncv, b = g_owner[g];
      x_cv[3 * size_t(i)] = xcv[3 * size_t(b)] + g_shift[3 * g] * L0;
      x_cv[3 * size_t(i) + 1] = xcv[3 * size_t(b) + 1] + g_shift[3 * g + 1] * L1;
      x_cv[3 * size_t(i) + 2] = xcv[3 * size_t(b) + 2] + g_shift[3 * g + 2] * L2;
    }
  }
}

// ---------------------------------------------------------------------------
// 5. per-face and per-cell factors
// ---------------------------------------------------------------------------
__global__ void k_area_over_delta(int nfa, const int* cvofa, const double* n_fa, const double* x_cv, double* aod) {
  for (int ifa = blockIdx.x * blockDim.x + threadIdx.x; ifa < nfa; ifa += gridDim.x * blockDim.x) {
    const double* n = &n_fa[3 * size_t(ifa)];
    double v = 0.0;
    const double area2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    if (area2 > 0.0) {
      const int c0 = cvofa[2 * ifa], c1 = cvofa[2 * ifa + 1];
      const double dx[3] = {x_cv[3 * size_t(c1)] - x_cv[3 * size_t(c0)],
                            x_cv[3 * size_t(c1) + 1] - x_cv[3 * size_t(c0) + 1],
                            x_cv[3 * size_t(c1) + 2] - x_cv[3 * size_t(c0) + 2]};
      const double dp = dx[0] * n[0] + dx[1] * n[1] + dx[2] * n[2];
      if (dp > 0.0) v = area2 / dp;
    }
    aod[ifa] = v;
  }
}

__global__ void k_in_count(int nef_i, const int* cvoef, int* cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nef_i; i += gridDim.x * blockDim.x)
    atomicAdd(&cnt[cvoef[2 * size_t(i) + 1]], 1);
}
__global__ void k_in_fill(int nef_i, const int* cvoef, int* fill, int* inc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nef_i; i += gridDim.x * blockDim.x)
    inc[atomicAdd(&fill[cvoef[2 * size_t(i) + 1]], 1)] = i;
}

__device__ __forceinline__ double mag3(const double* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
__device__ __forceinline__ double dist3(const double* a, const double* b) {
  const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

// Sums in the host's order: internal faces by face index (the faces where the
// cell is second come from lower buckets, so first), then periodic sides.
__global__ void k_cell_factors(Mesh M, const int* inc_i, int* inc, const int* ioff, i64 nef_i, const i64* poff,
                               const int* cvoef, const double* c_ef, const double* x_cv,
                               double* cmag, double* dcmag, double* sav) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < M.ncv; a += gridDim.x * blockDim.x) {
    const int b = inc_i[a], e = inc_i[a + 1];
    for (int i = b + 1; i < e; ++i) {
      const int v = inc[i];
      int j = i - 1;
      while (j >= b && inc[j] > v) {
        inc[j + 1] = inc[j];
        --j;
      }
      inc[j + 1] = v;
    }
    double cm_sum = 0.0, dc = 0.0;
    auto add = [&](size_t ief) {
      const double cm = mag3(&c_ef[3 * ief]);
      const int c0 = cvoef[2 * ief], c1 = cvoef[2 * ief + 1];
      cm_sum += cm;
      dc += dist3(&x_cv[3 * size_t(c1)], &x_cv[3 * size_t(c0)]) * cm;
    };
    for (int i = b; i < e; ++i) add(size_t(inc[i]));
    for (int i = ioff[a]; i < ioff[a + 1]; ++i) add(size_t(i));
    for (i64 k = poff[a]; k < poff[a + 1]; ++k) add(size_t(nef_i + k));
    double area_sum = 0.0;
    for (int foc = M.faocv_i[a]; foc < M.faocv_i[a + 1]; ++foc) area_sum += mag3(&M.n_fa[3 * size_t(M.loc[foc])]);
    cmag[a] = cm_sum;
    dcmag[a] = dc / area_sum;
    sav[a] = area_sum / M.vol[a];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Failure {
  int code;
  std::string what;
};

void ck(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    throw Failure{CGX_E_OOM, std::string("cgx_operators_build: device allocation failed (") + what + ")"};
  }
  if (e != cudaSuccess) throw Failure{CGX_E_CUDA, std::string("cgx_operators_build: ") + what + ": " + cudaGetErrorString(e)};
}

// device allocations released together
struct Pool {
  std::vector<void*> ptrs;
  template <class T>
  T* get(size_t n, const char* what) {
    void* p = nullptr;
    ck(cudaMalloc(&p, sizeof(T) * (n ? n : 1)), what);
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  void release(void* p) {
    for (auto& q : ptrs)
      if (q == p) {
        cudaFree(q);
        q = nullptr;
      }
  }
  ~Pool() {
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};


// staged copies (csrc/host_staging.h) with this file's error handling
struct Staging {
  cgx_staging::Staging st;
  explicit Staging(cudaStream_t s) : st(s) { ck(st.init(), "pinned staging buffers"); }
  void put(void* dst, const void* src, size_t bytes, const char* what) { ck(st.put(dst, src, bytes), what); }
  void get(void* dst, const void* src, size_t bytes, const char* what) { ck(st.get(dst, src, bytes), what); }
};

template <class T>
T* upload(Pool& P, Staging& st, const T* h, size_t n, const char* what) {
  T* d = P.get<T>(n, what);
  st.put(d, h, sizeof(T) * n, what);
  return d;
}

template <class T>
T* download(Staging& st, const T* d, size_t n, const char* what) {
  T* h = static_cast<T*>(std::malloc(sizeof(T) * (n ? n : 1)));
  if (!h) throw std::bad_alloc();
  st.get(h, d, sizeof(T) * n, what);
  return h;
}

template <class T>
T* host_copy(const T* src, size_t n) {
  T* h = static_cast<T*>(std::malloc(sizeof(T) * (n ? n : 1)));
  if (!h) throw std::bad_alloc();
  cgx_staging::par_memcpy(h, src, sizeof(T) * n);
  return h;
}

// exclusive scan of cnt[0..n] into off[0..n]: off[n] is the total when
// cnt[n] == 0.  Accumulates in the output type.
template <class Tin, class Tout>
void excl_scan(Pool& P, const Tin* cnt, Tout* off, size_t n, cudaStream_t s) {
  size_t bytes = 0;
  ck(cub::DeviceScan::ExclusiveScan(nullptr, bytes, cnt, off, cuda::std::plus<Tout>{}, Tout(0), int64_t(n + 1), s),
     "scan size");
  void* tmp = P.get<char>(bytes, "scan temp");
  ck(cub::DeviceScan::ExclusiveScan(tmp, bytes, cnt, off, cuda::std::plus<Tout>{}, Tout(0), int64_t(n + 1), s),
     "scan");
  P.release(tmp);
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return int(b);
}

template <class T>
T read_scalar(const T* d, cudaStream_t s) {
  T v;
  ck(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, s), "read count");
  ck(cudaStreamSynchronize(s), "sync");
  return v;
}

void check_err(const int* d_err, cudaStream_t s) {
  int e[ERR_SLOTS];
  ck(cudaMemcpyAsync(e, d_err, sizeof(e), cudaMemcpyDeviceToHost, s), "read flags");
  ck(cudaStreamSynchronize(s), "sync");
  if (e[ERR_INPUT]) throw Failure{CGX_E_ARG, "cgx_operators_build: inconsistent compact mesh (cell or ghost index out of range)"};
  if (e[ERR_THIN]) throw Failure{CGX_E_ARG, "cgx_operators_build: box too thin (extended stencil reaches a cell's own image)"};
  if (e[ERR_ROW]) throw Failure{CGX_E_ARG, "cgx_operators_build: operator row longer than 384 entries"};
  if (e[ERR_INTERNAL]) throw Failure{CGX_E_CUDA, "cgx_operators_build: internal error (operator term without an image)"};
}

int build(const cgx_compact_desc* in, double f_int, double sigma_thresh, int device, cgx_meshgen_out** out,
          float* device_ms) {
  const int ncv = in->ncv, ncv_g = in->ncv_g, nfa = in->nfa, nfa_i = in->nfa_i;
  const int ng1 = ncv_g - ncv;
  ck(cudaSetDevice(device), "cudaSetDevice");
  cudaStream_t s;
  ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  cudaEvent_t ev0, ev1;
  ck(cudaEventCreate(&ev0), "event");
  ck(cudaEventCreate(&ev1), "event");
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } eg{ev0, ev1};
  Pool P;
  Staging st(s);

  Mesh M;
  M.ncv = ncv;
  M.ncv_g = ncv_g;
  M.nfa = nfa;
  M.nfa_i = nfa_i;
  M.L0 = in->L[0];
  M.L1 = in->L[1];
  M.L2 = in->L[2];
  M.f_int = f_int;
  M.cvofa = upload(P, st, in->cvofa, 2 * size_t(nfa), "cvofa");
  M.n_fa = upload(P, st, in->n_fa, 3 * size_t(nfa), "n_fa");
  M.x_fa = upload(P, st, in->x_fa, 3 * size_t(nfa), "x_fa");
  M.vol = upload(P, st, in->vol_cv, size_t(ncv), "vol_cv");
  M.xcv = upload(P, st, in->x_cv, 3 * size_t(ncv), "x_cv");
  M.g_owner = upload(P, st, in->icv_owner_g, size_t(ng1), "icv_owner_g");
  M.g_shift = upload(P, st, in->shift_g, 3 * size_t(ng1), "shift_g");
  {
    // boundary faces per cell (host counting sort, stable in face index)
    const int nbf = in->nbf;
    std::vector<int> bi(size_t(ncv) + 1, 0), bv(size_t(std::max(nbf, 1)), 0);
    for (int f = 0; f < nbf; ++f) {
      const int c = in->cvobf[f];
      if (c < 0 || c >= ncv) throw Failure{CGX_E_ARG, "cgx_operators_build: cvobf out of range"};
      ++bi[size_t(c) + 1];
    }
    for (int a = 0; a < ncv; ++a) bi[size_t(a) + 1] += bi[size_t(a)];
    std::vector<int> fill(bi.begin(), bi.end() - 1);
    for (int f = 0; f < nbf; ++f) bv[size_t(fill[size_t(in->cvobf[f])]++)] = f;
    M.bfocv_i = upload(P, st, bi.data(), size_t(ncv) + 1, "bfocv_i");
    M.bfocv_v = upload(P, st, bv.data(), bv.size(), "bfocv_v");
    static const double kNoG[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    M.Gij = upload(P, st, nbf > 0 ? in->Gij_bf : kNoG, nbf > 0 ? 9 * size_t(nbf) : size_t(9), "Gij_bf");
  }
  int* d_err = P.get<int>(ERR_SLOTS, "flags");
  ck(cudaMemsetAsync(d_err, 0, sizeof(int) * ERR_SLOTS, s), "memset");
  M.err = d_err;
  ck(cudaEventRecord(ev0, s), "event");

  // 1. local faces, cvocv
  int* cnt = P.get<int>(size_t(ncv) + 1, "face counts");
  ck(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  k_check_ghosts<<<grid_for(ng1, kThreads), kThreads, 0, s>>>(ncv, ng1, M.g_owner, M.g_shift, d_err);
  k_face_count<<<grid_for(nfa, kThreads), kThreads, 0, s>>>(M, cnt);
  ck(cudaGetLastError(), "k_face_count");
  check_err(d_err, s);
  int* faocv_i = P.get<int>(size_t(ncv) + 1, "faocv_i");
  excl_scan(P, cnt, faocv_i, ncv, s);
  const int nloc = read_scalar(faocv_i + ncv, s);
  int* loc = P.get<int>(size_t(nloc), "local faces");
  ck(cudaMemcpyAsync(cnt, faocv_i, sizeof(int) * ncv, cudaMemcpyDeviceToDevice, s), "copy");
  k_face_fill<<<grid_for(nfa, kThreads), kThreads, 0, s>>>(M, cnt, loc);
  M.faocv_i = faocv_i;
  M.loc = loc;
  const size_t ncoc = size_t(nloc) + ncv;
  int* cvocv_i = P.get<int>(size_t(ncv) + 1, "cvocv_i");
  int* cvocv_v = P.get<int>(ncoc, "cvocv_v");
  k_cell_faces<<<grid_for(ncv, kThreads), kThreads, 0, s>>>(M, loc, cvocv_i, cvocv_v);
  M.cvocv_i = cvocv_i;
  M.cvocv_v = cvocv_v;

  // 2. gradient coefficients
  double* gc = P.get<double>(3 * ncoc, "grad coeff");
  int* d_nthr = P.get<int>(1, "n_threshold");
  ck(cudaMemsetAsync(d_nthr, 0, sizeof(int), s), "memset");
  k_grad_coeff<<<grid_for(ncv, 128), 128, 0, s>>>(M, sigma_thresh, gc, d_nthr);
  ck(cudaGetLastError(), "k_grad_coeff");
  M.gc = gc;

  // 3. operator rows
  const size_t row_smem = size_t(kRowWarps) * 2 * kHash * sizeof(i64);
  ck(cudaFuncSetAttribute(k_row_count, cudaFuncAttributeMaxDynamicSharedMemorySize, int(row_smem)), "smem attr");
  ck(cudaFuncSetAttribute(k_row_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, int(row_smem)), "smem attr");
  const int row_grid = grid_for(size_t(ncv), kRowWarps);
  i64* rcnt = P.get<i64>(size_t(ncv) + 1, "row counts");
  ck(cudaMemsetAsync(rcnt, 0, sizeof(i64) * (size_t(ncv) + 1), s), "memset");
  k_row_count<<<row_grid, kRowWarps * 32, row_smem, s>>>(M, rcnt);
  ck(cudaGetLastError(), "k_row_count");
  check_err(d_err, s);
  i64* drow_i = P.get<i64>(size_t(ncv) + 1, "drow_i");
  excl_scan(P, rcnt, drow_i, ncv, s);
  P.release(rcnt);
  const i64 nnz = read_scalar(drow_i + ncv, s);
  i64* dkey = P.get<i64>(size_t(nnz), "D keys");
  double* dval = P.get<double>(3 * size_t(nnz), "D values");
  k_row_fill<<<row_grid, kRowWarps * 32, row_smem, s>>>(M, drow_i, dkey, dval);
  ck(cudaGetLastError(), "k_row_fill");

  // 4. extended faces
  int* bcnt = P.get<int>(size_t(ncv) + 1, "bucket counts");
  ck(cudaMemsetAsync(bcnt, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  const int emit_grid = grid_for(size_t(ncv), 8);
  k_ef_emit<<<emit_grid, 256, 0, s>>>(ncv, drow_i, dkey, dval, 0, bcnt, nullptr, nullptr, nullptr, nullptr);
  ck(cudaGetLastError(), "k_ef_emit");
  i64* boff = P.get<i64>(size_t(ncv) + 1, "bucket offsets");
  excl_scan(P, bcnt, boff, ncv, s);
  const i64 nfaces = read_scalar(boff + ncv, s);
  i64* fkey = P.get<i64>(size_t(nfaces), "face keys");
  double* fn = P.get<double>(3 * size_t(nfaces), "face n");
  double* fc = P.get<double>(3 * size_t(nfaces), "face c");
  ck(cudaMemsetAsync(bcnt, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  k_ef_emit<<<emit_grid, 256, 0, s>>>(ncv, drow_i, dkey, dval, 1, bcnt, boff, fkey, fn, fc);
  ck(cudaGetLastError(), "k_ef_emit");
  P.release(dkey);
  P.release(dval);
  i64* skey = P.get<i64>(size_t(nfaces), "sorted face keys");
  double* sn = P.get<double>(3 * size_t(nfaces), "sorted n");
  double* sc = P.get<double>(3 * size_t(nfaces), "sorted c");
  int* ni = P.get<int>(size_t(ncv) + 1, "internal counts");
  int* np = P.get<int>(size_t(ncv) + 1, "periodic counts");
  ck(cudaMemsetAsync(ni, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  ck(cudaMemsetAsync(np, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  k_ef_bucket_sort<<<grid_for(ncv, 128), 128, 0, s>>>(ncv, boff, fkey, fn, fc, skey, sn, sc, ni, np);
  ck(cudaGetLastError(), "k_ef_bucket_sort");
  P.release(fkey);
  P.release(fn);
  P.release(fc);
  i64* ioff64 = P.get<i64>(size_t(ncv) + 1, "internal offsets");
  excl_scan(P, ni, ioff64, ncv, s);
  i64* poff = P.get<i64>(size_t(ncv) + 1, "periodic offsets");
  excl_scan(P, np, poff, ncv, s);
  const i64 nef_i64 = read_scalar(ioff64 + ncv, s);
  const i64 nper = read_scalar(poff + ncv, s);
  if (nef_i64 + nper > i64(INT_MAX)) throw Failure{CGX_E_ARG, "cgx_operators_build: too many extended faces"};
  const int nef_i = int(nef_i64), nef = int(nef_i64 + nper);
  int* ioff = P.get<int>(size_t(ncv) + 1, "internal offsets (int)");
  excl_scan(P, ni, ioff, ncv, s);
  P.release(ioff64);
  int* cvoef = P.get<int>(2 * size_t(nef), "cvoef");
  double* n_ef = P.get<double>(3 * size_t(nef), "n_ef");
  double* c_ef = P.get<double>(3 * size_t(nef), "c_ef");
  int* pfill = np;  // reused as fill counters
  ck(cudaMemsetAsync(pfill, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  i64* pkey = P.get<i64>(size_t(nper), "periodic keys");
  double* pn = P.get<double>(3 * size_t(nper), "periodic n");
  double* pc = P.get<double>(3 * size_t(nper), "periodic c");
  k_ef_split<<<grid_for(ncv, 128), 128, 0, s>>>(ncv, boff, skey, sn, sc, ioff, cvoef, n_ef, c_ef, poff, pfill,
                                                pkey, pn, pc);
  ck(cudaGetLastError(), "k_ef_split");
  P.release(skey);
  P.release(sn);
  P.release(sc);
  i64* pkey_sorted = P.get<i64>(size_t(nper), "periodic keys sorted");
  k_ef_periodic_sort<<<grid_for(ncv, 128), 128, 0, s>>>(ncv, nef_i64, poff, pkey, pn, pc, pkey_sorted, cvoef, n_ef,
                                                        c_ef);
  ck(cudaGetLastError(), "k_ef_periodic_sort");
  P.release(pkey);
  P.release(pn);
  P.release(pc);

  // level-2 ghosts: images of periodic sides that are not level-1 ghosts,
  // numbered in order of first use over the sides
  i64* gkey = P.get<i64>(size_t(ng1), "ghost keys");
  int* gid = P.get<int>(size_t(ng1), "ghost ids");
  i64* gkey_s = P.get<i64>(size_t(ng1), "ghost keys sorted");
  int* gid_s = P.get<int>(size_t(ng1), "ghost ids sorted");
  k_ghost_keys<<<grid_for(ng1, kThreads), kThreads, 0, s>>>(ng1, M.g_owner, M.g_shift, gkey, gid);
  {
    size_t bytes = 0;
    ck(cub::DeviceRadixSort::SortPairs(nullptr, bytes, gkey, gkey_s, gid, gid_s, ng1, 0, 64, s), "sort size");
    void* tmp = P.get<char>(bytes, "sort temp");
    ck(cub::DeviceRadixSort::SortPairs(tmp, bytes, gkey, gkey_s, gid, gid_s, ng1, 0, 64, s), "sort");
    P.release(tmp);
  }
  int* gcomp = P.get<int>(size_t(nper), "side ghosts");
  i64* seq = P.get<i64>(size_t(nper), "side order");
  k_ghost_lookup<<<grid_for(nper, kThreads), kThreads, 0, s>>>(nper, pkey_sorted, ng1, gkey_s, gid_s, ncv, gcomp,
                                                              seq);
  i64* skey2 = P.get<i64>(size_t(nper), "side keys sorted");
  i64* sval2 = P.get<i64>(size_t(nper), "side order sorted");
  {
    size_t bytes = 0;
    ck(cub::DeviceRadixSort::SortPairs(nullptr, bytes, pkey_sorted, skey2, seq, sval2, nper, 0, 64, s),
       "sort size");
    void* tmp = P.get<char>(bytes, "sort temp");
    ck(cub::DeviceRadixSort::SortPairs(tmp, bytes, pkey_sorted, skey2, seq, sval2, nper, 0, 64, s), "sort");
    P.release(tmp);
  }
  int* isnew = P.get<int>(size_t(nper) + 1, "new ghost flags");
  ck(cudaMemsetAsync(isnew, 0, sizeof(int) * (size_t(nper) + 1), s), "memset");
  k_ghost_heads<<<grid_for(nper, kThreads), kThreads, 0, s>>>(nper, skey2, sval2, gcomp, isnew);
  int* newrank = P.get<int>(size_t(nper) + 1, "new ghost ranks");
  excl_scan(P, isnew, newrank, size_t(nper), s);
  const int ng2 = read_scalar(newrank + nper, s);
  const int ncv_g2 = ncv_g + ng2;
  int* g_owner = P.get<int>(size_t(ncv_g2 - ncv), "ghost owners");
  int* g_shift = P.get<int>(3 * size_t(ncv_g2 - ncv), "ghost shifts");
  k_ghost_copy<<<grid_for(ng1, kThreads), kThreads, 0, s>>>(ng1, M.g_owner, M.g_shift, g_owner, g_shift);
  k_ghost_assign<<<grid_for(nper, kThreads), kThreads, 0, s>>>(nper, nef_i64, ncv, ncv_g, ng1, skey2, sval2, gcomp,
                                                              newrank, cvoef, g_owner, g_shift);
  ck(cudaGetLastError(), "k_ghost_assign");
  double* x_cv = P.get<double>(3 * size_t(ncv_g2), "x_cv");
  k_x_cv<<<grid_for(ncv_g2, kThreads), kThreads, 0, s>>>(ncv, ncv_g2, M.L0, M.L1, M.L2, M.xcv, g_owner, g_shift,
                                                         x_cv);

  // 5. factors
  double* aod = P.get<double>(size_t(nfa), "area_over_delta_fa");
  k_area_over_delta<<<grid_for(nfa, kThreads), kThreads, 0, s>>>(nfa, M.cvofa, M.n_fa, x_cv, aod);
  int* icnt = P.get<int>(size_t(ncv) + 1, "incoming counts");
  ck(cudaMemsetAsync(icnt, 0, sizeof(int) * (size_t(ncv) + 1), s), "memset");
  k_in_count<<<grid_for(nef_i, kThreads), kThreads, 0, s>>>(nef_i, cvoef, icnt);
  int* inc_i = P.get<int>(size_t(ncv) + 1, "incoming offsets");
  excl_scan(P, icnt, inc_i, ncv, s);
  int* inc = P.get<int>(size_t(nef_i), "incoming faces");
  ck(cudaMemcpyAsync(icnt, inc_i, sizeof(int) * ncv, cudaMemcpyDeviceToDevice, s), "copy");
  k_in_fill<<<grid_for(nef_i, kThreads), kThreads, 0, s>>>(nef_i, cvoef, icnt, inc);
  double* cmag = P.get<double>(size_t(ncv), "cmag");
  double* dcmag = P.get<double>(size_t(ncv), "dcmag_hat");
  double* sav = P.get<double>(size_t(ncv), "sa_to_vol");
  k_cell_factors<<<grid_for(ncv, 128), 128, 0, s>>>(M, inc_i, inc, ioff, nef_i64, poff, cvoef, c_ef, x_cv, cmag,
                                                    dcmag, sav);
  ck(cudaGetLastError(), "k_cell_factors");
  ck(cudaEventRecord(ev1, s), "event");
  check_err(d_err, s);

  // download into the generator's layout
  cgx_meshgen_out* m = static_cast<cgx_meshgen_out*>(std::calloc(1, sizeof(cgx_meshgen_out)));
  if (!m) throw std::bad_alloc();
  struct OutGuard {
    cgx_meshgen_out* m;
    ~OutGuard() {
      if (m) cgx_operators_free(m);
    }
  } og{m};
  m->ncv = ncv;
  m->ncv_g = ncv_g;
  m->ncv_g2 = ncv_g2;
  m->nfa = nfa;
  m->nfa_i = nfa_i;
  m->nef = nef;
  m->nef_i = nef_i;
  m->n_threshold = read_scalar(d_nthr, s);
  m->h = in->h;
  m->cvofa = reinterpret_cast<int(*)[2]>(host_copy(in->cvofa, 2 * size_t(nfa)));
  m->n_fa = reinterpret_cast<double(*)[3]>(host_copy(in->n_fa, 3 * size_t(nfa)));
  m->x_fa = reinterpret_cast<double(*)[3]>(host_copy(in->x_fa, 3 * size_t(nfa)));
  m->vol_cv = host_copy(in->vol_cv, size_t(ncv));
  if (in->x_vv) m->x_vv = reinterpret_cast<double(*)[3]>(host_copy(in->x_vv, 3 * size_t(ncv)));
  m->area_over_delta_fa = download(st, aod, size_t(nfa), "aod");
  m->x_cv = reinterpret_cast<double(*)[3]>(download(st, x_cv, 3 * size_t(ncv_g2), "x_cv"));
  m->cvocv_i = download(st, cvocv_i, size_t(ncv) + 1, "cvocv_i");
  m->cvocv_v = download(st, cvocv_v, ncoc, "cvocv_v");
  m->cvocv_grad_coeff = reinterpret_cast<double(*)[3]>(download(st, gc, 3 * ncoc, "grad coeff"));
  m->cvoef = reinterpret_cast<int(*)[2]>(download(st, cvoef, 2 * size_t(nef), "cvoef"));
  m->n_ef = reinterpret_cast<double(*)[3]>(download(st, n_ef, 3 * size_t(nef), "n_ef"));
  m->c_ef = reinterpret_cast<double(*)[3]>(download(st, c_ef, 3 * size_t(nef), "c_ef"));
  m->cmag_cv = download(st, cmag, size_t(ncv), "cmag");
  m->dcmag_hat_cv = download(st, dcmag, size_t(ncv), "dcmag_hat");
  m->sa_to_vol_ratio = download(st, sav, size_t(ncv), "sa_to_vol");
  m->icv_owner_g = download(st, g_owner, size_t(ncv_g2 - ncv), "icv_owner_g");
  m->shift_g = reinterpret_cast<int(*)[3]>(download(st, g_shift, 3 * size_t(ncv_g2 - ncv), "shift_g"));
  m->nbf = in->nbf;
  m->nbf_zones = in->nbf_zones;
  if (in->nbf > 0) {
    const size_t nb = size_t(in->nbf);
    m->cvobf = host_copy(in->cvobf, nb);
    if (in->zone_bf) m->zone_bf = host_copy(in->zone_bf, nb);
    if (in->n_bf) m->n_bf = reinterpret_cast<double(*)[3]>(host_copy(in->n_bf, 3 * nb));
    if (in->x_bf) m->x_bf = reinterpret_cast<double(*)[3]>(host_copy(in->x_bf, 3 * nb));
    if (in->area_bf) m->area_bf = host_copy(in->area_bf, nb);
    if (in->area_over_delta_bf) m->area_over_delta_bf = host_copy(in->area_over_delta_bf, nb);
    m->Gij_bf = reinterpret_cast<double(*)[3][3]>(host_copy(in->Gij_bf, 9 * nb));
  }
  ck(cudaStreamSynchronize(s), "download");
  if (device_ms) ck(cudaEventElapsedTime(device_ms, ev0, ev1), "elapsed");
  *out = m;
  og.m = nullptr;
  return CGX_OK;
}

}  // namespace

extern "C" void cgx_operators_free(cgx_meshgen_out* m) {
  if (!m) return;
  std::free(m->cvofa);
  std::free(m->n_fa);
  std::free(m->x_fa);
  std::free(m->area_over_delta_fa);
  std::free(m->vol_cv);
  std::free(m->x_cv);
  std::free(m->x_vv);
  std::free(m->cvocv_i);
  std::free(m->cvocv_v);
  std::free(m->cvocv_grad_coeff);
  std::free(m->cvoef);
  std::free(m->n_ef);
  std::free(m->c_ef);
  std::free(m->cmag_cv);
  std::free(m->dcmag_hat_cv);
  std::free(m->sa_to_vol_ratio);
  std::free(m->icv_owner_g);
  std::free(m->shift_g);
  std::free(m->cvobf);
  std::free(m->zone_bf);
  std::free(m->n_bf);
  std::free(m->x_bf);
  std::free(m->area_bf);
  std::free(m->area_over_delta_bf);
  std::free(m->Gij_bf);
  std::free(m);
}

extern "C" int cgx_operators_build(const cgx_compact_desc* in, double interp_factor, double sigma_thresh,
                                   int device, cgx_meshgen_out** out, float* device_ms) {
  if (!out) {
    cgx::set_last_error("cgx_operators_build: out is NULL");
    return CGX_E_ARG;
  }
  *out = nullptr;
  if (!in || in->ncv < 1 || in->ncv_g < in->ncv || in->nfa < 0 || in->nfa_i < 0 || in->nfa_i > in->nfa ||
      !in->cvofa || !in->n_fa || !in->x_fa || !in->vol_cv || !in->x_cv ||
      (in->ncv_g > in->ncv && (!in->icv_owner_g || !in->shift_g)) || !(in->L[0] > 0) || !(in->L[1] > 0) ||
      !(in->L[2] > 0) || !(interp_factor >= 0.0) || !(sigma_thresh >= 0.0) || in->nbf < 0 ||
      (in->nbf > 0 && (!in->cvobf || !in->Gij_bf))) {
    cgx::set_last_error("cgx_operators_build: invalid argument");
    return CGX_E_ARG;
  }
  try {
    return build(in, interp_factor, sigma_thresh, device, out, device_ms);
  } catch (const Failure& f) {
    cgx::set_last_error(f.what);
    return f.code;
  } catch (const std::bad_alloc&) {
    cgx::set_last_error("cgx_operators_build: out of host memory");
    return CGX_E_OOM;
  }
}
