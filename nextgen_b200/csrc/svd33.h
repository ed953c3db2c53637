// svd33.h -- one-sided Jacobi SVD of a 3x3 matrix (Hestenes' method), shared
// by the host operator build (meshgen.cpp) and the device one (cgx_ops.cu) so
// that both evaluate the same operations in the same order.  The device file
// is compiled without multiply-add contraction, like the host's SSE2 code, so
// the two give the same bits.
//
// A is column major, A[j*3+i] = A(i,j), as in the reference's calcSvd33
// calling convention (src/core/common/SvdNew.hpp).  On return U (column major,
// columns = left singular vectors for nonzero sigma), V (column major),
// sigma >= 0 (unsorted).
#ifndef CGX_SVD33_H
#define CGX_SVD33_H

#include <math.h>

#ifdef __CUDACC__
#define CGX_HD __host__ __device__
#else
#define CGX_HD
#endif

CGX_HD inline void svd33(const double* A, double* U, double* V, double* sigma) {
  double W[9];
  for (int k = 0; k < 9; ++k) W[k] = A[k];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) V[j * 3 + i] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 2; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        double alpha = 0, beta = 0, gamma = 0;
        for (int k = 0; k < 3; ++k) {
          alpha += W[p * 3 + k] * W[p * 3 + k];
          beta += W[q * 3 + k] * W[q * 3 + k];
          gamma += W[p * 3 + k] * W[q * 3 + k];
        }
        if (alpha == 0.0 || beta == 0.0) continue;
        const double rel = fabs(gamma) / sqrt(alpha * beta);
        off = (off < rel) ? rel : off;
        if (rel < 1e-15) continue;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int k = 0; k < 3; ++k) {
          const double wp = W[p * 3 + k], wq = W[q * 3 + k];
          W[p * 3 + k] = c * wp - s * wq;
          W[q * 3 + k] = s * wp + c * wq;
          const double vp = V[p * 3 + k], vq = V[q * 3 + k];
          V[p * 3 + k] = c * vp - s * vq;
          V[q * 3 + k] = s * vp + c * vq;
        }
      }
    }
    if (off < 1e-15) break;
  }
  for (int j = 0; j < 3; ++j) {
    double nrm = 0;
    for (int k = 0; k < 3; ++k) nrm += W[j * 3 + k] * W[j * 3 + k];
    nrm = sqrt(nrm);
    sigma[j] = nrm;
    for (int k = 0; k < 3; ++k) U[j * 3 + k] = (nrm > 0) ? W[j * 3 + k] / nrm : 0.0;
  }
}

#endif
