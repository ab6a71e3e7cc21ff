// Hex8 geometry at the 2x2x2 Gauss points (shared by the element kernels).
#pragma once
#include "feab_common.cuh"

namespace feab {

// Gauss-Legendre 2-point abscissa exactly as numpy.polynomial.legendre.leggauss(2) returns it
// (0x1.279a74590331cp-1); weights are exactly 1.0.
#define FEAB_GAUSS2 0.5773502691896257

struct Mat6 {
  double d[36];
};

// Natural coordinates of Gauss point q in the reference's order: xi outer, eta, zeta inner
// (fea_engine/src/fea_engine/elements/base.py:92-94).
__device__ __forceinline__ void gauss_point(int q, double& xi, double& eta, double& zeta) {
  xi = (q & 4) ? FEAB_GAUSS2 : -FEAB_GAUSS2;
  eta = (q & 2) ? FEAB_GAUSS2 : -FEAB_GAUSS2;
  zeta = (q & 1) ? FEAB_GAUSS2 : -FEAB_GAUSS2;
}

// Corner signs of Hex8Solid3D.shape_and_derivs (elements/solids.py:133-142).
__device__ __forceinline__ double xi_sign(int k) { return (k == 1 || k == 2 || k == 5 || k == 6) ? 1.0 : -1.0; }
__device__ __forceinline__ double eta_sign(int k) { return (k == 2 || k == 3 || k == 6 || k == 7) ? 1.0 : -1.0; }
__device__ __forceinline__ double zeta_sign(int k) { return k >= 4 ? 1.0 : -1.0; }

// Natural derivatives dN/dxi, dN/deta, dN/dzeta of node k at (xi, eta, zeta).
__device__ __forceinline__ void dshape(int k, double xi, double eta, double zeta, double& dx, double& de, double& dz) {
  const double sx = xi_sign(k), se = eta_sign(k), sz = zeta_sign(k);
  dx = 0.125 * sx * (1.0 + eta * se) * (1.0 + zeta * sz);
  de = 0.125 * se * (1.0 + xi * sx) * (1.0 + zeta * sz);
  dz = 0.125 * sz * (1.0 + xi * sx) * (1.0 + eta * se);
}

// Determinant and inverse of a 3x3 matrix by cofactors; returns det.
__device__ __forceinline__ double invert3(const double (&J)[3][3], double (&inv)[3][3]) {
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double r = 1.0 / det;
  inv[0][0] = c00 * r;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
  inv[1][0] = c01 * r;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
  inv[2][0] = c02 * r;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
  return det;
}

// J = dN @ X (J[i][j] = sum_k dN[i][k] X[k][j]), its determinant and inverse.
// Returns det; inv = J^-1, so physical gradients are g_k = inv @ dN[:, k]
// (np.linalg.solve(J, dN) in elements/solids.py:147).
__device__ __forceinline__ double jacobian_inverse(const double (&X)[8][3], double xi, double eta, double zeta,
                                                   double (&inv)[3][3]) {
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double a, b, c;
    dshape(k, xi, eta, zeta, a, b, c);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      J[0][j] += a * X[k][j];
      J[1][j] += b * X[k][j];
      J[2][j] += c * X[k][j];
    }
  }
  return invert3(J, inv);
}

// Packed upper-block index of node pair (a, b), a <= b: rows of the upper triangle in order.
__host__ __device__ __forceinline__ int packed_block(int a, int b) { return a * 8 - (a * (a - 1)) / 2 + (b - a); }

}  // namespace feab
