// Hex8 element kernels: stiffness (a), element-by-element apply, SIMP adjoint (VJP).
#include <algorithm>
#include "feab_hex8.cuh"

namespace feab {
namespace {

constexpr int kKeElems = 16;          // elements per block
constexpr int kKeThreads = kKeElems * 8;  // one thread per (element, Gauss point) in phase 1

// Node pair (a, b), a <= b, of packed block index pr (inverse of packed_block).
__device__ __forceinline__ void pair_of(int pr, int& a, int& b) {
  a = 0;
#pragma unroll
  for (int k = 1; k < 8; ++k)
    if (pr >= packed_block(k, k)) a = k;
  b = a + (pr - packed_block(a, a));
}

// ke = sum_q B^T D B detJ w for the 36 node pairs a <= b of each element.
// Phase 1: thread (element, q) computes the physical gradients g[k] = J^-1 dN[:, k] and
// w*detJ into shared memory.  Phase 2: thread per (element, pair) contracts
// K_ab[i][j] = sum_q wdet * sum_{s,t} B_a[s][i] D[s][t] B_b[t][j], using the 3 non-zeros
// per column of B (row pattern of elements/solids.py:150-162).
// BBAR (Hex8SolidBbar, elements/solids.py:225-257): B is replaced by the mean-dilatation
// B-bar = B - (m m^T / 3) B + (m m^T / 3) B-averaged, B-averaged = sum_q B detJ w / sum_q detJ w
// (m = [1 1 1 0 0 0]); in the three normal-strain rows the column of node k, component j becomes
// delta_ij g_k,i - g_k,j / 3 + gbar_k,j / 3 with gbar_k the volume-averaged gradient, so the
// columns have 5 non-zeros and phase 2 contracts the full 6 x 3 column blocks.
template <bool BBAR>
__global__ void __launch_bounds__(kKeThreads) k_hex8_ke(const double* __restrict__ coords, const int32_t* __restrict__ conn,
                                                        int64_t n_elem, Mat6 D, const double* __restrict__ scale,
                                                        double thickness, double* __restrict__ ke, int layout,
                                                        feab_device_status* st) {
  __shared__ double sX[kKeElems][8][3];
  __shared__ double sG[kKeElems][8][8][3];
  __shared__ double sW[kKeElems][8];
  __shared__ double sGbar[BBAR ? kKeElems : 1][8][3];
  const int t = threadIdx.x;
  const int64_t e0 = (int64_t)blockIdx.x * kKeElems;
  {
    const int el = t >> 3, k = t & 7;
    const int64_t e = e0 + el;
    if (e < n_elem) {
      const int64_t n = conn[e * 8 + k];
      sX[el][k][0] = coords[n * 3 + 0];
      sX[el][k][1] = coords[n * 3 + 1];
      sX[el][k][2] = coords[n * 3 + 2];
    }
  }
  __syncthreads();
  {
    const int el = t >> 3, q = t & 7;
    const int64_t e = e0 + el;
    if (e < n_elem) {
      double X[8][3];
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) X[k][j] = sX[el][k][j];
      double xi, eta, zeta, inv[3][3];
      gauss_point(q, xi, eta, zeta);
      const double det = jacobian_inverse(X, xi, eta, zeta, inv);
      if (!(fabs(det) >= 1e-300)) set_status(reinterpret_cast<int*>(st), FEAB_DEGENERATE_ELEMENT, e);
      sW[el][q] = det;  // w = 1 for the 2-point rule
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        double a, b, c;
        dshape(k, xi, eta, zeta, a, b, c);
#pragma unroll
        for (int i = 0; i < 3; ++i) sG[el][q][k][i] = inv[i][0] * a + inv[i][1] * b + inv[i][2] * c;
      }
    }
  }
  __syncthreads();
  if (BBAR) {
    // thread (element, k): the volume-averaged gradient of node k (Gauss points in rule order)
    const int el = t >> 3, k = t & 7;
    if (e0 + el < n_elem) {
      double gx = 0.0, gy = 0.0, gz = 0.0, vol = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double w = sW[el][q];
        gx += sG[el][q][k][0] * w;
        gy += sG[el][q][k][1] * w;
        gz += sG[el][q][k][2] * w;
        vol += w;
      }
      sGbar[el][k][0] = gx / vol;
      sGbar[el][k][1] = gy / vol;
      sGbar[el][k][2] = gz / vol;
    }
    __syncthreads();
  }
  for (int task = t; task < kKeElems * 36; task += kKeThreads) {
    const int el = task / 36, pr = task % 36;
    const int64_t e = e0 + el;
    if (e >= n_elem) break;
    int a, b;
    pair_of(pr, a, b);
    double K[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (BBAR) {
      // B-bar column blocks Ba, Bb (6 x 3) at each Gauss point; K_ab += w Ba^T D Bb
      const double (&ga)[3] = sGbar[el][a];
      const double (&gb)[3] = sGbar[el][b];
#pragma unroll 1
      for (int q = 0; q < 8; ++q) {
        const double w = sW[el][q];
        double Ba[6][3], Bb[6][3];
        auto column = [&](const double (&g)[3], const double (&gbar)[3], double (&B)[6][3]) {
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const double vol = (gbar[j] - g[j]) / 3.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) B[i][j] = (i == j ? g[i] : 0.0) + vol;
          }
          B[3][0] = g[1];
          B[3][1] = g[0];
          B[3][2] = 0.0;
          B[4][0] = 0.0;
          B[4][1] = g[2];
          B[4][2] = g[1];
          B[5][0] = g[2];
          B[5][1] = 0.0;
          B[5][2] = g[0];
        };
        const double gqa[3] = {sG[el][q][a][0], sG[el][q][a][1], sG[el][q][a][2]};
        const double gqb[3] = {sG[el][q][b][0], sG[el][q][b][1], sG[el][q][b][2]};
        column(gqa, ga, Ba);
        column(gqb, gb, Bb);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double DB[6];
#pragma unroll
          for (int s = 0; s < 6; ++s) {
            double v = 0.0;
#pragma unroll
            for (int r = 0; r < 6; ++r) v += D.d[s * 6 + r] * Bb[r][j];
            DB[s] = v;
          }
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            double v = 0.0;
#pragma unroll
            for (int s = 0; s < 6; ++s) v += Ba[s][i] * DB[s];
            K[i][j] += w * v;
          }
        }
      }
    } else
#pragma unroll 2
    for (int q = 0; q < 8; ++q) {
      const double w = sW[el][q];
      const double ax = sG[el][q][a][0], ay = sG[el][q][a][1], az = sG[el][q][a][2];
      const double bx = sG[el][q][b][0], by = sG[el][q][b][1], bz = sG[el][q][b][2];
      double DB[6][3];
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        DB[s][0] = D.d[s * 6 + 0] * bx + D.d[s * 6 + 3] * by + D.d[s * 6 + 5] * bz;
        DB[s][1] = D.d[s * 6 + 1] * by + D.d[s * 6 + 3] * bx + D.d[s * 6 + 4] * bz;
        DB[s][2] = D.d[s * 6 + 2] * bz + D.d[s * 6 + 4] * by + D.d[s * 6 + 5] * bx;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        K[0][j] += w * (ax * DB[0][j] + ay * DB[3][j] + az * DB[5][j]);
        K[1][j] += w * (ay * DB[1][j] + ax * DB[3][j] + az * DB[4][j]);
        K[2][j] += w * (az * DB[2][j] + ay * DB[4][j] + ax * DB[5][j]);
      }
    }
    if (a == b) {  // diagonal node block: mirror the upper triangle so ke is exactly symmetric
      K[1][0] = K[0][1];
      K[2][0] = K[0][2];
      K[2][1] = K[1][2];
    }
    const double f = thickness * (scale ? scale[e] : 1.0);
    if (layout == FEAB_HEX8_KE_PACKED) {
      double* o = ke + (e * 36 + pr) * 9;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = K[i][j] * f;
    } else {
      double* o = ke + e * 576;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          o[(3 * a + i) * 24 + 3 * b + j] = K[i][j] * f;
          if (a != b) o[(3 * b + j) * 24 + 3 * a + i] = K[i][j] * f;
        }
    }
  }
}

// Consistent mass (Element.mass, elements/base.py:711-731): me = sum_q Nm^T R Nm |detJ| w t, so the
// (a, b) node block is m_ab R t with m_ab = sum_q N_a N_b |detJ| w and R the 3x3 density matrix.
// Thread (element, q) forms |detJ_q| into shared memory; thread (element, pair a <= b) sums m_ab
// over the Gauss points in rule order and writes the block (packed) or both blocks (full).
__global__ void __launch_bounds__(kKeThreads) k_hex8_mass(const double* __restrict__ coords,
                                                          const int32_t* __restrict__ conn, int64_t n_elem, Mat6 R,
                                                          const double* __restrict__ scale, double thickness,
                                                          double* __restrict__ me, int layout,
                                                          feab_device_status* st) {
  __shared__ double sX[kKeElems][8][3];
  __shared__ double sDet[kKeElems][8];
  const int t = threadIdx.x;
  const int64_t e0 = (int64_t)blockIdx.x * kKeElems;
  {
    const int el = t >> 3, k = t & 7;
    const int64_t e = e0 + el;
    if (e < n_elem) {
      const int64_t n = conn[e * 8 + k];
      sX[el][k][0] = coords[n * 3 + 0];
      sX[el][k][1] = coords[n * 3 + 1];
      sX[el][k][2] = coords[n * 3 + 2];
    }
  }
  __syncthreads();
  {
    const int el = t >> 3, q = t & 7;
    const int64_t e = e0 + el;
    if (e < n_elem) {
      double X[8][3];
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) X[k][j] = sX[el][k][j];
      double xi, eta, zeta, inv[3][3];
      gauss_point(q, xi, eta, zeta);
      const double det = jacobian_inverse(X, xi, eta, zeta, inv);
      if (!(fabs(det) >= 1e-300)) set_status(reinterpret_cast<int*>(st), FEAB_DEGENERATE_ELEMENT, e);
      sDet[el][q] = fabs(det);  // w = 1 for the 2-point rule
    }
  }
  __syncthreads();
  for (int task = t; task < kKeElems * 36; task += kKeThreads) {
    const int el = task / 36, pr = task % 36;
    const int64_t e = e0 + el;
    if (e >= n_elem) break;
    int a, b;
    pair_of(pr, a, b);
    double m = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      double xi, eta, zeta;
      gauss_point(q, xi, eta, zeta);
      const double Na = 0.125 * (1.0 + xi * xi_sign(a)) * (1.0 + eta * eta_sign(a)) * (1.0 + zeta * zeta_sign(a));
      const double Nb = 0.125 * (1.0 + xi * xi_sign(b)) * (1.0 + eta * eta_sign(b)) * (1.0 + zeta * zeta_sign(b));
      m += Na * Nb * sDet[el][q];
    }
    const double f = m * thickness * (scale ? scale[e] : 1.0);
    if (layout == FEAB_HEX8_KE_PACKED) {
      double* o = me + (e * 36 + pr) * 9;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = R.d[i * 3 + j] * f;
    } else {
      double* o = me + e * 576;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          o[(3 * a + i) * 24 + 3 * b + j] = R.d[i * 3 + j] * f;
          if (a != b) o[(3 * b + j) * 24 + 3 * a + i] = R.d[i * 3 + j] * f;
        }
    }
  }
}

// y[3a+i] = sum over elements e of a, local nodes lb, dofs j: K_e(la,lb)[i][j] v[3 b + j].
// One warp per node; 72 (lb, i, j) terms per element spread over the lanes.
__global__ void k_hex8_apply(const double* __restrict__ ke, const int32_t* __restrict__ conn,
                             const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc_elem, int32_t n_nodes,
                             const double* __restrict__ v, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (a >= n_nodes) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int k = inc_ptr[a]; k < inc_ptr[a + 1]; ++k) {
    const int64_t e = inc_elem[k];
    const int cl = conn[e * 8 + (lane & 7)];
    const unsigned m = __ballot_sync(FEAB_FULL_MASK, lane < 8 && cl == a);
    const int la = __ffs(m) - 1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int t = lane + 32 * r;
      const int lb = min(t / 9, 7);
      const int b = __shfl_sync(FEAB_FULL_MASK, cl, lb);
      if (t < 72) {
        const int i = (t % 9) / 3, j = t % 3;
        const double val = la <= lb ? ke[(e * 36 + packed_block(la, lb)) * 9 + i * 3 + j]
                                    : ke[(e * 36 + packed_block(lb, la)) * 9 + j * 3 + i];
        const double c = val * v[(int64_t)b * 3 + j];
        acc[0] += i == 0 ? c : 0.0;
        acc[1] += i == 1 ? c : 0.0;
        acc[2] += i == 2 ? c : 0.0;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) acc[i] = warp_sum(acc[i]);
  if (lane < 3) y[(int64_t)a * 3 + lane] = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : acc[2]);
}

// out[e] = -p (1 - rho_min) rho_e^(p-1) * sum_q eps(lam)^T D eps(u) detJ w  (= lam_e^T K0_e u_e).
__global__ void k_hex8_simp_vjp(const double* __restrict__ coords, const int32_t* __restrict__ conn, int64_t n_elem,
                                Mat6 D, const double* __restrict__ rho, double penal, double rho_min,
                                const double* __restrict__ u, const double* __restrict__ lam, double* __restrict__ out,
                                feab_device_status* st) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  double X[8][3], U[8][3], L[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int64_t n = conn[e * 8 + k];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      X[k][j] = coords[n * 3 + j];
      U[k][j] = u[n * 3 + j];
      L[k][j] = lam[n * 3 + j];
    }
  }
  double energy = 0.0;
#pragma unroll 1
  for (int q = 0; q < 8; ++q) {
    double xi, eta, zeta, inv[3][3];
    gauss_point(q, xi, eta, zeta);
    const double det = jacobian_inverse(X, xi, eta, zeta, inv);
    if (!(fabs(det) >= 1e-300)) set_status(reinterpret_cast<int*>(st), FEAB_DEGENERATE_ELEMENT, e);
    double eu[6] = {0, 0, 0, 0, 0, 0}, el[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      double a, b, c;
      dshape(k, xi, eta, zeta, a, b, c);
      const double gx = inv[0][0] * a + inv[0][1] * b + inv[0][2] * c;
      const double gy = inv[1][0] * a + inv[1][1] * b + inv[1][2] * c;
      const double gz = inv[2][0] * a + inv[2][1] * b + inv[2][2] * c;
      eu[0] += gx * U[k][0];
      eu[1] += gy * U[k][1];
      eu[2] += gz * U[k][2];
      eu[3] += gy * U[k][0] + gx * U[k][1];
      eu[4] += gz * U[k][1] + gy * U[k][2];
      eu[5] += gz * U[k][0] + gx * U[k][2];
      el[0] += gx * L[k][0];
      el[1] += gy * L[k][1];
      el[2] += gz * L[k][2];
      el[3] += gy * L[k][0] + gx * L[k][1];
      el[4] += gz * L[k][1] + gy * L[k][2];
      el[5] += gz * L[k][0] + gx * L[k][2];
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double di = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) di += D.d[i * 6 + j] * eu[j];
      s += el[i] * di;
    }
    energy += s * det;
  }
  const double r = rho[e];
  out[e] = -penal * (1.0 - rho_min) * pow(r, penal - 1.0) * energy;
}

}  // namespace
}  // namespace feab

using namespace feab;

static bool load_mat6(const double* D_host, Mat6* out) {
  if (!D_host) return false;
  for (int i = 0; i < 36; ++i) out->d[i] = D_host[i];
  return true;
}

static int32_t element_stiffness(bool bbar, const double* coords, const int32_t* conn, int64_t n_elem,
                                 const double* D_host, const double* scale, double thickness, double* ke_out,
                                 int32_t layout, feab_device_status* status, cudaStream_t s) {
  Mat6 D;
  if (!coords || !conn || !ke_out || n_elem < 0 || !load_mat6(D_host, &D)) return FEAB_BAD_ARG;
  if (layout != FEAB_HEX8_KE_PACKED && layout != FEAB_HEX8_KE_FULL) return FEAB_BAD_ARG;
  if (n_elem == 0) return FEAB_OK;
  const int64_t grid = (n_elem + kKeElems - 1) / kKeElems;
  count_launches(1);
  if (bbar)
    k_hex8_ke<true><<<(unsigned)grid, kKeThreads, 0, s>>>(coords, conn, n_elem, D, scale, thickness, ke_out, layout,
                                                          status);
  else
    k_hex8_ke<false><<<(unsigned)grid, kKeThreads, 0, s>>>(coords, conn, n_elem, D, scale, thickness, ke_out, layout,
                                                           status);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_hex8_element_stiffness(const double* coords, const int32_t* conn, int64_t n_elem,
                                               const double* D_host, const double* scale, double thickness,
                                               double* ke_out, int32_t layout, feab_device_status* status,
                                               cudaStream_t s) {
  return element_stiffness(false, coords, conn, n_elem, D_host, scale, thickness, ke_out, layout, status, s);
}

extern "C" int32_t feab_hex8_bbar_element_stiffness(const double* coords, const int32_t* conn, int64_t n_elem,
                                                    const double* D_host, const double* scale, double thickness,
                                                    double* ke_out, int32_t layout, feab_device_status* status,
                                                    cudaStream_t s) {
  return element_stiffness(true, coords, conn, n_elem, D_host, scale, thickness, ke_out, layout, status, s);
}

extern "C" int32_t feab_hex8_element_mass(const double* coords, const int32_t* conn, int64_t n_elem,
                                          const double* R_host, const double* scale, double thickness, double* me_out,
                                          int32_t layout, feab_device_status* status, cudaStream_t s) {
  if (!coords || !conn || !me_out || !R_host || n_elem < 0) return FEAB_BAD_ARG;
  if (layout != FEAB_HEX8_KE_PACKED && layout != FEAB_HEX8_KE_FULL) return FEAB_BAD_ARG;
  Mat6 R;  // the 3x3 density matrix in the first 9 entries
  for (int i = 0; i < 36; ++i) R.d[i] = i < 9 ? R_host[i] : 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < i; ++j)
      if (R.d[i * 3 + j] != R.d[j * 3 + i]) return FEAB_BAD_ARG;  // the packed blocks assume R = R^T
  if (n_elem == 0) return FEAB_OK;
  const int64_t grid = (n_elem + kKeElems - 1) / kKeElems;
  count_launches(1);
  k_hex8_mass<<<(unsigned)grid, kKeThreads, 0, s>>>(coords, conn, n_elem, R, scale, thickness, me_out, layout, status);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_hex8_apply(const double* ke_packed, const int32_t* conn, const int32_t* inc_ptr,
                                   const int32_t* inc_elem, int32_t n_nodes, const double* v, double* y,
                                   cudaStream_t s) {
  if (!ke_packed || !conn || !inc_ptr || !inc_elem || !v || !y || n_nodes <= 0) return FEAB_BAD_ARG;
  const int wpb = 8;
  count_launches(1);
  k_hex8_apply<<<(n_nodes + wpb - 1) / wpb, wpb * 32, 0, s>>>(ke_packed, conn, inc_ptr, inc_elem, n_nodes, v, y);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_hex8_simp_vjp(const double* coords, const int32_t* conn, int64_t n_elem, const double* D_host,
                                      const double* rho, double penal, double rho_min, const double* u,
                                      const double* lam, double* out, feab_device_status* status, cudaStream_t s) {
  Mat6 D;
  if (!coords || !conn || !rho || !u || !lam || !out || n_elem < 0 || !load_mat6(D_host, &D)) return FEAB_BAD_ARG;
  if (n_elem == 0) return FEAB_OK;
  const int threads = 128;
  count_launches(1);
  k_hex8_simp_vjp<<<(unsigned)((n_elem + threads - 1) / threads), threads, 0, s>>>(coords, conn, n_elem, D, rho, penal,
                                                                                    rho_min, u, lam, out, status);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
