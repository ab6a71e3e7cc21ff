// Hex8 strain / stress recovery (fea_engine/src/fea_engine/recovery.py:196-227, :258-334):
// values at the 2x2x2 Gauss points, sigma = D B u (or the engineering strain B u), moved to the
// corner nodes by the lumped L2 projection
//   value_a = sum_e sum_q N_a(q) |detJ| w val_q / sum_e sum_q N_a(q) |detJ| w
// over the elements e sharing node a, plus the volume-averaged element values
//   elem_e = sum_q |detJ| w val_q / sum_q |detJ| w,
// and optionally the von Mises stress of both (recovery.py:386-420).
//
// Two kernels.  k_recover_elements: 8 threads per element, thread q first evaluates Gauss point q
// (val_q, |detJ| w) into shared memory, then thread c projects onto corner c, writing the
// element's corner record (6 numerators + denominator, padded to 64 bytes) to scratch, and
// threads 0-5 form the element average.  k_recover_nodes: one thread per node adds the corner
// records of its elements (16-byte loads) in ascending element order, the order of the
// reference's np.add.at over the connectivity, so the result is deterministic with no atomics.
#include "feab_hex8.cuh"

namespace feab {
namespace {

constexpr int kRecElems = 16;                 // elements per 128-thread block
constexpr int kRecThreads = kRecElems * 8;
constexpr int kRecord = 8;                    // doubles per (element, corner): 6 numerators, denominator, pad


// Trilinear shape function of corner c at Gauss point q (elements/solids.py:133-142).
__device__ __forceinline__ double shape_at(int c, int q) {
  double xi, eta, zeta;
  gauss_point(q, xi, eta, zeta);
  return 0.125 * (1.0 + xi * xi_sign(c)) * (1.0 + eta * eta_sign(c)) * (1.0 + zeta * zeta_sign(c));
}

__device__ __forceinline__ double mises(const double (&s)[6]) {
  const double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
  return sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

__global__ void __launch_bounds__(kRecThreads) k_recover_elements(const double* __restrict__ coords,
                                                                  const int32_t* __restrict__ conn, int64_t n_elem,
                                                                  Mat6 D, int use_d, const double* __restrict__ u,
                                                                  double* __restrict__ rec, double* __restrict__ elem,
                                                                  double* __restrict__ elem_vm,
                                                                  feab_device_status* st) {
  __shared__ double sX[kRecElems][8][3];
  __shared__ double sU[kRecElems][8][3];
  __shared__ double sV[kRecElems][8][7];       // per Gauss point: val (6), |detJ| w
  const int le = threadIdx.x >> 3, t = threadIdx.x & 7;
  const int64_t e = (int64_t)blockIdx.x * kRecElems + le;
  const bool live = e < n_elem;
  if (live) {
    const int64_t n = conn[e * 8 + t];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      sX[le][t][j] = coords[n * 3 + j];
      sU[le][t][j] = u[n * 3 + j];
    }
  }
  __syncthreads();
  if (live) {
    // thread t = Gauss point q
    double X[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) X[k][j] = sX[le][k][j];
    double xi, eta, zeta, inv[3][3];
    gauss_point(t, xi, eta, zeta);
    const double det = jacobian_inverse(X, xi, eta, zeta, inv);
    if (!(fabs(det) >= 1e-300)) set_status(reinterpret_cast<int*>(st), FEAB_DEGENERATE_ELEMENT, e);
    double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      double a, b, c;
      dshape(k, xi, eta, zeta, a, b, c);
      const double gx = inv[0][0] * a + inv[0][1] * b + inv[0][2] * c;
      const double gy = inv[1][0] * a + inv[1][1] * b + inv[1][2] * c;
      const double gz = inv[2][0] * a + inv[2][1] * b + inv[2][2] * c;
      const double ux = sU[le][k][0], uy = sU[le][k][1], uz = sU[le][k][2];
      // B rows xx, yy, zz, xy, yz, xz with engineering shear (recovery.py:169-193)
      eps[0] += gx * ux;
      eps[1] += gy * uy;
      eps[2] += gz * uz;
      eps[3] += gy * ux + gx * uy;
      eps[4] += gz * uy + gy * uz;
      eps[5] += gz * ux + gx * uz;
    }
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      double v = eps[s];
      if (use_d) {
        v = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) v += D.d[s * 6 + j] * eps[j];
      }
      sV[le][t][s] = v;
    }
    sV[le][t][6] = fabs(det);  // Gauss weights are 1
  }
  __syncthreads();
  if (live) {
    // thread t = corner c: sum over the Gauss points in rule order
    double num[6] = {0, 0, 0, 0, 0, 0}, den = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double wn = sV[le][q][6] * shape_at(t, q);
#pragma unroll
      for (int s = 0; s < 6; ++s) num[s] += wn * sV[le][q][s];
      den += wn;
    }
    double2* r = reinterpret_cast<double2*>(rec + (e * 8 + t) * kRecord);
    r[0] = make_double2(num[0], num[1]);
    r[1] = make_double2(num[2], num[3]);
    r[2] = make_double2(num[4], num[5]);
    r[3] = make_double2(den, 0.0);
  }
  if (elem || elem_vm) {
    // thread t < 6: component t of the element average (every lane takes part in the shuffles)
    double avg = 0.0;
    if (live) {
      double acc = 0.0, vol = 0.0;
      const int s = t < 6 ? t : 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        acc += sV[le][q][6] * sV[le][q][s];
        vol += sV[le][q][6];
      }
      avg = acc / vol;
      if (elem && t < 6) elem[e * 6 + t] = avg;
    }
    if (elem_vm) {
      // the 8 threads of an element are 8 consecutive lanes of one warp
      double s6[6];
      const int base = threadIdx.x & 31 & ~7;
#pragma unroll
      for (int j = 0; j < 6; ++j) s6[j] = __shfl_sync(FEAB_FULL_MASK, avg, base + j);
      if (live && t == 0) elem_vm[e] = mises(s6);
    }
  }
}

__global__ void k_recover_nodes(const int32_t* __restrict__ conn, const int32_t* __restrict__ inc_ptr,
                                const int32_t* __restrict__ inc_elem, int32_t n_nodes, const double* __restrict__ rec,
                                double* __restrict__ nodal, double* __restrict__ nodal_vm) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  double num[6] = {0, 0, 0, 0, 0, 0}, den = 0.0;
  for (int k = inc_ptr[a]; k < inc_ptr[a + 1]; ++k) {
    const int64_t e = inc_elem[k];
    const int4 c0 = *reinterpret_cast<const int4*>(conn + e * 8);
    const int4 c1 = *reinterpret_cast<const int4*>(conn + e * 8 + 4);
    const int c = c0.x == a ? 0 : c0.y == a ? 1 : c0.z == a ? 2 : c0.w == a ? 3
                : c1.x == a ? 4 : c1.y == a ? 5 : c1.z == a ? 6 : 7;
    const double2* r = reinterpret_cast<const double2*>(rec + (e * 8 + c) * kRecord);
    const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
    num[0] += r0.x;
    num[1] += r0.y;
    num[2] += r1.x;
    num[3] += r1.y;
    num[4] += r2.x;
    num[5] += r2.y;
    den += r3.x;
  }
  double v[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) v[s] = den > 0.0 ? num[s] / den : 0.0;
  if (nodal) {
    double2* o = reinterpret_cast<double2*>(nodal + (int64_t)a * 6);
    o[0] = make_double2(v[0], v[1]);
    o[1] = make_double2(v[2], v[3]);
    o[2] = make_double2(v[4], v[5]);
  }
  if (nodal_vm) nodal_vm[a] = mises(v);
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_hex8_recover_scratch_bytes(int64_t n_elem) {
  return n_elem > 0 ? sizeof(double) * (size_t)kRecord * 8 * (size_t)n_elem : 0;
}

extern "C" int32_t feab_hex8_recover(const double* coords, const int32_t* conn, int64_t n_elem, int32_t n_nodes,
                                     const int32_t* inc_ptr, const int32_t* inc_elem, const double* D_host,
                                     const double* u, double* nodal, double* nodal_vm, double* elem, double* elem_vm,
                                     void* scratch, size_t scratch_bytes, feab_device_status* status,
                                     cudaStream_t s) {
  if (!coords || !conn || !inc_ptr || !inc_elem || !u || n_elem <= 0 || n_nodes <= 0) return FEAB_BAD_ARG;
  if (!nodal && !nodal_vm && !elem && !elem_vm) return FEAB_BAD_ARG;
  if (!scratch || scratch_bytes < feab_hex8_recover_scratch_bytes(n_elem)) return FEAB_BAD_ARG;
  // the record, connectivity and nodal accesses are 16-byte vector accesses
  if ((reinterpret_cast<uintptr_t>(scratch) & 15u) || (reinterpret_cast<uintptr_t>(conn) & 15u) ||
      (reinterpret_cast<uintptr_t>(nodal) & 15u))
    return FEAB_BAD_ARG;
  if ((nodal_vm || elem_vm) && !D_host) return FEAB_BAD_ARG;  // von Mises is of the stress
  if (n_elem > (int64_t)INT32_MAX * kRecElems) return FEAB_BAD_ARG;
  Mat6 D;
  for (int i = 0; i < 36; ++i) D.d[i] = D_host ? D_host[i] : 0.0;
  double* rec = static_cast<double*>(scratch);
  const int64_t grid = (n_elem + kRecElems - 1) / kRecElems;
  k_recover_elements<<<(unsigned)grid, kRecThreads, 0, s>>>(coords, conn, n_elem, D, D_host ? 1 : 0, u, rec, elem,
                                                             elem_vm, status);
  if (nodal || nodal_vm) {
    const int threads = 256;
    k_recover_nodes<<<(n_nodes + threads - 1) / threads, threads, 0, s>>>(conn, inc_ptr, inc_elem, n_nodes, rec, nodal,
                                                                         nodal_vm);
    count_launches(2);
  } else {
    count_launches(1);
  }
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
