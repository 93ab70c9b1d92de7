// kernels_setup.cuh -- one-time FP64 setup on the GPU: per-GLL-point
// Jacobians, P1-interpolated material, folded stiffness records (stored in
// the problem precision) and the element-local diagonal mass.
//
// Reference arithmetic restated: HexP1::inverseJacobianAtPoint
// (HexP1.cpp:189-240), QuadP1::inverseJacobianAtPoint (QuadP1.h:79-90, with
// the correct dN/dr(s), dN/ds(r) arguments), ParAtIntPts (TensorQuad.cpp:
// 309-323, Hexahedra.cpp:635-656), Elastic3D::attachMaterialProperties
// (Elastic3D.cpp:33-54), assembleElementMassMatrix (Scalar.cpp:34-39,
// Elastic3D.cpp:63-67), Order2Newmark::initializeGlobalDofs
// (Order2Newmark.cpp:32-66).
#pragma once

#include <cstdint>

#include "kernels_material.cuh"

namespace salvus {

constexpr int kMaxN = 11;

struct GllTable {
  double xi[kMaxN];
  double w[kMaxN];
};

__device__ __forceinline__ void p1_jac_dev(int dim, const double *v, const double *ref,
                                           double *detJ, double *invJ) {
  if (dim == 2) {
    const double sg[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    double J0 = 0, J1 = 0, J2 = 0, J3 = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double dr = 0.25 * sg[k][0] * (1 + sg[k][1] * ref[1]);
      double ds = 0.25 * sg[k][1] * (1 + sg[k][0] * ref[0]);
      J0 += dr * v[2 * k]; J1 += dr * v[2 * k + 1];
      J2 += ds * v[2 * k]; J3 += ds * v[2 * k + 1];
    }
    double d = J0 * J3 - J1 * J2;
    *detJ = d;
    invJ[0] = J3 / d; invJ[1] = -J1 / d; invJ[2] = -J2 / d; invJ[3] = J0 / d;
    return;
  }
  const double sg[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double a = 1 + sg[k][0] * ref[0], b = 1 + sg[k][1] * ref[1], c = 1 + sg[k][2] * ref[2];
    double d0 = 0.125 * sg[k][0] * b * c, d1 = 0.125 * sg[k][1] * a * c,
           d2 = 0.125 * sg[k][2] * a * b;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      J[m] += d0 * v[3 * k + m];
      J[3 + m] += d1 * v[3 * k + m];
      J[6 + m] += d2 * v[3 * k + m];
    }
  }
  double m00 = J[4] * J[8] - J[5] * J[7], m01 = J[5] * J[6] - J[3] * J[8],
         m02 = J[3] * J[7] - J[4] * J[6];
  double d = J[0] * m00 + J[1] * m01 + J[2] * m02;
  double id = 1.0 / d;
  *detJ = d;
  invJ[0] = m00 * id;
  invJ[1] = (J[2] * J[7] - J[1] * J[8]) * id;
  invJ[2] = (J[1] * J[5] - J[2] * J[4]) * id;
  invJ[3] = m01 * id;
  invJ[4] = (J[0] * J[8] - J[2] * J[6]) * id;
  invJ[5] = (J[2] * J[3] - J[0] * J[5]) * id;
  invJ[6] = m02 * id;
  invJ[7] = (J[1] * J[6] - J[0] * J[7]) * id;
  invJ[8] = (J[0] * J[4] - J[1] * J[3]) * id;
}

__device__ __forceinline__ double p1_interp_dev(int dim, const double *vals, const double *ref) {
  if (dim == 2) {
    return 0.25 * ((1 - ref[0]) * (1 - ref[1]) * vals[0] + (1 + ref[0]) * (1 - ref[1]) * vals[1] +
                   (1 + ref[0]) * (1 + ref[1]) * vals[2] + (1 - ref[0]) * (1 + ref[1]) * vals[3]);
  }
  const double sg[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    s += 0.125 * (1 + sg[k][0] * ref[0]) * (1 + sg[k][1] * ref[1]) * (1 + sg[k][2] * ref[2]) *
         vals[k];
  return s;
}

// One thread per element point.  Writes the stiffness record (FP32 packed
// with connectivity, or FP64) and the element-local mass w detJ (rho).
// Records:
//   acoustic : G = w detJ vp^2 invJ^T invJ (symmetric; 3 or 6 words)
//   elastic  : invJ (row-major [x_a][xi_b], 9 words), lambda w detJ, mu w detJ
//              (transversely isotropic: A C F L N w detJ, kernels_material.cuh)
// FP32 elastic records (12 words with connectivity, 16 transversely
// isotropic) are stored as float4 planes per element, [E][3|4][P] float4:
// plane 0 = invJ 0-3, plane 1 = invJ 4-7, plane 2 = (invJ 8, m0, m1, conn),
// plane 3 = (m2, m3, m4, 0), so that consecutive points of one plane are
// consecutive 16-byte words (contiguous warp loads).
// Meshes of fluid and solid quadrilaterals (physics 3): records are stored per
// class, fluid elements first ([Ef] acoustic quad records) then solid ones
// (elastic 2-D records); cls_k[e] is the element's index within its class.
template <typename real, bool kPackConn>
__global__ void geometry_kernel(int64_t E, int dim, int n, int P, int physics, int rw,
                                const double *__restrict__ vtx, const double *__restrict__ par,
                                const int32_t *__restrict__ conn, GllTable gll,
                                real *__restrict__ rec, double *__restrict__ mass_local,
                                const int32_t *__restrict__ cls_k = nullptr, int64_t Ef = 0,
                                bool ti = false) {
  int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= E * P) return;
  const int64_t e = tid / P;
  const int p = (int)(tid - e * P);
  const int nv = dim == 2 ? 4 : 8;
  const int i = p % n, j = (p / n) % n, k = p / (n * n);
  double ref[3] = {gll.xi[i], gll.xi[j], dim == 3 ? gll.xi[k] : 0.0};
  double wq = gll.w[i] * gll.w[j] * (dim == 3 ? gll.w[k] : 1.0);
  double v[24];
  for (int a = 0; a < nv * dim; ++a) v[a] = vtx[e * nv * dim + a];
  double detJ, iJ[9];
  p1_jac_dev(dim, v, ref, &detJ, iJ);
  const double wd = wq * detJ;
  real *out = rec + tid * rw;
  if (physics == 3) {
    // FLUID VP RHO C11 C13 C33 C55 per element vertex
    auto at = [&](int k) {
      double vals[4];
      for (int a = 0; a < 4; ++a) vals[a] = par[((int64_t)k * E + e) * 4 + a];
      return p1_interp_dev(2, vals, ref);
    };
    const int64_t k = cls_k[e];
    if (par[e * 4] == 1.0) {
      const double vp = at(1), sc = wd * vp * vp;
      const double g3[3] = {sc * (iJ[0] * iJ[0] + iJ[2] * iJ[2]),
                            sc * (iJ[0] * iJ[1] + iJ[2] * iJ[3]),
                            sc * (iJ[1] * iJ[1] + iJ[3] * iJ[3])};
      if constexpr (kPackConn) {
        real *o = rec + (k * P + p) * 4;
        for (int a = 0; a < 3; ++a) o[a] = (real)g3[a];
        reinterpret_cast<int32_t *>(o)[3] = conn[tid];
      } else {
        real *o = rec + (k * P + p) * 3;
        for (int a = 0; a < 3; ++a) o[a] = (real)g3[a];
      }
      mass_local[tid] = wd;  // Scalar mass (Scalar.cpp:34-39)
    } else {
      const double w8[8] = {iJ[0], iJ[1], iJ[2], iJ[3],
                            wd * at(3), wd * at(4), wd * at(5), wd * at(6)};
      for (int a = 0; a < 8; ++a) {
        if constexpr (kPackConn)
          rec[Ef * P * 4 + ((k * 2 + a / 4) * P + p) * 4 + a % 4] = (real)w8[a];
        else
          rec[Ef * P * 3 + (k * P + p) * 8 + a] = (real)w8[a];
      }
      mass_local[tid] = wd * at(2);  // Elastic2D mass: rho (Elastic2D.cpp:45-50)
    }
    return;
  }
  if (physics == 2) {
    // elastic 2-D quads: RHO, C11, C13, C33, C55 at the point (Elastic2D.cpp:29-37,
    // 57-60); record invJ (4 words) and C * w detJ (4 words), FP32 as two
    // float4 planes [E][2][P] (kernels_elastic2d.cuh), FP64 as [E][P][8]
    double cp[5];
    for (int k = 0; k < 5; ++k) {
      double vals[4];
      for (int a = 0; a < 4; ++a) vals[a] = par[((int64_t)k * E + e) * 4 + a];
      cp[k] = p1_interp_dev(2, vals, ref);
    }
    double w8[8] = {iJ[0], iJ[1], iJ[2], iJ[3], wd * cp[1], wd * cp[2], wd * cp[3], wd * cp[4]};
    for (int a = 0; a < 8; ++a) {
      if constexpr (kPackConn) rec[((e * 2 + a / 4) * P + p) * 4 + a % 4] = (real)w8[a];
      else out[a] = (real)w8[a];
    }
    mass_local[tid] = wd * cp[0];  // Elastic2D mass: rho (Elastic2D.cpp:45-50)
    return;
  }
  if (physics == 0) {
    double vals[8];
    for (int a = 0; a < nv; ++a) vals[a] = par[e * nv + a];
    double vp = p1_interp_dev(dim, vals, ref);
    double s = wd * vp * vp;
    if (dim == 2) {
      // G_bc = sum_a invJ[a][b] invJ[a][c]
      double g00 = iJ[0] * iJ[0] + iJ[2] * iJ[2];
      double g01 = iJ[0] * iJ[1] + iJ[2] * iJ[3];
      double g11 = iJ[1] * iJ[1] + iJ[3] * iJ[3];
      out[0] = (real)(s * g00); out[1] = (real)(s * g01); out[2] = (real)(s * g11);
    } else {
      int q = 0;
      for (int b = 0; b < 3; ++b)
        for (int c = b; c < 3; ++c) {
          double g = iJ[0 * 3 + b] * iJ[0 * 3 + c] + iJ[1 * 3 + b] * iJ[1 * 3 + c] +
                     iJ[2 * 3 + b] * iJ[2 * 3 + c];
          out[q++] = (real)(s * g);
        }
    }
    mass_local[tid] = wd;  // Scalar mass: no density (Scalar.cpp:34-39)
  } else {
    // elastic 3-D: P1-interpolated RHO VP VS (isotropic) or RHO VPV VPH VSV
    // VSH ETA (transversely isotropic), then the folded constants
    // (Elastic3D.cpp:42-53, kernels_material.cuh)
    const int npar = ti ? 6 : 3;
    double pv[6];
    for (int q = 0; q < npar; ++q) {
      double vals[8];
      for (int a = 0; a < 8; ++a) vals[a] = par[((int64_t)q * E + e) * 8 + a];
      pv[q] = p1_interp_dev(3, vals, ref);
    }
    double mc[5];
    const int nm = ti ? 5 : 2;
    if (ti) elastic_constants_ti(pv, mc);
    else elastic_constants_iso(pv[0], pv[1], pv[2], mc);
    if constexpr (kPackConn) {
      // float4 planes [E][3|4][P]: invJ 0-3 | invJ 4-7 | invJ 8, m0, m1, conn
      // | m2, m3, m4, 0 (transversely isotropic only)
      const int planes = ti ? 4 : 3;
      real w16[16];
      for (int a = 0; a < 9; ++a) w16[a] = (real)iJ[a];
      w16[9] = (real)(wd * mc[0]);
      w16[10] = (real)(wd * mc[1]);
      w16[11] = 0;
      reinterpret_cast<int32_t *>(w16)[11] = conn[tid];
      for (int a = 0; a < 4; ++a) w16[12 + a] = a < 3 && ti ? (real)(wd * mc[2 + a]) : (real)0;
      for (int a = 0; a < 4 * planes; ++a)
        rec[((e * planes + a / 4) * P + p) * 4 + a % 4] = w16[a];
    } else {
      for (int a = 0; a < 9; ++a) out[a] = (real)iJ[a];
      for (int a = 0; a < nm; ++a) out[9 + a] = (real)(wd * mc[a]);
    }
    mass_local[tid] = wd * pv[0];
    return;
  }
  if (kPackConn) {
    int32_t c = conn[tid];
    reinterpret_cast<int32_t *>(out)[rw - (dim == 3 && physics == 0 ? 2 : 1)] = c;
    if (dim == 3 && physics == 0) reinterpret_cast<int32_t *>(out)[rw - 1] = 0;
  }
}

// FP32 records of elastic hexahedra that are all parallelepipeds
// (kernels_hex_affine.cuh): one thread per element point writes the folded
// material planes mat[m][e*P + p] (w detJ at the point times the constants
// of the P1-interpolated parameters, as geometry_kernel) and the
// element-local mass; point 0 of each element also writes invJ at the
// element centre to jac[e][9] (constant over an affine element).
__global__ void affine_hex_records_kernel(int64_t E, int n, int P, bool ti,
                                          const double *__restrict__ vtx,
                                          const double *__restrict__ par, GllTable gll,
                                          float *__restrict__ mat, float *__restrict__ jac,
                                          double *__restrict__ mass_local) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= E * P) return;
  const int64_t e = tid / P;
  const int p = (int)(tid - e * P);
  const int i = p % n, j = (p / n) % n, k = p / (n * n);
  const double ref[3] = {gll.xi[i], gll.xi[j], gll.xi[k]};
  const double wq = gll.w[i] * gll.w[j] * gll.w[k];
  double v[24];
  for (int a = 0; a < 24; ++a) v[a] = vtx[e * 24 + a];
  double detJ, iJ[9];
  p1_jac_dev(3, v, ref, &detJ, iJ);
  const double wd = wq * detJ;
  const int npar = ti ? 6 : 3;
  double pv[6];
  for (int q = 0; q < npar; ++q) {
    double vals[8];
    for (int a = 0; a < 8; ++a) vals[a] = par[((int64_t)q * E + e) * 8 + a];
    pv[q] = p1_interp_dev(3, vals, ref);
  }
  double mc[5];
  const int nm = ti ? 5 : 2;
  if (ti) elastic_constants_ti(pv, mc);
  else elastic_constants_iso(pv[0], pv[1], pv[2], mc);
  for (int q = 0; q < nm; ++q) mat[(int64_t)q * E * P + tid] = (float)(wd * mc[q]);
  mass_local[tid] = wd * pv[0];
  if (p == 0) {
    const double c0[3] = {0.0, 0.0, 0.0};
    double d0, J0[9];
    p1_jac_dev(3, v, c0, &d0, J0);
    for (int a = 0; a < 9; ++a) jac[e * 9 + a] = (float)J0[a];
  }
}

// Diagonal mass by node gather in ascending element order, then reciprocal.
__global__ void mass_gather_kernel(int64_t G, const int32_t *__restrict__ off,
                                   const int32_t *__restrict__ idx,
                                   const double *__restrict__ mass_local,
                                   double *__restrict__ mi64, float *__restrict__ mi32) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  double s = 0.0;
  for (int32_t q = off[g]; q < off[g + 1]; ++q) s += mass_local[idx[q]];
  double m = 1.0 / s;
  mi64[g] = m;
  mi32[g] = (float)m;
}

}  // namespace salvus
