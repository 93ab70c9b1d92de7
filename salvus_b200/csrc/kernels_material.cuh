// kernels_material.cuh -- Elastic3D Hooke's law at one quadrature point,
// with the quadrature weight and detJ folded into the constants.
//
// Reference: Elastic3D::attachMaterialProperties (Elastic3D.cpp:33-54) builds
// the transversely isotropic constants of a vertical symmetry axis from RHO,
// VPV, VPH, VSV, VSH, ETA:
//   c11 = c22 = rho VPH^2   c33 = rho VPV^2   c44 = c55 = rho VSV^2
//   c66 = rho VSH^2         c12 = c11 - 2 c66  c13 = c23 = ETA (c11 - 2 c44)
// and Elastic3D::computeStress (Elastic3D.cpp:106-118) applies them to the
// Voigt strains e = (xx, yy, zz, yz, xz, xy) with engineering shears
// (Elastic3D.cpp:76-82).  Here g[c][a] = d u_c / d x_a.
//
// Isotropic models (VPH = VPV = VP, VSH = VSV = VS, ETA = 1) reduce to
// lambda = rho (VP^2 - 2 VS^2), mu = rho VS^2; the kernels keep that two-
// constant form as their fast path.  Transversely isotropic records hold the
// five independent constants (A, C, F, L, N) = (c11, c33, c13, c44, c66).
#pragma once

namespace salvus {

// Number of folded material constants per point.
template <bool TI>
struct ElasticMat {
  static constexpr int kWords = TI ? 5 : 2;
};

// sigma = C : eps with lambda', mu' (w detJ folded in).
template <typename real>
__device__ __forceinline__ void stress_iso(const real g[3][3], real lam, real mu,
                                           real sig[3][3]) {
  const real tr = g[0][0] + g[1][1] + g[2][2];
  const real sxx = lam * tr + 2 * mu * g[0][0];
  const real syy = lam * tr + 2 * mu * g[1][1];
  const real szz = lam * tr + 2 * mu * g[2][2];
  const real sxy = mu * (g[0][1] + g[1][0]);
  const real sxz = mu * (g[0][2] + g[2][0]);
  const real syz = mu * (g[1][2] + g[2][1]);
  sig[0][0] = sxx; sig[0][1] = sxy; sig[0][2] = sxz;
  sig[1][0] = sxy; sig[1][1] = syy; sig[1][2] = syz;
  sig[2][0] = sxz; sig[2][1] = syz; sig[2][2] = szz;
}

// Transversely isotropic (vertical axis), constants m = (A, C, F, L, N) with
// w detJ folded in; c12 = A - 2 N (Elastic3D.cpp:51).
template <typename real>
__device__ __forceinline__ void stress_ti(const real g[3][3], const real m[5], real sig[3][3]) {
  const real A = m[0], Cc = m[1], F = m[2], L = m[3], Nn = m[4];
  const real c12 = A - 2 * Nn;
  const real e0 = g[0][0], e1 = g[1][1], e2 = g[2][2];
  const real e3 = g[1][2] + g[2][1];  // yz
  const real e4 = g[0][2] + g[2][0];  // xz
  const real e5 = g[0][1] + g[1][0];  // xy
  const real sxx = A * e0 + c12 * e1 + F * e2;
  const real syy = c12 * e0 + A * e1 + F * e2;
  const real szz = F * e0 + F * e1 + Cc * e2;
  const real syz = L * e3, sxz = L * e4, sxy = Nn * e5;
  sig[0][0] = sxx; sig[0][1] = sxy; sig[0][2] = sxz;
  sig[1][0] = sxy; sig[1][1] = syy; sig[1][2] = syz;
  sig[2][0] = sxz; sig[2][1] = syz; sig[2][2] = szz;
}

// FP64 constants of one point from its (P1-interpolated) parameters:
// isotropic (rho, vp, vs) -> (lambda, mu); TI (rho, vpv, vph, vsv, vsh, eta)
// -> (A, C, F, L, N).  Elastic3D.cpp:42-53.
__host__ __device__ inline void elastic_constants_iso(double rho, double vp, double vs,
                                                      double out[2]) {
  const double mu = rho * vs * vs;
  out[0] = rho * vp * vp - 2.0 * mu;
  out[1] = mu;
}
__host__ __device__ inline void elastic_constants_ti(const double p[6], double out[5]) {
  const double rho = p[0], vpv = p[1], vph = p[2], vsv = p[3], vsh = p[4], eta = p[5];
  const double c11 = rho * vph * vph, c33 = rho * vpv * vpv;
  const double c44 = rho * vsv * vsv, c66 = rho * vsh * vsh;
  out[0] = c11;
  out[1] = c33;
  out[2] = eta * (c11 - 2.0 * c44);
  out[3] = c44;
  out[4] = c66;
}

}  // namespace salvus
