// Pointwise physics of the entropy-variable DG discretisation, evaluated per
// integration point by one thread. Each function states the reference routine
// whose arithmetic it follows; the operation order is kept where it matters
// for FP64 agreement.
#pragma once

#include <cuda_runtime.h>

namespace vcpg {

// Gas constants (include/VCP3D_CurviLinear.hpp:174-186).
constexpr double kGam = 1.4;
constexpr double kPrLam = 0.72;
constexpr double kPrTurb = 0.90;
constexpr double kFactHFLam = kGam / kPrLam;    // factHeatFlux_Lam
constexpr double kFactHFTurb = kGam / kPrTurb;  // factHeatFlux_Turb
constexpr double kLamOverMu = -2.0 / 3.0;       // lambdaOverMu
constexpr double kRGas = 287.058;                 // RGas (include/VCP3D_CurviLinear.hpp:177)
constexpr double kCp = kGam * kRGas / (kGam - 1.0);  // Cp

// Math in the compute precision T (double for the FP64 form, float for the mixed form).
__device__ __forceinline__ double Exp(double x) { return exp(x); }
__device__ __forceinline__ float Exp(float x) { return expf(x); }
__device__ __forceinline__ double Log(double x) { return log(x); }
__device__ __forceinline__ double Pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float Pow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ float Log(float x) { return logf(x); }
__device__ __forceinline__ double Sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float Sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double Fabs(double x) { return fabs(x); }
__device__ __forceinline__ float Fabs(float x) { return fabsf(x); }
__device__ __forceinline__ double Fmax(double x, double y) { return fmax(x, y); }
__device__ __forceinline__ float Fmax(float x, float y) { return fmaxf(x, y); }
__device__ __forceinline__ double Fmin(double x, double y) { return fmin(x, y); }
__device__ __forceinline__ float Fmin(float x, float y) { return fminf(x, y); }
__device__ __forceinline__ double Fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float Fma(float a, float b, float c) { return fmaf(a, b, c); }
// Reads an FP64 input (state, metric) from global memory into the compute precision.
template <typename T>
__device__ __forceinline__ T LdT(const double *p) { return T(__ldg(p)); }

// Entropy variables -> rho, u, v, w, p, eKin (ElementClass::VolumeResidual,
// src/ElementClass.cpp:4187-4196).
template <typename T>
__device__ __forceinline__ void EntropyToPrim(const T V0, const T V1, const T V2,
                                              const T V3, const T V4, T &rho,
                                              T &u, T &v, T &w, T &p,
                                              T &eKin) {
  const T gm1 = T(kGam) - T(1.0);
  const T ov1mg = -T(1.0) / gm1;
  const T V4Inv = T(1.0) / V4;
  u = -V4Inv * V1;
  v = -V4Inv * V2;
  w = -V4Inv * V3;
  eKin = T(0.5) * (u * u + v * v + w * w);
  const T s = T(kGam) - gm1 * (V0 - V4 * eKin);
  // rho = (-V4 exp(s))^(-1/(gam-1)) (the reference's POW(-V4*EXP(s), ov1mg)),
  // evaluated as exp(ov1mg (log(-V4) + s)): one exponential and one logarithm.
  rho = Exp(ov1mg * (Log(-V4) + s));
  p = -rho * V4Inv;
}

// Face-state primitive variables as computed inside InviscidFluxesFace
// (src/FluxesFace.cpp:710-728): note the "0.5 * V4 * vTot2" grouping.
template <typename T>
__device__ __forceinline__ void FaceStatePrim(const T *V, T &rho, T &u, T &v,
                                              T &w, T &p, T &vTot2) {
  const T gm1 = T(kGam) - T(1.0);
  const T ov1mg = -T(1.0) / gm1;
  const T V4Inv = T(1.0) / V[4];
  u = -V4Inv * V[1];
  v = -V4Inv * V[2];
  w = -V4Inv * V[3];
  vTot2 = u * u + v * v + w * w;
  const T s = T(kGam) - gm1 * (V[0] - T(0.5) * V[4] * vTot2);
  // rho = (-V4 exp(s))^(-1/(gam-1)), as in EntropyToPrim.
  rho = Exp(ov1mg * (Log(-V[4]) + s));
  p = -V4Inv * rho;
}

// Eddy viscosity of the subgrid-scale models (src/SGSModel.cpp): sgs 1 WALE
// (C_w = 0.325), sgs 2 Vreman (c = 0.07), 0 none. g holds the velocity gradient
// du/dx, dv/dx, dw/dx, du/dy, dv/dy, dw/dy, du/dz, dv/dz, dw/dz; the result is
// rho times the model's kinematic eddy viscosity.
template <typename T>
__device__ __forceinline__ T EddyViscosity(const int sgs, const T lenScale, const T rho,
                                           const T *g) {
  const T third = T(1.0) / T(3.0), epsSmall = T(1.e-30);
  const T dudx = g[0], dvdx = g[1], dwdx = g[2], dudy = g[3], dvdy = g[4], dwdy = g[5];
  const T dudz = g[6], dvdz = g[7], dwdz = g[8];
  if (sgs == 1) {
    const T len = T(0.325) * lenScale, len2 = len * len;
    const T S11 = dudx, S22 = dvdy, S33 = dwdz;
    const T S12 = T(0.5) * (dudy + dvdx), S13 = T(0.5) * (dudz + dwdx), S23 = T(0.5) * (dvdz + dwdy);
    T Sd11 = dudx * dudx + dudy * dvdx + dudz * dwdx;
    T Sd22 = dvdx * dudy + dvdy * dvdy + dvdz * dwdy;
    T Sd33 = dwdx * dudz + dwdy * dvdz + dwdz * dwdz;
    const T Sd12 = T(0.5) * (dudx * dudy + dudy * dvdy + dudz * dwdy + dvdx * dudx + dvdy * dvdx +
                             dvdz * dwdx);
    const T Sd13 = T(0.5) * (dudx * dudz + dudy * dvdz + dudz * dwdz + dwdx * dudx + dwdy * dvdx +
                             dwdz * dwdx);
    const T Sd23 = T(0.5) * (dvdx * dudz + dvdy * dvdz + dvdz * dwdz + dwdx * dudy + dwdy * dvdy +
                             dwdz * dwdy);
    const T thirdTrace = third * (Sd11 + Sd22 + Sd33);
    Sd11 -= thirdTrace;
    Sd22 -= thirdTrace;
    Sd33 -= thirdTrace;
    const T sumS = S11 * S11 + S22 * S22 + S33 * S33 + T(2.0) * (S12 * S12 + S13 * S13 + S23 * S23);
    const T sumSd = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 +
                    T(2.0) * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
    const T sumSdPow3_2 = sumSd * Sqrt(sumSd);
    const T sumSdPow5_4 = Sqrt(sumSdPow3_2 * sumSd);
    const T sumSPow5_2 = sumS * sumS * Sqrt(sumS);
    const T denom = sumSPow5_2 + sumSdPow5_4;
    return rho * (len2 * sumSdPow3_2 / Fmax(denom, epsSmall));
  }
  if (sgs == 2) {
    const T len2 = lenScale * lenScale;
    T a11 = dudx, a22 = dvdy, a33 = dwdz;
    const T tmp = third * (a11 + a22 + a33);
    a11 -= tmp;
    a22 -= tmp;
    a33 -= tmp;
    const T a12 = dudy, a13 = dudz, a23 = dvdz, a21 = dvdx, a31 = dwdx, a32 = dwdy;
    const T b11 = len2 * (a11 * a11 + a12 * a12 + a13 * a13);
    const T b12 = len2 * (a11 * a21 + a12 * a22 + a13 * a23);
    const T b13 = len2 * (a11 * a31 + a12 * a32 + a13 * a33);
    const T b22 = len2 * (a21 * a21 + a22 * a22 + a23 * a23);
    const T b23 = len2 * (a21 * a31 + a22 * a32 + a23 * a33);
    const T b33 = len2 * (a31 * a31 + a32 * a32 + a33 * a33);
    T B = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
    B = (B + Fabs(B)) * T(0.5);
    const T denom = a11 * a11 + a22 * a22 + a33 * a33 + a12 * a12 + a13 * a13 + a23 * a23 +
                    a21 * a21 + a31 * a31 + a32 * a32;
    return rho * T(0.07) * Sqrt(B / Fmax(denom, epsSmall));
  }
  return T(0.0);
}

// Ismail-Roe entropy-stable flux, entropy-variable branch of InviscidFluxesFace
// (src/FluxesFace.cpp:813-975). Returns the flux times area*weight.
template <typename T>
__device__ __forceinline__ void IsmailRoeFlux(const T *VL, const T *VR, const T nx,
                                              const T ny, const T nz, const T Area,
                                              T *f, const T factU = T(1.0)) {
  const T gam = T(kGam), gm1 = gam - T(1.0), ovgm1 = T(1.0) / (gam - T(1.0));
  const T gp1Ovg = (gam + T(1.0)) / gam, gm1Ovg = gm1 / gam;
  const T beta = T(1.0) / T(6.0), alphaMax = T(0.0);
  T rhoL, vxL, vyL, vzL, pL, v2L, rhoR, vxR, vyR, vzR, pR, v2R;
  FaceStatePrim(VL, rhoL, vxL, vyL, vzL, pL, v2L);
  FaceStatePrim(VR, rhoR, vxR, vyR, vzR, pR, v2R);
  const T dV0 = VR[0] - VL[0], dV1 = VR[1] - VL[1], dV2 = VR[2] - VL[2];
  const T dV3 = VR[3] - VL[3], dV4 = VR[4] - VL[4];
  const T z0L = Sqrt(rhoL / pL), z0R = Sqrt(rhoR / pR);
  const T z1L = vxL * z0L, z1R = vxR * z0R;
  const T z2L = vyL * z0L, z2R = vyR * z0R;
  const T z3L = vzL * z0L, z3R = vzR * z0R;
  const T z4L = Sqrt(rhoL * pL), z4R = Sqrt(rhoR * pR);
  const T z0Avg = T(0.5) * (z0L + z0R), z1Avg = T(0.5) * (z1L + z1R);
  const T z2Avg = T(0.5) * (z2L + z2R), z3Avg = T(0.5) * (z3L + z3R);
  const T z4Avg = T(0.5) * (z4L + z4R);
  // Logarithmic means with the series expansion for nearly equal states.
  T zeta = z0L / z0R, fz = (zeta - T(1.0)) / (zeta + T(1.0)), uz = fz * fz, F;
  if (uz < T(0.01))
    F = T(1.0) + uz / T(3.0) + uz * uz / T(5.0) + uz * uz * uz / T(7.0) + uz * uz * uz * uz / T(9.0);
  else
    F = Log(zeta) / (T(2.0) * fz);
  const T z0LogAvg = z0Avg / F;
  zeta = z4L / z4R; fz = (zeta - T(1.0)) / (zeta + T(1.0)); uz = fz * fz;
  if (uz < T(0.01))
    F = T(1.0) + uz / T(3.0) + uz * uz / T(5.0) + uz * uz * uz / T(7.0) + uz * uz * uz * uz / T(9.0);
  else
    F = Log(zeta) / (T(2.0) * fz);
  const T z4LogAvg = z4Avg / F;
  const T oneOvz0Avg = T(1.0) / z0Avg;
  const T rhoAvg = z0Avg * z4LogAvg;
  const T p1Avg = oneOvz0Avg * z4Avg;
  const T p2Avg = T(0.5) * (gp1Ovg * z4LogAvg / z0LogAvg + gm1Ovg * p1Avg);
  const T vxAvg = oneOvz0Avg * z1Avg, vyAvg = oneOvz0Avg * z2Avg, vzAvg = oneOvz0Avg * z3Avg;
  const T vnAvg = vxAvg * nx + vyAvg * ny + vzAvg * nz;
  const T kinAvg = T(0.5) * (vxAvg * vxAvg + vyAvg * vyAvg + vzAvg * vzAvg);
  const T a2Avg = gam * p2Avg / rhoAvg;
  const T aAvg = Sqrt(a2Avg);
  const T HAvg = a2Avg * ovgm1 + kinAvg;
  const T EAvg = HAvg - p2Avg / rhoAvg;
  const T ovaAvg = T(1.0) / aAvg, ova2Avg = T(1.0) / a2Avg;
  T abv1 = rhoAvg * (vxAvg * dV1 + vyAvg * dV2 + vzAvg * dV3);
  T abv2 = abv1 + rhoAvg * (dV0 + HAvg * dV4);
  const T dr = abv1 + rhoAvg * (dV0 + EAvg * dV4);
  const T dru = vxAvg * abv2 + p2Avg * dV1;
  const T drv = vyAvg * abv2 + p2Avg * dV2;
  const T drw = vzAvg * abv2 + p2Avg * dV3;
  const T drE = HAvg * abv1 + rhoAvg * EAvg * (dV0 + HAvg * dV4) + p2Avg * kinAvg * dV4;
  T lam1 = Fabs(vnAvg + aAvg), lam2 = Fabs(vnAvg - aAvg), lam3 = Fabs(vnAvg);
  lam1 *= T(0.5) * (T(1.0) + beta + alphaMax);
  lam2 *= T(0.5) * (T(1.0) + beta + alphaMax);
  lam3 *= T(0.5);
  abv1 = T(0.5) * (lam1 + lam2);
  abv2 = T(0.5) * (lam1 - lam2);
  const T abv3 = abv1 - lam3;
  const T abv4 = gm1 * (kinAvg * dr - vxAvg * dru - vyAvg * drv - vzAvg * drw + drE);
  const T abv5 = nx * dru + ny * drv + nz * drw - vnAvg * dr;
  const T abv6 = abv3 * abv4 * ova2Avg + abv2 * abv5 * ovaAvg;
  const T abv7 = abv2 * abv4 * ovaAvg + abv3 * abv5;
  // factU (the reference's factUNorm): 1 for internal faces and open boundaries,
  // 0 for walls (no mass and convective transport through the face).
  T f0 = factU * rhoAvg * vnAvg;
  T f1 = factU * rhoAvg * vnAvg * vxAvg + p1Avg * nx;
  T f2 = factU * rhoAvg * vnAvg * vyAvg + p1Avg * ny;
  T f3 = factU * rhoAvg * vnAvg * vzAvg + p1Avg * nz;
  T f4 = factU * rhoAvg * vnAvg * HAvg;
  f0 -= factU * (lam3 * dr + abv6);
  f1 -= factU * (lam3 * dru + vxAvg * abv6 + nx * abv7);
  f2 -= factU * (lam3 * drv + vyAvg * abv6 + ny * abv7);
  f3 -= factU * (lam3 * drw + vzAvg * abv6 + nz * abv7);
  f4 -= factU * (lam3 * drE + HAvg * abv6 + vnAvg * abv7);
  f[0] = f0 * Area; f[1] = f1 * Area; f[2] = f2 * Area; f[3] = f3 * Area; f[4] = f4 * Area;
}

// Roe flux with entropy fix, entropy-variable branch of InviscidFluxesFace
// (src/FluxesFace.cpp:694-809). halfArea = 0.5 * weight * area.
template <typename T>
__device__ __forceinline__ void RoeFlux(const T *VL, const T *VR, const T nx,
                                        const T ny, const T nz, const T halfArea,
                                        T *f, const T factU = T(1.0)) {
  const T gam = T(kGam), gm1 = gam - T(1.0), ovgm1 = T(1.0) / (gam - T(1.0));
  const T Delta = T(0.001);
  T rhoL, vxL, vyL, vzL, pL, v2L, rhoR, vxR, vyR, vzR, pR, v2R;
  FaceStatePrim(VL, rhoL, vxL, vyL, vzL, pL, v2L);
  FaceStatePrim(VR, rhoR, vxR, vyR, vzR, pR, v2R);
  const T rEL = pL * ovgm1 + T(0.5) * rhoL * v2L;
  const T rER = pR * ovgm1 + T(0.5) * rhoR * v2R;
  const T dr = rhoR - rhoL;
  const T dru = rhoR * vxR - rhoL * vxL;
  const T drv = rhoR * vyR - rhoL * vyL;
  const T drw = rhoR * vzR - rhoL * vzL;
  const T drE = rER - rEL;
  const T zL = Sqrt(rhoL), zR = Sqrt(rhoR);
  T tmp = T(1.0) / (zL + zR);
  const T rHL = rEL + pL, rHR = rER + pR;
  const T uAvg = tmp * (zL * vxL + zR * vxR);
  const T vAvg = tmp * (zL * vyL + zR * vyR);
  const T wAvg = tmp * (zL * vzL + zR * vzR);
  const T HAvg = tmp * (rHL / zL + rHR / zR);
  const T alphaAvg = T(0.5) * (uAvg * uAvg + vAvg * vAvg + wAvg * wAvg);
  tmp = gm1 * (HAvg - alphaAvg);
  const T a2Avg = Fabs(tmp);
  const T aAvg = Sqrt(a2Avg);
  const T vnAvg = uAvg * nx + vAvg * ny + wAvg * nz;
  const T ovaAvg = T(1.0) / aAvg, ova2Avg = T(1.0) / a2Avg;
  T lam1 = Fabs(vnAvg + aAvg), lam2 = Fabs(vnAvg - aAvg), lam3 = Fabs(vnAvg);
  tmp = Delta * Fmax(lam1, lam2);
  lam1 = Fmax(lam1, tmp); lam2 = Fmax(lam2, tmp); lam3 = Fmax(lam3, tmp);
  const T abv1 = T(0.5) * (lam1 + lam2);
  const T abv2 = T(0.5) * (lam1 - lam2);
  const T abv3 = abv1 - lam3;
  const T abv4 = gm1 * (alphaAvg * dr - uAvg * dru - vAvg * drv - wAvg * drw + drE);
  const T abv5 = nx * dru + ny * drv + nz * drw - vnAvg * dr;
  const T abv6 = abv3 * abv4 * ova2Avg + abv2 * abv5 * ovaAvg;
  const T abv7 = abv2 * abv4 * ovaAvg + abv3 * abv5;
  const T vnL = vxL * nx + vyL * ny + vzL * nz;
  const T vnR = vxR * nx + vyR * ny + vzR * nz;
  const T pa = halfArea * (pL + pR);
  const T fact = factU * halfArea;
  f[0] = fact * (rhoL * vnL + rhoR * vnR - (lam3 * dr + abv6));
  f[1] = fact * (rhoL * vxL * vnL + rhoR * vxR * vnR - (lam3 * dru + uAvg * abv6 + nx * abv7)) + pa * nx;
  f[2] = fact * (rhoL * vyL * vnL + rhoR * vyR * vnR - (lam3 * drv + vAvg * abv6 + ny * abv7)) + pa * ny;
  f[3] = fact * (rhoL * vzL * vnL + rhoR * vzR * vnR - (lam3 * drw + wAvg * abv6 + nz * abv7)) + pa * nz;
  f[4] = fact * (rEL * vnL + rER * vnR + pL * vnL + pR * vnR - (lam3 * drE + HAvg * abv6 + vnAvg * abv7));
}

// Viscous normal flux, interior penalty and symmetrizing fluxes of one face
// point for entropy variables: ViscousFluxesFace (src/FluxesFace.cpp:1290-1651,
// entropy branch, no SGS model) followed by PenAndSymFluxesSymmVar
// (src/FluxesFace.cpp:1152-1284). hfMult = 0 for a wall with a prescribed heat
// flux (the conductive terms vanish) and qWallArea = w * area * q_wall is then
// added to the energy flux between the two, as the reference does.
//   VL, VR      left/right entropy variables
//   gx, gy, gz  averaged Cartesian gradients of the entropy variables
//   nnx..nnz    unit normal times factNorm (-1 when the own element is on the
//               right of a boundary face); wf, area: face weight and area
//   tau         penalty parameter (p+1)^2 C_pen / lenScale
// Subtracts the viscous flux from f, adds the penalty terms, and returns the
// Cartesian symmetrizing fluxes in sx, sy, sz (component 0 is zero).
template <typename T>
__device__ __forceinline__ void ViscousPenaltySymFlux(
    const T *VL, const T *VR, const T *gx, const T *gy, const T *gz,
    const T nnx, const T nny, const T nnz, const T wf,
    const T area, const T mu, const T tau, const T thetaSym, T *f,
    T *sx, T *sy, T *sz, const T hfMult = T(1.0), const T qWallArea = T(0.0),
    const int sgs = 0, const T lenLES = T(0.0), T *eddyOut = nullptr,
    T *viscForce = nullptr) {
  const T factHFLam = hfMult * T(kFactHFLam), factHFTurb = hfMult * T(kFactHFTurb);
  const T gm1 = T(kGam) - T(1.0), ovgm1 = T(1.0) / gm1, ov1mg = -ovgm1;
  const T V1 = T(0.5) * (VL[1] + VR[1]);
  const T V2 = T(0.5) * (VL[2] + VR[2]), V3 = T(0.5) * (VL[3] + VR[3]);
  const T V4 = T(0.5) * (VL[4] + VR[4]);
  const T V4Inv = T(1.0) / V4;
  const T u = -V4Inv * V1, v = -V4Inv * V2, w = -V4Inv * V3;
  const T dudx = -V4Inv * (gx[1] + u * gx[4]);
  const T dvdx = -V4Inv * (gx[2] + v * gx[4]);
  const T dwdx = -V4Inv * (gx[3] + w * gx[4]);
  const T dudy = -V4Inv * (gy[1] + u * gy[4]);
  const T dvdy = -V4Inv * (gy[2] + v * gy[4]);
  const T dwdy = -V4Inv * (gy[3] + w * gy[4]);
  const T dudz = -V4Inv * (gz[1] + u * gz[4]);
  const T dvdz = -V4Inv * (gz[2] + v * gz[4]);
  const T dwdz = -V4Inv * (gz[3] + w * gz[4]);
  // Eddy viscosity of the averaged state (ViscousFluxesFace step 2).
  T eddy = T(0.0);
  if (sgs) {
    const T V0 = T(0.5) * (VL[0] + VR[0]);
    const T eKin = T(0.5) * (u * u + v * v + w * w);
    const T s = T(kGam) - gm1 * (V0 - V4 * eKin);
    const T rho = Pow(-V4 * Exp(s), ov1mg);
    const T gv[9] = {dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz};
    eddy = EddyViscosity(sgs, lenLES, rho, gv);
    if (eddyOut) *eddyOut = eddy;
  }
  const T fe = -V4Inv * V4Inv * ov1mg;
  const T dedx = fe * gx[4], dedy = fe * gy[4], dedz = fe * gz[4];
  const T dV1 = VL[1] - VR[1], dV2 = VL[2] - VR[2], dV3 = VL[3] - VR[3];
  const T dV4 = VL[4] - VR[4];
  const T pOvRho = -V4Inv;

  // Viscous normal flux (src/FluxesFace.cpp:1565-1614): the reference scales the
  // metric normal by factNorm * w * area; nnx already carries factNorm.
  {
    const T Area = wf * area;
    const T nx = Area * nnx, ny = Area * nny, nz = Area * nnz;
    const T lamDivVel = T(kLamOverMu) * (dudx + dvdy + dwdz);
    const T muTot = mu + eddy;
    const T tauxx = muTot * (T(2.0) * dudx + lamDivVel);
    const T tauyy = muTot * (T(2.0) * dvdy + lamDivVel);
    const T tauzz = muTot * (T(2.0) * dwdz + lamDivVel);
    const T tauxy = muTot * (dudy + dvdx);
    const T tauxz = muTot * (dudz + dwdx);
    const T tauyz = muTot * (dvdz + dwdy);
    const T factHeatTot = mu * factHFLam + eddy * factHFTurb;
    const T qx = -factHeatTot * dedx, qy = -factHeatTot * dedy, qz = -factHeatTot * dedz;
    f[1] -= tauxx * nx + tauxy * ny + tauxz * nz;
    f[2] -= tauxy * nx + tauyy * ny + tauyz * nz;
    f[3] -= tauxz * nx + tauyz * ny + tauzz * nz;
    if (viscForce) {
      // Viscous wall force of the point (src/FluxesFace.cpp:1590-1612).
      viscForce[0] = -(tauxx * nx + tauxy * ny + tauxz * nz);
      viscForce[1] = -(tauxy * nx + tauyy * ny + tauyz * nz);
      viscForce[2] = -(tauxz * nx + tauyz * ny + tauzz * nz);
    }
    f[4] -= (u * tauxx + v * tauxy + w * tauxz - qx) * nx +
            (u * tauxy + v * tauyy + w * tauyz - qy) * ny +
            (u * tauxz + v * tauyz + w * tauzz - qz) * nz;
    if (hfMult == T(0.0)) f[4] += qWallArea;
  }

  // Penalty and symmetrizing fluxes (src/FluxesFace.cpp:1180-1283).
  const T lam = T(kLamOverMu), lamp1 = T(kLamOverMu) + T(1.0), lamp2 = T(kLamOverMu) + T(2.0);
  const T e = pOvRho * ovgm1;
  const T factFlux = pOvRho * wf * area * (mu + eddy);
  T nx = factFlux * nnx, ny = factFlux * nny, nz = factFlux * nnz;
  const T factHeatFlux = (mu * factHFLam + eddy * factHFTurb) / (mu + eddy);
  const T abvE = u * u + v * v + w * w + factHeatFlux * e;
  const T K11_11 = lamp2, K11_14 = u * lamp2, K11_22 = T(1.0), K11_24 = v, K11_33 = T(1.0),
               K11_34 = w, K11_44 = abvE + u * u * lamp1;
  const T K22_11 = T(1.0), K22_14 = u, K22_22 = lamp2, K22_24 = v * lamp2, K22_33 = T(1.0),
               K22_34 = w, K22_44 = abvE + v * v * lamp1;
  const T K33_11 = T(1.0), K33_14 = u, K33_22 = T(1.0), K33_24 = v, K33_33 = lamp2,
               K33_34 = w * lamp2, K33_44 = abvE + w * w * lamp1;
  const T K12_12 = lam, K12_14 = v * lam, K12_21 = T(1.0), K12_24 = u, K12_41 = v,
               K12_42 = u * lam, K12_44 = u * v * lamp1;
  const T K13_13 = lam, K13_14 = w * lam, K13_31 = T(1.0), K13_34 = u, K13_41 = w,
               K13_43 = u * lam, K13_44 = u * w * lamp1;
  const T K23_23 = lam, K23_24 = w * lam, K23_32 = T(1.0), K23_34 = v, K23_42 = w,
               K23_43 = v * lam, K23_44 = v * w * lamp1;
  const T un = u * nnx + v * nny + w * nnz;
  const T dVn = dV1 * nnx + dV2 * nny + dV3 * nnz;
  const T ttau = tau * factFlux;
  const T abvMom = lamp1 * (dVn + un * dV4);
  f[1] += ttau * (abvMom * nnx + dV1 + u * dV4);
  f[2] += ttau * (abvMom * nny + dV2 + v * dV4);
  f[3] += ttau * (abvMom * nnz + dV3 + w * dV4);
  f[4] += ttau * (lamp1 * un * dVn + u * dV1 + v * dV2 + w * dV3 + (abvE + lamp1 * un * un) * dV4);
  nx *= T(0.5) * thetaSym;
  ny *= T(0.5) * thetaSym;
  nz *= T(0.5) * thetaSym;
  sx[0] = T(0.0);
  sx[1] = -(K11_11 * dV1 + K11_14 * dV4) * nx - (K12_12 * dV2 + K12_14 * dV4) * ny -
          (K13_13 * dV3 + K13_14 * dV4) * nz;
  sx[2] = -(K11_22 * dV2 + K11_24 * dV4) * nx - (K12_21 * dV1 + K12_24 * dV4) * ny;
  sx[3] = -(K11_33 * dV3 + K11_34 * dV4) * nx - (K13_31 * dV1 + K13_34 * dV4) * nz;
  sx[4] = -(K11_14 * dV1 + K11_24 * dV2 + K11_34 * dV3 + K11_44 * dV4) * nx -
          (K12_41 * dV1 + K12_42 * dV2 + K12_44 * dV4) * ny -
          (K13_41 * dV1 + K13_43 * dV3 + K13_44 * dV4) * nz;
  sy[0] = T(0.0);
  sy[1] = -(K12_21 * dV2 + K12_41 * dV4) * nx - (K22_11 * dV1 + K22_14 * dV4) * ny;
  sy[2] = -(K12_12 * dV1 + K12_42 * dV4) * nx - (K22_22 * dV2 + K22_24 * dV4) * ny -
          (K23_23 * dV3 + K23_24 * dV4) * nz;
  sy[3] = -(K22_33 * dV3 + K22_34 * dV4) * ny - (K23_32 * dV2 + K23_34 * dV4) * nz;
  sy[4] = -(K12_14 * dV1 + K12_24 * dV2 + K12_44 * dV4) * nx -
          (K22_14 * dV1 + K22_24 * dV2 + K22_34 * dV3 + K22_44 * dV4) * ny -
          (K23_42 * dV2 + K23_43 * dV3 + K23_44 * dV4) * nz;
  sz[0] = T(0.0);
  sz[1] = -(K13_31 * dV3 + K13_41 * dV4) * nx - (K33_11 * dV1 + K33_14 * dV4) * nz;
  sz[2] = -(K23_32 * dV3 + K23_42 * dV4) * ny - (K33_22 * dV2 + K33_24 * dV4) * nz;
  sz[3] = -(K13_13 * dV1 + K13_43 * dV4) * nx - (K23_23 * dV2 + K23_43 * dV4) * ny -
          (K33_33 * dV3 + K33_34 * dV4) * nz;
  sz[4] = -(K13_14 * dV1 + K13_34 * dV3 + K13_44 * dV4) * nx -
          (K23_24 * dV2 + K23_34 * dV3 + K23_44 * dV4) * ny -
          (K33_14 * dV1 + K33_24 * dV2 + K33_34 * dV3 + K33_44 * dV4) * nz;
}

}  // namespace vcpg
