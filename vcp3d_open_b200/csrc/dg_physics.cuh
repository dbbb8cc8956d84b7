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

struct FluxParams {
  double mu;          // non-dimensional laminar viscosity
  double tau_pen;     // (p+1)^2 * C_pen (divided by the length scale per face)
  double theta_sym;   // symmetrizing-term parameter
  int riemann;        // 0 Roe, 1 Ismail-Roe
};

// Entropy variables -> rho, u, v, w, p, eKin (ElementClass::VolumeResidual,
// src/ElementClass.cpp:4187-4196).
__device__ __forceinline__ void EntropyToPrim(const double V0, const double V1, const double V2,
                                              const double V3, const double V4, double &rho,
                                              double &u, double &v, double &w, double &p,
                                              double &eKin) {
  const double gm1 = kGam - 1.0;
  const double ov1mg = -1.0 / gm1;
  const double V4Inv = 1.0 / V4;
  u = -V4Inv * V1;
  v = -V4Inv * V2;
  w = -V4Inv * V3;
  eKin = 0.5 * (u * u + v * v + w * w);
  const double s = kGam - gm1 * (V0 - V4 * eKin);
  const double tmp = -V4 * exp(s);
  rho = pow(tmp, ov1mg);
  p = -rho * V4Inv;
}

// Face-state primitive variables as computed inside InviscidFluxesFace
// (src/FluxesFace.cpp:710-728): note the "0.5 * V4 * vTot2" grouping.
__device__ __forceinline__ void FaceStatePrim(const double *V, double &rho, double &u, double &v,
                                              double &w, double &p, double &vTot2) {
  const double gm1 = kGam - 1.0;
  const double ov1mg = -1.0 / gm1;
  const double V4Inv = 1.0 / V[4];
  u = -V4Inv * V[1];
  v = -V4Inv * V[2];
  w = -V4Inv * V[3];
  vTot2 = u * u + v * v + w * w;
  const double s = kGam - gm1 * (V[0] - 0.5 * V[4] * vTot2);
  const double tmp = -V[4] * exp(s);
  rho = pow(tmp, ov1mg);
  p = -V4Inv * rho;
}

// Ismail-Roe entropy-stable flux, entropy-variable branch of InviscidFluxesFace
// (src/FluxesFace.cpp:813-975). Returns the flux times area*weight.
__device__ __forceinline__ void IsmailRoeFlux(const double *VL, const double *VR, const double nx,
                                              const double ny, const double nz, const double Area,
                                              double *f) {
  const double gam = kGam, gm1 = gam - 1.0, ovgm1 = 1.0 / (gam - 1.0);
  const double gp1Ovg = (gam + 1.0) / gam, gm1Ovg = gm1 / gam;
  const double beta = 1.0 / 6.0, alphaMax = 0.0;
  double rhoL, vxL, vyL, vzL, pL, v2L, rhoR, vxR, vyR, vzR, pR, v2R;
  FaceStatePrim(VL, rhoL, vxL, vyL, vzL, pL, v2L);
  FaceStatePrim(VR, rhoR, vxR, vyR, vzR, pR, v2R);
  const double dV0 = VR[0] - VL[0], dV1 = VR[1] - VL[1], dV2 = VR[2] - VL[2];
  const double dV3 = VR[3] - VL[3], dV4 = VR[4] - VL[4];
  const double z0L = sqrt(rhoL / pL), z0R = sqrt(rhoR / pR);
  const double z1L = vxL * z0L, z1R = vxR * z0R;
  const double z2L = vyL * z0L, z2R = vyR * z0R;
  const double z3L = vzL * z0L, z3R = vzR * z0R;
  const double z4L = sqrt(rhoL * pL), z4R = sqrt(rhoR * pR);
  const double z0Avg = 0.5 * (z0L + z0R), z1Avg = 0.5 * (z1L + z1R);
  const double z2Avg = 0.5 * (z2L + z2R), z3Avg = 0.5 * (z3L + z3R);
  const double z4Avg = 0.5 * (z4L + z4R);
  // Logarithmic means with the series expansion for nearly equal states.
  double zeta = z0L / z0R, fz = (zeta - 1.0) / (zeta + 1.0), uz = fz * fz, F;
  if (uz < 0.01)
    F = 1.0 + uz / 3.0 + uz * uz / 5.0 + uz * uz * uz / 7.0 + uz * uz * uz * uz / 9.0;
  else
    F = log(zeta) / (2.0 * fz);
  const double z0LogAvg = z0Avg / F;
  zeta = z4L / z4R; fz = (zeta - 1.0) / (zeta + 1.0); uz = fz * fz;
  if (uz < 0.01)
    F = 1.0 + uz / 3.0 + uz * uz / 5.0 + uz * uz * uz / 7.0 + uz * uz * uz * uz / 9.0;
  else
    F = log(zeta) / (2.0 * fz);
  const double z4LogAvg = z4Avg / F;
  const double oneOvz0Avg = 1.0 / z0Avg;
  const double rhoAvg = z0Avg * z4LogAvg;
  const double p1Avg = oneOvz0Avg * z4Avg;
  const double p2Avg = 0.5 * (gp1Ovg * z4LogAvg / z0LogAvg + gm1Ovg * p1Avg);
  const double vxAvg = oneOvz0Avg * z1Avg, vyAvg = oneOvz0Avg * z2Avg, vzAvg = oneOvz0Avg * z3Avg;
  const double vnAvg = vxAvg * nx + vyAvg * ny + vzAvg * nz;
  const double kinAvg = 0.5 * (vxAvg * vxAvg + vyAvg * vyAvg + vzAvg * vzAvg);
  const double a2Avg = gam * p2Avg / rhoAvg;
  const double aAvg = sqrt(a2Avg);
  const double HAvg = a2Avg * ovgm1 + kinAvg;
  const double EAvg = HAvg - p2Avg / rhoAvg;
  const double ovaAvg = 1.0 / aAvg, ova2Avg = 1.0 / a2Avg;
  double abv1 = rhoAvg * (vxAvg * dV1 + vyAvg * dV2 + vzAvg * dV3);
  double abv2 = abv1 + rhoAvg * (dV0 + HAvg * dV4);
  const double dr = abv1 + rhoAvg * (dV0 + EAvg * dV4);
  const double dru = vxAvg * abv2 + p2Avg * dV1;
  const double drv = vyAvg * abv2 + p2Avg * dV2;
  const double drw = vzAvg * abv2 + p2Avg * dV3;
  const double drE = HAvg * abv1 + rhoAvg * EAvg * (dV0 + HAvg * dV4) + p2Avg * kinAvg * dV4;
  double lam1 = fabs(vnAvg + aAvg), lam2 = fabs(vnAvg - aAvg), lam3 = fabs(vnAvg);
  lam1 *= 0.5 * (1.0 + beta + alphaMax);
  lam2 *= 0.5 * (1.0 + beta + alphaMax);
  lam3 *= 0.5;
  abv1 = 0.5 * (lam1 + lam2);
  abv2 = 0.5 * (lam1 - lam2);
  const double abv3 = abv1 - lam3;
  const double abv4 = gm1 * (kinAvg * dr - vxAvg * dru - vyAvg * drv - vzAvg * drw + drE);
  const double abv5 = nx * dru + ny * drv + nz * drw - vnAvg * dr;
  const double abv6 = abv3 * abv4 * ova2Avg + abv2 * abv5 * ovaAvg;
  const double abv7 = abv2 * abv4 * ovaAvg + abv3 * abv5;
  // factUNorm == 1 for internal faces and the boundary faces handled here.
  double f0 = rhoAvg * vnAvg;
  double f1 = rhoAvg * vnAvg * vxAvg + p1Avg * nx;
  double f2 = rhoAvg * vnAvg * vyAvg + p1Avg * ny;
  double f3 = rhoAvg * vnAvg * vzAvg + p1Avg * nz;
  double f4 = rhoAvg * vnAvg * HAvg;
  f0 -= (lam3 * dr + abv6);
  f1 -= (lam3 * dru + vxAvg * abv6 + nx * abv7);
  f2 -= (lam3 * drv + vyAvg * abv6 + ny * abv7);
  f3 -= (lam3 * drw + vzAvg * abv6 + nz * abv7);
  f4 -= (lam3 * drE + HAvg * abv6 + vnAvg * abv7);
  f[0] = f0 * Area; f[1] = f1 * Area; f[2] = f2 * Area; f[3] = f3 * Area; f[4] = f4 * Area;
}

// Roe flux with entropy fix, entropy-variable branch of InviscidFluxesFace
// (src/FluxesFace.cpp:694-809). halfArea = 0.5 * weight * area.
__device__ __forceinline__ void RoeFlux(const double *VL, const double *VR, const double nx,
                                        const double ny, const double nz, const double halfArea,
                                        double *f) {
  const double gam = kGam, gm1 = gam - 1.0, ovgm1 = 1.0 / (gam - 1.0);
  const double Delta = 0.001;
  double rhoL, vxL, vyL, vzL, pL, v2L, rhoR, vxR, vyR, vzR, pR, v2R;
  FaceStatePrim(VL, rhoL, vxL, vyL, vzL, pL, v2L);
  FaceStatePrim(VR, rhoR, vxR, vyR, vzR, pR, v2R);
  const double rEL = pL * ovgm1 + 0.5 * rhoL * v2L;
  const double rER = pR * ovgm1 + 0.5 * rhoR * v2R;
  const double dr = rhoR - rhoL;
  const double dru = rhoR * vxR - rhoL * vxL;
  const double drv = rhoR * vyR - rhoL * vyL;
  const double drw = rhoR * vzR - rhoL * vzL;
  const double drE = rER - rEL;
  const double zL = sqrt(rhoL), zR = sqrt(rhoR);
  double tmp = 1.0 / (zL + zR);
  const double rHL = rEL + pL, rHR = rER + pR;
  const double uAvg = tmp * (zL * vxL + zR * vxR);
  const double vAvg = tmp * (zL * vyL + zR * vyR);
  const double wAvg = tmp * (zL * vzL + zR * vzR);
  const double HAvg = tmp * (rHL / zL + rHR / zR);
  const double alphaAvg = 0.5 * (uAvg * uAvg + vAvg * vAvg + wAvg * wAvg);
  tmp = gm1 * (HAvg - alphaAvg);
  const double a2Avg = fabs(tmp);
  const double aAvg = sqrt(a2Avg);
  const double vnAvg = uAvg * nx + vAvg * ny + wAvg * nz;
  const double ovaAvg = 1.0 / aAvg, ova2Avg = 1.0 / a2Avg;
  double lam1 = fabs(vnAvg + aAvg), lam2 = fabs(vnAvg - aAvg), lam3 = fabs(vnAvg);
  tmp = Delta * fmax(lam1, lam2);
  lam1 = fmax(lam1, tmp); lam2 = fmax(lam2, tmp); lam3 = fmax(lam3, tmp);
  const double abv1 = 0.5 * (lam1 + lam2);
  const double abv2 = 0.5 * (lam1 - lam2);
  const double abv3 = abv1 - lam3;
  const double abv4 = gm1 * (alphaAvg * dr - uAvg * dru - vAvg * drv - wAvg * drw + drE);
  const double abv5 = nx * dru + ny * drv + nz * drw - vnAvg * dr;
  const double abv6 = abv3 * abv4 * ova2Avg + abv2 * abv5 * ovaAvg;
  const double abv7 = abv2 * abv4 * ovaAvg + abv3 * abv5;
  const double vnL = vxL * nx + vyL * ny + vzL * nz;
  const double vnR = vxR * nx + vyR * ny + vzR * nz;
  const double pa = halfArea * (pL + pR);
  const double fact = halfArea;
  f[0] = fact * (rhoL * vnL + rhoR * vnR - (lam3 * dr + abv6));
  f[1] = fact * (rhoL * vxL * vnL + rhoR * vxR * vnR - (lam3 * dru + uAvg * abv6 + nx * abv7)) + pa * nx;
  f[2] = fact * (rhoL * vyL * vnL + rhoR * vyR * vnR - (lam3 * drv + vAvg * abv6 + ny * abv7)) + pa * ny;
  f[3] = fact * (rhoL * vzL * vnL + rhoR * vzR * vnR - (lam3 * drw + wAvg * abv6 + nz * abv7)) + pa * nz;
  f[4] = fact * (rEL * vnL + rER * vnR + pL * vnL + pR * vnR - (lam3 * drE + HAvg * abv6 + vnAvg * abv7));
}

// Viscous normal flux, interior penalty and symmetrizing fluxes of one face
// point for entropy variables: ViscousFluxesFace (src/FluxesFace.cpp:1290-1651,
// entropy branch, no SGS model, no prescribed heat flux) followed by
// PenAndSymFluxesSymmVar (src/FluxesFace.cpp:1152-1284).
//   VL, VR      left/right entropy variables
//   gx, gy, gz  averaged Cartesian gradients of the entropy variables
//   nnx..nnz    unit normal times factNorm; wf, area: face weight and area
//   tau         penalty parameter (p+1)^2 C_pen / lenScale
// Subtracts the viscous flux from f, adds the penalty terms, and returns the
// Cartesian symmetrizing fluxes in sx, sy, sz (component 0 is zero).
__device__ __forceinline__ void ViscousPenaltySymFlux(
    const double *VL, const double *VR, const double *gx, const double *gy, const double *gz,
    const double nnx, const double nny, const double nnz, const double factNorm, const double wf,
    const double area, const double mu, const double tau, const double thetaSym, double *f,
    double *sx, double *sy, double *sz) {
  const double gm1 = kGam - 1.0, ovgm1 = 1.0 / gm1, ov1mg = -ovgm1;
  const double V1 = 0.5 * (VL[1] + VR[1]);
  const double V2 = 0.5 * (VL[2] + VR[2]), V3 = 0.5 * (VL[3] + VR[3]);
  const double V4 = 0.5 * (VL[4] + VR[4]);
  const double V4Inv = 1.0 / V4;
  const double u = -V4Inv * V1, v = -V4Inv * V2, w = -V4Inv * V3;
  // (rho of the averaged state is only needed by an SGS model.)
  const double dudx = -V4Inv * (gx[1] + u * gx[4]);
  const double dvdx = -V4Inv * (gx[2] + v * gx[4]);
  const double dwdx = -V4Inv * (gx[3] + w * gx[4]);
  const double dudy = -V4Inv * (gy[1] + u * gy[4]);
  const double dvdy = -V4Inv * (gy[2] + v * gy[4]);
  const double dwdy = -V4Inv * (gy[3] + w * gy[4]);
  const double dudz = -V4Inv * (gz[1] + u * gz[4]);
  const double dvdz = -V4Inv * (gz[2] + v * gz[4]);
  const double dwdz = -V4Inv * (gz[3] + w * gz[4]);
  const double fe = -V4Inv * V4Inv * ov1mg;
  const double dedx = fe * gx[4], dedy = fe * gy[4], dedz = fe * gz[4];
  const double dV1 = VL[1] - VR[1], dV2 = VL[2] - VR[2], dV3 = VL[3] - VR[3];
  const double dV4 = VL[4] - VR[4];
  const double pOvRho = -V4Inv;

  // Viscous normal flux (src/FluxesFace.cpp:1565-1614).
  {
    const double Area = factNorm * wf * area;
    const double nx = Area * nnx, ny = Area * nny, nz = Area * nnz;
    const double lamDivVel = kLamOverMu * (dudx + dvdy + dwdz);
    const double muTot = mu + 0.0;
    const double tauxx = muTot * (2.0 * dudx + lamDivVel);
    const double tauyy = muTot * (2.0 * dvdy + lamDivVel);
    const double tauzz = muTot * (2.0 * dwdz + lamDivVel);
    const double tauxy = muTot * (dudy + dvdx);
    const double tauxz = muTot * (dudz + dwdx);
    const double tauyz = muTot * (dvdz + dwdy);
    const double factHeatTot = mu * kFactHFLam + 0.0 * kFactHFTurb;
    const double qx = -factHeatTot * dedx, qy = -factHeatTot * dedy, qz = -factHeatTot * dedz;
    f[1] -= tauxx * nx + tauxy * ny + tauxz * nz;
    f[2] -= tauxy * nx + tauyy * ny + tauyz * nz;
    f[3] -= tauxz * nx + tauyz * ny + tauzz * nz;
    f[4] -= (u * tauxx + v * tauxy + w * tauxz - qx) * nx +
            (u * tauxy + v * tauyy + w * tauyz - qy) * ny +
            (u * tauxz + v * tauyz + w * tauzz - qz) * nz;
  }

  // Penalty and symmetrizing fluxes (src/FluxesFace.cpp:1180-1283).
  const double lam = kLamOverMu, lamp1 = kLamOverMu + 1.0, lamp2 = kLamOverMu + 2.0;
  const double e = pOvRho * ovgm1;
  const double factFlux = pOvRho * wf * area * (mu + 0.0);
  double nx = factFlux * nnx, ny = factFlux * nny, nz = factFlux * nnz;
  const double factHeatFlux = (mu * kFactHFLam + 0.0 * kFactHFTurb) / (mu + 0.0);
  const double abvE = u * u + v * v + w * w + factHeatFlux * e;
  const double K11_11 = lamp2, K11_14 = u * lamp2, K11_22 = 1.0, K11_24 = v, K11_33 = 1.0,
               K11_34 = w, K11_44 = abvE + u * u * lamp1;
  const double K22_11 = 1.0, K22_14 = u, K22_22 = lamp2, K22_24 = v * lamp2, K22_33 = 1.0,
               K22_34 = w, K22_44 = abvE + v * v * lamp1;
  const double K33_11 = 1.0, K33_14 = u, K33_22 = 1.0, K33_24 = v, K33_33 = lamp2,
               K33_34 = w * lamp2, K33_44 = abvE + w * w * lamp1;
  const double K12_12 = lam, K12_14 = v * lam, K12_21 = 1.0, K12_24 = u, K12_41 = v,
               K12_42 = u * lam, K12_44 = u * v * lamp1;
  const double K13_13 = lam, K13_14 = w * lam, K13_31 = 1.0, K13_34 = u, K13_41 = w,
               K13_43 = u * lam, K13_44 = u * w * lamp1;
  const double K23_23 = lam, K23_24 = w * lam, K23_32 = 1.0, K23_34 = v, K23_42 = w,
               K23_43 = v * lam, K23_44 = v * w * lamp1;
  const double un = u * nnx + v * nny + w * nnz;
  const double dVn = dV1 * nnx + dV2 * nny + dV3 * nnz;
  const double ttau = tau * factFlux;
  const double abvMom = lamp1 * (dVn + un * dV4);
  f[1] += ttau * (abvMom * nnx + dV1 + u * dV4);
  f[2] += ttau * (abvMom * nny + dV2 + v * dV4);
  f[3] += ttau * (abvMom * nnz + dV3 + w * dV4);
  f[4] += ttau * (lamp1 * un * dVn + u * dV1 + v * dV2 + w * dV3 + (abvE + lamp1 * un * un) * dV4);
  nx *= 0.5 * thetaSym;
  ny *= 0.5 * thetaSym;
  nz *= 0.5 * thetaSym;
  sx[0] = 0.0;
  sx[1] = -(K11_11 * dV1 + K11_14 * dV4) * nx - (K12_12 * dV2 + K12_14 * dV4) * ny -
          (K13_13 * dV3 + K13_14 * dV4) * nz;
  sx[2] = -(K11_22 * dV2 + K11_24 * dV4) * nx - (K12_21 * dV1 + K12_24 * dV4) * ny;
  sx[3] = -(K11_33 * dV3 + K11_34 * dV4) * nx - (K13_31 * dV1 + K13_34 * dV4) * nz;
  sx[4] = -(K11_14 * dV1 + K11_24 * dV2 + K11_34 * dV3 + K11_44 * dV4) * nx -
          (K12_41 * dV1 + K12_42 * dV2 + K12_44 * dV4) * ny -
          (K13_41 * dV1 + K13_43 * dV3 + K13_44 * dV4) * nz;
  sy[0] = 0.0;
  sy[1] = -(K12_21 * dV2 + K12_41 * dV4) * nx - (K22_11 * dV1 + K22_14 * dV4) * ny;
  sy[2] = -(K12_12 * dV1 + K12_42 * dV4) * nx - (K22_22 * dV2 + K22_24 * dV4) * ny -
          (K23_23 * dV3 + K23_24 * dV4) * nz;
  sy[3] = -(K22_33 * dV3 + K22_34 * dV4) * ny - (K23_32 * dV2 + K23_34 * dV4) * nz;
  sy[4] = -(K12_14 * dV1 + K12_24 * dV2 + K12_44 * dV4) * nx -
          (K22_14 * dV1 + K22_24 * dV2 + K22_34 * dV3 + K22_44 * dV4) * ny -
          (K23_42 * dV2 + K23_43 * dV3 + K23_44 * dV4) * nz;
  sz[0] = 0.0;
  sz[1] = -(K13_31 * dV3 + K13_41 * dV4) * nx - (K33_11 * dV1 + K33_14 * dV4) * nz;
  sz[2] = -(K23_32 * dV3 + K23_42 * dV4) * ny - (K33_22 * dV2 + K33_24 * dV4) * nz;
  sz[3] = -(K13_13 * dV1 + K13_43 * dV4) * nx - (K23_23 * dV2 + K23_43 * dV4) * ny -
          (K33_33 * dV3 + K33_34 * dV4) * nz;
  sz[4] = -(K13_14 * dV1 + K13_34 * dV3 + K13_44 * dV4) * nx -
          (K23_24 * dV2 + K23_34 * dV3 + K23_44 * dV4) * ny -
          (K33_14 * dV1 + K33_24 * dV2 + K33_34 * dV3 + K33_44 * dV4) * nz;
}

}  // namespace vcpg
