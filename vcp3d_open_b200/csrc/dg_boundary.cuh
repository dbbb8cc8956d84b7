// Characteristic (PC-NSCBC) boundary faces, always in FP64 (also in the mixed
// form). Two kernels run before every residual of a block with open boundaries:
//
//   BoundaryTraceKernel  one CTA per boundary face: the element's trace on the
//                        face (value and the three parametric derivatives, the
//                        TPSAG[IJK] contractions) and its area-weighted projected
//                        Mach number (WeightedMachElement, src/BoundaryState.cpp:935-994);
//   BoundaryFluxKernel   one CTA per boundary face: the boundary-averaged Mach
//                        number of its block face (SolverClass::AverageDataNSCBC,
//                        src/SolverClass.cpp:2492-2581), the boundary state and
//                        gradient (ConvertEntropyToPrimitive, the outflow / static
//                        / total inflow LODI corrections and ReconstructBoundaryStateAndGradient,
//                        src/BoundaryState.cpp:1002-1289, 1300-1568, 1579-1847), and
//                        the face fluxes of FluxesBoundaryFace (src/FluxesFace.cpp:16-214).
//
// The fluxes are written per boundary face in the roles the residual kernel's
// face distribution consumes: [0] fast-axis symmetrizing flux, [1] normal flux
// (the contribution to the own element), [2] face-normal symmetrizing flux,
// [3] slow-axis symmetrizing flux, each [5][M^2].
#pragma once

#include <cuda_runtime.h>

#include "dg_physics.cuh"
#include "dg_residual.cuh"
#include "dg_tensor.cuh"
#include "open_boundary.h"

namespace vcpg {

struct BoundaryArgs {
  const double *sol;           // [nE][5][K^3]
  const double *face_metric;   // [nE][6][13][M^2]
  const double *elem_scalars;  // [nE][15]
  const int *bface;            // [nB][kBfStride]
  const double *bpresc;        // [nB][kPrescStride]
  const double *pc;            // [M^2][M^2]
  const double *dlq;           // [M][M]
  double *btrace;              // [nB][4][5][M^2]: value, d/dr, d/ds, d/dt
  double *bmach;               // [nB] area-weighted projected Mach number
  double *bmach_local;         // [nB] the same averaged over the face's own area
  // Optional [nB]: per face, the outlet's element-local Mach number (the value of
  // its subface's last face, which a partitioned block may hold on another
  // rank); null: bmach_local of the face's kBfLast row.
  const double *bmach_last;
  // Optional [6]: per block face, the sum of the weights over the whole block
  // (a partitioned block sums across its slabs); null: this list's own faces.
  const double *bmach_sums;
  double *bflux;               // [nB][4][5][M^2]
  int nB;
  double mu, tau_num, theta_sym;
  int riemann, metric_compat;
  int sgs;                     // enum vcpg_sgs
  unsigned long long *eddymax; // optional: bits of the max eddy viscosity
  double *bforce;              // optional [nB][6]: pressure (0-2) and viscous (3-5)
                               // force of each wall face, monitoring only
  const BlockFaceCfg *cfgs;    // [nCases][6] per case and block face
  // Several cases per launch (null case_state: one case): the case slot is entry
  // kBfCase of the boundary-face row; only faces of cases in state `require` run.
  const int *case_state;
  const double *case_par;      // [nCases][kCasePar]
  int require;
};

// True when boundary face row bf belongs to a case this launch processes.
__device__ __forceinline__ bool BoundaryFaceActive(const BoundaryArgs &a, const int *bf) {
  if (!a.case_state) return true;
  const int c = bf[kBfCase];
  return c >= 0 && a.case_state[c] == a.require;
}

__device__ __forceinline__ int BFastParam(const int d) { return d == 0 ? 1 : 0; }

// Shared memory of BoundaryTraceKernel in doubles; dynamic above the 48 KB of
// static shared memory (degrees 7-9).
template <int K, int M> struct BoundaryTraceSmem {
  static constexpr int N = 5 * K * K * K + 10 * K * K + 15 * K * M + 22 * M * M;
  static constexpr bool DYN = N * 8 > 48 * 1024;
};

template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) BoundaryTraceKernel(const BoundaryArgs a) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K, K2 = K * K, M2 = M * M;
  using SM = BoundaryTraceSmem<K, M>;
  __shared__ double s_static[SM::DYN ? 1 : SM::N];
  extern __shared__ __align__(16) double sm_bt[];
  double *s_sol = SM::DYN ? sm_bt : s_static;
  double *s_bn = s_sol + 5 * KD, *s_bnd = s_bn + 5 * K2;
  double *s_t1a = s_bnd + 5 * K2, *s_t1b = s_t1a + 5 * K * M, *s_t1c = s_t1b + 5 * K * M;
  double *s_tr = s_t1c + 5 * K * M, *s_w = s_tr + 4 * 5 * M2;
  const int b = blockIdx.x;
  if (b >= a.nB) return;
  const int *bf = a.bface + b * kBfStride;
  if (!BoundaryFaceActive(a, bf)) return;
  const int e = bf[kBfElem], f = bf[kBfFace], d = f / 2, side = f % 2;
  const double *src = a.sol + (size_t)e * 5 * KD;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = src[i];
  __syncthreads();
  // Face-normal evaluation (first stage of TPSAG[IJK]); face arrays [slow][fast].
  for (int line = threadIdx.x; line < 5 * K2; line += NT) {
    const int v = line / K2, r2 = line - v * K2, sl = r2 / K, fa = r2 - sl * K;
    int base, ns;
    if (d == 0) { base = sl * K2 + fa * K; ns = 1; }
    else if (d == 1) { base = sl * K2 + fa; ns = K; }
    else { base = sl * K + fa; ns = K2; }
    const double *bsrc = s_sol + v * KD + base;
    double a0 = 0.0, d0 = 0.0;
#pragma unroll
    for (int n = 0; n < K; ++n) {
      const double x = bsrc[n * ns];
      a0 = fma(Ops<SLOT>().face[side * K + n], x, a0);
      d0 = fma(Ops<SLOT>().dface[side * K + n], x, d0);
    }
    s_bn[line] = a0;
    s_bnd[line] = d0;
  }
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 0, 5, K, K, 1, K, M, false>(s_bn, s_t1a);
  Contract<NT, SLOT, K, M, kDLeg, 0, 5, K, K, 1, K, M, false>(s_bn, s_t1b);
  Contract<NT, SLOT, K, M, kLeg, 0, 5, K, K, 1, K, M, false>(s_bnd, s_t1c);
  __syncthreads();
  // Slow axis: value, slow derivative (from t1a), fast derivative (t1b), normal (t1c).
  const int pFast = BFastParam(d), pSlow = 3 - d - pFast;
  Contract<NT, SLOT, K, M, kLeg, 1, 5, M, K, 1, K, M, false>(s_t1a, s_tr);
  Contract<NT, SLOT, K, M, kDLeg, 1, 5, M, K, 1, K, M, false>(s_t1a, s_tr + (1 + pSlow) * 5 * M2);
  Contract<NT, SLOT, K, M, kLeg, 1, 5, M, K, 1, K, M, false>(s_t1b, s_tr + (1 + pFast) * 5 * M2);
  Contract<NT, SLOT, K, M, kLeg, 1, 5, M, K, 1, K, M, false>(s_t1c, s_tr + (1 + d) * 5 * M2);
  __syncthreads();
  double *dst = a.btrace + (size_t)b * 4 * 5 * M2;
  for (int i = threadIdx.x; i < 4 * 5 * M2; i += NT) dst[i] = s_tr[i];
  // Area-weighted Mach number projected on the normal parametric direction, and
  // its average over the element face (BCStandardCharacteristicSubfaceClass::
  // WeightedMachElement, src/BoundaryState.cpp:935-994).
  const double *fm = a.face_metric + ((size_t)e * 6 + f) * 13 * M2;
  const int I0 = 4 + 3 * bf[kBfGrad];
  for (int l = threadIdx.x; l < M2; l += NT) {
    const double magn = fm[3 * M2 + l];
    const double wts = Ops<SLOT>().w[l % M] * Ops<SLOT>().w[l / M];
    const double rrx = fm[I0 * M2 + l], rry = fm[(I0 + 1) * M2 + l], rrz = fm[(I0 + 2) * M2 + l];
    const double magrr = sqrt(rrx * rrx + rry * rry + rrz * rrz);
    const double V4Inv = 1.0 / s_tr[4 * M2 + l];
    const double u = -V4Inv * s_tr[1 * M2 + l], v = -V4Inv * s_tr[2 * M2 + l],
                 w = -V4Inv * s_tr[3 * M2 + l];
    const double aa = sqrt(-kGam * V4Inv);
    const double urr = (u * rrx + v * rry + w * rrz) / magrr;
    s_w[l] = wts * magn * (urr / aa);
    s_w[M2 + l] = wts * magn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // Only characteristic faces enter the boundary average (the weighted Mach
    // number of the other subfaces is zero, SubfaceBaseClass::WeightedMachElement).
    double m = 0.0, area = 0.0;
    for (int l = 0; l < M2; ++l) {
      m += s_w[l];
      area += s_w[M2 + l];
    }
    a.bmach[b] = bf[kBfType] < VCPG_BC_WALL_HEAT_FLUX ? m : 0.0;
    if (a.bmach_local) a.bmach_local[b] = m / area;
  }
}

// Fluxes of one boundary face whose condition is a boundary state
// (FluxesBoundaryFace, src/FluxesFace.cpp:16-214, without wall model or NSCBC):
// the Cartesian gradient of the interior state (metric indexed as in the
// parity mode), the right state of the subface's ComputeBoundaryState
// (src/BoundaryState.cpp:124-828, entropy-variable branches), the Riemann flux
// with the wall factor (0 on walls), the viscous, penalty and symmetrizing fluxes
// with the interior gradient (heat-flux walls: no conduction, the prescribed
// flux added), and the four distribution inputs per face point.
template <int K, int M, int NT>
__device__ __forceinline__ void WeakBoundaryFlux(const BoundaryArgs &a, const int b,
                                                 const int e, const int f, const int type,
                                                 const double mu, const double *fm,
                                                 const double *tr, const double *pres) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int M2 = M * M;
  const int d = f / 2;
  const double factNorm = (f % 2 == 0) ? -1.0 : 1.0;
  const double gm1 = kGam - 1.0, ovgm1 = 1.0 / gm1, govgm1 = kGam * ovgm1, ovg = 1.0 / kGam;
  const double lenScale = a.elem_scalars[(size_t)e * 15 + d];
  double *out = a.bflux + (size_t)b * 4 * 5 * M2;
  const int pFast = BFastParam(d), pSlow = 3 - d - pFast;
  const bool forces = a.bforce && (type == VCPG_BC_WALL_HEAT_FLUX ||
                                   type == VCPG_BC_WALL_ISOTHERMAL ||
                                   type == VCPG_BC_WALL_INVISCID);
  double force[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int l = threadIdx.x; l < M2; l += NT) {
    const int li = l / M, lj = l - li * M;
    double VL[5], VR[5], gx[5], gy[5], gz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      VL[n] = tr[n * M2 + l];
      const int mi = a.metric_compat ? (n < M2 ? n : 0) : l;
      const double dvdr = tr[(5 + n) * M2 + l], dvds = tr[(10 + n) * M2 + l],
                   dvdt = tr[(15 + n) * M2 + l];
      gx[n] = dvdr * fm[4 * M2 + mi] + dvds * fm[7 * M2 + mi] + dvdt * fm[10 * M2 + mi];
      gy[n] = dvdr * fm[5 * M2 + mi] + dvds * fm[8 * M2 + mi] + dvdt * fm[11 * M2 + mi];
      gz[n] = dvdr * fm[6 * M2 + mi] + dvds * fm[9 * M2 + mi] + dvdt * fm[12 * M2 + mi];
    }
    const double nx = factNorm * fm[0 * M2 + l], ny = factNorm * fm[1 * M2 + l],
                 nz = factNorm * fm[2 * M2 + l];
    double factU = 1.0, hfMult = 1.0, qWall = 0.0;
    switch (type) {
      case VCPG_BC_WALL_HEAT_FLUX:
      case VCPG_BC_WALL_ISOTHERMAL: {
        VR[0] = VL[0] - 0.5 * (VL[1] * VL[1] + VL[2] * VL[2] + VL[3] * VL[3]) / VL[4];
        VR[1] = VR[2] = VR[3] = 0.0;
        VR[4] = type == VCPG_BC_WALL_HEAT_FLUX ? VL[4] : pres[0];
        factU = 0.0;
        if (type == VCPG_BC_WALL_HEAT_FLUX) { hfMult = 0.0; qWall = pres[0]; }
        break;
      }
      case VCPG_BC_WALL_INVISCID: {
        // ApplyInviscidWallBC (src/BoundaryState.cpp:40-118): the normal part of
        // V1..V3 removed with the face's unit normal.
        const double m0 = fm[0 * M2 + l], m1 = fm[1 * M2 + l], m2 = fm[2 * M2 + l];
        const double Vn = VL[1] * m0 + VL[2] * m1 + VL[3] * m2;
        VR[0] = VL[0] - 0.5 * Vn * Vn / VL[4];
        VR[1] = VL[1] - Vn * m0;
        VR[2] = VL[2] - Vn * m1;
        VR[3] = VL[3] - Vn * m2;
        VR[4] = VL[4];
        factU = 0.0;
        break;
      }
      case VCPG_BC_FARFIELD:
      case VCPG_BC_INFLOW_SUPERSONIC:
#pragma unroll
        for (int n = 0; n < 5; ++n) VR[n] = pres[n];
        break;
      case VCPG_BC_INFLOW_SUBSONIC: {
        // Riemann invariant extrapolated, scaled by the total enthalpy; the
        // velocity magnitude from the quadratic with the prescribed direction,
        // the Mach number clipped to 1 (src/BoundaryState.cpp:505-590).
        const double V4Inv = 1.0 / VL[4];
        const double u = -V4Inv * VL[1], v = -V4Inv * VL[2], w = -V4Inv * VL[3];
        const double a2 = -kGam * V4Inv, aa = sqrt(a2);
        const double un = u * nx + v * ny + w * nz;
        double riemann = 2.0 * aa * ovgm1 + un;
        const double H = a2 * ovgm1 + 0.5 * (u * u + v * v + w * w);
        riemann *= sqrt(pres[1] / H);
        const double alpha = nx * pres[2] + ny * pres[3] + nz * pres[4];
        const double qa = 1.0 + 0.5 * gm1 * alpha * alpha;
        const double qb = -gm1 * alpha * riemann;
        const double qc = 0.5 * gm1 * riemann * riemann - 2.0 * pres[1];
        double dd = qb * qb - 4.0 * qa * qc;
        dd = sqrt(fmax(0.0, dd));
        double qR = (-qb + dd) / (2.0 * qa);
        qR = fmax(0.0, qR);
        double qR2 = qR * qR;
        double aR2 = gm1 * (pres[1] - 0.5 * qR2);
        double MR2 = qR2 / aR2;
        MR2 = fmin(1.0, MR2);
        const double tmp = 1.0 / (1.0 + 0.5 * gm1 * MR2);
        aR2 = gm1 * pres[1] * tmp;
        qR2 = MR2 * aR2;
        qR = sqrt(qR2);
        const double pR = pres[0] * pow(tmp, govgm1);
        const double rhoR = kGam * pR / aR2;
        const double pRInv = 1.0 / pR;
        const double sR = log(pR / pow(rhoR, kGam));
        VR[0] = (kGam - sR) * ovgm1 - 0.5 * pRInv * rhoR * qR2;
        VR[1] = rhoR * pRInv * qR * pres[2];
        VR[2] = rhoR * pRInv * qR * pres[3];
        VR[3] = rhoR * pRInv * qR * pres[4];
        VR[4] = -rhoR * pRInv;
        break;
      }
      case VCPG_BC_OUTFLOW_SUBSONIC: {
        // Entropy, tangential velocity and the acoustic Riemann invariant
        // extrapolated, the back pressure imposed (src/BoundaryState.cpp:736-785).
        const double V4Inv = 1.0 / VL[4];
        const double u = -V4Inv * VL[1], v = -V4Inv * VL[2], w = -V4Inv * VL[3];
        const double eKin = 0.5 * (u * u + v * v + w * w);
        const double sL = kGam - gm1 * (VL[0] - VL[4] * eKin);
        const double aa = sqrt(-kGam * V4Inv);
        const double un = u * nx + v * ny + w * nz;
        const double riemann = 2.0 * aa * ovgm1 + un;
        const double pR = pres[0];
        const double rhoR = pow(pR / exp(sL), ovg);
        const double aR = sqrt(kGam * pR / rhoR);
        const double unR = riemann - 2.0 * aR * ovgm1;
        const double uR = u + (unR - un) * nx, vR = v + (unR - un) * ny, wR = w + (unR - un) * nz;
        const double pRInv = 1.0 / pR;
        VR[0] = (kGam - sL) * ovgm1 - 0.5 * pRInv * rhoR * (uR * uR + vR * vR + wR * wR);
        VR[1] = rhoR * pRInv * uR;
        VR[2] = rhoR * pRInv * vR;
        VR[3] = rhoR * pRInv * wR;
        VR[4] = -rhoR * pRInv;
        break;
      }
      default:  // VCPG_BC_OUTFLOW_SUPERSONIC: the interior state
#pragma unroll
        for (int n = 0; n < 5; ++n) VR[n] = VL[n];
        break;
    }
    const double wf = Ops<SLOT>().w[lj] * Ops<SLOT>().w[li];
    const double area = fm[3 * M2 + l];
    double flux[5], sx[5], sy[5], sz[5];
    if (a.riemann == 1)
      IsmailRoeFlux(VL, VR, nx, ny, nz, wf * area, flux, factU);
    else
      RoeFlux(VL, VR, nx, ny, nz, 0.5 * wf * area, flux, factU);
    double eddy = 0.0, visc[3];
    ViscousPenaltySymFlux(VL, VR, gx, gy, gz, nx, ny, nz, wf, area, mu,
                          a.tau_num / lenScale, a.theta_sym, flux, sx, sy, sz, hfMult,
                          wf * area * qWall, a.sgs, a.elem_scalars[(size_t)e * 15 + 3], &eddy,
                          forces ? visc : nullptr);
    if (a.sgs && a.eddymax && eddy > 0.0)
      atomicMax(a.eddymax, (unsigned long long)__double_as_longlong(eddy));
    if (forces) {
      // Pressure force: the mean of both states' pressures on the normal
      // pointing into the boundary (src/FluxesFace.cpp:997-1011).
      double r, uu, vv, ww, pL, pR, q2;
      FaceStatePrim(VL, r, uu, vv, ww, pL, q2);
      FaceStatePrim(VR, r, uu, vv, ww, pR, q2);
      const double abv = 0.5 * wf * area * (pL + pR);
      force[0] += abv * nx;
      force[1] += abv * ny;
      force[2] += abv * nz;
      force[3] += visc[0];
      force[4] += visc[1];
      force[5] += visc[2];
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int mi = a.metric_compat ? (n < M2 ? n : 0) : l;
      double sym[3];
#pragma unroll
      for (int p = 0; p < 3; ++p)
        sym[p] = sx[n] * fm[(4 + 3 * p) * M2 + mi] + sy[n] * fm[(5 + 3 * p) * M2 + mi] +
                 sz[n] * fm[(6 + 3 * p) * M2 + mi];
      out[(0 * 5 + n) * M2 + l] = sym[pFast];
      out[(1 * 5 + n) * M2 + l] = flux[n];
      out[(2 * 5 + n) * M2 + l] = sym[d];
      out[(3 * 5 + n) * M2 + l] = sym[pSlow];
    }
  }
  if (forces) {
    // Face sums of the six force components (warp shuffles, then warp order).
    __shared__ double s_force[6][NT / 32];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double v = force[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) s_force[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
      double v = 0.0;
      for (int w = 0; w < NT / 32; ++w) v += s_force[threadIdx.x][w];
      a.bforce[(size_t)b * 6 + threadIdx.x] = v;
    }
  }
}

// Boundary state and fluxes of one boundary face (characteristic conditions
// here, the others in WeakBoundaryFlux).
template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) BoundaryFluxKernel(const BoundaryArgs a) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int M2 = M * M;
  __shared__ double s_B[5 * M2], s_dqn[5 * M2], s_VR[5 * M2], s_dVr[5 * M2];
  __shared__ double s_mach;
  const int b = blockIdx.x;
  if (b >= a.nB) return;
  const int *bf = a.bface + b * kBfStride;
  if (!BoundaryFaceActive(a, bf)) return;
  const int e = bf[kBfElem], f = bf[kBfFace], type = bf[kBfType], d = f / 2;
  const int ig[3] = {bf[kBfGrad], bf[kBfGrad + 1], bf[kBfGrad + 2]};
  const int cs = a.case_state ? bf[kBfCase] : 0;
  const BlockFaceCfg c = a.cfgs[cs * 6 + f];
  const double mu = a.case_state ? a.case_par[cs * kCasePar + kParMu] : a.mu;
  const double factNorm = (f % 2 == 0) ? -1.0 : 1.0;
  const double *fm = a.face_metric + ((size_t)e * 6 + f) * 13 * M2;
  const double *tr = a.btrace + (size_t)b * 4 * 5 * M2;
  const double *pres = a.bpresc + (size_t)b * kPrescStride;
  if (type >= VCPG_BC_WALL_HEAT_FLUX) {   // the same branch for every thread of the CTA
    WeakBoundaryFlux<K, M, NT>(a, b, e, f, type, mu, fm, tr, pres);
    return;
  }

  // Boundary-averaged projected Mach number of this block face (sum in element order).
  if (threadIdx.x == 0) {
    double m = 0.0;
    if (a.bmach_sums) {
      m = a.bmach_sums[f];
    } else {
      for (int i = 0; i < c.count; ++i) m += a.bmach[c.first + i];
    }
    if (fabs(c.area) > 1.e-30) m /= c.area;
    s_mach = m;
  }
  __syncthreads();
  // The outlet's Mach number: the boundary average, or with "Outlet use local
  // (element) averaged Mach number" the average over the element face of the
  // subface's last element (the value the reference's subface member holds,
  // src/BoundaryState.cpp:1327); the inlets always take the boundary average.
  const double Mach = (type == VCPG_BC_OUTFLOW_NSCBC && c.localMach && a.bmach_local)
                          ? (a.bmach_last ? a.bmach_last[b] : a.bmach_local[bf[kBfLast]])
                          : s_mach;
  const double Mavg2 = Mach * Mach;
  const double gm1 = kGam - 1.0, ovgm1 = 1.0 / gm1;
  const int I0 = 4 + 3 * ig[0], J0 = 4 + 3 * ig[1], K0 = 4 + 3 * ig[2];

  // Characteristic correction of the normal derivative and the B vector of the
  // PC reconstruction, per face point.
  for (int l = threadIdx.x; l < M2; l += NT) {
    double V[5], dV[3][5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      V[n] = tr[n * M2 + l];
#pragma unroll
      for (int q = 0; q < 3; ++q) dV[q][n] = tr[((1 + ig[q]) * 5 + n) * M2 + l];
    }
    // ConvertEntropyToPrimitive (src/BoundaryState.cpp:1002-1106).
    const double V4Inv = 1.0 / V[4];
    const double u = -V4Inv * V[1], v = -V4Inv * V[2], w = -V4Inv * V[3];
    const double ek = 0.5 * (u * u + v * v + w * w);
    const double s = kGam - gm1 * (V[0] - V[4] * ek);
    const double a2 = -kGam * V4Inv;
    const double rho = pow(-V[4] * exp(s), -ovgm1);
    const double p = a2 * rho / kGam;
    const double povrho = -V4Inv;
    const double E = ovgm1 * povrho + ek;
    const double H = E + povrho;
    const double J[16] = {rho, rho * u, rho * v, rho * w, rho * E, povrho, povrho * u, povrho,
                          povrho * v, povrho, povrho * w, p, p * u, p * v, p * w, p * H};
    double dQ[3][5];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double *x = dV[q];
      dQ[q][0] = J[0] * x[0] + J[1] * x[1] + J[2] * x[2] + J[3] * x[3] + J[4] * x[4];
      dQ[q][1] = J[5] * x[1] + J[6] * x[4];
      dQ[q][2] = J[7] * x[2] + J[8] * x[4];
      dQ[q][3] = J[9] * x[3] + J[10] * x[4];
      dQ[q][4] = J[11] * x[0] + J[12] * x[1] + J[13] * x[2] + J[14] * x[3] + J[15] * x[4];
    }
    const double rr[3] = {fm[I0 * M2 + l], fm[(I0 + 1) * M2 + l], fm[(I0 + 2) * M2 + l]};
    const double magrr = sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
    const double ovmagrr = 1.0 / magrr;
    const double rn[3] = {rr[0] * ovmagrr, rr[1] * ovmagrr, rr[2] * ovmagrr};
    const double drhodr = dQ[0][0], dudr = dQ[0][1], dvdr = dQ[0][2], dwdr = dQ[0][3],
                 dpdr = dQ[0][4];
    const double ovrho = 1.0 / rho;
    const double aa2 = kGam * p * ovrho;
    const double aa = sqrt(aa2);
    const double ova2 = 1.0 / aa2, rhoa = rho * aa, ovrhoa = 1.0 / rhoa, rhova = rho / aa;
    const double ur = u * rr[0] + v * rr[1] + w * rr[2];
    const double arr = aa * magrr;
    const double lmb1 = ur - arr, lmb3 = ur + arr;
    const double ovlmb1 = 1.0 / lmb1, ovlmb3 = 1.0 / lmb3;
    const double dsdr = drhodr - ova2 * dpdr;
    const double dw1dr = rn[1] * dwdr - rn[2] * dvdr;
    const double dw2dr = rn[2] * dudr - rn[0] * dwdr;
    const double dw3dr = rn[0] * dvdr - rn[1] * dudr;
    const double durdr = rn[0] * dudr + rn[1] * dvdr + rn[2] * dwdr;
    double LL[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // Inverses of the acoustic eigenvalues that rebuild the normal derivative.
    double ov1 = ovlmb1, ov3 = ovlmb3;
    if (type == VCPG_BC_OUTFLOW_NSCBC) {
      // BCOutflowCharacteristicSubfaceClass::ComputeBoundaryState (src/BoundaryState.cpp:1300-1568).
      const double sign = (c.iPhi == 0) ? -1.0 : 1.0;
      const double kk = 0.5 * c.sigma * (1.0 - Mavg2) / c.len;
      const double bl = (c.betaL < 0.0) ? Mach : c.betaL;
      const double bt = (c.betaT < 0.0) ? Mach : c.betaT;
      const double cbl = c.oneMinusBeta ? fmin(1.0, 1.0 - bl) : fmin(1.0, bl);
      const double cbt = c.oneMinusBeta ? fmin(1.0, 1.0 - bt) : fmin(1.0, bt);
      const double pInf = pres[0];
      const double ss[3] = {fm[J0 * M2 + l], fm[(J0 + 1) * M2 + l], fm[(J0 + 2) * M2 + l]};
      const double tt[3] = {fm[K0 * M2 + l], fm[(K0 + 1) * M2 + l], fm[(K0 + 2) * M2 + l]};
      const double duds = dQ[1][1], dudt = dQ[2][1];
      const double dvds = dQ[1][2], dvdt = dQ[2][2];
      const double dwds = dQ[1][3], dwdt = dQ[2][3];
      const double dpds = dQ[1][4], dpdt = dQ[2][4];
      const double us = u * ss[0] + v * ss[1] + w * ss[2];
      const double ut = u * tt[0] + v * tt[1] + w * tt[2];
      const double ars = aa * (rn[0] * ss[0] + rn[1] * ss[1] + rn[2] * ss[2]);
      const double art = aa * (rn[0] * tt[0] + rn[1] * tt[1] + rn[2] * tt[2]);
      const double durds = rn[0] * duds + rn[1] * dvds + rn[2] * dwds;
      const double durdt = rn[0] * dudt + rn[1] * dvdt + rn[2] * dwdt;
      LL[0] = 0.5 * lmb1 * (ovrhoa * dpdr - durdr);
      LL[1] = (rn[0] * dsdr - dw1dr);
      LL[2] = (rn[1] * dsdr - dw2dr);
      LL[3] = (rn[2] * dsdr - dw3dr);
      LL[4] = 0.5 * lmb3 * (ovrhoa * dpdr + durdr);
      const double LT = 0.5 * ovrhoa * (us + sign * ars) * dpds + sign * 0.5 * us * durds +
                        0.5 * ovrhoa * (ut + sign * art) * dpdt + sign * 0.5 * ut * durdt;
      const double TT = -0.5 * aa * (ss[0] * duds + ss[1] * dvds + ss[2] * dwds +
                                     tt[0] * dudt + tt[1] * dvdt + tt[2] * dwdt);
      LL[c.iPhi] = kk * ovrho * magrr * (p - pInf) - cbl * LT + cbt * TT;
    } else if (type == VCPG_BC_INFLOW_TOTAL_NSCBC) {
      // BCInflowTotalCharacteristicSubfaceClass::ComputeBoundaryState
      // (src/BoundaryState.cpp:1848-2238): the incoming amplitudes relax the total
      // pressure, total temperature and the two direction cosines v/|u|, w/|u|
      // towards the prescribed values; the 4x4 system is solved in closed form by
      // elimination in the order of the reference (E, F, G, H coefficients). The
      // eigenvalues use the unit normal here.
      const int iPsi = c.iPhi == 0 ? 4 : 0;
      const double kk = -c.inSigma / c.inLen;
      const double urn = u * rn[0] + v * rn[1] + w * rn[2];
      const double l1 = urn - aa, l3 = urn + aa;
      ov1 = 1.0 / l1;
      ov3 = 1.0 / l3;
      const double ovl2 = 1.0 / urn;
      const double w1 = rn[1] * w - rn[2] * v, w2 = rn[2] * u - rn[0] * w,
                   w3 = rn[0] * v - rn[1] * u;
      const double ova = 1.0 / aa, ovrg = 1.0 / kRGas, ovcp = 1.0 / kCp;
      if (c.incoming) {
        LL[0] = 0.5 * l1 * (ovrhoa * dpdr - durdr);
        LL[4] = 0.5 * l3 * (ovrhoa * dpdr + durdr);
      }
      const double magU2 = 2.0 * ek, magU = sqrt(magU2);
      const double ff = 1.0 + 0.5 * gm1 * magU2 / aa2;
      const double T = p * ovrho * ovrg;
      const double Pt = p * pow(ff, kGam * ovgm1), Tt = T * ff;
      const double Zt = v / magU, Zp = w / magU;
      const double ka = kk * aa;
      const double X1 = ka * (Pt - pres[0]), X2 = ka * (Tt - pres[1]);
      const double X3 = ka * (Zt - pres[3]), X4 = ka * (Zp - pres[4]);
      const double rPtTt = ovrg * Pt / Tt, Ttovrho = Tt * ovrho, gaPt = kGam * ova * Pt;
      const double ekovrho = ek * ovrho, gm1eka = gm1 * ek * ova, gm1aTt = gm1 * ova * Tt;
      const double ovU2 = 1.0 / magU2;
      const double gp = gm1eka + urn, gmn = gm1eka - urn;
      const double f1 = w1 - rn[0] * ekovrho, f2 = w2 - rn[1] * ekovrho, f3 = w3 - rn[2] * ekovrho;
      const double A1 = gp * rPtTt - gaPt, A2 = f1 * rPtTt, A3 = f2 * rPtTt, A4 = f3 * rPtTt,
                   A5 = gmn * rPtTt - gaPt;
      const double B1 = gp * ovcp - gm1aTt, B2 = f1 * ovcp + rn[0] * Ttovrho,
                   B3 = f2 * ovcp + rn[1] * Ttovrho, B4 = f3 * ovcp + rn[2] * Ttovrho,
                   B5 = gmn * ovcp - gm1aTt;
      const double C1 = (rn[1] * magU - urn * Zt) * ovU2, C2 = -(rn[2] * magU + w1 * Zt) * ovU2,
                   C3 = (-w2 * Zt) * ovU2, C4 = (rn[0] * magU - w3 * Zt) * ovU2, C5 = -C1;
      const double D1 = (rn[2] * magU - urn * Zp) * ovU2, D2 = (rn[1] * magU - w1 * Zp) * ovU2,
                   D3 = -(rn[0] * magU + w2 * Zp) * ovU2, D4 = (-w3 * Zp) * ovU2, D5 = -D1;
      const double Y1 = LL[iPsi] * A1, Y2 = LL[iPsi] * B1, Y3 = LL[iPsi] * C1,
                   Y4 = LL[iPsi] * D1;
      const double ovA2 = 1.0 / A2;
      const double E0 = ovA2 * X1, E3 = -ovA2 * A3, E4 = -ovA2 * A4, E5 = -ovA2 * A5,
                   P2 = -ovA2 * Y1;
      const double ovF = 1.0 / (D3 + D2 * E3);
      const double F0 = ovF * (X4 - D2 * E0), F4 = -ovF * (D4 + D2 * E4),
                   F5 = -ovF * (D5 + D2 * E5), P3 = -ovF * (Y4 + D2 * P2);
      const double ovG = 1.0 / (C4 + C2 * E4 + C3 * F4 + C2 * E3 * F4);
      const double G0 = ovG * (X3 - C2 * E0 - C3 * F0 - C2 * E3 * F0),
                   G5 = -ovG * (C5 + C2 * E5 + C3 * F5 + C2 * E3 * F5),
                   P4 = -ovG * (Y3 + C2 * P2 + C3 * P3 + C2 * E3 * P3);
      const double ovH = 1.0 / (B5 + B2 * E5 + B3 * F5 + B4 * G5 + B2 * E3 * F5 + B2 * E4 * G5 +
                                B3 * F4 * G5 + B2 * E3 * F4 * G5);
      const double H0 = ovH * (X2 - B2 * E0 - B3 * F0 - B4 * G0 - B2 * E3 * F0 - B2 * E4 * G0 -
                               B3 * F4 * G0 - B2 * E3 * F4 * G0);
      const double P5 = -ovH * (Y2 + B2 * P2 + B3 * P3 + B4 * P4 + B2 * E3 * P3 + B2 * E4 * P4 +
                                B3 * F4 * P4 + B2 * E3 * F4 * P4);
      LL[c.iPhi] = H0 + P5;
      LL[3] = G0 + G5 * LL[c.iPhi] + P4;
      LL[2] = F0 + F4 * LL[3] + F5 * LL[c.iPhi] + P3;
      LL[1] = E0 + E3 * LL[2] + E4 * LL[3] + E5 * LL[c.iPhi] + P2;
      LL[1] *= ovl2;
      LL[2] *= ovl2;
      LL[3] *= ovl2;
      (void)dsdr; (void)dw1dr; (void)dw2dr; (void)dw3dr;
    } else {
      // BCInflowStaticCharacteristicSubfaceClass::ComputeBoundaryState
      // (src/BoundaryState.cpp:1579-1847).
      const double sign = (factNorm > 0.0) ? -1.0 : 1.0;
      const double ka = sign * 0.5 * c.inSigma * (1.0 - Mavg2) / c.inLen;
      const double ku = c.inSigma / c.inLen;
      const double ovlmb2 = 1.0 / ur;
      if (c.incoming) {
        LL[0] = 0.5 * lmb1 * (ovrhoa * dpdr - durdr);
        LL[4] = 0.5 * lmb3 * (ovrhoa * dpdr + durdr);
      }
      const double drho = rho - pres[0], du = u - pres[1], dv = v - pres[2], dw = w - pres[3];
      const double kaol = ku * aa * ovlmb2;
      LL[c.iPhi] = ka * aa * (rr[0] * du + rr[1] * dv + rr[2] * dw);
      LL[1] = kaol * (rr[2] * dv - rr[1] * dw + rr[0] * drho);
      LL[2] = kaol * (rr[0] * dw - rr[2] * du + rr[1] * drho);
      LL[3] = kaol * (rr[1] * du - rr[0] * dv + rr[2] * drho);
      (void)dsdr; (void)dw1dr; (void)dw2dr; (void)dw3dr;
    }
    // Boundary-conforming normal derivative of the primitive variables.
    double dn[5];
    dn[0] = ov1 * rhova * LL[0] + rn[0] * LL[1] + rn[1] * LL[2] + rn[2] * LL[3] +
            ov3 * rhova * LL[4];
    dn[1] = -ov1 * rn[0] * LL[0] - rn[2] * LL[2] + rn[1] * LL[3] + ov3 * rn[0] * LL[4];
    dn[2] = -ov1 * rn[1] * LL[0] + rn[2] * LL[1] - rn[0] * LL[3] + ov3 * rn[1] * LL[4];
    dn[3] = -ov1 * rn[2] * LL[0] - rn[1] * LL[1] + rn[0] * LL[2] + ov3 * rn[2] * LL[4];
    dn[4] = ov1 * rhoa * LL[0] + ov3 * rhoa * LL[4];
    const double q[5] = {rho, u, v, w, p};
    const double dqr[5] = {drhodr, dudr, dvdr, dwdr, dpdr};
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      s_dqn[n * M2 + l] = dn[n];
      s_B[n * M2 + l] = dn[n] - (dqr[n] - q[n] * c.dell);
    }
  }
  __syncthreads();

  // PC reconstruction of the boundary primitive state, then entropy variables and
  // the entropy-variable normal derivative (src/BoundaryState.cpp:1114-1230).
  for (int l = threadIdx.x; l < M2; l += NT) {
    double q[5];
    const double *A = a.pc + (size_t)l * M2;
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      double t = 0.0;
      for (int j = 0; j < M2; ++j) t += A[j] * s_B[n * M2 + j];
      q[n] = factNorm < 0.0 ? -t : t;
    }
    const double rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
    const double s = log(p / pow(rho, kGam));
    const double dr = s_dqn[0 * M2 + l], du = s_dqn[1 * M2 + l], dv = s_dqn[2 * M2 + l],
                 dw = s_dqn[3 * M2 + l], dp = s_dqn[4 * M2 + l];
    const double ovrho = 1.0 / rho, ovp = 1.0 / p, rovp = rho * ovp;
    const double ek = 0.5 * (u * u + v * v + w * w);
    double VR[5];
    VR[0] = -rovp * ek + (kGam - s) * ovgm1;
    VR[1] = rovp * u;
    VR[2] = rovp * v;
    VR[3] = rovp * w;
    VR[4] = -rovp;
    const double govgm1 = kGam * ovgm1;
    const double D[16] = {govgm1 * ovrho - ovp * ek, -VR[1], -VR[2], -VR[3],
                          ovp * (rovp * ek - ovgm1), u * ovp, rovp, -ovp * VR[1], v * ovp,
                          rovp, -ovp * VR[2], w * ovp, rovp, -ovp * VR[3], -ovp, ovp * rovp};
    s_dVr[0 * M2 + l] = D[0] * dr + D[1] * du + D[2] * dv + D[3] * dw + D[4] * dp;
    s_dVr[1 * M2 + l] = D[5] * dr + D[6] * du + D[7] * dp;
    s_dVr[2 * M2 + l] = D[8] * dr + D[9] * dv + D[10] * dp;
    s_dVr[3 * M2 + l] = D[11] * dr + D[12] * dw + D[13] * dp;
    s_dVr[4 * M2 + l] = D[14] * dr + D[15] * dp;
#pragma unroll
    for (int n = 0; n < 5; ++n) s_VR[n * M2 + l] = VR[n];
  }
  __syncthreads();

  // Transverse derivatives of the reconstructed state (derivative along the slow
  // face index into the first transverse slot, along the fast index into the
  // second, src/BoundaryState.cpp:1266-1288), Cartesian gradients of both sides
  // and their average (src/FluxesFace.cpp:108-148), and the face fluxes.
  const double lenScale = a.elem_scalars[(size_t)e * 15 + d];
  for (int l = threadIdx.x; l < M2; l += NT) {
    const int li = l / M, lj = l - li * M;
    double VL[5], VR[5], gR[3][5], gL[3][5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      VL[n] = tr[n * M2 + l];
      VR[n] = s_VR[n * M2 + l];
      double ds = 0.0, dt = 0.0;
      for (int k = 0; k < M; ++k) {
        ds += a.dlq[li * M + k] * s_VR[n * M2 + k * M + lj];
        dt += a.dlq[lj * M + k] * s_VR[n * M2 + li * M + k];
      }
      gR[ig[0]][n] = s_dVr[n * M2 + l];
      gR[ig[1]][n] = ds;
      gR[ig[2]][n] = dt;
#pragma unroll
      for (int q = 0; q < 3; ++q) gL[q][n] = tr[((1 + q) * 5 + n) * M2 + l];
    }
    double gx[5], gy[5], gz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int mi = a.metric_compat ? (n < M2 ? n : 0) : l;
      const double drdx = fm[4 * M2 + mi], dsdx = fm[7 * M2 + mi], dtdx = fm[10 * M2 + mi];
      const double drdy = fm[5 * M2 + mi], dsdy = fm[8 * M2 + mi], dtdy = fm[11 * M2 + mi];
      const double drdz = fm[6 * M2 + mi], dsdz = fm[9 * M2 + mi], dtdz = fm[12 * M2 + mi];
      const double xR = gR[0][n] * drdx + gR[1][n] * dsdx + gR[2][n] * dtdx;
      const double yR = gR[0][n] * drdy + gR[1][n] * dsdy + gR[2][n] * dtdy;
      const double zR = gR[0][n] * drdz + gR[1][n] * dsdz + gR[2][n] * dtdz;
      const double xL = gL[0][n] * drdx + gL[1][n] * dsdx + gL[2][n] * dtdx;
      const double yL = gL[0][n] * drdy + gL[1][n] * dsdy + gL[2][n] * dtdy;
      const double zL = gL[0][n] * drdz + gL[1][n] * dsdz + gL[2][n] * dtdz;
      gx[n] = 0.5 * (xL + xR);
      gy[n] = 0.5 * (yL + yR);
      gz[n] = 0.5 * (zL + zR);
    }
    const double wf = Ops<SLOT>().w[lj] * Ops<SLOT>().w[li];
    const double nx = factNorm * fm[0 * M2 + l], ny = factNorm * fm[1 * M2 + l],
                 nz = factNorm * fm[2 * M2 + l];
    const double area = fm[3 * M2 + l];
    double flux[5], sx[5], sy[5], sz[5];
    if (a.riemann == 1)
      IsmailRoeFlux(VL, VR, nx, ny, nz, wf * area, flux);
    else
      RoeFlux(VL, VR, nx, ny, nz, 0.5 * wf * area, flux);
    double eddy = 0.0;
    ViscousPenaltySymFlux(VL, VR, gx, gy, gz, nx, ny, nz, wf, area, mu,
                          a.tau_num / lenScale, a.theta_sym, flux, sx, sy, sz, 1.0, 0.0, a.sgs,
                          a.elem_scalars[(size_t)e * 15 + 3], &eddy);
    if (a.sgs && a.eddymax && eddy > 0.0)
      atomicMax(a.eddymax, (unsigned long long)__double_as_longlong(eddy));
    double *out = a.bflux + (size_t)b * 4 * 5 * M2;
    const int pFast = BFastParam(d), pSlow = 3 - d - pFast;
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int mi = a.metric_compat ? (n < M2 ? n : 0) : l;
      double sym[3];
#pragma unroll
      for (int p = 0; p < 3; ++p)
        sym[p] = sx[n] * fm[(4 + 3 * p) * M2 + mi] + sy[n] * fm[(5 + 3 * p) * M2 + mi] +
                 sz[n] * fm[(6 + 3 * p) * M2 + mi];
      out[(0 * 5 + n) * M2 + l] = sym[pFast];
      out[(1 * 5 + n) * M2 + l] = flux[n];
      out[(2 * 5 + n) * M2 + l] = sym[d];
      out[(3 * 5 + n) * M2 + l] = sym[pSlow];
    }
  }
}

}  // namespace vcpg
