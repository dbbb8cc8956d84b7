// Fused FP64 DG residual kernel: one CTA per element computes the volume
// terms, all six faces and the generalised mass-matrix solve of its element.
//
// Reference path (per element, SolverClass::Residual, src/SolverClass.cpp:3381-3795):
//   VolumeResidual (src/ElementClass.cpp:3809-4534)
//   I/J/KFaceResiduals (src/ElementClass.cpp:2582-3404) with FluxesInternalFace
//     (src/FluxesFace.cpp:220-343)
//   neighbour Min-face residual accumulation (src/SolverClass.cpp:3616-3732)
//   MultiplyResInverseMassMatrix -> CG_EntropyVarMassMatrix (src/CG_MassMatrix.cpp:250-504)
//
// Every interior face is evaluated by both of its elements with identical
// inputs, so the two sides see bit-identical fluxes and no cross-element
// write (and no atomic) is needed. The residual of an element is accumulated
// in the reference's order: volume (x, y, z), own Min faces (i, j, k), then
// the Max-face contributions each summed from zero and added (i, j, k).
#pragma once

#include "dg_physics.cuh"
#include "dg_tensor.cuh"

namespace vcpg {

struct ResidualArgs {
  const double *sol;           // [nE][5][K^3]
  double *res;                 // [nE][5][K^3] residual after the mass-matrix solve
  double *res_raw;             // optional [nE][5][K^3] residual before the solve
  const double *vol_metric;    // [nE][10][M^3]
  const double *face_metric;   // [nE][6][13][M^2]
  const double *elem_scalars;  // [nE][15]
  const int *nbr;              // [nE][6]
  int n_elem;
  double mu;                   // non-dimensional viscosity
  double tau_num;              // (p+1)^2 * relative penalty parameter
  double theta_sym;
  int riemann;                 // 0 Roe, 1 Ismail-Roe
  int metric_compat;           // 1: metric indexed by the variable index
  unsigned long long *mach2max;  // optional: bits of max Mach^2 (non-negative double)
  int *status;                 // [0] CG iteration cap hits, [1] boundary face without BC
  unsigned long long *cg_stats;  // [0] CG iterations, [1] element solves (cumulative)
};

// Arguments of the CFL time-step kernel (kernels.cu).
struct TimeStepArgs {
  const double *sol;
  const double *elem_scalars;
  int n_elem;
  int n_poly;
  double cfl, mu, p_ref, u_ref, rho_ref;
  unsigned long long *dt_bits;
  int *status;  // [2]: negative a^2 seen
};

template <int NT>
__device__ __forceinline__ double BlockSum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

template <int NT>
__device__ __forceinline__ double BlockMax(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = red[0];
#pragma unroll
  for (int i = 1; i < NT / 32; ++i) s = fmax(s, red[i]);
  return s;
}

// Block-wide (sum a, sum b, max c) with one pair of barriers; red needs 3*NT/32.
template <int NT>
__device__ __forceinline__ void BlockReduce3(double &a, double &b, double &c, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c = fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) { red[w] = a; red[NT / 32 + w] = b; red[2 * (NT / 32) + w] = c; }
  __syncthreads();
  a = 0.0; b = 0.0; c = red[2 * (NT / 32)];
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) {
    a += red[i];
    b += red[NT / 32 + i];
    c = fmax(c, red[2 * (NT / 32) + i]);
  }
}

// Shared-memory plan (doubles) of the fused kernel for a (K, M) pair.
template <int K, int M> struct Plan {
  static constexpr int KD = K * K * K, MD = M * M * M, M2 = M * M;
  static constexpr int TK = 5 * K * K * M;      // first-stage buffer
  static constexpr int TJ = 5 * K * M * M;      // second-stage buffer
  // Volume phase: tK, tJ, Var, dX, dY, dZ.
  static constexpr int VOL = TK + TJ + 20 * MD;
  // Face phase: per face-side trace (value + 3 derivatives) 20*M2, two sides,
  // three faces at a time, plus normal-evaluation and stage buffers.
  // Face phase: BN/BND 60 K^2, three fast-axis buffers 90 K M, traces 120 M^2.
  static constexpr int FACE = 60 * K * K + 90 * K * M + 120 * M2;
  // CG phase: z, p, Ap, x, pInt and the contraction buffers.
  static constexpr int CG = 20 * KD + 5 * MD + TK + TJ;
  static constexpr int WORK = VOL > FACE ? (VOL > CG ? VOL : CG) : (FACE > CG ? FACE : CG);
  // Persistent: sol, R, CG point data (8 per point), J*w, reduction scratch,
  // face vectors (basis and derivative at r = -1, +1).
  static constexpr int PERSIST = 10 * KD + 9 * MD + 64 + 4 * kKMax;
  static constexpr int TOTAL = PERSIST + WORK;
  static constexpr size_t BYTES = sizeof(double) * (size_t)TOTAL;
  // Threads per CTA and the CTAs per SM that the shared memory allows (227 KB).
  static constexpr int NT = K >= 5 ? 256 : 128;
  static constexpr int MIN_BLOCKS =
      (int)(227 * 1024 / BYTES) < 1 ? 1 : ((int)(227 * 1024 / BYTES) > 4 ? 4 : (int)(227 * 1024 / BYTES));
};


// ---------------------------------------------------------------------------
// Volume phase: solution and gradients at the integration points
// (TPSAGV), pointwise fluxes, and the three transposed contractions (TPAVR)
// into s_R. Also stores the CG point data (rho, u, v, w, p, rhoE, dUdV(4,4))
// and J*w.  Follows ElementClass::VolumeResidual, src/ElementClass.cpp:3809-4443.
// ---------------------------------------------------------------------------
template <int NT, int K, int M>
__device__ __forceinline__ void VolumePhase(const ResidualArgs &a, const int e,
                                            const double *s_sol, double *s_R, double *s_cgp,
                                            double *s_jw, double *work, double *s_red) {
  constexpr int SLOT = Slot<K, M>::value;
  using P = Plan<K, M>;
  constexpr int MD = P::MD, KD = P::KD, M2 = P::M2;
  double *tK = work, *tJ = work + P::TK, *Var = tJ + P::TJ;
  double *dX = Var + 5 * MD, *dY = dX + 5 * MD, *dZ = dY + 5 * MD;

  // TPSAGV (include/TensorProductSolAndGradVolume.hpp:5-249): k, then j, then i.
  Contract<NT, SLOT, K, M, kLeg, 2, 5, K, K, K, K, M, false>(s_sol, tK);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false>(tK, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false>(tJ, Var);
  Contract<NT, SLOT, K, M, kDLeg, 0, 5, K, M, M, K, M, false>(tJ, dX);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLeg, 1, 5, K, K, M, K, M, false>(tK, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false>(tJ, dY);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLeg, 2, 5, K, K, K, K, M, false>(s_sol, tK);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false>(tK, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false>(tJ, dZ);
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_R[i] = 0.0;
  __syncthreads();

  const double *vm = a.vol_metric + (size_t)e * 10 * MD;
  const double gm1 = kGam - 1.0, ov1mg = -1.0 / gm1;
  double mach2 = 0.0;
  for (int l = threadIdx.x; l < MD; l += NT) {
    const int i = l % M, j = (l / M) % M, k = l / M2;
    // Parametric -> Cartesian gradients (src/ElementClass.cpp:3856-3875). In the
    // compatibility mode the metric of point n is used for variable n.
    double V[5], gx[5], gy[5], gz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int mi = a.metric_compat ? n : l;
      const double dvdr = dX[n * MD + l], dvds = dY[n * MD + l], dvdt = dZ[n * MD + l];
      gx[n] = dvdr * __ldg(vm + 1 * MD + mi) + dvds * __ldg(vm + 4 * MD + mi) +
              dvdt * __ldg(vm + 7 * MD + mi);
      gy[n] = dvdr * __ldg(vm + 2 * MD + mi) + dvds * __ldg(vm + 5 * MD + mi) +
              dvdt * __ldg(vm + 8 * MD + mi);
      gz[n] = dvdr * __ldg(vm + 3 * MD + mi) + dvds * __ldg(vm + 6 * MD + mi) +
              dvdt * __ldg(vm + 9 * MD + mi);
      V[n] = Var[n * MD + l];
    }
    // Entropy -> primitive variables, velocity and internal-energy gradients
    // (src/ElementClass.cpp:4183-4257).
    double rho, u, v, w, p, eKin;
    EntropyToPrim(V[0], V[1], V[2], V[3], V[4], rho, u, v, w, p, eKin);
    const double V4Inv = 1.0 / V[4];
    const double rE = -p * ov1mg + rho * eKin;
    const double dudx = -V4Inv * (gx[1] + u * gx[4]), dudy = -V4Inv * (gy[1] + u * gy[4]),
                 dudz = -V4Inv * (gz[1] + u * gz[4]);
    const double dvdx = -V4Inv * (gx[2] + v * gx[4]), dvdy = -V4Inv * (gy[2] + v * gy[4]),
                 dvdz = -V4Inv * (gz[2] + v * gz[4]);
    const double dwdx = -V4Inv * (gx[3] + w * gx[4]), dwdy = -V4Inv * (gy[3] + w * gy[4]),
                 dwdz = -V4Inv * (gz[3] + w * gz[4]);
    const double fact = -V4Inv * V4Inv * ov1mg;
    const double dedx = gx[4] * fact, dedy = gy[4] * fact, dedz = gz[4] * fact;
    const double rH = rE + p;
    s_cgp[0 * MD + l] = rho;
    s_cgp[1 * MD + l] = u;
    s_cgp[2 * MD + l] = v;
    s_cgp[3 * MD + l] = w;
    s_cgp[4 * MD + l] = p;
    s_cgp[5 * MD + l] = rE;
    s_cgp[6 * MD + l] = rE * rH / rho + p * eKin;  // dUdV(4,4)
    mach2 = fmax(mach2, rho * (u * u + v * v + w * w) / (kGam * p));

    // Inviscid + viscous fluxes times -J w and the metric (src/ElementClass.cpp:4320-4416).
    const double Wl = c_ops[SLOT].w[i] * c_ops[SLOT].w[j] * c_ops[SLOT].w[k];
    const double Jl = __ldg(vm + l);
    s_jw[l] = Wl * Jl;
    const double weight = -Jl * Wl;
    const double ru = rho * u, rv = rho * v, rw = rho * w;
    const double muTot = a.mu + 0.0;
    const double factHeatFluxTot = a.mu * kFactHFLam + 0.0 * kFactHFTurb;
    const double divVelTerm = kLamOverMu * (dudx + dvdy + dwdz);
    const double tauxx = muTot * (2.0 * dudx + divVelTerm);
    const double tauyy = muTot * (2.0 * dvdy + divVelTerm);
    const double tauzz = muTot * (2.0 * dwdz + divVelTerm);
    const double tauxy = muTot * (dudy + dvdx);
    const double tauxz = muTot * (dudz + dwdx);
    const double tauyz = muTot * (dvdz + dwdy);
    const double qx = -factHeatFluxTot * dedx, qy = -factHeatFluxTot * dedy,
                 qz = -factHeatFluxTot * dedz;
    const double fx[5] = {ru, ru * u - tauxx + p, rv * u - tauxy, rw * u - tauxz,
                          (rE + p) * u - (u * tauxx + v * tauxy + w * tauxz - qx)};
    const double fy[5] = {rv, ru * v - tauxy, rv * v - tauyy + p, rw * v - tauyz,
                          (rE + p) * v - (u * tauxy + v * tauyy + w * tauyz - qy)};
    const double fz[5] = {rw, ru * w - tauxz, rv * w - tauyz, rw * w - tauzz + p,
                          (rE + p) * w - (u * tauxz + v * tauyz + w * tauzz - qz)};
    const double drdx = weight * __ldg(vm + 1 * MD + l), drdy = weight * __ldg(vm + 2 * MD + l),
                 drdz = weight * __ldg(vm + 3 * MD + l);
    const double dsdx = weight * __ldg(vm + 4 * MD + l), dsdy = weight * __ldg(vm + 5 * MD + l),
                 dsdz = weight * __ldg(vm + 6 * MD + l);
    const double dtdx = weight * __ldg(vm + 7 * MD + l), dtdy = weight * __ldg(vm + 8 * MD + l),
                 dtdz = weight * __ldg(vm + 9 * MD + l);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      dX[n * MD + l] = fx[n] * drdx + fy[n] * drdy + fz[n] * drdz;
      dY[n * MD + l] = fx[n] * dsdx + fy[n] * dsdy + fz[n] * dsdz;
      dZ[n * MD + l] = fx[n] * dtdx + fy[n] * dtdy + fz[n] * dtdz;
    }
  }
  if (a.mach2max) {
    const double m = BlockMax<NT>(mach2, s_red);
    if (threadIdx.x == 0) atomicMax(a.mach2max, (unsigned long long)__double_as_longlong(m));
  }
  __syncthreads();

  // TPAVR for the three flux directions (src/ElementClass.cpp:4425-4443).
  Contract<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false>(dX, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false>(tJ, tK);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegT, 0, 5, M, K, K, M, K, true>(tK, s_R);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false>(dY, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegT, 1, 5, M, M, K, M, K, false>(tJ, tK);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true>(tK, s_R);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegT, 2, 5, M, M, M, M, K, false>(dZ, tJ);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false>(tJ, tK);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true>(tK, s_R);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Face phase. The faces are processed in two groups -- the Min faces of the
// three directions, then the Max faces -- and every stage of a group runs over
// all three faces and both sides of each face at once, so a group needs three
// barriers for its six traces and three for its distributions.
//
// Trace t = 2 d + s: face direction d (0 i, 1 j, 2 k), s = 0 own side, s = 1
// neighbour side. Face arrays are [slow][fast] with (slow, fast) = (k, j), (k, i),
// (j, i) for d = 0, 1, 2, as in the reference's TPSAG[IJK] outputs. Trace
// storage TR[q][t][v][M^2]: q = 0 value, 1 face-normal derivative, 2 fast-axis
// derivative, 3 slow-axis derivative.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int FastParam(const int d) { return d == 0 ? 1 : 0; }

// Trace quantity q holding parametric derivative p (0 r, 1 s, 2 t) for direction d.
__device__ __forceinline__ int DerivSlot(const int d, const int p) {
  return p == d ? 1 : (p == FastParam(d) ? 2 : 3);
}

// Face-normal evaluation of the six sides of a group (first stage of TPSAG[IJK]).
template <int NT, int SLOT, int K>
__device__ __forceinline__ void FaceNormalBatch(const double *s_sol, const double *gsol,
                                                const int nb0, const int nb1, const int nb2,
                                                const int g, const double *s_fv, double *bn,
                                                double *bnd) {
  constexpr int KD = K * K * K, L = 5 * K * K;
  for (int line = threadIdx.x; line < 6 * L; line += NT) {
    const int t = line / L, r = line - t * L;
    const int d = t >> 1, nbr = (t & 1);
    const int side = nbr ? 1 - g : g;
    const int v = r / (K * K), r2 = r - v * K * K, sl = r2 / K, f = r2 - sl * K;
    int base, ns;
    if (d == 0) { base = sl * K * K + f * K; ns = 1; }
    else if (d == 1) { base = sl * K * K + f; ns = K; }
    else { base = sl * K + f; ns = K * K; }
    base += v * KD;
    const double *fv = s_fv + side * K, *dfv = s_fv + (2 + side) * K;
    double a0 = 0.0, d0 = 0.0;
    if (nbr) {
      const int nb = d == 0 ? nb0 : (d == 1 ? nb1 : nb2);
      if (nb >= 0) {
        const double *b = gsol + (size_t)nb * 5 * KD + base;
#pragma unroll
        for (int n = 0; n < K; ++n) {
          const double x = __ldg(b + n * ns);
          a0 = fma(fv[n], x, a0);
          d0 = fma(dfv[n], x, d0);
        }
      }
    } else {
      const double *b = s_sol + base;
#pragma unroll
      for (int n = 0; n < K; ++n) {
        const double x = b[n * ns];
        a0 = fma(fv[n], x, a0);
        d0 = fma(dfv[n], x, d0);
      }
    }
    bn[line] = a0;
    bnd[line] = d0;
  }
}

// Parametric -> Cartesian gradient of one side at face point pt from TR.
template <int M2>
__device__ __forceinline__ void TraceCartesianGrad(const double *TR, const int t, const int d,
                                                   const int pt, const double *fm,
                                                   const int compat, double *gx, double *gy,
                                                   double *gz) {
  const int qr = DerivSlot(d, 0), qs = DerivSlot(d, 1), qt = DerivSlot(d, 2);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    const int mi = compat ? n : pt;
    const double dvdr = TR[((qr * 6 + t) * 5 + n) * M2 + pt];
    const double dvds = TR[((qs * 6 + t) * 5 + n) * M2 + pt];
    const double dvdt = TR[((qt * 6 + t) * 5 + n) * M2 + pt];
    gx[n] = dvdr * __ldg(fm + 4 * M2 + mi) + dvds * __ldg(fm + 7 * M2 + mi) +
            dvdt * __ldg(fm + 10 * M2 + mi);
    gy[n] = dvdr * __ldg(fm + 5 * M2 + mi) + dvds * __ldg(fm + 8 * M2 + mi) +
            dvdt * __ldg(fm + 11 * M2 + mi);
    gz[n] = dvdr * __ldg(fm + 6 * M2 + mi) + dvds * __ldg(fm + 9 * M2 + mi) +
            dvdt * __ldg(fm + 12 * M2 + mi);
  }
}

// Fluxes of one interior face point (FluxesInternalFace, src/FluxesFace.cpp:220-343),
// seen from the own side. Writes the own-side distribution inputs by role:
// P1[role][d][v][M2] with role 0 fast-axis symmetrizing flux, 1 normal flux (with
// the own side's sign), 2 face-normal symmetrizing flux; P2[d][v][M2] the
// slow-axis symmetrizing flux.
template <int K, int M>
__device__ __forceinline__ void GroupFacePoint(const ResidualArgs &a, const int g, const int d,
                                               const int pt, const double *TR,
                                               const double *fmOwn, const double *fmNb,
                                               const double lenScale, double *P1, double *P2) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int M2 = M * M;
  const int tOwn = 2 * d, tNb = 2 * d + 1;
  // g == 0: own Min face, the neighbour is the left state; g == 1: own Max face.
  const int tL = g == 0 ? tNb : tOwn, tR = g == 0 ? tOwn : tNb;
  const double *fmL = g == 0 ? fmNb : fmOwn, *fmR = g == 0 ? fmOwn : fmNb;
  double VL[5], VR[5], gxL[5], gyL[5], gzL[5], gxR[5], gyR[5], gzR[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    VL[n] = TR[(tL * 5 + n) * M2 + pt];
    VR[n] = TR[(tR * 5 + n) * M2 + pt];
  }
  TraceCartesianGrad<M2>(TR, tL, d, pt, fmL, a.metric_compat, gxL, gyL, gzL);
  TraceCartesianGrad<M2>(TR, tR, d, pt, fmR, a.metric_compat, gxR, gyR, gzR);
  double gx[5], gy[5], gz[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    gx[n] = 0.5 * (gxL[n] + gxR[n]);
    gy[n] = 0.5 * (gyL[n] + gyR[n]);
    gz[n] = 0.5 * (gzL[n] + gzR[n]);
  }
  const int f = pt % M, sl = pt / M;
  const double wf = c_ops[SLOT].w[f] * c_ops[SLOT].w[sl];
  const double nx = 1.0 * __ldg(fmL + 0 * M2 + pt), ny = 1.0 * __ldg(fmL + 1 * M2 + pt),
               nz = 1.0 * __ldg(fmL + 2 * M2 + pt);
  const double area = __ldg(fmL + 3 * M2 + pt);
  double flux[5];
  if (a.riemann == 1)
    IsmailRoeFlux(VL, VR, nx, ny, nz, wf * area, flux);
  else
    RoeFlux(VL, VR, nx, ny, nz, 0.5 * wf * area, flux);
  double sx[5], sy[5], sz[5];
  ViscousPenaltySymFlux(VL, VR, gx, gy, gz, nx, ny, nz, 1.0, wf, area, a.mu,
                        a.tau_num / lenScale, a.theta_sym, flux, sx, sy, sz);
  const double *fm = g == 0 ? fmR : fmL;  // the own side's metric
  const int pFast = FastParam(d);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    const int mi = a.metric_compat ? n : pt;
    double sym[3];
#pragma unroll
    for (int p = 0; p < 3; ++p)
      sym[p] = sx[n] * __ldg(fm + (4 + 3 * p) * M2 + mi) +
               sy[n] * __ldg(fm + (5 + 3 * p) * M2 + mi) +
               sz[n] * __ldg(fm + (6 + 3 * p) * M2 + mi);
    const int o = (d * 5 + n) * M2 + pt;
    P1[1 * 15 * M2 + o] = g == 0 ? -flux[n] : flux[n];
    P1[2 * 15 * M2 + o] = sym[d];
    P1[0 * 15 * M2 + o] = sym[pFast];
    P2[o] = sym[3 - d - pFast];
  }
}

template <int NT, int K, int M>
__device__ __forceinline__ void FacePhase(const ResidualArgs &a, const int e, const double *s_sol,
                                          double *s_R, const double *s_fv, double *work) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K, M2 = M * M, K2 = K * K;
  static_assert(2 * M <= 3 * K && K <= 2 * M, "face-phase buffer aliasing");
  double *BN = work, *BND = BN + 30 * K2;        // 60 K^2
  double *T1a = BND + 30 * K2, *T1b = T1a + 30 * K * M, *T1c = T1b + 30 * K * M;  // 90 K M
  double *TR = T1c + 30 * K * M;                 // 120 M^2
  double *P1 = T1a, *P2 = T1a + 45 * M2;         // distribution inputs (in T1)
  double *Q1 = TR, *Q2 = TR + 45 * K * M;        // after the slow-axis contraction (in TR)
  double *RF = BN, *RFN = RF + 15 * K2, *RS = RFN + 30 * K2;  // after the fast axis (in BN)
  const double *sc = a.elem_scalars + (size_t)e * 15;
  for (int g = 0; g < 2; ++g) {
    const int nb0 = a.nbr[e * 6 + 0 + g], nb1 = a.nbr[e * 6 + 2 + g], nb2 = a.nbr[e * 6 + 4 + g];
    // Traces of the six sides (TPSAG[IJK]): normal, fast axis, slow axis.
    FaceNormalBatch<NT, SLOT, K>(s_sol, a.sol, nb0, nb1, nb2, g, s_fv, BN, BND);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLeg, 0, 30, K, K, 1, K, M, false>(BN, T1a);
    Contract<NT, SLOT, K, M, kDLeg, 0, 30, K, K, 1, K, M, false>(BN, T1b);
    Contract<NT, SLOT, K, M, kLeg, 0, 30, K, K, 1, K, M, false>(BND, T1c);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1a, TR);
    Contract<NT, SLOT, K, M, kDLeg, 1, 30, M, K, 1, K, M, false>(T1a, TR + 3 * 30 * M2);
    Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1b, TR + 2 * 30 * M2);
    Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1c, TR + 1 * 30 * M2);
    __syncthreads();
    // Pointwise fluxes of the three faces.
    for (int idx = threadIdx.x; idx < 3 * M2; idx += NT) {
      const int d = idx / M2, pt = idx - d * M2;
      const int nb = d == 0 ? nb0 : (d == 1 ? nb1 : nb2);
      if (nb < 0) {
        // Physical boundary faces are not part of this interior-face path.
        if (pt == 0) atomicAdd(a.status + 1, 1);
        for (int n = 0; n < 5; ++n) {
          const int o = (d * 5 + n) * M2 + pt;
          P1[o] = P1[15 * M2 + o] = P1[30 * M2 + o] = P2[o] = 0.0;
        }
        continue;
      }
      const double lenScale = fmin(sc[d], a.elem_scalars[(size_t)nb * 15 + d]);
      const double *fmOwn = a.face_metric + ((size_t)e * 6 + 2 * d + g) * 13 * M2;
      const double *fmNb = a.face_metric + ((size_t)nb * 6 + 2 * d + 1 - g) * 13 * M2;
      GroupFacePoint<K, M>(a, g, d, pt, TR, fmOwn, fmNb, lenScale, P1, P2);
    }
    __syncthreads();
    // Distribution (TPR[IJK]F): slow axis, fast axis, then the face-normal expansion.
    Contract<NT, SLOT, K, M, kLegT, 1, 45, M, M, 1, M, K, false>(P1, Q1);
    Contract<NT, SLOT, K, M, kDLegT, 1, 15, M, M, 1, M, K, false>(P2, Q2);
    __syncthreads();
    Contract<NT, SLOT, K, M, kDLegT, 0, 15, M, K, 1, M, K, false>(Q1, RF);
    Contract<NT, SLOT, K, M, kLegT, 0, 30, M, K, 1, M, K, false>(Q1 + 15 * K * M, RFN);
    Contract<NT, SLOT, K, M, kLegT, 0, 15, M, K, 1, M, K, false>(Q2, RS);
    __syncthreads();
    const double *fv = s_fv + g * K, *dfv = s_fv + (2 + g) * K;
    for (int idx = threadIdx.x; idx < 5 * KD; idx += NT) {
      const int v = idx / KD, r = idx - v * KD;
      const int k = r / K2, r2 = r - k * K2, j = r2 / K, i = r2 - j * K;
      double acc = s_R[idx];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int n = d == 0 ? i : (d == 1 ? j : k);
        const int sf = d == 0 ? k * K + j : (d == 1 ? k * K + i : j * K + i);
        const int o = (d * 5 + v) * K2 + sf;
        const double aF = fv[n], aD = dfv[n];
        const double tFlux = RFN[o], tN = RFN[15 * K2 + o], tFast = RF[o], tSlow = RS[o];
        // Reference order: normal flux, then the r, s, t symmetrizing fluxes.
        const int pFast = FastParam(d);
        double c = g == 0 ? acc : 0.0;
        c = fma(aF, tFlux, c);
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          if (p == d) c = fma(aD, tN, c);
          else if (p == pFast) c = fma(aF, tFast, c);
          else c = fma(aF, tSlow, c);
        }
        acc = g == 0 ? c : acc + c;
      }
      s_R[idx] = acc;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Generalised mass-matrix solve, CG_EntropyVarMassMatrix
// (src/CG_MassMatrix.cpp:250-504): flexible PCG with the element-centre
// dV/dU * 8/vol preconditioner, stop at ||r||_inf < 1e-10 ||r0||_inf, at most
// 100 iterations (the cap raises a status flag instead of aborting).
// r is s_R (overwritten); the solution is returned in x.
// ---------------------------------------------------------------------------
template <int NT, int K, int M>
__device__ __forceinline__ void MassSolve(const ResidualArgs &a, const int e, const double *s_sol,
                                          double *s_R, const double *s_cgp, const double *s_jw,
                                          double *work, double *s_red, double *&xOut) {
  constexpr int SLOT = Slot<K, M>::value;
  using P = Plan<K, M>;
  constexpr int KD = P::KD, MD = P::MD;
  double *z = work, *p = z + 5 * KD, *Ap = p + 5 * KD, *x = Ap + 5 * KD;
  double *pInt = x + 5 * KD, *tK = pInt + 5 * MD, *tJ = tK + P::TK;
  double *dvdu = s_red + 32;  // 15 preconditioner entries
  double *r = s_R;
  xOut = x;
  const double volElem = a.elem_scalars[(size_t)e * 15 + 5];
  const double JacInv = 8.0 / volElem;

  double m = 0.0;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) {
    m = fmax(m, fabs(r[i]));
    x[i] = 0.0;
  }
  const double rInitMax = BlockMax<NT>(m, s_red);
  if (!(rInitMax * JacInv > 1.e-10)) return;

  // Entropy variables at the element centre and dV/dU there (src/CG_MassMatrix.cpp:313-361).
  if (threadIdx.x < 5) {
    double V = 0.0;
    for (int l = 0; l < KD; ++l) V += c_ops[SLOT].center[l] * s_sol[threadIdx.x * KD + l];
    dvdu[threadIdx.x + 16] = V;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double gm1 = kGam - 1.0, ov1mg = 1.0 / (1.0 - kGam), govgm1 = kGam / gm1;
    const double V0 = dvdu[16], V1 = dvdu[17], V2 = dvdu[18], V3 = dvdu[19], V4 = dvdu[20];
    const double V4Inv = 1.0 / V4;
    const double u = -V4Inv * V1, v = -V4Inv * V2, w = -V4Inv * V3;
    const double eKin = 0.5 * (u * u + v * v + w * w);
    const double sEnt = kGam - gm1 * (V0 - V4 * eKin);
    const double tmp = -V4 * exp(sEnt);
    const double rho = pow(tmp, ov1mg);
    const double pr = -rho * V4Inv;
    const double pInv = 1.0 / pr;
    const double abv1 = gm1 * rho * pInv * pInv;
    const double abv2 = eKin * abv1;
    dvdu[0] = JacInv * (govgm1 / rho + abv2 * eKin);
    dvdu[1] = -JacInv * u * abv2;
    dvdu[2] = -JacInv * v * abv2;
    dvdu[3] = -JacInv * w * abv2;
    dvdu[4] = JacInv * (abv2 - pInv);
    dvdu[5] = JacInv * (abv1 * u * u + pInv);
    dvdu[6] = JacInv * abv1 * u * v;
    dvdu[7] = JacInv * abv1 * u * w;
    dvdu[8] = -JacInv * abv1 * u;
    dvdu[9] = JacInv * (abv1 * v * v + pInv);
    dvdu[10] = JacInv * abv1 * v * w;
    dvdu[11] = -JacInv * abv1 * v;
    dvdu[12] = JacInv * (abv1 * w * w + pInv);
    dvdu[13] = -JacInv * abv1 * w;
    dvdu[14] = JacInv * abv1;
  }
  __syncthreads();
  double D[15];
#pragma unroll
  for (int q = 0; q < 15; ++q) D[q] = dvdu[q];
  auto precond = [&](void) {
    for (int l = threadIdx.x; l < KD; l += NT) {
      const double r0 = r[l], r1 = r[KD + l], r2 = r[2 * KD + l], r3 = r[3 * KD + l],
                   r4 = r[4 * KD + l];
      z[l] = D[0] * r0 + D[1] * r1 + D[2] * r2 + D[3] * r3 + D[4] * r4;
      z[KD + l] = D[1] * r0 + D[5] * r1 + D[6] * r2 + D[7] * r3 + D[8] * r4;
      z[2 * KD + l] = D[2] * r0 + D[6] * r1 + D[9] * r2 + D[10] * r3 + D[11] * r4;
      z[3 * KD + l] = D[3] * r0 + D[7] * r1 + D[10] * r2 + D[12] * r3 + D[13] * r4;
      z[4 * KD + l] = D[4] * r0 + D[8] * r1 + D[11] * r2 + D[13] * r3 + D[14] * r4;
    }
  };
  precond();
  __syncthreads();
  double part = 0.0;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) {
    p[i] = z[i];
    part = fma(r[i], z[i], part);
  }
  double dotrz = BlockSum<NT>(part, s_red);

  int iter = 0;
  for (;; ++iter) {
    if (iter == 100) {
      if (threadIdx.x == 0) atomicAdd(a.status, 1);
      break;
    }
    // Ap = Leg^T3 (w J dU/dV (Leg3 p)) (src/CG_MassMatrix.cpp:408-443).
    Contract<NT, SLOT, K, M, kLeg, 2, 5, K, K, K, K, M, false>(p, tK);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false>(tK, tJ);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false>(tJ, pInt);
    __syncthreads();
    for (int l = threadIdx.x; l < MD; l += NT) {
      const double iw = s_jw[l];
      const double p0 = iw * pInt[l], p1 = iw * pInt[MD + l], p2 = iw * pInt[2 * MD + l],
                   p3 = iw * pInt[3 * MD + l], p4 = iw * pInt[4 * MD + l];
      const double rho = s_cgp[l], u = s_cgp[MD + l], v = s_cgp[2 * MD + l],
                   w = s_cgp[3 * MD + l], pr = s_cgp[4 * MD + l], rE = s_cgp[5 * MD + l];
      const double ru = rho * u, rv = rho * v, rw = rho * w, rH = rE + pr;
      const double d0 = rho, d1 = ru, d2 = rv, d3 = rw, d4 = rE, d5 = ru * u + pr, d6 = ru * v,
                   d7 = ru * w, d8 = rH * u, d9 = rv * v + pr, d10 = rv * w, d11 = rH * v,
                   d12 = rw * w + pr, d13 = rH * w, d14 = s_cgp[6 * MD + l];
      pInt[l] = d0 * p0 + d1 * p1 + d2 * p2 + d3 * p3 + d4 * p4;
      pInt[MD + l] = d1 * p0 + d5 * p1 + d6 * p2 + d7 * p3 + d8 * p4;
      pInt[2 * MD + l] = d2 * p0 + d6 * p1 + d9 * p2 + d10 * p3 + d11 * p4;
      pInt[3 * MD + l] = d3 * p0 + d7 * p1 + d10 * p2 + d12 * p3 + d13 * p4;
      pInt[4 * MD + l] = d4 * p0 + d8 * p1 + d11 * p2 + d13 * p3 + d14 * p4;
    }
    __syncthreads();
    Contract<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false>(pInt, tJ);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false>(tJ, tK);
    __syncthreads();
    Contract<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, false>(tK, Ap);
    __syncthreads();
    part = 0.0;
    for (int i = threadIdx.x; i < 5 * KD; i += NT) part = fma(p[i], Ap[i], part);
    const double alpha = dotrz / BlockSum<NT>(part, s_red);
    // Each thread owns whole DOFs: update x and r, precondition, and form the
    // partial sums of the three reductions that close the iteration.
    double zAp = 0.0, rzNew = 0.0, rMax = 0.0;
    for (int l = threadIdx.x; l < KD; l += NT) {
      double rr[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        x[q * KD + l] = fma(alpha, p[q * KD + l], x[q * KD + l]);
        rr[q] = fma(-alpha, Ap[q * KD + l], r[q * KD + l]);
        r[q * KD + l] = rr[q];
        rMax = fmax(rMax, fabs(rr[q]));
      }
      const double zz[5] = {
          D[0] * rr[0] + D[1] * rr[1] + D[2] * rr[2] + D[3] * rr[3] + D[4] * rr[4],
          D[1] * rr[0] + D[5] * rr[1] + D[6] * rr[2] + D[7] * rr[3] + D[8] * rr[4],
          D[2] * rr[0] + D[6] * rr[1] + D[9] * rr[2] + D[10] * rr[3] + D[11] * rr[4],
          D[3] * rr[0] + D[7] * rr[1] + D[10] * rr[2] + D[12] * rr[3] + D[13] * rr[4],
          D[4] * rr[0] + D[8] * rr[1] + D[11] * rr[2] + D[13] * rr[3] + D[14] * rr[4]};
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        z[q * KD + l] = zz[q];
        zAp = fma(zz[q], Ap[q * KD + l], zAp);
        rzNew = fma(rr[q], zz[q], rzNew);
      }
    }
    BlockReduce3<NT>(zAp, rzNew, rMax, s_red);
    if (rMax < 1.e-10 * rInitMax) break;
    const double beta = -alpha * zAp / dotrz;
    dotrz = rzNew;
    for (int i = threadIdx.x; i < 5 * KD; i += NT) p[i] = beta * p[i] + z[i];
    __syncthreads();
  }
  if (threadIdx.x == 0 && a.cg_stats) {
    atomicAdd(a.cg_stats, (unsigned long long)(iter + 1));
    atomicAdd(a.cg_stats + 1, 1ull);
  }
}

// ---------------------------------------------------------------------------
// The fused kernel.
// ---------------------------------------------------------------------------
template <int K, int M, int NT>
__global__ void __launch_bounds__(NT, Plan<K, M>::MIN_BLOCKS) ResidualKernel(const ResidualArgs a) {
  using P = Plan<K, M>;
  constexpr int KD = P::KD, MD = P::MD;
  extern __shared__ double smem[];
  double *s_sol = smem, *s_R = s_sol + 5 * KD, *s_cgp = s_R + 5 * KD, *s_jw = s_cgp + 8 * MD;
  double *s_red = s_jw + MD, *s_fv = s_red + 64, *work = s_fv + 4 * kKMax;
  const int e = blockIdx.x;
  if (e >= a.n_elem) return;
  const double *src = a.sol + (size_t)e * 5 * KD;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = src[i];
  if (threadIdx.x < 2 * K) {
    s_fv[threadIdx.x] = c_ops[Slot<K, M>::value].face[threadIdx.x];
    s_fv[2 * K + threadIdx.x] = c_ops[Slot<K, M>::value].dface[threadIdx.x];
  }
  __syncthreads();
  VolumePhase<NT, K, M>(a, e, s_sol, s_R, s_cgp, s_jw, work, s_red);
  FacePhase<NT, K, M>(a, e, s_sol, s_R, s_fv, work);
  if (a.res_raw) {
    double *dst = a.res_raw + (size_t)e * 5 * KD;
    for (int i = threadIdx.x; i < 5 * KD; i += NT) dst[i] = s_R[i];
  }
  __syncthreads();
  double *x;
  MassSolve<NT, K, M>(a, e, s_sol, s_R, s_cgp, s_jw, work, s_red, x);
  __syncthreads();
  double *dst = a.res + (size_t)e * 5 * KD;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) dst[i] = x[i];
}

}  // namespace vcpg
