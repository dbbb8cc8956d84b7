// CFL time step per element, ElementClass::ComputeTimeStep
// (src/ElementClass.cpp:1522-1644) with ComputePrimitiveVariablesNodalDOFs
// (:1500-1520) and the spectral-radius factors f1 / f2 of
// SolverClass::ExecuteTimeSynchronizationStep (src/SolverClass.cpp:2182-2189).
// The per-element arithmetic lives in ElementTimeStep, shared by the handle's
// TimeStepKernel (global minimum by an atomic min on the bit pattern of the
// positive double) and the allocation-free entry point (noalloc.cu).
#pragma once

#include "dg_residual.cuh"

namespace vcpg {

// Shared memory of TimeStepKernel in doubles; above the 48 KB of static shared
// memory (degrees 7-9) it is dynamic.
template <int K> struct TimeStepSmem {
  static constexpr int N = 15 * K * K * K + 64;
  static constexpr bool DYN = N * 8 > 48 * 1024;
};

// dt = CFL u_ref / (f1[p] radInv + f2[p] radVis) (src/ElementClass.cpp:1636-1643).
__device__ __forceinline__ double CflElementStep(const int n_poly, const double cfl,
                                                 const double uRef, const double radInvMax,
                                                 const double radVisMax) {
  const double f1[] = {2.0, 6.0, 12.0, 20.0, 28.0, 38.0, 50.0, 64.0, 80.0, 98.0};
  const double f2[] = {6.0, 36.0, 150.0, 420.0, 980.0, 1975.0, 3575.0, 7000.0, 14000.0, 28000.0};
  const double dtInv = f1[n_poly] * radInvMax + f2[n_poly] * radVisMax;
  return cfl * uRef / dtInv;
}

// The time step of one element without a subgrid-scale model: modal -> nodal
// (Legendre basis at the nodal DOFs), dimensional primitive variables,
// inviscid and viscous spectral radii. src: the element's modal state [5][K^3];
// sc: its 15 scalars (length scales, averaged normals). The three work arrays
// hold 5 K^3 doubles each, s_red 64. Returns, on thread 0 only, the element's
// step; *bad is set (thread 0) when a^2 is negative or not a number somewhere
// (the reference terminates on a^2 < 0; a NaN state is reported the same way).
template <int K, int M, int NT>
__device__ __forceinline__ double ElementTimeStep(const double *src, const double *sc,
                                                  const int n_poly, const double cfl,
                                                  const double mu, const double pRef,
                                                  const double uRef, const double rhoRef,
                                                  double *s_sol, double *s_t1, double *s_t2,
                                                  double *s_red, bool *bad) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = src[i];
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 2, 5, K, K, K, K, K, false>(s_sol, s_t1);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 1, 5, K, K, K, K, K, false>(s_t1, s_t2);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 0, 5, K, K, K, K, K, false>(s_t2, s_t1);
  __syncthreads();
  const double muDim = mu * pRef / uRef;
  const double dliInv = 1.0 / sc[0], dljInv = 1.0 / sc[1], dlkInv = 1.0 / sc[2];
  const double dli2Inv = dliInv * dliInv, dlj2Inv = dljInv * dljInv, dlk2Inv = dlkInv * dlkInv;
  const double dLen2Inv = dli2Inv + dlj2Inv + dlk2Inv;
  const double radVisOverNuLam = fmax(fmax(1.0, 2.0 + kLamOverMu), kFactHFLam) * dLen2Inv;
  double radInvMax = 0.0, radVisMax = 0.0, a2Bad = 0.0;
  for (int l = threadIdx.x; l < KD; l += NT) {
    double rho, u, v, w, p, eKin;
    EntropyToPrim(s_t1[l], s_t1[KD + l], s_t1[2 * KD + l], s_t1[3 * KD + l], s_t1[4 * KD + l],
                  rho, u, v, w, p, eKin);
    rho *= rhoRef; u *= uRef; v *= uRef; w *= uRef; p *= pRef;
    const double rhoInv = 1.0 / rho;
    const double a2 = kGam * p * rhoInv;
    const double velI = u * sc[6] + v * sc[7] + w * sc[8];
    const double velJ = u * sc[9] + v * sc[10] + w * sc[11];
    const double velK = u * sc[12] + v * sc[13] + w * sc[14];
    const double aa = sqrt(fabs(a2));
    const double radInv = (fabs(velI) + aa) * dliInv + (fabs(velJ) + aa) * dljInv +
                          (fabs(velK) + aa) * dlkInv;
    const double radVis = rhoInv * (muDim * radVisOverNuLam + 0.0);
    radInvMax = fmax(radInvMax, radInv);
    radVisMax = fmax(radVisMax, radVis);
    if (!(a2 >= 0.0)) a2Bad = 1.0;
  }
  radInvMax = BlockMax<NT>(radInvMax, s_red);
  radVisMax = BlockMax<NT>(radVisMax, s_red);
  a2Bad = BlockMax<NT>(a2Bad, s_red);
  if (threadIdx.x == 0) *bad = a2Bad != 0.0;
  return CflElementStep(n_poly, cfl, uRef, radInvMax, radVisMax);
}

template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) TimeStepKernel(const TimeStepArgs a) {
  constexpr int KD = K * K * K;
  using SM = TimeStepSmem<K>;
  __shared__ double s_static[SM::DYN ? 1 : SM::N];
  extern __shared__ __align__(16) double sm_ts[];
  double *s_sol = SM::DYN ? sm_ts : s_static;
  double *s_t1 = s_sol + 5 * KD, *s_t2 = s_t1 + 5 * KD, *s_red = s_t2 + 5 * KD;
  const int e = blockIdx.x;
  if (e >= a.n_elem) return;
  // Several cases per launch: per-case parameters, pending and running cases only.
  int cs = 0;
  double cfl = a.cfl, mu = a.mu, pRef = a.p_ref, uRef = a.u_ref, rhoRef = a.rho_ref;
  if (a.cases.elem_case) {
    cs = a.cases.elem_case[e];
    if (cs < 0) return;
    const int st = a.cases.state[cs];
    if (st != kCasePending && st != kCaseRunning) return;
    const double *pc = a.cases.par + cs * kCasePar;
    mu = pc[kParMu]; pRef = pc[kParPRef]; uRef = pc[kParURef]; rhoRef = pc[kParRhoRef];
    cfl = pc[kParCfl];
  }
  bool bad = false;
  const double dtElem = ElementTimeStep<K, M, NT>(a.sol + (size_t)e * 5 * KD,
                                                  a.elem_scalars + (size_t)e * 15, a.n_poly, cfl,
                                                  mu, pRef, uRef, rhoRef, s_sol, s_t1, s_t2,
                                                  s_red, &bad);
  if (threadIdx.x == 0) {
    if (bad) atomicAdd(a.status + 2, 1);
    atomicMin(a.dt_bits + cs, (unsigned long long)__double_as_longlong(dtElem));
  }
}

// The time step with a subgrid-scale model (the SGS branch of
// ElementClass::ComputeTimeStep): the eddy viscosity at the nodal DOFs from
// ComputeVelocityGradientsNodalDOFs (src/ElementClass.cpp:1649-1800; gradients of
// the entropy variables V1..V4 at the DOFs, the metric at the DOFs, dimensional
// velocity gradients) and the model, added to the viscous spectral radius.
// Dynamic shared memory: state, nodal values, two stage buffers (5 K^3 each)
// and the three parametric gradients of V1..V4 (12 K^3).
template <int K, int M, int NT>
__device__ __forceinline__ void TimeStepSgsElement(const TimeStepArgs &a, const int e,
                                                   double *sm_ts, double *s_red) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K;
  double *s_sol = sm_ts, *s_val = s_sol + 5 * KD, *tA = s_val + 5 * KD, *tB = tA + 5 * KD;
  double *gr = tB + 5 * KD;  // [3][4][KD]: d/dr, d/ds, d/dt of V1..V4
  int cs = 0;
  double cfl = a.cfl, mu = a.mu, pRef = a.p_ref, uRef = a.u_ref, rhoRef = a.rho_ref;
  if (a.cases.elem_case) {
    cs = a.cases.elem_case[e];
    if (cs < 0) return;
    const int st = a.cases.state[cs];
    if (st != kCasePending && st != kCaseRunning) return;
    const double *pc = a.cases.par + cs * kCasePar;
    mu = pc[kParMu]; pRef = pc[kParPRef]; uRef = pc[kParURef]; rhoRef = pc[kParRhoRef];
    cfl = pc[kParCfl];
  }
  const double *src = a.sol + (size_t)e * 5 * KD;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = src[i];
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 2, 5, K, K, K, K, K, false>(s_sol, tA);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 1, 5, K, K, K, K, K, false>(tA, tB);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 0, 5, K, K, K, K, K, false>(tB, s_val);
  __syncthreads();
  const double *V1 = s_sol + KD;  // entropy variables 1..4
  // d/dr: derivative along i (the last stage).
  Contract<NT, SLOT, K, M, kLegDof, 2, 4, K, K, K, K, K, false>(V1, tA);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 1, 4, K, K, K, K, K, false>(tA, tB);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegDof, 0, 4, K, K, K, K, K, false>(tB, gr);
  __syncthreads();
  // d/ds: derivative along j.
  Contract<NT, SLOT, K, M, kLegDof, 2, 4, K, K, K, K, K, false>(V1, tA);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegDof, 1, 4, K, K, K, K, K, false>(tA, tB);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 0, 4, K, K, K, K, K, false>(tB, gr + 4 * KD);
  __syncthreads();
  // d/dt: derivative along k.
  Contract<NT, SLOT, K, M, kDLegDof, 2, 4, K, K, K, K, K, false>(V1, tA);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 1, 4, K, K, K, K, K, false>(tA, tB);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 0, 4, K, K, K, K, K, false>(tB, gr + 8 * KD);
  __syncthreads();
  const double *sc = a.elem_scalars + (size_t)e * 15;
  const double *nm = a.vol_metric_dofs + (size_t)e * 10 * KD;
  const double muDim = mu * pRef / uRef;
  const double uRefInv = 1.0 / uRef;
  const double dliInv = 1.0 / sc[0], dljInv = 1.0 / sc[1], dlkInv = 1.0 / sc[2];
  const double dli2Inv = dliInv * dliInv, dlj2Inv = dljInv * dljInv, dlk2Inv = dlkInv * dlkInv;
  const double dLen2Inv = dli2Inv + dlj2Inv + dlk2Inv;
  const double radVisOverNuLam = fmax(fmax(1.0, 2.0 + kLamOverMu), kFactHFLam) * dLen2Inv;
  const double radVisOverNuTurb = fmax(fmax(1.0, 2.0 + kLamOverMu), kFactHFTurb) * dLen2Inv;
  double radInvMax = 0.0, radVisMax = 0.0, a2Bad = 0.0;
  for (int l = threadIdx.x; l < KD; l += NT) {
    double rho, u, v, w, p, eKin;
    EntropyToPrim(s_val[l], s_val[KD + l], s_val[2 * KD + l], s_val[3 * KD + l],
                  s_val[4 * KD + l], rho, u, v, w, p, eKin);
    rho *= rhoRef; u *= uRef; v *= uRef; w *= uRef; p *= pRef;
    // Velocity gradients in computational space from the entropy-variable
    // gradients, then Cartesian and dimensional.
    const double un = u * uRefInv, vn = v * uRefInv, wn = w * uRefInv;
    const double V4Inv = -p * uRefInv * uRefInv / rho;
    double dv[3][3];  // [velocity][parameter]
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double *G = gr + q * 4 * KD;
      const double d4 = G[3 * KD + l];
      dv[0][q] = -V4Inv * (G[l] + un * d4);
      dv[1][q] = -V4Inv * (G[KD + l] + vn * d4);
      dv[2][q] = -V4Inv * (G[2 * KD + l] + wn * d4);
    }
    const double drdx = nm[1 * KD + l], drdy = nm[2 * KD + l], drdz = nm[3 * KD + l];
    const double dsdx = nm[4 * KD + l], dsdy = nm[5 * KD + l], dsdz = nm[6 * KD + l];
    const double dtdx = nm[7 * KD + l], dtdy = nm[8 * KD + l], dtdz = nm[9 * KD + l];
    double g[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      g[c] = uRef * (dv[c][0] * drdx + dv[c][1] * dsdx + dv[c][2] * dtdx);
      g[3 + c] = uRef * (dv[c][0] * drdy + dv[c][1] * dsdy + dv[c][2] * dtdy);
      g[6 + c] = uRef * (dv[c][0] * drdz + dv[c][1] * dsdz + dv[c][2] * dtdz);
    }
    const double eddy = EddyViscosity(a.sgs, sc[3], rho, g);
    const double rhoInv = 1.0 / rho;
    const double a2 = kGam * p * rhoInv;
    const double velI = u * sc[6] + v * sc[7] + w * sc[8];
    const double velJ = u * sc[9] + v * sc[10] + w * sc[11];
    const double velK = u * sc[12] + v * sc[13] + w * sc[14];
    const double aa = sqrt(fabs(a2));
    const double radInv = (fabs(velI) + aa) * dliInv + (fabs(velJ) + aa) * dljInv +
                          (fabs(velK) + aa) * dlkInv;
    const double radVis = rhoInv * (muDim * radVisOverNuLam + eddy * radVisOverNuTurb);
    radInvMax = fmax(radInvMax, radInv);
    radVisMax = fmax(radVisMax, radVis);
    if (!(a2 >= 0.0)) a2Bad = 1.0;
  }
  radInvMax = BlockMax<NT>(radInvMax, s_red);
  radVisMax = BlockMax<NT>(radVisMax, s_red);
  a2Bad = BlockMax<NT>(a2Bad, s_red);
  if (threadIdx.x == 0) {
    if (a2Bad != 0.0) atomicAdd(a.status + 2, 1);
    const double dtElem = CflElementStep(a.n_poly, cfl, uRef, radInvMax, radVisMax);
    atomicMin(a.dt_bits + cs, (unsigned long long)__double_as_longlong(dtElem));
  }
}

// The 32 K^3 doubles of an element in shared memory, or above one CTA's shared
// memory (degree 9) in the handle's global scratch, one area per CTA of a grid
// that loops over the elements.
template <int K> struct TimeStepSgsSmem {
  static constexpr size_t BYTES = sizeof(double) * 32 * K * K * K;
  static constexpr bool BIG = BYTES > 227 * 1024;
};

template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) TimeStepSgsKernel(const TimeStepArgs a) {
  extern __shared__ __align__(16) double sm_ts[];
  __shared__ double s_red[64];
  if constexpr (TimeStepSgsSmem<K>::BIG) {
    double *base = reinterpret_cast<double *>(a.scratch) + (size_t)blockIdx.x * 32 * K * K * K;
    for (int e = blockIdx.x; e < a.n_elem; e += gridDim.x) {
      TimeStepSgsElement<K, M, NT>(a, e, base, s_red);
      __syncthreads();
    }
  } else {
    if ((int)blockIdx.x >= a.n_elem) return;
    TimeStepSgsElement<K, M, NT>(a, blockIdx.x, sm_ts, s_red);
  }
}

}  // namespace vcpg
