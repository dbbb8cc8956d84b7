// Kernel instantiations and launchers for every supported (K, M) pair:
// the fused residual kernel, the CFL time-step kernel and the Runge-Kutta
// stage updates.
#include <cstring>

#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "kernels.h"

namespace vcpg {

// ---------------------------------------------------------------------------
// Time step per element, ElementClass::ComputeTimeStep (src/ElementClass.cpp:1522-1644)
// with ComputePrimitiveVariablesNodalDOFs (:1500-1520); global minimum via an
// atomic min on the bit pattern of the (positive) double.
// ---------------------------------------------------------------------------


// Shared memory of TimeStepKernel in doubles; above the 48 KB of static shared
// memory (degrees 7-9) it is dynamic.
template <int K> struct TimeStepSmem {
  static constexpr int N = 15 * K * K * K + 64;
  static constexpr bool DYN = N * 8 > 48 * 1024;
};

template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) TimeStepKernel(const TimeStepArgs a) {
  constexpr int SLOT = Slot<K, M>::value;
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
  const double *src = a.sol + (size_t)e * 5 * KD;
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = src[i];
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 2, 5, K, K, K, K, K, false>(s_sol, s_t1);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 1, 5, K, K, K, K, K, false>(s_t1, s_t2);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLegDof, 0, 5, K, K, K, K, K, false>(s_t2, s_t1);
  __syncthreads();
  const double *sc = a.elem_scalars + (size_t)e * 15;
  const double muDim = mu * pRef / uRef;
  const double dliInv = 1.0 / sc[0], dljInv = 1.0 / sc[1], dlkInv = 1.0 / sc[2];
  const double dli2Inv = dliInv * dliInv, dlj2Inv = dljInv * dljInv, dlk2Inv = dlkInv * dlkInv;
  const double dLen2Inv = dli2Inv + dlj2Inv + dlk2Inv;
  const double radVisOverNuLam = fmax(fmax(1.0, 2.0 + kLamOverMu), kFactHFLam) * dLen2Inv;
  double radInvMax = 0.0, radVisMax = 0.0, a2Min = 1.e+10;
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
    a2Min = fmin(a2Min, a2);
  }
  radInvMax = BlockMax<NT>(radInvMax, s_red);
  radVisMax = BlockMax<NT>(radVisMax, s_red);
  a2Min = -BlockMax<NT>(-a2Min, s_red);
  if (threadIdx.x == 0) {
    if (a2Min < 0.0) atomicAdd(a.status + 2, 1);
    const double f1[] = {2.0, 6.0, 12.0, 20.0, 28.0, 38.0, 50.0, 64.0, 80.0, 98.0};
    const double f2[] = {6.0, 36.0, 150.0, 420.0, 980.0, 1975.0, 3575.0, 7000.0, 14000.0, 28000.0};
    const double dtInv = f1[a.n_poly] * radInvMax + f2[a.n_poly] * radVisMax;
    const double dtElem = cfl * uRef / dtInv;
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
  double radInvMax = 0.0, radVisMax = 0.0, a2Min = 1.e+10;
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
    a2Min = fmin(a2Min, a2);
  }
  radInvMax = BlockMax<NT>(radInvMax, s_red);
  radVisMax = BlockMax<NT>(radVisMax, s_red);
  a2Min = -BlockMax<NT>(-a2Min, s_red);
  if (threadIdx.x == 0) {
    if (a2Min < 0.0) atomicAdd(a.status + 2, 1);
    const double f1[] = {2.0, 6.0, 12.0, 20.0, 28.0, 38.0, 50.0, 64.0, 80.0, 98.0};
    const double f2[] = {6.0, 36.0, 150.0, 420.0, 980.0, 1975.0, 3575.0, 7000.0, 14000.0, 28000.0};
    const double dtInv = f1[a.n_poly] * radInvMax + f2[a.n_poly] * radVisMax;
    const double dtElem = cfl * uRef / dtInv;
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

// Reads the reduced time step (or the fixed one), records it and re-arms the reduction.
__global__ void FinalizeDtKernel(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                                 double *hist, int hist_cap, int *counter) {
  const double fx = *fixed_dt;
  const double dt = fx > 0.0 ? fx : __longlong_as_double((long long)*dt_bits);
  *d_dt = dt;
  const int c = *counter;
  if (c < hist_cap) hist[c] = dt;
  *counter = c + 1;
  *dt_bits = (unsigned long long)__double_as_longlong(1.e+10);
}

// Case of state entry i for several cases per launch (elem_case non-null):
// -1 unless the case is running. One case: 0.
__device__ __forceinline__ int StageCase(const CaseView &cv, const size_t i, const int elemSize) {
  if (!cv.elem_case) return 0;
  const int c = cv.elem_case[i / (size_t)elemSize];
  return (c >= 0 && cv.state[c] == kCaseRunning) ? c : -1;
}

// Per-case start of a time step in a bucket holding several cases: a pending
// case (its residual was evaluated earlier in this step) starts running; a
// running case that has taken its target steps is done (time step 0, skipped
// by every later kernel); otherwise its reduced CFL step is taken and counted.
__global__ void EnsembleFinalizeKernel(int n_cases, int *state, const int *target, int *done,
                                       unsigned long long *dt_bits, double *dt,
                                       double *sim_time) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cases) return;
  int st = state[c];
  if (st == kCasePending) st = kCaseRunning;
  if (st == kCaseRunning) {
    if (done[c] >= target[c]) {
      st = kCaseDone;
      dt[c] = 0.0;
    } else {
      const double d = __longlong_as_double((long long)dt_bits[c]);
      dt[c] = d;
      sim_time[c] += d;
      done[c] += 1;
    }
  }
  state[c] = st;
  dt_bits[c] = (unsigned long long)__double_as_longlong(1.e+10);
}

// SSP-RK3 stage (src/SolverClass.cpp:2368-2396); stage 0 also stores solOld.
__global__ void SspStageKernel(double *sol, double *solOld, const double *res, const double *d_dt,
                               double alpha, double beta, int copyOld, size_t n,
                               const CaseView cv, int elemSize) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = StageCase(cv, i, elemSize);
  if (c < 0) return;
  const double betaDt = beta * d_dt[c];
  const double oneMinAlpha = 1.0 - alpha;
  const double s = sol[i];
  double so;
  if (copyOld) { so = s; solOld[i] = s; } else { so = solOld[i]; }
  sol[i] = oneMinAlpha * s + alpha * so - betaDt * res[i];
}

// Low-storage RK stage: dU = a dU - dt R; U += b dU (a == 0 starts a new step).
__global__ void LsrkStageKernel(double *sol, double *du, const double *res, const double *d_dt,
                                double ca, double cb, size_t n, const CaseView cv, int elemSize) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = StageCase(cv, i, elemSize);
  if (c < 0) return;
  const double dt = d_dt[c];
  const double d = (ca == 0.0) ? -dt * res[i] : ca * du[i] - dt * res[i];
  du[i] = d;
  sol[i] = sol[i] + cb * d;
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
// Dynamic shared-memory limit of one residual-kernel variant, set once (outside
// any stream capture: ConfigureResidual runs before the first captured step).
template <int K, int M, typename T, bool OPEN>
static cudaError_t ConfigureKMT() {
  using P = Plan<K, M, T, OPEN>;
  static bool configured = false;
  if (configured || P::BIG) return cudaSuccess;
  cudaError_t err = cudaFuncSetAttribute(ResidualKernel<K, M, P::NT, T, OPEN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)P::BYTES);
  if (err == cudaSuccess) configured = true;
  return err;
}

template <int K, int M, typename T>
static cudaError_t ConfigureFluxKMT() {
  using P = FluxPlan<K, M, T>;
  static bool configured = false;
  if (configured || P::BIG) return cudaSuccess;
  cudaError_t err = cudaFuncSetAttribute(FaceFluxKernel<K, M, P::NT, T, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)P::BYTES);
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(FaceFluxKernel<K, M, P::NT, T, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::BYTES);
  if (err == cudaSuccess) configured = true;
  return err;
}

template <int K, int M>
static cudaError_t ConfigureBoundaryKM() {
  using SM = BoundaryTraceSmem<K, M>;
  constexpr int NT = M * M > 64 ? 128 : 64;
  if (!SM::DYN) return cudaSuccess;
  return cudaFuncSetAttribute(BoundaryTraceKernel<K, M, NT>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double) * SM::N));
}

template <int K, int M>
static cudaError_t ConfigureKM() {
  cudaError_t e = ConfigureBoundaryKM<K, M>();
  if (e == cudaSuccess) e = ConfigureFluxKMT<K, M, double>();
  if (e == cudaSuccess) e = ConfigureFluxKMT<K, M, float>();
  if (e == cudaSuccess) e = ConfigureKMT<K, M, double, false>();
  if (e == cudaSuccess) e = ConfigureKMT<K, M, float, false>();
  if (e == cudaSuccess) e = ConfigureKMT<K, M, double, true>();
  if (e == cudaSuccess) e = ConfigureKMT<K, M, float, true>();
  return e;
}

// One residual: the face fluxes, then the fused volume / distribution / mass-solve kernel.
template <int K, int M, typename T, bool OPEN>
static cudaError_t LaunchResidualKMT(const ResidualArgs &a, cudaStream_t st) {
  using P = Plan<K, M, T, OPEN>;
  using PF = FluxPlan<K, M, T>;
  cudaError_t err = ConfigureKMT<K, M, T, OPEN>();
  if (err == cudaSuccess) err = ConfigureFluxKMT<K, M, T>();
  if (err != cudaSuccess) return err;
  const int nFace = a.n_face_elem > 0 ? a.n_face_elem : a.n_elem;
  if ((P::BIG || PF::BIG) && (!a.scratch || a.scratch_ctas < 1)) return cudaErrorInvalidValue;
  const unsigned gridF = PF::BIG ? (nFace < a.scratch_ctas ? nFace : a.scratch_ctas) : nFace;
  const size_t smemF = PF::BIG ? 0 : PF::BYTES;
  if (a.sgs)
    FaceFluxKernel<K, M, PF::NT, T, true><<<gridF, PF::NT, smemF, st>>>(a);
  else
    FaceFluxKernel<K, M, PF::NT, T, false><<<gridF, PF::NT, smemF, st>>>(a);
  if constexpr (P::BIG)
    ResidualKernel<K, M, P::NT, T, OPEN>
        <<<a.n_elem < a.scratch_ctas ? a.n_elem : a.scratch_ctas, P::NT, 0, st>>>(a);
  else
    ResidualKernel<K, M, P::NT, T, OPEN><<<a.n_elem, P::NT, P::BYTES, st>>>(a);
  return cudaGetLastError();
}

// FP64 form or the mixed form (FP32 compute, FP64 inputs and outputs), each
// with or without open boundaries and sponge layers.
template <int K, int M>
static cudaError_t LaunchResidualKM(const ResidualArgs &a, cudaStream_t st) {
  if (a.open)
    return a.mixed ? LaunchResidualKMT<K, M, float, true>(a, st)
                   : LaunchResidualKMT<K, M, double, true>(a, st);
  return a.mixed ? LaunchResidualKMT<K, M, float, false>(a, st)
                 : LaunchResidualKMT<K, M, double, false>(a, st);
}

// The two characteristic-boundary kernels (dg_boundary.cuh).
template <int K, int M>
static cudaError_t LaunchBoundaryKM(const BoundaryArgs &a, cudaStream_t st) {
  constexpr int NT = M * M > 64 ? 128 : 64;
  using SM = BoundaryTraceSmem<K, M>;
  BoundaryTraceKernel<K, M, NT><<<a.nB, NT, SM::DYN ? sizeof(double) * SM::N : 0, st>>>(a);
  BoundaryFluxKernel<K, M, NT><<<a.nB, NT, 0, st>>>(a);
  return cudaGetLastError();
}

template <int K, int M>
static cudaError_t LaunchTimeStepKM(const TimeStepArgs &a, cudaStream_t st) {
  if (a.sgs) {
    using SG = TimeStepSgsSmem<K>;
    if constexpr (SG::BIG) {
      if (!a.scratch || a.scratch_ctas < 1) return cudaErrorInvalidValue;
      TimeStepSgsKernel<K, M, 64>
          <<<a.n_elem < a.scratch_ctas ? a.n_elem : a.scratch_ctas, 64, 0, st>>>(a);
    } else {
      TimeStepSgsKernel<K, M, 64><<<a.n_elem, 64, SG::BYTES, st>>>(a);
    }
  } else {
    using SM = TimeStepSmem<K>;
    TimeStepKernel<K, M, 64><<<a.n_elem, 64, SM::DYN ? sizeof(double) * SM::N : 0, st>>>(a);
  }
  return cudaGetLastError();
}

// Dynamic shared memory of the time-step kernels (before any capture).
template <int K, int M>
static cudaError_t ConfigureTimeStepKM() {
  constexpr size_t sgsSmem = sizeof(double) * 32 * K * K * K;
  cudaError_t e = cudaSuccess;
  if constexpr (sgsSmem <= 227 * 1024)
    e = cudaFuncSetAttribute(TimeStepSgsKernel<K, M, 64>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sgsSmem);
  using SM = TimeStepSmem<K>;
  if (e == cudaSuccess && SM::DYN)
    e = cudaFuncSetAttribute(TimeStepKernel<K, M, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * SM::N));
  return e;
}

// Every supported (K, M) pair (the open-boundary kernels exist for all of them).
#define VCPG_PAIRS(X) \
  X(2, 2) X(2, 3) X(3, 4) X(4, 5) X(5, 7) X(6, 8) X(7, 9) X(8, 12) X(9, 13) X(10, 14)
#define VCPG_PAIRS_OPEN(X) VCPG_PAIRS(X)

bool Supported(int K, int M) {
#define VCPG_IS(K_, M_) if (K == K_ && M == M_) return true;
  VCPG_PAIRS(VCPG_IS)
#undef VCPG_IS
  return false;
}

bool SupportsOpenBoundaries(int K, int M) {
#define VCPG_IS(K_, M_) if (K == K_ && M == M_) return true;
  VCPG_PAIRS_OPEN(VCPG_IS)
#undef VCPG_IS
  return false;
}

int SlotOf(int K, int M) {
#define VCPG_SLOT_OF(K_, M_) if (K == K_ && M == M_) return Slot<K_, M_>::value;
  VCPG_PAIRS(VCPG_SLOT_OF)
#undef VCPG_SLOT_OF
  return -1;
}

size_t ResidualSmemBytes(int K, int M) {
#define VCPG_SMEM(K_, M_) if (K == K_ && M == M_) return Plan<K_, M_>::BIG ? 0 : Plan<K_, M_>::BYTES;
  VCPG_PAIRS(VCPG_SMEM)
#undef VCPG_SMEM
  return 0;
}

template <int K, int M> static size_t ScratchBytesKM(int ctas) {
  size_t b = 0;
  auto take = [&b, ctas](bool big, size_t per) { if (big && per * ctas > b) b = per * ctas; };
  take(Plan<K, M, double, false>::BIG, sizeof(double) * Plan<K, M, double, false>::SCRATCH);
  take(Plan<K, M, double, true>::BIG, sizeof(double) * Plan<K, M, double, true>::SCRATCH);
  take(Plan<K, M, float, false>::BIG, sizeof(float) * Plan<K, M, float, false>::SCRATCH);
  take(Plan<K, M, float, true>::BIG, sizeof(float) * Plan<K, M, float, true>::SCRATCH);
  take(FluxPlan<K, M, double>::BIG, sizeof(double) * FluxPlan<K, M, double>::SCRATCH);
  take(FluxPlan<K, M, float>::BIG, sizeof(float) * FluxPlan<K, M, float>::SCRATCH);
  take(TimeStepSgsSmem<K>::BIG, TimeStepSgsSmem<K>::BYTES);
  return b;
}

size_t ResidualScratchBytes(int K, int M, int ctas) {
#define VCPG_SCRATCH(K_, M_) if (K == K_ && M == M_) return ScratchBytesKM<K_, M_>(ctas);
  VCPG_PAIRS(VCPG_SCRATCH)
#undef VCPG_SCRATCH
  return 0;
}

size_t FaceFluxBytesPerElement(int K, int M) {
  (void)K;
  return sizeof(double) * 3 * 20 * (size_t)M * M;
}

cudaError_t LaunchResidual(int K, int M, const ResidualArgs &a, cudaStream_t st) {
  if (a.n_elem <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) if (K == K_ && M == M_) return LaunchResidualKM<K_, M_>(a, st);
  VCPG_PAIRS(VCPG_LAUNCH)
#undef VCPG_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t ConfigureTimeStep(int K, int M) {
#define VCPG_CONF(K_, M_) if (K == K_ && M == M_) return ConfigureTimeStepKM<K_, M_>();
  VCPG_PAIRS(VCPG_CONF)
#undef VCPG_CONF
  return cudaErrorInvalidValue;
}

cudaError_t ConfigureResidual(int K, int M) {
#define VCPG_CONF(K_, M_) if (K == K_ && M == M_) return ConfigureKM<K_, M_>();
  VCPG_PAIRS(VCPG_CONF)
#undef VCPG_CONF
  return cudaErrorInvalidValue;
}

cudaError_t LaunchBoundary(int K, int M, const BoundaryArgs &a, cudaStream_t st) {
  if (a.nB <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) if (K == K_ && M == M_) return LaunchBoundaryKM<K_, M_>(a, st);
  VCPG_PAIRS_OPEN(VCPG_LAUNCH)
#undef VCPG_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t LaunchTimeStep(int K, int M, const TimeStepArgs &a, cudaStream_t st) {
  if (a.n_elem <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) if (K == K_ && M == M_) return LaunchTimeStepKM<K_, M_>(a, st);
  VCPG_PAIRS(VCPG_LAUNCH)
#undef VCPG_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t LaunchFinalizeDt(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                             double *hist, int hist_cap, int *counter, cudaStream_t st) {
  FinalizeDtKernel<<<1, 1, 0, st>>>(dt_bits, fixed_dt, d_dt, hist, hist_cap, counter);
  return cudaGetLastError();
}

cudaError_t LaunchEnsembleFinalize(int n_cases, int *state, const int *target, int *done,
                                   unsigned long long *dt_bits, double *dt, double *sim_time,
                                   cudaStream_t st) {
  if (n_cases <= 0) return cudaSuccess;
  EnsembleFinalizeKernel<<<(n_cases + 127) / 128, 128, 0, st>>>(n_cases, state, target, done,
                                                                dt_bits, dt, sim_time);
  return cudaGetLastError();
}

cudaError_t LaunchSspStage(double *sol, double *solOld, const double *res, const double *d_dt,
                           double alpha, double beta, int copyOld, size_t n, cudaStream_t st,
                           const CaseView &cv, int elemSize) {
  const int nt = 256;
  SspStageKernel<<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(sol, solOld, res, d_dt, alpha,
                                                               beta, copyOld, n, cv, elemSize);
  return cudaGetLastError();
}

cudaError_t LaunchLsrkStage(double *sol, double *du, const double *res, const double *d_dt,
                            double ca, double cb, size_t n, cudaStream_t st, const CaseView &cv,
                            int elemSize) {
  const int nt = 256;
  LsrkStageKernel<<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(sol, du, res, d_dt, ca, cb, n,
                                                                cv, elemSize);
  return cudaGetLastError();
}

cudaError_t UploadOperatorTable(const vcpg_operators *ops, int K, int M) {
  return UploadOperators(K, M, ops->leg_int, ops->dleg_int, ops->leg_face, ops->dleg_face,
                         ops->w_int, ops->leg_dofs, ops->dleg_dofs);
}

}  // namespace vcpg
