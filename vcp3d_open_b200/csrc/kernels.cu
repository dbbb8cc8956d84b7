// Kernel instantiations and launchers for every supported (K, M) pair:
// the fused residual kernel, the CFL time-step kernel and the Runge-Kutta
// stage updates.
#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "kernels.h"

namespace vcpg {

// ---------------------------------------------------------------------------
// Time step per element, ElementClass::ComputeTimeStep (src/ElementClass.cpp:1522-1644)
// with ComputePrimitiveVariablesNodalDOFs (:1500-1520); global minimum via an
// atomic min on the bit pattern of the (positive) double.
// ---------------------------------------------------------------------------


template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) TimeStepKernel(const TimeStepArgs a) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K;
  __shared__ double s_sol[5 * KD], s_t1[5 * KD], s_t2[5 * KD], s_red[64];
  const int e = blockIdx.x;
  if (e >= a.n_elem) return;
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
  const double muDim = a.mu * a.p_ref / a.u_ref;
  const double dliInv = 1.0 / sc[0], dljInv = 1.0 / sc[1], dlkInv = 1.0 / sc[2];
  const double dli2Inv = dliInv * dliInv, dlj2Inv = dljInv * dljInv, dlk2Inv = dlkInv * dlkInv;
  const double dLen2Inv = dli2Inv + dlj2Inv + dlk2Inv;
  const double radVisOverNuLam = fmax(fmax(1.0, 2.0 + kLamOverMu), kFactHFLam) * dLen2Inv;
  double radInvMax = 0.0, radVisMax = 0.0, a2Min = 1.e+10;
  for (int l = threadIdx.x; l < KD; l += NT) {
    double rho, u, v, w, p, eKin;
    EntropyToPrim(s_t1[l], s_t1[KD + l], s_t1[2 * KD + l], s_t1[3 * KD + l], s_t1[4 * KD + l],
                  rho, u, v, w, p, eKin);
    rho *= a.rho_ref; u *= a.u_ref; v *= a.u_ref; w *= a.u_ref; p *= a.p_ref;
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
    const double dtElem = a.cfl * a.u_ref / dtInv;
    atomicMin(a.dt_bits, (unsigned long long)__double_as_longlong(dtElem));
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

// SSP-RK3 stage (src/SolverClass.cpp:2368-2396); stage 0 also stores solOld.
__global__ void SspStageKernel(double *sol, double *solOld, const double *res, const double *d_dt,
                               double alpha, double beta, int copyOld, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double betaDt = beta * (*d_dt);
  const double oneMinAlpha = 1.0 - alpha;
  const double s = sol[i];
  double so;
  if (copyOld) { so = s; solOld[i] = s; } else { so = solOld[i]; }
  sol[i] = oneMinAlpha * s + alpha * so - betaDt * res[i];
}

// Low-storage RK stage: dU = a dU - dt R; U += b dU (a == 0 starts a new step).
__global__ void LsrkStageKernel(double *sol, double *du, const double *res, const double *d_dt,
                                double ca, double cb, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dt = *d_dt;
  const double d = (ca == 0.0) ? -dt * res[i] : ca * du[i] - dt * res[i];
  du[i] = d;
  sol[i] = sol[i] + cb * d;
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
template <int K, int M, typename T, bool OPEN>
static cudaError_t LaunchResidualKMT(const ResidualArgs &a, cudaStream_t st) {
  using P = Plan<K, M, T, OPEN>;
  constexpr int NT = P::NT;
  const size_t bytes = P::BYTES;
  static bool configured = false;
  if (!configured) {
    cudaError_t err = cudaFuncSetAttribute(ResidualKernel<K, M, NT, T, OPEN>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err != cudaSuccess) return err;
    configured = true;
  }
  ResidualKernel<K, M, NT, T, OPEN><<<a.n_elem, NT, bytes, st>>>(a);
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
  BoundaryTraceKernel<K, M, NT><<<a.nB, NT, 0, st>>>(a);
  BoundaryFluxKernel<K, M, NT><<<a.nB, NT, 0, st>>>(a);
  return cudaGetLastError();
}

template <int K, int M>
static cudaError_t LaunchTimeStepKM(const TimeStepArgs &a, cudaStream_t st) {
  TimeStepKernel<K, M, 64><<<a.n_elem, 64, 0, st>>>(a);
  return cudaGetLastError();
}

#define VCPG_DISPATCH(K_, M_, CALL) \
  if (K == K_ && M == M_) return CALL<K_, M_>

bool Supported(int K, int M) {
  return (K == 2 && M == 3) || (K == 3 && M == 4) || (K == 4 && M == 5) || (K == 5 && M == 7) ||
         (K == 6 && M == 8) || (K == 7 && M == 10);
}

int SlotOf(int K, int M) {
  if (K == 2 && M == 3) return Slot<2, 3>::value;
  if (K == 3 && M == 4) return Slot<3, 4>::value;
  if (K == 4 && M == 5) return Slot<4, 5>::value;
  if (K == 5 && M == 7) return Slot<5, 7>::value;
  if (K == 6 && M == 8) return Slot<6, 8>::value;
  if (K == 7 && M == 10) return Slot<7, 10>::value;
  return -1;
}

size_t ResidualSmemBytes(int K, int M) {
  if (K == 2 && M == 3) return Plan<2, 3>::BYTES;
  if (K == 3 && M == 4) return Plan<3, 4>::BYTES;
  if (K == 4 && M == 5) return Plan<4, 5>::BYTES;
  if (K == 5 && M == 7) return Plan<5, 7>::BYTES;
  if (K == 6 && M == 8) return Plan<6, 8>::BYTES;
  if (K == 7 && M == 10) return Plan<7, 10>::BYTES;
  return 0;
}

cudaError_t LaunchResidual(int K, int M, const ResidualArgs &a, cudaStream_t st) {
  if (a.n_elem <= 0) return cudaSuccess;
  if (K == 2 && M == 3) return LaunchResidualKM<2, 3>(a, st);
  if (K == 3 && M == 4) return LaunchResidualKM<3, 4>(a, st);
  if (K == 4 && M == 5) return LaunchResidualKM<4, 5>(a, st);
  if (K == 5 && M == 7) return LaunchResidualKM<5, 7>(a, st);
  if (K == 6 && M == 8) return LaunchResidualKM<6, 8>(a, st);
  return cudaErrorInvalidValue;
}

cudaError_t LaunchBoundary(int K, int M, const BoundaryArgs &a, cudaStream_t st) {
  if (a.nB <= 0) return cudaSuccess;
  if (K == 2 && M == 3) return LaunchBoundaryKM<2, 3>(a, st);
  if (K == 3 && M == 4) return LaunchBoundaryKM<3, 4>(a, st);
  if (K == 4 && M == 5) return LaunchBoundaryKM<4, 5>(a, st);
  if (K == 5 && M == 7) return LaunchBoundaryKM<5, 7>(a, st);
  if (K == 6 && M == 8) return LaunchBoundaryKM<6, 8>(a, st);
  return cudaErrorInvalidValue;
}

cudaError_t LaunchTimeStep(int K, int M, const TimeStepArgs &a, cudaStream_t st) {
  if (a.n_elem <= 0) return cudaSuccess;
  if (K == 2 && M == 3) return LaunchTimeStepKM<2, 3>(a, st);
  if (K == 3 && M == 4) return LaunchTimeStepKM<3, 4>(a, st);
  if (K == 4 && M == 5) return LaunchTimeStepKM<4, 5>(a, st);
  if (K == 5 && M == 7) return LaunchTimeStepKM<5, 7>(a, st);
  if (K == 6 && M == 8) return LaunchTimeStepKM<6, 8>(a, st);
  return cudaErrorInvalidValue;
}

cudaError_t LaunchFinalizeDt(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                             double *hist, int hist_cap, int *counter, cudaStream_t st) {
  FinalizeDtKernel<<<1, 1, 0, st>>>(dt_bits, fixed_dt, d_dt, hist, hist_cap, counter);
  return cudaGetLastError();
}

cudaError_t LaunchSspStage(double *sol, double *solOld, const double *res, const double *d_dt,
                           double alpha, double beta, int copyOld, size_t n, cudaStream_t st) {
  const int nt = 256;
  SspStageKernel<<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(sol, solOld, res, d_dt, alpha,
                                                               beta, copyOld, n);
  return cudaGetLastError();
}

cudaError_t LaunchLsrkStage(double *sol, double *du, const double *res, const double *d_dt,
                            double ca, double cb, size_t n, cudaStream_t st) {
  const int nt = 256;
  LsrkStageKernel<<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(sol, du, res, d_dt, ca, cb, n);
  return cudaGetLastError();
}

cudaError_t UploadOpTable(int slot, const OpTable &t) {
  return cudaMemcpyToSymbol(c_ops, &t, sizeof(OpTable), sizeof(OpTable) * (size_t)slot,
                            cudaMemcpyHostToDevice);
}

}  // namespace vcpg
