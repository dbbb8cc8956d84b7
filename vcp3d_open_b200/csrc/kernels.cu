// Dispatch over the supported (K, M) pairs (each pair's kernels are compiled
// from kernels_pair.cu into an object of their own), the launch geometry
// queries, and the kernels that do not depend on the pair: the time step's
// finalisation and the Runge-Kutta stage updates.
#include <cstring>

#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "dg_rk.cuh"
#include "dg_timestep.cuh"
#include "kernels.h"

namespace vcpg {

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
  double s = sol[i], so;
  if (copyOld) { so = s; solOld[i] = s; } else { so = solOld[i]; }
  SspUpdate(s, so, res[i], d_dt[c], alpha, beta);
  sol[i] = s;
}

// Low-storage RK stage: dU = a dU - dt R; U += b dU (a == 0 starts a new step).
__global__ void LsrkStageKernel(double *sol, double *du, const double *res, const double *d_dt,
                                double ca, double cb, size_t n, const CaseView cv, int elemSize) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = StageCase(cv, i, elemSize);
  if (c < 0) return;
  double s = sol[i], d = ca == 0.0 ? 0.0 : du[i];
  LsrkUpdate(s, d, res[i], d_dt[c], ca, cb);
  du[i] = d;
  sol[i] = s;
}

// The start of a single-case step: the time step (the reduced CFL step, or the
// fixed one) and the first stage's update with it, in one grid. Every block
// reads the reduced step first; the block that finishes last records it
// (d_dt for the stages fused into the residual kernels, the history) and
// re-arms the reduction. ticket: a zero-initialised counter, reset here.
__global__ void StartStepKernel(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                                double *hist, int hist_cap, int *counter, unsigned int *ticket,
                                double *sol, double *reg, const double *res, int kind,
                                double ca, double cb, size_t n) {
  const double fx = *fixed_dt;
  const double dt = fx > 0.0 ? fx : __longlong_as_double((long long)*dt_bits);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double s = sol[i];
    if (kind == kRkLowStorage) {
      double d = ca == 0.0 ? 0.0 : reg[i];
      LsrkUpdate(s, d, res[i], dt, ca, cb);
      reg[i] = d;
    } else {
      reg[i] = s;                     // solOld = sol
      SspUpdate(s, s, res[i], dt, ca, cb);
    }
    sol[i] = s;
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    *d_dt = dt;
    const int c = *counter;
    if (c < hist_cap) hist[c] = dt;
    *counter = c + 1;
    *dt_bits = (unsigned long long)__double_as_longlong(1.e+10);
    *ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
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

// Stage updates fused into the residual kernel where it prefetches their inputs
// (0: always the separate stage kernels).
#ifndef VCPG_FUSED_STAGES
#define VCPG_FUSED_STAGES 1
#endif

bool FusedStageUpdate(int K, int M, bool mixed, bool open) {
  if (!VCPG_FUSED_STAGES) return false;
#define VCPG_FUSED(K_, M_)                                                                   \
  if (K == K_ && M == M_)                                                                    \
    return mixed ? (open ? FusedUpdatePrefetch<K_, M_, float, true>::value                   \
                         : FusedUpdatePrefetch<K_, M_, float, false>::value)                 \
                 : (open ? FusedUpdatePrefetch<K_, M_, double, true>::value                  \
                         : FusedUpdatePrefetch<K_, M_, double, false>::value);
  VCPG_PAIRS(VCPG_FUSED)
#undef VCPG_FUSED
  return false;
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

cudaError_t LaunchResidual(int K, int M, const ResidualArgs &a, cudaStream_t st, int phase) {
  if (a.n_elem <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) \
  if (K == K_ && M == M_) return VCPG_PAIR_FN(LaunchResidual, K_, M_)(a, st, phase);
  VCPG_PAIRS(VCPG_LAUNCH)
#undef VCPG_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t ConfigureTimeStep(int K, int M) {
#define VCPG_CONF(K_, M_) if (K == K_ && M == M_) return VCPG_PAIR_FN(ConfigureTimeStep, K_, M_)();
  VCPG_PAIRS(VCPG_CONF)
#undef VCPG_CONF
  return cudaErrorInvalidValue;
}

cudaError_t ConfigureResidual(int K, int M) {
#define VCPG_CONF(K_, M_) if (K == K_ && M == M_) return VCPG_PAIR_FN(ConfigureResidual, K_, M_)();
  VCPG_PAIRS(VCPG_CONF)
#undef VCPG_CONF
  return cudaErrorInvalidValue;
}

cudaError_t LaunchBoundary(int K, int M, const BoundaryArgs &a, cudaStream_t st, int phase) {
  if (a.nB <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) \
  if (K == K_ && M == M_) return VCPG_PAIR_FN(LaunchBoundary, K_, M_)(a, st, phase);
  VCPG_PAIRS_OPEN(VCPG_LAUNCH)
#undef VCPG_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t LaunchTimeStep(int K, int M, const TimeStepArgs &a, cudaStream_t st) {
  if (a.n_elem <= 0) return cudaSuccess;
#define VCPG_LAUNCH(K_, M_) if (K == K_ && M == M_) return VCPG_PAIR_FN(LaunchTimeStep, K_, M_)(a, st);
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

// The states of listed elements, packed element after element for a neighbouring
// rank (vcpg_pack_send_list).
__global__ void GatherStatesKernel(const double *__restrict__ sol, const int *__restrict__ idx,
                                   const int count, const int per, double *__restrict__ out) {
  const size_t n = (size_t)count * per;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t e = t / per;
    out[t] = sol[(size_t)idx[e] * per + (t - e * per)];
  }
}

cudaError_t LaunchGatherStates(const double *sol, const int *idx, int count, int per, double *out,
                               cudaStream_t st) {
  const int nt = 256;
  const size_t n = (size_t)count * per;
  const size_t blocks = (n + nt - 1) / nt;
  GatherStatesKernel<<<(unsigned)(blocks < 148 * 8 ? blocks : 148 * 8), nt, 0, st>>>(
      sol, idx, count, per, out);
  return cudaGetLastError();
}

cudaError_t LaunchStartStep(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                            double *hist, int hist_cap, int *counter, unsigned int *ticket,
                            double *sol, double *reg, const double *res, int kind, double ca,
                            double cb, size_t n, cudaStream_t st) {
  // A grid of at most 8 resident blocks of 256 threads per SM (148 SMs).
  const int nt = 256;
  const size_t want = (n + nt - 1) / nt;
  const unsigned grid = (unsigned)(want < 148 * 8 ? (want > 0 ? want : 1) : 148 * 8);
  StartStepKernel<<<grid, nt, 0, st>>>(dt_bits, fixed_dt, d_dt, hist, hist_cap, counter, ticket,
                                       sol, reg, res, kind, ca, cb, n);
  return cudaGetLastError();
}

cudaError_t UploadOperatorTable(const vcpg_operators *ops, int K, int M) {
#define VCPG_UP(K_, M_) if (K == K_ && M == M_) return VCPG_PAIR_FN(Upload, K_, M_)(ops);
  VCPG_PAIRS(VCPG_UP)
#undef VCPG_UP
  return cudaErrorInvalidValue;
}

}  // namespace vcpg
