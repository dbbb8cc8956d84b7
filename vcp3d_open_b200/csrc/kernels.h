// Host-visible launchers of the device kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

#include "../../include/vcp3d_b200.h"
#include "dg_tensor.cuh"

namespace vcpg {

struct ResidualArgs;
struct TimeStepArgs;
struct BoundaryArgs;
struct CaseView;

// Every supported (K, M) pair: the reference's tensor-product dispatch
// (src/TensorProductVolumeResidualK2.cpp ... K10.cpp).
#define VCPG_PAIRS(X) \
  X(2, 2) X(2, 3) X(3, 4) X(4, 5) X(5, 7) X(6, 8) X(7, 9) X(8, 12) X(9, 13) X(10, 14)

// Per-pair entry points, defined by the pair's own object (kernels_pair.cu).
#define VCPG_PAIR_FN(name, K_, M_) Pair##name##_##K_##_##M_
#define VCPG_PAIR_DECLARE(K_, M_)                                                           \
  cudaError_t VCPG_PAIR_FN(LaunchResidual, K_, M_)(const ResidualArgs &a, cudaStream_t st,  \
                                                    int phase);                               \
  cudaError_t VCPG_PAIR_FN(LaunchBoundary, K_, M_)(const BoundaryArgs &a, cudaStream_t st,  \
                                                    int phase);                               \
  cudaError_t VCPG_PAIR_FN(LaunchTimeStep, K_, M_)(const TimeStepArgs &a, cudaStream_t st); \
  cudaError_t VCPG_PAIR_FN(ConfigureResidual, K_, M_)();                                    \
  cudaError_t VCPG_PAIR_FN(ConfigureTimeStep, K_, M_)();                                    \
  cudaError_t VCPG_PAIR_FN(Upload, K_, M_)(const vcpg_operators *ops);
VCPG_PAIRS(VCPG_PAIR_DECLARE)
#undef VCPG_PAIR_DECLARE

bool Supported(int K, int M);
// Whether a step applies the Runge-Kutta stage updates inside the residual
// kernel (its inputs prefetched into free shared memory) for this variant;
// otherwise the separate stage kernels apply them.
bool FusedStageUpdate(int K, int M, bool mixed, bool open);
int SlotOf(int K, int M);
size_t ResidualSmemBytes(int K, int M);
// Device bytes per element of the face-flux buffer (ResidualArgs::face_flux).
size_t FaceFluxBytesPerElement(int K, int M);
// The open-boundary kernels exist for this pair (degrees up to 6).
bool SupportsOpenBoundaries(int K, int M);
// Global scratch of the residual kernels for degrees whose element arrays exceed
// one CTA's shared memory (ResidualArgs::scratch), for a grid of `ctas` CTAs; 0
// when every variant of the pair runs in shared memory.
size_t ResidualScratchBytes(int K, int M, int ctas);
// Uploads the 1-D operators of a (K, M) pair (FP64 and FP32 copies) to the
// constant memory of this library's residual, boundary and time-step kernels.
cudaError_t UploadOperatorTable(const vcpg_operators *ops, int K, int M);
// Per-case step bookkeeping of a bucket holding several cases (csrc/ensemble.cu).
cudaError_t LaunchEnsembleFinalize(int n_cases, int *state, const int *target, int *done,
                                   unsigned long long *dt_bits, double *dt, double *sim_time,
                                   cudaStream_t st);

// One residual = FaceFluxKernel + ResidualKernel (2 launches). phase 1 launches
// only FaceFluxKernel, phase 2 only ResidualKernel (per-kernel timing).
cudaError_t LaunchResidual(int K, int M, const ResidualArgs &a, cudaStream_t st, int phase = 0);
// Sets the shared-memory limits of all residual-kernel variants of a (K, M) pair;
// call before capturing launches into a CUDA graph.
cudaError_t ConfigureResidual(int K, int M);
// Dynamic shared memory of the time-step kernels (with an SGS model, or degree >= 7).
cudaError_t ConfigureTimeStep(int K, int M);
// Boundary traces + Mach weights, then the boundary states and fluxes (2 launches).
// phase 1: the trace kernel only (traces and Mach weights).
cudaError_t LaunchBoundary(int K, int M, const BoundaryArgs &a, cudaStream_t st, int phase = 0);
cudaError_t LaunchTimeStep(int K, int M, const TimeStepArgs &a, cudaStream_t st);
cudaError_t LaunchFinalizeDt(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                             double *hist, int hist_cap, int *counter, cudaStream_t st);
// The start of a single-case step: the reduced (or fixed) time step recorded,
// the reduction re-armed, and the first stage's update (kind: enum RkKind,
// coefficients (a, b) or (alpha, beta)); reg is du or solOld.
cudaError_t LaunchStartStep(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                            double *hist, int hist_cap, int *counter, unsigned int *ticket,
                            double *sol, double *reg, const double *res, int kind, double ca,
                            double cb, size_t n, cudaStream_t st);
// out[i][:] = sol[idx[i]][:] for i < count, per doubles per element (the
// indices are checked on the host when the list is set).
cudaError_t LaunchGatherStates(const double *sol, const int *idx, int count, int per, double *out,
                               cudaStream_t st);
// Stage updates; d_dt holds one time step per case (one entry for a single case).
cudaError_t LaunchSspStage(double *sol, double *solOld, const double *res, const double *d_dt,
                           double alpha, double beta, int copyOld, size_t n, cudaStream_t st,
                           const CaseView &cv, int elemSize);
cudaError_t LaunchLsrkStage(double *sol, double *du, const double *res, const double *d_dt,
                            double ca, double cb, size_t n, cudaStream_t st, const CaseView &cv,
                            int elemSize);

}  // namespace vcpg
