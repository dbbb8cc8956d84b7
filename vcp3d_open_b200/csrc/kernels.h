// Host-visible launchers of the device kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

#include "dg_tensor.cuh"

namespace vcpg {

struct ResidualArgs;
struct TimeStepArgs;
struct BoundaryArgs;

bool Supported(int K, int M);
int SlotOf(int K, int M);
size_t ResidualSmemBytes(int K, int M);
cudaError_t UploadOpTable(int slot, const OpTable &t);

cudaError_t LaunchResidual(int K, int M, const ResidualArgs &a, cudaStream_t st);
// Boundary traces + Mach weights, then the boundary states and fluxes (2 launches).
cudaError_t LaunchBoundary(int K, int M, const BoundaryArgs &a, cudaStream_t st);
cudaError_t LaunchTimeStep(int K, int M, const TimeStepArgs &a, cudaStream_t st);
cudaError_t LaunchFinalizeDt(unsigned long long *dt_bits, const double *fixed_dt, double *d_dt,
                             double *hist, int hist_cap, int *counter, cudaStream_t st);
cudaError_t LaunchSspStage(double *sol, double *solOld, const double *res, const double *d_dt,
                           double alpha, double beta, int copyOld, size_t n, cudaStream_t st);
cudaError_t LaunchLsrkStage(double *sol, double *du, const double *res, const double *d_dt,
                            double ca, double cb, size_t n, cudaStream_t st);

}  // namespace vcpg
