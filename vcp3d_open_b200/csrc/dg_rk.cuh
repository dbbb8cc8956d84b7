// Runge-Kutta stage updates of one state entry, shared by the stand-alone stage
// kernels (kernels.cu) and the residual kernel's epilogue (dg_residual.cuh), so
// that the fused and the separate updates round identically (explicit fused
// multiply-adds, nothing left to the compiler's contraction choices).
//
// SSP-RK3 (SolverClass::ExecuteTimeSynchronizationStep, src/SolverClass.cpp:2368-2396):
//   sol = (1 - alpha) sol + alpha solOld - beta dt res
// Low-storage RK4 (Carpenter-Kennedy 5-stage 2N, an added scheme):
//   du = a du - dt res   (a = 0 starts a new step);   sol += b du
#pragma once

#include <cuda_runtime.h>

namespace vcpg {

// Fused-update kinds of ResidualArgs::rk_kind.
enum RkKind { kRkNone = 0, kRkLowStorage = 1, kRkSsp = 2 };

__device__ __forceinline__ void LsrkUpdate(double &sol, double &du, const double res,
                                           const double dt, const double a, const double b) {
  const double mdr = -dt * res;
  const double d = (a == 0.0) ? mdr : __fma_rn(a, du, mdr);
  du = d;
  sol = __fma_rn(b, d, sol);
}

__device__ __forceinline__ void SspUpdate(double &sol, const double solOld, const double res,
                                          const double dt, const double alpha,
                                          const double beta) {
  const double betaDt = beta * dt;
  const double t = __fma_rn(alpha, solOld, (1.0 - alpha) * sol);
  sol = __fma_rn(-betaDt, res, t);
}

}  // namespace vcpg
