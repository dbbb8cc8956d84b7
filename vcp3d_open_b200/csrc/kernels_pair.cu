// Kernels of one (K, M) pair: the residual kernels (face fluxes and the fused
// volume / distribution / mass-solve kernel, FP64 and mixed, with and without
// open boundaries), the characteristic-boundary kernels and the CFL time-step
// kernels. build.py compiles this file once per supported pair, with
// -DVCPG_PAIR_K=K -DVCPG_PAIR_M=M, so the pairs compile in parallel; each
// object holds its own constant-memory operator table (PairUpload).
#include <cstring>

#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "dg_timestep.cuh"
#include "kernels.h"

#if !defined(VCPG_PAIR_K) || !defined(VCPG_PAIR_M)
#error "compile with -DVCPG_PAIR_K=<K> -DVCPG_PAIR_M=<M>"
#endif

namespace vcpg {

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
// phase 0 launches both, 1 only FaceFluxKernel, 2 only ResidualKernel (timing).
template <int K, int M, typename T, bool OPEN>
static cudaError_t LaunchResidualKMT(const ResidualArgs &a, cudaStream_t st, int phase) {
  using P = Plan<K, M, T, OPEN>;
  using PF = FluxPlan<K, M, T>;
  cudaError_t err = ConfigureKMT<K, M, T, OPEN>();
  if (err == cudaSuccess) err = ConfigureFluxKMT<K, M, T>();
  if (err != cudaSuccess) return err;
  const int nFace = a.n_face_elem > 0 ? a.n_face_elem : a.n_elem;
  if ((P::BIG || PF::BIG) && (!a.scratch || a.scratch_ctas < 1)) return cudaErrorInvalidValue;
  const unsigned gridF = PF::BIG ? (nFace < a.scratch_ctas ? nFace : a.scratch_ctas) : nFace;
  const size_t smemF = PF::BIG ? 0 : PF::BYTES;
  if (phase != 2) {
    if (a.sgs)
      FaceFluxKernel<K, M, PF::NT, T, true><<<gridF, PF::NT, smemF, st>>>(a);
    else
      FaceFluxKernel<K, M, PF::NT, T, false><<<gridF, PF::NT, smemF, st>>>(a);
  }
  if (phase == 1) return cudaGetLastError();
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
static cudaError_t LaunchResidualKM(const ResidualArgs &a, cudaStream_t st, int phase) {
  if (a.open)
    return a.mixed ? LaunchResidualKMT<K, M, float, true>(a, st, phase)
                   : LaunchResidualKMT<K, M, double, true>(a, st, phase);
  return a.mixed ? LaunchResidualKMT<K, M, float, false>(a, st, phase)
                 : LaunchResidualKMT<K, M, double, false>(a, st, phase);
}

// The two characteristic-boundary kernels (dg_boundary.cuh).
template <int K, int M>
static cudaError_t LaunchBoundaryKM(const BoundaryArgs &a, cudaStream_t st, int phase) {
  constexpr int NT = M * M > 64 ? 128 : 64;
  using SM = BoundaryTraceSmem<K, M>;
  BoundaryTraceKernel<K, M, NT><<<a.nB, NT, SM::DYN ? sizeof(double) * SM::N : 0, st>>>(a);
  if (phase != 1) BoundaryFluxKernel<K, M, NT><<<a.nB, NT, 0, st>>>(a);
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

template <int K, int M>
static cudaError_t PairUploadKM(const vcpg_operators *ops) {
  return UploadOperators(K, M, ops->leg_int, ops->dleg_int, ops->leg_face, ops->dleg_face,
                         ops->w_int, ops->leg_dofs, ops->dleg_dofs);
}

#define VCPG_PAIR_DEFINE(K_, M_)                                                              \
  cudaError_t VCPG_PAIR_FN(LaunchResidual, K_, M_)(const ResidualArgs &a, cudaStream_t st,  \
                                                    int phase) {                              \
    return LaunchResidualKM<K_, M_>(a, st, phase);                                            \
  }                                                                                           \
  cudaError_t VCPG_PAIR_FN(LaunchBoundary, K_, M_)(const BoundaryArgs &a, cudaStream_t st,  \
                                                    int phase) {                              \
    return LaunchBoundaryKM<K_, M_>(a, st, phase);                                            \
  }                                                                                           \
  cudaError_t VCPG_PAIR_FN(LaunchTimeStep, K_, M_)(const TimeStepArgs &a, cudaStream_t st) {  \
    return LaunchTimeStepKM<K_, M_>(a, st);                                                   \
  }                                                                                           \
  cudaError_t VCPG_PAIR_FN(ConfigureResidual, K_, M_)() { return ConfigureKM<K_, M_>(); }     \
  cudaError_t VCPG_PAIR_FN(ConfigureTimeStep, K_, M_)() { return ConfigureTimeStepKM<K_, M_>(); } \
  cudaError_t VCPG_PAIR_FN(Upload, K_, M_)(const vcpg_operators *ops) {                       \
    return PairUploadKM<K_, M_>(ops);                                                         \
  }
VCPG_PAIR_DEFINE(VCPG_PAIR_K, VCPG_PAIR_M)
#undef VCPG_PAIR_DEFINE

}  // namespace vcpg
