// Allocation-free CFL time step: vcpg_time_step_noalloc (include/vcp3d_b200.h).
//
// Who needs this: a host program that hands all of its device memory to its
// own pool allocator (a framework's caching allocator, or a driver that budgets
// the memory of many resident cases itself) must not call cudaMalloc/cudaFree
// behind the pool's back -- the memory would be invisible to the pool's
// accounting, and those calls can synchronise the device. Such a caller already
// owns the state and the geometry on the device; this entry point computes the
// global time step from them without allocating anything.
//
// Its only scratch -- one double per element for the per-element steps plus one
// status slot -- is the static device array below, 2 MiB for the stated limit of
// VCPG_NOALLOC_MAX_ELEMS elements. Every GPU that loads this library holds it
// until the process exits. All calls share it and each call overwrites it, so
// calls that overlap on the GPU (other streams, other host threads) race; the
// caller must order them. The status slot is cleared at the start of every call.
// Every call also reads the status back and synchronises the caller's stream,
// so a call cannot be captured into a CUDA graph.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/vcp3d_b200.h"
#include "dg_residual.cuh"
#include "dg_timestep.cuh"
#include "kernels.h"

namespace {

using namespace vcpg;

constexpr int64_t kMaxElems = VCPG_NOALLOC_MAX_ELEMS;
constexpr int64_t kStatusSlot = kMaxElems;  // 1.0 when a negative a^2 was seen

static __device__ __align__(256) double g_noalloc_scratch[kMaxElems + 32];

// Device address of g_noalloc_scratch per device; looked up once per device.
std::mutex g_setup_mutex;
double *g_scratch_ptr[256] = {};

int ScratchForCurrentDevice(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return VCPG_E_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p)
      return VCPG_E_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return VCPG_OK;
}

// Per-element step into scratch[e]: the arithmetic of the handle's time step
// (ElementTimeStep, dg_timestep.cuh).
template <int K, int M, int NT>
__global__ void __launch_bounds__(NT) NoAllocElementDtKernel(const double *sol,
                                                             const double *scalars, int n_elem,
                                                             int n_poly, double cfl, double mu,
                                                             double p_ref, double u_ref,
                                                             double rho_ref, double *scratch) {
  constexpr int KD = K * K * K;
  __shared__ double s_sol[5 * KD], s_t1[5 * KD], s_t2[5 * KD], s_red[64];
  const int e = blockIdx.x;
  if (e >= n_elem) return;
  bool bad = false;
  const double dt = ElementTimeStep<K, M, NT>(sol + (size_t)e * 5 * KD, scalars + (size_t)e * 15,
                                              n_poly, cfl, mu, p_ref, u_ref, rho_ref, s_sol, s_t1,
                                              s_t2, s_red, &bad);
  if (threadIdx.x == 0) {
    if (bad) scratch[kStatusSlot] = 1.0;
    scratch[e] = dt;
  }
}

// Minimum of scratch[0, n) into *out (one block).
__global__ void __launch_bounds__(1024) NoAllocMinKernel(const double *scratch, int n,
                                                         double *out) {
  __shared__ double s_red[64];
  double m = 1.e+10;
  for (int i = threadIdx.x; i < n; i += 1024) m = fmin(m, scratch[i]);
  m = -BlockMax<1024>(-m, s_red);
  if (threadIdx.x == 0) *out = m;
}

template <int K, int M>
cudaError_t LaunchKM(const vcpg_params *p, const double *sol, const double *sc, int n,
                     double *scratch, double *d_dt, cudaStream_t st) {
  NoAllocElementDtKernel<K, M, 64><<<n, 64, 0, st>>>(sol, sc, n, p->n_poly, p->cfl, p->mu,
                                                     p->p_ref, p->u_ref, p->rho_ref, scratch);
  NoAllocMinKernel<<<1, 1024, 0, st>>>(scratch, n, d_dt);
  return cudaGetLastError();
}

}  // namespace

extern "C" int vcpg_time_step_noalloc(const vcpg_params *params, const vcpg_operators *ops,
                                      const double *d_sol, const double *d_elem_scalars,
                                      double *d_dt, void *stream) {
  if (!params || !ops || !d_sol || !d_elem_scalars || !d_dt) return VCPG_E_INVALID;
  const int K = params->n_poly + 1, M = params->n_int_1d;
  const int64_t nE = (int64_t)params->n_elem[0] * params->n_elem[1] * params->n_elem[2];
  // The eddy viscosity of an SGS model needs the nodal-DOF metric of a handle.
  if (params->sgs_model != VCPG_SGS_NONE) return VCPG_E_INVALID;
  if (nE <= 0) return VCPG_E_INVALID;
  if (nE > kMaxElems) return VCPG_E_ADMISSION;  // beyond the static scratch array
  // This kernel keeps 15 K^3 doubles in static shared memory: up to degree 6.
  if (!Supported(K, M) || K > 7) return VCPG_E_UNSUPPORTED_KM;
  double *scratch = nullptr;
  int rc = ScratchForCurrentDevice(&scratch);
  if (rc != VCPG_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // Operators of this (K, M) pair into this file's constant memory, ordered on
  // the caller's stream before the kernels that read them.
  if (UploadOperators(K, M, ops->leg_int, ops->dleg_int, ops->leg_face, ops->dleg_face,
                      ops->w_int, ops->leg_dofs, nullptr, st, true) != cudaSuccess)
    return VCPG_E_CUDA;
  if (cudaMemsetAsync(scratch + kStatusSlot, 0, sizeof(double), st) != cudaSuccess)
    return VCPG_E_CUDA;
  cudaError_t e = cudaErrorInvalidValue;
  const int n = (int)nE;
  if (K == 2 && M == 3) e = LaunchKM<2, 3>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 3 && M == 4) e = LaunchKM<3, 4>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 4 && M == 5) e = LaunchKM<4, 5>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 5 && M == 7) e = LaunchKM<5, 7>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 6 && M == 8) e = LaunchKM<6, 8>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 2 && M == 2) e = LaunchKM<2, 2>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  else if (K == 7 && M == 9) e = LaunchKM<7, 9>(params, d_sol, d_elem_scalars, n, scratch, d_dt, st);
  if (e != cudaSuccess) return VCPG_E_CUDA;
  double status = 0.0;
  if (cudaMemcpyAsync(&status, scratch + kStatusSlot, sizeof(double), cudaMemcpyDeviceToHost,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return VCPG_E_CUDA;
  return status != 0.0 ? VCPG_E_NEG_A2 : VCPG_OK;
}
