// Measured attempt: the 1-D line contractions of the sum-factorised residual
// (TPSAGV / TPAVR stages, include/TensorProductSolAndGradVolume.hpp:5-249) as
// Blackwell tensor-core tiles, against the FP32 fused multiply-add lines of the
// mixed-form residual kernel (dg_tensor.cuh, ContractL).
//
// One stage maps 128 lines of K inputs to M outputs: D[128 x 8] = X[128 x 8] B[8 x 8]
// with K, M <= 8 (degrees 4 and 5: K = 5, M = 7 and K = 6, M = 8), the inputs
// and the operator zero-padded to 8. The tensor-core variants stage X and the
// operator in shared memory in the K-major, no-swizzle canonical layout
// (8-row x 16-byte core matrices; LBO 128 B between the two K halves, SBO 256 B
// between 8-row groups), issue tcgen05.mma kind::tf32 from one thread with the
// accumulator in tensor memory, signal completion through tcgen05.commit on an
// mbarrier, and read D back with tcgen05.ld (thread t of warp w holds line
// 32 w + t). Variant 1 rounds the data and the operator to TF32 once; variant 2
// is the split "3xTF32" form, X B ~ Xhi Bhi + Xhi Blo + Xlo Bhi with hi =
// tf32(v), lo = tf32(v - hi), three MMAs into one accumulator. Variant 0 is the
// FMA path: one thread per line, its K inputs read from shared memory, M
// sequential FMA chains, the operator from shared memory; variant 3 is the same
// with the operator in constant memory, as the residual kernel holds it.
//
// Every variant runs `reps` chained stages per tile inside shared memory, as a
// residual kernel does between its global loads and stores: the stage writes its
// M outputs (the stage's result) and its first K outputs, scaled, as the next
// stage's inputs (for the tensor-core variants in the MMA layout, converted to
// TF32 and made visible to the tensor core's proxy). Only the last stage's
// outputs go to global memory. Used by python -m vcp3d_open_b200.tc_experiment;
// not part of the residual path.
//
// Waits on the mbarrier are bounded (2^26 polls); a wait that runs out sets an
// error flag, the CTA stops issuing work, waits once more (bounded) for its MMAs
// in flight and frees its tensor memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/vcp3d_b200.h"

namespace {

constexpr int kTile = 128;       // lines per MMA (M of the MMA)
constexpr int kN = 8;            // outputs per line, padded (N of the MMA)
constexpr int kKPad = 8;         // inputs per line, padded (one tf32 K step)
constexpr int kTmemCols = 32;    // smallest tensor-memory allocation
constexpr long long kPollLimit = 1ll << 26;

// Byte offset of element (row r, k) of a [rows x 8] K-major tile in the canonical
// no-swizzle layout: [row group][K half][8 rows][4 values].
__device__ __forceinline__ int CoreOffset(const int r, const int k) {
  return (r >> 3) * 256 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint32_t SmemAddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t SmemDesc(const void *tile) {
  const uint64_t a = (uint64_t)(SmemAddr(tile) & 0x3FFFFu) >> 4;
  return a | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor: D F32, A and B TF32, both K-major, N = 8, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ float ToTf32(const float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void Mma(const uint32_t tmem, const uint64_t a, const uint64_t b,
                                    const uint32_t accumulate) {
  // No output lane disabled (the four-word lane mask of cta_group::1 is zero).
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void Commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   SmemAddr(mbar))
               : "memory");
}

// Bounded wait for phase `parity` of the mbarrier; false when it ran out.
__device__ __forceinline__ bool WaitParity(uint64_t *mbar, const uint32_t parity) {
  const uint32_t a = SmemAddr(mbar);
  for (long long i = 0; i < kPollLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void LoadD8(const uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Tensor-core stages. Shared memory: X tiles (hi, lo) [2 buffers], operator tiles
// (hi, lo), the stage output [128][8]. 128 threads.
template <int K, int M, bool SPLIT>
__global__ void __launch_bounds__(128) TcContractKernel(const float *x, const float *op,
                                                        float *y, int n_tiles, int reps,
                                                        float scale, int *error) {
  __shared__ __align__(128) unsigned char s_x[2][2][kTile * kKPad * 4];  // [buf][hi/lo]
  __shared__ __align__(128) unsigned char s_b[2][kN * kKPad * 4];        // [hi/lo]
  __shared__ __align__(16) float s_out[kTile][kN];
  __shared__ __align__(8) uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(SmemAddr(&s_mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     SmemAddr(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // The operator B[k][n] (rows n of the K-major tile), hi and lo parts, zero-padded.
  for (int i = tid; i < kN * kKPad; i += 128) {
    const int n = i / kKPad, k = i % kKPad;
    const float b = (n < M && k < K) ? op[k * M + n] : 0.0f;
    const float hi = ToTf32(b);
    *reinterpret_cast<float *>(s_b[0] + CoreOffset(n, k)) = hi;
    *reinterpret_cast<float *>(s_b[1] + CoreOffset(n, k)) = ToTf32(b - hi);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t myLanes = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    // This thread's line into buffer 0 (hi and lo), inputs zero-padded to 8.
    const float *src = x + ((size_t)tile * kTile + tid) * K;
    int buf = 0;
#pragma unroll
    for (int k = 0; k < kKPad; ++k) {
      const float v = k < K ? src[k] : 0.0f;
      const float hi = ToTf32(v);
      *reinterpret_cast<float *>(s_x[0][0] + CoreOffset(tid, k)) = hi;
      *reinterpret_cast<float *>(s_x[0][1] + CoreOffset(tid, k)) = ToTf32(v - hi);
    }
    for (int r = 0; r < reps; ++r) {
      // Make the generic-proxy stores of this stage's inputs visible to the MMA.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (s_fail) break;
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        Mma(tmem, SmemDesc(s_x[buf][0]), SmemDesc(s_b[0]), 0u);
        if (SPLIT) {
          Mma(tmem, SmemDesc(s_x[buf][0]), SmemDesc(s_b[1]), 1u);
          Mma(tmem, SmemDesc(s_x[buf][1]), SmemDesc(s_b[0]), 1u);
        }
        Commit(&s_mbar);
      }
      if (!WaitParity(&s_mbar, phase)) {
        atomicExch(&s_fail, 1);
        atomicExch(error, 1);
        break;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float d[8];
      LoadD8(myLanes, d);
      // The stage's output, and the next stage's inputs (first K outputs, scaled).
#pragma unroll
      for (int m = 0; m < kN; ++m) s_out[tid][m] = d[m];
      const int nb = buf ^ 1;
#pragma unroll
      for (int k = 0; k < kKPad; ++k) {
        const float v = k < K ? scale * d[k] : 0.0f;
        const float hi = ToTf32(v);
        *reinterpret_cast<float *>(s_x[nb][0] + CoreOffset(tid, k)) = hi;
        *reinterpret_cast<float *>(s_x[nb][1] + CoreOffset(tid, k)) = ToTf32(v - hi);
      }
      buf = nb;
    }
    if (s_fail) break;
    __syncthreads();
    float *dst = y + ((size_t)tile * kTile + tid) * M;
#pragma unroll
    for (int m = 0; m < M; ++m) dst[m] = s_out[tid][m];
  }
  if (s_fail && tid == 0) {
    // Let any MMA still in flight finish before the tensor memory is freed.
    Commit(&s_mbar);
    WaitParity(&s_mbar, phase);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}

// The operator in constant memory (variant 3: the residual kernel's operand source).
__constant__ float c_probe_op[kKPad * kN];

// FMA stages: one thread per line, inputs and outputs in shared memory; the
// operator read from shared memory (variant 0, as a TMA- or bulk-copied operator
// table would be) or from the constant bank (variant 3, uniform operands).
template <int K, int M, bool CONST_OP>
__global__ void __launch_bounds__(128) FmaContractKernel(const float *x, const float *op,
                                                         float *y, int n_tiles, int reps,
                                                         float scale) {
  __shared__ float s_x[2][kTile][kKPad];
  __shared__ float s_out[kTile][kN];
  __shared__ float s_op[K * M];
  const int tid = threadIdx.x;
  for (int i = tid; i < K * M; i += 128) s_op[i] = op[i];
  __syncthreads();
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const float *src = x + ((size_t)tile * kTile + tid) * K;
#pragma unroll
    for (int k = 0; k < K; ++k) s_x[0][tid][k] = src[k];
    int buf = 0;
    for (int r = 0; r < reps; ++r) {
      __syncthreads();
      float xv[K];
#pragma unroll
      for (int k = 0; k < K; ++k) xv[k] = s_x[buf][tid][k];
      float d[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < K; ++k)
          acc = fmaf(CONST_OP ? c_probe_op[k * M + m] : s_op[k * M + m], xv[k], acc);
        d[m] = acc;
        s_out[tid][m] = acc;
      }
      const int nb = buf ^ 1;
#pragma unroll
      for (int k = 0; k < K; ++k) s_x[nb][tid][k] = scale * d[k];
      buf = nb;
    }
    __syncthreads();
    float *dst = y + ((size_t)tile * kTile + tid) * M;
#pragma unroll
    for (int m = 0; m < M; ++m) dst[m] = s_out[tid][m];
  }
}

template <int K, int M>
cudaError_t Launch(int variant, const float *x, const float *op, float *y, int n_tiles,
                   int reps, float scale, int *err, int grid, cudaStream_t st) {
  if (variant == 0)
    FmaContractKernel<K, M, false><<<grid, 128, 0, st>>>(x, op, y, n_tiles, reps, scale);
  else if (variant == 3)
    FmaContractKernel<K, M, true><<<grid, 128, 0, st>>>(x, op, y, n_tiles, reps, scale);
  else if (variant == 1)
    TcContractKernel<K, M, false><<<grid, 128, 0, st>>>(x, op, y, n_tiles, reps, scale, err);
  else
    TcContractKernel<K, M, true><<<grid, 128, 0, st>>>(x, op, y, n_tiles, reps, scale, err);
  return cudaGetLastError();
}

}  // namespace

extern "C" int vcpg_line_contraction_probe(int32_t variant, int32_t K, int32_t M,
                                           int64_t n_lines, int32_t reps, float scale,
                                           const float *x, const float *op, float *y,
                                           double *ms) {
  if (variant < 0 || variant > 3 || reps < 1 || n_lines < kTile || n_lines % kTile || !x ||
      !op || !y || !ms)
    return VCPG_E_INVALID;
  if (!((K == 5 && M == 7) || (K == 6 && M == 8))) return VCPG_E_UNSUPPORTED_KM;
  const int n_tiles = (int)(n_lines / kTile);
  float *dx = nullptr, *dop = nullptr, *dy = nullptr;
  int *derr = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = VCPG_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == VCPG_OK) rc = VCPG_E_CUDA;
    return rc == VCPG_OK;
  };
  int dev = 0, sms = 0;
  if (ok(cudaGetDevice(&dev)) && ok(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) &&
      ok(cudaMalloc((void **)&dx, sizeof(float) * n_lines * K)) &&
      ok(cudaMalloc((void **)&dop, sizeof(float) * K * M)) &&
      ok(cudaMalloc((void **)&dy, sizeof(float) * n_lines * M)) &&
      ok(cudaMalloc((void **)&derr, sizeof(int))) && ok(cudaMemset(derr, 0, sizeof(int))) &&
      ok(cudaMemcpy(dx, x, sizeof(float) * n_lines * K, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(dop, op, sizeof(float) * K * M, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpyToSymbol(c_probe_op, op, sizeof(float) * K * M)) &&
      ok(cudaEventCreate(&e0)) && ok(cudaEventCreate(&e1))) {
    // Four resident CTAs per SM (tensor memory: 4 x 32 of 512 columns).
    const int grid = n_tiles < 4 * sms ? n_tiles : 4 * sms;
    cudaError_t (*launch)(int, const float *, const float *, float *, int, int, float, int *,
                          int, cudaStream_t) =
        K == 5 ? Launch<5, 7> : Launch<6, 8>;
    if (ok(launch(variant, dx, dop, dy, n_tiles, reps, scale, derr, grid, nullptr)) &&
        ok(cudaDeviceSynchronize()) && ok(cudaEventRecord(e0)) &&
        ok(launch(variant, dx, dop, dy, n_tiles, reps, scale, derr, grid, nullptr)) &&
        ok(cudaEventRecord(e1)) && ok(cudaEventSynchronize(e1))) {
      float t = 0.f;
      int herr = 0;
      if (ok(cudaEventElapsedTime(&t, e0, e1)) &&
          ok(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost)) &&
          ok(cudaMemcpy(y, dy, sizeof(float) * n_lines * M, cudaMemcpyDeviceToHost))) {
        *ms = t;
        if (herr) rc = VCPG_E_CUDA;
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(dx);
  cudaFree(dop);
  cudaFree(dy);
  cudaFree(derr);
  return rc;
}
