// Sum-factorisation building blocks for one element processed by one CTA.
//
// All element arrays live in shared memory, variable-major and i fastest:
//   volume DOFs      [nv][K][K][K]      (k, j, i)
//   volume int. pts  [nv][M][M][M]
//   face arrays      [nv][S][F]         (S = slow, F = fast in-face axis)
// A 1-D operator is applied along one axis; every thread owns whole lines,
// loads the line into registers once and produces all outputs of the line
// with a sequential fused multiply-add chain over the input index, which is
// the summation order of the reference's tensor-product templates
// (include/TensorProductSolAndGradVolume.hpp:5-249,
//  include/TensorProductVolumeResidual.hpp:5-96,
//  include/TensorProductSolAndGrad[IJK]Face.hpp, include/TensorProductRes[IJK]Face.hpp).
//
// The 1-D operator values sit in constant memory, one table per (K, M) pair;
// with compile-time indices every coefficient is a uniform constant-bank
// operand of the FMA.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace vcpg {

constexpr int kKMax = 7;   // up to polynomial degree 6
constexpr int kMMax = 10;

struct OpTable {
  double leg[kKMax * kMMax];        // leg[k * M + m]: basis k at Gauss point m
  double dleg[kKMax * kMMax];       // derivative
  double face[2 * kKMax];           // [side][k], side 0: r = -1, side 1: r = +1
  double dface[2 * kKMax];
  double w[kMMax];                  // 1-D Gauss weights
  double legdof[kKMax * kKMax];     // legdof[k * K + i]: basis k at nodal DOF i
  double center[kKMax * kKMax * kKMax];
  // FP32 copies for the mixed-precision form.
  float legf[kKMax * kMMax];
  float dlegf[kKMax * kMMax];
  float facef[2 * kKMax];
  float dfacef[2 * kKMax];
  float wf[kMMax];
  float centerf[kKMax * kKMax * kKMax];
};

// Supported (K, M) pairs and their constant-memory slot.
template <int K, int M> struct Slot;
template <> struct Slot<2, 3> { static constexpr int value = 0; };
template <> struct Slot<3, 4> { static constexpr int value = 1; };
template <> struct Slot<4, 5> { static constexpr int value = 2; };
template <> struct Slot<5, 7> { static constexpr int value = 3; };
template <> struct Slot<6, 8> { static constexpr int value = 4; };
template <> struct Slot<7, 10> { static constexpr int value = 5; };
constexpr int kNumSlots = 6;

// One copy per translation unit; only kernels.cu launches kernels and uploads it.
static __constant__ OpTable c_ops[kNumSlots];

// Operator selection for a line transform.
enum OpSel {
  kLeg = 0,    // K -> M: out[m] = sum_k leg[k][m] in[k]
  kDLeg = 1,   // K -> M with the derivative
  kLegT = 2,   // M -> K: out[k] = sum_m leg[k][m] in[m]   (transposed operator)
  kDLegT = 3,  // M -> K with the derivative
  kLegDof = 4  // K -> K: out[i] = sum_k legdof[k][i] in[k]   (modal -> nodal)
};

template <int SLOT, int K, int M, int OP, typename T = double>
__device__ __forceinline__ T Coef(const int c, const int o) {
  if constexpr (std::is_same<T, float>::value) {
    if (OP == kLeg) return c_ops[SLOT].legf[c * M + o];
    if (OP == kDLeg) return c_ops[SLOT].dlegf[c * M + o];
    if (OP == kLegT) return c_ops[SLOT].legf[o * M + c];
    return c_ops[SLOT].dlegf[o * M + c];
  } else {
    if (OP == kLeg) return c_ops[SLOT].leg[c * M + o];
    if (OP == kDLeg) return c_ops[SLOT].dleg[c * M + o];
    if (OP == kLegT) return c_ops[SLOT].leg[o * M + c];
    if (OP == kLegDof) return c_ops[SLOT].legdof[c * K + o];
    return c_ops[SLOT].dleg[o * M + c];
  }
}

// Face basis values (side 0: r = -1, side 1: r = +1), 1-D weights and the centre
// basis in the compute precision.
template <int SLOT, typename T>
__device__ __forceinline__ T FaceVal(const int i) {
  if constexpr (std::is_same<T, float>::value) return c_ops[SLOT].facef[i];
  else return c_ops[SLOT].face[i];
}
template <int SLOT, typename T>
__device__ __forceinline__ T FaceDer(const int i) {
  if constexpr (std::is_same<T, float>::value) return c_ops[SLOT].dfacef[i];
  else return c_ops[SLOT].dface[i];
}
template <int SLOT, typename T>
__device__ __forceinline__ T Weight1D(const int i) {
  if constexpr (std::is_same<T, float>::value) return c_ops[SLOT].wf[i];
  else return c_ops[SLOT].w[i];
}
template <int SLOT, typename T>
__device__ __forceinline__ T CenterBasis(const int i) {
  if constexpr (std::is_same<T, float>::value) return c_ops[SLOT].centerf[i];
  else return c_ops[SLOT].center[i];
}

// Apply a 1-D operator along axis AX of in[NV][D2][D1][D0] (D_AX == NIN) and
// write (ACC: add) out[NV][D2'][D1'][D0'] where D_AX' == NOUT.
template <int NT, int SLOT, int K, int M, int OP, int AX, int NV, int D0, int D1, int D2,
          int NIN, int NOUT, bool ACC, typename T = double>
__device__ __forceinline__ void Contract(const T *__restrict__ in, T *__restrict__ out) {
  constexpr int O0 = AX == 0 ? NOUT : D0;
  constexpr int O1 = AX == 1 ? NOUT : D1;
  constexpr int O2 = AX == 2 ? NOUT : D2;
  // Non-contracted extents, the faster one first.
  constexpr int A = AX == 0 ? D1 : D0;
  constexpr int B = AX == 2 ? D1 : D2;
  constexpr int NLINES = NV * A * B;
  constexpr int IS = AX == 0 ? 1 : (AX == 1 ? D0 : D0 * D1);
  constexpr int OS = AX == 0 ? 1 : (AX == 1 ? O0 : O0 * O1);
  for (int line = threadIdx.x; line < NLINES; line += NT) {
    const int v = line / (A * B);
    const int r = line - v * (A * B);
    const int b = r / A;
    const int a = r - b * A;
    int ib, ob;
    if (AX == 0) {
      ib = ((v * D2 + b) * D1 + a) * D0;
      ob = ((v * O2 + b) * O1 + a) * O0;
    } else if (AX == 1) {
      ib = (v * D2 + b) * D1 * D0 + a;
      ob = (v * O2 + b) * O1 * O0 + a;
    } else {
      ib = v * D2 * D1 * D0 + b * D0 + a;
      ob = v * O2 * O1 * O0 + b * O0 + a;
    }
    T x[NIN];
#pragma unroll
    for (int c = 0; c < NIN; ++c) x[c] = in[ib + c * IS];
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      T acc = T(0);
#pragma unroll
      for (int c = 0; c < NIN; ++c) acc = fma(Coef<SLOT, K, M, OP, T>(c, o), x[c], acc);
      if (ACC)
        out[ob + o * OS] += acc;
      else
        out[ob + o * OS] = acc;
    }
  }
}

}  // namespace vcpg
