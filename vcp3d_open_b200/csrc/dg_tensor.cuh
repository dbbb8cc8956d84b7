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
// The 1-D operator values sit in constant memory, one exactly sized table per
// (K, M) pair; with compile-time indices every coefficient is a uniform
// constant-bank operand of the FMA.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace vcpg {

constexpr int kKMax = 10;   // up to polynomial degree 9
constexpr int kMMax = 14;

// The 1-D operators of one (K, M) pair, sized exactly (constant memory holds
// every supported pair's table).
template <int K, int M> struct OpTableKM {
  double leg[K * M];           // leg[k * M + m]: basis k at Gauss point m
  double dleg[K * M];          // derivative
  double face[2 * K];          // [side][k], side 0: r = -1, side 1: r = +1
  double dface[2 * K];
  double w[M];                 // 1-D Gauss weights
  double legdof[K * K];        // legdof[k * K + i]: basis k at nodal DOF i
  double dlegdof[K * K];       // its derivative (time step with an SGS model)
  // FP32 copies for the mixed-precision form.
  float legf[K * M];
  float dlegf[K * M];
  float facef[2 * K];
  float dfacef[2 * K];
  float wf[M];
};

// Supported (K, M) pairs -- the reference's tensor-product dispatch
// (src/TensorProductVolumeResidualK2.cpp ... K10.cpp) -- and their slots.
#define VCPG_SLOTS(X) \
  X(0, 2, 2) X(1, 2, 3) X(2, 3, 4) X(3, 4, 5) X(4, 5, 7) X(5, 6, 8) X(6, 7, 9) X(7, 8, 12) \
  X(8, 9, 13) X(9, 10, 14)
constexpr int kNumSlots = 10;

template <int K, int M> struct Slot;
template <int SLOT> struct SlotOps;
// One copy per translation unit: every unit that launches kernels uploads its
// own (UploadOperators).
#define VCPG_SLOT_DECL(S_, K_, M_)                                                          \
  template <> struct Slot<K_, M_> { static constexpr int value = S_; };                     \
  static __constant__ OpTableKM<K_, M_> c_ops##S_;                                          \
  template <> struct SlotOps<S_> {                                                          \
    __device__ static __forceinline__ const OpTableKM<K_, M_> &get() { return c_ops##S_; } \
  };
VCPG_SLOTS(VCPG_SLOT_DECL)
#undef VCPG_SLOT_DECL

template <int SLOT> __device__ __forceinline__ decltype(auto) Ops() { return SlotOps<SLOT>::get(); }

// Fills and uploads the table of one pair from the C-ABI operator arrays of
// this unit's copy (legdof / dlegdof may be absent: zeros). With a stream the
// copy is ordered on that stream (the host table is staged before the call
// returns); without one it is a synchronous copy.
template <int K, int M, typename Sym>
static inline cudaError_t UploadOperatorsKM(const Sym &sym, const double *leg, const double *dleg,
                                            const double *face, const double *dface,
                                            const double *w, const double *legdof,
                                            const double *dlegdof, cudaStream_t st,
                                            bool async) {
  OpTableKM<K, M> t{};
  for (int i = 0; i < K * M; ++i) {
    t.leg[i] = leg[i];
    t.dleg[i] = dleg[i];
    t.legf[i] = (float)leg[i];    // rounded once from the FP64 operators
    t.dlegf[i] = (float)dleg[i];
  }
  for (int i = 0; i < 2 * K; ++i) {
    t.face[i] = face[i];
    t.dface[i] = dface[i];
    t.facef[i] = (float)face[i];
    t.dfacef[i] = (float)dface[i];
  }
  for (int m = 0; m < M; ++m) {
    t.w[m] = w[m];
    t.wf[m] = (float)w[m];
  }
  for (int i = 0; i < K * K; ++i) {
    t.legdof[i] = legdof ? legdof[i] : 0.0;
    t.dlegdof[i] = dlegdof ? dlegdof[i] : 0.0;
  }
  if (async) return cudaMemcpyToSymbolAsync(sym, &t, sizeof(t), 0, cudaMemcpyHostToDevice, st);
  return cudaMemcpyToSymbol(sym, &t, sizeof(t), 0, cudaMemcpyHostToDevice);
}

static inline cudaError_t UploadOperators(int K, int M, const double *leg, const double *dleg,
                                          const double *face, const double *dface,
                                          const double *w, const double *legdof,
                                          const double *dlegdof, cudaStream_t st = nullptr,
                                          bool async = false) {
#define VCPG_SLOT_UPLOAD(S_, K_, M_)                                                  \
  if (K == K_ && M == M_)                                                             \
    return UploadOperatorsKM<K_, M_>(c_ops##S_, leg, dleg, face, dface, w, legdof, dlegdof, \
                                     st, async);
  VCPG_SLOTS(VCPG_SLOT_UPLOAD)
#undef VCPG_SLOT_UPLOAD
  return cudaErrorInvalidValue;
}

// Operator selection for a line transform.
enum OpSel {
  kLeg = 0,    // K -> M: out[m] = sum_k leg[k][m] in[k]
  kDLeg = 1,   // K -> M with the derivative
  kLegT = 2,   // M -> K: out[k] = sum_m leg[k][m] in[m]   (transposed operator)
  kDLegT = 3,  // M -> K with the derivative
  kLegDof = 4,  // K -> K: out[i] = sum_k legdof[k][i] in[k]   (modal -> nodal)
  kDLegDof = 5  // K -> K with the derivative
};

template <int SLOT, int K, int M, int OP, typename T = double>
__device__ __forceinline__ T Coef(const int c, const int o) {
  if constexpr (std::is_same<T, float>::value) {
    if (OP == kLeg) return Ops<SLOT>().legf[c * M + o];
    if (OP == kDLeg) return Ops<SLOT>().dlegf[c * M + o];
    if (OP == kLegT) return Ops<SLOT>().legf[o * M + c];
    return Ops<SLOT>().dlegf[o * M + c];
  } else {
    if (OP == kLeg) return Ops<SLOT>().leg[c * M + o];
    if (OP == kDLeg) return Ops<SLOT>().dleg[c * M + o];
    if (OP == kLegT) return Ops<SLOT>().leg[o * M + c];
    if (OP == kLegDof) return Ops<SLOT>().legdof[c * K + o];
    if (OP == kDLegDof) return Ops<SLOT>().dlegdof[c * K + o];
    return Ops<SLOT>().dleg[o * M + c];
  }
}

// Face basis values (side 0: r = -1, side 1: r = +1) and 1-D weights in the
// compute precision.
template <int SLOT, typename T>
__device__ __forceinline__ T FaceVal(const int i) {
  if constexpr (std::is_same<T, float>::value) return Ops<SLOT>().facef[i];
  else return Ops<SLOT>().face[i];
}
template <int SLOT, typename T>
__device__ __forceinline__ T FaceDer(const int i) {
  if constexpr (std::is_same<T, float>::value) return Ops<SLOT>().dfacef[i];
  else return Ops<SLOT>().dface[i];
}
template <int SLOT, typename T>
__device__ __forceinline__ T Weight1D(const int i) {
  if constexpr (std::is_same<T, float>::value) return Ops<SLOT>().wf[i];
  else return Ops<SLOT>().w[i];
}

// Strides (in elements) of an array [NV][D2][D1][D0] with unit stride along D0:
// S1 along D1, S2 along D2, SV between variables. Padded strides keep the
// lines that one warp touches on distinct shared-memory banks.
template <int S1_, int S2_, int SV_> struct Lay {
  static constexpr int S1 = S1_, S2 = S2_, SV = SV_;
};
template <int D0, int D1, int D2> using Dense = Lay<D0, D0 * D1, D0 * D1 * D2>;

// Apply a 1-D operator along axis AX of in[NV][D2][D1][D0] (layout LI, D_AX ==
// NIN) and write (ACC: add) out[NV][D2'][D1'][D0'] (layout LO) where D_AX' == NOUT.
template <int NT, int SLOT, int K, int M, int OP, int AX, int NV, int D0, int D1, int D2,
          int NIN, int NOUT, bool ACC, typename T, typename LI, typename LO>
__device__ __forceinline__ void ContractL(const T *__restrict__ in, T *__restrict__ out) {
  // Non-contracted extents, the faster one first.
  constexpr int A = AX == 0 ? D1 : D0;
  constexpr int B = AX == 2 ? D1 : D2;
  constexpr int NLINES = NV * A * B;
  constexpr int IS = AX == 0 ? 1 : (AX == 1 ? LI::S1 : LI::S2);
  constexpr int OS = AX == 0 ? 1 : (AX == 1 ? LO::S1 : LO::S2);
  for (int line = threadIdx.x; line < NLINES; line += NT) {
    const int v = line / (A * B);
    const int r = line - v * (A * B);
    const int b = r / A;
    const int a = r - b * A;
    int ib, ob;
    if (AX == 0) {
      ib = v * LI::SV + b * LI::S2 + a * LI::S1;
      ob = v * LO::SV + b * LO::S2 + a * LO::S1;
    } else if (AX == 1) {
      ib = v * LI::SV + b * LI::S2 + a;
      ob = v * LO::SV + b * LO::S2 + a;
    } else {
      ib = v * LI::SV + b * LI::S1 + a;
      ob = v * LO::SV + b * LO::S1 + a;
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

// Dense layouts on both sides.
template <int NT, int SLOT, int K, int M, int OP, int AX, int NV, int D0, int D1, int D2,
          int NIN, int NOUT, bool ACC, typename T = double>
__device__ __forceinline__ void Contract(const T *__restrict__ in, T *__restrict__ out) {
  constexpr int O0 = AX == 0 ? NOUT : D0;
  constexpr int O1 = AX == 1 ? NOUT : D1;
  constexpr int O2 = AX == 2 ? NOUT : D2;
  ContractL<NT, SLOT, K, M, OP, AX, NV, D0, D1, D2, NIN, NOUT, ACC, T, Dense<D0, D1, D2>,
            Dense<O0, O1, O2>>(in, out);
}

// Padded shared-memory layouts of the mass-matrix CG arrays, chosen per (K, M)
// and element size by minimising the shared-memory wavefronts of one iteration
// in a bank model (16 eight-byte or 32 four-byte banks; the warps' lines as the
// CG steps assign them at the launch's threads per CTA):
//   P  DOF vectors z, p, Ap, x      [5][K][K][K]
//   A  k-transformed                [5][M][K][K]   (forward)
//   B  k,j-transformed              [5][M][M][K]   (forward)
//   C  integration points           [5][M][M][M]
//   D  k-transformed back           [5][K][M][M]
//   E  k,j-transformed back         [5][K][K][M]
template <int K, int M, int ES> struct CgLayout {
  using P = Dense<K, K, K>;
  using A = Dense<K, K, M>;
  using B = Dense<K, M, M>;
  using C = Dense<M, M, M>;
  using D = Dense<M, M, K>;
  using E = Dense<M, K, K>;
};
#define VCPG_CG_LAYOUT(K_, M_, ES_, P_, A_, B_, C_, D_, E_)                                \
  template <> struct CgLayout<K_, M_, ES_> {                                              \
    using P = Lay<P_>; using A = Lay<A_>; using B = Lay<B_>;                              \
    using C = Lay<C_>; using D = Lay<D_>; using E = Lay<E_>;                              \
  };
#define VCPG_L(a, b, c) a, b, c
VCPG_CG_LAYOUT(2, 3, 8, VCPG_L(2, 5, 10), VCPG_L(2, 5, 18), VCPG_L(3, 9, 27), VCPG_L(3, 11, 41),
               VCPG_L(3, 13, 26), VCPG_L(3, 8, 19))
VCPG_CG_LAYOUT(3, 4, 8, VCPG_L(3, 9, 27), VCPG_L(3, 10, 41), VCPG_L(4, 19, 76), VCPG_L(4, 16, 64),
               VCPG_L(4, 18, 54), VCPG_L(7, 21, 63))
VCPG_CG_LAYOUT(4, 5, 8, VCPG_L(4, 17, 68), VCPG_L(4, 18, 90), VCPG_L(5, 28, 140),
               VCPG_L(5, 26, 137), VCPG_L(5, 26, 105), VCPG_L(8, 37, 148))
VCPG_CG_LAYOUT(5, 7, 8, VCPG_L(5, 25, 125), VCPG_L(6, 37, 259), VCPG_L(5, 37, 259),
               VCPG_L(7, 49, 343), VCPG_L(7, 55, 275), VCPG_L(10, 55, 275))
VCPG_CG_LAYOUT(6, 8, 8, VCPG_L(6, 36, 217), VCPG_L(6, 38, 308), VCPG_L(6, 54, 432),
               VCPG_L(8, 64, 512), VCPG_L(8, 72, 432), VCPG_L(9, 56, 336))
VCPG_CG_LAYOUT(2, 3, 4, VCPG_L(2, 5, 12), VCPG_L(2, 6, 18), VCPG_L(2, 6, 18), VCPG_L(3, 11, 41),
               VCPG_L(3, 17, 41), VCPG_L(4, 15, 35))
VCPG_CG_LAYOUT(3, 4, 4, VCPG_L(3, 11, 41), VCPG_L(3, 9, 43), VCPG_L(6, 29, 116),
               VCPG_L(4, 16, 64), VCPG_L(4, 20, 60), VCPG_L(5, 20, 60))
VCPG_CG_LAYOUT(4, 5, 4, VCPG_L(4, 16, 65), VCPG_L(4, 20, 100), VCPG_L(4, 20, 100),
               VCPG_L(5, 25, 125), VCPG_L(6, 37, 148), VCPG_L(8, 37, 148))
VCPG_CG_LAYOUT(5, 7, 4, VCPG_L(5, 25, 125), VCPG_L(5, 26, 185), VCPG_L(5, 37, 259),
               VCPG_L(7, 49, 343), VCPG_L(7, 53, 273), VCPG_L(9, 45, 225))
VCPG_CG_LAYOUT(6, 8, 4, VCPG_L(6, 36, 217), VCPG_L(6, 38, 304), VCPG_L(8, 70, 560),
               VCPG_L(8, 64, 512), VCPG_L(8, 72, 432), VCPG_L(9, 56, 336))
#undef VCPG_L
#undef VCPG_CG_LAYOUT

}  // namespace vcpg
