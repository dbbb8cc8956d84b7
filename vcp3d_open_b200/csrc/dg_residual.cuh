// Fused FP64 DG residual kernel: one CTA per element computes the volume
// terms, all six faces and the generalised mass-matrix solve of its element.
//
// Reference path (per element, SolverClass::Residual, src/SolverClass.cpp:3381-3795):
//   VolumeResidual (src/ElementClass.cpp:3809-4534)
//   I/J/KFaceResiduals (src/ElementClass.cpp:2582-3404) with FluxesInternalFace
//     (src/FluxesFace.cpp:220-343)
//   neighbour Min-face residual accumulation (src/SolverClass.cpp:3616-3732)
//   MultiplyResInverseMassMatrix -> CG_EntropyVarMassMatrix (src/CG_MassMatrix.cpp:250-504)
//
// Every interior face is evaluated by both of its elements with identical
// inputs, so the two sides see bit-identical fluxes and no cross-element
// write (and no atomic) is needed. The residual of an element is accumulated
// in the reference's order: volume (x, y, z), own Min faces (i, j, k), then
// the Max-face contributions each summed from zero and added (i, j, k).
#pragma once

#include <type_traits>

#include "dg_physics.cuh"
#include "dg_rk.cuh"
#include "dg_tensor.cuh"

namespace vcpg {

// States of a case in a bucket that holds several cases (csrc/ensemble.cu).
enum CaseState { kCaseFree = 0, kCasePending = 1, kCaseRunning = 2, kCaseDone = 3 };
// Per-case parameters, [nCases][kCasePar].
enum CasePar { kParMu = 0, kParPRef = 1, kParURef = 2, kParRhoRef = 3, kParCfl = 4, kCasePar = 8 };

// Per-case view of a bucket holding several cases of one (K, M) pair; a null
// elem_case means a single case (case 0) whose parameters are the scalars of
// the launch arguments.
struct CaseView {
  const int *elem_case;  // [nE] case slot of each element, -1 = unused element
  const int *state;      // [nCases] enum CaseState
  const double *par;     // [nCases][kCasePar]
  int require;           // the state a residual or boundary launch processes
};

struct ResidualArgs {
  const double *sol;           // [nE][5][K^3]
  double *res;                 // [nE][5][K^3] residual after the mass-matrix solve
  double *res_raw;             // optional [nE][5][K^3] residual before the solve
  const double *vol_metric;    // [nE][10][M^3]
  const double *face_metric;   // [nE][6][13][M^2]
  const double *elem_scalars;  // [nE][15]
  const int *nbr;              // [nE][6]
  int n_elem;                  // elements whose residual is computed
  // Elements whose Min-face fluxes FaceFluxKernel computes (0: n_elem). More than
  // n_elem in a partitioned block: the ghost elements above the owned ones.
  int n_face_elem;
  // First element of the launch's range: FaceFluxKernel covers elements
  // [face_first, face_first + n_face_elem), ResidualKernel [res_first,
  // res_first + n_elem) (0 and the counts above for a whole block; ranges split
  // a partitioned residual around the halo exchange).
  int face_first, res_first;
  double mu;                   // non-dimensional viscosity
  double tau_num;              // (p+1)^2 * relative penalty parameter
  double theta_sym;
  int riemann;                 // 0 Roe, 1 Ismail-Roe
  int metric_compat;           // 1: metric indexed by the variable index
  unsigned long long *mach2max;  // optional: bits of max Mach^2 (non-negative double)
  int sgs;                     // enum vcpg_sgs: subgrid-scale model
  unsigned long long *eddymax;   // optional: bits of the max eddy viscosity
  int *status;                 // [0] CG iteration cap hits, [1] boundary face without BC
  unsigned long long *cg_stats;  // [0] CG iterations, [1] element solves (cumulative)
  double cg_tol;               // relative CG stopping tolerance (1e-10 in the FP64 form)
  int mixed;                   // 1: FP32 compute (contractions, fluxes, mass solve)
  // Open boundaries (null / 0 for a block without them). Boundary faces carry
  // nbr = -2 - b, b indexing bflux; nbr = -1 is a physical face without a BC.
  int open;                    // 1: launch the variant with boundary faces and sponges
  const double *bflux;         // [nB][4][5][M^2] boundary-face fluxes (dg_boundary.cuh)
  const int *sponge_idx;       // [nE] sponge-layer index or -1
  const double *damp_fn;       // [nS][3][M^3] damping function per direction
  const double *damp_state;    // [nS][5][M^3] conservative damping state
  const double *cml;           // [nS][6] 1/sigma per direction, layer orientation
  int cml_on;                  // characteristic matching layer in sponge elements
  CaseView cases;              // several cases per launch (null elem_case: one case)
  // [nE][3][20][M^2] fluxes of every element's Min faces in the compute precision
  // (FaceFluxKernel writes them, the residual kernel reads them).
  void *face_flux;
  const double *center;        // [K^3] 3-D basis at the element centre (CG preconditioner)
  // Degrees whose element arrays exceed the shared memory of one CTA: one
  // global scratch area per CTA of a grid that loops over the elements.
  void *scratch;
  int scratch_ctas;            // CTAs the scratch areas hold (the grid of those degrees)
  int body_force;              // 1: the body-force source with fbody
  double fbody[3];             // body force per unit volume / p_ref
  // Runge-Kutta stage update fused into the epilogue (enum RkKind; single-case
  // steps): the element's residual updates its own state in place (no other CTA
  // of the residual kernel reads it) and is written to res only with
  // rk_store_res. kRkNone writes res.
  int rk_kind;
  int rk_store_res;
  double rk_a, rk_b;           // low-storage (a, b) or SSP (alpha, beta)
  const double *rk_dt;         // the step's time step (device)
  double *rk_sol;              // the state (the array sol points to)
  double *rk_reg;              // du (low-storage) or solOld (SSP)
};

// Whether the residual kernel of (K, M, T, OPEN) fetches the fused stage update's
// inputs asynchronously into its free work area (MassSolve); without that the
// epilogue's dependent loads lengthen every element (degrees 7-9 with their
// element arrays in global scratch, and the mixed form of degrees 5 and 6), and a
// step there applies the updates with the separate stage kernels.
template <int K, int M, typename T, bool OPEN> struct FusedUpdatePrefetch;

// Final value r of residual entry gi (after the mass-matrix solve): stored, or
// applied to the state by the fused stage update, whose inputs are the entry's
// state sol0 and its second register reg0 (du or solOld).
__device__ __forceinline__ void StoreResidual(const ResidualArgs &a, const size_t gi,
                                              const double r, const double dt,
                                              const double sol0, const double reg0) {
  if (a.rk_kind == kRkNone || a.rk_store_res) a.res[gi] = r;
  if (a.rk_kind == kRkNone) return;
  double s = sol0, g = reg0;
  if (a.rk_kind == kRkLowStorage) {
    LsrkUpdate(s, g, r, dt, a.rk_a, a.rk_b);
    a.rk_reg[gi] = g;
  } else {
    SspUpdate(s, g, r, dt, a.rk_a, a.rk_b);
  }
  a.rk_sol[gi] = s;
}

// Arguments of the CFL time-step kernels (dg_timestep.cuh).
struct TimeStepArgs {
  const double *sol;
  const double *elem_scalars;
  int n_elem;
  int n_poly;
  double cfl, mu, p_ref, u_ref, rho_ref;
  unsigned long long *dt_bits;  // per case: bits of the minimum over its elements
  int *status;  // [2]: negative a^2 seen
  CaseView cases;  // several cases: per-case parameters and time steps
  int sgs;                          // enum vcpg_sgs
  const double *vol_metric_dofs;    // [nE][10][K^3] metric at the nodal DOFs (with sgs)
  void *scratch;                    // degree 9 with a model: 32 K^3 doubles per CTA
  int scratch_ctas;
};

// Asynchronous 8-byte copy global -> shared (cp.async; the calling thread waits
// for its own copies with CpAsyncWaitAll).
__device__ __forceinline__ void CpAsync8(double *dst_smem, const double *src_gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src_gmem) : "memory");
}
// One bulk copy (the TMA engine's 1-D form, no multicast) of `bytes` from global
// to this CTA's shared memory, completing on the mbarrier `bar` (both 16-byte
// aligned, bytes a multiple of 16); issued by one thread after
// BulkBarrierInit and an arrive that expects the bytes.
__device__ __forceinline__ void BulkBarrierInit(unsigned long long *bar) {
  const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void BulkCopyToShared(void *dst_smem, const void *src_gmem,
                                                 const unsigned bytes,
                                                 unsigned long long *bar) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst_smem));
  const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
               ::"r"(b), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(d), "l"(src_gmem), "r"(bytes), "r"(b) : "memory");
}
// Waits for phase 0 of the mbarrier with a bounded number of polls; false when
// the bound ran out (the caller records it).
__device__ __forceinline__ bool BulkWait(unsigned long long *bar) {
  const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  for (int i = 0; i < (1 << 24); ++i) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(b) : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void CpAsyncWaitAll() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int NT, typename T>
__device__ __forceinline__ T BlockSum(T v, T *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T s = T(0.0);
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

template <int NT, typename T>
__device__ __forceinline__ T BlockMax(T v, T *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T s = red[0];
#pragma unroll
  for (int i = 1; i < NT / 32; ++i) s = Fmax(s, red[i]);
  return s;
}

// Single-barrier block reductions for loops that alternate two scratch areas:
// the caller guarantees that no thread still reads `red` from its previous use
// (a barrier lies between that read and this call).
template <int NT, typename T>
__device__ __forceinline__ T BlockSum1(T v, T *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  T s = T(0.0);
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

// Block-wide (sum a, sum b, max c) with one barrier, under the same condition
// as BlockSum1; red needs 3*NT/32.
template <int NT, typename T>
__device__ __forceinline__ void BlockReduce3(T &a, T &b, T &c, T *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c = Fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[w] = a; red[NT / 32 + w] = b; red[2 * (NT / 32) + w] = c; }
  __syncthreads();
  a = T(0.0); b = T(0.0); c = red[2 * (NT / 32)];
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) {
    a += red[i];
    b += red[NT / 32 + i];
    c = Fmax(c, red[2 * (NT / 32) + i]);
  }
}

// Upper bounds of the CTAs per SM that __launch_bounds__ asks the register
// allocator for (a higher value caps the registers per thread lower: 4 CTAs of
// 128 threads allow 128 registers, 6 allow 80, 8 allow 64), where the shared
// memory would allow more. Chosen by measurement on B200 (bench.py, TGV and
// pulse workloads, degrees 2-5): more, smaller-register CTAs pay for the FP32
// form of degrees 2 and 3 (16-44 % per step despite small spills) and for the
// face-flux kernel of every degree up to 5 (FP64 degree 3: 5 CTAs without the
// neighbour staging, which leaves room for 4 only, +5 %); the FP64 residual
// kernel of degree 2 and the FP32 one of degrees 4-5 lose with more.
#ifndef VCPG_CAP_RES_FP64
#define VCPG_CAP_RES_FP64 4          // FP64 residual kernel, 128-thread CTAs
#endif
#ifndef VCPG_CAP_RES_FP64_SMALL
#define VCPG_CAP_RES_FP64_SMALL 4    // the same, degrees <= 2
#endif
#ifndef VCPG_CAP_RES_FP32_K4
#define VCPG_CAP_RES_FP32_K4 6       // FP32 residual kernel, degree 3
#endif
#ifndef VCPG_CAP_RES_FP32_SMALL
#define VCPG_CAP_RES_FP32_SMALL 8    // FP32 residual kernel, degrees <= 2
#endif
#ifndef VCPG_CAP_RES_FP32_256
#define VCPG_CAP_RES_FP32_256 3      // FP32 residual kernel, 256-thread CTAs (degrees >= 4)
#endif
#ifndef VCPG_CAP_FLUX_FP64_SMALL
#define VCPG_CAP_FLUX_FP64_SMALL 6   // FP64 face-flux kernel, degrees <= 2
#endif
#ifndef VCPG_CAP_FLUX_FP64_K4
#define VCPG_CAP_FLUX_FP64_K4 5      // FP64 face-flux kernel, degree 3 (no neighbour staging then)
#endif
#ifndef VCPG_CAP_FLUX_FP32_K4
#define VCPG_CAP_FLUX_FP32_K4 8      // FP32 face-flux kernel, degree 3
#endif
#ifndef VCPG_CAP_FLUX_FP32_SMALL
#define VCPG_CAP_FLUX_FP32_SMALL 8   // FP32 face-flux kernel, degrees <= 2
#endif
#ifndef VCPG_CAP_FLUX_FP64_BIG
#define VCPG_CAP_FLUX_FP64_BIG 2     // FP64 face-flux kernel, 160-thread CTAs (degrees >= 4)
#endif
#ifndef VCPG_CAP_FLUX_FP32_BIG
#define VCPG_CAP_FLUX_FP32_BIG 4     // FP32 face-flux kernel, 160-thread CTAs
#endif

// Shared-memory plan (doubles) of the fused kernel for a (K, M) pair.
template <int K, int M, typename T = double, bool OPEN = false> struct Plan {
  static constexpr int KD = K * K * K, MD = M * M * M, M2 = M * M;
  static constexpr int TK = 5 * K * K * M;      // first-stage buffer
  static constexpr int TJ = 5 * K * M * M;      // second-stage buffer
  // Face phase: the distribution inputs of the six faces (120 M^2) and their
  // slow-axis results (120 K M); the traces and fluxes are computed by
  // FaceFluxKernel.
  static constexpr int FACE = 120 * M2 + 120 * K * M;
  // CG phase: z, p, Ap, x, pInt and the contraction buffers (padded layouts).
  using CL = CgLayout<K, M, (int)sizeof(T)>;
  static constexpr int CG_TK = 5 * (CL::A::SV > CL::E::SV ? CL::A::SV : CL::E::SV);
  static constexpr int CG_TJ = 5 * (CL::B::SV > CL::D::SV ? CL::B::SV : CL::D::SV);
  // The last 32 entries hold the preconditioner and the centre's entropy variables.
  static constexpr int CG = 20 * CL::P::SV + 5 * CL::C::SV + CG_TK + CG_TJ + 32;
  // Volume phase: tK, tJ, Var, dX, dY, dZ (+ the matching-layer source when
  // OPEN). tK and tJ take the CG's padded layouts where that does not enlarge
  // the shared memory of the kernel.
  static constexpr int VOL_DENSE = TK + TJ + 20 * MD + (OPEN ? 5 * MD : 0);
  static constexpr int VOL_PAD = CG_TK + CG_TJ + 20 * MD + (OPEN ? 5 * MD : 0);
  static constexpr int OTHER = FACE > CG ? FACE : CG;
  static constexpr bool PADVOL = VOL_PAD <= (VOL_DENSE > OTHER ? VOL_DENSE : OTHER);
  static constexpr int VOL = PADVOL ? VOL_PAD : VOL_DENSE;
  static constexpr int VTK = PADVOL ? CG_TK : TK, VTJ = PADVOL ? CG_TJ : TJ;
  using VA = std::conditional_t<PADVOL, typename CL::A, Dense<K, K, M>>;
  using VB = std::conditional_t<PADVOL, typename CL::B, Dense<K, M, M>>;
  using VD = std::conditional_t<PADVOL, typename CL::D, Dense<M, M, K>>;
  using VE = std::conditional_t<PADVOL, typename CL::E, Dense<M, K, K>>;
  // Threads per CTA and CTAs per SM (through __launch_bounds__ they bound the
  // registers per thread). FP64: 128 threads cover the widest contraction stage
  // of degrees <= 3 in one or two passes; from degree 4 on 256 threads (degree
  // 4 at 2 CTAs of 256 against 2 of 128: ResidualKernel 1.59 -> 1.41 ms on the
  // 40x20x20 pulse, 21.2 -> 20.5 ms on TGV 48^3, measured on B200). FP32: 256
  // threads from degree 4 up. As many CTAs as the shared memory allows, up to
  // the VCPG_CAP_RES_* bounds.
  static constexpr bool FP64 = sizeof(T) == 8;
  static constexpr int NT = K <= 4 ? 128 : 256;
  static constexpr int CAP =
      FP64 ? (K <= 3 ? VCPG_CAP_RES_FP64_SMALL : VCPG_CAP_RES_FP64)
           : (NT == 256 ? VCPG_CAP_RES_FP32_256
                        : (K == 4 ? VCPG_CAP_RES_FP32_K4 : VCPG_CAP_RES_FP32_SMALL));
  // Persistent: sol, R, CG point data (rho, u, v, w, p per point), J*w, reduction scratch,
  // face vectors (basis and derivative at r = -1, +1).
  // Face vectors: basis and derivative at r = -1, +1 (4 K values, room for 28 at least).
  static constexpr int FV = 4 * (K > 7 ? K : 7);
  // Reduction scratch: two areas of 3 values per warp of up to 512 threads.
  static constexpr int RED = 96;
  static constexpr int PERSIST = 10 * KD + 6 * MD + RED + FV;
  // The work area: the largest phase, widened to hold the volume metric (10 M^3
  // FP64 values) after the volume phase's arrays for VolumeMetricPrefetch where
  // that keeps the CTAs per SM (228 KB per SM, 1 KB reserved per CTA).
  static constexpr int WORK0 = VOL > OTHER ? VOL : OTHER;
  static constexpr int A16 = 16 / (int)sizeof(T);   // values per 16 bytes
  static constexpr int VPF_OFF = ((PERSIST + VOL + A16 - 1) / A16) * A16 - PERSIST;
  static constexpr int VPF = VPF_OFF + (int)(80 * (size_t)MD / sizeof(T));
  static constexpr size_t B0 = sizeof(T) * (size_t)(PERSIST + WORK0);
  static constexpr size_t B1 = sizeof(T) * (size_t)(PERSIST + VPF);
  static constexpr int F0 = (int)(233472 / (B0 + 1024)), F1 = (int)(233472 / (B1 + 1024));
  static constexpr int L0 = F0 < CAP ? F0 : CAP, L1 = F1 < CAP ? F1 : CAP;
  static constexpr bool WIDEN = VPF > WORK0 && L1 >= 1 && L1 >= L0 && B1 <= 227 * 1024;
  static constexpr int WORK = WIDEN ? VPF : WORK0;
  static constexpr int TOTAL = PERSIST + WORK;
  static constexpr size_t BYTES = sizeof(T) * (size_t)TOTAL;
  // Above the 227 KB of one CTA (degrees 7-9 in FP64): the arrays live in a
  // global scratch area per CTA (stride SCRATCH, 16-byte aligned) of a grid that
  // loops over the elements.
  static constexpr bool BIG = BYTES > 227 * 1024;
  static constexpr int SCRATCH = (TOTAL + 3) / 4 * 4;
  static constexpr int FIT = (int)(227 * 1024 / BYTES);
  static constexpr int MIN_BLOCKS = FIT < 1 ? 1 : (FIT > CAP ? CAP : FIT);
};


template <int K, int M, typename T, bool OPEN> struct FusedUpdatePrefetch {
  using PK = Plan<K, M, T, OPEN>;
  static constexpr int KD = K * K * K;
  static constexpr int OFF = (Plan<K, M, T>::CG + 1) / 2 * 2;   // in T, 8-byte aligned
  static constexpr bool value =
      !PK::BIG && (long)(PK::WORK - OFF) * (long)sizeof(T) >=
                      (sizeof(T) == 4 ? 2L : 1L) * 5 * KD * 8;
};

// ---------------------------------------------------------------------------
// Characteristic matching layer source of one integration point
// (src/ElementClass.cpp:3885-4108): the incoming-wave LODI amplitudes of each
// direction, weighted by -J w sigma_d / sigma_max, written to bufC[5][M^3].
// V: entropy variables; gx, gy, gz: their Cartesian gradients.
// ---------------------------------------------------------------------------
template <int M, typename T>
__device__ __forceinline__ void MatchingLayerSource(const ResidualArgs &a, const int sp,
                                                    const int l, const T *V, const T *gx,
                                                    const T *gy, const T *gz, const T rho,
                                                    const T u, const T v, const T w, const T p,
                                                    const T ek, const T rE, const T weight,
                                                    T *bufC) {
  constexpr int MD = M * M * M;
  const double *fn = a.damp_fn + (size_t)sp * 3 * MD;
  const double *cm = a.cml + (size_t)sp * 6;
  const T gm1 = T(kGam) - T(1.0), ovgm1 = T(1.0) / gm1;
  const T wx = weight * T(cm[0]) * LdT<T>(fn + l);
  const T wy = weight * T(cm[1]) * LdT<T>(fn + MD + l);
  const T wz = weight * T(cm[2]) * LdT<T>(fn + 2 * MD + l);
  const T nx = T(cm[3]), ny = T(cm[4]), nz = T(cm[5]);
  const T V4Inv = T(1.0) / V[4];
  const T H = rE / rho - V4Inv;
  const T a2 = -T(kGam) * V4Inv;
  const T c = Sqrt(a2);
  const T rhoa = rho * c, ovra = T(1.0) / rhoa, ova2 = T(1.0) / a2, rova = rho / c;
  const T rhou = rho * u, rhov = rho * v, rhow = rho * w;
  // Jacobian entropy -> primitive (rows rho, u, v, w, p).
  const T J11 = rho, J12 = rhou, J13 = rhov, J14 = rhow, J15 = rE;
  const T J22 = -V4Inv, J25 = -V4Inv * u, J33 = -V4Inv, J35 = -V4Inv * v;
  const T J44 = -V4Inv, J45 = -V4Inv * w;
  const T J51 = p, J52 = p * u, J53 = p * v, J54 = p * w, J55 = p * H;
  T dq[3][5];
  const T *g[3] = {gx, gy, gz};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const T *x = g[q];
    dq[q][0] = J11 * x[0] + J12 * x[1] + J13 * x[2] + J14 * x[3] + J15 * x[4];
    dq[q][1] = J22 * x[1] + J25 * x[4];
    dq[q][2] = J33 * x[2] + J35 * x[4];
    dq[q][3] = J44 * x[3] + J45 * x[4];
    dq[q][4] = J51 * x[0] + J52 * x[1] + J53 * x[2] + J54 * x[3] + J55 * x[4];
  }
  // Eigenvalues with the outgoing ones removed.
  const T vel[3] = {u, v, w}, dir[3] = {nx, ny, nz};
  T l1[3], l2[3], l3[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    l1[q] = vel[q] - c; l2[q] = vel[q]; l3[q] = vel[q] + c;
    if (dir[q] * l1[q] > T(0.0)) l1[q] = T(0.0);
    if (dir[q] * l2[q] > T(0.0)) l2[q] = T(0.0);
    if (dir[q] * l3[q] > T(0.0)) l3[q] = T(0.0);
  }
  // Wave amplitudes and P = S L per direction.
  const T Lx1 = T(0.5) * l1[0] * (ovra * dq[0][4] - dq[0][1]);
  const T Lx2 = l2[0] * (dq[0][0] - ova2 * dq[0][4]);
  const T Lx3 = l2[0] * (dq[0][3]);
  const T Lx4 = l2[0] * (-dq[0][2]);
  const T Lx5 = T(0.5) * l3[0] * (ovra * dq[0][4] + dq[0][1]);
  const T Ly1 = T(0.5) * l1[1] * (ovra * dq[1][4] - dq[1][2]);
  const T Ly2 = l2[1] * (-dq[1][3]);
  const T Ly3 = l2[1] * (dq[1][0] - ova2 * dq[1][4]);
  const T Ly4 = l2[1] * (dq[1][1]);
  const T Ly5 = T(0.5) * l3[1] * (ovra * dq[1][4] + dq[1][2]);
  const T Lz1 = T(0.5) * l1[2] * (ovra * dq[2][4] - dq[2][3]);
  const T Lz2 = l2[2] * (dq[2][2]);
  const T Lz3 = l2[2] * (-dq[2][1]);
  const T Lz4 = l2[2] * (dq[2][0] - ova2 * dq[2][4]);
  const T Lz5 = T(0.5) * l3[2] * (ovra * dq[2][4] + dq[2][3]);
  const T Lx51 = Lx5 + Lx1, Ly51 = Ly5 + Ly1, Lz51 = Lz5 + Lz1;
  const T P[3][5] = {{rova * (Lx51) + Lx2, (Lx5 - Lx1), -Lx4, Lx3, rhoa * (Lx51)},
                     {rova * (Ly51) + Ly3, Ly4, (Ly5 - Ly1), -Ly2, rhoa * (Ly51)},
                     {rova * (Lz51) + Lz4, -Lz3, Lz2, (Lz5 - Lz1), rhoa * (Lz51)}};
  const T wd[3] = {wx, wy, wz};
  T out[5];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const T *P_ = P[q];
    const T t0 = wd[q] * (P_[0]);
    const T t1 = wd[q] * (u * P_[0] + rho * P_[1]);
    const T t2 = wd[q] * (v * P_[0] + rho * P_[2]);
    const T t3 = wd[q] * (w * P_[0] + rho * P_[3]);
    const T t4 = wd[q] * (ek * P_[0] + rhou * P_[1] + rhov * P_[2] + rhow * P_[3] + ovgm1 * P_[4]);
    if (q == 0) { out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3; out[4] = t4; }
    else { out[0] += t0; out[1] += t1; out[2] += t2; out[3] += t3; out[4] += t4; }
  }
#pragma unroll
  for (int n = 0; n < 5; ++n) bufC[n * MD + l] = out[n];
}

// The element's volume metric (10 M^3 doubles) is fetched asynchronously into
// the part of the work area above the volume phase's arrays, while the
// interpolation contractions run, where it fits that space (FP64 up to degree 3).
template <int K, int M, typename T, bool OPEN> struct VolumeMetricPrefetch {
  using P = Plan<K, M, T, OPEN>;
  // In T from the work area, 16-byte aligned in shared memory (the work area
  // starts PERSIST values after the 16-byte aligned base).
  static constexpr int OFF = P::VPF_OFF;
  static constexpr unsigned BYTES = 80u * M * M * M;   // 10 M^3 FP64 values
  static constexpr bool value =
      !P::BIG && (long)(P::WORK - OFF) * (long)sizeof(T) >= (long)BYTES;
};

// ---------------------------------------------------------------------------
// Volume phase: solution and gradients at the integration points
// (TPSAGV), pointwise fluxes, and the three transposed contractions (TPAVR)
// into s_R. Also stores the CG point data (rho, u, v, w, p)
// and J*w.  Follows ElementClass::VolumeResidual, src/ElementClass.cpp:3809-4443.
// ---------------------------------------------------------------------------
// vms: the element's volume metric staged in shared memory (VolumeMetricPrefetch),
// or null to read it from global memory.
template <int NT, int K, int M, typename T, bool OPEN>
__device__ __forceinline__ void VolumePhase(const ResidualArgs &a, const int e, const double mu,
                                            const T *s_sol, T *s_R, T *s_cgp,
                                            T *s_jw, T *work, T *s_red, const double *vms,
                                            unsigned long long *bar) {
  constexpr int SLOT = Slot<K, M>::value;
  using P = Plan<K, M, T, OPEN>;
  constexpr int MD = P::MD, KD = P::KD, M2 = P::M2;
  T *tK = work, *tJ = work + P::VTK, *Var = tJ + P::VTJ;
  T *dX = Var + 5 * MD, *dY = dX + 5 * MD, *dZ = dY + 5 * MD;
  T *bufC = dZ + 5 * MD;  // matching-layer source (OPEN only)
  const int sp = OPEN ? a.sponge_idx[e] : -1;
  const bool cmlHere = OPEN && sp >= 0 && a.cml_on;

  // TPSAGV (include/TensorProductSolAndGradVolume.hpp:5-249): k, then j, then i.
  ContractL<NT, SLOT, K, M, kLeg, 2, 5, K, K, K, K, M, false, T, Dense<K, K, K>, typename P::VA>(s_sol, tK);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false, T, typename P::VA, typename P::VB>(tK, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false, T, typename P::VB, Dense<M, M, M>>(tJ, Var);
  ContractL<NT, SLOT, K, M, kDLeg, 0, 5, K, M, M, K, M, false, T, typename P::VB, Dense<M, M, M>>(tJ, dX);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kDLeg, 1, 5, K, K, M, K, M, false, T, typename P::VA, typename P::VB>(tK, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false, T, typename P::VB, Dense<M, M, M>>(tJ, dY);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kDLeg, 2, 5, K, K, K, K, M, false, T, Dense<K, K, K>, typename P::VA>(s_sol, tK);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false, T, typename P::VA, typename P::VB>(tK, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLeg, 0, 5, K, M, M, K, M, false, T, typename P::VB, Dense<M, M, M>>(tJ, dZ);
  for (int i = threadIdx.x; i < 5 * KD; i += NT) s_R[i] = T(0.0);
  if constexpr (VolumeMetricPrefetch<K, M, T, OPEN>::value) {
    // A wait that runs out is recorded and followed by one more bounded wait for
    // the copy, which must not land after the work area is reused.
    if (!BulkWait(bar)) {
      if (threadIdx.x == 0) atomicAdd(a.status + 3, 1);
      BulkWait(bar);
    }
  }
  __syncthreads();

  const double *vm = a.vol_metric + (size_t)e * 10 * MD;
  constexpr bool kVPref = VolumeMetricPrefetch<K, M, T, OPEN>::value;
  auto Vm = [&](const int i) -> T {
    if constexpr (kVPref) return T(vms[i]);
    else return LdT<T>(vm + i);
  };
  const T gm1 = T(kGam) - T(1.0), ov1mg = -T(1.0) / gm1;
  T mach2 = T(0.0), eddyMax = T(0.0);
  for (int l = threadIdx.x; l < MD; l += NT) {
    const int i = l % M, j = (l / M) % M, k = l / M2;
    // Parametric -> Cartesian gradients (src/ElementClass.cpp:3856-3875). In the
    // compatibility mode the metric of point n is used for variable n.
    T V[5], gx[5], gy[5], gz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      const int mi = a.metric_compat ? n : l;
      const T dvdr = dX[n * MD + l], dvds = dY[n * MD + l], dvdt = dZ[n * MD + l];
      gx[n] = dvdr * Vm(1 * MD + mi) + dvds * Vm(4 * MD + mi) +
              dvdt * Vm(7 * MD + mi);
      gy[n] = dvdr * Vm(2 * MD + mi) + dvds * Vm(5 * MD + mi) +
              dvdt * Vm(8 * MD + mi);
      gz[n] = dvdr * Vm(3 * MD + mi) + dvds * Vm(6 * MD + mi) +
              dvdt * Vm(9 * MD + mi);
      V[n] = Var[n * MD + l];
    }
    // Entropy -> primitive variables, velocity and internal-energy gradients
    // (src/ElementClass.cpp:4183-4257).
    T rho, u, v, w, p, eKin;
    EntropyToPrim(V[0], V[1], V[2], V[3], V[4], rho, u, v, w, p, eKin);
    const T V4Inv = T(1.0) / V[4];
    const T rE = -p * ov1mg + rho * eKin;
    const T dudx = -V4Inv * (gx[1] + u * gx[4]), dudy = -V4Inv * (gy[1] + u * gy[4]),
                 dudz = -V4Inv * (gz[1] + u * gz[4]);
    const T dvdx = -V4Inv * (gx[2] + v * gx[4]), dvdy = -V4Inv * (gy[2] + v * gy[4]),
                 dvdz = -V4Inv * (gz[2] + v * gz[4]);
    const T dwdx = -V4Inv * (gx[3] + w * gx[4]), dwdy = -V4Inv * (gy[3] + w * gy[4]),
                 dwdz = -V4Inv * (gz[3] + w * gz[4]);
    const T fact = -V4Inv * V4Inv * ov1mg;
    const T dedx = gx[4] * fact, dedy = gy[4] * fact, dedz = gz[4] * fact;
    const T rH = rE + p;
    s_cgp[0 * MD + l] = rho;
    s_cgp[1 * MD + l] = u;
    s_cgp[2 * MD + l] = v;
    s_cgp[3 * MD + l] = w;
    s_cgp[4 * MD + l] = p;
    mach2 = Fmax(mach2, rho * (u * u + v * v + w * w) / (T(kGam) * p));
    if (OPEN && cmlHere)
      MatchingLayerSource<M>(a, sp, l, V, gx, gy, gz, rho, u, v, w, p, eKin, rE,
                             -Vm(l) * Weight1D<SLOT, T>(i) * Weight1D<SLOT, T>(j) *
                                 Weight1D<SLOT, T>(k),
                             bufC);

    // Inviscid + viscous fluxes times -J w and the metric (src/ElementClass.cpp:4320-4416).
    const T Wl = Weight1D<SLOT, T>(i) * Weight1D<SLOT, T>(j) * Weight1D<SLOT, T>(k);
    const T Jl = Vm(l);
    s_jw[l] = Wl * Jl;
    const T weight = -Jl * Wl;
    const T ru = rho * u, rv = rho * v, rw = rho * w;
    T eddy = T(0.0);
    if (a.sgs) {
      // Eddy viscosity at the point (src/ElementClass.cpp:4272-4310).
      const T gv[9] = {dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz};
      eddy = EddyViscosity(a.sgs, T(a.elem_scalars[(size_t)e * 15 + 3]), rho, gv);
      eddyMax = Fmax(eddyMax, eddy);
    }
    const T muTot = T(mu) + eddy;
    const T factHeatFluxTot = T(mu) * T(kFactHFLam) + eddy * T(kFactHFTurb);
    const T divVelTerm = T(kLamOverMu) * (dudx + dvdy + dwdz);
    const T tauxx = muTot * (T(2.0) * dudx + divVelTerm);
    const T tauyy = muTot * (T(2.0) * dvdy + divVelTerm);
    const T tauzz = muTot * (T(2.0) * dwdz + divVelTerm);
    const T tauxy = muTot * (dudy + dvdx);
    const T tauxz = muTot * (dudz + dwdx);
    const T tauyz = muTot * (dvdz + dwdy);
    const T qx = -factHeatFluxTot * dedx, qy = -factHeatFluxTot * dedy,
                 qz = -factHeatFluxTot * dedz;
    const T fx[5] = {ru, ru * u - tauxx + p, rv * u - tauxy, rw * u - tauxz,
                          (rE + p) * u - (u * tauxx + v * tauxy + w * tauxz - qx)};
    const T fy[5] = {rv, ru * v - tauxy, rv * v - tauyy + p, rw * v - tauyz,
                          (rE + p) * v - (u * tauxy + v * tauyy + w * tauyz - qy)};
    const T fz[5] = {rw, ru * w - tauxz, rv * w - tauyz, rw * w - tauzz + p,
                          (rE + p) * w - (u * tauxz + v * tauyz + w * tauzz - qz)};
    const T drdx = weight * Vm(1 * MD + l), drdy = weight * Vm(2 * MD + l),
                 drdz = weight * Vm(3 * MD + l);
    const T dsdx = weight * Vm(4 * MD + l), dsdy = weight * Vm(5 * MD + l),
                 dsdz = weight * Vm(6 * MD + l);
    const T dtdx = weight * Vm(7 * MD + l), dtdy = weight * Vm(8 * MD + l),
                 dtdz = weight * Vm(9 * MD + l);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      dX[n * MD + l] = fx[n] * drdx + fy[n] * drdy + fz[n] * drdz;
      dY[n * MD + l] = fx[n] * dsdx + fy[n] * dsdy + fz[n] * dsdz;
      dZ[n * MD + l] = fx[n] * dtdx + fy[n] * dtdy + fz[n] * dtdz;
    }
  }
  if (a.mach2max) {
    const T m = BlockMax<NT>(mach2, s_red);
    if (threadIdx.x == 0) atomicMax(a.mach2max, (unsigned long long)__double_as_longlong((double)m));
  }
  if (a.sgs && a.eddymax) {
    const T m = BlockMax<NT>(eddyMax, s_red);
    if (threadIdx.x == 0) atomicMax(a.eddymax, (unsigned long long)__double_as_longlong((double)m));
  }
  __syncthreads();

  // The matching-layer source initialises the residual (src/ElementClass.cpp:3885-4117).
  if (OPEN && cmlHere) {
    ContractL<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(bufC, tJ);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R);
    __syncthreads();
  }
  // TPAVR for the three flux directions (src/ElementClass.cpp:4425-4443).
  ContractL<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(dX, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kDLegT, 0, 5, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(dY, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kDLegT, 1, 5, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kDLegT, 2, 5, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(dZ, tJ);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
  __syncthreads();
  ContractL<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R);
  __syncthreads();
  // Sponge-layer damping J w sum_d sigma_d (U - U_damp) (src/ElementClass.cpp:4450-4489).
  if (OPEN && sp >= 0) {
    const double *fn = a.damp_fn + (size_t)sp * 3 * MD;
    const double *ds = a.damp_state + (size_t)sp * 5 * MD;
    for (int l = threadIdx.x; l < MD; l += NT) {
      const T sigma = s_jw[l] * (LdT<T>(fn + l) + LdT<T>(fn + MD + l) + LdT<T>(fn + 2 * MD + l));
      const T rho = s_cgp[0 * MD + l];
      dX[0 * MD + l] = sigma * (rho - LdT<T>(ds + 0 * MD + l));
      dX[1 * MD + l] = sigma * (rho * s_cgp[1 * MD + l] - LdT<T>(ds + 1 * MD + l));
      dX[2 * MD + l] = sigma * (rho * s_cgp[2 * MD + l] - LdT<T>(ds + 2 * MD + l));
      dX[3 * MD + l] = sigma * (rho * s_cgp[3 * MD + l] - LdT<T>(ds + 3 * MD + l));
      const T u = s_cgp[1 * MD + l], v = s_cgp[2 * MD + l], w = s_cgp[3 * MD + l];
      const T rE = -s_cgp[4 * MD + l] * (-T(1.0) / (T(kGam) - T(1.0))) +
                   rho * (T(0.5) * (u * u + v * v + w * w));
      dX[4 * MD + l] = sigma * (rE - LdT<T>(ds + 4 * MD + l));
    }
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(dX, tJ);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 0, 5, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R);
    __syncthreads();
  }
  // Body force per unit volume (src/ElementClass.cpp:4495-4533): the source
  // -J w (f, u . f) on the momentum and energy residuals.
  if (a.body_force) {
    const T fx = T(a.fbody[0]), fy = T(a.fbody[1]), fz = T(a.fbody[2]);
    for (int l = threadIdx.x; l < MD; l += NT) {
      const T weight = -s_jw[l];
      const T u = s_cgp[1 * MD + l], v = s_cgp[2 * MD + l], w = s_cgp[3 * MD + l];
      dX[0 * MD + l] = weight * fx;
      dX[1 * MD + l] = weight * fy;
      dX[2 * MD + l] = weight * fz;
      dX[3 * MD + l] = weight * (u * fx + v * fy + w * fz);
    }
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 2, 4, M, M, M, M, K, false, T, Dense<M, M, M>, typename P::VD>(dX, tJ);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 1, 4, M, M, K, M, K, false, T, typename P::VD, typename P::VE>(tJ, tK);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 0, 4, M, K, K, M, K, true, T, typename P::VE, Dense<K, K, K>>(tK, s_R + KD);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Face phase. The faces are processed in two groups -- the Min faces of the
// three directions, then the Max faces -- and every stage of a group runs over
// all three faces and both sides of each face at once, so a group needs three
// barriers for its six traces and three for its distributions.
//
// Trace t = 2 d + s: face direction d (0 i, 1 j, 2 k), s = 0 own side, s = 1
// neighbour side. Face arrays are [slow][fast] with (slow, fast) = (k, j), (k, i),
// (j, i) for d = 0, 1, 2, as in the reference's TPSAG[IJK] outputs. Trace
// storage TR[q][t][v][M^2]: q = 0 value, 1 face-normal derivative, 2 fast-axis
// derivative, 3 slow-axis derivative.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int FastParam(const int d) { return d == 0 ? 1 : 0; }

// Trace quantity q holding parametric derivative p (0 r, 1 s, 2 t) for direction d.
__device__ __forceinline__ int DerivSlot(const int d, const int p) {
  return p == d ? 1 : (p == FastParam(d) ? 2 : 3);
}

// Face-normal evaluation of the six sides of a group (first stage of TPSAG[IJK]).
// s_nb: the three neighbours' states staged in shared memory ([3][5 K^3], in
// the order of the directions), or null to read them from gsol.
template <int NT, int SLOT, int K, typename T>
__device__ __forceinline__ void FaceNormalBatch(const T *s_sol, const double *gsol,
                                                const double *s_nb,
                                                const int nb0, const int nb1, const int nb2,
                                                const int g, const T *s_fv, T *bn,
                                                T *bnd) {
  constexpr int KD = K * K * K, L = 5 * K * K;
  for (int line = threadIdx.x; line < 6 * L; line += NT) {
    const int t = line / L, r = line - t * L;
    const int d = t >> 1, nbr = (t & 1);
    const int side = nbr ? 1 - g : g;
    const int v = r / (K * K), r2 = r - v * K * K, sl = r2 / K, f = r2 - sl * K;
    int base, ns;
    if (d == 0) { base = sl * K * K + f * K; ns = 1; }
    else if (d == 1) { base = sl * K * K + f; ns = K; }
    else { base = sl * K + f; ns = K * K; }
    base += v * KD;
    const T *fv = s_fv + side * K, *dfv = s_fv + (2 + side) * K;
    T a0 = T(0.0), d0 = T(0.0);
    if (nbr) {
      const int nb = d == 0 ? nb0 : (d == 1 ? nb1 : nb2);
      if (nb >= 0) {
        if (s_nb) {
          const double *b = s_nb + d * 5 * KD + base;
#pragma unroll
          for (int n = 0; n < K; ++n) {
            const T x = T(b[n * ns]);
            a0 = Fma(fv[n], x, a0);
            d0 = Fma(dfv[n], x, d0);
          }
        } else {
          const double *b = gsol + (size_t)nb * 5 * KD + base;
#pragma unroll
          for (int n = 0; n < K; ++n) {
            const T x = LdT<T>(b + n * ns);
            a0 = Fma(fv[n], x, a0);
            d0 = Fma(dfv[n], x, d0);
          }
        }
      }
    } else {
      const T *b = s_sol + base;
#pragma unroll
      for (int n = 0; n < K; ++n) {
        const T x = b[n * ns];
        a0 = Fma(fv[n], x, a0);
        d0 = Fma(dfv[n], x, d0);
      }
    }
    bn[line] = a0;
    bnd[line] = d0;
  }
}

// Parametric -> Cartesian gradient of one side at face point pt from TR.
template <int M2, typename T>
__device__ __forceinline__ void TraceCartesianGrad(const T *TR, const int t, const int d,
                                                   const int pt, const double *fm,
                                                   const int compat, T *gx, T *gy,
                                                   T *gz) {
  const int qr = DerivSlot(d, 0), qs = DerivSlot(d, 1), qt = DerivSlot(d, 2);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    // With fewer than 5 face points (M = 2) variable 4 reads the padding, which
    // holds point 0's metric (src/ElementClass.cpp:1163-1173).
    const int mi = compat ? (n < M2 ? n : 0) : pt;
    const T dvdr = TR[((qr * 6 + t) * 5 + n) * M2 + pt];
    const T dvds = TR[((qs * 6 + t) * 5 + n) * M2 + pt];
    const T dvdt = TR[((qt * 6 + t) * 5 + n) * M2 + pt];
    gx[n] = dvdr * LdT<T>(fm + 4 * M2 + mi) + dvds * LdT<T>(fm + 7 * M2 + mi) +
            dvdt * LdT<T>(fm + 10 * M2 + mi);
    gy[n] = dvdr * LdT<T>(fm + 5 * M2 + mi) + dvds * LdT<T>(fm + 8 * M2 + mi) +
            dvdt * LdT<T>(fm + 11 * M2 + mi);
    gz[n] = dvdr * LdT<T>(fm + 6 * M2 + mi) + dvds * LdT<T>(fm + 9 * M2 + mi) +
            dvdt * LdT<T>(fm + 12 * M2 + mi);
  }
}

// Fluxes of one interior face point (FluxesInternalFace, src/FluxesFace.cpp:220-343)
// from the traces TR of the face's two sides: tL / tR are the trace slots of the
// lower (left) and upper (right) element, fmL / fmR their face metrics; the
// normal is the left element's. Writes the normal flux and the Cartesian
// symmetrizing fluxes (component 0 of those is zero) to out[20][M^2]:
// 0-4 flux, 5-9 x, 10-14 y, 15-19 z.
template <int K, int M, bool SGS, typename T>
__device__ __forceinline__ void FacePointFlux(const ResidualArgs &a, const double mu, const int d,
                                              const int pt, const T *TR, const int tL,
                                              const int tR, const double *fmL,
                                              const double *fmR, const T lenScale, T *out,
                                              const T lenLES, T &eddy) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int M2 = M * M;
  T VL[5], VR[5], gxL[5], gyL[5], gzL[5], gxR[5], gyR[5], gzR[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    VL[n] = TR[(tL * 5 + n) * M2 + pt];
    VR[n] = TR[(tR * 5 + n) * M2 + pt];
  }
  TraceCartesianGrad<M2>(TR, tL, d, pt, fmL, a.metric_compat, gxL, gyL, gzL);
  TraceCartesianGrad<M2>(TR, tR, d, pt, fmR, a.metric_compat, gxR, gyR, gzR);
  T gx[5], gy[5], gz[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    gx[n] = T(0.5) * (gxL[n] + gxR[n]);
    gy[n] = T(0.5) * (gyL[n] + gyR[n]);
    gz[n] = T(0.5) * (gzL[n] + gzR[n]);
  }
  const int f = pt % M, sl = pt / M;
  const T wf = Weight1D<SLOT, T>(f) * Weight1D<SLOT, T>(sl);
  const T nx = T(1.0) * LdT<T>(fmL + 0 * M2 + pt), ny = T(1.0) * LdT<T>(fmL + 1 * M2 + pt),
               nz = T(1.0) * LdT<T>(fmL + 2 * M2 + pt);
  const T area = LdT<T>(fmL + 3 * M2 + pt);
  T flux[5];
  if (a.riemann == 1)
    IsmailRoeFlux(VL, VR, nx, ny, nz, wf * area, flux);
  else
    RoeFlux(VL, VR, nx, ny, nz, T(0.5) * wf * area, flux);
  T sx[5], sy[5], sz[5];
  ViscousPenaltySymFlux(VL, VR, gx, gy, gz, nx, ny, nz, wf, area, T(mu),
                        T(a.tau_num) / lenScale, T(a.theta_sym), flux, sx, sy, sz, T(1.0),
                        T(0.0), SGS ? a.sgs : 0, lenLES, &eddy);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    out[n * M2 + pt] = flux[n];
    out[(5 + n) * M2 + pt] = sx[n];
    out[(10 + n) * M2 + pt] = sy[n];
    out[(15 + n) * M2 + pt] = sz[n];
  }
}

// Distribution inputs of the six faces (TPR[IJK]F), both sides g = 0 (Min
// faces) and g = 1 (Max faces), grouped by the operators they take; within a
// group [g][d][v][B] (B = M^2 face points, later K^2 after both axes):
//   set 0 (PA, 30 blocks)   fast-axis symmetrizing flux: slow Leg^T, fast DLeg^T
//   set 1 (PB, 30 blocks)   normal flux:                 slow Leg^T, fast Leg^T
//   set 2 (PB, 30 blocks)   face-normal symmetrizing flux (expanded with the
//                           derivative of the face basis)
//   set 3 (PC, 30 blocks)   slow-axis symmetrizing flux: slow DLeg^T, fast Leg^T
// Sets 0-2 are contiguous, so one slow-axis contraction covers them.
template <int B>
__device__ __forceinline__ int RoleIndex(const int set, const int g, const int d, const int v,
                                         const int pt) {
  return ((set * 2 + g) * 15 + d * 5 + v) * B + pt;
}

// The roles of the fluxes F[20][M^2] (FacePointFlux layout) of one face point
// for side g of the element: the normal flux with the own side's sign (the own
// element is the right state of its Min faces) and the symmetrizing fluxes
// turned parametric with the own side's metric fm.
template <int K, int M, typename T>
__device__ __forceinline__ void FaceRoles(const ResidualArgs &a, const int g, const int d,
                                          const int pt, const T *F, const double *fm, T *P) {
  constexpr int M2 = M * M;
  const int pFast = FastParam(d);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    const int mi = a.metric_compat ? (n < M2 ? n : 0) : pt;
    const T flux = F[n * M2 + pt], sx = F[(5 + n) * M2 + pt], sy = F[(10 + n) * M2 + pt],
            sz = F[(15 + n) * M2 + pt];
    T sym[3];
#pragma unroll
    for (int p = 0; p < 3; ++p)
      sym[p] = sx * LdT<T>(fm + (4 + 3 * p) * M2 + mi) + sy * LdT<T>(fm + (5 + 3 * p) * M2 + mi) +
               sz * LdT<T>(fm + (6 + 3 * p) * M2 + mi);
    P[RoleIndex<M2>(0, g, d, n, pt)] = sym[pFast];
    P[RoleIndex<M2>(1, g, d, n, pt)] = g == 0 ? -flux : flux;
    P[RoleIndex<M2>(2, g, d, n, pt)] = sym[d];
    P[RoleIndex<M2>(3, g, d, n, pt)] = sym[3 - d - pFast];
  }
}

// Face fluxes of an element's three Min faces (each interior face is computed
// once, by its upper element): the traces of both sides (TPSAG[IJK]) and the
// pointwise fluxes, into face_flux[e][d][20][M^2]. Boundary faces are skipped
// (their fluxes come from the boundary kernels).
template <int NT, int K, int M, typename T, bool SGS>
__device__ __forceinline__ void MinFaceFluxes(const ResidualArgs &a, const int e, const double mu,
                                              const T *s_sol, const T *s_fv, T *work,
                                              const double *s_nb) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int M2 = M * M, K2 = K * K;
  static_assert(K <= M, "face-flux buffer aliasing");
  T *T1a = work, *T1b = T1a + 30 * K * M, *T1c = T1b + 30 * K * M;  // 90 K M
  T *BN = T1c + 30 * K * M, *BND = BN + 30 * K2;  // 60 K^2
  T *TR = BN;                               // 120 M^2 (BN is dead when TR is written)
  const int nb0 = a.nbr[e * 6 + 0], nb1 = a.nbr[e * 6 + 2], nb2 = a.nbr[e * 6 + 4];
  FaceNormalBatch<NT, SLOT, K>(s_sol, a.sol, s_nb, nb0, nb1, nb2, 0, s_fv, BN, BND);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 0, 30, K, K, 1, K, M, false>(BN, T1a);
  Contract<NT, SLOT, K, M, kDLeg, 0, 30, K, K, 1, K, M, false>(BN, T1b);
  Contract<NT, SLOT, K, M, kLeg, 0, 30, K, K, 1, K, M, false>(BND, T1c);
  __syncthreads();
  Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1a, TR);
  Contract<NT, SLOT, K, M, kDLeg, 1, 30, M, K, 1, K, M, false>(T1a, TR + 3 * 30 * M2);
  Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1b, TR + 2 * 30 * M2);
  Contract<NT, SLOT, K, M, kLeg, 1, 30, M, K, 1, K, M, false>(T1c, TR + 1 * 30 * M2);
  __syncthreads();
  const double *sc = a.elem_scalars + (size_t)e * 15;
  T *out = reinterpret_cast<T *>(a.face_flux) + (size_t)e * 3 * 20 * M2;
  T eddyMax = T(0.0);
  for (int idx = threadIdx.x; idx < 3 * M2; idx += NT) {
    const int d = idx / M2, pt = idx - d * M2;
    const int nb = d == 0 ? nb0 : (d == 1 ? nb1 : nb2);
    if (nb < 0) continue;
    const T lenScale = Fmin(T(sc[d]), T(a.elem_scalars[(size_t)nb * 15 + d]));
    // LES length of the face: the mean of both elements' (src/ElementClass.cpp:2655).
    const T lenLES = T(0.5) * (T(sc[3]) + T(a.elem_scalars[(size_t)nb * 15 + 3]));
    const double *fmOwn = a.face_metric + ((size_t)e * 6 + 2 * d) * 13 * M2;
    const double *fmNb = a.face_metric + ((size_t)nb * 6 + 2 * d + 1) * 13 * M2;
    // The lower element (the neighbour, trace slot 2d+1) is the left state.
    T eddy = T(0.0);
    FacePointFlux<K, M, SGS>(a, mu, d, pt, TR, 2 * d + 1, 2 * d, fmNb, fmOwn, lenScale,
                        out + d * 20 * M2, lenLES, eddy);
    eddyMax = Fmax(eddyMax, eddy);
  }
  if (SGS && a.eddymax) {
    // Largest eddy viscosity of the faces for the monitoring data.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) eddyMax = Fmax(eddyMax, __shfl_xor_sync(0xffffffffu, eddyMax, o));
    if ((threadIdx.x & 31) == 0 && eddyMax > T(0.0))
      atomicMax(a.eddymax, (unsigned long long)__double_as_longlong((double)eddyMax));
  }
}

template <int NT, int K, int M, typename T, bool OPEN>
__device__ __forceinline__ void FacePhase(const ResidualArgs &a, const int e, T *s_R,
                                          const T *s_fv, T *work) {
  constexpr int SLOT = Slot<K, M>::value;
  constexpr int KD = K * K * K, M2 = M * M, K2 = K * K;
  // P [120 M^2] (RoleIndex order), Q [120 K M] after the slow axis, R [120 K^2]
  // after the fast axis in P's place.
  static_assert(K <= M, "face-phase buffer aliasing");
  T *P = work, *Q = work + 120 * M2, *R = work;
  const T *faceFlux = reinterpret_cast<const T *>(a.face_flux);
  for (int idx = threadIdx.x; idx < 6 * M2; idx += NT) {
    const int f = idx / M2, pt = idx - f * M2;
    const int g = f / 3, d = f - 3 * g;
    const int nb = a.nbr[e * 6 + 2 * d + g];
    if (OPEN && nb <= -2) {
      // Characteristic boundary face: fluxes from BoundaryFluxKernel (FP64),
      // roles [0] fast-axis sym, [1] flux, [2] normal sym, [3] slow-axis sym.
      const double *bf = a.bflux + (size_t)(-2 - nb) * 4 * 5 * M2;
#pragma unroll
      for (int n = 0; n < 5; ++n)
#pragma unroll
        for (int set = 0; set < 4; ++set)
          P[RoleIndex<M2>(set, g, d, n, pt)] = T(bf[(set * 5 + n) * M2 + pt]);
      continue;
    }
    if (nb < 0) {
      // A physical boundary face without a boundary condition.
      if (pt == 0) atomicAdd(a.status + 1, 1);
      for (int n = 0; n < 5; ++n)
        for (int set = 0; set < 4; ++set) P[RoleIndex<M2>(set, g, d, n, pt)] = T(0.0);
      continue;
    }
    // The face's fluxes were computed by its upper element: this element for
    // its Min faces, the neighbour for this element's Max faces.
    const int upper = g == 0 ? e : nb;
    const T *F = faceFlux + ((size_t)upper * 3 + d) * 20 * M2;
    const double *fmOwn = a.face_metric + ((size_t)e * 6 + 2 * d + g) * 13 * M2;
    FaceRoles<K, M>(a, g, d, pt, F, fmOwn, P);
  }
  __syncthreads();
  // Slow axis, fast axis, then the face-normal expansion.
  Contract<NT, SLOT, K, M, kLegT, 1, 90, M, M, 1, M, K, false>(P, Q);
  Contract<NT, SLOT, K, M, kDLegT, 1, 30, M, M, 1, M, K, false>(P + 90 * M2, Q + 90 * K * M);
  __syncthreads();
  Contract<NT, SLOT, K, M, kDLegT, 0, 30, M, K, 1, M, K, false>(Q, R);
  Contract<NT, SLOT, K, M, kLegT, 0, 90, M, K, 1, M, K, false>(Q + 30 * K * M, R + 30 * K2);
  __syncthreads();
  for (int idx = threadIdx.x; idx < 5 * KD; idx += NT) {
    const int v = idx / KD, r = idx - v * KD;
    const int k = r / K2, r2 = r - k * K2, j = r2 / K, i = r2 - j * K;
    T acc = s_R[idx];
    // Reference order: the own Min faces (i, j, k) accumulate onto the volume
    // term; each Max face's contribution is summed from zero and added.
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const T *fv = s_fv + g * K, *dfv = s_fv + (2 + g) * K;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int n = d == 0 ? i : (d == 1 ? j : k);
        const int sf = d == 0 ? k * K + j : (d == 1 ? k * K + i : j * K + i);
        const T aF = fv[n], aD = dfv[n];
        const T tFast = R[RoleIndex<K2>(0, g, d, v, sf)], tFlux = R[RoleIndex<K2>(1, g, d, v, sf)],
                tN = R[RoleIndex<K2>(2, g, d, v, sf)], tSlow = R[RoleIndex<K2>(3, g, d, v, sf)];
        // Normal flux, then the r, s, t symmetrizing fluxes.
        const int pFast = FastParam(d);
        T c = g == 0 ? acc : T(0.0);
        c = Fma(aF, tFlux, c);
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          if (p == d) c = Fma(aD, tN, c);
          else if (p == pFast) c = Fma(aF, tFast, c);
          else c = Fma(aF, tSlow, c);
        }
        acc = g == 0 ? c : acc + c;
      }
    }
    s_R[idx] = acc;
  }
  __syncthreads();
}

// The first and the last transform of the mass-matrix operator, with the work
// that shares their loads: p = beta p + z before the forward k transform (from
// the second iteration on), and the partial sum of p . Ap after the backward
// i transform. Lines, summation order and coefficients are those of
// ContractL<..., AX = 2, ...> and ContractL<..., AX = 0, ...>; LP is the layout
// of the DOF vectors, LO / LI of the transformed arrays.
template <int NT, int SLOT, int K, int M, typename T, typename LP, typename LO>
__device__ __forceinline__ void KForwardUpdate(T *__restrict__ p, const T *__restrict__ z,
                                               const T beta, const bool update,
                                               T *__restrict__ out) {
  constexpr int K2 = K * K, NLINES = 5 * K2;
  for (int line = threadIdx.x; line < NLINES; line += NT) {
    const int v = line / K2, r = line - v * K2;
    const int j = r / K, i = r - j * K;
    const int ib = v * LP::SV + j * LP::S1 + i, ob = v * LO::SV + j * LO::S1 + i;
    T xv[K];
#pragma unroll
    for (int c = 0; c < K; ++c) xv[c] = p[ib + c * LP::S2];
    if (update) {
#pragma unroll
      for (int c = 0; c < K; ++c) {
        xv[c] = Fma(beta, xv[c], z[ib + c * LP::S2]);
        p[ib + c * LP::S2] = xv[c];
      }
    }
#pragma unroll
    for (int o = 0; o < M; ++o) {
      T acc = T(0);
#pragma unroll
      for (int c = 0; c < K; ++c) acc = fma(Coef<SLOT, K, M, kLeg, T>(c, o), xv[c], acc);
      out[ob + o * LO::S2] = acc;
    }
  }
}

template <int NT, int SLOT, int K, int M, typename T, typename LI, typename LP, bool DOT = true>
__device__ __forceinline__ T IBackwardDot(const T *__restrict__ in, const T *__restrict__ p,
                                          T *__restrict__ Ap) {
  constexpr int K2 = K * K, NLINES = 5 * K2;
  T part = T(0);
  for (int line = threadIdx.x; line < NLINES; line += NT) {
    const int v = line / K2, r = line - v * K2;
    const int kk = r / K, kj = r - kk * K;
    const int ib = v * LI::SV + kk * LI::S2 + kj * LI::S1;
    const int ob = v * LP::SV + kk * LP::S2 + kj * LP::S1;
    T xv[M];
#pragma unroll
    for (int c = 0; c < M; ++c) xv[c] = in[ib + c];
#pragma unroll
    for (int o = 0; o < K; ++o) {
      T acc = T(0);
#pragma unroll
      for (int c = 0; c < M; ++c) acc = fma(Coef<SLOT, K, M, kLegT, T>(c, o), xv[c], acc);
      Ap[ob + o] = acc;
      if constexpr (DOT) part = Fma(p[ob + o], acc, part);
    }
  }
  return part;
}

// w J dU/dV at one integration point from the stored point data (rho, u, v, w, p)
// (src/CG_MassMatrix.cpp:408-443 with dU/dV as in the volume phase): d[0..14] the
// symmetric 5x5 matrix by rows of its upper triangle, d[15] = w J.
template <int MD, typename T>
__device__ __forceinline__ void PointOperator(const T *s_cgp, const T *s_jw, const int l, T d[16]) {
  const T rho = s_cgp[l], u = s_cgp[MD + l], v = s_cgp[2 * MD + l], w = s_cgp[3 * MD + l],
          pr = s_cgp[4 * MD + l];
  const T eKin = T(0.5) * (u * u + v * v + w * w);
  const T rE = -pr * (-T(1.0) / (T(kGam) - T(1.0))) + rho * eKin;
  const T ru = rho * u, rv = rho * v, rw = rho * w, rH = rE + pr;
  d[0] = rho; d[1] = ru; d[2] = rv; d[3] = rw; d[4] = rE;
  d[5] = ru * u + pr; d[6] = ru * v; d[7] = ru * w; d[8] = rH * u;
  d[9] = rv * v + pr; d[10] = rv * w; d[11] = rH * v;
  d[12] = rw * w + pr; d[13] = rH * w;
  d[14] = rE * rH / rho + pr * eKin;
  d[15] = s_jw[l];
}

// ---------------------------------------------------------------------------
// Generalised mass-matrix solve, CG_EntropyVarMassMatrix
// (src/CG_MassMatrix.cpp:250-504): flexible PCG with the element-centre
// dV/dU * 8/vol preconditioner, stop at ||r||_inf < 1e-10 ||r0||_inf, at most
// 100 iterations (the cap raises a status flag instead of aborting).
// r is s_R (dense, overwritten); the solution goes through StoreResidual (the
// residual array, or the fused Runge-Kutta stage update of the element).
//
// One iteration is seven barrier-separated steps: k, j transforms to the
// integration points (the first with the search-direction update), the
// i transform fused with the point operator (one thread per point, its
// w J dU/dV kept in registers where the register budget allows),
// k, j, i transforms back (the last with the partial sums of p . Ap), and the
// update of x, r and z with the three sums that close the iteration. The two
// reductions use one barrier each and alternate their scratch areas. The CG
// arrays use the padded layouts of CgLayout. The update is DOF-local.
// Where every thread owns at most one DOF (K^3 <= threads) the iteration has
// nine steps: the owner keeps x, r and the search direction p in registers,
// forms p = z + beta p itself and stores it for the forward transforms (one more
// barrier), and forms the partial sums of p . Ap from its registers after the
// backward i transform (one more barrier); z then never passes through shared
// memory and the first and last transforms read only their lines.
// ---------------------------------------------------------------------------
template <int NT, int K, int M, typename T, bool OPEN>
__device__ __forceinline__ void MassSolve(const ResidualArgs &a, const int e, const T *s_sol,
                                          T *s_R, const T *s_cgp, const T *s_jw,
                                          T *work, T *s_red) {
  constexpr int SLOT = Slot<K, M>::value;
  using P = Plan<K, M, T>;
  using L = typename P::CL;
  using LP = typename L::P;
  using LB = typename L::B;
  using LC = typename L::C;
  constexpr int KD = P::KD, MD = P::MD, M2 = M * M, K2 = K * K;
  constexpr int PP = (MD + NT - 1) / NT;   // integration points per thread
  // Point operators held in registers: one point per thread, or two when the
  // launch bounds leave at least 168 registers per thread.
  constexpr bool kRegD = PP == 1 || (PP == 2 && 65536 / (NT * P::MIN_BLOCKS) >= 168);
  constexpr bool kOwn = KD <= NT;   // x, r and p of the owned DOF in registers
  T *z = work, *p = z + 5 * LP::SV, *Ap = p + 5 * LP::SV, *x = Ap + 5 * LP::SV;
  T *pInt = x + 5 * LP::SV, *tK = pInt + 5 * LC::SV, *tJ = tK + P::CG_TK;
  T *dvdu = tJ + P::CG_TJ;  // 15 preconditioner entries, then V at the centre
  T *redA = s_red, *redB = s_red + 32;
  T *r = s_R;
  const T volElem = a.elem_scalars[(size_t)e * 15 + 5];
  const T JacInv = T(8.0) / volElem;
  // Padded offset of DOF l = (k K + j) K + i.
  auto off = [](const int l) { return (l / K2) * LP::S2 + ((l / K) % K) * LP::S1 + l % K; };

  // The owned DOF's iterate, residual and search direction (kOwn).
  T xo[5], ro[5], po[5];
  T m = T(0.0);
  if constexpr (kOwn) {
    const int l = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      ro[q] = l < KD ? r[q * KD + l] : T(0.0);
      xo[q] = T(0.0);
      po[q] = T(0.0);
      m = Fmax(m, Fabs(ro[q]));
    }
  } else {
    for (int i = threadIdx.x; i < 5 * KD; i += NT) m = Fmax(m, Fabs(r[i]));
    for (int l = threadIdx.x; l < KD; l += NT) {
#pragma unroll
      for (int q = 0; q < 5; ++q) x[q * LP::SV + off(l)] = T(0.0);
    }
  }
  // Inputs of a fused stage update (the state's second register, and in the
  // mixed form the FP64 state itself; the FP64 form takes the state from s_sol)
  // are fetched asynchronously into the part of the work area that the CG
  // leaves free, each entry by the thread that applies the update to it.
  const size_t g0 = (size_t)e * 5 * KD;
  // The launched kernel's plan (its work area; shared memory unless BIG).
  constexpr bool kMixed = sizeof(T) == 4;
  constexpr int kPrefOff = FusedUpdatePrefetch<K, M, T, OPEN>::OFF;
  constexpr bool kPrefetch = FusedUpdatePrefetch<K, M, T, OPEN>::value;
  double *pref = reinterpret_cast<double *>(work + kPrefOff);
  const bool fused = a.rk_kind != kRkNone;
  if (kPrefetch && fused) {
    for (int l = threadIdx.x; l < KD; l += NT) {
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        CpAsync8(pref + q * KD + l, a.rk_reg + g0 + q * KD + l);
        if (kMixed) CpAsync8(pref + 5 * KD + q * KD + l, a.rk_sol + g0 + q * KD + l);
      }
    }
    CpAsyncCommit();
  }
  // Entry idx = q K^3 + l of the element: stored or applied (same thread as its prefetch).
  auto finish = [&](const int idx, const double r, const double dt) {
    if (!fused) { a.res[g0 + idx] = r; return; }
    double s0, r0;
    if constexpr (kPrefetch) {
      r0 = pref[idx];
      s0 = kMixed ? pref[5 * KD + idx] : double(s_sol[idx]);
    } else {
      r0 = a.rk_reg[g0 + idx];
      s0 = kMixed ? a.rk_sol[g0 + idx] : double(s_sol[idx]);
    }
    StoreResidual(a, g0 + idx, r, dt, s0, r0);
  };
  const T rInitMax = BlockMax<NT>(m, s_red);
  if (!(rInitMax * JacInv > T(1.e-10))) {
    const double dtStage = fused ? *a.rk_dt : 0.0;
    if (kPrefetch && fused) CpAsyncWaitAll();
    for (int l = threadIdx.x; l < KD; l += NT)
#pragma unroll
      for (int q = 0; q < 5; ++q) finish(q * KD + l, 0.0, dtStage);
    return;
  }

  // Entropy variables at the element centre and dV/dU there (src/CG_MassMatrix.cpp:313-361).
  if (threadIdx.x < 5) {
    T V = T(0.0);
    for (int l = 0; l < KD; ++l) V += T(a.center[l]) * s_sol[threadIdx.x * KD + l];
    dvdu[threadIdx.x + 16] = V;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const T gm1 = T(kGam) - T(1.0), ov1mg = T(1.0) / (T(1.0) - T(kGam)), govgm1 = T(kGam) / gm1;
    const T V0 = dvdu[16], V1 = dvdu[17], V2 = dvdu[18], V3 = dvdu[19], V4 = dvdu[20];
    const T V4Inv = T(1.0) / V4;
    const T u = -V4Inv * V1, v = -V4Inv * V2, w = -V4Inv * V3;
    const T eKin = T(0.5) * (u * u + v * v + w * w);
    const T sEnt = T(kGam) - gm1 * (V0 - V4 * eKin);
    const T tmp = -V4 * exp(sEnt);
    const T rho = pow(tmp, ov1mg);
    const T pr = -rho * V4Inv;
    const T pInv = T(1.0) / pr;
    const T abv1 = gm1 * rho * pInv * pInv;
    const T abv2 = eKin * abv1;
    dvdu[0] = JacInv * (govgm1 / rho + abv2 * eKin);
    dvdu[1] = -JacInv * u * abv2;
    dvdu[2] = -JacInv * v * abv2;
    dvdu[3] = -JacInv * w * abv2;
    dvdu[4] = JacInv * (abv2 - pInv);
    dvdu[5] = JacInv * (abv1 * u * u + pInv);
    dvdu[6] = JacInv * abv1 * u * v;
    dvdu[7] = JacInv * abv1 * u * w;
    dvdu[8] = -JacInv * abv1 * u;
    dvdu[9] = JacInv * (abv1 * v * v + pInv);
    dvdu[10] = JacInv * abv1 * v * w;
    dvdu[11] = -JacInv * abv1 * v;
    dvdu[12] = JacInv * (abv1 * w * w + pInv);
    dvdu[13] = -JacInv * abv1 * w;
    dvdu[14] = JacInv * abv1;
  }
  __syncthreads();
  // The preconditioner: read as shared-memory broadcasts where it is applied
  // when x, r and p take registers, else held in registers.
  T Dr[kOwn ? 1 : 15];
  if constexpr (!kOwn) {
#pragma unroll
    for (int q = 0; q < 15; ++q) Dr[q] = dvdu[q];
  }
  auto D = [&](const int q) -> T {
    if constexpr (kOwn) return dvdu[q];
    else return Dr[q];
  };
  // The i-direction basis values and the point operators of this thread's points.
  T lc[PP][K];
  T dd[kRegD ? PP : 1][16];
#pragma unroll
  for (int n = 0; n < PP; ++n) {
    const int l = threadIdx.x + n * NT;
    if (l < MD) {
#pragma unroll
      for (int c = 0; c < K; ++c) lc[n][c] = Coef<SLOT, K, M, kLeg, T>(c, l % M);
      if constexpr (kRegD) PointOperator<MD>(s_cgp, s_jw, l, dd[n]);
    }
  }
  T part = T(0.0);
  for (int l = threadIdx.x; l < KD; l += NT) {
    T rr[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) rr[q] = kOwn ? ro[q] : r[q * KD + l];
    const T zz[5] = {
        D(0) * rr[0] + D(1) * rr[1] + D(2) * rr[2] + D(3) * rr[3] + D(4) * rr[4],
        D(1) * rr[0] + D(5) * rr[1] + D(6) * rr[2] + D(7) * rr[3] + D(8) * rr[4],
        D(2) * rr[0] + D(6) * rr[1] + D(9) * rr[2] + D(10) * rr[3] + D(11) * rr[4],
        D(3) * rr[0] + D(7) * rr[1] + D(10) * rr[2] + D(12) * rr[3] + D(13) * rr[4],
        D(4) * rr[0] + D(8) * rr[1] + D(11) * rr[2] + D(13) * rr[3] + D(14) * rr[4]};
    const int o = off(l);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      if constexpr (!kOwn) z[q * LP::SV + o] = zz[q];
      p[q * LP::SV + o] = zz[q];
      if constexpr (kOwn) po[q] = zz[q];
      part = Fma(rr[q], zz[q], part);
    }
  }
  T dotrz = BlockSum<NT>(part, s_red);

  int iter = 0;
  T beta = T(0.0);
  for (;; ++iter) {
    if (iter == 100) {
      if (threadIdx.x == 0) atomicAdd(a.status, 1);
      break;
    }
    // Ap = Leg^T3 (w J dU/dV (Leg3 p)) (src/CG_MassMatrix.cpp:408-443).
    KForwardUpdate<NT, SLOT, K, M, T, LP, typename L::A>(p, z, beta, !kOwn && iter > 0, tK);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLeg, 1, 5, K, K, M, K, M, false, T, typename L::A, LB>(tK, tJ);
    __syncthreads();
#pragma unroll
    for (int n = 0; n < PP; ++n) {
      const int l = threadIdx.x + n * NT;
      if (l < MD) {
        const int mk = l / M2, mj = (l / M) % M, mi = l % M;
        const T *src = tJ + mk * LB::S2 + mj * LB::S1;  // tJ[v][mk][mj][0..K-1]
        T q[5];
#pragma unroll
        for (int vv = 0; vv < 5; ++vv) {
          T acc = T(0);
#pragma unroll
          for (int c = 0; c < K; ++c) acc = fma(lc[n][c], src[vv * LB::SV + c], acc);
          q[vv] = acc;
        }
        T dl[16];
        if constexpr (kRegD) {
#pragma unroll
          for (int i = 0; i < 16; ++i) dl[i] = dd[n][i];
        } else {
          PointOperator<MD>(s_cgp, s_jw, l, dl);
        }
        const T iw = dl[15];
        const T p0 = iw * q[0], p1 = iw * q[1], p2 = iw * q[2], p3 = iw * q[3], p4 = iw * q[4];
        T *dstp = pInt + mk * LC::S2 + mj * LC::S1 + mi;
        dstp[0] = dl[0] * p0 + dl[1] * p1 + dl[2] * p2 + dl[3] * p3 + dl[4] * p4;
        dstp[LC::SV] = dl[1] * p0 + dl[5] * p1 + dl[6] * p2 + dl[7] * p3 + dl[8] * p4;
        dstp[2 * LC::SV] = dl[2] * p0 + dl[6] * p1 + dl[9] * p2 + dl[10] * p3 + dl[11] * p4;
        dstp[3 * LC::SV] = dl[3] * p0 + dl[7] * p1 + dl[10] * p2 + dl[12] * p3 + dl[13] * p4;
        dstp[4 * LC::SV] = dl[4] * p0 + dl[8] * p1 + dl[11] * p2 + dl[13] * p3 + dl[14] * p4;
      }
    }
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 2, 5, M, M, M, M, K, false, T, LC, typename L::D>(pInt, tJ);
    __syncthreads();
    ContractL<NT, SLOT, K, M, kLegT, 1, 5, M, M, K, M, K, false, T, typename L::D,
              typename L::E>(tJ, tK);
    __syncthreads();
    T alpha;
    if constexpr (kOwn) {
      IBackwardDot<NT, SLOT, K, M, T, typename L::E, LP, false>(tK, p, Ap);
      __syncthreads();
      T pAp = T(0.0);
      if (threadIdx.x < KD) {
        const int o = off(threadIdx.x);
#pragma unroll
        for (int q = 0; q < 5; ++q) pAp = Fma(po[q], Ap[q * LP::SV + o], pAp);
      }
      alpha = dotrz / BlockSum1<NT>(pAp, redA);
    } else {
      alpha = dotrz /
              BlockSum1<NT>(IBackwardDot<NT, SLOT, K, M, T, typename L::E, LP>(tK, p, Ap), redA);
    }
    // Each thread owns whole DOFs: update x and r, precondition, and form the
    // partial sums of the three reductions that close the iteration.
    T zAp = T(0.0), rzNew = T(0.0), rMax = T(0.0);
    T zn[5] = {T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
    for (int l = threadIdx.x; l < KD; l += NT) {
      const int o = off(l);
      T rr[5], ap[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        ap[q] = Ap[q * LP::SV + o];
        if constexpr (kOwn) {
          xo[q] = Fma(alpha, po[q], xo[q]);
          rr[q] = Fma(-alpha, ap[q], ro[q]);
          ro[q] = rr[q];
        } else {
          x[q * LP::SV + o] = Fma(alpha, p[q * LP::SV + o], x[q * LP::SV + o]);
          rr[q] = Fma(-alpha, ap[q], r[q * KD + l]);
          r[q * KD + l] = rr[q];
        }
        rMax = Fmax(rMax, Fabs(rr[q]));
      }
      const T zz[5] = {
          D(0) * rr[0] + D(1) * rr[1] + D(2) * rr[2] + D(3) * rr[3] + D(4) * rr[4],
          D(1) * rr[0] + D(5) * rr[1] + D(6) * rr[2] + D(7) * rr[3] + D(8) * rr[4],
          D(2) * rr[0] + D(6) * rr[1] + D(9) * rr[2] + D(10) * rr[3] + D(11) * rr[4],
          D(3) * rr[0] + D(7) * rr[1] + D(10) * rr[2] + D(12) * rr[3] + D(13) * rr[4],
          D(4) * rr[0] + D(8) * rr[1] + D(11) * rr[2] + D(13) * rr[3] + D(14) * rr[4]};
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        if constexpr (!kOwn) z[q * LP::SV + o] = zz[q];
        zn[q] = zz[q];
        zAp = Fma(zz[q], ap[q], zAp);
        rzNew = Fma(rr[q], zz[q], rzNew);
      }
    }
    BlockReduce3<NT>(zAp, rzNew, rMax, redB);
    if (rMax < T(a.cg_tol) * rInitMax) break;
    beta = -alpha * zAp / dotrz;
    dotrz = rzNew;
    // The owner forms the next search direction p = z + beta p and stores it
    // for the forward transforms.
    if constexpr (kOwn) {
      if (threadIdx.x < KD) {
        const int o = off(threadIdx.x);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          po[q] = Fma(beta, po[q], zn[q]);
          p[q * LP::SV + o] = po[q];
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0 && a.cg_stats) {
    atomicAdd(a.cg_stats, (unsigned long long)(iter + 1));
    atomicAdd(a.cg_stats + 1, 1ull);
  }
  // Every thread stores the iterate of the DOFs it owns (it wrote their
  // entries of x itself in the last update).
  const double dtStage = fused ? *a.rk_dt : 0.0;
  if (kPrefetch && fused) CpAsyncWaitAll();
  for (int l = threadIdx.x; l < KD; l += NT) {
    const int o = off(l);
#pragma unroll
    for (int q = 0; q < 5; ++q)
      finish(q * KD + l, double(kOwn ? xo[q] : x[q * LP::SV + o]), dtStage);
  }
}

// ---------------------------------------------------------------------------
// The fused kernel.
// ---------------------------------------------------------------------------
// One element's residual: volume terms, face distribution and mass solve, with
// the element arrays at smem (shared memory, or the CTA's global scratch area).
template <int K, int M, int NT, typename T, bool OPEN>
__device__ __forceinline__ void ResidualElement(const ResidualArgs &a, const int e, T *smem) {
  using P = Plan<K, M, T, OPEN>;
  constexpr int KD = P::KD, MD = P::MD;
  T *s_sol = smem, *s_R = s_sol + 5 * KD, *s_cgp = s_R + 5 * KD, *s_jw = s_cgp + 5 * MD;
  T *s_red = s_jw + MD, *s_fv = s_red + P::RED, *work = s_fv + P::FV;
  // Several cases per launch: skip unused elements and cases in another state.
  double mu = a.mu;
  if (a.cases.elem_case) {
    const int cs = a.cases.elem_case[e];
    if (cs < 0 || a.cases.state[cs] != a.cases.require) return;
    mu = a.cases.par[cs * kCasePar + kParMu];
  }
  using VP = VolumeMetricPrefetch<K, M, T, OPEN>;
  double *vms = VP::value ? reinterpret_cast<double *>(work + VP::OFF) : nullptr;
  // The element's volume metric: one bulk copy into the work area above the
  // volume phase's arrays, in flight during the interpolation contractions.
  __shared__ __align__(8) unsigned long long s_bar;
  if constexpr (VP::value) {
    if (threadIdx.x == 0) {
      BulkBarrierInit(&s_bar);
      BulkCopyToShared(vms, a.vol_metric + (size_t)e * 10 * P::MD, VP::BYTES, &s_bar);
    }
  }
  // The element's state: one bulk copy where it is FP64 in shared memory and its
  // size a multiple of 16 bytes (even K), else converted element by element.
  const double *src = a.sol + (size_t)e * 5 * KD;
  constexpr bool kBulkState = !P::BIG && sizeof(T) == 8 && (40 * KD) % 16 == 0;
  __shared__ __align__(8) unsigned long long s_bar_state;
  if constexpr (kBulkState) {
    if (threadIdx.x == 0) {
      BulkBarrierInit(&s_bar_state);
      BulkCopyToShared(s_sol, src, 40u * KD, &s_bar_state);
    }
  } else {
    for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = T(src[i]);
  }
  if (threadIdx.x < 2 * K) {
    s_fv[threadIdx.x] = FaceVal<Slot<K, M>::value, T>(threadIdx.x);
    s_fv[2 * K + threadIdx.x] = FaceDer<Slot<K, M>::value, T>(threadIdx.x);
  }
  __syncthreads();   // also orders the barrier's initialisation before the waits
  if constexpr (kBulkState) {
    if (!BulkWait(&s_bar_state)) {
      if (threadIdx.x == 0) atomicAdd(a.status + 3, 1);
      BulkWait(&s_bar_state);
    }
  }
  VolumePhase<NT, K, M, T, OPEN>(a, e, mu, s_sol, s_R, s_cgp, s_jw, work, s_red, vms, &s_bar);
  FacePhase<NT, K, M, T, OPEN>(a, e, s_R, s_fv, work);
  if (a.res_raw) {
    double *dst = a.res_raw + (size_t)e * 5 * KD;
    for (int i = threadIdx.x; i < 5 * KD; i += NT) dst[i] = double(s_R[i]);
  }
  __syncthreads();
  MassSolve<NT, K, M, T, OPEN>(a, e, s_sol, s_R, s_cgp, s_jw, work, s_red);
}

template <int K, int M, int NT, typename T, bool OPEN>
__global__ void __launch_bounds__(NT, (Plan<K, M, T, OPEN>::MIN_BLOCKS)) ResidualKernel(const ResidualArgs a) {
  using P = Plan<K, M, T, OPEN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if constexpr (P::BIG) {
    T *base = reinterpret_cast<T *>(a.scratch) + (size_t)blockIdx.x * P::SCRATCH;
    for (int i = blockIdx.x; i < a.n_elem; i += gridDim.x) {
      ResidualElement<K, M, NT, T, OPEN>(a, a.res_first + i, base);
      __syncthreads();
    }
  } else {
    if ((int)blockIdx.x >= a.n_elem) return;
    ResidualElement<K, M, NT, T, OPEN>(a, a.res_first + (int)blockIdx.x,
                                       reinterpret_cast<T *>(smem_raw));
  }
}

// Staging of the lower neighbours' states in the face-flux kernel's shared
// memory (FluxPlan::NB_PREF); 0 reads them per line from global memory.
#ifndef VCPG_FACE_NB_STAGING
#define VCPG_FACE_NB_STAGING 1
#endif

// Shared memory (in T) and launch shape of the face-flux kernel.
template <int K, int M, typename T = double> struct FluxPlan {
  static constexpr int KD = K * K * K, M2 = M * M;
  static constexpr int FV = 4 * (K > 7 ? K : 7);
  static constexpr int TOTAL = 5 * KD + FV + 90 * K * M + 120 * M2;
  static constexpr size_t BASE_BYTES = sizeof(T) * (size_t)TOTAL;
  // Above one CTA's shared memory: global scratch per CTA, elements in a loop.
  static constexpr bool BIG = BASE_BYTES > 227 * 1024;
  static constexpr int SCRATCH = (TOTAL + 3) / 4 * 4;
  // Launch shape measured on B200: 128 threads for degree <= 3; from degree 4
  // on, 160 threads (the 3 M^2 face points of a group in one pass); CTAs per SM
  // up to the VCPG_CAP_FLUX_* bounds.
  static constexpr bool FP64 = sizeof(T) == 8;
  static constexpr int NT = K <= 4 ? 128 : 160;
  static constexpr int CAP =
      K <= 3 ? (FP64 ? VCPG_CAP_FLUX_FP64_SMALL : VCPG_CAP_FLUX_FP32_SMALL)
      : K == 4 ? (FP64 ? VCPG_CAP_FLUX_FP64_K4 : VCPG_CAP_FLUX_FP32_K4)
               : (FP64 ? VCPG_CAP_FLUX_FP64_BIG : VCPG_CAP_FLUX_FP32_BIG);
  static constexpr int FIT = (int)(227 * 1024 / BASE_BYTES);
  static constexpr int MIN_BLOCKS = FIT < 1 ? 1 : (FIT > CAP ? CAP : FIT);
  // The three lower neighbours' FP64 states staged in shared memory (after the
  // T arrays, 8-byte aligned) where that keeps MIN_BLOCKS CTAs per SM: one burst
  // of coalesced asynchronous copies instead of strided per-line global loads.
  static constexpr int NB_OFF = (TOTAL * (int)sizeof(T) + 7) / 8;   // in doubles
  static constexpr size_t NB_BYTES = 8 * ((size_t)NB_OFF + 15 * (size_t)KD);
  // (228 KB per SM with 1 KB reserved per CTA), from degree 4 on: measured on B200,
  // the staging takes FaceFluxKernel from 4.62 to 4.50 ms at degree 4 (TGV 48^3,
  // FP64) but from 0.75 to 0.80 ms at degree 2 (TGV 40^3, FP64; FP32 0.52 to 0.55).
  static constexpr bool NB_PREF = VCPG_FACE_NB_STAGING && !BIG && K >= 5 &&
                                  (int)(233472 / (NB_BYTES + 1024)) >= MIN_BLOCKS;
  static constexpr size_t BYTES = NB_PREF ? NB_BYTES : BASE_BYTES;
};

// The fluxes of every interior face, computed once by the face's upper element
// (its Min faces), before the residual kernel distributes them to both sides.
template <int K, int M, int NT, typename T, bool SGS>
__device__ __forceinline__ void FaceFluxElement(const ResidualArgs &a, const int e, T *smem) {
  using FP = FluxPlan<K, M, T>;
  constexpr int KD = K * K * K;
  T *s_sol = smem, *s_fv = s_sol + 5 * KD, *work = s_fv + FP::FV;
  double mu = a.mu;
  if (a.cases.elem_case) {
    const int cs = a.cases.elem_case[e];
    if (cs < 0 || a.cases.state[cs] != a.cases.require) return;
    mu = a.cases.par[cs * kCasePar + kParMu];
  }
  // The lower neighbours' states (i, j, k), fetched asynchronously while the
  // element's own state is converted.
  double *s_nb = FP::NB_PREF ? reinterpret_cast<double *>(smem) + FP::NB_OFF : nullptr;
  if constexpr (FP::NB_PREF) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int nb = a.nbr[e * 6 + 2 * d];
      if (nb < 0) continue;
      const double *g = a.sol + (size_t)nb * 5 * KD;
      for (int i = threadIdx.x; i < 5 * KD; i += NT) CpAsync8(s_nb + d * 5 * KD + i, g + i);
    }
    CpAsyncCommit();
  }
  // The element's own state: one bulk copy where it is FP64 in shared memory and
  // its size a multiple of 16 bytes (even K), else converted value by value.
  const double *src = a.sol + (size_t)e * 5 * KD;
  constexpr bool kBulkState = !FP::BIG && sizeof(T) == 8 && (40 * KD) % 16 == 0;
  __shared__ __align__(8) unsigned long long s_bar_state;
  if constexpr (kBulkState) {
    if (threadIdx.x == 0) {
      BulkBarrierInit(&s_bar_state);
      BulkCopyToShared(s_sol, src, 40u * KD, &s_bar_state);
    }
  } else {
    for (int i = threadIdx.x; i < 5 * KD; i += NT) s_sol[i] = T(src[i]);
  }
  if constexpr (FP::NB_PREF) CpAsyncWaitAll();
  if (threadIdx.x < 2 * K) {
    s_fv[threadIdx.x] = FaceVal<Slot<K, M>::value, T>(threadIdx.x);
    s_fv[2 * K + threadIdx.x] = FaceDer<Slot<K, M>::value, T>(threadIdx.x);
  }
  __syncthreads();   // also orders the barrier's initialisation before the waits
  if constexpr (kBulkState) {
    if (!BulkWait(&s_bar_state)) {
      if (threadIdx.x == 0) atomicAdd(a.status + 3, 1);
      BulkWait(&s_bar_state);
    }
  }
  MinFaceFluxes<NT, K, M, T, SGS>(a, e, mu, s_sol, s_fv, work, s_nb);
}

// SGS: with a subgrid-scale model (without one the kernel carries none of its code).
template <int K, int M, int NT, typename T, bool SGS>
__global__ void __launch_bounds__(NT, (FluxPlan<K, M, T>::MIN_BLOCKS)) FaceFluxKernel(const ResidualArgs a) {
  using P = FluxPlan<K, M, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n_face_elem > 0 ? a.n_face_elem : a.n_elem;
  if constexpr (P::BIG) {
    T *base = reinterpret_cast<T *>(a.scratch) + (size_t)blockIdx.x * P::SCRATCH;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
      FaceFluxElement<K, M, NT, T, SGS>(a, a.face_first + i, base);
      __syncthreads();
    }
  } else {
    if ((int)blockIdx.x >= n) return;
    FaceFluxElement<K, M, NT, T, SGS>(a, a.face_first + (int)blockIdx.x,
                                      reinterpret_cast<T *>(smem_raw));
  }
}

}  // namespace vcpg
