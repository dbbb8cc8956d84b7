// C ABI of the library (include/vcp3d_b200.h): handle management, uploads,
// one residual, the CFL time step and CUDA-graph-captured time steps.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/vcp3d_b200.h"
#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "host_setup.h"
#include "kernels.h"
#include "open_boundary.h"


using namespace vcpg;

constexpr int kSendLists = 6;   // per direction, towards the rank below and above

struct vcpg_handle {
  vcpg_params prm{};
  int K = 0, M = 0, KD = 0, MD = 0, M2 = 0;
  int64_t nE = 0;
  // Partition (vcpg_set_partition): residual, time step and stages run on the
  // first nOwned elements, face fluxes on the first nFace; both nE otherwise.
  int64_t nOwned = 0, nFace = 0;
  // vcpg_residual_part: part 0 computes the face fluxes of [0, fluxReady) and the
  // residuals of [0, resReady) (vcpg_set_partition_parts), part 1 the rest.
  int64_t fluxReady = 0, resReady = 0;
  // Owned elements sent to neighbouring ranks (vcpg_set_send_list).
  int *d_send[kSendLists] = {};
  int32_t nSend[kSendLists] = {};
  cudaStream_t stream = nullptr;
  double *d_sol = nullptr, *d_solOld = nullptr, *d_res = nullptr, *d_resRaw = nullptr;
  double *d_vol = nullptr, *d_face = nullptr, *d_sc = nullptr;
  int *d_nbr = nullptr;
  unsigned long long *d_dtbits = nullptr, *d_mach2 = nullptr, *d_eddymax = nullptr;
  double *d_nmetric = nullptr;   // [nE][10][K^3] metric at the nodal DOFs (SGS model)
  double *d_dt = nullptr, *d_fixed = nullptr, *d_hist = nullptr;
  int *d_status = nullptr, *d_counter = nullptr;
  unsigned int *d_ticket = nullptr;   // last-block ticket of StartStepKernel
  unsigned long long *d_cgstats = nullptr;
  int hist_cap = 0;
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int graph_launches[2] = {0, 0};
  int64_t launches = 0;
  bool res_valid = false;  // d_res holds the residual of d_sol
  // Open boundaries (vcpg_set_open_boundary): characteristic boundary faces and sponges.
  bool open = false;
  int nB = 0;
  int *d_bface = nullptr;
  double *d_bpresc = nullptr, *d_pc = nullptr, *d_dlq = nullptr;
  double *d_btrace = nullptr, *d_bmach = nullptr, *d_bflux = nullptr;
  double *d_bforce = nullptr;   // [nB][6] wall-face forces of a monitored residual
  double *d_center = nullptr;   // [K^3] 3-D basis at the element centre
  void *d_scratch = nullptr;    // element arrays of degrees above one CTA's shared memory
  int scratch_ctas = 0;
  BlockFaceCfg *d_cfg = nullptr;
  void *d_fflux = nullptr;  // fluxes of every element's Min faces (FaceFluxKernel)
  int *d_sponge = nullptr;
  double *d_dampfn = nullptr, *d_dampst = nullptr, *d_cml = nullptr;
  int cml_on = 0;
  BlockFaceCfg cfg[6] = {};
  // Block-wide Mach sums per block face (vcpg_set_boundary_mach_sums).
  double *d_bmachsums = nullptr;
  bool use_bmach_sums = false;
  // Partitioned blocks: per boundary row its row in the block's list and the
  // block row of its subface's last face; the outlets' element-local Mach
  // numbers set per residual (vcpg_set_boundary_outlet_mach) where a last face
  // lies on another rank.
  std::vector<int> bBlockRow, bBlockLast;
  bool remoteLast = false;
  double *d_bmachlast = nullptr;
  bool use_bmachlast = false;
  std::string err;
};

namespace {

const double kLsA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kLsB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};

int Fail(vcpg_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

int CudaFail(vcpg_handle *h, cudaError_t e, const char *what) {
  return Fail(h, VCPG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VCPG_CUDA(h, call)                                   \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return CudaFail((h), e_, #call); \
  } while (0)

ResidualArgs MakeResidualArgs(vcpg_handle *h, double *rawOut, unsigned long long *mach) {
  ResidualArgs a{};
  a.sol = h->d_sol;
  a.res = h->d_res;
  a.res_raw = rawOut;
  a.vol_metric = h->d_vol;
  a.face_metric = h->d_face;
  a.elem_scalars = h->d_sc;
  a.nbr = h->d_nbr;
  a.center = h->d_center;
  a.scratch = h->d_scratch;
  a.scratch_ctas = h->scratch_ctas;
  a.n_elem = (int)h->nOwned;
  a.n_face_elem = (int)h->nFace;
  a.body_force = (h->prm.body_force[0] != 0.0 || h->prm.body_force[1] != 0.0 ||
                  h->prm.body_force[2] != 0.0) ? 1 : 0;
  const double pRefInv = 1.0 / h->prm.p_ref;
  for (int c = 0; c < 3; ++c) a.fbody[c] = pRefInv * h->prm.body_force[c];
  a.mu = h->prm.mu;
  a.tau_num = (double)((h->prm.n_poly + 1) * (h->prm.n_poly + 1)) * h->prm.rel_penalty;
  a.theta_sym = h->prm.theta_sym;
  a.riemann = h->prm.riemann;
  a.metric_compat = h->prm.metric_index_compat;
  a.mach2max = mach;
  a.sgs = h->prm.sgs_model;
  a.eddymax = mach ? h->d_eddymax : nullptr;   // with the monitoring data
  a.status = h->d_status;
  a.cg_stats = h->d_cgstats;
  // The mixed form computes the residual in FP32; its mass-matrix CG stops at a
  // tolerance FP32 can reach (1e-5 relative), the FP64 form at the reference's 1e-10.
  a.mixed = h->prm.precision == VCPG_MIXED ? 1 : 0;
  a.cg_tol = a.mixed ? 1.e-5 : 1.e-10;
  a.open = h->open ? 1 : 0;
  a.bflux = h->d_bflux;
  a.sponge_idx = h->d_sponge;
  a.damp_fn = h->d_dampfn;
  a.damp_state = h->d_dampst;
  a.cml = h->d_cml;
  a.cml_on = h->cml_on;
  a.face_flux = h->d_fflux;
  return a;
}

TimeStepArgs MakeTimeStepArgs(vcpg_handle *h) {
  TimeStepArgs t{};
  t.sol = h->d_sol;
  t.elem_scalars = h->d_sc;
  t.n_elem = (int)h->nOwned;
  t.scratch = h->d_scratch;
  t.scratch_ctas = h->scratch_ctas;
  t.n_poly = h->prm.n_poly;
  t.cfl = h->prm.cfl;
  t.mu = h->prm.mu;
  t.p_ref = h->prm.p_ref;
  t.u_ref = h->prm.u_ref;
  t.rho_ref = h->prm.rho_ref;
  t.dt_bits = h->d_dtbits;
  t.status = h->d_status;
  t.sgs = h->prm.sgs_model;
  t.vol_metric_dofs = h->d_nmetric;
  return t;
}

// Reads and clears the device status words; maps them to an error code.
int CheckStatus(vcpg_handle *h) {
  int st[4] = {0, 0, 0, 0};
  VCPG_CUDA(h, cudaMemcpyAsync(st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  if (st[0] || st[1] || st[2] || st[3])
    VCPG_CUDA(h, cudaMemsetAsync(h->d_status, 0, sizeof(st), h->stream));
  if (st[0]) return Fail(h, VCPG_E_CG_NOCONV, "mass-matrix CG reached 100 iterations in " +
                                                  std::to_string(st[0]) + " element solve(s)");
  if (st[2]) return Fail(h, VCPG_E_NEG_A2, "negative or not-a-number square speed of sound in the time step");
  if (st[1]) return Fail(h, VCPG_E_INVALID, "physical boundary face without a boundary condition");
  if (st[3]) return Fail(h, VCPG_E_CUDA, "an asynchronous copy into shared memory did not complete "
                                          "within its wait bound");
  return VCPG_OK;
}

BoundaryArgs MakeBoundaryArgs(vcpg_handle *h) {
  BoundaryArgs b{};
  b.sol = h->d_sol;
  b.face_metric = h->d_face;
  b.elem_scalars = h->d_sc;
  b.bface = h->d_bface;
  b.bpresc = h->d_bpresc;
  b.pc = h->d_pc;
  b.dlq = h->d_dlq;
  b.btrace = h->d_btrace;
  b.bmach = h->d_bmach;
  b.bmach_local = h->d_bmach ? h->d_bmach + h->nB : nullptr;   // [nB, 2 nB)
  b.bmach_sums = h->use_bmach_sums ? h->d_bmachsums : nullptr;
  b.bmach_last = h->use_bmachlast ? h->d_bmachlast : nullptr;
  b.bflux = h->d_bflux;
  b.nB = h->nB;
  b.mu = h->prm.mu;
  b.tau_num = (double)((h->prm.n_poly + 1) * (h->prm.n_poly + 1)) * h->prm.rel_penalty;
  b.theta_sym = h->prm.theta_sym;
  b.riemann = h->prm.riemann;
  b.metric_compat = h->prm.metric_index_compat;
  b.sgs = h->prm.sgs_model;
  b.cfgs = h->d_cfg;
  return b;
}

// One residual evaluation: the characteristic boundary kernels (when the block
// has characteristic faces) and the fused residual kernel. Returns the launches.
int EnqueueResidual(vcpg_handle *h, const ResidualArgs &a, int *launches) {
  int n = 0;
  if (h->open && h->nB > 0) {
    BoundaryArgs b = MakeBoundaryArgs(h);
    b.eddymax = a.eddymax;
    // Wall forces only for a residual with monitoring data (mach2max set).
    b.bforce = (a.mach2max && h->prm.monitor_forces) ? h->d_bforce : nullptr;
    VCPG_CUDA(h, LaunchBoundary(h->K, h->M, b, h->stream));
    n += 2;
  }
  VCPG_CUDA(h, LaunchResidual(h->K, h->M, a, h->stream));
  n += 2;
  if (launches) *launches = n;
  return VCPG_OK;
}

// Uploads a block's (or a part's) open-boundary data to the handle.
int InstallOpenBoundary(vcpg_handle *h, const OpenBoundaryHost &ob_host) {
  int rc = VCPG_OK;
  const int M2 = h->M2, MD = h->MD;
  auto upload = [&](void **dst, const void *src, size_t bytes) -> int {
    if (bytes == 0) return VCPG_OK;
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    if (src) {
      e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return CudaFail(h, e, "cudaMemcpy open boundary");
    }
    return VCPG_OK;
  };
  const size_t nB = (size_t)ob_host.nB, nS = (size_t)ob_host.nS;
  if ((rc = upload((void **)&h->d_bface, ob_host.bface.data(), sizeof(int) * ob_host.bface.size())) ||
      (rc = upload((void **)&h->d_bpresc, ob_host.bpresc.data(), sizeof(double) * ob_host.bpresc.size())) ||
      (rc = upload((void **)&h->d_pc, ob_host.pc.data(), sizeof(double) * ob_host.pc.size())) ||
      (rc = upload((void **)&h->d_dlq, ob_host.dlq.data(), sizeof(double) * ob_host.dlq.size())) ||
      (rc = upload((void **)&h->d_btrace, nullptr, sizeof(double) * nB * 4 * 5 * M2)) ||
      (rc = upload((void **)&h->d_bmach, nullptr, sizeof(double) * nB * 2)) ||
      (rc = upload((void **)&h->d_bforce, nullptr, sizeof(double) * nB * 6)) ||
      (rc = upload((void **)&h->d_bflux, nullptr, sizeof(double) * nB * 4 * 5 * M2)) ||
      (rc = upload((void **)&h->d_sponge, ob_host.spongeIdx.data(), sizeof(int) * ob_host.spongeIdx.size())) ||
      (rc = upload((void **)&h->d_dampfn, ob_host.dampFn.data(), sizeof(double) * nS * 3 * MD)) ||
      (rc = upload((void **)&h->d_dampst, ob_host.dampState.data(), sizeof(double) * nS * 5 * MD)) ||
      (rc = upload((void **)&h->d_cml, ob_host.cml.data(), sizeof(double) * nS * 6)) ||
      (rc = upload((void **)&h->d_cfg, ob_host.cfg, sizeof(BlockFaceCfg) * 6)))
    return rc;
  // Boundary faces are coded in the neighbour table as -2 - (boundary-face index).
  VCPG_CUDA(h, cudaMemcpy(h->d_nbr, ob_host.nbrCode.data(), sizeof(int32_t) * ob_host.nbrCode.size(),
                          cudaMemcpyHostToDevice));
  h->nB = ob_host.nB;
  h->cml_on = ob_host.cmlOn;
  h->bBlockRow = ob_host.blockRow;
  h->bBlockLast = ob_host.blockLast;
  h->remoteLast = false;
  for (int f = 0; f < 6; ++f) {
    const BlockFaceCfg &c = ob_host.cfg[f];
    for (int r = c.first; r < c.first + c.count; ++r)
      if (c.localMach && ob_host.bface[(size_t)r * kBfStride + kBfLast] < 0) h->remoteLast = true;
  }
  for (int f = 0; f < 6; ++f) h->cfg[f] = ob_host.cfg[f];
  h->open = true;
  h->res_valid = false;
  // Captured steps hold the previous launch sequence.
  for (int s = 0; s < 2; ++s) {
    if (h->exec[s]) { cudaGraphExecDestroy(h->exec[s]); h->exec[s] = nullptr; }
    if (h->graph[s]) { cudaGraphDestroy(h->graph[s]); h->graph[s] = nullptr; }
  }
  return VCPG_OK;
}

int ResidualLaunches(const vcpg_handle *h) { return (h->open && h->nB > 0) ? 4 : 2; }

bool FusedSteps(const vcpg_handle *h) {
  return FusedStageUpdate(h->K, h->M, h->prm.precision == VCPG_MIXED, h->open);
}

// One time step of a single case: the CFL time step, then the first stage's
// update together with recording the step (StartStepKernel), then per stage a
// residual whose kernel applies the next stage's update to its element in its
// epilogue; the last stage's residual is stored (the next step's first stage
// uses it). SSP-RK3: 2 + 3 residuals' launches, low-storage RK4: 2 + 5. Where
// the residual kernel cannot prefetch the update's inputs (FusedStageUpdate),
// the step records the time step (FinalizeDtKernel) and runs a stage kernel
// before each residual instead.
int EnqueueStep(vcpg_handle *h, int scheme) {
  const size_t n = (size_t)h->nOwned * 5 * h->KD;
  TimeStepArgs t = MakeTimeStepArgs(h);
  VCPG_CUDA(h, LaunchTimeStep(h->K, h->M, t, h->stream));
  const double alphaRK[] = {1.0, 3.0 / 4.0, 1.0 / 3.0};
  const double betaRK[] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  const bool ssp = scheme == VCPG_SSPRK3;
  const int stages = ssp ? 3 : 5;
  const int kind = ssp ? kRkSsp : kRkLowStorage;
  auto coefA = [&](int s) { return ssp ? alphaRK[s] : kLsA[s]; };
  auto coefB = [&](int s) { return ssp ? betaRK[s] : kLsB[s]; };
  if (!FusedSteps(h)) {
    // The fixed step lives in device memory (d_fixed); a non-positive value selects the CFL step.
    VCPG_CUDA(h, LaunchFinalizeDt(h->d_dtbits, h->d_fixed, h->d_dt, h->d_hist, h->hist_cap,
                                  h->d_counter, h->stream));
    const ResidualArgs a = MakeResidualArgs(h, nullptr, nullptr);
    for (int s = 0; s < stages; ++s) {
      if (ssp)
        VCPG_CUDA(h, LaunchSspStage(h->d_sol, h->d_solOld, h->d_res, h->d_dt, alphaRK[s],
                                    betaRK[s], s == 0, n, h->stream, CaseView{}, 5 * h->KD));
      else
        VCPG_CUDA(h, LaunchLsrkStage(h->d_sol, h->d_solOld, h->d_res, h->d_dt, kLsA[s], kLsB[s],
                                     n, h->stream, CaseView{}, 5 * h->KD));
      int rc = EnqueueResidual(h, a, nullptr);
      if (rc) return rc;
    }
    return VCPG_OK;
  }
  VCPG_CUDA(h, LaunchStartStep(h->d_dtbits, h->d_fixed, h->d_dt, h->d_hist, h->hist_cap,
                               h->d_counter, h->d_ticket, h->d_sol, h->d_solOld, h->d_res, kind,
                               coefA(0), coefB(0), n, h->stream));
  for (int s = 0; s < stages; ++s) {
    ResidualArgs a = MakeResidualArgs(h, nullptr, nullptr);
    if (s + 1 < stages) {
      a.rk_kind = kind;
      a.rk_a = coefA(s + 1);
      a.rk_b = coefB(s + 1);
      a.rk_dt = h->d_dt;
      a.rk_sol = h->d_sol;
      a.rk_reg = h->d_solOld;
      a.rk_store_res = 0;
    }
    int rc = EnqueueResidual(h, a, nullptr);
    if (rc) return rc;
  }
  return VCPG_OK;
}

}  // namespace

extern "C" {

const char *vcpg_last_error(const vcpg_handle *h) { return h ? h->err.c_str() : "null handle"; }

int vcpg_destroy(vcpg_handle *h) {
  if (!h) return VCPG_OK;
  for (int s = 0; s < 2; ++s) {
    if (h->exec[s]) cudaGraphExecDestroy(h->exec[s]);
    if (h->graph[s]) cudaGraphDestroy(h->graph[s]);
  }
  void *bufs[] = {h->d_sol, h->d_solOld, h->d_res, h->d_resRaw, h->d_vol, h->d_face, h->d_sc,
                  h->d_nbr, h->d_dtbits, h->d_mach2, h->d_dt, h->d_fixed, h->d_hist,
                  h->d_status, h->d_counter, h->d_ticket, h->d_cgstats, h->d_bface, h->d_bpresc, h->d_pc,
                  h->d_dlq, h->d_btrace, h->d_bmach, h->d_bflux, h->d_sponge, h->d_dampfn,
                  h->d_dampst, h->d_cml, h->d_cfg, h->d_fflux, h->d_eddymax, h->d_nmetric,
                  h->d_bforce, h->d_center, h->d_scratch, h->d_bmachsums, h->d_bmachlast};
  for (void *p : bufs)
    if (p) cudaFree(p);
  for (int *p : h->d_send)
    if (p) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return VCPG_OK;
}

int vcpg_create(const vcpg_params *params, const vcpg_operators *ops, const vcpg_geometry *geom,
                vcpg_handle **out) {
  if (!params || !ops || !geom || !out) return VCPG_E_INVALID;
  *out = nullptr;
  vcpg_handle *h = new vcpg_handle();
  h->prm = *params;
  h->K = params->n_poly + 1;
  h->M = params->n_int_1d;
  h->KD = h->K * h->K * h->K;
  h->MD = h->M * h->M * h->M;
  h->M2 = h->M * h->M;
  h->nE = (int64_t)params->n_elem[0] * params->n_elem[1] * params->n_elem[2];
  if (h->nE <= 0 || h->nE > (int64_t)2147483647) {
    int rc = Fail(h, VCPG_E_INVALID, "invalid element count");
    *out = h;
    return rc;
  }
  h->nOwned = h->nFace = h->nE;
  if (!Supported(h->K, h->M) || h->K > kKMax || h->M > kMMax) {
    int rc = Fail(h, VCPG_E_UNSUPPORTED_KM, "no kernel for K=" + std::to_string(h->K) +
                                                " M=" + std::to_string(h->M));
    *out = h;
    return rc;
  }
  if (params->precision != VCPG_FP64 && params->precision != VCPG_MIXED) {
    int rc = Fail(h, VCPG_E_INVALID, "precision must be VCPG_FP64 or VCPG_MIXED");
    *out = h;
    return rc;
  }
  if (params->monitor_forces && !(params->mach > 0.0 && params->ref_area > 0.0)) {
    int rc = Fail(h, VCPG_E_INVALID, "force monitoring needs mach > 0 and ref_area > 0");
    *out = h;
    return rc;
  }
  if (params->sgs_model < VCPG_SGS_NONE || params->sgs_model > VCPG_SGS_VREMAN ||
      (params->sgs_model != VCPG_SGS_NONE && (!ops->dleg_dofs || !geom->vol_metric_dofs))) {
    int rc = Fail(h, VCPG_E_INVALID, "sgs_model must be VCPG_SGS_NONE, _WALE or _VREMAN; a model "
                                     "needs ops->dleg_dofs and geom->vol_metric_dofs");
    *out = h;
    return rc;
  }
  *out = h;
  const int K = h->K, M = h->M;
  // Operator table into the (K, M) constant slot.
  VCPG_CUDA(h, UploadOperatorTable(ops, K, M));

  VCPG_CUDA(h, ConfigureResidual(K, M));
  VCPG_CUDA(h, ConfigureTimeStep(K, M));
  VCPG_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  const size_t nState = (size_t)h->nE * 5 * h->KD;
  auto alloc = [&](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return VCPG_OK;
  };
  int rc;
  if ((rc = alloc((void **)&h->d_sol, nState * 8))) return rc;
  if ((rc = alloc((void **)&h->d_solOld, nState * 8))) return rc;
  if ((rc = alloc((void **)&h->d_res, nState * 8))) return rc;
  if ((rc = alloc((void **)&h->d_fflux, (size_t)h->nE * FaceFluxBytesPerElement(K, M)))) return rc;
  if ((rc = alloc((void **)&h->d_vol, (size_t)h->nE * 10 * h->MD * 8))) return rc;
  if ((rc = alloc((void **)&h->d_face, (size_t)h->nE * 6 * 13 * h->M2 * 8))) return rc;
  if ((rc = alloc((void **)&h->d_sc, (size_t)h->nE * 15 * 8))) return rc;
  if ((rc = alloc((void **)&h->d_nbr, (size_t)h->nE * 6 * sizeof(int)))) return rc;
  if ((rc = alloc((void **)&h->d_dtbits, sizeof(unsigned long long)))) return rc;
  if ((rc = alloc((void **)&h->d_mach2, sizeof(unsigned long long)))) return rc;
  if ((rc = alloc((void **)&h->d_eddymax, sizeof(unsigned long long)))) return rc;
  if (params->sgs_model != VCPG_SGS_NONE) {
    if ((rc = alloc((void **)&h->d_nmetric, (size_t)h->nE * 10 * h->KD * 8))) return rc;
    VCPG_CUDA(h, cudaMemcpy(h->d_nmetric, geom->vol_metric_dofs, (size_t)h->nE * 10 * h->KD * 8,
                            cudaMemcpyHostToDevice));
  }
  if ((rc = alloc((void **)&h->d_center, (size_t)h->KD * 8))) return rc;
  VCPG_CUDA(h, cudaMemcpy(h->d_center, ops->basis_center, (size_t)h->KD * 8,
                          cudaMemcpyHostToDevice));
  {
    // Degrees 7-9 (FP64) loop one CTA per SM over the elements with global scratch.
    int dev = 0, sms = 0;
    VCPG_CUDA(h, cudaGetDevice(&dev));
    VCPG_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t sb = ResidualScratchBytes(K, M, sms);
    if (sb > 0) {
      if ((rc = alloc(&h->d_scratch, sb))) return rc;
      h->scratch_ctas = sms;
    }
  }
  if ((rc = alloc((void **)&h->d_dt, sizeof(double)))) return rc;
  if ((rc = alloc((void **)&h->d_fixed, sizeof(double)))) return rc;
  if ((rc = alloc((void **)&h->d_status, 4 * sizeof(int)))) return rc;
  if ((rc = alloc((void **)&h->d_counter, sizeof(int)))) return rc;
  if ((rc = alloc((void **)&h->d_ticket, sizeof(unsigned int)))) return rc;
  VCPG_CUDA(h, cudaMemsetAsync(h->d_ticket, 0, sizeof(unsigned int), h->stream));
  if ((rc = alloc((void **)&h->d_cgstats, 2 * sizeof(unsigned long long)))) return rc;
  VCPG_CUDA(h, cudaMemsetAsync(h->d_cgstats, 0, 2 * sizeof(unsigned long long), h->stream));
  h->hist_cap = 1024;
  if ((rc = alloc((void **)&h->d_hist, (size_t)h->hist_cap * 8))) return rc;
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_vol, geom->vol_metric, (size_t)h->nE * 10 * h->MD * 8,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_face, geom->face_metric, (size_t)h->nE * 6 * 13 * h->M2 * 8,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_sc, geom->elem_scalars, (size_t)h->nE * 15 * 8,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_nbr, geom->neighbors, (size_t)h->nE * 6 * sizeof(int),
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaMemsetAsync(h->d_sol, 0, nState * 8, h->stream));
  VCPG_CUDA(h, cudaMemsetAsync(h->d_solOld, 0, nState * 8, h->stream));
  VCPG_CUDA(h, cudaMemsetAsync(h->d_res, 0, nState * 8, h->stream));
  VCPG_CUDA(h, cudaMemsetAsync(h->d_status, 0, 4 * sizeof(int), h->stream));
  const double big = 1.e+10;
  unsigned long long bits;
  std::memcpy(&bits, &big, 8);
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_dtbits, &bits, 8, cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_set_state(vcpg_handle *h, const double *modal) {
  if (!h || !modal) return VCPG_E_INVALID;
  h->res_valid = false;
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_sol, modal, (size_t)h->nE * 5 * h->KD * 8,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_get_state(vcpg_handle *h, double *modal) {
  if (!h || !modal) return VCPG_E_INVALID;
  VCPG_CUDA(h, cudaMemcpyAsync(modal, h->d_sol, (size_t)h->nE * 5 * h->KD * 8,
                               cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_get_residual(vcpg_handle *h, double *res) {
  if (!h || !res) return VCPG_E_INVALID;
  VCPG_CUDA(h, cudaMemcpyAsync(res, h->d_res, (size_t)h->nE * 5 * h->KD * 8,
                               cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_get_raw_residual(vcpg_handle *h, double *res) {
  if (!h || !res) return VCPG_E_INVALID;
  if (!h->d_resRaw) return Fail(h, VCPG_E_INVALID, "no raw residual kept");
  VCPG_CUDA(h, cudaMemcpyAsync(res, h->d_resRaw, (size_t)h->nE * 5 * h->KD * 8,
                               cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_residual(vcpg_handle *h, double *monitoring, int32_t keep_raw) {
  if (!h) return VCPG_E_INVALID;
  if (h->remoteLast && !h->use_bmachlast)
    return Fail(h, VCPG_E_INVALID, "outlet Mach numbers of subfaces whose last face lies on "
                                   "another rank: vcpg_set_boundary_outlet_mach first");
  if (keep_raw && !h->d_resRaw) {
    cudaError_t e = cudaMalloc((void **)&h->d_resRaw, (size_t)h->nE * 5 * h->KD * 8);
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, "cudaMalloc raw residual");
  }
  const bool forces = monitoring && h->prm.monitor_forces && h->d_bforce && h->nB > 0;
  if (monitoring) {
    VCPG_CUDA(h, cudaMemsetAsync(h->d_mach2, 0, 8, h->stream));
    VCPG_CUDA(h, cudaMemsetAsync(h->d_eddymax, 0, 8, h->stream));
    if (forces)   // faces that are no walls keep zeros
      VCPG_CUDA(h, cudaMemsetAsync(h->d_bforce, 0, sizeof(double) * 6 * h->nB, h->stream));
  }
  ResidualArgs a = MakeResidualArgs(h, keep_raw ? h->d_resRaw : nullptr,
                                    monitoring ? h->d_mach2 : nullptr);
  int nl = 0;
  int rc = EnqueueResidual(h, a, &nl);
  if (rc) return rc;
  h->launches += nl;
  rc = CheckStatus(h);
  h->res_valid = rc == VCPG_OK;
  if (monitoring) {
    unsigned long long bits = 0;
    VCPG_CUDA(h, cudaMemcpy(&bits, h->d_mach2, 8, cudaMemcpyDeviceToHost));
    double m2;
    std::memcpy(&m2, &bits, 8);
    VCPG_CUDA(h, cudaMemcpy(&bits, h->d_eddymax, 8, cudaMemcpyDeviceToHost));
    double eddyMax;
    std::memcpy(&eddyMax, &bits, 8);
    // Force coefficients (src/SolverClass.cpp:3754-3783): pressure and viscous
    // forces of the wall faces, summed in boundary-face order and scaled by
    // 2 / (gamma M^2 A_ref); zero without force monitoring or walls.
    for (int i = 0; i < 6; ++i) monitoring[i] = 0.0;
    if (forces) {
      std::vector<double> bf((size_t)6 * h->nB);
      VCPG_CUDA(h, cudaMemcpy(bf.data(), h->d_bforce, sizeof(double) * bf.size(),
                              cudaMemcpyDeviceToHost));
      for (int b = 0; b < h->nB; ++b)
        for (int i = 0; i < 6; ++i) monitoring[i] += bf[(size_t)b * 6 + i];
      const double factCoef = 2.0 / (1.4 * h->prm.mach * h->prm.mach * h->prm.ref_area);
      for (int i = 0; i < 6; ++i) monitoring[i] *= factCoef;
    }
    monitoring[6] = m2;
    monitoring[7] = eddyMax;   // maximum eddy viscosity of the volume and face points
  }
  return rc;
}

int vcpg_time_residual_kernels(vcpg_handle *h, int32_t reps, double *ms) {
  if (!h || reps < 1 || !ms) return VCPG_E_INVALID;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  for (auto &e : ev) VCPG_CUDA(h, cudaEventCreate(&e));
  const ResidualArgs a = MakeResidualArgs(h, nullptr, nullptr);
  const bool open = h->open && h->nB > 0;
  double acc[3] = {0.0, 0.0, 0.0};
  cudaError_t err = cudaSuccess;
  for (int r = 0; r < reps && err == cudaSuccess; ++r) {
    err = cudaEventRecord(ev[0], h->stream);
    if (err == cudaSuccess && open) err = LaunchBoundary(h->K, h->M, MakeBoundaryArgs(h), h->stream);
    if (err == cudaSuccess) err = cudaEventRecord(ev[1], h->stream);
    if (err == cudaSuccess) err = LaunchResidual(h->K, h->M, a, h->stream, 1);
    if (err == cudaSuccess) err = cudaEventRecord(ev[2], h->stream);
    if (err == cudaSuccess) err = LaunchResidual(h->K, h->M, a, h->stream, 2);
    if (err == cudaSuccess) err = cudaEventRecord(ev[3], h->stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[3]);
    for (int k = 0; k < 3 && err == cudaSuccess; ++k) {
      float t = 0.f;
      err = cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  VCPG_CUDA(h, err);
  h->launches += (int64_t)reps * ResidualLaunches(h);
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / reps;
  const int rc = CheckStatus(h);
  h->res_valid = rc == VCPG_OK;
  return rc;
}

int vcpg_time_step(vcpg_handle *h, double *dt) {
  if (!h || !dt) return VCPG_E_INVALID;
  TimeStepArgs t = MakeTimeStepArgs(h);
  VCPG_CUDA(h, LaunchTimeStep(h->K, h->M, t, h->stream));
  h->launches += 1;
  unsigned long long bits = 0;
  VCPG_CUDA(h, cudaMemcpyAsync(&bits, h->d_dtbits, 8, cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(dt, &bits, 8);
  const double big = 1.e+10;
  std::memcpy(&bits, &big, 8);
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_dtbits, &bits, 8, cudaMemcpyHostToDevice, h->stream));
  return CheckStatus(h);
}

int vcpg_step(vcpg_handle *h, int32_t scheme, int32_t n_steps, double fixed_dt,
              double *dt_history) {
  if (!h || n_steps < 0 || (scheme != VCPG_SSPRK3 && scheme != VCPG_LSRK4)) return VCPG_E_INVALID;
  if (h->nOwned != h->nE)
    return Fail(h, VCPG_E_INVALID, "a partitioned block steps stage by stage (vcpg_rk_stage) "
                                   "with the halo exchanged before every residual");
  if (n_steps == 0) return VCPG_OK;
  if (n_steps > h->hist_cap) {
    // Grow the history buffer; graphs hold the old pointer and are rebuilt.
    for (int s = 0; s < 2; ++s) {
      if (h->exec[s]) { cudaGraphExecDestroy(h->exec[s]); h->exec[s] = nullptr; }
      if (h->graph[s]) { cudaGraphDestroy(h->graph[s]); h->graph[s] = nullptr; }
    }
    cudaFree(h->d_hist);
    h->d_hist = nullptr;
    h->hist_cap = n_steps;
    cudaError_t e = cudaMalloc((void **)&h->d_hist, (size_t)h->hist_cap * 8);
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, "cudaMalloc dt history");
  }
  if (!h->res_valid) {
    // The first stage uses the residual of the current state: evaluate it once
    // after a new state was set (later steps reuse the last stage's residual).
    int nl = 0;
    int rc0 = EnqueueResidual(h, MakeResidualArgs(h, nullptr, nullptr), &nl);
    if (rc0) return rc0;
    h->launches += nl;
  }
  const double fx = fixed_dt > 0.0 ? fixed_dt : -1.0;
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_fixed, &fx, 8, cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
  if (!h->exec[scheme]) {
    VCPG_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = EnqueueStep(h, scheme);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return CudaFail(h, e, "cudaStreamEndCapture");
    h->graph[scheme] = g;
    VCPG_CUDA(h, cudaGraphInstantiate(&h->exec[scheme], g, 0));
    h->graph_launches[scheme] = 2 + (scheme == VCPG_SSPRK3 ? 3 : 5) *
                                        (ResidualLaunches(h) + (FusedSteps(h) ? 0 : 1));
  }
  for (int s = 0; s < n_steps; ++s) VCPG_CUDA(h, cudaGraphLaunch(h->exec[scheme], h->stream));
  h->launches += (int64_t)n_steps * h->graph_launches[scheme];
  if (dt_history)
    VCPG_CUDA(h, cudaMemcpyAsync(dt_history, h->d_hist, (size_t)n_steps * 8,
                                 cudaMemcpyDeviceToHost, h->stream));
  const int rc = CheckStatus(h);
  h->res_valid = rc == VCPG_OK;
  return rc;
}

int vcpg_synchronization_step(vcpg_handle *h, double dt_sync, int32_t max_steps,
                              int32_t *n_steps, double *monitoring) {
  if (!h || !(dt_sync > 0.0) || max_steps < 1) return VCPG_E_INVALID;
  // SolverClass::ExecuteTimeSynchronizationStep (src/SolverClass.cpp:2177-2422):
  // SSP-RK3 steps with the CFL step of the current state; the step that would
  // reach 0.99 of the synchronisation time is shortened to end on it exactly.
  double elapsed = 0.0;
  int32_t taken = 0;
  bool reached = false;
  while (!reached) {
    if (taken == max_steps) {
      if (n_steps) *n_steps = taken;
      return Fail(h, VCPG_E_INVALID, "synchronization time not reached within max_steps");
    }
    double dt = 0.0;
    int rc = vcpg_time_step(h, &dt);
    if (rc) return rc;
    if (elapsed + dt >= 0.99 * dt_sync) {
      dt = dt_sync - elapsed;
      reached = true;
    }
    elapsed += dt;
    rc = vcpg_step(h, VCPG_SSPRK3, 1, dt, nullptr);
    if (rc) return rc;
    ++taken;
  }
  if (n_steps) *n_steps = taken;
  // The reference fills the monitoring data in the last stage's residual, the
  // residual of the new state: evaluate it once more with monitoring.
  if (monitoring) return vcpg_residual(h, monitoring, 0);
  return VCPG_OK;
}

int vcpg_sync(vcpg_handle *h) {
  if (!h) return VCPG_E_INVALID;
  return CheckStatus(h);
}

int vcpg_set_partition(vcpg_handle *h, int32_t n_owned, int32_t n_face_ghost) {
  if (!h) return VCPG_E_INVALID;
  if (n_owned < 1 || n_face_ghost < 0 || (int64_t)n_owned + n_face_ghost > h->nE)
    return Fail(h, VCPG_E_INVALID, "partition: need 1 <= n_owned and n_owned + n_face_ghost "
                                   "<= the handle's elements");
  if (h->open)
    return Fail(h, VCPG_E_INVALID, "partition: declare the partition before the open boundaries "
                                   "(vcpg_set_open_boundary_partition)");
  h->nOwned = n_owned;
  h->nFace = (int64_t)n_owned + n_face_ghost;
  h->fluxReady = h->resReady = 0;   // no overlap until vcpg_set_partition_parts
  h->res_valid = false;
  for (int s = 0; s < 2; ++s) {
    if (h->exec[s]) { cudaGraphExecDestroy(h->exec[s]); h->exec[s] = nullptr; }
    if (h->graph[s]) { cudaGraphDestroy(h->graph[s]); h->graph[s] = nullptr; }
  }
  return VCPG_OK;
}

int vcpg_set_partition_parts(vcpg_handle *h, int32_t flux_ready, int32_t res_ready) {
  if (!h) return VCPG_E_INVALID;
  if (h->nOwned == h->nE)
    return Fail(h, VCPG_E_INVALID, "partition parts: a partitioned handle only");
  if (res_ready < 0 || res_ready > flux_ready || flux_ready > h->nOwned)
    return Fail(h, VCPG_E_INVALID, "partition parts: need 0 <= res_ready <= flux_ready <= "
                                   "n_owned");
  h->fluxReady = flux_ready;
  h->resReady = res_ready;
  return VCPG_OK;
}

int vcpg_set_send_list(vcpg_handle *h, int32_t list, const int32_t *elems, int32_t count) {
  if (!h || list < 0 || list >= kSendLists || count < 0 || (count > 0 && !elems))
    return VCPG_E_INVALID;
  for (int32_t i = 0; i < count; ++i)
    if (elems[i] < 0 || elems[i] >= h->nOwned)
      return Fail(h, VCPG_E_INVALID, "send list: elements must be owned");
  if (h->d_send[list]) {
    VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->d_send[list]);
    h->d_send[list] = nullptr;
  }
  h->nSend[list] = count;
  if (count == 0) return VCPG_OK;
  cudaError_t e = cudaMalloc((void **)&h->d_send[list], sizeof(int32_t) * count);
  if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, "cudaMalloc send list");
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_send[list], elems, sizeof(int32_t) * count,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_pack_send_list(vcpg_handle *h, int32_t list, double *d_buf) {
  if (!h || list < 0 || list >= kSendLists) return VCPG_E_INVALID;
  if (h->nSend[list] == 0) return VCPG_OK;
  if (!d_buf) return VCPG_E_INVALID;
  VCPG_CUDA(h, LaunchGatherStates(h->d_sol, h->d_send[list], h->nSend[list], 5 * h->KD, d_buf,
                                  h->stream));
  h->launches += 1;
  return VCPG_OK;
}

int vcpg_pack_states(vcpg_handle *h, int32_t first, int32_t count, double *d_buf) {
  if (!h || !d_buf || first < 0 || count < 0 || (int64_t)first + count > h->nE)
    return VCPG_E_INVALID;
  const size_t per = (size_t)5 * h->KD;
  VCPG_CUDA(h, cudaMemcpyAsync(d_buf, h->d_sol + (size_t)first * per, sizeof(double) * per * count,
                               cudaMemcpyDeviceToDevice, h->stream));
  return VCPG_OK;
}

int vcpg_unpack_states(vcpg_handle *h, int32_t first, int32_t count, const double *d_buf) {
  if (!h || !d_buf || first < 0 || count < 0 || (int64_t)first + count > h->nE)
    return VCPG_E_INVALID;
  const size_t per = (size_t)5 * h->KD;
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_sol + (size_t)first * per, d_buf, sizeof(double) * per * count,
                               cudaMemcpyDeviceToDevice, h->stream));
  h->res_valid = false;
  return VCPG_OK;
}

int vcpg_rk_stage(vcpg_handle *h, int32_t scheme, int32_t stage, double dt) {
  if (!h || !(dt > 0.0)) return VCPG_E_INVALID;
  if (!((scheme == VCPG_SSPRK3 && stage >= 0 && stage < 3) ||
        (scheme == VCPG_LSRK4 && stage >= 0 && stage < 5)))
    return Fail(h, VCPG_E_INVALID, "rk stage: SSP-RK3 stages 0-2, LSRK4 stages 0-4");
  // The stage kernels read the step from device memory.
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_dt, &dt, 8, cudaMemcpyHostToDevice, h->stream));
  const size_t n = (size_t)h->nOwned * 5 * h->KD;
  if (scheme == VCPG_SSPRK3) {
    const double alphaRK[] = {1.0, 3.0 / 4.0, 1.0 / 3.0};
    const double betaRK[] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
    VCPG_CUDA(h, LaunchSspStage(h->d_sol, h->d_solOld, h->d_res, h->d_dt, alphaRK[stage],
                                betaRK[stage], stage == 0, n, h->stream, CaseView{}, 5 * h->KD));
  } else {
    VCPG_CUDA(h, LaunchLsrkStage(h->d_sol, h->d_solOld, h->d_res, h->d_dt, kLsA[stage],
                                 kLsB[stage], n, h->stream, CaseView{}, 5 * h->KD));
  }
  h->launches += 1;
  h->res_valid = false;
  return VCPG_OK;
}

void *vcpg_stream(vcpg_handle *h) { return h ? (void *)h->stream : nullptr; }

int64_t vcpg_launch_count(const vcpg_handle *h) { return h ? h->launches : 0; }

int vcpg_stats(vcpg_handle *h, int64_t *cg_iterations, int64_t *element_solves) {
  if (!h) return VCPG_E_INVALID;
  unsigned long long st[2] = {0, 0};
  VCPG_CUDA(h, cudaMemcpyAsync(st, h->d_cgstats, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cg_iterations) *cg_iterations = (int64_t)st[0];
  if (element_solves) *element_solves = (int64_t)st[1];
  return VCPG_OK;
}

int vcpg_set_open_boundary(vcpg_handle *h, const vcpg_open_boundary *ob,
                           const vcpg_geometry *geom, int32_t p_grid, int32_t dof_location,
                           const double *grid_nodes) {
  return vcpg_set_open_boundary_subfaces(h, ob, nullptr, 0, geom, p_grid, dof_location,
                                         grid_nodes);
}

int vcpg_set_open_boundary_subfaces(vcpg_handle *h, const vcpg_open_boundary *ob,
                                    const vcpg_subface *subfaces, int32_t n_subfaces,
                                    const vcpg_geometry *geom, int32_t p_grid,
                                    int32_t dof_location, const double *grid_nodes) {
  if (!h || !ob || !geom || n_subfaces < 0 || (n_subfaces > 0 && !subfaces))
    return VCPG_E_INVALID;
  if (h->open) return Fail(h, VCPG_E_INVALID, "open boundaries are already configured");
  if (h->nOwned != h->nE)
    return Fail(h, VCPG_E_INVALID, "open boundaries of a partitioned block: "
                                   "vcpg_set_open_boundary_partition");
  if (!SupportsOpenBoundaries(h->K, h->M))
    return Fail(h, VCPG_E_UNSUPPORTED_KM, "no open-boundary kernels for this degree");
  OpenBoundaryHost ob_host;
  std::string err;
  int rc = BuildOpenBoundary(h->prm, *ob, *geom, p_grid, dof_location, grid_nodes, ob_host, err,
                             subfaces, n_subfaces);
  if (rc != VCPG_OK) return Fail(h, rc, err);
  return InstallOpenBoundary(h, ob_host);
}

int vcpg_set_open_boundary_partition(vcpg_handle *h, const vcpg_open_boundary *ob,
                                     const vcpg_subface *subfaces, int32_t n_subfaces,
                                     const int32_t *block_n_elem, const vcpg_geometry *block_geom,
                                     int32_t p_grid, int32_t dof_location,
                                     const double *block_grid_nodes,
                                     const int64_t *local_to_global) {
  if (!h || !ob || !block_n_elem || !block_geom || !local_to_global || n_subfaces < 0 ||
      (n_subfaces > 0 && !subfaces))
    return VCPG_E_INVALID;
  if (h->open) return Fail(h, VCPG_E_INVALID, "open boundaries are already configured");
  if (h->nOwned == h->nE)
    return Fail(h, VCPG_E_INVALID, "declare the partition first (vcpg_set_partition)");
  if (!SupportsOpenBoundaries(h->K, h->M))
    return Fail(h, VCPG_E_UNSUPPORTED_KM, "no open-boundary kernels for this degree");
  vcpg_params bp = h->prm;
  for (int d = 0; d < 3; ++d) bp.n_elem[d] = block_n_elem[d];
  const int64_t nBlock = (int64_t)bp.n_elem[0] * bp.n_elem[1] * bp.n_elem[2];
  for (int64_t l = 0; l < h->nE; ++l)
    if (local_to_global[l] < 0 || local_to_global[l] >= nBlock)
      return Fail(h, VCPG_E_INVALID, "local_to_global: element index outside the block");
  OpenBoundaryHost block, local;
  std::string err;
  int rc = BuildOpenBoundary(bp, *ob, *block_geom, p_grid, dof_location, block_grid_nodes, block,
                             err, subfaces, n_subfaces);
  if (rc != VCPG_OK) return Fail(h, rc, err);
  std::vector<int32_t> nbr((size_t)h->nE * 6);
  VCPG_CUDA(h, cudaMemcpy(nbr.data(), h->d_nbr, sizeof(int32_t) * nbr.size(),
                          cudaMemcpyDeviceToHost));
  SliceOpenBoundary(block, local_to_global, h->nE, h->nOwned, nbr.data(), h->MD, local);
  return InstallOpenBoundary(h, local);
}

int vcpg_boundary_mach_weights(vcpg_handle *h, double *weights, int32_t *counts) {
  if (!h || !counts) return VCPG_E_INVALID;
  for (int f = 0; f < 6; ++f) counts[f] = h->open ? h->cfg[f].count : 0;
  if (!h->open || h->nB == 0 || !weights) return VCPG_OK;   // NULL weights: the counts only
  VCPG_CUDA(h, LaunchBoundary(h->K, h->M, MakeBoundaryArgs(h), h->stream, 1));
  h->launches += 1;
  VCPG_CUDA(h, cudaMemcpyAsync(weights, h->d_bmach, sizeof(double) * h->nB,
                               cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_boundary_rows(vcpg_handle *h, int32_t *block_rows, int32_t *block_last) {
  if (!h || !block_rows || !block_last) return VCPG_E_INVALID;
  if (!h->open) return Fail(h, VCPG_E_INVALID, "no open boundaries");
  for (int b = 0; b < h->nB; ++b) {
    const bool sliced = (size_t)b < h->bBlockRow.size();
    block_rows[b] = sliced ? h->bBlockRow[b] : b;
    block_last[b] = sliced ? h->bBlockLast[b] : -1;
  }
  return VCPG_OK;
}

int vcpg_boundary_local_mach(vcpg_handle *h, double *values) {
  if (!h || !values) return VCPG_E_INVALID;
  if (!h->open || h->nB == 0) return VCPG_OK;
  VCPG_CUDA(h, cudaMemcpyAsync(values, h->d_bmach + h->nB, sizeof(double) * h->nB,
                               cudaMemcpyDeviceToHost, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  return VCPG_OK;
}

int vcpg_set_boundary_outlet_mach(vcpg_handle *h, const double *values) {
  if (!h) return VCPG_E_INVALID;
  if (!values) { h->use_bmachlast = false; return VCPG_OK; }
  if (!h->open || h->nB == 0) return VCPG_OK;
  if (!h->d_bmachlast) {
    cudaError_t e = cudaMalloc((void **)&h->d_bmachlast, sizeof(double) * h->nB);
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, "cudaMalloc outlet Mach numbers");
  }
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_bmachlast, values, sizeof(double) * h->nB,
                               cudaMemcpyHostToDevice, h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  h->use_bmachlast = true;
  return VCPG_OK;
}

int vcpg_set_boundary_mach_sums(vcpg_handle *h, const double *sums) {
  if (!h) return VCPG_E_INVALID;
  if (!sums) { h->use_bmach_sums = false; return VCPG_OK; }
  if (!h->d_bmachsums) {
    cudaError_t e = cudaMalloc((void **)&h->d_bmachsums, 6 * sizeof(double));
    if (e != cudaSuccess) return Fail(h, VCPG_E_OOM, "cudaMalloc Mach sums");
  }
  VCPG_CUDA(h, cudaMemcpyAsync(h->d_bmachsums, sums, 6 * sizeof(double), cudaMemcpyHostToDevice,
                               h->stream));
  VCPG_CUDA(h, cudaStreamSynchronize(h->stream));
  h->use_bmach_sums = true;
  return VCPG_OK;
}

int vcpg_residual_part(vcpg_handle *h, int32_t part) {
  if (!h || (part != 0 && part != 1)) return VCPG_E_INVALID;
  if (h->remoteLast && !h->use_bmachlast)
    return Fail(h, VCPG_E_INVALID, "outlet Mach numbers of subfaces whose last face lies on "
                                   "another rank: vcpg_set_boundary_outlet_mach first");
  if (h->nOwned == h->nE)
    return Fail(h, VCPG_E_INVALID, "residual parts: a partitioned handle only");
  const int64_t nO = h->nOwned, nF = h->nFace, fR = h->fluxReady, rR = h->resReady;
  int n = 0;
  auto launch = [&](int phase, int64_t first, int64_t count) -> int {
    if (count <= 0) return VCPG_OK;
    ResidualArgs a = MakeResidualArgs(h, nullptr, nullptr);
    a.n_elem = a.n_face_elem = (int)count;
    if (phase == 1) a.face_first = (int)first; else a.res_first = (int)first;
    VCPG_CUDA(h, LaunchResidual(h->K, h->M, a, h->stream, phase));
    ++n;
    return VCPG_OK;
  };
  int rc = VCPG_OK;
  if (part == 0) {
    // No ghost state needed: the boundary kernels (the handle's own boundary
    // faces), the face fluxes of the owned elements whose lower neighbours are
    // owned, the residuals of the owned elements without ghost neighbours.
    if (h->open && h->nB > 0) {
      VCPG_CUDA(h, LaunchBoundary(h->K, h->M, MakeBoundaryArgs(h), h->stream));
      n += 2;
    }
    if ((rc = launch(1, 0, fR)) || (rc = launch(2, 0, rR))) return rc;
    h->launches += n;
    h->res_valid = false;
    return VCPG_OK;
  }
  // After the ghost states are in: the remaining owned and the face ghosts' face
  // fluxes, the remaining residuals.
  if ((rc = launch(1, fR, nF - fR)) || (rc = launch(2, rR, nO - rR))) return rc;
  h->launches += n;
  rc = CheckStatus(h);
  h->res_valid = rc == VCPG_OK;
  return rc;
}

}  // extern "C"
