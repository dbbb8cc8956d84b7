// Served ensemble (include/vcp3d_b200.h, vcpg_ensemble_*): many cases resident
// on one GPU in per-degree buckets, stepped together, joining and leaving
// between steps.
//
// A bucket owns pre-allocated arenas -- elements (state, RK register, residual,
// metrics, neighbours, case slot), characteristic boundary faces, sponge
// elements -- and a table of case slots. A case occupies one contiguous range
// of each arena (first fit) and one slot. Every kernel of a bucket step runs
// over the arenas' high-water marks and skips elements / faces whose case is not
// in the state that launch processes (dg_residual.cuh CaseView), so a step is a
// fixed launch sequence captured once as a CUDA graph (re-captured when a high
// water mark moves):
//
//   residual of the pending cases (new arrivals), CFL step of pending and running
//   cases, per-case finalize (pending -> running; running -> done after the
//   target steps), then the RK stages with the residuals of the running cases.
//
// Streams: each bucket steps on its own stream, so different degrees overlap on
// the device. Uploads of arriving cases and the clearing of retired ranges go on
// one upload stream; the bucket stream waits for an arrival's upload before the
// case's state becomes pending (on the bucket stream, so a case never starts in
// the middle of a step). Results of finished cases are read on a copy stream:
// kernels never write a done case, so the copy does not wait for running steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/vcp3d_b200.h"
#include "dg_boundary.cuh"
#include "dg_residual.cuh"
#include "kernels.h"
#include "open_boundary.h"

using namespace vcpg;

namespace {

const double kLsA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kLsB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};

// First-fit allocator of index ranges in [0, capacity).
class RangeAllocator {
 public:
  void Reset(int64_t cap) {
    free_.clear();
    cap_ = cap;
    if (cap > 0) free_[0] = cap;
  }
  bool Alloc(int64_t n, int64_t *first) {
    if (n == 0) { *first = 0; return true; }
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *first = it->first;
        const int64_t rest = it->second - n, start = it->first + n;
        free_.erase(it);
        if (rest > 0) free_[start] = rest;
        return true;
      }
    }
    return false;
  }
  void Free(int64_t first, int64_t n) {
    if (n == 0) return;
    auto next = free_.lower_bound(first);
    int64_t s = first, len = n;
    if (next != free_.end() && next->first == first + n) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == first) {
        s = prev->first;
        len += prev->second;
        free_.erase(prev);
      }
    }
    free_[s] = len;
  }
  // End of the last allocated range.
  int64_t HighWater() const {
    if (free_.empty()) return cap_;
    auto last = std::prev(free_.end());
    return (last->first + last->second == cap_) ? last->first : cap_;
  }

 private:
  std::map<int64_t, int64_t> free_;
  int64_t cap_ = 0;
};

struct HostCase {
  int deg = 0, slot = -1;
  int64_t eFirst = 0, nE = 0, bFirst = 0, nB = 0, sFirst = 0, nS = 0;
  bool reported = false;
  // Recorded on the bucket stream after the slot became pending: until it has
  // completed, the slot's device state may still be its previous occupant's.
  cudaEvent_t admitted = nullptr;
};

struct Bucket {
  int deg = -1, K = 0, M = 0, KD = 0, MD = 0, M2 = 0;
  int64_t capE = 0, capB = 0, capS = 0;
  int capC = 0;
  cudaStream_t stream = nullptr;
  // Element arena.
  double *sol = nullptr, *solOld = nullptr, *res = nullptr, *vol = nullptr, *face = nullptr,
         *sc = nullptr;
  int *nbr = nullptr, *elemCase = nullptr, *spongeIdx = nullptr;
  void *fflux = nullptr;  // Min-face fluxes (FaceFluxKernel)
  // Boundary-face and sponge arenas.
  int *bface = nullptr;
  double *bpresc = nullptr, *btrace = nullptr, *bmach = nullptr, *bflux = nullptr;
  double *pc = nullptr, *dlq = nullptr;
  double *dampFn = nullptr, *dampSt = nullptr, *cml = nullptr;
  double *center = nullptr;  // [K^3] 3-D basis at the element centre
  // Case slots.
  int *state = nullptr, *target = nullptr, *done = nullptr, *status = nullptr;
  double *par = nullptr, *dt = nullptr, *simTime = nullptr;
  unsigned long long *dtBits = nullptr, *cgStats = nullptr;
  BlockFaceCfg *cfgs = nullptr;
  RangeAllocator elems, bfaces, sponge;
  std::vector<int64_t> slotCase;  // case id per slot, -1 = free
  int resident = 0;
  bool opsReady = false, pcReady = false;
  // Solution-DOF positions of the operator table (1 LGL, 0 equidistant; the grid
  // node positions do not enter it): the bucket's first case fixes them, since
  // the time step evaluates the basis at the nodal DOFs.
  int dofLoc = -1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t graphE = -1, graphB = -1;
  int graphLaunches = 0;
  // Steps in flight on the bucket stream (a step waits when kMaxInflight are queued).
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int evHead = 0, evCount = 0;
};

constexpr int kMaxInflight = 2;

}  // namespace

struct vcpg_ensemble {
  vcpg_ensemble_config cfg{};
  Bucket b[8];
  cudaStream_t upload = nullptr, copy = nullptr;
  std::map<int64_t, HostCase> cases;
  std::vector<int> hostState;
  int64_t nextId = 1, launches = 0;
  std::string err;
};

namespace {

int Fail(vcpg_ensemble *e, int code, const std::string &msg) {
  if (e) e->err = msg;
  return code;
}

#define ENS_CUDA(e, call)                                                            \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return Fail((e), VCPG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int IntegrationPoints(int deg) {
  // nPolyIntRule = 3p, M = nPolyIntRule / 2 + 1 (src/StandardElementClass.cpp:665).
  return (3 * deg) / 2 + 1;
}

int64_t ElementBytes(int K, int M) {
  const int64_t KD = (int64_t)K * K * K, MD = (int64_t)M * M * M, M2 = (int64_t)M * M;
  return 8 * (3 * 5 * KD + 10 * MD + 6 * 13 * M2 + 15 + 3 * 20 * M2) + 4 * (6 + 2);
}

int64_t BFaceBytes(int M) { return 8 * (4 + 2 * 4 * 5 * (int64_t)M * M + 2) + 4 * kBfStride; }

int64_t SpongeBytes(int M) { return 8 * (8 * (int64_t)M * M * M + 6); }

}  // namespace

namespace {

void FreeBucket(Bucket &b) {
  for (cudaEvent_t ev : b.ev)
    if (ev) cudaEventDestroy(ev);
  if (b.exec) cudaGraphExecDestroy(b.exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  void *bufs[] = {b.fflux, b.sol, b.solOld, b.res, b.vol, b.face, b.sc, b.nbr, b.elemCase, b.spongeIdx,
                  b.bface, b.bpresc, b.btrace, b.bmach, b.bflux, b.pc, b.dlq, b.dampFn,
                  b.dampSt, b.cml, b.state, b.target, b.done, b.status, b.par, b.dt,
                  b.simTime, b.dtBits, b.cgStats, b.cfgs, b.center};
  for (void *p : bufs)
    if (p) cudaFree(p);
  if (b.stream) cudaStreamDestroy(b.stream);
  b = Bucket{};
}

int AllocBucket(vcpg_ensemble *e, Bucket &b, int deg, int64_t capE, int64_t capB, int64_t capS,
                int capC) {
  b.deg = deg;
  b.K = deg + 1;
  b.M = IntegrationPoints(deg);
  b.KD = b.K * b.K * b.K;
  b.MD = b.M * b.M * b.M;
  b.M2 = b.M * b.M;
  b.capE = capE; b.capB = capB; b.capS = capS; b.capC = capC;
  // Buckets hold degrees whose kernels run in shared memory and have the
  // open-boundary kernels (up to degree 6).
  if (!Supported(b.K, b.M) || !SupportsOpenBoundaries(b.K, b.M) ||
      ResidualScratchBytes(b.K, b.M, 1) > 0)
    return Fail(e, VCPG_E_UNSUPPORTED_KM, "no kernel for degree " + std::to_string(deg));
  ENS_CUDA(e, ConfigureResidual(b.K, b.M));
  ENS_CUDA(e, cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  for (int i = 0; i < kMaxInflight; ++i)
    ENS_CUDA(e, cudaEventCreateWithFlags(&b.ev[i], cudaEventDisableTiming));
  auto alloc = [&](void **p, size_t bytes) -> int {
    if (bytes == 0) return VCPG_OK;
    cudaError_t err = cudaMalloc(p, bytes);
    if (err != cudaSuccess)
      return Fail(e, VCPG_E_OOM, std::string("cudaMalloc bucket arena: ") + cudaGetErrorString(err));
    return VCPG_OK;
  };
  const size_t E = (size_t)capE, B = (size_t)capB, S = (size_t)capS, C = (size_t)capC;
  const size_t nState = E * 5 * b.KD;
  int rc;
  if ((rc = alloc((void **)&b.sol, 8 * nState)) || (rc = alloc((void **)&b.solOld, 8 * nState)) ||
      (rc = alloc((void **)&b.res, 8 * nState)) ||
      (rc = alloc((void **)&b.fflux, E * FaceFluxBytesPerElement(b.K, b.M))) ||
      (rc = alloc((void **)&b.vol, 8 * E * 10 * b.MD)) ||
      (rc = alloc((void **)&b.face, 8 * E * 6 * 13 * b.M2)) ||
      (rc = alloc((void **)&b.sc, 8 * E * 15)) || (rc = alloc((void **)&b.nbr, 4 * E * 6)) ||
      (rc = alloc((void **)&b.elemCase, 4 * E)) || (rc = alloc((void **)&b.spongeIdx, 4 * E)) ||
      (rc = alloc((void **)&b.bface, 4 * B * kBfStride)) ||
      (rc = alloc((void **)&b.bpresc, 8 * B * kPrescStride)) ||
      (rc = alloc((void **)&b.btrace, 8 * B * 4 * 5 * b.M2)) ||
      (rc = alloc((void **)&b.bmach, 8 * 2 * B)) ||
      (rc = alloc((void **)&b.bflux, 8 * B * 4 * 5 * b.M2)) ||
      (rc = alloc((void **)&b.pc, 8 * (size_t)b.M2 * b.M2)) ||
      (rc = alloc((void **)&b.dlq, 8 * (size_t)b.M * b.M)) ||
      (rc = alloc((void **)&b.dampFn, 8 * S * 3 * b.MD)) ||
      (rc = alloc((void **)&b.dampSt, 8 * S * 5 * b.MD)) ||
      (rc = alloc((void **)&b.cml, 8 * S * 6)) || (rc = alloc((void **)&b.state, 4 * C)) ||
      (rc = alloc((void **)&b.target, 4 * C)) || (rc = alloc((void **)&b.done, 4 * C)) ||
      (rc = alloc((void **)&b.status, 4 * 4)) || (rc = alloc((void **)&b.par, 8 * C * kCasePar)) ||
      (rc = alloc((void **)&b.dt, 8 * C)) || (rc = alloc((void **)&b.simTime, 8 * C)) ||
      (rc = alloc((void **)&b.dtBits, 8 * C)) || (rc = alloc((void **)&b.cgStats, 8 * 2)) ||
      (rc = alloc((void **)&b.cfgs, sizeof(BlockFaceCfg) * C * 6)) ||
      (rc = alloc((void **)&b.center, 8 * (size_t)b.KD)))
    return rc;
  // Unused elements and faces carry case -1; every slot starts free.
  ENS_CUDA(e, cudaMemsetAsync(b.elemCase, 0xFF, 4 * E, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.spongeIdx, 0xFF, 4 * E, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.nbr, 0xFF, 4 * E * 6, b.stream));
  if (B) ENS_CUDA(e, cudaMemsetAsync(b.bface, 0xFF, 4 * B * kBfStride, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.state, 0, 4 * C, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.done, 0, 4 * C, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.status, 0, 16, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.cgStats, 0, 16, b.stream));
  ENS_CUDA(e, cudaMemsetAsync(b.cfgs, 0, sizeof(BlockFaceCfg) * C * 6, b.stream));
  std::vector<unsigned long long> big(C, (unsigned long long)0x4202a05f20000000ULL);  // 1e10
  ENS_CUDA(e, cudaMemcpyAsync(b.dtBits, big.data(), 8 * C, cudaMemcpyHostToDevice, b.stream));
  ENS_CUDA(e, cudaStreamSynchronize(b.stream));
  b.elems.Reset(capE);
  b.bfaces.Reset(capB);
  b.sponge.Reset(capS);
  b.slotCase.assign(C, -1);
  return VCPG_OK;
}

ResidualArgs BucketResidualArgs(const vcpg_ensemble *e, const Bucket &b, int require) {
  ResidualArgs a{};
  a.sol = b.sol;
  a.res = b.res;
  a.vol_metric = b.vol;
  a.face_metric = b.face;
  a.elem_scalars = b.sc;
  a.nbr = b.nbr;
  a.n_elem = (int)b.elems.HighWater();
  a.tau_num = (double)(b.K * b.K) * e->cfg.rel_penalty;
  a.theta_sym = e->cfg.theta_sym;
  a.riemann = e->cfg.riemann;
  a.metric_compat = e->cfg.metric_index_compat;
  a.status = b.status;
  a.cg_stats = b.cgStats;
  a.mixed = e->cfg.precision == VCPG_MIXED ? 1 : 0;
  a.cg_tol = a.mixed ? 1.e-5 : 1.e-10;
  a.open = (b.capB > 0 || b.capS > 0) ? 1 : 0;
  a.bflux = b.bflux;
  a.sponge_idx = b.spongeIdx;
  a.damp_fn = b.dampFn;
  a.damp_state = b.dampSt;
  a.cml = b.cml;
  a.cml_on = b.capS > 0 ? 1 : 0;
  a.cases = CaseView{b.elemCase, b.state, b.par, require};
  a.face_flux = b.fflux;
  a.center = b.center;
  return a;
}

BoundaryArgs BucketBoundaryArgs(const vcpg_ensemble *e, const Bucket &b, int require) {
  BoundaryArgs a{};
  a.sol = b.sol;
  a.face_metric = b.face;
  a.elem_scalars = b.sc;
  a.bface = b.bface;
  a.bpresc = b.bpresc;
  a.pc = b.pc;
  a.dlq = b.dlq;
  a.btrace = b.btrace;
  a.bmach = b.bmach;
  a.bmach_local = b.bmach + b.capB;   // [capB, 2 capB)
  a.bflux = b.bflux;
  a.nB = (int)b.bfaces.HighWater();
  a.tau_num = (double)(b.K * b.K) * e->cfg.rel_penalty;
  a.theta_sym = e->cfg.theta_sym;
  a.riemann = e->cfg.riemann;
  a.metric_compat = e->cfg.metric_index_compat;
  a.cfgs = b.cfgs;
  a.case_state = b.state;
  a.case_par = b.par;
  a.require = require;
  return a;
}

// One residual of the cases in state `require`: boundary kernels, residual kernel.
int EnqueueBucketResidual(vcpg_ensemble *e, Bucket &b, int require, int *launches) {
  if (b.bfaces.HighWater() > 0) {
    ENS_CUDA(e, LaunchBoundary(b.K, b.M, BucketBoundaryArgs(e, b, require), b.stream));
    *launches += 2;
  }
  ENS_CUDA(e, LaunchResidual(b.K, b.M, BucketResidualArgs(e, b, require), b.stream));
  *launches += 2;
  return VCPG_OK;
}

// The launch sequence of one bucket step (captured into the bucket's graph).
int EnqueueBucketStep(vcpg_ensemble *e, Bucket &b, int *launches) {
  const int64_t hwE = b.elems.HighWater();
  const size_t n = (size_t)hwE * 5 * b.KD;
  int rc = EnqueueBucketResidual(e, b, kCasePending, launches);
  if (rc) return rc;
  TimeStepArgs t{};
  t.sol = b.sol;
  t.elem_scalars = b.sc;
  t.n_elem = (int)hwE;
  t.n_poly = b.deg;
  t.dt_bits = b.dtBits;
  t.status = b.status;
  t.cases = CaseView{b.elemCase, b.state, b.par, kCaseRunning};
  ENS_CUDA(e, LaunchTimeStep(b.K, b.M, t, b.stream));
  ENS_CUDA(e, LaunchEnsembleFinalize(b.capC, b.state, b.target, b.done, b.dtBits, b.dt, b.simTime,
                                     b.stream));
  *launches += 2;
  const CaseView cv{b.elemCase, b.state, b.par, kCaseRunning};
  if (e->cfg.scheme == VCPG_SSPRK3) {
    const double alphaRK[] = {1.0, 3.0 / 4.0, 1.0 / 3.0};
    const double betaRK[] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
    for (int s = 0; s < 3; ++s) {
      ENS_CUDA(e, LaunchSspStage(b.sol, b.solOld, b.res, b.dt, alphaRK[s], betaRK[s], s == 0, n,
                                 b.stream, cv, 5 * b.KD));
      *launches += 1;
      if ((rc = EnqueueBucketResidual(e, b, kCaseRunning, launches))) return rc;
    }
  } else {
    for (int s = 0; s < 5; ++s) {
      ENS_CUDA(e, LaunchLsrkStage(b.sol, b.solOld, b.res, b.dt, kLsA[s], kLsB[s], n, b.stream, cv,
                                  5 * b.KD));
      *launches += 1;
      if ((rc = EnqueueBucketResidual(e, b, kCaseRunning, launches))) return rc;
    }
  }
  return VCPG_OK;
}

int CaptureBucketStep(vcpg_ensemble *e, Bucket &b) {
  if (b.exec) { cudaGraphExecDestroy(b.exec); b.exec = nullptr; }
  if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
  ENS_CUDA(e, cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
  int launches = 0;
  int rc = EnqueueBucketStep(e, b, &launches);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(b.stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (ce != cudaSuccess) return Fail(e, VCPG_E_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
  b.graph = g;
  ENS_CUDA(e, cudaGraphInstantiate(&b.exec, g, 0));
  b.graphE = b.elems.HighWater();
  b.graphB = b.bfaces.HighWater();
  b.graphLaunches = launches;
  return VCPG_OK;
}

int CheckBucketStatus(vcpg_ensemble *e, Bucket &b) {
  int st[4] = {0, 0, 0, 0};
  ENS_CUDA(e, cudaMemcpyAsync(st, b.status, sizeof(st), cudaMemcpyDeviceToHost, b.stream));
  ENS_CUDA(e, cudaStreamSynchronize(b.stream));
  if (st[0] || st[1] || st[2] || st[3]) {
    ENS_CUDA(e, cudaMemsetAsync(b.status, 0, sizeof(st), b.stream));
    if (st[3]) return Fail(e, VCPG_E_CUDA, "an asynchronous copy into shared memory did not "
                                           "complete within its wait bound");
    if (st[0]) return Fail(e, VCPG_E_CG_NOCONV, "mass-matrix CG reached 100 iterations (degree " +
                                                   std::to_string(b.deg) + ")");
    if (st[2]) return Fail(e, VCPG_E_NEG_A2, "negative or not-a-number square speed of sound in the time step");
    return Fail(e, VCPG_E_INVALID, "physical boundary face without a boundary condition");
  }
  return VCPG_OK;
}

}  // namespace

extern "C" {

int64_t vcpg_ensemble_footprint(int32_t n_poly, int32_t n_int_1d, int64_t n_elem,
                                int64_t n_bfaces, int64_t n_sponge) {
  const int K = n_poly + 1, M = n_int_1d;
  return n_elem * ElementBytes(K, M) + n_bfaces * BFaceBytes(M) + n_sponge * SpongeBytes(M);
}

const char *vcpg_ensemble_last_error(const vcpg_ensemble *ens) {
  return ens ? ens->err.c_str() : "null ensemble";
}

int vcpg_ensemble_destroy(vcpg_ensemble *ens) {
  if (!ens) return VCPG_OK;
  for (auto &kv : ens->cases)
    if (kv.second.admitted) cudaEventDestroy(kv.second.admitted);
  for (Bucket &b : ens->b)
    if (b.deg >= 0) FreeBucket(b);
  if (ens->upload) cudaStreamDestroy(ens->upload);
  if (ens->copy) cudaStreamDestroy(ens->copy);
  delete ens;
  return VCPG_OK;
}

int vcpg_ensemble_create(const vcpg_ensemble_config *cfg, vcpg_ensemble **out) {
  if (!cfg || !out) return VCPG_E_INVALID;
  *out = nullptr;
  vcpg_ensemble *e = new vcpg_ensemble();
  e->cfg = *cfg;
  *out = e;
  if (cfg->precision != VCPG_FP64 && cfg->precision != VCPG_MIXED)
    return Fail(e, VCPG_E_INVALID, "precision must be VCPG_FP64 or VCPG_MIXED");
  if (cfg->scheme != VCPG_SSPRK3 && cfg->scheme != VCPG_LSRK4)
    return Fail(e, VCPG_E_INVALID, "unknown scheme");
  if (cfg->max_cases < 1) return Fail(e, VCPG_E_INVALID, "max_cases must be positive");
  ENS_CUDA(e, cudaStreamCreateWithFlags(&e->upload, cudaStreamNonBlocking));
  ENS_CUDA(e, cudaStreamCreateWithFlags(&e->copy, cudaStreamNonBlocking));
  for (int p = 1; p <= 6; ++p) {
    if (cfg->bucket_elems[p] <= 0) continue;
    if (cfg->bucket_bfaces[p] < 0 || cfg->bucket_sponge[p] < 0)
      return Fail(e, VCPG_E_INVALID, "negative bucket capacity");
    int rc = AllocBucket(e, e->b[p], p, cfg->bucket_elems[p], cfg->bucket_bfaces[p],
                         cfg->bucket_sponge[p], cfg->max_cases);
    if (rc) return rc;
  }
  return VCPG_OK;
}

int vcpg_ensemble_submit(vcpg_ensemble *ens, const vcpg_params *params,
                         const vcpg_operators *ops, const vcpg_geometry *geom,
                         const double *modal_state, int32_t n_steps,
                         const vcpg_open_boundary *ob, int32_t p_grid, int32_t dof_location,
                         const double *grid_nodes, int64_t *case_id) {
  return vcpg_ensemble_submit_subfaces(ens, params, ops, geom, modal_state, n_steps, ob, nullptr,
                                       0, p_grid, dof_location, grid_nodes, case_id);
}

int vcpg_ensemble_submit_subfaces(vcpg_ensemble *ens, const vcpg_params *params,
                                  const vcpg_operators *ops, const vcpg_geometry *geom,
                                  const double *modal_state, int32_t n_steps,
                                  const vcpg_open_boundary *ob, const vcpg_subface *subfaces,
                                  int32_t n_subfaces, int32_t p_grid, int32_t dof_location,
                                  const double *grid_nodes, int64_t *case_id) {
  if (!ens || !params || !ops || !geom || !modal_state || !case_id || n_steps < 0 ||
      n_subfaces < 0 || (n_subfaces > 0 && (!subfaces || !ob)))
    return VCPG_E_INVALID;
  vcpg_ensemble *e = ens;
  if (params->sgs_model != VCPG_SGS_NONE)
    return Fail(e, VCPG_E_INVALID, "subgrid-scale models run on single-case handles");
  const int deg = params->n_poly;
  if (deg < 1 || deg > 6 || e->b[deg].deg != deg)
    return Fail(e, VCPG_E_INVALID, "no bucket for degree " + std::to_string(deg));
  Bucket &b = e->b[deg];
  if (params->n_int_1d != b.M)
    return Fail(e, VCPG_E_INVALID, "integration rule differs from the bucket's (3p)");
  if (params->precision != e->cfg.precision || params->riemann != e->cfg.riemann ||
      params->metric_index_compat != e->cfg.metric_index_compat ||
      params->theta_sym != e->cfg.theta_sym || params->rel_penalty != e->cfg.rel_penalty)
    return Fail(e, VCPG_E_INVALID, "case settings differ from the ensemble's shared settings");
  const int solLgl =
      (dof_location == VCPG_DOFS_LGL || dof_location == VCPG_DOFS_LGL_GRID_EQUI) ? 1 : 0;
  if (b.opsReady && solLgl != b.dofLoc)
    return Fail(e, VCPG_E_INVALID,
                "solution-DOF positions differ from the bucket's (its first case fixed them)");
  const int64_t nE = (int64_t)params->n_elem[0] * params->n_elem[1] * params->n_elem[2];
  if (nE <= 0) return Fail(e, VCPG_E_INVALID, "invalid element count");
  const int KD = b.KD, MD = b.MD, M2 = b.M2;

  // Sizes first (cheap), so that a refused case costs no set-up work.
  int64_t nB = 0, nS = 0;
  if (ob) {
    // A block face with subfaces takes its conditions from them (none periodic).
    bool sub[6] = {false, false, false, false, false, false};
    for (int32_t s = 0; s < n_subfaces; ++s)
      if (subfaces[s].face >= 0 && subfaces[s].face < 6) sub[subfaces[s].face] = true;
    for (int64_t e2 = 0; e2 < nE; ++e2)
      for (int f = 0; f < 6; ++f)
        if (geom->neighbors[e2 * 6 + f] < 0 && (ob->bc[f] != VCPG_BC_NONE || sub[f])) ++nB;
    const int n3[3] = {params->n_elem[0], params->n_elem[1], params->n_elem[2]};
    for (int k = 0; k < n3[2]; ++k)
      for (int j = 0; j < n3[1]; ++j)
        for (int i = 0; i < n3[0]; ++i) {
          const int idx[3] = {i, j, k};
          bool in = false;
          for (int d = 0; d < 3; ++d)
            in = in || idx[d] < ob->sponge_elems[2 * d] ||
                 idx[d] >= n3[d] - ob->sponge_elems[2 * d + 1];
          if (in) ++nS;
        }
  } else {
    for (int64_t i = 0; i < nE * 6; ++i)
      if (geom->neighbors[i] < 0)
        return Fail(e, VCPG_E_INVALID, "the case has boundary faces but no boundary conditions");
  }
  if ((nB > 0 && b.capB == 0) || (nS > 0 && b.capS == 0))
    return Fail(e, VCPG_E_ADMISSION, "the bucket has no boundary-face or sponge arena");

  // Admission: a free slot and contiguous ranges in the three arenas.
  int slot = -1;
  for (int s = 0; s < b.capC; ++s)
    if (b.slotCase[s] < 0) { slot = s; break; }
  int64_t eFirst = 0, bFirst = 0, sFirst = 0;
  if (slot < 0) return Fail(e, VCPG_E_ADMISSION, "no free case slot");
  if (!b.elems.Alloc(nE, &eFirst)) return Fail(e, VCPG_E_ADMISSION, "no room for the elements");
  if (!b.bfaces.Alloc(nB, &bFirst)) {
    b.elems.Free(eFirst, nE);
    return Fail(e, VCPG_E_ADMISSION, "no room for the boundary faces");
  }
  if (!b.sponge.Alloc(nS, &sFirst)) {
    b.elems.Free(eFirst, nE);
    b.bfaces.Free(bFirst, nB);
    return Fail(e, VCPG_E_ADMISSION, "no room for the sponge elements");
  }
  auto rollback = [&]() {
    b.elems.Free(eFirst, nE);
    b.bfaces.Free(bFirst, nB);
    b.sponge.Free(sFirst, nS);
  };

  // Open boundaries of this case (host set-up), with local indices.
  OpenBoundaryHost obh;
  if (ob) {
    std::string err;
    int rc = BuildOpenBoundary(*params, *ob, *geom, p_grid, dof_location, grid_nodes, obh, err,
                               subfaces, n_subfaces);
    if (rc) { rollback(); return Fail(e, rc, err); }
    if (obh.nB != nB || obh.nS != nS) {
      rollback();
      return Fail(e, VCPG_E_INVALID, "boundary-face or sponge count mismatch");
    }
  }

  // Bucket-wide operators on first use.
  if (!b.opsReady) {
    cudaError_t ce = UploadOperatorTable(ops, b.K, b.M);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(b.center, ops->basis_center, 8 * (size_t)b.KD, cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) { rollback(); return Fail(e, VCPG_E_CUDA, cudaGetErrorString(ce)); }
    b.opsReady = true;
    b.dofLoc = solLgl;
  }
  if (nB > 0 && !b.pcReady) {
    cudaError_t ce = cudaMemcpy(b.pc, obh.pc.data(), 8 * obh.pc.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(b.dlq, obh.dlq.data(), 8 * obh.dlq.size(), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) { rollback(); return Fail(e, VCPG_E_CUDA, cudaGetErrorString(ce)); }
    b.pcReady = true;
  }

  // Host copies with arena offsets.
  std::vector<int32_t> nbr(geom->neighbors, geom->neighbors + nE * 6);
  if (ob) nbr = obh.nbrCode;
  for (auto &v : nbr) v = v >= 0 ? (int32_t)(v + eFirst) : (v <= -2 ? (int32_t)(v - bFirst) : v);
  std::vector<int32_t> ecase(nE, slot), sidx(nE, -1);
  if (ob)
    for (int64_t i = 0; i < nE; ++i)
      sidx[i] = obh.spongeIdx[i] >= 0 ? (int32_t)(obh.spongeIdx[i] + sFirst) : -1;
  std::vector<int> brows(obh.bface);
  for (int64_t r = 0; r < nB; ++r) {
    brows[r * kBfStride + kBfElem] += (int)eFirst;
    brows[r * kBfStride + kBfCase] = slot;
    if (brows[r * kBfStride + kBfLast] >= 0) brows[r * kBfStride + kBfLast] += (int)bFirst;
  }
  BlockFaceCfg cfgs[6];
  for (int f = 0; f < 6; ++f) {
    cfgs[f] = obh.cfg[f];
    cfgs[f].first += (int)bFirst;
  }
  double par[kCasePar] = {0.0};
  par[kParMu] = params->mu;
  par[kParPRef] = params->p_ref;
  par[kParURef] = params->u_ref;
  par[kParRhoRef] = params->rho_ref;
  par[kParCfl] = params->cfl;
  const int zero = 0, tgt = n_steps;
  const double zeroD = 0.0;

  // Uploads on the upload stream (pageable copies: this thread waits for them,
  // the buckets keep computing).
  cudaStream_t up = e->upload;
  auto cp = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, up) : cudaSuccess;
  };
  cudaError_t ce = cudaSuccess;
  const size_t E = (size_t)nE;
  if (ce == cudaSuccess) ce = cp(b.sol + (size_t)eFirst * 5 * KD, modal_state, 8 * E * 5 * KD);
  if (ce == cudaSuccess) ce = cp(b.vol + (size_t)eFirst * 10 * MD, geom->vol_metric, 8 * E * 10 * MD);
  if (ce == cudaSuccess)
    ce = cp(b.face + (size_t)eFirst * 6 * 13 * M2, geom->face_metric, 8 * E * 6 * 13 * M2);
  if (ce == cudaSuccess) ce = cp(b.sc + (size_t)eFirst * 15, geom->elem_scalars, 8 * E * 15);
  if (ce == cudaSuccess) ce = cp(b.nbr + (size_t)eFirst * 6, nbr.data(), 4 * E * 6);
  if (ce == cudaSuccess) ce = cp(b.spongeIdx + eFirst, sidx.data(), 4 * E);
  if (ce == cudaSuccess && nB) ce = cp(b.bface + (size_t)bFirst * kBfStride, brows.data(), 4 * brows.size());
  if (ce == cudaSuccess && nB)
    ce = cp(b.bpresc + (size_t)bFirst * kPrescStride, obh.bpresc.data(), 8 * obh.bpresc.size());
  if (ce == cudaSuccess && nS) ce = cp(b.dampFn + (size_t)sFirst * 3 * MD, obh.dampFn.data(), 8 * obh.dampFn.size());
  if (ce == cudaSuccess && nS) ce = cp(b.dampSt + (size_t)sFirst * 5 * MD, obh.dampState.data(), 8 * obh.dampState.size());
  if (ce == cudaSuccess && nS) ce = cp(b.cml + (size_t)sFirst * 6, obh.cml.data(), 8 * obh.cml.size());
  if (ce == cudaSuccess) ce = cp(b.cfgs + (size_t)slot * 6, cfgs, sizeof(cfgs));
  if (ce == cudaSuccess) ce = cp(b.par + (size_t)slot * kCasePar, par, sizeof(par));
  if (ce == cudaSuccess) ce = cp(b.target + slot, &tgt, 4);
  if (ce == cudaSuccess) ce = cp(b.done + slot, &zero, 4);
  if (ce == cudaSuccess) ce = cp(b.simTime + slot, &zeroD, 8);
  // The case slot goes last: kernels only touch elements whose slot is pending
  // or running, and the slot becomes pending on the bucket stream below.
  if (ce == cudaSuccess) ce = cp(b.elemCase + eFirst, ecase.data(), 4 * E);
  cudaEvent_t ev = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventRecord(ev, up);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b.stream, ev, 0);
  const int pending = kCasePending;
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(b.state + slot, &pending, 4, cudaMemcpyHostToDevice, b.stream);
  if (ev) cudaEventDestroy(ev);
  cudaEvent_t admitted = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&admitted, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventRecord(admitted, b.stream);
  if (ce != cudaSuccess) {
    if (admitted) cudaEventDestroy(admitted);
    rollback();
    return Fail(e, VCPG_E_CUDA, cudaGetErrorString(ce));
  }

  const int64_t id = e->nextId++;
  HostCase hc;
  hc.deg = deg; hc.slot = slot;
  hc.eFirst = eFirst; hc.nE = nE; hc.bFirst = bFirst; hc.nB = nB; hc.sFirst = sFirst; hc.nS = nS;
  hc.admitted = admitted;
  e->cases[id] = hc;
  b.slotCase[slot] = id;
  b.resident += 1;
  *case_id = id;
  return VCPG_OK;
}

int vcpg_ensemble_step(vcpg_ensemble *ens) {
  if (!ens) return VCPG_E_INVALID;
  vcpg_ensemble *e = ens;
  for (Bucket &b : e->b) {
    if (b.deg < 0 || b.resident == 0) continue;
    if (!b.exec || b.graphE != b.elems.HighWater() || b.graphB != b.bfaces.HighWater()) {
      int rc = CaptureBucketStep(e, b);
      if (rc) return rc;
    }
    // Bound the queue: wait for the oldest step when kMaxInflight are in flight.
    while (b.evCount > 0 && cudaEventQuery(b.ev[b.evHead]) == cudaSuccess) {
      b.evHead = (b.evHead + 1) % kMaxInflight;
      --b.evCount;
    }
    if (b.evCount == kMaxInflight) {
      ENS_CUDA(e, cudaEventSynchronize(b.ev[b.evHead]));
      b.evHead = (b.evHead + 1) % kMaxInflight;
      --b.evCount;
    }
    ENS_CUDA(e, cudaGraphLaunch(b.exec, b.stream));
    ENS_CUDA(e, cudaEventRecord(b.ev[(b.evHead + b.evCount) % kMaxInflight], b.stream));
    ++b.evCount;
    e->launches += b.graphLaunches;
  }
  return VCPG_OK;
}

int vcpg_ensemble_poll(vcpg_ensemble *ens, int64_t *done_ids, int32_t max_ids, int32_t *n_done) {
  if (!ens || !n_done || (max_ids > 0 && !done_ids)) return VCPG_E_INVALID;
  vcpg_ensemble *e = ens;
  *n_done = 0;
  for (Bucket &b : e->b) {
    if (b.deg < 0 || b.resident == 0) continue;
    // The state words are read while steps may run: a done case is final.
    e->hostState.resize(b.capC);
    ENS_CUDA(e, cudaMemcpyAsync(e->hostState.data(), b.state, 4 * (size_t)b.capC,
                                cudaMemcpyDeviceToHost, e->copy));
    ENS_CUDA(e, cudaStreamSynchronize(e->copy));
    for (int s = 0; s < b.capC && *n_done < max_ids; ++s) {
      const int64_t id = b.slotCase[s];
      if (id < 0 || e->hostState[s] != kCaseDone) continue;
      HostCase &hc = e->cases[id];
      if (hc.reported) continue;
      if (cudaEventQuery(hc.admitted) != cudaSuccess) continue;  // stale state word
      hc.reported = true;
      done_ids[(*n_done)++] = id;
    }
  }
  return VCPG_OK;
}

int vcpg_ensemble_retire(vcpg_ensemble *ens, int64_t case_id, double *modal_state,
                         double *sim_time) {
  if (!ens) return VCPG_E_INVALID;
  vcpg_ensemble *e = ens;
  auto it = e->cases.find(case_id);
  if (it == e->cases.end()) return Fail(e, VCPG_E_INVALID, "unknown case id");
  HostCase hc = it->second;
  Bucket &b = e->b[hc.deg];
  if (cudaEventQuery(hc.admitted) != cudaSuccess)
    return Fail(e, VCPG_E_INVALID, "the case has not completed its steps");
  int st = 0;
  ENS_CUDA(e, cudaMemcpyAsync(&st, b.state + hc.slot, 4, cudaMemcpyDeviceToHost, e->copy));
  ENS_CUDA(e, cudaStreamSynchronize(e->copy));
  if (st != kCaseDone) return Fail(e, VCPG_E_INVALID, "the case has not completed its steps");
  // Kernels do not write done cases: read them on the copy stream.
  if (modal_state)
    ENS_CUDA(e, cudaMemcpyAsync(modal_state, b.sol + (size_t)hc.eFirst * 5 * b.KD,
                                8 * (size_t)hc.nE * 5 * b.KD, cudaMemcpyDeviceToHost, e->copy));
  double t = 0.0;
  ENS_CUDA(e, cudaMemcpyAsync(&t, b.simTime + hc.slot, 8, cudaMemcpyDeviceToHost, e->copy));
  ENS_CUDA(e, cudaStreamSynchronize(e->copy));
  if (sim_time) *sim_time = t;
  // Unmark the ranges on the upload stream (ordered before any later arrival's
  // uploads into them) and free the slot on the bucket stream.
  ENS_CUDA(e, cudaMemsetAsync(b.elemCase + hc.eFirst, 0xFF, 4 * (size_t)hc.nE, e->upload));
  if (hc.nB)
    ENS_CUDA(e, cudaMemsetAsync(b.bface + (size_t)hc.bFirst * kBfStride, 0xFF,
                                4 * (size_t)hc.nB * kBfStride, e->upload));
  const int freeState = kCaseFree;
  ENS_CUDA(e, cudaMemcpyAsync(b.state + hc.slot, &freeState, 4, cudaMemcpyHostToDevice, b.stream));
  ENS_CUDA(e, cudaStreamSynchronize(e->upload));
  b.elems.Free(hc.eFirst, hc.nE);
  b.bfaces.Free(hc.bFirst, hc.nB);
  b.sponge.Free(hc.sFirst, hc.nS);
  b.slotCase[hc.slot] = -1;
  b.resident -= 1;
  cudaEventDestroy(hc.admitted);
  e->cases.erase(it);
  return VCPG_OK;
}

int vcpg_ensemble_sync(vcpg_ensemble *ens) {
  if (!ens) return VCPG_E_INVALID;
  vcpg_ensemble *e = ens;
  ENS_CUDA(e, cudaStreamSynchronize(e->upload));
  for (Bucket &b : e->b) {
    if (b.deg < 0) continue;
    int rc = CheckBucketStatus(e, b);
    if (rc) return rc;
  }
  return VCPG_OK;
}

int vcpg_ensemble_stats(vcpg_ensemble *ens, int32_t *resident, int64_t *launches) {
  if (!ens) return VCPG_E_INVALID;
  int r = 0;
  for (Bucket &b : ens->b)
    if (b.deg >= 0) r += b.resident;
  if (resident) *resident = r;
  if (launches) *launches = ens->launches;
  return VCPG_OK;
}

}  // extern "C"
