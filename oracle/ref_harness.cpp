// Test infrastructure only (oracle build). Not part of the product.
//
// Command-line driver around the UNMODIFIED reference VCP3D sources (compiled
// from their own files by oracle/Makefile into oracle/_ref/). It reproduces
// the initialisation sequence of the reference main program
// (src/VCP3D_CurviLinear.cpp:25-100) and then either dumps the discretisation
// data, evaluates one residual, or drives a number of time steps, writing the
// results to a small tagged binary file that the Python tests read.
//
//   vcp3d_ref <param.cfg> dump     <out.bin>
//   vcp3d_ref <param.cfg> residual <out.bin> [--state <in.bin>]
//   vcp3d_ref <param.cfg> run      <out.bin> --scheme ssprk3|lsrk4 --steps N
//                                  [--dt DT] [--state <in.bin>] [--time]
//                                  [--every E]   (also <out.bin>.<n> every E steps)
//   vcp3d_ref <param.cfg> sync     <out.bin> --steps N
//
// The residual command replicates the loop structure of SolverClass::Residual
// (src/SolverClass.cpp:3381-3795) so that the residual can be captured both
// before and after the mass-matrix solve. The run command replicates the
// stage loop of SolverClass::ExecuteTimeSynchronizationStep
// (src/SolverClass.cpp:2177-2422) with a CFL-limited (or fixed) time step and
// without the synchronisation-time clip, and calls the reference's own
// SolverClass::Residual for every stage. The low-storage RK4 scheme has no
// counterpart in the reference; it drives the same Residual with the
// Carpenter-Kennedy (1994) five-stage 2N-storage coefficients. The sync command
// calls the reference's own ExecuteTimeSynchronizationStep N times after the
// initial residual, as the reference main program does.

#include <fstream>
#include <iostream>
#include <iomanip>
#include <sstream>
#include <string>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <algorithm>
#include <list>
#include <map>
#include <set>
#include <vector>
#include <random>
#include <cassert>
#include <cstdint>
#include <signal.h>
#include <omp.h>
#include <unistd.h>
#include <chrono>

// The harness reads solver internals; expose them without touching the sources.
#define private public
#define protected public
#include "VCP3D_CurviLinear.hpp"
#undef private
#undef protected

// Globals that the reference main program defines (src/VCP3D_CurviLinear.cpp:9-20).
int rank, nRanks;
ENUM_SIGNAL CurrentSignal;
su2double rhoDim;
su2double pDim;
su2double pRef;
su2double uRef;
su2double rhoRef;
su2double mu;

namespace {

// ---------------------------------------------------------------------------
// Tagged binary container: "VCPR" then records of
//   char name[32]; int32 ndim; int64 dims[ndim]; float64 data[prod(dims)].
// ---------------------------------------------------------------------------
struct Writer {
  FILE *f;
  explicit Writer(const char *path) {
    f = std::fopen(path, "wb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
    std::fwrite("VCPR", 1, 4, f);
  }
  ~Writer() { if (f) std::fclose(f); }
  void rec(const std::string &name, const std::vector<int64_t> &dims,
           const double *data) {
    char nm[32] = {0};
    std::strncpy(nm, name.c_str(), 31);
    std::fwrite(nm, 1, 32, f);
    int32_t nd = (int32_t)dims.size();
    std::fwrite(&nd, 4, 1, f);
    int64_t n = 1;
    for (int64_t d : dims) { std::fwrite(&d, 8, 1, f); n *= d; }
    std::fwrite(data, 8, (size_t)n, f);
  }
};

struct Record { std::vector<int64_t> dims; std::vector<double> data; };

std::map<std::string, Record> ReadRecords(const char *path) {
  std::map<std::string, Record> out;
  FILE *f = std::fopen(path, "rb");
  if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
  char magic[4];
  if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "VCPR", 4)) {
    std::fprintf(stderr, "%s: bad magic\n", path); std::exit(2);
  }
  for (;;) {
    char nm[32];
    if (std::fread(nm, 1, 32, f) != 32) break;
    int32_t nd;
    if (std::fread(&nd, 4, 1, f) != 1) break;
    Record r; r.dims.resize(nd);
    int64_t n = 1;
    for (int i = 0; i < nd; ++i) { if (std::fread(&r.dims[i], 8, 1, f) != 1) std::exit(2); n *= r.dims[i]; }
    r.data.resize(n);
    if (std::fread(r.data.data(), 8, (size_t)n, f) != (size_t)n) std::exit(2);
    out[std::string(nm)] = r;
  }
  std::fclose(f);
  return out;
}

// Owned elements in the reference's storage order (i fastest, then j, then k).
template <class F> void ForEachElem(SolverClass &s, F f) {
  for (int k = 1; k <= s.mNElemPerRankK; ++k)
    for (int j = 1; j <= s.mNElemPerRankJ; ++j)
      for (int i = 1; i <= s.mNElemPerRankI; ++i) f(s.mElements[i][j][k]);
}

int NElem(SolverClass &s) { return s.mNElemPerRankI * s.mNElemPerRankJ * s.mNElemPerRankK; }

// Gather one per-element field [elem][var][pad] into a flat array.
std::vector<double> Gather(SolverClass &s, std::vector<su2double *> ElementClass::*field,
                           int nv, int pad) {
  std::vector<double> out;
  out.reserve((size_t)NElem(s) * nv * pad);
  ForEachElem(s, [&](ElementClass *e) {
    for (int v = 0; v < nv; ++v)
      for (int m = 0; m < pad; ++m) out.push_back((e->*field)[v][m]);
  });
  return out;
}

void Scatter(SolverClass &s, std::vector<su2double *> ElementClass::*field, int nv,
             int pad, const std::vector<double> &in) {
  size_t p = 0;
  ForEachElem(s, [&](ElementClass *e) {
    for (int v = 0; v < nv; ++v)
      for (int m = 0; m < pad; ++m) (e->*field)[v][m] = in[p++];
  });
}

std::vector<su2double *> MakeWorkArray(SolverClass &s) {
  const int nDOFsPad = s.mStandardHex.mNDOFsPad;
  const int nIntPad = s.mStandardHex.mNIntegrationPad;
  const int n1 = std::max(15 * nVar + 1, 5 * nVar);
  const int n2 = std::max(nIntPad, nDOFsPad);
  std::vector<su2double *> w(n1);
  for (int i = 0; i < n1; ++i) w[i] = (su2double *)AllocateMemory(n2 * sizeof(su2double));
  return w;
}

void FreeWorkArray(std::vector<su2double *> &w) {
  for (auto &p : w) FreeMemory((void **)&p);
}

// Mirrors the time-step part of ExecuteTimeSynchronizationStep
// (src/SolverClass.cpp:2180-2275): minimum of ElementClass::ComputeTimeStep.
su2double GlobalTimeStep(SolverClass &s) {
  const su2double f1[] = {2.0, 6.0, 12.0, 20.0, 28.0, 38.0, 50.0, 64.0, 80.0, 98.0};
  const su2double f2[] = {6.0, 36.0, 150.0, 420.0, 980.0, 1975.0, 3575.0, 7000.0,
                          14000.0, 28000.0};
  const int nDOFs = s.mStandardHex.mNDOFs;
  su2double deltaT = 1.e+10;
#pragma omp parallel
  {
    std::vector<su2double *> solNodal(nVar + 1);
    for (int m = 0; m <= nVar; ++m)
      solNodal[m] = (su2double *)AllocateMemory(s.mStandardHex.mNDOFsPad * sizeof(su2double));
    (void)nDOFs;
    // Gradients of the nodal solution, used by the eddy viscosity of an SGS model.
    std::vector<su2double *> gradSolNodal;
    if (s.mInputParam->mSGSModelType != NO_SGS_MODEL) {
      gradSolNodal.resize(3 * nVar);
      for (auto &p : gradSolNodal)
        p = (su2double *)AllocateMemory(s.mStandardHex.mNDOFsPad * sizeof(su2double));
    }
#pragma omp for schedule(static), collapse(3), reduction(min : deltaT)
    for (int k = 1; k <= s.mNElemPerRankK; ++k)
      for (int j = 1; j <= s.mNElemPerRankJ; ++j)
        for (int i = 1; i <= s.mNElemPerRankI; ++i) {
          const su2double dt = s.mElements[i][j][k]->ComputeTimeStep(
              s.mInputParam, &s.mStandardHex, f1, f2, solNodal.data(), gradSolNodal.data());
          deltaT = std::min(deltaT, dt);
        }
    for (auto &p : solNodal) FreeMemory((void **)&p);
    for (auto &p : gradSolNodal) FreeMemory((void **)&p);
  }
  return deltaT;
}

void CopySolToOld(SolverClass &s) {
  const int nDOFsPad = s.mStandardHex.mNDOFsPad;
#pragma omp parallel for collapse(3), schedule(static)
  for (int k = 1; k <= s.mNElemPerRankK; ++k)
    for (int j = 1; j <= s.mNElemPerRankJ; ++j)
      for (int i = 1; i <= s.mNElemPerRankI; ++i)
        for (int l = 0; l < nVar; ++l)
          for (int m = 0; m < nDOFsPad; ++m)
            s.mElements[i][j][k]->mSolOld[l][m] = s.mElements[i][j][k]->mSol[l][m];
}

// SSP-RK3 stage update, src/SolverClass.cpp:2368-2396.
void SspStageUpdate(SolverClass &s, su2double alpha, su2double betaDt) {
  const int nDOFsPad = s.mStandardHex.mNDOFsPad;
  const su2double oneMinAlpha = one - alpha;
#pragma omp parallel for collapse(3), schedule(static)
  for (int k = 1; k <= s.mNElemPerRankK; ++k)
    for (int j = 1; j <= s.mNElemPerRankJ; ++j)
      for (int i = 1; i <= s.mNElemPerRankI; ++i)
        for (int l = 0; l < nVar; ++l) {
          su2double *sol = s.mElements[i][j][k]->mSol[l];
          const su2double *solOld = s.mElements[i][j][k]->mSolOld[l];
          const su2double *res = s.mElements[i][j][k]->mRes[l];
          for (int m = 0; m < nDOFsPad; ++m)
            sol[m] = oneMinAlpha * sol[m] + alpha * solOld[m] - betaDt * res[m];
        }
}

// Low-storage RK4 stage: dU = a dU - dt res; U += b dU. mSolOld holds dU.
void LsrkStageUpdate(SolverClass &s, su2double a, su2double b, su2double dt) {
  const int nDOFsPad = s.mStandardHex.mNDOFsPad;
#pragma omp parallel for collapse(3), schedule(static)
  for (int k = 1; k <= s.mNElemPerRankK; ++k)
    for (int j = 1; j <= s.mNElemPerRankJ; ++j)
      for (int i = 1; i <= s.mNElemPerRankI; ++i)
        for (int l = 0; l < nVar; ++l) {
          su2double *sol = s.mElements[i][j][k]->mSol[l];
          su2double *du = s.mElements[i][j][k]->mSolOld[l];
          const su2double *res = s.mElements[i][j][k]->mRes[l];
          for (int m = 0; m < nDOFsPad; ++m) {
            du[m] = a * du[m] - dt * res[m];
            sol[m] = sol[m] + b * du[m];
          }
        }
}

const double kLsA[5] = {0.0, -567301805773.0 / 1357537059087.0,
                        -2404267990393.0 / 2016746695238.0,
                        -3550918686646.0 / 2091501179385.0,
                        -1275806237668.0 / 842570457699.0};
const double kLsB[5] = {1432997174477.0 / 9575080441755.0,
                        5161836677717.0 / 13612068292357.0,
                        1720146321549.0 / 2090206949498.0,
                        3134564353537.0 / 4481467310338.0,
                        2277821191437.0 / 14882151754819.0};

void DoResidual(SolverClass &s, su2double *mon, bool monitor) {
  if (s.mInputParam->mNSCBC_Specified) s.AverageDataNSCBC();
  s.Residual(mon, monitor);
}

void DumpSetup(SolverClass &s, Writer &w) {
  StandardElementClass &sh = s.mStandardHex;
  InputParamClass *ip = s.mInputParam;
  const double params[] = {(double)s.mNElemPerRankI, (double)s.mNElemPerRankJ,
                           (double)s.mNElemPerRankK, (double)sh.mNPoly,
                           (double)sh.mNDOFs1D, (double)sh.mNIntegration1D,
                           (double)sh.mNDOFsPad, (double)sh.mNIntegrationPad,
                           (double)sh.mNIntegration2DPad, (double)sh.mNDOFs1DPad,
                           (double)sh.mNIntegration1DPad, (double)ip->mRiemannSolver,
                           (double)ip->mThetaSym, (double)ip->mRelativePenaltyParameter,
                           (double)ip->mCFL};
  w.rec("params", {(int64_t)(sizeof(params) / sizeof(double))}, params);
  const double refc[] = {pRef, uRef, rhoRef, mu};
  w.rec("refcond", {4}, refc);
  const int K = sh.mNDOFs1D, M = sh.mNIntegration1D, KP = sh.mNDOFs1DPad,
            MP = sh.mNIntegration1DPad;
  w.rec("legInt1D", {K, MP}, sh.mLegendreInt1D);
  w.rec("derLegInt1D", {K, MP}, sh.mDerLegendreInt1D);
  w.rec("legInt1DT", {M, KP}, sh.mLegendreInt1DTranspose);
  w.rec("derLegInt1DT", {M, KP}, sh.mDerLegendreInt1DTranspose);
  w.rec("legMinFace1D", {KP}, sh.mLegendreMinFace1D);
  w.rec("legMaxFace1D", {KP}, sh.mLegendreMaxFace1D);
  w.rec("derLegMinFace1D", {KP}, sh.mDerLegendreMinFace1D);
  w.rec("derLegMaxFace1D", {KP}, sh.mDerLegendreMaxFace1D);
  w.rec("intWeights", {sh.mNIntegrationPad}, sh.mIntWeights);
  w.rec("intWeightsFace", {sh.mNIntegration2DPad}, sh.mIntWeightsFace);
  w.rec("basisCenter", {sh.mNDOFs}, sh.mBasisCenter);
  w.rec("legDOFs1D", {K, KP}, sh.mLegendreDOFs1D);
  w.rec("derLegDOFs1D", {K, KP}, sh.mDerLegendreDOFs1D);
  w.rec("vandInv1D", {K, KP}, sh.mVandermonde1DInverse);
  w.rec("rInt1D", {M}, sh.mRIntegration1D.data());
  w.rec("wInt1D", {M}, sh.mIntegrationWeights1D.data());
  w.rec("rDOFs1D", {K}, sh.mRDOFs1D.data());

  const int nE = NElem(s);
  const int nIntPad = sh.mNIntegrationPad, n2Pad = sh.mNIntegration2DPad;
  w.rec("volMetric", {nE, 13, nIntPad}, Gather(s, &ElementClass::mVolMetricInt, 13, nIntPad).data());
  std::vector<su2double *> ElementClass::*faces[6] = {
      &ElementClass::mSurfMetricIntIMin, &ElementClass::mSurfMetricIntIMax,
      &ElementClass::mSurfMetricIntJMin, &ElementClass::mSurfMetricIntJMax,
      &ElementClass::mSurfMetricIntKMin, &ElementClass::mSurfMetricIntKMax};
  const char *fnames[6] = {"surfIMin", "surfIMax", "surfJMin", "surfJMax", "surfKMin", "surfKMax"};
  for (int f = 0; f < 6; ++f)
    w.rec(fnames[f], {nE, 16, n2Pad}, Gather(s, faces[f], 16, n2Pad).data());
  std::vector<double> scal;
  ForEachElem(s, [&](ElementClass *e) {
    const double v[] = {e->mLenScaleIDir, e->mLenScaleJDir, e->mLenScaleKDir,
                        e->mLenScaleLES, e->mLenScaleVolume, e->mVolElem,
                        e->mAveNormIDir[0], e->mAveNormIDir[1], e->mAveNormIDir[2],
                        e->mAveNormJDir[0], e->mAveNormJDir[1], e->mAveNormJDir[2],
                        e->mAveNormKDir[0], e->mAveNormKDir[1], e->mAveNormKDir[2]};
    scal.insert(scal.end(), v, v + 15);
  });
  w.rec("elemScalars", {nE, 15}, scal.data());
  const int nGrid = (ip->mNPolyGridDOFs + 1) * (ip->mNPolyGridDOFs + 1) * (ip->mNPolyGridDOFs + 1);
  w.rec("gridNodes", {nE, 3, nGrid}, Gather(s, &ElementClass::mCoorNodalGridDOFs, 3, nGrid).data());
  w.rec("solDOFCoor", {nE, 3, sh.mNDOFs},
        Gather(s, &ElementClass::mCoorNodalSolDOFs, 3, sh.mNDOFs).data());
  w.rec("sol", {nE, 5, sh.mNDOFsPad}, Gather(s, &ElementClass::mSol, 5, sh.mNDOFsPad).data());
}

// Residual with the loop structure of SolverClass::Residual; captures the
// residual before the mass-matrix solve as well.
void ResidualWithCapture(SolverClass &s, Writer &w) {
  StandardElementClass &sh = s.mStandardHex;
  const int nDOFsPad = sh.mNDOFsPad;
  if (s.mInputParam->mNSCBC_Specified) s.AverageDataNSCBC();
  std::vector<su2double *> wa = MakeWorkArray(s);
  su2double Mach2Max = zero, EddyVisMax = -one;
  su2double forceCoef[6] = {0, 0, 0, 0, 0, 0};
  ForEachElem(s, [&](ElementClass *e) {
    e->VolumeResidual(s.mInputParam, &sh, wa.data(), true, Mach2Max, EddyVisMax);
  });
  const int nE = NElem(s);
  w.rec("resVolume", {nE, 5, nDOFsPad}, Gather(s, &ElementClass::mRes, 5, nDOFsPad).data());
  w.rec("dUdV", {nE, 15, sh.mNIntegrationPad},
        Gather(s, &ElementClass::mDUdVInt, 15, sh.mNIntegrationPad).data());
  ForEachElem(s, [&](ElementClass *e) {
    e->IFaceResiduals(s.mInputParam, &sh, s.mElements, wa.data(), true, EddyVisMax, forceCoef);
  });
  ForEachElem(s, [&](ElementClass *e) {
    e->JFaceResiduals(s.mInputParam, &sh, s.mElements, wa.data(), true, EddyVisMax, forceCoef);
  });
  ForEachElem(s, [&](ElementClass *e) {
    e->KFaceResiduals(s.mInputParam, &sh, s.mElements, wa.data(), true, EddyVisMax, forceCoef);
  });
  for (int dir = 0; dir < 3; ++dir)
    for (int k = 1; k <= s.mNElemPerRankK; ++k)
      for (int j = 1; j <= s.mNElemPerRankJ; ++j)
        for (int i = 1; i <= s.mNElemPerRankI; ++i) {
          ElementClass *e = s.mElements[i][j][k];
          ElementClass *nb = dir == 0 ? s.mElements[i + 1][j][k]
                           : dir == 1 ? s.mElements[i][j + 1][k] : s.mElements[i][j][k + 1];
          if (!nb) continue;
          std::vector<su2double *> &src = dir == 0 ? nb->mResIMin : dir == 1 ? nb->mResJMin : nb->mResKMin;
          for (int l = 0; l < nVar; ++l)
            for (int m = 0; m < nDOFsPad; ++m) e->mRes[l][m] += src[l][m];
        }
  w.rec("resRaw", {nE, 5, nDOFsPad}, Gather(s, &ElementClass::mRes, 5, nDOFsPad).data());
  ForEachElem(s, [&](ElementClass *e) {
    e->MultiplyResInverseMassMatrix(s.mInputParam, &sh, wa.data());
  });
  w.rec("res", {nE, 5, nDOFsPad}, Gather(s, &ElementClass::mRes, 5, nDOFsPad).data());
  const su2double factCoef = two / (GamConstant * s.mInputParam->mMach *
                                    s.mInputParam->mMach * s.mInputParam->mReferenceArea);
  double mon[8];
  for (int i = 0; i < 6; ++i) mon[i] = forceCoef[i] * factCoef;
  mon[6] = Mach2Max; mon[7] = EddyVisMax;
  w.rec("monitor", {8}, mon);
  FreeWorkArray(wa);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <param.cfg> dump|residual|run|sync <out.bin> [options]\n", argv[0]);
    return 2;
  }
  std::string cfg = argv[1], cmd = argv[2], out = argv[3];
  std::string scheme = "ssprk3", statePath;
  int steps = 1, every = 0;
  double fixedDt = -1.0;
  bool timeIt = false;
  for (int a = 4; a < argc; ++a) {
    std::string o = argv[a];
    if (o == "--scheme" && a + 1 < argc) scheme = argv[++a];
    else if (o == "--steps" && a + 1 < argc) steps = std::atoi(argv[++a]);
    else if (o == "--dt" && a + 1 < argc) fixedDt = std::atof(argv[++a]);
    else if (o == "--state" && a + 1 < argc) statePath = argv[++a];
    else if (o == "--time") timeIt = true;
    else if (o == "--every" && a + 1 < argc) every = std::atoi(argv[++a]);
    else { std::fprintf(stderr, "unknown option %s\n", o.c_str()); return 2; }
  }
  // Resolve output/state paths before changing into the case directory.
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) return 2;
  auto absPath = [&](const std::string &p) {
    return (p.empty() || p[0] == '/') ? p : std::string(cwd) + "/" + p;
  };
  out = absPath(out);
  statePath = absPath(statePath);
  std::string dir = ".", base = cfg;
  const size_t slash = cfg.rfind('/');
  if (slash != std::string::npos) { dir = cfg.substr(0, slash); base = cfg.substr(slash + 1); }
  if (chdir(dir.c_str()) != 0) { std::perror("chdir"); return 2; }

  // Initialisation sequence of src/VCP3D_CurviLinear.cpp:28-90.
  int ac = 2;
  char *avArr[3] = {argv[0], argv[1], NULL};
  char **av = avArr;
  StartUpCode(&ac, &av);
  InputParamClass inputParam;
  std::vector<char> cfgName(base.begin(), base.end());
  cfgName.push_back(0);
  inputParam.ReadInputParameters(cfgName.data());
  if (inputParam.mSpongeLayer || inputParam.mCharacteristicMatchingLayer)
    inputParam.ReadSpongeLayerData(cfgName.data());
  inputParam.ReadSubfaceInformation(cfgName.data());
  inputParam.ReadBoundaryData(cfgName.data());
  inputParam.ComputeReferenceConditions();
  SolverClass solver(&inputParam);
  solver.ReadGrid();
  solver.ComputeMetricTerms();
  solver.BoundingBoxFluctuations();
  solver.InitSol();
  if (inputParam.mRestart) solver.ReadRestartSolution();
  if (inputParam.mSpongeLayer) solver.InitSpongeLayer();
  solver.PrescribedDataIntegrationPoints();
  solver.AddFluctuations();
  if (inputParam.mNSCBC_Specified) solver.InitNSCBC();

  const int nDOFsPad = solver.mStandardHex.mNDOFsPad;
  if (!statePath.empty()) {
    auto recs = ReadRecords(statePath.c_str());
    if (!recs.count("sol")) { std::fprintf(stderr, "state file has no 'sol'\n"); return 2; }
    Scatter(solver, &ElementClass::mSol, 5, nDOFsPad, recs["sol"].data);
  }

  Writer w(out.c_str());
  const int nE = NElem(solver);
  if (cmd == "dump") {
    DumpSetup(solver, w);
  } else if (cmd == "residual") {
    w.rec("sol", {nE, 5, nDOFsPad}, Gather(solver, &ElementClass::mSol, 5, nDOFsPad).data());
    ResidualWithCapture(solver, w);
    const double dt = GlobalTimeStep(solver);
    w.rec("dt", {1}, &dt);
  } else if (cmd == "run") {
    su2double mon[8];
    std::vector<double> dtHist;
    DoResidual(solver, mon, true);
    const int nStages = scheme == "lsrk4" ? 5 : 3;
    const su2double alphaRK[] = {one, three / four, one / three};
    const su2double betaRK[] = {one, one / four, two / three};
    auto t0 = std::chrono::steady_clock::now();
    for (int step = 0; step < steps; ++step) {
      const su2double dt = fixedDt > 0 ? fixedDt : GlobalTimeStep(solver);
      dtHist.push_back(dt);
      if (scheme == "lsrk4") {
        const int nDP = nDOFsPad;
        ForEachElem(solver, [&](ElementClass *e) {
          for (int l = 0; l < nVar; ++l)
            for (int m = 0; m < nDP; ++m) e->mSolOld[l][m] = zero;
        });
        for (int st = 0; st < nStages; ++st) {
          LsrkStageUpdate(solver, kLsA[st], kLsB[st], dt);
          DoResidual(solver, mon, st == nStages - 1);
        }
      } else if (scheme == "ssprk3") {
        CopySolToOld(solver);
        for (int st = 0; st < nStages; ++st) {
          SspStageUpdate(solver, alphaRK[st], betaRK[st] * dt);
          DoResidual(solver, mon, st == nStages - 1);
        }
      } else {
        std::fprintf(stderr, "unknown scheme %s\n", scheme.c_str());
        return 2;
      }
      // Sample files for long runs: the state and the steps so far.
      if (every > 0 && (step + 1) % every == 0) {
        Writer ws((out + "." + std::to_string(step + 1)).c_str());
        ws.rec("sol", {nE, 5, nDOFsPad}, Gather(solver, &ElementClass::mSol, 5, nDOFsPad).data());
        ws.rec("dtHist", {(int64_t)dtHist.size()}, dtHist.data());
      }
    }
    auto t1 = std::chrono::steady_clock::now();
    const double secs = std::chrono::duration<double>(t1 - t0).count();
    if (timeIt)
      std::printf("VCP3D_REF_TIMING steps=%d seconds=%.9e threads=%d dofs=%d\n", steps, secs,
                  omp_get_max_threads(), nE * solver.mStandardHex.mNDOFs);
    w.rec("sol", {nE, 5, nDOFsPad}, Gather(solver, &ElementClass::mSol, 5, nDOFsPad).data());
    w.rec("res", {nE, 5, nDOFsPad}, Gather(solver, &ElementClass::mRes, 5, nDOFsPad).data());
    w.rec("dtHist", {(int64_t)dtHist.size()}, dtHist.data());
    w.rec("monitor", {8}, mon);
    w.rec("seconds", {1}, &secs);
  } else if (cmd == "sync") {
    // The reference main program's loop (src/VCP3D_CurviLinear.cpp:88-116):
    // the residual of the initial state, then --steps calls of the reference's
    // own ExecuteTimeSynchronizationStep.
    su2double mon[8];
    DoResidual(solver, mon, true);
    auto t0 = std::chrono::steady_clock::now();
    for (int step = 0; step < steps; ++step) solver.ExecuteTimeSynchronizationStep(mon);
    auto t1 = std::chrono::steady_clock::now();
    const double secs = std::chrono::duration<double>(t1 - t0).count();
    const double nrk = (double)solver.mCurrentTimeStep;
    w.rec("sol", {nE, 5, nDOFsPad}, Gather(solver, &ElementClass::mSol, 5, nDOFsPad).data());
    w.rec("monitor", {8}, mon);
    w.rec("rkSteps", {1}, &nrk);
    w.rec("seconds", {1}, &secs);
  } else {
    std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
  }
  std::fflush(stdout);
  return 0;
}
