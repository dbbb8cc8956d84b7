// Metric terms on the device: vcpg_setup_geometry_device computes what
// vcpg_setup_geometry computes on the host (the restatement of
// ElementClass::ComputeMetricTerms / FinalMetric[IJK]Face / ComputeLengthScales,
// src/ElementClass.cpp:927-1022, 1027-1407, 1907-2092), one CTA per element.
//
// This file is compiled without multiply-add contraction (-fmad=false): the
// contractions use explicit fma in the host's order and every other product and
// sum rounds separately, as on the host, so both produce the same doubles. The
// cube root of the element volume (the volume length scale) is taken on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/vcp3d_b200.h"
#include "host_setup.h"

namespace vcpg {
namespace {

constexpr int kMetricThreads = 128;

// out = op applied along axis ax of in[n2][n1][n0]; op is [nin][nout]; the
// summation runs over the input index with fused multiply-adds, as the host's
// ApplyAxis does. Callers separate consecutive calls with a barrier.
__device__ void ApplyAxisD(const double *in, int n0, int n1, int n2, int ax, const double *op,
                           int nout, double *out) {
  const int nin = ax == 0 ? n0 : (ax == 1 ? n1 : n2);
  const int o0 = ax == 0 ? nout : n0, o1 = ax == 1 ? nout : n1, o2 = ax == 2 ? nout : n2;
  for (int idx = threadIdx.x; idx < o0 * o1 * o2; idx += blockDim.x) {
    const int c0 = idx % o0, c1 = (idx / o0) % o1, c2 = idx / (o0 * o1);
    const int o = ax == 0 ? c0 : (ax == 1 ? c1 : c2);
    double acc = 0.0;
    for (int c = 0; c < nin; ++c) {
      const int i0 = ax == 0 ? c : c0, i1 = ax == 1 ? c : c1, i2 = ax == 2 ? c : c2;
      acc = fma(op[c * nout + o], in[(i2 * n1 + i1) * n0 + i0], acc);
    }
    out[idx] = acc;
  }
}

struct MetricArgs {
  const double *nodes;       // [nE][3][Kg^3]
  const double *lagInt;      // [Kg][M]
  const double *dlagInt;     // [Kg][M]
  const double *lagFace;     // [2][Kg]
  const double *dlagFace;    // [2][Kg]
  const double *wInt;        // [M]
  double *vol;               // [nE][10][M^3]
  double *face;              // [nE][6][13][M^2]
  double *scalars;           // [nE][15] (entries 3 and 4 are finished on the host)
  int *bad;                  // elements with a non-positive Jacobian
  int nE, Kg, M;
};

__global__ void __launch_bounds__(kMetricThreads) ElementMetricsKernel(const MetricArgs a) {
  const int e = blockIdx.x;
  if (e >= a.nE) return;
  const int Kg = a.Kg, M = a.M, KG3 = Kg * Kg * Kg, MD = M * M * M, M2 = M * M;
  extern __shared__ double sm[];
  double *g = sm;                         // 3 Kg^3
  double *t1 = g + 3 * KG3;               // Kg^3 (>= Kg^2 M and >= Kg^2)
  double *t2 = t1 + Kg * Kg * (Kg > M ? Kg : M);  // Kg M^2 (>= Kg M)
  double *dc = t2 + Kg * M * M + Kg * M;  // [3][3][MD], faces use [3][3][M2]
  double *ops = dc + 9 * MD;              // lagInt, dlagInt, lagFace, dlagFace, wInt
  double *lag = ops, *dlag = lag + Kg * M, *lagF = dlag + Kg * M, *dlagF = lagF + 2 * Kg;
  double *wI = dlagF + 2 * Kg;
  for (int i = threadIdx.x; i < 3 * KG3; i += blockDim.x) g[i] = a.nodes[(size_t)e * 3 * KG3 + i];
  for (int i = threadIdx.x; i < Kg * M; i += blockDim.x) {
    lag[i] = a.lagInt[i];
    dlag[i] = a.dlagInt[i];
  }
  for (int i = threadIdx.x; i < 2 * Kg; i += blockDim.x) {
    lagF[i] = a.lagFace[i];
    dlagF[i] = a.dlagFace[i];
  }
  for (int i = threadIdx.x; i < M; i += blockDim.x) wI[i] = a.wInt[i];
  __syncthreads();

  // Volume: derivatives of the coordinates at the integration points (k, j, i).
  for (int x = 0; x < 3; ++x)
    for (int q = 0; q < 3; ++q) {
      ApplyAxisD(g + x * KG3, Kg, Kg, Kg, 2, q == 2 ? dlag : lag, M, t1);
      __syncthreads();
      ApplyAxisD(t1, Kg, Kg, M, 1, q == 1 ? dlag : lag, M, t2);
      __syncthreads();
      ApplyAxisD(t2, Kg, M, M, 0, q == 0 ? dlag : lag, M, dc + (q * 3 + x) * MD);
      __syncthreads();
    }
  double *vol = a.vol + (size_t)e * 10 * MD;
  for (int l = threadIdx.x; l < MD; l += blockDim.x) {
    const double dxdr = dc[0 * MD + l], dydr = dc[1 * MD + l], dzdr = dc[2 * MD + l];
    const double dxds = dc[3 * MD + l], dyds = dc[4 * MD + l], dzds = dc[5 * MD + l];
    const double dxdt = dc[6 * MD + l], dydt = dc[7 * MD + l], dzdt = dc[8 * MD + l];
    const double J = dxdr * (dyds * dzdt - dzds * dydt) - dxds * (dydr * dzdt - dzdr * dydt) +
                     dxdt * (dydr * dzds - dzdr * dyds);
    if (!(J > 0.0)) atomicAdd(a.bad, 1);
    const double Jinv = 1.0 / J;
    vol[0 * MD + l] = J;
    vol[1 * MD + l] = Jinv * (dyds * dzdt - dzds * dydt);
    vol[2 * MD + l] = Jinv * (dzds * dxdt - dxds * dzdt);
    vol[3 * MD + l] = Jinv * (dxds * dydt - dyds * dxdt);
    vol[4 * MD + l] = Jinv * (dzdr * dydt - dydr * dzdt);
    vol[5 * MD + l] = Jinv * (dxdr * dzdt - dzdr * dxdt);
    vol[6 * MD + l] = Jinv * (dydr * dxdt - dxdr * dydt);
    vol[7 * MD + l] = Jinv * (dydr * dzds - dzdr * dyds);
    vol[8 * MD + l] = Jinv * (dzdr * dxds - dxdr * dzds);
    vol[9 * MD + l] = Jinv * (dxdr * dyds - dydr * dxds);
  }
  __syncthreads();

  // Faces: face-normal evaluation, then the fast and the slow in-face axes.
  double *faceOut = a.face + (size_t)e * 6 * 13 * M2;
  for (int f = 0; f < 6; ++f) {
    const int d = f / 2, side = f % 2;
    const double *fv = lagF + side * Kg, *dfv = dlagF + side * Kg;
    const int fastAx = d == 0 ? 1 : 0, slowAx = d == 2 ? 1 : 2;
    for (int x = 0; x < 3; ++x)
      for (int q = 0; q < 3; ++q) {
        int n[3] = {Kg, Kg, Kg};
        ApplyAxisD(g + x * KG3, n[0], n[1], n[2], d, q == d ? dfv : fv, 1, t1);
        __syncthreads();
        n[d] = 1;
        ApplyAxisD(t1, n[0], n[1], n[2], fastAx, q == fastAx ? dlag : lag, M, t2);
        __syncthreads();
        n[fastAx] = M;
        ApplyAxisD(t2, n[0], n[1], n[2], slowAx, q == slowAx ? dlag : lag, M,
                   dc + (q * 3 + x) * M2);
        __syncthreads();
      }
    double *fm = faceOut + (size_t)f * 13 * M2;
    for (int l = threadIdx.x; l < M2; l += blockDim.x) {
      const double dxdr = dc[0 * M2 + l], dydr = dc[1 * M2 + l], dzdr = dc[2 * M2 + l];
      const double dxds = dc[3 * M2 + l], dyds = dc[4 * M2 + l], dzds = dc[5 * M2 + l];
      const double dxdt = dc[6 * M2 + l], dydt = dc[7 * M2 + l], dzdt = dc[8 * M2 + l];
      double nx, ny, nz;
      if (d == 0) {
        nx = dyds * dzdt - dydt * dzds; ny = dxdt * dzds - dxds * dzdt; nz = dxds * dydt - dxdt * dyds;
      } else if (d == 1) {
        nx = dydt * dzdr - dydr * dzdt; ny = dxdr * dzdt - dxdt * dzdr; nz = dxdt * dydr - dxdr * dydt;
      } else {
        nx = dydr * dzds - dyds * dzdr; ny = dxds * dzdr - dxdr * dzds; nz = dxdr * dyds - dxds * dydr;
      }
      const double lenNorm = sqrt(nx * nx + ny * ny + nz * nz);
      const double invLen = 1.0 / lenNorm;
      fm[0 * M2 + l] = nx * invLen;
      fm[1 * M2 + l] = ny * invLen;
      fm[2 * M2 + l] = nz * invLen;
      fm[3 * M2 + l] = lenNorm;
      const double Jinv = 1.0 / (dxdr * (dyds * dzdt - dzds * dydt) - dxds * (dydr * dzdt - dzdr * dydt) +
                                 dxdt * (dydr * dzds - dzdr * dyds));
      fm[4 * M2 + l] = (dyds * dzdt - dzds * dydt) * Jinv;
      fm[5 * M2 + l] = (dzds * dxdt - dxds * dzdt) * Jinv;
      fm[6 * M2 + l] = (dxds * dydt - dyds * dxdt) * Jinv;
      fm[7 * M2 + l] = (dzdr * dydt - dydr * dzdt) * Jinv;
      fm[8 * M2 + l] = (dxdr * dzdt - dzdr * dxdt) * Jinv;
      fm[9 * M2 + l] = (dydr * dxdt - dxdr * dydt) * Jinv;
      fm[10 * M2 + l] = (dydr * dzds - dzdr * dyds) * Jinv;
      fm[11 * M2 + l] = (dzdr * dxds - dxdr * dzds) * Jinv;
      fm[12 * M2 + l] = (dxdr * dyds - dydr * dxds) * Jinv;
    }
    __syncthreads();
  }

  // Element volume, directional length scales and averaged normals, summed in
  // the host's order by one thread.
  if (threadIdx.x == 0) {
    double *sc = a.scalars + (size_t)e * 15;
    double volElem = 0.0;
    for (int k = 0, l = 0; k < M; ++k)
      for (int j = 0; j < M; ++j)
        for (int i = 0; i < M; ++i, ++l) volElem += wI[i] * wI[j] * wI[k] * vol[l];
    sc[5] = volElem;
    for (int dd = 0; dd < 3; ++dd) {
      const double *fmin = faceOut + (size_t)(2 * dd) * 13 * M2, *fmax = fmin + 13 * M2;
      double s = 0.0, a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int j = 0, l = 0; j < M; ++j)
        for (int i = 0; i < M; ++i, ++l) {
          const double w = wI[i] * wI[j];
          a0 += w * (fmin[l] * fmin[3 * M2 + l] + fmax[l] * fmax[3 * M2 + l]);
          a1 += w * (fmin[M2 + l] * fmin[3 * M2 + l] + fmax[M2 + l] * fmax[3 * M2 + l]);
          a2 += w * (fmin[2 * M2 + l] * fmin[3 * M2 + l] + fmax[2 * M2 + l] * fmax[3 * M2 + l]);
          s += w * (fmin[3 * M2 + l] + fmax[3 * M2 + l]);
        }
      sc[dd] = 2.0 * volElem / s;
      sc[6 + 3 * dd] = a0 / s;
      sc[7 + 3 * dd] = a1 / s;
      sc[8 + 3 * dd] = a2 / s;
    }
  }
}

}  // namespace
}  // namespace vcpg

using vcpg::host::StdElement;

extern "C" {

int vcpg_setup_geometry_device(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                               const int32_t periodic[3], const double *grid_nodes,
                               double *leg_int, double *dleg_int, double *leg_face,
                               double *dleg_face, double *w_int, double *leg_dofs,
                               double *basis_center, double *vol_metric, double *face_metric,
                               double *elem_scalars, int32_t *neighbors) {
  if (!params || !grid_nodes || p_grid < 1 || !vol_metric || !face_metric || !elem_scalars)
    return VCPG_E_INVALID;
  const int K = params->n_poly + 1, M = params->n_int_1d, Kg = p_grid + 1;
  const int nI = params->n_elem[0], nJ = params->n_elem[1], nK = params->n_elem[2];
  if (K < 2 || M < 1 || nI < 1 || nJ < 1 || nK < 1 || Kg > 10 || M > 16) return VCPG_E_INVALID;
  StdElement se;
  try {
    se = vcpg::host::BuildStdElement(K, M, Kg, vcpg::host::SolLgl(dof_location), vcpg::host::GridLgl(dof_location));
  } catch (const std::exception &) {
    return VCPG_E_INVALID;
  }
  if (leg_int) std::memcpy(leg_int, se.leg.data(), sizeof(double) * K * M);
  if (dleg_int) std::memcpy(dleg_int, se.dleg.data(), sizeof(double) * K * M);
  if (leg_face) std::memcpy(leg_face, se.face.data(), sizeof(double) * 2 * K);
  if (dleg_face) std::memcpy(dleg_face, se.dface.data(), sizeof(double) * 2 * K);
  if (w_int) std::memcpy(w_int, se.wInt.data(), sizeof(double) * M);
  if (leg_dofs) std::memcpy(leg_dofs, se.legdof.data(), sizeof(double) * K * K);
  if (basis_center) std::memcpy(basis_center, se.center.data(), sizeof(double) * K * K * K);
  if (neighbors) vcpg::host::BlockNeighbors(nI, nJ, nK, periodic, neighbors);

  const int64_t nE = (int64_t)nI * nJ * nK;
  const int KG3 = Kg * Kg * Kg, MD = M * M * M, M2 = M * M;
  const size_t smem = sizeof(double) * ((size_t)3 * KG3 + Kg * Kg * std::max(Kg, M) +
                                        Kg * M * M + Kg * M + 9 * MD + 2 * Kg * M + 4 * Kg + M);
  // One element's arrays above the shared memory of a CTA (degree 9 with 14
  // points per direction): the host set-up, whose doubles the kernel reproduces.
  if (smem > 227 * 1024)
    return vcpg_setup_geometry(params, p_grid, dof_location, periodic, grid_nodes, leg_int,
                               dleg_int, leg_face, dleg_face, w_int, leg_dofs, basis_center,
                               vol_metric, face_metric, elem_scalars, neighbors);
  // Elements per pass: device buffers of at most about 1 GiB.
  const size_t perElem = sizeof(double) * ((size_t)3 * KG3 + 10 * MD + 78 * M2 + 15);
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(nE, (int64_t)((1ull << 30) / perElem)));
  std::vector<double> ops;
  ops.insert(ops.end(), se.lagInt.begin(), se.lagInt.end());
  ops.insert(ops.end(), se.dlagInt.begin(), se.dlagInt.end());
  ops.insert(ops.end(), se.lagFace.begin(), se.lagFace.end());
  ops.insert(ops.end(), se.dlagFace.begin(), se.dlagFace.end());
  ops.insert(ops.end(), se.wInt.begin(), se.wInt.end());
  double *dOps = nullptr, *dNodes = nullptr, *dVol = nullptr, *dFace = nullptr, *dSc = nullptr;
  int *dBad = nullptr;
  int rc = VCPG_OK, bad = 0;
  cudaError_t ce = cudaMalloc((void **)&dOps, sizeof(double) * ops.size());
  if (ce == cudaSuccess) ce = cudaMalloc((void **)&dNodes, sizeof(double) * 3 * KG3 * chunk);
  if (ce == cudaSuccess) ce = cudaMalloc((void **)&dVol, sizeof(double) * 10 * MD * chunk);
  if (ce == cudaSuccess) ce = cudaMalloc((void **)&dFace, sizeof(double) * 78 * M2 * chunk);
  if (ce == cudaSuccess) ce = cudaMalloc((void **)&dSc, sizeof(double) * 15 * chunk);
  if (ce == cudaSuccess) ce = cudaMalloc((void **)&dBad, sizeof(int));
  if (ce == cudaSuccess) ce = cudaMemcpy(dOps, ops.data(), sizeof(double) * ops.size(), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemset(dBad, 0, sizeof(int));
  if (ce == cudaSuccess && smem > 48 * 1024)
    ce = cudaFuncSetAttribute(vcpg::ElementMetricsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
  for (int64_t e0 = 0; ce == cudaSuccess && e0 < nE; e0 += chunk) {
    const int64_t n = std::min(chunk, nE - e0);
    ce = cudaMemcpy(dNodes, grid_nodes + e0 * 3 * KG3, sizeof(double) * 3 * KG3 * n,
                    cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) break;
    vcpg::MetricArgs a{dNodes, dOps, dOps + Kg * M, dOps + 2 * Kg * M, dOps + 2 * Kg * M + 2 * Kg,
                       dOps + 2 * Kg * M + 4 * Kg, dVol, dFace, dSc, dBad, (int)n, Kg, M};
    vcpg::ElementMetricsKernel<<<(unsigned)n, vcpg::kMetricThreads, smem>>>(a);
    ce = cudaGetLastError();
    if (ce == cudaSuccess)
      ce = cudaMemcpy(vol_metric + e0 * 10 * MD, dVol, sizeof(double) * 10 * MD * n, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(face_metric + e0 * 78 * M2, dFace, sizeof(double) * 78 * M2 * n, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(elem_scalars + e0 * 15, dSc, sizeof(double) * 15 * n, cudaMemcpyDeviceToHost);
  }
  if (ce == cudaSuccess) ce = cudaMemcpy(&bad, dBad, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dOps); cudaFree(dNodes); cudaFree(dVol); cudaFree(dFace); cudaFree(dSc); cudaFree(dBad);
  if (ce != cudaSuccess) {
    cudaGetLastError();   // a failed call leaves no error behind for later launches
    return VCPG_E_CUDA;
  }
  if (bad) rc = VCPG_E_INVALID;   // a non-positive Jacobian, as the host version rejects
  // The volume length scale: cube root on the host, as vcpg_setup_geometry takes it.
  for (int64_t e = 0; e < nE; ++e) {
    double *sc = elem_scalars + e * 15;
    const double lenVol = std::pow(sc[5], 1.0 / 3.0);
    sc[3] = lenVol / params->n_poly;
    sc[4] = lenVol;
  }
  return rc;
}

}  // extern "C"
