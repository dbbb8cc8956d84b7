// Host-side pre-processing: standard-element operators, metric terms, length
// scales and the nodal -> modal state conversion. This is the part of the
// reference solver's set-up that feeds the hot path, re-implemented from the
// mathematics it follows:
//   operators      StandardElementClass::DataStandardElement (src/StandardElementClass.cpp:105-911)
//   Legendre basis orthonormal Jacobi recursion (NormJacobi, src/StandAloneFunctions.cpp:329-383;
//                  Hesthaven & Warburton, "Nodal Discontinuous Galerkin Methods", 2008, JacobiP)
//   metrics        ElementClass::ComputeMetricTerms (src/ElementClass.cpp:1027-1407),
//                  FinalMetric[IJK]Face (:1907-2092)
//   length scales  ElementClass::ComputeLengthScales (src/ElementClass.cpp:927-1022)
//   state          SolverClass::ReadRestartSolution (src/SolverClass.cpp:3310-3366)
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "host_setup.h"

namespace vcpg {
namespace host {

// Orthonormal Jacobi polynomial P_n^(alpha,beta)(x) by the three-term recursion.
double NormJacobi(int n, int alpha, int beta, double x) {
  const double ap1 = alpha + 1, bp1 = beta + 1, apb = alpha + beta;
  const double apbp1 = apb + 1, apbp2 = apb + 2, apbp3 = apb + 3;
  const double b2ma2 = (double)(beta * beta - alpha * alpha);
  double gap1 = 1.0, gbp1 = 1.0, gapbp2 = 1.0;
  for (int i = 2; i <= alpha; ++i) gap1 *= i;
  for (int i = 2; i <= beta; ++i) gbp1 *= i;
  for (int i = 2; i <= alpha + beta + 1; ++i) gapbp2 *= i;
  double pm1 = std::sqrt(std::pow(0.5, apbp1) * gapbp2 / (gap1 * gbp1));
  double p = 0.5 * pm1 * (apbp2 * x + alpha - beta) * std::sqrt(apbp3 / (ap1 * bp1));
  if (n == 0) return pm1;
  for (int i = 2; i <= n; ++i) {
    const int j = i - 1;
    double t = 2 * j + apb;
    const double aim1 = 2.0 * std::sqrt(j * (j + apb) * (j + alpha) * (j + beta) / ((t - 1.0) * (t + 1.0))) / t;
    const double bi = b2ma2 / (t * (t + 2.0));
    t = 2 * i + apb;
    const double ai = 2.0 * std::sqrt(i * (i + apb) * (i + alpha) * (i + beta) / ((t - 1.0) * (t + 1.0))) / t;
    const double pn = ((x - bi) * p - aim1 * pm1) / ai;
    pm1 = p;
    p = pn;
  }
  return p;
}

// d/dx of the orthonormal Jacobi polynomial: sqrt(n(n+a+b+1)) P_{n-1}^(a+1,b+1).
double GradNormJacobi(int n, int alpha, int beta, double x) {
  if (n == 0) return 0.0;
  return std::sqrt((double)n * (n + alpha + beta + 1)) * NormJacobi(n - 1, alpha + 1, beta + 1, x);
}

// Gauss-Legendre points and weights on [-1, 1]: Newton iteration on P_n.
void GaussLegendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double z = -std::cos(pi * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    if (n == 1) { p1 = z; p0 = 1.0; }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
  for (int i = 0; i < n / 2; ++i) {  // exact symmetry
    const double xs = 0.5 * (x[n - 1 - i] - x[i]);
    x[i] = -xs;
    x[n - 1 - i] = xs;
    const double ws = 0.5 * (w[i] + w[n - 1 - i]);
    w[i] = w[n - 1 - i] = ws;
  }
}

// Nodal DOF locations (LocationDOFs1D, src/StandAloneFunctions.cpp:182-327):
// closed-form Gauss-Lobatto points up to 7 nodes, Newton iteration beyond.
void DofLocations(int n, int lgl, std::vector<double> &r) {
  r.assign(n, 0.0);
  if (!lgl) {
    const double dh = 2.0 / (n - 1);
    for (int i = 0; i < n; ++i) r[i] = -1.0 + i * dh;
    return;
  }
  switch (n) {
    case 1: r[0] = 0.0; return;
    case 2: r = {-1.0, 1.0}; return;
    case 3: r = {-1.0, 0.0, 1.0}; return;
    case 4: { const double a = std::sqrt(1.0 / 5.0); r = {-1.0, -a, a, 1.0}; return; }
    case 5: { const double a = std::sqrt(3.0 / 7.0); r = {-1.0, -a, 0.0, a, 1.0}; return; }
    case 6: {
      const double t1 = 2.0 * std::sqrt(7.0) / 21.0;
      const double t2 = std::sqrt(1.0 / 3.0 + t1), t3 = std::sqrt(1.0 / 3.0 - t1);
      r = {-1.0, -t2, -t3, t3, t2, 1.0};
      return;
    }
    case 7: {
      const double t1 = 2.0 * std::sqrt(5.0 / 3.0) / 11.0;
      const double t2 = std::sqrt(5.0 / 11.0 + t1), t3 = std::sqrt(5.0 / 11.0 - t1);
      r = {-1.0, -t2, -t3, 0.0, t3, t2, 1.0};
      return;
    }
    default: break;
  }
  // Interior LGL points are the roots of P'_{n-1}.
  const int N = n - 1;
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double x = -std::cos(pi * i / N);
    for (int it = 0; it < 100 && i > 0 && i < N; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= N; ++k) {
        const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      const double dx = (x * p1 - p0) / (n * p1);
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    r[i] = x;
  }
  r[0] = -1.0;
  r[N] = 1.0;
}

// In-place inverse of a row-major n x n matrix (Gauss-Jordan, partial pivoting).
void Invert(int n, std::vector<double> &A) {
  std::vector<double> B(n * n, 0.0);
  for (int i = 0; i < n; ++i) B[i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (A[p * n + c] == 0.0) throw std::runtime_error("singular Vandermonde matrix");
    if (p != c)
      for (int k = 0; k < n; ++k) { std::swap(A[p * n + k], A[c * n + k]); std::swap(B[p * n + k], B[c * n + k]); }
    const double inv = 1.0 / A[c * n + c];
    for (int k = 0; k < n; ++k) { A[c * n + k] *= inv; B[c * n + k] *= inv; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = A[r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; B[r * n + k] -= f * B[c * n + k]; }
    }
  }
  A = B;
}

}  // namespace host
}  // namespace vcpg

namespace vcpg {
namespace host {

namespace {

// out = op applied along axis ax of in[n2][n1][n0]; op is [nin][nout].
std::vector<double> ApplyAxis(const std::vector<double> &in, int n0, int n1, int n2, int ax,
                              const double *op, int nout) {
  const int nin = ax == 0 ? n0 : (ax == 1 ? n1 : n2);
  const int o0 = ax == 0 ? nout : n0, o1 = ax == 1 ? nout : n1, o2 = ax == 2 ? nout : n2;
  std::vector<double> out((size_t)o0 * o1 * o2, 0.0);
  for (int c2 = 0; c2 < o2; ++c2)
    for (int c1 = 0; c1 < o1; ++c1)
      for (int c0 = 0; c0 < o0; ++c0) {
        const int o = ax == 0 ? c0 : (ax == 1 ? c1 : c2);
        double acc = 0.0;
        for (int c = 0; c < nin; ++c) {
          const int i0 = ax == 0 ? c : c0, i1 = ax == 1 ? c : c1, i2 = ax == 2 ? c : c2;
          acc = std::fma(op[c * nout + o], in[((size_t)i2 * n1 + i1) * n0 + i0], acc);
        }
        out[((size_t)c2 * o1 + c1) * o0 + c0] = acc;
      }
  return out;
}

}  // namespace

StdElement BuildStdElement(int K, int M, int Kg, int dofLgl, int gridLgl) {
  StdElement se;
  se.K = K; se.M = M; se.Kg = Kg;
  GaussLegendre(M, se.rInt, se.wInt);
  DofLocations(K, dofLgl, se.rDof);
  DofLocations(Kg, gridLgl, se.rGrid);
  se.leg.resize(K * M); se.dleg.resize(K * M);
  for (int k = 0; k < K; ++k)
    for (int m = 0; m < M; ++m) {
      se.leg[k * M + m] = NormJacobi(k, 0, 0, se.rInt[m]);
      se.dleg[k * M + m] = GradNormJacobi(k, 0, 0, se.rInt[m]);
    }
  se.face.resize(2 * K); se.dface.resize(2 * K);
  for (int k = 0; k < K; ++k) {
    se.face[k] = NormJacobi(k, 0, 0, -1.0);
    se.face[K + k] = NormJacobi(k, 0, 0, 1.0);
    se.dface[k] = GradNormJacobi(k, 0, 0, -1.0);
    se.dface[K + k] = GradNormJacobi(k, 0, 0, 1.0);
  }
  se.legdof.resize(K * K);
  for (int k = 0; k < K; ++k)
    for (int i = 0; i < K; ++i) se.legdof[k * K + i] = NormJacobi(k, 0, 0, se.rDof[i]);
  std::vector<double> c0(K);
  for (int k = 0; k < K; ++k) c0[k] = NormJacobi(k, 0, 0, 0.0);
  se.center.resize(K * K * K);
  for (int k = 0, ii = 0; k < K; ++k)
    for (int j = 0; j < K; ++j)
      for (int i = 0; i < K; ++i, ++ii) se.center[ii] = c0[i] * c0[j] * c0[k];
  // Inverse Vandermonde matrix of the nodal DOFs: V(i, k) = P_k(r_i).
  std::vector<double> V(K * K);
  for (int i = 0; i < K; ++i)
    for (int k = 0; k < K; ++k) V[i * K + k] = NormJacobi(k, 0, 0, se.rDof[i]);
  Invert(K, V);  // V now holds (V^-1)(k, i) at [k * K + i]
  se.vandInv.resize(K * K);
  for (int c = 0; c < K; ++c)
    for (int o = 0; o < K; ++o) se.vandInv[c * K + o] = V[o * K + c];
  // Grid Lagrange basis = Vandermonde(points) * inverse Vandermonde(grid nodes).
  std::vector<double> Vg(Kg * Kg);
  for (int i = 0; i < Kg; ++i)
    for (int k = 0; k < Kg; ++k) Vg[i * Kg + k] = NormJacobi(k, 0, 0, se.rGrid[i]);
  Invert(Kg, Vg);  // (Vg^-1)(k, j) at [k * Kg + j]
  se.lagInt.assign(Kg * M, 0.0); se.dlagInt.assign(Kg * M, 0.0);
  for (int j = 0; j < Kg; ++j)
    for (int m = 0; m < M; ++m)
      for (int k = 0; k < Kg; ++k) {
        se.lagInt[j * M + m] += NormJacobi(k, 0, 0, se.rInt[m]) * Vg[k * Kg + j];
        se.dlagInt[j * M + m] += GradNormJacobi(k, 0, 0, se.rInt[m]) * Vg[k * Kg + j];
      }
  se.lagDof.assign(Kg * K, 0.0); se.dlagDof.assign(Kg * K, 0.0);
  for (int j = 0; j < Kg; ++j)
    for (int m = 0; m < K; ++m)
      for (int k = 0; k < Kg; ++k) {
        se.lagDof[j * K + m] += NormJacobi(k, 0, 0, se.rDof[m]) * Vg[k * Kg + j];
        se.dlagDof[j * K + m] += GradNormJacobi(k, 0, 0, se.rDof[m]) * Vg[k * Kg + j];
      }
  se.dlegdof.resize(K * K);
  for (int k = 0; k < K; ++k)
    for (int i = 0; i < K; ++i) se.dlegdof[k * K + i] = GradNormJacobi(k, 0, 0, se.rDof[i]);
  se.lagFace.assign(2 * Kg, 0.0); se.dlagFace.assign(2 * Kg, 0.0);
  se.lagFace[0] = 1.0;
  se.lagFace[Kg + Kg - 1] = 1.0;
  for (int j = 0; j < Kg; ++j)
    for (int k = 0; k < Kg; ++k) {
      se.dlagFace[j] += GradNormJacobi(k, 0, 0, -1.0) * Vg[k * Kg + j];
      se.dlagFace[Kg + j] += GradNormJacobi(k, 0, 0, 1.0) * Vg[k * Kg + j];
    }
  return se;
}

void ElementMetrics(const StdElement &se, const double *gridNodes, double *vol, double *face,
                    double *scalars, int nPoly) {
  const int Kg = se.Kg, M = se.M, MD = M * M * M, M2 = M * M;
  const int KG3 = Kg * Kg * Kg;
  // Volume: coordinates derivatives at the integration points (k, then j, then i).
  std::vector<double> dc((size_t)9 * MD);  // [param][coord][point]
  for (int x = 0; x < 3; ++x) {
    std::vector<double> g(gridNodes + x * KG3, gridNodes + (x + 1) * KG3);
    for (int q = 0; q < 3; ++q) {
      std::vector<double> t = ApplyAxis(g, Kg, Kg, Kg, 2, (q == 2 ? se.dlagInt : se.lagInt).data(), M);
      t = ApplyAxis(t, Kg, Kg, M, 1, (q == 1 ? se.dlagInt : se.lagInt).data(), M);
      t = ApplyAxis(t, Kg, M, M, 0, (q == 0 ? se.dlagInt : se.lagInt).data(), M);
      for (int l = 0; l < MD; ++l) dc[(q * 3 + x) * MD + l] = t[l];
    }
  }
  for (int l = 0; l < MD; ++l) {
    const double dxdr = dc[(0 * 3 + 0) * MD + l], dydr = dc[(0 * 3 + 1) * MD + l], dzdr = dc[(0 * 3 + 2) * MD + l];
    const double dxds = dc[(1 * 3 + 0) * MD + l], dyds = dc[(1 * 3 + 1) * MD + l], dzds = dc[(1 * 3 + 2) * MD + l];
    const double dxdt = dc[(2 * 3 + 0) * MD + l], dydt = dc[(2 * 3 + 1) * MD + l], dzdt = dc[(2 * 3 + 2) * MD + l];
    const double J = dxdr * (dyds * dzdt - dzds * dydt) - dxds * (dydr * dzdt - dzdr * dydt) +
                     dxdt * (dydr * dzds - dzdr * dyds);
    if (!(J > 0.0)) throw std::runtime_error("negative or zero Jacobian");
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
  // Faces: face-normal evaluation, then the fast and the slow in-face axes.
  for (int f = 0; f < 6; ++f) {
    const int d = f / 2, side = f % 2;
    const double *fv = se.lagFace.data() + side * Kg, *dfv = se.dlagFace.data() + side * Kg;
    const int fastAx = d == 0 ? 1 : 0, slowAx = d == 2 ? 1 : 2;
    std::vector<double> fdc((size_t)9 * M2);  // [param][coord][point]
    for (int x = 0; x < 3; ++x) {
      std::vector<double> g(gridNodes + x * KG3, gridNodes + (x + 1) * KG3);
      for (int q = 0; q < 3; ++q) {
        int n[3] = {Kg, Kg, Kg};
        std::vector<double> t = ApplyAxis(g, n[0], n[1], n[2], d, q == d ? dfv : fv, 1);
        n[d] = 1;
        t = ApplyAxis(t, n[0], n[1], n[2], fastAx, (q == fastAx ? se.dlagInt : se.lagInt).data(), M);
        n[fastAx] = M;
        t = ApplyAxis(t, n[0], n[1], n[2], slowAx, (q == slowAx ? se.dlagInt : se.lagInt).data(), M);
        for (int l = 0; l < M2; ++l) fdc[(q * 3 + x) * M2 + l] = t[l];
      }
    }
    double *fm = face + (size_t)f * 13 * M2;
    for (int l = 0; l < M2; ++l) {
      const double dxdr = fdc[(0 * 3 + 0) * M2 + l], dydr = fdc[(0 * 3 + 1) * M2 + l], dzdr = fdc[(0 * 3 + 2) * M2 + l];
      const double dxds = fdc[(1 * 3 + 0) * M2 + l], dyds = fdc[(1 * 3 + 1) * M2 + l], dzds = fdc[(1 * 3 + 2) * M2 + l];
      const double dxdt = fdc[(2 * 3 + 0) * M2 + l], dydt = fdc[(2 * 3 + 1) * M2 + l], dzdt = fdc[(2 * 3 + 2) * M2 + l];
      double nx, ny, nz;
      if (d == 0) {
        nx = dyds * dzdt - dydt * dzds; ny = dxdt * dzds - dxds * dzdt; nz = dxds * dydt - dxdt * dyds;
      } else if (d == 1) {
        nx = dydt * dzdr - dydr * dzdt; ny = dxdr * dzdt - dxdt * dzdr; nz = dxdt * dydr - dxdr * dydt;
      } else {
        nx = dydr * dzds - dyds * dzdr; ny = dxds * dzdr - dxdr * dzds; nz = dxdr * dyds - dxds * dydr;
      }
      const double lenNorm = std::sqrt(nx * nx + ny * ny + nz * nz);
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
  }
  // Length scales and averaged normals (ElementClass::ComputeLengthScales).
  double volElem = 0.0;
  for (int k = 0, l = 0; k < M; ++k)
    for (int j = 0; j < M; ++j)
      for (int i = 0; i < M; ++i, ++l) volElem += se.wInt[i] * se.wInt[j] * se.wInt[k] * vol[l];
  const double lenVol = std::pow(volElem, 1.0 / 3.0);
  scalars[3] = lenVol / nPoly;
  scalars[4] = lenVol;
  scalars[5] = volElem;
  for (int d = 0; d < 3; ++d) {
    const double *fmin = face + (size_t)(2 * d) * 13 * M2, *fmax = fmin + 13 * M2;
    double s = 0.0, a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 0, l = 0; j < M; ++j)
      for (int i = 0; i < M; ++i, ++l) {
        const double w = se.wInt[i] * se.wInt[j];
        a0 += w * (fmin[l] * fmin[3 * M2 + l] + fmax[l] * fmax[3 * M2 + l]);
        a1 += w * (fmin[M2 + l] * fmin[3 * M2 + l] + fmax[M2 + l] * fmax[3 * M2 + l]);
        a2 += w * (fmin[2 * M2 + l] * fmin[3 * M2 + l] + fmax[2 * M2 + l] * fmax[3 * M2 + l]);
        s += w * (fmin[3 * M2 + l] + fmax[3 * M2 + l]);
      }
    scalars[d] = 2.0 * volElem / s;
    scalars[6 + 3 * d] = a0 / s;
    scalars[7 + 3 * d] = a1 / s;
    scalars[8 + 3 * d] = a2 / s;
  }
}

void NodalMetrics(const StdElement &se, const double *gridNodes, double *out) {
  const int Kg = se.Kg, K = se.K, KD = K * K * K, KG3 = Kg * Kg * Kg;
  std::vector<double> dc((size_t)9 * KD);  // [param][coord][DOF]
  for (int x = 0; x < 3; ++x) {
    std::vector<double> g(gridNodes + x * KG3, gridNodes + (x + 1) * KG3);
    for (int q = 0; q < 3; ++q) {
      std::vector<double> t = ApplyAxis(g, Kg, Kg, Kg, 2, (q == 2 ? se.dlagDof : se.lagDof).data(), K);
      t = ApplyAxis(t, Kg, Kg, K, 1, (q == 1 ? se.dlagDof : se.lagDof).data(), K);
      t = ApplyAxis(t, Kg, K, K, 0, (q == 0 ? se.dlagDof : se.lagDof).data(), K);
      for (int l = 0; l < KD; ++l) dc[((size_t)q * 3 + x) * KD + l] = t[l];
    }
  }
  for (int l = 0; l < KD; ++l) {
    const double dxdr = dc[0 * KD + l], dydr = dc[1 * KD + l], dzdr = dc[2 * KD + l];
    const double dxds = dc[3 * KD + l], dyds = dc[4 * KD + l], dzds = dc[5 * KD + l];
    const double dxdt = dc[6 * KD + l], dydt = dc[7 * KD + l], dzdt = dc[8 * KD + l];
    const double J = dxdr * (dyds * dzdt - dzds * dydt) - dxds * (dydr * dzdt - dzdr * dydt) +
                     dxdt * (dydr * dzds - dzdr * dyds);
    if (!(J > 0.0)) throw std::runtime_error("negative or zero Jacobian at a nodal DOF");
    const double Jinv = 1.0 / J;
    out[0 * KD + l] = J;
    out[1 * KD + l] = Jinv * (dyds * dzdt - dzds * dydt);
    out[2 * KD + l] = Jinv * (dzds * dxdt - dxds * dzdt);
    out[3 * KD + l] = Jinv * (dxds * dydt - dyds * dxdt);
    out[4 * KD + l] = Jinv * (dzdr * dydt - dydr * dzdt);
    out[5 * KD + l] = Jinv * (dxdr * dzdt - dzdr * dxdt);
    out[6 * KD + l] = Jinv * (dydr * dxdt - dxdr * dydt);
    out[7 * KD + l] = Jinv * (dydr * dzds - dzdr * dyds);
    out[8 * KD + l] = Jinv * (dzdr * dxds - dxdr * dzds);
    out[9 * KD + l] = Jinv * (dxdr * dyds - dydr * dxds);
  }
}

void BlockNeighbors(int nI, int nJ, int nK, const int32_t periodic[3], int32_t *neighbors) {
  const int n[3] = {nI, nJ, nK};
  for (int k = 0; k < nK; ++k)
    for (int j = 0; j < nJ; ++j)
      for (int i = 0; i < nI; ++i) {
        const int64_t e = ((int64_t)k * nJ + j) * nI + i;
        const int idx[3] = {i, j, k};
        for (int d = 0; d < 3; ++d)
          for (int s = 0; s < 2; ++s) {
            int c[3] = {idx[0], idx[1], idx[2]};
            c[d] += s == 0 ? -1 : 1;
            int32_t nb = -1;
            if (c[d] < 0 || c[d] >= n[d]) {
              if (periodic && periodic[d]) c[d] = (c[d] + n[d]) % n[d];
              else c[d] = -1;
            }
            if (c[d] >= 0) nb = (int32_t)(((int64_t)c[2] * nJ + c[1]) * nI + c[0]);
            neighbors[e * 6 + 2 * d + s] = nb;
          }
      }
}

}  // namespace host
}  // namespace vcpg
