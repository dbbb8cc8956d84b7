// Host-side set-up of open boundaries: the characteristic boundary-face list and
// its configuration, the polynomial-correction (PC) operators, the boundary
// areas, and the sponge-layer / characteristic-matching-layer data.
//
// Reference routines whose results this reproduces:
//   PC matrix, Lagrange operators   StandardElementClass::AssemblePolynomialCorrectionOperators
//                                   and ValuesLagrangeBasis1D (src/StandardElementClass.cpp:181-394)
//   boundary indices                BCStandardCharacteristicSubfaceClass::IdentifyBoundaryIndices
//                                   (src/BoundaryState.cpp:829-928)
//   NSCBC parameters                ConfigureParamNSCBC (src/SubfaceClasses.cpp:1349-1436)
//   prescribed data                 ConvertPrescribedData (src/SubfaceClasses.cpp:1304-1318, 1473-1495)
//   boundary areas                  ElementClass::ComputeSurfaceAreaBoundary (src/ElementClass.cpp:303-330)
//   sponge layer                    SolverClass::InitSpongeLayer / SetUpSpongeLayer[IJK]M(IN|AX),
//                                   ElementClass::ConfigureSpongeLayer / InitializeDampingState
//                                   (src/SpongeLayer.cpp:13-665, 844-1000)
#include "open_boundary.h"

#include <cmath>
#include <cstring>
#include <stdexcept>

#include "host_setup.h"

namespace vcpg {
namespace {

constexpr double kGamma = 1.4;
constexpr double kRGas = 287.058;                      // RGas (include/VCP3D_CurviLinear.hpp:177)
constexpr double kCp = kGamma * kRGas / (kGamma - 1.0);  // Cp
constexpr double kEpsThreshold = 1.e-10;  // include/VCP3D_CurviLinear.hpp:137

// Lagrange basis on `nodes` at `pts`: val[j * nP + i] = L_j(pts[i]) and its
// derivative, through the Legendre Vandermonde matrices as in
// StandardElementClass::LagrangianBasisFunctions (src/StandardElementClass.cpp:498-600).
void Lagrange(const std::vector<double> &nodes, const std::vector<double> &pts,
              std::vector<double> &val, std::vector<double> &der) {
  const int n = (int)nodes.size(), nP = (int)pts.size();
  std::vector<double> V(n * n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) V[i * n + k] = host::NormJacobi(k, 0, 0, nodes[i]);
  host::Invert(n, V);  // (V^-1)(k, j) at [k * n + j]
  val.assign((size_t)n * nP, 0.0);
  der.assign((size_t)n * nP, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < nP; ++i)
      for (int k = 0; k < n; ++k) {
        val[j * nP + i] += host::NormJacobi(k, 0, 0, pts[i]) * V[k * n + j];
        der[j * nP + i] += host::GradNormJacobi(k, 0, 0, pts[i]) * V[k * n + j];
      }
}

// Coordinates of the integration points of one element from its grid nodes
// gridNodes[3][Kg^3] with the grid Lagrange basis lag[Kg][M]: out[3][M^3],
// contracted one axis at a time (k, then j, then i).
void IntegrationPointCoordinates(const double *gridNodes, int Kg, int M,
                                 const std::vector<double> &lag, double *out) {
  const int KG3 = Kg * Kg * Kg, MD = M * M * M;
  std::vector<double> t1((size_t)M * Kg * Kg), t2((size_t)M * M * Kg);
  for (int x = 0; x < 3; ++x) {
    const double *g = gridNodes + x * KG3;  // [c][b][a]
    for (int k = 0; k < M; ++k)
      for (int b = 0; b < Kg; ++b)
        for (int a = 0; a < Kg; ++a) {
          double acc = 0.0;
          for (int c = 0; c < Kg; ++c) acc += lag[c * M + k] * g[(c * Kg + b) * Kg + a];
          t1[((size_t)k * Kg + b) * Kg + a] = acc;
        }
    for (int k = 0; k < M; ++k)
      for (int j = 0; j < M; ++j)
        for (int a = 0; a < Kg; ++a) {
          double acc = 0.0;
          for (int b = 0; b < Kg; ++b) acc += lag[b * M + j] * t1[((size_t)k * Kg + b) * Kg + a];
          t2[((size_t)k * M + j) * Kg + a] = acc;
        }
    for (int k = 0; k < M; ++k)
      for (int j = 0; j < M; ++j)
        for (int i = 0; i < M; ++i) {
          double acc = 0.0;
          for (int a = 0; a < Kg; ++a) acc += lag[a * M + i] * t2[((size_t)k * M + j) * Kg + a];
          out[x * MD + (k * M + j) * M + i] = acc;
        }
  }
}

// Parametric axis of the face normal and the transverse axes, from the face
// metric at point 0: the normal is the axis whose metric gradient is parallel
// to the unit normal (cosine within 1e-10 of one).
bool IdentifyBoundaryIndices(const double *fm, int M2, int grad[3]) {
  const double nx = fm[0 * M2], ny = fm[1 * M2], nz = fm[2 * M2];
  int found = -1;
  for (int i = 0; i < 3; ++i) {
    const double gx = fm[(4 + 3 * i) * M2], gy = fm[(5 + 3 * i) * M2], gz = fm[(6 + 3 * i) * M2];
    const double len = std::sqrt(gx * gx + gy * gy + gz * gz);
    const double cosT = (nx * gx + ny * gy + nz * gz) / len;
    if (std::fabs(cosT - 1.0) < kEpsThreshold) {
      if (found >= 0) return false;
      found = i;
    }
  }
  if (found < 0) return false;
  grad[0] = found;
  grad[1] = found == 0 ? 1 : 0;
  grad[2] = found == 2 ? 1 : 2;
  return true;
}

}  // namespace

// Non-dimensional prescribed data of a boundary condition through a boundary
// state, as the subfaces' ConvertPrescribedData / PrescribedDataFromFreeStream
// produce them (src/SubfaceClasses.cpp:542-620, 739-751, 863-915, 1026-1109,
// 1169-1180): heat flux / (p_ref u_ref); for the isothermal wall the value
// -p_ref / (R rho_ref T_wall) that becomes the wall's V4; for the far field and
// the supersonic inflow the entropy variables of the state; for the subsonic
// inflow p_t / p_ref, the total enthalpy Cp T_t / u_ref^2 and the unit
// direction; for the subsonic outflow p / p_ref.
static void EntropyFromPrimitive(double rho, double u, double v, double w, double p,
                                 double *V) {
  const double ovgm1 = 1.0 / (kGamma - 1.0);
  const double s = std::log(p / std::pow(rho, kGamma));
  const double pInv = 1.0 / p;
  V[0] = (kGamma - s) * ovgm1 - 0.5 * pInv * rho * (u * u + v * v + w * w);
  V[1] = rho * u * pInv;
  V[2] = rho * v * pInv;
  V[3] = rho * w * pInv;
  V[4] = -rho * pInv;
}

static void WeakBoundaryData(int type, const vcpg_open_boundary &ob, int f,
                             const vcpg_params &prm, double *pres) {
  const double rhoRefInv = 1.0 / prm.rho_ref, uRefInv = 1.0 / prm.u_ref,
               pRefInv = 1.0 / prm.p_ref;
  switch (type) {
    case VCPG_BC_WALL_HEAT_FLUX:
      pres[0] = ob.wall_data[f] * (1.0 / (prm.p_ref * prm.u_ref));
      break;
    case VCPG_BC_WALL_ISOTHERMAL:
      pres[0] = (-prm.p_ref / (kRGas * prm.rho_ref)) / ob.wall_data[f];
      break;
    case VCPG_BC_FARFIELD: {
      const double *q = ob.free_stream;
      EntropyFromPrimitive(q[0] / prm.rho_ref, q[1] / prm.u_ref, q[2] / prm.u_ref,
                           q[3] / prm.u_ref, q[4] / prm.p_ref, pres);
      break;
    }
    case VCPG_BC_INFLOW_SUPERSONIC: {
      const double *q = ob.inflow_super[f];
      EntropyFromPrimitive(q[0] * rhoRefInv, q[1] * uRefInv, q[2] * uRefInv, q[3] * uRefInv,
                           q[4] * pRefInv, pres);
      break;
    }
    case VCPG_BC_INFLOW_SUBSONIC: {
      const double *t = ob.inflow_total[f];
      const double len2 = t[2] * t[2] + t[3] * t[3] + t[4] * t[4];
      const double lenInv = 1.0 / std::sqrt(len2);
      pres[0] = t[0] * pRefInv;
      pres[1] = t[1] * (kCp * uRefInv * uRefInv);
      pres[2] = t[2] * lenInv;
      pres[3] = t[3] * lenInv;
      pres[4] = t[4] * lenInv;
      break;
    }
    case VCPG_BC_OUTFLOW_SUBSONIC:
      pres[0] = ob.p_out[f] * pRefInv;
      break;
    default:
      break;
  }
}

int BuildOpenBoundary(const vcpg_params &prm, const vcpg_open_boundary &ob,
                      const vcpg_geometry &geom, int pGrid, int dofLocation,
                      const double *gridNodes, OpenBoundaryHost &out, std::string &err,
                      const vcpg_subface *subfaces, int nSubfaces) {
  try {
    const int K = prm.n_poly + 1, M = prm.n_int_1d, M2 = M * M, MD = M * M * M;
    const int nI = prm.n_elem[0], nJ = prm.n_elem[1], nK = prm.n_elem[2];
    const int64_t nE = (int64_t)nI * nJ * nK;
    if (!geom.face_metric || !geom.neighbors) { err = "geometry arrays missing"; return VCPG_E_INVALID; }
    auto badBc = [](int bc) { return bc < VCPG_BC_NONE || bc > VCPG_BC_OUTFLOW_SUPERSONIC; };
    for (int f = 0; f < 6; ++f)
      if (badBc(ob.bc[f])) {
        err = "unknown boundary condition on face " + std::to_string(f);
        return VCPG_E_INVALID;
      }
    // Subfaces: per subface a copy of ob carrying the subface's condition and
    // prescribed data in its block face's slots, so that every element face reads
    // its settings from one vcpg_open_boundary.
    if (nSubfaces < 0 || (nSubfaces > 0 && !subfaces)) { err = "invalid subface list"; return VCPG_E_INVALID; }
    std::vector<vcpg_open_boundary> subOb((size_t)nSubfaces, ob);
    bool faceHasSub[6] = {false, false, false, false, false, false};
    const int nIdx[3] = {nI, nJ, nK};
    for (int s2 = 0; s2 < nSubfaces; ++s2) {
      const vcpg_subface &sf = subfaces[s2];
      if (sf.face < 0 || sf.face > 5 || badBc(sf.bc)) {
        err = "subface " + std::to_string(s2) + ": invalid block face or boundary condition";
        return VCPG_E_INVALID;
      }
      const int fd = sf.face / 2, a0 = fd == 0 ? 1 : 0, a1 = fd == 2 ? 1 : 2;
      if (sf.elem_begin[0] < 0 || sf.elem_begin[1] < 0 || sf.elem_end[0] > nIdx[a0] ||
          sf.elem_end[1] > nIdx[a1] || sf.elem_begin[0] >= sf.elem_end[0] ||
          sf.elem_begin[1] >= sf.elem_end[1]) {
        err = "subface " + std::to_string(s2) + ": element range outside its block face";
        return VCPG_E_INVALID;
      }
      faceHasSub[sf.face] = true;
      vcpg_open_boundary &o = subOb[s2];
      const int f = sf.face;
      o.bc[f] = sf.bc;
      o.p_out[f] = sf.p_out;
      for (int q = 0; q < 4; ++q) o.inflow[f][q] = sf.inflow[q];
      for (int q = 0; q < 5; ++q) o.inflow_total[f][q] = sf.inflow_total[q];
      o.wall_data[f] = sf.wall_data;
      for (int q = 0; q < 5; ++q) o.inflow_super[f][q] = sf.inflow_super[q];
    }
    // The settings of element e's block face f: its subface's, or ob's (which
    // subface in *which: -1 for ob).
    auto settingsOf = [&](int64_t e, int f, std::string &why,
                          int *which) -> const vcpg_open_boundary * {
      *which = -1;
      if (!faceHasSub[f]) return &ob;
      const int64_t idx[3] = {e % nI, (e / nI) % nJ, e / ((int64_t)nI * nJ)};
      const int fd = f / 2, a0 = fd == 0 ? 1 : 0, a1 = fd == 2 ? 1 : 2;
      const vcpg_open_boundary *hit = nullptr;
      int hits = 0;
      for (int s2 = 0; s2 < nSubfaces; ++s2) {
        const vcpg_subface &sf = subfaces[s2];
        if (sf.face != f) continue;
        if (idx[a0] >= sf.elem_begin[0] && idx[a0] < sf.elem_end[0] &&
            idx[a1] >= sf.elem_begin[1] && idx[a1] < sf.elem_end[1]) {
          hit = &subOb[s2];
          *which = s2;
          ++hits;
        }
      }
      if (hits != 1)
        why = "element " + std::to_string(e) + " face " + std::to_string(f) + " is covered by " +
              std::to_string(hits) + " subfaces (exactly one expected)";
      return hits == 1 ? hit : nullptr;
    };

    // 1-D operators: Lagrange basis of the solution DOFs at the Gauss points, its
    // derivative at the DOFs, and the Lagrange derivative on the Gauss points.
    std::vector<double> rInt, wInt, rDof;
    host::GaussLegendre(M, rInt, wInt);
    host::DofLocations(K, host::SolLgl(dofLocation), rDof);
    std::vector<double> lqv, lqd, ldv, ldd, qqv, qqd;
    Lagrange(rDof, rInt, lqv, lqd);   // lqv[j * M + i] = L_j(q_i)
    Lagrange(rDof, rDof, ldv, ldd);   // ldd[j * K + i] = L_j'(r_i)
    Lagrange(rInt, rInt, qqv, qqd);   // qqd[k * M + i] = l_k'(q_i)
    const double c0 = -ldd[0];        // -L_0'(r_0)
    out.dlq.assign(M * M, 0.0);
    for (int i = 0; i < M; ++i)
      for (int k = 0; k < M; ++k) out.dlq[i * M + k] = qqd[k * M + i];

    // PC matrix A = L2D (dL2D^T dL2D)^-1 dL2D^T with dL2D = c0 L2D, where L2D maps
    // the K^2 face DOFs to the M^2 face integration points.
    const int K2 = K * K;
    std::vector<double> L2D((size_t)M2 * K2), dL2D((size_t)M2 * K2);
    for (int i1 = 0; i1 < M; ++i1)
      for (int i2 = 0; i2 < M; ++i2)
        for (int j1 = 0; j1 < K; ++j1)
          for (int j2 = 0; j2 < K; ++j2) {
            const double v = lqv[j1 * M + i1] * lqv[j2 * M + i2];
            L2D[(size_t)(i1 * M + i2) * K2 + j1 * K + j2] = v;
            dL2D[(size_t)(i1 * M + i2) * K2 + j1 * K + j2] = v * c0;
          }
    std::vector<double> LS((size_t)K2 * K2, 0.0);
    for (int i = 0; i < K2; ++i)
      for (int j = 0; j < K2; ++j)
        for (int k = 0; k < M2; ++k) LS[i * K2 + j] += dL2D[(size_t)k * K2 + i] * dL2D[(size_t)k * K2 + j];
    host::Invert(K2, LS);
    std::vector<double> PCt((size_t)K2 * M2, 0.0);
    for (int i = 0; i < K2; ++i)
      for (int j = 0; j < M2; ++j) {
        double t = 0.0;
        for (int k = 0; k < K2; ++k) t += LS[i * K2 + k] * dL2D[(size_t)j * K2 + k];
        PCt[(size_t)i * M2 + j] = t;
      }
    out.pc.assign((size_t)M2 * M2, 0.0);
    for (int i = 0; i < M2; ++i)
      for (int j = 0; j < M2; ++j) {
        double t = 0.0;
        for (int k = 0; k < K2; ++k) t += L2D[(size_t)i * K2 + k] * PCt[(size_t)k * M2 + j];
        out.pc[(size_t)i * M2 + j] = t;
      }

    // Boundary faces, per block face in element order (the order of the
    // reference's boundary sums), and their configuration.
    out.nbrCode.assign(geom.neighbors, geom.neighbors + nE * 6);
    out.bface.clear();
    out.bpresc.clear();
    out.nB = 0;
    for (int f = 0; f < 6; ++f) {
      BlockFaceCfg &c = out.cfg[f];
      c = BlockFaceCfg{};
      c.type = faceHasSub[f] ? -1 : ob.bc[f];
      c.first = out.nB;
      const double factNorm = (f % 2 == 0) ? -1.0 : 1.0;
      c.dell = factNorm * c0;
      c.iPhi = factNorm > 0.0 ? 0 : 4;
      c.sigma = ob.outlet_sigma; c.len = ob.outlet_len;
      c.betaL = ob.outlet_beta_l; c.betaT = ob.outlet_beta_t;
      c.oneMinusBeta = ob.outlet_one_minus_beta ? 1 : 0;
      c.inSigma = ob.inlet_sigma; c.inLen = ob.inlet_len;
      c.incoming = ob.inlet_incoming ? 1 : 0;
      c.localMach = ob.outlet_local_mach ? 1 : 0;
      std::vector<int> rowSub;   // subface of each of this block face's rows
      for (int64_t e = 0; e < nE; ++e) {
        if (geom.neighbors[e * 6 + f] >= 0) continue;
        std::string why;
        int which = -1;
        const vcpg_open_boundary *o = settingsOf(e, f, why, &which);
        if (!o) { err = why; return VCPG_E_INVALID; }
        const int type = o->bc[f];
        if (type == VCPG_BC_NONE) continue;  // stays -1: flagged by the residual kernel
        if (type == VCPG_BC_INFLOW_TOTAL_NSCBC || type == VCPG_BC_INFLOW_SUBSONIC) {
          const double *t = o->inflow_total[f];
          const double dl = std::sqrt(t[2] * t[2] + t[3] * t[3] + t[4] * t[4]);
          if (!(t[0] > 0.0) || !(t[1] > 0.0) || !(dl > 0.0)) {
            err = "total inflow needs a positive total pressure, total temperature and a "
                  "velocity direction on face " + std::to_string(f);
            return VCPG_E_INVALID;
          }
        }
        const bool weak = type >= VCPG_BC_WALL_HEAT_FLUX;
        const double len = type == VCPG_BC_OUTFLOW_NSCBC ? c.len : c.inLen;
        if (!weak && !(len > 0.0)) {
          err = "characteristic length must be positive on face " + std::to_string(f);
          return VCPG_E_INVALID;
        }
        const double *fm = geom.face_metric + ((size_t)e * 6 + f) * 13 * M2;
        const int fd = f / 2;
        int grad[3] = {fd, fd == 0 ? 1 : 0, fd == 2 ? 1 : 2};
        if (!weak && !IdentifyBoundaryIndices(fm, M2, grad)) {
          err = "could not identify the boundary indices of element " + std::to_string(e) +
                " face " + std::to_string(f) + " (characteristic faces must be aligned with "
                "a parametric direction)";
          return VCPG_E_INVALID;
        }
        const int b = out.nB++;
        rowSub.push_back(which);
        int row[kBfStride] = {(int)e, f, type, grad[0], grad[1], grad[2], 0, b};
        out.bface.insert(out.bface.end(), row, row + kBfStride);
        double pres[kPrescStride] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (type == VCPG_BC_OUTFLOW_NSCBC) {
          pres[0] = o->p_out[f] / prm.p_ref;
        } else if (type == VCPG_BC_INFLOW_STATIC_NSCBC) {
          pres[0] = o->inflow[f][0] / prm.rho_ref;
          pres[1] = o->inflow[f][1] / prm.u_ref;
          pres[2] = o->inflow[f][2] / prm.u_ref;
          pres[3] = o->inflow[f][3] / prm.u_ref;
        } else if (type == VCPG_BC_INFLOW_TOTAL_NSCBC) {
          // BCInflowTotalCharacteristicSubfaceClass::ConvertPrescribedData
          // (src/SubfaceClasses.cpp:1577-1608): p_t / p_ref, T_t / (p_ref / rho_ref)
          // (the gas constant stays in the boundary formulas), unit direction.
          const double *t = o->inflow_total[f];
          const double dl = std::sqrt(t[2] * t[2] + t[3] * t[3] + t[4] * t[4]);
          pres[0] = t[0] / prm.p_ref;
          pres[1] = t[1] / (prm.p_ref / prm.rho_ref);
          pres[2] = t[2] / dl;
          pres[3] = t[3] / dl;
          pres[4] = t[4] / dl;
        } else {
          WeakBoundaryData(type, *o, f, prm, pres);
        }
        out.bpresc.insert(out.bpresc.end(), pres, pres + kPrescStride);
        out.nbrCode[e * 6 + f] = -2 - b;
        for (int l = 0; l < M2; ++l) c.area += wInt[l % M] * wInt[l / M] * fm[3 * M2 + l];
      }
      c.count = out.nB - c.first;
      // The last face of each subface (rows are in element order): index by
      // subface (+1, so that the whole-face settings -1 take slot 0).
      std::vector<int> lastOf((size_t)nSubfaces + 1, -1);
      for (int r = 0; r < c.count; ++r) lastOf[(size_t)(rowSub[r] + 1)] = c.first + r;
      for (int r = 0; r < c.count; ++r)
        out.bface[(size_t)(c.first + r) * kBfStride + kBfLast] = lastOf[(size_t)(rowSub[r] + 1)];
    }

    // Sponge layers and the characteristic matching layer.
    const int *nb = ob.sponge_elems;
    bool anySponge = false;
    for (int f = 0; f < 6; ++f) {
      if (nb[f] < 0) { err = "negative sponge-layer thickness"; return VCPG_E_INVALID; }
      anySponge = anySponge || nb[f] > 0;
    }
    out.spongeIdx.assign(nE, -1);
    out.nS = 0;
    out.dampFn.clear(); out.dampState.clear(); out.cml.clear();
    out.cmlOn = ob.cml ? 1 : 0;
    if (ob.cml && !anySponge) { err = "the matching layer acts in sponge elements: no sponge given"; return VCPG_E_INVALID; }
    if (anySponge) {
      if (!gridNodes || pGrid < 1) { err = "sponge layers need the grid nodes"; return VCPG_E_INVALID; }
      const int Kg = pGrid + 1, KG3 = Kg * Kg * Kg;
      std::vector<double> rGrid, lgv, lgd;
      host::DofLocations(Kg, host::GridLgl(dofLocation), rGrid);
      Lagrange(rGrid, rInt, lgv, lgd);
      const int n[3] = {nI, nJ, nK};
      // Layer membership per element and direction: bit 2 d = min side, 2 d + 1 = max side.
      std::vector<int> flags(nE, 0);
      for (int k = 0; k < nK; ++k)
        for (int j = 0; j < nJ; ++j)
          for (int i = 0; i < nI; ++i) {
            const int idx[3] = {i, j, k};
            int fl = 0;
            for (int d = 0; d < 3; ++d) {
              if (idx[d] < nb[2 * d]) fl |= 1 << (2 * d);
              if (idx[d] >= n[d] - nb[2 * d + 1]) fl |= 1 << (2 * d + 1);
              if (((fl >> (2 * d)) & 3) == 3) {
                err = "sponge layers of opposite faces overlap";
                return VCPG_E_INVALID;
              }
            }
            flags[((int64_t)k * nJ + j) * nI + i] = fl;
          }
      // Extent of each layer: coordinate of the element's first DOF and of the
      // last DOF along the layer direction (grid corners).
      double lo[6], hi[6];
      for (int f = 0; f < 6; ++f) { lo[f] = 1.e+30; hi[f] = -1.e+30; }
      for (int64_t e = 0; e < nE; ++e)
        for (int f = 0; f < 6; ++f) {
          if (!((flags[e] >> f) & 1)) continue;
          const int d = f / 2;
          const int last = d == 0 ? Kg - 1 : (d == 1 ? (Kg - 1) * Kg : (Kg - 1) * Kg * Kg);
          const double *g = gridNodes + e * 3 * KG3 + d * KG3;
          lo[f] = std::min(lo[f], g[0]);
          hi[f] = std::max(hi[f], g[last]);
        }
      std::vector<double> xyz(3 * MD);
      const double gm1 = kGamma - 1.0;
      const double *st = ob.sponge_state;
      const double rhoS = st[0] / prm.rho_ref, uS = st[1] / prm.u_ref, vS = st[2] / prm.u_ref,
                   wS = st[3] / prm.u_ref, pS = st[4] / prm.p_ref;
      const double cons[5] = {rhoS, rhoS * uS, rhoS * vS, rhoS * wS,
                              pS / gm1 + 0.5 * rhoS * (uS * uS + vS * vS + wS * wS)};
      for (int64_t e = 0; e < nE; ++e) {
        if (!flags[e]) continue;
        const int s = out.nS++;
        out.spongeIdx[e] = s;
        IntegrationPointCoordinates(gridNodes + e * 3 * KG3, Kg, M, lgv, xyz.data());
        double cm[6] = {0.0, 0.0, 0.0, 1.0, 1.0, 1.0};
        for (int d = 0; d < 3; ++d) {
          const bool mn = (flags[e] >> (2 * d)) & 1, mx = (flags[e] >> (2 * d + 1)) & 1;
          if (mn) cm[3 + d] = -1.0;
          for (int l = 0; l < MD; ++l) {
            double val = 0.0;
            if (mn || mx) {
              const int f = mn ? 2 * d : 2 * d + 1;
              const double ss = ob.sponge_sigma[f], aa = ob.sponge_alpha[f];
              const double x0 = mn ? hi[f] : lo[f];
              const double x = xyz[d * MD + l];
              if (mn ? x > x0 : x < x0) { err = "inconsistent sponge layer location"; return VCPG_E_INVALID; }
              val = ss * std::pow(std::fabs(x - x0) / (hi[f] - lo[f]), aa);
            }
            out.dampFn.push_back(val);
          }
          if (mn || mx) {
            const double ss = ob.sponge_sigma[mn ? 2 * d : 2 * d + 1];
            cm[d] = ob.cml ? (std::fabs(ss) < 1.0e-4 ? 1.0 : 1.0 / ss) : 0.0;
          }
        }
        for (int v = 0; v < 5; ++v)
          for (int l = 0; l < MD; ++l) out.dampState.push_back(cons[v]);
        out.cml.insert(out.cml.end(), cm, cm + 6);
      }
    }
    return VCPG_OK;
  } catch (const std::exception &ex) {
    err = ex.what();
    return VCPG_E_INVALID;
  }
}

void SliceOpenBoundary(const OpenBoundaryHost &block, const int64_t *localToGlobal, int64_t nLocal,
                       int64_t nOwned, const int32_t *localNbr, int MD, OpenBoundaryHost &out) {
  std::vector<int64_t> localOf(block.nbrCode.size() / 6, -1);   // block element -> owned local
  for (int64_t l = 0; l < nOwned; ++l) localOf[localToGlobal[l]] = l;
  out = OpenBoundaryHost{};
  out.pc = block.pc;
  out.dlq = block.dlq;
  out.cmlOn = block.cmlOn;
  // Boundary faces of owned elements, block order kept (per block face, element order).
  std::vector<int> newIndex((size_t)block.nB, -1);
  for (int f = 0; f < 6; ++f) {
    out.cfg[f] = block.cfg[f];            // areas and settings of the whole block face
    out.cfg[f].first = out.nB;
    for (int b = block.cfg[f].first; b < block.cfg[f].first + block.cfg[f].count; ++b) {
      const int *row = &block.bface[(size_t)b * kBfStride];
      const int64_t l = localOf[row[kBfElem]];
      if (l < 0) continue;
      newIndex[b] = out.nB++;
      out.blockRow.push_back(b);
      out.blockLast.push_back(row[kBfLast]);
      out.bface.insert(out.bface.end(), row, row + kBfStride);
      out.bface[out.bface.size() - kBfStride + kBfElem] = (int)l;
      out.bface[out.bface.size() - kBfStride + kBfLast] = -1;   // remapped below
      out.bpresc.insert(out.bpresc.end(), block.bpresc.begin() + (size_t)b * kPrescStride,
                        block.bpresc.begin() + (size_t)(b + 1) * kPrescStride);
    }
    out.cfg[f].count = out.nB - out.cfg[f].first;
  }
  for (int b = 0; b < block.nB; ++b) {
    const int nb = newIndex[b];
    const int last = block.bface[(size_t)b * kBfStride + kBfLast];
    if (nb >= 0 && last >= 0 && newIndex[last] >= 0)
      out.bface[(size_t)nb * kBfStride + kBfLast] = newIndex[last];
  }
  // Neighbour table: the handle's, with the owned elements' boundary faces coded.
  out.nbrCode.assign(localNbr, localNbr + nLocal * 6);
  for (int64_t l = 0; l < nOwned; ++l) {
    const int64_t g = localToGlobal[l];
    for (int f = 0; f < 6; ++f) {
      const int c = block.nbrCode[g * 6 + f];
      if (c <= -2) out.nbrCode[l * 6 + f] = -2 - newIndex[-2 - c];
      else if (c == -1) out.nbrCode[l * 6 + f] = -1;
    }
  }
  // Sponge elements among the owned ones, in local order.
  out.spongeIdx.assign(nLocal, -1);
  for (int64_t l = 0; l < nOwned; ++l) {
    const int s = block.spongeIdx[localToGlobal[l]];
    if (s < 0) continue;
    out.spongeIdx[l] = out.nS++;
    out.dampFn.insert(out.dampFn.end(), block.dampFn.begin() + (size_t)s * 3 * MD,
                      block.dampFn.begin() + (size_t)(s + 1) * 3 * MD);
    out.dampState.insert(out.dampState.end(), block.dampState.begin() + (size_t)s * 5 * MD,
                         block.dampState.begin() + (size_t)(s + 1) * 5 * MD);
    out.cml.insert(out.cml.end(), block.cml.begin() + (size_t)s * 6,
                   block.cml.begin() + (size_t)(s + 1) * 6);
  }
}

}  // namespace vcpg
