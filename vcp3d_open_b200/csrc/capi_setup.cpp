// Host-side entry points of the C ABI: geometry/operator set-up from a grid
// and the nodal-conservative -> modal-entropy conversion of an initial state.
#include <cmath>
#include <cstring>
#include <exception>
#include <vector>

#include "../../include/vcp3d_b200.h"
#include "host_setup.h"

using vcpg::host::StdElement;

extern "C" {

int vcpg_setup_geometry(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                        const int32_t periodic[3], const double *grid_nodes, double *leg_int,
                        double *dleg_int, double *leg_face, double *dleg_face, double *w_int,
                        double *leg_dofs, double *basis_center, double *vol_metric,
                        double *face_metric, double *elem_scalars, int32_t *neighbors) {
  if (!params || !grid_nodes || p_grid < 1) return VCPG_E_INVALID;
  try {
    const int K = params->n_poly + 1, M = params->n_int_1d, Kg = p_grid + 1;
    const int nI = params->n_elem[0], nJ = params->n_elem[1], nK = params->n_elem[2];
    if (K < 2 || M < 1 || nI < 1 || nJ < 1 || nK < 1) return VCPG_E_INVALID;
    // The grid nodes of the generated cases sit at the LGL (or equidistant) positions
    // matching dof_location, as ElementClass::LGLDistribution detects.
    StdElement se = vcpg::host::BuildStdElement(K, M, Kg, vcpg::host::SolLgl(dof_location), vcpg::host::GridLgl(dof_location));
    if (leg_int) std::memcpy(leg_int, se.leg.data(), sizeof(double) * K * M);
    if (dleg_int) std::memcpy(dleg_int, se.dleg.data(), sizeof(double) * K * M);
    if (leg_face) std::memcpy(leg_face, se.face.data(), sizeof(double) * 2 * K);
    if (dleg_face) std::memcpy(dleg_face, se.dface.data(), sizeof(double) * 2 * K);
    if (w_int) std::memcpy(w_int, se.wInt.data(), sizeof(double) * M);
    if (leg_dofs) std::memcpy(leg_dofs, se.legdof.data(), sizeof(double) * K * K);
    if (basis_center) std::memcpy(basis_center, se.center.data(), sizeof(double) * K * K * K);
    const int64_t nE = (int64_t)nI * nJ * nK;
    const int MD = M * M * M, M2 = M * M, KG3 = Kg * Kg * Kg;
    for (int64_t e = 0; e < nE; ++e) {
      double sc[15];
      vcpg::host::ElementMetrics(se, grid_nodes + e * 3 * KG3,
                                 vol_metric ? vol_metric + e * 10 * MD : nullptr,
                                 face_metric ? face_metric + e * 6 * 13 * M2 : nullptr, sc,
                                 params->n_poly);
      if (elem_scalars) std::memcpy(elem_scalars + e * 15, sc, sizeof(sc));
    }
    if (neighbors) vcpg::host::BlockNeighbors(nI, nJ, nK, periodic, neighbors);
  } catch (const std::exception &) {
    return VCPG_E_INVALID;
  }
  return VCPG_OK;
}

int vcpg_setup_nodal_metrics(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                             const double *grid_nodes, double *dleg_dofs,
                             double *vol_metric_dofs) {
  if (!params || !grid_nodes || p_grid < 1) return VCPG_E_INVALID;
  try {
    const int K = params->n_poly + 1, M = params->n_int_1d, Kg = p_grid + 1;
    const int64_t nE = (int64_t)params->n_elem[0] * params->n_elem[1] * params->n_elem[2];
    if (K < 2 || M < 1 || nE < 1) return VCPG_E_INVALID;
    StdElement se = vcpg::host::BuildStdElement(K, M, Kg, vcpg::host::SolLgl(dof_location), vcpg::host::GridLgl(dof_location));
    if (dleg_dofs) std::memcpy(dleg_dofs, se.dlegdof.data(), sizeof(double) * K * K);
    const int KD = K * K * K, KG3 = Kg * Kg * Kg;
    if (vol_metric_dofs)
      for (int64_t e = 0; e < nE; ++e)
        vcpg::host::NodalMetrics(se, grid_nodes + e * 3 * KG3, vol_metric_dofs + e * 10 * KD);
  } catch (const std::exception &) {
    return VCPG_E_INVALID;
  }
  return VCPG_OK;
}

int vcpg_vandermonde_inverse(int32_t n_poly, int32_t dof_location, double *vand_inv) {
  if (n_poly < 1 || n_poly > 9 || !vand_inv) return VCPG_E_INVALID;
  const int K = n_poly + 1;
  try {
    const std::vector<double> v =
        vcpg::host::BuildStdElement(K, K, K, vcpg::host::SolLgl(dof_location), 1).vandInv;
    std::memcpy(vand_inv, v.data(), sizeof(double) * K * K);
  } catch (const std::exception &) {
    return VCPG_E_INVALID;
  }
  return VCPG_OK;
}

int vcpg_nodal_conservative_to_modal(const vcpg_params *params, const double *vand_inv,
                                     const double *cons, double *modal, int64_t n_elem) {
  if (!params || !cons || !modal || n_elem < 0) return VCPG_E_INVALID;
  const int K = params->n_poly + 1, KD = K * K * K;
  std::vector<double> vinv;
  if (!vand_inv) {  // LGL nodal DOFs
    vinv = vcpg::host::BuildStdElement(K, K, K, 1, 1).vandInv;
    vand_inv = vinv.data();
  }
  const double gam = 1.4, gm1 = gam - 1.0, ovgm1 = 1.0 / gm1;
  const double rhoRefInv = 1.0 / params->rho_ref, uRefInv = 1.0 / params->u_ref,
               pRefInv = 1.0 / params->p_ref;
  std::vector<double> nod(5 * KD), t1(5 * KD), t2(5 * KD);
  for (int64_t e = 0; e < n_elem; ++e) {
    const double *c = cons + e * 5 * KD;
    for (int l = 0; l < KD; ++l) {
      double rho = c[l];
      const double rhoInv = 1.0 / rho;
      double u = rhoInv * c[KD + l], v = rhoInv * c[2 * KD + l], w = rhoInv * c[3 * KD + l];
      double p = gm1 * (c[4 * KD + l] - 0.5 * (u * c[KD + l] + v * c[2 * KD + l] + w * c[3 * KD + l]));
      rho *= rhoRefInv; u *= uRefInv; v *= uRefInv; w *= uRefInv; p *= pRefInv;
      const double s = std::log(p / std::pow(rho, gam));
      const double pInv = 1.0 / p;
      nod[l] = (gam - s) * ovgm1 - 0.5 * rho * (u * u + v * v + w * w) * pInv;
      nod[KD + l] = rho * u * pInv;
      nod[2 * KD + l] = rho * v * pInv;
      nod[3 * KD + l] = rho * w * pInv;
      nod[4 * KD + l] = -rho * pInv;
    }
    // Nodal -> modal with the inverse Vandermonde matrix along k, j, then i.
    for (int var = 0; var < 5; ++var) {
      const double *b = nod.data() + var * KD;
      double *o1 = t1.data() + var * KD, *o2 = t2.data() + var * KD;
      double *o3 = modal + e * 5 * KD + var * KD;
      for (int kk = 0; kk < K; ++kk)
        for (int j = 0; j < K; ++j)
          for (int i = 0; i < K; ++i) {
            double acc = 0.0;
            for (int c2 = 0; c2 < K; ++c2) acc = std::fma(vand_inv[c2 * K + kk], b[(c2 * K + j) * K + i], acc);
            o1[(kk * K + j) * K + i] = acc;
          }
      for (int kk = 0; kk < K; ++kk)
        for (int jj = 0; jj < K; ++jj)
          for (int i = 0; i < K; ++i) {
            double acc = 0.0;
            for (int c2 = 0; c2 < K; ++c2) acc = std::fma(vand_inv[c2 * K + jj], o1[(kk * K + c2) * K + i], acc);
            o2[(kk * K + jj) * K + i] = acc;
          }
      for (int kk = 0; kk < K; ++kk)
        for (int jj = 0; jj < K; ++jj)
          for (int ii = 0; ii < K; ++ii) {
            double acc = 0.0;
            for (int c2 = 0; c2 < K; ++c2) acc = std::fma(vand_inv[c2 * K + ii], o2[(kk * K + jj) * K + c2], acc);
            o3[(kk * K + jj) * K + ii] = acc;
          }
    }
  }
  return VCPG_OK;
}

}  // extern "C"
