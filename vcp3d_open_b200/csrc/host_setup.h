// Host-side pre-processing of the hot path's inputs (see host_setup.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace vcpg {
namespace host {

// The location code of the C ABI (enum vcpg_dof_location): LGL solution DOFs and
// LGL grid nodes.
inline int SolLgl(int loc) { return loc == 1 || loc == 3; }
inline int GridLgl(int loc) { return loc == 1 || loc == 2; }

double NormJacobi(int n, int alpha, int beta, double x);
double GradNormJacobi(int n, int alpha, int beta, double x);
void GaussLegendre(int n, std::vector<double> &x, std::vector<double> &w);
void DofLocations(int n, int lgl, std::vector<double> &r);
void Invert(int n, std::vector<double> &A);

// Standard-element operators. Matrices are row-major [input][output]:
// op[c * nout + o] multiplies input c for output o.
struct StdElement {
  int K = 0, M = 0, Kg = 0;
  std::vector<double> rInt, wInt, rDof, rGrid;
  std::vector<double> leg, dleg;         // [K][M]   modal basis at the Gauss points
  std::vector<double> face, dface;       // [2][K]   modal basis at r = -1, +1
  std::vector<double> legdof;            // [K][K]   modal basis k at nodal DOF i
  std::vector<double> center;            // [K^3]    3-D modal basis at the centre
  std::vector<double> vandInv;           // [K][K]   nodal c -> modal o
  std::vector<double> lagInt, dlagInt;   // [Kg][M]  grid Lagrange basis at the Gauss points
  std::vector<double> lagFace, dlagFace; // [2][Kg]  grid Lagrange basis at r = -1, +1
  std::vector<double> lagDof, dlagDof;   // [Kg][K]  grid Lagrange basis at the nodal DOFs
  std::vector<double> dlegdof;           // [K][K]   derivative of modal basis k at DOF i
};

StdElement BuildStdElement(int K, int M, int Kg, int dofLgl, int gridLgl);

// Metric terms of one element from its grid nodes gridNodes[3][Kg^3]:
// vol[10][M^3] (J, dr/dx .. dt/dz), face[6][13][M^2], scalars[15].
void ElementMetrics(const StdElement &se, const double *gridNodes, double *vol, double *face,
                    double *scalars, int nPoly);

// Metric terms at the nodal solution DOFs (ComputeCoorNodalSolDOFs): out[10][K^3]
// with J and the nine inverse-Jacobian terms, in the layout of the volume metric.
void NodalMetrics(const StdElement &se, const double *gridNodes, double *out);

// Face neighbours of a single block, elements i fastest: [nE][6] (iMin, iMax,
// jMin, jMax, kMin, kMax), -1 on a non-periodic block face.
void BlockNeighbors(int nI, int nJ, int nK, const int32_t periodic[3], int32_t *neighbors);

}  // namespace host
}  // namespace vcpg
