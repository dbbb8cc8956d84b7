// Open-boundary set-up shared by the host builder (open_boundary.cpp) and the
// device kernels (dg_boundary.cuh): characteristic boundary faces, the
// polynomial-correction operators and the sponge / matching-layer data.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vcp3d_b200.h"

namespace vcpg {

// Per block face (0 iMin .. 5 kMax) settings of the characteristic boundaries
// on it (the element faces' conditions are in the boundary-face list; a block
// face with several subfaces may hold outlets and inlets).
struct BlockFaceCfg {
  int type;            // enum vcpg_bc of the whole face, -1 with several conditions
  int first, count;    // range of this block face's entries in the boundary-face list
  int iPhi;            // index of the incoming acoustic wave amplitude (0 or 4)
  int oneMinusBeta;    // outlet: transverse terms weighted by (1 - beta)
  int incoming;        // inlet: keep the outgoing acoustic amplitudes of the interior
  double dell;         // factNorm * (-dL_0(r_0)): Lagrange derivative at the boundary DOF
  double area;         // sum of w * area over the block face's physical element faces
                       // (SolverClass::InitNSCBC)
  double sigma, len;   // outlet: normal relaxation coefficient and characteristic length
  double betaL, betaT; // outlet transverse relaxation coefficients
  double inSigma, inLen;  // inlet: normal relaxation coefficient and characteristic length
  int localMach;          // outlet: the element-local averaged Mach number (kBfLast's face)
};

// Entries of one boundary face in the boundary-face list (ints).
enum BFaceField {
  kBfElem = 0,   // element index
  kBfFace = 1,   // block face / element face 0..5 (2 d + side)
  kBfType = 2,   // enum vcpg_bc
  kBfGrad = 3,   // 3 entries: parametric axis of the normal, first and second transverse
  kBfCase = 6,   // case slot when a launch holds several cases (0 for one case)
  kBfLast = 7,   // list index of the last face (in element order) of this face's subface
  kBfStride = 8
};

// Non-dimensional prescribed values per boundary face: outflow p; static inflow
// rho, u, v, w; total inflow p_t, T_t (scaled by p_ref / rho_ref), direction x, y, z.
constexpr int kPrescStride = 5;

struct OpenBoundaryHost {
  int nB = 0;                       // boundary faces with a characteristic BC
  std::vector<int> bface;           // [nB][kBfStride]
  std::vector<double> bpresc;       // [nB][kPrescStride] non-dimensional prescribed data
  std::vector<double> pc;           // [M^2][M^2] polynomial-correction matrix
  std::vector<double> dlq;          // [M][M]: dlq[i * M + k] = dL_k(q_i), Lagrange basis
                                    // on the Gauss points
  BlockFaceCfg cfg[6] = {};
  // Sliced lists (SliceOpenBoundary): per row, its row in the whole block's list
  // and the block row of its subface's last face (-1 without).
  std::vector<int> blockRow, blockLast;
  std::vector<int32_t> nbrCode;     // [nE][6] neighbour table with boundary faces coded
                                    // as -2 - (index in the boundary-face list)
  int nS = 0;                       // sponge elements
  std::vector<int32_t> spongeIdx;   // [nE] sponge index or -1
  std::vector<double> dampFn;       // [nS][3][M^3] damping function per direction
  std::vector<double> dampState;    // [nS][5][M^3] conservative damping state
  std::vector<double> cml;          // [nS][6]: 1/sigma per direction, layer orientation
  int cmlOn = 0;
};

// Builds the open-boundary data of a block (optionally with several subfaces
// per block face, vcpg_subface). Returns a vcpg status and sets err.
int BuildOpenBoundary(const vcpg_params &prm, const vcpg_open_boundary &ob,
                      const vcpg_geometry &geom, int pGrid, int dofLocation,
                      const double *gridNodes, OpenBoundaryHost &out, std::string &err,
                      const vcpg_subface *subfaces = nullptr, int nSubfaces = 0);

// The part of a block's open-boundary data that a partitioned handle needs: boundary
// faces and sponge elements of its owned local elements (local_to_global[l]:
// block index of local element l, the first nOwned owned), in block order, the
// block faces' areas of the whole block, and the handle's neighbour table
// (localNbr, [nLocal][6]) with its boundary faces coded.
void SliceOpenBoundary(const OpenBoundaryHost &block, const int64_t *localToGlobal, int64_t nLocal,
                       int64_t nOwned, const int32_t *localNbr, int MD, OpenBoundaryHost &out);

}  // namespace vcpg
