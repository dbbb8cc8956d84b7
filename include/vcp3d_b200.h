/*
 * vcp3d_b200.h -- C ABI of the B200 (sm_100a) implementation of the VCP3D
 * explicit DG residual and time step.
 *
 * The library replaces the per-element work inside the reference solver's
 * residual and Runge-Kutta stage calls:
 *
 *   SolverClass::Residual(su2double *monitoringData, bool)      include/SolverClass.hpp:72-73
 *   SolverClass::ExecuteTimeSynchronizationStep(su2double *)    include/SolverClass.hpp:50
 *   ElementClass::ComputeTimeStep(...)                          include/ElementClass.hpp:312-317
 *
 * Everything crosses the boundary as plain pointers and sizes. A handle owns
 * all device memory and one CUDA stream; the solution stays resident on the
 * device between calls and host pointers are only borrowed for the duration
 * of a call. Every entry point returns VCPG_OK (0) or one of the error codes
 * below; vcpg_last_error() gives the message. The reference aborts the
 * process in these situations (Terminate, src/StandAloneFunctions.cpp:628-674);
 * a host shim that wants that behaviour maps a non-zero code to Terminate.
 *
 * Array conventions (all double precision, row-major, no padding):
 *   K = n_poly + 1 (DOFs per direction), M = n_int_1d (integration points per
 *   direction). Elements are numbered i fastest, then j, then k. Within an
 *   element, DOFs and volume integration points are numbered i fastest; face
 *   integration points follow the reference's face layout (i-faces: j fastest
 *   then k; j-faces: i fastest then k; k-faces: i fastest then j).
 *   Solution and residual: [n_elem][5][K^3], modal coefficients of the
 *   entropy variables (the reference's mSol / mRes without padding).
 */
#ifndef VCP3D_B200_H
#define VCP3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum vcpg_status {
  VCPG_OK = 0,
  VCPG_E_CUDA = 1,            /* a CUDA runtime call failed                      */
  VCPG_E_CG_NOCONV = 2,       /* mass-matrix CG hit its iteration cap (100)      */
  VCPG_E_NEG_A2 = 3,          /* negative speed of sound squared in the time step */
  VCPG_E_NONFINITE = 4,       /* a non-finite value appeared in the state         */
  VCPG_E_OOM = 5,             /* device allocation failed                         */
  VCPG_E_UNSUPPORTED_KM = 6,  /* (K, M) pair without a compiled kernel            */
  VCPG_E_ADMISSION = 7,       /* request does not fit the device memory budget    */
  VCPG_E_INVALID = 8          /* invalid argument                                 */
};

enum vcpg_riemann { VCPG_ROE = 0, VCPG_ISMAIL_ROE = 1 };
enum vcpg_precision { VCPG_FP64 = 0, VCPG_MIXED = 1 };
enum vcpg_scheme { VCPG_SSPRK3 = 0, VCPG_LSRK4 = 1 };
/* "Subgrid scale model" (src/SGSModel.cpp): WALE (C_w = 0.325) or Vreman (c = 0.07),
 * with the element's LES length scale (elem_scalars[3]). */
enum vcpg_sgs { VCPG_SGS_NONE = 0, VCPG_SGS_WALE = 1, VCPG_SGS_VREMAN = 2 };

/* Face numbering used by every per-face array: 0 iMin, 1 iMax, 2 jMin, 3 jMax, 4 kMin, 5 kMax. */

typedef struct vcpg_params {
  int32_t n_elem[3];          /* elements in i, j, k                                 */
  int32_t n_poly;             /* polynomial degree of the solution, K = n_poly + 1    */
  int32_t n_int_1d;           /* integration points per direction, M                  */
  int32_t riemann;            /* enum vcpg_riemann                                   */
  int32_t metric_index_compat;/* 1: gradient and symmetrizing-flux transforms index
                                 the metric by the variable index as the reference
                                 does (src/ElementClass.cpp:3865-3873,
                                 src/FluxesFace.cpp:272-282, 325-332); 0: by point */
  int32_t precision;          /* enum vcpg_precision. VCPG_MIXED: the residual
                                 (contractions, fluxes, mass solve) computes in
                                 FP32 with a 1e-5 CG tolerance; state, metrics,
                                 time step and RK updates stay FP64            */
  double theta_sym;           /* "Theta parameter symmetrizing terms"                */
  double rel_penalty;         /* "Relative penalty parameter"                        */
  double cfl;                 /* "CFL number"                                        */
  double mu;                  /* non-dimensional laminar viscosity                   */
  double p_ref, u_ref, rho_ref; /* reference conditions (dimensional)                */
  int32_t sgs_model;          /* enum vcpg_sgs; a model needs ops->dleg_dofs and
                                 geom->vol_metric_dofs (vcpg_setup_nodal_metrics)  */
  int32_t monitor_forces;     /* "Monitor forces": with wall faces (heat flux,
                                 isothermal, inviscid) the monitoring data's entries
                                 0-2 are the pressure and 3-5 the viscous force
                                 coefficients in x, y, z (src/FluxesFace.cpp:997-1011,
                                 1586-1612, src/SolverClass.cpp:3754-3783); else 0 */
  double mach;                /* "Mach number" (force coefficients)                  */
  double ref_area;            /* "Reference area force coefficients" (default 1)     */
  double body_force[3];       /* "Body force per unit volume (x,y,z)", dimensional
                                 (N/m^3): the source -J w (0, f, u.f) / p_ref of the
                                 volume residual (src/ElementClass.cpp:4495-4533)    */
} vcpg_params;

/* Standard-element operators (StandardElementClass, src/StandardElementClass.cpp:105-911). */
typedef struct vcpg_operators {
  const double *leg_int;      /* [K][M] orthonormal Legendre basis at the 1-D Gauss points */
  const double *dleg_int;     /* [K][M] its derivative                                     */
  const double *leg_face;     /* [2][K] basis at r = -1 (min face) and r = +1 (max face)    */
  const double *dleg_face;    /* [2][K] derivative at r = -1 and r = +1                     */
  const double *w_int;        /* [M]    1-D Gauss weights                                   */
  const double *leg_dofs;     /* [K][K] basis at the 1-D nodal DOFs (time-step conversion)  */
  const double *basis_center; /* [K^3]  3-D basis at the element centre (CG preconditioner) */
  const double *dleg_dofs;    /* [K][K] derivative of basis k at nodal DOF i (time step with
                                 an SGS model; may be NULL without one)                    */
} vcpg_operators;

/* Per-element geometry (ElementClass::ComputeMetricTerms, src/ElementClass.cpp:1027-1407). */
typedef struct vcpg_geometry {
  const double *vol_metric;   /* [n_elem][10][M^3]: J, dr/dx dr/dy dr/dz ds/dx ... dt/dz   */
  const double *face_metric;  /* [n_elem][6][13][M^2]: unit normal (3), area, 9 terms      */
  const double *elem_scalars; /* [n_elem][15]: lenI lenJ lenK lenLES lenVol volElem,
                                 averaged unit normals of the i, j, k directions (9)       */
  const int32_t *neighbors;   /* [n_elem][6]: neighbour element per face, -1 = boundary    */
  const double *vol_metric_dofs; /* [n_elem][10][K^3]: J and the inverse-Jacobian terms at
                                 the nodal solution DOFs (mVolMetricSolDOFs); needed with
                                 an SGS model (time step), may be NULL without one       */
} vcpg_geometry;

typedef struct vcpg_handle vcpg_handle;

/* Creates a solver on the current CUDA device; uploads operators and geometry. */
int vcpg_create(const vcpg_params *params, const vcpg_operators *ops,
                const vcpg_geometry *geom, vcpg_handle **out);
int vcpg_destroy(vcpg_handle *h);
const char *vcpg_last_error(const vcpg_handle *h);

/* Parametric positions of the nodal solution DOFs and of the grid nodes
 * ("Location of the DOFs"; the reference detects the grid's own spacing,
 * ElementClass::LGLDistribution, src/ElementClass.cpp:3406-3622). */
enum vcpg_dof_location {
  VCPG_DOFS_EQUIDISTANT = 0,     /* equidistant solution DOFs and grid nodes */
  VCPG_DOFS_LGL = 1,             /* LGL solution DOFs and grid nodes         */
  VCPG_DOFS_EQUI_GRID_LGL = 2,   /* equidistant solution DOFs, LGL grid      */
  VCPG_DOFS_LGL_GRID_EQUI = 3    /* LGL solution DOFs, equidistant grid      */
};

/* Host-side set-up from a high-order grid (the product's own restatement of the
 * reference's operator and metric pre-processing). grid_nodes is the per-element
 * grid, [n_elem][3][(p_grid+1)^3], nodes and solution DOFs at the parametric
 * positions of dof_location (enum vcpg_dof_location). Fills caller-allocated arrays with the
 * shapes documented in vcpg_operators / vcpg_geometry; neighbors are filled for
 * a block that is periodic in every direction listed in periodic[3]. */
int vcpg_setup_geometry(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                        const int32_t periodic[3], const double *grid_nodes,
                        double *leg_int, double *dleg_int, double *leg_face,
                        double *dleg_face, double *w_int, double *leg_dofs,
                        double *basis_center, double *vol_metric, double *face_metric,
                        double *elem_scalars, int32_t *neighbors);

/* Metric terms at the nodal solution DOFs (ElementClass::ComputeCoorNodalSolDOFs,
 * src/ElementClass.cpp:816-918) and the derivative of the modal basis at the 1-D
 * nodal DOFs: the inputs an SGS model's time step needs. vol_metric_dofs
 * [n_elem][10][K^3], dleg_dofs [K][K]; host computation. */
int vcpg_setup_nodal_metrics(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                             const double *grid_nodes, double *dleg_dofs,
                             double *vol_metric_dofs);

/* The same set-up with the metric terms computed on the current CUDA device (one
 * CTA per element; the same doubles as vcpg_setup_geometry, which runs the
 * identical arithmetic on the host). Same arguments and outputs; the grid nodes
 * go to the device in passes of at most about 1 GiB of buffers. */
int vcpg_setup_geometry_device(const vcpg_params *params, int32_t p_grid, int32_t dof_location,
                               const int32_t periodic[3], const double *grid_nodes,
                               double *leg_int, double *dleg_int, double *leg_face,
                               double *dleg_face, double *w_int, double *leg_dofs,
                               double *basis_center, double *vol_metric, double *face_metric,
                               double *elem_scalars, int32_t *neighbors);

/* Converts dimensional conservative variables at the nodal DOFs
 * ([n_elem][5][K^3]) to modal entropy-variable coefficients, as
 * SolverClass::ReadRestartSolution does (src/SolverClass.cpp:3310-3366).
 * vand_inv is the [K][K] inverse 1-D Vandermonde matrix of the nodal DOFs,
 * vand_inv[c * K + o] mapping nodal value c to mode o; NULL selects the LGL
 * nodal DOFs. */
/* The [K][K] inverse 1-D Vandermonde matrix of the nodal solution DOFs of
 * dof_location (StandardElementClass, src/StandardElementClass.cpp:860-880), the
 * vand_inv argument of vcpg_nodal_conservative_to_modal. */
int vcpg_vandermonde_inverse(int32_t n_poly, int32_t dof_location, double *vand_inv);

int vcpg_nodal_conservative_to_modal(const vcpg_params *params, const double *vand_inv,
                                     const double *cons, double *modal, int64_t n_elem);

/* State transfer (host <-> device), [n_elem][5][K^3]. vcpg_set_state marks the
 * stored residual as stale. */
int vcpg_set_state(vcpg_handle *h, const double *modal);
int vcpg_get_state(vcpg_handle *h, double *modal);
int vcpg_get_residual(vcpg_handle *h, double *res);

/* One residual evaluation of the current state: volume + face terms followed
 * by the generalised mass-matrix solve (SolverClass::Residual). monitoring
 * receives the reference's 8 monitoring values when non-NULL. The residual
 * before the mass-matrix solve is kept when keep_raw is non-zero and can be
 * read with vcpg_get_raw_residual. */
int vcpg_residual(vcpg_handle *h, double *monitoring, int32_t keep_raw);
int vcpg_get_raw_residual(vcpg_handle *h, double *res);

/* Global CFL time step (minimum of ElementClass::ComputeTimeStep, non-dimensional). */
int vcpg_time_step(vcpg_handle *h, double *dt);

/* n_steps full time steps with the given scheme (SSP-RK3 as in
 * ExecuteTimeSynchronizationStep, or five-stage low-storage RK4). If
 * fixed_dt > 0 it is used as the non-dimensional step, otherwise the CFL step
 * is recomputed on the device at the start of every step. The first stage uses
 * the residual of the current state, as in the reference main program
 * (src/VCP3D_CurviLinear.cpp:94); when the state was set since the last
 * residual, vcpg_step evaluates it first (one extra launch). dt_history, when
 * non-NULL, receives the n_steps time steps. The step sequence is captured in
 * a CUDA graph on first use. */
int vcpg_step(vcpg_handle *h, int32_t scheme, int32_t n_steps, double fixed_dt,
              double *dt_history);

/* One synchronization time step (SolverClass::ExecuteTimeSynchronizationStep,
 * src/SolverClass.cpp:2177-2422): SSP-RK3 steps with the CFL step of the
 * current state until the non-dimensional time dt_sync (the reference's
 * "Synchronization time step" times u_ref) is reached; the step that would pass
 * 0.99 dt_sync is shortened to end on dt_sync exactly. Reads one time step back
 * to the host per RK step. n_steps (optional) receives the number of RK steps;
 * monitoring (optional) the 8 monitoring values of the final state, at the cost
 * of one more residual. More than max_steps RK steps is an error. */
int vcpg_synchronization_step(vcpg_handle *h, double dt_sync, int32_t max_steps,
                              int32_t *n_steps, double *monitoring);

/* Synchronises the handle's stream and reports the first device-side error
 * (CG cap, negative a^2) recorded since the last call. */
int vcpg_sync(vcpg_handle *h);

/* The handle's CUDA stream (cudaStream_t) for callers that time or order work. */
void *vcpg_stream(vcpg_handle *h);

/* ---- A block split across GPUs (the reference's DistributeGrid,
 * src/SolverClass.cpp:1537-1584, with the halo exchange of Residual). ----
 * A rank's handle holds its owned elements first, then ghost copies of the
 * neighbouring ranks' elements. vcpg_set_partition declares elements
 * [0, n_owned) owned: residual, time step (local minimum) and stages run on
 * them. Elements [n_owned, n_owned + n_face_ghost) are ghosts whose Min faces
 * towards owned elements are evaluated here (their other lower neighbours -1);
 * the remaining elements are ghosts that only provide their state. Open
 * boundaries of a partitioned block: vcpg_set_open_boundary_partition; vcpg_step and
 * vcpg_synchronization_step are rejected, a step being: vcpg_time_step, the
 * minimum over ranks, then per stage vcpg_rk_stage, the exchange of the ghost
 * states (vcpg_pack_send_list or vcpg_pack_states, the transport, then
 * vcpg_unpack_states) and vcpg_residual (or vcpg_residual_part 0 and 1 around
 * the exchange). */
int vcpg_set_partition(vcpg_handle *h, int32_t n_owned, int32_t n_face_ghost);

/* Device-to-device copies, on the handle's stream, between the states of
 * elements [first, first + count) and a device buffer of count * 5 K^3
 * doubles (element-major, as the state). */
int vcpg_pack_states(vcpg_handle *h, int32_t first, int32_t count, double *d_buf);
int vcpg_unpack_states(vcpg_handle *h, int32_t first, int32_t count, const double *d_buf);

/* One Runge-Kutta stage of step dt with the current residual on the owned
 * elements (the stage loop of ExecuteTimeSynchronizationStep,
 * src/SolverClass.cpp:2368-2396): SSP-RK3 stage 0-2 (stage 0 keeps the state
 * as the step's start) or LSRK4 stage 0-4. */
int vcpg_rk_stage(vcpg_handle *h, int32_t scheme, int32_t stage, double dt);

/* Number of this library's kernel launches issued since creation. */
int64_t vcpg_launch_count(const vcpg_handle *h);

/* Cumulative mass-matrix CG statistics since creation: total iterations and
 * element solves (the reference's per-element CG, src/CG_MassMatrix.cpp:395-492). */
int vcpg_stats(vcpg_handle *h, int64_t *cg_iterations, int64_t *element_solves);

/* Measurement hook (no counterpart in the reference): evaluates the residual
 * of the current state `reps` times with CUDA events on the handle's stream
 * around each kernel and returns the average milliseconds per launch:
 * ms[0] the two characteristic-boundary kernels (0 without such faces),
 * ms[1] FaceFluxKernel, ms[2] ResidualKernel. The device residual afterwards
 * is that of the current state, as after vcpg_residual. */
int vcpg_time_residual_kernels(vcpg_handle *h, int32_t reps, double *ms);

/* Measurement hook (no counterpart in the reference): the line contraction of
 * one sum-factorisation stage, 128 lines per tile, run `reps` times per tile
 * from shared memory to shared memory, with variant 0 FP32 fused multiply-adds
 * (the mixed form's residual kernel), 1 TF32 tensor-core tiles (tcgen05.mma
 * kind::tf32, accumulator in tensor memory), 2 the same with the operands split
 * into TF32 high and low parts (three MMAs, FP32-level accuracy), 3 the FP32
 * lines with the operator in constant memory instead of shared memory. K inputs and
 * M outputs per line, (K, M) = (5, 7) or (6, 8); x [n_lines][K], op [K][M]
 * (op[k * M + m]), y [n_lines][M] receives the last stage's outputs (each
 * stage's next inputs are its first K outputs times scale). n_lines a multiple
 * of 128; ms receives the device time of the timed launch (after a warm-up
 * launch). Allocates its own device buffers. */
int vcpg_line_contraction_probe(int32_t variant, int32_t K, int32_t M, int64_t n_lines,
                                int32_t reps, float scale, const float *x, const float *op,
                                float *y, double *ms);

/* Allocation-free CFL time step. This entry point has no counterpart in the
 * reference solver. It is for callers that cannot call cudaMalloc: programs
 * whose device memory all belongs to their own pool allocator (a framework's
 * caching allocator, or a driver budgeting many resident cases) and that must
 * not allocate or free behind that pool, whose accounting would not see it and
 * whose work cudaMalloc/cudaFree could stall by synchronising the device.
 * The caller passes device arrays it already owns: d_sol [n_elem][5][K^3],
 * d_elem_scalars [n_elem][15] (as in vcpg_geometry) and d_dt (one double,
 * receives the same global time step vcpg_time_step returns). No handle is
 * used and nothing is allocated: the only scratch (one double per element and
 * a status slot) is a static device array of the library sized for
 * VCPG_NOALLOC_MAX_ELEMS elements (2 MiB), held by every GPU that loads the
 * library until the process exits. Larger n_elem returns VCPG_E_ADMISSION
 * before any device work. The first call on each device looks up the array's
 * device address with that device current. All calls share the array and
 * overwrite it: calls that overlap on the GPU (different streams or host
 * threads) race, so order them. Each call uploads the operators and launches
 * its kernels on `stream` (a cudaStream_t, NULL = legacy default stream), then
 * reads its status back and synchronises that stream before returning, so it
 * cannot be captured into a CUDA graph. VCPG_E_NEG_A2 reports a negative (or
 * not-a-number) speed of sound squared in the state. */
#define VCPG_NOALLOC_MAX_ELEMS 262144
int vcpg_time_step_noalloc(const vcpg_params *params, const vcpg_operators *ops,
                           const double *d_sol, const double *d_elem_scalars, double *d_dt,
                           void *stream);

/* ------------------------------------------------------------------------- */
/* Open boundaries: characteristic (PC-NSCBC) boundary conditions, sponge     */
/* layers and the characteristic matching layer.                              */
/* ------------------------------------------------------------------------- */

/* Boundary condition of one block face (face numbering as above). */
enum vcpg_bc {
  VCPG_BC_NONE = 0,                 /* interior / periodic: the face has neighbours     */
  VCPG_BC_OUTFLOW_NSCBC = 1,        /* "BCOutflowNSCBC": prescribed static pressure,
                                       BCOutflowCharacteristicSubfaceClass
                                       (src/BoundaryState.cpp:1300-1568)              */
  VCPG_BC_INFLOW_STATIC_NSCBC = 2,  /* "BCInflowStaticNSCBC": prescribed density and
                                       velocity, BCInflowStaticCharacteristicSubfaceClass
                                       (src/BoundaryState.cpp:1579-1847)              */
  VCPG_BC_INFLOW_TOTAL_NSCBC = 3,   /* "BCInflowTotalNSCBC": prescribed total pressure,
                                       total temperature and velocity direction,
                                       BCInflowTotalCharacteristicSubfaceClass
                                       (src/BoundaryState.cpp:1848-2238)              */
  /* Boundary conditions through a boundary state (FluxesBoundaryFace,
   * src/FluxesFace.cpp:16-214, with the subface's ComputeBoundaryState,
   * src/BoundaryState.cpp:124-828); no wall model. */
  VCPG_BC_WALL_HEAT_FLUX = 4,       /* "BCWallHeatFlux": wall_data = heat flux (W/m^2)  */
  VCPG_BC_WALL_ISOTHERMAL = 5,      /* "BCWallIsothermal": wall_data = temperature (K)  */
  VCPG_BC_WALL_INVISCID = 6,        /* "BCWallInviscid"                                 */
  VCPG_BC_FARFIELD = 7,             /* "BCFarfield": the free stream (free_stream)      */
  VCPG_BC_INFLOW_SUBSONIC = 8,      /* "BCInflowSubsonic": total pressure, total
                                       temperature and direction in inflow_total        */
  VCPG_BC_INFLOW_SUPERSONIC = 9,    /* "BCInflowSupersonic": inflow_super               */
  VCPG_BC_OUTFLOW_SUBSONIC = 10,    /* "BCOutflowSubsonic": static pressure in p_out    */
  VCPG_BC_OUTFLOW_SUPERSONIC = 11   /* "BCOutflowSupersonic"                            */
};

/* The reference's "NSCBC tuning parameters", "Prescribed boundary data" and
 * "Sponge layer information" blocks (src/InputParamClass.cpp:406-431, 1196-1330).
 * Dimensional prescribed values are non-dimensionalised with the handle's
 * reference conditions, as ConvertPrescribedData does (src/SubfaceClasses.cpp). */
typedef struct vcpg_open_boundary {
  int32_t bc[6];                  /* enum vcpg_bc per block face                       */
  double p_out[6];                /* outflow: static pressure (Pa)                     */
  double inflow[6][4];            /* static inflow: density, velocity x, y, z          */
  double outlet_len;              /* "Outlet characteristic length"                    */
  double outlet_sigma;            /* "Outlet normal relaxation (sigma)"                */
  double outlet_beta_l;           /* "Outlet coupled transverse relaxation (beta_l)";
                                     negative: use the boundary-averaged Mach number   */
  double outlet_beta_t;           /* "Outlet uncoupled transverse relaxation (beta_t)" */
  int32_t outlet_one_minus_beta;  /* "Outlet use one minus beta transverse relaxation" */
  int32_t inlet_incoming;         /* "Inlet use outgoing wave amplitude"               */
  double inlet_len;               /* "Inlet characteristic length"                     */
  double inlet_sigma;             /* "Inlet normal relaxation (sigma)"                 */
  int32_t sponge_elems[6];        /* sponge-layer thickness in elements per block face */
  double sponge_sigma[6];         /* damping constant per block face                   */
  double sponge_alpha[6];         /* damping exponent per block face                   */
  int32_t cml;                    /* "Characteristic matching layer" in sponge elements */
  double sponge_state[5];         /* damping (averaged) state: density, velocity x, y,
                                     z, pressure, dimensional                          */
  double inflow_total[6][5];      /* total inflow (characteristic or subsonic): total
                                     pressure (Pa), total temperature (K), velocity
                                     direction x, y, z                                 */
  double wall_data[6];            /* heat-flux wall: heat flux (W/m^2); isothermal
                                     wall: wall temperature (K)                        */
  double inflow_super[6][5];      /* supersonic inflow: density, velocity x, y, z,
                                     pressure                                          */
  double free_stream[5];          /* far field: density, velocity x, y, z, pressure
                                     (the reference's free stream, dimensional)        */
  int32_t outlet_local_mach;      /* "Outlet use local (element) averaged Mach number":
                                     the characteristic outflow of a subface uses the
                                     projected Mach number averaged over one element
                                     face -- as in the reference run on one thread, the
                                     face of the subface's last element in element order,
                                     whose value the reference's subface-wide member
                                     holds when the residual runs
                                     (src/BoundaryState.cpp:990, 1327); in a
                                     partitioned block see
                                     vcpg_set_boundary_outlet_mach.                    */
} vcpg_open_boundary;

/* Configures open boundaries on a handle whose geometry has boundary faces
 * (neighbors == -1 on the faces listed in bc). geom must be the same host
 * arrays given to vcpg_create; grid_nodes ([n_elem][3][(p_grid+1)^3], nodes at
 * the dof_location positions as in vcpg_setup_geometry) are needed when any
 * sponge_elems is non-zero and may be NULL otherwise. Every later residual
 * first averages the projected Mach number over each characteristic boundary
 * (SolverClass::AverageDataNSCBC, src/SolverClass.cpp:2492-2581) and builds the
 * boundary states and fluxes in FP64 (also in the mixed form). Characteristic
 * faces must be aligned with a parametric direction
 * (IdentifyBoundaryIndices, src/BoundaryState.cpp:829-928), otherwise
 * VCPG_E_INVALID. Call once, after vcpg_create and before the first residual. */
int vcpg_set_open_boundary(vcpg_handle *h, const vcpg_open_boundary *ob,
                           const vcpg_geometry *geom, int32_t p_grid, int32_t dof_location,
                           const double *grid_nodes);

/* One subface of a block face: an entry of the reference's "Subface
 * information" with its prescribed boundary data (InputParamClass::
 * ReadSubfaceInformation / ReadBoundaryData, src/InputParamClass.cpp:1340-1580;
 * element ranges as mapped by SolverClass, src/SolverClass.cpp:1640-1660). It
 * covers the element faces of block face `face` whose in-plane element indices
 * lie in [elem_begin, elem_end) along the face's two in-plane directions taken
 * in i, j, k order (j and k on i faces, i and k on j faces, i and j on k faces;
 * 0-based, end exclusive), with its own condition and prescribed data (the
 * fields of vcpg_open_boundary for one face, same units). */
typedef struct vcpg_subface {
  int32_t face;                   /* block face 0 iMin .. 5 kMax                       */
  int32_t elem_begin[2];          /* first element index, both in-plane directions    */
  int32_t elem_end[2];            /* one past the last                                 */
  int32_t bc;                     /* enum vcpg_bc                                      */
  double p_out;                   /* outflow: static pressure (Pa)                     */
  double inflow[4];               /* static inflow: density, velocity x, y, z          */
  double inflow_total[5];         /* total inflow: p_t (Pa), T_t (K), direction x, y, z */
  double wall_data;               /* heat flux (W/m^2) or wall temperature (K)         */
  double inflow_super[5];         /* supersonic inflow: density, velocity, pressure    */
} vcpg_subface;

/* vcpg_set_open_boundary with several subfaces per block face. A block face
 * named by at least one subface takes the condition and prescribed data of
 * each element face from the subface that covers it; its subfaces must cover
 * every one of its element faces exactly once (else VCPG_E_INVALID). The other
 * block faces keep ob->bc and ob's per-face data. The NSCBC tuning parameters
 * of ob apply to every characteristic subface (outlet and inlet settings
 * separately). As in the reference, the projected Mach number of a
 * characteristic subface is averaged over the characteristic element faces of
 * its whole block face and divided by the area of all of that block face's
 * physical element faces (SolverClass::InitNSCBC / AverageDataNSCBC,
 * src/SolverClass.cpp:2447-2581; ElementClass::ComputeSurfaceAreaBoundary /
 * AverageMachNSCBC, src/ElementClass.cpp:303-509). n_subfaces = 0 is
 * vcpg_set_open_boundary. */
int vcpg_set_open_boundary_subfaces(vcpg_handle *h, const vcpg_open_boundary *ob,
                                    const vcpg_subface *subfaces, int32_t n_subfaces,
                                    const vcpg_geometry *geom, int32_t p_grid,
                                    int32_t dof_location, const double *grid_nodes);

/* Open boundaries of a partitioned block (after vcpg_set_partition): the
 * set-up of the whole block (ob and the subfaces as for
 * vcpg_set_open_boundary_subfaces; block_n_elem, block_geom and
 * block_grid_nodes describe the whole block), of which the handle keeps the
 * boundary faces and sponge elements of its owned elements. local_to_global
 * gives the block index of each of the handle's elements. Boundary areas and
 * sponge extents are those of the whole block, as the reference's rank sums
 * and minima / maxima make them (src/SolverClass.cpp:2478-2481,
 * src/SpongeLayer.cpp:135-136). The boundary-averaged Mach number spans the
 * ranks: before each residual the caller gathers every rank's
 * vcpg_boundary_mach_weights, sums each block face's weights in block element
 * order (the ranks' lists merged by element index) and passes the sums to
 * vcpg_set_boundary_mach_sums (src/SolverClass.cpp:2556-2560). */
int vcpg_set_open_boundary_partition(vcpg_handle *h, const vcpg_open_boundary *ob,
                                     const vcpg_subface *subfaces, int32_t n_subfaces,
                                     const int32_t *block_n_elem, const vcpg_geometry *block_geom,
                                     int32_t p_grid, int32_t dof_location,
                                     const double *block_grid_nodes,
                                     const int64_t *local_to_global);

/* The area-weighted projected Mach numbers of the handle's characteristic
 * boundary faces for its current state (ElementClass::AverageMachNSCBC,
 * src/ElementClass.cpp:357-509; zero on other boundary faces), in the handle's
 * boundary-face order: counts[f] faces of block face f, f = 0..5 in turn;
 * weights needs their total (NULL: only the counts are returned).
 * Synchronises the handle's stream. */
int vcpg_boundary_mach_weights(vcpg_handle *h, double *weights, int32_t *counts);

/* Per block face, the sum of the Mach weights over the whole block, which the
 * next residuals divide by the block face's area in place of summing the
 * handle's own faces; NULL returns to the handle's own sums. */
int vcpg_set_boundary_mach_sums(vcpg_handle *h, const double *sums);

/* The outlet's element-local averaged Mach number ("Outlet use local averaged
 * Mach number") in a partitioned block: the reference's subface member holds the
 * value of the subface's last element face (src/BoundaryState.cpp:990, 1327),
 * which may lie on another rank. vcpg_boundary_rows gives per boundary row of
 * the handle its row in the whole block's boundary-face list (block face by
 * block face, element order) and the block row of its subface's last face (-1
 * without); vcpg_boundary_local_mach the rows' face-averaged Mach numbers of the
 * last boundary trace (vcpg_boundary_mach_weights runs one); with these the
 * ranks exchange the last faces' values and vcpg_set_boundary_outlet_mach sets
 * per row the value its outlet uses (NULL: the handle's own last face). A
 * partitioned handle whose last faces lie elsewhere refuses residuals until it
 * is set. */
int vcpg_boundary_rows(vcpg_handle *h, int32_t *block_rows, int32_t *block_last);
int vcpg_boundary_local_mach(vcpg_handle *h, double *values);
int vcpg_set_boundary_outlet_mach(vcpg_handle *h, const double *values);

/* A residual of a partitioned handle in two parts, so that the halo exchange
 * can run meanwhile: part 0 needs no ghost state (the boundary kernels, the
 * face fluxes of elements [0, flux_ready) and the residuals of elements
 * [0, res_ready) of vcpg_set_partition_parts); part 1, after the ghost states
 * are unpacked, completes the residual (the face fluxes of the remaining owned
 * elements and of the face ghosts, the remaining residuals). Part 0 then part
 * 1 equals vcpg_residual without monitoring data. The overlap of the
 * reference's Residual (src/SolverClass.cpp:3428-3611). */
int vcpg_residual_part(vcpg_handle *h, int32_t part);

/* What part 0 of vcpg_residual_part computes, for a handle whose owned
 * elements are ordered so that [0, flux_ready) have only owned lower
 * neighbours and [0, res_ready) have no ghost neighbour at all
 * (0 <= res_ready <= flux_ready <= n_owned). vcpg_set_partition resets both to
 * 0: part 0 then runs the boundary kernels only. */
int vcpg_set_partition_parts(vcpg_handle *h, int32_t flux_ready, int32_t res_ready);

/* The owned elements whose states go to a neighbouring rank, as list
 * `list` (0 <= list < 6: per direction, towards the rank below and above);
 * vcpg_pack_send_list gathers their states in list order, on the handle's
 * stream, into a device buffer of count * 5 K^3 doubles (the neighbour's ghost
 * elements, unpacked there with vcpg_unpack_states). The reference's
 * DistributeGrid halo (src/SolverClass.cpp:1537-1584) between the blocks of a
 * 3-D split. */
int vcpg_set_send_list(vcpg_handle *h, int32_t list, const int32_t *elems, int32_t count);
int vcpg_pack_send_list(vcpg_handle *h, int32_t list, double *d_buf);

/* ------------------------------------------------------------------------- */
/* Served ensemble: many cases resident on one GPU, batched by degree.        */
/* ------------------------------------------------------------------------- */
/* This has no counterpart in the reference solver, which runs one case per
 * process. An ensemble keeps every admitted case's state and geometry resident
 * in per-degree buckets: pre-allocated arenas of elements, boundary faces and
 * sponge elements. One time step of a bucket advances all of its running cases
 * together -- one launch of each fused kernel over the bucket's elements,
 * captured once as a CUDA graph -- each case with its own CFL time step and
 * parameters. Buckets run on their own streams, so different degrees overlap
 * on the device. Cases join (vcpg_ensemble_submit) and leave
 * (vcpg_ensemble_retire) between steps: continuous batching. A case's result
 * does not depend on the other cases in the mix (every element reads only its
 * own case's data). Not thread-safe: one host thread drives an ensemble. */

typedef struct vcpg_ensemble vcpg_ensemble;

typedef struct vcpg_ensemble_config {
  int32_t precision;            /* enum vcpg_precision, all cases                     */
  int32_t scheme;               /* enum vcpg_scheme, all cases                        */
  int32_t riemann;              /* enum vcpg_riemann, all cases                       */
  int32_t metric_index_compat;  /* as in vcpg_params, all cases                       */
  double theta_sym;             /* as in vcpg_params, all cases                       */
  double rel_penalty;           /* as in vcpg_params, all cases                       */
  int64_t bucket_elems[8];      /* element capacity of the bucket of degree p (index
                                   p, 1..6); 0 = no bucket for that degree            */
  int64_t bucket_bfaces[8];     /* characteristic boundary faces per bucket           */
  int64_t bucket_sponge[8];     /* sponge elements per bucket                         */
  int32_t max_cases;            /* case slots per bucket                              */
} vcpg_ensemble_config;

/* Allocates every bucket's arenas on the current device (the admission budget). */
int vcpg_ensemble_create(const vcpg_ensemble_config *cfg, vcpg_ensemble **out);
int vcpg_ensemble_destroy(vcpg_ensemble *ens);
const char *vcpg_ensemble_last_error(const vcpg_ensemble *ens);

/* Device bytes one case occupies in its bucket (its admission footprint). */
int64_t vcpg_ensemble_footprint(int32_t n_poly, int32_t n_int_1d, int64_t n_elem,
                                int64_t n_bfaces, int64_t n_sponge);

/* Admits a case to run n_steps time steps: the inputs of vcpg_create (params
 * must match the ensemble's shared settings and the bucket's degree), its
 * modal state (as vcpg_set_state) and, when ob is non-NULL, its open
 * boundaries (as vcpg_set_open_boundary). Returns VCPG_E_ADMISSION, with
 * nothing changed, when the bucket has no contiguous room for the case's
 * elements, boundary faces or sponge elements, or no free case slot; the
 * caller keeps the request and submits it again after cases retire. The
 * uploads are ordered on the bucket's stream before its next step; the case
 * first evaluates its residual inside that step and then steps with the rest. */
int vcpg_ensemble_submit(vcpg_ensemble *ens, const vcpg_params *params,
                         const vcpg_operators *ops, const vcpg_geometry *geom,
                         const double *modal_state, int32_t n_steps,
                         const vcpg_open_boundary *ob, int32_t p_grid, int32_t dof_location,
                         const double *grid_nodes, int64_t *case_id);

/* vcpg_ensemble_submit for a case with several subfaces per block face (as
 * vcpg_set_open_boundary_subfaces): the reference's mSubfaces[f][l]
 * (src/SolverClass.cpp:1646-1652) for a served case. */
int vcpg_ensemble_submit_subfaces(vcpg_ensemble *ens, const vcpg_params *params,
                                  const vcpg_operators *ops, const vcpg_geometry *geom,
                                  const double *modal_state, int32_t n_steps,
                                  const vcpg_open_boundary *ob, const vcpg_subface *subfaces,
                                  int32_t n_subfaces, int32_t p_grid, int32_t dof_location,
                                  const double *grid_nodes, int64_t *case_id);

/* Enqueues one time step of every bucket with resident cases; does not wait. */
int vcpg_ensemble_step(vcpg_ensemble *ens);

/* Non-blocking: ids of cases that have completed their steps since the last
 * poll (at most max_ids), from the most recent step whose state copy has
 * arrived. */
int vcpg_ensemble_poll(vcpg_ensemble *ens, int64_t *done_ids, int32_t max_ids,
                       int32_t *n_done);

/* Copies a completed case's modal state ([n_elem][5][K^3]) and simulated time
 * to the host and frees its slots for new cases. */
int vcpg_ensemble_retire(vcpg_ensemble *ens, int64_t case_id, double *modal_state,
                         double *sim_time);

/* Waits for all enqueued work; reports device-side errors (CG cap, a^2 < 0). */
int vcpg_ensemble_sync(vcpg_ensemble *ens);

/* Resident (pending or running) cases and this library's launches so far. */
int vcpg_ensemble_stats(vcpg_ensemble *ens, int32_t *resident, int64_t *launches);

#ifdef __cplusplus
}
#endif

#endif /* VCP3D_B200_H */
