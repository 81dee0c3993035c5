/*
 * bosss_b200.h -- C-ABI of the B200-native DG operator evaluator.
 *
 * This is the drop-in boundary below BoSSS's C# operator API. The C# side keeps
 * its registration (`new DifferentialOperator(...)`, `EquationComponents[cod].Add(..)`,
 * `Commit()`) and its evaluator interface (`GetEvaluatorEx(..).Evaluate(alpha, beta, out)`);
 * a GPU evaluator class translates the committed operator into the plain
 * descriptors below and calls these functions through P/Invoke.
 *
 * Conventions
 *  - every entry point returns an int status: 0 = OK, negative = error;
 *    `bosss_b200_last_error` returns the message of the last failing call of
 *    the calling thread.
 *  - all vectors are FP64 in the reference's cell-major DOF layout
 *    `idx = j * N_per_cell + fieldOffset[f] + n`
 *    (UnsetteledCoordinateMapping.cs:696-706), j = local cell index.
 *  - host pointers are only read/written during the call (C# pins them with
 *    `fixed`/GCHandle for the duration of the call) and are never retained.
 *  - one handle = one CUDA stream; calls on one handle must be serialised by
 *    the caller (the reference evaluators are not thread-safe either).
 *  - `stream` arguments of the *_device entry points: NULL selects the handle's own
 *    (non-blocking) stream; pass cudaStreamLegacy ((void*)1) for the legacy default
 *    stream.
 *  - there is no CPU fallback: a component with no device functor makes
 *    `bosss_b200_create` fail with BOSSS_ERR_UNSUPPORTED_COMPONENT.
 */
#ifndef BOSSS_B200_H
#define BOSSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BOSSS_B200_VERSION_MAJOR 0
#define BOSSS_B200_VERSION_MINOR 3
#define BOSSS_B200_VERSION_PATCH 0

#define BOSSS_MAX_VARS 8
#define BOSSS_MAX_COMPONENTS 32
#define BOSSS_MAX_PARAMS 24

/* ---- status codes (DifferentialOperator.cs:1022-1023, 1590-1591 throw on the same conditions) ---- */
enum bosss_status {
    BOSSS_OK = 0,
    BOSSS_ERR_BAD_ARG = -1,                 /* wrong sizes, unsupported option (e.g. SubGridBoundaryTreatment) */
    BOSSS_ERR_UNSUPPORTED_COMPONENT = -2,   /* a registered equation component has no device functor */
    BOSSS_ERR_CUDA = -3,                    /* a CUDA runtime call failed */
    BOSSS_ERR_TIMEOUT = -4,                 /* a bounded device-side wait ran out */
    BOSSS_ERR_NAN = -5,                     /* opt-in NaN/Inf check tripped */
    BOSSS_ERR_NO_DEVICE = -6,               /* no CUDA device / library built without one */
    BOSSS_ERR_OUT_OF_MEMORY = -7
};

/* ---- equation components with device functors ----
 * Each value names the reference class whose pointwise semantics the device
 * functor reproduces. Parameters are passed in `bosss_component.params`. */
enum bosss_component_type {
    /* ScalarTransportFlux (2D) / ScalarTransportFlux3D, ScalarTransport/TransportFlux.cs:29-191.
     * INonlinearFlux, one argument; the velocity parameter fields are constant:
     * params[0..D-1] = velocity. */
    BOSSS_COMP_SCALAR_TRANSPORT_FLUX = 1,
    /* SIPLaplace, NSECommon/ipLaplace.cs:30-269 (IVolumeForm + IEdgeForm), one argument.
     * Nu(x, p) is generalised to nu(u) = params[1] + params[2]*u^2 (params[2] = 0 is the
     * reference's constant-viscosity form).
     * params[0] = penalty_base, params[3] = boundary kind (0 = Dirichlet, 1 = Neumann g_N=0),
     * Dirichlet value g_D(x) = params[4] + sum_d params[5+d]*x_d + sum_d params[8+d]*x_d^2. */
    BOSSS_COMP_SIP_LAPLACE = 2,
    /* Constant volume source (INonlinearSource, NECQuadratureVolume.cs:465-489): params[0] = s,
     * contributes  s * v. */
    BOSSS_COMP_CONSTANT_SOURCE = 3,
    /* OptimizedHLLC{Density,Momentum,Energy}Flux,
     * CompressibleFlowCommon/Convection/OptimizedHLLC*Flux.cs; arguments = all D+2 conservative
     * variables (rho, m_0..m_{D-1}, rhoE). params[0] = gamma, params[1] = Mach;
     * momentum: params[2] = component index. Boundary faces (non-periodic directions) take the
     * outer state from the boundary-state table (bosss_b200_set_boundary_state) and evaluate
     * the inner-edge HLLC flux with it, as OptimizedHLLCFlux.BorderEdgeFlux
     * (OptimizedHLLCFlux.cs:61-131) does with the state of its boundary-condition map; the
     * table holds prescribed states (inflow / far field), bosss_b200_set_boundary_kinds marks
     * supersonic-outlet and adiabatic-slip-wall nodes, whose outer states follow the inner one.
     * Such grids run on the generic kernel. */
    BOSSS_COMP_HLLC_DENSITY_FLUX = 10,
    BOSSS_COMP_HLLC_MOMENTUM_FLUX = 11,
    BOSSS_COMP_HLLC_ENERGY_FLUX = 12,
    /* OptimizedSIPG{Density,Momentum,Energy}Flux, CNS/Diffusion/OptimizedSIPG*Flux.cs: the
     * viscous terms of the compressible Navier-Stokes equations (SIPG); arguments = the D+2
     * conservative variables (rho, m_0..m_{D-1}, rhoE); params[0] gamma, [1] Mach, [2] Reynolds,
     * [3] Prandtl, [4] bulk/shear viscosity ratio (ViscosityRatio), [5] viscosity law (0: mu = 1,
     * 1: Sutherland), [6] Sutherland S/T0, [7] SIPGPenaltyScaling, [8] momentum component.
     * Boundary faces take the outer state from the boundary-state table
     * (bosss_b200_set_boundary_state), which the C# side fills from its boundary-condition
     * map (GetBoundaryState at the nodes of bosss_b200_boundary_nodes); not adiabatic walls. */
    BOSSS_COMP_CNS_SIPG_DENSITY_FLUX = 20,
    BOSSS_COMP_CNS_SIPG_MOMENTUM_FLUX = 21,
    BOSSS_COMP_CNS_SIPG_ENERGY_FLUX = 22
};

/* ---- quadrature-order functions, QuadOrderFunc.cs ---- */
enum bosss_quad_order_kind {
    BOSSS_QUAD_FIXED = 0,          /* FixedOrder(order) */
    BOSSS_QUAD_LINEAR = 1,         /* Linear() = SumOfMaxDegrees(1, false) */
    BOSSS_QUAD_NONLINEAR = 2,      /* NonLinear(deg) = SumOfMaxDegrees(deg, false) */
    BOSSS_QUAD_MAXDEG_TIMES_TWO = 3,
    BOSSS_QUAD_SUM_OF_MAX_DEGREES = 4  /* SumOfMaxDegrees(deg, RoundUp = true) */
};

typedef struct bosss_component {
    int32_t type;                      /* enum bosss_component_type */
    int32_t codomain;                  /* EquationComponents[codomain].Add(..) */
    int32_t n_args;                    /* length of ArgumentOrdering */
    int32_t args[BOSSS_MAX_VARS];      /* ArgumentOrdering as domain-variable indices */
    double params[BOSSS_MAX_PARAMS];
} bosss_component;

typedef struct bosss_op_desc {
    int32_t n_domain;                          /* number of domain variables */
    int32_t n_codomain;                        /* number of codomain variables */
    int32_t domain_degree[BOSSS_MAX_VARS];     /* DG degree per domain field */
    int32_t codomain_degree[BOSSS_MAX_VARS];   /* DG degree per codomain field */
    int32_t quad_kind;                         /* enum bosss_quad_order_kind */
    int32_t quad_param;                        /* order (FIXED) or nonlinear degree */
    int32_t n_components;
    bosss_component components[BOSSS_MAX_COMPONENTS];
} bosss_op_desc;

/* Uniform Cartesian grid, Grid2D.Cartesian2DGrid / Grid3D.Cartesian3DGrid with linspace nodes. */
enum bosss_cell_order {
    /* the generator's local order on one process: x slowest, last axis fastest
     * (Grid3D.cs:232-249: j = (ix*nY + iy)*nZ + iz; Grid2D: j = ix*nY + iy) */
    BOSSS_CELLS_GENERATOR = 0,
    /* GlobalID order: 3D x fastest (GlobalID = ix + iy*nX + iz*nX*nY, Grid3D.cs:248);
     * 2D GlobalID = ix*nY + iy (Grid2D.cs:182), the same as the generator order */
    BOSSS_CELLS_GLOBALID = 1
};

typedef struct bosss_grid_desc {
    int32_t dim;           /* 2 or 3 */
    int32_t n[3];          /* cells per direction */
    double lo[3];          /* domain lower corner */
    double hi[3];          /* domain upper corner */
    int32_t periodic[3];   /* 1 = periodic in that direction */
    int32_t cell_order;    /* enum bosss_cell_order */
    /* Part of a partitioned grid (domain decomposition, Transceiver.cs): this grid is the
     * cells [global_offset, global_offset + n) of a global grid with global_n cells and
     * periodicity global_periodic per direction (the offset may be negative, or reach past
     * global_n, where a ghost layer wraps around a periodic direction). For a part, lo and hi
     * are the box of the GLOBAL grid: cell widths and node coordinates are computed exactly
     * as on the whole grid, so a part's results equal the whole grid's (to the last bit of the
 * VJP, which can move with the tile a cell shares with its neighbours). The SIP
     * penalty's cell length scale (GridData_CellData.cs:663-684) counts the global boundary,
     * not the edge of the part. All zero: the grid is the whole grid. */
    int32_t global_n[3];
    int32_t global_offset[3];
    int32_t global_periodic[3];
} bosss_grid_desc;

enum bosss_precision {
    BOSSS_PRECISION_FP64 = 0,        /* plain FP64 path */
    /* Split precision: the residual's volume contractions (basis -> quadrature nodes, the
     * dgemm of DGField_Evaluation.cs:100-110, and the projection onto the test-function
     * gradients, NECQuadratureVolume.cs:689-716) run on the tensor cores. Each FP64 operand
     * row is scaled by a power of two and split exactly into 5 signed 8-bit slices; the
     * slice products accumulate exactly in 32-bit integers and are recombined in FP64, so
     * results agree with the FP64 path to about 1e-13 relative. The pointwise fluxes, the
     * face terms and JVP / VJP stay FP64. Built for 3D Euler (HLLC) with DG degree <= 3 and
     * 4 Gauss nodes per direction, whole grids (create() rejects other operators and parts
     * of partitioned grids with BOSSS_ERR_BAD_ARG). */
    BOSSS_PRECISION_SPLIT_FP32 = 1
};

typedef struct bosss_options {
    int32_t device;        /* CUDA device ordinal */
    int32_t precision;     /* enum bosss_precision */
    int32_t check_nan;     /* 1 = scan outputs for NaN/Inf, fail with BOSSS_ERR_NAN */
    int32_t kernel;        /* 0 = automatic, 1 = generic fused kernel, 2 = slab kernel (3D systems),
                              3 = slab volume pass + face-once face kernels (3D Euler, whole periodic
                              grids; residual and VJP, each face's HLLC flux evaluated once) */
    int32_t reserved[8];
} bosss_options;

typedef struct bosss_handle bosss_handle;
typedef struct bosss_bsr bosss_bsr;

/* ---- library ---- */
int bosss_b200_version(int32_t* major, int32_t* minor, int32_t* patch);
/* Copies the last error message of the calling thread (NUL-terminated, truncated to len). */
int bosss_b200_last_error(char* buf, size_t len);
/* Number of CUDA devices visible (0 when none). */
int bosss_b200_device_count(int32_t* count);

/* ---- operator evaluator ----
 * create: DifferentialOperator.GetEvaluatorEx (DifferentialOperator.cs:1013-1033) with
 * CompileQuadratureRules (:205-216); uploads basis tables and grid constants once. */
int bosss_b200_create(const bosss_op_desc* op, const bosss_grid_desc* grid,
                      const bosss_options* opt, bosss_handle** out);
int bosss_b200_destroy(bosss_handle* h);
/* DOF counts of the domain and codomain mappings, and the quadrature nodes per direction. */
int bosss_b200_get_sizes(const bosss_handle* h, int64_t* n_domain_dofs, int64_t* n_codomain_dofs,
                         int32_t* quad_nodes_1d);
/* The kernel path in effect for `mode` (0 residual, 1 JVP, 2 VJP): 1 generic fused kernel,
 * 2 slab kernel, 3 slab volume pass + face-once face kernels, 4 tensor-core volume kernel +
 * face terms (split-precision residual); and the kernel launches of one whole-grid call. */
int bosss_b200_kernel_info(const bosss_handle* h, int32_t mode, int32_t* kernel, int32_t* launches);

/* EvaluatorNonLin.Evaluate (DifferentialOperator.cs:1584-1661):
 *   out = beta*out + alpha*Op(U),  host buffers (copies in and out inside the call; above
 *   16 MB they stream by chunks of planes of the slowest grid direction on two copy streams,
 *   overlapped with the evaluation of the chunks whose neighbour planes have arrived). */
int bosss_b200_evaluate(bosss_handle* h, double alpha, double beta, const double* U,
                        double* out, double time);
/* Same, device-resident buffers (U, out are device pointers), enqueued on `stream`
 * (cudaStream_t, NULL = the handle's stream); returns after enqueueing. */
int bosss_b200_evaluate_device(bosss_handle* h, double alpha, double beta, const double* U_dev,
                               double* out_dev, double time, void* stream);

/* Boundary-state table of an operator whose boundary terms take a prescribed outer state
 * (the CNS viscous components, the HLLC fluxes on non-periodic grids): boundary_nodes returns the number of boundary face nodes
 * and, if xyz is not NULL, their physical coordinates (D per node), numbered cell by cell
 * (local order), then face direction d, then side (lower, upper), then the face's Gauss node
 * (the direction after d fastest); set_boundary_state uploads n_nodes * n_domain values, the
 * outer state of every domain variable at every node -- what the reference's
 * boundary-condition map returns there (CompressibleBoundaryCondMap.GetBoundaryState, e.g.
 * SupersonicInlet.cs:45-66). Evaluations of such an operator on a grid with boundary faces
 * fail with BOSSS_ERR_BAD_ARG until the table is set. */
int bosss_b200_boundary_nodes(const bosss_handle* h, int64_t* n_nodes, double* xyz);
int bosss_b200_set_boundary_state(bosss_handle* h, const double* state);
/* Boundary-condition kind of every boundary face node (same numbering), for the HLLC fluxes:
 * 0 the table's outer state (SupersonicInlet and other prescribed states; the default), 1 the
 * inner state (SupersonicOutlet.GetBoundaryState), 2 the inner state with the normal momentum
 * reflected, m - 2 (m . n) n (AdiabaticSlipWall.GetBoundaryState without wall velocities).
 * Kinds 1 and 2 depend on the state, so they enter the JVP and VJP. Other operators accept
 * kind 0 only. When no node has kind 0 the boundary-state table is not needed. */
int bosss_b200_set_boundary_kinds(bosss_handle* h, const int32_t* kinds);

/* Directional derivative J(U)*V of the nonlinear operator; replaces the FD `dirder`
 * of the matrix-free Newton-GMRES (Newton.cs:1450-1495). Host buffers. */
int bosss_b200_jvp(bosss_handle* h, const double* U, const double* V, double* JV, double time);
/* Adjoint product J(U)^T * W (transpose of the Jacobian that
 * EvaluatorLinear.ComputeMatrix / FDJacobianBuilder assemble, DifferentialOperator.cs:1740-1838,
 * 2558-2858). Host buffers. */
int bosss_b200_vjp(bosss_handle* h, const double* U, const double* W, double* JTW, double time);
/* Residual and adjoint product at the same state in one call, host buffers:
 * R = beta*R + alpha*Op(U) and JTW = J(U)^T W. U and W cross PCIe once for both products;
 * like the single-product host entry points, inputs and outputs stream by chunks of grid
 * planes, overlapped with the evaluation (residual + adjoint pair of an adjoint-based
 * optimisation step; in the reference, EvaluatorNonLin.Evaluate plus the transpose of
 * EvaluatorLinear.ComputeMatrix applied to W, DifferentialOperator.cs:1584-1661, 1766-1838). */
int bosss_b200_residual_vjp(bosss_handle* h, double alpha, double beta, const double* U, double* R, const double* W,
                            double* JTW, double time);
int bosss_b200_jvp_device(bosss_handle* h, const double* U_dev, const double* V_dev, double* JV_dev,
                          double time, void* stream);
int bosss_b200_vjp_device(bosss_handle* h, const double* U_dev, const double* W_dev, double* JTW_dev,
                          double time, void* stream);
/* Blocks until all work enqueued on the handle's stream is done; reports device-side errors. */
int bosss_b200_synchronize(bosss_handle* h);

/* ---- block-sparse matrix (BlockMsrMatrix, BoSSS.Platform/LinAlg/BlockMsrMatrix.cs:186) ----
 * Block rows = cells of the codomain mapping, block columns = cells of the domain mapping,
 * every stored block dense (row_block x col_block), row-major within the block.
 * row_ptr[n_block_rows+1], col_idx[nnz_blocks], values[nnz_blocks*row_block*col_block]. */
int bosss_b200_bsr_create(int64_t n_block_rows, int64_t n_block_cols, int32_t row_block,
                          int32_t col_block, const int64_t* row_ptr, const int32_t* col_idx,
                          const double* values, int32_t device, bosss_bsr** out);
int bosss_b200_bsr_destroy(bosss_bsr* A);
/* BlockMsrMatrix.SpMV (BlockMsrMatrix.cs:2554-2990): y = beta*y + alpha*A*x, host buffers. */
int bosss_b200_bsr_spmv(bosss_bsr* A, double alpha, const double* x, double beta, double* y);
/* Device-resident variant on `stream` (NULL = the matrix's stream). */
int bosss_b200_bsr_spmv_device(bosss_bsr* A, double alpha, const double* x_dev, double beta,
                               double* y_dev, void* stream);
/* Reads the matrix back (same layout as bosss_b200_bsr_create's inputs). row_ptr/col_idx/values
 * may be NULL to query sizes only. */
int bosss_b200_bsr_get(const bosss_bsr* A, int64_t* n_block_rows, int64_t* n_block_cols,
                       int32_t* row_block, int32_t* col_block, int64_t* nnz_blocks,
                       int64_t* row_ptr, int32_t* col_idx, double* values);

/* ---- solvers ----
 * Options and report of the Krylov solvers. The matrix-free Newton-GMRES replaces the
 * reference's Newton with MatrixFreeGMRES and the FD `dirder` (Newton.cs:1231-1495) by the
 * exact JVP; bosss_b200_bsr_solve is restarted GMRES in FP32 inside FP64 iterative
 * refinement on an assembled block-sparse matrix. */
typedef struct bosss_solver_opts {
    double rtol;            /* outer relative tolerance on the residual 2-norm */
    double atol;            /* outer absolute tolerance */
    int32_t max_outer;      /* Newton steps (newton_solve) / refinement steps (bsr_solve) */
    int32_t restart;        /* GMRES restart length m (<= 200) */
    int32_t max_krylov;     /* GMRES iterations per outer step */
    int32_t precond;        /* 0 = none, 1 = block-Jacobi on the cell blocks of the Jacobian,
                               2 = multigrid V-cycle (bosss_b200_pmg_create; newton_solve and
                               batch_solve with scalar operators only) */
    double inner_rtol;      /* relative tolerance of each inner (Krylov) solve */
    int32_t precond_update; /* newton_solve: rebuild the preconditioner (Jacobian assembly +
                               setup) every this many Newton steps, the reference's
                               constant_newton_it (Newton.cs:70, 762); 0 or 1: every step */
    int32_t reserved[7];
} bosss_solver_opts;

typedef struct bosss_solver_report {
    int32_t outer_iters;    /* Newton / refinement steps taken */
    int32_t krylov_iters;   /* total GMRES iterations */
    int32_t converged;      /* 1 if the outer tolerance was met */
    int32_t reserved0;
    double residual0;       /* initial residual 2-norm */
    double residual;        /* final residual 2-norm */
    double reserved[6];
} bosss_solver_report;

/* Solve Op(U) = 0 by Newton's method; each step solves J(U) dU = -Op(U) with matrix-free
 * right-preconditioned GMRES on the exact JVP. U: host buffer, initial guess in, solution out. */
int bosss_b200_newton_solve(bosss_handle* h, double* U, double time, const bosss_solver_opts* opt,
                            bosss_solver_report* rep);
/* Solve A x = b (square block-sparse A) with FP32 GMRES inside FP64 iterative refinement;
 * x: host buffer, initial guess in, solution out. */
int bosss_b200_bsr_solve(bosss_bsr* A, const double* b, double* x, const bosss_solver_opts* opt,
                         bosss_solver_report* rep);

/* Multigrid preconditioner of a scalar operator's cell-block Jacobian A (from
 * bosss_b200_compute_jacobian) on the handle's whole Cartesian grid (ClassicMultigrid.Solve,
 * ClassicMultigrid.cs:335-420, over the p-levels of LevelPmg and the aggregation grids of
 * CoarseningAlgorithms.CreateSequence): p-levels of degree K, K-1, ..., 1 (leading sub-blocks of
 * the hierarchical basis, one block-Jacobi sweep before and after the coarse correction), the
 * piecewise-constant level and its 2x2x2 aggregates (two damped Jacobi sweeps each side), a
 * dense coarsest solve. One V-cycle per apply, a fixed linear operator (suitable as a right
 * preconditioner of GMRES). A is copied; it may be destroyed after create. */
typedef struct bosss_pmg bosss_pmg;
int bosss_b200_pmg_create(const bosss_handle* h, const bosss_bsr* A, bosss_pmg** out);
/* x = M^-1 b, device vectors, enqueued on `stream` (NULL: the preconditioner's stream). */
int bosss_b200_pmg_apply_device(bosss_pmg* M, const double* b_dev, double* x_dev, void* stream);
/* Number of p-levels and structured levels, unknowns of the coarsest level, and whether the
 * coarsest level is solved directly (1) or by Jacobi sweeps (0, singular coarsest matrix). */
int bosss_b200_pmg_info(const bosss_pmg* M, int32_t* n_p_levels, int32_t* n_h_levels, int64_t* coarsest,
                        int32_t* coarsest_direct);
int bosss_b200_pmg_destroy(bosss_pmg* M);

/* Jacobian assembly of the operator at state U into a new block-sparse matrix
 * (EvaluatorLinear.ComputeMatrix, LECVolumeQuadrature2.cs:132 / LECEdgeQuadrature2.cs:127 ->
 * BlockMsrMatrix.AccBlock): exact linearisation, cell-block pattern = self + face neighbours. */
int bosss_b200_compute_jacobian(bosss_handle* h, const double* U, double time, bosss_bsr** out);

/* ---- batched evaluation ----
 * Many independent operator instances (own grid, DG degree and quadrature rule each,
 * same physics family; device path: 3D scalar transport / advection-diffusion) evaluated
 * by ONE persistent launch per mode: CTAs pull (instance, cell tile) work items from a
 * queue in device memory. Vectors are the concatenation of the instances' vectors
 * (offsets from bosss_b200_batch_get_sizes). The residual + VJP pair can be captured once
 * into a CUDA graph and replayed; an autotuner picks the cell tiles per work item for each
 * (degree, quadrature nodes) class and the queue order, persisted in a small text table.
 * Tile kernel per mode (opt->kernel): 0 = automatic (register-blocked slab tiles when every
 * instance has at most 5 nodes per direction; else the generic tiles),
 * 1 = generic tiles, 2 = slab tiles wherever every instance allows them. */
typedef struct bosss_batch bosss_batch;

enum bosss_eval_mode { BOSSS_MODE_RESIDUAL = 0, BOSSS_MODE_JVP = 1, BOSSS_MODE_VJP = 2 };

int bosss_b200_batch_create(int32_t n, const bosss_op_desc* ops, const bosss_grid_desc* grids,
                            const bosss_options* opt, bosss_batch** out);
int bosss_b200_batch_destroy(bosss_batch* b);
/* prefix offsets (n+1 entries each) of the instances in the concatenated vectors */
int bosss_b200_batch_get_sizes(const bosss_batch* b, int64_t* domain_offsets, int64_t* codomain_offsets);
/* mode RESIDUAL: out = beta*out + alpha*Op(U); JVP: out = J(U) V; VJP: out = J(U)^T V. Host buffers. */
int bosss_b200_batch_evaluate(bosss_batch* b, int32_t mode, double alpha, double beta, const double* U,
                              const double* V, double* out, double time);
int bosss_b200_batch_evaluate_device(bosss_batch* b, int32_t mode, double alpha, double beta, const double* U_dev,
                                     const double* V_dev, double* out_dev, double time, void* stream);
/* capture R = Op(U) and G = J(U)^T W for all instances into a CUDA graph (device buffers) */
int bosss_b200_batch_capture(bosss_batch* b, const double* U_dev, const double* W_dev, double* R_dev, double* G_dev,
                             double time);
int bosss_b200_batch_replay(bosss_batch* b, void* stream);
/* time candidate tile counts per (degree, nodes) class and the queue order on the given
 * buffers; reads/writes the text table at table_path (NULL: no persistence) */
int bosss_b200_batch_autotune(bosss_batch* b, const double* U_dev, const double* W_dev, double* R_dev, double* G_dev,
                              const char* table_path);
/* The autotuned choice: tiles per work item of the (K, Q) class, and the schedule in *lpt:
 * 1 = persistent queue longest first, 0 = persistent queue in instance order, 2 = one launch
 * per (K, Q) class with the single-grid launch configuration. */
int bosss_b200_batch_tiles(const bosss_batch* b, int32_t K, int32_t Q, int32_t* tiles, int32_t* lpt);

/* Per-instance implicit-step solves over the batch: for every instance i
 *   (I/dt[i] + J_i(U)) x_i = b_i          (transpose = 0; JVP as the operator)
 *   (I/dt[i] + J_i(U))^T x_i = b_i        (transpose = 1; the adjoint system on the VJP)
 * -- the system of ImplicitEuler.PerformTimeStep, (diag(1/dt) + M) x = state/dt - affine
 * (ImplicitEuler.cs:86-116; the mass matrix of the orthonormal basis is the identity), and its
 * adjoint. FP32 GMRES(restart) on
 * FP32 vectors, the operator applied in FP64, inside FP64 iterative refinement until
 * ||b_i - A_i x_i|| <= max(rtol ||b_i||, atol) (defaults: rtol 1e-10, 30 refinement steps,
 * inner tolerance 1e-3; SoftGMRES.cs on a BlockMsrMatrix in the reference, here
 * matrix-free); precond 1 (default): block-Jacobi on the diagonal cell blocks of
 * I/dt + J_i, probed with a face-neighbour colouring; 2: one multigrid V-cycle
 * (bosss_b200_pmg_create) on the assembled I/dt + J_i, or its transpose for the adjoint
 * systems (scalar operators); 0: none. Device vectors (concatenated
 * instance vectors, bosss_b200_batch_get_sizes offsets): U the state of the linearisation
 * (NULL: zero; the Jacobian of the linear advection-diffusion family does not depend on it),
 * b the right-hand sides, x the initial guesses in and the solutions out. reports: NULL or
 * n entries. The instances are solved largest first by 4 host threads, each on its own
 * stream with its own work arrays. Returns after the solves have completed. */
int bosss_b200_batch_solve(bosss_batch* b, int32_t transpose, const double* dt, const double* U_dev,
                           const double* b_dev, double* x_dev, const bosss_solver_opts* opt,
                           bosss_solver_report* reports);

/* ---- XDG: per-species bulk evaluation with moment-fitted cut-cell rules ----
 * XEvaluatorNonlin.Evaluate, bulk part (XSpatialOperatorMk2_XEvaluators.cs:372-511): for
 * species A (phi < 0) and B (phi >= 0) the species' bulk operator (XLaplace_Bulk =
 * SIPLaplace with nu = mu_s, XLaplace.cs:50-120, plus sources) is integrated over the
 * cells and faces that contain the species; cut cells and cut faces use per-item rules
 * fitted to the moments of the species part (LevelSetComboRuleFactory2.cs:300-528:
 * candidate nodes = tensor Gauss nodes inside the species part, moments integrated on the
 * device, minimum-norm least-squares weights as DGELSY returns them, IMatrixExtensions.cs:
 * 2318-2340). Level-set (interface) terms are not part of this evaluator.
 * Vectors are species frames: a full-grid DG vector per species (J * Np, the reference's
 * cell-major layout); entries of cells without the species are ignored and returned 0. */
enum bosss_levelset_type { BOSSS_LEVELSET_SPHERE = 1 };   /* phi = |x - c| - r, params = c[3], r */

typedef struct bosss_levelset_desc {
    int32_t type;
    double params[8];
} bosss_levelset_desc;

typedef struct bosss_xdg_opts {
    int32_t cut_nodes_1d;       /* candidate Gauss nodes per direction (default 5) */
    int32_t fallback_nodes_1d;  /* candidates for species parts with < 8 nodes (default 9) */
    int32_t moment_degree;      /* fitted polynomial degree (default min(2k, 4)); <0: default */
    int32_t subdivision;        /* moment integration: S x S coarse boxes, cut ones S x S again (default 8) */
    int32_t rule;               /* cut-cell rule family: 0 = moment fitting on Gauss-node subsets (default),
                                   1 = Saye-type recursive Gauss rules (the reference's default,
                                   SayeGaussRule_*.cs), cut_nodes_1d Gauss nodes per direction and
                                   piece; moments are still integrated and the rules' residual
                                   against them is reported as the fit residual */
    int32_t reserved[7];
} bosss_xdg_opts;

typedef struct bosss_xdg bosss_xdg;

int bosss_b200_xdg_create(const bosss_op_desc* opA, const bosss_op_desc* opB, const bosss_grid_desc* grid,
                          const bosss_levelset_desc* ls, const bosss_xdg_opts* xopt, const bosss_options* opt,
                          bosss_xdg** out);
int bosss_b200_xdg_destroy(bosss_xdg* X);
/* cells with the species, cut cells / cut faces with rules, node-count range, lowest fitted
 * degree and the largest relative moment residual of the fitted rules */
int bosss_b200_xdg_info(const bosss_xdg* X, int32_t species, int64_t* n_cells, int64_t* n_cut_cells,
                        int64_t* n_cut_faces, int32_t* min_nodes, int32_t* max_nodes, int32_t* min_degree,
                        double* max_fit_residual);
/* rules of a species: n_items[2] = {items, nodes}; item_info[5 per item] = (cell, dim (3 volume,
 * 2 face), face direction, face side, fitted degree); node_offsets[items+1]; nodes[3 per node]
 * (reference coordinates of the cell, or of the face in its two in-plane directions);
 * weights[nodes]; vol_flags[J] and face_flags[J*6] (0 absent, 1 standard rule, 2 cut rule).
 * Any output pointer may be NULL. */
/* Saye-type rule of one species part of a box, host computation (no device needed): the part
 * {phi < 0} (species -1) or {phi >= 0} (species +1) of the cell [center - h/2, center + h/2]
 * (dim 3) or of its face normal to `dir` through `center` (dim 2; center[dir] is the face
 * coordinate), nodes_1d Gauss nodes per direction and piece. Nodes in reference coordinates
 * of the cell / face ([-1,1]^dim, 3 per node, unused entries 0), weights in the reference
 * measure. Call with nodes = weights = NULL to get the count in *n_nodes, then with arrays of
 * that size. */
int bosss_b200_saye_rule(const bosss_levelset_desc* ls, int32_t dim, int32_t dir, int32_t species,
                         const double* center, const double* h, int32_t nodes_1d, int64_t* n_nodes, double* nodes,
                         double* weights);
int bosss_b200_xdg_get_rules(const bosss_xdg* X, int32_t species, int64_t* n_items, int64_t* item_info,
                             int64_t* node_offsets, double* nodes, double* weights, unsigned char* vol_flags,
                             unsigned char* face_flags);
/* the fitted moments, 35 per item (unused trailing entries 0): int over the species part of the
 * reference basis functions of degree <= moment_degree (3D items) or of the face basis (faces) */
int bosss_b200_xdg_get_moments(const bosss_xdg* X, int32_t species, double* moments);
int bosss_b200_xdg_evaluate(bosss_xdg* X, int32_t species, double alpha, double beta, const double* U, double* out,
                            double time);
/* Cell length scales of a species' SIP penalty: the CoefficientSet.CellLengthScales that
 * XLaplace_Bulk and the base SIPLaplace read (XLaplace.cs:104-113, 193-198; ipLaplace.cs:131-141;
 * inner faces max(1/len[in], 1/len[out]), boundary faces 2/len[in]) and that the interface term
 * reads for both species (XLaplace.cs:261-297, max(1/len_A[j], 1/len_B[j])). len: J values in the
 * grid's cell order. Default, computed at create from the fitted rules as
 * MultiphaseAgglomerator.LengthScaleAgg does without agglomeration (MultiphaseAgglomerator.cs:744-944):
 * len = species volume / (interface area + the species' part of every face of the cell), at
 * least machine epsilon * h, and 1e10 times the uncut length scale for cells whose volume
 * fraction is <= 1e-10; NaN for cells without the species. set: the caller's scales (e.g. the
 * agglomerated ones of its cell agglomerator, XOperatorFactoryBase.cs:93-105), finite and
 * positive on every cell of the species; NULL restores the default. */
int bosss_b200_xdg_get_length_scales(const bosss_xdg* X, int32_t species, double* len);
int bosss_b200_xdg_set_length_scales(bosss_xdg* X, int32_t species, const double* len);
int bosss_b200_xdg_evaluate_device(bosss_xdg* X, int32_t species, double alpha, double beta, const double* U_dev,
                                   double* out_dev, double time, void* stream);

/* Level-set interface term of the two-phase Poisson problem: XLaplace_Interface.InnerEdgeForm
 * (src/L3-solution/BoSSS.Solution.XNSECommon/XLaplace.cs:205-345) integrated over the level-set
 * surface of every cut cell, as NECQuadratureLevelSet.EvaluateEx / SaveIntegrationResults do
 * (src/L2-foundation/BoSSS.Foundation.XDG/NECQuadratureLevelSet.cs:35-664).
 * setup: mu_A (phi < 0), mu_B (phi > 0), penalty base factor and mode as the XLaplace_Interface
 * constructor (mode BOSSS_IFACE_SWIP or BOSSS_IFACE_SIP, the reference's enum order); builds the
 * surface rules of the sphere on the host (nodes_1d Gauss nodes per interval; <= 0: 6).
 * The penalty's size factor is max(1/len_A[j], 1/len_B[j]) of the species' cell length scales
 * (bosss_b200_xdg_get_length_scales). */
enum bosss_iface_mode { BOSSS_IFACE_SWIP = 0, BOSSS_IFACE_SIP = 1 };
int bosss_b200_xdg_interface_setup(bosss_xdg* X, double mu_A, double mu_B, double penalty_base, int32_t mode,
                                   int32_t nodes_1d);
/* counts[2] = {cut cells with surface nodes, nodes}; then (any may be NULL) the cells, node
 * offsets (cells + 1), nodes in reference coordinates of the cell (3 per node), weights (physical
 * surface measure) and unit normals grad(phi)/|grad(phi)| (3 per node, from A into B) */
int bosss_b200_xdg_interface_get_rules(const bosss_xdg* X, int64_t* counts, int64_t* cells, int64_t* node_offsets,
                                       double* nodes, double* weights, double* normals);
/* out_A += alpha * (interface term tested with species A), out_B likewise; U_A, U_B and the
 * outputs are the species' coefficient vectors of bosss_b200_xdg_evaluate (cell-major, all cells) */
int bosss_b200_xdg_interface_evaluate(bosss_xdg* X, double alpha, const double* U_A, const double* U_B,
                                      double* out_A, double* out_B);
int bosss_b200_xdg_interface_evaluate_device(bosss_xdg* X, double alpha, const double* U_A_dev,
                                             const double* U_B_dev, double* out_A_dev, double* out_B_dev,
                                             void* stream);

/* ---- explicit Runge-Kutta time stepping ----
 * RungeKutta.Perform / PerformStage (TimeStepping/RungeKutta.cs:240-330) with the change rate
 * of ExplicitEuler.ComputeChangeRate (ExplicitEuler.cs:223-229): for s = 0..stages-1
 *   u_s = U - dt * sum_{r<s} a[s][r] k_r,   k_s = Op(u_s)   (evaluated at time + c[s]*dt),
 * then U <- U - dt * sum_s b[s] k_s. `a` is stages x stages row-major and strictly lower
 * triangular (explicit), `b` and `c` have `stages` entries, stages <= 8. The operator must be
 * square (domain DOFs == codomain DOFs). Named tableaus (RungeKuttaScheme.cs) are supplied by
 * the caller; the Python mirror carries them. */
int bosss_b200_rk_work_size(const bosss_handle* h, int32_t stages, int64_t* n_doubles);
/* nsteps steps on device buffers: U_dev in/out, work_dev of bosss_b200_rk_work_size doubles.
 * use_graph != 0: one step is captured into a CUDA graph once and the graph is launched nsteps
 * times (one residual launch and one stage-combination launch per stage). Asynchronous on
 * `stream` (NULL: the handle's stream). */
int bosss_b200_rk_steps_device(bosss_handle* h, int32_t stages, const double* a, const double* b, const double* c,
                               double dt, int32_t nsteps, double time, double* U_dev, double* work_dev,
                               int32_t use_graph, void* stream);
/* Same with a host state vector U (copied in, stepped with a captured graph, copied back). */
int bosss_b200_rk_steps(bosss_handle* h, int32_t stages, const double* a, const double* b, const double* c, double dt,
                        int32_t nsteps, double time, double* U);

/* Residual (mode 0), JVP (1) or VJP (2) on the cells [cell_begin, cell_end) of the handle's
 * grid only, device buffers, enqueued on `stream` (NULL: the handle's stream): the cells'
 * outputs are written (residual: out = beta*out + alpha*R; JVP / VJP: out = the product,
 * alpha and beta unused), nothing else is. U and V hold the whole
 * grid, so the cells' face neighbours are read. This is the building block of partitioned
 * evaluation with ghost layers: the interior of a part is evaluated while the halo exchange
 * of its ghost cells is in flight, the cells next to the ghosts afterwards
 * (EvaluatorNonLin.Evaluate with MPI, DifferentialOperator.cs:1599-1627). */
int bosss_b200_apply_device(bosss_handle* h, int32_t mode, double alpha, double beta, const double* U_dev,
                            const double* V_dev, double* out_dev, double time, int64_t cell_begin,
                            int64_t cell_end, void* stream);

/* Batched evaluation that allocates no device memory (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: hosts whose device memory belongs to another
 * allocator, or loops that must not synchronise the device with an allocation. Same
 * persistent kernel as the batch above, but its scratch (work-queue counter, instance
 * table, tile prefix sums) lives in a fixed 1 MiB device array inside the library, held
 * by every GPU that loads the library until exit: at most 512 instances per call; larger
 * batches are rejected with BOSSS_ERR_BAD_ARG. `instances`: n handles from
 * bosss_b200_create (which allocates no device memory), same physics family (3D scalar
 * transport / advection-diffusion); vectors are the caller's device buffers, the
 * concatenation of the instances' vectors in the given order; modes as above. Whole grids
 * only: a part of a partitioned grid is rejected with BOSSS_ERR_BAD_ARG. The first call on
 * a device looks up the array's device address; make that first call before any stream
 * capture. Every call overwrites the shared array (the queue counter is cleared by each
 * call): calls on one stream are ordered by the stream, but calls whose kernels overlap on
 * the GPU (other streams, other threads) race. The call does not wait for its kernel: it
 * returns once the launch is enqueued. Its small instance table is copied from pageable
 * host memory, which the CUDA runtime stages before the copy call returns. */
int bosss_b200_batch_evaluate_noalloc(int32_t n, bosss_handle* const* instances, int32_t mode, double alpha,
                                      double beta, const double* U_dev, const double* V_dev, double* out_dev,
                                      double time, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BOSSS_B200_H */
