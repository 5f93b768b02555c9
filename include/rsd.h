/* rsd.h - C ABI of the B200 (sm_100a) backend for the Residuum heat-equation hot path.
 *
 * Plain pointers, sizes and status codes; no exceptions, no C++ or torch types cross this line.
 * Each entry point names the reference interface it stands in for (paths relative to the
 * Residuum reference tree).  Device pointers are CUDA global-memory pointers on the context's
 * device; "host" arguments are ordinary CPU memory.
 *
 * Conventions
 *   - every function returns RSD_OK (0) or a negative RSD_E* code; rsd_last_error_string()
 *     describes the last failure on the calling thread;
 *   - one rsd_ctx owns one CUDA stream; calls on a context are ordered on that stream and
 *     return after their results are complete unless documented otherwise;
 *   - solver non-convergence is not an error: it is report.converged == 0, as the reference's
 *     solvers return false with a filled SolverReport (linalg/solver/iterative/cg/Solver.tpp:110-117).
 */
#ifndef RSD_H
#define RSD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSD_OK 0
#define RSD_EINVAL (-1)       /* bad argument, size or unsupported discretization */
#define RSD_ENOMEM (-2)       /* device allocation failed */
#define RSD_ECUDA (-3)        /* CUDA runtime error */
#define RSD_EBREAKDOWN (-5)   /* Krylov breakdown with a non-finite scalar */
#define RSD_ENAN (-6)         /* non-finite value detected */
#define RSD_EPARSE (-7)       /* expression string could not be compiled */
#define RSD_ETIMEOUT (-8)     /* a bounded device wait gave up */

typedef struct rsd_ctx rsd_ctx;
typedef struct rsd_csr rsd_csr;
typedef struct rsd_mesh rsd_mesh;
typedef struct rsd_heat rsd_heat;

/* CopyKind (include/linalg/types/backend/cuda/CopyKind.hpp:9-14) */
enum { RSD_H2H = 0, RSD_H2D = 1, RSD_D2H = 2, RSD_D2D = 3 };

/* LinearSolverConfig::Type / PreconditionerConfig::Type (include/solver/config/LinearSolverConfig.hpp) */
enum { RSD_CG = 0, RSD_GMRES = 1 };
enum { RSD_IDENTITY = 0, RSD_JACOBI = 1 };
enum { RSD_FP64 = 0, RSD_MIXED = 1 };
enum { RSD_TOL_RELATIVE = 0, RSD_TOL_ABSOLUTE = 1 };
/* LinearSolverConfig::OperatorType (include/solver/config/LinearSolverConfig.hpp:49-56) */
enum { RSD_OP_CSR = 0, RSD_OP_FEM = 1 };

/* SolverReport (include/linalg/solver/base/SolverReport.hpp:12-28) plus device-path extras */
typedef struct rsd_report {
	int32_t converged;
	int32_t status;              /* RSD_OK or the RSD_E* that stopped the solve */
	int64_t iterations;
	double initialResidual;      /* ||b - A x0|| */
	double finalResidual;        /* ||r_k|| of the recurrence (reference semantics) */
	double finalResidualRel;     /* finalResidual / (initialResidual + 1e-50) */
	double trueResidualRel;      /* mixed precision: ||b - A64 x|| / ||r0||, recomputed in FP64 */
	int64_t refinements;         /* mixed precision: FP64 residual replacements */
} rsd_report;

/* cg::Config / gmres::Config (linalg/solver/iterative/{cg,gmres}/Config.hpp) plus precision */
typedef struct rsd_solver_cfg {
	int32_t type;                /* RSD_CG or RSD_GMRES */
	int32_t precond;             /* RSD_IDENTITY or RSD_JACOBI */
	int32_t precision;           /* RSD_FP64 or RSD_MIXED (FP32 inner, FP64 residual) */
	int32_t tol_type;            /* RSD_TOL_RELATIVE or RSD_TOL_ABSOLUTE */
	double tol;
	int64_t max_iters;
	int64_t krylov_dim;          /* GMRES restart length m */
	double reliable_delta;       /* mixed CG: FP64 residual replacement when |r| falls by this factor; 0: adaptive,
	                                from 0.1, set at each replacement from the recurrence/true residual gap, in [1e-4, 0.1]
	                                (the batched solver: [1e-3, 0.1]) */
	int32_t operator_type;       /* RSD_OP_CSR, or RSD_OP_FEM: the heat stages assemble no matrix and solve with the
	                                matrix-free operator (FEMOperator: element-kernel products, Jacobi from the
	                                element diagonal; CG or GMRES in FP64).  rsd_solve and rsd_batch_solve take RSD_OP_CSR. */
	int32_t reserved;            /* zero */
} rsd_solver_cfg;

/* ---- lifetime (linalg/types/backend/CUDA.hpp:23-73 has no context; these give it one) ---- */
int rsd_ctx_create(int device, rsd_ctx** out);
int rsd_ctx_destroy(rsd_ctx* ctx);
int rsd_ctx_sync(rsd_ctx* ctx);
void* rsd_ctx_stream(rsd_ctx* ctx);
const char* rsd_last_error_string(void);
int rsd_version(int32_t* major, int32_t* minor);
/* Compile an expression (the subset the heat problem's expression strings take) on the host without a
 * device: RSD_OK and the evaluation stack depth its program needs, or RSD_EPARSE with the reason,
 * e.g. a depth above the device machine's 16 entries.  No counterpart in the reference (exprtk
 * compiles in the reference's ScalarExpression / TemperatureExpression constructors). */
int rsd_expr_check(const char* expr, int32_t* depth);
/* Tracing (the reference has only its benchmark Timer, include/benchmark/core/Timer.hpp:10-24):
 * when enabled, every launch of the kernel families "spmv_dot_f64", "spmv_dot_f32", "cg_update",
 * "cg_pupdate", "reliable_update", "assemble_matrix", "assemble_vector", "spmv", "cg_persist" (the
 * mixed solve's persistent kernel, one launch per solve) is bracketed by CUDA events on the context
 * stream; rsd_ctx_profile_get returns launches and summed device time.
 * Enabling (or disabling) resets the totals. */
int rsd_ctx_profile(rsd_ctx* ctx, int32_t enable);
int rsd_ctx_profile_get(rsd_ctx* ctx, const char* family, int64_t* launches, double* total_ms);

/* ---- memory: CUDA::alloc / copy / zero / set (linalg/types/backend/CUDA.hpp:30-71) ---- */
int rsd_alloc(rsd_ctx* ctx, size_t bytes, void** dptr);
int rsd_free(rsd_ctx* ctx, void* dptr);
/* Device memory that host code may also read (managed memory, resident on the device): the backend
 * tag's vectors use it because the reference's NewtonRunner reads the stage residual's entries on the
 * host (solver/nonlinear/Newton.hpp:45, fem/dof/DOFResidualNorms.hpp:13-24); read it only after the
 * context's stream has finished with it.  Freed with rsd_free.  No counterpart in the reference's
 * CUDA tag, which allocates with cudaMalloc (linalg/types/backend/CUDA.hpp:30-37). */
int rsd_alloc_managed(rsd_ctx* ctx, size_t bytes, void** dptr);
int rsd_memcpy(rsd_ctx* ctx, void* dst, const void* src, size_t bytes, int32_t kind);
int rsd_memset_zero(rsd_ctx* ctx, void* dptr, size_t bytes);
int rsd_fill_f64(rsd_ctx* ctx, double* x, int64_t n, double value);
int rsd_fill_f32(rsd_ctx* ctx, float* x, int64_t n, float value);

/* ---- BLAS-1: operations::dot/axpy/axpby/scal/copy/multiply/norm
 *      (linalg/operations/VectorOps.hpp:10-36, backend/cpu/VectorOps.tpp:7-86).
 *      Reductions are deterministic (fixed two-stage order) and return to host memory. ---- */
int rsd_dot(rsd_ctx* ctx, int64_t n, const double* x, const double* y, double* out);
int rsd_nrm2(rsd_ctx* ctx, int64_t n, const double* x, double* out);
int rsd_axpy(rsd_ctx* ctx, int64_t n, double alpha, const double* x, double* y);
int rsd_axpby(rsd_ctx* ctx, int64_t n, double alpha, double beta, const double* x, double* y);
int rsd_scal(rsd_ctx* ctx, int64_t n, double alpha, double* x);
int rsd_copy(rsd_ctx* ctx, int64_t n, const double* x, double* y);
int rsd_mul(rsd_ctx* ctx, int64_t n, const double* x, const double* y, double* z);

/* ---- CSR matrix: CSRMatrix<Real, CUDA> (linalg/types/CSRMatrix.hpp:14-88).  Host input uses
 *      the reference's 64-bit Index; the device copy holds 32-bit rowPtr/colIdx (nnz < 2^31). ---- */
int rsd_csr_create(rsd_ctx* ctx, int64_t nrows, int64_t nnz, const int64_t* row_ptr, const int64_t* col_idx,
                   const double* values, rsd_csr** out);
int rsd_csr_destroy(rsd_csr* A);
int rsd_csr_info(const rsd_csr* A, int64_t* nrows, int64_t* nnz);
/* The execution layout's size (no counterpart in the reference, whose CSR has one layout): SELL-32
 * slots (entries including padding), slices of 32 rows, and the slices stored as stencil slices
 * (no column indices); any output may be NULL. */
int rsd_csr_layout(const rsd_csr* A, int64_t* sell_slots, int64_t* slices, int64_t* stencil_slices);
/* Mirrored stencil slices of the layout (no counterpart in the reference): slices whose entries at
 * negative column offsets the mixed CG's FP32 SpMV reads from the mirror rows' own entries while the
 * values are known symmetric to the last bit (as the row-gather assembly of 4- and 8-node elements
 * writes them); `active` is 1 when the current values qualify.  Either output may be NULL. */
int rsd_csr_mirrored(const rsd_csr* A, int64_t* mirrored_slices, int32_t* active);
/* device pointer to the CSR-order values (writes through it are allowed until the next call on A) */
int rsd_csr_values(rsd_ctx* ctx, rsd_csr* A, double** dvalues);
int rsd_csr_set_values(rsd_ctx* ctx, rsd_csr* A, const double* host_values);
int rsd_csr_get_values(rsd_ctx* ctx, rsd_csr* A, double* host_values);
int rsd_csr_get_pattern(rsd_ctx* ctx, const rsd_csr* A, int64_t* host_row_ptr, int64_t* host_col_idx);
/* operations::matvec (linalg/operations/backend/cpu/MatrixOps.tpp:5-23), device vectors */
int rsd_spmv(rsd_ctx* ctx, const rsd_csr* A, const double* x, double* y);
/* FP32 copy of the values (refreshed from FP64) and its SpMV, for the mixed-precision path */
int rsd_csr_sync_f32(rsd_ctx* ctx, rsd_csr* A);
int rsd_spmv_f32(rsd_ctx* ctx, const rsd_csr* A, const float* x, float* y);
/* CSROperator::diagonal (linalg/operator/CSROperator.hpp:40-45), operations::lump (MatrixOps.tpp:25-43) */
int rsd_csr_diagonal(rsd_ctx* ctx, const rsd_csr* A, double* d);
int rsd_csr_lump(rsd_ctx* ctx, const rsd_csr* A, double* d);
/* Jacobi::update (linalg/solver/preconditioner/Jacobi.hpp:23-36): invD = |d|>1e-300 ? 1/d : 1 */
int rsd_jacobi_setup(rsd_ctx* ctx, const rsd_csr* A, double* inv_diag);
/* Execution layout and launch shape of SpMV and the Krylov kernels: lanes_per_row 0 selects the
 * SELL-32 layout (one thread per row, slices of 32 rows stored column-major; the default),
 * 1..32 (power of two) CSR with that many lanes per row; block_threads 64..512 (power of two),
 * 0 for the default.  The autotuner times every choice and keeps the fastest. */
int rsd_csr_set_launch(rsd_csr* A, int32_t lanes_per_row, int32_t block_threads);
int rsd_csr_autotune(rsd_ctx* ctx, rsd_csr* A, int32_t* lanes_per_row, int32_t* block_threads, double* best_us);
/* Measured FP64 FMA throughput of the device (non-tensor pipe), in TFLOP/s, for the element
 * assembly's roofline: independent FMA chains on every SM, timed with CUDA events.  No counterpart
 * in the reference (a measurement helper). */
int rsd_measure_fp64_rate(rsd_ctx* ctx, double* tflops);

/* ---- Krylov solves: CGRunner / GMRESRunner::solve (linalg/solver/iterative/cg/Solver.tpp:13-119,
 *      gmres/Solver.tpp:3-170) through LinearSolverRunner::solve(b, x, report)
 *      (linalg/solver/base/LinearSolverRunner.hpp:16); b and x are device vectors. ---- */
int rsd_solve(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* report);
/* FP64 CG (cfg->type RSD_CG, cfg->precision RSD_FP64; identity or Jacobi) that allocates nothing:
 * no counterpart in the reference.  Same kernels, grids and reductions as rsd_solve's FP64 CG, so
 * the same iterates and report, but its scratch (residual, search direction, A p, inverse diagonal,
 * reduction partials and device scalars) is one file-scope device array of 8 MiB + 19 KiB, which
 * limits A to at most 262,144 rows; larger matrices are rejected with RSD_EINVAL and a message.
 * The scalars and reduction tickets that must start at zero are cleared on the stream by each call.
 * The array is shared by every call on a device: calls that overlap on one device (two host threads,
 * or two streams in flight) race on it and must be serialized by the caller.  The call synchronizes
 * the stream and reads its report into pageable host memory, so it cannot be used inside a stream
 * capture.  The first call on a device looks up the array's device address and keeps it for the
 * life of the process: a primary context torn down and recreated (cudaDeviceReset) leaves that
 * address stale, so do not reset the device between calls. */
int rsd_cg_solve_static(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x,
                        rsd_report* report);

/* ---- mesh: mesh::Data (include/mesh/Data.hpp:13-35), host arrays in that layout ---- */
int rsd_mesh_create(rsd_ctx* ctx, int32_t nsd, int32_t order, int64_t num_nodes, int64_t num_elements,
                    const double* xyz, const int64_t* ien, const int32_t* rng, rsd_mesh** out);
int rsd_mesh_destroy(rsd_mesh* m);
/* PMSH, the reference's binary mesh file (MeshIO::readBinary, src/io/MeshIO.cpp:84-151; layout as
 * MeshIO::writeBinary writes it, include/io/MeshIO.hpp:16-35).  rsd_pmsh_read runs on the host without a
 * device: the header into info and, when the arrays are given (each may be NULL), xyz (num_nodes *
 * spatial_dim), ien (num_elements * nodes_per_element, 64-bit) and rng (num_elements * faces_per_element).
 * rsd_mesh_read_pmsh reads a Lagrange quadrilateral or hexahedral mesh of equal order in every direction
 * into a device mesh.  Malformed files give RSD_EINVAL with the reason. */
typedef struct rsd_pmsh_info {
	int32_t parametric_dim, spatial_dim;
	int32_t family;              /* mesh::ElementFamily: 0 Quad, 1 Tri, 2 Hex, 3 Tet, 4 Wedge */
	int32_t basis;               /* mesh::BasisType: 0 Lagrange, 1 Spline */
	int64_t num_nodes, num_elements;
	int32_t nodes_per_element, faces_per_element;
	int32_t num_orders, order[3];
	int32_t iga;                 /* extraction operators present */
} rsd_pmsh_info;
int rsd_pmsh_read(const char* path, rsd_pmsh_info* info, double* xyz, int64_t* ien, int32_t* rng);
int rsd_mesh_read_pmsh(rsd_ctx* ctx, const char* path, rsd_mesh** out);

/* ---- heat problem: HeatProblem<CUDA, HeatEquation<NSD,NSD,Family>>
 *      (application/heateq/problem/HeatProblem.hpp:34-206).  Expression strings use the
 *      reference's exprtk syntax subset (numbers, t x y z T, pi, + - * / ^, unary -, sin cos tan
 *      exp log sqrt abs). ---- */
typedef struct rsd_heat_desc {
	int32_t nq;                      /* Gauss points per direction */
	double k_const;                  /* conductivity when k_expr is NULL */
	const char* k_expr;              /* k(T), or NULL */
	const char* dk_expr;             /* dk/dT(T), or NULL (0) */
	const double* k_elem;            /* host, one multiplier per element, or NULL */
	double rho, cp;                  /* density, specific heat (cp when cp_expr is NULL) */
	const char* src_expr;            /* volumetric source f(t,x,y,z), or NULL (0) */
	const char* dirichlet_expr[6];   /* Dirichlet value per boundary tag 0..5; NULL = tag not essential */
	/* ConductivityModel (equation/heateq/evaluator/ConductivityModel.hpp:60-96) with an anisotropic
	 * shape: K = k * k_tensor, k being k_const or k(T) (set k_const = 1 for the reference's constant
	 * Anisotropic type); host, nsd x nsd row-major, or NULL for the isotropic K = k I */
	const double* k_tensor;
	/* SpecificHeatModel (equation/heateq/evaluator/SpecificHeatModel.hpp:35-61), TemperatureDependent:
	 * cp(T) and dcp/dT(T) (the latter feeds TangentMassForm), or NULL for the constant cp */
	const char* cp_expr;
	const char* dcp_expr;
	/* further essential tags of any value >= 0 (EssentialBoundaryRegistry takes any tag,
	 * fem/boundary/EssentialBoundaryRegistry.hpp:15-59): num_dirichlet pairs of a tag and its
	 * Dirichlet expression, registered after the dirichlet_expr entries (a tag given twice keeps the
	 * later expression) */
	int32_t num_dirichlet;
	const int32_t* dirichlet_tags;
	const char* const* dirichlet_exprs;
} rsd_heat_desc;

/* constructor + TopologicalDOF::buildConstraints + Assembler::createMatrix
 * (HeatProblem.tpp:4-176, topology/TopologicalDOF.tpp:34-111, fem/assembly/backend/cpu/Assembler.tpp:8-76) */
int rsd_heat_create(rsd_ctx* ctx, const rsd_mesh* m, const rsd_heat_desc* desc, rsd_heat** out);
int rsd_heat_destroy(rsd_heat* h);
int rsd_heat_info(const rsd_heat* h, int64_t* num_free, int64_t* nnz);
int rsd_heat_dofmap(rsd_ctx* ctx, const rsd_heat* h, int32_t* host_topo_to_alg, int32_t* host_alg_to_topo);
int rsd_heat_matrix(rsd_heat* h, rsd_csr** A);       /* the problem's K/J storage (owned by h) */
/* HeatProblem::createMatrix (HeatProblem.hpp:62, Assembler::createMatrix): a new matrix with h's
 * pattern, sharing h's pattern arrays, with zero values of its own; destroy it with rsd_csr_destroy
 * before h. */
int rsd_heat_create_matrix(rsd_ctx* ctx, rsd_heat* h, rsd_csr** A);
/* HeatProblem::loadNodalField, Expression mode (HeatProblem.tpp:185-205): U[free dof of node v] =
 * expr(t, x_v, y_v, z_v) for every free node (the initial condition); U device, num_free entries */
int rsd_heat_eval_nodal(rsd_ctx* ctx, rsd_heat* h, const char* expr, double t, double* U);
int rsd_heat_set_time(rsd_ctx* ctx, rsd_heat* h, double t);   /* re-evaluates Dirichlet node values */
int rsd_heat_set_k_elem(rsd_ctx* ctx, rsd_heat* h, const double* k_elem_device);

/* Assembler::assembleMatrix (fem/assembly/backend/cpu/Assembler.tpp:86-140): zero A, then
 * scatter c_diff*Diffusion + c_mass*Mass + c_tdiff*TangentDiffusion + c_tmass*TangentMass.
 * U (free DOFs; Dirichlet values injected, GatherMode::Full) and Udot (GatherMode::Free) are
 * device vectors or NULL (zero).  A must have h's pattern (rsd_heat_matrix or a copy). */
int rsd_assemble_matrix(rsd_ctx* ctx, rsd_heat* h, double c_diff, double c_mass, double c_tdiff, double c_tmass,
                        const double* U, const double* Udot, rsd_csr* A);
/* Assembler::assembleVector (Assembler.tpp:199-255) with the stages' form/operand pairings:
 * which 0: load (SourceForm); 1: Diffusion on U (Full); 2: rho*cp*Mass on U (Full);
 * 3: rho*cp*Mass on Udot (Free); 4: Diffusion + coef*Mass on operand (Free; FEMOperator::apply);
 * 10: Diffusion + TangentDiffusion + coef*Mass on operand at the state U (the Jacobian's product) */
int rsd_assemble_vector(rsd_ctx* ctx, rsd_heat* h, int32_t which, double coef, const double* U, const double* Udot,
                        const double* operand, double* out);
/* The LinearSolverRunner HeatProblem::makeLinearRunner builds for OperatorType::FEM
 * (application/heateq/problem/HeatProblem.tpp:274-289) over FEMOperator (linalg/operator/FEMOperator.hpp:39-56)
 * with the forms Diffusion + c_mass*Mass: solves A x = b without a matrix, every product an element
 * pass (rsd_assemble_vector mode 4 with the iterate as the k(T) state), Jacobi from the element
 * diagonal (Assembler::assembleDiagonal).  cfg: type RSD_CG or RSD_GMRES, precision RSD_FP64;
 * operator_type is not read.  b, x device vectors of num_free entries; x holds the initial guess. */
int rsd_heat_solve_fem(rsd_ctx* ctx, rsd_heat* h, double c_mass, const rsd_solver_cfg* cfg, const double* b, double* x,
                       rsd_report* report);
/* The LinearSolverRunner HeatProblem::makeLinearRunner builds for OperatorType::FEM with any of the
 * stages' form compositions (SteadyStage.hpp:37, BackwardEulerStage.hpp:43-46): Diffusion
 * + c_tdiff TangentDiffusion + c_mass Mass + c_tmass TangentMass, models at the state U (Full gather)
 * and the rate Udot (TangentMass); U NULL or U == x binds the state to the iterate, as the linear
 * stages do.  Jacobi from the same forms' element diagonal.  cfg as for rsd_heat_solve_fem. */
int rsd_heat_solve_fem_forms(rsd_ctx* ctx, rsd_heat* h, double c_tdiff, double c_mass, double c_tmass, const double* U,
                             const double* Udot, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* report);
/* A flux boundary condition given by one expression per spatial component, q(t, x, y, z), on a
 * boundary tag of any value >= 0 (HeatProblem.tpp:98-105, FluxBoundaryForm); flux_expr NULL clears
 * the tag's flux.
 * The stages then add its integrals to the right-hand side as HeatProblem::applyNatural does. */
int rsd_heat_set_flux(rsd_ctx* ctx, rsd_heat* h, int32_t tag, const char* const* flux_expr);
/* BoundaryApplicator::applyNaturalBCs (fem/boundary/backend/cpu/BoundaryApplicator.tpp:66-140) at the
 * problem's current time: F += sum over flux faces of the integral of (q . n) N_a, scattered Free */
int rsd_apply_natural(rsd_ctx* ctx, rsd_heat* h, double* F);
/* HeatProblem::computeNodalField (application/heateq/problem/HeatProblem.tpp:293-303) through
 * QuantityEvaluator::evaluateNodalField with SimpleAverageRecovery (fem/quantity/backend/cpu/
 * QuantityEvaluator.tpp:205-257): field RSD_FIELD_HEAT_FLUX (HeatFluxField, Q = -k grad T, nsd
 * components per node) or RSD_FIELD_CONDUCTIVITY (ConductivityField, 1 per node) from the free-DOF
 * temperature U (device); out: device, nnodes * components (node-major); scratch: device, nnodes. */
enum { RSD_FIELD_HEAT_FLUX = 0, RSD_FIELD_CONDUCTIVITY = 1 };
int rsd_heat_nodal_field(rsd_ctx* ctx, rsd_heat* h, int32_t field, const double* U, double* out, double* scratch);
/* HeatFlux monitors (MonitorConfig::Quantity::HeatFlux, HeatProblem.tpp:410-440) at the problem's current
 * time, per requested boundary tag:
 *   RSD_FLUX_STRONG: BoundaryQuadratureMonitorGroup with HeatFluxIntegrand
 *     (fem/quantity/BoundaryQuadratureMonitorGroup.hpp, equation/heateq/quantity/HeatFluxIntegrand.hpp):
 *     the sum over the tag's faces and Gauss points of -(K grad T) . n w (n area-scaled);
 *   RSD_FLUX_WEAK: BoundaryReactionMonitorGroup (fem/quantity/BoundaryReactionMonitorGroup.hpp): the
 *     element vectors of source - Diffusion(U) [- rho cp Mass(Udot) when `transient`] summed over the
 *     tag's face nodes (each node once per element and tag, faces in order, as QuantityEvaluator.tpp:92-200).
 * RSD_REDUCE_AVERAGE divides each value by the tag's measure (sum of |n| w).  U (free DOFs, Dirichlet
 * values injected) and Udot are device vectors; values and measures (may be NULL) are host arrays of
 * ntags.  A monitor combination (coefficients times tags, MonitorConfig::terms) is a linear combination
 * of the per-tag values. */
enum { RSD_FLUX_WEAK = 0, RSD_FLUX_STRONG = 1 };
enum { RSD_REDUCE_INTEGRAL = 0, RSD_REDUCE_AVERAGE = 1 };
int rsd_heat_boundary_flux(rsd_ctx* ctx, rsd_heat* h, int32_t method, int32_t reduction, int32_t transient, int32_t ntags,
                           const int32_t* tags, const double* U, const double* Udot, double* values, double* measures);
/* BoundaryApplicator::applyEssentialBCs (fem/boundary/backend/cpu/BoundaryApplicator.tpp:7-64) */
int rsd_apply_dirichlet_lift(rsd_ctx* ctx, rsd_heat* h, double c_diff, double c_mass, double* F);
/* Assembler::assembleDiagonal (Assembler.tpp:142-197) */
int rsd_assemble_diagonal(rsd_ctx* ctx, rsd_heat* h, double c_diff, double c_mass, const double* U, double* d);

/* ---- stages ---- */
/* SteadyStage linear assemble + solve (solver/stage/SteadyStage.hpp:60-84); U device in/out.
 * With cfg->operator_type RSD_OP_FEM the stages assemble no matrix (the stages' needsK() is false
 * for a matrix-free operator) and solve as rsd_heat_solve_fem does. */
int rsd_heat_steady(rsd_ctx* ctx, rsd_heat* h, const rsd_solver_cfg* cfg, double* U, rsd_report* report);
/* BackwardEulerRunner::step over BackwardEulerStage, linear mode
 * (solver/timestepper/BackwardEuler.hpp:32-70, solver/stage/BackwardEulerStage.hpp:71-124):
 * advances h's time by dt from Uprev to U (both device; U holds the warm start on entry), then
 * copies U into Uprev; residual_norm receives the stage's residualNorm() (may be NULL). */
int rsd_heat_be_step(rsd_ctx* ctx, rsd_heat* h, double dt, const rsd_solver_cfg* cfg, double* U, double* Uprev,
                     rsd_report* report, double* residual_norm);
/* The same step for a caller whose state U_host lives in host memory (in: the state to advance from,
 * also the step's previous state; out: the new state): uploaded to device vectors h keeps (allocated
 * on the first call), stepped, and copied back, with one synchronization; the copies overlap the
 * matrix assembly and the residual pass on a second stream.  Pinned host memory gives full-speed
 * copies.  No counterpart in the reference (its CUDA tag keeps vectors on the device). */
int rsd_heat_be_step_host(rsd_ctx* ctx, rsd_heat* h, double dt, const rsd_solver_cfg* cfg, double* U_host,
                          rsd_report* report, double* residual_norm);
/* NewtonRunner::solve over SteadyStage nonlinear mode (solver/nonlinear/Newton.hpp:32-83,
 * solver/stage/SteadyStage.hpp:89-116): R = F - K(T)T, J = K + K_T, J dU = R, U += dU.
 * linear->operator_type RSD_OP_FEM: J is not assembled; each product of the linear solve is an element
 * pass of Diffusion + TangentDiffusion at the Newton state (the reference's FEMOperator over the
 * Jacobian forms), Jacobi from that operator's element diagonal.  With a nonzero dk/dT the Jacobian
 * K + K_T is not symmetric: solve it with GMRES (linear->type RSD_GMRES); CG has no convergence
 * guarantee there and may stop at max_iters unconverged, reported as such. */
int rsd_heat_newton(rsd_ctx* ctx, rsd_heat* h, double abs_tol, double rel_tol, int64_t max_iters,
                    const rsd_solver_cfg* linear, double* U, rsd_report* report);

/* ---- batched solves (no counterpart in the reference, whose solvers take one system): many
 *      independent systems A_i x_i = b_i of any sizes in one persistent launch.  Each CTA takes the
 *      next problem from a device queue (largest first) and runs the whole CG+Jacobi for it.
 *      cfg->type must be RSD_CG; RSD_MIXED gives FP32 inner iterations with FP64 residual
 *      replacement (convergence on the FP64 residual), RSD_FP64 plain FP64 PCG.  The batch keeps
 *      the matrices by reference: they must outlive it and keep their patterns. ---- */
typedef struct rsd_batch rsd_batch;
int rsd_batch_create(rsd_ctx* ctx, int32_t count, rsd_csr* const* A, rsd_batch** out);
int rsd_batch_destroy(rsd_batch* batch);
/* b, x: host arrays of count device pointers (x holds the initial guesses on entry);
 * reports: host array of count reports, or NULL */
int rsd_batch_solve(rsd_ctx* ctx, rsd_batch* batch, const rsd_solver_cfg* cfg, const double* const* b,
                    double* const* x, rsd_report* reports);

/* ---- adjoint pair, in the shape of an autograd Function (no counterpart in the reference) ----
 * Steady linear heat with per-element conductivity k_e = k_const * exp(theta_e) (rsd_heat_desc's
 * k_expr must be unset).  theta: device, one value per element; T, dJdT: device, free DOFs;
 * dJdtheta: device, one value per element.
 * forward:  sets k_e from theta, assembles K(theta), F and the Dirichlet lift, solves K T = F
 *           (T holds the warm start on entry).
 * backward: rebuilds K(theta) (nothing is saved between the calls), solves the adjoint system
 *           K lambda = dJ/dT, and returns dJ/dtheta_e = -k_e * int_e grad(lambda) . grad(T) with T
 *           carrying its Dirichlet values.  For J = 0.5 ||T - T_obs||^2 pass dJdT = T - T_obs. */
int rsd_heat_forward(rsd_ctx* ctx, rsd_heat* h, const double* theta, const rsd_solver_cfg* cfg, double* T,
                     rsd_report* report);
int rsd_heat_backward(rsd_ctx* ctx, rsd_heat* h, const double* theta, const double* T, const double* dJdT,
                      const rsd_solver_cfg* cfg, double* dJdtheta, rsd_report* report);

/* ---- transient adjoint pair, in the shape of an autograd Function (no counterpart in the
 * reference): the linear Backward-Euler steps of rsd_heat_be_step (BackwardEulerStage.hpp:71-124)
 * with k_e = k_const * exp(theta_e), constant cp and the assembled operator.
 * forward:  U = the state after nsteps steps of dt from U0 at time t0 (U0, U device, num_free);
 *           report: iterations summed over the steps, converged if every step converged.
 * backward: dJdtheta (device, one per element) = the gradient of a terminal objective J(U_N) whose
 *           derivative dJdU (device, num_free) is given, by the discrete adjoint of the same steps:
 *           mu_N = A^-1 dJ/dU_N, mu_k = A^-1 M mu_{k+1} / dt with A = K + M/dt, and
 *           dJ/dtheta_e = -k_e sum_k int_e grad mu_k . K0 grad U_k.  The forward states are recomputed,
 *           not kept: every ceil(sqrt(nsteps))-th state is checkpointed and each segment is replayed
 *           from its checkpoint during the reverse sweep, so about 2 sqrt(nsteps) states are held
 *           (states_held, may be NULL) for about nsteps extra forward steps.  report: iterations = the
 *           adjoint solves' total, refinements = the forward solves' total (replays included).
 * The conductivity tensor, if any, must be symmetric (A^T = A); k_expr and cp_expr must be unset. */
int rsd_heat_transient_forward(rsd_ctx* ctx, rsd_heat* h, const double* theta, double t0, double dt, int64_t nsteps,
                               const rsd_solver_cfg* cfg, const double* U0, double* U, rsd_report* report);
int rsd_heat_transient_backward(rsd_ctx* ctx, rsd_heat* h, const double* theta, double t0, double dt, int64_t nsteps,
                                const double* U0, const double* dJdU, const rsd_solver_cfg* cfg, double* dJdtheta,
                                rsd_report* report, int64_t* states_held);

#ifdef __cplusplus
}
#endif
#endif
