/* Test infrastructure, not product code.
 *
 * Plain-C CPU restatement of the Residuum heat-equation hot path, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU legs to check the CUDA backend.  Every function
 * cites the reference file:line it restates (paths relative to the reference checkout).
 *
 * Parity pins: tests/test_oracle_cpu.py checks this restatement against the reference's own
 * known-answer tests and against oracle/_ref (the reference templates compiled unmodified).
 */
#ifndef RSD_ORACLE_H
#define RSD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* mesh::Data (include/mesh/Data.hpp:13-35): xyz node-major, ien element-major, rng per face */
typedef struct ro_mesh {
	int32_t nsd, order;
	int64_t nnodes, nelem;
	int32_t npe, nfaces;
	double* xyz;
	int64_t* ien;
	int32_t* rng;
} ro_mesh;

/* BlockMesh2D/3D::generate (src/mesh/generator/BlockMesh2D.cpp:6-117, BlockMesh3D.cpp:6-139) */
int ro_mesh_block(int32_t nsd, const int32_t* nel, const double* lo, const double* hi, int32_t order, ro_mesh* m);
void ro_mesh_free(ro_mesh* m);

/* problem description: models, forms and boundary data, expression strings in the reference's
 * exprtk syntax (numbers, t x y z T, pi, + - * / ^, unary -, sin cos tan exp log sqrt abs) */
typedef struct ro_model {
	int32_t nq;               /* Gauss points per direction */
	const char* k_expr;       /* k(T); NULL: constant k_const */
	const char* dk_expr;      /* dk/dT(T); NULL: 0 */
	double k_const;
	const double* k_elem;     /* per-element conductivity multiplier or NULL */
	double rho, cp;
	const char* src_expr;     /* f(t,x,y,z); NULL: 0 */
	const char* bc_expr[6];   /* Dirichlet value per boundary tag; NULL: tag not essential */
} ro_model;

typedef struct ro_report {
	int32_t converged;
	int64_t iterations;
	double initialResidual, finalResidual, finalResidualRel;
} ro_report;

typedef struct ro_problem ro_problem;

ro_problem* ro_problem_create(const ro_mesh* m, const ro_model* model);
void ro_problem_destroy(ro_problem* p);
const char* ro_last_error(void);
int64_t ro_num_free(const ro_problem* p);
int64_t ro_nnz(const ro_problem* p);
void ro_dofmap(const ro_problem* p, int32_t* t2a, int32_t* a2t, int32_t* ctag);
void ro_pattern(const ro_problem* p, int64_t* rowPtr, int64_t* col);
void ro_set_time(ro_problem* p, double t);
void ro_bc_node_values(const ro_problem* p, double* g);

/* element loops */
void ro_assemble_matrix(ro_problem* p, double cDiff, double cMass, double cTDiff, double cTMass,
                        const double* U, const double* Udot, double* val);
void ro_assemble_vector(ro_problem* p, int32_t which, double coef, const double* U, const double* Udot,
                        const double* operand, double* out);
void ro_lift(ro_problem* p, double cDiff, double cMass, double* F);
int ro_set_flux(ro_problem* p, int32_t tag, const char* const* exprs);
void ro_natural(ro_problem* p, double* F);
void ro_nodal_field(ro_problem* p, int32_t field, const double* U, double* out);
void ro_diagonal(ro_problem* p, double cDiff, double cMass, const double* U, double* d);
void ro_adjoint_gradient(ro_problem* p, const double* T, const double* lam, double* grad);

/* linear algebra */
void ro_spmv(int64_t n, const int64_t* rowPtr, const int64_t* col, const double* val, const double* x, double* y);
int ro_csr_solve(int32_t solverType, int32_t precond, int64_t n, const int64_t* rowPtr, const int64_t* col,
                 const double* val, const double* b, double* x, double tol, int64_t maxit, int64_t krylov,
                 ro_report* rep);

/* the matrix-free operator (LinearSolverConfig operator type "fem"): CG over element-pass products */
int ro_fem_solve(ro_problem* p, double coef, int32_t precond, const double* b, double* x, double tol, int64_t maxit,
                 ro_report* rep);
/* 0: the stages solve with the assembled matrix (CSR); 1: with the matrix-free operator (CG only) */
void ro_set_operator(ro_problem* p, int32_t op);

/* stages */
int ro_steady(ro_problem* p, int32_t solverType, int32_t precond, double tol, int64_t maxit, int64_t krylov,
              double* U, ro_report* rep);
int ro_backward_euler(ro_problem* p, double dt, int64_t nsteps, int32_t solverType, int32_t precond, double tol,
                      int64_t maxit, int64_t krylov, double* U, double* resPerStep, int64_t* itersPerStep);
int ro_newton(ro_problem* p, double absTol, double relTol, int64_t maxit, int32_t solverType, int32_t precond,
              double tol, int64_t linMaxit, int64_t krylov, double* U, ro_report* rep);

/* expression evaluation (exposed for parser cross-checks) */
int ro_expr_eval(const char* src, double t, double x, double y, double z, double T, double* out);

#ifdef __cplusplus
}
#endif
#endif
