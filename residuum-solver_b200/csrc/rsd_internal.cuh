// Internal declarations shared by the sm_100a translation units of librsd_cuda.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rsd.h"

namespace rsd {

// ---------------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);

#define RSD_CUDA(call)                                                   \
	do {                                                                 \
		cudaError_t e_ = (call);                                         \
		if (e_ != cudaSuccess) return ::rsd::cuda_error(e_, #call);      \
	} while (0)

#define RSD_CHECK(expr)                      \
	do {                                     \
		int rc_ = (expr);                    \
		if (rc_ != RSD_OK) return rc_;       \
	} while (0)

// ---------------------------------------------------------------------------------------------
// launch geometry: B200 has 148 SMs; grids are sized as multiples of the SM count
// ---------------------------------------------------------------------------------------------
constexpr int kReduceThreads = 256;
constexpr int kMaxPartials = 148 * 8;   // one partial per block of a reduction grid

// device scalars of one reduction / Krylov iteration (kept on the device, read by the next kernel)
struct DevScalars {
	double rz, pAp, alpha, beta, rr, res0, res, rzNew;
	double rel, spare0, spare1, spare2;
	int32_t done, converged, status, pad;
	int64_t iter;
	uint32_t ticket;      // last-block-done counter (reset by the last block)
	uint32_t ticket2;
};

struct rsd_scratch {
	double* partials = nullptr;    // kMaxPartials * 4 doubles
	DevScalars* scal = nullptr;    // device scalars
	DevScalars* hscal = nullptr;   // pinned host mirror
	double* hbuf = nullptr;        // pinned host staging (64 doubles)
};

}  // namespace rsd

namespace rsd {
// per-kernel-family launch timing with CUDA events on the context stream (off by default)
enum ProfFamily { PF_SPMV_DOT_F64, PF_SPMV_DOT_F32, PF_CG_UPDATE, PF_CG_PUPDATE, PF_RELIABLE, PF_ASM_MATRIX,
                  PF_ASM_VECTOR, PF_SPMV, PF_CG_PERSIST, PF_COUNT };
struct Profiler {
	bool on = false;
	std::vector<cudaEvent_t> pool;
	std::vector<int> fam;          // family of each recorded pair
	size_t used = 0;               // events in use (pairs * 2)
	int64_t launches[PF_COUNT] = {};
	double total_ms[PF_COUNT] = {};
};
}  // namespace rsd

struct rsd_ctx {
	int device = 0;
	int num_sms = 148;
	cudaStream_t stream = nullptr;
	cudaStream_t copy = nullptr;       // second stream: D2H of a step's state beside its residual pass (lazy)
	cudaEvent_t copyReady = nullptr, uploaded = nullptr;
	rsd::rsd_scratch s;
	rsd::Profiler prof;
	void* graphs = nullptr;        // cached CG solve graphs (rsd_krylov.cu)
	void* ws = nullptr;            // Krylov workspace of this context (grow-only)
	size_t wsBytes = 0;
};

namespace rsd {
// bracket one launch: prof_begin returns the pair index or -1 when profiling is off
int prof_begin(rsd_ctx* ctx, int family);
void prof_end(rsd_ctx* ctx, int pair);
int prof_flush(rsd_ctx* ctx);   // fold recorded pairs into the totals (synchronizes the stream)
}  // namespace rsd

// A CSR matrix (the API's storage, CSRMatrix's layout with 32-bit indices) plus its SELL-32
// execution layout: rows in slices of 32, each slice padded to its longest row rounded up to even
// and stored as column-major pairs, so that each lane reads two consecutive entries of its row in
// one load, a warp's loads are contiguous and consecutive rows' gathers of x are neighbours.  Entry
// j of row i lives at sStart[i/32] + 64 (j/2) + 2 (i%32) + j%2; padding has value 0 and repeats a
// column of the row.  Values may be current in either layout (csrValid/sellValid).
struct rsd_csr {
	int64_t n = 0, nnz = 0;
	int32_t* rowPtr = nullptr;     // n+1
	int32_t* col = nullptr;        // nnz
	double* val = nullptr;         // nnz
	int32_t* diag = nullptr;       // n: position of the diagonal entry or -1
	// SELL-32
	int64_t nslices = 0, ssize = 0;
	int32_t* sStart = nullptr;     // nslices+1
	int32_t* sCol = nullptr;       // ssize
	double* sVal = nullptr;        // ssize
	int32_t* sSrc = nullptr;       // ssize: CSR position of the slot, -1 for padding
	int32_t* sDiag = nullptr;      // n: slot of the diagonal entry or -1
	// narrow columns: sBase[s] + sCol16[slot] == sCol[slot], present when every slice's columns
	// lie within 65,535 of its smallest (then the SELL kernels read 2 instead of 4 bytes per slot)
	uint16_t* sCol16 = nullptr;    // ssize
	int32_t* sBase = nullptr;      // nslices
	// stencil slices: sUni[s] >= 0 when the 32 rows of slice s share one pattern of column offsets,
	// sOffs[sUni[s] + j] = column - row of entry j; the slice's columns are then not read
	int32_t* sUni = nullptr;       // nslices (or null when no slice qualifies)
	int32_t* sOffs = nullptr;      // distinct patterns, concatenated
	int64_t nStencil = 0;          // slices stored as stencil slices
	// row order of the slices: slot row r of the layout holds matrix row sPerm[r] (rows of one column
	// pattern grouped within windows, so that slices pad less and share stencil patterns), sIperm
	// the inverse; both null when slot row r is row r
	int32_t* sPerm = nullptr;      // n
	int32_t* sIperm = nullptr;     // n
	// mirrored stencil slices (symmetric matrices): slice s reads its first sNeg[s] entries (the
	// negative offsets o) from the mirror rows r + o, entry sMk[sMir[s] + j] of their slice; 0 reads the
	// slice whole.  Used while symVersion == version (values assembled symmetric to the last bit).
	int32_t* sNeg = nullptr;       // nslices (or null)
	int32_t* sMir = nullptr;       // nslices
	uint8_t* sMk = nullptr;        // mirrored entries, concatenated
	int64_t nMirrored = 0;         // slices that read mirrored entries
	uint64_t symVersion = 0;       // value version known symmetric (0: none)
	bool csrValid = true, sellValid = false;
	int format = 0;                // SpMV layout: 0 SELL-32 (narrow columns when present), 1 CSR vector with `lanes` lanes per row
	int lanes = 0;                 // CSR SpMV lanes per row (0: default from nnz/row)
	int block = 0;                 // SpMV threads per block (0: default)
	bool owns_pattern = true;
	uint64_t version = 1;          // bumped whenever the FP64 values may have changed
	// FP32 copy of the values for the mixed-precision path, in the layout `fmt32` (lazily created)
	float* val32 = nullptr;        // max(ssize, nnz)
	int fmt32 = -1;
	uint64_t version32 = 0;        // FP64 version the FP32 copy was made from
};

namespace rsd {
int sell_sync(rsd_ctx* ctx, rsd_csr* A);     // SELL values current (from CSR if needed)
int csr_sync(rsd_ctx* ctx, rsd_csr* A);      // CSR values current (from SELL if needed)
int f32_sync(rsd_ctx* ctx, rsd_csr* A);      // FP32 copy current, in the execution layout
void free_graph_cache(rsd_ctx* ctx);         // release the context's cached solve graphs
int exec_sync(rsd_ctx* ctx, rsd_csr* A);     // FP64 values current in the execution layout
int share_pattern(rsd_ctx* ctx, const rsd_csr* src, rsd_csr** out);   // src's pattern, own zero values
}  // namespace rsd

namespace rsd {

// ---------------------------------------------------------------------------------------------
// expressions: host compiler + device stack machine (bytecode shared by every kernel)
// ---------------------------------------------------------------------------------------------
constexpr int kExprMax = 48;
constexpr int kExprStack = 16;   // evaluation stack of the device machine
enum ExprOp : int8_t { E_CONST, E_VAR, E_ADD, E_SUB, E_MUL, E_DIV, E_POW, E_NEG, E_SIN, E_COS, E_TAN, E_EXP, E_LOG, E_SQRT, E_ABS };
struct DevExpr {
	int32_t n = 0;          // 0: expression absent
	int32_t depth = 0;      // evaluation stack depth the program needs (at most kExprStack)
	int8_t op[kExprMax];
	int8_t arg[kExprMax];   // variable index (t x y z T) for E_VAR, constant slot for E_CONST
	double c[kExprMax];
};
int compile_expr(const char* src, DevExpr* out);
double eval_expr_host(const DevExpr& e, double t, double x, double y, double z, double T);

// ---------------------------------------------------------------------------------------------
// reductions and vector kernels (rsd_blas.cu)
// ---------------------------------------------------------------------------------------------
int reduce_grid(rsd_ctx* ctx, int64_t n);
int dot_device(rsd_ctx* ctx, int64_t n, const double* x, const double* y, double* host_out);
int spmv_f64(rsd_ctx* ctx, const rsd_csr* A, const double* x, double* y);
int spmv_f32(rsd_ctx* ctx, const rsd_csr* A, const float* x, float* y);
int build_diag_index(rsd_ctx* ctx, rsd_csr* A);
int default_lanes(const rsd_csr* A);

// ---------------------------------------------------------------------------------------------
// Krylov (rsd_krylov.cu)
// ---------------------------------------------------------------------------------------------
int solve(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep);

}  // namespace rsd

// ---------------------------------------------------------------------------------------------
// mesh and heat problem (rsd_core.cu / rsd_assemble.cu / rsd_heat.cu)
// ---------------------------------------------------------------------------------------------
struct rsd_mesh {
	int32_t nsd = 0, order = 0, npe = 0, nfaces = 0;
	int64_t nnodes = 0, nelem = 0;
	std::vector<double> h_xyz;
	std::vector<int32_t> h_ien;     // element-major, 32-bit
	std::vector<int32_t> h_rng;
	double* xyz = nullptr;          // device, node-major (x,y[,z])
	int32_t* ien = nullptr;         // device, element-major
};

struct rsd_heat {
	const rsd_mesh* m = nullptr;
	int32_t nq1 = 2;                // Gauss points per direction
	double k_const = 1.0, rho = 1.0, cp = 1.0;
	rsd::DevExpr kExpr, dkExpr, srcExpr;
	rsd::DevExpr cpExpr, dcpExpr;   // cp(T), dcp/dT (SpecificHeatModel, TemperatureDependent)
	bool aniso = false;             // K = k * kS (ConductivityModel, Anisotropic): kS nsd x nsd row-major
	double kS[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
	// essential boundary tags (any value >= 0) and their Dirichlet expressions, in registration order
	std::vector<int32_t> essTags;
	std::vector<rsd::DevExpr> bcExpr;
	std::vector<int32_t> h_t2a, h_a2t;
	std::vector<int32_t> h_ctag;     // per node: index into essTags / bcExpr of its constraint, -1 if free
	int64_t n = 0;
	int32_t* t2a = nullptr;         // device, per node (-1: constrained)
	double* g = nullptr;            // device, Dirichlet value per node at the current time
	double* kElem = nullptr;        // device, per element (or null)
	double* tables = nullptr;       // device: N, dNdxi, w per quadrature point
	int nq = 0;                     // total quadrature points
	double time = 0.0;
	rsd_csr* K = nullptr;           // matrix with the problem's pattern
	int32_t* bElems = nullptr;      // device: elements with at least one constrained node (lift)
	int64_t nbElems = 0;
	double* gPrev = nullptr;        // device: Dirichlet values at the previous time (time-dependent BCs)
	bool gPrevValid = false;
	uint8_t* ranks = nullptr;       // device: element -> column-rank map for K's pattern
	bool slotsTried = false;
	// affine elements (constant Jacobian): flag per element, and the reference-element integrals
	// [NT + 1][npe][npe] of the gradient products and of the mass (NT = 3 in 2D, 6 in 3D)
	uint8_t* affine = nullptr;      // device, per element
	double* geo = nullptr;          // device, 8 per element: table coefficients (6), |J|, 0
	bool affineTried = false, anyAffine = false, allAffine = false;
	double* ktab = nullptr;         // device
	// row -> (element, local node) adjacency of the free rows, element order (row-gather assembly)
	int32_t* adjPtr = nullptr;      // device, n + 1
	int32_t* adj = nullptr;         // device, e * npe + a
	int32_t* erow = nullptr;        // device, [e][a]: t2a[ien[e][a]] (sum-factorized operator products), or null
	// flux boundary conditions: tag -> one expression per spatial component (three slots per tag)
	std::vector<int32_t> fluxTags;
	std::vector<rsd::DevExpr> fluxExpr;
	rsd::DevExpr* dFlux = nullptr;  // device copy of fluxExpr
	int32_t* nFaces = nullptr;      // device: (element, face, flux index) of the faces whose tag carries a flux
	int64_t nnFaces = 0;
	rsd::DevExpr* dBc = nullptr;    // device copy of bcExpr
	int32_t* cNodes = nullptr;      // device: the constrained nodes, then their bcExpr indices
	int64_t ncNodes = 0;
	bool adjTried = false;
	int32_t maxSlice = 0;           // longest SELL-32 slice of K, in entries per row
	// stage scratch
	double *F = nullptr, *R = nullptr, *Udot = nullptr, *ms = nullptr, *dU = nullptr;
	double *hostU = nullptr, *hostUprev = nullptr;   // device state of rsd_heat_be_step_host
	double dt = 0.0;
};

namespace rsd {
int build_dofmap(rsd_heat* h);
int face_nodes(int nsd, int p, int f, int* out);      // element-local nodes of face f (getFaceNodes order)
bool device_setup();                                  // DOF map and pattern on the device (RSD_HOST_SETUP=1: host)
int device_dofmap(rsd_ctx* ctx, rsd_heat* h);         // needs h->t2a allocated
int device_pattern(rsd_ctx* ctx, const rsd_heat* h, std::vector<int32_t>& rp, std::vector<int32_t>& col, bool* fallback);
int build_pattern(rsd_ctx* ctx, const rsd_heat* h, rsd_csr** out);
int upload_bc_values(rsd_ctx* ctx, rsd_heat* h);
int assemble_matrix(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double cTDiff, double cTMass,
                    const double* U, const double* Udot, rsd_csr* A);
int assemble_vector(rsd_ctx* ctx, rsd_heat* h, int which, double coef, const double* U, const double* Udot,
                    const double* operand, double* out, double outScale, bool accumulate);
int assemble_diagonal(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, const double* U, double* d,
                      double cTDiff = 0.0, double cTMass = 0.0, const double* Udot = nullptr);
int assemble_lift(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double* F);
// which 4: Diffusion + coef Mass (the stages' operator); 10: Diffusion + cTDiff TangentDiffusion + coef Mass
// + cTMass TangentMass (the Jacobian), both with the state U read through k(T), cp(T), dk/dT and grad T,
// and the rate Udot read by TangentMass
int apply_operator(rsd_ctx* ctx, rsd_heat* h, double coef, const double* U, const double* V, double* out,
                   const int32_t* skip, int which = 4, double cTDiff = 1.0, double cTMass = 0.0,
                   const double* Udot = nullptr);
int set_flux(rsd_ctx* ctx, rsd_heat* h, int tag, const char* const* exprs);
int apply_natural(rsd_ctx* ctx, rsd_heat* h, double* F);
int nodal_field(rsd_ctx* ctx, rsd_heat* h, int field, const double* U, double* out, double* scratch);
int boundary_flux(rsd_ctx* ctx, rsd_heat* h, int method, int ntags, const int32_t* tags, const double* U, const double* Udot,
                  bool transient, double* out);
// state null: the iterate x is the state (the stages' linear solves); which, cTDiff, cTMass and Udot as
// for apply_operator
int solve_fem(rsd_ctx* ctx, rsd_heat* h, double coef, const rsd_solver_cfg* cfg, const double* b, double* x,
              rsd_report* rep, int which = 4, const double* state = nullptr, double cTDiff = 1.0,
              double cTMass = 0.0, const double* Udot = nullptr);
int build_tables(rsd_ctx* ctx, rsd_heat* h);
}  // namespace rsd
