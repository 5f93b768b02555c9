// HeatProblem-equivalent object on the device and the stage-level drivers built on it:
// steady linear solve, one Backward-Euler step and the Newton loop.
#include <cmath>
#include <cstring>
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {

int build_tables(rsd_ctx* ctx, rsd_heat* h);
int assemble_lift(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double* F);

static bool uses_time(const DevExpr& e) {
	for (int i = 0; i < e.n; ++i) if (e.op[i] == E_VAR && e.arg[i] == 0) return true;
	return false;
}

// Dirichlet value per constrained node at time t: the constraint tag's expression at the node's
// coordinates, as gatherElementVector evaluates it (fem/assembly/backend/cpu/ElementMap.tpp:55-65)
// g[node] = the Dirichlet expression of the node's constraint (tags[i]: its index into bc) at (t, x)
__global__ void k_bc_values(int64_t nc, const int32_t* __restrict__ nodes, const int32_t* __restrict__ tags,
                            const double* __restrict__ xyz, int nsd, const DevExpr* __restrict__ bc, double t,
                            double* __restrict__ g) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t v = nodes[i];
		const double* x = xyz + (int64_t)v * nsd;
		g[v] = eval_expr(bc[tags[i]], t, x[0], x[1], nsd == 3 ? x[2] : 0.0, 0.0);
	}
}

// gatherElementVector's Dirichlet values (fem/assembly/backend/cpu/ElementMap.tpp:55-65) for every
// constrained node at time t, evaluated on the device into dst (free nodes keep zero); the constrained
// node list and the compiled expressions go to the device on the first call
static int bc_values_to(rsd_ctx* ctx, rsd_heat* h, double t, double* dst) {
	const rsd_mesh* m = h->m;
	if (!h->dBc) {
		std::vector<int32_t> cn, ct;
		for (int64_t i = 0; i < m->nnodes; ++i)
			if (h->h_t2a[i] < 0) { cn.push_back((int32_t)i); ct.push_back(h->h_ctag[i]); }
		h->ncNodes = (int64_t)cn.size();
		const size_t ne = std::max<size_t>(h->bcExpr.size(), 1);
		RSD_CUDA(cudaMalloc(&h->dBc, sizeof(DevExpr) * ne));
		RSD_CUDA(cudaMalloc(&h->cNodes, sizeof(int32_t) * 2 * std::max<int64_t>(h->ncNodes, 1)));
		if (!h->bcExpr.empty())
			RSD_CUDA(cudaMemcpyAsync(h->dBc, h->bcExpr.data(), sizeof(DevExpr) * h->bcExpr.size(), cudaMemcpyHostToDevice, ctx->stream));
		if (h->ncNodes) {
			RSD_CUDA(cudaMemcpyAsync(h->cNodes, cn.data(), sizeof(int32_t) * cn.size(), cudaMemcpyHostToDevice, ctx->stream));
			RSD_CUDA(cudaMemcpyAsync(h->cNodes + h->ncNodes, ct.data(), sizeof(int32_t) * ct.size(), cudaMemcpyHostToDevice, ctx->stream));
		}
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));   // the host lists go out of scope
	}
	if (dst != h->g && dst != h->gPrev) return set_error(RSD_EINVAL, "Dirichlet values go to g or gPrev");
	if (h->ncNodes) {
		k_bc_values<<<vec_grid(ctx, h->ncNodes), 256, 0, ctx->stream>>>(h->ncNodes, h->cNodes, h->cNodes + h->ncNodes,
		                                                                m->xyz, m->nsd, h->dBc, t, dst);
		RSD_CUDA(cudaGetLastError());
	}
	return RSD_OK;
}

int upload_bc_values(rsd_ctx* ctx, rsd_heat* h) { return bc_values_to(ctx, h, h->time, h->g); }

static bool bc_time_dependent(const rsd_heat* h) {
	for (const DevExpr& e : h->bcExpr) if (uses_time(e)) return true;
	return false;
}

static int set_time(rsd_ctx* ctx, rsd_heat* h, double t) {
	const bool changed = t != h->time;
	h->time = t;
	if (changed && bc_time_dependent(h)) return upload_bc_values(ctx, h);
	return RSD_OK;
}

// U[t2a[v]] = f(t, x_v) for every free node v (HeatProblem::loadNodalField, Expression mode)
__global__ void k_eval_nodal(int64_t nn, const int32_t* __restrict__ t2a, const double* __restrict__ xyz, int nsd,
                             const DevExpr f, double t, double* __restrict__ U) {
	for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nn; v += (int64_t)gridDim.x * blockDim.x) {
		const int32_t r = t2a[v];
		if (r < 0) continue;
		const double* x = xyz + v * nsd;
		U[r] = eval_expr(f, t, x[0], nsd > 1 ? x[1] : 0.0, nsd > 2 ? x[2] : 0.0, 0.0);
	}
}

__global__ void k_be_rate(int64_t n, double inv_dt, const double* __restrict__ U, const double* __restrict__ Up, double* __restrict__ Ud) {
	// copy(U, Udot); axpby(-1/dt, 1/dt, Uprev, Udot)  (BackwardEulerStage.hpp:73-74)
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		Ud[i] = inv_dt * U[i] + (-inv_dt) * Up[i];
}
// k_e = exp(theta_e): the per-element conductivity multiplier of the adjoint pair
__global__ void k_exp_theta(int64_t ne, const double* __restrict__ theta, double* __restrict__ kElem) {
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
		kElem[e] = exp(theta[e]);
}
// dJ/dtheta_e = -(dk_e/dtheta_e) * k0 * g_e with dk_e/dtheta_e = k_e and g_e = int_e grad(lambda) . grad(T)
__global__ void k_adjoint_scale(int64_t ne, const double* __restrict__ kElem, double k0, double* __restrict__ g) {
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
		g[e] = -(kElem[e] * k0) * g[e];
}

// acc[e] += g[e]: the transient gradient's sum over steps
__global__ void k_accumulate(int64_t ne, const double* __restrict__ g, double* __restrict__ acc) {
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
		acc[e] += g[e];
}

// |F - R| with the deterministic grid reduction: axpby(1, -1, F, R) then norm(R)
// (BackwardEulerStage.hpp:120-122), without storing F - R
__global__ void k_diff_norm(int64_t n, const double* __restrict__ F, const double* __restrict__ R, double* partials,
                            unsigned* ticket, double* out) {
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double d = -1.0 * R[i] + 1.0 * F[i];
		v[0] += d * d;
	}
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

static void free_heat(rsd_heat* h) {
	cudaFree(h->t2a); cudaFree(h->g); cudaFree(h->kElem); cudaFree(h->tables); cudaFree(h->bElems); cudaFree(h->gPrev);
	cudaFree(h->ranks); cudaFree(h->affine); cudaFree(h->geo); cudaFree(h->ktab); cudaFree(h->adjPtr); cudaFree(h->adj); cudaFree(h->erow); cudaFree(h->dFlux); cudaFree(h->nFaces); cudaFree(h->dBc); cudaFree(h->cNodes);
	cudaFree(h->hostU); cudaFree(h->hostUprev);
	cudaFree(h->F); cudaFree(h->R); cudaFree(h->Udot); cudaFree(h->ms); cudaFree(h->dU);
	if (h->K) rsd_csr_destroy(h->K);
	delete h;
}

}  // namespace rsd

using namespace rsd;

extern "C" {

int rsd_heat_create(rsd_ctx* ctx, const rsd_mesh* m, const rsd_heat_desc* d, rsd_heat** out) {
	if (!ctx || !m || !d || !out) return set_error(RSD_EINVAL, "null argument");
	if (d->nq < 1 || d->nq > 5) return set_error(RSD_EINVAL, "quadrature points per direction must be 1..5 (kMaxQuadraturePoints1D)");
	RSD_CUDA(cudaSetDevice(ctx->device));
	rsd_heat* h = new rsd_heat();
	h->m = m;
	h->nq1 = d->nq;
	h->k_const = d->k_const;
	h->rho = d->rho;
	h->cp = d->cp;
	int rc;
	if ((rc = compile_expr(d->k_expr, &h->kExpr)) || (rc = compile_expr(d->dk_expr, &h->dkExpr)) || (rc = compile_expr(d->src_expr, &h->srcExpr)) ||
	    (rc = compile_expr(d->cp_expr, &h->cpExpr)) || (rc = compile_expr(d->dcp_expr, &h->dcpExpr))) { delete h; return rc; }
	if (d->dcp_expr && !d->cp_expr) { delete h; return set_error(RSD_EINVAL, "dcp_expr given without cp_expr"); }
	if (d->k_tensor) {
		h->aniso = true;
		for (int i = 0; i < 9; ++i) h->kS[i] = 0.0;
		for (int i = 0; i < m->nsd; ++i)
			for (int j = 0; j < m->nsd; ++j) {
				const double v = d->k_tensor[i * m->nsd + j];
				if (!std::isfinite(v)) { delete h; return set_error(RSD_EINVAL, "conductivity tensor entry is not finite"); }
				h->kS[i * 3 + j] = v;
			}
	}
	// essential tags: dirichlet_expr[0..5], then the tag list (a repeated tag keeps its later expression,
	// as the reference evaluates every entry registered on a tag in turn)
	auto add_bc = [&](int32_t tag, const char* src) -> int {
		if (tag < 0) return set_error(RSD_EINVAL, "boundary tags are >= 0");
		DevExpr ex;
		RSD_CHECK(compile_expr(src, &ex));
		for (size_t i = 0; i < h->essTags.size(); ++i)
			if (h->essTags[i] == tag) { h->bcExpr[i] = ex; return RSD_OK; }
		h->essTags.push_back(tag);
		h->bcExpr.push_back(ex);
		return RSD_OK;
	};
	for (int t = 0; t < 6; ++t)
		if (d->dirichlet_expr[t] && (rc = add_bc(t, d->dirichlet_expr[t]))) { delete h; return rc; }
	if (d->num_dirichlet < 0 || (d->num_dirichlet > 0 && (!d->dirichlet_tags || !d->dirichlet_exprs))) { delete h; return set_error(RSD_EINVAL, "bad Dirichlet tag list"); }
	for (int32_t i = 0; i < d->num_dirichlet; ++i) {
		if (!d->dirichlet_exprs[i]) { delete h; return set_error(RSD_EINVAL, "Dirichlet tag without an expression"); }
		if ((rc = add_bc(d->dirichlet_tags[i], d->dirichlet_exprs[i]))) { delete h; return rc; }
	}
	cudaError_t e;
	const int64_t nn = m->nnodes;
	if ((e = cudaMalloc(&h->t2a, sizeof(int32_t) * nn)) != cudaSuccess) { free_heat(h); return cuda_error(e, "dof map allocation"); }
	const bool onDevice = device_setup();
	if (onDevice) {
		if ((rc = device_dofmap(ctx, h))) { free_heat(h); return rc; }
	} else {
		build_dofmap(h);
	}
	const int64_t n = std::max<int64_t>(h->n, 1);
	if ((e = cudaMalloc(&h->g, sizeof(double) * nn)) != cudaSuccess ||
	    (e = cudaMalloc(&h->F, sizeof(double) * n)) != cudaSuccess || (e = cudaMalloc(&h->R, sizeof(double) * n)) != cudaSuccess ||
	    (e = cudaMalloc(&h->Udot, sizeof(double) * n)) != cudaSuccess || (e = cudaMalloc(&h->ms, sizeof(double) * n)) != cudaSuccess ||
	    (e = cudaMalloc(&h->dU, sizeof(double) * n)) != cudaSuccess) {
		free_heat(h);
		return cuda_error(e, "heat problem allocation");
	}
	if (!onDevice && (e = cudaMemcpyAsync(h->t2a, h->h_t2a.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) { free_heat(h); return cuda_error(e, "dof map upload"); }
	if (d->k_elem) {
		if ((e = cudaMalloc(&h->kElem, sizeof(double) * m->nelem)) != cudaSuccess ||
		    (e = cudaMemcpyAsync(h->kElem, d->k_elem, sizeof(double) * m->nelem, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) {
			free_heat(h);
			return cuda_error(e, "element conductivity upload");
		}
	}
	{
		// elements touching a constrained node: the only ones the Dirichlet lift can change
		std::vector<int32_t> be;
		for (int64_t el = 0; el < m->nelem; ++el)
			for (int a = 0; a < m->npe; ++a)
				if (h->h_t2a[m->h_ien[el * m->npe + a]] < 0) { be.push_back((int32_t)el); break; }
		h->nbElems = (int64_t)be.size();
		if (h->nbElems &&
		    ((e = cudaMalloc(&h->bElems, sizeof(int32_t) * be.size())) != cudaSuccess ||
		     (e = cudaMemcpyAsync(h->bElems, be.data(), sizeof(int32_t) * be.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)) {
			free_heat(h);
			return cuda_error(e, "boundary element list");
		}
		if ((e = cudaMalloc(&h->gPrev, sizeof(double) * nn)) != cudaSuccess) { free_heat(h); return cuda_error(e, "allocation"); }
		// Dirichlet values are written for the constrained nodes only: the free nodes' entries stay zero
		if ((e = cudaMemsetAsync(h->g, 0, sizeof(double) * nn, ctx->stream)) != cudaSuccess ||
		    (e = cudaMemsetAsync(h->gPrev, 0, sizeof(double) * nn, ctx->stream)) != cudaSuccess) { free_heat(h); return cuda_error(e, "allocation"); }
	}
	if ((rc = build_tables(ctx, h)) || (rc = upload_bc_values(ctx, h)) || (rc = build_pattern(ctx, h, &h->K))) { free_heat(h); return rc; }
	*out = h;
	return RSD_OK;
}

int rsd_heat_destroy(rsd_heat* h) {
	if (!h) return RSD_OK;
	cudaDeviceSynchronize();
	free_heat(h);
	return RSD_OK;
}

int rsd_heat_info(const rsd_heat* h, int64_t* num_free, int64_t* nnz) {
	if (!h) return set_error(RSD_EINVAL, "null problem");
	if (num_free) *num_free = h->n;
	if (nnz) *nnz = h->K->nnz;
	return RSD_OK;
}

int rsd_heat_dofmap(rsd_ctx* ctx, const rsd_heat* h, int32_t* t2a, int32_t* a2t) {
	(void)ctx;
	if (!h) return set_error(RSD_EINVAL, "null problem");
	if (t2a) std::memcpy(t2a, h->h_t2a.data(), sizeof(int32_t) * h->h_t2a.size());
	if (a2t) std::memcpy(a2t, h->h_a2t.data(), sizeof(int32_t) * h->h_a2t.size());
	return RSD_OK;
}

int rsd_heat_matrix(rsd_heat* h, rsd_csr** A) {
	if (!h || !A) return set_error(RSD_EINVAL, "null argument");
	*A = h->K;
	return RSD_OK;
}

int rsd_heat_create_matrix(rsd_ctx* ctx, rsd_heat* h, rsd_csr** A) {
	if (!ctx || !h || !A) return set_error(RSD_EINVAL, "null argument");
	RSD_CUDA(cudaSetDevice(ctx->device));
	return share_pattern(ctx, h->K, A);
}

int rsd_heat_eval_nodal(rsd_ctx* ctx, rsd_heat* h, const char* expr, double t, double* U) {
	if (!ctx || !h || !expr || (h->n && !U)) return set_error(RSD_EINVAL, "null argument");
	DevExpr f;
	RSD_CHECK(compile_expr(expr, &f));
	const int64_t nn = h->m->nnodes;
	if (nn) {
		k_eval_nodal<<<vec_grid(ctx, nn), 256, 0, ctx->stream>>>(nn, h->t2a, h->m->xyz, h->m->nsd, f, t, U);
		RSD_CUDA(cudaGetLastError());
	}
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_set_time(rsd_ctx* ctx, rsd_heat* h, double t) {
	if (!ctx || !h) return set_error(RSD_EINVAL, "null argument");
	h->time = t;
	return upload_bc_values(ctx, h);
}

int rsd_heat_set_k_elem(rsd_ctx* ctx, rsd_heat* h, const double* k) {
	if (!ctx || !h) return set_error(RSD_EINVAL, "null argument");
	if (!k) { cudaFree(h->kElem); h->kElem = nullptr; return RSD_OK; }
	if (!h->kElem) RSD_CUDA(cudaMalloc(&h->kElem, sizeof(double) * h->m->nelem));
	RSD_CUDA(cudaMemcpyAsync(h->kElem, k, sizeof(double) * h->m->nelem, cudaMemcpyDeviceToDevice, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_assemble_matrix(rsd_ctx* ctx, rsd_heat* h, double cd, double cm, double ct, double ctm, const double* U,
                        const double* Udot, rsd_csr* A) {
	if (!ctx || !h || !A) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(assemble_matrix(ctx, h, cd, cm, ct, ctm, U, Udot, A));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_assemble_vector(rsd_ctx* ctx, rsd_heat* h, int32_t which, double coef, const double* U, const double* Udot,
                        const double* operand, double* out) {
	if (!ctx || !h || !out || which < 0 || (which > 4 && which != 10)) return set_error(RSD_EINVAL, "bad argument");
	RSD_CHECK(assemble_vector(ctx, h, which, coef, U, Udot, operand, out, 1.0, false));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_set_flux(rsd_ctx* ctx, rsd_heat* h, int32_t tag, const char* const* flux_expr) {
	if (!ctx || !h) return set_error(RSD_EINVAL, "null argument");
	return set_flux(ctx, h, tag, flux_expr);
}

int rsd_apply_natural(rsd_ctx* ctx, rsd_heat* h, double* F) {
	if (!ctx || !h || (h->n && !F)) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(apply_natural(ctx, h, F));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_nodal_field(rsd_ctx* ctx, rsd_heat* h, int32_t field, const double* U, double* out, double* scratch) {
	if (!ctx || !h || !out || !scratch || (h->n && !U)) return set_error(RSD_EINVAL, "null argument");
	if (field != RSD_FIELD_HEAT_FLUX && field != RSD_FIELD_CONDUCTIVITY) return set_error(RSD_EINVAL, "unknown nodal field");
	RSD_CHECK(nodal_field(ctx, h, field, U, out, scratch));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_solve_fem(rsd_ctx* ctx, rsd_heat* h, double c_mass, const rsd_solver_cfg* cfg, const double* b, double* x,
                       rsd_report* rep) {
	if (!ctx || !h || !cfg) return set_error(RSD_EINVAL, "null argument");
	return solve_fem(ctx, h, c_mass, cfg, b, x, rep);
}

int rsd_heat_solve_fem_forms(rsd_ctx* ctx, rsd_heat* h, double c_tdiff, double c_mass, double c_tmass, const double* U,
                             const double* Udot, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	if (!ctx || !h || !cfg) return set_error(RSD_EINVAL, "null argument");
	if (!std::isfinite(c_tdiff) || !std::isfinite(c_mass) || !std::isfinite(c_tmass)) return set_error(RSD_EINVAL, "form coefficients must be finite");
	// the state is the iterate itself when none is given or when it is the solution vector (the
	// stages bind the state to the vector the solver updates)
	const double* state = (U == nullptr || U == x) ? nullptr : U;
	if (c_tdiff == 0.0 && c_tmass == 0.0) return solve_fem(ctx, h, c_mass, cfg, b, x, rep, 4, state);
	return solve_fem(ctx, h, c_mass, cfg, b, x, rep, 10, state, c_tdiff, c_tmass, Udot);
}

int rsd_heat_boundary_flux(rsd_ctx* ctx, rsd_heat* h, int32_t method, int32_t reduction, int32_t transient, int32_t ntags,
                           const int32_t* tags, const double* U, const double* Udot, double* values, double* measures) {
	if (!ctx || !h || ntags < 0 || (ntags && (!tags || !values)) || (h->n && !U)) return set_error(RSD_EINVAL, "null argument");
	if (method != RSD_FLUX_WEAK && method != RSD_FLUX_STRONG) return set_error(RSD_EINVAL, "unknown flux evaluation method");
	if (reduction != RSD_REDUCE_INTEGRAL && reduction != RSD_REDUCE_AVERAGE) return set_error(RSD_EINVAL, "unknown monitor reduction");
	if (ntags == 0) return RSD_OK;
	double* d = nullptr;
	RSD_CUDA(cudaMalloc(&d, sizeof(double) * 2 * ntags));
	int rc = boundary_flux(ctx, h, method, ntags, tags, U, Udot, transient != 0, d);
	std::vector<double> hv(2 * ntags, 0.0);
	if (rc == RSD_OK) {
		const cudaError_t e = cudaMemcpy(hv.data(), d, sizeof(double) * 2 * ntags, cudaMemcpyDeviceToHost);
		if (e != cudaSuccess) rc = cuda_error(e, "monitor values");
	}
	cudaFree(d);
	RSD_CHECK(rc);
	for (int t = 0; t < ntags; ++t) {
		const double meas = hv[2 * t + 1];
		values[t] = reduction == RSD_REDUCE_AVERAGE ? hv[2 * t] / meas : hv[2 * t];
		if (measures) measures[t] = meas;
	}
	return RSD_OK;
}

int rsd_apply_dirichlet_lift(rsd_ctx* ctx, rsd_heat* h, double cd, double cm, double* F) {
	if (!ctx || !h || !F) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(assemble_lift(ctx, h, cd, cm, F));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_assemble_diagonal(rsd_ctx* ctx, rsd_heat* h, double cd, double cm, const double* U, double* d) {
	if (!ctx || !h || !d) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(assemble_diagonal(ctx, h, cd, cm, U, d));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

// SteadyStage linear: assemble K, load, lift; solve K U = F (solver/stage/SteadyStage.hpp:60-84)
int rsd_heat_steady(rsd_ctx* ctx, rsd_heat* h, const rsd_solver_cfg* cfg, double* U, rsd_report* rep) {
	if (!ctx || !h || !cfg || !U) return set_error(RSD_EINVAL, "null argument");
	const bool fem = cfg->operator_type == RSD_OP_FEM;   // isSparse() false: no K (SteadyStage.hpp:62-64)
	if (!fem) RSD_CHECK(assemble_matrix(ctx, h, 1.0, 0.0, 0.0, 0.0, U, nullptr, h->K));
	RSD_CHECK(assemble_vector(ctx, h, 0, 0.0, U, nullptr, nullptr, h->F, 1.0, false));
	RSD_CHECK(apply_natural(ctx, h, h->F));                                                  // applyNatural
	RSD_CHECK(assemble_lift(ctx, h, 1.0, 0.0, h->F));
	return fem ? solve_fem(ctx, h, 0.0, cfg, h->F, U, rep) : solve(ctx, h->K, cfg, h->F, U, rep);
}

// one BackwardEulerRunner::step, linear mode (solver/timestepper/BackwardEuler.hpp:32-70 over
// solver/stage/BackwardEulerStage.hpp:71-124)
}  // extern "C" (reopened below)

namespace rsd {
static int ensure_copy_stream(rsd_ctx* ctx) {
	if (ctx->copy) return RSD_OK;
	RSD_CUDA(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
	RSD_CUDA(cudaEventCreateWithFlags(&ctx->copyReady, cudaEventDisableTiming));
	RSD_CUDA(cudaEventCreateWithFlags(&ctx->uploaded, cudaEventDisableTiming));
	return RSD_OK;
}

// BackwardEulerRunner::step on device vectors U, Uprev.  With host_in the state is first uploaded
// into U and Uprev on the second stream, and a matrix that does not depend on the state (no k(T))
// is assembled meanwhile; with host_out the new U is copied to that host buffer on the second stream
// beside the residual pass.  One synchronization at the end.
static int be_step(rsd_ctx* ctx, rsd_heat* h, double dt, const rsd_solver_cfg* cfg, double* U, double* Uprev,
                   rsd_report* rep, double* residual_norm, const double* host_in, double* host_out) {
	const int64_t n = h->n;
	const double t = h->time + dt, inv = 1.0 / dt;
	const int gv = vec_grid(ctx, n);
	if (host_in || host_out) RSD_CHECK(ensure_copy_stream(ctx));
	if (host_in) {
		RSD_CUDA(cudaMemcpyAsync(U, host_in, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->copy));
		RSD_CUDA(cudaMemcpyAsync(Uprev, U, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->copy));
		RSD_CUDA(cudaEventRecord(ctx->uploaded, ctx->copy));
	}
	// K + M/dt reads the state only through k(T); without it, it goes first while the state uploads.
	// A matrix-free operator needs no K (BackwardEulerStage::needsK, BackwardEulerStage.hpp:76-78).
	const bool fem = cfg->operator_type == RSD_OP_FEM;
	const bool early = !fem && host_in && h->kExpr.n == 0 && h->dkExpr.n == 0;
	h->dt = dt;
	RSD_CHECK(set_time(ctx, h, t));
	// Dirichlet values at t - dt for the mass right-hand side (gathered Full at currentTime_ - dt_)
	h->gPrevValid = bc_time_dependent(h);
	if (h->gPrevValid) RSD_CHECK(bc_values_to(ctx, h, t - dt, h->gPrev));
	if (early) RSD_CHECK(assemble_matrix(ctx, h, 1.0, inv, 0.0, 0.0, U, h->Udot, h->K));      // K + M/dt
	if (host_in) RSD_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->uploaded, 0));
	k_be_rate<<<gv, 256, 0, ctx->stream>>>(n, inv, U, Uprev, h->Udot);
	if (!early && !fem) RSD_CHECK(assemble_matrix(ctx, h, 1.0, inv, 0.0, 0.0, U, h->Udot, h->K));    // K + M/dt
	RSD_CHECK(assemble_vector(ctx, h, 7, inv, Uprev, nullptr, nullptr, h->F, 1.0, false));  // load + (1/dt) M Uprev
	RSD_CHECK(apply_natural(ctx, h, h->F));                                                  // applyNatural
	RSD_CHECK(assemble_lift(ctx, h, 1.0, inv, h->F));                                      // F -= (K + M/dt) G
	if (fem) RSD_CHECK(solve_fem(ctx, h, inv, cfg, h->F, U, rep));
	else RSD_CHECK(solve(ctx, h->K, cfg, h->F, U, rep));
	if (host_out) {
		// the new state is final: copy it to the host on the second stream while the residual pass runs
		RSD_CUDA(cudaEventRecord(ctx->copyReady, ctx->stream));
		RSD_CUDA(cudaStreamWaitEvent(ctx->copy, ctx->copyReady, 0));
		RSD_CUDA(cudaMemcpyAsync(host_out, U, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->copy));
	}
	if (residual_norm) {
		// BackwardEulerStage::residualNorm (:113-124) with the Udot of this step's assemble():
		// K U (Full) + M Udot in one element pass, then |F - R|
		RSD_CHECK(assemble_vector(ctx, h, 8, 0.0, U, h->Udot, nullptr, h->R, 1.0, false));
		double* dres = &ctx->s.scal[3].spare1;
		k_diff_norm<<<red_grid(ctx, n), kReduceThreads, 0, ctx->stream>>>(n, h->F, h->R, ctx->s.partials, &ctx->s.scal[3].ticket, dres);
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaMemcpyAsync(ctx->s.hbuf + 8, dres, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	}
	RSD_CUDA(cudaMemcpyAsync(Uprev, U, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));   // advance()
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (host_in || host_out) RSD_CUDA(cudaStreamSynchronize(ctx->copy));
	if (residual_norm) *residual_norm = ctx->s.hbuf[8];
	return RSD_OK;
}
}  // namespace rsd

extern "C" {

int rsd_heat_be_step(rsd_ctx* ctx, rsd_heat* h, double dt, const rsd_solver_cfg* cfg, double* U, double* Uprev,
                     rsd_report* rep, double* residual_norm) {
	if (!ctx || !h || !cfg || !U || !Uprev || !(dt > 0)) return set_error(RSD_EINVAL, "bad argument");
	return be_step(ctx, h, dt, cfg, U, Uprev, rep, residual_norm, nullptr, nullptr);
}

// The same step for a caller whose state lives in host memory: the state is uploaded to device
// vectors the problem keeps (allocated on the first call), the step's previous state is that same
// state (BackwardEulerRunner::step keeps Uprev = U between steps), and the new state is copied back,
// everything on the context stream with one synchronization.  Pinned host memory makes the copies
// run at full link speed.
int rsd_heat_be_step_host(rsd_ctx* ctx, rsd_heat* h, double dt, const rsd_solver_cfg* cfg, double* U_host,
                          rsd_report* rep, double* residual_norm) {
	if (!ctx || !h || !cfg || !U_host || !(dt > 0)) return set_error(RSD_EINVAL, "bad argument");
	const int64_t n = h->n;
	const size_t bytes = sizeof(double) * std::max<int64_t>(n, 1);
	if (!h->hostU) {
		cudaError_t e;
		if ((e = cudaMalloc(&h->hostU, bytes)) != cudaSuccess || (e = cudaMalloc(&h->hostUprev, bytes)) != cudaSuccess) {
			cudaFree(h->hostU);
			h->hostU = nullptr;
			return cuda_error(e, "device state for host-buffer steps");
		}
	}
	return be_step(ctx, h, dt, cfg, h->hostU, h->hostUprev, rep, residual_norm, U_host, U_host);
}

// NewtonRunner::solve over SteadyStage nonlinear mode (solver/nonlinear/Newton.hpp:32-83)
int rsd_heat_newton(rsd_ctx* ctx, rsd_heat* h, double abs_tol, double rel_tol, int64_t max_iters,
                    const rsd_solver_cfg* lin, double* U, rsd_report* rep) {
	if (!ctx || !h || !lin || !U) return set_error(RSD_EINVAL, "bad argument");
	const bool fem = lin->operator_type == RSD_OP_FEM;   // needsJ() false: J is applied, not assembled
	const int64_t n = h->n;
	rsd_report R{};
	double res0 = 0.0;
	for (int64_t it = 0; it < max_iters; ++it) {
		// assembleLoad and assembleResidual (K(T) T, Full gather) in one element pass: R = F - K(T) T
		RSD_CHECK(assemble_vector(ctx, h, 9, 0.0, U, nullptr, nullptr, h->R, 1.0, false));
		RSD_CHECK(apply_natural(ctx, h, h->R));   // F includes the natural boundary terms
		double rr = 0.0;
		RSD_CHECK(dot_device(ctx, n, h->R, h->R, &rr));
		const double res = std::sqrt(rr);
		if (it == 0) res0 = res;
		const double rel = res0 > 0.0 ? res / res0 : 0.0;
		R.iterations = it;
		R.initialResidual = res0; R.finalResidual = res; R.finalResidualRel = rel; R.trueResidualRel = rel;
		if (!std::isfinite(res)) { R.status = RSD_ENAN; break; }
		if (res < abs_tol || rel < rel_tol) { R.converged = 1; break; }
		if (!fem) RSD_CHECK(assemble_matrix(ctx, h, 1.0, 0.0, 1.0, 0.0, U, nullptr, h->K));   // J = K + K_T
		RSD_CUDA(cudaMemsetAsync(h->dU, 0, sizeof(double) * n, ctx->stream));
		rsd_report lr;
		if (fem) RSD_CHECK(solve_fem(ctx, h, 0.0, lin, h->R, h->dU, &lr, 10, U));           // J(U) applied per product
		else RSD_CHECK(solve(ctx, h->K, lin, h->R, h->dU, &lr));
		R.refinements += lr.iterations;                                                      // total inner iterations
		if (!lr.converged) { R.status = lr.status; break; }
		RSD_CHECK(rsd_axpy(ctx, n, 1.0, h->dU, U));                                           // U += dU
		if (it == max_iters - 1) R.iterations = max_iters;
	}
	if (rep) *rep = R;
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

// ---- adjoint pair (no counterpart in the reference; the gradient's element loop follows
// DiffusionForm::computeElementLevelMatrix, equation/heateq/form/DiffusionForm.hpp:11-52) ----
static int adjoint_check(rsd_ctx* ctx, rsd_heat* h, const double* theta, const rsd_solver_cfg* cfg) {
	if (!ctx || !h || !theta || !cfg) return set_error(RSD_EINVAL, "null argument");
	if (h->kExpr.n) return set_error(RSD_EINVAL, "the adjoint pair needs a constant conductivity (k_expr unset)");
	if (h->aniso)
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < i; ++j)
				if (h->kS[i * 3 + j] != h->kS[j * 3 + i])
					return set_error(RSD_EINVAL, "the adjoint pair solves K^T with K: the conductivity tensor must be symmetric");
	if (!h->kElem) RSD_CUDA(cudaMalloc(&h->kElem, sizeof(double) * std::max<int64_t>(h->m->nelem, 1)));
	const int64_t ne = h->m->nelem;
	if (ne) {
		k_exp_theta<<<vec_grid(ctx, ne), 256, 0, ctx->stream>>>(ne, theta, h->kElem);
		RSD_CUDA(cudaGetLastError());
	}
	return RSD_OK;
}

int rsd_heat_forward(rsd_ctx* ctx, rsd_heat* h, const double* theta, const rsd_solver_cfg* cfg, double* T, rsd_report* rep) {
	if (!T) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(adjoint_check(ctx, h, theta, cfg));
	RSD_CHECK(assemble_matrix(ctx, h, 1.0, 0.0, 0.0, 0.0, T, nullptr, h->K));
	RSD_CHECK(assemble_vector(ctx, h, 0, 0.0, T, nullptr, nullptr, h->F, 1.0, false));
	RSD_CHECK(apply_natural(ctx, h, h->F));
	RSD_CHECK(assemble_lift(ctx, h, 1.0, 0.0, h->F));
	RSD_CHECK(solve(ctx, h->K, cfg, h->F, T, rep));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_backward(rsd_ctx* ctx, rsd_heat* h, const double* theta, const double* T, const double* dJdT,
                      const rsd_solver_cfg* cfg, double* dJdtheta, rsd_report* rep) {
	if (!T || !dJdT || !dJdtheta) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(adjoint_check(ctx, h, theta, cfg));
	// K(theta) again (the forward's matrix may have been overwritten since); K is symmetric, so the
	// adjoint system K^T lambda = dJ/dT is solved with the same matrix
	RSD_CHECK(assemble_matrix(ctx, h, 1.0, 0.0, 0.0, 0.0, T, nullptr, h->K));
	const int64_t n = h->n, ne = h->m->nelem;
	double* lam = h->dU;
	RSD_CUDA(cudaMemsetAsync(lam, 0, sizeof(double) * std::max<int64_t>(n, 1), ctx->stream));
	RSD_CHECK(solve(ctx, h->K, cfg, dJdT, lam, rep));
	// g_e = int_e grad(lambda) . grad(T) (T with its Dirichlet values, lambda zero there), then scale
	RSD_CHECK(assemble_vector(ctx, h, 6, 0.0, T, nullptr, lam, dJdtheta, 1.0, false));
	if (ne) {
		k_adjoint_scale<<<vec_grid(ctx, ne), 256, 0, ctx->stream>>>(ne, h->kElem, h->k_const, dJdtheta);
		RSD_CUDA(cudaGetLastError());
	}
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}


}  // extern "C"

// ---- transient adjoint pair (no counterpart in the reference): N Backward-Euler steps of the linear
// stage (BackwardEulerStage.hpp:71-124, BackwardEuler.hpp:32-70) with k_e = k_const exp(theta_e), and
// the gradient of a terminal objective J(U_N) by the discrete adjoint of those steps.  With
// A = K(theta) + M/dt the steps are A U_k = M U_{k-1} / dt + f_k (f_k: load and Dirichlet lift at t_k),
// and only K depends on theta, so with mu_N = A^-1 dJ/dU_N and mu_k = A^-1 M mu_{k+1} / dt
// (A symmetric) dJ/dtheta_e = -k_e sum_k int_e grad(mu_k) . K0 grad(U_k), U_k carrying its Dirichlet
// values at t_k.  The reverse sweep needs U_k in reverse order: the forward sweep keeps every C-th state
// (C = ceil(sqrt N)) and each segment's states are recomputed from its checkpoint when the sweep
// reaches it, so ceil(N / C) + C + 1 states are held instead of N, for about N extra forward steps.
namespace rsd {

static int transient_check(rsd_ctx* ctx, rsd_heat* h, const double* theta, const rsd_solver_cfg* cfg, double dt, int64_t nsteps) {
	RSD_CHECK(adjoint_check(ctx, h, theta, cfg));
	if (h->cpExpr.n) return set_error(RSD_EINVAL, "the transient adjoint pair needs a constant specific heat (cp_expr unset)");
	if (cfg->operator_type != RSD_OP_CSR) return set_error(RSD_EINVAL, "the transient adjoint pair solves with the assembled matrix (operator_type RSD_OP_CSR)");
	if (!(dt > 0) || nsteps < 0) return set_error(RSD_EINVAL, "dt must be > 0 and nsteps >= 0");
	return RSD_OK;
}

// steps first..last-1 -> first+1..last from the state in U (Uprev its copy), times t0 + k dt
static int steps(rsd_ctx* ctx, rsd_heat* h, double t0, double dt, int64_t first, int64_t last, const rsd_solver_cfg* cfg,
                 double* U, double* Uprev, rsd_report* total) {
	for (int64_t k = first; k < last; ++k) {
		h->time = t0 + (double)k * dt;   // be_step advances it and re-evaluates the Dirichlet values
		rsd_report r{};
		RSD_CHECK(be_step(ctx, h, dt, cfg, U, Uprev, &r, nullptr, nullptr, nullptr));
		if (total) {
			total->iterations += r.iterations;
			if (!r.converged) { total->converged = 0; if (r.status != RSD_OK) total->status = r.status; }
		}
	}
	return RSD_OK;
}

}  // namespace rsd

extern "C" {

int rsd_heat_transient_forward(rsd_ctx* ctx, rsd_heat* h, const double* theta, double t0, double dt, int64_t nsteps,
                               const rsd_solver_cfg* cfg, const double* U0, double* U, rsd_report* rep) {
	if (!U0 || !U) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(transient_check(ctx, h, theta, cfg, dt, nsteps));
	const int64_t n = h->n;
	double* Uprev = h->dU;
	RSD_CUDA(cudaMemcpyAsync(U, U0, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
	RSD_CUDA(cudaMemcpyAsync(Uprev, U0, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
	rsd_report total{};
	total.converged = 1;
	RSD_CHECK(steps(ctx, h, t0, dt, 0, nsteps, cfg, U, Uprev, &total));
	if (rep) *rep = total;
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

int rsd_heat_transient_backward(rsd_ctx* ctx, rsd_heat* h, const double* theta, double t0, double dt, int64_t nsteps,
                                const double* U0, const double* dJdU, const rsd_solver_cfg* cfg, double* dJdtheta,
                                rsd_report* rep, int64_t* states_held) {
	if (!U0 || !dJdU || !dJdtheta) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(transient_check(ctx, h, theta, cfg, dt, nsteps));
	const int64_t n = h->n, ne = h->m->nelem, N = nsteps;
	cudaStream_t st = ctx->stream;
	RSD_CUDA(cudaMemsetAsync(dJdtheta, 0, sizeof(double) * std::max<int64_t>(ne, 1), st));
	if (rep) *rep = rsd_report{};
	if (N == 0 || n == 0) {
		if (rep) rep->converged = 1;
		if (states_held) *states_held = 0;
		RSD_CUDA(cudaStreamSynchronize(st));
		return RSD_OK;
	}
	const int64_t C = (int64_t)std::ceil(std::sqrt((double)N));
	const int64_t nseg = (N + C - 1) / C;
	const int64_t ns = (n + 31) & ~int64_t(31);   // 256-byte aligned vectors
	// checkpoints (nseg), one segment (C + 1), the adjoint pair mu / mu_next, the right-hand side, the
	// step's previous state; per element the step's gradient term
	const int64_t nvec = nseg + (C + 1) + 4;
	double* buf = nullptr;
	double* gstep = nullptr;
	RSD_CUDA(cudaMalloc(&buf, sizeof(double) * ns * nvec));
	if (cudaMalloc(&gstep, sizeof(double) * std::max<int64_t>(ne, 1)) != cudaSuccess) {
		cudaFree(buf);
		return set_error(RSD_ENOMEM, "transient adjoint scratch");
	}
	auto run = [&]() -> int {
		double* ck = buf;
		double* seg = ck + ns * nseg;
		double* mu = seg + ns * (C + 1);
		double* muNext = mu + ns;
		double* rhs = muNext + ns;
		double* Uprev = rhs + ns;
		rsd_report fwd{};
		fwd.converged = 1;
		// forward sweep: keep the state at the start of every segment
		double* U = seg;
		RSD_CUDA(cudaMemcpyAsync(U, U0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
		RSD_CUDA(cudaMemcpyAsync(Uprev, U0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
		for (int64_t s = 0; s < nseg; ++s) {
			RSD_CUDA(cudaMemcpyAsync(ck + ns * s, U, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
			if (s + 1 < nseg) RSD_CHECK(steps(ctx, h, t0, dt, s * C, (s + 1) * C, cfg, U, Uprev, &fwd));
		}
		// reverse sweep, segment by segment
		rsd_report adj{};
		adj.converged = 1;
		RSD_CUDA(cudaMemsetAsync(muNext, 0, sizeof(double) * n, st));
		for (int64_t s = nseg - 1; s >= 0; --s) {
			const int64_t start = s * C, len = std::min(C, N - start);
			// seg[j] = U_{start + j}, j = 0..len (recomputed from the checkpoint)
			RSD_CUDA(cudaMemcpyAsync(seg, ck + ns * s, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
			for (int64_t j = 1; j <= len; ++j) {
				double* Uj = seg + ns * j;
				RSD_CUDA(cudaMemcpyAsync(Uj, seg + ns * (j - 1), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
				RSD_CUDA(cudaMemcpyAsync(Uprev, Uj, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
				RSD_CHECK(steps(ctx, h, t0, dt, start + j - 1, start + j, cfg, Uj, Uprev, &fwd));
			}
			// h->K holds A = K + M/dt from the steps just taken (theta is fixed)
			for (int64_t j = len; j >= 1; --j) {
				const int64_t k = start + j;
				const double* b = dJdU;
				if (k < N) {
					// M mu_{k+1} / dt: rho cp Mass on a free vector (zero on the Dirichlet nodes)
					RSD_CHECK(assemble_vector(ctx, h, 3, 0.0, nullptr, muNext, nullptr, rhs, 1.0 / dt, false));
					b = rhs;
				}
				RSD_CUDA(cudaMemcpyAsync(mu, muNext, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));   // warm start
				rsd_report r{};
				RSD_CHECK(solve(ctx, h->K, cfg, b, mu, &r));
				adj.iterations += r.iterations;
				if (!r.converged) { adj.converged = 0; if (r.status != RSD_OK) adj.status = r.status; }
				// int_e grad(mu_k) . K0 grad(U_k) with U_k's Dirichlet values at t_k
				h->time = t0 + (double)k * dt;
				RSD_CHECK(upload_bc_values(ctx, h));
				RSD_CHECK(assemble_vector(ctx, h, 6, 0.0, seg + ns * j, nullptr, mu, gstep, 1.0, false));
				if (ne) k_accumulate<<<vec_grid(ctx, ne), 256, 0, st>>>(ne, gstep, dJdtheta);
				RSD_CUDA(cudaGetLastError());
				std::swap(mu, muNext);
			}
		}
		if (ne) k_adjoint_scale<<<vec_grid(ctx, ne), 256, 0, st>>>(ne, h->kElem, h->k_const, dJdtheta);
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaStreamSynchronize(st));
		if (rep) {
			rep->converged = adj.converged && fwd.converged;
			rep->status = adj.status != RSD_OK ? adj.status : fwd.status;
			rep->iterations = adj.iterations;        // adjoint solves
			rep->refinements = fwd.iterations;       // forward solves, the recomputed segments included
		}
		if (states_held) *states_held = nseg + C + 1;
		return RSD_OK;
	};
	const int rc = run();
	cudaStreamSynchronize(st);
	cudaFree(buf);
	cudaFree(gstep);
	return rc;
}

}  // extern "C"
