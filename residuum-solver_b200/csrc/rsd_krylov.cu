// Krylov solvers on the device: PCG (FP64, and FP32-inner with FP64 reliable updates) and
// restarted right-preconditioned GMRES(m) with modified Gram-Schmidt.
//
// PCG keeps every scalar (alpha, beta, r.z, |r|) in device memory: each iteration is three
// kernels on one stream (SpMV + p.Ap, update + r.r/r.z, p update), each grid reduction finishing
// in its last block, so no iteration waits on the host.  The host only polls the done flag once
// per chunk of iterations; kernels of an already-finished solve return immediately.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {

namespace {

struct CgScal {
	double rz, pAp, alpha, beta, res0, res, rel, rmax, res64, trueRel;
	int64_t iter, refinements;
	int32_t done, converged, reliable, apply_xy, status, pad;
	unsigned ticket;
};
static_assert(sizeof(CgScal) <= sizeof(DevScalars), "CgScal must fit a DevScalars slot");
static CgScal* scal_slot(rsd_ctx* ctx, int k) { return reinterpret_cast<CgScal*>(&ctx->s.scal[k]); }

__device__ __forceinline__ bool is_done(const CgScal* S) { return *((volatile const int32_t*)&S->done) != 0; }

// ---- FP64 PCG: linalg/solver/iterative/cg/Solver.tpp:13-119 ----------------------------------
// r = b - A x; z = M r; p = z; rz = r.z; res0 = |r|   (Solver.tpp:31-63)
template <int L>
__global__ void __launch_bounds__(256) k_cg_init(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                 const double* __restrict__ x, double* __restrict__ r, double* __restrict__ p,
                                                 const double* __restrict__ invD, CgScal* S, double* partials, double tol,
                                                 int relMode, int64_t maxIters) {
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[2] = {0.0, 0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double ax = row_dot<L, double, double>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) {
			const double ri = ldh(b + row, pol.first) + (-1.0) * ax;
			const double zi = invD ? ri * ldh(invD + row, pol.first) : ri;
			sth(r + row, ri, pol.first);
			sth(p + row, zi, pol.last);
			v[0] += ri * ri;
			v[1] += ri * zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res0 = sqrt(v[0]);
		S->res0 = res0; S->rz = v[1]; S->iter = 0; S->res = res0; S->rel = 1.0;
		S->refinements = 0; S->reliable = 0; S->apply_xy = 0; S->status = 0;
		const double crit = relMode ? res0 / (res0 + 1e-50) : res0;
		if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (maxIters <= 1) { S->done = 1; S->converged = 0; S->iter = maxIters; S->rel = res0 / (res0 + 1e-50); }
		else { S->done = 0; S->converged = 0; }
	}
}

// Ap = A p; alpha = rz / p.Ap   (Solver.tpp:69-73)
template <int L>
__global__ void __launch_bounds__(256) k_cg_spmv_dot(int64_t n, MatView<double> A, const double* __restrict__ p,
                                                     double* __restrict__ Ap, CgScal* S, double* partials) {
	if (is_done(S)) return;
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[1] = {0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double s = row_dot<L, double, double>(A, p, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) { sth(Ap + row, s, pol.first); v[0] += ldh(p + row, pol.last) * s; }
	}
	if (grid_sum<1>(v, partials, &S->ticket)) {
		S->pAp = v[0];
		S->alpha = S->rz / v[0];
		if (!isfinite(S->alpha)) { S->done = 1; S->converged = 0; S->status = RSD_EBREAKDOWN; }
	}
}

// x += alpha p; r -= alpha Ap; res = |r|; convergence; z = M r; beta = r.z_new / r.z  (Solver.tpp:74-106)
__global__ void __launch_bounds__(256) k_cg_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                   const double* __restrict__ p, const double* __restrict__ Ap,
                                                   const double* __restrict__ invD, CgScal* S, double* partials, double tol,
                                                   int relMode, int64_t maxIters) {
	if (is_done(S)) return;
	const double alpha = S->alpha;
	const L2Pol pol = make_l2pol();
	double v[2] = {0.0, 0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		sth(x + i, ldh_rw(x + i, pol.first) + alpha * ldh(p + i, pol.first), pol.first);
		const double ri = ldh_rw(r + i, pol.first) + (-alpha) * ldh(Ap + i, pol.first);
		sth(r + i, ri, pol.first);
		const double zi = invD ? ri * ldh(invD + i, pol.first) : ri;
		v[0] += ri * ri;
		v[1] += ri * zi;
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const int64_t k = S->iter + 1;
		const double res = sqrt(v[0]);
		const double rel = res / (S->res0 + 1e-50);
		S->res = res; S->rel = rel; S->iter = k;
		const double crit = relMode ? rel : res;
		if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; }
		else if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (k + 1 >= maxIters) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->beta = v[1] / S->rz; S->rz = v[1]; }
	}
}

// p = beta p + z   (Solver.tpp:103-104: scal then axpy)
__global__ void __launch_bounds__(256) k_cg_pupdate(int64_t n, double* __restrict__ p, const double* __restrict__ r,
                                                    const double* __restrict__ invD, const CgScal* S) {
	if (is_done(S)) return;
	const double beta = S->beta;
	const L2Pol pol = make_l2pol();
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double ri = ldh(r + i, pol.first);
		const double zi = invD ? ri * ldh(invD + i, pol.first) : ri;
		sth(p + i, ldh_rw(p + i, pol.first) * beta + 1.0 * zi, pol.last);   // the next SpMV gathers p
	}
}

// ---- mixed precision PCG: FP32 matrix, vectors and recurrence; FP64 x, reductions and residual
// replacement (reliable updates, Sleijpen & van der Vorst 1996): whenever the FP32 recurrence
// residual drops by `delta` since the last replacement, or claims convergence, the true residual
// r = b - A64 (x + y) is recomputed in FP64 and replaces the recurrence residual; the FP32
// correction y is folded into x.  Convergence is declared on the FP64 residual only.
// r0 = b - A64 x in FP64
template <int L>
__global__ void __launch_bounds__(256) k_mx_init(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                 const double* __restrict__ x, float* __restrict__ r, float* __restrict__ p,
                                                 float* __restrict__ y, const float* __restrict__ invD, CgScal* S,
                                                 double* partials, double tol, int relMode, int64_t maxIters) {
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[2] = {0.0, 0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double ax = row_dot<L, double, double>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) {
			const double r64 = ldh(b + row, pol.first) - ax;
			const float ri = (float)r64;
			const float zi = invD ? ri * ldh(invD + row, pol.first) : ri;
			sth(r + row, ri, pol.first); sth(p + row, zi, pol.last); sth(y + row, 0.0f, pol.first);
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res0 = sqrt(v[0]);
		S->res0 = res0; S->rmax = res0; S->res = res0; S->res64 = res0; S->rel = 1.0; S->trueRel = 1.0;
		S->rz = v[1]; S->iter = 0; S->refinements = 0; S->reliable = 0; S->apply_xy = 0; S->status = 0;
		const double crit = relMode ? res0 / (res0 + 1e-50) : res0;
		if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (maxIters <= 1) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->done = 0; S->converged = 0; }
	}
}

template <int L>
__global__ void __launch_bounds__(256) k_mx_spmv_dot(int64_t n, MatView<float> A, const float* __restrict__ p,
                                                     float* __restrict__ Ap, CgScal* S, double* partials) {
	if (is_done(S)) return;
	if (blockIdx.x == 0 && threadIdx.x == 0) { S->reliable = 0; S->apply_xy = 0; }
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[1] = {0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const float s = row_dot<L, float, float>(A, p, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) { sth(Ap + row, s, pol.first); v[0] += (double)ldh(p + row, pol.last) * (double)s; }
	}
	if (grid_sum<1>(v, partials, &S->ticket)) {
		S->pAp = v[0];
		S->alpha = S->rz / v[0];
		if (!isfinite(S->alpha)) { S->done = 1; S->converged = 0; S->status = RSD_EBREAKDOWN; }
	}
}

__global__ void __launch_bounds__(256) k_mx_update(int64_t n, float* __restrict__ y, float* __restrict__ r,
                                                   const float* __restrict__ p, const float* __restrict__ Ap,
                                                   const float* __restrict__ invD, CgScal* S, double* partials, double tol,
                                                   int relMode, int64_t maxIters, double delta) {
	if (is_done(S)) return;
	const float alpha = (float)S->alpha;
	const L2Pol pol = make_l2pol();
	double v[2] = {0.0, 0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		sth(y + i, ldh_rw(y + i, pol.first) + alpha * ldh(p + i, pol.first), pol.first);
		const float ri = ldh_rw(r + i, pol.first) - alpha * ldh(Ap + i, pol.first);
		sth(r + i, ri, pol.first);
		const float zi = invD ? ri * ldh(invD + i, pol.first) : ri;
		v[0] += (double)ri * (double)ri;
		v[1] += (double)ri * (double)zi;
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const int64_t k = S->iter + 1;
		const double res = sqrt(v[0]);
		S->res = res; S->iter = k;
		const double crit = relMode ? res / (S->res0 + 1e-50) : res;
		if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; return; }
		if (crit < tol || res < delta * S->rmax || k + 1 >= maxIters) {
			S->reliable = 1;                    // FP64 residual replacement next
		} else {
			S->beta = v[1] / S->rz; S->rz = v[1];
		}
	}
}

// reliable update: r64 = b - A64 (x + y), r = (float) r64, rz with the new r
template <int L>
__global__ void __launch_bounds__(256) k_mx_reliable(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                     const double* __restrict__ x, const float* __restrict__ y,
                                                     float* __restrict__ r, const float* __restrict__ invD, CgScal* S,
                                                     double* partials, double tol, int relMode, int64_t maxIters) {
	if (is_done(S) || !*((volatile const int32_t*)&S->reliable)) return;
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[2] = {0.0, 0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double s = row_sum<L, double, double>(A, row, n, rl.lane, pol,
		                                            [&](int c) { return ldh(x + c, pol.last) + (double)ldh(y + c, pol.last); });
		if (rl.lane == 0 && row < n) {
			const double r64 = ldh(b + row, pol.first) - s;
			const float ri = (float)r64;
			const float zi = invD ? ri * ldh(invD + row, pol.first) : ri;
			sth(r + row, ri, pol.first);
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res = sqrt(v[0]);
		const double rel = res / (S->res0 + 1e-50);
		S->res64 = res; S->trueRel = rel; S->rmax = res; S->res = res; S->rel = rel;
		S->refinements += 1;
		S->apply_xy = 1;
		const double crit = relMode ? rel : res;
		if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; }
		else if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (S->iter + 1 >= maxIters) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->beta = v[1] / S->rz; S->rz = v[1]; }
	}
}

// fold y into x after a replacement; p = beta p + z
__global__ void __launch_bounds__(256) k_mx_pupdate(int64_t n, double* __restrict__ x, float* __restrict__ y,
                                                    float* __restrict__ p, const float* __restrict__ r,
                                                    const float* __restrict__ invD, const CgScal* S) {
	const int apply = *((volatile const int32_t*)&S->apply_xy);
	const int done = is_done(S);
	if (!apply && done) return;
	const float beta = (float)S->beta;
	const L2Pol pol = make_l2pol();
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		if (apply) {
			sth(x + i, ldh_rw(x + i, pol.first) + (double)ldh_rw(y + i, pol.first), pol.first);
			sth(y + i, 0.0f, pol.first);
		}
		if (!done) {
			const float ri = ldh(r + i, pol.first);
			const float zi = invD ? ri * ldh(invD + i, pol.first) : ri;
			sth(p + i, ldh_rw(p + i, pol.first) * beta + zi, pol.last);   // the next SpMV gathers p
		}
	}
}

__global__ void k_invdiag32(int64_t n, const int32_t* __restrict__ dpos, const double* __restrict__ val, float* __restrict__ d) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t q = dpos[i];
		const double v = q >= 0 ? val[q] : 0.0;
		d[i] = (float)((fabs(v) > 1e-300) ? 1.0 / v : 1.0);
	}
}
__global__ void k_invdiag64(int64_t n, const int32_t* __restrict__ dpos, const double* __restrict__ val, double* __restrict__ d) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t q = dpos[i];
		const double v = q >= 0 ? val[q] : 0.0;
		d[i] = (fabs(v) > 1e-300) ? 1.0 / v : 1.0;
	}
}

// ||b - A x|| in FP64 (device scalar)
template <int L>
__global__ void __launch_bounds__(256) k_true_res(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                  const double* __restrict__ x, double* partials, unsigned* ticket, double* out) {
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[1] = {0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double ax = row_dot<L, double, double>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) { const double ri = ldh(b + row, pol.first) - ax; v[0] += ri * ri; }
	}
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

// ---- workspace -------------------------------------------------------------------------------
struct Workspace {
	void* base = nullptr;
	size_t bytes = 0;
	int device = -1;
};
static Workspace g_ws[16];

static int get_ws(rsd_ctx* ctx, size_t bytes, void** out) {
	Workspace& w = g_ws[ctx->device & 15];
	if (w.bytes < bytes || w.device != ctx->device) {
		if (w.base) { cudaStreamSynchronize(ctx->stream); cudaFree(w.base); w.base = nullptr; w.bytes = 0; }
		RSD_CUDA(cudaMalloc(&w.base, bytes));
		w.bytes = bytes;
		w.device = ctx->device;
	}
	*out = w.base;
	return RSD_OK;
}

static int row_blocks(const rsd_ctx* ctx, int64_t n, int L, int block = 256) {
	int64_t b = (n * std::max(L, 1) + block - 1) / block;
	b = std::min<int64_t>(b, std::min<int64_t>(kMaxPartials, (int64_t)ctx->num_sms * (2048 / block)));
	return (int)std::max<int64_t>(b, 1);
}
static int vec_blocks(const rsd_ctx* ctx, int64_t n) {
	int64_t b = (n + 255) / 256;
	b = std::min<int64_t>(b, std::min<int64_t>(kMaxPartials, (int64_t)ctx->num_sms * 8));
	return (int)std::max<int64_t>(b, 1);
}

static int finish_report(rsd_ctx* ctx, CgScal* S, rsd_report* rep) {
	CgScal h;
	RSD_CUDA(cudaMemcpyAsync(&h, S, sizeof(CgScal), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (rep) {
		rep->converged = h.converged;
		rep->status = h.status;
		rep->iterations = h.iter;
		rep->initialResidual = h.res0;
		rep->finalResidual = h.res;
		rep->finalResidualRel = h.res / (h.res0 + 1e-50);
		rep->refinements = h.refinements;
		rep->trueResidualRel = h.trueRel;
	}
	return RSD_OK;
}

// launches issued after the solve finished returned immediately: drop them from the timing
static void discard_idle(rsd_ctx* ctx, const std::vector<int>& pairs, int per_iter, int64_t iters) {
	for (size_t k = (size_t)std::max<int64_t>(iters, 0) * per_iter; k < pairs.size(); ++k) ctx->prof.fam[pairs[k]] = -1;
}

// poll the done flag of an iteration chunk without stalling the launch pipeline
struct Poller {
	rsd_ctx* ctx;
	CgScal* S;
	int32_t* hflag;
	cudaEvent_t ev[2];
	int k = 0;
	bool pending[2] = {false, false};
	int init() {
		RSD_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
		RSD_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
		return RSD_OK;
	}
	~Poller() { cudaEventDestroy(ev[0]); cudaEventDestroy(ev[1]); }
	// enqueue a flag read behind the chunk just launched; returns true once an earlier chunk saw done
	int post(bool* finished) {
		const int slot = k & 1;
		RSD_CUDA(cudaMemcpyAsync(&hflag[slot], &S->done, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaEventRecord(ev[slot], ctx->stream));
		pending[slot] = true;
		const int prev = slot ^ 1;
		*finished = false;
		if (pending[prev]) {
			RSD_CUDA(cudaEventSynchronize(ev[prev]));
			pending[prev] = false;
			*finished = hflag[prev] != 0;
		}
		++k;
		return RSD_OK;
	}
};

static int cg_fp64(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	RSD_CHECK(exec_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	void* wsv;
	RSD_CHECK(get_ws(ctx, sizeof(double) * (4 * n + 64), &wsv));
	double* r = (double*)wsv;
	double* p = r + n;
	double* Ap = p + n;
	double* invD = cfg->precond == RSD_JACOBI ? Ap + n : nullptr;
	CgScal* S = scal_slot(ctx, 0);
	RSD_CUDA(cudaMemsetAsync(S, 0, sizeof(CgScal), ctx->stream));
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	const int gr = row_blocks(ctx, n, L), gv = vec_blocks(ctx, n);
	// Jacobi::update on every solve (cg/Solver.tpp:22)
	if (invD) k_invdiag64<<<gv, 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
	RSD_DISPATCH_L(L, (k_cg_init<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, r, p, invD, S, ctx->s.partials, cfg->tol, rel, cfg->max_iters)));
	RSD_CUDA(cudaGetLastError());
	Poller poll{ctx, S, (int32_t*)ctx->s.hbuf};
	RSD_CHECK(poll.init());
	const int chunk = 8;
	bool fin = false;
	std::vector<int> pairs;
	for (int64_t it = 0; it < cfg->max_iters + 2 * chunk && !fin; it += chunk) {
		for (int c = 0; c < chunk; ++c) {
			int pr = prof_begin(ctx, PF_SPMV_DOT_F64);
			RSD_DISPATCH_L(L, (k_cg_spmv_dot<LL><<<gr, 256, 0, ctx->stream>>>(n, V, p, Ap, S, ctx->s.partials)));
			prof_end(ctx, pr);
			int pu = prof_begin(ctx, PF_CG_UPDATE);
			k_cg_update<<<gv, 256, 0, ctx->stream>>>(n, x, r, p, Ap, invD, S, ctx->s.partials, cfg->tol, rel, cfg->max_iters);
			prof_end(ctx, pu);
			int pp = prof_begin(ctx, PF_CG_PUPDATE);
			k_cg_pupdate<<<gv, 256, 0, ctx->stream>>>(n, p, r, invD, S);
			prof_end(ctx, pp);
			if (pr >= 0) { pairs.push_back(pr); pairs.push_back(pu); pairs.push_back(pp); }
		}
		RSD_CUDA(cudaGetLastError());
		RSD_CHECK(poll.post(&fin));
	}
	RSD_CHECK(finish_report(ctx, S, rep));
	discard_idle(ctx, pairs, 3, rep ? rep->iterations : 0);
	// FP64 check of the final iterate: ||b - A x|| / ||r0||
	double* tr = &scal_slot(ctx, 1)->res;
	RSD_DISPATCH_L(L, (k_true_res<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, ctx->s.partials, &scal_slot(ctx, 1)->ticket, tr)));
	RSD_CUDA(cudaGetLastError());
	double h = 0.0;
	RSD_CUDA(cudaMemcpyAsync(&h, tr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (rep) rep->trueResidualRel = h / (rep->initialResidual + 1e-50);
	return RSD_OK;
}

static int cg_mixed(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	RSD_CHECK(f32_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	const MatView<float> V32 = view32(A);
	void* wsv;
	RSD_CHECK(get_ws(ctx, sizeof(float) * (5 * n + 64), &wsv));
	float* r = (float*)wsv;
	float* p = r + n;
	float* Ap = p + n;
	float* y = Ap + n;
	float* invD = cfg->precond == RSD_JACOBI ? y + n : nullptr;
	CgScal* S = scal_slot(ctx, 0);
	RSD_CUDA(cudaMemsetAsync(S, 0, sizeof(CgScal), ctx->stream));
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	const double delta = cfg->reliable_delta > 0 ? cfg->reliable_delta : 0.1;
	const int gr = row_blocks(ctx, n, L), gv = vec_blocks(ctx, n);
	if (invD) k_invdiag32<<<gv, 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
	RSD_DISPATCH_L(L, (k_mx_init<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, r, p, y, invD, S, ctx->s.partials, cfg->tol, rel, cfg->max_iters)));
	RSD_CUDA(cudaGetLastError());
	Poller poll{ctx, S, (int32_t*)ctx->s.hbuf};
	RSD_CHECK(poll.init());
	const int chunk = 8;
	bool fin = false;
	std::vector<int> pairs;
	for (int64_t it = 0; it < cfg->max_iters + 2 * chunk && !fin; it += chunk) {
		for (int c = 0; c < chunk; ++c) {
			int pr = prof_begin(ctx, PF_SPMV_DOT_F32);
			RSD_DISPATCH_L(L, (k_mx_spmv_dot<LL><<<gr, 256, 0, ctx->stream>>>(n, V32, p, Ap, S, ctx->s.partials)));
			prof_end(ctx, pr);
			int pu = prof_begin(ctx, PF_CG_UPDATE);
			k_mx_update<<<gv, 256, 0, ctx->stream>>>(n, y, r, p, Ap, invD, S, ctx->s.partials, cfg->tol, rel, cfg->max_iters, delta);
			prof_end(ctx, pu);
			int pq = prof_begin(ctx, PF_RELIABLE);
			RSD_DISPATCH_L(L, (k_mx_reliable<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, y, r, invD, S, ctx->s.partials, cfg->tol, rel, cfg->max_iters)));
			prof_end(ctx, pq);
			int pp = prof_begin(ctx, PF_CG_PUPDATE);
			k_mx_pupdate<<<gv, 256, 0, ctx->stream>>>(n, x, y, p, r, invD, S);
			prof_end(ctx, pp);
			if (pr >= 0) { pairs.push_back(pr); pairs.push_back(pu); pairs.push_back(pq); pairs.push_back(pp); }
		}
		RSD_CUDA(cudaGetLastError());
		RSD_CHECK(poll.post(&fin));
	}
	RSD_CHECK(finish_report(ctx, S, rep));
	discard_idle(ctx, pairs, 4, rep ? rep->iterations : 0);
	if (rep) { rep->finalResidual = rep->trueResidualRel * rep->initialResidual; rep->finalResidualRel = rep->trueResidualRel; }
	return RSD_OK;
}

// ---- GMRES(m): linalg/solver/iterative/gmres/Solver.tpp:3-170 ---------------------------------
// Device: SpMV, preconditioner, the MGS dot/axpy pairs (each h_ij stays on the device), norms and
// scalings.  Host: the (m+1) x m Hessenberg, Givens rotations and back substitution, as the
// reference keeps them (gmres/Workspace.hpp:26-31); one column is read back per Arnoldi step.
__global__ void k_dot_to(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* partials,
                         unsigned* ticket, double* out, int sqrtOut) {
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) v[0] += a[i] * b[i];
	if (grid_sum<1>(v, partials, ticket)) *out = sqrtOut ? sqrt(v[0]) : v[0];
}
// w += (-h) q, h read from the device
__global__ void k_axpy_neg_dev(int64_t n, const double* __restrict__ h, const double* __restrict__ q, double* __restrict__ w) {
	const double a = -(*h);
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) w[i] += a * q[i];
}
// q = w * (1/hn) unless breakdown (hn <= 1e-14)
__global__ void k_scale_copy(int64_t n, const double* __restrict__ w, const double* __restrict__ hn, double* __restrict__ q) {
	const double h = *hn;
	if (h <= 1e-14) return;
	const double s = 1.0 / h;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) q[i] = w[i] * s;
}
__global__ void k_prec(int64_t n, const double* __restrict__ invD, const double* __restrict__ r, double* __restrict__ z) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) z[i] = invD ? r[i] * invD[i] : r[i];
}
__global__ void k_resid(int64_t n, const double* __restrict__ b, const double* __restrict__ Ax, double* __restrict__ r) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) r[i] = b[i] + (-1.0) * Ax[i];
}
__global__ void k_scal_dev(int64_t n, double a, double* __restrict__ x) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] *= a;
}
// z = sum_i y_i Q_i (accumulated in basis order, as the reference's axpy sequence)
__global__ void k_combine(int64_t n, int m, const double* __restrict__ Q, const double* __restrict__ yv, double* __restrict__ z) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		double s = 0.0;
		for (int k = 0; k < m; ++k) s += yv[k] * Q[(int64_t)k * n + i];
		z[i] = s;
	}
}

static int gmres_fp64(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	const int64_t m = std::max<int64_t>(1, cfg->krylov_dim);
	void* wsv;
	RSD_CHECK(get_ws(ctx, sizeof(double) * ((m + 4) * n + 4 * (m + 2) + 64), &wsv));
	double* Q = (double*)wsv;
	double* w = Q + (m + 1) * n;
	double* z = w + n;
	double* invD = cfg->precond == RSD_JACOBI ? z + n : nullptr;
	double* dH = z + 2 * n;          // device column buffer: h_0..h_{j+1}, plus y
	double* dY = dH + (m + 2);
	const int gv = vec_blocks(ctx, n), grd = red_grid(ctx, n);
	unsigned* ticket = &scal_slot(ctx, 2)->ticket;
	const bool relMode = cfg->tol_type == RSD_TOL_RELATIVE;
	const double breakdownTol = 1e-14, eps = 1e-50;
	std::vector<double> H((m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), yv(m), col(m + 2);
	auto Hat = [&](int64_t i, int64_t j) -> double& { return H[j * (m + 1) + i]; };
	RSD_CHECK(exec_sync(ctx, A));
	if (invD) k_invdiag64<<<gv, 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
	auto residual = [&](double* beta) -> int {
		RSD_CHECK(spmv_f64(ctx, A, x, w));
		k_resid<<<gv, 256, 0, ctx->stream>>>(n, b, w, Q);
		k_dot_to<<<grd, kReduceThreads, 0, ctx->stream>>>(n, Q, Q, ctx->s.partials, ticket, dH, 1);
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaMemcpyAsync(ctx->s.hbuf, dH, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		*beta = ctx->s.hbuf[0];
		return RSD_OK;
	};
	double res0;
	RSD_CHECK(residual(&res0));
	auto converged = [&](double res) { return (relMode ? res / (res0 + eps) : res) < cfg->tol; };
	rsd_report R{};
	R.initialResidual = res0;
	if (converged(res0)) {
		R.converged = 1; R.finalResidual = res0; R.finalResidualRel = 1.0; R.iterations = 0; R.trueResidualRel = res0 / (res0 + eps);
		if (rep) *rep = R;
		return RSD_OK;
	}
	int64_t total = 0;
	double beta = res0;
	while (total < cfg->max_iters) {
		k_scal_dev<<<gv, 256, 0, ctx->stream>>>(n, 1.0 / beta, Q);
		g[0] = beta;
		for (int64_t i = 1; i <= m; ++i) g[i] = 0.0;
		int64_t mLocal = 0;
		bool breakdown = false;
		for (int64_t j = 0; j < m; ++j) {
			double* qj = Q + j * n;
			k_prec<<<gv, 256, 0, ctx->stream>>>(n, invD, qj, z);
			RSD_CHECK(spmv_f64(ctx, A, z, w));
			for (int64_t i = 0; i <= j; ++i) {
				k_dot_to<<<grd, kReduceThreads, 0, ctx->stream>>>(n, Q + i * n, w, ctx->s.partials, ticket, dH + i, 0);
				k_axpy_neg_dev<<<gv, 256, 0, ctx->stream>>>(n, dH + i, Q + i * n, w);
			}
			k_dot_to<<<grd, kReduceThreads, 0, ctx->stream>>>(n, w, w, ctx->s.partials, ticket, dH + j + 1, 1);
			k_scale_copy<<<gv, 256, 0, ctx->stream>>>(n, w, dH + j + 1, Q + (j + 1) * n);
			RSD_CUDA(cudaGetLastError());
			RSD_CUDA(cudaMemcpyAsync(col.data(), dH, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, ctx->stream));
			RSD_CUDA(cudaStreamSynchronize(ctx->stream));
			for (int64_t i = 0; i <= j; ++i) Hat(i, j) = col[i];
			const double hNext = col[j + 1];
			++total;
			breakdown = hNext <= breakdownTol;
			for (int64_t i = 0; i < j; ++i) {
				const double h1 = Hat(i, j), h2 = Hat(i + 1, j);
				Hat(i, j) = cs[i] * h1 + sn[i] * h2;
				Hat(i + 1, j) = -sn[i] * h1 + cs[i] * h2;
			}
			const double hjj = Hat(j, j);
			const double denom = std::sqrt(hjj * hjj + hNext * hNext);
			if (denom <= breakdownTol) { cs[j] = 1.0; sn[j] = 0.0; }
			else { cs[j] = hjj / denom; sn[j] = hNext / denom; }
			Hat(j, j) = cs[j] * hjj + sn[j] * hNext;
			const double gj = g[j];
			g[j] = cs[j] * gj;
			g[j + 1] = -sn[j] * gj;
			mLocal = j + 1;
			if (!std::isfinite(g[j + 1])) { R.status = RSD_EBREAKDOWN; break; }
			if (converged(std::fabs(g[j + 1])) || breakdown || total >= cfg->max_iters) break;
		}
		for (int64_t ii = 0; ii < mLocal; ++ii) {
			const int64_t i = mLocal - 1 - ii;
			double s = g[i];
			for (int64_t k = i + 1; k < mLocal; ++k) s -= Hat(i, k) * yv[k];
			yv[i] = s / Hat(i, i);
		}
		RSD_CUDA(cudaMemcpyAsync(dY, yv.data(), sizeof(double) * mLocal, cudaMemcpyHostToDevice, ctx->stream));
		k_combine<<<gv, 256, 0, ctx->stream>>>(n, (int)mLocal, Q, dY, z);
		k_prec<<<gv, 256, 0, ctx->stream>>>(n, invD, z, w);
		RSD_CHECK(rsd_axpy(ctx, n, 1.0, w, x));
		RSD_CHECK(residual(&beta));
		if (R.status || converged(beta) || breakdown || total >= cfg->max_iters) break;
	}
	R.converged = R.status ? 0 : converged(beta);
	R.finalResidual = beta;
	R.finalResidualRel = beta / (res0 + eps);
	R.iterations = total;
	R.trueResidualRel = beta / (res0 + eps);
	if (rep) *rep = R;
	return RSD_OK;
}

// ---- FP64 PCG over a static device scratch ---------------------------------------------------
// The same kernels, grids and reductions as cg_fp64 (so the same iterates, bit for bit), with every
// scratch buffer carved from one file-scope device array instead of the context's workspace: the
// call allocates nothing.  The array is sized for kStaticMaxRows rows; one array per device, shared
// by every call on that device.
constexpr int64_t kStaticMaxRows = int64_t(1) << 18;                 // 262,144 rows
constexpr size_t kStaticHeadBytes = 2 * sizeof(DevScalars) + sizeof(double) * 2 * kMaxPartials;
constexpr size_t kStaticHeadAligned = (kStaticHeadBytes + 255) & ~size_t(255);
constexpr size_t kStaticScratchBytes = kStaticHeadAligned + sizeof(double) * 4 * kStaticMaxRows;   // 8 MiB + 19 KiB
static_assert(sizeof(DevScalars) % 8 == 0, "the partials after the two scalar slots stay 8-byte aligned");

}  // namespace

static __device__ __align__(256) unsigned char g_cg_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kStaticMaxDevices = 64;
static std::mutex g_static_mu;
static void* g_static_ptr[kStaticMaxDevices];

// device address of this device's scratch, looked up once per device
static int static_scratch(rsd_ctx* ctx, unsigned char** out) {
	if (ctx->device < 0 || ctx->device >= kStaticMaxDevices) return set_error(RSD_EINVAL, "device index out of range for the static scratch table");
	std::lock_guard<std::mutex> lk(g_static_mu);
	if (!g_static_ptr[ctx->device]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_cg_static_scratch);
		if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(static CG scratch)");
		g_static_ptr[ctx->device] = p;
	}
	*out = (unsigned char*)g_static_ptr[ctx->device];
	return RSD_OK;
}

static int cg_fp64_static(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	unsigned char* base = nullptr;
	RSD_CHECK(static_scratch(ctx, &base));
	CgScal* S = reinterpret_cast<CgScal*>(base);
	CgScal* S1 = reinterpret_cast<CgScal*>(base + sizeof(DevScalars));
	double* partials = reinterpret_cast<double*>(base + 2 * sizeof(DevScalars));
	double* r = reinterpret_cast<double*>(base + kStaticHeadAligned);
	double* p = r + n;
	double* Ap = p + n;
	double* invD = cfg->precond == RSD_JACOBI ? Ap + n : nullptr;
	// the reduction tickets and the done/converged flags must start at zero on every call
	RSD_CUDA(cudaMemsetAsync(base, 0, 2 * sizeof(DevScalars), ctx->stream));
	RSD_CHECK(exec_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	const int gr = row_blocks(ctx, n, L), gv = vec_blocks(ctx, n);
	if (invD) k_invdiag64<<<gv, 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
	RSD_DISPATCH_L(L, (k_cg_init<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, r, p, invD, S, partials, cfg->tol, rel, cfg->max_iters)));
	RSD_CUDA(cudaGetLastError());
	const int chunk = 8;
	for (int64_t it = 0; it < cfg->max_iters + 2 * chunk; it += chunk) {
		for (int c = 0; c < chunk; ++c) {
			RSD_DISPATCH_L(L, (k_cg_spmv_dot<LL><<<gr, 256, 0, ctx->stream>>>(n, V, p, Ap, S, partials)));
			k_cg_update<<<gv, 256, 0, ctx->stream>>>(n, x, r, p, Ap, invD, S, partials, cfg->tol, rel, cfg->max_iters);
			k_cg_pupdate<<<gv, 256, 0, ctx->stream>>>(n, p, r, invD, S);
		}
		RSD_CUDA(cudaGetLastError());
		int32_t done = 0;   // pageable host word: the copy returns once the flag has been read
		RSD_CUDA(cudaMemcpyAsync(&done, &S->done, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		if (done) break;
	}
	RSD_CHECK(finish_report(ctx, S, rep));
	double* tr = &S1->res;
	RSD_DISPATCH_L(L, (k_true_res<LL><<<gr, 256, 0, ctx->stream>>>(n, V, b, x, partials, &S1->ticket, tr)));
	RSD_CUDA(cudaGetLastError());
	double h = 0.0;
	RSD_CUDA(cudaMemcpyAsync(&h, tr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (rep) rep->trueResidualRel = h / (rep->initialResidual + 1e-50);
	return RSD_OK;
}

}  // namespace

int solve(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	if (!ctx || !A || !cfg || (A->n && (!b || !x))) return set_error(RSD_EINVAL, "null argument");
	if (cfg->max_iters < 0 || !(cfg->tol >= 0)) return set_error(RSD_EINVAL, "bad solver configuration");
	if (rep) *rep = rsd_report{};
	if (A->n == 0) { if (rep) rep->converged = 1; return RSD_OK; }
	RSD_CUDA(cudaSetDevice(ctx->device));
	if (cfg->type == RSD_CG) return cfg->precision == RSD_MIXED ? cg_mixed(ctx, A, cfg, b, x, rep) : cg_fp64(ctx, A, cfg, b, x, rep);
	if (cfg->type == RSD_GMRES) {
		if (cfg->krylov_dim <= 0) return set_error(RSD_EINVAL, "GMRES needs krylov_dim >= 1");
		return gmres_fp64(ctx, A, cfg, b, x, rep);
	}
	return set_error(RSD_EINVAL, "unknown solver type");
}

}  // namespace rsd

extern "C" int rsd_solve(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	return rsd::solve(ctx, A, cfg, b, x, rep);
}

extern "C" int rsd_cg_solve_static(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x,
                                   rsd_report* rep) {
	using namespace rsd;
	if (!ctx || !A || !cfg || (A->n && (!b || !x))) return set_error(RSD_EINVAL, "null argument");
	if (cfg->type != RSD_CG || cfg->precision != RSD_FP64)
		return set_error(RSD_EINVAL, "rsd_cg_solve_static runs FP64 CG only (type RSD_CG, precision RSD_FP64)");
	if (cfg->max_iters < 0 || !(cfg->tol >= 0)) return set_error(RSD_EINVAL, "bad solver configuration");
	if (A->n > kStaticMaxRows) {
		char msg[160];
		snprintf(msg, sizeof msg, "rsd_cg_solve_static: %lld rows exceed the static scratch limit of %lld rows",
		         (long long)A->n, (long long)kStaticMaxRows);
		return set_error(RSD_EINVAL, msg);
	}
	if (rep) *rep = rsd_report{};
	if (A->n == 0) { if (rep) rep->converged = 1; return RSD_OK; }
	RSD_CUDA(cudaSetDevice(ctx->device));
	return cg_fp64_static(ctx, A, cfg, b, x, rep);
}
