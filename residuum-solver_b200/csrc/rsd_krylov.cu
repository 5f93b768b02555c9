// Krylov solvers on the device: PCG (FP64, and FP32-inner with FP64 reliable updates) and
// restarted right-preconditioned GMRES(m) with classical Gram-Schmidt applied twice.
//
// PCG keeps every scalar (alpha, beta, r.z, |r|) in device memory: an FP64 iteration is three
// kernels on one stream (SpMV + p.Ap, update + r.r/r.z, p update), a mixed one two (SpMV + z.Az,
// then one vector pass of the single-reduction form), each grid reduction finishing in its last
// block, so no iteration waits on the host.  A solve is one CUDA graph (a device-side WHILE loop);
// with plain launches the host polls the done flag once per chunk of iterations, and kernels of an
// already-finished solve return immediately.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <mutex>
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {

namespace {

// threads per block of the CG SpMV+dot kernels and of the vector update kernels; each block ends
// with one ticket atomic of the grid reduction, so fewer, larger blocks shorten the reduction tail
// (measured on the 128^3 system: 512 / 1024 gave 3% on the solve over 256 / 256)
constexpr int kST = 512;
constexpr int kVT = 1024;

struct CgScal {
	double rz, pAp, alpha, beta, res0, res, rhoPrev, rmax, res64, trueRel;   // mixed: rhoPrev = previous r.z
	double dcur;                      // mixed: current replacement threshold
	int64_t iter;
	int32_t refinements, done, converged, reliable, status, pad0, pad;
	unsigned ticket;
};
static_assert(sizeof(CgScal) <= sizeof(DevScalars), "CgScal must fit a DevScalars slot");
static CgScal* scal_slot(rsd_ctx* ctx, int k) { return reinterpret_cast<CgScal*>(&ctx->s.scal[k]); }

__device__ __forceinline__ bool is_done(const CgScal* S) { return *((volatile const int32_t*)&S->done) != 0; }

// Graph mode: the whole solve is one CUDA graph whose iterations run under a conditional WHILE node
// (and, for mixed precision, the FP64 residual replacement under a nested IF node).  The kernels
// steer both from the device: the p-update sets the WHILE condition from the done flag, the update
// sets the IF condition from the replacement flag.  `limit` bounds the body executions of one launch
// (max_iters plus slack) so that the loop ends even if no kernel ever declared the solve done.
struct GraphCtl {
	unsigned long long hw, hr;   // cudaGraphConditionalHandle of the WHILE and IF nodes
	int32_t on, limit;
};

__device__ __forceinline__ void graph_continue(CgScal* S, const GraphCtl& gc) {
	const int32_t bodies = S->pad + 1;   // body executions in this launch (pad starts at zero)
	S->pad = bodies;
	bool go = !is_done(S);
	if (go && bodies >= gc.limit) {
		S->done = 1; S->converged = 0; S->status = RSD_ETIMEOUT;
		go = false;
	}
	cudaGraphSetConditional(gc.hw, go ? 1u : 0u);
}

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
			const int64_t i = mat_row(A, row);
			const double ri = ldh(b + i, pol.first) + (-1.0) * ax;
			const double zi = invD ? ri * ldh(invD + i, pol.last) : ri;
			sth(r + i, ri, pol.last);
			sth(p + i, zi, pol.last);
			v[0] += ri * ri;
			v[1] += ri * zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res0 = sqrt(v[0]);
		S->res0 = res0; S->rz = v[1]; S->iter = 0; S->res = res0;
		S->refinements = 0; S->reliable = 0; S->status = 0;
		const double crit = relMode ? res0 / (res0 + 1e-50) : res0;
		if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (maxIters <= 1) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->done = 0; S->converged = 0; }
	}
}

// Ap = A p; alpha = rz / p.Ap   (Solver.tpp:69-73)
template <int L>
__global__ void __launch_bounds__(kST, kRowBlocks) k_cg_spmv_dot(int64_t n, MatView<double> A, const double* __restrict__ p,
                                                     double* __restrict__ Ap, CgScal* S, double* partials) {
	if (is_done(S)) return;
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[1] = {0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double s = row_dot<L, double, double>(A, p, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) { const int64_t i = mat_row(A, row); sth(Ap + i, s, pol.last); v[0] += ldh(p + i, pol.last) * s; }
	}
	if (grid_sum<1>(v, partials, &S->ticket)) {
		S->pAp = v[0];
		S->alpha = S->rz / v[0];
		if (!isfinite(S->alpha)) { S->done = 1; S->converged = 0; S->status = RSD_EBREAKDOWN; }
	}
}

// x += alpha p; r -= alpha Ap; res = |r|; convergence; z = M r; beta = r.z_new / r.z  (Solver.tpp:74-106)
__global__ void __launch_bounds__(kVT) k_cg_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                   const double* __restrict__ p, const double* __restrict__ Ap,
                                                   const double* __restrict__ invD, CgScal* S, double* partials, double tol,
                                                   int relMode, int64_t maxIters, int vec) {
	if (is_done(S)) return;
	const double alpha = S->alpha;
	const L2Pol pol = make_l2pol();
	const uint64_t h = pol.last;
	double v[2] = {0.0, 0.0};
	packet_loop<double>(n, vec, [&](int64_t i, int w) {
		if (w > 1) {
			Pk<double> X = ldp_rw(x + i, h), P = ldp(p + i, h), R = ldp_rw(r + i, h), Q = ldp(Ap + i, h), D;
			if (invD) D = ldp(invD + i, h);
#pragma unroll
			for (int k = 0; k < Pk<double>::W; ++k) {
				X.v[k] = X.v[k] + alpha * P.v[k];
				const double ri = R.v[k] + (-alpha) * Q.v[k];
				R.v[k] = ri;
				const double zi = invD ? ri * D.v[k] : ri;
				v[0] += ri * ri;
				v[1] += ri * zi;
			}
			stp(x + i, X, h);
			stp(r + i, R, h);
		} else {
			sth(x + i, ldh_rw(x + i, h) + alpha * ldh(p + i, h), h);
			const double ri = ldh_rw(r + i, h) + (-alpha) * ldh(Ap + i, h);
			sth(r + i, ri, h);
			const double zi = invD ? ri * ldh(invD + i, h) : ri;
			v[0] += ri * ri;
			v[1] += ri * zi;
		}
	});
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const int64_t k = S->iter + 1;
		const double res = sqrt(v[0]);
		const double rel = res / (S->res0 + 1e-50);
		S->res = res; S->iter = k;
		const double crit = relMode ? rel : res;
		if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; }
		else if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (k + 1 >= maxIters) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->beta = v[1] / S->rz; S->rz = v[1]; }
	}
}

// p = beta p + z   (Solver.tpp:103-104: scal then axpy)
__global__ void __launch_bounds__(kVT) k_cg_pupdate(int64_t n, double* __restrict__ p, const double* __restrict__ r,
                                                    const double* __restrict__ invD, CgScal* S, GraphCtl gc) {
	if (gc.on && blockIdx.x == 0 && threadIdx.x == 0) graph_continue(S, gc);
	if (is_done(S)) return;
	const double beta = S->beta;
	const L2Pol pol = make_l2pol();
	const uint64_t h = pol.last;   // the next SpMV gathers p
	packet_loop<double>(n, true, [&](int64_t i, int w) {
		if (w > 1) {
			Pk<double> P = ldp_rw(p + i, h), R = ldp(r + i, h), D;
			if (invD) D = ldp(invD + i, h);
#pragma unroll
			for (int k = 0; k < Pk<double>::W; ++k) P.v[k] = P.v[k] * beta + 1.0 * (invD ? R.v[k] * D.v[k] : R.v[k]);
			stp(p + i, P, h);
		} else {
			const double ri = ldh(r + i, h);
			const double zi = invD ? ri * ldh(invD + i, h) : ri;
			sth(p + i, ldh_rw(p + i, h) * beta + 1.0 * zi, h);
		}
	});
}

// ---- mixed precision PCG: FP32 matrix, vectors and recurrence; FP64 x, reductions and residual
// replacement (reliable updates, Sleijpen & van der Vorst 1996): whenever the FP32 recurrence
// residual drops by `delta` since the last replacement, or claims convergence, the FP32
// correction y is folded into x (x += y, y = 0) and the true residual r = b - A64 x is recomputed
// in FP64 to replace the recurrence residual.  Convergence is declared on the FP64 residual only.
// The iteration is the single-reduction form (k_mx_step): one SpMV and one vector pass.
// r0 = b - A64 x in FP64, z0 = M r0, y = 0
template <int L>
__global__ void __launch_bounds__(256) k_mx_init(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                 const double* __restrict__ x, float* __restrict__ z,
                                                 float* __restrict__ y, const float* __restrict__ invD, CgScal* S,
                                                 double* partials, double tol, int relMode, int64_t maxIters, double delta) {
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[2] = {0.0, 0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double ax = row_dot<L, double, double>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) {
			const int64_t i = mat_row(A, row);
			const double r64 = ldh(b + i, pol.first) - ax;
			const float ri = (float)r64;
			const float zi = invD ? ri * ldh(invD + i, pol.last) : ri;
			sth(z + i, zi, pol.last); sth(y + i, 0.0f, pol.last);
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res0 = sqrt(v[0]);
		S->res0 = res0; S->rmax = res0; S->res = res0; S->res64 = res0; S->rhoPrev = 0.0; S->trueRel = 1.0;
		S->rz = v[1]; S->iter = 0; S->refinements = 0; S->reliable = 0; S->status = 0;
		S->dcur = delta;
		const double crit = relMode ? res0 / (res0 + 1e-50) : res0;
		if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (maxIters <= 1) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->done = 0; S->converged = 0; }
	}
}

// w = A32 z and mu = z.w (FP64 sum)
template <int L>
__global__ void __launch_bounds__(kST, kRowBlocks) k_mx_spmv_dot(int64_t n, MatView<float> A, const float* __restrict__ z,
                                                     float* __restrict__ w, CgScal* S, double* partials) {
	if (is_done(S)) return;
	if (blockIdx.x == 0 && threadIdx.x == 0) S->reliable = 0;
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[1] = {0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const float s = row_dot<L, float, float>(A, z, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) { const int64_t i = mat_row(A, row); sth(w + i, s, pol.last); v[0] += (double)ldh(z + i, pol.last) * (double)s; }
	}
	if (grid_sum<1>(v, partials, &S->ticket)) S->pAp = v[0];
}

// The vector pass of the single-reduction iteration (Chronopoulos & Gear 1989): with rho = r.z,
// mu = z.Az and the previous rho and alpha on the device, beta = rho / rho_prev and
// alpha = rho / (mu - beta rho / alpha_prev) (the first pass: beta = 0, alpha = rho / mu); then
// p = z + beta p, s = w + beta s (s = A p by recurrence, w = A z), y += alpha p, and the residual
// update carried on z alone (Jacobi: r = D z, so z -= alpha M s and r = z / M for the sums), with
// rho = r.z and |r| in one reduction.  In exact arithmetic these are the iterates of
// the two-reduction PCG; the pass replaces its update and p-update kernels and one grid-wide
// reduction per iteration.  In graph mode its first thread also sets the loop condition from the
// done flag as the previous body left it (replacement included), so a solve ends one idle body after
// the body that finished it, with no extra node per iteration.
__global__ void __launch_bounds__(kVT) k_mx_step(int64_t n, float* __restrict__ y,
                                                 float* __restrict__ z, float* __restrict__ p, float* __restrict__ s,
                                                 const float* __restrict__ w, const float* __restrict__ invD, CgScal* S,
                                                 double* partials, double tol, int relMode, int64_t maxIters, GraphCtl gc) {
	if (gc.on && blockIdx.x == 0 && threadIdx.x == 0) graph_continue(S, gc);
	if (is_done(S)) return;
	const double rho = S->rz, mu = S->pAp, rhoPrev = S->rhoPrev;
	const bool first = !(rhoPrev != 0.0);
	const double beta = first ? 0.0 : rho / rhoPrev;
	const double alpha = first ? rho / mu : rho / (mu - beta * rho / S->alpha);
	const float fa = (float)alpha, fb = (float)beta;
	const L2Pol pol = make_l2pol();
	const uint64_t h = pol.last;
	double v[2] = {0.0, 0.0};
	packet_loop<float>(n, true, [&](int64_t i, int wd) {
		if (wd > 1) {
			Pk<float> Z = ldp_rw(z + i, h), W = ldp(w + i, h), Y = ldp_rw(y + i, h), P, Q, D;
			if (first) { P = Z; Q = W; }
			else {
				P = ldp_rw(p + i, h); Q = ldp_rw(s + i, h);
#pragma unroll
				for (int k = 0; k < Pk<float>::W; ++k) { P.v[k] = Z.v[k] + fb * P.v[k]; Q.v[k] = W.v[k] + fb * Q.v[k]; }
			}
			if (invD) D = ldp(invD + i, h);
#pragma unroll
			for (int k = 0; k < Pk<float>::W; ++k) {
				Y.v[k] = Y.v[k] + fa * P.v[k];
				const float zi = invD ? Z.v[k] - fa * (Q.v[k] * D.v[k]) : Z.v[k] - fa * Q.v[k];
				const float ri = invD ? zi / D.v[k] : zi;
				Z.v[k] = zi;
				v[0] += (double)ri * (double)ri;
				v[1] += (double)ri * (double)zi;
			}
			stp(p + i, P, h); stp(s + i, Q, h); stp(y + i, Y, h); stp(z + i, Z, h);
		} else {
			const float zo = ldh_rw(z + i, h), wo = ldh(w + i, h);
			const float pi = first ? zo : zo + fb * ldh_rw(p + i, h);
			const float si = first ? wo : wo + fb * ldh_rw(s + i, h);
			sth(p + i, pi, h); sth(s + i, si, h);
			sth(y + i, ldh_rw(y + i, h) + fa * pi, h);
			const float di = invD ? ldh(invD + i, h) : 1.0f;
			const float zi = invD ? zo - fa * (si * di) : zo - fa * si;
			const float ri = invD ? zi / di : zi;
			sth(z + i, zi, h);
			v[0] += (double)ri * (double)ri;
			v[1] += (double)ri * (double)zi;
		}
	});
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const int64_t k = S->iter + 1;
		const double res = sqrt(v[0]);
		S->res = res; S->iter = k;
		if (!isfinite(alpha)) { S->done = 1; S->converged = 0; S->status = RSD_EBREAKDOWN; }
		else if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; }
		else {
			S->alpha = alpha; S->beta = beta; S->rhoPrev = rho; S->rz = v[1];
			const double crit = relMode ? res / (S->res0 + 1e-50) : res;
			if (crit < tol || res < S->dcur * S->rmax || k + 1 >= maxIters) S->reliable = 1;   // FP64 replacement next
		}
		if (gc.on) cudaGraphSetConditional(gc.hr, S->reliable ? 1u : 0u);
	}
}

// before a replacement: fold the FP32 correction into the FP64 iterate, x += y, y = 0
__global__ void __launch_bounds__(kVT) k_mx_fold(int64_t n, double* __restrict__ x, float* __restrict__ y, const CgScal* S) {
	if (is_done(S) || !*((volatile const int32_t*)&S->reliable)) return;
	const L2Pol pol = make_l2pol();
	const uint64_t h = pol.last;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		sth(x + i, ldh_rw(x + i, h) + (double)ldh_rw(y + i, h), h);
		sth(y + i, 0.0f, h);
	}
}

// reliable update (after the fold): r64 = b - A64 x, z = M (float) r64, rho = r.z with the new r
// (p, s and the previous rho and alpha carry on)
template <int L>
__global__ void __launch_bounds__(kST, kRowBlocks) k_mx_reliable(int64_t n, MatView<double> A, const double* __restrict__ b,
                                                     const double* __restrict__ x,
                                                     float* __restrict__ z, const float* __restrict__ invD, CgScal* S, double* partials,
                                                     double tol, int relMode, int64_t maxIters, int adaptive) {
	if (is_done(S) || !*((volatile const int32_t*)&S->reliable)) return;
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	double v[2] = {0.0, 0.0};
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const double ax = row_dot<L, double, double>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) {
			const int64_t i = mat_row(A, row);
			const double r64 = ldh(b + i, pol.first) - ax;
			const float ri = (float)r64;
			const float zi = invD ? ri * ldh(invD + i, pol.last) : ri;
			sth(z + i, zi, pol.last);
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		}
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res = sqrt(v[0]);
		const double rel = res / (S->res0 + 1e-50);
		if (adaptive) S->dcur = next_delta(S->dcur, S->res, res, kDeltaFloorCg);
		S->res64 = res; S->trueRel = rel; S->rmax = res; S->res = res;
		S->refinements += 1;
		const double crit = relMode ? rel : res;
		if (!isfinite(res)) { S->done = 1; S->converged = 0; S->status = RSD_ENAN; }
		else if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (S->iter + 1 >= maxIters) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else S->rz = v[1];
	}
}

// ---- the mixed solve as one persistent cooperative kernel ---------------------------------------
// The iteration of the kernels above (k_mx_spmv_dot, k_mx_step, and the replacement k_mx_fold +
// k_mx_reliable when due) run by one cooperative launch whose blocks stay resident for the whole
// solve: a grid barrier separates the phases, and every block sums the phase's per-block partials
// itself (the same partials in the same order, so every block holds the same scalars and takes the
// same decisions).  What it saves over one launch per phase is each kernel's ramp, its dependent
// scalar loads at the start and its last-block reduction tail.  Each barrier waits a bounded time;
// a barrier that gives up ends the solve with RSD_ETIMEOUT.
constexpr int kPersistSlots = 5;                        // partial slots: SpMV 0; step 1, 2; replacement 3, 4
constexpr unsigned long long kBarrierPolls = 1ull << 24;  // the first 4096 back to back, then 64 ns apart: about a second

__device__ __forceinline__ bool grid_barrier(unsigned long long* count, unsigned long long target) {
	__shared__ int ok;
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		atomicAdd(count, 1ull);
		unsigned long long polls = 0;
		int good = 1;
		while (*(volatile unsigned long long*)count < target) {
			if (++polls > kBarrierPolls) { good = 0; break; }
			if (polls > 4096) __nanosleep(64);
		}
		__threadfence();
		ok = good;
	}
	__syncthreads();
	return ok != 0;
}

// every block's NCH sums, then (after the barrier) their totals in every block: the partials of
// slot c + blockIdx.x, summed strided and by block_sum as grid_sum's last block does
template <int NCH>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NCH], double* partials, int slot0, unsigned long long* count,
                                               unsigned long long& gen) {
	__shared__ double tot[NCH];
	block_sum<NCH>(v);
	if (threadIdx.x == 0)
#pragma unroll
		for (int c = 0; c < NCH; ++c) partials[(size_t)(slot0 + c) * kMaxPartials + blockIdx.x] = v[c];
	gen += gridDim.x;
	if (!grid_barrier(count, gen)) return false;
	double acc[NCH];
#pragma unroll
	for (int c = 0; c < NCH; ++c) {
		acc[c] = 0.0;
		for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[c] += __ldcg(&partials[(size_t)(slot0 + c) * kMaxPartials + b]);
	}
	block_sum<NCH>(acc);
	if (threadIdx.x == 0)
#pragma unroll
		for (int c = 0; c < NCH; ++c) tot[c] = acc[c];
	__syncthreads();
#pragma unroll
	for (int c = 0; c < NCH; ++c) v[c] = tot[c];
	return true;
}

struct MxPersistArgs {
	int64_t n;
	MatView<float> A32;
	MatView<double> A64;
	const double* b;
	double* x;
	float *z, *p, *s, *w, *y;
	const float* invD;
	CgScal* S;
	double* partials;            // kPersistSlots slots of kMaxPartials
	unsigned long long* count;   // barrier arrivals (zeroed before the launch)
	double tol;
	int relMode, adaptive;
	int64_t maxIters;
};

template <int L>
__global__ void __launch_bounds__(kST, kRowBlocks) k_mx_persist(const MxPersistArgs a) {
	const L2Pol pol = make_l2pol();
	const int64_t n = a.n;
	CgScal* S = a.S;
	// the state k_mx_init left, read once; from here on every block carries the same copy
	double rho = S->rz, rhoPrev = S->rhoPrev, alphaPrev = S->alpha, betaPrev = S->beta;
	const double res0 = S->res0;
	double res = S->res, rmax = S->rmax, dcur = S->dcur, res64 = S->res64, trueRel = S->trueRel;
	int64_t iter = S->iter;
	int refinements = S->refinements, done = S->done, converged = S->converged, status = S->status;
	unsigned long long gen = 0;
	const uint64_t h = pol.last;
	for (int64_t guard = 0; !done && guard <= a.maxIters + 2; ++guard) {
		// w = A32 z, mu = z.w
		double vA[1] = {0.0};
		{
			const RowLoop<L> rl;
			for (int64_t base = rl.base; base < n; base += rl.step) {
				const int64_t row = base + rl.sub;
				// z was written by this launch: coherent loads (the .nc path holds no such guarantee)
				const float sr = row_sum<L, float, float>(a.A32, row, n, rl.lane, pol, [&](int c) { return ldh_rw(a.z + c, pol.last); });
				if (rl.lane == 0 && row < n) {
					const int64_t i = mat_row(a.A32, row);
					sth(a.w + i, sr, pol.last);
					vA[0] += (double)ldh_rw(a.z + i, pol.last) * (double)sr;
				}
			}
		}
		if (!grid_allreduce<1>(vA, a.partials, 0, a.count, gen)) { status = RSD_ETIMEOUT; done = 1; break; }
		const double mu = vA[0];
		// the single-reduction vector pass (k_mx_step)
		const bool first = !(rhoPrev != 0.0);
		const double beta = first ? 0.0 : rho / rhoPrev;
		const double alpha = first ? rho / mu : rho / (mu - beta * rho / alphaPrev);
		const float fa = (float)alpha, fb = (float)beta;
		double vB[2] = {0.0, 0.0};
		packet_loop<float>(n, true, [&](int64_t i, int wd) {
			if (wd > 1) {
				Pk<float> Z = ldp_rw(a.z + i, h), W = ldp_rw(a.w + i, h), Y = ldp_rw(a.y + i, h), P, Q, D;
				if (first) { P = Z; Q = W; }
				else {
					P = ldp_rw(a.p + i, h); Q = ldp_rw(a.s + i, h);
#pragma unroll
					for (int k = 0; k < Pk<float>::W; ++k) { P.v[k] = Z.v[k] + fb * P.v[k]; Q.v[k] = W.v[k] + fb * Q.v[k]; }
				}
				if (a.invD) D = ldp(a.invD + i, h);
#pragma unroll
				for (int k = 0; k < Pk<float>::W; ++k) {
					Y.v[k] = Y.v[k] + fa * P.v[k];
					const float zi = a.invD ? Z.v[k] - fa * (Q.v[k] * D.v[k]) : Z.v[k] - fa * Q.v[k];
					const float ri = a.invD ? zi / D.v[k] : zi;
					Z.v[k] = zi;
					vB[0] += (double)ri * (double)ri;
					vB[1] += (double)ri * (double)zi;
				}
				stp(a.p + i, P, h); stp(a.s + i, Q, h); stp(a.y + i, Y, h); stp(a.z + i, Z, h);
			} else {
				const float zo = ldh_rw(a.z + i, h), wo = ldh_rw(a.w + i, h);
				const float pi = first ? zo : zo + fb * ldh_rw(a.p + i, h);
				const float si = first ? wo : wo + fb * ldh_rw(a.s + i, h);
				sth(a.p + i, pi, h); sth(a.s + i, si, h);
				sth(a.y + i, ldh_rw(a.y + i, h) + fa * pi, h);
				const float di = a.invD ? ldh(a.invD + i, h) : 1.0f;
				const float zi = a.invD ? zo - fa * (si * di) : zo - fa * si;
				const float ri = a.invD ? zi / di : zi;
				sth(a.z + i, zi, h);
				vB[0] += (double)ri * (double)ri;
				vB[1] += (double)ri * (double)zi;
			}
		});
		if (!grid_allreduce<2>(vB, a.partials, 1, a.count, gen)) { status = RSD_ETIMEOUT; done = 1; break; }
		const int64_t k = iter + 1;
		res = sqrt(vB[0]);
		iter = k;
		bool reliable = false;
		if (!isfinite(alpha)) { done = 1; converged = 0; status = RSD_EBREAKDOWN; }
		else if (!isfinite(res)) { done = 1; converged = 0; status = RSD_ENAN; }
		else {
			alphaPrev = alpha; betaPrev = beta; rhoPrev = rho; rho = vB[1];
			const double crit = a.relMode ? res / (res0 + 1e-50) : res;
			reliable = crit < a.tol || res < dcur * rmax || k + 1 >= a.maxIters;
		}
		if (done || !reliable) continue;
		// replacement: x += y, y = 0; then r64 = b - A64 x, z = M r (k_mx_fold, k_mx_reliable)
		for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
			sth(a.x + i, ldh_rw(a.x + i, h) + (double)ldh_rw(a.y + i, h), h);
			sth(a.y + i, 0.0f, h);
		}
		gen += gridDim.x;
		if (!grid_barrier(a.count, gen)) { status = RSD_ETIMEOUT; done = 1; break; }
		double vR[2] = {0.0, 0.0};
		{
			const RowLoop<L> rl;
			for (int64_t base = rl.base; base < n; base += rl.step) {
				const int64_t row = base + rl.sub;
				const double ax = row_sum<L, double, double>(a.A64, row, n, rl.lane, pol, [&](int c) { return ldh_rw(a.x + c, pol.last); });
				if (rl.lane == 0 && row < n) {
					const int64_t i = mat_row(a.A64, row);
					const double r64 = ldh(a.b + i, pol.first) - ax;
					const float ri = (float)r64;
					const float zi = a.invD ? ri * ldh(a.invD + i, pol.last) : ri;
					sth(a.z + i, zi, pol.last);
					vR[0] += r64 * r64;
					vR[1] += (double)ri * (double)zi;
				}
			}
		}
		if (!grid_allreduce<2>(vR, a.partials, 3, a.count, gen)) { status = RSD_ETIMEOUT; done = 1; break; }
		const double rt = sqrt(vR[0]);
		const double rel = rt / (res0 + 1e-50);
		if (a.adaptive) dcur = next_delta(dcur, res, rt, kDeltaFloorCg);
		res64 = rt; trueRel = rel; rmax = rt; res = rt;
		refinements += 1;
		const double crit = a.relMode ? rel : rt;
		if (!isfinite(rt)) { done = 1; converged = 0; status = RSD_ENAN; }
		else if (crit < a.tol) { done = 1; converged = 1; }
		else if (iter + 1 >= a.maxIters) { done = 1; converged = 0; iter = a.maxIters; }
		else rho = vR[1];
	}
	if (!done) { done = 1; converged = 0; }   // the guard ran out (cannot happen with a finite maxIters)
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		S->rz = rho; S->rhoPrev = rhoPrev; S->alpha = alphaPrev; S->beta = betaPrev;
		S->res = res; S->rmax = rmax; S->dcur = dcur; S->res64 = res64; S->trueRel = trueRel;
		S->iter = iter; S->refinements = refinements; S->done = done; S->converged = converged; S->status = status;
		S->reliable = 0;
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
		if (rl.lane == 0 && row < n) { const double ri = ldh(b + mat_row(A, row), pol.first) - ax; v[0] += ri * ri; }
	}
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

// ---- workspace -------------------------------------------------------------------------------
// One grow-only buffer per context, used only on that context's stream: contexts on one device (one
// per host thread, say) never share Krylov vectors, and a grow waits only for this context's own work.
static int get_ws(rsd_ctx* ctx, size_t bytes, void** out) {
	if (ctx->wsBytes < bytes) {
		if (ctx->ws) {
			RSD_CUDA(cudaStreamSynchronize(ctx->stream));
			cudaFree(ctx->ws);
			ctx->ws = nullptr;
			ctx->wsBytes = 0;
		}
		RSD_CUDA(cudaMalloc(&ctx->ws, bytes));
		ctx->wsBytes = bytes;
	}
	*out = ctx->ws;
	return RSD_OK;
}

// The SpMV kernels are capped at 32 registers (8 blocks of 256 per SM): they are latency-bound on
// the value/column -> gather chain, and full occupancy measured 20-25% faster than the 40-register
// build.
// grids of the row kernels (n rows, max(L,1) threads each) and vector kernels (n entries): one
// full wave of each kernel's resident blocks; used inside functions that define ctx, n and L
#define RG(kern) wave_blocks(ctx, kern, 256, n * std::max(L, 1))
#define VG(kern) wave_blocks(ctx, kern, 256, n)
#define RGB(kern, bt) wave_blocks(ctx, kern, bt, n * std::max(L, 1))
#define VGB(kern, bt) wave_blocks(ctx, kern, bt, n)

// workspace vectors start 256-byte aligned: every warp's 32 consecutive entries then fall in whole
// 32-byte sectors
static int64_t pad_len(int64_t n) { return (n + 63) & ~int64_t(63); }

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

// ---- graph mode plumbing ---------------------------------------------------------------------
// A solve's graph is cached on the context per precision and rebuilt only when anything it
// captured changes (pointers, sizes, launch shapes, tolerances).
struct CgKey {
	const void* p[14];
	int64_t i[8];
	double d[2];
	bool operator==(const CgKey& o) const { return std::memcmp(this, &o, sizeof(CgKey)) == 0; }
};
struct CgGraph {
	CgKey key{};
	bool valid = false;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	void release() {
		if (exec) cudaGraphExecDestroy(exec);
		if (graph) cudaGraphDestroy(graph);
		exec = nullptr; graph = nullptr; valid = false;
	}
};
struct GraphCache {
	CgGraph cg[2];   // 0: FP64, 1: mixed
};

static bool graph_mode(const rsd_ctx* ctx) {
	if (ctx->prof.on) return false;              // per-kernel timing needs the plain launches
	const char* e = getenv("RSD_CG_GRAPH");
	return !(e && e[0] == '0');
}

// the persistent mixed solve (k_mx_persist) needs cooperative launches; RSD_CG_PERSIST=0 keeps the
// per-phase kernels (as a graph, or as plain launches under RSD_CG_GRAPH=0 or profiling, which then
// times each phase)
static bool persist_mode(const rsd_ctx* ctx) {
	const char* e = getenv("RSD_CG_PERSIST");
	if (e && e[0] == '0') return false;
	const char* g = getenv("RSD_CG_GRAPH");
	if (g && g[0] == '0') return false;
	int coop = 0;
	cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device);
	return coop != 0;
}

static GraphCache* graph_cache(rsd_ctx* ctx) {
	if (!ctx->graphs) ctx->graphs = new GraphCache();
	return static_cast<GraphCache*>(ctx->graphs);
}

// leaf nodes of the work captured so far on the stream
static int capture_leaves(cudaStream_t s, const cudaGraphNode_t** deps, size_t* nd) {
	cudaStreamCaptureStatus st;
	RSD_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, deps, nd));
	if (st != cudaStreamCaptureStatusActive) return set_error(RSD_ECUDA, "stream capture is not active");
	return RSD_OK;
}

// add a conditional node of `type` to `g` behind `deps`; returns the node and its body graph
static int add_conditional(cudaGraph_t g, const cudaGraphNode_t* deps, size_t nd, cudaGraphConditionalHandle h,
                           cudaGraphConditionalNodeType type, cudaGraphNode_t* node, cudaGraph_t* body) {
	cudaGraphNodeParams np{};
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = h;
	np.conditional.type = type;
	np.conditional.size = 1;
	RSD_CUDA(cudaGraphAddNode(node, g, deps, nd, &np));
	*body = np.conditional.phGraph_out[0];
	return RSD_OK;
}

// Build prologue -> WHILE(body_a -> [IF(reliable)] -> body_b) -> epilogue into one executable graph.
// Each stage function launches its kernels on ctx->stream, which is being captured.
template <typename Pro, typename BodyA, typename Rel, typename BodyB, typename Epi>
static int build_cg_graph(rsd_ctx* ctx, bool with_if, int32_t limit, Pro prologue, BodyA body_a, Rel reliable,
                          BodyB body_b, Epi epilogue, CgGraph* G) {
	cudaStream_t s = ctx->stream;
	G->release();
	RSD_CUDA(cudaGraphCreate(&G->graph, 0));
	cudaGraphConditionalHandle hw = 0, hr = 0;
	RSD_CUDA(cudaGraphConditionalHandleCreate(&hw, G->graph, 1, cudaGraphCondAssignDefault));
	auto fail = [&](int rc) {
		cudaGraph_t junk = nullptr;
		cudaStreamCaptureStatus st;
		if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) cudaStreamEndCapture(s, &junk);
		cudaGetLastError();
		G->release();
		return rc;
	};
	int rc;
	// prologue, then the WHILE node behind it
	RSD_CUDA(cudaStreamBeginCaptureToGraph(s, G->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
	if ((rc = prologue()) != RSD_OK) return fail(rc);
	const cudaGraphNode_t* deps = nullptr;
	size_t nd = 0;
	if ((rc = capture_leaves(s, &deps, &nd)) != RSD_OK) return fail(rc);
	cudaGraphNode_t wnode;
	cudaGraph_t body;
	if ((rc = add_conditional(G->graph, deps, nd, hw, cudaGraphCondTypeWhile, &wnode, &body)) != RSD_OK) return fail(rc);
	cudaGraph_t out = nullptr;
	if (cudaStreamEndCapture(s, &out) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "end capture (prologue)"));
	// the loop body
	cudaGraph_t ifBody = nullptr;
	if (with_if && cudaGraphConditionalHandleCreate(&hr, body, 0, cudaGraphCondAssignDefault) != cudaSuccess)
		return fail(cuda_error(cudaGetLastError(), "conditional handle (IF)"));
	const GraphCtl gc{hw, hr, 1, limit};
	if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
		return fail(cuda_error(cudaGetLastError(), "begin capture (body)"));
	if ((rc = body_a(gc)) != RSD_OK) return fail(rc);
	if (with_if) {
		if ((rc = capture_leaves(s, &deps, &nd)) != RSD_OK) return fail(rc);
		cudaGraphNode_t inode;
		if ((rc = add_conditional(body, deps, nd, hr, cudaGraphCondTypeIf, &inode, &ifBody)) != RSD_OK) return fail(rc);
		if (cudaStreamUpdateCaptureDependencies(s, &inode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
			return fail(cuda_error(cudaGetLastError(), "capture dependencies (IF)"));
	}
	if ((rc = body_b(gc)) != RSD_OK) return fail(rc);
	if (cudaStreamEndCapture(s, &out) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "end capture (body)"));
	if (with_if) {
		if (cudaStreamBeginCaptureToGraph(s, ifBody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
			return fail(cuda_error(cudaGetLastError(), "begin capture (IF body)"));
		if ((rc = reliable()) != RSD_OK) return fail(rc);
		if (cudaStreamEndCapture(s, &out) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "end capture (IF body)"));
	}
	// epilogue behind the WHILE node
	if (cudaStreamBeginCaptureToGraph(s, G->graph, &wnode, nullptr, 1, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
		return fail(cuda_error(cudaGetLastError(), "begin capture (epilogue)"));
	if ((rc = epilogue()) != RSD_OK) return fail(rc);
	if (cudaStreamEndCapture(s, &out) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "end capture (epilogue)"));
	if (cudaGraphInstantiate(&G->exec, G->graph, 0) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "graph instantiate"));
	G->valid = true;
	return RSD_OK;
}

static int32_t body_limit(int64_t max_iters) { return (int32_t)std::min<int64_t>(max_iters + 4, INT32_MAX - 1); }

static int cg_fp64(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	RSD_CHECK(exec_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	void* wsv;
	const int64_t ns = pad_len(n);
	RSD_CHECK(get_ws(ctx, sizeof(double) * 4 * ns, &wsv));
	double* r = (double*)wsv;
	double* p = r + ns;
	double* Ap = p + ns;
	double* invD = cfg->precond == RSD_JACOBI ? Ap + ns : nullptr;
	const int xvec = reinterpret_cast<uintptr_t>(x) % 16 == 0;   // 16-byte packets on x too
	CgScal* S = scal_slot(ctx, 0);
	CgScal* S1 = scal_slot(ctx, 1);
	double* partials = ctx->s.partials;
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	const double tol = cfg->tol;
	const int64_t maxIt = cfg->max_iters;
	cudaStream_t st = ctx->stream;
	auto prologue = [&]() -> int {
		RSD_CUDA(cudaMemsetAsync(S, 0, sizeof(CgScal), st));
		// Jacobi::update on every solve (cg/Solver.tpp:22)
		if (invD) k_invdiag64<<<VG(k_invdiag64), 256, 0, st>>>(n, exec_diag(A), exec_val(A), invD);
		RSD_DISPATCH_L(L, (k_cg_init<LL><<<RG(k_cg_init<LL>), 256, 0, st>>>(n, V, b, x, r, p, invD, S, partials, tol, rel, maxIt)));
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	auto body_a = [&](GraphCtl) -> int {
		RSD_DISPATCH_L(L, (k_cg_spmv_dot<LL><<<RGB(k_cg_spmv_dot<LL>, kST), kST, 0, st>>>(n, V, p, Ap, S, partials)));
		k_cg_update<<<VGB(k_cg_update, kVT), kVT, 0, st>>>(n, x, r, p, Ap, invD, S, partials, tol, rel, maxIt, xvec);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	auto body_b = [&](GraphCtl gc) -> int {
		k_cg_pupdate<<<VGB(k_cg_pupdate, kVT), kVT, 0, st>>>(n, p, r, invD, S, gc);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	// FP64 check of the final iterate: ||b - A x|| into S1->res
	auto epilogue = [&]() -> int {
		RSD_DISPATCH_L(L, (k_true_res<LL><<<RG(k_true_res<LL>), 256, 0, st>>>(n, V, b, x, partials, &S1->ticket, &S1->res)));
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	if (graph_mode(ctx)) {
		CgGraph& G = graph_cache(ctx)->cg[0];
		CgKey key{};
		const void* ptrs[] = {A, V.ptr, V.col, V.val, exec_diag(A), b, x, r, invD, S, partials};
		std::copy(std::begin(ptrs), std::end(ptrs), key.p);
		const int64_t ints[] = {n, L, maxIt, rel};
		std::copy(std::begin(ints), std::end(ints), key.i);
		key.d[0] = tol;
		if (!G.valid || !(G.key == key)) {
			RSD_CHECK(build_cg_graph(ctx, false, body_limit(maxIt), prologue, body_a, [] { return RSD_OK; }, body_b, epilogue, &G));
			G.key = key;
		}
		RSD_CUDA(cudaGraphLaunch(G.exec, st));
		RSD_CHECK(finish_report(ctx, S, rep));
	} else {
		RSD_CHECK(prologue());
		Poller poll{ctx, S, (int32_t*)ctx->s.hbuf};
		RSD_CHECK(poll.init());
		const int chunk = 8;
		bool fin = false;
		std::vector<int> pairs;
		const GraphCtl off{0, 0, 0, 0};
		for (int64_t it = 0; it < maxIt + 2 * chunk && !fin; it += chunk) {
			for (int c = 0; c < chunk; ++c) {
				int pr = prof_begin(ctx, PF_SPMV_DOT_F64);
				RSD_DISPATCH_L(L, (k_cg_spmv_dot<LL><<<RGB(k_cg_spmv_dot<LL>, kST), kST, 0, st>>>(n, V, p, Ap, S, partials)));
				prof_end(ctx, pr);
				int pu = prof_begin(ctx, PF_CG_UPDATE);
				k_cg_update<<<VGB(k_cg_update, kVT), kVT, 0, st>>>(n, x, r, p, Ap, invD, S, partials, tol, rel, maxIt, xvec);
				prof_end(ctx, pu);
				int pp = prof_begin(ctx, PF_CG_PUPDATE);
				k_cg_pupdate<<<VGB(k_cg_pupdate, kVT), kVT, 0, st>>>(n, p, r, invD, S, off);
				prof_end(ctx, pp);
				if (pr >= 0) { pairs.push_back(pr); pairs.push_back(pu); pairs.push_back(pp); }
			}
			RSD_CUDA(cudaGetLastError());
			RSD_CHECK(poll.post(&fin));
		}
		RSD_CHECK(finish_report(ctx, S, rep));
		discard_idle(ctx, pairs, 3, rep ? rep->iterations : 0);
		RSD_CHECK(epilogue());
	}
	double h = 0.0;
	RSD_CUDA(cudaMemcpyAsync(&h, &S1->res, sizeof(double), cudaMemcpyDeviceToHost, st));
	RSD_CUDA(cudaStreamSynchronize(st));
	if (rep) rep->trueResidualRel = h / (rep->initialResidual + 1e-50);
	return RSD_OK;
}

static int cg_mixed(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	const int64_t n = A->n;
	RSD_CHECK(f32_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	// the mirrored reads of a symmetric matrix are opt-in (RSD_SYM_SPMV=1): on the 128^3 BE system they
	// cut the value stream to 57 % but the dependent mirror loads (slice start, then value) made the
	// step slower (7.17 against 4.53 ms)
	const char* symEnv = getenv("RSD_SYM_SPMV");
	const MatView<float> V32 = (symEnv && symEnv[0] == '1') ? view32_sym(A) : view32(A);
	void* wsv;
	const int64_t ns = pad_len(n);
	// six FP32 vectors, then the persistent kernel's partial slots and barrier count
	const size_t vecBytes = sizeof(float) * 6 * ns;
	RSD_CHECK(get_ws(ctx, vecBytes + sizeof(double) * kPersistSlots * kMaxPartials + 256, &wsv));
	double* pslots = (double*)((char*)wsv + vecBytes);
	unsigned long long* pcount = (unsigned long long*)(pslots + kPersistSlots * kMaxPartials);
	// the residual is carried as z = M r alone (r = D z for the reductions)
	float* z = (float*)wsv;  // M r, the vector the SpMV multiplies
	float* p = z + ns;
	float* sv = p + ns;      // A p, by recurrence
	float* w = sv + ns;      // A z
	float* y = w + ns;
	float* invD = cfg->precond == RSD_JACOBI ? y + ns : nullptr;
	CgScal* S = scal_slot(ctx, 0);
	double* partials = ctx->s.partials;
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	// a fixed threshold when the configuration gives one, else adaptive from 0.1
	const int adaptive = !(cfg->reliable_delta > 0);
	const double delta = adaptive ? 0.1 : cfg->reliable_delta;
	const double tol = cfg->tol;
	const int64_t maxIt = cfg->max_iters;
	cudaStream_t st = ctx->stream;
	auto prologue = [&]() -> int {
		RSD_CUDA(cudaMemsetAsync(S, 0, sizeof(CgScal), st));
		if (invD) k_invdiag32<<<VG(k_invdiag32), 256, 0, st>>>(n, exec_diag(A), exec_val(A), invD);
		RSD_DISPATCH_L(L, (k_mx_init<LL><<<RG(k_mx_init<LL>), 256, 0, st>>>(n, V, b, x, z, y, invD, S, partials, tol, rel, maxIt, delta)));
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	// one iteration: w = A z with mu = z.w, then the single-reduction vector pass
	auto spmv = [&]() {
		RSD_DISPATCH_L(L, (k_mx_spmv_dot<LL><<<RGB(k_mx_spmv_dot<LL>, kST), kST, 0, st>>>(n, V32, z, w, S, partials)));
	};
	auto step = [&](GraphCtl gc) {
		// 512-thread blocks on the SpMV's grid: the partition k_mx_persist uses, so that both paths
		// give the same sums, bit for bit
		k_mx_step<<<VGB(k_mx_step, kST), kST, 0, st>>>(n, y, z, p, sv, w, invD, S, partials, tol, rel, maxIt, gc);
	};
	auto body_a = [&](GraphCtl gc) -> int {
		spmv();
		step(gc);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	auto reliable = [&]() -> int {
		k_mx_fold<<<VGB(k_mx_fold, kVT), kVT, 0, st>>>(n, x, y, S);
		RSD_DISPATCH_L(L, (k_mx_reliable<LL><<<RGB(k_mx_reliable<LL>, kST), kST, 0, st>>>(n, V, b, x, z, invD, S, partials, tol, rel, maxIt, adaptive)));
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	auto body_b = [&](GraphCtl) -> int { return RSD_OK; };   // the step kernel sets the loop condition
	if (L <= 0 && persist_mode(ctx)) {
		// the whole iteration in one cooperative launch (SELL-32 layouts)
		RSD_CHECK(prologue());
		RSD_CUDA(cudaMemsetAsync(pcount, 0, sizeof(unsigned long long), st));
		MxPersistArgs args{n, V32, V, b, x, z, p, sv, w, y, invD, S, pslots, pcount, tol, rel, adaptive, maxIt};
		void* params[] = {&args};
		auto go = [&](const void* kern) -> int {
			int per = 0;
			RSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kST, 0));
			const int grid = std::min(std::max(per, 1) * ctx->num_sms, kMaxPartials);
			RSD_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kST), params, 0, st));
			return RSD_OK;
		};
		const int pf = prof_begin(ctx, PF_CG_PERSIST);
		RSD_CHECK(L == -1 ? go((const void*)k_mx_persist<-1>) : go((const void*)k_mx_persist<0>));
		prof_end(ctx, pf);
		RSD_CHECK(finish_report(ctx, S, rep));
	} else if (graph_mode(ctx)) {
		CgGraph& G = graph_cache(ctx)->cg[1];
		CgKey key{};
		const void* ptrs[] = {A, V.ptr, V.col, V.val, V32.val, exec_diag(A), b, x, z, invD, S, partials, V32.neg};
		std::copy(std::begin(ptrs), std::end(ptrs), key.p);
		const int64_t ints[] = {n, L, maxIt, rel};
		std::copy(std::begin(ints), std::end(ints), key.i);
		key.d[0] = tol;
		key.d[1] = adaptive ? -1.0 : delta;
		if (!G.valid || !(G.key == key)) {
			RSD_CHECK(build_cg_graph(ctx, true, body_limit(maxIt), prologue, body_a, reliable, body_b, [] { return RSD_OK; }, &G));
			G.key = key;
		}
		RSD_CUDA(cudaGraphLaunch(G.exec, st));
		RSD_CHECK(finish_report(ctx, S, rep));
	} else {
		RSD_CHECK(prologue());
		Poller poll{ctx, S, (int32_t*)ctx->s.hbuf};
		RSD_CHECK(poll.init());
		const int chunk = 8;
		bool fin = false;
		std::vector<int> pairs;
		const GraphCtl off{0, 0, 0, 0};
		for (int64_t it = 0; it < maxIt + 2 * chunk && !fin; it += chunk) {
			for (int c = 0; c < chunk; ++c) {
				int pr = prof_begin(ctx, PF_SPMV_DOT_F32);
				spmv();
				prof_end(ctx, pr);
				int pu = prof_begin(ctx, PF_CG_UPDATE);
				step(off);
				prof_end(ctx, pu);
				int pq = prof_begin(ctx, PF_RELIABLE);
				RSD_CHECK(reliable());
				prof_end(ctx, pq);
				if (pr >= 0) { pairs.push_back(pr); pairs.push_back(pu); pairs.push_back(pq); }
			}
			RSD_CUDA(cudaGetLastError());
			RSD_CHECK(poll.post(&fin));
		}
		RSD_CHECK(finish_report(ctx, S, rep));
		discard_idle(ctx, pairs, 3, rep ? rep->iterations : 0);
	}
	if (rep) { rep->finalResidual = rep->trueResidualRel * rep->initialResidual; rep->finalResidualRel = rep->trueResidualRel; }
	return RSD_OK;
}

// ---- PCG over the matrix-free operator: cg/Solver.tpp:13-119 with the operator products of
// FEMOperator::apply (linalg/operator/FEMOperator.hpp:39-43) and Jacobi::update over
// FEMOperator::diagonal (FEMOperator.hpp:49-51).  The products are element passes (apply_operator),
// the rest the FP64 CG kernels above. ------------------------------------------------------------

// Jacobi::update's inversion (preconditioner/Jacobi.hpp:29-32): d = 1/d where |d| > 1e-300, else 1
__global__ void k_inv_guarded(int64_t n, double* __restrict__ d) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double v = d[i];
		d[i] = (fabs(v) > 1e-300) ? 1.0 / v : 1.0;
	}
}

// r holds A x on entry: r = b - A x; z = M r; p = z; rz = r.z; res0 = |r|   (Solver.tpp:31-63)
__global__ void __launch_bounds__(256) k_fem_init(int64_t n, const double* __restrict__ b, double* __restrict__ r,
                                                  double* __restrict__ p, const double* __restrict__ invD, CgScal* S,
                                                  double* partials, double tol, int relMode, int64_t maxIters) {
	double v[2] = {0.0, 0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double ri = b[i] + (-1.0) * r[i];
		const double zi = invD ? ri * invD[i] : ri;
		r[i] = ri;
		p[i] = zi;
		v[0] += ri * ri;
		v[1] += ri * zi;
	}
	if (grid_sum<2>(v, partials, &S->ticket)) {
		const double res0 = sqrt(v[0]);
		S->res0 = res0; S->rz = v[1]; S->iter = 0; S->res = res0;
		S->refinements = 0; S->reliable = 0; S->status = 0;
		const double crit = relMode ? res0 / (res0 + 1e-50) : res0;
		if (crit < tol) { S->done = 1; S->converged = 1; }
		else if (maxIters <= 1) { S->done = 1; S->converged = 0; S->iter = maxIters; }
		else { S->done = 0; S->converged = 0; }
	}
}

// alpha = rz / p.Ap   (Solver.tpp:69-73), Ap from the element pass
__global__ void __launch_bounds__(256) k_fem_alpha(int64_t n, const double* __restrict__ p, const double* __restrict__ Ap,
                                                   CgScal* S, double* partials) {
	if (is_done(S)) return;
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		v[0] += p[i] * Ap[i];
	if (grid_sum<1>(v, partials, &S->ticket)) {
		S->pAp = v[0];
		S->alpha = S->rz / v[0];
		if (!isfinite(S->alpha)) { S->done = 1; S->converged = 0; S->status = RSD_EBREAKDOWN; }
	}
}

// |b - A x| into *out, A x in ax
__global__ void __launch_bounds__(256) k_fem_true_res(int64_t n, const double* __restrict__ b, const double* __restrict__ ax,
                                                      double* partials, unsigned* ticket, double* out) {
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double d = b[i] + (-1.0) * ax[i];
		v[0] += d * d;
	}
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

// Plain launches in chunks of 8 iterations behind a done-flag poll; after the solve has finished the
// remaining launches of a chunk return at once (the element pass through its skip flag).
static int cg_fem(rsd_ctx* ctx, rsd_heat* h, double coef, const rsd_solver_cfg* cfg, const double* b, double* x,
                  rsd_report* rep, int which, const double* state, double cTD, double cTM, const double* Udot) {
	const double* U = state ? state : x;   // the operator's state
	const int64_t n = h->n;
	void* wsv;
	const int64_t ns = pad_len(n);
	RSD_CHECK(get_ws(ctx, sizeof(double) * 4 * ns, &wsv));
	double* r = (double*)wsv;
	double* p = r + ns;
	double* Ap = p + ns;
	double* invD = cfg->precond == RSD_JACOBI ? Ap + ns : nullptr;
	const int xvec = reinterpret_cast<uintptr_t>(x) % 16 == 0;
	CgScal* S = scal_slot(ctx, 0);
	CgScal* S1 = scal_slot(ctx, 1);
	double* partials = ctx->s.partials;
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	const double tol = cfg->tol;
	const int64_t maxIt = cfg->max_iters;
	cudaStream_t st = ctx->stream;
	RSD_CUDA(cudaMemsetAsync(S, 0, sizeof(CgScal), st));
	// Jacobi::update on every solve (cg/Solver.tpp:22); the operator's state is the iterate x
	if (invD) {
		RSD_CHECK(assemble_diagonal(ctx, h, 1.0, coef, U, invD, which == 10 ? cTD : 0.0, which == 10 ? cTM : 0.0, Udot));
		k_inv_guarded<<<vec_grid(ctx, n), 256, 0, st>>>(n, invD);
	}
	RSD_CHECK(apply_operator(ctx, h, coef, U, x, r, nullptr, which, cTD, cTM, Udot));
	k_fem_init<<<VG(k_fem_init), 256, 0, st>>>(n, b, r, p, invD, S, partials, tol, rel, maxIt);
	RSD_CUDA(cudaGetLastError());
	Poller poll{ctx, S, (int32_t*)ctx->s.hbuf};
	RSD_CHECK(poll.init());
	const int chunk = 8;
	bool fin = false;
	const GraphCtl off{0, 0, 0, 0};
	for (int64_t it = 0; it < maxIt + 2 * chunk && !fin; it += chunk) {
		for (int c = 0; c < chunk; ++c) {
			RSD_CHECK(apply_operator(ctx, h, coef, U, p, Ap, &S->done, which, cTD, cTM, Udot));
			k_fem_alpha<<<VG(k_fem_alpha), 256, 0, st>>>(n, p, Ap, S, partials);
			k_cg_update<<<VGB(k_cg_update, kVT), kVT, 0, st>>>(n, x, r, p, Ap, invD, S, partials, tol, rel, maxIt, xvec);
			k_cg_pupdate<<<VGB(k_cg_pupdate, kVT), kVT, 0, st>>>(n, p, r, invD, S, off);
		}
		RSD_CUDA(cudaGetLastError());
		RSD_CHECK(poll.post(&fin));
	}
	RSD_CHECK(finish_report(ctx, S, rep));
	// FP64 check of the final iterate: ||b - A x||
	RSD_CHECK(apply_operator(ctx, h, coef, U, x, Ap, nullptr, which, cTD, cTM, Udot));
	k_fem_true_res<<<VG(k_fem_true_res), 256, 0, st>>>(n, b, Ap, partials, &S1->ticket, &S1->res);
	RSD_CUDA(cudaGetLastError());
	double hres = 0.0;
	RSD_CUDA(cudaMemcpyAsync(&hres, &S1->res, sizeof(double), cudaMemcpyDeviceToHost, st));
	RSD_CUDA(cudaStreamSynchronize(st));
	if (rep) rep->trueResidualRel = hres / (rep->initialResidual + 1e-50);
	return RSD_OK;
}

}  // namespace


void free_graph_cache(rsd_ctx* ctx) {
	if (!ctx->graphs) return;
	GraphCache* c = static_cast<GraphCache*>(ctx->graphs);
	for (CgGraph& g : c->cg) g.release();
	delete c;
	ctx->graphs = nullptr;
}

namespace {

// ---- GMRES(m): linalg/solver/iterative/gmres/Solver.tpp:3-170 ---------------------------------
// Right-preconditioned restarted GMRES.  Device: the preconditioned SpMV (Jacobi folded into the
// gather, w = A (M^-1 q)), the orthogonalization and the scalings; host: the (m+1) x m Hessenberg,
// Givens rotations and back substitution as the reference computes them (gmres/Solver.tpp:88-126), on
// the device: one thread applies the previous rotations to the new Hessenberg column, forms the next
// rotation, updates g and decides whether the cycle ends (convergence on |g_{j+1}|, breakdown, the
// iteration limit, a non-finite value); every kernel of the following steps reads that decision and
// returns at once, so the host launches a whole cycle without waiting and reads the outcome once per
// cycle.  The products and sums use explicit round-to-nearest operations (no fused multiply-add), the
// same arithmetic as the host loop they replace.
// Orthogonalization is classical Gram-Schmidt applied twice (CGS2): each pass is one kernel for
// all j+1 projections Q^T w and one for w -= Q h.  In exact arithmetic it equals the reference's
// modified Gram-Schmidt; in floating point CGS2 keeps the basis orthogonal to working precision as
// MGS does, with 4 launches per step instead of 2(j+1).
// T = double is FP64 GMRES; T = float is the mixed variant: FP32 matrix and Krylov basis, FP64
// reductions, x and the restart residual r = b - A64 x, convergence declared on that FP64 residual.

// w = A (M^-1 q) with M^-1 = diag(invD) (identity when invD is null)
template <int L, typename T>
__global__ void __launch_bounds__(256, 2 * kRowBlocks) k_gm_spmv(int64_t n, MatView<T> A, const T* __restrict__ q,
                                                 const T* __restrict__ invD, T* __restrict__ w, const int32_t* stop) {
	if (stop && *(volatile const int32_t*)stop) return;   // uniform over the launch
	const L2Pol pol = make_l2pol();
	const RowLoop<L> rl;
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const T s = row_sum<L, T, T>(A, row, n, rl.lane, pol, [&](int c) {
			return invD ? ldh(invD + c, pol.last) * ldh(q + c, pol.last) : ldh(q + c, pol.last);
		});
		if (rl.lane == 0 && row < n) sth(w + mat_row(A, row), s, pol.last);
	}
}

// h[i] = Q_i . w for i = blockIdx.y (FP64 accumulation; last-block-done reduction per i)
template <typename T>
__global__ void k_gm_mdot(int64_t n, const T* __restrict__ Q, int64_t ldq, const T* __restrict__ w, double* partials,
                          unsigned* tickets, double* h, const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	const int i = blockIdx.y;
	const T* __restrict__ qi = Q + (int64_t)i * ldq;
	double v[1] = {0.0};
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
		v[0] += (double)qi[e] * (double)w[e];
	if (grid_sum<1>(v, partials + (size_t)i * kMaxPartials, tickets + i)) h[i] = v[0];
}

// w -= sum_{i<k} h[i] Q_i (basis order)
template <typename T>
__global__ void k_gm_mupdate(int64_t n, const T* __restrict__ Q, int64_t ldq, int k, const double* __restrict__ h,
                             T* __restrict__ w, const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
		double s = (double)w[e];
		for (int i = 0; i < k; ++i) s -= h[i] * (double)Q[(int64_t)i * ldq + e];
		w[e] = (T)s;
	}
}

// The fused classical Gram-Schmidt passes for k <= KMAX basis vectors (k uniform over the launch):
// each thread keeps k running sums over its elements, a block sums them in a fixed tree (warp
// shuffles, then the warps in order), one partial per (sum, block), and the last block to arrive adds
// each sum's partials in block order (a warp per sum: lanes over strided partials, then a shuffle
// tree) into out[i].  Deterministic for a given grid.  256-thread blocks.
constexpr int kGmFusedThreads = 256, kGmFusedMax = 32;
template <int KMAX>
__device__ __forceinline__ void gm_multi_sum(double (&acc)[KMAX], int k, double* partials, unsigned* ticket, double* out) {
	__shared__ double sm[KMAX][kGmFusedThreads / 32];
	__shared__ bool last;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int i = 0; i < KMAX; ++i)
		if (i < k) {
			const double v = group_sum<32>(acc[i]);
			if (lane == 0) sm[i][warp] = v;
		}
	__syncthreads();
	if (threadIdx.x < k) {
		double s = 0.0;
		for (int wi = 0; wi < nw; ++wi) s += sm[threadIdx.x][wi];
		partials[(size_t)threadIdx.x * kMaxPartials + blockIdx.x] = s;
		__threadfence();
	}
	__syncthreads();
	if (threadIdx.x == 0) last = atomicInc(ticket, gridDim.x - 1) == gridDim.x - 1;
	__syncthreads();
	if (!last) return;
	__threadfence();
	for (int i = warp; i < k; i += nw) {
		double s = 0.0;
		for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(&partials[(size_t)i * kMaxPartials + b]);
		s = group_sum<32>(s);
		if (lane == 0) out[i] = s;
	}
}

// CGS pass 1: h[i] = Q_i . w for i < k, w read once per element
template <typename T, int KMAX>
__global__ void __launch_bounds__(kGmFusedThreads, 1) k_gm_mdot_k(int64_t n, const T* __restrict__ Q, int64_t ldq, int k,
                                                             const T* __restrict__ w, double* partials, unsigned* ticket,
                                                             double* h, const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	double acc[KMAX];
#pragma unroll
	for (int i = 0; i < KMAX; ++i) acc[i] = 0.0;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
		const double we = (double)w[e];
		// every load unconditional (sums past k read vector k - 1 again and are never reduced), so the
		// compiler issues them all before the first multiply-add
#pragma unroll
		for (int i = 0; i < KMAX; ++i) acc[i] += (double)__ldg(Q + (int64_t)min(i, k - 1) * ldq + e) * we;
	}
	gm_multi_sum<KMAX>(acc, k, partials, ticket, h);
}

// CGS pass 1's update fused with pass 2's dots: w -= sum_{i<k} h1[i] Q_i (basis order, FP64 per
// element, stored in T, as k_gm_mupdate), then h2[i] = Q_i . w with the stored w
template <typename T, int KMAX>
__global__ void __launch_bounds__(kGmFusedThreads, 1) k_gm_update_mdot(int64_t n, const T* __restrict__ Q, int64_t ldq, int k,
                                                                  const double* __restrict__ h1, T* __restrict__ w,
                                                                  double* partials, unsigned* ticket, double* h2,
                                                                  const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	__shared__ double hs[KMAX];
	if (threadIdx.x < KMAX) hs[threadIdx.x] = threadIdx.x < k ? h1[threadIdx.x] : 0.0;
	__syncthreads();
	double acc[KMAX];
#pragma unroll
	for (int i = 0; i < KMAX; ++i) acc[i] = 0.0;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
		double s = (double)w[e];
		// unconditional loads (past k: vector k - 1 again, times a zero coefficient, which leaves s
		// unchanged), so that they all issue before the first multiply-add
#pragma unroll
		for (int i = 0; i < KMAX; ++i) s -= hs[i] * (double)__ldg(Q + (int64_t)min(i, k - 1) * ldq + e);
		const T wn = (T)s;
		w[e] = wn;
		const double wd = (double)wn;
#pragma unroll
		for (int i = 0; i < KMAX; ++i) acc[i] += (double)__ldg(Q + (int64_t)min(i, k - 1) * ldq + e) * wd;
	}
	gm_multi_sum<KMAX>(acc, k, partials, ticket, h2);
}

// The Hessenberg least-squares state of one GMRES cycle on the device (gmres/Workspace.hpp:26-31)
struct GmState {
	int32_t stop, mLocal, status, breakdown;
	double tol, denom;    // |g_{j+1}| / denom < tol ends the cycle (denom: res0 + 1e-50 when relative, else 1)
	int64_t budget;       // Arnoldi steps this cycle may take (the iteration limit's remainder)
};

// Arnoldi step j: the new column (the two CGS passes' coefficients, hNext), the previous rotations, the
// next rotation, g; ends the cycle on convergence, breakdown (hNext <= 1e-14), the step budget or a
// non-finite g (gmres/Solver.tpp:88-110).  One warp: the lanes stage the column and the rotations in
// shared memory, lane 0 runs the rotations in order (the column entry it carries in a register), the
// lanes write the column back.
constexpr int kGmMaxDim = 256;
struct GmGivensArgs {
	GmState* S;
	int j, m;
	const double* h1;
	const double* h2;
	double *H, *cs, *sn, *g;
};
// run by one warp (lanes 0..31) with hNext, the new column's last entry, in *hNextp
__device__ __forceinline__ void gm_givens_warp(const GmGivensArgs& a, const double* __restrict__ hNextp) {
	__shared__ double hj[kGmMaxDim], c[kGmMaxDim], sv[kGmMaxDim];
	const int lane = threadIdx.x & 31, j = a.j;
	const int ld = a.m + 1;   // H column-major: H(i, j) at j * (m + 1) + i
	double* Hj = a.H + (int64_t)j * ld;
	for (int i = lane; i <= j; i += 32) hj[i] = __dadd_rn(a.h1[i], a.h2[i]);
	for (int i = lane; i < j; i += 32) { c[i] = a.cs[i]; sv[i] = a.sn[i]; }
	__syncwarp();
	if (lane == 0) {
		GmState* S = a.S;
		const double hNext = *hNextp;
		double x = hj[0];
		for (int i = 0; i < j; ++i) {
			const double b = hj[i + 1];
			hj[i] = __dadd_rn(__dmul_rn(c[i], x), __dmul_rn(sv[i], b));
			x = __dadd_rn(__dmul_rn(-sv[i], x), __dmul_rn(c[i], b));
		}
		const double hjj = x;
		const double denom = sqrt(__dadd_rn(__dmul_rn(hjj, hjj), __dmul_rn(hNext, hNext)));
		double cj, sj;
		if (denom <= 1e-14) { cj = 1.0; sj = 0.0; }
		else { cj = hjj / denom; sj = hNext / denom; }
		a.cs[j] = cj; a.sn[j] = sj;
		hj[j] = __dadd_rn(__dmul_rn(cj, hjj), __dmul_rn(sj, hNext));
		const double gj = a.g[j];
		a.g[j] = __dmul_rn(cj, gj);
		const double gn = __dmul_rn(-sj, gj);
		a.g[j + 1] = gn;
		S->mLocal = j + 1;
		const bool brk = hNext <= 1e-14;
		S->breakdown = brk;
		if (!isfinite(gn)) { S->status = RSD_EBREAKDOWN; S->stop = 1; }
		else if (fabs(gn) / S->denom < S->tol || brk || j + 1 >= S->budget || j + 1 >= a.m) S->stop = 1;
	}
	__syncwarp();
	for (int i = lane; i <= j; i += 32) Hj[i] = hj[i];
}

__global__ void __launch_bounds__(32) k_gm_givens(const GmGivensArgs a, const double* __restrict__ hNextp) {
	if (*(volatile const int32_t*)&a.S->stop) return;   // uniform over the warp
	gm_givens_warp(a, hNextp);
}

// CGS pass 2's update fused with the norm: w -= sum_{i<k} h2[i] Q_i, then out = ||w|| of the stored w;
// the last block to finish (it holds the norm) then runs the step's Givens update in its first warp
// when ga.S is set, which saves the step a launch of its own
template <typename T, int KMAX>
__global__ void __launch_bounds__(kGmFusedThreads, 1) k_gm_update_nrm(int64_t n, const T* __restrict__ Q, int64_t ldq, int k,
                                                                 const double* __restrict__ h2, T* __restrict__ w,
                                                                 double* partials, unsigned* ticket, double* out,
                                                                 const int32_t* stop, const GmGivensArgs ga) {
	if (*(volatile const int32_t*)stop) return;
	__shared__ double hs[KMAX];
	if (threadIdx.x < KMAX) hs[threadIdx.x] = threadIdx.x < k ? h2[threadIdx.x] : 0.0;
	__syncthreads();
	double v[1] = {0.0};
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
		double s = (double)w[e];
		// unconditional loads (past k: vector k - 1 again, times a zero coefficient, which leaves s
		// unchanged), so that they all issue before the first multiply-add
#pragma unroll
		for (int i = 0; i < KMAX; ++i) s -= hs[i] * (double)__ldg(Q + (int64_t)min(i, k - 1) * ldq + e);
		const T wn = (T)s;
		w[e] = wn;
		v[0] += (double)wn * (double)wn;
	}
	__shared__ int lastBlock;
	const bool last = grid_sum<1>(v, partials, ticket);   // thread 0 of the last block
	if (last) *out = sqrt(v[0]);
	if (ga.S) {
		if (threadIdx.x == 0) lastBlock = last;
		__syncthreads();
		if (lastBlock && threadIdx.x < 32) gm_givens_warp(ga, out);
	}
}

template <typename T, int KMAX>
static int gm_fused_k(rsd_ctx* ctx, int64_t n, const T* Q, int64_t ldq, int k, T* w, double* parts, unsigned* tk,
                      unsigned* tn, double* h1, double* h2, double* nrm, const int32_t* stop, const GmGivensArgs& ga) {
	cudaStream_t st = ctx->stream;
	const int g1 = wave_blocks(ctx, k_gm_mdot_k<T, KMAX>, kGmFusedThreads, n);
	const int g2 = wave_blocks(ctx, k_gm_update_mdot<T, KMAX>, kGmFusedThreads, n);
	const int g3 = wave_blocks(ctx, k_gm_update_nrm<T, KMAX>, kGmFusedThreads, n);
	k_gm_mdot_k<T, KMAX><<<g1, kGmFusedThreads, 0, st>>>(n, Q, ldq, k, w, parts, tk, h1, stop);
	k_gm_update_mdot<T, KMAX><<<g2, kGmFusedThreads, 0, st>>>(n, Q, ldq, k, h1, w, parts, tk, h2, stop);
	k_gm_update_nrm<T, KMAX><<<g3, kGmFusedThreads, 0, st>>>(n, Q, ldq, k, h2, w, parts, tn, nrm, stop, ga);
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}
template <typename T>
static int gm_fused(rsd_ctx* ctx, int64_t n, const T* Q, int64_t ldq, int k, T* w, double* parts, unsigned* tk,
                    unsigned* tn, double* h1, double* h2, double* nrm, const int32_t* stop, const GmGivensArgs& ga) {
	if (k <= 4) return gm_fused_k<T, 4>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
	if (k <= 8) return gm_fused_k<T, 8>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
	if (k <= 12) return gm_fused_k<T, 12>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
	if (k <= 16) return gm_fused_k<T, 16>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
	if (k <= 24) return gm_fused_k<T, 24>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
	return gm_fused_k<T, kGmFusedMax>(ctx, n, Q, ldq, k, w, parts, tk, tn, h1, h2, nrm, stop, ga);
}

// out = ||w||
template <typename T>
__global__ void k_gm_nrm2(int64_t n, const T* __restrict__ w, double* partials, unsigned* ticket, double* out,
                          const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	double v[1] = {0.0};
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
		v[0] += (double)w[e] * (double)w[e];
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

// q = w / hn unless breakdown (hn <= 1e-14)
template <typename T>
__global__ void k_gm_scale(int64_t n, const T* __restrict__ w, const double* __restrict__ hn, T* __restrict__ q,
                           const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	const double h = *hn;
	if (h <= 1e-14) return;
	const double s = 1.0 / h;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		q[i] = (T)((double)w[i] * s);
}

// q0 = (b - Ax) / beta in T, with beta read from the device
template <typename T>
__global__ void k_gm_start(int64_t n, const double* __restrict__ b, const double* __restrict__ Ax,
                           const double* __restrict__ beta, T* __restrict__ q) {
	const double s = 1.0 / *beta;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		q[i] = (T)((b[i] + (-1.0) * Ax[i]) * s);
}

// ||b - Ax||
__global__ void k_gm_resnorm(int64_t n, const double* __restrict__ b, const double* __restrict__ Ax, double* partials,
                             unsigned* ticket, double* out) {
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double r = b[i] + (-1.0) * Ax[i];
		v[0] += r * r;
	}
	if (grid_sum<1>(v, partials, ticket)) *out = sqrt(v[0]);
}

// back substitution H(0:m, 0:m) y = g(0:m) for the cycle's m = mLocal steps: one warp stages the
// triangle and g in shared memory, lane 0 solves in the serial order (cycles whose triangle does not
// fit solve from global memory)
constexpr int kGmBacksubDim = 64;
__global__ void __launch_bounds__(32) k_gm_backsub(const GmState* S, int m, const double* __restrict__ H,
                                                   const double* __restrict__ g, double* __restrict__ y) {
	__shared__ double Hs[kGmBacksubDim * (kGmBacksubDim + 1)], gs[kGmBacksubDim], ys[kGmBacksubDim];
	const int ml = S->mLocal, ld = m + 1, lane = threadIdx.x;
	// the triangle's columns 0..ml-1 span ml * ld entries (ld = m + 1): staged when they fit
	const bool staged = ml <= kGmBacksubDim && (int64_t)ml * ld <= (int64_t)kGmBacksubDim * (kGmBacksubDim + 1);
	if (staged) {
		for (int q = lane; q < ml * ld; q += 32) Hs[q] = H[q];   // columns 0..ml-1
		for (int i = lane; i < ml; i += 32) gs[i] = g[i];
	}
	__syncwarp();
	if (lane == 0) {
		const double* Hp = staged ? Hs : H;
		const double* gp = staged ? gs : g;
		double* yp = staged ? ys : y;
		for (int i = ml - 1; i >= 0; --i) {
			double s = gp[i];
			for (int k = i + 1; k < ml; ++k) s = __dsub_rn(s, __dmul_rn(Hp[(int64_t)k * ld + i], yp[k]));
			yp[i] = s / Hp[(int64_t)i * ld + i];
		}
	}
	__syncwarp();
	if (staged)
		for (int i = lane; i < ml; i += 32) y[i] = ys[i];
}

// x += M^-1 (sum_i y_i Q_i), accumulated in basis order in FP64, over the cycle's S->mLocal vectors
template <typename T>
__global__ void k_gm_update_x(int64_t n, const GmState* S, const T* __restrict__ Q, int64_t ldq, const double* __restrict__ yv,
                              const T* __restrict__ invD, double* __restrict__ x) {
	const int m = S->mLocal;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		double s = 0.0;
		for (int k = 0; k < m; ++k) s += yv[k] * (double)Q[(int64_t)k * ldq + i];
		x[i] += invD ? (double)invD[i] * s : s;
	}
}

template <typename T>
__global__ void k_gm_invdiag(int64_t n, const int32_t* __restrict__ dpos, const double* __restrict__ val, T* __restrict__ d) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t q = dpos[i];
		const double v = q >= 0 ? val[q] : 0.0;
		d[i] = (T)((fabs(v) > 1e-300) ? 1.0 / v : 1.0);
	}
}

// The operator of a GMRES solve: an assembled matrix (CSR/SELL, FP64 or its FP32 copy) ...
template <typename T>
struct GmCsrOp {
	rsd_ctx* ctx;
	rsd_csr* A;
	int64_t n;
	int prepare() { return sizeof(T) == 4 ? f32_sync(ctx, A) : exec_sync(ctx, A); }
	int invdiag(T* invD, const double*) {
		k_gm_invdiag<T><<<vec_grid(ctx, n), 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	}
	// w = A (M^-1 q); the launch returns at once when *stop != 0
	int prec_apply(const T* q, const T* invD, T* w, T*, const double*, const int32_t* stop) {
		const int L = exec_lanes(A);
		const MatView<T> V = exec_view<T>(A);
		RSD_DISPATCH_L(L, (k_gm_spmv<LL, T><<<wave_blocks(ctx, k_gm_spmv<LL, T>, 256, n * std::max(LL, 1)), 256, 0, ctx->stream>>>(n, V, q, invD, w, stop)));
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	}
	int apply64(const double* x, double* Ax) { return spmv_f64(ctx, A, x, Ax); }
};

// ... or the matrix-free operator (FEMOperator, FP64): every product an element pass with the
// iterate as the k(T) state, Jacobi from the element diagonal at the initial iterate
__global__ void k_gm_scale_by(int64_t n, const double* __restrict__ q, const double* __restrict__ d, double* __restrict__ out,
                              const int32_t* stop) {
	if (*(volatile const int32_t*)stop) return;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		out[i] = d ? q[i] * d[i] : q[i];
}
struct GmFemOp {
	rsd_ctx* ctx;
	rsd_heat* h;
	double coef;
	int64_t n;
	int which;
	const double* state;   // null: the iterate
	double cTD, cTM;       // TangentDiffusion / TangentMass coefficients of the Jacobian's product (which 10)
	const double* Udot;
	int prepare() { return RSD_OK; }
	int invdiag(double* invD, const double* x) {
		RSD_CHECK(assemble_diagonal(ctx, h, 1.0, coef, state ? state : x, invD, which == 10 ? cTD : 0.0, which == 10 ? cTM : 0.0, Udot));
		k_inv_guarded<<<vec_grid(ctx, n), 256, 0, ctx->stream>>>(n, invD);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	}
	int prec_apply(const double* q, const double* invD, double* w, double* tmp, const double* x, const int32_t* stop) {
		k_gm_scale_by<<<vec_grid(ctx, n), 256, 0, ctx->stream>>>(n, q, invD, tmp, stop);
		RSD_CUDA(cudaGetLastError());
		return apply_operator(ctx, h, coef, state ? state : x, tmp, w, stop, which, cTD, cTM, Udot);
	}
	int apply64(const double* x, double* Ax) { return apply_operator(ctx, h, coef, state ? state : x, x, Ax, nullptr, which, cTD, cTM, Udot); }
};

template <typename T, typename Op>
static int gmres_core(rsd_ctx* ctx, Op& op, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	constexpr bool kMixed = sizeof(T) == 4;
	const int64_t n = op.n;
	const int64_t m = std::max<int64_t>(1, cfg->krylov_dim);
	if (m + 1 > kGmMaxDim - 1) return set_error(RSD_EINVAL, "GMRES krylov_dim above 254");
	RSD_CHECK(op.prepare());
	const int64_t ns = pad_len(n);
	// workspace: Q (m+1 vectors), w, invD and a scratch vector in T; Ax in FP64; partials for m+1
	// reductions; tickets; H columns
	const size_t qBytes = sizeof(T) * (size_t)(m + 4) * ns;
	const size_t axBytes = sizeof(double) * (size_t)ns;
	const size_t pBytes = sizeof(double) * (size_t)(m + 1) * kMaxPartials;
	// the device least-squares state: H ((m + 1) m), cs, sn (m), g (m + 1), y (m), the two CGS passes'
	// coefficients (m + 2 each), the next norm, and the control block
	const size_t hBytes = sizeof(double) * (size_t)((m + 1) * m + 2 * m + (m + 1) + m + 2 * (m + 2) + 8) + sizeof(GmState) + 64;
	const size_t tBytes = sizeof(unsigned) * (size_t)(m + 2);
	void* wsv;
	RSD_CHECK(get_ws(ctx, qBytes + axBytes + pBytes + hBytes + tBytes + 1024, &wsv));
	char* base = (char*)wsv;
	T* Q = (T*)base;
	T* w = Q + (m + 1) * ns;
	T* invD = cfg->precond == RSD_JACOBI ? w + ns : nullptr;
	T* tmp = w + 2 * ns;
	double* Ax = (double*)(base + qBytes);
	double* parts = (double*)(base + qBytes + axBytes);
	double* dH = (double*)(base + qBytes + axBytes + pBytes);
	double* dCs = dH + (m + 1) * m;
	double* dSn = dCs + m;
	double* dG = dSn + m;
	double* dY = dG + (m + 1);
	double* dH1 = dY + m;
	double* dH2 = dH1 + (m + 2);
	double* dNorm = dH2 + (m + 2);
	GmState* dS = (GmState*)(((uintptr_t)(dNorm + 8) + 63) & ~uintptr_t(63));
	unsigned* tickets = (unsigned*)(base + qBytes + axBytes + pBytes + hBytes);
	cudaStream_t st = ctx->stream;
	RSD_CUDA(cudaMemsetAsync(tickets, 0, tBytes, st));
	const int gv = vec_grid(ctx, n), grd = red_grid(ctx, n);
	const bool relMode = cfg->tol_type == RSD_TOL_RELATIVE;
	const double eps = 1e-50;
	if (invD) RSD_CHECK(op.invdiag(invD, x));
	// FP64 residual of the current x; q0 = r / beta
	auto residual = [&](double* beta) -> int {
		RSD_CHECK(op.apply64(x, Ax));
		k_gm_resnorm<<<grd, kReduceThreads, 0, st>>>(n, b, Ax, parts, tickets + m + 1, dNorm);
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaMemcpyAsync(ctx->s.hbuf, dNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
		RSD_CUDA(cudaStreamSynchronize(st));
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
	int64_t total = 0, cycles = 0;
	double beta = res0;
	GmState* hS = reinterpret_cast<GmState*>(ctx->s.hbuf + 16);   // pinned staging
	while (total < cfg->max_iters) {
		// a cycle: g = (beta, 0, ...), the control block, q0; then every Arnoldi step launched at once
		GmState s0{};
		s0.tol = cfg->tol;
		s0.denom = relMode ? res0 + eps : 1.0;
		s0.budget = std::min<int64_t>(m, cfg->max_iters - total);
		*hS = s0;
		RSD_CUDA(cudaMemcpyAsync(dS, hS, sizeof(GmState), cudaMemcpyHostToDevice, st));
		RSD_CUDA(cudaMemsetAsync(dG, 0, sizeof(double) * (m + 1), st));
		RSD_CUDA(cudaMemcpyAsync(dG, dNorm, sizeof(double), cudaMemcpyDeviceToDevice, st));
		k_gm_start<T><<<gv, 256, 0, st>>>(n, b, Ax, dNorm, Q);
		++cycles;
		const int32_t* stop = &dS->stop;
		for (int64_t j = 0; j < s0.budget; ++j) {
			const T* qj = Q + j * ns;
			RSD_CHECK(op.prec_apply(qj, invD, w, tmp, x, stop));
			const int k = (int)(j + 1);
			if (k <= kGmFusedMax) {
				// the two CGS passes in three streaming kernels: dots; update + dots; update + norm
				// the Givens update runs in the last block of the third kernel
				const GmGivensArgs ga{dS, (int)j, (int)m, dH1, dH2, dH, dCs, dSn, dG};
				RSD_CHECK(gm_fused(ctx, n, Q, ns, k, w, parts, tickets + m, tickets + m + 1, dH1, dH2, dNorm, stop, ga));
			} else {
				for (double* dh : {dH1, dH2}) {
					k_gm_mdot<T><<<dim3(grd, k), kReduceThreads, 0, st>>>(n, Q, ns, w, parts, tickets, dh, stop);
					k_gm_mupdate<T><<<gv, 256, 0, st>>>(n, Q, ns, k, dh, w, stop);
				}
				k_gm_nrm2<T><<<grd, kReduceThreads, 0, st>>>(n, w, parts, tickets + m + 1, dNorm, stop);
			}
			if (k > kGmFusedMax) k_gm_givens<<<1, 32, 0, st>>>(GmGivensArgs{dS, (int)j, (int)m, dH1, dH2, dH, dCs, dSn, dG}, dNorm);
			// after the Givens update: a step that ended the cycle (stop) leaves q_{j+1}, which no one
			// reads, unwritten
			k_gm_scale<T><<<gv, 256, 0, st>>>(n, w, dNorm, Q + (j + 1) * ns, stop);
			RSD_CUDA(cudaGetLastError());
		}
		k_gm_backsub<<<1, 32, 0, st>>>(dS, (int)m, dH, dG, dY);
		k_gm_update_x<T><<<gv, 256, 0, st>>>(n, dS, Q, ns, dY, invD, x);
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaMemcpyAsync(hS, dS, sizeof(GmState), cudaMemcpyDeviceToHost, st));
		RSD_CHECK(residual(&beta));   // synchronizes: the control block is on the host too
		total += hS->mLocal;
		if (hS->status) R.status = hS->status;
		if (R.status || converged(beta) || total >= cfg->max_iters) break;
		if (hS->breakdown && !kMixed) break;   // FP64: the Krylov space is exhausted; mixed: restart in FP64
	}
	R.converged = R.status ? 0 : converged(beta);
	R.finalResidual = beta;
	R.finalResidualRel = beta / (res0 + eps);
	R.iterations = total;
	R.trueResidualRel = beta / (res0 + eps);
	R.refinements = kMixed ? cycles : 0;
	if (rep) *rep = R;
	return RSD_OK;
}

template <typename T>
static int gmres_run(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	GmCsrOp<T> op{ctx, A, A->n};
	return gmres_core<T>(ctx, op, cfg, b, x, rep);
}

// ---- FP64 PCG over a static device scratch ---------------------------------------------------
// The same kernels, grids and reductions as cg_fp64 (so the same iterates, bit for bit), with every
// scratch buffer carved from one file-scope device array instead of the context's workspace: the
// call allocates nothing.  The array is sized for kStaticMaxRows rows; one array per device, shared
// by every call on that device.
constexpr int64_t kStaticMaxRows = int64_t(1) << 18;                 // 262,144 rows (a multiple of 64)
constexpr size_t kStaticHeadBytes = 2 * sizeof(DevScalars) + sizeof(double) * 2 * kMaxPartials;
constexpr size_t kStaticHeadAligned = (kStaticHeadBytes + 255) & ~size_t(255);
constexpr size_t kStaticScratchBytes = kStaticHeadAligned + sizeof(double) * 4 * kStaticMaxRows;   // 8 MiB + 19 KiB
static_assert(sizeof(DevScalars) % 8 == 0, "the partials after the two scalar slots stay 8-byte aligned");

}  // namespace

static __device__ __align__(256) unsigned char g_cg_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kStaticMaxDevices = 64;
static std::mutex g_static_mu;
// the static scratch's device address per device, looked up on the first call and kept for the life
// of the process: it assumes the primary context outlives every call (no cudaDeviceReset between them)
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
	const int64_t ns = pad_len(n);   // kStaticMaxRows is a multiple of the padding
	double* r = reinterpret_cast<double*>(base + kStaticHeadAligned);
	double* p = r + ns;
	double* Ap = p + ns;
	double* invD = cfg->precond == RSD_JACOBI ? Ap + ns : nullptr;
	const int xvec = reinterpret_cast<uintptr_t>(x) % 16 == 0;
	// the reduction tickets and the done/converged flags must start at zero on every call
	RSD_CUDA(cudaMemsetAsync(base, 0, 2 * sizeof(DevScalars), ctx->stream));
	RSD_CHECK(exec_sync(ctx, A));
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	if (invD) k_invdiag64<<<VG(k_invdiag64), 256, 0, ctx->stream>>>(n, exec_diag(A), exec_val(A), invD);
	RSD_DISPATCH_L(L, (k_cg_init<LL><<<RG(k_cg_init<LL>), 256, 0, ctx->stream>>>(n, V, b, x, r, p, invD, S, partials, cfg->tol, rel, cfg->max_iters)));
	RSD_CUDA(cudaGetLastError());
	const int chunk = 8;
	for (int64_t it = 0; it < cfg->max_iters + 2 * chunk; it += chunk) {
		for (int c = 0; c < chunk; ++c) {
			RSD_DISPATCH_L(L, (k_cg_spmv_dot<LL><<<RGB(k_cg_spmv_dot<LL>, kST), kST, 0, ctx->stream>>>(n, V, p, Ap, S, partials)));
			k_cg_update<<<VGB(k_cg_update, kVT), kVT, 0, ctx->stream>>>(n, x, r, p, Ap, invD, S, partials, cfg->tol, rel, cfg->max_iters, xvec);
			k_cg_pupdate<<<VGB(k_cg_pupdate, kVT), kVT, 0, ctx->stream>>>(n, p, r, invD, S, GraphCtl{0, 0, 0, 0});
		}
		RSD_CUDA(cudaGetLastError());
		int32_t done = 0;   // pageable host word: the copy returns once the flag has been read
		RSD_CUDA(cudaMemcpyAsync(&done, &S->done, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		if (done) break;
	}
	RSD_CHECK(finish_report(ctx, S, rep));
	double* tr = &S1->res;
	RSD_DISPATCH_L(L, (k_true_res<LL><<<RG(k_true_res<LL>), 256, 0, ctx->stream>>>(n, V, b, x, partials, &S1->ticket, tr)));
	RSD_CUDA(cudaGetLastError());
	double h = 0.0;
	RSD_CUDA(cudaMemcpyAsync(&h, tr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (rep) rep->trueResidualRel = h / (rep->initialResidual + 1e-50);
	return RSD_OK;
}

}  // namespace

int solve_fem(rsd_ctx* ctx, rsd_heat* h, double coef, const rsd_solver_cfg* cfg, const double* b, double* x,
              rsd_report* rep, int which, const double* state, double cTD, double cTM, const double* Udot) {
	if (!ctx || !h || !cfg || (h->n && (!b || !x))) return set_error(RSD_EINVAL, "null argument");
	if (cfg->max_iters < 0 || !(cfg->tol >= 0)) return set_error(RSD_EINVAL, "bad solver configuration");
	if (cfg->type != RSD_CG && cfg->type != RSD_GMRES) return set_error(RSD_EINVAL, "unknown solver type");
	if (cfg->precision != RSD_FP64) return set_error(RSD_EINVAL, "the matrix-free operator solves in FP64 (precision RSD_FP64)");
	if (cfg->type == RSD_GMRES && cfg->krylov_dim <= 0) return set_error(RSD_EINVAL, "GMRES needs krylov_dim >= 1");
	if (rep) *rep = rsd_report{};
	if (h->n == 0) { if (rep) rep->converged = 1; return RSD_OK; }
	RSD_CUDA(cudaSetDevice(ctx->device));
	if (cfg->type == RSD_GMRES) {
		GmFemOp op{ctx, h, coef, h->n, which, state, cTD, cTM, Udot};
		return gmres_core<double>(ctx, op, cfg, b, x, rep);
	}
	return cg_fem(ctx, h, coef, cfg, b, x, rep, which, state, cTD, cTM, Udot);
}

int solve(rsd_ctx* ctx, rsd_csr* A, const rsd_solver_cfg* cfg, const double* b, double* x, rsd_report* rep) {
	if (!ctx || !A || !cfg || (A->n && (!b || !x))) return set_error(RSD_EINVAL, "null argument");
	if (cfg->max_iters < 0 || !(cfg->tol >= 0)) return set_error(RSD_EINVAL, "bad solver configuration");
	if (cfg->operator_type != RSD_OP_CSR)
		return set_error(RSD_EINVAL, "a matrix solve takes operator_type RSD_OP_CSR (the matrix-free operator is rsd_heat_solve_fem)");
	if (rep) *rep = rsd_report{};
	if (A->n == 0) { if (rep) rep->converged = 1; return RSD_OK; }
	RSD_CUDA(cudaSetDevice(ctx->device));
	if (cfg->type == RSD_CG) return cfg->precision == RSD_MIXED ? cg_mixed(ctx, A, cfg, b, x, rep) : cg_fp64(ctx, A, cfg, b, x, rep);
	if (cfg->type == RSD_GMRES) {
		if (cfg->krylov_dim <= 0) return set_error(RSD_EINVAL, "GMRES needs krylov_dim >= 1");
		return cfg->precision == RSD_MIXED ? gmres_run<float>(ctx, A, cfg, b, x, rep) : gmres_run<double>(ctx, A, cfg, b, x, rep);
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
	if (cfg->type != RSD_CG || cfg->precision != RSD_FP64 || cfg->operator_type != RSD_OP_CSR)
		return set_error(RSD_EINVAL, "rsd_cg_solve_static runs FP64 CG on a matrix only (type RSD_CG, precision RSD_FP64, operator_type RSD_OP_CSR)");
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
