// BLAS-1, deterministic reductions, SpMV (SELL-32 and CSR-vector, FP64 / FP32), layout syncs,
// diagonal, lump, Jacobi setup and the SpMV launch autotuner.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {

// ---------------------------------------------------------------------------------------------
// vector kernels: operations::axpy/axpby/scal/copy/multiply (linalg/operations/backend/cpu/VectorOps.tpp)
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_fill(T* x, int64_t n, T v) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = v;
}
__global__ void k_axpby(int64_t n, double a, double b, const double* __restrict__ x, double* __restrict__ y) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] = b * y[i] + a * x[i];
}
__global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] += a * x[i];
}
__global__ void k_scal(int64_t n, double a, double* __restrict__ x) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] *= a;
}
__global__ void k_mul(int64_t n, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ z) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) z[i] = x[i] * y[i];
}

// dot product with the deterministic grid reduction; the total lands in *out (device)
__global__ void k_dot(int64_t n, const double* __restrict__ x, const double* __restrict__ y, double* partials,
                      unsigned* ticket, double* out) {
	double v[1] = {0.0};
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) v[0] += x[i] * y[i];
	if (grid_sum<1>(v, partials, ticket)) *out = v[0];
}

int dot_device(rsd_ctx* ctx, int64_t n, const double* x, const double* y, double* host_out) {
	k_dot<<<red_grid(ctx, n), kReduceThreads, 0, ctx->stream>>>(n, x, y, ctx->s.partials, &ctx->s.scal[3].ticket, &ctx->s.scal[3].spare0);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaMemcpyAsync(ctx->s.hbuf, &ctx->s.scal[3].spare0, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	*host_out = ctx->s.hbuf[0];
	return RSD_OK;
}

// ---------------------------------------------------------------------------------------------
// layout syncs between CSR (API order) and SELL-32 (execution order)
// ---------------------------------------------------------------------------------------------
__global__ void k_sell_from_csr(int64_t ssize, const int32_t* __restrict__ src, const double* __restrict__ val, double* __restrict__ sval) {
	for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ssize; s += (int64_t)gridDim.x * blockDim.x) {
		const int32_t q = src[s];
		sval[s] = q >= 0 ? val[q] : 0.0;
	}
}
__global__ void k_csr_from_sell(int64_t ssize, const int32_t* __restrict__ src, const double* __restrict__ sval, double* __restrict__ val) {
	for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < ssize; s += (int64_t)gridDim.x * blockDim.x) {
		const int32_t q = src[s];
		if (q >= 0) val[q] = sval[s];
	}
}
__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

int sell_sync(rsd_ctx* ctx, rsd_csr* A) {
	if (A->sellValid) return RSD_OK;
	if (A->ssize) {
		k_sell_from_csr<<<vec_grid(ctx, A->ssize), 256, 0, ctx->stream>>>(A->ssize, A->sSrc, A->val, A->sVal);
		RSD_CUDA(cudaGetLastError());
	}
	A->sellValid = true;
	return RSD_OK;
}

int csr_sync(rsd_ctx* ctx, rsd_csr* A) {
	if (A->csrValid) return RSD_OK;
	if (A->ssize) {
		k_csr_from_sell<<<vec_grid(ctx, A->ssize), 256, 0, ctx->stream>>>(A->ssize, A->sSrc, A->sVal, A->val);
		RSD_CUDA(cudaGetLastError());
	}
	A->csrValid = true;
	return RSD_OK;
}

int exec_sync(rsd_ctx* ctx, rsd_csr* A) { return A->format == 0 ? sell_sync(ctx, A) : csr_sync(ctx, A); }

int f32_sync(rsd_ctx* ctx, rsd_csr* A) {
	RSD_CHECK(exec_sync(ctx, A));
	if (!A->val32) RSD_CUDA(cudaMalloc(&A->val32, sizeof(float) * std::max<int64_t>(std::max(A->ssize, A->nnz), 1)));
	if (A->version32 == A->version && A->fmt32 == A->format) return RSD_OK;
	const int64_t len = A->format == 0 ? A->ssize : A->nnz;
	if (len) {
		k_to_f32<<<vec_grid(ctx, len), 256, 0, ctx->stream>>>(len, exec_val(A), A->val32);
		RSD_CUDA(cudaGetLastError());
	}
	A->version32 = A->version;
	A->fmt32 = A->format;
	return RSD_OK;
}

// ---------------------------------------------------------------------------------------------
// SpMV: operations::matvec (linalg/operations/backend/cpu/MatrixOps.tpp:5-23), SELL-32 (L == 0,
// a warp per slice) or CSR-vector (L lanes per row)
// ---------------------------------------------------------------------------------------------
template <int L, typename T>
__global__ void __launch_bounds__(512, kRowBlocks) k_spmv(int64_t n, MatView<T> A, const T* __restrict__ x, T* __restrict__ y) {
	const L2Pol pol = make_l2pol();
	RowLoop<L> rl;
	for (int64_t base = rl.base; base < n; base += rl.step) {
		const int64_t row = base + rl.sub;
		const T s = row_dot<L, T, T>(A, x, row, n, rl.lane, pol);
		if (rl.lane == 0 && row < n) sth(y + mat_row(A, row), s, pol.first);
	}
}

int default_lanes(const rsd_csr* A) {
	if (A->lanes) return A->lanes;
	const double avg = A->n ? (double)A->nnz / (double)A->n : 1.0;
	if (avg <= 6) return 2;
	if (avg <= 40) return 4;
	if (avg <= 96) return 8;
	return 16;
}

// one full wave of the kernel's resident blocks (grid-stride loop over the rows)
#define SPMV_GRID(kern, L, block) wave_blocks(ctx, kern, block, A->n * std::max(L, 1), INT64_MAX)

int spmv_f64(rsd_ctx* ctx, const rsd_csr* Ac, const double* x, double* y) {
	rsd_csr* A = const_cast<rsd_csr*>(Ac);
	if (A->n == 0) return RSD_OK;
	RSD_CHECK(exec_sync(ctx, A));
	const int block = A->block ? A->block : 256;
	const int L = exec_lanes(A);
	const MatView<double> V = view64(A);
	RSD_DISPATCH_L(L, (k_spmv<LL, double><<<SPMV_GRID((k_spmv<LL, double>), LL, block), block, 0, ctx->stream>>>(A->n, V, x, y)));
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

int spmv_f32(rsd_ctx* ctx, const rsd_csr* Ac, const float* x, float* y) {
	rsd_csr* A = const_cast<rsd_csr*>(Ac);
	if (A->n == 0) return RSD_OK;
	RSD_CHECK(f32_sync(ctx, A));
	const int block = A->block ? A->block : 256;
	const int L = exec_lanes(A);
	const MatView<float> V = view32(A);
	RSD_DISPATCH_L(L, (k_spmv<LL, float><<<SPMV_GRID((k_spmv<LL, float>), LL, block), block, 0, ctx->stream>>>(A->n, V, x, y)));
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

// CSROperator::diagonal (linalg/operator/CSROperator.hpp:40-45) through the precomputed diagonal
// slot; Jacobi::update's inverse (linalg/solver/preconditioner/Jacobi.hpp:31-34) when invert is set
__global__ void k_diag(int64_t n, const int32_t* __restrict__ dpos, const double* __restrict__ val, double* __restrict__ d, int invert) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t p = dpos[i];
		const double v = p >= 0 ? val[p] : 0.0;
		d[i] = invert ? ((fabs(v) > 1e-300) ? 1.0 / v : 1.0) : v;
	}
}

// operations::lump (MatrixOps.tpp:25-43): row sums over the SELL-32 layout (padding adds zeros)
__global__ void k_lump(int64_t n, MatView<double> A, double* __restrict__ d) {
	const L2Pol pol = make_l2pol();
	for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x)
		d[mat_row(A, row)] = row_sum<0, double, double>(A, row, n, 0, pol, [](int) { return 1.0; });
}

}  // namespace rsd

using namespace rsd;

extern "C" {

int rsd_fill_f64(rsd_ctx* c, double* x, int64_t n, double v) {
	if (!c || (n && !x)) return set_error(RSD_EINVAL, "null argument");
	if (!n) return RSD_OK;
	k_fill<double><<<vec_grid(c, n), 256, 0, c->stream>>>(x, n, v);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_fill_f32(rsd_ctx* c, float* x, int64_t n, float v) {
	if (!c || (n && !x)) return set_error(RSD_EINVAL, "null argument");
	if (!n) return RSD_OK;
	k_fill<float><<<vec_grid(c, n), 256, 0, c->stream>>>(x, n, v);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_dot(rsd_ctx* c, int64_t n, const double* x, const double* y, double* out) {
	if (!c || !out || (n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	return dot_device(c, n, x, y, out);
}

int rsd_nrm2(rsd_ctx* c, int64_t n, const double* x, double* out) {
	double d = 0.0;
	RSD_CHECK(rsd_dot(c, n, x, x, &d));
	*out = std::sqrt(d);
	return RSD_OK;
}

#define RSD_VEC_LAUNCH(kernel, ...)                                        \
	do {                                                                   \
		if (!n) return RSD_OK;                                             \
		kernel<<<vec_grid(c, n), 256, 0, c->stream>>>(n, __VA_ARGS__);     \
		RSD_CUDA(cudaGetLastError());                                      \
		RSD_CUDA(cudaStreamSynchronize(c->stream));                        \
		return RSD_OK;                                                     \
	} while (0)

int rsd_axpy(rsd_ctx* c, int64_t n, double a, const double* x, double* y) {
	if (!c || (n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	RSD_VEC_LAUNCH(k_axpy, a, x, y);
}
int rsd_axpby(rsd_ctx* c, int64_t n, double a, double b, const double* x, double* y) {
	if (!c || (n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	RSD_VEC_LAUNCH(k_axpby, a, b, x, y);
}
int rsd_scal(rsd_ctx* c, int64_t n, double a, double* x) {
	if (!c || (n && !x)) return set_error(RSD_EINVAL, "null argument");
	RSD_VEC_LAUNCH(k_scal, a, x);
}
int rsd_copy(rsd_ctx* c, int64_t n, const double* x, double* y) {
	if (!c || (n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	if (!n) return RSD_OK;
	RSD_CUDA(cudaMemcpyAsync(y, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}
int rsd_mul(rsd_ctx* c, int64_t n, const double* x, const double* y, double* z) {
	if (!c || (n && (!x || !y || !z))) return set_error(RSD_EINVAL, "null argument");
	RSD_VEC_LAUNCH(k_mul, x, y, z);
}

int rsd_spmv(rsd_ctx* c, const rsd_csr* A, const double* x, double* y) {
	if (!c || !A || (A->n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	const int pr = prof_begin(c, PF_SPMV);
	RSD_CHECK(spmv_f64(c, A, x, y));
	prof_end(c, pr);
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_sync_f32(rsd_ctx* c, rsd_csr* A) {
	if (!c || !A) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(f32_sync(c, A));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_spmv_f32(rsd_ctx* c, const rsd_csr* A, const float* x, float* y) {
	if (!c || !A || (A->n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	if (!A->val32) return set_error(RSD_EINVAL, "FP32 values not created: call rsd_csr_sync_f32 first");
	RSD_CHECK(spmv_f32(c, A, x, y));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_diagonal(rsd_ctx* c, const rsd_csr* Ac, double* d) {
	rsd_csr* A = const_cast<rsd_csr*>(Ac);
	if (!c || !A || (A->n && !d)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	RSD_CHECK(exec_sync(c, A));
	k_diag<<<vec_grid(c, A->n), 256, 0, c->stream>>>(A->n, exec_diag(A), exec_val(A), d, 0);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_jacobi_setup(rsd_ctx* c, const rsd_csr* Ac, double* invD) {
	rsd_csr* A = const_cast<rsd_csr*>(Ac);
	if (!c || !A || (A->n && !invD)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	RSD_CHECK(exec_sync(c, A));
	k_diag<<<vec_grid(c, A->n), 256, 0, c->stream>>>(A->n, exec_diag(A), exec_val(A), invD, 1);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_lump(rsd_ctx* c, const rsd_csr* Ac, double* d) {
	rsd_csr* A = const_cast<rsd_csr*>(Ac);
	if (!c || !A || (A->n && !d)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	RSD_CHECK(sell_sync(c, A));
	k_lump<<<vec_grid(c, A->n), 256, 0, c->stream>>>(A->n, MatView<double>{A->sStart, A->sCol, A->sVal, nullptr, nullptr, nullptr, nullptr, A->sPerm}, d);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

}  // extern "C" (reopened below)

namespace rsd {
// eight independent FMA chains per thread; the sum is stored only under a condition the host never
// meets, so that the chains are not removed
__global__ void __launch_bounds__(256) k_fma64(double* out, int iters, double a, double b) {
	double x[8];
#pragma unroll
	for (int k = 0; k < 8; ++k) x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
	for (int i = 0; i < iters; ++i)
#pragma unroll
		for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
	double s = 0.0;
#pragma unroll
	for (int k = 0; k < 8; ++k) s += x[k];
	if (s == -1.0) out[0] = s;
}
}  // namespace rsd

extern "C" {

int rsd_measure_fp64_rate(rsd_ctx* c, double* tflops) {
	if (!c || !tflops) return set_error(RSD_EINVAL, "null argument");
	const int iters = 4096, threads = 256, blocks = c->num_sms * 8;
	cudaEvent_t e0, e1;
	RSD_CUDA(cudaEventCreate(&e0));
	RSD_CUDA(cudaEventCreate(&e1));
	float best = 1e30f;
	for (int rep = 0; rep < 4; ++rep) {
		RSD_CUDA(cudaEventRecord(e0, c->stream));
		k_fma64<<<blocks, threads, 0, c->stream>>>(c->s.partials, iters, 0.9999999, 1e-9);
		RSD_CUDA(cudaEventRecord(e1, c->stream));
		RSD_CUDA(cudaEventSynchronize(e1));
		float ms = 0.0f;
		RSD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
		if (rep > 0) best = std::min(best, ms);   // the first launch warms up
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	*tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e12;
	return RSD_OK;
}

// SpMV launch autotuner: times SELL-32 and CSR-vector with 2..32 lanes per row, each at 128, 256
// and 512 threads per block, with CUDA events (median of 5 launches after 2 warm-ups), and keeps
// the fastest in A's launch settings.
int rsd_csr_autotune(rsd_ctx* c, rsd_csr* A, int32_t* lanes_out, int32_t* block_out, double* best_us) {
	if (!c || !A) return set_error(RSD_EINVAL, "null argument");
	if (A->n == 0) { if (lanes_out) *lanes_out = 0; if (block_out) *block_out = 256; if (best_us) *best_us = 0; return RSD_OK; }
	double *x = nullptr, *y = nullptr;
	RSD_CUDA(cudaMalloc(&x, sizeof(double) * A->n));
	RSD_CUDA(cudaMalloc(&y, sizeof(double) * A->n));
	k_fill<double><<<vec_grid(c, A->n), 256, 0, c->stream>>>(x, A->n, 1.0);
	RSD_CHECK(sell_sync(c, A));
	RSD_CHECK(csr_sync(c, A));
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	const int lanes[] = {0, 2, 4, 8, 16, 32};   // 0: SELL-32
	const int blocks[] = {128, 256, 512};
	int bestL = 0, bestB = 256;
	double best = 1e30;
	const int savedF = A->format, savedL = A->lanes, savedB = A->block;
	int rc = RSD_OK;
	for (int L : lanes)
		for (int B : blocks) {
			A->format = L ? 1 : 0; A->lanes = L; A->block = B;
			std::vector<float> ts;
			for (int rep = 0; rep < 7 && rc == RSD_OK; ++rep) {
				cudaEventRecord(e0, c->stream);
				rc = spmv_f64(c, A, x, y);
				cudaEventRecord(e1, c->stream);
				cudaEventSynchronize(e1);
				float ms = 0.f;
				cudaEventElapsedTime(&ms, e0, e1);
				if (rep >= 2) ts.push_back(ms);
			}
			if (rc != RSD_OK) break;
			std::sort(ts.begin(), ts.end());
			const double us = 1e3 * ts[ts.size() / 2];
			if (us < best) { best = us; bestL = L; bestB = B; }
		}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(x);
	cudaFree(y);
	if (rc != RSD_OK) { A->format = savedF; A->lanes = savedL; A->block = savedB; return rc; }
	A->format = bestL ? 1 : 0;
	A->lanes = bestL;
	A->block = bestB;
	if (lanes_out) *lanes_out = bestL;
	if (block_out) *block_out = bestB;
	if (best_us) *best_us = best;
	return RSD_OK;
}

}  // extern "C"
