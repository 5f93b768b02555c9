// BLAS-1, deterministic reductions, CSR SpMV (FP64 / FP32), diagonal, lump and Jacobi setup.
#include <algorithm>
#include <cmath>

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
// SpMV: operations::matvec (linalg/operations/backend/cpu/MatrixOps.tpp:5-23) as vector-CSR:
// a group of L lanes per row, streaming 4-byte columns and 8/4-byte values, x through L2.
// ---------------------------------------------------------------------------------------------
template <int L, typename T>
__global__ void __launch_bounds__(256) k_spmv(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                              const T* __restrict__ val, const T* __restrict__ x, T* __restrict__ y) {
	const int lane = threadIdx.x & (L - 1);
	const int64_t g0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / L;
	const int64_t gs = ((int64_t)gridDim.x * blockDim.x) / L;
	// warp-uniform trip count: the whole warp iterates while any of its groups has a row
	const int64_t warp0 = g0 - ((threadIdx.x & 31) / L);
	for (int64_t base = warp0; base < n; base += gs) {
		const int64_t row = base + ((threadIdx.x & 31) / L);
		const T s = csr_row<L, T, T>(rp, col, val, x, row, n, lane);
		if (lane == 0 && row < n) y[row] = s;
	}
}

int default_lanes(const rsd_csr* A) {
	if (A->lanes) return A->lanes;
	const double avg = A->n ? (double)A->nnz / (double)A->n : 1.0;
	if (avg <= 6) return 2;
	if (avg <= 14) return 4;
	if (avg <= 40) return 4;
	if (avg <= 96) return 8;
	return 16;
}

template <typename T>
static int spmv_t(rsd_ctx* ctx, const rsd_csr* A, const T* val, const T* x, T* y) {
	if (A->n == 0) return RSD_OK;
	const int L = default_lanes(A);
	const int block = A->block ? A->block : 256;
	int64_t blocks = (A->n * L + block - 1) / block;
	blocks = std::min<int64_t>(blocks, (int64_t)ctx->num_sms * (2048 / block));
	dim3 g((unsigned)std::max<int64_t>(blocks, 1));
	switch (L) {
		case 1: k_spmv<1, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
		case 2: k_spmv<2, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
		case 4: k_spmv<4, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
		case 8: k_spmv<8, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
		case 16: k_spmv<16, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
		default: k_spmv<32, T><<<g, block, 0, ctx->stream>>>(A->n, A->rowPtr, A->col, val, x, y); break;
	}
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

int spmv_f64(rsd_ctx* ctx, const rsd_csr* A, const double* x, double* y) { return spmv_t<double>(ctx, A, A->val, x, y); }
int spmv_f32(rsd_ctx* ctx, const rsd_csr* A, const float* x, float* y) { return spmv_t<float>(ctx, A, A->val32, x, y); }

__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// CSROperator::diagonal (linalg/operator/CSROperator.hpp:40-45) via the precomputed diagonal slot;
// a missing diagonal is an error in the reference (std::out_of_range) and 0 here, flagged by the caller
__global__ void k_diag(int64_t n, const int32_t* __restrict__ dpos, const double* __restrict__ val, double* __restrict__ d, int invert) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t p = dpos[i];
		const double v = p >= 0 ? val[p] : 0.0;
		// Jacobi::update (linalg/solver/preconditioner/Jacobi.hpp:31-34)
		d[i] = invert ? ((fabs(v) > 1e-300) ? 1.0 / v : 1.0) : v;
	}
}

// operations::lump (MatrixOps.tpp:25-43): row sums, one group of 4 lanes per row
__global__ void k_lump(int64_t n, const int32_t* __restrict__ rp, const double* __restrict__ val, double* __restrict__ d) {
	const int lane = threadIdx.x & 3;
	const int64_t g0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 4, gs = ((int64_t)gridDim.x * blockDim.x) / 4;
	const int64_t warp0 = g0 - ((threadIdx.x & 31) / 4);
	for (int64_t base = warp0; base < n; base += gs) {
		const int64_t row = base + ((threadIdx.x & 31) / 4);
		double s = 0.0;
		if (row < n) for (int p = rp[row] + lane; p < rp[row + 1]; p += 4) s += val[p];
		s = group_sum<4>(s);
		if (lane == 0 && row < n) d[row] = s;
	}
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
	RSD_CHECK(spmv_f64(c, A, x, y));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_sync_f32(rsd_ctx* c, rsd_csr* A) {
	if (!c || !A) return set_error(RSD_EINVAL, "null argument");
	if (!A->val32) RSD_CUDA(cudaMalloc(&A->val32, sizeof(float) * std::max<int64_t>(A->nnz, 1)));
	if (A->nnz) {
		k_to_f32<<<vec_grid(c, A->nnz), 256, 0, c->stream>>>(A->nnz, A->val, A->val32);
		RSD_CUDA(cudaGetLastError());
	}
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	A->version32 = A->version;
	return RSD_OK;
}

int rsd_spmv_f32(rsd_ctx* c, const rsd_csr* A, const float* x, float* y) {
	if (!c || !A || (A->n && (!x || !y))) return set_error(RSD_EINVAL, "null argument");
	if (!A->val32) return set_error(RSD_EINVAL, "FP32 values not created: call rsd_csr_sync_f32 first");
	RSD_CHECK(spmv_f32(c, A, x, y));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_diagonal(rsd_ctx* c, const rsd_csr* A, double* d) {
	if (!c || !A || (A->n && !d)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	k_diag<<<vec_grid(c, A->n), 256, 0, c->stream>>>(A->n, A->diag, A->val, d, 0);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_jacobi_setup(rsd_ctx* c, const rsd_csr* A, double* invD) {
	if (!c || !A || (A->n && !invD)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	k_diag<<<vec_grid(c, A->n), 256, 0, c->stream>>>(A->n, A->diag, A->val, invD, 1);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

// SpMV launch autotuner: times every lanes-per-row x block combination on this matrix with CUDA
// events (median of 5 launches after 2 warm-ups) and keeps the fastest in A's launch settings.
int rsd_csr_autotune(rsd_ctx* c, rsd_csr* A, int32_t* lanes_out, int32_t* block_out, double* best_us) {
	if (!c || !A) return set_error(RSD_EINVAL, "null argument");
	if (A->n == 0) { if (lanes_out) *lanes_out = 2; if (block_out) *block_out = 256; if (best_us) *best_us = 0; return RSD_OK; }
	double *x = nullptr, *y = nullptr;
	RSD_CUDA(cudaMalloc(&x, sizeof(double) * A->n));
	RSD_CUDA(cudaMalloc(&y, sizeof(double) * A->n));
	k_fill<double><<<vec_grid(c, A->n), 256, 0, c->stream>>>(x, A->n, 1.0);
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	const int lanes[] = {2, 4, 8, 16, 32};
	const int blocks[] = {128, 256, 512};
	int bestL = default_lanes(A), bestB = 256;
	double best = 1e30;
	const int savedL = A->lanes, savedB = A->block;
	int rc = RSD_OK;
	for (int L : lanes)
		for (int B : blocks) {
			A->lanes = L; A->block = B;
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
	if (rc != RSD_OK) { A->lanes = savedL; A->block = savedB; return rc; }
	A->lanes = bestL;
	A->block = bestB;
	if (lanes_out) *lanes_out = bestL;
	if (block_out) *block_out = bestB;
	if (best_us) *best_us = best;
	return RSD_OK;
}

int rsd_csr_lump(rsd_ctx* c, const rsd_csr* A, double* d) {
	if (!c || !A || (A->n && !d)) return set_error(RSD_EINVAL, "null argument");
	if (!A->n) return RSD_OK;
	k_lump<<<vec_grid(c, A->n * 4), 256, 0, c->stream>>>(A->n, A->rowPtr, A->val, d);
	RSD_CUDA(cudaGetLastError());
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

}  // extern "C"
