// Device building blocks shared by the kernels: warp/block reductions, the deterministic
// last-block-done grid reduction, streaming loads, the CSR row product and the expression VM.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "rsd_internal.cuh"

namespace rsd {

// streaming loads for data read exactly once (matrix values/columns): evict-first in L1/L2 so
// that the gathered vector keeps its place in the 126 MB L2
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
template <typename T>
__device__ __forceinline__ T ld_ro(const T* p) { return __ldg(p); }

template <int W, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
	for (int off = W / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
	return v;
}

// block-wide sum of NCH values; thread 0 receives the totals (fixed order -> deterministic)
template <int NCH>
__device__ __forceinline__ void block_sum(double (&v)[NCH]) {
	__shared__ double sm[NCH][32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
	for (int c = 0; c < NCH; ++c) v[c] = group_sum<32>(v[c]);
	if (lane == 0)
#pragma unroll
		for (int c = 0; c < NCH; ++c) sm[c][warp] = v[c];
	__syncthreads();
	if (warp == 0) {
#pragma unroll
		for (int c = 0; c < NCH; ++c) {
			double t = lane < nw ? sm[c][lane] : 0.0;
			v[c] = group_sum<32>(t);
		}
	}
	__syncthreads();
}

// Every block deposits its NCH partial sums; the last block to arrive sums all partials in block
// order and returns true on thread 0 with the totals in v.  The ticket wraps back to zero.
template <int NCH>
__device__ __forceinline__ bool grid_sum(double (&v)[NCH], double* partials, unsigned* ticket) {
	__shared__ bool last;
	block_sum<NCH>(v);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int c = 0; c < NCH; ++c) partials[c * kMaxPartials + blockIdx.x] = v[c];
		__threadfence();
		last = atomicInc(ticket, gridDim.x - 1) == gridDim.x - 1;
	}
	__syncthreads();
	if (!last) return false;
	__threadfence();
	double acc[NCH];
#pragma unroll
	for (int c = 0; c < NCH; ++c) {
		acc[c] = 0.0;
		for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[c] += __ldcg(&partials[c * kMaxPartials + b]);
	}
	block_sum<NCH>(acc);
#pragma unroll
	for (int c = 0; c < NCH; ++c) v[c] = acc[c];
	return threadIdx.x == 0;
}

// one CSR row times x by a group of L lanes; every lane of the group returns the full sum
template <int L, typename T, typename AccT>
__device__ __forceinline__ AccT csr_row(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                       const T* __restrict__ val, const T* __restrict__ x, int64_t row, int64_t n,
                                       int lane) {
	AccT s = AccT(0);
	if (row < n) {
		const int b = rp[row], e = rp[row + 1];
#pragma unroll 4
		for (int p = b + lane; p < e; p += L) s += (AccT)ld_stream(val + p) * (AccT)ld_ro(x + ld_stream(col + p));
	}
	return group_sum<L>(s);
}

// expression stack machine (bytecode from compile_expr)
__device__ __forceinline__ double eval_expr(const DevExpr& e, double t, double x, double y, double z, double T) {
	double st[16];
	int sp = 0;
	for (int i = 0; i < e.n; ++i) {
		const int op = e.op[i];
		const int a = e.arg[i];
		switch (op) {
			case E_CONST: st[sp++] = e.c[a]; break;
			case E_VAR: st[sp++] = a == 0 ? t : a == 1 ? x : a == 2 ? y : a == 3 ? z : T; break;
			case E_ADD: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
			case E_SUB: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
			case E_MUL: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
			case E_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
			case E_POW: --sp; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
			case E_NEG: st[sp - 1] = -st[sp - 1]; break;
			case E_SIN: st[sp - 1] = sin(st[sp - 1]); break;
			case E_COS: st[sp - 1] = cos(st[sp - 1]); break;
			case E_TAN: st[sp - 1] = tan(st[sp - 1]); break;
			case E_EXP: st[sp - 1] = exp(st[sp - 1]); break;
			case E_LOG: st[sp - 1] = log(st[sp - 1]); break;
			case E_SQRT: st[sp - 1] = sqrt(st[sp - 1]); break;
			default: st[sp - 1] = fabs(st[sp - 1]); break;
		}
		if (sp >= 16) return 0.0;
	}
	return e.n ? st[0] : 0.0;
}

inline int vec_grid(const rsd_ctx* ctx, int64_t n, int threads = 256) {
	int64_t b = (n + threads - 1) / threads;
	const int64_t cap = (int64_t)ctx->num_sms * 8;
	if (b > cap) b = cap;
	if (b < 1) b = 1;
	return (int)b;
}

inline int red_grid(const rsd_ctx* ctx, int64_t n) {
	int64_t b = (n + kReduceThreads * 4 - 1) / (kReduceThreads * 4);
	const int64_t cap = std::min<int64_t>(kMaxPartials, (int64_t)ctx->num_sms * 4);
	if (b > cap) b = cap;
	if (b < 1) b = 1;
	return (int)b;
}

}  // namespace rsd
