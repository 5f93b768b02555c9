// Device building blocks shared by the kernels: warp/block reductions, the deterministic
// last-block-done grid reduction, L2-hinted loads, the CSR / SELL-32 row products and the
// expression VM.
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

// ---- explicit L2 eviction priorities -------------------------------------------------------
// The Krylov loops stream the matrix (hundreds of MB) and several vectors per iteration through
// L2, while the SpMV gathers one vector (p) at column indices.  If other vector traffic evicts p,
// the gathers turn into latency-bound DRAM misses (measured: 147 us -> 265 us for the FP64 128^3
// SpMV after three vector writes).  So: matrix streams and single-use vector traffic are loaded and
// stored evict-first, the gathered vector evict-last.
struct L2Pol {
	uint64_t first, last, normal;
};
__device__ __forceinline__ L2Pol make_l2pol() {
	L2Pol p;
	asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p.first));
	asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p.last));
	asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p.normal));
	return p;
}
__device__ __forceinline__ double ldh(const double* a, uint64_t pol) {
	double v;
	asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ float ldh(const float* a, uint64_t pol) {
	float v;
	asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ uint16_t ldh(const uint16_t* a, uint64_t pol) {
	unsigned short v;
	asm volatile("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ uint32_t ldh(const uint32_t* a, uint64_t pol) {
	uint32_t v;
	asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
	return v;
}
// pairs of consecutive entries (8- or 16-byte aligned)
__device__ __forceinline__ float2 ldh2(const float* a, uint64_t pol) {
	float2 v;
	asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ double2 ldh2(const double* a, uint64_t pol) {
	double2 v;
	asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ int2 ldh2(const int32_t* a, uint64_t pol) {
	int2 v;
	asm volatile("ld.global.nc.L2::cache_hint.v2.s32 {%0,%1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ int32_t ldh(const int32_t* a, uint64_t pol) {
	int32_t v;
	asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
	return v;
}
// coherent (non-.nc) load, for data written earlier in the same kernel's lifetime by other blocks
__device__ __forceinline__ double ldh_rw(const double* a, uint64_t pol) {
	double v;
	asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ float ldh_rw(const float* a, uint64_t pol) {
	float v;
	asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
	return v;
}
__device__ __forceinline__ void sth(double* a, double v, uint64_t pol) {
	asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void sth(float* a, float v, uint64_t pol) {
	asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}

// 32 bytes per lane in one load (sm_100's 256-bit vector loads), read-only path; p 32-byte aligned
__device__ __forceinline__ void ld_nc_v4(const double* p, double& a, double& b, double& c, double& d) {
	asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}

// 16-byte packets for the element-wise Krylov kernels (4 floats or 2 doubles per load/store)
template <typename T> struct Pk;
template <> struct Pk<float> { static constexpr int W = 4; float v[4]; };
template <> struct Pk<double> { static constexpr int W = 2; double v[2]; };
__device__ __forceinline__ Pk<float> ldp(const float* a, uint64_t pol) {
	Pk<float> r;
	asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
	             : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]) : "l"(a), "l"(pol));
	return r;
}
__device__ __forceinline__ Pk<float> ldp_rw(const float* a, uint64_t pol) {
	Pk<float> r;
	asm volatile("ld.global.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
	             : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]) : "l"(a), "l"(pol));
	return r;
}
__device__ __forceinline__ void stp(float* a, const Pk<float>& r, uint64_t pol) {
	asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
	             ::"l"(a), "f"(r.v[0]), "f"(r.v[1]), "f"(r.v[2]), "f"(r.v[3]), "l"(pol) : "memory");
}
__device__ __forceinline__ Pk<double> ldp(const double* a, uint64_t pol) {
	Pk<double> r;
	asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;" : "=d"(r.v[0]), "=d"(r.v[1]) : "l"(a), "l"(pol));
	return r;
}
__device__ __forceinline__ Pk<double> ldp_rw(const double* a, uint64_t pol) {
	Pk<double> r;
	asm volatile("ld.global.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;" : "=d"(r.v[0]), "=d"(r.v[1]) : "l"(a), "l"(pol));
	return r;
}
__device__ __forceinline__ void stp(double* a, const Pk<double>& r, uint64_t pol) {
	asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1,%2}, %3;" ::"l"(a), "d"(r.v[0]), "d"(r.v[1]), "l"(pol) : "memory");
}

// Element-wise loop over [0, n): f(i0, W) on 16-byte packets (i0 a multiple of W) when `vec`, the
// scalar tail (and everything when !vec) as f(i, 1).  f must handle both widths.
template <typename T, typename F>
__device__ __forceinline__ void packet_loop(int64_t n, bool vec, F f) {
	constexpr int W = Pk<T>::W;
	const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
	const int64_t nv = vec ? n / W : 0;
	for (int64_t iv = tid; iv < nv; iv += nth) f(iv * W, W);
	for (int64_t i = nv * W + tid; i < n; i += nth) f(i, 1);
}

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

// The matrix as a kernel sees it: CSR (ptr = row pointer) or SELL-32 (ptr = slice starts), with
// the values in the precision of the kernel.
template <typename T>
struct MatView {
	const int32_t* __restrict__ ptr;
	const int32_t* __restrict__ col;
	const T* __restrict__ val;
	const uint16_t* __restrict__ col16 = nullptr;   // SELL-32 narrow columns (L == -1)
	const int32_t* __restrict__ base = nullptr;
	const int32_t* __restrict__ uni = nullptr;      // SELL-32 stencil slices (L <= 0), or null
	const int32_t* __restrict__ offs = nullptr;
	const int32_t* __restrict__ perm = nullptr;     // SELL-32: matrix row of each slot row, or null (identity)
	// mirrored stencil slices of a symmetric matrix (FP32 row sums only), or null: slice s takes its
	// first neg[s] entries from the mirror rows, entry mk[mir[s] + j] of their slices
	const int32_t* __restrict__ neg = nullptr;
	const int32_t* __restrict__ mir = nullptr;
	const uint8_t* __restrict__ mk = nullptr;
};

// the matrix row a kernel's slot row `row` (< n) stands for
template <typename T>
__device__ __forceinline__ int64_t mat_row(const MatView<T>& A, int64_t row) { return A.perm ? (int64_t)A.perm[row] : row; }

// Resident blocks of 512 threads per SM the SELL-32 row-sum kernels are compiled for: 2 leaves 64
// registers per thread, enough for the 64 bytes of values in flight per lane of row_sum (eight FP32
// pairs or four FP64 pairs).  Measured at 128^3: FP32 SpMV 49 us and FP64 85 us, against 53 / 90 us
// with four pairs at 3 blocks, 58 us (FP32) with two pairs at 4 blocks
constexpr int kRowBlocks = 2;

// sum over one row of val * xf(column).  L == 0: SELL-32, one thread per row (entries 32 slots
// apart, so a warp's value/column loads are contiguous); L == -1: SELL-32 with 16-bit column
// offsets from the slice base; L > 0: CSR with a group of L lanes per row, every lane of the group
// receiving the total.  Values and columns stream evict-first; xf reads the gathered vector with
// evict-last.
// RND8: FP32 values in rounds of eight pairs (the SpMV kernels, compiled for the registers it needs);
// false keeps the rounds at four pairs, for callers that hold much other state in registers.
template <int L, typename T, typename AccT, bool RND8 = true, typename XF>
__device__ __forceinline__ AccT row_sum(const MatView<T>& A, int64_t row, int64_t n, int lane, const L2Pol& pol, XF xf) {
	AccT s = AccT(0);
	if (row < n) {
		if constexpr (L <= 0) {
			// the slice's (even) length is the same for the whole warp; a lane reads its row in pairs
			// of consecutive entries, two pairs at a time (values, columns, then the gathers), and sums
			// them in row order
			const int64_t sl = row >> 5;
			const int s0 = A.ptr[sl];
			const int npair = (A.ptr[sl + 1] - s0) >> 6;
			const int q0 = s0 + 2 * (int)(row & 31);
			const T* __restrict__ vp = A.val + q0;
			uint64_t vpol = pol.first;   // the value stream: read once, unless mirrored reads follow
			auto run = [&](auto colpair, int jp) {
				// 64 bytes of values per step (eight FP32 pairs or four FP64 pairs: their value loads,
				// pattern offsets and gathers issued together), then two pairs, then one; the SpMV
				// kernels get the registers for it (kRowBlocks)
				if constexpr (sizeof(T) == 4 && RND8) {
					for (; jp + 8 <= npair; jp += 8) {
						decltype(ldh2(vp, pol.first)) vv[8];
						AccT xv[16];
#pragma unroll
						for (int k = 0; k < 8; ++k) vv[k] = ldh2(vp + 64 * (jp + k), vpol);
#pragma unroll
						for (int k = 0; k < 8; ++k) {
							const int2 c = colpair(jp + k);
							xv[2 * k] = xf(c.x);
							xv[2 * k + 1] = xf(c.y);
						}
#pragma unroll
						for (int k = 0; k < 8; ++k) {
							s += (AccT)vv[k].x * xv[2 * k];
							s += (AccT)vv[k].y * xv[2 * k + 1];
						}
					}
				}
				for (; jp + 4 <= npair; jp += 4) {
					const auto va = ldh2(vp + 64 * jp, vpol), vb = ldh2(vp + 64 * (jp + 1), vpol);
					const auto vc = ldh2(vp + 64 * (jp + 2), vpol), vd = ldh2(vp + 64 * (jp + 3), vpol);
					const int2 ca = colpair(jp), cb = colpair(jp + 1), cc = colpair(jp + 2), cd = colpair(jp + 3);
					const AccT x0 = xf(ca.x), x1 = xf(ca.y), x2 = xf(cb.x), x3 = xf(cb.y);
					const AccT x4 = xf(cc.x), x5 = xf(cc.y), x6 = xf(cd.x), x7 = xf(cd.y);
					s += (AccT)va.x * x0;
					s += (AccT)va.y * x1;
					s += (AccT)vb.x * x2;
					s += (AccT)vb.y * x3;
					s += (AccT)vc.x * x4;
					s += (AccT)vc.y * x5;
					s += (AccT)vd.x * x6;
					s += (AccT)vd.y * x7;
				}
				for (; jp + 2 <= npair; jp += 2) {
					const auto va = ldh2(vp + 64 * jp, vpol), vb = ldh2(vp + 64 * (jp + 1), vpol);
					const int2 ca = colpair(jp), cb = colpair(jp + 1);
					const AccT x0 = xf(ca.x), x1 = xf(ca.y), x2 = xf(cb.x), x3 = xf(cb.y);
					s += (AccT)va.x * x0;
					s += (AccT)va.y * x1;
					s += (AccT)vb.x * x2;
					s += (AccT)vb.y * x3;
				}
				for (; jp < npair; ++jp) {
					const auto va = ldh2(vp + 64 * jp, vpol);
					const int2 ca = colpair(jp);
					const AccT x0 = xf(ca.x), x1 = xf(ca.y);
					s += (AccT)va.x * x0;
					s += (AccT)va.y * x1;
				}
			};
			// a stencil slice (the branch is uniform over the warp, which holds the slice): the column
			// of entry j is row + offset j, read once per warp from the shared pattern
			const int u = A.uni ? A.uni[sl] : -1;
			if (u >= 0) {
				const int32_t* __restrict__ op = A.offs + u;
				const int r = (int)mat_row(A, row);   // the stencil's offsets are relative to the matrix row
				auto by_load = [&]() {
					run([&](int jp) {
						const int2 o = ldh2(op + 2 * jp, pol.last);
						return make_int2(r + o.x, r + o.y);
					}, 0);
				};
				if constexpr (sizeof(T) == 4) {
					// FP32 values: a stencil slice fills the warp, so lane k holds pattern entry k (read once
					// per slice) and the offsets come by shuffle instead of a load per pair (for FP64 values
					// the extra register spills under the 32-register budget, so those keep the loads)
					if (npair <= 16) {
						const int mine = __ldg(op + min((int)(row & 31), 2 * npair - 1));
						auto colpair = [&](int jp) {
							return make_int2(r + __shfl_sync(0xffffffffu, mine, 2 * jp), r + __shfl_sync(0xffffffffu, mine, 2 * jp + 1));
						};
						const int nn = A.neg ? A.neg[sl] : 0;
						if (nn > 0) {
							// a mirrored slice of a symmetric matrix: entries 0..nn-1 (negative offsets o)
							// from the mirror rows r + o, whose own reads of them went by a few slices ago
							// (still in L2), then this row's entries from nn on; the sum keeps the pattern
							// order, so it equals the whole row's to the last bit
							vpol = pol.normal;
							const uint8_t* __restrict__ mk = A.mk + A.mir[sl];
							for (int j = 0; j < nn; j += 8) {
								T mv[8];
								AccT mx[8];
#pragma unroll
								for (int k = 0; k < 8; ++k) {
									const int jj = min(j + k, nn - 1);   // clamped: every load issues
									const int m = r + __shfl_sync(0xffffffffu, mine, jj);
									const int e = mk[jj];
									mv[k] = A.val[A.ptr[m >> 5] + 64 * (e >> 1) + 2 * (m & 31) + (e & 1)];
									mx[k] = xf(m);
								}
#pragma unroll
								for (int k = 0; k < 8; ++k)
									if (j + k < nn) s += (AccT)mv[k] * mx[k];
							}
							int jp = nn >> 1;
							if (nn & 1) {   // entry nn is the second of pair nn / 2
								const auto va = ldh2(vp + 64 * jp, vpol);
								s += (AccT)va.y * xf(r + __shfl_sync(0xffffffffu, mine, nn));
								++jp;
							}
							run(colpair, jp);
						} else {
							run(colpair, 0);
						}
					} else {
						by_load();
					}
				} else {
					by_load();
				}
			} else if constexpr (L < 0) {
				const int cb = A.base[sl];
				const uint16_t* __restrict__ cp16 = A.col16 + q0;
				run([&](int jp) {
					const uint32_t w = ldh(reinterpret_cast<const uint32_t*>(cp16 + 64 * jp), pol.first);
					return make_int2(cb + (int)(w & 0xFFFFu), cb + (int)(w >> 16));
				}, 0);
			} else {
				const int32_t* __restrict__ cp32 = A.col + q0;
				run([&](int jp) { return ldh2(cp32 + 64 * jp, pol.first); }, 0);
			}
		} else {
			const int e = A.ptr[row + 1];
#pragma unroll 4
			for (int q = A.ptr[row] + lane; q < e; q += L) s += (AccT)ldh(A.val + q, pol.first) * xf(ldh(A.col + q, pol.first));
		}
	}
	if constexpr (L > 1) s = group_sum<L>(s);
	return s;
}

template <int L, typename T, typename AccT>
__device__ __forceinline__ AccT row_dot(const MatView<T>& A, const T* __restrict__ x, int64_t row, int64_t n, int lane, const L2Pol& pol) {
	return row_sum<L, T, AccT>(A, row, n, lane, pol, [&](int c) { return (AccT)ldh(x + c, pol.last); });
}

// Row-loop geometry shared by the row kernels: a group of G = max(L,1) threads per row, rows
// handed out warp by warp so that a warp's rows are consecutive (a whole SELL slice when L == 0).
template <int L>
struct RowLoop {
	static constexpr int G = L > 0 ? L : 1;
	int lane;
	int64_t base, step, sub;
	__device__ __forceinline__ RowLoop() {
		lane = threadIdx.x & (G - 1);
		sub = (threadIdx.x & 31) / G;
		const int64_t g0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
		base = g0 - sub;
		step = ((int64_t)gridDim.x * blockDim.x) / G;
	}
};

// Adaptive replacement threshold of the mixed-precision solvers.  The FP32 recurrence residual drifts
// from the true one by roughly eps32 * cond(A) * ||A|| ||x|| whatever the current residual is, so its
// relative error grows in proportion to the reduction since the last replacement.  With d the
// relative gap seen at this replacement (threshold delta), the threshold that keeps the next gap
// near 1% is 100 d delta, kept within [lo, 0.1]: well-conditioned systems replace rarely,
// ill-conditioned ones often.  The floor is the solver's (measured): the single CG solve takes
// kDeltaFloorCg, the batched solver kDeltaFloorBatch, where a lower floor cost iterations.
constexpr double kDeltaFloorCg = 1e-4, kDeltaFloorBatch = 1e-3;
__host__ __device__ __forceinline__ double next_delta(double delta, double recurrence, double true_res, double lo) {
	const double d = fabs(recurrence - true_res) / fmax(true_res, 1e-300);
	return fmin(0.1, fmax(lo, 100.0 * d * delta));
}

// expression stack machine (bytecode from compile_expr, which rejects programs deeper than kExprStack
// and records each program's depth).  The stack lives in registers: D slots indexed only by
// compile-time constants (s[0] the top), a push shifting the slots up and a binary operator folding
// the top two and shifting down.  A stack array indexed by a running stack pointer lives in local
// memory instead, and inlined into the boundary-reaction monitor kernel (an element loop that keeps
// per-node local arrays live across its quadrature points) it was given the storage of the element's
// rate array (nvcc 12.9, sm_100a): the source value overwrote a nodal rate from the second point on
// (test_heat_flux_monitors pins the monitor against the reference).
template <int D>
__device__ __forceinline__ double eval_expr_d(const DevExpr& e, double t, double x, double y, double z, double T) {
	double s[D];
#pragma unroll
	for (int k = 0; k < D; ++k) s[k] = 0.0;
	for (int i = 0; i < e.n; ++i) {
		const int op = e.op[i];
		const int a = e.arg[i];
		if (op == E_CONST || op == E_VAR) {
			const double v = op == E_CONST ? e.c[a] : (a == 0 ? t : a == 1 ? x : a == 2 ? y : a == 3 ? z : T);
#pragma unroll
			for (int k = D - 1; k > 0; --k) s[k] = s[k - 1];
			s[0] = v;
		} else if (op <= E_POW) {
			const double l = s[1], r = s[0];
			double v;
			switch (op) {
				case E_ADD: v = l + r; break;
				case E_SUB: v = l - r; break;
				case E_MUL: v = l * r; break;
				case E_DIV: v = l / r; break;
				default: v = pow(l, r); break;
			}
			s[0] = v;
#pragma unroll
			for (int k = 1; k < D - 1; ++k) s[k] = s[k + 1];
		} else {
			double v = s[0];
			switch (op) {
				case E_NEG: v = -v; break;
				case E_SIN: v = sin(v); break;
				case E_COS: v = cos(v); break;
				case E_TAN: v = tan(v); break;
				case E_EXP: v = exp(v); break;
				case E_LOG: v = log(v); break;
				case E_SQRT: v = sqrt(v); break;
				default: v = fabs(v); break;
			}
			s[0] = v;
		}
	}
	return e.n ? s[0] : 0.0;
}
__device__ __forceinline__ double eval_expr(const DevExpr& e, double t, double x, double y, double z, double T) {
	if (e.depth <= 4) return eval_expr_d<4>(e, t, x, y, z, T);
	if (e.depth <= 8) return eval_expr_d<8>(e, t, x, y, z, T);
	return eval_expr_d<kExprStack>(e, t, x, y, z, T);
}

// lanes per row of the execution layout: -1 for SELL-32 with narrow columns, 0 for SELL-32, else
// the CSR group size
inline int exec_lanes(const rsd_csr* A) { return A->format == 0 ? (A->sCol16 ? -1 : 0) : default_lanes(A); }
inline MatView<double> view64(const rsd_csr* A) {
	return A->format == 0 ? MatView<double>{A->sStart, A->sCol, A->sVal, A->sCol16, A->sBase, A->sUni, A->sOffs, A->sPerm}
	                      : MatView<double>{A->rowPtr, A->col, A->val};
}
inline MatView<float> view32(const rsd_csr* A) {
	return A->format == 0 ? MatView<float>{A->sStart, A->sCol, A->val32, A->sCol16, A->sBase, A->sUni, A->sOffs, A->sPerm}
	                      : MatView<float>{A->rowPtr, A->col, A->val32};
}
// the FP32 view with the mirrored slices when the values are known symmetric (the mixed CG's SpMV)
inline MatView<float> view32_sym(const rsd_csr* A) {
	MatView<float> V = view32(A);
	if (A->format == 0 && A->nMirrored && A->symVersion == A->version && !A->sPerm) {
		V.neg = A->sNeg; V.mir = A->sMir; V.mk = A->sMk;
	}
	return V;
}
template <typename T>
inline MatView<T> exec_view(const rsd_csr* A) {
	if constexpr (sizeof(T) == 4) return view32(A);
	else return view64(A);
}
// diagonal position and values of the execution layout
inline const int32_t* exec_diag(const rsd_csr* A) { return A->format == 0 ? A->sDiag : A->diag; }
inline const double* exec_val(const rsd_csr* A) { return A->format == 0 ? A->sVal : A->val; }

#define RSD_DISPATCH_L(L, CALL)                          \
	switch (L) {                                         \
		case -1: { constexpr int LL = -1; CALL; } break; \
		case 0: { constexpr int LL = 0; CALL; } break;   \
		case 1: { constexpr int LL = 1; CALL; } break;   \
		case 2: { constexpr int LL = 2; CALL; } break;   \
		case 4: { constexpr int LL = 4; CALL; } break;   \
		case 8: { constexpr int LL = 8; CALL; } break;   \
		case 16: { constexpr int LL = 16; CALL; } break; \
		default: { constexpr int LL = 32; CALL; } break; \
	}

// resident blocks per SM of `kernel` at `block` threads (cached per kernel and block size)
int resident_blocks(const void* kernel, int block);

// grid of a grid-stride kernel: the blocks `threads` need, at most one full wave of resident blocks
// (so no block starts after the first ones finish) and at most `cap` (the reduction partials)
template <typename K>
inline int wave_blocks(const rsd_ctx* ctx, K* kernel, int block, int64_t threads, int64_t cap = kMaxPartials) {
	const int64_t need = (threads + block - 1) / block;
	const int64_t wave = (int64_t)ctx->num_sms * resident_blocks((const void*)kernel, block);
	return (int)std::max<int64_t>(1, std::min(std::min(need, wave), cap));
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
