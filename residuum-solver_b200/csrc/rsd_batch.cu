// Batched solves of many independent, uneven systems in one persistent launch (a "CSR of CSRs":
// the batch indexes its problems, each problem is an rsd_csr in its SELL-32 execution layout).
//
// Each CTA takes the next problem from a device-side queue (problems ordered by size, largest
// first, so the longest solves start first), runs the whole preconditioned CG for it with
// block-level reductions and __syncthreads between phases, writes the problem's report and takes
// the next one.  No CTA ever waits for another, so the launch cannot deadlock, and the loop of every
// solve is bounded by max_iters.
//
// Precision: TI = float is the mixed scheme of the single-system solver (FP32 matrix and vectors,
// FP64 reductions, FP64 residual replacement when the recurrence residual falls by delta or claims
// convergence, convergence declared on the FP64 residual); TI = double is plain FP64 PCG
// (cg/Solver.tpp:13-119 per problem).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "rsd_kernels.cuh"

struct rsd_batch {
	int32_t count = 0;
	std::vector<rsd_csr*> A;
	std::vector<int32_t> order;        // problems by nnz, descending
	void* desc = nullptr;              // device BatchProb[count]
	void* out = nullptr;               // device BatchOut[count]
	int32_t* dorder = nullptr;         // device order[count]
	int32_t* next = nullptr;           // device queue head
	void* ws = nullptr;                // device workspace, 5 vectors per problem
	size_t wsBytes = 0;
};

namespace rsd {
namespace {

namespace cg = cooperative_groups;

constexpr int kBT = 1024;              // threads per CTA: 32 warps keep enough gathers in flight
constexpr int kBW = kBT / 32;

template <typename TI>
struct BatchProb {
	int64_t n, nslices;
	MatView<TI> A;                     // execution layout, inner precision
	MatView<double> A64;               // FP64 values (residuals)
	const int32_t* sDiag;
	const double* b;
	double* x;
	TI *r, *p, *Ap, *y, *invD;
};

struct BatchOut {
	int64_t iterations, refinements;
	double res0, res, trueRel;
	int32_t converged, status;
};

// The problem descriptor (two matrix views and the vector pointers, about 60 registers' worth) is
// copied into shared memory once per problem and read from there: held in registers it pushed the
// solver loop into local-memory spills.
template <typename TI>
__device__ __forceinline__ void load_prob(uint64_t* pbuf, const BatchProb<TI>* src) {
	static_assert(sizeof(BatchProb<TI>) % 8 == 0, "descriptor of whole 8-byte words");
	const uint64_t* w = reinterpret_cast<const uint64_t*>(src);
	for (int k = threadIdx.x; k < (int)(sizeof(BatchProb<TI>) / 8); k += blockDim.x) pbuf[k] = w[k];
}

// block-wide sums of NCH doubles; every thread receives the totals (fixed order: deterministic)
template <int NCH, int NW = kBW>
__device__ __forceinline__ void bsum(double (&v)[NCH], double (*sm)[kBW]) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int c = 0; c < NCH; ++c) v[c] = group_sum<32>(v[c]);
	if (lane == 0)
#pragma unroll
		for (int c = 0; c < NCH; ++c) sm[c][warp] = v[c];
	__syncthreads();
#pragma unroll
	for (int c = 0; c < NCH; ++c) {
		double t = 0.0;
		for (int w = 0; w < NW; ++w) t += sm[c][w];
		v[c] = t;
	}
	__syncthreads();
}

// rows of one problem, one SELL slice per warp at a time; f(row, rowSum) for the rows < n
template <int L, typename T, typename XF, typename F>
__device__ __forceinline__ void slice_rows(const MatView<T>& A, int64_t n, int64_t nslices, const L2Pol& pol, XF xf, F f) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int64_t sl = warp; sl < nslices; sl += kBW) {
		const int64_t row = sl * 32 + lane;
		const double s = (double)row_sum<L, T, T, false>(A, row, n, 0, pol, xf);
		if (row < n) f(mat_row(A, row), s);
	}
}

template <typename TI, int L>
__device__ void solve_one(const BatchProb<TI>& P, BatchOut* out, double tol, int relMode, int64_t maxIt, double delta,
                          int adaptive, double (*sm)[kBW]) {
	constexpr bool kMixed = sizeof(TI) == 4;
	constexpr int PW = 16 / sizeof(TI);   // entries per 16-byte packet
	struct Vec { TI v[PW]; };
	auto ldv = [](const TI* a) { Vec o; *reinterpret_cast<uint4*>(&o) = *reinterpret_cast<const uint4*>(a); return o; };
	auto stv = [](TI* a, const Vec& o) { *reinterpret_cast<uint4*>(a) = *reinterpret_cast<const uint4*>(&o); };
	const int64_t n = P.n;
	const L2Pol pol = make_l2pol();
	TI* __restrict__ r = P.r;
	TI* __restrict__ p = P.p;
	TI* __restrict__ Ap = P.Ap;
	TI* __restrict__ y = P.y;
	TI* __restrict__ invD = P.invD;
	double* __restrict__ x = P.x;
	const int tid = threadIdx.x;
	// Jacobi::update (Jacobi.hpp:31-34); z = M r through zr()
	for (int64_t i = tid; i < n; i += kBT) {
		if (invD) {
			const int32_t q = P.sDiag[i];
			const double d = q >= 0 ? P.A64.val[q] : 0.0;
			invD[i] = (TI)(fabs(d) > 1e-300 ? 1.0 / d : 1.0);
		}
		y[i] = (TI)0;
	}
	__syncthreads();
	auto zr = [&](int64_t i, TI ri) -> TI { return invD ? ri * invD[i] : ri; };
	// r = b - A64 x; z = M r; p = z
	auto residual64 = [&](double (&v)[2]) {
		v[0] = v[1] = 0.0;
		slice_rows<L, double>(P.A64, n, P.nslices, pol, [&](int c) { return x[c] + (double)y[c]; }, [&](int64_t i, double ax) {
			const double r64 = P.b[i] - ax;
			const TI ri = (TI)r64;
			const TI zi = zr(i, ri);
			r[i] = ri;
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		});
	};
	double v[2];
	residual64(v);
	bsum<2>(v, sm);
	for (int64_t i = tid; i < n; i += kBT) p[i] = zr(i, r[i]);
	__syncthreads();
	const double res0 = sqrt(v[0]);
	double rz = v[1], res = res0, rmax = res0, trueRel = 1.0;
	int64_t it = 0, refinements = 0;
	int32_t converged = 0, status = 0;
	auto crit = [&](double rr) { return relMode ? rr / (res0 + 1e-50) : rr; };
	if (crit(res0) < tol || n == 0) converged = 1;
	while (!converged && !status && it < maxIt - 1) {
		// Ap = A p, alpha = r.z / p.Ap
		double w[1] = {0.0};
		slice_rows<L, TI>(P.A, n, P.nslices, pol, [&](int c) { return (TI)p[c]; }, [&](int64_t i, double s) {
			Ap[i] = (TI)s;
			w[0] += (double)p[i] * (double)(TI)s;
		});
		bsum<1>(w, sm);
		const double alpha = rz / w[0];
		if (!isfinite(alpha)) { status = RSD_EBREAKDOWN; break; }
		const TI a = (TI)alpha;
		double u[2] = {0.0, 0.0};
		auto upd = [&](int64_t i, TI pi, TI api, TI ri0, TI di) {
			if (kMixed) y[i] = y[i] + a * pi;
			else x[i] = x[i] + alpha * (double)pi;    // FP64: x += alpha p as cg/Solver.tpp:74-76
			const TI ri = ri0 - a * api;
			const TI zi = invD ? ri * di : ri;
			u[0] += (double)ri * (double)ri;
			u[1] += (double)ri * (double)zi;
			return ri;
		};
		// 16-byte packets (the workspace vectors start 256-byte aligned), then the scalar tail
		for (int64_t iv = tid; iv < n / PW; iv += kBT) {
			const int64_t i0 = iv * PW;
			Vec P = ldv(p + i0), AP = ldv(Ap + i0), R = ldv(r + i0), D{};
			if (invD) D = ldv(invD + i0);
#pragma unroll
			for (int k = 0; k < PW; ++k) R.v[k] = upd(i0 + k, P.v[k], AP.v[k], R.v[k], D.v[k]);
			stv(r + i0, R);
		}
		for (int64_t i = (n / PW) * PW + tid; i < n; i += kBT) r[i] = upd(i, p[i], Ap[i], r[i], invD ? invD[i] : (TI)1);
		bsum<2>(u, sm);
		++it;
		res = sqrt(u[0]);
		if (!isfinite(res)) { status = RSD_ENAN; break; }
		double rzNew = u[1];
		const bool replace = kMixed && (crit(res) < tol || res < delta * rmax || it + 1 >= maxIt);
		if (replace) {
			// FP64 residual replacement: r = b - A64 (x + y), then fold y into x
			residual64(v);
			bsum<2>(v, sm);
			for (int64_t i = tid; i < n; i += kBT) { x[i] += (double)y[i]; y[i] = (TI)0; }
			const double recurrence = res;
			res = sqrt(v[0]);
			if (adaptive) delta = next_delta(delta, recurrence, res, kDeltaFloorBatch);
			rmax = res;
			trueRel = res / (res0 + 1e-50);
			rzNew = v[1];
			++refinements;
			if (crit(res) < tol) { converged = 1; break; }
		} else if (!kMixed && crit(res) < tol) {
			converged = 1;
			break;
		}
		const TI beta = (TI)(rzNew / rz);
		rz = rzNew;
		__syncthreads();
		for (int64_t iv = tid; iv < n / PW; iv += kBT) {
			const int64_t i0 = iv * PW;
			Vec P = ldv(p + i0), R = ldv(r + i0), D{};
			if (invD) D = ldv(invD + i0);
#pragma unroll
			for (int k = 0; k < PW; ++k) P.v[k] = P.v[k] * beta + (invD ? R.v[k] * D.v[k] : R.v[k]);
			stv(p + i0, P);
		}
		for (int64_t i = (n / PW) * PW + tid; i < n; i += kBT) p[i] = p[i] * beta + zr(i, r[i]);
		__syncthreads();
	}
	if (kMixed && !converged) {
		// stopped early: fold the remaining FP32 correction into the FP64 iterate
		__syncthreads();
		for (int64_t i = tid; i < n; i += kBT) { x[i] += (double)y[i]; y[i] = (TI)0; }
	}
	if (!kMixed) trueRel = res / (res0 + 1e-50);
	if (tid == 0) {
		out->iterations = converged ? it : (status ? it : maxIt);
		out->refinements = refinements;
		out->res0 = res0;
		out->res = res;
		out->trueRel = trueRel;
		out->converged = converged;
		out->status = status;
	}
	__syncthreads();
}

// ---- teams: one problem over the CTAs of a thread-block cluster -----------------------------------
// The work per problem grows about as rows^1.5 (its CG iterations grow with the grid size), so with
// one CTA per problem the largest problems outlast the rest of the batch by far.  A cluster of
// CTAs solves each problem instead: the rows (slices) and vector entries are dealt across the CTAs,
// the reductions add the CTAs' block sums through distributed shared memory in rank order (the same
// totals in every CTA, deterministic), and a cluster barrier orders each phase's global writes before
// the next phase reads them.  Same formulas as solve_one.
// Team shape: TM CTAs of TT threads (kBT; the size is chosen per batch, launch_teams).  Measured on
// the 256-problem batch (mixed / FP64 ms), teams of 1024-thread CTAs: one CTA per problem 159 / 177,
// 2 CTAs 99.0 / 112.0, 3 CTAs 117.4 / 124.9, 4 CTAs 133.7 / 135.6, 8 CTAs 215 / 199; 512-thread CTAs
// (128 registers, no spills): 4 x 512 150 / 153, 8 x 512 194 / 196.

template <int NCH, int TT, int TM>
__device__ __forceinline__ void team_sum(double (&v)[NCH], double (*sm)[kBW], double (*xch)[4], int& parity) {
	cg::cluster_group cl = cg::this_cluster();
	bsum<NCH, TT / 32>(v, sm);
	if (threadIdx.x == 0)
#pragma unroll
		for (int c = 0; c < NCH; ++c) xch[parity][c] = v[c];
	cl.sync();
	double t[NCH];
#pragma unroll
	for (int c = 0; c < NCH; ++c) t[c] = 0.0;
	for (int r = 0; r < TM; ++r) {
		const double* rem = cl.map_shared_rank(&xch[parity][0], r);
#pragma unroll
		for (int c = 0; c < NCH; ++c) t[c] += rem[c];
	}
#pragma unroll
	for (int c = 0; c < NCH; ++c) v[c] = t[c];
	parity ^= 1;   // the next sum writes the other slot: a CTA still reading this one has not passed it
}

// the team's share of one problem's slices; f(row, rowSum) for the rows < n
template <int L, typename T, int TT, int TM, typename XF, typename F>
__device__ __forceinline__ void team_rows(const MatView<T>& A, int64_t n, int64_t nslices, int rank, const L2Pol& pol, XF xf, F f) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int64_t sl = (int64_t)rank * (TT / 32) + warp; sl < nslices; sl += (TT / 32) * TM) {
		const int64_t row = sl * 32 + lane;
		const double s = (double)row_sum<L, T, T, false>(A, row, n, 0, pol, xf);
		if (row < n) f(mat_row(A, row), s);
	}
}

template <typename TI, int L, int TT, int TM>
__device__ void solve_team(const BatchProb<TI>& P, BatchOut* out, double tol, int relMode, int64_t maxIt, double delta,
                           int adaptive, double (*sm)[kBW], double (*xch)[4]) {
	constexpr bool kMixed = sizeof(TI) == 4;
	constexpr int PW = 16 / sizeof(TI);
	struct Vec { TI v[PW]; };
	auto ldv = [](const TI* a) { Vec o; *reinterpret_cast<uint4*>(&o) = *reinterpret_cast<const uint4*>(a); return o; };
	auto stv = [](TI* a, const Vec& o) { *reinterpret_cast<uint4*>(a) = *reinterpret_cast<const uint4*>(&o); };
	cg::cluster_group cl = cg::this_cluster();
	const int rank = (int)cl.block_rank();
	const int64_t n = P.n;
	const L2Pol pol = make_l2pol();
	TI* __restrict__ r = P.r;
	TI* __restrict__ p = P.p;
	TI* __restrict__ Ap = P.Ap;
	TI* __restrict__ y = P.y;
	TI* __restrict__ invD = P.invD;
	double* __restrict__ x = P.x;
	const int64_t gt = (int64_t)rank * TT + threadIdx.x, gs = (int64_t)TT * TM;   // entry deal
	int parity = 0;
	for (int64_t i = gt; i < n; i += gs) {
		if (invD) {
			const int32_t q = P.sDiag[i];
			const double d = q >= 0 ? P.A64.val[q] : 0.0;
			invD[i] = (TI)(fabs(d) > 1e-300 ? 1.0 / d : 1.0);
		}
		y[i] = (TI)0;
	}
	cl.sync();
	auto zr = [&](int64_t i, TI ri) -> TI { return invD ? ri * invD[i] : ri; };
	auto residual64 = [&](double (&v)[2]) {
		v[0] = v[1] = 0.0;
		team_rows<L, double, TT, TM>(P.A64, n, P.nslices, rank, pol, [&](int c) { return x[c] + (double)y[c]; }, [&](int64_t i, double ax) {
			const double r64 = P.b[i] - ax;
			const TI ri = (TI)r64;
			const TI zi = zr(i, ri);
			r[i] = ri;
			v[0] += r64 * r64;
			v[1] += (double)ri * (double)zi;
		});
	};
	double v[2];
	residual64(v);
	team_sum<2, TT, TM>(v, sm, xch, parity);
	for (int64_t i = gt; i < n; i += gs) p[i] = zr(i, r[i]);
	cl.sync();
	const double res0 = sqrt(v[0]);
	double rz = v[1], res = res0, rmax = res0, trueRel = 1.0;
	int64_t it = 0, refinements = 0;
	int32_t converged = 0, status = 0;
	auto crit = [&](double rr) { return relMode ? rr / (res0 + 1e-50) : rr; };
	if (crit(res0) < tol || n == 0) converged = 1;
	while (!converged && !status && it < maxIt - 1) {
		double w[1] = {0.0};
		team_rows<L, TI, TT, TM>(P.A, n, P.nslices, rank, pol, [&](int c) { return (TI)p[c]; }, [&](int64_t i, double s) {
			Ap[i] = (TI)s;
			w[0] += (double)p[i] * (double)(TI)s;
		});
		team_sum<1, TT, TM>(w, sm, xch, parity);
		const double alpha = rz / w[0];
		if (!isfinite(alpha)) { status = RSD_EBREAKDOWN; break; }
		const TI a = (TI)alpha;
		double u[2] = {0.0, 0.0};
		auto upd = [&](int64_t i, TI pi, TI api, TI ri0, TI di) {
			if (kMixed) y[i] = y[i] + a * pi;
			else x[i] = x[i] + alpha * (double)pi;
			const TI ri = ri0 - a * api;
			const TI zi = invD ? ri * di : ri;
			u[0] += (double)ri * (double)ri;
			u[1] += (double)ri * (double)zi;
			return ri;
		};
		for (int64_t iv = gt; iv < n / PW; iv += gs) {
			const int64_t i0 = iv * PW;
			Vec Pv = ldv(p + i0), AP = ldv(Ap + i0), R = ldv(r + i0), D{};
			if (invD) D = ldv(invD + i0);
#pragma unroll
			for (int k = 0; k < PW; ++k) R.v[k] = upd(i0 + k, Pv.v[k], AP.v[k], R.v[k], D.v[k]);
			stv(r + i0, R);
		}
		for (int64_t i = (n / PW) * PW + gt; i < n; i += gs) r[i] = upd(i, p[i], Ap[i], r[i], invD ? invD[i] : (TI)1);
		team_sum<2, TT, TM>(u, sm, xch, parity);
		++it;
		res = sqrt(u[0]);
		if (!isfinite(res)) { status = RSD_ENAN; break; }
		double rzNew = u[1];
		const bool replace = kMixed && (crit(res) < tol || res < delta * rmax || it + 1 >= maxIt);
		if (replace) {
			residual64(v);
			team_sum<2, TT, TM>(v, sm, xch, parity);
			for (int64_t i = gt; i < n; i += gs) { x[i] += (double)y[i]; y[i] = (TI)0; }
			const double recurrence = res;
			res = sqrt(v[0]);
			if (adaptive) delta = next_delta(delta, recurrence, res, kDeltaFloorBatch);
			rmax = res;
			trueRel = res / (res0 + 1e-50);
			rzNew = v[1];
			++refinements;
			if (crit(res) < tol) { converged = 1; break; }
		} else if (!kMixed && crit(res) < tol) {
			converged = 1;
			break;
		}
		const TI beta = (TI)(rzNew / rz);
		rz = rzNew;
		for (int64_t iv = gt; iv < n / PW; iv += gs) {
			const int64_t i0 = iv * PW;
			Vec Pv = ldv(p + i0), R = ldv(r + i0), D{};
			if (invD) D = ldv(invD + i0);
#pragma unroll
			for (int k = 0; k < PW; ++k) Pv.v[k] = Pv.v[k] * beta + (invD ? R.v[k] * D.v[k] : R.v[k]);
			stv(p + i0, Pv);
		}
		for (int64_t i = (n / PW) * PW + gt; i < n; i += gs) p[i] = p[i] * beta + zr(i, r[i]);
		cl.sync();   // the next product gathers p from every CTA's share
	}
	if (kMixed && !converged) {
		cl.sync();
		for (int64_t i = gt; i < n; i += gs) { x[i] += (double)y[i]; y[i] = (TI)0; }
	}
	if (!kMixed) trueRel = res / (res0 + 1e-50);
	if (rank == 0 && threadIdx.x == 0) {
		out->iterations = converged ? it : (status ? it : maxIt);
		out->refinements = refinements;
		out->res0 = res0;
		out->res = res;
		out->trueRel = trueRel;
		out->converged = converged;
		out->status = status;
	}
	cl.sync();   // the workspace vectors of this problem are not reused, but the exchange slots are
}

template <typename TI, int TT, int TM>
__global__ void __launch_bounds__(TT, 1) k_batch_cg_team(const BatchProb<TI>* probs, const int32_t* order, int32_t count,
                                                       int32_t* next, BatchOut* outs, double tol, int relMode,
                                                       int64_t maxIt, double delta, int adaptive) {
	__shared__ double sm[2][kBW];
	__shared__ double xch[2][4];
	__shared__ int32_t job;
	__shared__ alignas(16) uint64_t pbuf[sizeof(BatchProb<TI>) / 8];
	const BatchProb<TI>& P = *reinterpret_cast<const BatchProb<TI>*>(pbuf);
	cg::cluster_group cl = cg::this_cluster();
	for (;;) {
		if (cl.block_rank() == 0 && threadIdx.x == 0) job = atomicAdd(next, 1);
		cl.sync();
		const int32_t j = *cl.map_shared_rank(&job, 0);
		if (j < count) load_prob(pbuf, probs + order[j]);
		cl.sync();   // every CTA has read the job (and its descriptor) before rank 0 takes the next
		if (j >= count) return;
		const int32_t pi = order[j];
		if (P.A.col16) solve_team<TI, -1, TT, TM>(P, outs + pi, tol, relMode, maxIt, delta, adaptive, sm, xch);
		else solve_team<TI, 0, TT, TM>(P, outs + pi, tol, relMode, maxIt, delta, adaptive, sm, xch);
	}
}

template <typename TI>
__global__ void __launch_bounds__(kBT) k_batch_cg(const BatchProb<TI>* probs, const int32_t* order, int32_t count,
                                                  int32_t* next, BatchOut* outs, double tol, int relMode,
                                                  int64_t maxIt, double delta, int adaptive) {
	__shared__ double sm[2][kBW];
	__shared__ int32_t job;
	__shared__ alignas(16) uint64_t pbuf[sizeof(BatchProb<TI>) / 8];
	const BatchProb<TI>& P = *reinterpret_cast<const BatchProb<TI>*>(pbuf);
	for (;;) {
		if (threadIdx.x == 0) job = atomicAdd(next, 1);
		__syncthreads();
		const int32_t j = job;
		if (j < count) load_prob(pbuf, probs + order[j]);
		__syncthreads();
		if (j >= count) return;
		const int32_t pi = order[j];
		if (P.A.col16) solve_one<TI, -1>(P, outs + pi, tol, relMode, maxIt, delta, adaptive, sm);
		else solve_one<TI, 0>(P, outs + pi, tol, relMode, maxIt, delta, adaptive, sm);
	}
}

int64_t pad_len(int64_t n) { return (n + 63) & ~int64_t(63); }

// launch configuration of the team kernel: clusters of TM CTAs of TT threads; *clusters = how many
// are resident at once
template <typename TI, int TT, int TM>
int team_config(rsd_ctx* ctx, cudaLaunchConfig_t& lc, cudaLaunchAttribute* at, int* clusters) {
	lc = cudaLaunchConfig_t{};
	at[0].id = cudaLaunchAttributeClusterDimension;
	at[0].val.clusterDim.x = TM; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
	lc.blockDim = dim3(TT);
	lc.dynamicSmemBytes = 0;
	lc.stream = ctx->stream;
	lc.attrs = at;
	lc.numAttrs = 1;
	lc.gridDim = dim3(TM * ctx->num_sms);
	*clusters = 0;
	RSD_CUDA(cudaOccupancyMaxActiveClusters(clusters, (const void*)k_batch_cg_team<TI, TT, TM>, &lc));
	return RSD_OK;
}

// one launch of the team kernel with as many clusters as are resident (at most one per problem),
// taking problems from the queue
template <typename TI, int TT, int TM>
int launch_team(rsd_ctx* ctx, rsd_batch* B, int32_t count, const rsd_solver_cfg* cfg, int rel, double delta, int adaptive) {
	cudaLaunchConfig_t lc;
	cudaLaunchAttribute at[1];
	int clusters = 0;
	RSD_CHECK((team_config<TI, TT, TM>(ctx, lc, at, &clusters)));
	clusters = std::max(1, std::min(count, clusters));
	lc.gridDim = dim3(TM * clusters);
	RSD_CUDA(cudaLaunchKernelEx(&lc, k_batch_cg_team<TI, TT, TM>, (const BatchProb<TI>*)B->desc, (const int32_t*)B->dorder, count,
	                            B->next, (BatchOut*)B->out, cfg->tol, rel, cfg->max_iters, delta, adaptive));
	return RSD_OK;
}

// The team size for a batch of `count` problems (forced: 2, 4 or 8 CTAs, 0 to choose).  A batch
// solve ends when its largest problem does, and that problem's iterations shorten with more SMs on
// it, while smaller teams run more problems at once and span fewer SMs per reduction.  Measured
// (1024-thread CTAs, mixed ms): 256 problems 99.0 with teams of 2, 133.7 with 4, 215 with 8; 64
// problems 78.1 with 2, 44.4 with 4.  Rule: the smallest team whose resident clusters number at most
// two thirds of the problems (every cluster then solves 1.5 problems or more), else 8.
template <typename TI>
int launch_teams(rsd_ctx* ctx, rsd_batch* B, int32_t count, const rsd_solver_cfg* cfg, int rel, double delta, int adaptive,
                 int forced) {
	int tm = forced;
	if (tm != 2 && tm != 4 && tm != 8) {
		cudaLaunchConfig_t lc;
		cudaLaunchAttribute at[1];
		int c2 = 0, c4 = 0;
		RSD_CHECK((team_config<TI, kBT, 2>(ctx, lc, at, &c2)));
		RSD_CHECK((team_config<TI, kBT, 4>(ctx, lc, at, &c4)));
		tm = 3 * c2 <= 2 * count ? 2 : (3 * c4 <= 2 * count ? 4 : 8);
	}
	if (tm == 2) return launch_team<TI, kBT, 2>(ctx, B, count, cfg, rel, delta, adaptive);
	if (tm == 4) return launch_team<TI, kBT, 4>(ctx, B, count, cfg, rel, delta, adaptive);
	return launch_team<TI, kBT, 8>(ctx, B, count, cfg, rel, delta, adaptive);
}

}  // namespace
}  // namespace rsd

using namespace rsd;

extern "C" {

int rsd_batch_create(rsd_ctx* ctx, int32_t count, rsd_csr* const* A, rsd_batch** out) {
	if (!ctx || !out || count < 0 || (count && !A)) return set_error(RSD_EINVAL, "null argument");
	for (int32_t i = 0; i < count; ++i)
		if (!A[i]) return set_error(RSD_EINVAL, "null matrix in the batch");
	RSD_CUDA(cudaSetDevice(ctx->device));
	rsd_batch* B = new rsd_batch();
	B->count = count;
	B->A.assign(A, A + count);
	B->order.resize(count);
	std::iota(B->order.begin(), B->order.end(), 0);
	std::stable_sort(B->order.begin(), B->order.end(), [&](int32_t a, int32_t b) { return A[a]->nnz > A[b]->nnz; });
	size_t floats = 0;
	for (int32_t i = 0; i < count; ++i) floats += 5 * (size_t)pad_len(A[i]->n);
	B->wsBytes = std::max<size_t>(floats * sizeof(double), 256);   // room for FP64 inner vectors too
	const size_t descBytes = std::max<size_t>(sizeof(BatchProb<double>) * count, 64);
	cudaError_t e;
	if ((e = cudaMalloc(&B->ws, B->wsBytes)) != cudaSuccess || (e = cudaMalloc(&B->desc, descBytes)) != cudaSuccess ||
	    (e = cudaMalloc(&B->out, sizeof(BatchOut) * std::max(count, 1))) != cudaSuccess ||
	    (e = cudaMalloc(&B->dorder, sizeof(int32_t) * std::max(count, 1))) != cudaSuccess ||
	    (e = cudaMalloc(&B->next, sizeof(int32_t))) != cudaSuccess) {
		cudaFree(B->ws); cudaFree(B->desc); cudaFree(B->out); cudaFree(B->dorder); cudaFree(B->next);
		delete B;
		return cuda_error(e, "cudaMalloc (batch)");
	}
	if (count) {   // on the context stream, which the solves run on (B->order outlives the copy)
		RSD_CUDA(cudaMemcpyAsync(B->dorder, B->order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	}
	*out = B;
	return RSD_OK;
}

int rsd_batch_destroy(rsd_batch* B) {
	if (!B) return RSD_OK;
	cudaFree(B->ws); cudaFree(B->desc); cudaFree(B->out); cudaFree(B->dorder); cudaFree(B->next);
	delete B;
	return RSD_OK;
}

int rsd_batch_solve(rsd_ctx* ctx, rsd_batch* B, const rsd_solver_cfg* cfg, const double* const* b, double* const* x,
                    rsd_report* reports) {
	if (!ctx || !B || !cfg || (B->count && (!b || !x))) return set_error(RSD_EINVAL, "null argument");
	if (cfg->type != RSD_CG) return set_error(RSD_EINVAL, "the batched solver runs CG");
	if (cfg->max_iters < 0 || !(cfg->tol >= 0)) return set_error(RSD_EINVAL, "bad solver configuration");
	if (cfg->operator_type != RSD_OP_CSR) return set_error(RSD_EINVAL, "the batched solver takes operator_type RSD_OP_CSR");
	const int32_t count = B->count;
	if (!count) return RSD_OK;
	RSD_CUDA(cudaSetDevice(ctx->device));
	const bool mixed = cfg->precision == RSD_MIXED;
	const bool jacobi = cfg->precond == RSD_JACOBI;
	const int adaptive = !(cfg->reliable_delta > 0);
	const double delta = adaptive ? 0.1 : cfg->reliable_delta;
	const int rel = cfg->tol_type == RSD_TOL_RELATIVE;
	auto fill = [&](auto tag) -> int {
		using TI = decltype(tag);
		std::vector<BatchProb<TI>> d(count);
		TI* w = static_cast<TI*>(B->ws);
		for (int32_t i = 0; i < count; ++i) {
			rsd_csr* A = B->A[i];
			if (!b[i] || !x[i]) return set_error(RSD_EINVAL, "null vector in the batch");
			A->format = 0;                                      // the persistent kernel reads SELL-32
			if (mixed) RSD_CHECK(f32_sync(ctx, A)); else RSD_CHECK(sell_sync(ctx, A));
			BatchProb<TI>& P = d[i];
			P.n = A->n;
			P.nslices = A->nslices;
			P.A = MatView<TI>{A->sStart, A->sCol, mixed ? (const TI*)A->val32 : (const TI*)A->sVal, A->sCol16, A->sBase, A->sUni, A->sOffs, A->sPerm};
			P.A64 = MatView<double>{A->sStart, A->sCol, A->sVal, A->sCol16, A->sBase, A->sUni, A->sOffs, A->sPerm};
			P.sDiag = A->sDiag;
			P.b = b[i];
			P.x = x[i];
			const int64_t ns = pad_len(A->n);
			P.r = w; P.p = w + ns; P.Ap = w + 2 * ns; P.y = w + 3 * ns; P.invD = jacobi ? w + 4 * ns : nullptr;
			w += 5 * ns;
		}
		RSD_CUDA(cudaMemcpyAsync(B->desc, d.data(), sizeof(BatchProb<TI>) * count, cudaMemcpyHostToDevice, ctx->stream));
		return RSD_OK;
	};
	RSD_CHECK(mixed ? fill(float()) : fill(double()));
	RSD_CUDA(cudaMemsetAsync(B->next, 0, sizeof(int32_t), ctx->stream));
	// teams of CTAs of kBT threads (thread-block clusters) per problem when the device launches
	// clusters (RSD_BATCH_TEAM=0: one CTA per problem; 2, 4 or 8: that team size)
	const char* teamEnv = getenv("RSD_BATCH_TEAM");
	int clusterOk = 0;
	cudaDeviceGetAttribute(&clusterOk, cudaDevAttrClusterLaunch, ctx->device);
	if (clusterOk && !(teamEnv && teamEnv[0] == '0')) {
		const int forced = teamEnv ? atoi(teamEnv) : 0;
		const int rc = mixed ? launch_teams<float>(ctx, B, count, cfg, rel, delta, adaptive, forced)
		                     : launch_teams<double>(ctx, B, count, cfg, rel, delta, adaptive, forced);
		RSD_CHECK(rc);
	} else {
	int occ = 0;
	const void* kern = mixed ? (const void*)k_batch_cg<float> : (const void*)k_batch_cg<double>;
	RSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBT, 0));
	const int grid = std::max(1, std::min(count, ctx->num_sms * std::max(occ, 1)));
	if (mixed)
		k_batch_cg<float><<<grid, kBT, 0, ctx->stream>>>((const BatchProb<float>*)B->desc, B->dorder, count, B->next,
		                                                (BatchOut*)B->out, cfg->tol, rel, cfg->max_iters, delta, adaptive);
	else
		k_batch_cg<double><<<grid, kBT, 0, ctx->stream>>>((const BatchProb<double>*)B->desc, B->dorder, count, B->next,
		                                                 (BatchOut*)B->out, cfg->tol, rel, cfg->max_iters, delta, adaptive);
	}
	RSD_CUDA(cudaGetLastError());
	std::vector<BatchOut> h(count);
	RSD_CUDA(cudaMemcpyAsync(h.data(), B->out, sizeof(BatchOut) * count, cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	if (reports)
		for (int32_t i = 0; i < count; ++i) {
			rsd_report& R = reports[i];
			R = rsd_report{};
			R.converged = h[i].converged;
			R.status = h[i].status;
			R.iterations = h[i].iterations;
			R.initialResidual = h[i].res0;
			R.finalResidual = mixed ? h[i].trueRel * h[i].res0 : h[i].res;
			R.finalResidualRel = mixed ? h[i].trueRel : h[i].res / (h[i].res0 + 1e-50);
			R.trueResidualRel = h[i].trueRel;
			R.refinements = h[i].refinements;
		}
	return RSD_OK;
}

}  // extern "C"
