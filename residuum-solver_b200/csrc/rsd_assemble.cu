// Element loops on the device: matrix assembly (K, M, tangents) with scatter-add into the
// precomputed CSR pattern, vector assembly (load, residuals, mass products, matrix-free operator,
// Dirichlet lifting), diagonal and the adjoint's element gradient.
//
// Layout: a group of G lanes (G = next power of two >= nodes per element, at most 32) owns one
// element; lane a owns local node a.  Quadrature tables (N, dN/dxi per point and node, weights)
// live in shared memory.  Per quadrature point the Jacobian and any interpolated field are summed
// over the group with xor shuffles (every lane gets the total), and row a of the element matrix is
// formed against the tables, which all lanes of a warp read at the same address (broadcast):
//     (dN_a/dx . dN_b/dx) = sum_al G_a[al] dN_b/dxi_al,   G_a = invJ^T dN_a/dx,
// so no per-point exchange of physical gradients between lanes is needed.  Each lane then adds its
// row into the CSR values with FP64 atomics (colour-free scatter) after a binary search of the
// column in its row (the rows are sorted; Assembler.tpp:8-76).
//
// Geometry follows JacobianTransform (fem/geometry/JacobianTransform.tpp): measure = sqrt(det(J^T J)),
// 2D gradient transform with the true inverse, 3D with the cofactor/det layout (:160-185).
#include <cmath>

#include "rsd_kernels.cuh"

namespace rsd {

struct AsmParams {
	int64_t nelem;
	int32_t nq;
	// vector kernels: 0 load, 1 diffusion(U), 2 mass(U), 3 mass(Udot), 4 operator(V), 5 lift, 6 adjoint,
	// 7 Backward-Euler right-hand side load + coef*mass(U), 8 stage residual diffusion(U) + mass(Udot),
	// 9 Newton residual load - diffusion(U)
	int32_t which;
	const int32_t* __restrict__ elist;  // element subset (lift: elements touching a constrained node) or null
	const double* __restrict__ xyz;
	const int32_t* __restrict__ ien;
	const int32_t* __restrict__ t2a;
	const double* __restrict__ g;       // Dirichlet value per node
	const double* __restrict__ gPrev;   // Dirichlet value per node at the previous time (which 7), or null
	const double* __restrict__ kElem;
	const double* __restrict__ tables;  // [nq][G][4] (N, dxi, deta, dzeta) then w[nq]
	double kConst, rho, cp, time;
	DevExpr kExpr, dkExpr, srcExpr;
	// matrix
	const int32_t* __restrict__ rp;
	const int32_t* __restrict__ col;
	double* __restrict__ val;
	double cDiff, cMass, cTDiff, cTMass;
	// vectors
	const double* __restrict__ U;
	const double* __restrict__ Udot;
	const double* __restrict__ V;
	double coef;
	double* __restrict__ out;
	double outScale;
};

template <int NSD, int P>
struct Elem {
	static constexpr int NPE = (P + 1) * (P + 1) * (NSD == 3 ? P + 1 : 1);
	static constexpr int G = NPE <= 4 ? 4 : NPE <= 8 ? 8 : NPE <= 16 ? 16 : 32;
	static constexpr int EPW = 32 / G;
};

constexpr int kAsmThreads = 128;

// geometry at one quadrature point: J summed over the group, then inverse layout and measure
template <int NSD, int G>
__device__ __forceinline__ void qp_geometry(const double (&xa)[3], const double (&dxi)[3], double (&inv)[9], double& measure) {
	double J[9];
#pragma unroll
	for (int i = 0; i < NSD; ++i)
#pragma unroll
		for (int al = 0; al < NSD; ++al) J[i * NSD + al] = group_sum<G>(dxi[al] * xa[i]);
	if (NSD == 2) {
		const double g0 = J[0] * J[0] + J[2] * J[2], g1 = J[0] * J[1] + J[2] * J[3], g3 = J[1] * J[1] + J[3] * J[3];
		const double detg = g0 * g3 - g1 * g1;
		const double detJ = J[0] * J[3] - J[1] * J[2];
		const double di = 1.0 / detJ;
		inv[0] = di * J[3]; inv[1] = -di * J[1]; inv[2] = -di * J[2]; inv[3] = di * J[0];
		measure = sqrt(detg);
	} else {
		double gm[9];
#pragma unroll
		for (int b = 0; b < 3; ++b)
#pragma unroll
			for (int a = 0; a < 3; ++a) gm[b * 3 + a] = J[a] * J[b] + J[3 + a] * J[3 + b] + J[6 + a] * J[6 + b];
		const double detg = gm[0] * (gm[4] * gm[8] - gm[5] * gm[7]) - gm[1] * (gm[3] * gm[8] - gm[5] * gm[6]) + gm[2] * (gm[3] * gm[7] - gm[4] * gm[6]);
		const double detJ = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
		const double di = 1.0 / detJ;
		inv[0] = di * (J[4] * J[8] - J[5] * J[7]);
		inv[1] = -di * (J[3] * J[8] - J[5] * J[6]);
		inv[2] = di * (J[3] * J[7] - J[4] * J[6]);
		inv[3] = -di * (J[1] * J[8] - J[2] * J[7]);
		inv[4] = di * (J[0] * J[8] - J[2] * J[6]);
		inv[5] = -di * (J[0] * J[7] - J[1] * J[6]);
		inv[6] = di * (J[1] * J[5] - J[2] * J[4]);
		inv[7] = -di * (J[0] * J[5] - J[2] * J[3]);
		inv[8] = di * (J[0] * J[4] - J[1] * J[3]);
		measure = sqrt(detg);
	}
}

template <int NSD>
__device__ __forceinline__ void phys_grad(const double (&inv)[9], const double (&dxi)[3], double (&dx)[3]) {
#pragma unroll
	for (int i = 0; i < NSD; ++i) {
		double s = 0.0;
#pragma unroll
		for (int al = 0; al < NSD; ++al) s += inv[i * NSD + al] * dxi[al];
		dx[i] = s;
	}
}

// element data for the lane: node, row, coordinates; returns false when the lane has no node
template <int NSD, int P>
__device__ __forceinline__ bool load_node(const AsmParams& prm, bool valid, int64_t e, int a, int32_t& node, int32_t& row, double (&xa)[3]) {
	using E = Elem<NSD, P>;
	xa[0] = xa[1] = xa[2] = 0.0;
	node = 0; row = -1;
	if (!valid || a >= E::NPE) return false;
	node = prm.ien[e * E::NPE + a];
	row = prm.t2a[node];
#pragma unroll
	for (int i = 0; i < NSD; ++i) xa[i] = prm.xyz[(int64_t)node * NSD + i];
	return true;
}

template <int NSD, int P>
__device__ __forceinline__ void load_tables(const AsmParams& prm, double* sm) {
	using E = Elem<NSD, P>;
	const int total = prm.nq * E::G * 4 + prm.nq;
	for (int i = threadIdx.x; i < total; i += blockDim.x) sm[i] = prm.tables[i];
	__syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Assembler::assembleMatrix (fem/assembly/backend/cpu/Assembler.tpp:86-140)
// ---------------------------------------------------------------------------------------------
template <int NSD, int P>
__global__ void __launch_bounds__(kAsmThreads) k_asm_matrix(const AsmParams prm) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, G = E::G, EPW = E::EPW;
	extern __shared__ double sm[];
	load_tables<NSD, P>(prm, sm);
	const double* tab = sm;
	const double* wq = sm + prm.nq * G * 4;
	const int lane = threadIdx.x & 31, a = lane % G, slot = lane / G;
	const int warpsPerBlock = blockDim.x >> 5;
	const int64_t warpId = (int64_t)blockIdx.x * warpsPerBlock + (threadIdx.x >> 5);
	const int64_t warpStride = (int64_t)gridDim.x * warpsPerBlock;
	const bool needState = prm.kExpr.n || prm.dkExpr.n || prm.cTDiff != 0.0 || prm.cTMass != 0.0;
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += warpStride * EPW) {
		const int64_t e = eb + slot;
		int32_t node, row;
		double xa[3];
		const bool has = load_node<NSD, P>(prm, e < prm.nelem, e, a, node, row, xa);
		double Ua = 0.0;
		if (has && needState) Ua = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node];
		const double ke = (prm.kElem && e < prm.nelem) ? prm.kElem[e] : 1.0;
		double Ke[NPE];
#pragma unroll
		for (int b = 0; b < NPE; ++b) Ke[b] = 0.0;
		for (int q = 0; q < prm.nq; ++q) {
			const double* tq = tab + (q * G) * 4;
			double Na = 0.0, dxi[3] = {0.0, 0.0, 0.0};
			if (a < NPE) {
				Na = tq[a * 4];
#pragma unroll
				for (int al = 0; al < NSD; ++al) dxi[al] = tq[a * 4 + 1 + al];
			}
			double inv[9], measure;
			qp_geometry<NSD, G>(xa, dxi, inv, measure);
			double dx[3];
			phys_grad<NSD>(inv, dxi, dx);
			double k = prm.kConst, dk = 0.0, gradT[3] = {0.0, 0.0, 0.0};
			if (needState) {
				const double T = group_sum<G>(Na * Ua);
#pragma unroll
				for (int i = 0; i < NSD; ++i) gradT[i] = group_sum<G>(dx[i] * Ua);
				if (prm.kExpr.n) k = eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, T);
				if (prm.dkExpr.n) dk = eval_expr(prm.dkExpr, 0.0, 0.0, 0.0, 0.0, T);
			}
			const double wm = measure * wq[q];
			// G_a = invJ^T dx  ->  dN_a/dx . dN_b/dx = G_a . dN_b/dxi
			double Ga[3];
#pragma unroll
			for (int al = 0; al < NSD; ++al) {
				double s = 0.0;
#pragma unroll
				for (int i = 0; i < NSD; ++i) s += inv[i * NSD + al] * dx[i];
				Ga[al] = s;
			}
			const double cd = prm.cDiff * ke * k * wm;
			const double cm = prm.cMass * prm.rho * prm.cp * Na * wm;
			double ct = 0.0;
			if (prm.cTDiff != 0.0) {
				double s = 0.0;
#pragma unroll
				for (int i = 0; i < NSD; ++i) s += dx[i] * dk * gradT[i];
				ct = prm.cTDiff * s * wm;
			}
#pragma unroll
			for (int b = 0; b < NPE; ++b) {
				const double* tb = tq + b * 4;   // same address across the warp: broadcast
				double gd = 0.0;
#pragma unroll
				for (int al = 0; al < NSD; ++al) gd += Ga[al] * tb[1 + al];
				Ke[b] += cd * gd + (cm + ct) * tb[0];
			}
		}
		// scatter row a (free rows only) into the CSR values
		const int base = lane - a;
#pragma unroll
		for (int b = 0; b < NPE; ++b) {
			const int32_t cb = __shfl_sync(0xffffffffu, row, base + b);
			if (has && row >= 0 && cb >= 0) {
				const int end = prm.rp[row + 1];
				int lo = prm.rp[row], hi = end;
				while (lo < hi) {
					const int mid = (lo + hi) >> 1;
					const int32_t cm2 = prm.col[mid];
					if (cm2 < cb) lo = mid + 1; else hi = mid;
				}
				if (lo < end && prm.col[lo] == cb) atomicAdd(prm.val + lo, Ke[b]);
			}
		}
	}
}

// ---------------------------------------------------------------------------------------------
// Assembler::assembleVector (Assembler.tpp:199-255), BoundaryApplicator::applyEssentialBCs
// (fem/boundary/backend/cpu/BoundaryApplicator.tpp:7-64) and the adjoint element gradient.
// The vector forms use sum_b (dN_a/dx . dN_b/dx) V_b = dN_a/dx . grad V with grad V summed over
// the group, and sum_b N_a N_b V_b = N_a V(x_q).
// ---------------------------------------------------------------------------------------------
template <int NSD, int P>
__global__ void __launch_bounds__(kAsmThreads) k_asm_vector(const AsmParams prm) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, G = E::G, EPW = E::EPW;
	extern __shared__ double sm[];
	load_tables<NSD, P>(prm, sm);
	const double* tab = sm;
	const double* wq = sm + prm.nq * G * 4;
	const int lane = threadIdx.x & 31, a = lane % G, slot = lane / G;
	const int warpsPerBlock = blockDim.x >> 5;
	const int64_t warpId = (int64_t)blockIdx.x * warpsPerBlock + (threadIdx.x >> 5);
	const int64_t warpStride = (int64_t)gridDim.x * warpsPerBlock;
	const int which = prm.which;
	const bool kT = prm.kExpr.n != 0;
	const bool hasLoad = which == 0 || which == 7 || which == 9;
	const bool opState = kT && which == 4;   // the operator takes k(T) from the state U, not the operand
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += warpStride * EPW) {
		const int64_t idx = eb + slot;
		const bool inRange = idx < prm.nelem;
		const int64_t e = inRange ? (prm.elist ? (int64_t)prm.elist[idx] : idx) : 0;
		int32_t node, row;
		double xa[3];
		const bool has = load_node<NSD, P>(prm, inRange, e, a, node, row, xa);
		// gathered operand V, second operand W (Udot) and state U (for k(T))
		double Va = 0.0, Wa = 0.0, Ua = 0.0;
		if (has) {
			const double fullU = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node];
			switch (which) {
				case 1: case 2: case 8: case 9: Va = fullU; break;                          // GatherMode::Full
				case 3: Va = (row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0; break;           // Free
				case 4: Va = (row >= 0 && prm.V) ? prm.V[row] : 0.0; break;                 // Free
				case 5: Va = row >= 0 ? 0.0 : prm.g[node]; break;                           // Constrained
				case 6: Va = (row >= 0 && prm.V) ? prm.V[row] : 0.0; Ua = fullU; break;     // lambda (Free), T (Full)
				case 7: Va = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : (prm.gPrev ? prm.gPrev[node] : prm.g[node]); break;
				default: break;
			}
			if (which == 8) Wa = (row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
			if (opState) Ua = fullU;
		}
		const double ke = (prm.kElem && inRange) ? prm.kElem[e] : 1.0;
		double Fa = 0.0, ge = 0.0;
		for (int q = 0; q < prm.nq; ++q) {
			const double* tq = tab + (q * G) * 4;
			double Na = 0.0, dxi[3] = {0.0, 0.0, 0.0};
			if (a < NPE) {
				Na = tq[a * 4];
#pragma unroll
				for (int al = 0; al < NSD; ++al) dxi[al] = tq[a * 4 + 1 + al];
			}
			double inv[9], measure;
			qp_geometry<NSD, G>(xa, dxi, inv, measure);
			double dx[3];
			phys_grad<NSD>(inv, dxi, dx);
			const double wm = measure * wq[q];
			if (hasLoad) {
				double xq[3] = {0.0, 0.0, 0.0};
#pragma unroll
				for (int i = 0; i < NSD; ++i) xq[i] = group_sum<G>(Na * xa[i]);
				const double f = prm.srcExpr.n ? eval_expr(prm.srcExpr, prm.time, xq[0], xq[1], NSD == 3 ? xq[2] : 0.0, 0.0) : 0.0;
				Fa += (f * Na) * wm;
				if (which == 0) continue;
			}
			const double Vq = group_sum<G>(Na * Va);
			double gv[3] = {0.0, 0.0, 0.0};
#pragma unroll
			for (int i = 0; i < NSD; ++i) gv[i] = group_sum<G>(dx[i] * Va);
			if (which == 6) {
				double gt[3];
#pragma unroll
				for (int i = 0; i < NSD; ++i) gt[i] = group_sum<G>(dx[i] * Ua);
				double s = 0.0;
#pragma unroll
				for (int i = 0; i < NSD; ++i) s += gv[i] * gt[i];
				ge += s * wm;
				continue;
			}
			double k = prm.kConst;
			if (kT) {
				// diffusion of U takes T from U itself; the operator from the state; the lift
				// interpolates no state, so k is taken at T = 0 there
				const double T = (which == 1 || which == 8 || which == 9) ? Vq : opState ? group_sum<G>(Na * Ua) : 0.0;
				k = eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, T);
			}
			double dd = 0.0;
#pragma unroll
			for (int i = 0; i < NSD; ++i) dd += dx[i] * gv[i];
			const double mass = prm.rho * prm.cp * Na * Vq;
			switch (which) {
				case 1: Fa += ke * k * dd * wm; break;
				case 2: case 3: Fa += mass * wm; break;
				case 4: Fa += (ke * k * dd + prm.coef * mass) * wm; break;
				case 5: Fa += (prm.cDiff * ke * k * dd + prm.cMass * mass) * wm; break;
				case 7: Fa += prm.coef * mass * wm; break;
				case 8: {
					const double Wq = group_sum<G>(Na * Wa);
					Fa += (ke * k * dd + prm.rho * prm.cp * Na * Wq) * wm;
					break;
				}
				case 9: Fa -= ke * k * dd * wm; break;
				default: break;
			}
		}
		if (which == 6) {
			if (a == 0 && inRange) prm.out[e] = ge;
		} else if (has && row >= 0) {
			atomicAdd(prm.out + row, prm.outScale * Fa);
		}
	}
}

// Assembler::assembleDiagonal (Assembler.tpp:142-197) for c_diff*Diffusion + c_mass*Mass
template <int NSD, int P>
__global__ void __launch_bounds__(kAsmThreads) k_asm_diag(const AsmParams prm) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, G = E::G, EPW = E::EPW;
	extern __shared__ double sm[];
	load_tables<NSD, P>(prm, sm);
	const double* tab = sm;
	const double* wq = sm + prm.nq * G * 4;
	const int lane = threadIdx.x & 31, a = lane % G, slot = lane / G;
	const int warpsPerBlock = blockDim.x >> 5;
	const int64_t warpId = (int64_t)blockIdx.x * warpsPerBlock + (threadIdx.x >> 5);
	const int64_t warpStride = (int64_t)gridDim.x * warpsPerBlock;
	const bool needT = prm.kExpr.n != 0;
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += warpStride * EPW) {
		const int64_t e = eb + slot;
		int32_t node, row;
		double xa[3];
		const bool has = load_node<NSD, P>(prm, e < prm.nelem, e, a, node, row, xa);
		double Ua = 0.0;
		if (has && needT) Ua = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node];
		const double ke = (prm.kElem && e < prm.nelem) ? prm.kElem[e] : 1.0;
		double Da = 0.0;
		for (int q = 0; q < prm.nq; ++q) {
			const double* tq = tab + (q * G) * 4;
			double Na = 0.0, dxi[3] = {0.0, 0.0, 0.0};
			if (a < NPE) {
				Na = tq[a * 4];
#pragma unroll
				for (int al = 0; al < NSD; ++al) dxi[al] = tq[a * 4 + 1 + al];
			}
			double inv[9], measure;
			qp_geometry<NSD, G>(xa, dxi, inv, measure);
			double dx[3];
			phys_grad<NSD>(inv, dxi, dx);
			double k = prm.kConst;
			if (needT) k = eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, group_sum<G>(Na * Ua));
			double dd = 0.0;
#pragma unroll
			for (int i = 0; i < NSD; ++i) dd += dx[i] * dx[i];
			Da += (prm.cDiff * ke * k * dd + prm.cMass * prm.rho * prm.cp * Na * Na) * measure * wq[q];
		}
		if (has && row >= 0) atomicAdd(prm.out + row, Da);
	}
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
// Lagrange1D::eval / evalFirstDerivative (fem/basis/Lagrange1D.tpp:4-51)
static void lagrange1d(int p, double xi, double* N, double* dN) {
	if (p == 1) { N[0] = 0.5 * (1.0 - xi); N[1] = 0.5 * (1.0 + xi); dN[0] = -0.5; dN[1] = 0.5; }
	else if (p == 2) {
		N[0] = 0.5 * xi * (xi - 1.0); N[1] = (1.0 - xi) * (1.0 + xi); N[2] = 0.5 * xi * (xi + 1.0);
		dN[0] = xi - 0.5; dN[1] = -2.0 * xi; dN[2] = xi + 0.5;
	} else {
		N[0] = (-9.0 / 16.0) * (xi - (1.0 / 3.0)) * (xi - 1.0) * (xi + (1.0 / 3.0));
		N[1] = (27.0 / 16.0) * (xi - 1.0) * (xi - (1.0 / 3.0)) * (xi + 1.0);
		N[2] = (-27.0 / 16.0) * (xi + (1.0 / 3.0)) * (xi - 1.0) * (xi + 1.0);
		N[3] = (9.0 / 16.0) * (xi - (1.0 / 3.0)) * (xi + 1.0) * (xi + (1.0 / 3.0));
		dN[0] = (-9.0 / 16.0) * (3.0 * xi * xi - 2.0 * xi - (1.0 / 9.0));
		dN[1] = (27.0 / 16.0) * (3.0 * xi * xi - (2.0 / 3.0) * xi - 1.0);
		dN[2] = (-27.0 / 16.0) * (3.0 * xi * xi + (2.0 / 3.0) * xi - 1.0);
		dN[3] = (9.0 / 16.0) * (3.0 * xi * xi + 2.0 * xi - (1.0 / 9.0));
	}
}

// Gauss-Legendre points and weights, the values GaussQuadrature1D tabulates
// (fem/quadrature/GaussQuadrature1D.tpp:4-71)
static void gauss_legendre(int n, double* x, double* w) {
	static const double X[6][5] = {{0}, {0.0}, {-0.5773502691896257, 0.5773502691896257},
		{-0.7745966692414834, 0.0, 0.7745966692414834},
		{-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526},
		{-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640}};
	static const double W[6][5] = {{0}, {2.0}, {1.0, 1.0}, {0.5555555555555556, 0.8888888888888889, 0.5555555555555556},
		{0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538},
		{0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665, 0.2369268850561891}};
	for (int i = 0; i < n; ++i) { x[i] = X[n][i]; w[i] = W[n][i]; }
}

static int group_width(int npe) { return npe <= 4 ? 4 : npe <= 8 ? 8 : npe <= 16 ? 16 : 32; }

// tensor-product tables in quadrature-point order (x fastest, GaussQuadratureHex.tpp:4-49) and
// node order (x fastest, LagrangeHex.tpp:4-55): [nq][G][4] = (N, dN/dxi, dN/deta, dN/dzeta), then w[nq]
int build_tables(rsd_heat* h) {
	const int nsd = h->m->nsd, p = h->m->order, q1 = h->nq1, G = group_width(h->m->npe);
	double gx[5], gw[5];
	gauss_legendre(q1, gx, gw);
	const int nq = nsd == 3 ? q1 * q1 * q1 : q1 * q1;
	std::vector<double> t(nq * G * 4 + nq, 0.0);
	int q = 0;
	for (int k = 0; k < (nsd == 3 ? q1 : 1); ++k)
		for (int j = 0; j < q1; ++j)
			for (int i = 0; i < q1; ++i, ++q) {
				double Nx[4], Ny[4], Nz[4] = {1, 1, 1, 1}, dx[4], dy[4], dz[4] = {0, 0, 0, 0};
				lagrange1d(p, gx[i], Nx, dx);
				lagrange1d(p, gx[j], Ny, dy);
				if (nsd == 3) lagrange1d(p, gx[k], Nz, dz);
				t[nq * G * 4 + q] = nsd == 3 ? gw[i] * gw[j] * gw[k] : gw[i] * gw[j];
				int a = 0;
				for (int c = 0; c < (nsd == 3 ? p + 1 : 1); ++c)
					for (int b = 0; b <= p; ++b)
						for (int aa = 0; aa <= p; ++aa, ++a) {
							double* e = &t[(q * G + a) * 4];
							if (nsd == 2) { e[0] = Nx[aa] * Ny[b]; e[1] = dx[aa] * Ny[b]; e[2] = Nx[aa] * dy[b]; }
							else {
								e[0] = Nx[aa] * Ny[b] * Nz[c];
								e[1] = dx[aa] * Ny[b] * Nz[c];
								e[2] = Nx[aa] * dy[b] * Nz[c];
								e[3] = Nx[aa] * Ny[b] * dz[c];
							}
						}
			}
	h->nq = nq;
	if (h->tables) cudaFree(h->tables);
	RSD_CUDA(cudaMalloc(&h->tables, sizeof(double) * t.size()));
	RSD_CUDA(cudaMemcpy(h->tables, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice));
	return RSD_OK;
}

static AsmParams params_for(const rsd_heat* h) {
	AsmParams p{};
	p.nelem = h->m->nelem;
	p.nq = h->nq;
	p.xyz = h->m->xyz;
	p.ien = h->m->ien;
	p.t2a = h->t2a;
	p.g = h->g;
	p.kElem = h->kElem;
	p.tables = h->tables;
	p.kConst = h->k_const;
	p.rho = h->rho;
	p.cp = h->cp;
	p.time = h->time;
	p.kExpr = h->kExpr;
	p.dkExpr = h->dkExpr;
	p.srcExpr = h->srcExpr;
	p.outScale = 1.0;
	return p;
}

static int launch_one(void (*kern)(const AsmParams), dim3 gr, size_t smem, rsd_ctx* ctx, const AsmParams& p) {
	if (smem > 48 * 1024) RSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	kern<<<gr, kAsmThreads, smem, ctx->stream>>>(p);
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

#define RSD_ASM_DISPATCH(KERNEL)                                                              \
	static int launch_##KERNEL(rsd_ctx* ctx, const rsd_heat* h, const AsmParams& p) {         \
		const int nsd = h->m->nsd, ord = h->m->order, G = group_width(h->m->npe);             \
		const size_t smem = sizeof(double) * (h->nq * G * 4 + h->nq);                         \
		const int epb = (kAsmThreads / 32) * (32 / G);                                        \
		int64_t blocks = (p.nelem + epb - 1) / epb;                                           \
		blocks = std::min<int64_t>(blocks, (int64_t)ctx->num_sms * 16);                       \
		dim3 gr((unsigned)std::max<int64_t>(blocks, 1));                                      \
		if (nsd == 2 && ord == 1) return launch_one(KERNEL<2, 1>, gr, smem, ctx, p);          \
		if (nsd == 2 && ord == 2) return launch_one(KERNEL<2, 2>, gr, smem, ctx, p);          \
		if (nsd == 2 && ord == 3) return launch_one(KERNEL<2, 3>, gr, smem, ctx, p);          \
		if (nsd == 3 && ord == 1) return launch_one(KERNEL<3, 1>, gr, smem, ctx, p);          \
		if (nsd == 3 && ord == 2) return launch_one(KERNEL<3, 2>, gr, smem, ctx, p);          \
		return set_error(RSD_EINVAL, "unsupported element");                                  \
	}

RSD_ASM_DISPATCH(k_asm_matrix)
RSD_ASM_DISPATCH(k_asm_vector)
RSD_ASM_DISPATCH(k_asm_diag)

int assemble_matrix(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double cTDiff, double cTMass,
                    const double* U, const double* Udot, rsd_csr* A) {
	if (A->n != h->n || A->nnz != h->K->nnz) return set_error(RSD_EINVAL, "matrix does not have the problem's pattern");
	AsmParams p = params_for(h);
	p.rp = A->rowPtr; p.col = A->col; p.val = A->val;
	p.cDiff = cDiff; p.cMass = cMass; p.cTDiff = cTDiff; p.cTMass = cTMass;
	p.U = U; p.Udot = Udot;
	RSD_CUDA(cudaMemsetAsync(A->val, 0, sizeof(double) * std::max<int64_t>(A->nnz, 1), ctx->stream));
	A->version++;
	const int pr = prof_begin(ctx, PF_ASM_MATRIX);
	const int rc = launch_k_asm_matrix(ctx, h, p);
	prof_end(ctx, pr);
	return rc;
}

int assemble_vector(rsd_ctx* ctx, rsd_heat* h, int which, double coef, const double* U, const double* Udot,
                    const double* operand, double* out, double outScale, bool accumulate) {
	AsmParams p = params_for(h);
	p.which = which; p.coef = coef; p.U = U; p.Udot = Udot; p.V = operand; p.out = out; p.outScale = outScale;
	if (which == 7 && h->gPrevValid) p.gPrev = h->gPrev;
	if (!accumulate) {
		const int64_t len = which == 6 ? h->m->nelem : h->n;
		RSD_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * std::max<int64_t>(len, 1), ctx->stream));
	}
	const int pr = prof_begin(ctx, PF_ASM_VECTOR);
	const int rc = launch_k_asm_vector(ctx, h, p);
	prof_end(ctx, pr);
	return rc;
}

// the lift visits only elements with a constrained node: every other element adds exact zeros
int assemble_lift(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double* F) {
	if (h->nbElems == 0) return RSD_OK;
	AsmParams p = params_for(h);
	p.which = 5; p.cDiff = cDiff; p.cMass = cMass; p.out = F; p.outScale = -1.0;
	p.elist = h->bElems; p.nelem = h->nbElems;
	const int pr = prof_begin(ctx, PF_ASM_VECTOR);
	const int rc = launch_k_asm_vector(ctx, h, p);
	prof_end(ctx, pr);
	return rc;
}

int assemble_diagonal(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, const double* U, double* d) {
	AsmParams p = params_for(h);
	p.cDiff = cDiff; p.cMass = cMass; p.U = U; p.out = d;
	RSD_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * std::max<int64_t>(h->n, 1), ctx->stream));
	return launch_k_asm_diag(ctx, h, p);
}

}  // namespace rsd
