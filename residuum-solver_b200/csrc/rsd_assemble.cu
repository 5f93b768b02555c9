// Element loops on the device: matrix assembly (K, M, tangents) with scatter-add into the
// precomputed CSR pattern, vector assembly (load, residuals, mass products, matrix-free operator,
// Dirichlet lifting), diagonal and the adjoint's element gradient.
//
// Layout: a group of G lanes (G = next power of two >= nodes per element, at most 32) owns one
// element, several elements per warp.  Each element goes through three phases:
//   1. lane a stages node a (coordinates and the gathered fields) in shared memory;
//   2. lane q evaluates quadrature point q (q = lane, lane + G, ...): Jacobian, inverse layout,
//      measure, interpolated state and fields, the conductivity model and the source, written
//      once as a per-point record (no point is evaluated twice and no shuffle is needed);
//   3. lane a forms its row of the element matrix (or its vector entry) from the records, which
//      the lanes of a group read at one address (broadcast), and from the shape-function tables:
//          dN_a/dx . dN_b/dx = sum_al G_a[al] dN_b/dxi_al,   G_a = invJ^T dN_a/dx,
//      where dN_b/dxi at a point is the same table entry for every lane of the warp.
// Matrix rows are added with FP64 atomics (colour-free scatter) straight into the SELL-32 execution
// layout of the values, at positions from a precomputed element -> slot map, or, without the map,
// after a binary search of the column in the sorted CSR row (fem/assembly/backend/cpu/Assembler.tpp:8-76).
//
// Geometry follows JacobianTransform (fem/geometry/JacobianTransform.tpp): measure = sqrt(det(J^T J)),
// 2D gradient transform with the true inverse, 3D with the cofactor/det layout (:160-185).
#include <cmath>
#include <map>
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {

// Position j of CSR entry q (column c) of row `row` in its SELL-32 slice: the rank within the row,
// or in a stencil slice the index of the offset c - row in the slice's sorted pattern (whose padding
// repeats the last offset, so the first match is the entry).  iperm: the row's slot row in a layout
// whose slices hold the rows in another order, or null
__device__ __forceinline__ int32_t sell_rank(const int32_t* sStart, const int32_t* sUni, const int32_t* sOffs,
                                             const int32_t* iperm, const int32_t* rp, int32_t row, int32_t q, int32_t c) {
	const int32_t sl = (iperm ? iperm[row] : row) >> 5;
	const int32_t u = sUni ? sUni[sl] : -1;
	if (u < 0) return q - rp[row];
	const int32_t* pat = sOffs + u;
	const int32_t off = c - row;
	int lo = 0, hi = (sStart[sl + 1] - sStart[sl]) >> 5;
	while (lo < hi) {
		const int mid = (lo + hi) >> 1;
		if (pat[mid] < off) lo = mid + 1; else hi = mid;
	}
	return lo;
}

// SELL-32 slot of CSR entry q (column c) of row `row`
__device__ __forceinline__ int32_t sell_slot(const int32_t* sStart, const int32_t* sUni, const int32_t* sOffs,
                                             const int32_t* iperm, const int32_t* rp, int32_t row, int32_t q, int32_t c) {
	const int32_t j = sell_rank(sStart, sUni, sOffs, iperm, rp, row, q, c);
	const int32_t sr = iperm ? iperm[row] : row;
	return sStart[sr >> 5] + 64 * (j >> 1) + 2 * (sr & 31) + (j & 1);
}

struct AsmParams {
	int64_t nelem;
	int32_t nq;
	int32_t pts;   // per-point records staged per element: nq, or 0 when every element of the launch is affine
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
	DevExpr cpExpr, dcpExpr;            // cp(T), dcp/dT (n = 0: the constant cp)
	int32_t aniso;                      // K = k kS (anisotropic shape), else k I
	double kS[9];                       // row-major, stride 3
	// matrix: CSR pattern for the column search, SELL-32 slice starts and values for the scatter
	const int32_t* __restrict__ rp;
	const int32_t* __restrict__ col;
	const int32_t* __restrict__ sStart;
	const int32_t* __restrict__ sUni;   // stencil slices (pattern start per slice, -1 for none), or null
	const int32_t* __restrict__ sOffs;
	const int32_t* __restrict__ sPerm;  // slot row -> matrix row of the layout, or null (identity)
	const int32_t* __restrict__ sIperm; // matrix row -> slot row, or null
	double* __restrict__ val;
	float* __restrict__ val32;          // row-gather assembly: the FP32 copy written alongside, or null
	// element -> column-rank map [e][a][b]: the SELL-32 position j (sell_rank) of column t2a[node_b] in
	// row t2a[node_a] (0xFF when either DOF is constrained), rows of (NPE rounded up to 8) bytes; or null
	const uint8_t* __restrict__ ranks;
	// affine fast path (launch-uniform `fast`): per-element flags and the reference integrals
	int32_t fast;
	const uint8_t* __restrict__ affine;
	const double* __restrict__ geo;     // per affine element: the 6 coefficients of the tables, |J|, 0
	const double* __restrict__ ktab;
	double cDiff, cMass, cTDiff, cTMass;
	// vectors
	const double* __restrict__ U;
	const double* __restrict__ Udot;
	const double* __restrict__ V;
	double coef;
	double* __restrict__ out;
	double outScale;
	// vector kernels: the whole launch returns at once when *skip != 0 (a finished solve's flag), or null
	const int32_t* __restrict__ skip;
	const int32_t* __restrict__ erow;   // [e][a]: the free row of node a of element e (-1: constrained), or null
};

template <int NSD, int P>
struct Elem {
	static constexpr int NPE = (P + 1) * (P + 1) * (NSD == 3 ? P + 1 : 1);
	static constexpr int G = NPE <= 4 ? 4 : NPE <= 8 ? 8 : NPE <= 16 ? 16 : 32;
	static constexpr int EPW = 32 / G;
};

constexpr int kAsmThreads = 128;
constexpr int kAsmWarps = kAsmThreads / 32;

// per-point record: inverse layout (9), w*measure, k, dk, grad T (3), V, grad V (3), W, f, cp, dcp/dT, T rate
constexpr int R_INV = 0, R_WM = 9, R_K = 10, R_DK = 11, R_GT = 12, R_V = 15, R_GV = 16, R_W = 19, R_F = 20, R_CP = 21,
              R_DCP = 22, R_TR = 23, REC = 24;
// per-node staging: x (3), U, V, W, rate of U
constexpr int N_X = 0, N_U = 3, N_V = 4, N_W = 5, N_R = 6, NREC = 7;

__host__ __device__ inline int table_stride(int G) { return G * 4 + 1; }                      // odd: no bank conflicts across q
__host__ __device__ inline int node_area(int npe) { return npe * NREC + 1; }
__host__ __device__ inline int point_area(int nq) { return nq * REC + 1; }
// reference-integral tables of the affine path: NT gradient-product tables and the mass table, rows
// of npe entries padded to an odd stride (a group's lanes read distinct rows without bank conflicts)
__host__ __device__ inline int ktab_count(int nsd) { return nsd == 3 ? 7 : 4; }
__host__ __device__ inline int ktab_stride(int npe) { return npe | 1; }

size_t asm_smem_bytes(int npe, int nq, int nsd, bool fast, int pts) {
	const int G = npe <= 4 ? 4 : npe <= 8 ? 8 : npe <= 16 ? 16 : 32;
	const int EPW = 32 / G;
	const size_t kt = fast ? (size_t)ktab_count(nsd) * npe * ktab_stride(npe) : 0;
	return sizeof(double) * ((size_t)nq * table_stride(G) + nq + (size_t)kAsmWarps * EPW * (node_area(npe) + point_area(pts)) + kt);
}

// what phase 2 must evaluate
struct Needs {
	bool state;    // T, grad T (k(T), cp(T), tangents)
	bool field;    // V, grad V
	bool field2;   // W (second operand, mass only)
	bool load;     // x_q and f(t, x_q)
	bool rate;     // the rate of T (TangentMassForm)
};

// the conductivity's shape applied to a vector: out = kS v (anisotropic) or v
template <int NSD>
__device__ __forceinline__ void shape_apply(const AsmParams& prm, const double* v, double* out) {
	if (!prm.aniso) {
#pragma unroll
		for (int i = 0; i < NSD; ++i) out[i] = v[i];
		return;
	}
#pragma unroll
	for (int i = 0; i < NSD; ++i) {
		double s = 0.0;
#pragma unroll
		for (int j = 0; j < NSD; ++j) s += prm.kS[i * 3 + j] * v[j];
		out[i] = s;
	}
}
// out = kS^T v
template <int NSD>
__device__ __forceinline__ void shape_apply_t(const AsmParams& prm, const double* v, double* out) {
	if (!prm.aniso) {
#pragma unroll
		for (int i = 0; i < NSD; ++i) out[i] = v[i];
		return;
	}
#pragma unroll
	for (int j = 0; j < NSD; ++j) {
		double s = 0.0;
#pragma unroll
		for (int i = 0; i < NSD; ++i) s += prm.kS[i * 3 + j] * v[i];
		out[j] = s;
	}
}
// grad N_a . K grad V / k with K = k kS: the diffusion integrand's direction part
template <int NSD>
__device__ __forceinline__ double shape_dot(const AsmParams& prm, const double* ga, const double* gv) {
	double sv[3];
	shape_apply<NSD>(prm, gv, sv);
	double s = 0.0;
#pragma unroll
	for (int i = 0; i < NSD; ++i) s += ga[i] * sv[i];
	return s;
}

template <int NSD, int P>
__device__ __forceinline__ void stage_tables(const AsmParams& prm, double* sm) {
	using E = Elem<NSD, P>;
	const int TS = table_stride(E::G);
	for (int i = threadIdx.x; i < prm.nq * E::G * 4; i += blockDim.x) {
		const int q = i / (E::G * 4), r = i % (E::G * 4);
		sm[q * TS + r] = prm.tables[i];
	}
	for (int i = threadIdx.x; i < prm.nq; i += blockDim.x) sm[prm.nq * TS + i] = prm.tables[prm.nq * E::G * 4 + i];
	__syncthreads();
}

// Geometry of one point from its Jacobian J[i * NSD + al] = dx_i/dxi_al: returns det(J^T J) (the
// squared measure) and, when INV, the inverse layout inv[i * NSD + al] = (J^-T)_{i al}.
template <int NSD, bool INV>
__device__ __forceinline__ double jac_geom(const double (&J)[9], double (&inv)[9]) {
	double detg;
	if (NSD == 2) {
		const double g0 = J[0] * J[0] + J[2] * J[2], g1 = J[0] * J[1] + J[2] * J[3], g3 = J[1] * J[1] + J[3] * J[3];
		detg = g0 * g3 - g1 * g1;
		if (INV) {
			const double di = 1.0 / (J[0] * J[3] - J[1] * J[2]);
			inv[0] = di * J[3]; inv[1] = -di * J[1]; inv[2] = -di * J[2]; inv[3] = di * J[0];
		}
	} else {
		double gm[9];
#pragma unroll
		for (int b = 0; b < 3; ++b)
#pragma unroll
			for (int a = 0; a < 3; ++a) gm[b * 3 + a] = J[a] * J[b] + J[3 + a] * J[3 + b] + J[6 + a] * J[6 + b];
		detg = gm[0] * (gm[4] * gm[8] - gm[5] * gm[7]) - gm[1] * (gm[3] * gm[8] - gm[5] * gm[6]) + gm[2] * (gm[3] * gm[7] - gm[4] * gm[6]);
		if (INV) {
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
		}
	}
	return detg;
}

// phase 2: one quadrature point, all inputs from the staged node data.  GRAD = false (mass and load
// terms only): no inverse Jacobian, no gradients and no conductivity model are evaluated.
template <int NSD, int P, bool GRAD>
__device__ __forceinline__ void eval_point(const AsmParams& prm, const Needs& nd, const double* tq, double w,
                                           const double* nodes, double ke, double* rec) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE;
	double J[9];
#pragma unroll
	for (int i = 0; i < NSD * NSD; ++i) J[i] = 0.0;
	double Tq = 0.0, Rq = 0.0, Vq = 0.0, Wq = 0.0, xq[3] = {0.0, 0.0, 0.0}, dT[3] = {0.0, 0.0, 0.0}, dV[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
	for (int b = 0; b < NPE; ++b) {
		const double* t = tq + b * 4;
		const double* nb = nodes + b * NREC;
#pragma unroll
		for (int i = 0; i < NSD; ++i)
#pragma unroll
			for (int al = 0; al < NSD; ++al) J[i * NSD + al] += t[1 + al] * nb[N_X + i];
		if (nd.state) {
			Tq += t[0] * nb[N_U];
			if (GRAD)
#pragma unroll
				for (int al = 0; al < NSD; ++al) dT[al] += t[1 + al] * nb[N_U];
		}
		if (nd.rate) Rq += t[0] * nb[N_R];
		if (nd.field) {
			Vq += t[0] * nb[N_V];
			if (GRAD)
#pragma unroll
				for (int al = 0; al < NSD; ++al) dV[al] += t[1 + al] * nb[N_V];
		}
		if (nd.field2) Wq += t[0] * nb[N_W];
		if (nd.load)
#pragma unroll
			for (int i = 0; i < NSD; ++i) xq[i] += t[0] * nb[N_X + i];
	}
	double inv[9];
	const double detg = jac_geom<NSD, GRAD>(J, inv);
	// SpecificHeatModel (SpecificHeatModel.hpp:35-61): cp and dcp/dT at the point's T
	rec[R_CP] = prm.cpExpr.n ? eval_expr(prm.cpExpr, 0.0, 0.0, 0.0, 0.0, nd.state ? Tq : 0.0) : prm.cp;
	rec[R_DCP] = prm.dcpExpr.n ? eval_expr(prm.dcpExpr, 0.0, 0.0, 0.0, 0.0, nd.state ? Tq : 0.0) : 0.0;
	rec[R_TR] = Rq;
	if (!GRAD) {
		rec[R_WM] = sqrt(detg) * w;
		if (nd.field) rec[R_V] = Vq;
		if (nd.field2) rec[R_W] = Wq;
		rec[R_K] = 0.0;
		rec[R_DK] = 0.0;
		if (nd.load) rec[R_F] = prm.srcExpr.n ? eval_expr(prm.srcExpr, prm.time, xq[0], xq[1], NSD == 3 ? xq[2] : 0.0, 0.0) : 0.0;
		return;
	}
#pragma unroll
	for (int i = 0; i < NSD * NSD; ++i) rec[R_INV + i] = inv[i];
	rec[R_WM] = sqrt(detg) * w;
	// physical gradients of the interpolated fields: grad_i = sum_al inv[i][al] d/dxi_al
	if (nd.state) {
#pragma unroll
		for (int i = 0; i < NSD; ++i) {
			double s = 0.0;
#pragma unroll
			for (int al = 0; al < NSD; ++al) s += inv[i * NSD + al] * dT[al];
			rec[R_GT + i] = s;
		}
	}
	if (nd.field) {
		rec[R_V] = Vq;
#pragma unroll
		for (int i = 0; i < NSD; ++i) {
			double s = 0.0;
#pragma unroll
			for (int al = 0; al < NSD; ++al) s += inv[i * NSD + al] * dV[al];
			rec[R_GV + i] = s;
		}
	}
	if (nd.field2) rec[R_W] = Wq;
	// models: k(T) and dk/dT (ConductivityModel.hpp:60-96), the per-element factor applies to diffusion
	const double k = prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, nd.state ? Tq : 0.0) : prm.kConst;
	rec[R_K] = ke * k;
	rec[R_DK] = prm.dkExpr.n ? eval_expr(prm.dkExpr, 0.0, 0.0, 0.0, 0.0, nd.state ? Tq : 0.0) : 0.0;
	if (nd.load) rec[R_F] = prm.srcExpr.n ? eval_expr(prm.srcExpr, prm.time, xq[0], xq[1], NSD == 3 ? xq[2] : 0.0, 0.0) : 0.0;
}

// lane a's physical gradient at a point: dx_i = sum_al inv[i][al] dN_a/dxi_al
template <int NSD>
__device__ __forceinline__ void node_grad(const double* rec, const double* ta, double (&dx)[3]) {
#pragma unroll
	for (int i = 0; i < NSD; ++i) {
		double s = 0.0;
#pragma unroll
		for (int al = 0; al < NSD; ++al) s += rec[R_INV + i * NSD + al] * ta[1 + al];
		dx[i] = s;
	}
}

// Affine elements: with J constant, sum_q w_q |J| (J^-T dN_a).(J^-T dN_b) = |J| sum_{al,be} C_{al be}
// S^{al be}_ab with C = J^-1 J^-T and S the reference integrals sum_q w_q dN_a/dxi_al dN_b/dxi_be.
// C is symmetric, so the tables hold S^{al al} and S^{al be} + S^{be al} (al < be): coefficient k of
// table k in the order (00, 11, [22,] 01, [02, 12]).
template <int NSD>
__device__ __forceinline__ void coefs_from_inv(const double (&inv)[9], double (&c)[6]) {
	auto C = [&](int al, int be) {
		double t = 0.0;
#pragma unroll
		for (int i = 0; i < NSD; ++i) t += inv[i * NSD + al] * inv[i * NSD + be];
		return t;
	};
	if (NSD == 3) { c[0] = C(0, 0); c[1] = C(1, 1); c[2] = C(2, 2); c[3] = C(0, 1); c[4] = C(0, 2); c[5] = C(1, 2); }
	else { c[0] = C(0, 0); c[1] = C(1, 1); c[2] = C(0, 1); c[3] = c[4] = c[5] = 0.0; }
}

// row a of the affine element's gradient form applied to v: sum_k c_k sum_b T_k[a][b] v_b
template <int NSD, int NPE, int KS>
__device__ __forceinline__ double affine_grad_row(const double* kt, const double (&c)[6], int a, const double* v, int vstride) {
	constexpr int NT = NSD == 3 ? 6 : 3;
	double s = 0.0;
#pragma unroll
	for (int k = 0; k < NT; ++k) {
		const double* row = kt + (k * NPE + a) * KS;
		double t = 0.0;
#pragma unroll 9
		for (int b = 0; b < NPE; ++b) t += row[b] * v[b * vstride];
		s += c[k] * t;
	}
	return s;
}

// row a of the reference mass matrix applied to v
template <int NSD, int NPE, int KS>
__device__ __forceinline__ double affine_mass_row(const double* kt, int a, const double* v, int vstride) {
	constexpr int NT = NSD == 3 ? 6 : 3;
	const double* row = kt + (NT * NPE + a) * KS;
	double t = 0.0;
#pragma unroll 9
	for (int b = 0; b < NPE; ++b) t += row[b] * v[b * vstride];
	return t;
}

// the warp-uniform element loop shared by every kernel: EPW elements per warp per trip
#define RSD_ELEMENT_LOOP_BEGIN                                                                   \
	using E = Elem<NSD, P>;                                                                      \
	constexpr int NPE = E::NPE, G = E::G, EPW = E::EPW;                                           \
	extern __shared__ double sm[];                                                               \
	stage_tables<NSD, P>(prm, sm);                                                               \
	const int TS = table_stride(G);                                                              \
	const double* tab = sm;                                                                      \
	const double* wq = sm + prm.nq * TS;                                                         \
	const int lane = threadIdx.x & 31, a = lane % G, slot = lane / G, warp = threadIdx.x >> 5;   \
	double* wbase = sm + prm.nq * TS + prm.nq + (size_t)warp * EPW * (node_area(NPE) + point_area(prm.pts)); \
	double* nodes = wbase + slot * (node_area(NPE) + point_area(prm.pts));                       \
	double* recs = nodes + node_area(NPE);                                                       \
	const int64_t warpId = (int64_t)blockIdx.x * kAsmWarps + warp;                               \
	const int64_t warpStride = (int64_t)gridDim.x * kAsmWarps;                                   \
	constexpr int KS = NPE | 1;                                                                  \
	double* kt = sm + prm.nq * TS + prm.nq + (size_t)kAsmWarps * EPW * (node_area(NPE) + point_area(prm.pts)); \
	if (prm.fast) {                                                                              \
		for (int i = threadIdx.x; i < ktab_count(NSD) * NPE * NPE; i += blockDim.x)              \
			kt[(i / NPE) * KS + i % NPE] = prm.ktab[i];                                          \
		__syncthreads();                                                                         \
	}                                                                                            \
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += warpStride * EPW) {                    \
		const int64_t idx = eb + slot;                                                           \
		const bool inRange = idx < prm.nelem;                                                    \
		const int64_t e = inRange ? (prm.elist ? (int64_t)prm.elist[idx] : idx) : 0;             \
		const bool aff = prm.fast && inRange && (prm.pts == 0 || prm.affine[e]);                \
		const bool has = inRange && a < NPE;                                                     \
		int32_t node = 0, row = -1;                                                              \
		if (has) {                                                                               \
			node = prm.ien[e * NPE + a];                                                         \
			row = prm.t2a[node];                                                                 \
		}                                                                                        \
		const double ke = (prm.kElem && inRange) ? prm.kElem[e] : 1.0;

#define RSD_STAGE_NODE(Uv, Vv, Wv) RSD_STAGE_NODE_R(Uv, Vv, Wv, 0.0)
#define RSD_STAGE_NODE_R(Uv, Vv, Wv, Rv)                                                         \
		if (has) {                                                                               \
			double* nb = nodes + a * NREC;                                                       \
			if (!aff)   /* an affine element's geometry is precomputed */                        \
				_Pragma("unroll") for (int i = 0; i < NSD; ++i) nb[N_X + i] = prm.xyz[(int64_t)node * NSD + i]; \
			nb[N_U] = (Uv); nb[N_V] = (Vv); nb[N_W] = (Wv); nb[N_R] = (Rv);                      \
		}                                                                                        \
		__syncwarp();                                                                            \
		if (!aff && inRange)                                                                     \
			for (int q = a; q < prm.nq; q += G)                                                  \
				eval_point<NSD, P, kGrad>(prm, nd, tab + q * TS, wq[q], nodes, ke, recs + q * REC);     \
		__syncwarp();

#define RSD_ELEMENT_LOOP_END                                                                     \
		__syncwarp();                                                                            \
	}

// ---------------------------------------------------------------------------------------------
// Assembler::assembleMatrix (fem/assembly/backend/cpu/Assembler.tpp:86-140):
// c_diff*Diffusion + c_mass*Mass + c_tdiff*TangentDiffusion + c_tmass*TangentMass, the models at the
// state U (Full gather) and the rate Udot (Free gather; TangentMassForm reads it)
// ---------------------------------------------------------------------------------------------
template <int NSD, int P>
__global__ void __launch_bounds__(kAsmThreads) k_asm_matrix(const AsmParams prm) {
	constexpr bool kGrad = true;
	Needs nd{};
	nd.state = prm.kExpr.n || prm.dkExpr.n || prm.cTDiff != 0.0 || (prm.cpExpr.n && (prm.cMass != 0.0 || prm.cTMass != 0.0));
	nd.rate = prm.cTMass != 0.0 && prm.dcpExpr.n != 0;
	RSD_ELEMENT_LOOP_BEGIN
	const double Ua = (has && nd.state) ? (row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node]) : 0.0;
	const double Ra = (has && nd.rate && row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
	RSD_STAGE_NODE_R(Ua, 0.0, 0.0, Ra)
	double Ke[NPE];
#pragma unroll
	for (int b = 0; b < NPE; ++b) Ke[b] = 0.0;
	if (has && aff) {
		// c_diff k |J| sum_k c_k T_k + c_mass rho cp |J| M, from the reference integrals
		const double* gp = prm.geo + e * 8;
		double c[6];
#pragma unroll
		for (int k = 0; k < 6; ++k) c[k] = gp[k];
		const double cd = prm.cDiff * ke * prm.kConst * gp[6];
		const double cm = prm.cMass * prm.rho * prm.cp * gp[6];
		constexpr int NT = NSD == 3 ? 6 : 3;
#pragma unroll
		for (int b = 0; b < NPE; ++b) {
			double g = 0.0;
#pragma unroll
			for (int k = 0; k < NT; ++k) g += c[k] * kt[(k * NPE + a) * KS + b];
			Ke[b] = cd * g + cm * kt[(NT * NPE + a) * KS + b];
		}
	} else if (has) {
		for (int q = 0; q < prm.nq; ++q) {
			const double* rec = recs + q * REC;
			const double* tq = tab + q * TS;
			const double* ta = tq + a * 4;
			double dx[3], ky[3];
			node_grad<NSD>(rec, ta, dx);
			// DiffusionForm: grad N_a . kS grad N_b = (kS^T grad N_a) . J^-T dN_b/dxi
			shape_apply_t<NSD>(prm, dx, ky);
			double Ga[3];
#pragma unroll
			for (int al = 0; al < NSD; ++al) {
				double s = 0.0;
#pragma unroll
				for (int i = 0; i < NSD; ++i) s += rec[R_INV + i * NSD + al] * ky[i];
				Ga[al] = s;
			}
			const double wm = rec[R_WM];
			const double cd = prm.cDiff * rec[R_K] * wm;
			// MassForm rho cp(T) N_a N_b, TangentMassForm rho dcp/dT T_rate N_a N_b
			double cm = (prm.cMass * prm.rho * rec[R_CP] + prm.cTMass * prm.rho * rec[R_DCP] * rec[R_TR]) * ta[0] * wm;
			if (prm.cTDiff != 0.0)   // TangentDiffusionForm: grad N_a . dk/dT kS grad T N_b
				cm += prm.cTDiff * rec[R_DK] * shape_dot<NSD>(prm, dx, rec + R_GT) * wm;
#pragma unroll
			for (int b = 0; b < NPE; ++b) {
				const double* tb = tq + b * 4;   // one address for the whole warp: broadcast
				double gd = 0.0;
#pragma unroll
				for (int al = 0; al < NSD; ++al) gd += Ga[al] * tb[1 + al];
				Ke[b] += cd * gd + cm * tb[0];
			}
		}
	}
	// scatter row a (free rows only) into the SELL-32 values: entry j of row r sits at
	// sStart[r / 32] + 64 (j / 2) + 2 (r % 32) + j % 2, and the rank map gives j for each element column
	if (prm.ranks) {
		constexpr int RB = (NPE + 7) & ~7;
		if (has && row >= 0) {
			const unsigned long long* rk = reinterpret_cast<const unsigned long long*>(prm.ranks + ((int64_t)e * NPE + a) * RB);
			unsigned long long w[RB / 8];
#pragma unroll
			for (int k = 0; k < RB / 8; ++k) w[k] = __ldcs(rk + k);
			const int32_t sr = prm.sIperm ? prm.sIperm[row] : row;
			double* rowBase = prm.val + prm.sStart[sr >> 5] + 2 * (sr & 31);
#pragma unroll
			for (int b = 0; b < NPE; ++b) {
				const int j = (int)((w[b >> 3] >> (8 * (b & 7))) & 0xFF);
				if (j != 0xFF) atomicAdd(rowBase + 64 * (j >> 1) + (j & 1), Ke[b]);
			}
		}
	} else {
		const int base = lane - a;
#pragma unroll
		for (int b = 0; b < NPE; ++b) {
			const int32_t cb = __shfl_sync(0xffffffffu, row, base + b);
			if (has && row >= 0 && cb >= 0) {
				const int end = prm.rp[row + 1];
				int lo = prm.rp[row], hi = end;
				while (lo < hi) {
					const int mid = (lo + hi) >> 1;
					if (prm.col[mid] < cb) lo = mid + 1; else hi = mid;
				}
				if (lo < end && prm.col[lo] == cb)
					atomicAdd(prm.val + sell_slot(prm.sStart, prm.sUni, prm.sOffs, prm.sIperm, prm.rp, row, lo, cb), Ke[b]);
			}
		}
	}
	RSD_ELEMENT_LOOP_END
}

// element -> column-rank map, built once per pattern: rank[e][a][b] = position of column
// t2a[node_b] within row t2a[node_a] (rows hold at most 254 entries), 0xFF when either DOF is
// constrained
// Assembler::assembleMatrix when every element of the launch is affine, gathered by row: a warp owns
// a SELL-32 slice and lane l its row 32 s + l.  The lane adds row a of every adjacent element (e, a),
// in element order, into its column of a shared-memory image of the slice [entry][lane], which the
// warp then writes out in the pair layout.  Every value is written once: no zero fill, no atomics,
// and the sums are deterministic.
// the 1D factors of the reference integrals of 4- and 8-node elements on the problem's Gauss rule:
// K = int N_i' N_j', M = int N_i N_j, G = int N_i' N_j (the 2D and 3D tables are their products)
struct Q1Fac {
	double K[2][2], M[2][2], G[2][2];
};

constexpr int kRowWarps = 4;
template <int NSD, int P>
__global__ void __launch_bounds__(32 * kRowWarps) k_asm_matrix_rows(const AsmParams prm, const int32_t* __restrict__ adjPtr,
                                                                     const int32_t* __restrict__ adj, int64_t n, int32_t maxLen) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, KS = NPE | 1, NT = NSD == 3 ? 6 : 3, RB = (NPE + 7) & ~7;
	extern __shared__ double sm[];
	double* kt = sm;
	for (int i = threadIdx.x; i < ktab_count(NSD) * NPE * NPE; i += blockDim.x) kt[(i / NPE) * KS + i % NPE] = prm.ktab[i];
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	double* acc = sm + ktab_count(NSD) * NPE * KS + (size_t)warp * maxLen * 32 + lane;   // this lane's column
	const int64_t ns = (n + 31) >> 5;
	for (int64_t s = (int64_t)blockIdx.x * kRowWarps + warp; s < ns; s += (int64_t)gridDim.x * kRowWarps) {
		const int32_t s0 = prm.sStart[s];
		const int len = (prm.sStart[s + 1] - s0) >> 5;
		for (int j = 0; j < len; ++j) acc[j * 32] = 0.0;
		const int64_t srow = 32 * s + lane;
		if (srow < n) {
			const int64_t row = prm.sPerm ? prm.sPerm[srow] : srow;   // the matrix row this lane holds
			// elements in batches of ABATCH: all their loads first, then the sums (in element order)
			constexpr int ABATCH = 4;
			const int32_t q1 = adjPtr[row + 1];
			for (int32_t q0 = adjPtr[row]; q0 < q1; q0 += ABATCH) {
				int32_t ea[ABATCH];
				double gk[ABATCH][8];
				unsigned long long w[ABATCH][RB / 8];
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) ea[k] = q0 + k < q1 ? adj[q0 + k] : -1;
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) {
					if (ea[k] < 0) continue;
					const int32_t e = ea[k] / NPE;
					const double2* gp = reinterpret_cast<const double2*>(prm.geo + (int64_t)e * 8);
#pragma unroll
					for (int i = 0; i < 4; ++i) { const double2 v = gp[i]; gk[k][2 * i] = v.x; gk[k][2 * i + 1] = v.y; }
					gk[k][7] = prm.kElem ? prm.kElem[e] : 1.0;   // slot 7 of the record is spare
					const unsigned long long* rk = reinterpret_cast<const unsigned long long*>(prm.ranks + (int64_t)ea[k] * RB);
#pragma unroll
					for (int i = 0; i < RB / 8; ++i) w[k][i] = __ldcs(rk + i);
				}
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) {
					if (ea[k] < 0) continue;
					const int32_t a = ea[k] - (ea[k] / NPE) * NPE;
					const double cd = prm.cDiff * gk[k][7] * prm.kConst * gk[k][6];
					const double cm = prm.cMass * prm.rho * prm.cp * gk[k][6];
#pragma unroll
					for (int b = 0; b < NPE; ++b) {
						const int j = (int)((w[k][b >> 3] >> (8 * (b & 7))) & 0xFF);
						if (j != 0xFF) {
							double g = 0.0;
#pragma unroll
							for (int t = 0; t < NT; ++t) g += gk[k][t] * kt[(t * NPE + a) * KS + b];
							acc[j * 32] += cd * g + cm * kt[(NT * NPE + a) * KS + b];
						}
					}
				}
			}
		}
		// pair jp of lane l sits at s0 + 64 jp + 2 l; a lane reads only its own column of the image
		double2* out = reinterpret_cast<double2*>(prm.val + s0) + lane;
		for (int jp = 0; jp < (len >> 1); ++jp) out[32 * jp] = make_double2(acc[(2 * jp) * 32], acc[(2 * jp + 1) * 32]);
		if (prm.val32) {   // the mixed solver's copy, rounded as the conversion kernel rounds
			float2* out32 = reinterpret_cast<float2*>(prm.val32 + s0) + lane;
			for (int jp = 0; jp < (len >> 1); ++jp)
				out32[32 * jp] = make_float2((float)acc[(2 * jp) * 32], (float)acc[(2 * jp + 1) * 32]);
		}
	}
}

// The same row gather for 4- and 8-node elements with the reference integrals formed in registers
// from their 1D factors: on the tensor-product rule the reference-element integral of
// dN_a/dxi_s dN_b/dxi_t (symmetrised for s != t) and of N_a N_b is a product over the directions of
// the 1D integrals K = int N_i' N_j', M = int N_i N_j and G = int N_i' N_j with i, j the nodes' 1D
// indices (bit d of the local node number).  The table kernel above reads 7 shared-memory entries
// per (row, element, column) and was bound by the shared-memory pipe; here the element's row is formed
// with the last direction factored out (about 14 FP64 operations per entry, no memory), and every row
// sums its elements in element order.  Compiled for 4 resident 128-thread blocks (128 registers):
// 0.408 ms per 128^3 assembly against 0.420 ms for the unfactored products at the compiler's choice.
template <int NSD>
__global__ void __launch_bounds__(32 * kRowWarps, 4) k_asm_matrix_rows_q1(const AsmParams prm, const Q1Fac f,
                                                                        const int32_t* __restrict__ adjPtr,
                                                                        const int32_t* __restrict__ adj, int64_t n, int32_t maxLen) {
	constexpr int NPE = NSD == 3 ? 8 : 4, RB = 8;
	extern __shared__ double sm[];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	double* acc = sm + (size_t)warp * maxLen * 32 + lane;   // this lane's column of the slice image
	const int64_t ns = (n + 31) >> 5;
	for (int64_t s = (int64_t)blockIdx.x * kRowWarps + warp; s < ns; s += (int64_t)gridDim.x * kRowWarps) {
		const int32_t s0 = prm.sStart[s];
		const int len = (prm.sStart[s + 1] - s0) >> 5;
		for (int j = 0; j < len; ++j) acc[j * 32] = 0.0;
		const int64_t srow = 32 * s + lane;
		if (srow < n) {
			const int64_t row = prm.sPerm ? prm.sPerm[srow] : srow;   // the matrix row this lane holds
			constexpr int ABATCH = 2;
			const int32_t q1 = adjPtr[row + 1];
			for (int32_t q0 = adjPtr[row]; q0 < q1; q0 += ABATCH) {
				int32_t ea[ABATCH];
				double gk[ABATCH][8];
				unsigned long long w[ABATCH];
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) ea[k] = q0 + k < q1 ? adj[q0 + k] : -1;
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) {
					if (ea[k] < 0) continue;
					const int32_t e = ea[k] / NPE;
					// the 64-byte geometry record (64-byte aligned) in two 32-byte loads
					const double* gp = prm.geo + (int64_t)e * 8;
					ld_nc_v4(gp, gk[k][0], gk[k][1], gk[k][2], gk[k][3]);
					ld_nc_v4(gp + 4, gk[k][4], gk[k][5], gk[k][6], gk[k][7]);
					gk[k][7] = prm.kElem ? prm.kElem[e] : 1.0;
					w[k] = __ldcs(reinterpret_cast<const unsigned long long*>(prm.ranks + (int64_t)ea[k] * RB));
				}
#pragma unroll
				for (int k = 0; k < ABATCH; ++k) {
					if (ea[k] < 0) continue;
					const int a = ea[k] - (ea[k] / NPE) * NPE;
					const double cd = prm.cDiff * gk[k][7] * prm.kConst * gk[k][6];
					const double cm = prm.cMass * prm.rho * prm.cp * gk[k][6];
					// the 1D factors of this row's node, per direction d and 1D column index c
					double Km[3][2], Mm[3][2], Gr[3][2], Gc[3][2];
#pragma unroll
					for (int d = 0; d < NSD; ++d) {
						const int ia = (a >> d) & 1;
#pragma unroll
						for (int c = 0; c < 2; ++c) {
							Km[d][c] = ia ? f.K[1][c] : f.K[0][c];
							Mm[d][c] = ia ? f.M[1][c] : f.M[0][c];
							Gr[d][c] = ia ? f.G[1][c] : f.G[0][c];   // int N_a' N_b
							Gc[d][c] = ia ? f.G[c][1] : f.G[c][0];   // int N_a N_b'
						}
					}
					// entry (a, b) = cd sum_t C_t S_t(a, b) + cm M(a, b) with S_t and M products of the
					// 1D factors; the last direction is factored out, entry = M_z A + K_z B + (G_z C + G'_z D)
					// with A..D per column pair of the other directions.  The two sums of mirrored products
					// (the cross terms, and G_z C + G'_z D, whose C and D trade places when a and b do) are
					// rounded without contraction, so that entries (a, b) and (b, a) come out equal
					double c[6];
#pragma unroll
					for (int t = 0; t < 6; ++t) c[t] = cd * gk[k][t];
					constexpr int NB = NSD == 3 ? 4 : 2;   // column pairs / columns of the other directions
#pragma unroll
					for (int bl = 0; bl < NB; ++bl) {
						const int b0 = bl & 1, b1 = (bl >> 1) & 1;
						double A, B = 0.0, Cz = 0.0, Dz = 0.0;
						if constexpr (NSD == 3) {
							const double m01 = Mm[0][b0] * Mm[1][b1];
							const double x01 = __dadd_rn(__dmul_rn(Gr[0][b0], Gc[1][b1]), __dmul_rn(Gc[0][b0], Gr[1][b1]));
							A = c[0] * (Km[0][b0] * Mm[1][b1]);
							A += c[1] * (Mm[0][b0] * Km[1][b1]);
							A += c[3] * x01;
							A += cm * m01;
							B = c[2] * m01;
							const double p4 = c[4] * Mm[1][b1], p5 = c[5] * Mm[0][b0];
							Cz = __dadd_rn(__dmul_rn(p4, Gc[0][b0]), __dmul_rn(p5, Gc[1][b1]));   // coefficient of G_z (row)
							Dz = __dadd_rn(__dmul_rn(p4, Gr[0][b0]), __dmul_rn(p5, Gr[1][b1]));   // coefficient of G'_z
						} else {
							A = 0.0;
						}
#pragma unroll
						for (int bz = 0; bz < 2; ++bz) {
							const int b = NSD == 3 ? bl | (bz << 2) : (bl | (bz << 1));
							const int j = (int)((w[k] >> (8 * b)) & 0xFF);
							if (j == 0xFF) continue;
							double v;
							if constexpr (NSD == 3) {
								v = Mm[2][bz] * A;
								v += Km[2][bz] * B;
								v += __dadd_rn(__dmul_rn(Gr[2][bz], Cz), __dmul_rn(Gc[2][bz], Dz));
							} else {
								// 2D: entry = cd (C0 K_x M_y + C1 M_x K_y + C2 (G_x G'_y + G'_x G_y)) + cm M_x M_y
								const int bx = bl;
								const double mm = Mm[0][bx] * Mm[1][bz];
								const double x01 = __dadd_rn(__dmul_rn(Gr[0][bx], Gc[1][bz]), __dmul_rn(Gc[0][bx], Gr[1][bz]));
								v = c[0] * (Km[0][bx] * Mm[1][bz]);
								v += c[1] * (Mm[0][bx] * Km[1][bz]);
								v += c[2] * x01;
								v += cm * mm;
							}
							acc[j * 32] += v;
						}
					}
				}
			}
		}
		double2* out = reinterpret_cast<double2*>(prm.val + s0) + lane;
		for (int jp = 0; jp < (len >> 1); ++jp) out[32 * jp] = make_double2(acc[(2 * jp) * 32], acc[(2 * jp + 1) * 32]);
		if (prm.val32) {
			float2* out32 = reinterpret_cast<float2*>(prm.val32 + s0) + lane;
			for (int jp = 0; jp < (len >> 1); ++jp)
				out32[32 * jp] = make_float2((float)acc[(2 * jp) * 32], (float)acc[(2 * jp + 1) * 32]);
		}
	}
}

template <int NSD, int P>
__global__ void k_build_slots(int64_t nelem, const int32_t* __restrict__ ien, const int32_t* __restrict__ t2a,
                              const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                              const int32_t* __restrict__ sStart, const int32_t* __restrict__ sUni,
                              const int32_t* __restrict__ sOffs, const int32_t* __restrict__ iperm,
                              uint8_t* __restrict__ ranks, int32_t stride) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE;
	const int64_t total = nelem * NPE;
	for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
		const int64_t e = t / NPE;
		const int a = (int)(t % NPE);
		const int32_t row = t2a[ien[e * NPE + a]];
		uint8_t* out = ranks + t * stride;
		for (int b = 0; b < NPE; ++b) {
			const int32_t cb = t2a[ien[e * NPE + b]];
			int32_t s = 0xFF;
			if (row >= 0 && cb >= 0) {
				const int end = rp[row + 1];
				int lo = rp[row], hi = end;
				while (lo < hi) {
					const int mid = (lo + hi) >> 1;
					if (col[mid] < cb) lo = mid + 1; else hi = mid;
				}
				if (lo < end && col[lo] == cb) s = sell_rank(sStart, sUni, sOffs, iperm, rp, row, lo, cb);
			}
			out[b] = (uint8_t)s;
		}
		for (int b = NPE; b < stride; ++b) out[b] = 0xFF;
	}
}

// ---------------------------------------------------------------------------------------------
// Assembler::assembleVector (Assembler.tpp:199-255), BoundaryApplicator::applyEssentialBCs
// (fem/boundary/backend/cpu/BoundaryApplicator.tpp:7-64) and the adjoint element gradient:
// sum_b (dN_a/dx . dN_b/dx) V_b = dN_a/dx . grad V and sum_b N_a N_b V_b = N_a V(x_q), with V and
// grad V evaluated once per point in phase 2.
// ---------------------------------------------------------------------------------------------
template <int NSD, int P, int W>
__global__ void __launch_bounds__(kAsmThreads) k_asm_vector(const AsmParams prm) {
	constexpr int which = W;
	// the diffusion-type terms need gradients; load and mass terms only the measure
	constexpr bool kGrad = W == 1 || W == 4 || W == 5 || W == 6 || W == 8 || W == 9 || W == 10;
	Needs nd{};
	nd.load = which == 0 || which == 7 || which == 9;
	nd.field = which != 0;
	nd.field2 = which == 8;
	// k(T): diffusion of U takes T from U itself (staged as V, mirrored into U), the operator from the state;
	// cp(T): every mass term takes T from the state (the mass right-hand side's state is U_prev itself)
	constexpr bool kMass = W == 2 || W == 3 || W == 4 || W == 7 || W == 8 || W == 10;
	nd.state = (prm.kExpr.n != 0 && (which == 1 || which == 4 || which == 8 || which == 9)) || which == 6 || which == 10 ||
	           (kMass && prm.cpExpr.n != 0);
	nd.rate = W == 10 && prm.cTMass != 0.0 && prm.dcpExpr.n != 0;
	if (prm.skip && *(volatile const int32_t*)prm.skip) return;   // uniform over the launch
	RSD_ELEMENT_LOOP_BEGIN
	double Va = 0.0, Wa = 0.0, Ua = 0.0;
	if (has) {
		const double fullU = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node];
		switch (which) {
			case 1: case 2: case 8: case 9: Va = fullU; break;                          // GatherMode::Full
			case 3: Va = (row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0; break;           // Free
			case 4: case 10: Va = (row >= 0 && prm.V) ? prm.V[row] : 0.0; break;        // Free
			case 5: Va = row >= 0 ? 0.0 : prm.g[node]; break;                           // Constrained
			case 6: Va = (row >= 0 && prm.V) ? prm.V[row] : 0.0; break;                 // lambda (Free)
			case 7: Va = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : (prm.gPrev ? prm.gPrev[node] : prm.g[node]); break;
			default: break;
		}
		if (which == 8) Wa = (row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
		Ua = (which == 3 || which == 4 || which == 6 || which == 10) ? fullU : Va;
	}
	const double Ra = (has && nd.rate && row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
	RSD_STAGE_NODE_R(Ua, Va, Wa, Ra)
	double Fa = 0.0, ge = 0.0;
	if (has && aff) {
		// reference integrals (no load term and no state here: the host enables this path only then;
		// without state the conductivity model is evaluated at T = 0, as on the quadrature path)
		const double* gp = prm.geo + e * 8;
		const double detJ = gp[6];
		double kdV = 0.0;
		if constexpr (kGrad) {
			double c[6];
#pragma unroll
			for (int k = 0; k < 6; ++k) c[k] = gp[k];
			const double k0 = prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, 0.0) : prm.kConst;
			kdV = ke * k0 * detJ * affine_grad_row<NSD, NPE, KS>(kt, c, a, nodes + N_V, NREC);
		}
		const double massV = prm.rho * prm.cp * detJ * affine_mass_row<NSD, NPE, KS>(kt, a, nodes + N_V, NREC);
		switch (which) {
			case 1: Fa = kdV; break;
			case 2: case 3: Fa = massV; break;
			case 4: Fa = kdV + prm.coef * massV; break;
			case 5: Fa = prm.cDiff * kdV + prm.cMass * massV; break;
			case 7: Fa = prm.coef * massV; break;
			case 8: Fa = kdV + prm.rho * prm.cp * detJ * affine_mass_row<NSD, NPE, KS>(kt, a, nodes + N_W, NREC); break;
			case 9: Fa = -kdV; break;
			default: break;
		}
	} else if (has) {
		for (int q = 0; q < prm.nq; ++q) {
			const double* rec = recs + q * REC;
			const double* ta = tab + q * TS + a * 4;
			const double wm = rec[R_WM];
			const double Na = ta[0];
			if (which == 6) {
				// adjoint: grad lambda . kS grad T with unit conductivity, summed once per point
				if (a == 0) ge += shape_dot<NSD>(prm, rec + R_GV, rec + R_GT) * wm;
				continue;
			}
			if (nd.load) Fa += (rec[R_F] * Na) * wm;
			if (which == 0) continue;
			double kd = 0.0, tg = 0.0;
			if constexpr (kGrad) {
				double dx[3];
				node_grad<NSD>(rec, ta, dx);
				kd = rec[R_K] * shape_dot<NSD>(prm, dx, rec + R_GV);      // per-element factor included
				if (which == 10)                           // TangentDiffusionForm: grad N_a . dk/dT kS grad T
					tg = rec[R_DK] * shape_dot<NSD>(prm, dx, rec + R_GT);
			}
			const double mass = prm.rho * rec[R_CP] * Na * rec[R_V];
			switch (which) {
				case 1: Fa += kd * wm; break;
				case 2: case 3: Fa += mass * wm; break;
				case 4: Fa += (kd + prm.coef * mass) * wm; break;
				case 10:   // + c_tdiff TangentDiffusionForm + c_tmass TangentMassForm (rho dcp/dT T_rate N_a V)
					Fa += (kd + prm.cTDiff * tg * rec[R_V] + prm.coef * mass + prm.cTMass * prm.rho * rec[R_DCP] * rec[R_TR] * Na * rec[R_V]) * wm;
					break;
				case 5: Fa += (prm.cDiff * kd + prm.cMass * mass) * wm; break;
				case 7: Fa += prm.coef * mass * wm; break;
				case 8: Fa += (kd + prm.rho * rec[R_CP] * Na * rec[R_W]) * wm; break;
				case 9: Fa -= kd * wm; break;
				default: break;
			}
		}
	}
	if (which == 6) {
		if (a == 0 && inRange) prm.out[e] = ge;
	} else if (has && row >= 0) {
		atomicAdd(prm.out + row, prm.outScale * Fa);
	}
	RSD_ELEMENT_LOOP_END
}

// The vector modes of k_asm_vector for problems whose elements are all affine, with one thread per
// element (4- and 8-node elements): a warp keeps 32 elements' gathers in flight instead of 32 / G,
// and the reference integrals (staged in shared memory, rows of npe) are read by all lanes at once.
// Each element's rows are formed as in the group kernel's affine branch, in the same order.
// Applying a reference integral of an 8-node element to the element vector as a Kronecker product
// of 1D factors, one direction at a time: out[a] = sum_b A[a_d][b_d] in[b] over the node pairs
// that differ only in bit d (16 multiply-adds instead of 64)
template <int AX>
__device__ __forceinline__ void kron_stage(const double (&A)[2][2], const double (&in)[8], double (&out)[8]) {
	constexpr int S = 1 << AX;
#pragma unroll
	for (int a = 0; a < 8; ++a) {
		const int i = (a >> AX) & 1, b0 = a & ~S;
		out[a] = A[i][0] * in[b0] + A[i][1] * in[b0 | S];
	}
}
// (Ax (x) Ay) applied in x and y to a vector already contracted in z
__device__ __forceinline__ void kron_xy(const double (&Ax)[2][2], const double (&Ay)[2][2], const double (&in)[8],
                                        double (&out)[8]) {
	double t[8];
	kron_stage<1>(Ay, in, t);
	kron_stage<0>(Ax, t, out);
}

template <int NSD, int P, int W>
__global__ void __launch_bounds__(256) k_asm_vector_elem(const AsmParams prm, const Q1Fac fac) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, NT = NSD == 3 ? 6 : 3;
	constexpr bool kGrad = W == 1 || W == 4 || W == 5 || W == 8 || W == 9;
	static_assert(NPE == 4 || NPE == 8, "one thread per element for 4- and 8-node elements");
	if (prm.skip && *(volatile const int32_t*)prm.skip) return;   // uniform over the launch
	// 8-node elements apply the reference integrals as Kronecker products of the 1D factors (no table
	// reads: the table products were bound by the shared-memory pipe); 4-node ones read the tables
	extern __shared__ double kt[];
	if constexpr (NSD == 2) {
		for (int i = threadIdx.x; i < (NT + 1) * NPE * NPE; i += blockDim.x) kt[i] = prm.ktab[i];
		__syncthreads();
	}
	double GT[2][2];
#pragma unroll
	for (int i = 0; i < 2; ++i)
#pragma unroll
		for (int j = 0; j < 2; ++j) GT[i][j] = fac.G[j][i];
	const double k0 = kGrad ? (prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, 0.0) : prm.kConst) : 0.0;
	for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < prm.nelem; idx += (int64_t)gridDim.x * blockDim.x) {
		const int64_t e = prm.elist ? (int64_t)prm.elist[idx] : idx;
		double gk[8];
		ld_nc_v4(prm.geo + e * 8, gk[0], gk[1], gk[2], gk[3]);   // the 64-byte record in two 32-byte loads
		ld_nc_v4(prm.geo + e * 8 + 4, gk[4], gk[5], gk[6], gk[7]);
		const double ke = prm.kElem ? prm.kElem[e] : 1.0;
		int32_t rows[NPE];
		double V[NPE], Wv[NPE];
#pragma unroll
		for (int a = 0; a < NPE; ++a) {
			const int32_t node = prm.ien[e * NPE + a];
			const int32_t row = prm.t2a[node];
			rows[a] = row;
			double Va = 0.0;
			switch (W) {
				case 1: case 2: case 8: case 9: Va = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node]; break;
				case 3: Va = (row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0; break;
				case 4: Va = (row >= 0 && prm.V) ? prm.V[row] : 0.0; break;
				case 5: Va = row >= 0 ? 0.0 : prm.g[node]; break;
				case 7: Va = row >= 0 ? (prm.U ? prm.U[row] : 0.0) : (prm.gPrev ? prm.gPrev[node] : prm.g[node]); break;
				default: break;
			}
			V[a] = Va;
			Wv[a] = (W == 8 && row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
		}
		const double detJ = gk[6];
		if constexpr (NSD == 3) {
			// the element vector's diffusion and mass products, all rows at once
			double kd[8], mv[8], mw[8];
			{
				double zM[8];
				kron_stage<2>(fac.M, V, zM);
				kron_xy(fac.M, fac.M, zM, mv);
				if constexpr (W == 8) {
					double wz[8];
					kron_stage<2>(fac.M, Wv, wz);
					kron_xy(fac.M, fac.M, wz, mw);
				}
				if constexpr (kGrad) {
					double zK[8], zG[8], zGT[8], t[8], u[8];
					kron_stage<2>(fac.K, V, zK);
					kron_stage<2>(fac.G, V, zG);
					kron_stage<2>(GT, V, zGT);
					const double c = ke * k0 * detJ;
					// g = C00 S00 V + C11 S11 V + C22 S22 V + C01 S01 V + C02 S02 V + C12 S12 V
					kron_xy(fac.K, fac.M, zM, t);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] = gk[0] * t[a];
					kron_xy(fac.M, fac.K, zM, t);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] += gk[1] * t[a];
					kron_xy(fac.M, fac.M, zK, t);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] += gk[2] * t[a];
					kron_xy(fac.G, GT, zM, t);
					kron_xy(GT, fac.G, zM, u);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] += gk[3] * (t[a] + u[a]);
					kron_xy(fac.G, fac.M, zGT, t);
					kron_xy(GT, fac.M, zG, u);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] += gk[4] * (t[a] + u[a]);
					kron_xy(fac.M, fac.G, zGT, t);
					kron_xy(fac.M, GT, zG, u);
#pragma unroll
					for (int a = 0; a < 8; ++a) kd[a] = c * (kd[a] + gk[5] * (t[a] + u[a]));
				}
			}
#pragma unroll
			for (int a = 0; a < NPE; ++a) {
				const double kdV = kGrad ? kd[a] : 0.0;
				const double massV = prm.rho * prm.cp * detJ * mv[a];
				double Fa = 0.0;
				switch (W) {
					case 1: Fa = kdV; break;
					case 2: case 3: Fa = massV; break;
					case 4: Fa = kdV + prm.coef * massV; break;
					case 5: Fa = prm.cDiff * kdV + prm.cMass * massV; break;
					case 7: Fa = prm.coef * massV; break;
					case 8: Fa = kdV + prm.rho * prm.cp * detJ * mw[a]; break;
					case 9: Fa = -kdV; break;
					default: break;
				}
				if (rows[a] >= 0) atomicAdd(prm.out + rows[a], prm.outScale * Fa);
			}
			continue;
		}
#pragma unroll
		for (int a = 0; a < NPE; ++a) {
			double kdV = 0.0;
			if constexpr (kGrad) {
				double g = 0.0;
#pragma unroll
				for (int k = 0; k < NT; ++k) {
					const double* row = kt + (k * NPE + a) * NPE;
					double t = 0.0;
#pragma unroll
					for (int b = 0; b < NPE; ++b) t += row[b] * V[b];
					g += gk[k] * t;
				}
				kdV = ke * k0 * detJ * g;
			}
			const double* mrow = kt + (NT * NPE + a) * NPE;
			double mv = 0.0, mw = 0.0;
#pragma unroll
			for (int b = 0; b < NPE; ++b) {
				mv += mrow[b] * V[b];
				if (W == 8) mw += mrow[b] * Wv[b];
			}
			const double massV = prm.rho * prm.cp * detJ * mv;
			double Fa = 0.0;
			switch (W) {
				case 1: Fa = kdV; break;
				case 2: case 3: Fa = massV; break;
				case 4: Fa = kdV + prm.coef * massV; break;
				case 5: Fa = prm.cDiff * kdV + prm.cMass * massV; break;
				case 7: Fa = prm.coef * massV; break;
				case 8: Fa = kdV + prm.rho * prm.cp * detJ * mw; break;
				case 9: Fa = -kdV; break;
				default: break;
			}
			if (rows[a] >= 0) atomicAdd(prm.out + rows[a], prm.outScale * Fa);
		}
	}
}

// 1D Lagrange values and derivatives at the Gauss points, [q][j] = N_j(xi_q), N_j'(xi_q), and the
// Gauss weights: the factors of the tensor-product shape functions and quadrature
struct Tab1D {
	double B[4][4], D[4][4], w[4];
};

// The operator product (which 4: Diffusion + coef*Mass on the operand, gathered Free) of an all-affine
// mesh of tensor-product elements with P+1 Gauss points per direction, by sum factorization.  A
// group of G lanes holds one element, lane a on node a = ix + N1 iy + N1^2 iz, which is also
// quadrature point (ix, iy, iz).  Reference gradients and values at the points come from 1D
// contractions along x, y, z (the values of the other lanes along one axis by shuffle); the flux
// w |J| k C grad (C = J^-1 J^-T from the element's coefficients, the same integrals as the tables of
// the affine path, evaluated by the same Gauss rule) and the mass term go back by the transposed
// contractions.  Per element that is 2 x (1 + 2 + 3) contractions of N1 shuffles in 3D instead of
// NPE^2 table entries per form.
template <int NSD, int P>
__global__ void __launch_bounds__(256) k_apply_sumfac(const AsmParams prm, const Tab1D tab) {
	using E = Elem<NSD, P>;
	constexpr int N1 = P + 1, NPE = E::NPE, G = E::G, EPW = 32 / G;
	static_assert(NPE <= 32, "one element per group of at most 32 lanes");
	if (prm.skip && *(volatile const int32_t*)prm.skip) return;   // uniform over the launch
	__shared__ Tab1D st;
	if (threadIdx.x == 0) st = tab;
	__syncthreads();
	const int lane = threadIdx.x & 31, a = lane % G, base = lane - a;
	const bool act = a < NPE;
	const int ax = act ? a % N1 : 0, ay = act ? (a / N1) % N1 : 0, az = (act && NSD == 3) ? a / (N1 * N1) : 0;
	// the lane's rows (forward) and columns (backward) of the 1D factors, read from shared memory
	const double* Bx = st.B[ax];
	const double* Dx = st.D[ax];
	const double* By = st.B[ay];
	const double* Dy = st.D[ay];
	const double* Bz = st.B[az];
	const double* Dz = st.D[az];
	auto BT = [&](int q, int i) { return st.B[q][i]; };
	auto DT = [&](int q, int i) { return st.D[q][i]; };
	const double wq = st.w[ax] * st.w[ay] * (NSD == 3 ? st.w[az] : 1.0);
	const double k0 = prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, 0.0) : prm.kConst;
	const double massc = prm.coef * prm.rho * prm.cp;
	// the value of lane (i, j, k) of this group
	auto at = [&](double v, int i, int j, int k) { return __shfl_sync(0xffffffffu, v, base + i + N1 * j + N1 * N1 * k); };
	const int64_t warpId = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int64_t step = (((int64_t)gridDim.x * blockDim.x) >> 5) * EPW;
	auto rowOf = [&](int64_t ee) -> int32_t { return (act && ee < prm.nelem) ? prm.erow[ee * NPE + a] : -1; };
	auto valOf = [&](int32_t r) -> double { return (r >= 0 && prm.V) ? prm.V[r] : 0.0; };
	// loads run ahead of the element being computed: its operand values one element ahead, the rows two
	const int64_t e0 = warpId * EPW + lane / G;
	int32_t rowCur = rowOf(e0), rowNext = rowOf(e0 + step);
	double uCur = valOf(rowCur);
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += step) {
		const int64_t e = eb + lane / G;
		const bool in = e < prm.nelem;
		const int32_t row = rowCur;
		const double u = uCur;
		uCur = valOf(rowNext);
		rowCur = rowNext;
		rowNext = rowOf(e + 2 * step);
		double c[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, detJ = 0.0, ke = 1.0;
		if (in) {
			const double2* gp2 = reinterpret_cast<const double2*>(prm.geo + e * 8);
			const double2 g0 = gp2[0], g1 = gp2[1], g2 = gp2[2], g3 = gp2[3];
			c[0] = g0.x; c[1] = g0.y; c[2] = g1.x; c[3] = g1.y; c[4] = g2.x; c[5] = g2.y; detJ = g3.x;
			if (prm.kElem) ke = prm.kElem[e];
		}
		double F = 0.0;
		if constexpr (NSD == 3) {
			// forward: x, then y, then z
			double xb = 0.0, xd = 0.0;
#pragma unroll
			for (int j = 0; j < N1; ++j) { const double v = at(u, j, ay, az); xb += Bx[j] * v; xd += Dx[j] * v; }
			double ybb = 0.0, ydb = 0.0, ybd = 0.0;
#pragma unroll
			for (int j = 0; j < N1; ++j) {
				const double vb = at(xb, ax, j, az), vd = at(xd, ax, j, az);
				ybb += By[j] * vb; ydb += Dy[j] * vb; ybd += By[j] * vd;
			}
			double val = 0.0, gz = 0.0, gy = 0.0, gx = 0.0;
#pragma unroll
			for (int j = 0; j < N1; ++j) {
				const double vbb = at(ybb, ax, ay, j), vdb = at(ydb, ax, ay, j), vbd = at(ybd, ax, ay, j);
				val += Bz[j] * vbb; gz += Dz[j] * vbb; gy += Bz[j] * vdb; gx += Bz[j] * vbd;
			}
			// the point's flux and mass term (c: C00, C11, C22, C01, C02, C12)
			const double s = ke * k0 * detJ * wq;
			const double fx = s * (c[0] * gx + c[3] * gy + c[4] * gz);
			const double fy = s * (c[3] * gx + c[1] * gy + c[5] * gz);
			const double fz = s * (c[4] * gx + c[5] * gy + c[2] * gz);
			const double m = massc * detJ * wq * val;
			// backward: z, then y, then x (transposed factors)
			double A1 = 0.0, A2 = 0.0, A3 = 0.0;
#pragma unroll
			for (int q = 0; q < N1; ++q) {
				const double vx = at(fx, ax, ay, q), vy = at(fy, ax, ay, q), vz = at(fz, ax, ay, q), vm = at(m, ax, ay, q);
				const double bq = BT(q, az);
				A1 += bq * vx; A2 += bq * vy; A3 += DT(q, az) * vz + bq * vm;
			}
			double C1 = 0.0, C2 = 0.0;
#pragma unroll
			for (int q = 0; q < N1; ++q) {
				const double v1 = at(A1, ax, q, az), v2 = at(A2, ax, q, az), v3 = at(A3, ax, q, az);
				const double bq = BT(q, ay);
				C1 += bq * v1; C2 += DT(q, ay) * v2 + bq * v3;
			}
#pragma unroll
			for (int q = 0; q < N1; ++q) {
				const double v1 = at(C1, q, ay, az), v2 = at(C2, q, ay, az);
				F += DT(q, ax) * v1 + BT(q, ax) * v2;
			}
		} else {
			double xb = 0.0, xd = 0.0;
#pragma unroll
			for (int j = 0; j < N1; ++j) { const double v = at(u, j, ay, 0); xb += Bx[j] * v; xd += Dx[j] * v; }
			double val = 0.0, gy = 0.0, gx = 0.0;
#pragma unroll
			for (int j = 0; j < N1; ++j) {
				const double vb = at(xb, ax, j, 0), vd = at(xd, ax, j, 0);
				val += By[j] * vb; gy += Dy[j] * vb; gx += By[j] * vd;
			}
			// c: C00, C11, C01
			const double s = ke * k0 * detJ * wq;
			const double fx = s * (c[0] * gx + c[2] * gy);
			const double fy = s * (c[2] * gx + c[1] * gy);
			const double m = massc * detJ * wq * val;
			double A1 = 0.0, A2 = 0.0;
#pragma unroll
			for (int q = 0; q < N1; ++q) {
				const double vx = at(fx, ax, q, 0), vy = at(fy, ax, q, 0), vm = at(m, ax, q, 0);
				const double bq = BT(q, ay);
				A1 += bq * vx; A2 += DT(q, ay) * vy + bq * vm;
			}
#pragma unroll
			for (int q = 0; q < N1; ++q) {
				const double v1 = at(A1, q, ay, 0), v2 = at(A2, q, ay, 0);
				F += DT(q, ax) * v1 + BT(q, ax) * v2;
			}
		}
		if (row >= 0) atomicAdd(prm.out + row, prm.outScale * F);
	}
}

// The same product for 27-node hexahedra with three lanes per element: lane k of an element owns its
// nodes, and quadrature points, in the plane z = k.  The x and y contractions stay in the lane's
// registers; only the z contraction crosses lanes, by shuffles among the element's three lanes
// (forward: this plane's partial sums of the other two planes; backward: the other two points'
// contributions to this plane's nodes).  The quadrature points are visited one x-point at a time, so
// a lane keeps the x-contracted lines of its plane, one x-point's temporaries and its nine node sums
// live.  Ten elements per warp; lanes 30 and 31 compute on nothing and write nothing.
__global__ void __launch_bounds__(128, 3) k_apply_hex27_planes(const AsmParams prm, const Tab1D t) {
	constexpr int EPW = 10, NPE = 27;
	if (prm.skip && *(volatile const int32_t*)prm.skip) return;   // uniform over the launch
	const int lane = threadIdx.x & 31, grp = lane / 3, k = lane - 3 * grp;
	const bool act = grp < EPW;
	// planes k+1 and k+2 (mod 3) and their lanes; lanes 30/31 (no element) wrap into the warp harmlessly
	const int k1 = k == 2 ? 0 : k + 1, k2 = k == 0 ? 2 : k - 1;
	const int src1 = (3 * grp + k1) & 31, src2 = (3 * grp + k2) & 31;
	auto sel = [](int i, double a, double b, double c) { return i == 0 ? a : (i == 1 ? b : c); };
	// row k of the 1D tables (point z = k) at nodes k, k+1, k+2, and the point's weight
	const double cB0 = sel(k, t.B[0][0], t.B[1][1], t.B[2][2]);
	const double cB1 = sel(k, t.B[0][1], t.B[1][2], t.B[2][0]);
	const double cB2 = sel(k, t.B[0][2], t.B[1][0], t.B[2][1]);
	const double cD0 = sel(k, t.D[0][0], t.D[1][1], t.D[2][2]);
	const double cD1 = sel(k, t.D[0][1], t.D[1][2], t.D[2][0]);
	const double cD2 = sel(k, t.D[0][2], t.D[1][0], t.D[2][1]);
	const double wk = sel(k, t.w[0], t.w[1], t.w[2]);
	const double k0 = prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, 0.0) : prm.kConst;
	const double massc = prm.coef * prm.rho * prm.cp;
	const int64_t warpId = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int64_t step = (((int64_t)gridDim.x * blockDim.x) >> 5) * EPW;
	// the rows and operand values of this lane's plane (nodes (i, j, k), index i + 3 j) of element ee
	auto load = [&](int64_t ee, int32_t (&rw)[9], double (&uv)[9]) {
		const bool ok = act && ee < prm.nelem;
#pragma unroll
		for (int a = 0; a < 9; ++a) rw[a] = ok ? prm.erow[ee * NPE + 9 * k + a] : -1;
#pragma unroll
		for (int a = 0; a < 9; ++a) uv[a] = (rw[a] >= 0 && prm.V) ? prm.V[rw[a]] : 0.0;
	};
	int32_t rowN[9];
	double uN[9];
	load(warpId * EPW + grp, rowN, uN);
	for (int64_t eb = warpId * EPW; eb < prm.nelem; eb += step) {   // warp-uniform trip count
		const int64_t e = eb + grp;
		const bool in = act && e < prm.nelem;
		int32_t row[9];
		double u[9];
#pragma unroll
		for (int a = 0; a < 9; ++a) { row[a] = rowN[a]; u[a] = uN[a]; }
		load(e + step, rowN, uN);   // the next element's plane, in flight during this one
		double c[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, detJ = 0.0, ke = 1.0;
		if (in) {
			const double2* gp2 = reinterpret_cast<const double2*>(prm.geo + e * 8);
			const double2 g0 = gp2[0], g1 = gp2[1], g2 = gp2[2], g3 = gp2[3];
			c[0] = g0.x; c[1] = g0.y; c[2] = g1.x; c[3] = g1.y; c[4] = g2.x; c[5] = g2.y; detJ = g3.x;
			if (prm.kElem) ke = prm.kElem[e];
		}
		const double sK = ke * k0 * detJ * wk, sM = massc * detJ * wk;
		// x: xb[q][j] = sum_i B[q][i] u(i, j), xd with D
		double xb[3][3], xd[3][3];
#pragma unroll
		for (int q = 0; q < 3; ++q)
#pragma unroll
			for (int j = 0; j < 3; ++j) {
				xb[q][j] = t.B[q][0] * u[3 * j] + t.B[q][1] * u[3 * j + 1] + t.B[q][2] * u[3 * j + 2];
				xd[q][j] = t.D[q][0] * u[3 * j] + t.D[q][1] * u[3 * j + 1] + t.D[q][2] * u[3 * j + 2];
			}
		double F[9];
#pragma unroll
		for (int a = 0; a < 9; ++a) F[a] = 0.0;
#pragma unroll
		for (int q1 = 0; q1 < 3; ++q1) {
			double A1[3], A2[3], A3[3];
#pragma unroll
			for (int q2 = 0; q2 < 3; ++q2) {
				// y: this plane's node values contracted to the point (q1, q2)
				const double bb = t.B[q2][0] * xb[q1][0] + t.B[q2][1] * xb[q1][1] + t.B[q2][2] * xb[q1][2];
				const double db = t.D[q2][0] * xb[q1][0] + t.D[q2][1] * xb[q1][1] + t.D[q2][2] * xb[q1][2];
				const double bd = t.B[q2][0] * xd[q1][0] + t.B[q2][1] * xd[q1][1] + t.B[q2][2] * xd[q1][2];
				// z: the other planes' sums, then value and reference gradient at the point (q1, q2, k)
				const double bb1 = __shfl_sync(0xffffffffu, bb, src1), bb2 = __shfl_sync(0xffffffffu, bb, src2);
				const double db1 = __shfl_sync(0xffffffffu, db, src1), db2 = __shfl_sync(0xffffffffu, db, src2);
				const double bd1 = __shfl_sync(0xffffffffu, bd, src1), bd2 = __shfl_sync(0xffffffffu, bd, src2);
				const double val = cB0 * bb + cB1 * bb1 + cB2 * bb2;
				const double gz = cD0 * bb + cD1 * bb1 + cD2 * bb2;
				const double gy = cB0 * db + cB1 * db1 + cB2 * db2;
				const double gx = cB0 * bd + cB1 * bd1 + cB2 * bd2;
				// the point's flux and mass term (c: C00, C11, C22, C01, C02, C12)
				const double s = sK * t.w[q1] * t.w[q2];
				const double fx = s * (c[0] * gx + c[3] * gy + c[4] * gz);
				const double fy = s * (c[3] * gx + c[1] * gy + c[5] * gz);
				const double fz = s * (c[4] * gx + c[5] * gy + c[2] * gz);
				const double m = sM * t.w[q1] * t.w[q2] * val;
				// back along z: this point's share of its own plane's nodes plus the shares the points
				// of planes k+2 and k+1 computed for this plane (their "+1" and "+2" targets)
				const double o3a = cD1 * fz + cB1 * m, o3b = cD2 * fz + cB2 * m;
				A1[q2] = cB0 * fx + __shfl_sync(0xffffffffu, cB1 * fx, src2) + __shfl_sync(0xffffffffu, cB2 * fx, src1);
				A2[q2] = cB0 * fy + __shfl_sync(0xffffffffu, cB1 * fy, src2) + __shfl_sync(0xffffffffu, cB2 * fy, src1);
				A3[q2] = cD0 * fz + cB0 * m + __shfl_sync(0xffffffffu, o3a, src2) + __shfl_sync(0xffffffffu, o3b, src1);
			}
			// back along y to the nodes j of this x-point, then along x into the node sums
#pragma unroll
			for (int j = 0; j < 3; ++j) {
				const double C1 = t.B[0][j] * A1[0] + t.B[1][j] * A1[1] + t.B[2][j] * A1[2];
				const double C2 = t.D[0][j] * A2[0] + t.D[1][j] * A2[1] + t.D[2][j] * A2[2]
				                + t.B[0][j] * A3[0] + t.B[1][j] * A3[1] + t.B[2][j] * A3[2];
#pragma unroll
				for (int i = 0; i < 3; ++i) F[3 * j + i] += t.D[q1][i] * C1 + t.B[q1][i] * C2;
			}
		}
#pragma unroll
		for (int a = 0; a < 9; ++a)
			if (row[a] >= 0) atomicAdd(prm.out + row[a], prm.outScale * F[a]);
	}
}

// erow[e][a] = t2a[ien[e][a]]
__global__ void k_build_erow(int64_t count, const int32_t* __restrict__ ien, const int32_t* __restrict__ t2a,
                             int32_t* __restrict__ erow) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
		erow[i] = t2a[ien[i]];
}

// Assembler::assembleDiagonal (Assembler.tpp:142-197) for c_diff*Diffusion + c_mass*Mass
// + c_tdiff*TangentDiffusion + c_tmass*TangentMass
template <int NSD, int P>
__global__ void __launch_bounds__(kAsmThreads) k_asm_diag(const AsmParams prm) {
	constexpr bool kGrad = true;
	Needs nd{};
	nd.state = prm.kExpr.n != 0 || prm.cTDiff != 0.0 || (prm.cpExpr.n != 0 && (prm.cMass != 0.0 || prm.cTMass != 0.0));
	nd.rate = prm.cTMass != 0.0 && prm.dcpExpr.n != 0;
	RSD_ELEMENT_LOOP_BEGIN
	const double Ua = (has && nd.state) ? (row >= 0 ? (prm.U ? prm.U[row] : 0.0) : prm.g[node]) : 0.0;
	const double Ra = (has && nd.rate && row >= 0 && prm.Udot) ? prm.Udot[row] : 0.0;
	RSD_STAGE_NODE_R(Ua, 0.0, 0.0, Ra)
	double Da = 0.0;
	if (has) {
		for (int q = 0; q < prm.nq; ++q) {
			const double* rec = recs + q * REC;
			const double* ta = tab + q * TS + a * 4;
			double dx[3];
			node_grad<NSD>(rec, ta, dx);
			const double dd = shape_dot<NSD>(prm, dx, dx);
			double tg = 0.0;
			if (prm.cTDiff != 0.0) tg = rec[R_DK] * shape_dot<NSD>(prm, dx, rec + R_GT);
			const double mc = prm.cMass * prm.rho * rec[R_CP] + prm.cTMass * prm.rho * rec[R_DCP] * rec[R_TR];
			Da += (prm.cDiff * rec[R_K] * dd + mc * ta[0] * ta[0] + prm.cTDiff * tg * ta[0]) * rec[R_WM];
		}
	}
	if (has && row >= 0) atomicAdd(prm.out + row, Da);
	RSD_ELEMENT_LOOP_END
}

// 1D Gauss rule of the boundary quadrature (points and weights, up to 5 points)
struct FaceRule {
	double x[5], w[5];
	int n;
};

__host__ __device__ static inline void lagrange1d(int p, double xi, double* N, double* dN);

// BoundaryApplicator::applyNaturalBCs (fem/boundary/backend/cpu/BoundaryApplicator.tpp:66-140) with
// FluxBoundaryForm (equation/heateq/form/FluxBoundaryForm.hpp:22-34): for every boundary face whose
// tag carries a flux q(t, x), F_a += sum_q sum_i (q_i(t, x_q) N_a(q)) n_i(q) w_q over the face's nodes,
// with the point mapped into the element (LagrangeQuad/Hex::mapFaceToElement), n = cof(J) nRef
// (JacobianTransform::computeBoundaryNormal), w the reference face weight, scattered Free.  One
// thread per face; faces holds (element, face, flux index) triplets.
template <int NSD, int P>
__global__ void __launch_bounds__(128) k_natural(int64_t nfaces, const int32_t* __restrict__ faces,
                                                 const double* __restrict__ xyz, const int32_t* __restrict__ ien,
                                                 const int32_t* __restrict__ t2a, const DevExpr* __restrict__ flux,
                                                 double time, FaceRule rule, double* __restrict__ F) {
	constexpr int N1 = P + 1, NPE = (NSD == 3) ? N1 * N1 * N1 : N1 * N1, NFN = (NSD == 3) ? N1 * N1 : N1;
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= nfaces) return;
	const int64_t e = faces[3 * i];
	const int f = faces[3 * i + 1], fx = faces[3 * i + 2];   // face, index of its flux expressions
	const int axis = f / 2;                       // the reference axis normal to the face
	const double side = (f & 1) ? 1.0 : -1.0;     // its reference coordinate on the face
	const int32_t* en = ien + e * NPE;
	double Fe[NFN];
#pragma unroll
	for (int a = 0; a < NFN; ++a) Fe[a] = 0.0;
	const int nqf = (NSD == 3) ? rule.n * rule.n : rule.n;
	for (int q = 0; q < nqf; ++q) {
		const int qs = q % rule.n, qt = q / rule.n;
		const double s = rule.x[qs], t = NSD == 3 ? rule.x[qt] : 0.0;
		const double w = NSD == 3 ? rule.w[qs] * rule.w[qt] : rule.w[qs];
		// element coordinates of the point: the face axis fixed, (s, t) on the others in order
		double xi[3] = {0.0, 0.0, 0.0};
		xi[axis] = side;
		{
			int k = 0;
#pragma unroll
			for (int d = 0; d < NSD; ++d)
				if (d != axis) xi[d] = (k++ == 0) ? s : t;
		}
		double Nd[3][4], dNd[3][4];
#pragma unroll
		for (int d = 0; d < NSD; ++d) lagrange1d(P, xi[d], Nd[d], dNd[d]);
		// x = sum N_a x_a, J[i][al] = sum dN_a/dxi_al x_a,i (JacobianTransform::mapToPhysical, computeJacobian)
		double x[3] = {0.0, 0.0, 0.0}, J[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
		for (int a = 0; a < NPE; ++a) {
			const int ix = a % N1, iy = (a / N1) % N1, iz = NSD == 3 ? a / (N1 * N1) : 0;
			double Na = Nd[0][ix] * Nd[1][iy], g[3];
			g[0] = dNd[0][ix] * Nd[1][iy];
			g[1] = Nd[0][ix] * dNd[1][iy];
			if (NSD == 3) { g[0] *= Nd[2][iz]; g[1] *= Nd[2][iz]; g[2] = Nd[0][ix] * Nd[1][iy] * dNd[2][iz]; Na *= Nd[2][iz]; }
			const double* xa = xyz + (int64_t)en[a] * NSD;
#pragma unroll
			for (int d = 0; d < NSD; ++d) {
				const double c = xa[d];
				x[d] += Na * c;
#pragma unroll
				for (int al = 0; al < NSD; ++al) J[d * NSD + al] += g[al] * c;
			}
		}
		// n = cof(J) nRef with nRef = side e_axis (JacobianTransform::computeMatrixCofactor)
		double n[3];
		if constexpr (NSD == 2) {
			const double cof[4] = {J[3], -J[2], -J[1], J[0]};
#pragma unroll
			for (int d = 0; d < 2; ++d) n[d] = cof[d * 2 + axis] * side;
		} else {
			const double cof[9] = {J[4] * J[8] - J[5] * J[7], -(J[3] * J[8] - J[5] * J[6]), J[3] * J[7] - J[4] * J[6],
			                       -(J[1] * J[8] - J[2] * J[7]), J[0] * J[8] - J[2] * J[6], -(J[0] * J[7] - J[1] * J[6]),
			                       J[1] * J[5] - J[2] * J[4], -(J[0] * J[5] - J[2] * J[3]), J[0] * J[4] - J[1] * J[3]};
#pragma unroll
			for (int d = 0; d < 3; ++d) n[d] = cof[d * 3 + axis] * side;
		}
		double val[3];
#pragma unroll
		for (int d = 0; d < NSD; ++d)
			val[d] = eval_expr(flux[fx * 3 + d], time, x[0], x[1], NSD == 3 ? x[2] : 0.0, 0.0);
		// the face's nodes: the face axis at its end, the other axes in order
#pragma unroll
		for (int b = 0; b < NFN; ++b) {
			const int u = b % N1, v = b / N1;
			int id[3];
			id[axis] = (f & 1) ? P : 0;
			{
				int k = 0;
#pragma unroll
				for (int d = 0; d < NSD; ++d)
					if (d != axis) id[d] = (k++ == 0) ? u : v;
			}
			double Nb = Nd[0][id[0]] * Nd[1][id[1]];
			if (NSD == 3) Nb *= Nd[2][id[2]];
#pragma unroll
			for (int d = 0; d < NSD; ++d) Fe[b] += (val[d] * Nb) * n[d] * w;
		}
	}
#pragma unroll
	for (int b = 0; b < NFN; ++b) {
		const int u = b % N1, v = b / N1;
		int id[3] = {0, 0, 0};
		id[axis] = (f & 1) ? P : 0;
		{
			int k = 0;
#pragma unroll
			for (int d = 0; d < NSD; ++d)
				if (d != axis) id[d] = (k++ == 0) ? u : v;
		}
		const int a = id[0] + N1 * id[1] + (NSD == 3 ? N1 * N1 * id[2] : 0);
		const int32_t row = t2a[en[a]];
		if (row >= 0) atomicAdd(F + row, Fe[b]);
	}
}

// QuantityEvaluator::evaluateNodalField (fem/quantity/backend/cpu/QuantityEvaluator.tpp:205-257) with
// SimpleAverageRecovery (fem/quantity/recovery/SimpleAverageRecovery.hpp): at every quadrature point of
// every element the field's value is added to each of the element's nodes with weight
// N_a |J| w, and the weights themselves are summed; k_nodal_finish divides.  field 0: HeatFluxField
// (Q = -K grad T, K = k(T) I times the element factor, equation/heateq/evaluator/HeatFluxField.hpp),
// 1: ConductivityField (K[0]).  The temperature is gathered Full (Dirichlet values on constrained
// nodes).  One thread per element.
template <int NSD, int P>
__global__ void __launch_bounds__(128) k_nodal_field(const AsmParams prm, int field, int G, double* __restrict__ acc,
                                                     double* __restrict__ wsum) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE;
	const int NC = field == 0 ? NSD : 1;
	const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (e >= prm.nelem) return;
	const int32_t* en = prm.ien + e * NPE;
	double Ue[NPE];
#pragma unroll
	for (int a = 0; a < NPE; ++a) {
		const int32_t v = en[a], r = prm.t2a[v];
		Ue[a] = r >= 0 ? (prm.U ? prm.U[r] : 0.0) : prm.g[v];
	}
	const double ke = prm.kElem ? prm.kElem[e] : 1.0;
	const double* wq = prm.tables + (size_t)prm.nq * G * 4;
	for (int q = 0; q < prm.nq; ++q) {
		const double* tq = prm.tables + (size_t)q * G * 4;
		double J[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, gxi[3] = {0.0, 0.0, 0.0}, T = 0.0;
		for (int a = 0; a < NPE; ++a) {
			const double* ta = tq + a * 4;
			const double* xa = prm.xyz + (int64_t)en[a] * NSD;
			T += ta[0] * Ue[a];
#pragma unroll
			for (int al = 0; al < NSD; ++al) {
				gxi[al] += ta[1 + al] * Ue[a];
#pragma unroll
				for (int i = 0; i < NSD; ++i) J[i * NSD + al] += ta[1 + al] * xa[i];
			}
		}
		double inv[9];
		const double meas = sqrt(jac_geom<NSD, true>(J, inv));
		const double k = ke * (prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, T) : prm.kConst);
		double val[3];
		if (field == 0) {
			// HeatFluxField: q = -K grad T with K = k kS
			double g[3], kg[3];
#pragma unroll
			for (int i = 0; i < NSD; ++i) {
				double gi = 0.0;
#pragma unroll
				for (int al = 0; al < NSD; ++al) gi += inv[i * NSD + al] * gxi[al];
				g[i] = gi;
			}
			shape_apply<NSD>(prm, g, kg);
#pragma unroll
			for (int i = 0; i < NSD; ++i) val[i] = -(k * kg[i]);
		} else {
			val[0] = prm.aniso ? k * prm.kS[0] : k;   // ConductivityField: K[0]
		}
		for (int a = 0; a < NPE; ++a) {
			const double wa = tq[a * 4] * meas * wq[q];
			const int64_t v = en[a];
			for (int c = 0; c < NC; ++c) atomicAdd(acc + v * NC + c, wa * val[c]);
			atomicAdd(wsum + v, wa);
		}
	}
}

// A face point of element e's face f: element coordinates, shape values and reference gradients at
// the point, the physical point, the Jacobian and the area-scaled outward normal n = cof(J) nRef
// (LagrangeQuad/Hex::mapFaceToElement, JacobianTransform::computeBoundaryNormal), as k_natural forms them.
template <int NSD, int P>
struct FacePoint {
	static constexpr int N1 = P + 1, NPE = (NSD == 3) ? N1 * N1 * N1 : N1 * N1;
	double N[NPE], dN[NPE][3], x[3], J[9], n[3];
	__device__ void eval(const double* __restrict__ xyz, const int32_t* en, int f, double s, double t) {
		const int axis = f / 2;
		const double side = (f & 1) ? 1.0 : -1.0;
		double xi[3] = {0.0, 0.0, 0.0};
		xi[axis] = side;
		{
			int k = 0;
#pragma unroll
			for (int d = 0; d < NSD; ++d)
				if (d != axis) xi[d] = (k++ == 0) ? s : t;
		}
		double Nd[3][4], dNd[3][4];
#pragma unroll
		for (int d = 0; d < NSD; ++d) lagrange1d(P, xi[d], Nd[d], dNd[d]);
#pragma unroll
		for (int i = 0; i < 9; ++i) J[i] = 0.0;
		x[0] = x[1] = x[2] = 0.0;
		for (int a = 0; a < NPE; ++a) {
			const int ix = a % N1, iy = (a / N1) % N1, iz = NSD == 3 ? a / (N1 * N1) : 0;
			double Na = Nd[0][ix] * Nd[1][iy];
			dN[a][0] = dNd[0][ix] * Nd[1][iy];
			dN[a][1] = Nd[0][ix] * dNd[1][iy];
			if (NSD == 3) { dN[a][0] *= Nd[2][iz]; dN[a][1] *= Nd[2][iz]; dN[a][2] = Nd[0][ix] * Nd[1][iy] * dNd[2][iz]; Na *= Nd[2][iz]; }
			N[a] = Na;
			const double* xa = xyz + (int64_t)en[a] * NSD;
#pragma unroll
			for (int d = 0; d < NSD; ++d) {
				x[d] += Na * xa[d];
#pragma unroll
				for (int al = 0; al < NSD; ++al) J[d * NSD + al] += dN[a][al] * xa[d];
			}
		}
		if constexpr (NSD == 2) {
			const double cof[4] = {J[3], -J[2], -J[1], J[0]};
#pragma unroll
			for (int d = 0; d < 2; ++d) n[d] = cof[d * 2 + axis] * side;
			n[2] = 0.0;
		} else {
			const double cof[9] = {J[4] * J[8] - J[5] * J[7], -(J[3] * J[8] - J[5] * J[6]), J[3] * J[7] - J[4] * J[6],
			                       -(J[1] * J[8] - J[2] * J[7]), J[0] * J[8] - J[2] * J[6], -(J[0] * J[7] - J[1] * J[6]),
			                       J[1] * J[5] - J[2] * J[4], -(J[0] * J[5] - J[2] * J[3]), J[0] * J[4] - J[1] * J[3]};
#pragma unroll
			for (int d = 0; d < 3; ++d) n[d] = cof[d * 3 + axis] * side;
		}
	}
};

// HeatFlux monitor, Strong method (BoundaryQuadratureMonitorGroup with HeatFluxIntegrand,
// equation/heateq/quantity/HeatFluxIntegrand.hpp:24-40, QuantityEvaluator.tpp:14-90): per listed face
// (element, face, tag slot) the sum over the face's Gauss points of -(K grad T) . n w, T gathered Full,
// K = k(T) kS times the element factor, and the face's measure sum |n| w; out[2 slot], out[2 slot + 1]
template <int NSD, int P>
__global__ void __launch_bounds__(128) k_flux_strong(const AsmParams prm, int64_t nfaces, const int32_t* __restrict__ faces,
                                                     FaceRule rule, double* __restrict__ out) {
	using FP = FacePoint<NSD, P>;
	constexpr int NPE = FP::NPE;
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= nfaces) return;
	const int64_t e = faces[3 * i];
	const int f = faces[3 * i + 1], slot = faces[3 * i + 2];
	const int32_t* en = prm.ien + e * NPE;
	double Ue[NPE];
	for (int a = 0; a < NPE; ++a) {
		const int32_t v = en[a], r = prm.t2a[v];
		Ue[a] = r >= 0 ? (prm.U ? prm.U[r] : 0.0) : prm.g[v];
	}
	const double ke = prm.kElem ? prm.kElem[e] : 1.0;
	double flux = 0.0, meas = 0.0;
	const int nqf = (NSD == 3) ? rule.n * rule.n : rule.n;
	FP fp;
	for (int q = 0; q < nqf; ++q) {
		const int qs = q % rule.n, qt = q / rule.n;
		const double w = NSD == 3 ? rule.w[qs] * rule.w[qt] : rule.w[qs];
		fp.eval(prm.xyz, en, f, rule.x[qs], NSD == 3 ? rule.x[qt] : 0.0);
		double inv[9];
		jac_geom<NSD, true>(fp.J, inv);
		double T = 0.0, gxi[3] = {0.0, 0.0, 0.0};
		for (int a = 0; a < NPE; ++a) {
			T += fp.N[a] * Ue[a];
#pragma unroll
			for (int al = 0; al < NSD; ++al) gxi[al] += fp.dN[a][al] * Ue[a];
		}
		double g[3], kg[3];
#pragma unroll
		for (int d = 0; d < NSD; ++d) {
			double v = 0.0;
#pragma unroll
			for (int al = 0; al < NSD; ++al) v += inv[d * NSD + al] * gxi[al];
			g[d] = v;
		}
		shape_apply<NSD>(prm, g, kg);
		const double k = ke * (prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, T) : prm.kConst);
		double fl = 0.0, nn = 0.0;
#pragma unroll
		for (int d = 0; d < NSD; ++d) { fl -= (k * kg[d]) * fp.n[d]; nn += fp.n[d] * fp.n[d]; }
		flux += fl * w;
		meas += sqrt(nn) * w;
	}
	atomicAdd(out + 2 * slot, flux);
	atomicAdd(out + 2 * slot + 1, meas);
}

// HeatFlux monitor, Weak method (BoundaryReactionMonitorGroup, QuantityEvaluator.tpp:92-200): per listed
// element the element vector of the source minus Diffusion on U (Full) minus, when transient, rho cp Mass
// on Udot (Free), models at the element's T; then, face by face in order, each face on a requested tag adds
// its Gauss measure to that tag and the entries of its nodes not already claimed by the same tag in this
// element.  ftag[i * nfaces + f] is the tag slot of face f of element elems[i], or -1.
template <int NSD, int P>
__global__ void __launch_bounds__(64) k_flux_weak(const AsmParams prm, int64_t nel, const int32_t* __restrict__ elems,
                                                  const int32_t* __restrict__ ftag, int nfaces, int G, FaceRule rule,
                                                  double* __restrict__ out) {
	using FP = FacePoint<NSD, P>;
	constexpr int N1 = P + 1, NPE = FP::NPE, NFN = (NSD == 3) ? N1 * N1 : N1;
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= nel) return;
	const int64_t e = elems[i];
	const int32_t* en = prm.ien + e * NPE;
	double Ue[NPE], Ud[NPE], Oe[NPE];
	for (int a = 0; a < NPE; ++a) {
		const int32_t v = en[a], r = prm.t2a[v];
		Ue[a] = r >= 0 ? (prm.U ? prm.U[r] : 0.0) : prm.g[v];
		Ud[a] = (r >= 0 && prm.Udot) ? prm.Udot[r] : 0.0;
		Oe[a] = 0.0;
	}
	const double ke = prm.kElem ? prm.kElem[e] : 1.0;
	const double* wq = prm.tables + (size_t)prm.nq * G * 4;
	for (int q = 0; q < prm.nq; ++q) {
		const double* tq = prm.tables + (size_t)q * G * 4;
		double J[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, gxi[3] = {0.0, 0.0, 0.0}, x[3] = {0.0, 0.0, 0.0};
		double T = 0.0, Tr = 0.0;
		for (int a = 0; a < NPE; ++a) {
			const double* ta = tq + a * 4;
			const double* xa = prm.xyz + (int64_t)en[a] * NSD;
			T += ta[0] * Ue[a];
			Tr += ta[0] * Ud[a];
#pragma unroll
			for (int d = 0; d < NSD; ++d) {
				x[d] += ta[0] * xa[d];
#pragma unroll
				for (int al = 0; al < NSD; ++al) J[d * NSD + al] += ta[1 + al] * xa[d];
			}
#pragma unroll
			for (int al = 0; al < NSD; ++al) gxi[al] += ta[1 + al] * Ue[a];
		}
		double inv[9];
		const double wm = sqrt(jac_geom<NSD, true>(J, inv)) * wq[q];
		double g[3], kg[3];
#pragma unroll
		for (int d = 0; d < NSD; ++d) {
			double v = 0.0;
#pragma unroll
			for (int al = 0; al < NSD; ++al) v += inv[d * NSD + al] * gxi[al];
			g[d] = v;
		}
		shape_apply<NSD>(prm, g, kg);
		const double k = ke * (prm.kExpr.n ? eval_expr(prm.kExpr, 0.0, 0.0, 0.0, 0.0, T) : prm.kConst);
		const double fsrc = prm.srcExpr.n ? eval_expr(prm.srcExpr, prm.time, x[0], x[1], NSD == 3 ? x[2] : 0.0, 0.0) : 0.0;
		const double cp = prm.cpExpr.n ? eval_expr(prm.cpExpr, 0.0, 0.0, 0.0, 0.0, T) : prm.cp;
		const double mass = prm.cMass != 0.0 ? prm.rho * cp * Tr : 0.0;   // cMass = 1: the transient term
		for (int a = 0; a < NPE; ++a) {
			const double* ta = tq + a * 4;
			double dN[3];
#pragma unroll
			for (int d = 0; d < NSD; ++d) {
				double v = 0.0;
#pragma unroll
				for (int al = 0; al < NSD; ++al) v += inv[d * NSD + al] * ta[1 + al];
				dN[d] = v;
			}
			double dk = 0.0;
#pragma unroll
			for (int d = 0; d < NSD; ++d) dk += dN[d] * kg[d];
			Oe[a] += (fsrc * ta[0]) * wm - (k * dk) * wm - (mass * ta[0]) * wm;
		}
	}
	int claimed[NPE];
	for (int a = 0; a < NPE; ++a) claimed[a] = -1;
	const int nqf = (NSD == 3) ? rule.n * rule.n : rule.n;
	FP fp;
	for (int f = 0; f < nfaces; ++f) {
		const int slot = ftag[i * nfaces + f];
		if (slot < 0) continue;
		double meas = 0.0;
		for (int q = 0; q < nqf; ++q) {
			const int qs = q % rule.n, qt = q / rule.n;
			const double w = NSD == 3 ? rule.w[qs] * rule.w[qt] : rule.w[qs];
			fp.eval(prm.xyz, en, f, rule.x[qs], NSD == 3 ? rule.x[qt] : 0.0);
			double nn = 0.0;
#pragma unroll
			for (int d = 0; d < NSD; ++d) nn += fp.n[d] * fp.n[d];
			meas += sqrt(nn) * w;
		}
		atomicAdd(out + 2 * slot + 1, meas);
		const int axis = f / 2;
		double r = 0.0;
		for (int b = 0; b < NFN; ++b) {
			const int u = b % N1, v = b / N1;
			int id[3] = {0, 0, 0};
			id[axis] = (f & 1) ? P : 0;
			{
				int k = 0;
#pragma unroll
				for (int d = 0; d < NSD; ++d)
					if (d != axis) id[d] = (k++ == 0) ? u : v;
			}
			const int a = id[0] + N1 * id[1] + (NSD == 3 ? N1 * N1 * id[2] : 0);
			if (claimed[a] != slot) { r += Oe[a]; claimed[a] = slot; }
		}
		atomicAdd(out + 2 * slot, r);
	}
}

__global__ void k_nodal_finish(int64_t nnodes, int nc, const double* __restrict__ wsum, double* __restrict__ acc) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnodes * nc; i += (int64_t)gridDim.x * blockDim.x)
		acc[i] /= wsum[i / nc];
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
// Lagrange1D::eval / evalFirstDerivative (fem/basis/Lagrange1D.tpp:4-51)
__host__ __device__ static inline void lagrange1d(int p, double xi, double* N, double* dN) {
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
int build_tables(rsd_ctx* ctx, rsd_heat* h) {
	const int nsd = h->m->nsd, p = h->m->order, q1 = h->nq1, G = group_width(h->m->npe);
	double gx[5], gw[5];
	gauss_legendre(q1, gx, gw);
	const int nq = nsd == 3 ? q1 * q1 * q1 : q1 * q1;
	if (asm_smem_bytes(h->m->npe, nq, nsd, false, nq) > 227 * 1024) return set_error(RSD_EINVAL, "too many quadrature points for this element");
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
	RSD_CUDA(cudaMemcpyAsync(h->tables, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, ctx->stream));
	// reference integrals of the affine path, by the same quadrature: the gradient products
	// (00, 11, [22,] 01, [02, 12]; off-diagonal pairs symmetrised) and the mass
	const int npe = h->m->npe, nt = ktab_count(nsd) - 1;
	const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
	const int pairs2[3][2] = {{0, 0}, {1, 1}, {0, 1}};
	std::vector<double> kt((size_t)(nt + 1) * npe * npe, 0.0);
	for (int k = 0; k <= nt; ++k)
		for (int a = 0; a < npe; ++a)
			for (int b = 0; b < npe; ++b) {
				double sum = 0.0;
				for (int qq = 0; qq < nq; ++qq) {
					const double w = t[(size_t)nq * G * 4 + qq];
					const double* ta = &t[((size_t)qq * G + a) * 4];
					const double* tb = &t[((size_t)qq * G + b) * 4];
					if (k == nt) { sum += w * ta[0] * tb[0]; continue; }
					const int al = nsd == 3 ? pairs[k][0] : pairs2[k][0], be = nsd == 3 ? pairs[k][1] : pairs2[k][1];
					sum += w * ta[1 + al] * tb[1 + be];
					if (al != be) sum += w * ta[1 + be] * tb[1 + al];
				}
				kt[((size_t)k * npe + a) * npe + b] = sum;
			}
	if (h->ktab) cudaFree(h->ktab);
	RSD_CUDA(cudaMalloc(&h->ktab, sizeof(double) * kt.size()));
	RSD_CUDA(cudaMemcpyAsync(h->ktab, kt.data(), sizeof(double) * kt.size(), cudaMemcpyHostToDevice, ctx->stream));
	// uploads go on the context stream (a pageable copy on the legacy stream may still be in flight when
	// it returns, unordered with the non-blocking context stream); the host tables die here
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

// An element is affine when its Jacobian is the same at every quadrature point, to 1e-13 of its
// largest entry (rounding of the node coordinates stays well below that on regular meshes).
template <int NSD, int P>
__global__ void k_affine(int64_t nelem, const int32_t* __restrict__ ien, const double* __restrict__ xyz,
                         const double* __restrict__ tables, int nq, uint8_t* __restrict__ flag, double* __restrict__ geo,
                         unsigned* count) {
	using E = Elem<NSD, P>;
	constexpr int NPE = E::NPE, G = E::G;
	const int64_t total = ((nelem + 31) / 32) * 32;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
		bool ok = false;
		if (e < nelem) {
			auto jac = [&](int q, double (&J)[9]) {
#pragma unroll
				for (int i = 0; i < 9; ++i) J[i] = 0.0;
				for (int b = 0; b < NPE; ++b) {
					const int64_t node = ien[e * NPE + b];
					const double* t = tables + ((size_t)q * G + b) * 4;
#pragma unroll
					for (int i = 0; i < NSD; ++i)
#pragma unroll
						for (int al = 0; al < NSD; ++al) J[i * NSD + al] += t[1 + al] * xyz[node * NSD + i];
				}
			};
			double J0[9], Jq[9];
			jac(0, J0);
			double jmax = 0.0;
#pragma unroll
			for (int i = 0; i < NSD * NSD; ++i) jmax = fmax(jmax, fabs(J0[i]));
			ok = jmax > 0.0;
			for (int q = 1; q < nq && ok; ++q) {
				jac(q, Jq);
#pragma unroll
				for (int i = 0; i < NSD * NSD; ++i) ok = ok && fabs(Jq[i] - J0[i]) <= 1e-13 * jmax;
			}
			flag[e] = ok ? 1 : 0;
			// the element's geometry from its first point, as the quadrature path evaluates it
			double inv[9], c[6];
			const double meas = sqrt(jac_geom<NSD, true>(J0, inv));
			coefs_from_inv<NSD>(inv, c);
			double* gp = geo + e * 8;
#pragma unroll
			for (int k = 0; k < 6; ++k) gp[k] = c[k];
			gp[6] = meas;
			gp[7] = 0.0;
		}
		const unsigned votes = __ballot_sync(0xffffffffu, ok);
		if ((threadIdx.x & 31) == 0 && votes) atomicAdd(count, (unsigned)__popc(votes));
	}
}

// Per-element affine flags (once per problem).  RSD_AFFINE=0 leaves every element on the
// quadrature path.
static int ensure_affine(rsd_ctx* ctx, rsd_heat* h) {
	if (h->affineTried) return RSD_OK;
	h->affineTried = true;
	const char* env = getenv("RSD_AFFINE");
	if (env && env[0] == '0') return RSD_OK;
	if (asm_smem_bytes(h->m->npe, h->nq, h->m->nsd, true, h->nq) > 227 * 1024 || !h->ktab) return RSD_OK;
	const int64_t ne = h->m->nelem;
	RSD_CUDA(cudaMalloc(&h->affine, std::max<int64_t>(ne, 1)));
	RSD_CUDA(cudaMalloc(&h->geo, sizeof(double) * 8 * std::max<int64_t>(ne, 1)));
	unsigned hcnt = 0;
	unsigned* dcnt = nullptr;
	RSD_CUDA(cudaMalloc(&dcnt, sizeof(unsigned)));
	RSD_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(unsigned), ctx->stream));
	const int blocks = (int)std::min<int64_t>((ne + 255) / 256, (int64_t)ctx->num_sms * 8);
	const int nsd = h->m->nsd, ord = h->m->order;
#define RSD_AFF(D, Q) k_affine<D, Q><<<std::max(blocks, 1), 256, 0, ctx->stream>>>(ne, h->m->ien, h->m->xyz, h->tables, h->nq, h->affine, h->geo, dcnt)
	if (nsd == 2 && ord == 1) RSD_AFF(2, 1);
	else if (nsd == 2 && ord == 2) RSD_AFF(2, 2);
	else if (nsd == 2 && ord == 3) RSD_AFF(2, 3);
	else if (nsd == 3 && ord == 1) RSD_AFF(3, 1);
	else RSD_AFF(3, 2);
#undef RSD_AFF
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpyAsync(&hcnt, dcnt, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
	cudaFree(dcnt);
	if (e != cudaSuccess) return cuda_error(e, "affine element flags");
	h->anyAffine = hcnt > 0;
	h->allAffine = (int64_t)hcnt == ne;
	return RSD_OK;
}

// The reference-element integrals hold isotropic gradient products and a constant rho cp: an
// anisotropic conductivity or cp(T) takes the quadrature path
static bool model_blocks_affine(const rsd_heat* h) { return h->aniso || h->cpExpr.n != 0; }

static AsmParams params_for(const rsd_heat* h) {
	AsmParams p{};
	p.nelem = h->m->nelem;
	p.nq = h->nq;
	p.pts = h->nq;
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
	p.cpExpr = h->cpExpr;
	p.dcpExpr = h->dcpExpr;
	p.aniso = h->aniso ? 1 : 0;
	for (int i = 0; i < 9; ++i) p.kS[i] = h->kS[i];
	p.outScale = 1.0;
	return p;
}

static int launch_one(void (*kern)(const AsmParams), dim3 gr, size_t smem, rsd_ctx* ctx, const AsmParams& p) {
	if (p.fast && !(p.affine && p.geo && p.ktab)) return set_error(RSD_EINVAL, "affine assembly path without its tables");
	if (smem > 48 * 1024) RSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	kern<<<gr, kAsmThreads, smem, ctx->stream>>>(p);
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

#define RSD_ASM_DISPATCH(KERNEL)                                                              \
	static int launch_##KERNEL(rsd_ctx* ctx, const rsd_heat* h, const AsmParams& p) {         \
		const int nsd = h->m->nsd, ord = h->m->order, G = group_width(h->m->npe);             \
		const size_t smem = asm_smem_bytes(h->m->npe, h->nq, nsd, p.fast != 0, p.pts);       \
		const int epb = kAsmWarps * (32 / G);                                                 \
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
RSD_ASM_DISPATCH(k_asm_diag)

// the vector kernel is specialised per operand mode, so that each mode compiles only its terms
template <int NSD, int P>
static int launch_vector_mode(rsd_ctx* ctx, dim3 gr, size_t smem, const AsmParams& p) {
	switch (p.which) {
		case 0: return launch_one(k_asm_vector<NSD, P, 0>, gr, smem, ctx, p);
		case 1: return launch_one(k_asm_vector<NSD, P, 1>, gr, smem, ctx, p);
		case 2: return launch_one(k_asm_vector<NSD, P, 2>, gr, smem, ctx, p);
		case 3: return launch_one(k_asm_vector<NSD, P, 3>, gr, smem, ctx, p);
		case 4: return launch_one(k_asm_vector<NSD, P, 4>, gr, smem, ctx, p);
		case 5: return launch_one(k_asm_vector<NSD, P, 5>, gr, smem, ctx, p);
		case 6: return launch_one(k_asm_vector<NSD, P, 6>, gr, smem, ctx, p);
		case 7: return launch_one(k_asm_vector<NSD, P, 7>, gr, smem, ctx, p);
		case 8: return launch_one(k_asm_vector<NSD, P, 8>, gr, smem, ctx, p);
		case 9: return launch_one(k_asm_vector<NSD, P, 9>, gr, smem, ctx, p);
		case 10: return launch_one(k_asm_vector<NSD, P, 10>, gr, smem, ctx, p);
		default: return set_error(RSD_EINVAL, "unknown vector assembly mode");
	}
}

// one thread per element for all-affine problems of 4- and 8-node elements (RSD_ELEM_VEC=0: the
// group kernel)
static Q1Fac q1_factors(const rsd_heat* h);
template <int NSD, int P>
static int launch_vector_elem(rsd_ctx* ctx, const rsd_heat* h, const AsmParams& p) {
	constexpr int NPE = Elem<NSD, P>::NPE, NT = NSD == 3 ? 6 : 3;
	const size_t smem = NSD == 3 ? 0 : sizeof(double) * (NT + 1) * NPE * NPE;
	const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((p.nelem + 255) / 256, (int64_t)ctx->num_sms * 16));
	const Q1Fac fac = q1_factors(h);
	auto go = [&](auto kern) -> int {
		kern<<<blocks, 256, smem, ctx->stream>>>(p, fac);
		RSD_CUDA(cudaGetLastError());
		return RSD_OK;
	};
	switch (p.which) {
		case 1: return go(k_asm_vector_elem<NSD, P, 1>);
		case 2: return go(k_asm_vector_elem<NSD, P, 2>);
		case 3: return go(k_asm_vector_elem<NSD, P, 3>);
		case 4: return go(k_asm_vector_elem<NSD, P, 4>);
		case 5: return go(k_asm_vector_elem<NSD, P, 5>);
		case 7: return go(k_asm_vector_elem<NSD, P, 7>);
		case 8: return go(k_asm_vector_elem<NSD, P, 8>);
		case 9: return go(k_asm_vector_elem<NSD, P, 9>);
		default: return set_error(RSD_EINVAL, "vector mode without a per-element affine kernel");
	}
}

static int launch_k_asm_vector(rsd_ctx* ctx, const rsd_heat* h, const AsmParams& p) {
	const int nsd = h->m->nsd, ord = h->m->order, G = group_width(h->m->npe);
	if (p.fast && p.pts == 0 && ord == 1 && p.which != 0 && p.which != 6 && p.nelem > 0) {
		const char* env = getenv("RSD_ELEM_VEC");
		if (!(env && env[0] == '0')) return nsd == 3 ? launch_vector_elem<3, 1>(ctx, h, p) : launch_vector_elem<2, 1>(ctx, h, p);
	}
	const size_t smem = asm_smem_bytes(h->m->npe, h->nq, nsd, p.fast != 0, p.pts);
	const int epb = kAsmWarps * (32 / G);
	int64_t blocks = (p.nelem + epb - 1) / epb;
	blocks = std::min<int64_t>(blocks, (int64_t)ctx->num_sms * 16);
	dim3 gr((unsigned)std::max<int64_t>(blocks, 1));
	if (nsd == 2 && ord == 1) return launch_vector_mode<2, 1>(ctx, gr, smem, p);
	if (nsd == 2 && ord == 2) return launch_vector_mode<2, 2>(ctx, gr, smem, p);
	if (nsd == 2 && ord == 3) return launch_vector_mode<2, 3>(ctx, gr, smem, p);
	if (nsd == 3 && ord == 1) return launch_vector_mode<3, 1>(ctx, gr, smem, p);
	if (nsd == 3 && ord == 2) return launch_vector_mode<3, 2>(ctx, gr, smem, p);
	return set_error(RSD_EINVAL, "unsupported element");
}

// Build the element -> column-rank map for h's pattern (once).  Skipped, leaving the binary-search
// scatter, when RSD_SLOT_MAP=0, when a row holds more than 254 entries, or when the map would take
// more than a quarter of free memory.
static int ensure_slots(rsd_ctx* ctx, rsd_heat* h) {
	if (h->ranks || h->slotsTried) return RSD_OK;
	h->slotsTried = true;
	const char* env = getenv("RSD_SLOT_MAP");
	if (env && env[0] == '0') return RSD_OK;
	const rsd_csr* K = h->K;
	// the longest row is the longest slice of the SELL-32 layout
	std::vector<int32_t> st(K->nslices + 1);
	RSD_CUDA(cudaMemcpyAsync(st.data(), K->sStart, sizeof(int32_t) * st.size(), cudaMemcpyDeviceToHost, ctx->stream));
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	for (int64_t i = 0; i < K->nslices; ++i) h->maxSlice = std::max<int32_t>(h->maxSlice, (st[i + 1] - st[i]) / 32);
	if (h->maxSlice > 254) return RSD_OK;
	const int npe = h->m->npe;
	const int stride = (npe + 7) & ~7;
	const size_t bytes = (size_t)h->m->nelem * npe * stride;
	size_t freeB = 0, totalB = 0;
	RSD_CUDA(cudaMemGetInfo(&freeB, &totalB));
	if (bytes > freeB / 4) return RSD_OK;
	if (cudaMalloc(&h->ranks, std::max<size_t>(bytes, 8)) != cudaSuccess) { cudaGetLastError(); h->ranks = nullptr; return RSD_OK; }
	const int64_t total = h->m->nelem * npe;
	const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 8);
	const int nsd = h->m->nsd, ord = h->m->order;
#define RSD_SLOTS(D, Q) k_build_slots<D, Q><<<std::max(blocks, 1), 256, 0, ctx->stream>>>(h->m->nelem, h->m->ien, h->t2a, K->rowPtr, K->col, K->sStart, K->sUni, K->sOffs, K->sIperm, h->ranks, stride)
	if (nsd == 2 && ord == 1) RSD_SLOTS(2, 1);
	else if (nsd == 2 && ord == 2) RSD_SLOTS(2, 2);
	else if (nsd == 2 && ord == 3) RSD_SLOTS(2, 3);
	else if (nsd == 3 && ord == 1) RSD_SLOTS(3, 1);
	else RSD_SLOTS(3, 2);
#undef RSD_SLOTS
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

// Row -> (element, local node) adjacency of the free rows (once per problem), for the row-gather
// assembly: built on the host in element order, so that every row sums its elements in that order.
static int ensure_adjacency(rsd_ctx* ctx, rsd_heat* h) {
	if (h->adjTried) return RSD_OK;
	h->adjTried = true;
	const int64_t ne = h->m->nelem, n = h->n;
	const int npe = h->m->npe;
	if (ne * npe >= INT32_MAX) return RSD_OK;
	std::vector<int32_t> ptr(n + 1, 0);
	for (int64_t t = 0; t < ne * npe; ++t) {
		const int32_t r = h->h_t2a[h->m->h_ien[t]];
		if (r >= 0) ++ptr[r + 1];
	}
	for (int64_t i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
	std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1), adj(std::max<int32_t>(ptr[n], 1));
	for (int64_t t = 0; t < ne * npe; ++t) {
		const int32_t r = h->h_t2a[h->m->h_ien[t]];
		if (r >= 0) adj[pos[r]++] = (int32_t)t;
	}
	cudaError_t e;
	if ((e = cudaMalloc(&h->adjPtr, sizeof(int32_t) * (n + 1))) != cudaSuccess ||
	    (e = cudaMalloc(&h->adj, sizeof(int32_t) * adj.size())) != cudaSuccess ||
	    (e = cudaMemcpyAsync(h->adjPtr, ptr.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
	    (e = cudaMemcpyAsync(h->adj, adj.data(), sizeof(int32_t) * adj.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
		cudaGetLastError();
		cudaFree(h->adjPtr); cudaFree(h->adj);
		h->adjPtr = nullptr; h->adj = nullptr;
	}
	return RSD_OK;
}

// the 1D factors of the 4- and 8-node reference integrals on the problem's rule
static Q1Fac q1_factors(const rsd_heat* h) {
	Q1Fac f{};
	double xq[5], wq[5], N[4], dN[4], Nq[5][2], dNq[5][2];
	gauss_legendre(h->nq1, xq, wq);
	for (int q = 0; q < h->nq1; ++q) {
		lagrange1d(1, xq[q], N, dN);
		for (int i = 0; i < 2; ++i) { Nq[q][i] = N[i]; dNq[q][i] = dN[i]; }
	}
	// K and M symmetric to the last bit (one evaluation per pair, mirrored), so that the row-gather
	// kernel's element entries (a, b) and (b, a) come out equal and so does the assembled matrix
	for (int i = 0; i < 2; ++i)
		for (int j = 0; j < 2; ++j) {
			double k = 0.0, m = 0.0, g = 0.0;
			for (int q = 0; q < h->nq1; ++q) {
				k += wq[q] * dNq[q][std::min(i, j)] * dNq[q][std::max(i, j)];
				m += wq[q] * Nq[q][std::min(i, j)] * Nq[q][std::max(i, j)];
				g += wq[q] * dNq[q][i] * Nq[q][j];
			}
			f.K[i][j] = k; f.M[i][j] = m; f.G[i][j] = g;
		}
	return f;
}

// the row-gather kernel for an all-affine launch with the slot map (RSD_ROW_ASM=0: the scatter)
static int launch_matrix_rows(rsd_ctx* ctx, rsd_heat* h, const AsmParams& p, bool* done, bool* symmetric) {
	*done = false;
	*symmetric = false;
	const char* env = getenv("RSD_ROW_ASM");
	if ((env && env[0] == '0') || !p.fast || p.pts != 0 || !p.ranks || h->maxSlice > 64) return RSD_OK;
	RSD_CHECK(ensure_adjacency(ctx, h));
	if (!h->adj) return RSD_OK;
	const int nsd = h->m->nsd, ord = h->m->order, npe = h->m->npe;
	const size_t smem = sizeof(double) * ((size_t)ktab_count(nsd) * npe * ktab_stride(npe) + (size_t)kRowWarps * h->maxSlice * 32);
	const int64_t ns = (h->n + 31) / 32;
	const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((ns + kRowWarps - 1) / kRowWarps, (int64_t)ctx->num_sms * 32));
	auto go = [&](auto kern) -> int {
		if (smem > 48 * 1024) RSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		kern<<<blocks, 32 * kRowWarps, smem, ctx->stream>>>(p, h->adjPtr, h->adj, h->n, h->maxSlice);
		RSD_CUDA(cudaGetLastError());
		*done = true;
		return RSD_OK;
	};
	if (ord == 1) {
		const Q1Fac f = q1_factors(h);
		const size_t smem1 = sizeof(double) * (size_t)kRowWarps * h->maxSlice * 32;
		auto go1 = [&](auto kern) -> int {
			if (smem1 > 48 * 1024) RSD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
			kern<<<blocks, 32 * kRowWarps, smem1, ctx->stream>>>(p, f, h->adjPtr, h->adj, h->n, h->maxSlice);
			RSD_CUDA(cudaGetLastError());
			*done = true;
			return RSD_OK;
		};
		const char* tabEnv = getenv("RSD_ROW_ASM_TABLES");
		if (!(tabEnv && tabEnv[0] == '1')) {
			// entries (a, b) and (b, a) of an element come out equal and every row sums its elements in
			// element order: the assembled values are symmetric to the last bit
			*symmetric = true;
			return nsd == 3 ? go1(k_asm_matrix_rows_q1<3>) : go1(k_asm_matrix_rows_q1<2>);
		}
	}
	if (nsd == 2 && ord == 1) return go(k_asm_matrix_rows<2, 1>);
	if (nsd == 2 && ord == 2) return go(k_asm_matrix_rows<2, 2>);
	if (nsd == 2 && ord == 3) return go(k_asm_matrix_rows<2, 3>);
	if (nsd == 3 && ord == 1) return go(k_asm_matrix_rows<3, 1>);
	if (nsd == 3 && ord == 2) return go(k_asm_matrix_rows<3, 2>);
	return RSD_OK;
}

int assemble_matrix(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double cTDiff, double cTMass,
                    const double* U, const double* Udot, rsd_csr* A) {
	if (A->n != h->n || A->nnz != h->K->nnz) return set_error(RSD_EINVAL, "matrix does not have the problem's pattern");
	RSD_CHECK(ensure_slots(ctx, h));
	AsmParams p = params_for(h);
	p.rp = A->rowPtr; p.col = A->col; p.sStart = A->sStart; p.sUni = A->sUni; p.sOffs = A->sOffs; p.val = A->sVal;
	p.sPerm = A->sPerm; p.sIperm = A->sIperm;
	// the slot map indexes h's pattern; another matrix of equal size may differ, so it searches
	if (A == h->K || A->rowPtr == h->K->rowPtr) p.ranks = h->ranks;
	p.cDiff = cDiff; p.cMass = cMass; p.cTDiff = cTDiff; p.cTMass = cTMass;
	// reference integrals for the affine elements when the coefficients are constant per element
	RSD_CHECK(ensure_affine(ctx, h));
	if (h->anyAffine && h->kExpr.n == 0 && h->dkExpr.n == 0 && cTDiff == 0.0 && cTMass == 0.0 && !model_blocks_affine(h)) {
		p.fast = 1; p.affine = h->affine; p.geo = h->geo; p.ktab = h->ktab; if (h->allAffine) p.pts = 0;
	}
	p.U = U; p.Udot = Udot;
	A->sellValid = true;
	A->csrValid = false;
	A->version++;
	const int pr = prof_begin(ctx, PF_ASM_MATRIX);
	bool rows = false, symmetric = false;
	// a matrix that already has an FP32 copy in the SELL layout gets it written by the row gather too
	if (A->val32 && A->format == 0) p.val32 = A->val32;
	int rc = launch_matrix_rows(ctx, h, p, &rows, &symmetric);
	if (rc == RSD_OK && rows && p.val32) { A->version32 = A->version; A->fmt32 = 0; }
	if (rc == RSD_OK && rows && symmetric) A->symVersion = A->version;
	if (rc == RSD_OK && !rows) {
		RSD_CUDA(cudaMemsetAsync(A->sVal, 0, sizeof(double) * std::max<int64_t>(A->ssize, 1), ctx->stream));
		rc = launch_k_asm_matrix(ctx, h, p);
	}
	prof_end(ctx, pr);
	return rc;
}

// the affine path of the vector kernels: every mode but the adjoint, with no state-dependent
// conductivity and no load term (both are evaluated per quadrature point)
static int affine_vector(rsd_ctx* ctx, rsd_heat* h, AsmParams& p) {
	RSD_CHECK(ensure_affine(ctx, h));
	const int w = p.which;
	const bool load = w == 0 || w == 7 || w == 9;
	const bool state = (h->kExpr.n != 0 && (w == 1 || w == 4 || w == 8 || w == 9)) || w == 10;
	if (h->anyAffine && w != 6 && !state && !(load && h->srcExpr.n != 0) && !model_blocks_affine(h)) {
		p.fast = 1; p.affine = h->affine; p.geo = h->geo; p.ktab = h->ktab; if (h->allAffine) p.pts = 0;
	}
	return RSD_OK;
}

int assemble_vector(rsd_ctx* ctx, rsd_heat* h, int which, double coef, const double* U, const double* Udot,
                    const double* operand, double* out, double outScale, bool accumulate) {
	if (which == 4 && !accumulate && outScale == 1.0) return apply_operator(ctx, h, coef, U, operand, out, nullptr, 4);
	AsmParams p = params_for(h);
	p.which = which; p.coef = coef; p.U = U; p.Udot = Udot; p.V = operand; p.out = out; p.outScale = outScale;
	if (which == 10) p.cTDiff = 1.0;   // the Jacobian's product: TangentDiffusion with coefficient 1
	if (which == 7 && h->gPrevValid) p.gPrev = h->gPrev;
	RSD_CHECK(affine_vector(ctx, h, p));
	if (!accumulate) {
		const int64_t len = which == 6 ? h->m->nelem : h->n;
		RSD_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * std::max<int64_t>(len, 1), ctx->stream));
	}
	const int pr = prof_begin(ctx, PF_ASM_VECTOR);
	const int rc = launch_k_asm_vector(ctx, h, p);
	prof_end(ctx, pr);
	return rc;
}

// FEMOperator::apply (linalg/operator/FEMOperator.hpp:39-43) for the forms Diffusion + coef * Mass:
// out = A(U) V over the free DOFs, the operand gathered Free (zero on constrained nodes) and the state
// U (Full) read only through k(T).  With skip, the element kernel returns at once once *skip != 0.
// Meshes of order 2 and 3 whose elements are all affine, with P+1 Gauss points per direction and at
// most 32 nodes per element, take the sum-factorized kernel (RSD_SUMFAC=0: the table kernels);
// 4- and 8-node elements keep the one-thread-per-element table kernel, which measured faster for them.
int apply_operator(rsd_ctx* ctx, rsd_heat* h, double coef, const double* U, const double* V, double* out,
                   const int32_t* skip, int which, double cTDiff, double cTMass, const double* Udot) {
	AsmParams p = params_for(h);
	p.which = which; p.coef = coef; p.U = U; p.V = V; p.out = out; p.skip = skip;
	if (which == 10) { p.cTDiff = cTDiff; p.cTMass = cTMass; p.Udot = Udot; }
	RSD_CHECK(affine_vector(ctx, h, p));
	RSD_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * std::max<int64_t>(h->n, 1), ctx->stream));
	const int pr = prof_begin(ctx, PF_ASM_VECTOR);
	const int nsd = h->m->nsd, ord = h->m->order;
	const int n1 = ord + 1, nq1 = h->nq1;
	const char* env = getenv("RSD_SUMFAC");
	int rc;
	if (p.fast && p.pts == 0 && nq1 == n1 && ord >= 2 && h->m->npe <= 32 && p.nelem > 0 && !(env && env[0] == '0')) {
		if (!h->erow) {
			// the element -> free-row map, once per problem
			const int64_t cnt = h->m->nelem * h->m->npe;
			int32_t* er = nullptr;
			RSD_CUDA(cudaMalloc(&er, sizeof(int32_t) * std::max<int64_t>(cnt, 1)));
			h->erow = er;
			k_build_erow<<<vec_grid(ctx, cnt), 256, 0, ctx->stream>>>(cnt, h->m->ien, h->t2a, h->erow);
			RSD_CUDA(cudaGetLastError());
		}
		p.erow = h->erow;
		Tab1D t{};
		double xq[5], wq[5], N[4], dN[4];
		gauss_legendre(n1, xq, wq);
		for (int q = 0; q < n1; ++q) {
			lagrange1d(ord, xq[q], N, dN);
			for (int j = 0; j < n1; ++j) { t.B[q][j] = N[j]; t.D[q][j] = dN[j]; }
			t.w[q] = wq[q];
		}
		const int epw = 32 / group_width(h->m->npe);
		const int64_t warpsNeeded = (p.nelem + epw - 1) / epw;
		const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((warpsNeeded + 7) / 8, (int64_t)ctx->num_sms * 8));
		auto go = [&](auto kern) -> int {
			kern<<<blocks, 256, 0, ctx->stream>>>(p, t);
			RSD_CUDA(cudaGetLastError());
			return RSD_OK;
		};
		const char* planes = getenv("RSD_SUMFAC_PLANES");
		if (nsd == 2 && ord == 2) rc = go(k_apply_sumfac<2, 2>);
		else if (nsd == 2 && ord == 3) rc = go(k_apply_sumfac<2, 3>);
		else if (planes && planes[0] == '0') rc = go(k_apply_sumfac<3, 2>);
		else {
			const int64_t wn = (p.nelem + 9) / 10;
			const int b = (int)std::max<int64_t>(1, std::min<int64_t>((wn + 3) / 4, (int64_t)ctx->num_sms * 3));   // resident: 3 per SM
			k_apply_hex27_planes<<<b, 128, 0, ctx->stream>>>(p, t);
			RSD_CUDA(cudaGetLastError());
			rc = RSD_OK;
		}
	} else {
		rc = launch_k_asm_vector(ctx, h, p);
	}
	prof_end(ctx, pr);
	return rc;
}

// the lift visits only elements with a constrained node: every other element adds exact zeros
int assemble_lift(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, double* F) {
	if (h->nbElems == 0) return RSD_OK;
	AsmParams p = params_for(h);
	p.which = 5; p.cDiff = cDiff; p.cMass = cMass; p.out = F; p.outScale = -1.0;
	p.elist = h->bElems; p.nelem = h->nbElems;
	RSD_CHECK(affine_vector(ctx, h, p));
	const int pr = prof_begin(ctx, PF_ASM_VECTOR);
	const int rc = launch_k_asm_vector(ctx, h, p);
	prof_end(ctx, pr);
	return rc;
}

// HeatProblem's flux boundary condition with an expression per spatial component
// (application/heateq/problem/HeatProblem.tpp:98-105): registers or clears tag's flux and rebuilds
// the list of boundary faces that carry one
int set_flux(rsd_ctx* ctx, rsd_heat* h, int tag, const char* const* exprs) {
	const rsd_mesh* m = h->m;
	if (tag < 0) return set_error(RSD_EINVAL, "boundary tags are >= 0");
	size_t slot = h->fluxTags.size();
	for (size_t i = 0; i < h->fluxTags.size(); ++i) if (h->fluxTags[i] == tag) slot = i;
	if (exprs) {
		DevExpr c[3];
		for (int d = 0; d < m->nsd; ++d) {
			if (!exprs[d]) return set_error(RSD_EINVAL, "a flux needs one expression per spatial component");
			RSD_CHECK(compile_expr(exprs[d], &c[d]));
		}
		if (slot == h->fluxTags.size()) { h->fluxTags.push_back(tag); h->fluxExpr.resize(3 * h->fluxTags.size()); }
		for (int d = 0; d < 3; ++d) h->fluxExpr[slot * 3 + d] = d < m->nsd ? c[d] : DevExpr{};
	} else if (slot < h->fluxTags.size()) {
		h->fluxTags.erase(h->fluxTags.begin() + slot);
		h->fluxExpr.erase(h->fluxExpr.begin() + 3 * slot, h->fluxExpr.begin() + 3 * slot + 3);
	}
	std::map<int32_t, int32_t> index;
	for (size_t i = 0; i < h->fluxTags.size(); ++i) index[h->fluxTags[i]] = (int32_t)i;
	std::vector<int32_t> fl;
	for (int64_t e = 0; e < m->nelem; ++e)
		for (int f = 0; f < m->nfaces; ++f) {
			const int32_t t = m->h_rng[e * m->nfaces + f];
			const auto it = t >= 0 ? index.find(t) : index.end();
			if (it != index.end()) { fl.push_back((int32_t)e); fl.push_back(f); fl.push_back(it->second); }
		}
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));   // no launch in flight reads the lists replaced here
	cudaFree(h->nFaces);
	h->nFaces = nullptr;
	cudaFree(h->dFlux);
	h->dFlux = nullptr;
	h->nnFaces = (int64_t)fl.size() / 3;
	if (!h->fluxExpr.empty()) {
		RSD_CUDA(cudaMalloc(&h->dFlux, sizeof(DevExpr) * h->fluxExpr.size()));
		RSD_CUDA(cudaMemcpyAsync(h->dFlux, h->fluxExpr.data(), sizeof(DevExpr) * h->fluxExpr.size(), cudaMemcpyHostToDevice, ctx->stream));
	}
	if (h->nnFaces) {
		RSD_CUDA(cudaMalloc(&h->nFaces, sizeof(int32_t) * fl.size()));
		RSD_CUDA(cudaMemcpyAsync(h->nFaces, fl.data(), sizeof(int32_t) * fl.size(), cudaMemcpyHostToDevice, ctx->stream));
	}
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	return RSD_OK;
}

// HeatProblem::applyNatural (HeatProblem.tpp:234-238) at the problem's current time: F += the flux
// integrals of every registered flux boundary
int apply_natural(rsd_ctx* ctx, rsd_heat* h, double* F) {
	if (h->nnFaces == 0) return RSD_OK;
	FaceRule r{};
	r.n = h->nq1;
	gauss_legendre(r.n, r.x, r.w);
	const int nsd = h->m->nsd, ord = h->m->order;
	const int blocks = (int)((h->nnFaces + 127) / 128);
#define RSD_NAT(D, Q) k_natural<D, Q><<<blocks, 128, 0, ctx->stream>>>(h->nnFaces, h->nFaces, h->m->xyz, h->m->ien, h->t2a, h->dFlux, h->time, r, F)
	if (nsd == 2 && ord == 1) RSD_NAT(2, 1);
	else if (nsd == 2 && ord == 2) RSD_NAT(2, 2);
	else if (nsd == 2 && ord == 3) RSD_NAT(2, 3);
	else if (nsd == 3 && ord == 1) RSD_NAT(3, 1);
	else if (nsd == 3 && ord == 2) RSD_NAT(3, 2);
	else return set_error(RSD_EINVAL, "unsupported element");
#undef RSD_NAT
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

// HeatProblem::computeNodalField (HeatProblem.tpp:293-303) for the heat flux (field 0, nsd components
// per node) or the conductivity (field 1): out has nnodes * components entries; scratch nnodes
int nodal_field(rsd_ctx* ctx, rsd_heat* h, int field, const double* U, double* out, double* scratch) {
	AsmParams p = params_for(h);
	p.U = U;
	const int nsd = h->m->nsd, ord = h->m->order, nc = field == 0 ? nsd : 1, G = group_width(h->m->npe);
	RSD_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * h->m->nnodes * nc, ctx->stream));
	RSD_CUDA(cudaMemsetAsync(scratch, 0, sizeof(double) * h->m->nnodes, ctx->stream));
	const int blocks = (int)std::max<int64_t>(1, (h->m->nelem + 127) / 128);
#define RSD_NF(D, Q) k_nodal_field<D, Q><<<blocks, 128, 0, ctx->stream>>>(p, field, G, out, scratch)
	if (nsd == 2 && ord == 1) RSD_NF(2, 1);
	else if (nsd == 2 && ord == 2) RSD_NF(2, 2);
	else if (nsd == 2 && ord == 3) RSD_NF(2, 3);
	else if (nsd == 3 && ord == 1) RSD_NF(3, 1);
	else if (nsd == 3 && ord == 2) RSD_NF(3, 2);
	else return set_error(RSD_EINVAL, "unsupported element");
#undef RSD_NF
	k_nodal_finish<<<vec_grid(ctx, h->m->nnodes * nc), 256, 0, ctx->stream>>>(h->m->nnodes, nc, scratch, out);
	RSD_CUDA(cudaGetLastError());
	return RSD_OK;
}

// HeatProblem's HeatFlux monitors (HeatProblem.tpp:410-440) at the problem's current time: per requested
// tag, the Strong (boundary quadrature) or Weak (boundary reaction) flux and the tag's measure, into
// out[2 t], out[2 t + 1] (device, zeroed here); transient adds the weak method's mass term on Udot
int boundary_flux(rsd_ctx* ctx, rsd_heat* h, int method, int ntags, const int32_t* tags, const double* U, const double* Udot,
                  bool transient, double* out) {
	const rsd_mesh* m = h->m;
	std::map<int32_t, int32_t> slot;
	for (int t = 0; t < ntags; ++t) {
		if (tags[t] < 0) return set_error(RSD_EINVAL, "boundary tags are >= 0");
		if (slot.count(tags[t])) return set_error(RSD_EINVAL, "a tag is requested twice");
		slot[tags[t]] = t;
	}
	AsmParams p = params_for(h);
	p.U = U;
	p.Udot = Udot;
	p.cMass = transient ? 1.0 : 0.0;
	FaceRule r{};
	r.n = h->nq1;
	gauss_legendre(r.n, r.x, r.w);
	RSD_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 2 * std::max(ntags, 1), ctx->stream));
	const int nsd = m->nsd, ord = m->order, nf = m->nfaces;
	std::vector<int32_t> list, ftag;
	for (int64_t e = 0; e < m->nelem; ++e) {
		bool any = false;
		for (int f = 0; f < nf; ++f) {
			const int32_t t = m->h_rng[e * nf + f];
			const auto it = t >= 0 ? slot.find(t) : slot.end();
			if (it == slot.end()) continue;
			if (method == RSD_FLUX_STRONG) { list.push_back((int32_t)e); list.push_back(f); list.push_back(it->second); }
			any = true;
		}
		if (method == RSD_FLUX_WEAK && any) {
			list.push_back((int32_t)e);
			for (int f = 0; f < nf; ++f) {
				const int32_t t = m->h_rng[e * nf + f];
				const auto it = t >= 0 ? slot.find(t) : slot.end();
				ftag.push_back(it == slot.end() ? -1 : it->second);
			}
		}
	}
	if (list.empty()) return RSD_OK;
	int32_t* dl = nullptr;
	RSD_CUDA(cudaMalloc(&dl, sizeof(int32_t) * (list.size() + ftag.size())));
	auto launch = [&]() -> int {
		RSD_CUDA(cudaMemcpyAsync(dl, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice, ctx->stream));
		if (!ftag.empty())
			RSD_CUDA(cudaMemcpyAsync(dl + list.size(), ftag.data(), sizeof(int32_t) * ftag.size(), cudaMemcpyHostToDevice, ctx->stream));
		if (method == RSD_FLUX_STRONG) {
			const int64_t cnt = (int64_t)list.size() / 3;
			const int blocks = (int)((cnt + 127) / 128);
#define RSD_FS(D, Q) k_flux_strong<D, Q><<<blocks, 128, 0, ctx->stream>>>(p, cnt, dl, r, out)
			if (nsd == 2 && ord == 1) RSD_FS(2, 1);
			else if (nsd == 2 && ord == 2) RSD_FS(2, 2);
			else if (nsd == 2 && ord == 3) RSD_FS(2, 3);
			else if (nsd == 3 && ord == 1) RSD_FS(3, 1);
			else if (nsd == 3 && ord == 2) RSD_FS(3, 2);
			else return set_error(RSD_EINVAL, "unsupported element");
#undef RSD_FS
		} else {
			const int64_t cnt = (int64_t)list.size();
			const int blocks = (int)((cnt + 63) / 64), G = group_width(m->npe);
#define RSD_FW(D, Q) k_flux_weak<D, Q><<<blocks, 64, 0, ctx->stream>>>(p, cnt, dl, dl + list.size(), nf, G, r, out)
			if (nsd == 2 && ord == 1) RSD_FW(2, 1);
			else if (nsd == 2 && ord == 2) RSD_FW(2, 2);
			else if (nsd == 2 && ord == 3) RSD_FW(2, 3);
			else if (nsd == 3 && ord == 1) RSD_FW(3, 1);
			else if (nsd == 3 && ord == 2) RSD_FW(3, 2);
			else return set_error(RSD_EINVAL, "unsupported element");
#undef RSD_FW
		}
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		return RSD_OK;
	};
	const int rc = launch();
	cudaFree(dl);
	return rc;
}

int assemble_diagonal(rsd_ctx* ctx, rsd_heat* h, double cDiff, double cMass, const double* U, double* d, double cTDiff,
                      double cTMass, const double* Udot) {
	AsmParams p = params_for(h);
	p.cDiff = cDiff; p.cMass = cMass; p.cTDiff = cTDiff; p.cTMass = cTMass; p.U = U; p.Udot = Udot; p.out = d;
	RSD_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * std::max<int64_t>(h->n, 1), ctx->stream));
	return launch_k_asm_diag(ctx, h, p);
}

}  // namespace rsd
