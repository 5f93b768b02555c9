// Context, memory, errors, expression compiler, mesh upload, DOF map and CSR pattern.
#include <algorithm>
#include <map>
#include <mutex>
#include <cctype>
#include <cmath>
#include <cstring>
#include <thread>

#include "rsd_internal.cuh"

namespace rsd {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
	g_last_error = msg;
	return code;
}

int cuda_error(cudaError_t e, const char* what) {
	const int code = (e == cudaErrorMemoryAllocation) ? RSD_ENOMEM : RSD_ECUDA;
	return set_error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------------
// expression compiler: recursive descent over the exprtk subset the reference's configurations use
// (src/utils/expression/ScalarExpression.cpp:3-30, equation/heateq/evaluator/TemperatureExpression.hpp:31-58)
// ---------------------------------------------------------------------------------------------
namespace {
struct Parser {
	const char* s;
	size_t pos = 0;
	bool err = false;
	DevExpr* e;
	int nconst = 0;
	void emit(ExprOp op, int arg = 0, double c = 0.0) {
		if (e->n >= kExprMax) { err = true; return; }
		e->op[e->n] = op;
		if (op == E_CONST) { e->c[nconst] = c; e->arg[e->n] = (int8_t)nconst++; }
		else e->arg[e->n] = (int8_t)arg;
		e->n++;
	}
	void ws() { while (s[pos] && std::isspace((unsigned char)s[pos])) pos++; }
	void primary() {
		ws();
		const char c = s[pos];
		if (c == '(') { pos++; expr(); ws(); if (s[pos] != ')') { err = true; return; } pos++; return; }
		if (std::isdigit((unsigned char)c) || c == '.') {
			char* end = nullptr;
			const double v = std::strtod(s + pos, &end);
			if (end == s + pos) { err = true; return; }
			pos = (size_t)(end - s);
			emit(E_CONST, 0, v);
			return;
		}
		if (std::isalpha((unsigned char)c) || c == '_') {
			std::string name;
			while (std::isalnum((unsigned char)s[pos]) || s[pos] == '_') name += s[pos++];
			static const char* vars[] = {"t", "x", "y", "z", "T"};
			for (int v = 0; v < 5; ++v) if (name == vars[v]) { emit(E_VAR, v); return; }
			if (name == "pi") { emit(E_CONST, 0, 3.14159265358979323846); return; }
			static const char* fns[] = {"sin", "cos", "tan", "exp", "log", "sqrt", "abs"};
			static const ExprOp fop[] = {E_SIN, E_COS, E_TAN, E_EXP, E_LOG, E_SQRT, E_ABS};
			for (int f = 0; f < 7; ++f)
				if (name == fns[f]) {
					ws();
					if (s[pos] != '(') { err = true; return; }
					pos++; expr(); ws();
					if (s[pos] != ')') { err = true; return; }
					pos++;
					emit(fop[f]);
					return;
				}
		}
		err = true;
	}
	void power() { primary(); ws(); if (s[pos] == '^') { pos++; unary(); emit(E_POW); } }
	void unary() {
		ws();
		if (s[pos] == '-') { pos++; unary(); emit(E_NEG); return; }
		if (s[pos] == '+') { pos++; unary(); return; }
		power();
	}
	void term() {
		unary();
		for (;;) { ws(); const char c = s[pos]; if (c != '*' && c != '/') return; pos++; unary(); emit(c == '*' ? E_MUL : E_DIV); }
	}
	void expr() {
		term();
		for (;;) { ws(); const char c = s[pos]; if (c != '+' && c != '-') return; pos++; term(); emit(c == '+' ? E_ADD : E_SUB); }
	}
};
}  // namespace

int compile_expr(const char* src, DevExpr* out) {
	*out = DevExpr();
	if (!src) return RSD_OK;
	Parser p{src, 0, false, out};
	p.expr();
	p.ws();
	if (p.err || src[p.pos] != 0 || out->n == 0) {
		*out = DevExpr();
		return set_error(RSD_EPARSE, std::string("cannot compile expression '") + src + "'");
	}
	// the stack depth the postfix program reaches: operands push one, binary operators pop one
	int sp = 0, depth = 0;
	for (int i = 0; i < out->n; ++i) {
		const int op = out->op[i];
		if (op == E_CONST || op == E_VAR) ++sp;
		else if (op == E_ADD || op == E_SUB || op == E_MUL || op == E_DIV || op == E_POW) --sp;
		depth = std::max(depth, sp);
	}
	if (depth > kExprStack) {
		*out = DevExpr();
		return set_error(RSD_EPARSE, std::string("expression '") + src + "' needs an evaluation stack of " + std::to_string(depth) +
		                 " entries; the device machine holds " + std::to_string(kExprStack));
	}
	out->depth = depth;
	return RSD_OK;
}

double eval_expr_host(const DevExpr& e, double t, double x, double y, double z, double T) {
	double st[kExprStack];
	int sp = 0;
	const double v[5] = {t, x, y, z, T};
	for (int i = 0; i < e.n; ++i) {
		switch (e.op[i]) {
			case E_CONST: st[sp++] = e.c[e.arg[i]]; break;
			case E_VAR: st[sp++] = v[e.arg[i]]; break;
			case E_ADD: sp--; st[sp - 1] = st[sp - 1] + st[sp]; break;
			case E_SUB: sp--; st[sp - 1] = st[sp - 1] - st[sp]; break;
			case E_MUL: sp--; st[sp - 1] = st[sp - 1] * st[sp]; break;
			case E_DIV: sp--; st[sp - 1] = st[sp - 1] / st[sp]; break;
			case E_POW: sp--; st[sp - 1] = std::pow(st[sp - 1], st[sp]); break;
			case E_NEG: st[sp - 1] = -st[sp - 1]; break;
			case E_SIN: st[sp - 1] = std::sin(st[sp - 1]); break;
			case E_COS: st[sp - 1] = std::cos(st[sp - 1]); break;
			case E_TAN: st[sp - 1] = std::tan(st[sp - 1]); break;
			case E_EXP: st[sp - 1] = std::exp(st[sp - 1]); break;
			case E_LOG: st[sp - 1] = std::log(st[sp - 1]); break;
			case E_SQRT: st[sp - 1] = std::sqrt(st[sp - 1]); break;
			default: st[sp - 1] = std::fabs(st[sp - 1]); break;
		}
	}
	return e.n ? st[0] : 0.0;
}

// ---------------------------------------------------------------------------------------------
// host parallel-for over [0, n)
// ---------------------------------------------------------------------------------------------
template <typename Fn>
static void parallel_for(int64_t n, Fn&& fn) {
	unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
	if (n < 65536) nt = 1;
	std::vector<std::thread> th;
	const int64_t chunk = (n + nt - 1) / nt;
	for (unsigned t = 0; t < nt; ++t) {
		const int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
		if (b >= e) break;
		th.emplace_back([=, &fn] { fn(b, e); });
	}
	for (auto& t : th) t.join();
}

// ---------------------------------------------------------------------------------------------
// TopologicalDOF::buildConstraints, Interleaved ordering (topology/TopologicalDOF.tpp:34-111):
// nodes on faces whose tag is essential are constrained; the constraint tag is the last face
// (in element, face order) that marked the node (h_ctag holds that tag's expression index); free nodes are numbered in ascending order.
// Face-node lists are LagrangeQuad/Hex::getFaceNodes (fem/basis/LagrangeQuad.tpp:136-155,
// fem/basis/LagrangeHex.tpp:263-304).
// ---------------------------------------------------------------------------------------------
int face_nodes(int nsd, int p, int f, int* out) {
	const int q = p + 1;
	int k = 0;
	if (nsd == 2) {
		for (int i = 0; i < q; ++i) out[k++] = f == 0 ? i * q : f == 1 ? i * q + p : f == 2 ? i : i + q * p;
		return k;
	}
	for (int j = 0; j < q; ++j)
		for (int i = 0; i < q; ++i) {
			int v;
			switch (f) {
				case 0: v = i * q + j * q * q; break;
				case 1: v = i * q + j * q * q + p; break;
				case 2: v = i + j * q * q; break;
				case 3: v = i + j * q * q + q * p; break;
				case 4: v = i + j * q; break;
				default: v = i + j * q + q * q * p; break;
			}
			out[k++] = v;
		}
	return k;
}

// the device builds the DOF map and the pattern unless RSD_HOST_SETUP=1 selects the host loops
bool device_setup() {
	const char* env = getenv("RSD_HOST_SETUP");
	return !(env && env[0] == '1');
}

int build_dofmap(rsd_heat* h) {
	const rsd_mesh* m = h->m;
	h->h_t2a.assign(m->nnodes, 0);
	h->h_ctag.assign(m->nnodes, -1);
	std::map<int32_t, int32_t> index;   // essential tag -> its expression
	for (size_t i = 0; i < h->essTags.size(); ++i) index[h->essTags[i]] = (int32_t)i;
	int fn[64];
	for (int64_t e = 0; e < m->nelem; ++e)
		for (int f = 0; f < m->nfaces; ++f) {
			const int32_t tag = m->h_rng[e * m->nfaces + f];
			if (tag < 0) continue;
			const auto it = index.find(tag);
			if (it == index.end()) continue;
			const int npf = face_nodes(m->nsd, m->order, f, fn);
			for (int i = 0; i < npf; ++i) {
				const int32_t node = m->h_ien[e * m->npe + fn[i]];
				h->h_t2a[node] = -1;
				h->h_ctag[node] = it->second;
			}
		}
	h->h_a2t.clear();
	h->h_a2t.reserve(m->nnodes);
	int64_t alg = 0;
	for (int64_t i = 0; i < m->nnodes; ++i) {
		if (h->h_t2a[i] == -1) continue;
		h->h_t2a[i] = (int32_t)alg++;
		h->h_a2t.push_back((int32_t)i);
	}
	h->n = alg;
	return RSD_OK;
}

// diagonal position per row (CSROperator::diagonal's getDataIndex, linalg/types/CSRMatrix.hpp:49-73)
static void diag_index(int64_t n, const int32_t* rp, const int32_t* col, int32_t* d) {
	parallel_for(n, [&](int64_t b, int64_t e) {
		for (int64_t i = b; i < e; ++i) {
			const int32_t* first = col + rp[i];
			const int32_t* last = col + rp[i + 1];
			const int32_t* it = std::lower_bound(first, last, (int32_t)i);
			d[i] = (it != last && *it == i) ? (int32_t)(it - col) : -1;
		}
	});
}

int resident_blocks(const void* kernel, int block) {
	static std::mutex mu;
	static std::map<std::pair<const void*, int>, int> cache;
	std::lock_guard<std::mutex> lk(mu);
	auto it = cache.find({kernel, block});
	if (it != cache.end()) return it->second;
	int occ = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, 0) != cudaSuccess || occ < 1) {
		cudaGetLastError();
		occ = 1;
	}
	cache[{kernel, block}] = occ;
	return occ;
}

static void free_csr_arrays(rsd_csr* A) {
	cudaFree(A->val); cudaFree(A->sVal); cudaFree(A->val32);
	if (!A->owns_pattern) return;   // the pattern belongs to the matrix it was shared from
	cudaFree(A->rowPtr); cudaFree(A->col); cudaFree(A->diag);
	cudaFree(A->sStart); cudaFree(A->sCol); cudaFree(A->sSrc); cudaFree(A->sDiag); cudaFree(A->sCol16); cudaFree(A->sBase); cudaFree(A->sUni); cudaFree(A->sOffs);
	cudaFree(A->sPerm); cudaFree(A->sIperm); cudaFree(A->sNeg); cudaFree(A->sMir); cudaFree(A->sMk);
}

// The row order of the SELL-32 slices (SELL-C-sigma): within windows of kSellWindow rows, rows sorted
// by length (longest first) and then by their column-offset pattern, stably, so that a slice holds
// rows of one kind (on a Q2 mesh: vertex, edge, face or interior nodes, whose rows have 125, 75, 45
// or 27 entries and one offset pattern each) instead of alternating kinds padded to the longest.
// Opt-in (RSD_SELL_SORT=1), and then used when it shrinks the padded layout by a tenth or more.  On
// the 48^3 Q2 Jacobian it cut the padding from 1.59 to 1.06 slots per entry but made GMRES's Arnoldi
// step slower (241 against 223 us FP64): a slice's rows are then every other row of a grid line, so
// the gathers touch twice the sectors, and fewer slices share one stencil pattern.  The rows past the
// last whole window keep their order.
constexpr int64_t kSellWindow = 32 * 16;
static bool sell_row_order(int64_t n, const std::vector<int32_t>& rp, const std::vector<int32_t>& col,
                           std::vector<int32_t>* perm) {
	const char* env = getenv("RSD_SELL_SORT");
	if (!(env && env[0] == '1') || n < kSellWindow) return false;
	auto padded = [&](const int32_t* order) {
		int64_t total = 0;
		for (int64_t s0 = 0; s0 < n; s0 += 32) {
			int32_t len = 0;
			for (int64_t i = s0; i < std::min<int64_t>(n, s0 + 32); ++i) {
				const int32_t r = order ? order[i] : (int32_t)i;
				len = std::max(len, rp[r + 1] - rp[r]);
			}
			total += 32 * (int64_t)((len + 1) & ~1);
		}
		return total;
	};
	std::vector<uint64_t> key(n);
	parallel_for(n, [&](int64_t b, int64_t e) {
		for (int64_t i = b; i < e; ++i) {
			uint64_t hsh = 1469598103934665603ull;   // FNV-1a over the offsets col - row
			for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
				hsh ^= (uint64_t)(uint32_t)(col[q] - (int32_t)i);
				hsh *= 1099511628211ull;
			}
			const uint64_t len = (uint64_t)(rp[i + 1] - rp[i]);
			key[i] = ((0xFFFFull - std::min<uint64_t>(len, 0xFFFF)) << 48) | (hsh >> 16);
		}
	});
	std::vector<int32_t> order(n);
	for (int64_t i = 0; i < n; ++i) order[i] = (int32_t)i;
	const int64_t windows = n / kSellWindow;
	parallel_for(windows, [&](int64_t b, int64_t e) {
		for (int64_t w = b; w < e; ++w)
			std::stable_sort(order.begin() + w * kSellWindow, order.begin() + (w + 1) * kSellWindow,
			                 [&](int32_t x, int32_t y) { return key[x] < key[y]; });
	});
	if (padded(order.data()) * 10 > padded(nullptr) * 9) return false;
	*perm = std::move(order);
	return true;
}

// A matrix with src's pattern and layout (shared, not copied) and zero values of its own.
int share_pattern(rsd_ctx* ctx, const rsd_csr* src, rsd_csr** out) {
	rsd_csr* A = new rsd_csr(*src);
	A->owns_pattern = false;
	A->val = nullptr; A->sVal = nullptr; A->val32 = nullptr;
	A->fmt32 = -1; A->version = 1; A->version32 = 0; A->symVersion = 0;
	cudaError_t e;
	if ((e = cudaMalloc(&A->val, sizeof(double) * std::max<int64_t>(A->nnz, 1))) != cudaSuccess ||
	    (e = cudaMalloc(&A->sVal, sizeof(double) * std::max<int64_t>(A->ssize, 1))) != cudaSuccess ||
	    (e = cudaMemsetAsync(A->val, 0, sizeof(double) * std::max<int64_t>(A->nnz, 1), ctx->stream)) != cudaSuccess ||
	    (e = cudaMemsetAsync(A->sVal, 0, sizeof(double) * std::max<int64_t>(A->ssize, 1), ctx->stream)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
		cudaFree(A->val); cudaFree(A->sVal);
		delete A;
		return cuda_error(e, "matrix values");
	}
	A->csrValid = true;
	A->sellValid = true;
	*out = A;
	return RSD_OK;
}

static int upload_csr(rsd_ctx* ctx, int64_t n, const std::vector<int32_t>& rp, const std::vector<int32_t>& col,
                      const double* hval, rsd_csr** out) {
	const int64_t nnz = rp[n];
	rsd_csr* A = new rsd_csr();
	A->n = n;
	A->nnz = nnz;
	std::vector<int32_t> d(n);
	diag_index(n, rp.data(), col.data(), d.data());
	// SELL-32 layout: slice s holds slot rows 32s..32s+31 (matrix rows prow(slot row): the identity
	// unless sell_row_order groups rows of one kind), padded to its longest row rounded up to even;
	// entries are stored in pairs, entry j of lane l at start[s] + 64 (j / 2) + 2 l + (j % 2), so that a
	// lane reads two consecutive entries of its row with one 8- or 16-byte load
	std::vector<int32_t> perm;
	const bool permuted = sell_row_order(n, rp, col, &perm);
	auto prow = [&](int64_t r) -> int64_t { return permuted ? (int64_t)perm[r] : r; };
	const int64_t ns = (n + 31) / 32;
	std::vector<int64_t> start(ns + 1, 0);
	for (int64_t s = 0; s < ns; ++s) {
		int32_t len = 0;
		for (int64_t i = 32 * s; i < std::min<int64_t>(n, 32 * s + 32); ++i) len = std::max(len, rp[prow(i) + 1] - rp[prow(i)]);
		start[s + 1] = start[s] + 32 * (int64_t)((len + 1) & ~1);
	}
	auto pos = [&](int64_t s, int64_t l, int64_t j) { return start[s] + 64 * (j >> 1) + 2 * l + (j & 1); };
	const int64_t ssize = start[ns];
	if (ssize > INT32_MAX) { delete A; return set_error(RSD_EINVAL, "padded SELL layout has 2^31 or more slots"); }
	std::vector<int32_t> sStart(ns + 1), sCol(std::max<int64_t>(ssize, 1)), sSrc(std::max<int64_t>(ssize, 1), -1), sDiag(std::max<int64_t>(n, 1), -1);
	std::vector<int32_t> sMin(std::max<int64_t>(ns, 1)), sMax(std::max<int64_t>(ns, 1));
	for (int64_t s = 0; s <= ns; ++s) sStart[s] = (int32_t)start[s];
	parallel_for(ns, [&](int64_t b, int64_t e) {
		for (int64_t s = b; s < e; ++s) {
			const int64_t len = (start[s + 1] - start[s]) / 32;
			const int64_t r0 = prow(32 * s);
			// padding repeats a column the row already holds (value 0), so that it reads nothing new
			const int32_t pad0 = rp[r0] < rp[r0 + 1] ? col[rp[r0]] : (int32_t)r0;
			int32_t lo = INT32_MAX, hi = INT32_MIN;
			for (int64_t l = 0; l < 32; ++l) {
				const bool in = 32 * s + l < n;
				const int64_t i = in ? prow(32 * s + l) : -1;   // the matrix row of the slot row
				const int32_t pad = in ? (rp[i] < rp[i + 1] ? col[rp[i + 1] - 1] : (int32_t)i) : pad0;
				for (int64_t j = 0; j < len; ++j) {
					const int64_t slot = pos(s, l, j);
					if (in && rp[i] + j < rp[i + 1]) { sCol[slot] = col[rp[i] + j]; sSrc[slot] = (int32_t)(rp[i] + j); }
					else sCol[slot] = pad;
					lo = std::min(lo, sCol[slot]);
					hi = std::max(hi, sCol[slot]);
				}
				if (in && d[i] >= 0) sDiag[i] = (int32_t)pos(s, l, d[i] - rp[i]);
			}
			sMin[s] = len ? lo : 0;
			sMax[s] = len ? hi : 0;
		}
	});
	// stencil slices: a full slice whose rows' column offsets (column - row) all belong to one sorted
	// pattern no longer than the slice's padded length stores that pattern once.  Entry j of every row
	// of the slice is then the pattern's offset j: a row without that column holds a zero there (its
	// column row + offset must lie in [0, n), so that the gather stays in range), and the padding
	// repeats the last offset.  Rows that differ only by missing neighbours (the ends of grid lines)
	// thus share the slice pattern, and the slice reads no column bytes.
	std::vector<int32_t> sUni(std::max<int64_t>(ns, 1), -1), offTable;
	{
		std::vector<std::vector<int32_t>> pat(ns);
		parallel_for(ns, [&](int64_t b, int64_t e) {
			std::vector<int32_t> u;
			for (int64_t s = b; s < e; ++s) {
				const int64_t r0 = 32 * s, len2 = (start[s + 1] - start[s]) / 32;
				if (r0 + 32 > n || len2 == 0) continue;
				u.clear();
				bool sorted = true;   // rows in increasing column order (the re-lay below matches in order)
				int64_t rmin = INT64_MAX, rmax = -1;
				for (int64_t l = 0; l < 32; ++l) {
					const int64_t i = prow(r0 + l);
					rmin = std::min(rmin, i);
					rmax = std::max(rmax, i);
					for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
						u.push_back(col[q] - (int32_t)i);
						sorted = sorted && (q == rp[i] || col[q - 1] < col[q]);
					}
				}
				if (!sorted) continue;
				std::sort(u.begin(), u.end());
				u.erase(std::unique(u.begin(), u.end()), u.end());
				if (u.empty() || (int64_t)u.size() > len2) continue;
				if (rmin + u.front() < 0 || rmax + (int64_t)u.back() >= n) continue;
				pat[s] = u;
				pat[s].resize(len2, u.back());
			}
		});
		std::map<std::vector<int32_t>, int32_t> seen;
		for (int64_t s = 0; s < ns; ++s) {
			if (pat[s].empty()) continue;
			auto it = seen.find(pat[s]);
			if (it == seen.end()) {
				it = seen.emplace(pat[s], (int32_t)offTable.size()).first;
				offTable.insert(offTable.end(), pat[s].begin(), pat[s].end());
			}
			sUni[s] = it->second;
			++A->nStencil;
		}
		// re-lay the stencil slices by pattern position (the CSR rank order above holds for the rest)
		parallel_for(ns, [&](int64_t b, int64_t e) {
			for (int64_t s = b; s < e; ++s) {
				if (sUni[s] < 0) continue;
				const int32_t* off = offTable.data() + sUni[s];
				const int64_t len = (start[s + 1] - start[s]) / 32;
				int32_t lo = INT32_MAX, hi = INT32_MIN;
				for (int64_t l = 0; l < 32; ++l) {
					const int64_t i = prow(32 * s + l);
					int32_t q = rp[i];
					sDiag[i] = -1;
					for (int64_t j = 0; j < len; ++j) {
						const int64_t slot = pos(s, l, j);
						const int32_t c = (int32_t)i + off[j];
						sCol[slot] = c;
						sSrc[slot] = -1;
						if (q < rp[i + 1] && col[q] == c) {
							sSrc[slot] = q;
							if (q == d[i]) sDiag[i] = (int32_t)slot;
							++q;
						}
						lo = std::min(lo, c);
						hi = std::max(hi, c);
					}
				}
				sMin[s] = lo;
				sMax[s] = hi;
			}
		});
	}
	const bool stencil = !offTable.empty();
	// mirrored stencil slices: for a symmetric matrix, entry (i, i + o) with o < 0 equals entry
	// (i + o, i), which the mirror row stores at offset -o; a slice qualifies when for each of its
	// negative offsets the mirror rows (one or two slices) are stencil slices holding -o at one common
	// position.  The SpMV then reads only its own entries from offset 0 on; the mirrored ones come from
	// rows a few slices back, still in L2.
	std::vector<int32_t> sNeg, sMir;
	std::vector<uint8_t> sMk;
	if (stencil && !permuted) {
		sNeg.assign(ns, 0);
		sMir.assign(ns, 0);
		auto find_off = [&](int64_t t, int32_t off) -> int {
			if (t < 0 || t >= ns || sUni[t] < 0) return -1;
			const int32_t* pt = offTable.data() + sUni[t];
			const int64_t lt = (start[t + 1] - start[t]) / 32;
			for (int64_t j = 0; j < lt; ++j)
				if (pt[j] == off) return (int)j;
			return -1;
		};
		for (int64_t sl = 0; sl < ns; ++sl) {
			if (sUni[sl] < 0) continue;
			const int32_t* pt = offTable.data() + sUni[sl];
			const int64_t len = (start[sl + 1] - start[sl]) / 32;
			int nneg = 0;
			while (nneg < len && pt[nneg] < 0) ++nneg;
			if (nneg == 0 || nneg > 32) continue;
			std::vector<uint8_t> mk(nneg);
			bool ok = true;
			for (int j = 0; j < nneg && ok; ++j) {
				const int64_t m0 = 32 * sl + pt[j], m1 = m0 + 31;   // the mirror rows of the slice's lanes
				const int a = find_off(m0 >> 5, -pt[j]), b = find_off(m1 >> 5, -pt[j]);
				ok = a >= 0 && a < 255 && a == b;
				if (ok) mk[j] = (uint8_t)a;
			}
			if (!ok) continue;
			sNeg[sl] = nneg;
			sMir[sl] = (int32_t)sMk.size();
			sMk.insert(sMk.end(), mk.begin(), mk.end());
			++A->nMirrored;
		}
	}
	// 16-bit columns: every slice's columns within 65,535 of the slice's smallest one
	bool narrow = ssize > 0;
	for (int64_t s = 0; s < ns && narrow; ++s) narrow = (int64_t)sMax[s] - sMin[s] <= 65535;
	std::vector<uint16_t> sCol16;
	if (narrow) {
		sCol16.resize(ssize);
		parallel_for(ns, [&](int64_t b, int64_t e) {
			for (int64_t s = b; s < e; ++s)
				for (int64_t q = start[s]; q < start[s + 1]; ++q) sCol16[q] = (uint16_t)(sCol[q] - sMin[s]);
		});
	}
	A->nslices = ns;
	A->ssize = ssize;
	auto fail = [&](cudaError_t e, const char* w) { free_csr_arrays(A); delete A; return cuda_error(e, w); };
	const size_t S = (size_t)std::max<int64_t>(ssize, 1);
	cudaError_t e;
	if ((e = cudaMalloc(&A->rowPtr, sizeof(int32_t) * (n + 1))) != cudaSuccess) return fail(e, "cudaMalloc rowPtr");
	if ((e = cudaMalloc(&A->col, sizeof(int32_t) * std::max<int64_t>(nnz, 1))) != cudaSuccess) return fail(e, "cudaMalloc col");
	if ((e = cudaMalloc(&A->val, sizeof(double) * std::max<int64_t>(nnz, 1))) != cudaSuccess) return fail(e, "cudaMalloc val");
	if ((e = cudaMalloc(&A->diag, sizeof(int32_t) * std::max<int64_t>(n, 1))) != cudaSuccess) return fail(e, "cudaMalloc diag");
	if ((e = cudaMalloc(&A->sStart, sizeof(int32_t) * (ns + 1))) != cudaSuccess) return fail(e, "cudaMalloc sStart");
	if ((e = cudaMalloc(&A->sCol, sizeof(int32_t) * S)) != cudaSuccess) return fail(e, "cudaMalloc sCol");
	if ((e = cudaMalloc(&A->sVal, sizeof(double) * S)) != cudaSuccess) return fail(e, "cudaMalloc sVal");
	if ((e = cudaMalloc(&A->sSrc, sizeof(int32_t) * S)) != cudaSuccess) return fail(e, "cudaMalloc sSrc");
	if ((e = cudaMalloc(&A->sDiag, sizeof(int32_t) * std::max<int64_t>(n, 1))) != cudaSuccess) return fail(e, "cudaMalloc sDiag");
	if ((e = cudaMemcpyAsync(A->rowPtr, rp.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload rowPtr");
	if (nnz && (e = cudaMemcpyAsync(A->col, col.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload col");
	if (n && (e = cudaMemcpyAsync(A->diag, d.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload diag");
	if ((e = cudaMemcpyAsync(A->sStart, sStart.data(), sizeof(int32_t) * (ns + 1), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sStart");
	if ((e = cudaMemcpyAsync(A->sCol, sCol.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sCol");
	if ((e = cudaMemcpyAsync(A->sSrc, sSrc.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sSrc");
	if ((e = cudaMemcpyAsync(A->sDiag, sDiag.data(), sizeof(int32_t) * std::max<int64_t>(n, 1), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sDiag");
	if (stencil) {
		if ((e = cudaMalloc(&A->sUni, sizeof(int32_t) * ns)) != cudaSuccess) return fail(e, "cudaMalloc sUni");
		if ((e = cudaMalloc(&A->sOffs, sizeof(int32_t) * offTable.size())) != cudaSuccess) return fail(e, "cudaMalloc sOffs");
		if ((e = cudaMemcpyAsync(A->sUni, sUni.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sUni");
		if ((e = cudaMemcpyAsync(A->sOffs, offTable.data(), sizeof(int32_t) * offTable.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sOffs");
	}
	if (A->nMirrored) {
		if ((e = cudaMalloc(&A->sNeg, sizeof(int32_t) * ns)) != cudaSuccess) return fail(e, "cudaMalloc sNeg");
		if ((e = cudaMalloc(&A->sMir, sizeof(int32_t) * ns)) != cudaSuccess) return fail(e, "cudaMalloc sMir");
		if ((e = cudaMalloc(&A->sMk, sMk.size())) != cudaSuccess) return fail(e, "cudaMalloc sMk");
		if ((e = cudaMemcpyAsync(A->sNeg, sNeg.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sNeg");
		if ((e = cudaMemcpyAsync(A->sMir, sMir.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sMir");
		if ((e = cudaMemcpyAsync(A->sMk, sMk.data(), sMk.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sMk");
	}
	if (permuted) {
		std::vector<int32_t> iperm(n);
		for (int64_t r = 0; r < n; ++r) iperm[perm[r]] = (int32_t)r;
		if ((e = cudaMalloc(&A->sPerm, sizeof(int32_t) * n)) != cudaSuccess) return fail(e, "cudaMalloc sPerm");
		if ((e = cudaMalloc(&A->sIperm, sizeof(int32_t) * n)) != cudaSuccess) return fail(e, "cudaMalloc sIperm");
		if ((e = cudaMemcpyAsync(A->sPerm, perm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sPerm");
		if ((e = cudaMemcpyAsync(A->sIperm, iperm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sIperm");
		// the host copy must outlive the asynchronous copies: synchronize before it goes out of scope
		if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(e, "upload sIperm");
	}
	if (narrow) {
		if ((e = cudaMalloc(&A->sCol16, sizeof(uint16_t) * ssize)) != cudaSuccess) return fail(e, "cudaMalloc sCol16");
		if ((e = cudaMalloc(&A->sBase, sizeof(int32_t) * ns)) != cudaSuccess) return fail(e, "cudaMalloc sBase");
		if ((e = cudaMemcpyAsync(A->sCol16, sCol16.data(), sizeof(uint16_t) * ssize, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sCol16");
		if ((e = cudaMemcpyAsync(A->sBase, sMin.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail(e, "upload sBase");
	}
	if (hval && nnz) e = cudaMemcpyAsync(A->val, hval, sizeof(double) * nnz, cudaMemcpyHostToDevice, ctx->stream);
	else e = cudaMemsetAsync(A->val, 0, sizeof(double) * std::max<int64_t>(nnz, 1), ctx->stream);
	if (e != cudaSuccess) return fail(e, "upload values");
	if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(e, "csr upload sync");
	A->csrValid = true;
	A->sellValid = false;
	*out = A;
	return RSD_OK;
}

// Assembler<CPU>::createMatrix (fem/assembly/backend/cpu/Assembler.tpp:8-76): row i holds the
// sorted, unique free columns of every element touching free DOF i.  Built per row from a
// node->element incidence list, in parallel on the host (one-time setup).
int build_pattern(rsd_ctx* ctx, const rsd_heat* h, rsd_csr** out) {
	if (device_setup()) {
		std::vector<int32_t> rp, col;
		bool fallback = false;
		RSD_CHECK(device_pattern(ctx, h, rp, col, &fallback));
		if (!fallback) return upload_csr(ctx, h->n, rp, col, nullptr, out);
	}
	const rsd_mesh* m = h->m;
	const int64_t n = h->n, nn = m->nnodes, ne = m->nelem;
	const int npe = m->npe;
	std::vector<int64_t> ioff(nn + 1, 0);
	for (int64_t i = 0; i < ne * npe; ++i) ioff[m->h_ien[i] + 1]++;
	for (int64_t i = 0; i < nn; ++i) ioff[i + 1] += ioff[i];
	std::vector<int32_t> inc(ne * npe);
	{
		std::vector<int64_t> cur(ioff.begin(), ioff.end() - 1);
		for (int64_t e = 0; e < ne; ++e)
			for (int a = 0; a < npe; ++a) inc[cur[m->h_ien[e * npe + a]]++] = (int32_t)e;
	}
	std::vector<int32_t> rp(n + 1, 0);
	auto row_cols = [&](int64_t r, std::vector<int32_t>& buf) {
		buf.clear();
		const int32_t node = h->h_a2t[r];
		for (int64_t k = ioff[node]; k < ioff[node + 1]; ++k) {
			const int32_t* en = &m->h_ien[(int64_t)inc[k] * npe];
			for (int b = 0; b < npe; ++b) { const int32_t c = h->h_t2a[en[b]]; if (c >= 0) buf.push_back(c); }
		}
		std::sort(buf.begin(), buf.end());
		buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
	};
	parallel_for(n, [&](int64_t b, int64_t e) {
		std::vector<int32_t> buf;
		for (int64_t r = b; r < e; ++r) { row_cols(r, buf); rp[r + 1] = (int32_t)buf.size(); }
	});
	int64_t total = 0;
	for (int64_t r = 0; r < n; ++r) {
		total += rp[r + 1];
		if (total > INT32_MAX) return set_error(RSD_EINVAL, "pattern has 2^31 or more non-zeros");
		rp[r + 1] = (int32_t)total;
	}
	std::vector<int32_t> col(total);
	parallel_for(n, [&](int64_t b, int64_t e) {
		std::vector<int32_t> buf;
		for (int64_t r = b; r < e; ++r) { row_cols(r, buf); std::copy(buf.begin(), buf.end(), col.begin() + rp[r]); }
	});
	return upload_csr(ctx, n, rp, col, nullptr, out);
}

// ---------------------------------------------------------------------------------------------
// per-kernel-family event timing
// ---------------------------------------------------------------------------------------------
static const char* kFamilyNames[PF_COUNT] = {"spmv_dot_f64", "spmv_dot_f32", "cg_update", "cg_pupdate", "reliable_update",
                                             "assemble_matrix", "assemble_vector", "spmv", "cg_persist"};

int prof_begin(rsd_ctx* ctx, int family) {
	Profiler& p = ctx->prof;
	if (!p.on) return -1;
	if (p.used + 2 > p.pool.size()) {
		if (p.used + 2 > 1 << 16) prof_flush(ctx);
		while (p.used + 2 > p.pool.size()) {
			cudaEvent_t e;
			if (cudaEventCreate(&e) != cudaSuccess) return -1;
			p.pool.push_back(e);
		}
	}
	const int pair = (int)(p.used / 2);
	cudaEventRecord(p.pool[p.used], ctx->stream);
	p.used += 2;
	if ((int)p.fam.size() <= pair) p.fam.resize(pair + 1);
	p.fam[pair] = family;
	return pair;
}

void prof_end(rsd_ctx* ctx, int pair) {
	if (pair < 0) return;
	cudaEventRecord(ctx->prof.pool[2 * pair + 1], ctx->stream);
}

int prof_flush(rsd_ctx* ctx) {
	Profiler& p = ctx->prof;
	if (!p.used) return RSD_OK;
	RSD_CUDA(cudaStreamSynchronize(ctx->stream));
	for (size_t k = 0; k < p.used / 2; ++k) {
		float ms = 0.f;
		if (p.fam[k] < 0) continue;
		if (cudaEventElapsedTime(&ms, p.pool[2 * k], p.pool[2 * k + 1]) == cudaSuccess) {
			p.launches[p.fam[k]] += 1;
			p.total_ms[p.fam[k]] += ms;
		}
	}
	p.used = 0;
	return RSD_OK;
}

}  // namespace rsd

using namespace rsd;

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

int rsd_ctx_profile(rsd_ctx* c, int32_t enable) {
	if (!c) return set_error(RSD_EINVAL, "null context");
	RSD_CHECK(prof_flush(c));
	c->prof.on = enable != 0;
	for (int f = 0; f < PF_COUNT; ++f) { c->prof.launches[f] = 0; c->prof.total_ms[f] = 0.0; }
	return RSD_OK;
}

int rsd_ctx_profile_get(rsd_ctx* c, const char* family, int64_t* launches, double* total_ms) {
	if (!c || !family) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(prof_flush(c));
	for (int f = 0; f < PF_COUNT; ++f)
		if (!std::strcmp(family, kFamilyNames[f])) {
			if (launches) *launches = c->prof.launches[f];
			if (total_ms) *total_ms = c->prof.total_ms[f];
			return RSD_OK;
		}
	return set_error(RSD_EINVAL, std::string("unknown kernel family ") + family);
}

const char* rsd_last_error_string(void) { return g_last_error.c_str(); }

int rsd_expr_check(const char* expr, int32_t* depth) {
	if (!expr) return set_error(RSD_EINVAL, "null expression");
	DevExpr e;
	RSD_CHECK(compile_expr(expr, &e));
	if (depth) *depth = e.depth;
	return RSD_OK;
}

int rsd_version(int32_t* major, int32_t* minor) {
	if (major) *major = 0;
	if (minor) *minor = 1;
	return RSD_OK;
}

int rsd_ctx_create(int device, rsd_ctx** out) {
	if (!out) return set_error(RSD_EINVAL, "null output");
	int count = 0;
	RSD_CUDA(cudaGetDeviceCount(&count));
	if (device < 0 || device >= count) return set_error(RSD_EINVAL, "no such CUDA device");
	RSD_CUDA(cudaSetDevice(device));
	rsd_ctx* c = new rsd_ctx();
	c->device = device;
	cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
	cudaError_t e;
	if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) { delete c; return cuda_error(e, "cudaStreamCreate"); }
	if ((e = cudaMalloc(&c->s.partials, sizeof(double) * kMaxPartials * 4)) != cudaSuccess ||
	    (e = cudaMalloc(&c->s.scal, sizeof(DevScalars) * 4)) != cudaSuccess ||
	    (e = cudaMallocHost(&c->s.hscal, sizeof(DevScalars) * 4)) != cudaSuccess ||
	    (e = cudaMallocHost(&c->s.hbuf, sizeof(double) * 64)) != cudaSuccess) {
		rsd_ctx_destroy(c);
		return cuda_error(e, "context scratch");
	}
	cudaMemsetAsync(c->s.scal, 0, sizeof(DevScalars) * 4, c->stream);
	cudaStreamSynchronize(c->stream);
	*out = c;
	return RSD_OK;
}

int rsd_ctx_destroy(rsd_ctx* c) {
	if (!c) return RSD_OK;
	cudaSetDevice(c->device);
	if (c->stream) cudaStreamSynchronize(c->stream);
	for (cudaEvent_t e : c->prof.pool) cudaEventDestroy(e);
	free_graph_cache(c);
	cudaFree(c->ws);
	cudaFree(c->s.partials);
	cudaFree(c->s.scal);
	cudaFreeHost(c->s.hscal);
	cudaFreeHost(c->s.hbuf);
	if (c->copy) { cudaStreamSynchronize(c->copy); cudaStreamDestroy(c->copy); }
	if (c->copyReady) cudaEventDestroy(c->copyReady);
	if (c->uploaded) cudaEventDestroy(c->uploaded);
	if (c->stream) cudaStreamDestroy(c->stream);
	delete c;
	return RSD_OK;
}

int rsd_ctx_sync(rsd_ctx* c) {
	if (!c) return set_error(RSD_EINVAL, "null context");
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

void* rsd_ctx_stream(rsd_ctx* c) { return c ? (void*)c->stream : nullptr; }

int rsd_alloc(rsd_ctx* c, size_t bytes, void** dptr) {
	if (!c || !dptr) return set_error(RSD_EINVAL, "null argument");
	RSD_CUDA(cudaSetDevice(c->device));
	*dptr = nullptr;
	RSD_CUDA(cudaMalloc(dptr, bytes ? bytes : 1));
	return RSD_OK;
}

int rsd_alloc_managed(rsd_ctx* c, size_t bytes, void** dptr) {
	if (!c || !dptr) return set_error(RSD_EINVAL, "null argument");
	RSD_CUDA(cudaSetDevice(c->device));
	RSD_CUDA(cudaMallocManaged(dptr, std::max<size_t>(bytes, 1), cudaMemAttachGlobal));
	// resident on the device: kernels read it at full speed; host reads map or migrate pages on demand
	if (cudaMemAdvise(*dptr, std::max<size_t>(bytes, 1), cudaMemAdviseSetPreferredLocation, c->device) != cudaSuccess) cudaGetLastError();
	return RSD_OK;
}

int rsd_free(rsd_ctx* c, void* dptr) {
	if (!c) return set_error(RSD_EINVAL, "null context");
	if (dptr) {
		RSD_CUDA(cudaStreamSynchronize(c->stream));
		RSD_CUDA(cudaFree(dptr));
	}
	return RSD_OK;
}

int rsd_memcpy(rsd_ctx* c, void* dst, const void* src, size_t bytes, int32_t kind) {
	if (!c) return set_error(RSD_EINVAL, "null context");
	if (bytes == 0) return RSD_OK;
	if (kind == RSD_H2H) { std::memmove(dst, src, bytes); return RSD_OK; }
	cudaMemcpyKind k = kind == RSD_H2D ? cudaMemcpyHostToDevice : kind == RSD_D2H ? cudaMemcpyDeviceToHost
	                 : kind == RSD_D2D ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault;
	RSD_CUDA(cudaMemcpyAsync(dst, src, bytes, k, c->stream));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_memset_zero(rsd_ctx* c, void* dptr, size_t bytes) {
	if (!c) return set_error(RSD_EINVAL, "null context");
	RSD_CUDA(cudaMemsetAsync(dptr, 0, bytes, c->stream));
	RSD_CUDA(cudaStreamSynchronize(c->stream));
	return RSD_OK;
}

int rsd_csr_create(rsd_ctx* c, int64_t nrows, int64_t nnz, const int64_t* row_ptr, const int64_t* col_idx,
                   const double* values, rsd_csr** out) {
	if (!c || !out || nrows < 0 || nnz < 0 || !row_ptr || (nnz && !col_idx)) return set_error(RSD_EINVAL, "bad CSR arguments");
	if (nnz > INT32_MAX || nrows > INT32_MAX) return set_error(RSD_EINVAL, "CSR too large for 32-bit indices");
	if (row_ptr[0] != 0 || row_ptr[nrows] != nnz) return set_error(RSD_EINVAL, "rowPtr does not span nnz");
	std::vector<int32_t> rp(nrows + 1), col(nnz);
	for (int64_t i = 0; i <= nrows; ++i) {
		if (i && row_ptr[i] < row_ptr[i - 1]) return set_error(RSD_EINVAL, "rowPtr not monotone");
		rp[i] = (int32_t)row_ptr[i];
	}
	for (int64_t p = 0; p < nnz; ++p) {
		if (col_idx[p] < 0 || col_idx[p] >= nrows) return set_error(RSD_EINVAL, "column index out of range");
		col[p] = (int32_t)col_idx[p];
	}
	RSD_CUDA(cudaSetDevice(c->device));
	return upload_csr(c, nrows, rp, col, values, out);
}

int rsd_csr_destroy(rsd_csr* A) {
	if (!A) return RSD_OK;
	cudaDeviceSynchronize();
	free_csr_arrays(A);
	delete A;
	return RSD_OK;
}

int rsd_csr_info(const rsd_csr* A, int64_t* nrows, int64_t* nnz) {
	if (!A) return set_error(RSD_EINVAL, "null matrix");
	if (nrows) *nrows = A->n;
	if (nnz) *nnz = A->nnz;
	return RSD_OK;
}

int rsd_csr_layout(const rsd_csr* A, int64_t* sell_slots, int64_t* slices, int64_t* stencil_slices) {
	if (!A) return set_error(RSD_EINVAL, "null matrix");
	if (sell_slots) *sell_slots = A->ssize;
	if (slices) *slices = A->nslices;
	if (stencil_slices) *stencil_slices = A->nStencil;
	return RSD_OK;
}

int rsd_csr_mirrored(const rsd_csr* A, int64_t* mirrored_slices, int32_t* active) {
	if (!A) return set_error(RSD_EINVAL, "null matrix");
	if (mirrored_slices) *mirrored_slices = A->nMirrored;
	if (active) *active = (A->format == 0 && A->nMirrored && A->symVersion == A->version && !A->sPerm) ? 1 : 0;
	return RSD_OK;
}

int rsd_csr_values(rsd_ctx* c, rsd_csr* A, double** dvalues) {
	if (!c || !A || !dvalues) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(csr_sync(c, A));
	*dvalues = A->val;
	// the caller may write through the pointer: the CSR layout becomes the current one
	A->sellValid = false;
	A->version++;
	return RSD_OK;
}

int rsd_csr_set_values(rsd_ctx* c, rsd_csr* A, const double* hv) {
	if (!c || !A || !hv) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(rsd_memcpy(c, A->val, hv, sizeof(double) * A->nnz, RSD_H2D));
	A->csrValid = true;
	A->sellValid = false;
	A->version++;
	return RSD_OK;
}

int rsd_csr_get_values(rsd_ctx* c, rsd_csr* A, double* hv) {
	if (!c || !A || !hv) return set_error(RSD_EINVAL, "null argument");
	RSD_CHECK(csr_sync(c, A));
	return rsd_memcpy(c, hv, A->val, sizeof(double) * A->nnz, RSD_D2H);
}

int rsd_csr_get_pattern(rsd_ctx* c, const rsd_csr* A, int64_t* hrp, int64_t* hcol) {
	if (!c || !A) return set_error(RSD_EINVAL, "null argument");
	std::vector<int32_t> rp(A->n + 1), col(A->nnz);
	RSD_CHECK(rsd_memcpy(c, rp.data(), A->rowPtr, sizeof(int32_t) * (A->n + 1), RSD_D2H));
	if (A->nnz) RSD_CHECK(rsd_memcpy(c, col.data(), A->col, sizeof(int32_t) * A->nnz, RSD_D2H));
	if (hrp) for (int64_t i = 0; i <= A->n; ++i) hrp[i] = rp[i];
	if (hcol) for (int64_t p = 0; p < A->nnz; ++p) hcol[p] = col[p];
	return RSD_OK;
}

int rsd_csr_set_launch(rsd_csr* A, int32_t lanes, int32_t block) {
	if (!A) return set_error(RSD_EINVAL, "null matrix");
	if (lanes && (lanes < 1 || lanes > 32 || (lanes & (lanes - 1)))) return set_error(RSD_EINVAL, "lanes per row must be a power of two in 1..32");
	if (block && (block < 64 || block > 512 || (block & (block - 1)))) return set_error(RSD_EINVAL, "block must be a power of two in 64..512");
	A->format = lanes ? 1 : 0;
	A->lanes = lanes;
	A->block = block;
	return RSD_OK;
}

int rsd_mesh_create(rsd_ctx* c, int32_t nsd, int32_t order, int64_t num_nodes, int64_t num_elements,
                    const double* xyz, const int64_t* ien, const int32_t* rng, rsd_mesh** out) {
	if (!c || !out || !xyz || !ien || !rng) return set_error(RSD_EINVAL, "null argument");
	if (nsd != 2 && nsd != 3) return set_error(RSD_EINVAL, "spatial dimension must be 2 or 3");
	if (order < 1 || order > 3) return set_error(RSD_EINVAL, "basis order must be 1..3 (kMaxBasisOrder)");
	int npe = (order + 1) * (order + 1) * (nsd == 3 ? order + 1 : 1);
	if (npe > 32) return set_error(RSD_EINVAL, "elements with more than 32 nodes (Q3 hex) are not supported");
	if (num_nodes <= 0 || num_nodes > INT32_MAX || num_elements <= 0 || num_elements * npe > INT32_MAX)
		return set_error(RSD_EINVAL, "mesh too large for 32-bit connectivity");
	rsd_mesh* m = new rsd_mesh();
	m->nsd = nsd; m->order = order; m->npe = npe; m->nfaces = nsd == 3 ? 6 : 4;
	m->nnodes = num_nodes; m->nelem = num_elements;
	m->h_xyz.assign(xyz, xyz + num_nodes * nsd);
	m->h_ien.resize(num_elements * npe);
	for (int64_t i = 0; i < num_elements * npe; ++i) {
		if (ien[i] < 0 || ien[i] >= num_nodes) { delete m; return set_error(RSD_EINVAL, "connectivity references a missing node"); }
		m->h_ien[i] = (int32_t)ien[i];
	}
	m->h_rng.assign(rng, rng + num_elements * m->nfaces);
	cudaError_t e;
	if ((e = cudaMalloc(&m->xyz, sizeof(double) * m->h_xyz.size())) != cudaSuccess ||
	    (e = cudaMalloc(&m->ien, sizeof(int32_t) * m->h_ien.size())) != cudaSuccess ||
	    (e = cudaMemcpyAsync(m->xyz, m->h_xyz.data(), sizeof(double) * m->h_xyz.size(), cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
	    (e = cudaMemcpyAsync(m->ien, m->h_ien.data(), sizeof(int32_t) * m->h_ien.size(), cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
		cudaFree(m->xyz); cudaFree(m->ien); delete m;
		return cuda_error(e, "mesh upload");
	}
	*out = m;
	return RSD_OK;
}

int rsd_mesh_destroy(rsd_mesh* m) {
	if (!m) return RSD_OK;
	cudaDeviceSynchronize();
	cudaFree(m->xyz);
	cudaFree(m->ien);
	delete m;
	return RSD_OK;
}

}  // extern "C"
