/* Test infrastructure, not product code: the plain-C CPU restatement of the Residuum
 * heat-equation hot path that the CUDA backend is checked against.  Loop orders follow the
 * reference so that sums accumulate in the same order; each function names the reference
 * file:line it restates (paths relative to the reference checkout). */
#include "rsd_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_err[256];
const char* ro_last_error(void) { return g_err; }

/* ============================================================================================
 * expression language (stands in for exprtk at src/utils/expression/ScalarExpression.cpp:3-30
 * and equation/heateq/evaluator/TemperatureExpression.hpp:31-58)
 * ========================================================================================== */
enum { OP_CONST, OP_VAR, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_POW, OP_NEG, OP_FN };
enum { FN_SIN, FN_COS, FN_TAN, FN_EXP, FN_LOG, FN_SQRT, FN_ABS };
typedef struct { int op, arg; double c; } ro_tok;
typedef struct { ro_tok t[256]; int n; } ro_prog;
typedef struct { const char* s; int pos; int err; ro_prog* p; } ro_parser;

static void emit(ro_parser* P, int op, int arg, double c) {
	if (P->p->n >= 256) { P->err = 1; return; }
	P->p->t[P->p->n].op = op; P->p->t[P->p->n].arg = arg; P->p->t[P->p->n].c = c; P->p->n++;
}
static void skip(ro_parser* P) { while (P->s[P->pos] && isspace((unsigned char)P->s[P->pos])) P->pos++; }
static void p_expr(ro_parser* P);
static void p_unary(ro_parser* P);
static void p_primary(ro_parser* P) {
	skip(P);
	const char* s = P->s + P->pos;
	if (*s == '(') { P->pos++; p_expr(P); skip(P); if (P->s[P->pos] != ')') { P->err = 1; return; } P->pos++; return; }
	if (isdigit((unsigned char)*s) || *s == '.') {
		char* end; double v = strtod(s, &end);
		if (end == s) { P->err = 1; return; }
		P->pos += (int)(end - s); emit(P, OP_CONST, 0, v); return;
	}
	if (isalpha((unsigned char)*s) || *s == '_') {
		char name[32]; int k = 0;
		while ((isalnum((unsigned char)s[k]) || s[k] == '_') && k < 31) { name[k] = s[k]; k++; }
		name[k] = 0; P->pos += k;
		if (!strcmp(name, "t")) { emit(P, OP_VAR, 0, 0); return; }
		if (!strcmp(name, "x")) { emit(P, OP_VAR, 1, 0); return; }
		if (!strcmp(name, "y")) { emit(P, OP_VAR, 2, 0); return; }
		if (!strcmp(name, "z")) { emit(P, OP_VAR, 3, 0); return; }
		if (!strcmp(name, "T")) { emit(P, OP_VAR, 4, 0); return; }
		if (!strcmp(name, "pi")) { emit(P, OP_CONST, 0, 3.14159265358979323846); return; }
		static const char* fns[] = {"sin", "cos", "tan", "exp", "log", "sqrt", "abs"};
		for (int f = 0; f < 7; ++f) if (!strcmp(name, fns[f])) {
			skip(P); if (P->s[P->pos] != '(') { P->err = 1; return; }
			P->pos++; p_expr(P); skip(P);
			if (P->s[P->pos] != ')') { P->err = 1; return; }
			P->pos++; emit(P, OP_FN, f, 0); return;
		}
	}
	P->err = 1;
}
static void p_power(ro_parser* P) {
	p_primary(P); skip(P);
	if (P->s[P->pos] == '^') { P->pos++; p_unary(P); emit(P, OP_POW, 0, 0); }
}
static void p_unary(ro_parser* P) {
	skip(P);
	if (P->s[P->pos] == '-') { P->pos++; p_unary(P); emit(P, OP_NEG, 0, 0); return; }
	if (P->s[P->pos] == '+') { P->pos++; p_unary(P); return; }
	p_power(P);
}
static void p_term(ro_parser* P) {
	p_unary(P);
	for (;;) {
		skip(P); char c = P->s[P->pos];
		if (c != '*' && c != '/') return;
		P->pos++; p_unary(P); emit(P, c == '*' ? OP_MUL : OP_DIV, 0, 0);
	}
}
static void p_expr(ro_parser* P) {
	p_term(P);
	for (;;) {
		skip(P); char c = P->s[P->pos];
		if (c != '+' && c != '-') return;
		P->pos++; p_term(P); emit(P, c == '+' ? OP_ADD : OP_SUB, 0, 0);
	}
}
static int compile_expr(const char* src, ro_prog* prog) {
	ro_parser P = {src, 0, 0, prog};
	prog->n = 0;
	p_expr(&P); skip(&P);
	if (P.err || P.s[P.pos] != 0 || prog->n == 0) { snprintf(g_err, sizeof g_err, "cannot parse expression '%s'", src); return -1; }
	return 0;
}
static double run_expr(const ro_prog* p, double t, double x, double y, double z, double T) {
	double st[64]; int sp = 0; const double v[5] = {t, x, y, z, T};
	for (int i = 0; i < p->n; ++i) {
		const ro_tok* k = &p->t[i];
		switch (k->op) {
			case OP_CONST: st[sp++] = k->c; break;
			case OP_VAR: st[sp++] = v[k->arg]; break;
			case OP_ADD: sp--; st[sp - 1] = st[sp - 1] + st[sp]; break;
			case OP_SUB: sp--; st[sp - 1] = st[sp - 1] - st[sp]; break;
			case OP_MUL: sp--; st[sp - 1] = st[sp - 1] * st[sp]; break;
			case OP_DIV: sp--; st[sp - 1] = st[sp - 1] / st[sp]; break;
			case OP_POW: sp--; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
			case OP_NEG: st[sp - 1] = -st[sp - 1]; break;
			case OP_FN: {
				double a = st[sp - 1], r = 0;
				switch (k->arg) { case FN_SIN: r = sin(a); break; case FN_COS: r = cos(a); break; case FN_TAN: r = tan(a); break;
					case FN_EXP: r = exp(a); break; case FN_LOG: r = log(a); break; case FN_SQRT: r = sqrt(a); break; default: r = fabs(a); }
				st[sp - 1] = r; break;
			}
		}
	}
	return st[0];
}
int ro_expr_eval(const char* src, double t, double x, double y, double z, double T, double* out) {
	ro_prog p;
	if (compile_expr(src, &p)) return -1;
	*out = run_expr(&p, t, x, y, z, T);
	return 0;
}

/* ============================================================================================
 * mesh generators: src/mesh/generator/BlockMesh2D.cpp:37-117, BlockMesh3D.cpp:26-139
 * ========================================================================================== */
int ro_mesh_block(int32_t nsd, const int32_t* nel, const double* lo, const double* hi, int32_t order, ro_mesh* m) {
	memset(m, 0, sizeof *m);
	if ((nsd != 2 && nsd != 3) || order < 1 || order > 3) { snprintf(g_err, sizeof g_err, "bad mesh"); return -1; }
	const int64_t nx = nel[0], ny = nel[1], nz = nsd == 3 ? nel[2] : 1;
	const int64_t p = order;
	const int64_t NX = nx * p + 1, NY = ny * p + 1, NZ = nsd == 3 ? nz * p + 1 : 1;
	m->nsd = nsd; m->order = order;
	m->npe = (int32_t)((p + 1) * (p + 1) * (nsd == 3 ? p + 1 : 1));
	m->nfaces = nsd == 3 ? 6 : 4;
	m->nnodes = NX * NY * NZ;
	m->nelem = nx * ny * nz;
	m->xyz = malloc(sizeof(double) * m->nnodes * nsd);
	m->ien = malloc(sizeof(int64_t) * m->nelem * m->npe);
	m->rng = malloc(sizeof(int32_t) * m->nelem * m->nfaces);
	const double dx = (hi[0] - lo[0]) / (double)(nx * p);
	const double dy = (hi[1] - lo[1]) / (double)(ny * p);
	const double dz = nsd == 3 ? (hi[2] - lo[2]) / (double)(nz * p) : 0.0;
	int64_t node = 0;
	for (int64_t k = 0; k < NZ; ++k)
		for (int64_t j = 0; j < NY; ++j)
			for (int64_t i = 0; i < NX; ++i, ++node) {
				m->xyz[nsd * node] = lo[0] + (double)i * dx;
				m->xyz[nsd * node + 1] = lo[1] + (double)j * dy;
				if (nsd == 3) m->xyz[nsd * node + 2] = lo[2] + (double)k * dz;
			}
	for (int64_t ez = 0; ez < nz; ++ez)
		for (int64_t ey = 0; ey < ny; ++ey)
			for (int64_t ex = 0; ex < nx; ++ex) {
				const int64_t e = ez * nx * ny + ey * nx + ex;
				for (int64_t a = 0; a < m->npe; ++a) {
					const int64_t ax = a % (p + 1), ay = (a / (p + 1)) % (p + 1), az = a / ((p + 1) * (p + 1));
					m->ien[e * m->npe + a] = (ez * p + az) * NY * NX + (ey * p + ay) * NX + (ex * p + ax);
				}
				int32_t* r = m->rng + e * m->nfaces;
				if (nsd == 2) {
					r[0] = ex == 0 ? 0 : -1; r[1] = ex == nx - 1 ? 1 : -1;
					r[2] = ey == 0 ? 2 : -1; r[3] = ey == ny - 1 ? 3 : -1;
				} else {
					r[0] = ex == 0 ? 0 : -1; r[1] = ex == nx - 1 ? 1 : -1;
					r[2] = ey == 0 ? 2 : -1; r[3] = ey == ny - 1 ? 3 : -1;
					r[4] = ez == 0 ? 4 : -1; r[5] = ez == nz - 1 ? 5 : -1;
				}
			}
	return 0;
}
void ro_mesh_free(ro_mesh* m) { free(m->xyz); free(m->ien); free(m->rng); memset(m, 0, sizeof *m); }

/* ============================================================================================
 * basis and quadrature
 * ========================================================================================== */
/* Lagrange1D::eval / evalFirstDerivative (fem/basis/Lagrange1D.tpp:4-51) */
static void lag1d(int p, double xi, double* N, double* dN) {
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
/* GaussQuadrature1D points/weights (fem/quadrature/GaussQuadrature1D.tpp:4-71): the standard
 * Gauss-Legendre nodes, at the same decimal precision as the reference table */
static void gauss1d(int n, double* xi, double* w) {
	static const double X[6][5] = {{0}, {0.0}, {-0.5773502691896257, 0.5773502691896257},
		{-0.7745966692414834, 0.0, 0.7745966692414834},
		{-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526},
		{-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640}};
	static const double W[6][5] = {{0}, {2.0}, {1.0, 1.0}, {0.5555555555555556, 0.8888888888888889, 0.5555555555555556},
		{0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538},
		{0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665, 0.2369268850561891}};
	for (int i = 0; i < n; ++i) { xi[i] = X[n][i]; w[i] = W[n][i]; }
}

#define RO_MAXN 64
#define RO_MAXQ 125

struct ro_problem {
	const ro_mesh* m;
	ro_model model;
	ro_prog kP, dkP, srcP, bcP[6];
	int hasK, hasDK, hasSrc, hasBC[6];
	double* kElem;
	int32_t* t2a; int32_t* a2t; int32_t* ctag;
	int64_t n, nnz;
	int64_t* rowPtr; int64_t* col;
	int nq;                    /* total quadrature points */
	double N[RO_MAXQ][RO_MAXN], dNdxi[RO_MAXQ][RO_MAXN * 3], qxi[RO_MAXQ][3], qw[RO_MAXQ];
	double time;
	double* g;                 /* Dirichlet value per node at the current time (constrained nodes) */
	int32_t opType;            /* LinearSolverConfig::OperatorType of the stages: 0 CSR, 1 FEM */
	ro_prog fluxP[6][3];       /* flux boundary conditions: per tag, one expression per component */
	int hasFlux[6];
};

int64_t ro_num_free(const ro_problem* p) { return p->n; }
int64_t ro_nnz(const ro_problem* p) { return p->nnz; }

/* LagrangeQuad / LagrangeHex getFaceNodes (fem/basis/LagrangeQuad.tpp:136-155,
 * fem/basis/LagrangeHex.tpp:263-304) */
static int face_nodes(int nsd, int p, int f, int64_t* out) {
	const int q = p + 1; int k = 0;
	if (nsd == 2) {
		for (int i = 0; i < q; ++i) out[k++] = f == 0 ? i * q : f == 1 ? i * q + p : f == 2 ? i : i + q * p;
		return k;
	}
	for (int j = 0; j < q; ++j)
		for (int i = 0; i < q; ++i) {
			int64_t v;
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

/* TopologicalDOF::buildConstraints, Interleaved ordering (topology/TopologicalDOF.tpp:34-111) */
static void build_dofmap(ro_problem* P) {
	const ro_mesh* m = P->m;
	for (int64_t i = 0; i < m->nnodes; ++i) { P->t2a[i] = 0; P->ctag[i] = -1; }
	int64_t fn[RO_MAXN];
	for (int64_t e = 0; e < m->nelem; ++e)
		for (int f = 0; f < m->nfaces; ++f) {
			const int32_t tag = m->rng[e * m->nfaces + f];
			if (tag < 0) continue;
			const int npf = face_nodes(m->nsd, m->order, f, fn);
			for (int i = 0; i < npf; ++i) {
				const int64_t node = m->ien[e * m->npe + fn[i]];
				if (tag > 5 || !P->hasBC[tag]) continue;
				P->t2a[node] = -1;       /* constrainedSet.insert */
				P->ctag[node] = tag;     /* constraintTags_[dof] = tag (last writer wins) */
			}
		}
	int64_t alg = 0;
	for (int64_t i = 0; i < m->nnodes; ++i) {
		if (P->t2a[i] == -1) continue;
		P->t2a[i] = (int32_t)alg; P->a2t[alg] = (int32_t)i; ++alg;
	}
	P->n = alg;
}

static int cmp_i64(const void* a, const void* b) { int64_t x = *(const int64_t*)a, y = *(const int64_t*)b; return (x > y) - (x < y); }

/* Assembler<CPU>::createMatrix (fem/assembly/backend/cpu/Assembler.tpp:8-76) */
static void build_pattern(ro_problem* P) {
	const ro_mesh* m = P->m;
	const int64_t n = P->n;
	int64_t* off = calloc(n + 1, sizeof(int64_t));
	for (int64_t e = 0; e < m->nelem; ++e) {
		const int64_t* nodes = m->ien + e * m->npe;
		for (int i = 0; i < m->npe; ++i) {
			const int32_t r = P->t2a[nodes[i]]; if (r < 0) continue;
			for (int k = 0; k < m->npe; ++k) if (P->t2a[nodes[k]] >= 0) off[r + 1]++;
		}
	}
	for (int64_t i = 0; i < n; ++i) off[i + 1] += off[i];
	int64_t* raw = malloc(sizeof(int64_t) * (off[n] ? off[n] : 1));
	int64_t* cur = malloc(sizeof(int64_t) * (n ? n : 1));
	memcpy(cur, off, sizeof(int64_t) * n);
	for (int64_t e = 0; e < m->nelem; ++e) {
		const int64_t* nodes = m->ien + e * m->npe;
		for (int i = 0; i < m->npe; ++i) {
			const int32_t r = P->t2a[nodes[i]]; if (r < 0) continue;
			for (int k = 0; k < m->npe; ++k) { const int32_t c = P->t2a[nodes[k]]; if (c >= 0) raw[cur[r]++] = c; }
		}
	}
	P->rowPtr = malloc(sizeof(int64_t) * (n + 1));
	P->rowPtr[0] = 0;
	for (int64_t i = 0; i < n; ++i) {
		int64_t* b = raw + off[i]; int64_t len = off[i + 1] - off[i];
		qsort(b, (size_t)len, sizeof(int64_t), cmp_i64);
		int64_t u = 0;
		for (int64_t j = 0; j < len; ++j) if (j == 0 || b[j] != b[u - 1]) b[u++] = b[j];
		P->rowPtr[i + 1] = P->rowPtr[i] + u;
	}
	P->nnz = P->rowPtr[n];
	P->col = malloc(sizeof(int64_t) * (P->nnz ? P->nnz : 1));
	for (int64_t i = 0; i < n; ++i) memcpy(P->col + P->rowPtr[i], raw + off[i], sizeof(int64_t) * (P->rowPtr[i + 1] - P->rowPtr[i]));
	free(raw); free(cur); free(off);
}

void ro_set_time(ro_problem* P, double t) {
	const ro_mesh* m = P->m;
	P->time = t;
	for (int64_t i = 0; i < m->nnodes; ++i) {
		P->g[i] = 0.0;
		if (P->t2a[i] >= 0) continue;
		const double* x = m->xyz + m->nsd * i;
		P->g[i] = run_expr(&P->bcP[P->ctag[i]], t, x[0], x[1], m->nsd == 3 ? x[2] : 0.0, 0.0);
	}
}
void ro_bc_node_values(const ro_problem* P, double* g) { memcpy(g, P->g, sizeof(double) * P->m->nnodes); }

ro_problem* ro_problem_create(const ro_mesh* m, const ro_model* model) {
	ro_problem* P = calloc(1, sizeof(ro_problem));
	P->m = m; P->model = *model;
	if (model->k_expr) { if (compile_expr(model->k_expr, &P->kP)) goto fail; P->hasK = 1; }
	if (model->dk_expr) { if (compile_expr(model->dk_expr, &P->dkP)) goto fail; P->hasDK = 1; }
	if (model->src_expr) { if (compile_expr(model->src_expr, &P->srcP)) goto fail; P->hasSrc = 1; }
	for (int t = 0; t < 6; ++t) if (model->bc_expr[t]) { if (compile_expr(model->bc_expr[t], &P->bcP[t])) goto fail; P->hasBC[t] = 1; }
	if (model->k_elem) { P->kElem = malloc(sizeof(double) * m->nelem); memcpy(P->kElem, model->k_elem, sizeof(double) * m->nelem); }
	P->model.k_elem = P->kElem;
	P->t2a = malloc(sizeof(int32_t) * m->nnodes); P->a2t = malloc(sizeof(int32_t) * m->nnodes);
	P->ctag = malloc(sizeof(int32_t) * m->nnodes); P->g = malloc(sizeof(double) * m->nnodes);
	build_dofmap(P);
	build_pattern(P);
	/* tensor-product tables: GaussQuadratureQuad/Hex::getPoints (x fastest) and
	 * LagrangeQuad/Hex::eval/evalGradient (fem/basis/LagrangeHex.tpp:4-55) */
	const int nd = m->nsd, q1 = model->nq, p = m->order;
	double gx[5], gw[5]; gauss1d(q1, gx, gw);
	int q = 0;
	for (int k = 0; k < (nd == 3 ? q1 : 1); ++k)
		for (int j = 0; j < q1; ++j)
			for (int i = 0; i < q1; ++i, ++q) {
				P->qxi[q][0] = gx[i]; P->qxi[q][1] = gx[j]; P->qxi[q][2] = nd == 3 ? gx[k] : 0.0;
				P->qw[q] = nd == 3 ? gw[i] * gw[j] * gw[k] : gw[i] * gw[j];
				double Nx[4], Ny[4], Nz[4], dx[4], dy[4], dz[4];
				lag1d(p, P->qxi[q][0], Nx, dx); lag1d(p, P->qxi[q][1], Ny, dy);
				if (nd == 3) lag1d(p, P->qxi[q][2], Nz, dz);
				int a = 0;
				for (int c = 0; c < (nd == 3 ? p + 1 : 1); ++c)
					for (int b = 0; b <= p; ++b)
						for (int aa = 0; aa <= p; ++aa, ++a) {
							if (nd == 2) {
								P->N[q][a] = Nx[aa] * Ny[b];
								P->dNdxi[q][a * 2] = dx[aa] * Ny[b]; P->dNdxi[q][a * 2 + 1] = Nx[aa] * dy[b];
							} else {
								P->N[q][a] = Nx[aa] * Ny[b] * Nz[c];
								P->dNdxi[q][a * 3] = dx[aa] * Ny[b] * Nz[c];
								P->dNdxi[q][a * 3 + 1] = Nx[aa] * dy[b] * Nz[c];
								P->dNdxi[q][a * 3 + 2] = Nx[aa] * Ny[b] * dz[c];
							}
						}
			}
	P->nq = q;
	ro_set_time(P, 0.0);
	return P;
fail:
	free(P);
	return NULL;
}

void ro_problem_destroy(ro_problem* P) {
	if (!P) return;
	free(P->kElem); free(P->t2a); free(P->a2t); free(P->ctag); free(P->g); free(P->rowPtr); free(P->col); free(P);
}
void ro_dofmap(const ro_problem* P, int32_t* t2a, int32_t* a2t, int32_t* ctag) {
	if (t2a) memcpy(t2a, P->t2a, sizeof(int32_t) * P->m->nnodes);
	if (a2t) memcpy(a2t, P->a2t, sizeof(int32_t) * P->n);
	if (ctag) memcpy(ctag, P->ctag, sizeof(int32_t) * P->m->nnodes);
}
void ro_pattern(const ro_problem* P, int64_t* rowPtr, int64_t* col) {
	memcpy(rowPtr, P->rowPtr, sizeof(int64_t) * (P->n + 1));
	memcpy(col, P->col, sizeof(int64_t) * P->nnz);
}

/* ============================================================================================
 * quadrature-point evaluation: EvalQuadraturePointVolume::evaluate
 * (equation/heateq/evaluator/EvalQuadraturePointVolume.hpp:64-85) over JacobianTransform
 * (fem/geometry/JacobianTransform.tpp:4-234, including the 2D J^-1 / 3D cofactor layout)
 * ========================================================================================== */
typedef struct {
	double x[3], N[RO_MAXN], dNdx[RO_MAXN * 3], measure, w;
	double T, Tdot, gradT[3], k, dk, rho, cp;
} ro_qp;

static void qp_eval(const ro_problem* P, int q, const double* coords, ro_qp* Q) {
	const int S = P->m->nsd, npe = P->m->npe;
	const double* dNdxi = P->dNdxi[q];
	double J[9], g[9], inv[9];
	for (int i = 0; i < S; ++i) Q->x[i] = 0.0;
	for (int a = 0; a < npe; ++a) for (int i = 0; i < S; ++i) Q->x[i] += P->N[q][a] * coords[a * S + i];
	for (int i = 0; i < S * S; ++i) J[i] = 0.0;
	for (int i = 0; i < S; ++i) for (int al = 0; al < S; ++al) for (int a = 0; a < npe; ++a) J[i * S + al] += dNdxi[a * S + al] * coords[a * S + i];
	for (int be = 0; be < S; ++be) for (int al = 0; al < S; ++al) {
		double s = 0.0;
		for (int i = 0; i < S; ++i) s += J[i * S + al] * J[i * S + be];
		g[be * S + al] = s; g[al * S + be] = s;
	}
	double detg, detJ;
	if (S == 2) {
		detg = (g[0] * g[3]) - (g[1] * g[2]);
		detJ = (J[0] * J[3]) - (J[1] * J[2]);
		const double di = 1.0 / detJ;
		inv[0] = di * J[3]; inv[1] = -di * J[1]; inv[2] = -di * J[2]; inv[3] = di * J[0];
	} else {
		detg = (g[0] * ((g[4] * g[8]) - (g[5] * g[7]))) - (g[1] * ((g[3] * g[8]) - (g[5] * g[6]))) + (g[2] * ((g[3] * g[7]) - (g[4] * g[6])));
		detJ = (J[0] * ((J[4] * J[8]) - (J[5] * J[7]))) - (J[1] * ((J[3] * J[8]) - (J[5] * J[6]))) + (J[2] * ((J[3] * J[7]) - (J[4] * J[6])));
		const double di = 1.0 / detJ;
		inv[0] = di * ((J[4] * J[8]) - (J[5] * J[7]));
		inv[1] = -di * ((J[3] * J[8]) - (J[5] * J[6]));
		inv[2] = di * ((J[3] * J[7]) - (J[4] * J[6]));
		inv[3] = -di * ((J[1] * J[8]) - (J[2] * J[7]));
		inv[4] = di * ((J[0] * J[8]) - (J[2] * J[6]));
		inv[5] = -di * ((J[0] * J[7]) - (J[1] * J[6]));
		inv[6] = di * ((J[1] * J[5]) - (J[2] * J[4]));
		inv[7] = -di * ((J[0] * J[5]) - (J[2] * J[3]));
		inv[8] = di * ((J[0] * J[4]) - (J[1] * J[3]));
	}
	Q->measure = sqrt(detg);
	Q->w = P->qw[q];
	for (int a = 0; a < npe; ++a) {
		Q->N[a] = P->N[q][a];
		for (int i = 0; i < S; ++i) {
			double s = 0.0;
			for (int al = 0; al < S; ++al) s += (inv[i * S + al] * dNdxi[a * S + al]);
			Q->dNdx[a * S + i] = s;
		}
	}
}

/* HeatStateVector::interpolate (equation/heateq/evaluator/HeatStateVector.hpp:53-56) and the
 * models: conductivity (ConductivityModel.hpp:60-96), density, specific heat */
static void qp_state(const ro_problem* P, ro_qp* Q, const double* Ue, const double* Re) {
	const int S = P->m->nsd, npe = P->m->npe;
	double u = 0.0, r = 0.0;
	for (int a = 0; a < npe; ++a) u += Q->N[a] * Ue[a];
	for (int i = 0; i < S; ++i) Q->gradT[i] = 0.0;
	for (int a = 0; a < npe; ++a) for (int i = 0; i < S; ++i) Q->gradT[i] += Q->dNdx[a * S + i] * Ue[a];
	for (int a = 0; a < npe; ++a) r += Q->N[a] * Re[a];
	Q->T = u; Q->Tdot = r;
	Q->k = P->hasK ? run_expr(&P->kP, 0, 0, 0, 0, u) : P->model.k_const;
	Q->dk = P->hasDK ? run_expr(&P->dkP, 0, 0, 0, 0, u) : 0.0;
	Q->rho = P->model.rho; Q->cp = P->model.cp;
}

/* gatherElementCoords / gatherElementVector Free|Full|Constrained
 * (fem/assembly/backend/cpu/ElementMap.tpp:4-75); vec NULL gathers zeros for free DOFs */
enum { G_FREE, G_FULL, G_CONSTRAINED };
static void gather(const ro_problem* P, const int64_t* nodes, int mode, const double* vec, const double* g, double* out) {
	for (int a = 0; a < P->m->npe; ++a) {
		const int32_t r = P->t2a[nodes[a]];
		if (r >= 0) out[a] = (mode != G_CONSTRAINED && vec) ? vec[r] : 0.0;
		else out[a] = (mode == G_FREE) ? 0.0 : g[nodes[a]];
	}
}
static void coords_of(const ro_problem* P, const int64_t* nodes, double* c) {
	const int S = P->m->nsd;
	for (int a = 0; a < P->m->npe; ++a) for (int i = 0; i < S; ++i) c[a * S + i] = P->m->xyz[nodes[a] * S + i];
}

/* forms, accumulated into Ke in FormRegistry order: Diffusion (DiffusionForm.hpp:11-31, scaled per
 * element by k_elem), TangentDiffusion (TangentDiffusionForm.hpp:11-56), Mass scaled by cMass
 * (MassForm.hpp:11-27 inside ScaledForm.hpp:21-33), TangentMass (TangentMassForm.hpp:11-27) */
static void element_matrix(const ro_problem* P, int64_t e, double cDiff, double cMass, double cTDiff, double cTMass,
                           const double* Ue, const double* Re, double* Ke) {
	const int S = P->m->nsd, npe = P->m->npe;
	const int64_t* nodes = P->m->ien + e * npe;
	double coords[RO_MAXN * 3];
	coords_of(P, nodes, coords);
	const double ke = P->kElem ? P->kElem[e] : 1.0;
	memset(Ke, 0, sizeof(double) * npe * npe);
	for (int q = 0; q < P->nq; ++q) {
		ro_qp Q; qp_eval(P, q, coords, &Q); qp_state(P, &Q, Ue, Re);
		for (int a = 0; a < npe; ++a) for (int b = 0; b < npe; ++b) {
			double* kab = &Ke[a * npe + b];
			if (cDiff != 0.0) {
				double integ = 0.0;
				for (int i = 0; i < S; ++i) {
					double mv = 0.0;
					for (int j = 0; j < S; ++j) mv += (i == j ? Q.k : 0.0) * Q.dNdx[b * S + j];
					integ += Q.dNdx[a * S + i] * mv;
				}
				const double v = integ * Q.measure * Q.w;
				*kab += (P->kElem ? ke * v : v) * cDiff;
			}
			if (cTDiff != 0.0) {
				double integ = 0.0;
				for (int i = 0; i < S; ++i) {
					double mv = 0.0;
					for (int j = 0; j < S; ++j) mv += (i == j ? Q.dk : 0.0) * Q.gradT[j];
					integ += Q.dNdx[a * S + i] * mv;
				}
				*kab += cTDiff * (integ * Q.N[b] * Q.measure * Q.w);
			}
			if (cMass != 0.0) *kab += cMass * (Q.rho * Q.cp * Q.N[a] * Q.N[b] * Q.measure * Q.w);
			if (cTMass != 0.0) *kab += cTMass * (Q.rho * 0.0 * Q.Tdot * Q.N[a] * Q.N[b] * Q.measure * Q.w);
		}
	}
}

/* Assembler<CPU>::assembleMatrix + scatterElementMatrix (Assembler.tpp:86-140,
 * ElementMap.tpp:115-184): the merge against the row's sorted columns is a lookup here */
static int64_t find_slot(const ro_problem* P, int64_t r, int64_t c) {
	int64_t lo = P->rowPtr[r], hi = P->rowPtr[r + 1];
	while (lo < hi) { int64_t mid = lo + (hi - lo) / 2; if (P->col[mid] == c) return mid; if (P->col[mid] < c) lo = mid + 1; else hi = mid; }
	return -1;
}
void ro_assemble_matrix(ro_problem* P, double cDiff, double cMass, double cTDiff, double cTMass,
                        const double* U, const double* Udot, double* val) {
	const int npe = P->m->npe;
	memset(val, 0, sizeof(double) * P->nnz);
	double Ke[RO_MAXN * RO_MAXN], Ue[RO_MAXN], Re[RO_MAXN];
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		gather(P, nodes, G_FULL, U, P->g, Ue);
		gather(P, nodes, G_FREE, Udot, P->g, Re);
		element_matrix(P, e, cDiff, cMass, cTDiff, cTMass, Ue, Re, Ke);
		for (int a = 0; a < npe; ++a) {
			const int32_t r = P->t2a[nodes[a]]; if (r < 0) continue;
			for (int b = 0; b < npe; ++b) {
				const int32_t c = P->t2a[nodes[b]]; if (c < 0) continue;
				val[find_slot(P, r, c)] += Ke[a * npe + b];
			}
		}
	}
}

/* vector forms at one quadrature point, accumulated into Fe in the reference's order:
 * DiffusionForm::computeElementLevelVector (DiffusionForm.hpp:33-52; buffered and scaled when a
 * per-element conductivity is set), MassForm::computeElementLevelVector (MassForm.hpp:18-27),
 * ScaledForm buffering (fem/form/ScaledForm.hpp:35-50) for the coefficient on the mass term */
static void qp_vector_forms(const ro_problem* P, const ro_qp* Q, int diff, int mass, double massCoef, int massScaled,
                            double ke, const double* V, double* Fe) {
	const int S = P->m->nsd, npe = P->m->npe;
	double buf[RO_MAXN];
	if (diff) {
		if (P->kElem) memset(buf, 0, sizeof(double) * npe);
		for (int a = 0; a < npe; ++a) for (int b = 0; b < npe; ++b) {
			double integ = 0.0;
			for (int i = 0; i < S; ++i) {
				double mv = 0.0;
				for (int j = 0; j < S; ++j) mv += (i == j ? Q->k : 0.0) * Q->dNdx[b * S + j];
				integ += Q->dNdx[a * S + i] * mv;
			}
			const double v = integ * V[b] * Q->measure * Q->w;
			if (P->kElem) buf[a] += v; else Fe[a] += v;
		}
		if (P->kElem) for (int a = 0; a < npe; ++a) Fe[a] += ke * buf[a];
	}
	if (mass) {
		if (massScaled) memset(buf, 0, sizeof(double) * npe);
		for (int a = 0; a < npe; ++a) for (int b = 0; b < npe; ++b) {
			const double m = Q->rho * Q->cp * Q->N[a] * Q->N[b] * V[b] * Q->measure * Q->w;
			if (massScaled) buf[a] += m; else Fe[a] += m;
		}
		if (massScaled) for (int a = 0; a < npe; ++a) Fe[a] += massCoef * buf[a];
	}
}

/* Assembler<CPU>::assembleVector (Assembler.tpp:199-255) for the form/operand pairings the
 * stages use: 0 load (SourceForm.hpp:22-32), 1 DiffusionForm on U (Full gather),
 * 2 rho*cp Mass on U (Full), 3 rho*cp Mass on Udot (Free), 4 Diffusion + coef*Mass on operand (Free) */
void ro_assemble_vector(ro_problem* P, int32_t which, double coef, const double* U, const double* Udot,
                        const double* operand, double* out) {
	const int S = P->m->nsd, npe = P->m->npe;
	memset(out, 0, sizeof(double) * P->n);
	double Ue[RO_MAXN], Re[RO_MAXN], Oe[RO_MAXN], Fe[RO_MAXN], coords[RO_MAXN * 3];
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		gather(P, nodes, G_FULL, U, P->g, Ue);
		gather(P, nodes, G_FREE, Udot, P->g, Re);
		gather(P, nodes, G_FREE, operand, P->g, Oe);
		coords_of(P, nodes, coords);
		const double ke = P->kElem ? P->kElem[e] : 1.0;
		memset(Fe, 0, sizeof Fe);
		for (int q = 0; q < P->nq; ++q) {
			ro_qp Q; qp_eval(P, q, coords, &Q); qp_state(P, &Q, Ue, Re);
			if (which == 0) {
				const double f = P->hasSrc ? run_expr(&P->srcP, P->time, Q.x[0], Q.x[1], S == 3 ? Q.x[2] : 0.0, 0.0) : 0.0;
				for (int a = 0; a < npe; ++a) Fe[a] += (f * Q.N[a]) * Q.measure * Q.w;
			} else if (which == 1) qp_vector_forms(P, &Q, 1, 0, 0.0, 0, ke, Ue, Fe);
			else if (which == 2) qp_vector_forms(P, &Q, 0, 1, 0.0, 0, ke, Ue, Fe);
			else if (which == 3) qp_vector_forms(P, &Q, 0, 1, 0.0, 0, ke, Re, Fe);
			else qp_vector_forms(P, &Q, 1, coef != 0.0, coef, 1, ke, Oe, Fe);
		}
		for (int a = 0; a < npe; ++a) { const int32_t r = P->t2a[nodes[a]]; if (r >= 0) out[r] += Fe[a]; }
	}
}

/* BoundaryApplicator<CPU>::applyEssentialBCs (fem/boundary/backend/cpu/BoundaryApplicator.tpp:7-64):
 * F += -1 * (Diffusion + cMass*Mass)(G_e) over every element, G_e the Dirichlet values at
 * constrained nodes and zero elsewhere.  The reference does not interpolate the state here, so a
 * temperature-dependent k is evaluated at T = 0 in this restatement (the reference reads an
 * unset qp.T; no configuration combines the lift with k(T)).  Elements without constrained
 * nodes add exact zeros and are skipped. */
void ro_lift(ro_problem* P, double cDiff, double cMass, double* F) {
	const int npe = P->m->npe;
	double Ge[RO_MAXN], Z[RO_MAXN] = {0}, Fe[RO_MAXN], coords[RO_MAXN * 3];
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		int any = 0;
		for (int a = 0; a < npe; ++a) any |= (P->t2a[nodes[a]] < 0);
		if (!any) continue;
		gather(P, nodes, G_CONSTRAINED, NULL, P->g, Ge);
		coords_of(P, nodes, coords);
		const double ke = P->kElem ? P->kElem[e] : 1.0;
		memset(Fe, 0, sizeof Fe);
		for (int q = 0; q < P->nq; ++q) {
			ro_qp Q; qp_eval(P, q, coords, &Q); qp_state(P, &Q, Z, Z);
			qp_vector_forms(P, &Q, cDiff != 0.0, cMass != 0.0, cMass, 1, ke, Ge, Fe);
		}
		for (int a = 0; a < npe; ++a) { const int32_t r = P->t2a[nodes[a]]; if (r >= 0) F[r] += -1.0 * Fe[a]; }
	}
}

/* Assembler<CPU>::assembleDiagonal (Assembler.tpp:142-197) */
void ro_diagonal(ro_problem* P, double cDiff, double cMass, const double* U, double* d) {
	const int npe = P->m->npe;
	double Ke[RO_MAXN * RO_MAXN], Ue[RO_MAXN], Z[RO_MAXN] = {0};
	memset(d, 0, sizeof(double) * P->n);
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		gather(P, nodes, G_FULL, U, P->g, Ue);
		element_matrix(P, e, cDiff, cMass, 0.0, 0.0, Ue, Z, Ke);
		for (int a = 0; a < npe; ++a) { const int32_t r = P->t2a[nodes[a]]; if (r >= 0) d[r] += Ke[a * npe + a]; }
	}
}

/* HeatProblem's flux boundary condition, one expression per spatial component
 * (application/heateq/problem/HeatProblem.tpp:98-105); NULL clears the tag */
int ro_set_flux(ro_problem* P, int32_t tag, const char* const* exprs) {
	if (tag < 0 || tag >= 2 * P->m->nsd) { snprintf(g_err, sizeof g_err, "boundary tag out of range"); return 1; }
	if (!exprs) { P->hasFlux[tag] = 0; return 0; }
	for (int d = 0; d < P->m->nsd; ++d) if (compile_expr(exprs[d], &P->fluxP[tag][d])) return 1;
	P->hasFlux[tag] = 1;
	return 0;
}

/* BoundaryApplicator<CPU>::applyNaturalBCs (fem/boundary/backend/cpu/BoundaryApplicator.tpp:66-140)
 * with FluxBoundaryForm (equation/heateq/form/FluxBoundaryForm.hpp:22-34) and the boundary
 * quadrature point of equation/heateq/evaluator/EvalQuadraturePointBoundary.hpp:74-103: for each
 * element face whose tag carries a flux, the face point is mapped into the element
 * (LagrangeQuad/Hex::mapFaceToElement), x and J from all element nodes, n = cof(J) nRef
 * (JacobianTransform::computeBoundaryNormal, nRef = +-e_axis by getFaceTopology), and
 * Fe[a] += (q_i N_a) n_i w over the face nodes (getFaceNodes), w the reference face weight; the
 * face vector is scattered Free with +1. */
void ro_natural(ro_problem* P, double* F) {
	const ro_mesh* m = P->m;
	const int S = m->nsd, p = m->order, q1 = p + 1, npe = m->npe, nf = m->nfaces;
	int any = 0;
	for (int t = 0; t < 6; ++t) any |= P->hasFlux[t];
	if (!any) return;
	int nb = 0;
	for (int i = 1; i <= 5; ++i) if ((int)round(pow((double)P->nq, 1.0 / S)) == i) nb = i;
	double gx[5], gw[5];
	gauss1d(nb, gx, gw);
	double coords[RO_MAXN * 3];
	int64_t fn[RO_MAXN];
	for (int64_t e = 0; e < m->nelem; ++e) {
		const int64_t* nodes = m->ien + e * npe;
		for (int f = 0; f < nf; ++f) {
			const int32_t tag = m->rng[e * nf + f];
			if (tag < 0 || tag >= 6 || !P->hasFlux[tag]) continue;
			coords_of(P, nodes, coords);
			const int npf = face_nodes(S, p, f, fn);
			const int axis = f / 2;
			const double side = (f & 1) ? 1.0 : -1.0;
			double Fe[RO_MAXN];
			memset(Fe, 0, sizeof Fe);
			const int nqf = S == 3 ? nb * nb : nb;
			for (int q = 0; q < nqf; ++q) {
				const int qs = q % nb, qt = q / nb;
				const double w = S == 3 ? gw[qs] * gw[qt] : gw[qs];
				double xi[3] = {0, 0, 0};
				xi[axis] = side;
				int k = 0;
				for (int d = 0; d < S; ++d) if (d != axis) xi[d] = (k++ == 0) ? gx[qs] : gx[qt];
				double Nd[3][4], dNd[3][4];
				for (int d = 0; d < S; ++d) lag1d(p, xi[d], Nd[d], dNd[d]);
				double N[RO_MAXN], x[3] = {0, 0, 0}, J[9] = {0};
				for (int a = 0; a < npe; ++a) {
					const int ix = a % q1, iy = (a / q1) % q1, iz = S == 3 ? a / (q1 * q1) : 0;
					double g[3];
					N[a] = Nd[0][ix] * Nd[1][iy] * (S == 3 ? Nd[2][iz] : 1.0);
					g[0] = dNd[0][ix] * Nd[1][iy] * (S == 3 ? Nd[2][iz] : 1.0);
					g[1] = Nd[0][ix] * dNd[1][iy] * (S == 3 ? Nd[2][iz] : 1.0);
					g[2] = S == 3 ? Nd[0][ix] * Nd[1][iy] * dNd[2][iz] : 0.0;
					for (int i = 0; i < S; ++i) {
						x[i] += N[a] * coords[a * S + i];
						for (int al = 0; al < S; ++al) J[i * S + al] += g[al] * coords[a * S + i];
					}
				}
				double cof[9], nrm[3];
				if (S == 2) { cof[0] = J[3]; cof[1] = -J[2]; cof[2] = -J[1]; cof[3] = J[0]; }
				else {
					cof[0] = (J[4] * J[8] - J[5] * J[7]); cof[1] = -(J[3] * J[8] - J[5] * J[6]); cof[2] = (J[3] * J[7] - J[4] * J[6]);
					cof[3] = -(J[1] * J[8] - J[2] * J[7]); cof[4] = (J[0] * J[8] - J[2] * J[6]); cof[5] = -(J[0] * J[7] - J[1] * J[6]);
					cof[6] = (J[1] * J[5] - J[2] * J[4]); cof[7] = -(J[0] * J[5] - J[2] * J[3]); cof[8] = (J[0] * J[4] - J[1] * J[3]);
				}
				for (int i = 0; i < S; ++i) nrm[i] = cof[i * S + axis] * side;
				double val[3];
				for (int d = 0; d < S; ++d) val[d] = run_expr(&P->fluxP[tag][d], P->time, x[0], x[1], S == 3 ? x[2] : 0.0, 0.0);
				for (int b = 0; b < npf; ++b)
					for (int d = 0; d < S; ++d) Fe[b] += (val[d] * N[fn[b]]) * nrm[d] * w;
			}
			for (int b = 0; b < npf; ++b) { const int32_t r = P->t2a[nodes[fn[b]]]; if (r >= 0) F[r] += Fe[b]; }
		}
	}
}

/* QuantityEvaluator::evaluateNodalField (fem/quantity/backend/cpu/QuantityEvaluator.tpp:205-257) with
 * SimpleAverageRecovery: per element and point, the field value (0: HeatFluxField, -k grad T;
 * 1: ConductivityField, k) is accumulated at every element node with weight N_a * measure * w, and
 * divided by the summed weights; T gathered Full.  out: nnodes * components. */
void ro_nodal_field(ro_problem* P, int32_t field, const double* U, double* out) {
	const int S = P->m->nsd, npe = P->m->npe, nc = field == 0 ? S : 1;
	const int64_t nn = P->m->nnodes;
	double* wsum = calloc((size_t)nn, sizeof(double));
	memset(out, 0, sizeof(double) * nn * nc);
	double Ue[RO_MAXN], Z[RO_MAXN] = {0}, coords[RO_MAXN * 3];
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		gather(P, nodes, G_FULL, U, P->g, Ue);
		coords_of(P, nodes, coords);
		const double ke = P->kElem ? P->kElem[e] : 1.0;
		for (int q = 0; q < P->nq; ++q) {
			ro_qp Q; qp_eval(P, q, coords, &Q); qp_state(P, &Q, Ue, Z);
			const double k = ke * Q.k;
			double val[3];
			if (field == 0) for (int i = 0; i < S; ++i) val[i] = -(k * Q.gradT[i]);
			else val[0] = k;
			for (int a = 0; a < npe; ++a) {
				const double wa = Q.N[a] * Q.measure * Q.w;
				for (int c = 0; c < nc; ++c) out[nodes[a] * nc + c] += wa * val[c];
				wsum[nodes[a]] += wa;
			}
		}
	}
	for (int64_t v = 0; v < nn; ++v) for (int c = 0; c < nc; ++c) out[v * nc + c] /= wsum[v];
	free(wsum);
}

/* adjoint: grad_e = lam_e^T Khat_e T_e with Khat_e the unit-conductivity element stiffness,
 * T_e gathered Full (Dirichlet values), lam_e gathered Free */
void ro_adjoint_gradient(ro_problem* P, const double* T, const double* lam, double* grad) {
	const int npe = P->m->npe;
	double Ke[RO_MAXN * RO_MAXN], Te[RO_MAXN], Le[RO_MAXN], Z[RO_MAXN] = {0};
	double* saved = P->kElem; double kc = P->model.k_const; int hk = P->hasK;
	P->kElem = NULL; P->model.k_const = 1.0; P->hasK = 0;
	for (int64_t e = 0; e < P->m->nelem; ++e) {
		const int64_t* nodes = P->m->ien + e * npe;
		gather(P, nodes, G_FULL, T, P->g, Te);
		gather(P, nodes, G_FREE, lam, P->g, Le);
		element_matrix(P, e, 1.0, 0.0, 0.0, 0.0, Z, Z, Ke);
		double g = 0.0;
		for (int a = 0; a < npe; ++a) for (int b = 0; b < npe; ++b) g += Le[a] * Ke[a * npe + b] * Te[b];
		grad[e] = g;
	}
	P->kElem = saved; P->model.k_const = kc; P->hasK = hk;
}

/* ============================================================================================
 * linear algebra: MatrixOps.tpp:5-23, VectorOps.tpp:7-86, Jacobi.hpp:23-40, CSROperator.hpp:40-45,
 * cg/Solver.tpp:13-119, gmres/Solver.tpp:3-170
 * ========================================================================================== */
void ro_spmv(int64_t n, const int64_t* rowPtr, const int64_t* col, const double* val, const double* x, double* y) {
	for (int64_t i = 0; i < n; ++i) {
		double s = 0.0;
		for (int64_t p = rowPtr[i]; p < rowPtr[i + 1]; ++p) s += val[p] * x[col[p]];
		y[i] = s;
	}
}
static double dot(int64_t n, const double* a, const double* b) { double s = 0.0; for (int64_t i = 0; i < n; ++i) s += a[i] * b[i]; return s; }
static void axpy(int64_t n, double a, const double* x, double* y) { for (int64_t i = 0; i < n; ++i) y[i] += a * x[i]; }

typedef struct { int64_t n; const int64_t* rp; const int64_t* col; const double* val; } ro_csr;
static void jacobi_setup(const ro_csr* A, int precond, double* invD) {
	for (int64_t i = 0; i < A->n; ++i) {
		if (!precond) { invD[i] = 1.0; continue; }
		double d = 0.0;
		int64_t lo = A->rp[i], hi = A->rp[i + 1];
		while (lo < hi) { int64_t mid = lo + (hi - lo) / 2; if (A->col[mid] == i) { d = A->val[mid]; break; } if (A->col[mid] < i) lo = mid + 1; else hi = mid; }
		invD[i] = (fabs(d) > 1e-300) ? 1.0 / d : 1.0;
	}
}
static void prec_apply(int64_t n, int precond, const double* invD, const double* r, double* z) {
	for (int64_t i = 0; i < n; ++i) z[i] = precond ? r[i] * invD[i] : r[i];
}

static int cg_solve(const ro_csr* A, int precond, const double* b, double* x, double tol, int64_t maxit, ro_report* rep) {
	const int64_t n = A->n;
	double* r = malloc(sizeof(double) * n); double* p = malloc(sizeof(double) * n);
	double* Ap = malloc(sizeof(double) * n); double* z = malloc(sizeof(double) * n); double* invD = malloc(sizeof(double) * n);
	jacobi_setup(A, precond, invD);
	ro_spmv(n, A->rp, A->col, A->val, x, Ap);
	for (int64_t i = 0; i < n; ++i) r[i] = b[i];
	axpy(n, -1.0, Ap, r);
	const double res0 = sqrt(dot(n, r, r));
	int ok = 0; int64_t it = 0; double res = res0;
	rep->initialResidual = res0;
	if (res0 / (res0 + 1e-50) < tol) { ok = 1; rep->finalResidual = res0; rep->finalResidualRel = 1.0; goto done; }
	prec_apply(n, precond, invD, r, z);
	memcpy(p, z, sizeof(double) * n);
	double rz = dot(n, r, z);
	for (int64_t k = 1; k < maxit; ++k) {
		ro_spmv(n, A->rp, A->col, A->val, p, Ap);
		const double alpha = rz / dot(n, p, Ap);
		axpy(n, alpha, p, x);
		axpy(n, -alpha, Ap, r);
		res = sqrt(dot(n, r, r));
		const double rel = res / (res0 + 1e-50);
		if (rel < tol) { ok = 1; it = k; rep->finalResidual = res; rep->finalResidualRel = rel; goto done; }
		prec_apply(n, precond, invD, r, z);
		const double rzn = dot(n, r, z);
		const double beta = rzn / rz;
		for (int64_t i = 0; i < n; ++i) p[i] *= beta;
		axpy(n, 1.0, z, p);
		rz = rzn;
	}
	res = sqrt(dot(n, r, r));
	it = maxit; rep->finalResidual = res; rep->finalResidualRel = res / (res0 + 1e-50);
done:
	rep->converged = ok; rep->iterations = it;
	free(r); free(p); free(Ap); free(z); free(invD);
	return ok ? 0 : 1;
}

static int gmres_solve(const ro_csr* A, int precond, const double* b, double* x, double tol, int64_t maxit, int64_t m, ro_report* rep) {
	const int64_t n = A->n;
	double* Q = malloc(sizeof(double) * n * (m + 1));
	double* w = malloc(sizeof(double) * n); double* z = malloc(sizeof(double) * n); double* invD = malloc(sizeof(double) * n);
	double* H = calloc((size_t)((m + 1) * m), sizeof(double));
	double* cs = calloc((size_t)m, sizeof(double)); double* sn = calloc((size_t)m, sizeof(double)); double* g = calloc((size_t)(m + 1), sizeof(double));
	double* y = calloc((size_t)m, sizeof(double));
#define HAT(i, j) H[(j) * (m + 1) + (i)]
	jacobi_setup(A, precond, invD);
	ro_spmv(n, A->rp, A->col, A->val, x, w);
	for (int64_t i = 0; i < n; ++i) Q[i] = b[i];
	axpy(n, -1.0, w, Q);
	const double res0 = sqrt(dot(n, Q, Q));
	rep->initialResidual = res0;
	int ok = 0; int64_t total = 0; double beta = res0;
	if (res0 / (res0 + 1e-50) < tol) { ok = 1; rep->finalResidual = res0; rep->finalResidualRel = 1.0; rep->iterations = 0; goto out; }
	while (total < maxit) {
		for (int64_t i = 0; i < n; ++i) Q[i] *= 1.0 / beta;
		g[0] = beta; for (int64_t i = 1; i <= m; ++i) g[i] = 0.0;
		int64_t mloc = 0; int brk = 0;
		for (int64_t j = 0; j < m; ++j) {
			prec_apply(n, precond, invD, Q + j * n, z);
			ro_spmv(n, A->rp, A->col, A->val, z, w);
			for (int64_t i = 0; i <= j; ++i) { const double h = dot(n, Q + i * n, w); HAT(i, j) = h; axpy(n, -h, Q + i * n, w); }
			const double hn = sqrt(dot(n, w, w));
			++total;
			brk = hn <= 1e-14;
			if (!brk) { memcpy(Q + (j + 1) * n, w, sizeof(double) * n); for (int64_t i = 0; i < n; ++i) Q[(j + 1) * n + i] *= 1.0 / hn; }
			for (int64_t i = 0; i < j; ++i) {
				const double h1 = HAT(i, j), h2 = HAT(i + 1, j);
				HAT(i, j) = cs[i] * h1 + sn[i] * h2;
				HAT(i + 1, j) = -sn[i] * h1 + cs[i] * h2;
			}
			const double hjj = HAT(j, j);
			const double den = sqrt(hjj * hjj + hn * hn);
			if (den <= 1e-14) { cs[j] = 1.0; sn[j] = 0.0; } else { cs[j] = hjj / den; sn[j] = hn / den; }
			HAT(j, j) = cs[j] * hjj + sn[j] * hn;
			const double gj = g[j];
			g[j] = cs[j] * gj; g[j + 1] = -sn[j] * gj;
			mloc = j + 1;
			if (fabs(g[j + 1]) / (res0 + 1e-50) < tol || brk || total >= maxit) break;
		}
		for (int64_t ii = 0; ii < mloc; ++ii) {
			const int64_t i = mloc - 1 - ii;
			double s = g[i];
			for (int64_t k = i + 1; k < mloc; ++k) s -= HAT(i, k) * y[k];
			y[i] = s / HAT(i, i);
		}
		memset(z, 0, sizeof(double) * n);
		for (int64_t i = 0; i < mloc; ++i) axpy(n, y[i], Q + i * n, z);
		prec_apply(n, precond, invD, z, w);
		axpy(n, 1.0, w, x);
		ro_spmv(n, A->rp, A->col, A->val, x, w);
		for (int64_t i = 0; i < n; ++i) Q[i] = b[i];
		axpy(n, -1.0, w, Q);
		beta = sqrt(dot(n, Q, Q));
		const int conv = beta / (res0 + 1e-50) < tol;
		if (conv || brk || total >= maxit) { ok = conv; break; }
	}
	rep->finalResidual = beta; rep->finalResidualRel = beta / (res0 + 1e-50); rep->iterations = total;
out:
	rep->converged = ok;
#undef HAT
	free(Q); free(w); free(z); free(invD); free(H); free(cs); free(sn); free(g); free(y);
	return ok ? 0 : 1;
}

int ro_csr_solve(int32_t solverType, int32_t precond, int64_t n, const int64_t* rowPtr, const int64_t* col,
                 const double* val, const double* b, double* x, double tol, int64_t maxit, int64_t krylov, ro_report* rep) {
	ro_csr A = {n, rowPtr, col, val};
	memset(rep, 0, sizeof *rep);
	return solverType == 0 ? cg_solve(&A, precond, b, x, tol, maxit, rep) : gmres_solve(&A, precond, b, x, tol, maxit, krylov, rep);
}

/* The LinearSolverRunner HeatProblem::makeLinearRunner builds for OperatorType::FEM
 * (application/heateq/problem/HeatProblem.tpp:274-289): cg/Solver.tpp:13-119 over FEMOperator
 * (linalg/operator/FEMOperator.hpp:39-56).  Every product is the element pass of which 4
 * (Diffusion + coef*Mass on the operand, gathered Free) with the state, read through k(T), being the
 * iterate x itself (the stages bind their state to the vector the solver updates); Jacobi::update
 * (preconditioner/Jacobi.hpp:23-33) inverts the element diagonal at the initial x. */
int ro_fem_solve(ro_problem* P, double coef, int32_t precond, const double* b, double* x, double tol, int64_t maxit,
                 ro_report* rep) {
	const int64_t n = P->n;
	memset(rep, 0, sizeof *rep);
	double* r = malloc(sizeof(double) * n); double* p = malloc(sizeof(double) * n);
	double* Ap = malloc(sizeof(double) * n); double* z = malloc(sizeof(double) * n); double* invD = malloc(sizeof(double) * n);
	if (precond) {
		ro_diagonal(P, 1.0, coef, x, invD);
		for (int64_t i = 0; i < n; ++i) invD[i] = (fabs(invD[i]) > 1e-300) ? 1.0 / invD[i] : 1.0;
	} else {
		for (int64_t i = 0; i < n; ++i) invD[i] = 1.0;
	}
	ro_assemble_vector(P, 4, coef, x, NULL, x, Ap);
	for (int64_t i = 0; i < n; ++i) r[i] = b[i];
	axpy(n, -1.0, Ap, r);
	const double res0 = sqrt(dot(n, r, r));
	int ok = 0; int64_t it = 0; double res = res0;
	rep->initialResidual = res0;
	if (res0 / (res0 + 1e-50) < tol) { ok = 1; rep->finalResidual = res0; rep->finalResidualRel = 1.0; goto done; }
	prec_apply(n, precond, invD, r, z);
	memcpy(p, z, sizeof(double) * n);
	double rz = dot(n, r, z);
	for (int64_t k = 1; k < maxit; ++k) {
		ro_assemble_vector(P, 4, coef, x, NULL, p, Ap);
		const double alpha = rz / dot(n, p, Ap);
		axpy(n, alpha, p, x);
		axpy(n, -alpha, Ap, r);
		res = sqrt(dot(n, r, r));
		const double rel = res / (res0 + 1e-50);
		if (rel < tol) { ok = 1; it = k; rep->finalResidual = res; rep->finalResidualRel = rel; goto done; }
		prec_apply(n, precond, invD, r, z);
		const double rzn = dot(n, r, z);
		const double beta = rzn / rz;
		for (int64_t i = 0; i < n; ++i) p[i] *= beta;
		axpy(n, 1.0, z, p);
		rz = rzn;
	}
	res = sqrt(dot(n, r, r));
	it = maxit; rep->finalResidual = res; rep->finalResidualRel = res / (res0 + 1e-50);
done:
	rep->converged = ok; rep->iterations = it;
	free(r); free(p); free(Ap); free(z); free(invD);
	return ok ? 0 : 1;
}

void ro_set_operator(ro_problem* P, int32_t op) { P->opType = op; }

/* ============================================================================================
 * stages
 * ========================================================================================== */
/* SteadyStage linear (solver/stage/SteadyStage.hpp:60-84, HeatProblem.tpp:217-270) */
int ro_steady(ro_problem* P, int32_t solverType, int32_t precond, double tol, int64_t maxit, int64_t krylov, double* U, ro_report* rep) {
	double* val = malloc(sizeof(double) * P->nnz); double* F = malloc(sizeof(double) * P->n);
	if (P->opType && solverType != 0) { free(val); free(F); snprintf(g_err, sizeof g_err, "matrix-free operator: CG only"); return 2; }
	if (!P->opType) ro_assemble_matrix(P, 1.0, 0.0, 0.0, 0.0, U, NULL, val);
	ro_assemble_vector(P, 0, 0.0, U, NULL, NULL, F);
	ro_natural(P, F);
	ro_lift(P, 1.0, 0.0, F);
	int rc = P->opType ? ro_fem_solve(P, 0.0, precond, F, U, tol, maxit, rep)
	                   : ro_csr_solve(solverType, precond, P->n, P->rowPtr, P->col, val, F, U, tol, maxit, krylov, rep);
	free(val); free(F);
	return rc;
}

/* BackwardEulerRunner::step over BackwardEulerStage, linear mode
 * (solver/timestepper/BackwardEuler.hpp:32-70, solver/stage/BackwardEulerStage.hpp:71-124):
 * dt clamped to tf - t, Udot = (U - Uprev)/dt, A = K + M/dt, F = load + (1/dt) M Uprev (Full
 * gather at t - dt) - lift, CG warm-started from U, then the stage's residual norm
 * |F - K U - M Udot| with the Udot of the assemble call */
int ro_backward_euler(ro_problem* P, double dt, int64_t nsteps, int32_t solverType, int32_t precond, double tol,
                      int64_t maxit, int64_t krylov, double* U, double* resPerStep, int64_t* itersPerStep) {
	const int64_t n = P->n;
	double* Uprev = malloc(sizeof(double) * n); double* Udot = malloc(sizeof(double) * n);
	double* F = malloc(sizeof(double) * n); double* ms = malloc(sizeof(double) * n); double* R = malloc(sizeof(double) * n);
	double* val = malloc(sizeof(double) * P->nnz);
	memcpy(Uprev, U, sizeof(double) * n);
	double time = 0.0; const double tf = dt * (double)nsteps;
	int rc = 0;
	if (P->opType && solverType != 0) { snprintf(g_err, sizeof g_err, "matrix-free operator: CG only"); rc = 2; nsteps = 0; }
	for (int64_t s = 0; s < nsteps && !(time >= tf - 1e-9); ++s) {
		double h = dt < tf - time ? dt : tf - time;
		const double t = time + h;
		for (int64_t i = 0; i < n; ++i) Udot[i] = (-1.0 / h) * Uprev[i] + (1.0 / h) * U[i];
		ro_set_time(P, t);
		if (!P->opType) ro_assemble_matrix(P, 1.0, 1.0 / h, 0.0, 0.0, U, Udot, val);
		ro_assemble_vector(P, 0, 0.0, U, Udot, NULL, F);
		ro_set_time(P, t - h);
		ro_assemble_vector(P, 2, 0.0, Uprev, NULL, NULL, ms);
		ro_set_time(P, t);
		axpy(n, 1.0 / h, ms, F);
		ro_natural(P, F);
		ro_lift(P, 1.0, 1.0 / h, F);
		ro_report rep;
		const int src = P->opType ? ro_fem_solve(P, 1.0 / h, precond, F, U, tol, maxit, &rep)
		                          : ro_csr_solve(solverType, precond, n, P->rowPtr, P->col, val, F, U, tol, maxit, krylov, &rep);
		if (src) { rc = 1; break; }
		if (itersPerStep) itersPerStep[s] = rep.iterations;
		ro_assemble_vector(P, 1, 0.0, U, Udot, NULL, R);
		ro_assemble_vector(P, 3, 0.0, U, Udot, NULL, ms);
		axpy(n, 1.0, ms, R);
		for (int64_t i = 0; i < n; ++i) R[i] = -1.0 * R[i] + 1.0 * F[i];
		if (resPerStep) resPerStep[s] = sqrt(dot(n, R, R));
		memcpy(Uprev, U, sizeof(double) * n);
		time += h;
	}
	free(Uprev); free(Udot); free(F); free(ms); free(R); free(val);
	return rc;
}

/* NewtonRunner::solve over SteadyStage nonlinear mode (solver/nonlinear/Newton.hpp:32-83,
 * solver/stage/SteadyStage.hpp:89-116): R = F - K(T) T (Full gather), J = K + K_T, J dU = R, U += dU */
int ro_newton(ro_problem* P, double absTol, double relTol, int64_t maxit, int32_t solverType, int32_t precond,
              double tol, int64_t linMaxit, int64_t krylov, double* U, ro_report* rep) {
	const int64_t n = P->n;
	double* F = malloc(sizeof(double) * n); double* R = malloc(sizeof(double) * n); double* dU = malloc(sizeof(double) * n);
	double* val = malloc(sizeof(double) * P->nnz);
	double res0 = 0.0; int ok = 0;
	memset(rep, 0, sizeof *rep);
	for (int64_t it = 0; it < maxit; ++it) {
		ro_assemble_vector(P, 0, 0.0, U, NULL, NULL, F);
		ro_natural(P, F);
		ro_assemble_vector(P, 1, 0.0, U, NULL, NULL, R);
		for (int64_t i = 0; i < n; ++i) R[i] = -1.0 * R[i] + 1.0 * F[i];
		const double res = sqrt(dot(n, R, R));
		if (it == 0) res0 = res;
		const double rel = res0 > 0.0 ? res / res0 : 0.0;
		if (res < absTol || rel < relTol) {
			ok = 1; rep->iterations = it; rep->initialResidual = res0; rep->finalResidual = res; rep->finalResidualRel = rel;
			break;
		}
		ro_assemble_matrix(P, 1.0, 0.0, 1.0, 0.0, U, NULL, val);
		memset(dU, 0, sizeof(double) * n);
		ro_report lr;
		if (ro_csr_solve(solverType, precond, n, P->rowPtr, P->col, val, R, dU, tol, linMaxit, krylov, &lr)) { ok = 0; rep->iterations = it; goto out; }
		axpy(n, 1.0, dU, U);
		if (it == maxit - 1) rep->iterations = maxit;
	}
out:
	rep->converged = ok;
	free(F); free(R); free(dU); free(val);
	return ok ? 0 : 1;
}
