// Drop-in check of the B200 backend tag: the reference's own cg::Solver and gmres::Solver templates,
// unmodified, instantiated once with the reference's CPU tag and once with rsd::residuum::B200,
// on the same systems.  Prints one JSON object with both runs' reports and the largest relative
// difference of the solutions.
//
// Build (needs the Residuum include/ tree and the built librsd_cuda.so): tests/cpp/build.py
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <optional>
#include <type_traits>
#include <vector>

#include "rsd_residuum.hpp"

#include "linalg/solver/iterative/cg/Solver.hpp"
#include "linalg/solver/iterative/gmres/Solver.hpp"
#include "linalg/solver/preconditioner/Identity.hpp"
#include "utils/logging/core/NullLogger.hpp"

using namespace residuum::linalg;
using CPU = types::backend::CPU;
using B200 = rsd::residuum::B200;

// 2D five-point operator on an N x N grid: -div(k grad u) + c * d/dx u with a variable k;
// c = 0 gives an SPD matrix (CG), c != 0 a nonsymmetric one (GMRES)
static types::CSRMatrix<double, CPU> five_point(Index N, double c) {
	const Index n = N * N;
	types::CSRMatrix<double, CPU> A(n, n);
	std::vector<Index> cols;
	std::vector<double> vals;
	A.rowPtr()[0] = 0;
	for (Index j = 0; j < N; ++j)
		for (Index i = 0; i < N; ++i) {
			const Index r = j * N + i;
			const double k = 1.0 + 0.5 * std::sin(0.37 * (double)i) * std::cos(0.23 * (double)j);
			auto put = [&](Index col, double v) { cols.push_back(col); vals.push_back(v); };
			if (j > 0) put(r - N, -k);
			if (i > 0) put(r - 1, -k - c);
			put(r, 4.0 * k + 0.01);
			if (i + 1 < N) put(r + 1, -k + c);
			if (j + 1 < N) put(r + N, -k);
			A.rowPtr()[r + 1] = cols.size();
		}
	A.resize(cols.size());
	std::copy(cols.begin(), cols.end(), A.colIdx());
	std::copy(vals.begin(), vals.end(), A.data());
	return A;
}

template <typename Vec>
static Vec make_vec(const std::vector<double>& h) {
	Vec v(h.size());
	Vec::backend_type::template copy<double>(v.data(), h.data(), h.size(), types::backend::CopyKind::HostToDevice);
	return v;
}
template <typename Vec>
static std::vector<double> to_host(const Vec& v) {
	std::vector<double> h(v.size());
	Vec::backend_type::template copy<double>(h.data(), v.data(), v.size(), types::backend::CopyKind::DeviceToHost);
	return h;
}

struct Run {
	bool converged;
	Index iterations;
	double res0, res;
	std::vector<double> x;
};

template <typename Backend, bool GMRES>
static Run solve(const types::CSRMatrix<double, CPU>& host, const std::vector<double>& bh) {
	using Vec = types::Vector<double, Backend>;
	using Mat = types::CSRMatrix<double, Backend>;
	using Op = op::CSROperator<Mat>;
	using Prec = solver::preconditioner::Jacobi<Vec>;
	using Log = residuum::utils::logging::NullLogger;
	std::optional<Mat> dev;
	if constexpr (!std::is_same_v<Backend, CPU>) dev.emplace(host);
	const Mat& A = [&]() -> const Mat& {
		if constexpr (std::is_same_v<Backend, CPU>) return host;
		else return *dev;
	}();
	Op op(A);
	Vec b = make_vec<Vec>(bh);
	Vec x(bh.size());
	x.zero();
	Prec M;
	Log log;
	solver::SolverReport<Vec> rep;
	bool ok;
	if constexpr (GMRES) {
		using S = solver::iterative::gmres::Solver<Op, Vec, Prec, Log>;
		typename S::Config cfg;
		cfg.tol = 1e-10; cfg.maxIters = 5000; cfg.krylovDim = 20;
		typename S::Workspace W(bh.size(), cfg.krylovDim);
		ok = S(cfg).solve(rep, log, W, M, op, b, x);
	} else {
		using S = solver::iterative::cg::Solver<Op, Vec, Prec, Log>;
		typename S::Config cfg;
		cfg.tol = 1e-10; cfg.maxIters = 5000;
		typename S::Workspace W(bh.size());
		ok = S(cfg).solve(rep, log, W, M, op, b, x);
	}
	return Run{ok, rep.iterations, rep.initialResidual, rep.finalResidual, to_host(x)};
}

static double rel_diff(const std::vector<double>& a, const std::vector<double>& b) {
	double d = 0.0, m = 0.0;
	for (size_t i = 0; i < a.size(); ++i) { d = std::max(d, std::fabs(a[i] - b[i])); m = std::max(m, std::fabs(b[i])); }
	return d / std::max(m, 1e-300);
}

static void report(const char* name, const Run& c, const Run& g, bool last) {
	std::printf("\"%s\": {\"cpu\": {\"converged\": %d, \"iterations\": %zu, \"res0\": %.17g, \"res\": %.17g}, "
	            "\"b200\": {\"converged\": %d, \"iterations\": %zu, \"res0\": %.17g, \"res\": %.17g}, \"x_rel_diff\": %.3e}%s",
	            name, (int)c.converged, (size_t)c.iterations, c.res0, c.res, (int)g.converged, (size_t)g.iterations, g.res0,
	            g.res, rel_diff(g.x, c.x), last ? "" : ", ");
}

int main() {
	try {
		const Index N = 96;
		std::vector<double> b(N * N);
		for (size_t i = 0; i < b.size(); ++i) b[i] = std::sin(0.001 * (double)(i * i % 9973)) + 0.5;
		auto spd = five_point(N, 0.0);
		auto nsy = five_point(N, 0.3);
		const Run c1 = solve<CPU, false>(spd, b), g1 = solve<B200, false>(spd, b);
		const Run c2 = solve<CPU, true>(nsy, b), g2 = solve<B200, true>(nsy, b);
		std::printf("{");
		report("cg_jacobi", c1, g1, false);
		report("gmres20_jacobi", c2, g2, true);
		std::printf("}\n");
	} catch (const std::exception& e) {
		std::printf("{\"error\": \"%s\"}\n", e.what());
		return 1;
	}
	return 0;
}
