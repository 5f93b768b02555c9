// Drop-in check of the heat problem on the B200 backend tag (include/rsd_residuum_heat.hpp): the
// reference's own HeatProblem<CPU, HeatEquation<NSD, NSD, Family>> and rsd::residuum::heat::HeatProblem
// are built from the same HeatConfig and mesh and solved by the same unmodified reference drivers,
// as HeatDispatcher::run drives them (src/application/heateq/HeatDispatcher.cpp): SteadyStage +
// driver::Steady (NewtonRunner inside the stage for a nonlinear solver), and
// timestepper::dispatchTransientStage (BackwardEulerStage + BackwardEulerRunner) + driver::Transient.
// Prints one JSON object: per case both drivers' return values and the largest difference of the
// final states relative to the largest reference value.
//
// Build (needs the Residuum include/ and src/ trees and the built librsd_cuda.so): tests/cpp/build.py
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "rsd_residuum_heat.hpp"

#include "application/heateq/problem/HeatProblem.hpp"
#include "equation/heateq/HeatEquation.hpp"
#include "mesh/generator/BlockMesh2D.hpp"
#include "mesh/generator/BlockMesh3D.hpp"
#include "solver/driver/Steady.hpp"
#include "solver/driver/Transient.hpp"
#include "solver/stage/SteadyStage.hpp"
#include "solver/timestepper/TimeStepperFactory.hpp"

using namespace residuum;
namespace hc = application::heateq::config;
namespace sc = solver::config;

struct Case {
	std::string name;
	int nsd = 3, order = 1;
	int nel[3] = {4, 4, 4};
	std::vector<std::pair<int, int>> retag;   // (block tag, new tag)
	hc::HeatConfig cfg;
	bool referenceSolvers = false;             // the B200 problem's CSR runners: the reference's cg/gmres templates
};

static hc::HeatConfig base(int nq) {
	hc::HeatConfig c;
	c.backend.type = sc::BackendConfig::Type::CPU;
	c.discretization.quadrature.xi = c.discretization.quadrature.eta = c.discretization.quadrature.zeta = nq;
	c.conductivity.type = hc::ConductivityConfig::Type::Constant;
	c.conductivity.value = 1.0;
	c.source.type = hc::SourceConfig::Type::VolumetricHeatSource;
	c.source.read.mode = sc::NodalFieldReadConfig::Mode::Expression;
	c.source.read.expression = "0";
	c.initialCondition.read.mode = sc::NodalFieldReadConfig::Mode::Expression;
	c.initialCondition.read.expression = "0";
	c.logging.linear.type = c.logging.nonlinear.type = c.logging.timestepper.type = c.logging.driver.type = sc::LoggerConfig::Type::None;
	return c;
}
static void value_bc(hc::HeatConfig& c, int tag, const std::string& e) {
	hc::BoundaryConditionConfig bc;
	bc.boundaryID = tag;
	bc.type = hc::BoundaryConditionConfig::Type::Value;
	bc.expression = e;
	bc.forms = {hc::BoundaryConditionConfig::Form::ValueBC};
	c.boundaryConditions.push_back(bc);
}
static void flux_bc(hc::HeatConfig& c, int tag, const std::vector<std::string>& e) {
	hc::BoundaryConditionConfig bc;
	bc.boundaryID = tag;
	bc.type = hc::BoundaryConditionConfig::Type::Flux;
	bc.fluxExpression = e;
	bc.forms = {hc::BoundaryConditionConfig::Form::FluxBC};
	c.boundaryConditions.push_back(bc);
}
static sc::LinearSolverConfig linear(bool gmres, double tol, bool fem = false, Index krylov = 30) {
	sc::LinearSolverConfig l;
	l.type = gmres ? sc::LinearSolverConfig::Type::GMRES : sc::LinearSolverConfig::Type::CG;
	l.operatorType = fem ? sc::LinearSolverConfig::OperatorType::FEM : sc::LinearSolverConfig::OperatorType::CSR;
	l.preconditioner.type = sc::PreconditionerConfig::Type::Jacobi;
	l.tolerance = tol;
	l.maxIterations = 20000;
	if (gmres) { sc::GMRESParams g; g.krylovDim = krylov; l.params = g; }
	return l;
}
static void transient(hc::HeatConfig& c, double dt, int steps, double rho, hc::SpecificHeatConfig cp) {
	c.solver.driver.type = sc::DriverConfig::Type::Transient;
	sc::TimeStepperConfig ts;
	ts.type = sc::TimeStepperConfig::Type::BackwardEuler;
	ts.t0 = 0.0;
	ts.tf = dt * steps;
	ts.stepSize.mode = sc::TimeStepSizeConfig::Mode::Constant;
	ts.stepSize.dt = dt;
	c.solver.timestepper = ts;
	c.density = hc::ScalarMaterialPropertyConfig{rho, "kg/m^3"};
	c.specificHeat = cp;
}
static hc::SpecificHeatConfig cp_const(double v) {
	hc::SpecificHeatConfig s;
	s.type = hc::SpecificHeatConfig::Type::Constant;
	s.value = v;
	return s;
}
static sc::NonlinearSolverConfig newton(const sc::LinearSolverConfig& l) {
	sc::NonlinearSolverConfig n;
	n.type = sc::NonlinearSolverConfig::Type::Newton;
	n.absoluteTolerance = 1e-10;
	n.relativeTolerance = 1e-10;
	n.maxIterations = 30;
	n.linearSolver = l;
	return n;
}

template <int NSD>
static mesh::Mesh make_mesh(const Case& k) {
	mesh::Mesh m = NSD == 2 ? mesh::generator::BlockMesh2D(k.nel[0], k.nel[1], 0, 1, 0, 1, k.order, k.order).generate()
	                        : mesh::generator::BlockMesh3D(k.nel[0], k.nel[1], k.nel[2], 0, 1, 0, 1, 0, 1, k.order, k.order, k.order).generate();
	for (auto& t : m.data.rng)
		for (auto [from, to] : k.retag)
			if (t == from) { t = to; break; }
	return m;
}

// HeatDispatcher::run's driver choice, on any problem type
template <typename P>
static bool drive(P& p, const hc::HeatConfig& cfg) {
	if (cfg.solver.driver.type == sc::DriverConfig::Type::Steady) {
		solver::stage::SteadyStage<P> stage(p);
		solver::driver::Steady<solver::stage::SteadyStage<P>> d;
		return d.solve(stage);
	}
	const auto& ts = *p.solverInstance().timestepper;
	return solver::timestepper::dispatchTransientStage(p, ts, cfg.logging.timestepper, p.equationLabel(), [](auto& stage, auto& stepper) {
		using StageT = std::decay_t<decltype(stage)>;
		solver::driver::Transient<StageT> d;
		return d.solve(stage, stepper);
	});
}

template <int NSD>
static void run(const Case& k, bool last) {
	static_assert(solver::problem::TransientCapableProblem<rsd::residuum::heat::HeatProblem<NSD>>);
	constexpr auto Fam = NSD == 2 ? mesh::ElementFamily::Quad : mesh::ElementFamily::Hex;
	using Bundle = equation::HeatEquation<NSD, NSD, Fam>;
	using CpuP = application::heateq::problem::HeatProblem<linalg::types::backend::CPU, Bundle>;
	const int nq = (int)k.cfg.discretization.quadrature.xi;
	typename Bundle::Basis basis = [&] { if constexpr (NSD == 2) return typename Bundle::Basis(k.order, k.order); else return typename Bundle::Basis(k.order, k.order, k.order); }();
	typename Bundle::QuadratureVolumeType qv = [&] { if constexpr (NSD == 2) return typename Bundle::QuadratureVolumeType(nq, nq); else return typename Bundle::QuadratureVolumeType(nq, nq, nq); }();
	typename Bundle::QuadratureBoundaryType qb = [&] { if constexpr (NSD == 2) return typename Bundle::QuadratureBoundaryType(nq); else return typename Bundle::QuadratureBoundaryType(nq, nq); }();
	CpuP cpu(k.cfg, make_mesh<NSD>(k), basis, qv, qb);
	const bool okCpu = drive(cpu, k.cfg);
	rsd::residuum::heat::HeatProblem<NSD> dev(k.cfg, make_mesh<NSD>(k));
	dev.useReferenceSolvers(k.referenceSolvers);
	const bool okDev = drive(dev, k.cfg);
	const std::vector<double> u = dev.solutionToHost();
	double d = 0.0, m = 0.0;
	const Index n = cpu.numFreeDOFs();
	for (Index i = 0; i < n; ++i) {
		d = std::max(d, std::fabs(u[i] - cpu.U().data()[i]));
		m = std::max(m, std::fabs(cpu.U().data()[i]));
	}
	std::printf("\"%s\": {\"cpu_ok\": %d, \"b200_ok\": %d, \"n\": %zu, \"n_b200\": %zu, \"max_abs\": %.17g, \"rel_diff\": %.3e}%s", k.name.c_str(), (int)okCpu,
	            (int)okDev, (size_t)n, (size_t)dev.numFreeDOFs(), m, d / std::max(m, 1e-300), last ? "" : ", ");
	std::fflush(stdout);
}

int main() {
	std::vector<Case> cases;
	{   // 2D steady, Dirichlet (1-x)(1-y) on every side, unit source
		Case k; k.name = "steady_q1_quad"; k.nsd = 2; k.nel[0] = 16; k.nel[1] = 16;
		k.cfg = base(2);
		k.cfg.source.read.expression = "1";
		for (int t = 0; t < 4; ++t) value_bc(k.cfg, t, "(1-x)*(1-y)");
		k.cfg.solver.linear = linear(false, 1e-10);
		cases.push_back(k);
	}
	{   // the same on the reference's own cg::Solver templates over the tag
		Case k = cases.back(); k.name = "steady_q1_quad_reference_solvers"; k.referenceSolvers = true;
		cases.push_back(k);
	}
	{   // 3D Backward Euler, 5 steps, sine initial condition (Transient driver)
		Case k; k.name = "be_q1_hex"; k.nel[0] = 6; k.nel[1] = 5; k.nel[2] = 4;
		k.cfg = base(2);
		k.cfg.initialCondition.read.expression = "sin(pi*x)*sin(pi*y)*sin(pi*z) + 0.1*x";
		k.cfg.source.read.expression = "1";
		for (int t = 0; t < 6; ++t) value_bc(k.cfg, t, "0");
		k.cfg.solver.linear = linear(false, 1e-10);
		transient(k.cfg, 1e-2, 5, 1.0, cp_const(1.0));
		cases.push_back(k);
	}
	{   // the same with the matrix-free operator
		Case k = cases.back(); k.name = "be_q1_hex_fem";
		k.cfg.solver.linear = linear(false, 1e-10, true);
		cases.push_back(k);
	}
	{   // 3D Q2 Newton, k(T) = 1 + 0.5 T, f = 10, T = 0 / 1 on x = 0 / 1 (GMRES(30) + Jacobi)
		Case k; k.name = "newton_q2_hex"; k.order = 2; k.nel[0] = k.nel[1] = k.nel[2] = 3;
		k.cfg = base(3);
		k.cfg.conductivity.type = hc::ConductivityConfig::Type::TemperatureDependentIsotropic;
		k.cfg.conductivity.valueExpression = "1 + 0.5*T";
		k.cfg.conductivity.gradientExpression = "0.5";
		k.cfg.source.read.expression = "10";
		value_bc(k.cfg, 0, "0");
		value_bc(k.cfg, 1, "1");
		k.cfg.solver.nonlinear = newton(linear(true, 1e-12));
		cases.push_back(k);
	}
	{   // the same Newton with the Jacobian applied matrix-free
		Case k = cases.back(); k.name = "newton_q2_hex_fem";
		k.cfg.solver.nonlinear = newton(linear(true, 1e-12, true));
		cases.push_back(k);
	}
	{   // anisotropic k(T) tensor, cp(T), Backward-Euler Newton (TangentMass active), a renumbered
	    // Dirichlet tag (9), a time-dependent Dirichlet value and a flux boundary
		Case k; k.name = "be_newton_cpT_aniso"; k.nel[0] = 4; k.nel[1] = 4; k.nel[2] = 3;
		k.retag = {{0, 9}};
		k.cfg = base(2);
		k.cfg.conductivity.type = hc::ConductivityConfig::Type::TemperatureDependentAnisotropic;
		k.cfg.conductivity.tensor = {{2.0, 0.3, 0.0}, {0.3, 1.0, 0.1}, {0.0, 0.1, 0.5}};
		k.cfg.conductivity.valueExpression = "1 + 0.2*T";
		k.cfg.conductivity.gradientExpression = "0.2";
		k.cfg.source.read.expression = "1 + x*y";
		k.cfg.initialCondition.read.expression = "x*y + 0.5*z";
		value_bc(k.cfg, 9, "0");
		value_bc(k.cfg, 1, "1 + 2*t");
		flux_bc(k.cfg, 2, {"1 + y", "0.5", "0"});
		hc::SpecificHeatConfig cp;
		cp.type = hc::SpecificHeatConfig::Type::TemperatureDependent;
		cp.valueExpression = "1 + 0.3*T";
		cp.gradientExpression = "0.3";
		k.cfg.solver.nonlinear = newton(linear(true, 1e-12));
		transient(k.cfg, 1e-2, 3, 2.0, cp);
		cases.push_back(k);
	}
	{   // constant anisotropic tensor, steady, CG (symmetric tensor), tag 7 renumbered from 3
		Case k; k.name = "steady_aniso_quad_q2"; k.nsd = 2; k.order = 2; k.nel[0] = 6; k.nel[1] = 5;
		k.retag = {{3, 7}};
		k.cfg = base(3);
		k.cfg.conductivity.type = hc::ConductivityConfig::Type::Anisotropic;
		k.cfg.conductivity.tensor = {{1.5, 0.4}, {0.4, 0.8}};
		k.cfg.source.read.expression = "2 - x";
		value_bc(k.cfg, 0, "x*y");
		value_bc(k.cfg, 7, "1");
		k.cfg.solver.linear = linear(false, 1e-12);
		cases.push_back(k);
	}
	try {
		std::printf("{");
		for (size_t i = 0; i < cases.size(); ++i) {
			const bool last = i + 1 == cases.size();
			if (cases[i].nsd == 2) run<2>(cases[i], last);
			else run<3>(cases[i], last);
		}
		std::printf("}\n");
	} catch (const std::exception& e) {
		std::printf("\"error\": \"%s\"}\n", e.what());
		return 1;
	}
	return 0;
}
