// Test infrastructure, not product code.
//
// C-ABI harness over the reference's own application layer: an UNMODIFIED
// application::heateq::problem::HeatProblem<CPU, equation::HeatEquation<NSD, NSD, Family>>
// (application/heateq/problem/HeatProblem.hpp:34-206, HeatProblem.tpp) built from a HeatConfig
// (application/heateq/config/HeatConfig.hpp) and driven the way HeatDispatcher::run drives it
// (src/application/heateq/HeatDispatcher.cpp): SteadyStage + driver::Steady for a steady
// configuration (NewtonRunner inside the stage when a nonlinear solver is configured), and
// timestepper::dispatchTransientStage (BackwardEulerStage + BackwardEulerRunner) + driver::Transient
// for a transient one.  Every model the configuration selects is the reference's own:
// ConductivityModel (constant, anisotropic tensor, k(T), k(T) times a tensor), SpecificHeatModel
// (constant or cp(T)), ScalarExpression sources / Dirichlet values and VectorExpression fluxes.
//
// The only project-written piece is the expression engine behind <exprtk.hpp> (oracle/exprtk), which
// the reference does not vendor; the mesh comes from the reference's BlockMesh2D/3D generator
// instead of a mesh file, optionally with its boundary tags renumbered.
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "application/heateq/problem/HeatProblem.hpp"
#include "equation/heateq/HeatEquation.hpp"
#include "mesh/generator/BlockMesh2D.hpp"
#include "mesh/generator/BlockMesh3D.hpp"
#include "io/MeshIO.hpp"
#include "solver/driver/Steady.hpp"
#include "solver/driver/Transient.hpp"
#include "solver/stage/SteadyStage.hpp"
#include "solver/timestepper/TimeStepperFactory.hpp"

using namespace residuum;

extern "C" {

// Problem description shared with oracle/__init__.py (ctypes mirror of this layout).
typedef struct refp_desc {
	int32_t nsd, order, nq;
	int32_t nel[3];
	double lo[3], hi[3];
	int32_t tag_map[6];      // block-mesh boundary tag t becomes tag_map[t] (t itself when negative)
	// ConductivityConfig::Type: 0 Constant, 1 Anisotropic, 2 TemperatureDependentIsotropic,
	// 3 TemperatureDependentAnisotropic
	int32_t k_type;
	double k_value;
	double k_tensor[9];      // nsd x nsd, row-major
	const char* k_expr;
	const char* dk_expr;
	double rho;
	int32_t cp_type;         // SpecificHeatConfig::Type: 0 Constant, 1 TemperatureDependent
	double cp_value;
	const char* cp_expr;
	const char* dcp_expr;
	const char* source;      // volumetric source expression f(t, x, y, z)
	const char* initial;     // initial condition expression
	int32_t nbc;             // boundary conditions (at most 16)
	int32_t bc_tag[16];
	int32_t bc_flux[16];     // 0: value (Dirichlet), 1: flux (one expression per spatial component)
	const char* bc_expr[16][3];
	// solver configuration
	int32_t transient;       // DriverConfig::Type: 0 Steady, 1 Transient (Backward Euler, constant step)
	int32_t nonlinear;       // 1: Newton (NonlinearSolverConfig), 0: linear
	double nl_abs, nl_rel;
	int64_t nl_maxit;
	int32_t lin_type;        // 0 CG, 1 GMRES
	int32_t precond;         // 0 Identity, 1 Jacobi
	int32_t op_type;         // 0 CSR, 1 FEM (matrix-free)
	double lin_tol;
	int64_t lin_maxit, krylov;
	double t0, tf, dt;
} refp_desc;

}  // extern "C"

namespace {

namespace hc = application::heateq::config;
namespace sc = solver::config;

thread_local std::string g_err;

hc::HeatConfig make_config(const refp_desc& d) {
	hc::HeatConfig c;
	c.backend.type = sc::BackendConfig::Type::CPU;
	c.discretization.quadrature.xi = c.discretization.quadrature.eta = c.discretization.quadrature.zeta = d.nq;
	auto tensor = [&]() {
		std::vector<std::vector<Real>> t(d.nsd, std::vector<Real>(d.nsd));
		for (int i = 0; i < d.nsd; ++i)
			for (int j = 0; j < d.nsd; ++j) t[i][j] = d.k_tensor[i * d.nsd + j];
		return t;
	};
	switch (d.k_type) {
		case 0: c.conductivity.type = hc::ConductivityConfig::Type::Constant; c.conductivity.value = d.k_value; break;
		case 1: c.conductivity.type = hc::ConductivityConfig::Type::Anisotropic; c.conductivity.tensor = tensor(); break;
		case 2: c.conductivity.type = hc::ConductivityConfig::Type::TemperatureDependentIsotropic; break;
		default: c.conductivity.type = hc::ConductivityConfig::Type::TemperatureDependentAnisotropic; c.conductivity.tensor = tensor(); break;
	}
	if (d.k_expr) c.conductivity.valueExpression = d.k_expr;
	if (d.dk_expr) c.conductivity.gradientExpression = d.dk_expr;
	c.source.type = hc::SourceConfig::Type::VolumetricHeatSource;
	c.source.read.mode = sc::NodalFieldReadConfig::Mode::Expression;
	c.source.read.expression = d.source ? d.source : "0";
	c.initialCondition.read.mode = sc::NodalFieldReadConfig::Mode::Expression;
	c.initialCondition.read.expression = d.initial ? d.initial : "0";
	for (int b = 0; b < d.nbc; ++b) {
		hc::BoundaryConditionConfig bc;
		bc.boundaryID = d.bc_tag[b];
		if (d.bc_flux[b]) {
			bc.type = hc::BoundaryConditionConfig::Type::Flux;
			for (int i = 0; i < d.nsd; ++i) bc.fluxExpression.push_back(d.bc_expr[b][i] ? d.bc_expr[b][i] : "0");
			bc.forms = {hc::BoundaryConditionConfig::Form::FluxBC};
		} else {
			bc.type = hc::BoundaryConditionConfig::Type::Value;
			bc.expression = d.bc_expr[b][0] ? d.bc_expr[b][0] : "0";
			bc.forms = {hc::BoundaryConditionConfig::Form::ValueBC};
		}
		c.boundaryConditions.push_back(bc);
	}
	sc::LinearSolverConfig lin;
	lin.type = d.lin_type ? sc::LinearSolverConfig::Type::GMRES : sc::LinearSolverConfig::Type::CG;
	lin.operatorType = d.op_type ? sc::LinearSolverConfig::OperatorType::FEM : sc::LinearSolverConfig::OperatorType::CSR;
	lin.preconditioner.type = d.precond ? sc::PreconditionerConfig::Type::Jacobi : sc::PreconditionerConfig::Type::Identity;
	lin.tolerance = d.lin_tol;
	lin.maxIterations = (Index)d.lin_maxit;
	if (d.lin_type) { sc::GMRESParams gp; gp.krylovDim = (Index)d.krylov; lin.params = gp; }
	if (d.nonlinear) {
		sc::NonlinearSolverConfig nl;
		nl.type = sc::NonlinearSolverConfig::Type::Newton;
		nl.absoluteTolerance = d.nl_abs;
		nl.relativeTolerance = d.nl_rel;
		nl.maxIterations = (Index)d.nl_maxit;
		nl.linearSolver = lin;
		c.solver.nonlinear = nl;
	} else {
		c.solver.linear = lin;
	}
	c.solver.driver.type = d.transient ? sc::DriverConfig::Type::Transient : sc::DriverConfig::Type::Steady;
	if (d.transient) {
		sc::TimeStepperConfig ts;
		ts.type = sc::TimeStepperConfig::Type::BackwardEuler;
		ts.t0 = d.t0;
		ts.tf = d.tf;
		ts.stepSize.mode = sc::TimeStepSizeConfig::Mode::Constant;
		ts.stepSize.dt = d.dt;
		c.solver.timestepper = ts;
		c.density = hc::ScalarMaterialPropertyConfig{d.rho, "kg/m^3"};
		hc::SpecificHeatConfig cp;
		cp.type = d.cp_type ? hc::SpecificHeatConfig::Type::TemperatureDependent : hc::SpecificHeatConfig::Type::Constant;
		cp.value = d.cp_value;
		if (d.cp_expr) cp.valueExpression = d.cp_expr;
		if (d.dcp_expr) cp.gradientExpression = d.dcp_expr;
		c.specificHeat = cp;
	}
	c.logging.linear.type = c.logging.nonlinear.type = c.logging.timestepper.type = c.logging.driver.type = sc::LoggerConfig::Type::None;
	return c;
}

mesh::Mesh make_mesh(const refp_desc& d) {
	mesh::Mesh m = d.nsd == 2
		? mesh::generator::BlockMesh2D(d.nel[0], d.nel[1], d.lo[0], d.hi[0], d.lo[1], d.hi[1], d.order, d.order).generate()
		: mesh::generator::BlockMesh3D(d.nel[0], d.nel[1], d.nel[2], d.lo[0], d.hi[0], d.lo[1], d.hi[1], d.lo[2], d.hi[2], d.order, d.order, d.order).generate();
	for (auto& t : m.data.rng)
		if (t >= 0 && t < 6 && d.tag_map[t] >= 0) t = d.tag_map[t];
	return m;
}

struct Base {
	virtual ~Base() = default;
	virtual int64_t numFree() = 0;
	virtual int64_t numNodes() = 0;
	virtual void dofmap(int32_t* t2a) = 0;
	virtual void mesh(double* xyz, int32_t* rng) = 0;
	virtual int run(double* U) = 0;
	virtual int64_t nnz() = 0;
	virtual void pattern(int64_t* rp, int64_t* col) = 0;
	virtual void assembleMatrix(int formset, double c, double t, const double* U, const double* Udot, double* val) = 0;
	virtual void assembleVector(int which, double t, const double* U, const double* Udot, double* out) = 0;
};

template <int NSD>
struct Problem final : Base {
	static constexpr auto Fam = NSD == 2 ? mesh::ElementFamily::Quad : mesh::ElementFamily::Hex;
	using Bundle = equation::HeatEquation<NSD, NSD, Fam>;
	using P = application::heateq::problem::HeatProblem<linalg::types::backend::CPU, Bundle>;
	using VecT = typename P::VectorT;
	using MatT = typename P::MatrixT;
	using StateT = typename P::StateVectorT;

	hc::HeatConfig cfg;
	int order = 1;
	std::unique_ptr<P> p;
	mesh::Mesh meshCopy;

	static typename Bundle::Basis basis(int o) {
		if constexpr (NSD == 2) return typename Bundle::Basis(o, o);
		else return typename Bundle::Basis(o, o, o);
	}
	static typename Bundle::QuadratureVolumeType quadVol(int q) {
		if constexpr (NSD == 2) return typename Bundle::QuadratureVolumeType(q, q);
		else return typename Bundle::QuadratureVolumeType(q, q, q);
	}
	static typename Bundle::QuadratureBoundaryType quadBdy(int q) {
		if constexpr (NSD == 2) return typename Bundle::QuadratureBoundaryType(q);
		else return typename Bundle::QuadratureBoundaryType(q, q);
	}

	explicit Problem(const refp_desc& d) : cfg(make_config(d)), order(d.order) {
		mesh::Mesh m = make_mesh(d);
		meshCopy = m;
		p = std::make_unique<P>(cfg, std::move(m), basis(d.order), quadVol(d.nq), quadBdy(d.nq));
	}
	int64_t numFree() override { return (int64_t)p->numFreeDOFs(); }
	int64_t numNodes() override { return (int64_t)meshCopy.data.numNodes; }
	// TopologicalDOF::buildConstraints over the configuration's value (essential) tags, as the
	// HeatProblem constructor builds it (HeatProblem.tpp:70-90, :129): topology -> algebraic map
	void dofmap(int32_t* t2a) override {
		using DirichletT = typename Bundle::template DirichletExpression<utils::expression::ScalarExpression>;
		topology::TopologicalDOF<1> topo(meshCopy, fem::dof::DOFOrdering::Interleaved);
		fem::boundary::EssentialBoundaryRegistry ess;
		for (const auto& bc : cfg.boundaryConditions) {
			if (bc.type != hc::BoundaryConditionConfig::Type::Value) continue;
			auto b = std::shared_ptr<fem::boundary::BoundaryCondition<DirichletT>>(new fem::boundary::BoundaryCondition<DirichletT>{bc.boundaryID, {fem::boundary::BCCategory::Essential}, DirichletT{bc.expression}});
			ess.template registerBC<DirichletT>(b);
		}
		topo.buildConstraints(basis(order), ess);
		for (Index i = 0; i < topo.numGlobalDOFs(); ++i) t2a[i] = (int32_t)topo.getTopoToAlg()[i];
	}
	void mesh(double* xyz, int32_t* rng) override {
		for (size_t i = 0; i < meshCopy.data.xyz.size(); ++i) xyz[i] = meshCopy.data.xyz[i];
		for (size_t i = 0; i < meshCopy.data.rng.size(); ++i) rng[i] = meshCopy.data.rng[i];
	}
	// HeatDispatcher::run (src/application/heateq/HeatDispatcher.cpp): Steady or Transient driver
	int run(double* U) override {
		bool ok;
		if (cfg.solver.driver.type == sc::DriverConfig::Type::Steady) {
			solver::stage::SteadyStage<P> stage(*p);
			solver::driver::Steady<solver::stage::SteadyStage<P>> driver;
			ok = driver.solve(stage);
		} else {
			const auto& ts = *p->solverInstance().timestepper;
			ok = solver::timestepper::dispatchTransientStage(*p, ts, cfg.logging.timestepper, p->equationLabel(), [](auto& stage, auto& stepper) {
				using StageT = std::decay_t<decltype(stage)>;
				solver::driver::Transient<StageT> driver;
				return driver.solve(stage, stepper);
			});
		}
		for (int64_t i = 0; i < numFree(); ++i) U[i] = p->U().data()[i];
		return ok ? 0 : 1;
	}
	std::unique_ptr<MatT> K;
	MatT& matrix() { if (!K) K = std::make_unique<MatT>(p->createMatrix()); return *K; }
	int64_t nnz() override { return (int64_t)matrix().rowPtr()[matrix().nRows()]; }
	void pattern(int64_t* rp, int64_t* col) override {
		MatT& A = matrix();
		for (Index i = 0; i <= A.nRows(); ++i) rp[i] = (int64_t)A.rowPtr()[i];
		for (Index q = 0; q < A.rowPtr()[A.nRows()]; ++q) col[q] = (int64_t)A.colIdx()[q];
	}
	// the stages' compositions (SteadyStage.hpp:37, BackwardEulerStage.hpp:43-46) of the problem's own
	// forms and models: formset 0 K; 1 K + c M; 2 K + K_T; 3 K + K_T + c M + M_T
	template <typename Fn>
	void withForms(int formset, double c, Fn&& fn) {
		using SF = std::decay_t<decltype(p->stiffnessForms())>;
		using MF = std::decay_t<decltype(p->massForms())>;
		using TF = std::decay_t<decltype(p->tangentStiffnessForms())>;
		using TMF = std::decay_t<decltype(p->tangentMassForms())>;
		using Scaled = fem::form::ScaledForm<1, MF>;
		using OpModel = fem::evaluator::ModelRegistry<std::decay_t<decltype(p->stiffnessModel())>, std::decay_t<decltype(p->massModel())>>;
		const OpModel opModel(p->stiffnessModel(), p->massModel());
		switch (formset) {
			case 0: fn(fem::form::FormRegistry<SF>(p->stiffnessForms()), p->stiffnessModel()); break;
			case 1: fn(fem::form::FormRegistry<SF, Scaled>(p->stiffnessForms(), Scaled(c)), opModel); break;
			case 2: fn(fem::form::FormRegistry<SF, TF>(p->stiffnessForms(), p->tangentStiffnessForms()), p->stiffnessModel()); break;
			case 3: fn(fem::form::FormRegistry<SF, TF, Scaled, TMF>(p->stiffnessForms(), p->tangentStiffnessForms(), Scaled(c), p->tangentMassForms()), opModel); break;
			default: throw std::invalid_argument("formset");
		}
	}
	void load(VecT& dst, const double* src) {
		for (int64_t i = 0; i < numFree(); ++i) dst.data()[i] = src ? src[i] : 0.0;
	}
	void assembleMatrix(int formset, double c, double t, const double* U, const double* Udot, double* val) override {
		load(p->U(), U);
		load(p->Udot(), Udot);
		StateT state;
		state.valueSource = &p->U();
		state.rateSource = &p->Udot();
		MatT& A = matrix();
		withForms(formset, c, [&](const auto& forms, const auto& model) { p->assembleMatrix(t, forms, model, state, A); });
		for (Index q = 0; q < A.rowPtr()[A.nRows()]; ++q) val[q] = A.data()[q];
	}
	// which 0: load (assembleLoad) + natural (applyNatural); 1: residual of the stiffness forms at U
	// (assembleResidual); 2: mass forms on Udot (BackwardEulerStage::residualNorm's second term)
	void assembleVector(int which, double t, const double* U, const double* Udot, double* out) override {
		load(p->U(), U);
		load(p->Udot(), Udot);
		const int64_t n = numFree();
		if (which == 0) {
			p->assembleLoad(t);
			p->applyNatural(t);
			for (int64_t i = 0; i < n; ++i) out[i] = p->F().data()[i];
			return;
		}
		VecT V(n);
		StateT state;
		state.valueSource = &p->U();
		state.rateSource = &p->Udot();
		if (which == 1) p->assembleResidual(t, p->stiffnessForms(), p->stiffnessModel(), state, V);
		else p->assembleVector(t, p->massForms(), p->massModel(), state, [](StateT& s) -> Real* { return s.rateBuffer(); }, V);
		for (int64_t i = 0; i < n; ++i) out[i] = V.data()[i];
	}
};

}  // namespace

extern "C" {

const char* refp_last_error(void) { return g_err.c_str(); }

void* refp_create(const refp_desc* d) {
	try {
		if (d->nsd == 2) return static_cast<Base*>(new Problem<2>(*d));
		if (d->nsd == 3) return static_cast<Base*>(new Problem<3>(*d));
		g_err = "nsd must be 2 or 3";
	} catch (const std::exception& e) { g_err = e.what(); }
	return nullptr;
}
void refp_destroy(void* h) { delete static_cast<Base*>(h); }
int64_t refp_num_free(void* h) { return static_cast<Base*>(h)->numFree(); }
int64_t refp_num_nodes(void* h) { return static_cast<Base*>(h)->numNodes(); }
void refp_mesh(void* h, double* xyz, int32_t* rng) { static_cast<Base*>(h)->mesh(xyz, rng); }
void refp_dofmap(void* h, int32_t* t2a) { static_cast<Base*>(h)->dofmap(t2a); }
int refp_run(void* h, double* U) {
	try { return static_cast<Base*>(h)->run(U); } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int64_t refp_nnz(void* h) { return static_cast<Base*>(h)->nnz(); }
void refp_pattern(void* h, int64_t* rp, int64_t* col) { static_cast<Base*>(h)->pattern(rp, col); }
int refp_assemble_matrix(void* h, int formset, double c, double t, const double* U, const double* Udot, double* val) {
	try { static_cast<Base*>(h)->assembleMatrix(formset, c, t, U, Udot, val); return 0; } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
// the reference's block mesh (tags renumbered by the description) written by MeshIO::writeBinary
int refp_write_pmsh(const refp_desc* d, const char* path) {
	try { io::MeshIO::writeBinary(make_mesh(*d), path); return 0; } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int refp_assemble_vector(void* h, int which, double t, const double* U, const double* Udot, double* out) {
	try { static_cast<Base*>(h)->assembleVector(which, t, U, Udot, out); return 0; } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

}  // extern "C"
