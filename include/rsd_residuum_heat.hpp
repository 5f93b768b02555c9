// rsd_residuum_heat.hpp - the heat problem on the B200 backend tag (C++20): a drop-in for
// residuum::application::heateq::problem::HeatProblem<BackendT, HeatEquation<NSD, NSD, Family>>
// (application/heateq/problem/HeatProblem.hpp:34-206, HeatProblem.tpp).
//
//     using Problem = rsd::residuum::heat::HeatProblem<3>;
//     Problem p(config, std::move(mesh));                    // the reference's own HeatConfig and mesh
//     residuum::solver::stage::SteadyStage<Problem> stage(p);   // unmodified reference stages,
//     residuum::solver::driver::Steady<decltype(stage)> d;      // drivers, runners and Newton
//     d.solve(stage);
//
// The class satisfies the reference's solver::problem::Problem and TransientCapableProblem concepts
// (solver/problem/Problem.hpp:16-50, TransientCapableProblem.hpp:13-25), so SteadyStage,
// BackwardEulerStage, NewtonRunner, BackwardEulerRunner, driver::Steady and driver::Transient run on
// it unchanged.  Its containers are the B200 tag's Vector / CSRMatrix (rsd_residuum.hpp) and every
// assembly, boundary application and linear solve goes to the C ABI (rsd.h):
//
//   * the forms and models it hands out are descriptors: the stages compose them with the
//     reference's own FormRegistry / ScaledForm / ModelRegistry (BackwardEulerStage.hpp:43-46), and
//     the problem reads the composition back by evaluating it once on a probe point, which yields the
//     coefficient of every form (Diffusion, Mass, TangentDiffusion, TangentMass, Source); that
//     selects the device assembly (rsd_assemble_matrix / rsd_assemble_vector / the Dirichlet lift);
//   * the state vector's buffers are tags, so a selector lambda (valueBuffer / rateBuffer /
//     operandBuffer) tells which vector an element form is evaluated against;
//   * makeLinearRunner gives rsd_solve over the stage's matrix (OperatorType::CSR, CG or GMRES,
//     Jacobi or identity, the linear solver configuration's tolerance and limits), or the matrix-free
//     operator over the same form composition (OperatorType::FEM, rsd_heat_solve_fem_forms); with
//     useReferenceSolvers(true) the CSR case instead builds the reference's own makeLinearSolverRunner
//     (cg::Solver / gmres::Solver templates) over CSROperator on the tag.
//
// Configuration coverage (HeatProblem.tpp:4-176): conductivity Constant, Anisotropic,
// TemperatureDependentIsotropic and TemperatureDependentAnisotropic; specific heat Constant or
// TemperatureDependent; expression sources, Dirichlet values (any tag >= 0) and fluxes; the initial
// condition's Expression mode.  Nodal input files (the File modes), field output (writeOutput) and
// monitors are not part of the device path: File modes throw, output and monitors do nothing.
// Errors throw std::runtime_error, as the reference's HeatProblem does.
#pragma once

#include <array>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rsd_residuum.hpp"

#include "application/heateq/config/HeatConfig.hpp"
#include "fem/dispatch/DiscretizationLimits.hpp"
#include "fem/dof/DOFOrdering.hpp"
#include "fem/evaluator/ModelRegistry.hpp"
#include "fem/form/FormRegistry.hpp"
#include "fem/form/ScaledForm.hpp"
#include "linalg/operator/CSROperator.hpp"
#include "linalg/solver/base/LinearSolverRunner.hpp"
#include "mesh/Mesh.hpp"
#include "solver/SolverInstance.hpp"
#include "solver/config/LoggingConfig.hpp"
#include "solver/linear/LinearSolverFactory.hpp"

namespace rsd::residuum::heat {

// ---------------------------------------------------------------------------------------------
// form and model descriptors
// ---------------------------------------------------------------------------------------------

// The probe point the compositions are evaluated on: five "nodes", one slot per form kind.
struct ProbePoint {
	static constexpr Index ParametricDim = 2;
	static constexpr Index SpatialDim = 2;
	Index nodesPerElement() const { return 5; }
};
static_assert(::residuum::fem::dispatch::kMaxNodesPerElement<ProbePoint::ParametricDim> >= 5,
              "the probe's slots must fit ScaledForm's element buffers");

enum FormSlot { kDiffusion = 0, kMass = 1, kTangentDiffusion = 2, kTangentMass = 3, kSource = 4, kSlots = 5 };

// A form that adds 1 to its slot: composed by FormRegistry / ScaledForm, the probe reads back
// sum(coefficient * slot) per kind.
template <int Slot>
struct FormTag {
	template <typename QP>
	void computeElementLevelMatrix(const QP&, Real* Ke) const { Ke[Slot] += Real(1); }
	template <typename QP>
	void computeElementLevelVector(const QP&, const Real*, Real* Oe) const { Oe[Slot] += Real(1); }
};
using DiffusionForm = FormTag<kDiffusion>;
using MassForm = FormTag<kMass>;
using TangentDiffusionForm = FormTag<kTangentDiffusion>;
using TangentMassForm = FormTag<kTangentMass>;
using SourceForm = FormTag<kSource>;

// the models live in the device problem (rsd_heat_desc); these name them for the stages' registries
struct ConductivityModel {};
struct MassModel {};

using Coefficients = std::array<double, kSlots>;

template <typename FormsT>
Coefficients matrix_coefficients(const FormsT& forms) {
	ProbePoint qp;
	Real Ke[kSlots * kSlots] = {};
	forms.computeElementLevelMatrix(qp, Ke);
	Coefficients c{};
	for (int k = 0; k < kSlots; ++k) c[k] = Ke[k];
	return c;
}
template <typename FormsT>
Coefficients vector_coefficients(const FormsT& forms) {
	ProbePoint qp;
	Real Ue[kSlots] = {}, Oe[kSlots] = {};
	forms.computeElementLevelVector(qp, Ue, Oe);
	Coefficients c{};
	for (int k = 0; k < kSlots; ++k) c[k] = Oe[k];
	return c;
}

// HeatStateVector's role (equation/heateq/evaluator/HeatStateVector.hpp:21-56): the vectors a form is
// evaluated against; the buffers are tags a selector lambda picks from.
template <typename VectorT>
struct HeatState {
	const VectorT* valueSource = nullptr;
	const VectorT* rateSource = nullptr;
	const VectorT* operandSource = nullptr;
	Real tags_[3] = {};
	Real* valueBuffer() { return &tags_[0]; }
	Real* rateBuffer() { return &tags_[1]; }
	Real* operandBuffer() { return &tags_[2]; }
};
enum class Operand { Value, Rate, Operand };
template <typename StateT, typename SelectorT>
Operand which_operand(SelectorT& selector) {
	StateT probe;
	Real* p = selector(probe);
	if (p == probe.valueBuffer()) return Operand::Value;
	if (p == probe.rateBuffer()) return Operand::Rate;
	return Operand::Operand;
}

// ---------------------------------------------------------------------------------------------
// the problem
// ---------------------------------------------------------------------------------------------
template <int NSD>
class HeatProblem {
public:
	using VectorT = ::residuum::linalg::types::Vector<double, B200>;
	using MatrixT = ::residuum::linalg::types::CSRMatrix<double, B200>;
	using StateVectorT = HeatState<VectorT>;
	static constexpr Index NumDOFs = 1;
	static constexpr Index SpatialDim = NSD;

	using StiffnessForms = ::residuum::fem::form::FormRegistry<DiffusionForm>;
	using MassForms = ::residuum::fem::form::FormRegistry<MassForm>;
	using TangentDiffusionForms = ::residuum::fem::form::FormRegistry<TangentDiffusionForm>;
	using TangentMassForms = ::residuum::fem::form::FormRegistry<TangentMassForm>;

	// HeatProblem(config, mesh, basis, quadratureVolume, quadratureBoundary) (HeatProblem.tpp:4):
	// the basis order comes from the mesh, the Gauss rule from config.discretization.quadrature
	HeatProblem(const ::residuum::application::heateq::config::HeatConfig& config, ::residuum::mesh::Mesh mesh)
		: config_(config), solverInstance_(::residuum::solver::resolveSolverInstance(config_.solver)), mesh_(std::move(mesh)) {
		namespace hc = ::residuum::application::heateq::config;
		namespace sc = ::residuum::solver::config;
		const auto& md = mesh_.data;
		if (md.spatialDim != (Index)NSD || md.parametricDim != (Index)NSD)
			throw std::runtime_error("HeatProblem<B200>: the mesh's dimensions differ from the problem's");
		if (md.basisType != ::residuum::mesh::BasisType::Lagrange) throw std::runtime_error("HeatProblem<B200>: Lagrange basis only");
		const Index order = md.basisOrder.empty() ? 1 : md.basisOrder[0];
		for (Index o : md.basisOrder)
			if (o != order) throw std::runtime_error("HeatProblem<B200>: the basis order must be equal in every direction");
		const auto& q = config_.discretization.quadrature;
		if (q.eta != q.xi || (NSD == 3 && q.zeta != q.xi))
			throw std::runtime_error("HeatProblem<B200>: the Gauss rule must have equal points in every direction");

		rsd_heat_desc d{};
		d.nq = (int32_t)q.xi;
		d.rho = 1.0;
		d.cp = 1.0;
		d.k_const = 1.0;
		std::vector<double> tensor;
		auto set_tensor = [&]() {
			const auto& t = config_.conductivity.tensor;
			if (t.size() != (size_t)NSD) throw std::runtime_error("ConductivityModel: tensor must be SpatialDim x SpatialDim");
			for (const auto& row : t) {
				if (row.size() != (size_t)NSD) throw std::runtime_error("ConductivityModel: tensor must be SpatialDim x SpatialDim");
				tensor.insert(tensor.end(), row.begin(), row.end());
			}
			d.k_tensor = tensor.data();
		};
		switch (config_.conductivity.type) {
			case hc::ConductivityConfig::Type::Constant: d.k_const = config_.conductivity.value; break;
			case hc::ConductivityConfig::Type::Anisotropic: set_tensor(); break;
			case hc::ConductivityConfig::Type::TemperatureDependentIsotropic:
				d.k_expr = config_.conductivity.valueExpression.c_str();
				d.dk_expr = config_.conductivity.gradientExpression.c_str();
				break;
			case hc::ConductivityConfig::Type::TemperatureDependentAnisotropic:
				set_tensor();
				d.k_expr = config_.conductivity.valueExpression.c_str();
				d.dk_expr = config_.conductivity.gradientExpression.c_str();
				break;
			default: throw std::runtime_error("HeatProblem: unsupported conductivity type");
		}
		const bool transient = ::residuum::solver::isTransient(solverInstance_.mode);
		if (transient) {
			if (!config_.density.has_value() || !config_.specificHeat.has_value())
				throw std::runtime_error("HeatProblem: 'materials.density' and 'materials.specific_heat' are required for a transient driver");
			if (!solverInstance_.timestepper) throw std::runtime_error("HeatProblem: solver.timestepper config is required for a transient driver");
			d.rho = config_.density->value;
			if (config_.specificHeat->type == hc::SpecificHeatConfig::Type::Constant) {
				d.cp = config_.specificHeat->value;
			} else if (config_.specificHeat->type == hc::SpecificHeatConfig::Type::TemperatureDependent) {
				d.cp_expr = config_.specificHeat->valueExpression.c_str();
				d.dcp_expr = config_.specificHeat->gradientExpression.c_str();
			} else {
				throw std::runtime_error("HeatProblem: unsupported specific heat type");
			}
		}
		if (config_.source.read.mode != sc::NodalFieldReadConfig::Mode::Expression)
			throw std::runtime_error("HeatProblem<B200>: nodal source files are not read by the device path");
		d.src_expr = config_.source.read.expression.c_str();
		std::vector<int32_t> tags;
		std::vector<const char*> exprs;
		for (const auto& bc : config_.boundaryConditions)
			for (auto form : bc.forms) {
				if (bc.mode == sc::NodalFieldReadConfig::Mode::File)
					throw std::runtime_error("HeatProblem<B200>: nodal boundary files are not read by the device path");
				if (form == hc::BoundaryConditionConfig::Form::ValueBC) {
					tags.push_back((int32_t)bc.boundaryID);
					exprs.push_back(bc.expression.c_str());
				} else if (bc.fluxExpression.size() != (size_t)NSD) {
					throw std::runtime_error("HeatProblem: flux boundary 'expression' must have SpatialDim components");
				}
			}
		d.num_dirichlet = (int32_t)tags.size();
		d.dirichlet_tags = tags.data();
		d.dirichlet_exprs = exprs.data();

		std::vector<int64_t> ien(md.ien.begin(), md.ien.end());
		std::vector<int32_t> rng(md.rng.begin(), md.rng.end());
		rsd_mesh* m = nullptr;
		check(rsd_mesh_create(B200::ctx(), NSD, (int32_t)order, (int64_t)md.numNodes, (int64_t)md.numElements, md.xyz.data(),
		                      ien.data(), rng.data(), &m));
		rmesh_.reset(m);
		rsd_heat* h = nullptr;
		check(rsd_heat_create(B200::ctx(), rmesh_.get(), &d, &h));
		heat_.reset(h);
		for (const auto& bc : config_.boundaryConditions)
			for (auto form : bc.forms)
				if (form == hc::BoundaryConditionConfig::Form::FluxBC) {
					std::vector<const char*> fx;
					for (const auto& e : bc.fluxExpression) fx.push_back(e.c_str());
					check(rsd_heat_set_flux(B200::ctx(), heat_.get(), (int32_t)bc.boundaryID, fx.data()));
				}
		int64_t n = 0, nnz = 0;
		check(rsd_heat_info(heat_.get(), &n, &nnz));
		numFree_ = (Index)n;

		F_ = std::make_unique<VectorT>(createVector());
		U_ = std::make_unique<VectorT>(createVector());
		U_prev_ = std::make_unique<VectorT>(createVector());
		Udot_ = std::make_unique<VectorT>(createVector());
		// initial condition (HeatProblem::loadNodalField, Expression mode)
		if (config_.initialCondition.read.mode != sc::NodalFieldReadConfig::Mode::Expression)
			throw std::runtime_error("HeatProblem<B200>: nodal initial-condition files are not read by the device path");
		check(rsd_heat_eval_nodal(B200::ctx(), heat_.get(), config_.initialCondition.read.expression.c_str(), 0.0, U_->data()));
		if (transient) ::residuum::linalg::operations::copy(*U_, *U_prev_);
	}

	HeatProblem(const HeatProblem&) = delete;
	HeatProblem& operator=(const HeatProblem&) = delete;

	// stateless forms and the models (HeatProblem.hpp:55-60)
	StiffnessForms stiffnessForms() const { return {}; }
	MassForms massForms() const { return {}; }
	TangentDiffusionForms tangentStiffnessForms() const { return {}; }
	TangentMassForms tangentMassForms() const { return {}; }
	const ConductivityModel& stiffnessModel() const { return conductivity_; }
	const MassModel& massModel() const { return mass_; }

	// HeatProblem::createMatrix / createVector (HeatProblem.hpp:62-63): the problem's pattern, zeros
	MatrixT createMatrix() const {
		rsd_csr* A = nullptr;
		check(rsd_heat_create_matrix(B200::ctx(), heat_.get(), &A));
		return MatrixT(A);
	}
	VectorT createVector() const {
		VectorT v(numFree_);
		v.zero();
		return v;
	}

	// HeatProblem::assembleLoad (HeatProblem.tpp:217-231)
	void assembleLoad(Real time) {
		setTime(time);
		check(rsd_assemble_vector(B200::ctx(), heat_.get(), 0, 0.0, nullptr, nullptr, nullptr, F_->data()));
	}
	// HeatProblem::applyNatural (HeatProblem.tpp:234-238)
	void applyNatural(Real time) {
		setTime(time);
		check(rsd_apply_natural(B200::ctx(), heat_.get(), F_->data()));
	}

	// HeatProblem::assembleMatrix (HeatProblem.tpp:240-246): K = sum of the composition's forms
	template <typename FormsT, typename ModelT>
	void assembleMatrix(Real time, const FormsT& forms, const ModelT&, StateVectorT& state, MatrixT& K) {
		const Coefficients c = matrix_coefficients(forms);
		setTime(time);
		check(rsd_assemble_matrix(B200::ctx(), heat_.get(), c[kDiffusion], c[kMass], c[kTangentDiffusion], c[kTangentMass],
		                          ptr(state.valueSource), ptr(state.rateSource), K.handle()));
	}

	// HeatProblem::assembleVector (HeatProblem.tpp:248-255): V = the composition applied to the
	// vector the selector names, with the models at the state
	template <typename FormsT, typename ModelT, typename SelectorT>
	void assembleVector(Real time, const FormsT& forms, const ModelT&, StateVectorT& state, SelectorT selector, VectorT& V) {
		const Coefficients c = vector_coefficients(forms);
		const Operand op = which_operand<StateVectorT>(selector);
		setTime(time);
		rsd_ctx* ctx = B200::ctx();
		const double* U = ptr(state.valueSource);
		const double* Ud = ptr(state.rateSource);
		if (op == Operand::Operand) {
			// FEMOperator::apply's composition on the operand: Diffusion + c_mass Mass (+ TangentDiffusion)
			if (c[kDiffusion] != 1.0 || c[kTangentMass] != 0.0 || (c[kTangentDiffusion] != 0.0 && c[kTangentDiffusion] != 1.0) || c[kSource] != 0.0)
				throw std::runtime_error("HeatProblem<B200>: operand products take Diffusion + c Mass [+ TangentDiffusion]");
			const int which = c[kTangentDiffusion] != 0.0 ? 10 : 4;
			check(rsd_assemble_vector(ctx, heat_.get(), which, c[kMass], U, Ud, ptr(state.operandSource), V.data()));
			return;
		}
		if (c[kTangentDiffusion] != 0.0 || c[kTangentMass] != 0.0)
			throw std::runtime_error("HeatProblem<B200>: tangent forms act on an operand");
		// one device pass per form kind present, summed into V
		struct Term { int which; double coef; };
		std::vector<Term> terms;
		if (op == Operand::Value) {
			if (c[kDiffusion] != 0.0) terms.push_back({1, c[kDiffusion]});   // Diffusion on U (Full)
			if (c[kMass] != 0.0) terms.push_back({2, c[kMass]});             // rho cp Mass on U (Full)
			if (c[kSource] != 0.0) terms.push_back({0, c[kSource]});         // SourceForm
		} else {
			if (c[kDiffusion] != 0.0 || c[kSource] != 0.0) throw std::runtime_error("HeatProblem<B200>: only Mass acts on the rate");
			if (c[kMass] != 0.0) terms.push_back({3, c[kMass]});             // rho cp(T(U)) Mass on Udot (Free)
		}
		if (terms.empty()) { V.zero(); return; }
		for (size_t i = 0; i < terms.size(); ++i) {
			VectorT& dst = i == 0 ? V : scratch();
			check(rsd_assemble_vector(ctx, heat_.get(), terms[i].which, 0.0, U, Ud, nullptr, dst.data()));
			if (i == 0) {
				if (terms[i].coef != 1.0) ::residuum::linalg::operations::scal(terms[i].coef, V);
			} else {
				::residuum::linalg::operations::axpy(terms[i].coef, dst, V);
			}
		}
	}

	// HeatProblem::assembleResidual (HeatProblem.tpp:257-263): always against the current solution
	template <typename FormsT, typename ModelT>
	void assembleResidual(Real time, const FormsT& forms, const ModelT& model, StateVectorT& state, VectorT& R) {
		assembleVector(time, forms, model, state, [](StateVectorT& s) -> Real* { return s.valueBuffer(); }, R);
	}

	// HeatProblem::applyEssential (HeatProblem.tpp:265-271): F -= the composition applied to the
	// Dirichlet values (BoundaryApplicator::applyEssentialBCs)
	template <typename FormsT, typename ModelT>
	void applyEssential(Real time, const FormsT& forms, const ModelT&, VectorT& F) {
		const Coefficients c = vector_coefficients(forms);
		if (c[kTangentDiffusion] != 0.0 || c[kTangentMass] != 0.0 || c[kSource] != 0.0)
			throw std::runtime_error("HeatProblem<B200>: the Dirichlet lift takes Diffusion and Mass");
		setTime(time);
		check(rsd_apply_dirichlet_lift(B200::ctx(), heat_.get(), c[kDiffusion], c[kMass], F.data()));
	}

	// HeatProblem::makeLinearRunner (HeatProblem.tpp:273-291)
	template <typename FormsT, typename ModelT>
	std::unique_ptr<::residuum::linalg::solver::LinearSolverRunner<VectorT>> makeLinearRunner(const Real* time, const FormsT& forms, const ModelT&,
	                                                                                           StateVectorT& state, MatrixT& K) {
		using OpType = ::residuum::solver::config::LinearSolverConfig::OperatorType;
		const auto& lin = *solverInstance_.linear;
		const rsd_solver_cfg cfg = solver_cfg(lin);
		if (lin.operatorType == OpType::CSR) {
			if (useReferenceSolvers_) {
				using Op = ::residuum::linalg::op::CSROperator<MatrixT>;
				return ::residuum::solver::linear::makeLinearSolverRunner<Op, VectorT>(Op(K), numFree_, lin, config_.logging.linear, equationLabel(),
				                                                                        dofNames(), freeDOFsPerField(), dofOrdering());
			}
			return std::make_unique<MatrixRunner>(K, cfg);
		}
		if (lin.operatorType == OpType::FEM) {
			const Coefficients c = matrix_coefficients(forms);
			if (c[kDiffusion] != 1.0 || c[kSource] != 0.0)
				throw std::runtime_error("HeatProblem<B200>: the matrix-free operator takes Diffusion with coefficient 1");
			return std::make_unique<FemRunner>(*this, time, state, c, cfg);
		}
		throw std::runtime_error("HeatProblem: unsupported operator");
	}

	Index numFreeDOFs() const { return numFree_; }
	std::vector<std::string> dofNames() const { return {"T"}; }
	Index freeDOFsPerField() const { return numFree_; }
	::residuum::fem::dof::DOFOrdering dofOrdering() const { return ::residuum::fem::dof::DOFOrdering::Interleaved; }
	const ::residuum::solver::SolverInstance& solverInstance() const { return solverInstance_; }
	std::string equationLabel() const { return "Heat Equation"; }
	const ::residuum::solver::config::LoggingConfig& loggingConfig() const { return config_.logging; }

	VectorT& U() { return *U_; }
	VectorT& F() { return *F_; }
	VectorT& U_prev() { return *U_prev_; }
	VectorT& Udot() { return *Udot_; }
	const VectorT& solution() const { return *U_; }
	void advance() { ::residuum::linalg::operations::copy(*U_, *U_prev_); }

	// field output and monitors are not part of the device path
	void writeOutput(Index, Real) const {}
	void writeLog() const {}
	void evaluateMonitors(Index, Real) const {}

	// CSR runners: the reference's own solver templates on the tag (true) or the device solver (false)
	void useReferenceSolvers(bool on) { useReferenceSolvers_ = on; }
	// the device problem, for calls of the C ABI beside the stages
	rsd_heat* device() const { return heat_.get(); }
	// the free DOF values on the host
	std::vector<double> solutionToHost() const {
		std::vector<double> h(numFree_);
		B200::copy<double>(h.data(), U_->data(), numFree_, ::residuum::linalg::types::backend::CopyKind::DeviceToHost);
		return h;
	}

private:
	static const double* ptr(const VectorT* v) { return v ? v->data() : nullptr; }

	void setTime(Real t) {
		if (timeSet_ && t == time_) return;
		check(rsd_heat_set_time(B200::ctx(), heat_.get(), t));
		time_ = t;
		timeSet_ = true;
	}
	VectorT& scratch() {
		if (!scratch_) scratch_ = std::make_unique<VectorT>(numFree_);
		return *scratch_;
	}

	// LinearSolverConfig -> the device solver's configuration (CG or GMRES(m), Jacobi or identity)
	static rsd_solver_cfg solver_cfg(const ::residuum::solver::config::LinearSolverConfig& lin) {
		namespace sc = ::residuum::solver::config;
		rsd_solver_cfg c{};
		switch (lin.type) {
			case sc::LinearSolverConfig::Type::CG: c.type = RSD_CG; break;
			case sc::LinearSolverConfig::Type::GMRES: c.type = RSD_GMRES; break;
			default: throw std::runtime_error("LinearSolverFactory: only CG and GMRES are implemented");
		}
		c.precond = lin.preconditioner.type == sc::PreconditionerConfig::Type::Jacobi ? RSD_JACOBI : RSD_IDENTITY;
		c.precision = RSD_FP64;
		c.tol_type = RSD_TOL_RELATIVE;
		c.tol = lin.tolerance;
		c.max_iters = (int64_t)lin.maxIterations;
		c.krylov_dim = 50;
		if (const auto* g = std::get_if<sc::GMRESParams>(&lin.params)) c.krylov_dim = (int64_t)g->krylovDim;
		c.operator_type = lin.operatorType == sc::LinearSolverConfig::OperatorType::FEM ? RSD_OP_FEM : RSD_OP_CSR;
		return c;
	}
	static void fill(const rsd_report& r, ::residuum::linalg::solver::SolverReport<VectorT>& report) {
		report.converged = r.converged != 0;
		report.iterations = (Index)r.iterations;
		report.initialResidual = r.initialResidual;
		report.finalResidual = r.finalResidual;
		report.finalResidualRel = r.finalResidualRel;
		if (r.status != RSD_OK) throw std::runtime_error(std::string("rsd: ") + rsd_last_error_string());
	}

	struct MatrixRunner final : ::residuum::linalg::solver::LinearSolverRunner<VectorT> {
		MatrixT& K;
		rsd_solver_cfg cfg;
		MatrixRunner(MatrixT& k, const rsd_solver_cfg& c) : K(k), cfg(c) { cfg.operator_type = RSD_OP_CSR; }
		bool solve(const VectorT& b, VectorT& x, ::residuum::linalg::solver::SolverReport<VectorT>& report) override {
			rsd_report r{};
			check(rsd_solve(B200::ctx(), K.handle(), &cfg, b.data(), x.data(), &r));
			fill(r, report);
			return report.converged;
		}
	};
	struct FemRunner final : ::residuum::linalg::solver::LinearSolverRunner<VectorT> {
		HeatProblem& p;
		const Real* time;
		StateVectorT& state;
		Coefficients c;
		rsd_solver_cfg cfg;
		FemRunner(HeatProblem& pr, const Real* t, StateVectorT& s, const Coefficients& co, const rsd_solver_cfg& cf)
			: p(pr), time(t), state(s), c(co), cfg(cf) {}
		bool solve(const VectorT& b, VectorT& x, ::residuum::linalg::solver::SolverReport<VectorT>& report) override {
			if (time) p.setTime(*time);
			rsd_report r{};
			check(rsd_heat_solve_fem_forms(B200::ctx(), p.heat_.get(), c[kTangentDiffusion], c[kMass], c[kTangentMass], ptr(state.valueSource),
			                               ptr(state.rateSource), &cfg, b.data(), x.data(), &r));
			fill(r, report);
			return report.converged;
		}
	};

	struct MeshDel { void operator()(rsd_mesh* m) const noexcept { rsd_mesh_destroy(m); } };
	struct HeatDel { void operator()(rsd_heat* h) const noexcept { rsd_heat_destroy(h); } };

	::residuum::application::heateq::config::HeatConfig config_;
	::residuum::solver::SolverInstance solverInstance_;
	::residuum::mesh::Mesh mesh_;
	std::unique_ptr<rsd_mesh, MeshDel> rmesh_;
	std::unique_ptr<rsd_heat, HeatDel> heat_;
	Index numFree_ = 0;
	ConductivityModel conductivity_;
	MassModel mass_;
	std::unique_ptr<VectorT> F_, U_, U_prev_, Udot_, scratch_;
	Real time_ = 0.0;
	bool timeSet_ = false;
	bool useReferenceSolvers_ = false;
};

}  // namespace rsd::residuum::heat
