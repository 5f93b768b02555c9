// Test infrastructure, not product code.
//
// C-ABI harness over the UNMODIFIED Residuum reference templates (linalg, fem, solver), compiled
// from the reference source tree by oracle/Makefile into oracle/_ref/libresiduum_ref.so.  It is
// the strongest available checker for the CUDA backend: every number it returns is produced by the
// reference's own Assembler<CPU>, BoundaryApplicator<CPU>, TopologicalDOF, cg::Solver,
// gmres::Solver, Jacobi, SteadyStage, BackwardEulerStage, NewtonRunner and BackwardEulerRunner.
//
// What is project-written here (plugins that the reference's concepts accept, no reference logic
// is re-implemented):
//   * closed-form models (conductivity k(T) = ka + kb*T, constant specific heat) standing in for
//     the exprtk-backed ConductivityModel / SpecificHeatModel (exprtk is not vendored with the
//     reference and is absent here; equation/heateq/evaluator/ConductivityModel.hpp:60-96 is the
//     behaviour mirrored);
//   * closed-form source and Dirichlet callables for SourceFunction / BoundaryValueFunction;
//   * ElementScaledDiffusion, a form that wraps the reference DiffusionForm and scales it by a
//     per-element conductivity recovered in gatherElementData (the reference Assembler calls it per
//     element, fem/assembly/backend/cpu/Assembler.tpp:118);
//   * RefHeatProblem, a Problem / TransientCapableProblem implementation mirroring
//     application/heateq/problem/HeatProblem.tpp:217-289 without YAML, IO, loggers or monitors,
//     so that the reference's own SteadyStage / BackwardEulerStage / NewtonRunner drive it.
//   * ref_adjoint_gradient: an FP64 element loop over the reference QP evaluator + DiffusionForm;
//   * ref_boundary_flux: the reference's own BoundaryQuadratureMonitorGroup (HeatFluxIntegrand) and
//     BoundaryReactionMonitorGroup composed as HeatProblem::makeMonitorGroup composes them
//     (application/heateq/problem/HeatProblem.tpp:368-440), evaluated with a full-precision callback.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "core/Types.hpp"
#include "linalg/types/Vector.hpp"
#include "linalg/types/CSRMatrix.hpp"
#include "linalg/operations/VectorOps.hpp"
#include "linalg/operations/MatrixOps.hpp"
#include "linalg/operator/CSROperator.hpp"
#include "linalg/operator/FEMOperator.hpp"
#include "fem/quantity/QuantityEvaluator.hpp"
#include "fem/quantity/BoundaryQuadratureMonitorGroup.hpp"
#include "fem/quantity/BoundaryReactionMonitorGroup.hpp"
#include "fem/quantity/QuantityForms.hpp"
#include "fem/dispatch/DiscretizationDispatch.hpp"
#include "equation/heateq/quantity/HeatFluxIntegrand.hpp"
#include "equation/heateq/evaluator/HeatBoundaryStateVector.hpp"
#include "equation/heateq/evaluator/EvalQuadraturePointBoundary.hpp"
#include "fem/quantity/recovery/SimpleAverageRecovery.hpp"
#include "equation/heateq/evaluator/HeatFluxField.hpp"
#include "equation/heateq/evaluator/ConductivityField.hpp"
#include "linalg/solver/iterative/cg/Solver.hpp"
#include "linalg/solver/iterative/gmres/Solver.hpp"
#include "linalg/solver/preconditioner/Jacobi.hpp"
#include "linalg/solver/preconditioner/Identity.hpp"
#include "utils/logging/core/NullLogger.hpp"
#include "fem/assembly/Assembler.hpp"
#include "fem/boundary/BoundaryApplicator.hpp"
#include "fem/basis/LagrangeHex.hpp"
#include "fem/basis/LagrangeQuad.hpp"
#include "fem/quadrature/GaussQuadratureHex.hpp"
#include "fem/quadrature/GaussQuadratureQuad.hpp"
#include "fem/geometry/JacobianTransform.hpp"
#include "fem/form/FormRegistry.hpp"
#include "fem/form/ScaledForm.hpp"
#include "fem/evaluator/ModelRegistry.hpp"
#include "equation/heateq/evaluator/EvalElement.hpp"
#include "equation/heateq/evaluator/EvalQuadraturePointVolume.hpp"
#include "equation/heateq/evaluator/HeatStateVector.hpp"
#include "equation/heateq/evaluator/DensityModel.hpp"
#include "equation/heateq/evaluator/DefaultModel.hpp"
#include "equation/heateq/evaluator/SourceFunction.hpp"
#include "equation/heateq/boundary/BoundaryValueFunction.hpp"
#include "equation/heateq/form/DiffusionForm.hpp"
#include "equation/heateq/form/MassForm.hpp"
#include "equation/heateq/form/TangentDiffusionForm.hpp"
#include "equation/heateq/form/TangentMassForm.hpp"
#include "equation/heateq/form/SourceForm.hpp"
#include "mesh/generator/BlockMesh2D.hpp"
#include "mesh/generator/BlockMesh3D.hpp"
#include "topology/TopologicalDOF.hpp"
#include "solver/SolverInstance.hpp"
#include "solver/config/LoggingConfig.hpp"
#include "solver/config/LinearSolverConfig.hpp"
#include "solver/config/NonlinearSolverConfig.hpp"
#include "solver/config/TimeStepperConfig.hpp"
#include "solver/linear/LinearSolverFactory.hpp"
#include "solver/stage/SteadyStage.hpp"
#include "solver/stage/BackwardEulerStage.hpp"
#include "solver/timestepper/BackwardEuler.hpp"
#include "solver/timestepper/ConstantStepSizePolicy.hpp"

using namespace residuum;
using CPU = linalg::types::backend::CPU;
using VecT = linalg::types::Vector<Real, CPU>;
using MatT = linalg::types::CSRMatrix<Real, CPU>;

extern "C" {

// Problem description shared with oracle/__init__.py (ctypes mirror of this layout).
typedef struct ref_desc {
	int32_t nsd;            // 2 (quad) or 3 (hex)
	int32_t order;          // Lagrange order in every direction
	int32_t nq;             // Gauss points per direction
	int32_t nx, ny, nz;     // elements per direction
	double lo[3], hi[3];    // block extents
	int32_t ess_mask;       // bit t set: boundary tag t carries an essential (Dirichlet) condition
	int32_t bc_kind;        // 0: per-tag constants bc_val[tag]; 1: g = x; 2: g = (1-x)(1-y)
	double bc_val[6];
	int32_t src_kind;       // 0: f = src_c; 1: f = src_c * x*y(*z)
	double src_c;
	double k_a, k_b;        // k(T) = k_a + k_b*T, dk/dT = k_b
	double rho, cp;         // density, specific heat (constant)
	const double* k_elem;   // optional per-element conductivity multiplier (numElements) or NULL
} ref_desc;

typedef struct ref_report {
	int32_t converged;
	int64_t iterations;
	double initialResidual, finalResidual, finalResidualRel;
} ref_report;

} // extern "C"

namespace {

// ---- closed-form plugins ---------------------------------------------------------------------

struct SourceCallable {
	int kind; double c; int nsd;
	void operator()(Real, const Real* x, Real* out) const {
		if (kind == 0) { out[0] = c; return; }
		Real p = c;
		for (int d = 0; d < nsd; ++d) p *= x[d];
		out[0] = p;
	}
};

struct DirichletCallable {
	int kind; double val;
	void operator()(Real, const Real* x, Real* out) const {
		if (kind == 0) out[0] = val;
		else if (kind == 1) out[0] = x[0];
		else out[0] = (1.0 - x[0]) * (1.0 - x[1]);
	}
};

// k(T) = ka + kb*T isotropic; mirrors ConductivityModel::eval/evalGradient
// (equation/heateq/evaluator/ConductivityModel.hpp:60-96) for an isotropic value/gradient pair.
template<typename QP>
struct LinearConductivity {
	Real ka = 1, kb = 0;
	void eval(QP& qp) const {
		Real k = (kb != 0.0) ? (ka + kb * qp.T.value()) : ka;
		for (Index i = 0; i < QP::SpatialDim; ++i)
			for (Index j = 0; j < QP::SpatialDim; ++j)
				qp.K[i * QP::SpatialDim + j] = (i == j) ? k : Real(0);
	}
	void evalGradient(QP& qp) const {
		Real dk = kb;
		for (Index i = 0; i < QP::SpatialDim; ++i)
			for (Index j = 0; j < QP::SpatialDim; ++j)
				qp.dKdT[i * QP::SpatialDim + j] = (i == j) ? dk : Real(0);
	}
};

// constant specific heat; mirrors SpecificHeatModel (…/SpecificHeatModel.hpp) in Constant mode
template<typename QP>
struct ConstantSpecificHeat {
	Real value = 1;
	void eval(QP& qp) const { qp.cp = value; }
	void evalGradient(QP& qp) const { qp.dcpdT = Real(0); }
};

// DiffusionForm scaled by a per-element conductivity recovered from the element's ien slice
template<typename QP>
struct ElementScaledDiffusion {
	const Index* ienBase = nullptr;
	Index npe = 1;
	const double* kElem = nullptr;
	mutable Real scale = 1;
	void gatherElementData(const Index* nodeIDs, Index) const {
		scale = kElem ? kElem[(nodeIDs - ienBase) / npe] : Real(1);
	}
	void computeElementLevelMatrix(const QP& qp, Real* Ke) const {
		if (!kElem) { equation::heateq::DiffusionForm<QP>::computeElementLevelMatrix(qp, Ke); return; }
		constexpr Index maxN = fem::dispatch::kMaxNodesPerElement<QP::ParametricDim>;
		Real buffer[maxN * maxN];
		std::memset(buffer, 0, sizeof(buffer));
		equation::heateq::DiffusionForm<QP>::computeElementLevelMatrix(qp, buffer);
		const Index n = qp.nodesPerElement();
		for (Index i = 0; i < n * n; ++i) Ke[i] += scale * buffer[i];
	}
	void computeElementLevelVector(const QP& qp, const Real* Ue, Real* Oe) const {
		if (!kElem) { equation::heateq::DiffusionForm<QP>::computeElementLevelVector(qp, Ue, Oe); return; }
		constexpr Index maxN = fem::dispatch::kMaxNodesPerElement<QP::ParametricDim>;
		Real buffer[maxN];
		std::memset(buffer, 0, sizeof(buffer));
		equation::heateq::DiffusionForm<QP>::computeElementLevelVector(qp, Ue, buffer);
		const Index n = qp.nodesPerElement();
		for (Index i = 0; i < n; ++i) Oe[i] += scale * buffer[i];
	}
};

// ---- type bundle per dimension ----------------------------------------------------------------

template<int NSD> struct Family;
template<> struct Family<2> {
	using Basis = fem::basis::LagrangeQuad;
	using Quad = fem::quadrature::GaussQuadratureQuad;
	static Basis basis(int p) { return Basis(p, p); }
	static Quad quad(int q) { return Quad(q, q); }
};
template<> struct Family<3> {
	using Basis = fem::basis::LagrangeHex;
	using Quad = fem::quadrature::GaussQuadratureHex;
	static Basis basis(int p) { return Basis(p, p, p); }
	static Quad quad(int q) { return Quad(q, q, q); }
};

struct Base {
	virtual ~Base() = default;
	virtual Index numNodes() const = 0;
	virtual Index numElems() const = 0;
	virtual Index numFree() const = 0;
	virtual void dofmap(int32_t* t2a, int32_t* a2t) = 0;
	virtual void mesh(double* xyz, int64_t* ien, int32_t* rng) = 0;
	virtual Index nnz() = 0;
	virtual void pattern(int64_t* rowPtr, int64_t* col) = 0;
	virtual void assembleMatrix(int formset, double massCoef, const double* U, const double* Udot, double* val) = 0;
	virtual void assembleVector(int which, double coef, const double* U, const double* Udot, const double* operand, double* out) = 0;
	virtual void lift(int formset, double massCoef, double* F) = 0;
	virtual void diagonal(int formset, double massCoef, const double* U, double* d) = 0;
	virtual int steady(int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, ref_report* rep) = 0;
	virtual int newton(double absTol, double relTol, int64_t maxit, int solverType, int precond, double tol, int64_t linMaxit, int64_t krylov, double* U, ref_report* rep) = 0;
	virtual int backwardEuler(double dt, int64_t nsteps, int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, double* residualPerStep, double* stepStats) = 0;
	virtual void adjointGradient(const double* T, const double* lam, double* grad) = 0;
	virtual void boundaryFlux(int method, int reduction, int transient, int ntags, const int32_t* tags, const double* U, const double* Udot, double* values) = 0;
	int opType = 0;   // LinearSolverConfig::OperatorType of the stages' linear solves: 0 CSR, 1 FEM
	virtual void nodalField(int field, const double* U, double* out) = 0;
};

template<int NSD>
struct RefHeatProblem final : Base {

	static constexpr Index NumDOFs = 1;
	using Fam = Family<NSD>;
	using EvalEle = equation::heateq::evaluator::EvalElement<typename Fam::Basis, NSD>;
	using EvalQP = equation::heateq::evaluator::EvalQuadraturePointVolume<EvalEle, typename Fam::Basis, fem::geometry::JacobianTransform<NSD, NSD>>;
	using VectorT = VecT;
	using MatrixT = MatT;
	using StateVectorT = equation::heateq::evaluator::HeatStateVector<1, NSD, NSD, VecT>;

	using Cond = LinearConductivity<EvalQP>;
	using Density = equation::heateq::evaluator::DensityModel<EvalQP>;
	using Cp = ConstantSpecificHeat<EvalQP>;
	using MassModelT = fem::evaluator::ModelRegistry<Density, Cp>;
	using OpModelT = fem::evaluator::ModelRegistry<Cond, Density, Cp>;

	using Diff = ElementScaledDiffusion<EvalQP>;
	using StiffnessForms = fem::form::FormRegistry<Diff>;
	using MassForms = fem::form::FormRegistry<equation::heateq::MassForm<EvalQP>>;
	using TangentDiffusionForms = fem::form::FormRegistry<equation::heateq::TangentDiffusionForm<EvalQP>>;
	using TangentMassForms = fem::form::FormRegistry<equation::heateq::TangentMassForm<EvalQP>>;
	using SourceFn = equation::heateq::evaluator::SourceFunction<NSD, 1, SourceCallable>;
	using SourceForms = fem::form::FormRegistry<equation::heateq::SourceForm<EvalQP, SourceFn>>;
	using DirichletFn = equation::heateq::BoundaryValueFunction<NSD, 1, DirichletCallable>;

	ref_desc d;
	std::vector<double> kElem;
	mesh::Mesh mesh_;
	std::unique_ptr<topology::TopologicalDOF<1>> topo_;
	fem::boundary::EssentialBoundaryRegistry ess_;
	typename Fam::Basis basis_;
	typename Fam::Quad quad_;
	EvalEle evalEle_;
	Cond cond_;
	Density density_;
	Cp cp_;
	MassModelT massModel_;
	OpModelT opModel_;
	equation::heateq::evaluator::DefaultModel<EvalQP> defaultModel_;
	Diff diff_;
	std::unique_ptr<StiffnessForms> stiff_;
	fem::assembly::Assembler<CPU> assembler_;
	SourceForms sourceForms_;

	// linear / nonlinear / time-stepper configuration consumed by the reference stages
	solver::config::LinearSolverConfig linCfg_;
	solver::config::NonlinearSolverConfig nlCfg_;
	solver::config::TimeStepperConfig tsCfg_;
	solver::config::LoggingConfig logCfg_;
	solver::SolverInstance inst_;

	std::unique_ptr<VecT> F_, U_, Uprev_, Udot_;

	static mesh::Mesh makeMesh(const ref_desc& d) {
		if (NSD == 2) return mesh::generator::BlockMesh2D(d.nx, d.ny, d.lo[0], d.hi[0], d.lo[1], d.hi[1], d.order, d.order).generate();
		return mesh::generator::BlockMesh3D(d.nx, d.ny, d.nz, d.lo[0], d.hi[0], d.lo[1], d.hi[1], d.lo[2], d.hi[2], d.order, d.order, d.order).generate();
	}

	explicit RefHeatProblem(const ref_desc& desc)
		: d(desc), mesh_(makeMesh(desc)), basis_(Fam::basis(desc.order)), quad_(Fam::quad(desc.nq)), evalEle_(basis_),
		  sourceForms_(SourceFn(SourceCallable{desc.src_kind, desc.src_c, NSD})) {
		if (desc.k_elem) kElem.assign(desc.k_elem, desc.k_elem + mesh_.data.numElements);
		d.k_elem = kElem.empty() ? nullptr : kElem.data();
		topo_ = std::make_unique<topology::TopologicalDOF<1>>(mesh_, fem::dof::DOFOrdering::Interleaved);
		cond_.ka = desc.k_a; cond_.kb = desc.k_b;
		density_.value = desc.rho;
		cp_.value = desc.cp;
		massModel_ = MassModelT(density_, cp_);
		opModel_ = OpModelT(cond_, density_, cp_);
		diff_.ienBase = mesh_.data.ien.data();
		diff_.npe = mesh_.data.nodesPerElement;
		diff_.kElem = d.k_elem;
		stiff_ = std::make_unique<StiffnessForms>(diff_);
		const int ntags = (NSD == 2) ? 4 : 6;
		for (int t = 0; t < ntags; ++t) {
			if (!(desc.ess_mask & (1 << t))) continue;
			auto bc = std::make_shared<fem::boundary::BoundaryCondition<DirichletFn>>(fem::boundary::BoundaryCondition<DirichletFn>{t, {fem::boundary::BCCategory::Essential}, DirichletFn(DirichletCallable{desc.bc_kind, desc.bc_val[t]})});
			ess_.template registerBC<DirichletFn>(bc);
		}
		topo_->buildConstraints(basis_, ess_);
		const Index n = topo_->numFreeDOFs();
		F_ = std::make_unique<VecT>(n); U_ = std::make_unique<VecT>(n); Uprev_ = std::make_unique<VecT>(n); Udot_ = std::make_unique<VecT>(n);
		F_->zero(); U_->zero(); Uprev_->zero(); Udot_->zero();
		logCfg_.linear.type = solver::config::LoggerConfig::Type::None;
		logCfg_.nonlinear.type = solver::config::LoggerConfig::Type::None;
		logCfg_.timestepper.type = solver::config::LoggerConfig::Type::None;
		logCfg_.driver.type = solver::config::LoggerConfig::Type::None;
	}

	// ---- Problem concept (solver/problem/Problem.hpp:16-50) -----------------------------------
	// a reference to one instance: FEMOperator keeps the forms it is given by reference
	const StiffnessForms& stiffnessForms() const { return *stiff_; }
	const OpModelT& stiffnessModel() const { return opModel_; }
	TangentDiffusionForms tangentStiffnessForms() const { return {}; }
	MassForms massForms() const { return {}; }
	const MassModelT& massModel() const { return massModel_; }
	TangentMassForms tangentMassForms() const { return {}; }
	MatT createMatrix() const { return fem::assembly::Assembler<CPU>::template createMatrix<1>(mesh_, *topo_); }
	VecT createVector() const { return fem::assembly::Assembler<CPU>::template createVector<1>(mesh_, *topo_); }

	// HeatProblem.tpp:217-231
	void assembleLoad(Real time) {
		F_->zero();
		StateVectorT state;
		state.valueSource = U_.get();
		auto sel = [](StateVectorT& s) -> Real* { return s.valueBuffer(); };
		fem::assembly::Assembler<CPU>::template assembleVector<1, EvalEle, EvalQP, equation::heateq::evaluator::DefaultModel<EvalQP>, typename Fam::Quad, StateVectorT, fem::assembly::FormsWithOperand<SourceForms, decltype(sel)>>(mesh_, *topo_, time, defaultModel_, evalEle_, quad_, state, *F_, &ess_, fem::assembly::FormsWithOperand<SourceForms, decltype(sel)>{sourceForms_, sel});
	}
	// no natural boundary conditions are registered in any configuration: zero flux, no contribution
	void applyNatural(Real) {}

	template<typename FormsT, typename ModelT>
	void assembleMatrix(Real time, const FormsT& forms, const ModelT& model, StateVectorT& state, MatT& K) {
		fem::assembly::Assembler<CPU>::template assembleMatrix<1, EvalEle, EvalQP, ModelT, FormsT, typename Fam::Quad, StateVectorT>(mesh_, *topo_, time, model, forms, evalEle_, quad_, state, K, &ess_);
	}
	template<typename FormsT, typename ModelT, typename SelectorT>
	void assembleVector(Real time, const FormsT& forms, const ModelT& model, StateVectorT& state, SelectorT selector, VecT& V) {
		fem::assembly::Assembler<CPU>::template assembleVector<1, EvalEle, EvalQP, ModelT, typename Fam::Quad, StateVectorT, fem::assembly::FormsWithOperand<FormsT, SelectorT>>(mesh_, *topo_, time, model, evalEle_, quad_, state, V, &ess_, fem::assembly::FormsWithOperand<FormsT, SelectorT>{forms, selector});
	}
	template<typename FormsT, typename ModelT>
	void assembleResidual(Real time, const FormsT& forms, const ModelT& model, StateVectorT& state, VecT& R) {
		assembleVector(time, forms, model, state, [](StateVectorT& s) -> Real* { return s.valueBuffer(); }, R);
	}
	template<typename FormsT, typename ModelT>
	void applyEssential(Real time, const FormsT& forms, const ModelT& model, VecT& F) {
		fem::boundary::BoundaryApplicator<CPU>::template applyEssentialBCs<1, EvalEle, EvalQP, ModelT, FormsT, typename Fam::Quad>(mesh_, *topo_, ess_, time, model, forms, evalEle_, quad_, F);
	}
	// forwards to the runner the reference factory built and keeps the last report, which the
	// stages' own solve() discards (solver/stage/SteadyStage.hpp:281-291)
	struct ReportingRunner final : linalg::solver::LinearSolverRunner<VecT> {
		std::unique_ptr<linalg::solver::LinearSolverRunner<VecT>> inner;
		linalg::solver::SolverReport<VecT>* sink;
		double* seconds;
		bool solve(const VecT& b, VecT& x, linalg::solver::SolverReport<VecT>& report) override {
			const auto t0 = std::chrono::steady_clock::now();
			bool ok = inner->solve(b, x, report);
			*seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
			*sink = report;
			return ok;
		}
	};
	linalg::solver::SolverReport<VecT> lastReport_;
	double lastSolveSeconds_ = 0.0;
	template<typename FormsT, typename ModelT>
	std::unique_ptr<linalg::solver::LinearSolverRunner<VecT>> makeLinearRunner(const Real* time, const FormsT& forms, const ModelT& model, StateVectorT& state, MatT& K) {
		using Op = linalg::op::CSROperator<MatT>;
		using FemOp = linalg::op::FEMOperator<fem::assembly::Assembler<CPU>, topology::TopologicalDOF<1>, EvalEle, EvalQP, ModelT, FormsT, typename Fam::Quad, StateVectorT, VecT>;
		auto r = std::make_unique<ReportingRunner>();
		// HeatProblem.tpp:274-289: the operator type of the linear solver config picks CSR or matrix-free
		if (inst_.linear->operatorType == solver::config::LinearSolverConfig::OperatorType::FEM)
			r->inner = solver::linear::makeLinearSolverRunner<FemOp, VecT>(FemOp(assembler_, mesh_, *topo_, time, model, forms, evalEle_, quad_, &ess_, state), topo_->numFreeDOFs(), *inst_.linear, logCfg_.linear, equationLabel(), dofNames(), topo_->numFreeDOFs(), fem::dof::DOFOrdering::Interleaved);
		else
			r->inner = solver::linear::makeLinearSolverRunner<Op, VecT>(Op(K), topo_->numFreeDOFs(), *inst_.linear, logCfg_.linear, equationLabel(), dofNames(), topo_->numFreeDOFs(), fem::dof::DOFOrdering::Interleaved);
		r->sink = &lastReport_;
		r->seconds = &lastSolveSeconds_;
		return r;
	}
	Index numFreeDOFs() const { return topo_->numFreeDOFs(); }
	std::vector<std::string> dofNames() const { return {"T"}; }
	Index freeDOFsPerField() const { return topo_->numFreeDOFs(); }
	fem::dof::DOFOrdering dofOrdering() const { return fem::dof::DOFOrdering::Interleaved; }
	const solver::SolverInstance& solverInstance() const { return inst_; }
	std::string equationLabel() const { return "Heat Equation"; }
	const solver::config::LoggingConfig& loggingConfig() const { return logCfg_; }
	VecT& U() { return *U_; }
	VecT& F() { return *F_; }
	VecT& U_prev() { return *Uprev_; }
	VecT& Udot() { return *Udot_; }
	void advance() { linalg::operations::copy(*U_, *Uprev_); }
	void writeOutput(Index, Real) const {}
	void evaluateMonitors(Index, Real) const {}

	// ---- harness entry points ----------------------------------------------------------------
	Index numNodes() const override { return mesh_.data.numNodes; }
	Index numElems() const override { return mesh_.data.numElements; }
	Index numFree() const override { return topo_->numFreeDOFs(); }
	void dofmap(int32_t* t2a, int32_t* a2t) override {
		for (Index i = 0; i < topo_->numGlobalDOFs(); ++i) t2a[i] = topo_->getTopoToAlg()[i];
		for (Index i = 0; i < topo_->numFreeDOFs(); ++i) a2t[i] = topo_->getAlgToTopo()[i];
	}
	void mesh(double* xyz, int64_t* ien, int32_t* rng) override {
		for (size_t i = 0; i < mesh_.data.xyz.size(); ++i) xyz[i] = mesh_.data.xyz[i];
		for (size_t i = 0; i < mesh_.data.ien.size(); ++i) ien[i] = (int64_t)mesh_.data.ien[i];
		for (size_t i = 0; i < mesh_.data.rng.size(); ++i) rng[i] = mesh_.data.rng[i];
	}
	std::unique_ptr<MatT> K_;
	MatT& K() { if (!K_) K_ = std::make_unique<MatT>(createMatrix()); return *K_; }
	Index nnz() override { return K().rowPtr()[K().nRows()]; }
	void pattern(int64_t* rowPtr, int64_t* col) override {
		MatT& A = K();
		for (Index i = 0; i <= A.nRows(); ++i) rowPtr[i] = (int64_t)A.rowPtr()[i];
		for (Index p = 0; p < A.rowPtr()[A.nRows()]; ++p) col[p] = (int64_t)A.colIdx()[p];
	}

	using MassScaled = fem::form::ScaledForm<1, MassForms>;
	// formset: 0 K; 1 K + c*M; 2 K + K_T; 3 K + K_T + c*M + M_T; 4 M (mass only, rho*cp)
	template<typename Fn>
	void withForms(int formset, double c, Fn&& fn) {
		switch (formset) {
			case 0: fn(fem::form::FormRegistry<StiffnessForms>(stiffnessForms())); break;
			case 1: fn(fem::form::FormRegistry<StiffnessForms, MassScaled>(stiffnessForms(), MassScaled(c))); break;
			case 2: fn(fem::form::FormRegistry<StiffnessForms, TangentDiffusionForms>(stiffnessForms(), TangentDiffusionForms{})); break;
			case 3: fn(fem::form::FormRegistry<StiffnessForms, TangentDiffusionForms, MassScaled, TangentMassForms>(stiffnessForms(), TangentDiffusionForms{}, MassScaled(c), TangentMassForms{})); break;
			case 4: fn(MassForms{}); break;
			default: throw std::invalid_argument("formset");
		}
	}
	void loadState(const double* U, const double* Udot) {
		const Index n = numFree();
		for (Index i = 0; i < n; ++i) { U_->data()[i] = U ? U[i] : 0.0; Udot_->data()[i] = Udot ? Udot[i] : 0.0; }
	}
	void assembleMatrix(int formset, double c, const double* U, const double* Udot, double* val) override {
		loadState(U, Udot);
		StateVectorT state; state.valueSource = U_.get(); state.rateSource = Udot_.get();
		MatT& A = K();
		withForms(formset, c, [&](const auto& forms) { assembleMatrix(0.0, forms, opModel_, state, A); });
		for (Index p = 0; p < A.rowPtr()[A.nRows()]; ++p) val[p] = A.data()[p];
	}
	// which: 0 load F (source); 1 Diffusion on U (Full gather, BC values injected);
	//        2 rho*cp*Mass on U; 3 rho*cp*Mass on Udot; 4 operator formset=1 (K + coef*M) on operand (Free gather)
	void assembleVector(int which, double coef, const double* U, const double* Udot, const double* operand, double* out) override {
		loadState(U, Udot);
		const Index n = numFree();
		VecT V(n), X(n);
		if (operand) for (Index i = 0; i < n; ++i) X.data()[i] = operand[i];
		StateVectorT state; state.valueSource = U_.get(); state.rateSource = Udot_.get();
		if (operand) state.operandSource = &X;
		auto selV = [](StateVectorT& s) -> Real* { return s.valueBuffer(); };
		auto selR = [](StateVectorT& s) -> Real* { return s.rateBuffer(); };
		auto selO = [](StateVectorT& s) -> Real* { return s.operandBuffer(); };
		if (which == 0) { assembleLoad(0.0); for (Index i = 0; i < n; ++i) out[i] = F_->data()[i]; return; }
		if (which == 1) assembleVector(0.0, stiffnessForms(), opModel_, state, selV, V);
		else if (which == 2) assembleVector(0.0, massForms(), massModel_, state, selV, V);
		else if (which == 3) assembleVector(0.0, massForms(), massModel_, state, selR, V);
		else if (which == 4) withForms(1, coef, [&](const auto& forms) { assembleVector(0.0, forms, opModel_, state, selO, V); });
		else throw std::invalid_argument("which");
		for (Index i = 0; i < n; ++i) out[i] = V.data()[i];
	}
	void lift(int formset, double c, double* F) override {
		const Index n = numFree();
		VecT V(n);
		for (Index i = 0; i < n; ++i) V.data()[i] = F[i];
		withForms(formset, c, [&](const auto& forms) { applyEssential(0.0, forms, opModel_, V); });
		for (Index i = 0; i < n; ++i) F[i] = V.data()[i];
	}
	void diagonal(int formset, double c, const double* U, double* dg) override {
		loadState(U, nullptr);
		const Index n = numFree();
		VecT D(n);
		StateVectorT state; state.valueSource = U_.get(); state.rateSource = Udot_.get();
		withForms(formset, c, [&](const auto& forms) {
			using FormsT = std::decay_t<decltype(forms)>;
			fem::assembly::Assembler<CPU>::template assembleDiagonal<1, EvalEle, EvalQP, OpModelT, FormsT, typename Fam::Quad, StateVectorT>(mesh_, *topo_, 0.0, opModel_, forms, evalEle_, quad_, state, D, &ess_);
		});
		for (Index i = 0; i < n; ++i) dg[i] = D.data()[i];
	}

	void setLinear(int solverType, int precond, double tol, int64_t maxit, int64_t krylov) {
		linCfg_.type = solverType == 0 ? solver::config::LinearSolverConfig::Type::CG : solver::config::LinearSolverConfig::Type::GMRES;
		linCfg_.operatorType = opType ? solver::config::LinearSolverConfig::OperatorType::FEM : solver::config::LinearSolverConfig::OperatorType::CSR;
		linCfg_.preconditioner.type = precond ? solver::config::PreconditionerConfig::Type::Jacobi : solver::config::PreconditionerConfig::Type::Identity;
		linCfg_.tolerance = tol;
		linCfg_.maxIterations = (Index)maxit;
		if (solverType != 0) { solver::config::GMRESParams gp; gp.krylovDim = (Index)krylov; linCfg_.params = gp; }
	}

	// SteadyStage linear mode (solver/stage/SteadyStage.hpp:60-84) driven as Steady::solve does
	int steady(int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, ref_report* rep) override {
		setLinear(solverType, precond, tol, maxit, krylov);
		inst_.mode = solver::SolverMode::SteadyLinear; inst_.linear = &linCfg_; inst_.nonlinear = nullptr; inst_.timestepper = nullptr;
		loadState(U, nullptr);
		solver::stage::SteadyStage<RefHeatProblem> stage(*this);
		stage.assemble();
		bool ok = stage.solve();
		const auto& report = lastReport_;
		if (rep) { rep->converged = ok; rep->iterations = (int64_t)report.iterations; rep->initialResidual = report.initialResidual; rep->finalResidual = report.finalResidual; rep->finalResidualRel = report.finalResidualRel; }
		for (Index i = 0; i < numFree(); ++i) U[i] = U_->data()[i];
		return ok ? 0 : 1;
	}

	// SteadyStage nonlinear mode + NewtonRunner (solver/nonlinear/Newton.hpp:32-83)
	int newton(double absTol, double relTol, int64_t maxit, int solverType, int precond, double tol, int64_t linMaxit, int64_t krylov, double* U, ref_report* rep) override {
		setLinear(solverType, precond, tol, linMaxit, krylov);
		nlCfg_.type = solver::config::NonlinearSolverConfig::Type::Newton;
		nlCfg_.absoluteTolerance = absTol; nlCfg_.relativeTolerance = relTol; nlCfg_.maxIterations = (Index)maxit;
		nlCfg_.linearSolver = linCfg_;
		inst_.mode = solver::SolverMode::SteadyNonlinear; inst_.linear = &nlCfg_.linearSolver; inst_.nonlinear = &nlCfg_; inst_.timestepper = nullptr;
		loadState(U, nullptr);
		solver::stage::SteadyStage<RefHeatProblem> stage(*this);
		linalg::solver::SolverReport<VecT> report;
		auto runner = solver::nonlinear::makeNonlinearSolverRunner<solver::stage::SteadyStage<RefHeatProblem>, VecT>(stage, nlCfg_, logCfg_.nonlinear, equationLabel(), dofNames(), numFree(), fem::dof::DOFOrdering::Interleaved);
		bool ok = runner->solve(report);
		if (rep) { rep->converged = ok; rep->iterations = (int64_t)report.iterations; rep->initialResidual = report.initialResidual; rep->finalResidual = report.finalResidual; rep->finalResidualRel = report.finalResidualRel; }
		for (Index i = 0; i < numFree(); ++i) U[i] = U_->data()[i];
		return ok ? 0 : 1;
	}

	// BackwardEulerStage + BackwardEulerRunner (solver/timestepper/BackwardEuler.hpp:32-70), linear mode
	// stepStats (optional, 3 per step): wall seconds of runner.step(), of its linear solve, CG iterations
	int backwardEuler(double dt, int64_t nsteps, int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, double* residualPerStep, double* stepStats) override {
		setLinear(solverType, precond, tol, maxit, krylov);
		tsCfg_.type = solver::config::TimeStepperConfig::Type::BackwardEuler;
		tsCfg_.t0 = 0.0; tsCfg_.tf = dt * (double)nsteps;
		tsCfg_.stepSize.dt = dt;
		tsCfg_.linearSolver = linCfg_;
		inst_.mode = solver::SolverMode::TransientLinear; inst_.linear = &linCfg_; inst_.nonlinear = nullptr; inst_.timestepper = &tsCfg_;
		loadState(U, nullptr);
		linalg::operations::copy(*U_, *Uprev_);
		solver::stage::BackwardEulerStage<RefHeatProblem> stage(*this);
		solver::timestepper::BackwardEulerRunner<solver::stage::BackwardEulerStage<RefHeatProblem>> runner(stage, tsCfg_, std::make_unique<solver::timestepper::ConstantStepSizePolicy>(dt), utils::logging::timestepper::Logger(utils::logging::NullLogger{}));
		int rc = 0;
		for (int64_t s = 0; s < nsteps && !runner.finished(); ++s) {
			const auto t0 = std::chrono::steady_clock::now();
			if (!runner.step()) { rc = 1; break; }
			const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
			if (stepStats) {
				stepStats[3 * s] = secs;
				stepStats[3 * s + 1] = lastSolveSeconds_;
				stepStats[3 * s + 2] = (double)lastReport_.iterations;
			}
			if (residualPerStep) residualPerStep[s] = stage.residualNorm();
		}
		for (Index i = 0; i < numFree(); ++i) U[i] = U_->data()[i];
		return rc;
	}

	// HeatProblem::computeNodalField (HeatProblem.tpp:293-303): the reference QuantityEvaluator with
	// SimpleAverageRecovery over the operator model; field 0 HeatFluxField, 1 ConductivityField
	void nodalField(int field, const double* U, double* out) override {
		loadState(U, nullptr);
		StateVectorT state;
		state.valueSource = U_.get();
		auto run = [&](auto fld) {
			using FieldT = decltype(fld);
			fem::quantity::QuantityEvaluator<CPU>::template evaluateNodalField<1, EvalEle, EvalQP, OpModelT, FieldT, typename Fam::Quad, fem::quantity::recovery::SimpleAverageRecovery, StateVectorT>(mesh_, *topo_, ess_, 0.0, opModel_, fld, evalEle_, quad_, state, fem::quantity::recovery::SimpleAverageRecovery{}, out);
		};
		if (field == 0) run(equation::heateq::evaluator::HeatFluxField<NSD>{});
		else run(equation::heateq::evaluator::ConductivityField{});
	}

	// HeatFlux monitors, one group per call: method 1 Strong (BoundaryQuadratureMonitorGroup over
	// ReducedQuantity<HeatFluxIntegrand, mode>), 0 Weak (BoundaryReactionMonitorGroup over the source,
	// the negated stiffness on the value and, when transient, the negated mass on the rate), each tag one
	// combination with coefficient 1 (MonitorConfig::terms)
	void boundaryFlux(int method, int reduction, int transient, int ntags, const int32_t* tags, const double* U, const double* Udot, double* values) override {
		using Traits = fem::dispatch::ElementTypeTraits<NSD == 2 ? mesh::ElementFamily::Quad : mesh::ElementFamily::Hex>;
		using QuadBdy = typename Traits::QuadratureBoundaryType;
		using EvalQPB = equation::heateq::evaluator::EvalQuadraturePointBoundary<EvalEle, typename Fam::Basis, fem::geometry::JacobianTransform<NSD, NSD>>;
		using BdyState = equation::heateq::evaluator::HeatBoundaryStateVector<1, NSD, NSD, VecT>;
		using CondBdy = LinearConductivity<EvalQPB>;
		const QuadBdy quadBdy = [&] { if constexpr (NSD == 2) return QuadBdy(d.nq); else return QuadBdy(d.nq, d.nq); }();
		loadState(U, Udot);
		auto collect = [&](fem::quantity::MonitorGroup& group) {
			for (int t = 0; t < ntags; ++t) {
				group.registerTag(tags[t]);
				const Index c = group.addCombination();
				group.addTerm(c, tags[t], 1.0);
			}
			group.evaluate(0.0, [&](Index c, const Real* v) { values[c] = v[0]; });
		};
		const auto mode = reduction ? fem::quantity::Reduction::Average : fem::quantity::Reduction::Integral;
		if (method == 1) {
			CondBdy condBdy = CondBdy{cond_.ka, cond_.kb};
			BdyState state;
			state.valueSource = U_.get();
			auto run = [&](auto tagMode) {
				constexpr auto M = decltype(tagMode)::value;
				using QF = fem::quantity::QuantityForms<fem::quantity::ReducedQuantity<equation::heateq::quantity::HeatFluxIntegrand<EvalQPB>, M>>;
				fem::quantity::BoundaryQuadratureMonitorGroup<CPU, 1, EvalEle, EvalQPB, CondBdy, QF, QuadBdy, BdyState> group(mesh_, *topo_, ess_, condBdy, QF{}, evalEle_, quadBdy, state);
				collect(group);
			};
			if (reduction) run(std::integral_constant<fem::quantity::Reduction, fem::quantity::Reduction::Average>{});
			else run(std::integral_constant<fem::quantity::Reduction, fem::quantity::Reduction::Integral>{});
			return;
		}
		StateVectorT state;
		state.valueSource = U_.get();
		state.rateSource = Udot_.get();
		auto selV = [](StateVectorT& s) -> Real* { return s.valueBuffer(); };
		auto selR = [](StateVectorT& s) -> Real* { return s.rateBuffer(); };
		using SrcForm = std::decay_t<decltype(sourceForms_.template get<0>())>;
		using NegStiff = fem::form::ScaledForm<1, StiffnessForms>;
		using NegMass = fem::form::ScaledForm<1, MassForms>;
		using SrcPair = fem::assembly::FormsWithOperand<SrcForm, decltype(selV)>;
		using StiffPair = fem::assembly::FormsWithOperand<NegStiff, decltype(selV)>;
		using MassPair = fem::assembly::FormsWithOperand<NegMass, decltype(selR)>;
		const NegStiff negStiff(Real(-1));
		const NegMass negMass(Real(-1));
		if (transient) {
			fem::quantity::BoundaryReactionMonitorGroup<CPU, 1, EvalEle, EvalQP, EvalQPB, OpModelT, typename Fam::Quad, QuadBdy, StateVectorT, SrcPair, StiffPair, MassPair> group(
				mesh_, *topo_, ess_, opModel_, evalEle_, quad_, quadBdy, state, mode, SrcPair{sourceForms_.template get<0>(), selV}, StiffPair{negStiff, selV}, MassPair{negMass, selR});
			collect(group);
		} else {
			fem::quantity::BoundaryReactionMonitorGroup<CPU, 1, EvalEle, EvalQP, EvalQPB, OpModelT, typename Fam::Quad, QuadBdy, StateVectorT, SrcPair, StiffPair> group(
				mesh_, *topo_, ess_, opModel_, evalEle_, quad_, quadBdy, state, mode, SrcPair{sourceForms_.template get<0>(), selV}, StiffPair{negStiff, selV});
			collect(group);
		}
	}

	// dJ/dk_e contribution lam_e^T Khat_e T_e for every element, with Khat_e the unit-conductivity
	// element stiffness built by the reference QP evaluator and DiffusionForm; T and lam are free
	// vectors (constrained entries contribute their Dirichlet value for T and zero for lam).
	void adjointGradient(const double* T, const double* lam, double* grad) override {
		const Index npe = mesh_.data.nodesPerElement;
		constexpr Index maxN = fem::dispatch::kMaxNodesPerElement<NSD>;
		Real xi[fem::dispatch::kMaxQuadraturePointsTotal<NSD> * NSD], w[fem::dispatch::kMaxQuadraturePointsTotal<NSD>];
		quad_.getPoints(xi); quad_.getWeights(w);
		loadState(T, nullptr);
		VecT L(numFree());
		for (Index i = 0; i < numFree(); ++i) L.data()[i] = lam[i];
		EvalEle ele = evalEle_;
		Cond unit; unit.ka = 1.0; unit.kb = 0.0;
		for (Index e = 0; e < mesh_.data.numElements; ++e) {
			Real Ke[maxN * maxN]; std::memset(Ke, 0, sizeof(Ke));
			const Index* nodes = mesh_.getElementNodes(e);
			Real coords[NSD * maxN];
			fem::assembly::gatherElementCoords<NSD>(mesh_, nodes, npe, coords);
			Real Te[maxN] = {0}, Le[maxN] = {0};
			fem::assembly::gatherElementVector<1, NSD, fem::assembly::GatherMode::Full>(nodes, npe, coords, *topo_, &ess_, 0.0, Te, U_.get());
			fem::assembly::gatherElementVector<1, NSD, fem::assembly::GatherMode::Free>(nodes, npe, coords, *topo_, &ess_, 0.0, Le, &L);
			ele.bindElement(coords, 0.0);
			EvalQP qp(ele);
			for (Index q = 0; q < quad_.numPointsTotal(); ++q) {
				qp.evaluate(&xi[NSD * q], w[q]);
				unit.eval(qp);
				equation::heateq::DiffusionForm<EvalQP>::computeElementLevelMatrix(qp, Ke);
			}
			Real g = 0;
			for (Index a = 0; a < npe; ++a) for (Index b = 0; b < npe; ++b) g += Le[a] * Ke[a * npe + b] * Te[b];
			grad[e] = g;
		}
	}
};

thread_local std::string g_err;

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void* ref_create(const ref_desc* d) {
	try {
		if (d->nsd == 2) return static_cast<Base*>(new RefHeatProblem<2>(*d));
		if (d->nsd == 3) return static_cast<Base*>(new RefHeatProblem<3>(*d));
		g_err = "nsd must be 2 or 3";
	} catch (const std::exception& e) { g_err = e.what(); }
	return nullptr;
}
void ref_destroy(void* h) { delete static_cast<Base*>(h); }
void ref_set_operator(void* h, int op) { static_cast<Base*>(h)->opType = op; }
void ref_nodal_field(void* h, int field, const double* U, double* out) { static_cast<Base*>(h)->nodalField(field, U, out); }
int64_t ref_num_nodes(void* h) { return (int64_t)static_cast<Base*>(h)->numNodes(); }
int64_t ref_num_elems(void* h) { return (int64_t)static_cast<Base*>(h)->numElems(); }
int64_t ref_num_free(void* h) { return (int64_t)static_cast<Base*>(h)->numFree(); }
void ref_dofmap(void* h, int32_t* t2a, int32_t* a2t) { static_cast<Base*>(h)->dofmap(t2a, a2t); }
void ref_mesh(void* h, double* xyz, int64_t* ien, int32_t* rng) { static_cast<Base*>(h)->mesh(xyz, ien, rng); }
int64_t ref_nnz(void* h) { return (int64_t)static_cast<Base*>(h)->nnz(); }
void ref_pattern(void* h, int64_t* rowPtr, int64_t* col) { static_cast<Base*>(h)->pattern(rowPtr, col); }
void ref_assemble_matrix(void* h, int formset, double c, const double* U, const double* Udot, double* val) { static_cast<Base*>(h)->assembleMatrix(formset, c, U, Udot, val); }
void ref_assemble_vector(void* h, int which, double coef, const double* U, const double* Udot, const double* operand, double* out) { static_cast<Base*>(h)->assembleVector(which, coef, U, Udot, operand, out); }
void ref_lift(void* h, int formset, double c, double* F) { static_cast<Base*>(h)->lift(formset, c, F); }
void ref_diagonal(void* h, int formset, double c, const double* U, double* d) { static_cast<Base*>(h)->diagonal(formset, c, U, d); }
int ref_steady(void* h, int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, ref_report* rep) {
	try { return static_cast<Base*>(h)->steady(solverType, precond, tol, maxit, krylov, U, rep); } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int ref_newton(void* h, double absTol, double relTol, int64_t maxit, int solverType, int precond, double tol, int64_t linMaxit, int64_t krylov, double* U, ref_report* rep) {
	try { return static_cast<Base*>(h)->newton(absTol, relTol, maxit, solverType, precond, tol, linMaxit, krylov, U, rep); } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int ref_backward_euler(void* h, double dt, int64_t nsteps, int solverType, int precond, double tol, int64_t maxit, int64_t krylov, double* U, double* resPerStep, double* stepStats) {
	try { return static_cast<Base*>(h)->backwardEuler(dt, nsteps, solverType, precond, tol, maxit, krylov, U, resPerStep, stepStats); } catch (const std::exception& e) { g_err = e.what(); return -1; }
}
void ref_adjoint_gradient(void* h, const double* T, const double* lam, double* grad) { static_cast<Base*>(h)->adjointGradient(T, lam, grad); }
int ref_boundary_flux(void* h, int method, int reduction, int transient, int ntags, const int32_t* tags, const double* U, const double* Udot, double* values) {
	try { static_cast<Base*>(h)->boundaryFlux(method, reduction, transient, ntags, tags, U, Udot, values); return 0; } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

// Generic CSR solve through the reference cg::Solver / gmres::Solver (linalg/solver/iterative/*),
// Jacobi or Identity preconditioning, NullLogger.  Row pointers and columns are 64-bit like the
// reference's Index.
int ref_csr_solve(int solverType, int precond, int64_t n, const int64_t* rowPtr, const int64_t* col, const double* val,
                  const double* b, double* x, double tol, int64_t maxit, int64_t krylov, ref_report* rep) {
	MatT A((Index)n, (Index)n);
	for (int64_t i = 0; i <= n; ++i) A.rowPtr()[i] = (Index)rowPtr[i];
	A.resize((Index)rowPtr[n]);
	for (int64_t p = 0; p < rowPtr[n]; ++p) { A.colIdx()[p] = (Index)col[p]; A.data()[p] = val[p]; }
	VecT B((Index)n), X((Index)n);
	for (int64_t i = 0; i < n; ++i) { B.data()[i] = b[i]; X.data()[i] = x[i]; }
	using Op = linalg::op::CSROperator<MatT>;
	Op op(A);
	utils::logging::NullLogger logger;
	linalg::solver::SolverReport<VecT> report;
	bool ok;
	auto run = [&](auto& M) {
		using PrecT = std::decay_t<decltype(M)>;
		if (solverType == 0) {
			using S = linalg::solver::iterative::cg::Solver<Op, VecT, PrecT, utils::logging::NullLogger>;
			typename S::Config cfg; cfg.tol = tol; cfg.maxIters = (Index)maxit;
			typename S::Workspace W((Index)n);
			S s(cfg);
			ok = s.solve(report, logger, W, M, op, B, X);
		} else {
			using S = linalg::solver::iterative::gmres::Solver<Op, VecT, PrecT, utils::logging::NullLogger>;
			typename S::Config cfg; cfg.tol = tol; cfg.maxIters = (Index)maxit; cfg.krylovDim = (Index)krylov;
			typename S::Workspace W((Index)n, (Index)krylov);
			S s(cfg);
			ok = s.solve(report, logger, W, M, op, B, X);
		}
	};
	if (precond) { linalg::solver::preconditioner::Jacobi<VecT> M; run(M); }
	else { linalg::solver::preconditioner::Identity<VecT> M; run(M); }
	for (int64_t i = 0; i < n; ++i) x[i] = X.data()[i];
	if (rep) { rep->converged = ok; rep->iterations = (int64_t)report.iterations; rep->initialResidual = report.initialResidual; rep->finalResidual = report.finalResidual; rep->finalResidualRel = report.finalResidualRel; }
	return ok ? 0 : 1;
}

// reference CSR SpMV (linalg/operations/backend/cpu/MatrixOps.tpp:5-23)
void ref_spmv(int64_t n, const int64_t* rowPtr, const int64_t* col, const double* val, const double* x, double* y) {
	MatT A((Index)n, (Index)n);
	for (int64_t i = 0; i <= n; ++i) A.rowPtr()[i] = (Index)rowPtr[i];
	A.resize((Index)rowPtr[n]);
	for (int64_t p = 0; p < rowPtr[n]; ++p) { A.colIdx()[p] = (Index)col[p]; A.data()[p] = val[p]; }
	VecT X((Index)n), Y((Index)n);
	for (int64_t i = 0; i < n; ++i) X.data()[i] = x[i];
	linalg::operations::matvec(A, X, Y);
	for (int64_t i = 0; i < n; ++i) y[i] = Y.data()[i];
}

} // extern "C"
