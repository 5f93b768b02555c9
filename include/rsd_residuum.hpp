// rsd_residuum.hpp - the B200 backend as a Residuum `Backend` tag (C++20).
//
// Include this header (with the Residuum `include/` directory on the include path) before
// instantiating any Residuum linear-algebra template with the tag `rsd::residuum::B200`:
//
//     using Vec = residuum::linalg::types::Vector<double, rsd::residuum::B200>;
//     using Mat = residuum::linalg::types::CSRMatrix<double, rsd::residuum::B200>;
//     using Op  = residuum::linalg::op::CSROperator<Mat>;
//     using M   = residuum::linalg::solver::preconditioner::Jacobi<Vec>;
//     residuum::linalg::solver::iterative::cg::Solver<Op, Vec, M, NullLogger> s(cfg);   // unmodified
//
// What it provides, all forwarding to the C ABI in rsd.h:
//   * B200: the tag's memory interface (Ptr / alloc / copy / zero / set), the same shape as the
//     reference's CPU and CUDA tags (linalg/types/backend/CPU.hpp:15-40, CUDA.hpp:23-73), on one
//     process-wide rsd context (device 0 unless B200::use() names another);
//   * CSRMatrix<T, B200>: a device CSR matrix (an rsd_csr: 32-bit indices, SELL-32 execution layout),
//     built from the reference's host CSRMatrix<T, CPU> (linalg/types/CSRMatrix.hpp:14-88) or taken
//     over from the C ABI (the heat problem's createMatrix);
//   * explicit specializations of operations::dot/axpy/axpby/scal/copy/multiply/norm
//     (linalg/operations/VectorOps.hpp:10-36) and operations::matvec/lump (MatrixOps.hpp:10-16) for
//     the tag's vector and matrix;
//   * CSROperator<CSRMatrix<double, B200>> (linalg/operator/CSROperator.hpp:14-48) and
//     Jacobi<Vector<double, B200>> (linalg/solver/preconditioner/Jacobi.hpp:15-50), whose reference
//     versions read matrix entries on the host.
// Errors throw std::runtime_error with the library's message, as the reference's CUDA tag throws.
// The heat problem itself on the tag is in rsd_residuum_heat.hpp.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rsd.h"

#include "core/Types.hpp"
#include "linalg/types/Vector.hpp"
#include "linalg/types/CSRMatrix.hpp"
#include "linalg/types/backend/cuda/CopyKind.hpp"
#include "linalg/operations/VectorOps.hpp"
#include "linalg/operations/MatrixOps.hpp"
#include "linalg/operator/CSROperator.hpp"
#include "linalg/solver/preconditioner/Jacobi.hpp"

namespace rsd::residuum {

inline void check(int rc) {
	if (rc != RSD_OK) throw std::runtime_error(std::string("rsd: ") + rsd_last_error_string());
}

class B200 {
public:
	// the context every tag operation runs on; created on first use on device 0
	static rsd_ctx* ctx() {
		rsd_ctx*& c = slot();
		if (!c) check(rsd_ctx_create(0, &c));
		return c;
	}
	// run the tag on an existing context (owned by the caller)
	static void use(rsd_ctx* c) { slot() = c; }

	template <typename T>
	struct Deleter {
		void operator()(T* p) const noexcept {
			if (p) rsd_free(ctx(), p);
		}
	};
	template <typename T>
	using Ptr = std::unique_ptr<T, Deleter<T>>;

	// vectors live in device-resident managed memory: the reference's NewtonRunner reads the stage
	// residual's entries on the host (solver/nonlinear/Newton.hpp:45), which plain device memory
	// would not allow; kernels see ordinary device memory
	template <typename T>
	static Ptr<T> alloc(Index n) {
		void* p = nullptr;
		check(rsd_alloc_managed(ctx(), sizeof(T) * (n ? n : 1), &p));
		return Ptr<T>(static_cast<T*>(p));
	}
	template <typename T>
	static void copy(T* dst, const T* src, Index n, ::residuum::linalg::types::backend::CopyKind kind) {
		check(rsd_memcpy(ctx(), dst, src, sizeof(T) * n, static_cast<int32_t>(kind)));
	}
	template <typename T>
	static void zero(T* p, Index n) {
		check(rsd_memset_zero(ctx(), p, sizeof(T) * n));
	}
	template <typename T>
	static void set(T* p, Index n, T v) {
		if constexpr (sizeof(T) == 8) check(rsd_fill_f64(ctx(), reinterpret_cast<double*>(p), (int64_t)n, (double)v));
		else check(rsd_fill_f32(ctx(), reinterpret_cast<float*>(p), (int64_t)n, (float)v));
	}

private:
	static rsd_ctx*& slot() {
		static rsd_ctx* c = nullptr;
		return c;
	}
};

}  // namespace rsd::residuum

namespace residuum::linalg::types {

// Device CSR matrix of the B200 tag.  The pattern and values come from the reference's host
// matrix; values can be replaced later with the same pattern.
template <typename T>
class CSRMatrix<T, rsd::residuum::B200> {
	static_assert(sizeof(T) == 8, "the B200 CSR matrix holds FP64 values");

public:
	using value_type = T;
	using backend_type = rsd::residuum::B200;

	// an empty matrix (the stages' MatrixT(0, 0) when no matrix is assembled)
	CSRMatrix(Index nRows, Index nCols) : nRows_(nRows), nCols_(nCols) {}
	// takes ownership of a device matrix from the C ABI (rsd_heat_create_matrix, rsd_csr_create)
	explicit CSRMatrix(rsd_csr* A) {
		int64_t n = 0, nnz = 0;
		rsd::residuum::check(rsd_csr_info(A, &n, &nnz));
		nRows_ = nCols_ = (Index)n;
		nNnz_ = (Index)nnz;
		A_.reset(A);
	}
	explicit CSRMatrix(const CSRMatrix<T, backend::CPU>& host) : nRows_(host.nRows()), nCols_(host.nCols()) {
		const Index nnz = host.rowPtr()[nRows_];
		std::vector<int64_t> rp(nRows_ + 1), col(nnz ? nnz : 1);
		for (Index i = 0; i <= nRows_; ++i) rp[i] = (int64_t)host.rowPtr()[i];
		for (Index p = 0; p < nnz; ++p) col[p] = (int64_t)host.colIdx()[p];
		rsd_csr* A = nullptr;
		rsd::residuum::check(rsd_csr_create(rsd::residuum::B200::ctx(), (int64_t)nRows_, (int64_t)nnz, rp.data(), col.data(),
		                                    reinterpret_cast<const double*>(host.data()), &A));
		A_.reset(A);
		nNnz_ = nnz;
	}
	CSRMatrix(const CSRMatrix&) = delete;
	CSRMatrix& operator=(const CSRMatrix&) = delete;
	CSRMatrix(CSRMatrix&&) noexcept = default;
	CSRMatrix& operator=(CSRMatrix&&) noexcept = default;

	Index nRows() const { return nRows_; }
	Index nCols() const { return nCols_; }
	Index nnz() const { return nNnz_; }
	rsd_csr* handle() const { return A_.get(); }

	// new values for the same pattern, from a host matrix in CSR order
	void setValues(const CSRMatrix<T, backend::CPU>& host) {
		rsd::residuum::check(rsd_csr_set_values(rsd::residuum::B200::ctx(), A_.get(), reinterpret_cast<const double*>(host.data())));
	}
	// CSR-order values back to the host
	std::vector<T> values() const {
		std::vector<T> v(nNnz_);
		rsd::residuum::check(rsd_csr_get_values(rsd::residuum::B200::ctx(), A_.get(), reinterpret_cast<double*>(v.data())));
		return v;
	}

private:
	struct Destroy {
		void operator()(rsd_csr* A) const noexcept { rsd_csr_destroy(A); }
	};
	Index nRows_ = 0, nCols_ = 0, nNnz_ = 0;
	std::unique_ptr<rsd_csr, Destroy> A_;
};

}  // namespace residuum::linalg::types

namespace residuum::linalg::operations {

using B200Vec = types::Vector<double, rsd::residuum::B200>;
using B200Mat = types::CSRMatrix<double, rsd::residuum::B200>;

template <>
inline double dot<B200Vec>(const B200Vec& x, const B200Vec& y) {
	double r = 0.0;
	rsd::residuum::check(rsd_dot(rsd::residuum::B200::ctx(), (int64_t)x.size(), x.data(), y.data(), &r));
	return r;
}
template <>
inline void axpy<B200Vec>(const double alpha, const B200Vec& x, B200Vec& y) {
	rsd::residuum::check(rsd_axpy(rsd::residuum::B200::ctx(), (int64_t)y.size(), alpha, x.data(), y.data()));
}
template <>
inline void axpby<B200Vec>(const double alpha, const double beta, const B200Vec& x, B200Vec& y) {
	rsd::residuum::check(rsd_axpby(rsd::residuum::B200::ctx(), (int64_t)y.size(), alpha, beta, x.data(), y.data()));
}
template <>
inline void scal<B200Vec>(const double alpha, B200Vec& x) {
	rsd::residuum::check(rsd_scal(rsd::residuum::B200::ctx(), (int64_t)x.size(), alpha, x.data()));
}
template <>
inline void copy<B200Vec>(const B200Vec& x, B200Vec& y) {
	rsd::residuum::check(rsd_copy(rsd::residuum::B200::ctx(), (int64_t)x.size(), x.data(), y.data()));
}
template <>
inline void multiply<B200Vec>(const B200Vec& x, const B200Vec& y, B200Vec& z) {
	rsd::residuum::check(rsd_mul(rsd::residuum::B200::ctx(), (int64_t)z.size(), x.data(), y.data(), z.data()));
}
template <>
inline double norm<B200Vec>(const B200Vec& x) {
	double r = 0.0;
	rsd::residuum::check(rsd_nrm2(rsd::residuum::B200::ctx(), (int64_t)x.size(), x.data(), &r));
	return r;
}
template <>
inline void matvec<B200Mat, B200Vec>(const B200Mat& A, const B200Vec& x, B200Vec& y) {
	rsd::residuum::check(rsd_spmv(rsd::residuum::B200::ctx(), A.handle(), x.data(), y.data()));
}
template <>
inline void lump<B200Mat, B200Vec>(const B200Mat& A, B200Vec& d) {
	rsd::residuum::check(rsd_csr_lump(rsd::residuum::B200::ctx(), A.handle(), d.data()));
}

}  // namespace residuum::linalg::operations

namespace residuum::linalg::op {

template <>
class CSROperator<types::CSRMatrix<double, rsd::residuum::B200>> {
public:
	using MatrixT = types::CSRMatrix<double, rsd::residuum::B200>;
	using value_type = double;

	const MatrixT& A;

	explicit CSROperator(const MatrixT& mat) : A(mat) {}

	template <typename VectorT>
	void apply(const VectorT& x, VectorT& y) const {
		operations::matvec(A, x, y);
	}
	Index size() const { return A.nRows(); }
	Index flopsPerApply() const { return 2 * A.nnz(); }
	template <typename VectorT>
	void diagonal(VectorT& d) const {
		rsd::residuum::check(rsd_csr_diagonal(rsd::residuum::B200::ctx(), A.handle(), d.data()));
	}
};

}  // namespace residuum::linalg::op

namespace residuum::linalg::solver::preconditioner {

// Jacobi::update/apply (Jacobi.hpp:23-40) on the device: invD = |d| > 1e-300 ? 1/d : 1, z = r .* invD
template <>
class Jacobi<types::Vector<double, rsd::residuum::B200>> {
public:
	using VectorT = types::Vector<double, rsd::residuum::B200>;
	using DataType = double;

	Jacobi() = default;

	template <typename OperatorT>
	requires linalg::op::DiagonalExtractable<OperatorT, VectorT>
	void update(const OperatorT& A) {
		if (!invDiag_) invDiag_ = std::make_unique<VectorT>(A.size());
		rsd::residuum::check(rsd_jacobi_setup(rsd::residuum::B200::ctx(), A.A.handle(), invDiag_->data()));
	}
	void apply(const VectorT& r, VectorT& z) { operations::multiply(r, *invDiag_, z); }
	Index flopsPerApply() const { return invDiag_ ? invDiag_->size() : Index(0); }

private:
	std::unique_ptr<VectorT> invDiag_;
};

}  // namespace residuum::linalg::solver::preconditioner
