// Test infrastructure, not product code.
//
// A project-written stand-in for the exprtk header library, which the reference includes as
// <exprtk.hpp> for its expression-driven models and boundary data but does not vendor (its CI
// fetches exprtk's master branch, no version pinned).  It implements only the part of exprtk's
// interface the reference calls:
//
//   symbol_table<T>::add_variable(name, T&), add_constants()          (pi, epsilon, inf)
//   expression<T>::register_symbol_table(table), value()
//   parser<T>::compile(source, expression) -> bool, error()
//
// (include/equation/heateq/evaluator/TemperatureExpression.hpp:38-58,
//  src/utils/expression/ScalarExpression.cpp:3-30, src/utils/expression/VectorExpression.cpp)
//
// over the expression subset the reference's configurations use: numbers, bound variables and
// constants, + - * / ^, unary minus and plus, parentheses, and the one-argument functions sin cos tan
// exp log sqrt abs.  Precedence follows the usual rules (^ above unary minus above * / above + -;
// -x^2 = -(x^2)).  A compiled expression is a postfix program whose variable slots point at the
// variables bound in the symbol table, so value() reads their current values, as exprtk's does.
// Anything outside the subset fails to compile with a message.
#pragma once

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace exprtk {

template <typename T>
class symbol_table {
public:
	bool add_variable(const std::string& name, T& ref) {
		vars_[name] = &ref;
		return true;
	}
	bool add_constant(const std::string& name, T value) {
		consts_[name] = value;
		return true;
	}
	bool add_constants() {
		add_constant("pi", T(3.14159265358979323846264338327950288L));
		add_constant("epsilon", std::numeric_limits<T>::epsilon());
		add_constant("inf", std::numeric_limits<T>::infinity());
		return true;
	}
	const T* variable(const std::string& name) const {
		auto it = vars_.find(name);
		return it == vars_.end() ? nullptr : it->second;
	}
	bool constant(const std::string& name, T& out) const {
		auto it = consts_.find(name);
		if (it == consts_.end()) return false;
		out = it->second;
		return true;
	}

private:
	std::map<std::string, T*> vars_;
	std::map<std::string, T> consts_;
};

namespace details {
enum class op { constant, variable, add, sub, mul, div, pow, neg, sin, cos, tan, exp, log, sqrt, abs };
template <typename T>
struct instruction {
	op code;
	T value = T(0);           // constant
	const T* var = nullptr;   // variable
};
template <typename T>
struct program {
	std::vector<instruction<T>> code;
	T run() const {
		std::vector<T> st;
		st.reserve(code.size());
		for (const auto& in : code) {
			switch (in.code) {
				case op::constant: st.push_back(in.value); break;
				case op::variable: st.push_back(*in.var); break;
				case op::neg: st.back() = -st.back(); break;
				case op::sin: st.back() = std::sin(st.back()); break;
				case op::cos: st.back() = std::cos(st.back()); break;
				case op::tan: st.back() = std::tan(st.back()); break;
				case op::exp: st.back() = std::exp(st.back()); break;
				case op::log: st.back() = std::log(st.back()); break;
				case op::sqrt: st.back() = std::sqrt(st.back()); break;
				case op::abs: st.back() = std::abs(st.back()); break;
				default: {
					const T b = st.back();
					st.pop_back();
					T& a = st.back();
					if (in.code == op::add) a = a + b;
					else if (in.code == op::sub) a = a - b;
					else if (in.code == op::mul) a = a * b;
					else if (in.code == op::div) a = a / b;
					else a = std::pow(a, b);
				}
			}
		}
		return st.empty() ? std::numeric_limits<T>::quiet_NaN() : st.back();
	}
};
}  // namespace details

template <typename T>
class expression {
public:
	void register_symbol_table(symbol_table<T>& table) { tables_.push_back(&table); }
	T value() const { return prog_ ? prog_->run() : std::numeric_limits<T>::quiet_NaN(); }

private:
	template <typename>
	friend class parser;
	std::vector<const symbol_table<T>*> tables_;
	std::shared_ptr<const details::program<T>> prog_;
};

template <typename T>
class parser {
public:
	bool compile(const std::string& source, expression<T>& expr) {
		src_ = source;
		pos_ = 0;
		error_.clear();
		tables_ = &expr.tables_;
		auto prog = std::make_shared<details::program<T>>();
		out_ = &prog->code;
		sum();
		ws();
		if (error_.empty() && pos_ != src_.size()) fail("unexpected '" + src_.substr(pos_, 1) + "'");
		if (error_.empty() && prog->code.empty()) fail("empty expression");
		out_ = nullptr;
		tables_ = nullptr;
		if (!error_.empty()) {
			expr.prog_.reset();
			return false;
		}
		expr.prog_ = std::move(prog);
		return true;
	}
	std::string error() const { return error_; }

private:
	using op = details::op;
	void fail(const std::string& msg) {
		if (error_.empty()) error_ = "ERR at position " + std::to_string(pos_) + ": " + msg;
	}
	void emit(op code, T value = T(0), const T* var = nullptr) { out_->push_back({code, value, var}); }
	void ws() {
		while (pos_ < src_.size() && std::isspace((unsigned char)src_[pos_])) ++pos_;
	}
	char peek() {
		ws();
		return pos_ < src_.size() ? src_[pos_] : '\0';
	}
	void sum() {
		product();
		for (char c = peek(); error_.empty() && (c == '+' || c == '-'); c = peek()) {
			++pos_;
			product();
			emit(c == '+' ? op::add : op::sub);
		}
	}
	void product() {
		signed_factor();
		for (char c = peek(); error_.empty() && (c == '*' || c == '/'); c = peek()) {
			++pos_;
			signed_factor();
			emit(c == '*' ? op::mul : op::div);
		}
	}
	void signed_factor() {
		const char c = peek();
		if (c == '-' || c == '+') {
			++pos_;
			signed_factor();
			if (c == '-') emit(op::neg);
			return;
		}
		power();
	}
	void power() {
		primary();
		if (error_.empty() && peek() == '^') {
			++pos_;
			signed_factor();
			emit(op::pow);
		}
	}
	void primary() {
		const char c = peek();
		if (c == '(') {
			++pos_;
			sum();
			if (peek() != ')') return fail("missing ')'");
			++pos_;
			return;
		}
		if (std::isdigit((unsigned char)c) || c == '.') {
			const char* begin = src_.c_str() + pos_;
			char* end = nullptr;
			const double v = std::strtod(begin, &end);
			if (end == begin) return fail("bad number");
			pos_ += (size_t)(end - begin);
			return emit(op::constant, T(v));
		}
		if (std::isalpha((unsigned char)c) || c == '_') {
			std::string name;
			while (pos_ < src_.size() && (std::isalnum((unsigned char)src_[pos_]) || src_[pos_] == '_')) name += src_[pos_++];
			static const std::map<std::string, op> functions = {{"sin", op::sin}, {"cos", op::cos}, {"tan", op::tan}, {"exp", op::exp},
			                                                     {"log", op::log}, {"sqrt", op::sqrt}, {"abs", op::abs}};
			auto f = functions.find(name);
			if (f != functions.end()) {
				if (peek() != '(') return fail("'" + name + "' needs an argument in parentheses");
				++pos_;
				sum();
				if (peek() != ')') return fail("missing ')'");
				++pos_;
				return emit(f->second);
			}
			for (const auto* table : *tables_) {
				if (const T* v = table->variable(name)) return emit(op::variable, T(0), v);
				T value;
				if (table->constant(name, value)) return emit(op::constant, value);
			}
			return fail("undefined symbol '" + name + "'");
		}
		fail(c ? std::string("unexpected '") + c + "'" : std::string("unexpected end of expression"));
	}

	std::string src_;
	size_t pos_ = 0;
	std::string error_;
	std::vector<details::instruction<T>>* out_ = nullptr;
	const std::vector<const symbol_table<T>*>* tables_ = nullptr;
};

}  // namespace exprtk
