/* Host shim standing in for the reference's CUDA linalg layer under its
 * solvers (TEST INFRASTRUCTURE, used only to build oracle/_ref/
 * libibref_solver.so): a dense host vector with the reductions solvers/pcg.h
 * and algo/chebyshev.h call (dot and the norm as plain sums in index order,
 * axpy, swap, scaling), and a matrix-free "sparse" matrix whose product is a
 * callback into the oracle's operator.  gemv with beta = 0 does not read y (the BLAS convention the
 * reference relies on for its uninitialised q). */
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <utility>
#include <vector>

namespace linalg {

template <typename T> struct dense {};
template <typename T> struct sparse {};
template <typename L> struct vector;
template <typename L> struct matrix;
inline constexpr struct zero_t {} zero;

template <>
struct vector<dense<double>> {
	std::vector<double> v;
	vector() = default;
	explicit vector(int n) : v((std::size_t) n) {}
	vector(int n, zero_t) : v((std::size_t) n, 0.0) {}
	int rows() const { return (int) v.size(); }
	int cols() const { return 1; }
	double* values() { return v.data(); }
	const double* values() const { return v.data(); }
};

using dvec = vector<dense<double>>;

using apply_fn = void (*)(const double*, double*, void*);

template <>
struct matrix<sparse<double>> {
	apply_fn apply = nullptr;
	void* ctx = nullptr;
	int n = 0;
	// the CSR members algo/gershgorin.h names (the bridge never calls it)
	int rows() const { return n; }
	int* starts() const { return nullptr; }
	int* indices() const { return nullptr; }
	double* values() const { return nullptr; }
};

template <>
struct matrix<dense<double>> {};

using smat = matrix<sparse<double>>;

struct extent { int rows, cols; };
inline extent size(const dvec& x) { return {x.rows(), 1}; }
template <typename... A> void fill(A&&...) {}

inline double dot(const dvec& a, const dvec& b)
{
	double s = 0.0;
	for (std::size_t i = 0; i < a.v.size(); ++i) s += a.v[i] * b.v[i];
	return s;
}

inline double abs(const dvec& a) { return std::sqrt(dot(a, a)); }

inline void axpy(double a, const dvec& x, dvec& y)
{
	for (std::size_t i = 0; i < y.v.size(); ++i) y.v[i] = a * x.v[i] + y.v[i];
}

inline void swap(dvec& a, dvec& b) { std::swap(a.v, b.v); }

inline dvec operator*(double s, dvec x)
{
	for (double& e : x.v) e = s * e;
	return x;
}

inline void gemv(double alpha, const smat& m, const dvec& x, double beta, dvec& y)
{
	std::vector<double> ax(x.v.size());
	m.apply(x.v.data(), ax.data(), m.ctx);
	if (y.v.size() != ax.size()) y.v.assign(ax.size(), 0.0);
	for (std::size_t i = 0; i < ax.size(); ++i)
		y.v[i] = beta == 0.0 ? alpha * ax[i] : alpha * ax[i] + beta * y.v[i];
}

} // namespace linalg
