/* Host shim standing in for the reference's CUDA linalg layer (TEST
 * INFRASTRUCTURE, used only to build oracle/_ref/libibref_forces.so): a
 * column-major host matrix with the members the reference's force code
 * touches (values, rows, cols, linalg::size, element-wise sums and scaling,
 * and the product that applies an operator). */
#pragma once
#include <cstddef>
#include <stdexcept>
#include <vector>

namespace linalg {

struct extent { int rows, cols; };
inline constexpr struct zero_t {} zero;

template <typename T> struct dense {};
template <typename L> struct matrix;
template <typename L> struct vector;

template <>
struct matrix<dense<double>> {
	int r = 0, c = 0;
	std::vector<double> v;
	matrix() = default;
	matrix(int rows, int cols) : r(rows), c(cols), v((std::size_t) rows * cols, 0.0) {}
	matrix(extent e) : matrix(e.rows, e.cols) {}
	matrix(extent e, zero_t) : matrix(e.rows, e.cols) {}
	double* values() { return v.data(); }
	const double* values() const { return v.data(); }
	int rows() const { return r; }
	int cols() const { return c; }
};

template <>
struct vector<dense<double>> : matrix<dense<double>> {
	vector() = default;
	explicit vector(int n) : matrix<dense<double>>(n, 1) {}
};

using hmatrix = matrix<dense<double>>;

inline extent size(const hmatrix& m) { return {m.rows(), m.cols()}; }

inline hmatrix operator+(const hmatrix& a, const hmatrix& b)
{
	if (a.r != b.r || a.c != b.c) throw std::invalid_argument("shape");
	hmatrix o(a.r, a.c);
	for (std::size_t i = 0; i < a.v.size(); ++i) o.v[i] = a.v[i] + b.v[i];
	return o;
}

inline hmatrix operator-(const hmatrix& a, const hmatrix& b)
{
	if (a.r != b.r || a.c != b.c) throw std::invalid_argument("shape");
	hmatrix o(a.r, a.c);
	for (std::size_t i = 0; i < a.v.size(); ++i) o.v[i] = a.v[i] - b.v[i];
	return o;
}

inline hmatrix operator*(double s, const hmatrix& a)
{
	hmatrix o(a.r, a.c);
	for (std::size_t i = 0; i < a.v.size(); ++i) o.v[i] = s * a.v[i];
	return o;
}

/* operator product, column-major, a plain summation loop */
inline hmatrix operator*(const hmatrix& a, const hmatrix& b)
{
	if (a.c != b.r) throw std::invalid_argument("shape");
	hmatrix o(a.r, b.c);
	for (int j = 0; j < b.c; ++j)
		for (int i = 0; i < a.r; ++i) {
			double s = 0.0;
			for (int k = 0; k < a.c; ++k) s += a.v[(std::size_t) k * a.r + i] * b.v[(std::size_t) j * b.r + k];
			o.v[(std::size_t) j * a.r + i] = s;
		}
	return o;
}

} // namespace linalg
