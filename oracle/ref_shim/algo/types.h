/* Host shim standing in for the reference's algo/types.h, which pulls in the
 * CUDA linalg layer.  fd/discretization.h needs only a sparse-matrix shape,
 * a launcher and the index base; the geometry functions used by the oracle
 * never call them. */
#pragma once
namespace linalg {
template <typename T> struct dense {};
template <typename T> struct sparse {};
template <typename T> struct matrix {};
template <typename T> struct vector {};
struct size { int rows, cols; };
}
namespace fd {
struct matrix {
	matrix(int, int, int = 0) {}
	int* starts() { return nullptr; }
	int* indices() { return nullptr; }
	double* values() { return nullptr; }
};
}
namespace util {
template <int nt = 128, int vt = 1, typename F, typename... A>
void transform(F&& f, int n, A&&... a) { for (int i = 0; i < n; ++i) f(i, a...); }
}
namespace algo {
static constexpr int indexing_base = 0;
using matrix = fd::matrix;
using vector = linalg::vector<linalg::dense<double>>;
}
