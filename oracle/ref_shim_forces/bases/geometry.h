/* Host shim for bases/geometry.h and the launcher (TEST INFRASTRUCTURE):
 * the geometry container's members as the reference's force loaders read
 * them, the operators' members as its forces apply them, the reference /
 * current tags, and util::transform as a host loop. */
#pragma once
#include <array>
#include "algo/cross.h"
#include "algo/dot.h"
#include "bases/types.h"
#include "util/math.h"

namespace util {
template <int nt = 128, int vt = 1, typename F, typename... A>
void transform(F&& f, int n, A&&... a) { for (int i = 0; i < n; ++i) f(i, a...); }
}

namespace bases {

inline constexpr struct {} reference;
inline constexpr struct {} current;

template <int dims>
struct geometry {
	static constexpr auto dimensions = dims;
	matrix position;
	std::array<matrix, dims> tangents;
	matrix normal;
	std::array<matrix, dims * (dims + 1) / 2> second_derivatives;
	matrix sigma;
};

template <int dims>
struct operators {
	int data_sites = 0, sample_sites = 0;
	matrix evaluator;
	std::array<matrix, dims> first_derivatives;
	std::array<matrix, dims * (dims + 1) / 2> second_derivatives;
	vector weights;
};

} // namespace bases
