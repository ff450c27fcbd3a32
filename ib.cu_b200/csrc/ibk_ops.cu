// Operator implementations and the (delta, dims, precision) dispatch table.
#include <cstdio>
#include "ibk_internal.h"
#include "ibk_direct.cuh"

namespace ibk {

namespace {

constexpr int kThreads = 128;

inline int blocks_for(long long n, int threads) { return (int) ((n + threads - 1) / threads); }

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status spread_impl(Plan& plan, const OpArgs& a, const double* fl, CompPtrs fe)
{
	using D = Delta<KIND, ORDER>;
	const GridGeom& g = *a.g;
	for (int c = 0; c < DIMS; ++c) {
		cudaError_t e = cudaMemsetAsync(fe.p[c], 0, sizeof(double) * (size_t) g.comp[c].size, a.stream);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
	}
	return launch(plan, "spread_direct_kernel", a.stream, [&] {
		spread_direct_kernel<D, DIMS><<<blocks_for(a.n, kThreads), kThreads, 0, a.stream>>>(g, a.n, a.x, fl, fe);
	});
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status interp_impl(Plan& plan, const OpArgs& a, ConstCompPtrs ue, double* ul)
{
	using D = Delta<KIND, ORDER>;
	return launch(plan, "interp_direct_kernel", a.stream, [&] {
		interp_direct_kernel<D, DIMS><<<blocks_for(a.n, kThreads), kThreads, 0, a.stream>>>(*a.g, a.n, a.x, ue, ul);
	});
}

template <int KIND, int ORDER, int DIMS>
ibk_status keys_impl(Plan& plan, const OpArgs& a, int comp, int* keys)
{
	using D = Delta<KIND, ORDER>;
	return launch(plan, "keys_kernel", a.stream, [&] {
		keys_kernel<D, DIMS><<<blocks_for(a.n, kThreads), kThreads, 0, a.stream>>>(*a.g, comp, a.n, a.x, keys);
	});
}

template <int KIND, int ORDER, int DIMS, int PREC>
constexpr OpTable make_table()
{
	return OpTable{&spread_impl<KIND, ORDER, DIMS, PREC>, &interp_impl<KIND, ORDER, DIMS, PREC>,
	               &keys_impl<KIND, ORDER, DIMS>};
}

struct Entry { int kind, order, dims, prec; OpTable ops; };

#define IBK_ENTRY(K, O, DIM, PR) Entry{K, O, DIM, PR, make_table<K, O, DIM, PR>()}
#define IBK_DELTA_ENTRIES(DIM, PR)                                          \
	IBK_ENTRY(kBspline, 1, DIM, PR), IBK_ENTRY(kBspline, 2, DIM, PR),     \
	IBK_ENTRY(kBspline, 3, DIM, PR), IBK_ENTRY(kBspline, 4, DIM, PR),     \
	IBK_ENTRY(kBspline, 5, DIM, PR), IBK_ENTRY(kPeskin, 0, DIM, PR),      \
	IBK_ENTRY(kRoma, 0, DIM, PR), IBK_ENTRY(kCosine, 0, DIM, PR),         \
	IBK_ENTRY(kHat, 0, DIM, PR)

const Entry kTable[] = {
	IBK_DELTA_ENTRIES(2, IBK_PRECISION_FP64),
	IBK_DELTA_ENTRIES(3, IBK_PRECISION_FP64),
};

} // namespace

const OpTable* find_ops(int kind, int order, int dims, int precision)
{
	if (kind != kBspline) order = 0;
	for (const Entry& e : kTable)
		if (e.kind == kind && e.order == order && e.dims == dims && e.prec == precision)
			return &e.ops;
	return nullptr;
}

} // namespace ibk
