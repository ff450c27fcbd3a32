// Conservation sums in FP64: total force and torque of the point forces, and
// the total of a spread force density (h^dims times the sum over faces).  In
// a periodic domain spreading conserves force, so the two totals agree; the
// reference has no such check of its own (its solver never sums either).
//
// Both are two-stage reductions with a fixed order: kSumBlocks blocks each
// sum a fixed grid-stride share of the elements and reduce it in shared
// memory by a fixed tree, then one block adds the partials the same way.
// The result is therefore the same on every run (no atomics), whatever the
// scheduling.
#include <string>
#include "ibk_internal.h"

namespace ibk {
namespace {

constexpr int kSumThreads = 256;
constexpr int kSumBlocks = 1024;
constexpr int kMoments = 6;     // force (3), torque (3)

// Tree sum of v over the block; thread 0 receives the total.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red)
{
	red[threadIdx.x] = v;
	__syncthreads();
#pragma unroll
	for (int s = NT / 2; s > 0; s >>= 1) {
		if ((int) threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
		__syncthreads();
	}
	const double t = red[0];
	__syncthreads();
	return t;
}

__global__ void __launch_bounds__(kSumThreads)
moment_partials_kernel(int n, int dims, const double* __restrict__ x, const double* __restrict__ fl,
                       double* __restrict__ partial)
{
	__shared__ double red[kSumThreads];
	double m[kMoments] = {0, 0, 0, 0, 0, 0};
	for (int p = blockIdx.x * kSumThreads + threadIdx.x; p < n; p += kSumBlocks * kSumThreads) {
		double xp[3] = {0, 0, 0}, fp[3] = {0, 0, 0};
		for (int d = 0; d < dims; ++d) {
			xp[d] = __ldg(x + (size_t) d * n + p);
			fp[d] = __ldg(fl + (size_t) d * n + p);
		}
		for (int d = 0; d < 3; ++d) m[d] = __dadd_rn(m[d], fp[d]);
		// x cross F (2-D: only the z component is non-zero)
		m[3] = __dadd_rn(m[3], __dsub_rn(__dmul_rn(xp[1], fp[2]), __dmul_rn(xp[2], fp[1])));
		m[4] = __dadd_rn(m[4], __dsub_rn(__dmul_rn(xp[2], fp[0]), __dmul_rn(xp[0], fp[2])));
		m[5] = __dadd_rn(m[5], __dsub_rn(__dmul_rn(xp[0], fp[1]), __dmul_rn(xp[1], fp[0])));
	}
	for (int k = 0; k < kMoments; ++k) {
		const double t = block_sum<kSumThreads>(m[k], red);
		if (threadIdx.x == 0) partial[(size_t) blockIdx.x * kMoments + k] = t;
	}
}

__global__ void __launch_bounds__(kSumThreads)
grid_partials_kernel(long long size, const double* __restrict__ fe, double* __restrict__ partial)
{
	__shared__ double red[kSumThreads];
	double s = 0.0;
	for (long long j = (long long) blockIdx.x * kSumThreads + threadIdx.x; j < size;
	     j += (long long) kSumBlocks * kSumThreads)
		s = __dadd_rn(s, __ldg(fe + j));
	const double t = block_sum<kSumThreads>(s, red);
	if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// out[k] = scale * sum over blocks of partial[b * stride + k], for k < count.
__global__ void __launch_bounds__(kSumThreads)
sum_partials_kernel(const double* __restrict__ partial, int stride, int count, double scale, double* __restrict__ out)
{
	__shared__ double red[kSumThreads];
	for (int k = 0; k < count; ++k) {
		double s = 0.0;
		for (int b = threadIdx.x; b < kSumBlocks; b += kSumThreads) s = __dadd_rn(s, partial[(size_t) b * stride + k]);
		const double t = block_sum<kSumThreads>(s, red);
		if (threadIdx.x == 0) out[k] = __dmul_rn(scale, t);
	}
}

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_force_moments(ibk_plan handle, int n, const double* x, const double* fl, double* out, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || !out || (n > 0 && (!x || !fl)) || n < 0)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or arrays, or negative count");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	ibk_status st = ensure_scratch(*plan, kSlotSums, sizeof(double) * kMoments * kSumBlocks, s);
	if (st != IBK_OK) return st;
	double* partial = static_cast<double*>(plan->scratch[kSlotSums].ptr);
	if ((st = launch(*plan, "moment_partials_kernel", s, [&] {
		moment_partials_kernel<<<kSumBlocks, kSumThreads, 0, s>>>(n, plan->g.dims, x, fl, partial);
	})) != IBK_OK) return st;
	return launch(*plan, "sum_partials_kernel", s, [&] {
		sum_partials_kernel<<<1, kSumThreads, 0, s>>>(partial, kMoments, kMoments, 1.0, out);
	});
}

ibk_status ibk_grid_totals(ibk_plan handle, double* const* fe, double* out, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || !fe || !out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or arrays");
	for (int c = 0; c < plan->g.dims; ++c)
		if (!fe[c]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null grid component");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	ibk_status st = ensure_scratch(*plan, kSlotSums, sizeof(double) * kMoments * kSumBlocks, s);
	if (st != IBK_OK) return st;
	double* partial = static_cast<double*>(plan->scratch[kSlotSums].ptr);
	const double cell = 1.0 / plan->g.res;      // h^dims
	for (int c = 0; c < plan->g.dims; ++c) {
		if ((st = launch(*plan, "grid_partials_kernel", s, [&] {
			grid_partials_kernel<<<kSumBlocks, kSumThreads, 0, s>>>(plan->g.comp[c].size, fe[c], partial);
		})) != IBK_OK) return st;
		if ((st = launch(*plan, "sum_partials_kernel", s, [&] {
			sum_partials_kernel<<<1, kSumThreads, 0, s>>>(partial, 1, 1, cell, out + c);
		})) != IBK_OK) return st;
	}
	return IBK_OK;
}

} // extern "C"
