// Per-point ("direct") kernels: one thread per Lagrangian point, no binning.
//
//   keys_kernel            ib::sweep::sort for one component (bit-exact keys)
//   interp_direct_kernel   ib::interpolate: gather M^dims nodes per component,
//                          summed in the reference's pattern order
//   spread_direct_kernel   ib::spread as global FP64 reductions into faces
//                          that the caller's stream has zeroed first
//
// These are the small-n / fallback-free baseline of the library; the tiled
// kernels (ibk_tiled.cuh) are the throughput path.
#pragma once
#include "ibk_device.cuh"

namespace ibk {

// Per point, per component: weights and node indices along each axis.
template <typename D, int DIMS, bool SPREAD>
struct AxisStencil {
	static constexpr int M = D::M;
	static constexpr int shift = (M - 1) >> 1;
	double w[DIMS][M];
	int node[DIMS][M];        // node index along the axis; -1 = dropped (spread)

	__device__ __forceinline__ void build(const GridGeom& g, const CompGeom& cg, const double* z) {
#pragma unroll
		for (int d = 0; d < DIMS; ++d) {
			AxisStep<M> a = axis_step<M>(g, cg, d, z[d]);
#pragma unroll
			for (int m = 0; m < M; ++m) {
				w[d][m] = D::phi64(__dadd_rn(a.delta, (double) (m - shift)));
				int j = node_index(g, cg, d, a.base + m - shift);
				const int p = cg.points[d];
				if (SPREAD) node[d][m] = (0 <= j && j < p) ? j : -1;
				else node[d][m] = j < 0 ? 0 : (j >= p ? p - 1 : j);
			}
		}
	}
};

template <typename D, int DIMS>
__global__ void __launch_bounds__(128)
keys_kernel(GridGeom g, int comp, int n, const double* __restrict__ x, int* __restrict__ keys)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const CompGeom& cg = g.comp[comp];
	int key = 0, weight = 1;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		AxisStep<D::M> a = axis_step<D::M>(g, cg, d, x[(size_t) d * n + p]);
		key += weight * a.key;                       // indexing::combine, clamped
		weight *= cg.points[d] + g.solid[d];
	}
	keys[p] = key;
}

template <typename D, int DIMS>
__global__ void __launch_bounds__(128)
interp_direct_kernel(GridGeom g, int n, const double* __restrict__ x, ConstCompPtrs ue,
                     double* __restrict__ ul)
{
	using P = Pattern<D::M, DIMS, D::every_other>;
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	double z[DIMS];
#pragma unroll
	for (int d = 0; d < DIMS; ++d) z[d] = x[(size_t) d * n + p];
#pragma unroll 1
	for (int c = 0; c < DIMS; ++c) {
		const CompGeom& cg = g.comp[c];
		AxisStencil<D, DIMS, false> st;
		st.build(g, cg, z);
		const double* __restrict__ u = ue.p[c];
		const int p0 = cg.points[0];
		const int p1 = DIMS > 1 ? cg.points[1] : 1;
		double v = 0.0;
#pragma unroll
		for (int e = 0; e < P::V; ++e) {
			const int m0 = P::m(e, 0);
			double w;
			long long k;
			if constexpr (DIMS == 3) {
				const int m1 = P::m(e, 1), m2 = P::m(e, 2);
				w = __dmul_rn(st.w[0][m0], __dmul_rn(st.w[1][m1], st.w[2][m2]));
				k = st.node[0][m0] + (long long) p0 * (st.node[1][m1] + (long long) p1 * st.node[2][m2]);
			} else {
				const int m1 = P::m(e, 1);
				w = __dmul_rn(st.w[0][m0], st.w[1][m1]);
				k = st.node[0][m0] + (long long) p0 * st.node[1][m1];
			}
			v = __dadd_rn(v, __dmul_rn(w, __ldg(u + k)));   // interpolate.h:71-72
		}
		ul[(size_t) c * n + p] = v;
	}
}

template <typename D, int DIMS>
__global__ void __launch_bounds__(128)
spread_direct_kernel(GridGeom g, int n, const double* __restrict__ x, const double* __restrict__ fl,
                     CompPtrs fe)
{
	using P = Pattern<D::M, DIMS, D::every_other>;
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	double z[DIMS];
#pragma unroll
	for (int d = 0; d < DIMS; ++d) z[d] = x[(size_t) d * n + p];
#pragma unroll 1
	for (int c = 0; c < DIMS; ++c) {
		const CompGeom& cg = g.comp[c];
		AxisStencil<D, DIMS, true> st;
		st.build(g, cg, z);
		const double f = __dmul_rn(g.res, fl[(size_t) c * n + p]);
		double* __restrict__ out = fe.p[c];
		const int p0 = cg.points[0];
		const int p1 = DIMS > 1 ? cg.points[1] : 1;
#pragma unroll
		for (int e = 0; e < P::V; ++e) {
			const int m0 = P::m(e, 0);
			double w;
			long long k;
			bool ok;
			if constexpr (DIMS == 3) {
				const int m1 = P::m(e, 1), m2 = P::m(e, 2);
				w = __dmul_rn(st.w[0][m0], __dmul_rn(st.w[1][m1], st.w[2][m2]));
				ok = (st.node[0][m0] | st.node[1][m1] | st.node[2][m2]) >= 0;
				k = st.node[0][m0] + (long long) p0 * (st.node[1][m1] + (long long) p1 * st.node[2][m2]);
			} else {
				const int m1 = P::m(e, 1);
				w = __dmul_rn(st.w[0][m0], st.w[1][m1]);
				ok = (st.node[0][m0] | st.node[1][m1]) >= 0;
				k = st.node[0][m0] + (long long) p0 * st.node[1][m1];
			}
			if (ok) atomicAdd(out + k, __dmul_rn(w, f));
		}
	}
}

} // namespace ibk
