// GPU restatement of the reference's own algorithm for spread and
// interpolate, for timing it on the same B200 (the reference's CUDA build
// does not compile with nvcc 12.9, so it cannot be timed as shipped).
//
// Labelled as a restatement: it follows the reference's kernel structure
// step by step with the reference's library calls (Thrust), not this
// repository's tiled kernels.  Per component (include/ib/novel.h:197-227):
//   K1  sort key of every point and the identity permutation (novel.h:68-90)
//   K2  thrust::sort_by_key of the keys with the permutation (novel.h:89)
//   K3  thrust::unique_copy to count the distinct keys, a host sync
//       (novel.h:58-66)
//   then per sweep of per_sweep = 8 stencil entries (novel.h:92-150):
//   K4  per sorted point, the sweep's 8 weights times the force
//   K5  thrust::reduce_by_key of those 8-vectors over equal keys
//   K6  per distinct key, plane i of buf += res * sum (errors_negative drops)
//   and finally
//   K7  combine: fe[t] = sum over the 8 planes of buf[i * size + t], and the
//       planes zeroed again (novel.h:153-167).
// Temporaries are allocated on every call, as the reference allocates them
// (novel.h:180-191, 213-215).  Interpolation is the reference's one thread
// per point gather in pattern order (include/ib/interpolate.h:49-76), which
// the library's interp_direct_kernel already restates.
//
// The index step and weights are the library's bit-exact restatements of
// the reference's (keys, origins and weights agree bit for bit), so the
// results agree with the library's FP64 path up to summation order.
#include <cstdio>
#include <string>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/functional.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>
#include <thrust/unique.h>
#include "ibk_direct.cuh"

namespace {

using namespace ibk;
using D = Delta<kBspline, 3>;
constexpr int DIMS = 3;
using P = Pattern<D::M, DIMS, D::every_other>;
constexpr int kPerSweep = 8;                    // largest divisor of 64 that is <= 10
constexpr int kSweeps = P::V / kPerSweep;

struct Values {
	double v[kPerSweep];
};

struct AddValues {
	__host__ __device__ Values operator()(const Values& a, const Values& b) const
	{
		Values r;
#pragma unroll
		for (int i = 0; i < kPerSweep; ++i) r.v[i] = a.v[i] + b.v[i];
		return r;
	}
};

// K1: sweep::sort (include/ib/sweep.h:64-77) of every point; perm = identity.
__global__ void keys_perm_kernel(GridGeom g, int comp, int n, const double* __restrict__ x, int* keys, int* perm)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const CompGeom& cg = g.comp[comp];
	int key = 0, weight = 1;
	for (int d = 0; d < DIMS; ++d) {
		AxisStep<D::M> a = axis_step<D::M>(g, cg, d, x[(size_t) d * n + p]);
		key += weight * a.key;
		weight *= cg.points[d] + g.solid[d];
	}
	keys[p] = key;
	perm[p] = p;
}

// K4: the sweep's weights times the force, per sorted point (novel.h:120-134).
__global__ void values_kernel(GridGeom g, int comp, int n, const double* __restrict__ x,
                              const double* __restrict__ fc, const int* __restrict__ perm, int sweep, Values* vals)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const CompGeom& cg = g.comp[comp];
	const int j = perm[t];
	const double f = fc[j];
	double w[DIMS][D::M];
	for (int d = 0; d < DIMS; ++d) {
		AxisStep<D::M> a = axis_step<D::M>(g, cg, d, x[(size_t) d * n + j]);
		for (int m = 0; m < D::M; ++m) w[d][m] = D::phi64(__dadd_rn(a.delta, (double) (m - P::shift)));
	}
	Values v;
#pragma unroll
	for (int i = 0; i < kPerSweep; ++i) {
		const int e = sweep * kPerSweep + i;
		const double wt = __dmul_rn(w[0][P::m(e, 0)], __dmul_rn(w[1][P::m(e, 1)], w[2][P::m(e, 2)]));
		v.v[i] = __dmul_rn(wt, f);
	}
	vals[t] = v;
}

// K6: per distinct key, its sweep's 8 grid indices (sweep::indices with
// errors_negative) and buf[i * size + j] += res * v[i] (novel.h:136-145).
__global__ void scatter_kernel(GridGeom g, int comp, int q, const int* __restrict__ ukeys,
                               const Values* __restrict__ uvals, int sweep, long long size, double* buf)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= q) return;
	const CompGeom& cg = g.comp[comp];
	int key = ukeys[t];
	int base[DIMS];
	for (int d = 0; d < DIMS; ++d) {                 // indexing::sorter::decompose
		const int wd = cg.points[d] + g.solid[d];
		base[d] = key % wd - g.solid[d];
		key /= wd;
	}
	const Values v = uvals[t];
	for (int i = 0; i < kPerSweep; ++i) {
		const int e = sweep * kPerSweep + i;
		long long k = 0, stride = 1;
		bool ok = true;
		for (int d = 0; d < DIMS; ++d) {
			const int node = node_index(g, cg, d, base[d] + P::m(e, d) - P::shift);
			ok = ok && node >= 0 && node < cg.points[d];
			k += (long long) node * stride;
			stride *= cg.points[d];
		}
		if (ok) buf[(size_t) i * size + k] += __dmul_rn(g.res, v.v[i]);
	}
}

// K7: fe[t] = sum of the planes, planes zeroed (novel.h:153-167).
__global__ void combine_kernel(long long size, double* buf, double* fe)
{
	const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= size) return;
	double s = 0.0;
	for (int i = 0; i < kPerSweep; ++i) {
		s = __dadd_rn(s, buf[(size_t) i * size + t]);
		buf[(size_t) i * size + t] = 0.0;
	}
	fe[t] = s;
}

std::string g_error;

bool ok(cudaError_t e, const char* what)
{
	if (e == cudaSuccess) return true;
	g_error = std::string(what) + ": " + cudaGetErrorString(e);
	cudaGetLastError();
	return false;
}

} // namespace

extern "C" {

const char* refgpu_last_error() { return g_error.c_str(); }

// Spread of n points (x, fl: dims*n device doubles) into fe[3] (device).
// g: the grid geometry in the library's device layout.  0 on success.
int refgpu_spread(const ibk::GridGeom* g, int n, const double* x, const double* fl, double* const* fe)
{
	if (n <= 0) return 0;
	long long max_size = 0;
	for (int c = 0; c < DIMS; ++c) max_size = g->comp[c].size > max_size ? g->comp[c].size : max_size;
	int *keys = nullptr, *perm = nullptr, *ukeys = nullptr, *scratch = nullptr;
	Values *vals = nullptr, *uvals = nullptr;
	double* buf = nullptr;
	bool good = ok(cudaMalloc(&keys, sizeof(int) * n), "cudaMalloc") &&
	            ok(cudaMalloc(&perm, sizeof(int) * n), "cudaMalloc") &&
	            ok(cudaMalloc(&buf, sizeof(double) * kPerSweep * (size_t) max_size), "cudaMalloc") &&
	            ok(cudaMemset(buf, 0, sizeof(double) * kPerSweep * (size_t) max_size), "cudaMemset");
	const int threads = 128, blocks = (n + threads - 1) / threads;
	for (int c = 0; c < DIMS && good; ++c) {
		const long long size = g->comp[c].size;
		keys_perm_kernel<<<blocks, threads>>>(*g, c, n, x, keys, perm);                         // K1
		thrust::sort_by_key(thrust::device, keys, keys + n, perm);                              // K2
		good = ok(cudaMalloc(&scratch, sizeof(int) * n), "cudaMalloc");                         // K3
		if (!good) break;
		const int q = (int) (thrust::unique_copy(thrust::device, keys, keys + n, scratch) - scratch);
		cudaFree(scratch);
		scratch = nullptr;
		good = ok(cudaMalloc(&vals, sizeof(Values) * n), "cudaMalloc") &&
		       ok(cudaMalloc(&uvals, sizeof(Values) * q), "cudaMalloc") &&
		       ok(cudaMalloc(&ukeys, sizeof(int) * q), "cudaMalloc");
		for (int s = 0; s < kSweeps && good; ++s) {
			values_kernel<<<blocks, threads>>>(*g, c, n, x, fl + (size_t) c * n, perm, s, vals);    // K4
			thrust::reduce_by_key(thrust::device, keys, keys + n, vals, ukeys, uvals,             // K5
			                      thrust::equal_to<int>(), AddValues());
			scatter_kernel<<<(q + threads - 1) / threads, threads>>>(*g, c, q, ukeys, uvals, s, size, buf);  // K6
		}
		combine_kernel<<<(int) ((size + threads - 1) / threads), threads>>>(size, buf, fe[c]);    // K7
		good = good && ok(cudaGetLastError(), "launch");
		cudaFree(vals);
		cudaFree(uvals);
		cudaFree(ukeys);
		vals = uvals = nullptr;
		ukeys = nullptr;
	}
	cudaFree(keys);
	cudaFree(perm);
	cudaFree(buf);
	return good ? 0 : 1;
}

// Interpolation of n points: ul[c*n + p] from ue[3] (device).
int refgpu_interpolate(const ibk::GridGeom* g, int n, const double* x, const double* const* ue, double* ul)
{
	if (n <= 0) return 0;
	ConstCompPtrs u;
	for (int c = 0; c < 3; ++c) u.p[c] = ue[c];
	const int threads = 128;
	interp_direct_kernel<D, DIMS><<<(n + threads - 1) / threads, threads>>>(*g, n, x, u, ul);
	return ok(cudaGetLastError(), "launch") ? 0 : 1;
}

} // extern "C"
