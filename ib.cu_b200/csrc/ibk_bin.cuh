// Binning: a counting sort of the Lagrangian points by (tile, reach class).
//
// Tiles are boxes of T0 x T1 x T2 grid cells.  A point's home tile is the
// tile holding its stencil origin for the components staggered by 1/2 along
// each axis; its reach class records, per axis, whether the stencil of ANY
// component reaches into the lower (0) or upper (2) neighbouring tile or stays
// inside (1).  Origins are the reference's exact ones (axis_step), so the
// classes are exact: the owner-computes spread kernel reads exactly the bins
// whose points can touch its faces.
//
//   bin_count_kernel    key = tile * 3^dims + class; warp-aggregated rank
//   bin_scan_kernel     exclusive scan of the bin counts (resets the counts)
//   bin_scatter_kernel  perm[offset[key] + rank] = point
// The non-template kernels are static: each translation unit that launches
// them carries its own copy.
#pragma once
#include "ibk_device.cuh"

namespace ibk {

// Exact stencil-node span of every component along axis d, relative to the
// origin `bh` of the components staggered by 1/2 along d.
template <int M>
struct AxisReach {
	int home;      // clamped origin used for the home tile
	int node_lo;   // lowest node (unwrapped, relative to the same index space)
	int node_hi;   // highest node
};

template <int M, int DIMS>
__device__ __forceinline__ AxisReach<M> axis_reach(const GridGeom& g, const TileGeom& tg, int d, double x)
{
	constexpr int lo_off = (M - 1) >> 1;      // offsets run -lo_off .. M - 1 - lo_off
	constexpr int hi_off = M - 1 - lo_off;
	const int half_comp = tg.tag_mac ? (d + 1) % DIMS : 0;
	const int bh = axis_step<M>(g, g.comp[half_comp], d, x).base;
	int lo = bh, hi = bh;
	if (tg.tag_mac) {
		int bo = axis_step<M>(g, g.comp[d], d, x).base;
		int diff = bo - bh;
		if (!g.solid[d]) {
			const int c = tg.cells[d];
			if (2 * diff > c) diff -= c;
			else if (2 * diff < -c) diff += c;
		}
		lo = min(bh, bh + diff);
		hi = max(bh, bh + diff);
	}
	AxisReach<M> r;
	r.home = bh < 0 ? 0 : (bh >= tg.cells[d] ? tg.cells[d] - 1 : bh);
	r.node_lo = lo - lo_off;
	r.node_hi = hi + hi_off;
	return r;
}

// Bin of point p: home tile * 3^dims + reach class.
template <int M, int DIMS>
__device__ __forceinline__ int bin_key(const GridGeom& g, const TileGeom& tg, const double* __restrict__ x,
                                       int n, int p)
{
	int tile = 0, cls = 0, ts = 1, cs = 1;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		AxisReach<M> r = axis_reach<M, DIMS>(g, tg, d, __ldg(x + (size_t) d * n + p));
		const int t = r.home / tg.T[d];
		const int tlo = t * tg.T[d];
		const int thi = min(tlo + tg.T[d], tg.cells[d]);
		int c = 1;
		if (tg.ntiles[d] > 1) c = r.node_lo < tlo ? 0 : (r.node_hi >= thi ? 2 : 1);
		tile += t * ts;
		ts *= tg.ntiles[d];
		cls += c * cs;
		cs *= 3;
	}
	return tile * tg.nclass + cls;
}

// Warp-aggregated rank of a point in its bin (one atomic per group of lanes
// sharing a key); with fbits != nullptr also raises binmax[key * 3 + c] to
// the group's largest FP32 |F| bit pattern.  Every lane of `mask` must call
// it, all with fbits null or all with fbits set.
template <int DIMS>
__device__ __forceinline__ void bin_rank(unsigned mask, int key, int* __restrict__ count, int2* __restrict__ kr_out,
                                         const unsigned* fbits, unsigned* __restrict__ binmax)
{
	const int lane = threadIdx.x & 31;
	const unsigned peers = __match_any_sync(mask, key);
	const int leader = __ffs(peers) - 1;
	int base = 0;
	if (lane == leader) base = atomicAdd(count + key, __popc(peers));
	base = __shfl_sync(peers, base, leader);
	*kr_out = make_int2(key, base + __popc(peers & ((1u << lane) - 1u)));
	if (fbits != nullptr) {
#pragma unroll
		for (int c = 0; c < DIMS; ++c) {
			const unsigned m = __reduce_max_sync(peers, fbits[c]);
			if (lane == leader && m != 0u) atomicMax(binmax + (size_t) key * kMaxDims + c, m);
		}
	}
}

// FP32 |f[c * n + p]| bit patterns of one point (0 past the end).
template <int DIMS>
__device__ __forceinline__ void force_bits(const double* __restrict__ f, int n, int p, bool active, unsigned* fbits)
{
#pragma unroll
	for (int c = 0; c < DIMS; ++c)
		fbits[c] = active ? __float_as_uint(fabsf((float) __ldg(f + (size_t) c * n + p))) : 0u;
}

// With f != nullptr (spread) the kernel also raises binmax[key * 3 + c] to
// the FP32 |F| of every point of the bin, per component; binmax starts at
// zero and, as all values are non-negative floats, compares as unsigned bit
// patterns.  The maximum does not depend on the order of the atomics.
template <int M, int DIMS>
__global__ void __launch_bounds__(256)
bin_count_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                 int* __restrict__ count, int2* __restrict__ key_rank,
                 const double* __restrict__ f, unsigned* __restrict__ binmax)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	const bool active = p < n;
	unsigned fbits[kMaxDims] = {0u, 0u, 0u};
	if (f != nullptr) force_bits<DIMS>(f, n, p, active, fbits);   // loads in flight with x's
	const int key = active ? bin_key<M, DIMS>(g, tg, x, n, p) : 0;
	const unsigned mask = __ballot_sync(0xffffffffu, active);
	if (!active) return;
	bin_rank<DIMS>(mask, key, count, key_rank + p, f != nullptr ? fbits : nullptr, binmax);
}

// Exclusive scan of the bin counts in two launches.  Each CTA owns a chunk
// of kScanChunk bins: the first kernel writes the chunk totals; the second
// scans the (few thousand at most) chunk totals in every CTA to get its
// chunk's offset, scans its chunk, and zeroes the counts for the next call.
constexpr int kScanThreads = 1024;
constexpr int kScanChunk = kScanThreads * 4;

__device__ __forceinline__ int block_exclusive_scan(int v, int& total)
{
	__shared__ int warp_sums[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += t;
	}
	if (lane == 31) warp_sums[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		int s = lane < (int) (blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int t = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += t;
		}
		warp_sums[lane] = s;
	}
	__syncthreads();
	total = warp_sums[31];
	const int r = (warp ? warp_sums[warp - 1] : 0) + incl - v;
	__syncthreads();
	return r;
}

static __global__ void __launch_bounds__(kScanThreads)
bin_chunk_sum_kernel(const int* __restrict__ count, int* __restrict__ chunk, int num_bins)
{
	const int i0 = blockIdx.x * kScanChunk + threadIdx.x * 4;
	int v = 0;
	if (i0 + 3 < num_bins) {
		const int4 q = *reinterpret_cast<const int4*>(count + i0);
		v = q.x + q.y + q.z + q.w;
	} else {
		for (int k = 0; k < 4; ++k) if (i0 + k < num_bins) v += count[i0 + k];
	}
	int total;
	block_exclusive_scan(v, total);
	if (threadIdx.x == 0) chunk[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(kScanThreads)
bin_scan_kernel(int* __restrict__ count, const int* __restrict__ chunk, int* __restrict__ offset,
                int num_bins, int nchunks)
{
	// offset of this chunk = sum of the totals of the chunks before it
	int pre = 0;
	for (int c = threadIdx.x; c < blockIdx.x; c += kScanThreads) pre += chunk[c];
	int base_total;
	{
		int dummy = block_exclusive_scan(pre, base_total);
		(void) dummy;
	}
	const int i0 = blockIdx.x * kScanChunk + threadIdx.x * 4;
	int v[4];
	const bool full = i0 + 3 < num_bins;
	if (full) {
		const int4 q = *reinterpret_cast<const int4*>(count + i0);
		v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
	} else {
		for (int k = 0; k < 4; ++k) v[k] = i0 + k < num_bins ? count[i0 + k] : 0;
	}
	int total;
	int run = base_total + block_exclusive_scan(v[0] + v[1] + v[2] + v[3], total);
	int o[4];
#pragma unroll
	for (int k = 0; k < 4; ++k) { o[k] = run; run += v[k]; }
	if (full) {
		*reinterpret_cast<int4*>(offset + i0) = make_int4(o[0], o[1], o[2], o[3]);
		*reinterpret_cast<int4*>(count + i0) = make_int4(0, 0, 0, 0);
	} else {
		for (int k = 0; k < 4; ++k) if (i0 + k < num_bins) { offset[i0 + k] = o[k]; count[i0 + k] = 0; }
	}
	if (blockIdx.x == nchunks - 1 && threadIdx.x == kScanThreads - 1) offset[num_bins] = run;
}

static __global__ void __launch_bounds__(256)
bin_scatter_kernel(int n, const int2* __restrict__ key_rank, const int* __restrict__ offset,
                   int* __restrict__ perm)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const int2 kr = key_rank[p];
	perm[__ldg(offset + kr.x) + kr.y] = p;
}

} // namespace ibk
