// Binning: a counting sort of the Lagrangian points by (tile, reach class)
// that leaves one 32-byte record per point in bin order.
//
// Tiles are boxes of T0 x T1 x T2 grid cells.  A point's home tile is the
// tile holding its stencil origin for the components staggered by 1/2 along
// each axis; its reach class records, per axis, whether the stencil of ANY
// component reaches into the lower (0) or upper (2) neighbouring tile or stays
// inside (1).  Origins are the reference's exact ones (axis_step), so the
// classes are exact: the owner-computes spread reads exactly the bins whose
// points can touch its faces.
//
// The record holds what the tile kernels need of the point, computed once
// with the reference's FP64 index step: per axis the exact stencil origin of
// the half-staggered components relative to the home tile, the difference
// to the origin along the component's own axis (MAC), the fractional
// offsets of both rounded to FP32, and the point's index.  The tile kernels
// read records contiguously, bin after bin, and never redo the FP64 step in
// the FP32C form (the FP64 form redoes it for its exact weights only).
//
//   bin_count_kernel    key = tile * 3^dims + class; warp-aggregated rank
//   bin_scan_kernel     exclusive scan of the bin counts (resets the counts)
//   bin_scatter_kernel  records[offset[key] + rank] = record of the point
// The non-template kernels are static: each translation unit that launches
// them carries its own copy.
#pragma once
#include "ibk_device.cuh"

namespace ibk {

// Sorted point record.  org: byte d (d < dims) = origin of the half-staggered
// components along axis d minus the first cell of the home tile (int8);
// byte 3 bits 2d..2d+1 = 1 + (origin along axis d of the component staggered
// along d) - (half-staggered origin), periodic differences folded to the
// nearest image, in {-1, 0, 1}.  dh / dn: sweep::difference of the half-
// staggered and own-axis components (include/ib/sweep.h:49-62), FP32.
struct __align__(16) PointRec {
	int org;
	float dh[kMaxDims];
	float dn[kMaxDims];
	int p;                  // point index (a batch numbers all its points)
};
static_assert(sizeof(PointRec) == 32, "point record layout");

__device__ __forceinline__ int rec_origin(int org, int d)
{
	return (int) (signed char) ((unsigned) org >> (8 * d));
}
__device__ __forceinline__ int rec_own_shift(int org, int d)
{
	return (int) (((unsigned) org >> (24 + 2 * d)) & 3u) - 1;
}

__device__ __forceinline__ PointRec load_rec(const PointRec* __restrict__ r)
{
	const int4 a = __ldg(reinterpret_cast<const int4*>(r));
	const int4 b = __ldg(reinterpret_cast<const int4*>(r) + 1);
	PointRec v;
	v.org = a.x;
	v.dh[0] = __int_as_float(a.y); v.dh[1] = __int_as_float(a.z); v.dh[2] = __int_as_float(a.w);
	v.dn[0] = __int_as_float(b.x); v.dn[1] = __int_as_float(b.y); v.dn[2] = __int_as_float(b.z);
	v.p = b.w;
	return v;
}

__device__ __forceinline__ void store_rec(PointRec* r, const PointRec& v)
{
	int4* q = reinterpret_cast<int4*>(r);
	q[0] = make_int4(v.org, __float_as_int(v.dh[0]), __float_as_int(v.dh[1]), __float_as_int(v.dh[2]));
	q[1] = make_int4(__float_as_int(v.dn[0]), __float_as_int(v.dn[1]), __float_as_int(v.dn[2]), v.p);
}

// Range of the own-axis origin shift (rec_own_shift) that a grid allows for
// component c along axis d: MAC components are shifted by 0 (periodic) or 1
// (solid) along their own axis against 1/2 for the others, so the own origin
// is the half one or one above it (periodic) / below it (solid); after the
// wall clamps of the sort key the shift stays in the same range.
__host__ __device__ inline void own_shift_range(const GridGeom& g, int tag_mac, int c, int d, int* lo, int* hi)
{
	*lo = 0;
	*hi = 0;
	if (!tag_mac || c != d) return;
	const double so = g.comp[d].shift[d], sh = g.comp[(d + 1) % g.dims].shift[d];
	if (so < sh) *hi = 1;
	else if (so > sh) *lo = -1;
}

// Bin of point p (home tile * 3^dims + reach class); with rec != nullptr the
// point's record as well (rec->p is left to the caller).
template <int M, int DIMS>
__device__ __forceinline__ int point_bin(const GridGeom& g, const TileGeom& tg, const double* __restrict__ x,
                                         int n, int p, PointRec* rec)
{
	constexpr int sh = (M - 1) >> 1;
	int tile = 0, cls = 0, ts = 1, cs = 1;
	unsigned org = 0;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		const double xd = __ldg(x + (size_t) d * n + p);
		const int hc = tg.tag_mac ? (d + 1) % DIMS : 0;
		const AxisStep<M> h = axis_step<M>(g, g.comp[hc], d, xd);
		int diff = 0;
		double dn = h.delta;
		if (tg.tag_mac) {
			const AxisStep<M> o = axis_step<M>(g, g.comp[d], d, xd);
			diff = o.base - h.base;
			if (!g.solid[d]) {
				const int c = tg.cells[d];
				if (2 * diff > c) diff -= c;
				else if (2 * diff < -c) diff += c;
			}
			dn = o.delta;
		}
		const int home = h.base < 0 ? 0 : (h.base >= tg.cells[d] ? tg.cells[d] - 1 : h.base);
		const int t = home / tg.T[d];
		const int lo = t * tg.T[d];
		const int thi = min(lo + tg.T[d], tg.cells[d]);
		const int node_lo = min(h.base, h.base + diff) - sh;
		const int node_hi = max(h.base, h.base + diff) + (M - 1 - sh);
		int c = 1;
		if (tg.ntiles[d] > 1) c = node_lo < lo ? 0 : (node_hi >= thi ? 2 : 1);
		tile += t * ts;
		ts *= tg.ntiles[d];
		cls += c * cs;
		cs *= 3;
		if (rec) {
			org |= ((unsigned) (h.base - lo) & 0xffu) << (8 * d);
			org |= (unsigned) (diff + 1) << (24 + 2 * d);
			rec->dh[d] = (float) h.delta;
			rec->dn[d] = (float) dn;
		}
	}
	if (rec) {
		rec->org = (int) org;
#pragma unroll
		for (int d = DIMS; d < kMaxDims; ++d) { rec->dh[d] = 0.0f; rec->dn[d] = 0.0f; }
	}
	return tile * tg.nclass + cls;
}

// Force statistics of the bins (spread only): binmax[bin * 3 + c] = the
// largest |f| of the bin's points as FP32 bits (f = FP32 res * F_c, the value
// the FP32C spread multiplies), from which a tile takes the largest term its
// fixed point must hold.  An integer maximum: independent of the order of
// the atomics (the binning order is not deterministic; this is).
struct BinStats {
	const double* f;        // forces (dims * n), nullptr: no statistics
	double res;             // product of the resolutions (1 / h^dims)
	unsigned* binmax;
};

template <int DIMS>
__device__ __forceinline__ void force_abs(const BinStats& st, int n, int p, float* a)
{
#pragma unroll
	for (int c = 0; c < DIMS; ++c) a[c] = fabsf((float) (st.res * __ldg(st.f + (size_t) c * n + p)));
}

// Warp-aggregated rank of a point in its bin: one atomic per group of lanes
// sharing a key; with statistics (a != nullptr) also the group's largest
// |f| per component.  Every lane of `mask` must call it.
template <int DIMS>
__device__ __forceinline__ void bin_rank(unsigned mask, int key, int* __restrict__ count, int2* __restrict__ kr_out,
                                         const float* a, unsigned* __restrict__ binmax)
{
	const int lane = threadIdx.x & 31;
	const unsigned peers = __match_any_sync(mask, key);
	const int leader = __ffs(peers) - 1;
	int base = 0;
	if (lane == leader) base = atomicAdd(count + key, __popc(peers));
	base = __shfl_sync(peers, base, leader);
	*kr_out = make_int2(key, base + __popc(peers & ((1u << lane) - 1u)));
	if (a != nullptr) {
#pragma unroll
		for (int c = 0; c < DIMS; ++c) {
			const unsigned m = __reduce_max_sync(peers, __float_as_uint(a[c]));
			if (lane == leader && m != 0u) atomicMax(binmax + (size_t) key * kMaxDims + c, m);
		}
	}
}

template <int M, int DIMS>
__global__ void __launch_bounds__(256)
bin_count_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                 int* __restrict__ count, int2* __restrict__ key_rank, BinStats st)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	const bool active = p < n;
	float a[kMaxDims] = {0.0f, 0.0f, 0.0f};
	if (st.f != nullptr && active) force_abs<DIMS>(st, n, p, a);   // loads in flight with x's
	const int key = active ? point_bin<M, DIMS>(g, tg, x, n, p, nullptr) : 0;
	const unsigned mask = __ballot_sync(0xffffffffu, active);
	if (!active) return;
	bin_rank<DIMS>(mask, key, count, key_rank + p, st.f != nullptr ? a : nullptr, st.binmax);
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

// The record of every point at its sorted position (the FP64 index step is
// recomputed here rather than stored by the count kernel: it costs less
// than writing and re-reading the records in input order).
template <int M, int DIMS>
__global__ void __launch_bounds__(256)
bin_scatter_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const int2* __restrict__ key_rank, const int* __restrict__ offset,
                   PointRec* __restrict__ recs)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const int2 kr = __ldg(key_rank + p);
	PointRec r;
	point_bin<M, DIMS>(g, tg, x, n, p, &r);
	r.p = p;
	store_rec(recs + __ldg(offset + kr.x) + kr.y, r);
}

} // namespace ibk
