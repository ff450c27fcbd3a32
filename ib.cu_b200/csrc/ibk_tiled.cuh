// Tiled kernels: the throughput path of spread and interpolate.
//
// Points are binned by (home tile, reach class) (ibk_bin.cuh).  One CTA owns
// one tile of T0 x T1 x T2 grid cells for every MAC component.
//
// spread_tile_kernel  -- owner computes.  The CTA visits every point whose
//   stencil can touch its tile (its own bins plus the neighbours' bins whose
//   reach class points at it), accumulates the in-tile contributions in shared
//   memory, and writes every face of its tile exactly once (zeros included).
//   No global atomics, no zero-fill pass: each face is written by one CTA.
//     FP64:  FP64 shared-memory accumulation.
//     FP32C: FP32 weights and products, each quantised to fixed point and
//            summed exactly (32-bit integer shared atomics folded into FP64
//            totals; order-independent).  See fix_add below.
//
// interp_tile_kernel  -- one CTA per (tile, component) stages the tile plus
//   its stencil halo in shared memory with one TMA bulk tensor copy; at a
//   domain edge the out-of-range slabs are then patched with loads that wrap
//   periodic halos and clamp wall halos exactly as the reference clamps node
//   indices.  Every point of the tile then gathers its M^dims nodes from
//   shared memory.
//     FP64:  exact weights, sums in the reference's pattern order (bit-exact).
//     FP32C: the staged values rounded to FP32 in shared memory (half the
//            shared-memory traffic of the gathers), FP32 weights, FP32 row
//            sums of M products, FP64 sum of the rows.
#pragma once
#include "ibk_device.cuh"
#include "ibk_bin.cuh"
#include "ibk_tma.cuh"

namespace ibk {

constexpr int kTileThreads = 256;

// Tile-local description of one dimension for one component.
struct TileAxis {
	int lo;      // first face index of the tile
	int hi;      // one past the last face owned by the tile (clipped to points)
};

__device__ __forceinline__ void tile_coords(const TileGeom& tg, int t, int* tc)
{
	tc[0] = t % tg.ntiles[0];
	int r = t / tg.ntiles[0];
	tc[1] = r % tg.ntiles[1];
	tc[2] = r / tg.ntiles[1];
}

// All M weights of one axis in FP32 for fractional offset delta.
template <typename D>
__device__ __forceinline__ void weights32(float delta, float* w)
{
	constexpr int M = D::M, sh = (M - 1) >> 1;
#pragma unroll
	for (int m = 0; m < M; ++m) w[m] = D::phi32(delta + (float) (m - sh));
}
// Cubic B-spline (bspline<3>) in closed form: t = -delta in [0, 1).
template <>
__device__ __forceinline__ void weights32<Delta<kBspline, 3>>(float delta, float* w)
{
	const float t = -delta, u = 1.0f - t;
	const float t2 = t * t, u2 = u * u;
	w[0] = u2 * u * (1.0f / 6.0f);
	w[1] = fmaf(0.5f * t, t2, 2.0f / 3.0f - t2);
	w[2] = fmaf(0.5f * u, u2, 2.0f / 3.0f - u2);
	w[3] = t2 * t * (1.0f / 6.0f);
}

// Largest weight of the dims-dimensional tensor-product stencil (bound used
// by the fixed-point scale).  phi <= 1 for every delta here; the cubic
// B-spline is at most 2/3 per axis.
template <typename D, int DIMS>
__host__ __device__ constexpr float max_weight()
{
	return (D::M == 4 && !D::every_other) ? (DIMS == 3 ? 8.0f / 27.0f : 4.0f / 9.0f) : 1.0f;
}

// ------------------------------------------------------------ ranges ---
// The bins a tile must visit: per axis five (neighbour offset, class)
// choices: (-1, upper), (0, lower), (0, inside), (0, upper), (+1, lower).
constexpr int kMaxRanges = 125;

struct RangeTable {
	int start[kMaxRanges];
	int pref[kMaxRanges + 1];
	int count;
	unsigned fmax_bits;     // spread: max over the candidate bins of binmax[bin][comp]
};

template <int DIMS>
__device__ __forceinline__ void build_ranges(const GridGeom& g, const TileGeom& tg, const int* tc,
                                             const int* __restrict__ off, RangeTable& rt, bool neighbours,
                                             const unsigned* __restrict__ binmax = nullptr, int comp = 0)
{
	const int nent = neighbours ? (DIMS == 3 ? 125 : 25) : 1;
	const int tid = threadIdx.x;
	int len = 0, st = 0;
	unsigned fm = 0;
	if (tid < nent) {
		int tile = 0, cls = 0, ts = 1, cs = 1;
		bool ok = true;
		int e = tid;
		for (int d = 0; d < DIMS; ++d) {
			int k = neighbours ? e % 5 : 1;
			e /= 5;
			int o = k == 0 ? -1 : (k == 4 ? 1 : 0);
			int c = k == 0 ? 2 : (k == 4 ? 0 : k - 1);
			int nt = tg.ntiles[d];
			int t = tc[d] + o;
			if (o != 0) {
				if (nt == 1) ok = false;
				else if (g.solid[d]) ok = ok && t >= 0 && t < nt;
				else t = (t + nt) % nt;
			}
			tile += t * ts;
			ts *= nt;
			cls += c * cs;
			cs *= 3;
		}
		if (!neighbours) {
			// the tile's own points: all classes, one contiguous range
			st = off[tile * tg.nclass];
			len = off[tile * tg.nclass + tg.nclass] - st;
		} else if (ok) {
			const int bin = tile * tg.nclass + cls;
			st = off[bin];
			len = off[bin + 1] - st;
			if (binmax != nullptr && len > 0) fm = binmax[(size_t) bin * kMaxDims + comp];
		}
		rt.start[tid] = st;
	}
	// block-wide exclusive scan of len over the first 128 threads
	__shared__ int warp_tot[4];
	__shared__ unsigned warp_fm[4];
	const int lane = tid & 31, warp = tid >> 5;
	int incl = (tid < 128) ? len : 0;
	if (tid < 128) {
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int v = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o) incl += v;
		}
		const unsigned wm = __reduce_max_sync(0xffffffffu, fm);
		if (lane == 31) {
			warp_tot[warp] = incl;
			warp_fm[warp] = wm;
		}
	}
	__syncthreads();
	if (tid < 128) {
		int base = 0;
		for (int w = 0; w < warp; ++w) base += warp_tot[w];
		if (tid < nent) rt.pref[tid] = base + incl - len;
		if (tid == nent - 1) {
			rt.pref[nent] = base + incl;
			rt.count = nent;
			rt.fmax_bits = max(max(warp_fm[0], warp_fm[1]), max(warp_fm[2], warp_fm[3]));
		}
	}
	__syncthreads();
}

// The point slot of candidate item (items number the tile's ranges back to
// back) for a thread whose items only increase: r is the range of its
// previous item (0 before the first) and moves forward past the ranges that
// end at or before item (pref[count] is past every item, so the walk stops).
__device__ __forceinline__ int range_walk(const RangeTable& rt, int& r, int item)
{
	while (rt.pref[r + 1] <= item) ++r;
	return rt.start[r] + (item - rt.pref[r]);
}

// ------------------------------------------------------------ spread ---

// arr[m] for a run-time m without dynamic register indexing.
template <int M, typename T>
__device__ __forceinline__ T select_m(const T* arr, int m)
{
	T r = arr[0];
#pragma unroll
	for (int k = 1; k < M; ++k) r = (m == k) ? arr[k] : r;
	return r;
}

template <typename D, int DIMS, int PREC>
struct SpreadSmem;
template <typename D, int DIMS>
struct SpreadSmem<D, DIMS, IBK_PRECISION_FP64> { using acc_t = double; };
template <typename D, int DIMS>
struct SpreadSmem<D, DIMS, IBK_PRECISION_FP32C> { using acc_t = int; };

// Fixed point of the FP32C spread.  Each FP32 product is scaled so that the
// largest possible term of the tile (max|w| * res * max|F| over the tile's
// candidate points) is below 2^22, rounded to an integer with the float magic
// number 1.5 * 2^23 (x + magic carries rint(x) in its low mantissa bits for
// |x| <= 2^22: an FADD and an integer subtract, no conversion instruction),
// and added to the face's 32-bit working word with one integer shared atomic.
// At most kFixChunk candidates are summed between folds (kFixChunk * 2^22 <
// 2^31, so a working word cannot overflow); each fold adds the working words
// exactly into an FP64 total per face (integers below 2^53 are exact in
// FP64).  The sum is therefore exact and independent of the order in which
// points are visited (the binning order is not deterministic; the result
// is); the only rounding is each product's quantisation to 2^-23 of the
// tile's largest possible term, and the final scaling is exact.
constexpr float kMagic = 12582912.0f;           // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr int kFixChunk = 511;                  // candidates between folds
constexpr int kFixTermLog2 = 22;                // largest term * scale < 2^22

__device__ __forceinline__ void fix_add(int* word, float s)
{
	atomicAdd(word, __float_as_int(s + kMagic) - kMagicBits);   // rint(s)
}

// fix_add of the product a * b, rounded once (rint of the exact product).
__device__ __forceinline__ void fix_add_product(int* word, float a, float b)
{
	atomicAdd(word, __float_as_int(__fmaf_rn(a, b, kMagic)) - kMagicBits);
}

// The fixed-point increments of a0 * b and a1 * b (each rounded once, as in
// fix_add_product), from one packed two-lane FP32 FMA.
__device__ __forceinline__ int2 fix_terms2(float a0, float a1, float b)
{
	float r0, r1;
	asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\t"
	    "mov.b64 pa, {%2, %3};\n\t"
	    "mov.b64 pb, {%4, %4};\n\t"
	    "mov.b64 pc, {%5, %5};\n\t"
	    "fma.rn.f32x2 pd, pa, pb, pc;\n\t"
	    "mov.b64 {%0, %1}, pd;\n\t}"
	    : "=f"(r0), "=f"(r1) : "f"(a0), "f"(a1), "f"(b), "f"(kMagic));
	return make_int2(__float_as_int(r0) - kMagicBits, __float_as_int(r1) - kMagicBits);
}

// One candidate point p of a spread tile [lo, hi): its in-tile stencil
// contributions added to the tile's accumulators (F is read only when the
// stencil touches the tile).  FP32C: the FP32 product res * F is scaled by
// the tile's fixed-point scale.
// contig: the tile spans no periodic axis whole, so the in-tile nodes of a
// stencil are consecutive along every axis and their accumulators sit at
// fixed offsets from the first one.
// near: contig, and every periodic axis has more cells than M + the tile's
// extent.  A stencil that meets the tile then does so after at most one shift
// by the period, which places its centre within half a period of the tile's
// centre; its in-tile nodes follow from the shifted position of node 0
// without wrapping every node.
template <typename D, int DIMS, int PREC>
__device__ __forceinline__ void spread_candidate(const GridGeom& g, const CompGeom& cg, int n,
                                                 const double* __restrict__ x, const double* __restrict__ fc,
                                                 int p, float scale, const int* lo, const int* hi, int S1, int S2,
                                                 bool contig, bool near, typename SpreadSmem<D, DIMS, PREC>::acc_t* acc)
{
	constexpr int M = D::M, sh = (M - 1) >> 1;
	int loc[DIMS][M];
	unsigned mask[DIMS];
	int lb[DIMS];           // near: tile-local position of node 0 (may lie outside)
	double dl[DIMS];
	bool any = true;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		AxisStep<M> a = axis_step<M>(g, cg, d, __ldg(x + (size_t) d * n + p));
		dl[d] = a.delta;
		unsigned mk = 0;
		if (near) {
			// spread drops nodes outside [0, points) (errors_negative) and this
			// tile owns [lo, hi): node m is in it iff 0 <= l + m < hi - lo
			int l = a.base - sh - lo[d];
			const int e = hi[d] - lo[d];
			if (!g.solid[d]) {
				const int C = cg.cells[d], twice = 2 * l + M - e;
				l += twice > C ? -C : (twice < -C ? C : 0);
			}
			const int m_lo = max(0, -l), m_hi = min(M, e - l);
			mk = m_hi > m_lo ? ((1u << m_hi) - 1u) & ~((1u << m_lo) - 1u) : 0u;
			lb[d] = l;
#pragma unroll
			for (int m = 0; m < M; ++m) loc[d][m] = l + m;
		} else {
			lb[d] = 0;
#pragma unroll
			for (int m = 0; m < M; ++m) {
				const int j = node_index(g, cg, d, a.base + m - sh);
				loc[d][m] = j - lo[d];
				mk |= (unsigned) (j >= lo[d] && j < hi[d]) << m;
			}
		}
		mask[d] = mk;
		any = any && mk;
	}
	if (!any) return;
	if constexpr (PREC == IBK_PRECISION_FP64) {
		const double f = __dmul_rn(g.res, __ldg(fc + p));
		double w[DIMS][M];
#pragma unroll
		for (int d = 0; d < DIMS; ++d)
#pragma unroll
			for (int m = 0; m < M; ++m)
				w[d][m] = (mask[d] >> m & 1u) ? D::phi64(__dadd_rn(dl[d], (double) (m - sh))) : 0.0;
#pragma unroll
		for (int m0 = 0; m0 < M; ++m0) w[0][m0] = __dmul_rn(w[0][m0], f);
#pragma unroll
		for (int r = 0; r < (DIMS == 3 ? M * M : M); ++r) {
			const int m1 = r % M, m2 = r / M;
			const unsigned rm = DIMS == 3 ? (mask[1] >> m1) & (mask[2] >> m2) & 1u : (mask[1] >> m1) & 1u;
			if (!rm) continue;   // rows outside the tile (mostly warp-uniform)
			const double w12 = DIMS == 3 ? __dmul_rn(w[1][m1], w[2][m2]) : w[1][m1];
			const int row = (DIMS == 3 ? loc[2][m2] * S2 : 0) + loc[1][m1] * S1;
#pragma unroll
			for (int m0 = 0; m0 < M; ++m0)
				if ((mask[0] >> m0) & rm)
					atomicAdd(acc + row + loc[0][m0], __dmul_rn(w[0][m0], w12));
		}
	} else {
		const float f = (float) (g.res * __ldg(fc + p)) * scale;
		float w[DIMS][M];
#pragma unroll
		for (int d = 0; d < DIMS; ++d) weights32<D>((float) dl[d], w[d]);
#pragma unroll
		for (int m0 = 0; m0 < M; ++m0) w[0][m0] *= f;
		if (contig) {
			// node (m0, m1, m2) at first + m2 * S2 + m1 * S1 + m0, where
			// first is the (possibly outside) position of node (0, 0, 0)
			if (!near) {
#pragma unroll
				for (int d = 0; d < DIMS; ++d) {
					int v = 0;
					bool found = false;
#pragma unroll
					for (int m = 0; m < M; ++m)
						if (!found && ((mask[d] >> m) & 1u)) { v = loc[d][m] - m; found = true; }
					lb[d] = v;
				}
			}
			const int first = (DIMS == 3 ? lb[2] * S2 : 0) + lb[1] * S1 + lb[0];
			int* base = acc + first;
			constexpr unsigned kFull = (1u << M) - 1u;
			const bool full = mask[0] == kFull && mask[1] == kFull && (DIMS < 3 || mask[2] == kFull);
			if (full) {
				// the whole stencil inside the tile: no per-node tests
#pragma unroll
				for (int r = 0; r < (DIMS == 3 ? M * M : M); ++r) {
					const int m1 = r % M, m2 = r / M;
					const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
					int* rowp = base + (DIMS == 3 ? m2 * S2 : 0) + m1 * S1;
#pragma unroll
					for (int m0 = 0; m0 + 1 < M; m0 += 2) {
						const int2 t = fix_terms2(w[0][m0], w[0][m0 + 1], w12);
						atomicAdd(rowp + m0, t.x);
						atomicAdd(rowp + m0 + 1, t.y);
					}
					if (M & 1) fix_add_product(rowp + (M - 1), w[0][M - 1], w12);
				}
			} else {
#pragma unroll
				for (int r = 0; r < (DIMS == 3 ? M * M : M); ++r) {
					const int m1 = r % M, m2 = r / M;
					const unsigned rm = DIMS == 3 ? (mask[1] >> m1) & (mask[2] >> m2) & 1u : (mask[1] >> m1) & 1u;
					if (!rm) continue;   // rows outside the tile (mostly warp-uniform)
					const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
					int* rowp = base + (DIMS == 3 ? m2 * S2 : 0) + m1 * S1;
#pragma unroll
					for (int m0 = 0; m0 + 1 < M; m0 += 2) {
						const int2 t = fix_terms2(w[0][m0], w[0][m0 + 1], w12);
						if ((mask[0] >> m0) & 1u) atomicAdd(rowp + m0, t.x);
						if ((mask[0] >> (m0 + 1)) & 1u) atomicAdd(rowp + m0 + 1, t.y);
					}
					if ((M & 1) && ((mask[0] >> (M - 1)) & 1u)) fix_add_product(rowp + (M - 1), w[0][M - 1], w12);
				}
			}
		} else {
#pragma unroll
			for (int r = 0; r < (DIMS == 3 ? M * M : M); ++r) {
				const int m1 = r % M, m2 = r / M;
				const unsigned rm = DIMS == 3 ? (mask[1] >> m1) & (mask[2] >> m2) & 1u : (mask[1] >> m1) & 1u;
				if (!rm) continue;
				const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
				const int row = (DIMS == 3 ? loc[2][m2] * S2 : 0) + loc[1][m1] * S1;
#pragma unroll
				for (int m0 = 0; m0 < M; ++m0)
					if ((mask[0] >> m0) & rm) fix_add_product(acc + row + loc[0][m0], w[0][m0], w12);
			}
		}
	}
}

// One (tile, component) of the spread; every thread of the CTA calls it.
// perm holds point indices offset by pbase (a batch numbers the points of
// all its instances consecutively); off and binmax are this grid's bins.
template <typename D, int DIMS, int PREC, int NT = kTileThreads>
__device__ __forceinline__ void spread_tile(const GridGeom& g, const TileGeom& tg, int n, const double* __restrict__ x,
                                            const double* __restrict__ fl, const int* __restrict__ perm, int pbase,
                                            const int* __restrict__ off, const unsigned* __restrict__ binmax,
                                            const CompPtrs& fe, int tile, int c)
{
	using acc_t = typename SpreadSmem<D, DIMS, PREC>::acc_t;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ RangeTable rt;

	const CompGeom& cg = g.comp[c];
	const int T0 = tg.T[0], T1 = tg.T[1], T2 = DIMS == 3 ? tg.T[2] : 1;
	const SpreadStrides ss = spread_strides(T0, T1, T2, DIMS);
	const int TV = ss.words;    // padded accumulator words
	// FP64: acc[TV] doubles.  FP32C: total[TV] doubles, then acc[TV] working words.
	double* total = reinterpret_cast<double*>(smem_raw);
	acc_t* acc = PREC == IBK_PRECISION_FP64 ? reinterpret_cast<acc_t*>(smem_raw)
	                                        : reinterpret_cast<acc_t*>(total + TV);
	int tc[3] = {0, 0, 0};
	tile_coords(tg, tile, tc);
	int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
	bool contig = true, near = true;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		lo[d] = tc[d] * tg.T[d];
		hi[d] = min(lo[d] + tg.T[d], cg.points[d]);
		contig = contig && (g.solid[d] || tg.ntiles[d] > 1);
		near = near && (g.solid[d] || D::M + tg.T[d] < cg.cells[d]);
	}
	near = near && contig;
	build_ranges<DIMS>(g, tg, tc, off, rt, true, binmax, c);
	const double* __restrict__ fc = fl + (size_t) c * n;
	const int e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = DIMS == 3 ? hi[2] - lo[2] : 1;
	double* __restrict__ out = fe.p[c];
	const int ncand = rt.pref[rt.count];
	if (ncand == 0) {
		// no point reaches the tile: its faces are zero
		for (int i = threadIdx.x; i < e1 * e2 * T0; i += NT) {
			const int l0 = i % T0;
			const int r = i / T0;
			if (l0 >= e0) continue;
			const int l1 = r % e1, l2 = r / e1;
			out[(size_t) (lo[0] + l0) + (size_t) cg.points[0] *
			    ((size_t) (lo[1] + l1) + (DIMS == 3 ? (size_t) cg.points[1] * (size_t) (lo[2] + l2) : 0))] = 0.0;
		}
		return;
	}
	for (int i = threadIdx.x; i < TV; i += NT) acc[i] = (acc_t) 0;
	if constexpr (PREC == IBK_PRECISION_FP32C)
		for (int i = threadIdx.x; i < TV; i += NT) total[i] = 0.0;
	__syncthreads();

	double inv_scale = 1.0;     // FP32C: back to force density (exact power of two)
	if constexpr (PREC == IBK_PRECISION_FP64) {
		int r = 0;
		for (int it = threadIdx.x; it < ncand; it += NT)
			spread_candidate<D, DIMS, PREC>(g, cg, n, x, fc, __ldg(perm + range_walk(rt, r, it)) - pbase, 0.0f,
			                                lo, hi, ss.S1, ss.S2, contig, near, acc);
	} else {
		// the tile's largest possible term, max|F| * max|w| * res (max|F| over
		// its candidate bins, rounded to FP32, hence the 1.001), is scaled to
		// below 2^22; at most kFixChunk candidates between folds
		const float bound = __uint_as_float(rt.fmax_bits) * 1.001f * max_weight<D, DIMS>() * (float) g.res + 1e-30f;
		int e;
		frexpf(bound, &e);                      // bound < 2^e
		const float scale = ldexpf(1.0f, min(kFixTermLog2 - e, 126));
		int r = 0;              // this thread's items increase across the chunks
		for (int base = 0; base < ncand; base += kFixChunk) {
			const int stop = min(ncand, base + kFixChunk);
			for (int it = base + threadIdx.x; it < stop; it += NT)
				spread_candidate<D, DIMS, PREC>(g, cg, n, x, fc, __ldg(perm + range_walk(rt, r, it)) - pbase, scale,
				                                lo, hi, ss.S1, ss.S2, contig, near, acc);
			// fold the working words into the exact FP64 totals
			__syncthreads();
			for (int i = threadIdx.x; i < TV; i += NT) {
				total[i] += (double) acc[i];
				acc[i] = 0;
			}
			__syncthreads();
		}
		inv_scale = 1.0 / (double) scale;
	}
	__syncthreads();

	// every face of the tile, written once
	for (int i = threadIdx.x; i < e1 * e2 * T0; i += NT) {
		const int l0 = i % T0;
		const int r = i / T0;
		if (l0 >= e0) continue;
		const int l1 = r % e1, l2 = r / e1;
		const size_t gi = (size_t) (lo[0] + l0) + (size_t) cg.points[0] *
			((size_t) (lo[1] + l1) + (DIMS == 3 ? (size_t) cg.points[1] * (size_t) (lo[2] + l2) : 0));
		const int li = (DIMS == 3 ? l2 * ss.S2 : 0) + l1 * ss.S1 + l0;
		if constexpr (PREC == IBK_PRECISION_FP64) out[gi] = acc[li];
		else out[gi] = total[li] * inv_scale;
	}
}

// NT threads per CTA; FP32C CTAs are capped at 64 registers per thread so
// that 1024 threads of them fit on an SM, FP64 ones (256 threads) at 85 so
// that three fit.
template <typename D, int DIMS, int PREC, int NT>
__global__ void __launch_bounds__(NT, PREC == IBK_PRECISION_FP32C ? 1024 / NT : 3)
spread_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const double* __restrict__ fl, const int* __restrict__ perm,
                   const int* __restrict__ off, const unsigned* __restrict__ binmax, CompPtrs fe)
{
	// grid: (tile, component)
	spread_tile<D, DIMS, PREC, NT>(g, tg, n, x, fl, perm, 0, off, binmax, fe, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ interp ---

// Halo of the staged region around the tile, per side.
template <int M> struct Halo {
	static constexpr int lo = 1 + ((M - 1) >> 1);
	static constexpr int hi = 1 + M / 2;
};

// Fold a region coordinate onto the grid: wrap periodic axes, clamp walls.
__device__ __forceinline__ int fold(const GridGeom& g, const CompGeom& cg, int d, int v)
{
	const int pd = cg.points[d];
	if (g.solid[d]) return v < 0 ? 0 : (v >= pd ? pd - 1 : v);
	if (v < 0 || v >= pd) v = wrap_index(v, cg.cells[d]);
	return v;
}

// Staged-region geometry shared by host and device: the x extent is padded to
// an even count so a TMA box row is a multiple of 16 bytes.
template <int M>
__host__ __device__ inline int region_extent(int T, int d)
{
	const int e = T + Halo<M>::lo + Halo<M>::hi;
	return d == 0 ? (e + 1) & ~1 : e;
}

// Epilogue of the serving step, applied to each interpolated velocity U of
// component c at point p: forward Euler advection and a linear spring to the
// point's reference position,
//   xn = x + dt * U,   fl = -k * (xn - xref)    (FP64, no contraction).
struct StepEpilogue {
	double* xn;             // 3n, advected positions
	double* fl;             // 3n, spring forces at xn
	const double* xref;     // 3n, reference positions
	double dt, k;
};

// One (tile, component) of the interpolation; every thread of the CTA calls
// it.  maps/use_tma select TMA staging (maps_global: the maps live in global
// memory, written by a copy before the launch); epi, when not null, adds the
// serving-step epilogue; ul may then be null.  Returns false only when a
// bounded wait for the staging copy gave up (the status word records it and
// the CTA must stop).
template <typename D, int DIMS, int PREC>
__device__ __forceinline__ bool interp_tile(const GridGeom& g, const TileGeom& tg, int n, const double* __restrict__ x,
                                            const int* __restrict__ perm, int pbase, const int* __restrict__ off,
                                            const ConstCompPtrs& ue, double* __restrict__ ul,
                                            const CUtensorMap* maps, int use_tma, bool maps_global, int* status,
                                            const StepEpilogue* epi, int t, int c)
{
	using P = Pattern<D::M, DIMS, D::every_other>;
	constexpr int M = D::M, sh = (M - 1) >> 1;
	constexpr int HL = Halo<M>::lo;
	// The region pointer is aligned to 128 bytes by hand (TMA destination);
	// the launch adds 128 bytes of slack for it.
	extern __shared__ __align__(16) unsigned char interp_smem[];
	double* reg = reinterpret_cast<double*>(interp_smem + ((128u - (smem_addr(interp_smem) & 127u)) & 127u));
	__shared__ __align__(8) uint64_t bar;

	const int start = __ldg(off + t * tg.nclass);
	const int end = __ldg(off + (t + 1) * tg.nclass);
	if (start == end) return true;
	const CompGeom& cg = g.comp[c];
	const double* __restrict__ u = ue.p[c];
	int tc[3] = {0, 0, 0};
	tile_coords(tg, t, tc);
	int rlo[3] = {0, 0, 0}, E[3] = {1, 1, 1};
	bool tma = use_tma != 0;        // stage with one bulk tensor copy
	bool interior = true;           // the region lies inside the grid
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		rlo[d] = tc[d] * tg.T[d] - HL;
		E[d] = region_extent<M>(tg.T[d], d);
		interior = interior && rlo[d] >= 0 && rlo[d] + E[d] <= cg.points[d];
	}
	// self-check of the TMA preconditions: 128-byte destination, x origin
	// on a 16-byte boundary; a violation is recorded and the region staged
	// by plain loads instead
	if (tma && (((smem_addr(reg) & 127u) != 0u) || (rlo[0] & 1) != 0)) {
		if (threadIdx.x == 0 && status) atomicExch(status, 2);
		tma = false;
	}
	// first point of this thread, fetched while the region is staged
	int it = start + threadIdx.x;
	int p_next = 0;
	double z_next[DIMS];
	if (it < end) {
		p_next = __ldg(perm + it) - pbase;
#pragma unroll
		for (int d = 0; d < DIMS; ++d) z_next[d] = __ldg(x + (size_t) d * n + p_next);
	}
	if (tma) {
		// one bulk tensor copy of the box; at a domain edge the box starts at a
		// negative or past-the-end coordinate and the copy zero-fills those
		// elements, which are patched below
		if (threadIdx.x == 0) mbar_init(&bar, 1);
		__syncthreads();
		if (threadIdx.x == 0) {
			if (maps_global) tensormap_acquire(maps + c);
			fence_proxy_async_smem();       // a persistent CTA's accesses to the previous tile's region
			mbar_arrive_expect_tx(&bar, (unsigned) (sizeof(double) * E[0] * E[1] * E[2]));
			if constexpr (DIMS == 3) tma_load_3d(reg, maps + c, rlo[0], rlo[1], rlo[2], &bar);
			else tma_load_2d(reg, maps + c, rlo[0], rlo[1], &bar);
		}
		// one thread polls the mbarrier; the others park at the CTA barrier
		// (no issue slots spent spinning)
		__shared__ int tma_ok;
		if (threadIdx.x == 0) tma_ok = mbar_wait_bounded(&bar, 0, status) ? 1 : 0;
		__syncthreads();
		if (!tma_ok) return false;
		if (threadIdx.x == 0) mbar_inval(&bar);   // every thread is past the wait
		if (!interior) {
			// out-of-range slabs: wrap periodic, clamp solid (interpolate.h:16-22)
#pragma unroll 1
			for (int d = 0; d < DIMS; ++d) {
				const int below = max(0, -rlo[d]);
				const int above_from = min(E[d], cg.points[d] - rlo[d]);
				const int other = (E[0] * E[1] * E[2]) / E[d];
#pragma unroll 1
				for (int side = 0; side < 2; ++side) {
					const int s0 = side == 0 ? 0 : max(above_from, 0);
					const int s1 = side == 0 ? below : E[d];
					const int cnt = (s1 - s0) * other;
					for (int i = threadIdx.x; i < cnt; i += kTileThreads) {
						// element i of the slab: coordinate along d, then the others
						int l[3] = {0, 0, 0};
						l[d] = s0 + i / other;
						int rest = i % other;
#pragma unroll
						for (int e = 0; e < DIMS; ++e) {
							if (e == d) continue;
							l[e] = rest % E[e];
							rest /= E[e];
						}
						size_t gi = 0, stride = 1;
#pragma unroll
						for (int e = 0; e < DIMS; ++e) {
							gi += (size_t) fold(g, cg, e, rlo[e] + l[e]) * stride;
							stride *= (size_t) cg.points[e];
						}
						reg[(DIMS == 3 ? (l[2] * E[1] + l[1]) : l[1]) * E[0] + l[0]] = __ldg(u + gi);
					}
				}
			}
			__syncthreads();
		}
	} else {
		// plain row copies that wrap periodic and clamp solid halos: a warp
		// per row, lanes along x, kRowsInFlight rows' loads issued before
		// their stores
		constexpr int kRowsInFlight = 4;
		constexpr int kWarps = kTileThreads / 32;
		const int rows = E[1] * E[2];
		const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
		for (int r0 = warp; r0 < rows; r0 += kWarps * kRowsInFlight) {
			double v[kRowsInFlight][2];
#pragma unroll
			for (int q = 0; q < kRowsInFlight; ++q) {
				const int r = r0 + q * kWarps;
				if (r >= rows) break;
				const int l1 = r % E[1], l2 = r / E[1];
				size_t rb = (size_t) fold(g, cg, 1, rlo[1] + l1);
				if (DIMS == 3) rb += (size_t) cg.points[1] * (size_t) fold(g, cg, 2, rlo[2] + l2);
				rb *= (size_t) cg.points[0];
#pragma unroll
				for (int h = 0; h < 2; ++h) {
					const int l0 = lane + 32 * h;
					if (l0 < E[0]) v[q][h] = __ldg(u + rb + fold(g, cg, 0, rlo[0] + l0));
				}
			}
#pragma unroll
			for (int q = 0; q < kRowsInFlight; ++q) {
				const int r = r0 + q * kWarps;
				if (r >= rows) break;
#pragma unroll
				for (int h = 0; h < 2; ++h) {
					const int l0 = lane + 32 * h;
					if (l0 < E[0]) reg[(size_t) r * E[0] + l0] = v[q][h];
				}
			}
		}
		// wider regions (x extent above 64) finish row by row
		if (E[0] > 64) {
			for (int r = warp; r < rows; r += kWarps) {
				const int l1 = r % E[1], l2 = r / E[1];
				size_t rb = (size_t) fold(g, cg, 1, rlo[1] + l1);
				if (DIMS == 3) rb += (size_t) cg.points[1] * (size_t) fold(g, cg, 2, rlo[2] + l2);
				rb *= (size_t) cg.points[0];
				for (int l0 = 64 + lane; l0 < E[0]; l0 += 32)
					reg[(size_t) r * E[0] + l0] = __ldg(u + rb + fold(g, cg, 0, rlo[0] + l0));
			}
		}
		__syncthreads();
	}
	if constexpr (PREC == IBK_PRECISION_FP32C) {
		// the staged FP64 values rounded to FP32 in place, in chunks: a chunk's
		// FP32 words land on FP64 elements that are read by then
		constexpr int kChunk = kTileThreads * 8;
		const int vol = E[0] * E[1] * E[2];
		float* regf = reinterpret_cast<float*>(reg);
		for (int b0 = 0; b0 < vol; b0 += kChunk) {
			double v8[8];
#pragma unroll
			for (int q = 0; q < 8; ++q) {
				const int i = b0 + q * kTileThreads + threadIdx.x;
				v8[q] = i < vol ? reg[i] : 0.0;
			}
			__syncthreads();
#pragma unroll
			for (int q = 0; q < 8; ++q) {
				const int i = b0 + q * kTileThreads + threadIdx.x;
				if (i < vol) regf[i] = (float) v8[q];
			}
			__syncthreads();
		}
	}
	for (; it < end; it += kTileThreads) {
		const int p = p_next;
		double z[DIMS];
#pragma unroll
		for (int d = 0; d < DIMS; ++d) z[d] = z_next[d];
		if (it + kTileThreads < end) {          // prefetch the next point
			p_next = __ldg(perm + it + kTileThreads) - pbase;
#pragma unroll
			for (int d = 0; d < DIMS; ++d) z_next[d] = __ldg(x + (size_t) d * n + p_next);
		}
		int loc[DIMS];          // local index of the stencil's first node
		double dl[DIMS];
		bool inside = true;
#pragma unroll
		for (int d = 0; d < DIMS; ++d) {
			AxisStep<M> a = axis_step<M>(g, cg, d, z[d]);
			dl[d] = a.delta;
			int b = a.base;
			if (!g.solid[d] && tg.ntiles[d] > 1) {
				const int cells = cg.cells[d];
				const int diff = b - (rlo[d] + HL);
				if (2 * diff > cells) b -= cells;
				else if (2 * diff < -cells) b += cells;
			}
			const int l = b - sh - rlo[d];
			loc[d] = l;
			inside = inside && l >= 0 && l + M <= E[d];
		}
		double v;
		if (inside) {
			const int base = DIMS == 3 ? (loc[2] * E[1] + loc[1]) * E[0] + loc[0] : loc[1] * E[0] + loc[0];
			if constexpr (PREC == IBK_PRECISION_FP64) {
				double w[DIMS][M];
#pragma unroll
				for (int d = 0; d < DIMS; ++d)
#pragma unroll
					for (int m = 0; m < M; ++m) w[d][m] = D::phi64(__dadd_rn(dl[d], (double) (m - sh)));
				v = 0.0;
#pragma unroll
				for (int e = 0; e < P::V; ++e) {
					const int m0 = P::m(e, 0), m1 = P::m(e, 1);
					double wt;
					int k;
					if constexpr (DIMS == 3) {
						const int m2 = P::m(e, 2);
						wt = __dmul_rn(w[0][m0], __dmul_rn(w[1][m1], w[2][m2]));
						k = base + (m2 * E[1] + m1) * E[0] + m0;
					} else {
						wt = __dmul_rn(w[0][m0], w[1][m1]);
						k = base + m1 * E[0] + m0;
					}
					v = __dadd_rn(v, __dmul_rn(wt, reg[k]));   // interpolate.h:71-72
				}
			} else {
				// FP32 weights and FP32 staged values; FP32 row sums, FP64 total
				float w32[DIMS][M];
#pragma unroll
				for (int d = 0; d < DIMS; ++d) weights32<D>((float) dl[d], w32[d]);
				const float* regf = reinterpret_cast<const float*>(reg);
				v = 0.0;
				constexpr int R = DIMS == 3 ? M * M : M;
#pragma unroll
				for (int r = 0; r < R; ++r) {
					const int m1 = r % M, m2 = r / M;
					const float* row = regf + base + (DIMS == 3 ? (m2 * E[1] + m1) * E[0] : m1 * E[0]);
					float rs = 0.0f;
#pragma unroll
					for (int m0 = 0; m0 < M; ++m0) rs = fmaf(w32[0][m0], row[m0], rs);
					const double w12 = DIMS == 3 ? (double) w32[1][m1] * (double) w32[2][m2] : (double) w32[1][m1];
					v = fma(w12, (double) rs, v);
				}
			}
		} else {
			// stencil leaves the staged region: exact global gather
			int gidx[DIMS][M];
			double w[DIMS][M];
#pragma unroll
			for (int d = 0; d < DIMS; ++d) {
				AxisStep<M> a = axis_step<M>(g, cg, d, z[d]);
#pragma unroll
				for (int m = 0; m < M; ++m) {
					const int j = node_index(g, cg, d, a.base + m - sh);
					const int pd = cg.points[d];
					gidx[d][m] = j < 0 ? 0 : (j >= pd ? pd - 1 : j);
					w[d][m] = D::phi64(__dadd_rn(a.delta, (double) (m - sh)));
				}
			}
			v = 0.0;
#pragma unroll
			for (int e = 0; e < P::V; ++e) {
				const int m0 = P::m(e, 0), m1 = P::m(e, 1);
				double wt;
				long long k;
				if constexpr (DIMS == 3) {
					const int m2 = P::m(e, 2);
					wt = __dmul_rn(w[0][m0], __dmul_rn(w[1][m1], w[2][m2]));
					k = gidx[0][m0] + (long long) cg.points[0] * (gidx[1][m1] + (long long) cg.points[1] * gidx[2][m2]);
				} else {
					wt = __dmul_rn(w[0][m0], w[1][m1]);
					k = gidx[0][m0] + (long long) cg.points[0] * gidx[1][m1];
				}
				v = __dadd_rn(v, __dmul_rn(wt, __ldg(u + k)));
			}
		}
		const size_t i = (size_t) c * n + p;
		if (ul != nullptr) ul[i] = v;
		if (epi != nullptr) {
			double zc = z[0];
#pragma unroll
			for (int d = 1; d < DIMS; ++d) zc = d == c ? z[d] : zc;
			const double xn = __dadd_rn(zc, __dmul_rn(epi->dt, v));
			epi->xn[i] = xn;
			epi->fl[i] = __dmul_rn(-epi->k, __dsub_rn(xn, __ldg(epi->xref + i)));
		}
	}
	return true;
}

template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads, D::M <= 4 ? 2 : 1)
interp_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const int* __restrict__ perm, const int* __restrict__ off,
                   ConstCompPtrs ue, double* __restrict__ ul,
                   const __grid_constant__ TmaMaps maps, int use_tma, int* status)
{
	// grid: (tile, component)
	interp_tile<D, DIMS, PREC>(g, tg, n, x, perm, 0, off, ue, ul, maps.map, use_tma, false, status, nullptr,
	                           blockIdx.x, blockIdx.y);
}

} // namespace ibk
