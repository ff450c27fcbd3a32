// Tiled kernels: the throughput path of spread and interpolate.
//
// Points are binned by (home tile, reach class) into 32-byte records in bin
// order (ibk_bin.cuh).  A tile is a box of T0 x T1 x T2 grid cells.
//
// spread_tile  -- owner computes.  The CTA visits every point whose stencil
//   can touch its tile (its own bins plus the neighbours' bins whose reach
//   class points at it), accumulates the in-tile contributions in shared
//   memory, and writes every face of its tile exactly once (zeros included).
//   No global atomics, no zero-fill pass: each face is written by one CTA.
//     FP32C: one CTA per tile for every component.  FP32 weights and
//            products, each rounded once to a per-(tile, component) fixed
//            point and summed exactly with 32-bit integer shared atomics
//            (order-independent; see the fixed-point notes below).
//     FP64:  one CTA per (tile, component), FP64 shared-memory accumulation,
//            the reference's exact weights.
//
// interp_tile  -- one CTA per (tile, component) stages the tile plus the
//   stencil halo of that component in shared memory with one TMA bulk tensor
//   copy; at a domain edge the out-of-range slabs are then patched with loads
//   that wrap periodic halos and clamp wall halos exactly as the reference
//   clamps node indices.  Every point of the tile then gathers its M^dims
//   nodes from shared memory.
//     FP64:  exact weights, sums in the reference's pattern order (bit-exact).
//     FP32C: the staged values rounded to FP32 in shared memory (half the
//            shared-memory traffic of the gathers), FP32 weights, FP32 row
//            sums of M products, FP64 sum of the rows.
#pragma once
#include <algorithm>
#include "ibk_device.cuh"
#include "ibk_bin.cuh"
#include "ibk_tma.cuh"

namespace ibk {

constexpr int kTileThreads = 256;

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

// Axis d of a packed per-axis int8 triple.
__device__ __forceinline__ int unpack8(int v, int d) { return (int) (signed char) ((unsigned) v >> (8 * d)); }

// ------------------------------------------------------------ ranges ---
// The bins a spread tile must visit.  Per axis five (neighbour offset,
// class) choices: (-1, upper), (0, lower), (0, inside), (0, upper),
// (+1, lower); the 3^dims choices with offset 0 on every axis are the tile's
// own bins, one contiguous range.  Non-empty ranges are compacted; each
// keeps the offset from this tile's first cell to its home tile's first cell
// (unwrapped across periodic boundaries) so a record's home-relative origin
// becomes a tile-local one by one addition.
constexpr int kMaxRanges = 128;

struct RangeTable {
	int start[kMaxRanges];
	int pref[kMaxRanges + 1];
	int shift[kMaxRanges];  // per axis int8: home tile's first cell - this tile's first cell
	int count;
};

// The bins' force maxima of a grid for the FP32C scale (see BinStats), or
// null.
struct BinStatsView {
	const unsigned* binmax;
};

template <int DIMS>
__device__ __forceinline__ void build_ranges(const GridGeom& g, const TileGeom& tg, const int* tc,
                                             const int* __restrict__ off, RangeTable& rt,
                                             BinStatsView bs = BinStatsView{nullptr}, unsigned* fmax = nullptr)
{
	constexpr int nent = DIMS == 3 ? 125 : 25;
	const int tid = threadIdx.x;
	int len = 0, st = 0;
	unsigned sft = 0;
	int sbin = -1;          // the bin whose statistics this thread contributes
	if (tid < nent) {
		int tile = 0, cls = 0, ts = 1, cs = 1;
		bool ok = true, home = true, first_home = true;
		int e = tid;
#pragma unroll
		for (int d = 0; d < DIMS; ++d) {
			const int k = e % 5;
			e /= 5;
			const int o = k == 0 ? -1 : (k == 4 ? 1 : 0);
			const int c = k == 0 ? 2 : (k == 4 ? 0 : k - 1);
			home = home && o == 0;
			first_home = first_home && k == 1;
			const int nt = tg.ntiles[d];
			int t = tc[d] + o;
			int lo_home = t * tg.T[d];
			if (o != 0) {
				if (nt == 1) ok = false;
				else if (g.solid[d]) ok = ok && t >= 0 && t < nt;
				else if (t < 0) { t = nt - 1; lo_home = t * tg.T[d] - tg.cells[d]; }
				else if (t >= nt) { t = 0; lo_home = tg.cells[d]; }
			}
			sft |= ((unsigned) (lo_home - tc[d] * tg.T[d]) & 0xffu) << (8 * d);
			tile += t * ts;
			ts *= nt;
			cls += c * cs;
			cs *= 3;
		}
		if (home) {
			if (first_home) {
				st = __ldg(off + tile * tg.nclass);
				len = __ldg(off + (tile + 1) * tg.nclass) - st;
			}
			sbin = tile * tg.nclass + cls;   // each home class bin once
		} else if (ok) {
			const int bin = tile * tg.nclass + cls;
			st = __ldg(off + bin);
			len = __ldg(off + bin + 1) - st;
			sbin = bin;
		}
	}
	if (fmax != nullptr) {
		// the largest |f| per component over the candidate bins (threads
		// 0..127 hold one bin each, or none)
		__shared__ unsigned part_m[4][kMaxDims];
		unsigned fm[kMaxDims] = {0u, 0u, 0u};
		if (sbin >= 0)
#pragma unroll
			for (int c = 0; c < DIMS; ++c) fm[c] = __ldg(bs.binmax + (size_t) sbin * kMaxDims + c);
		if (tid < 128)
#pragma unroll
			for (int c = 0; c < kMaxDims; ++c) {
				const unsigned m = __reduce_max_sync(0xffffffffu, fm[c]);
				if ((tid & 31) == 0) part_m[tid >> 5][c] = m;
			}
		__syncthreads();
		if (tid < kMaxDims)
			fmax[tid] = max(max(part_m[0][tid], part_m[1][tid]), max(part_m[2][tid], part_m[3][tid]));
	}
	// compaction: slot = number of non-empty entries before this one, pref =
	// exclusive sum of the lengths (the first 128 threads, 4 warps)
	__shared__ int warp_slots[4], warp_len[4];
	const int lane = tid & 31, warp = tid >> 5;
	const bool nz = len > 0;
	int incl = 0, before = 0;
	unsigned ball = 0;
	if (tid < 128) {
		ball = __ballot_sync(0xffffffffu, nz);
		before = __popc(ball & ((1u << lane) - 1u));
		incl = len;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int v = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o) incl += v;
		}
		if (lane == 31) {
			warp_slots[warp] = __popc(ball);
			warp_len[warp] = incl;
		}
	}
	__syncthreads();
	if (tid < 128) {
		int sb = 0, lb = 0;
		for (int w = 0; w < warp; ++w) { sb += warp_slots[w]; lb += warp_len[w]; }
		if (nz) {
			const int slot = sb + before;
			rt.start[slot] = st;
			rt.pref[slot] = lb + incl - len;
			rt.shift[slot] = (int) sft;
		}
		if (tid == 127) {
			const int cnt = sb + __popc(ball);
			rt.count = cnt;
			rt.pref[cnt] = lb + incl;
		}
	}
	__syncthreads();
}

// The record slot of candidate item (items number the tile's ranges back to
// back) for a thread whose items only increase: r is the range of its
// previous item (0 before the first) and moves forward past the ranges that
// end at or before item (pref[count] is past every item, so the walk stops).
__device__ __forceinline__ int range_walk(const RangeTable& rt, int& r, int item)
{
	while (rt.pref[r + 1] <= item) ++r;
	return rt.start[r] + (item - rt.pref[r]);
}

// ------------------------------------------------------------ spread ---

template <int PREC> struct SpreadAcc;
template <> struct SpreadAcc<IBK_PRECISION_FP64> { using type = double; };
template <> struct SpreadAcc<IBK_PRECISION_FP32C> { using type = int; };

// Fixed point of the FP32C spread.  Per (tile, component) a power-of-two
// scale is chosen so that every single |term| stays below 2^22, the largest
// term being max|w| * max|f| over the candidate bins (the binning's bin
// maxima, BinStats).  Each FP32 product is scaled, rounded once to an integer
// with the float magic number 1.5 * 2^23 (x + magic carries rint(x) in its
// low mantissa bits for |x| <= 2^22: an FFMA and an integer subtract, no
// conversion instruction) and added to the face's 32-bit word with one
// integer shared atomic.  A word holds the sum of up to kFoldChunk = 256
// such terms exactly (|sum| < 2^30 + 128 < 2^31).  When an occupancy bound
// shows that no face can receive more than 2 kFoldChunk terms
// (window_occupancy: the common case) every component is summed in one pass,
// the scale halved where the bound exceeds kFoldChunk; otherwise (very dense
// tiles) the components are summed one at a time and the words are folded
// into exact FP64 totals every kFoldChunk candidates.  Either way the sum is
// exact and independent of the order in which points are visited (the
// binning order is not deterministic; the result is); the only rounding is
// each product's quantisation to 2^-22 (at most 2^-21 where halved) of the
// tile's largest term.
constexpr float kMagic = 12582912.0f;           // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr int kFixSumLog2 = 30;                 // bound on sum |term| * scale
constexpr int kFixTermLog2 = 22;                // bound on one |term| * scale
// Candidates summed into a 32-bit word between folds in the folded form
// (kFoldChunk * 2^kFixTermLog2 = 2^kFixSumLog2).
constexpr int kFoldChunk = 256;

// The fixed-point increments of a0 * b and a1 * b (each rounded once), from
// one packed two-lane FP32 FMA.
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

__device__ __forceinline__ int fix_term(float a, float b)
{
	return __float_as_int(__fmaf_rn(a, b, kMagic)) - kMagicBits;
}

// Occupancy bound of a spread tile: an upper bound on the number of
// candidate points whose stencil can reach one face.  A point reaches face j
// (tile-local, along each axis) only if its half-staggered origin lies in a
// window of width W_d = M + (own-axis shift range) starting at
// j + sh - M + 1 - dhi_d.  The candidates' origins are counted on a grid of
// 2 x 2 x 2-cell blocks covering every window of the tile; a window spans at
// most ceil(W_d / 2) + 1 blocks per axis, and the largest box sum of that
// many blocks bounds the points reaching any face.  cnt: shared scratch of at
// least occupancy_words() ints (the accumulators, before they are zeroed).
// Every thread of the CTA calls it; the result is the same in every thread.
template <int M>
__host__ __device__ inline void occupancy_axis(const GridGeom& g, const TileGeom& tg, int d, int* A, int* nb, int* wb)
{
	constexpr int sh = (M - 1) >> 1;
	int dlo, dhi;
	own_shift_range(g, tg.tag_mac, d, d, &dlo, &dhi);
	const int W = M + dhi - dlo;                // window width in cells
	*A = sh - M + 1 - dhi;                      // window start for face 0
	*nb = (tg.T[d] + W - 1 + 1) >> 1;           // blocks covering every window
	*wb = (W + 1) / 2 + 1;                      // blocks one window can span
}

// Largest value of cnt[0 .. vol) over the CTA (every thread gets it).
template <int NT>
__device__ __forceinline__ int block_max(const int* cnt, int vol)
{
	__shared__ int warp_best[NT / 32];
	int best = 0;
	for (int i = threadIdx.x; i < vol; i += NT) best = max(best, cnt[i]);
	best = __reduce_max_sync(0xffffffffu, best);
	if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
	__syncthreads();
	best = 0;
#pragma unroll
	for (int w = 0; w < NT / 32; ++w) best = max(best, warp_best[w]);
	__syncthreads();
	return best;
}

// Box sums along one axis: out[i] = sum of in[i + k * stride], k < w, while
// the line index (i / stride) % n + k stays below n.
template <int NT>
__device__ __forceinline__ void box_axis(const int* in, int* out, int vol, int stride, int n, int w)
{
	for (int i = threadIdx.x; i < vol; i += NT) {
		const int pos = (i / stride) % n;
		int sum = 0;
		for (int k = 0; k < w && pos + k < n; ++k) sum += in[i + k * stride];
		out[i] = sum;
	}
	__syncthreads();
}

// cnt: shared scratch of at least 2 occupancy_words() ints.
template <int M, int DIMS, int NT>
__device__ __forceinline__ int window_occupancy(const GridGeom& g, const TileGeom& tg, const RangeTable& rt, int ncand,
                                                const PointRec* __restrict__ recs, int* cnt)
{
	int A0, A1, A2 = 0, N0, N1, N2 = 1, W0, W1, W2 = 1;
	occupancy_axis<M>(g, tg, 0, &A0, &N0, &W0);
	occupancy_axis<M>(g, tg, 1, &A1, &N1, &W1);
	if (DIMS == 3) occupancy_axis<M>(g, tg, 2, &A2, &N2, &W2);
	const int vol = N0 * N1 * N2;
	for (int i = threadIdx.x; i < vol; i += NT) cnt[i] = 0;
	__syncthreads();
	int r = 0;
	for (int it = threadIdx.x; it < ncand; it += NT) {
		const int org = __ldg(&recs[range_walk(rt, r, it)].org);
		const int sft = rt.shift[r];
		const int q0 = rec_origin(org, 0) + unpack8(sft, 0) - A0;
		const int q1 = rec_origin(org, 1) + unpack8(sft, 1) - A1;
		const int q2 = DIMS == 3 ? rec_origin(org, 2) + unpack8(sft, 2) - A2 : 0;
		const int b0 = q0 >> 1, b1 = q1 >> 1, b2 = q2 >> 1;
		if (q0 >= 0 && q1 >= 0 && q2 >= 0 && b0 < N0 && b1 < N1 && b2 < N2)
			atomicAdd(cnt + (b2 * N1 + b1) * N0 + b0, 1);
	}
	__syncthreads();
	// a window covers at most W0 W1 W2 blocks: when even the fullest block
	// times that stays within twice a fold chunk, the box sums are not needed
	const int densest = block_max<NT>(cnt, vol);
	if (densest * W0 * W1 * W2 <= 2 * kFoldChunk) return densest * W0 * W1 * W2;
	int* tmp = cnt + vol;
	box_axis<NT>(cnt, tmp, vol, 1, N0, W0);
	box_axis<NT>(tmp, cnt, vol, N0, N1, W1);
	if (DIMS == 3) {
		box_axis<NT>(cnt, tmp, vol, N0 * N1, N2, W2);
		return block_max<NT>(tmp, vol);
	}
	return block_max<NT>(cnt, vol);
}

// Ints of shared scratch window_occupancy needs for tiles tg.
template <int M>
__host__ __device__ inline size_t occupancy_words(const GridGeom& g, const TileGeom& tg)
{
	size_t v = 1;
	for (int d = 0; d < g.dims; ++d) {
		int A, nb, wb;
		occupancy_axis<M>(g, tg, d, &A, &nb, &wb);
		v *= (size_t) nb;
	}
	return 2 * v;     // the count grid and one buffer of box sums
}

__host__ __device__ inline size_t occupancy_words_rt(const GridGeom& g, const TileGeom& tg, int M)
{
	switch (M) {
	case 2: return occupancy_words<2>(g, tg);
	case 3: return occupancy_words<3>(g, tg);
	case 4: return occupancy_words<4>(g, tg);
	case 5: return occupancy_words<5>(g, tg);
	default: return occupancy_words<6>(g, tg);
	}
}

// The fixed-point scale of one component: the largest power of two with
// (largest term) * scale < 2^kFixTermLog2 and, for the one-pass form, nmax
// (largest term) * scale < 2^kFixSumLog2, the largest term being max|w| *
// max|f| (0 when the component's forces are all 0).  nmax <= kFoldChunk
// leaves the first bound the only one; up to 2 kFoldChunk costs at most one
// bit.
__device__ __forceinline__ float fix_scale(unsigned fmax_bits, float wmax, int nmax)
{
	if (fmax_bits == 0u) return 0.0f;
	const double term = (double) __uint_as_float(fmax_bits) * (double) wmax * 1.001;
	int ex_term, ex_sum;
	frexp(term, &ex_term);                       // largest term < 2^ex_term
	frexp(term * (double) max(nmax, 1), &ex_sum); // largest face sum < 2^ex_sum
	const int k = min(kFixTermLog2 - ex_term, kFixSumLog2 - ex_sum);
	return ldexpf(1.0f, max(-126, min(k, 126)));
}

// Shared-memory reduction (no return value) at a 32-bit shared address.
__device__ __forceinline__ void red_shared(unsigned addr, int v)
{
	asm volatile("red.shared.add.s32 [%0], %1;" :: "r"(addr), "r"(v) : "memory");
}

// The four reductions of one stencil row of a 4-point delta: node m0 at
// row + 4 m0 bytes, one block with immediate offsets.  Nodes outside the tile
// carry zero weight (their addresses stay inside the shared accumulators),
// so no node needs a predicate or a branch.
__device__ __forceinline__ void red_row4(unsigned row, int t0, int t1, int t2, int t3)
{
	asm volatile("red.shared.add.s32 [%0], %1;\n\tred.shared.add.s32 [%0+4], %2;\n\t"
	             "red.shared.add.s32 [%0+8], %3;\n\tred.shared.add.s32 [%0+12], %4;"
	             :: "r"(row), "r"(t0), "r"(t1), "r"(t2), "r"(t3) : "memory");
}

// The accumulators start kGuardWords after the dynamic shared memory: a
// row's out-of-tile columns (zero terms) may fall up to M - 1 words before
// the first row of the first component.
constexpr int kGuardWords = 8;

// In-tile node mask of one axis: bit m set when node (j0 + m) lies in [0, e).
template <int M>
__device__ __forceinline__ unsigned axis_mask(int j0, int e)
{
	const int mlo = max(0, -j0), mhi = min(M, e - j0);
	return mhi > mlo ? ((1u << mhi) - 1u) & ~((1u << mlo) - 1u) : 0u;
}

// One FP32C contribution set: the in-tile nodes of a point's stencil for one
// component.  l: tile-local stencil origin per axis; dl: fractional offsets;
// f: res * F * scale; e: faces of the tile per axis; acc: shared byte address
// of the component's accumulator words (row stride S1, plane stride S2);
// Rows outside the tile are predicated off: their lanes issue no shared
// access, so they add no bank traffic to the row's reductions.
template <typename D, int DIMS>
__device__ __forceinline__ void spread_fix(unsigned acc, const int* l, const float* dl, float f,
                                           const int* e, int S1, int S2)
{
	constexpr int M = D::M, sh = (M - 1) >> 1;
	unsigned mk[DIMS];
	bool any = true;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		mk[d] = axis_mask<M>(l[d] - sh, e[d]);
		any = any && mk[d] != 0u;
	}
	if (!any) return;
	float w[DIMS][M];
#pragma unroll
	for (int d = 0; d < DIMS; ++d) weights32<D>(dl[d], w[d]);
	// columns outside the tile: zero weight (in-row addresses stay inside the
	// accumulators: padding columns, a neighbouring row or the guard words)
#pragma unroll
	for (int m0 = 0; m0 < M; ++m0) w[0][m0] = (mk[0] >> m0) & 1u ? w[0][m0] * f : 0.0f;
	const int first = (l[0] - sh) + (l[1] - sh) * S1 + (DIMS == 3 ? (l[2] - sh) * S2 : 0);
	const unsigned base = acc + 4u * (unsigned) first;   // wraps for negative origins; in-tile nodes land inside
	constexpr int R = DIMS == 3 ? M * M : M;
#pragma unroll
	for (int r = 0; r < R; ++r) {
		const int m1 = r % M, m2 = r / M;
		const unsigned rm = DIMS == 3 ? (mk[1] >> m1) & (mk[2] >> m2) & 1u : (mk[1] >> m1) & 1u;
		const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
		const unsigned row = base + 4u * (unsigned) (m1 * S1 + (DIMS == 3 ? m2 * S2 : 0));
		if constexpr (M == 4) {
			const int2 a = fix_terms2(w[0][0], w[0][1], w12);
			const int2 b = fix_terms2(w[0][2], w[0][3], w12);
			if (rm) red_row4(row, a.x, a.y, b.x, b.y);
		} else {
#pragma unroll
			for (int m0 = 0; m0 + 1 < M; m0 += 2) {
				const int2 t = fix_terms2(w[0][m0], w[0][m0 + 1], w12);
				if (rm) {
					red_shared(row + 4u * m0, t.x);
					red_shared(row + 4u * (m0 + 1), t.y);
				}
			}
			if ((M & 1) && rm) red_shared(row + 4u * (M - 1), fix_term(w[0][M - 1], w12));
		}
	}
}

// Node index along axis d of a tile that spans a whole periodic axis (the
// stencil wraps inside the tile): the wrapped local index, always in range.
// Elsewhere the local index and whether it lies in [0, e).
__device__ __forceinline__ int local_node(int j, int e, int cells, bool wrap, bool& ok)
{
	if (wrap) {
		ok = true;
		return wrap_index(j, cells);
	}
	ok = j >= 0 && j < e;
	return j;
}

// The general form of spread_fix / spread_f64 for tiles with a wrapping
// axis: per-node local indices (each face of the tile may be reached from
// both sides of the period).
template <typename D, int DIMS, typename Acc, typename Term>
__device__ __forceinline__ void spread_wrapped(const int* l, const int* e, const int* cells, const bool* wrap,
                                               int S1, int S2, Acc&& add, Term&& weight_row)
{
	constexpr int M = D::M, sh = (M - 1) >> 1;
	int loc[DIMS][M];
	unsigned mk[DIMS];
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		mk[d] = 0u;
#pragma unroll
		for (int m = 0; m < M; ++m) {
			bool ok;
			loc[d][m] = local_node(l[d] - sh + m, e[d], cells[d], wrap[d], ok);
			mk[d] |= (unsigned) ok << m;
		}
	}
	constexpr int R = DIMS == 3 ? M * M : M;
#pragma unroll
	for (int r = 0; r < R; ++r) {
		const int m1 = r % M, m2 = r / M;
		const unsigned rm = DIMS == 3 ? (mk[1] >> m1) & (mk[2] >> m2) & 1u : (mk[1] >> m1) & 1u;
		if (!rm) continue;
		const int row = (DIMS == 3 ? loc[2][m2] * S2 : 0) + loc[1][m1] * S1;
#pragma unroll
		for (int m0 = 0; m0 < M; ++m0)
			if ((mk[0] >> m0) & 1u) add(row + loc[0][m0], weight_row(m0, m1, m2));
	}
}

// FP64 contribution set (the reference's arithmetic: w0 * (res F) times
// w1 * w2, exact weights), tile without wrapping axes.
template <typename D, int DIMS>
__device__ __forceinline__ void spread_f64(double* acc, const int* l, const double* dl, double f, const int* e,
                                           int S1, int S2)
{
	constexpr int M = D::M, sh = (M - 1) >> 1;
	unsigned mk[DIMS];
	bool any = true;
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		mk[d] = axis_mask<M>(l[d] - sh, e[d]);
		any = any && mk[d] != 0u;
	}
	if (!any) return;
	double w[DIMS][M];
#pragma unroll
	for (int d = 0; d < DIMS; ++d)
#pragma unroll
		for (int m = 0; m < M; ++m)
			w[d][m] = (mk[d] >> m & 1u) ? D::phi64(__dadd_rn(dl[d], (double) (m - sh))) : 0.0;
#pragma unroll
	for (int m0 = 0; m0 < M; ++m0) w[0][m0] = __dmul_rn(w[0][m0], f);
	const int first = (l[0] - sh) + (l[1] - sh) * S1 + (DIMS == 3 ? (l[2] - sh) * S2 : 0);
	constexpr int R = DIMS == 3 ? M * M : M;
#pragma unroll
	for (int r = 0; r < R; ++r) {
		const int m1 = r % M, m2 = r / M;
		const unsigned rm = DIMS == 3 ? (mk[1] >> m1) & (mk[2] >> m2) & 1u : (mk[1] >> m1) & 1u;
		if (!rm) continue;
		const double w12 = DIMS == 3 ? __dmul_rn(w[1][m1], w[2][m2]) : w[1][m1];
		double* row = acc + first + m1 * S1 + (DIMS == 3 ? m2 * S2 : 0);
#pragma unroll
		for (int m0 = 0; m0 < M; ++m0)
			if ((mk[0] >> m0) & 1u) atomicAdd(row + m0, __dmul_rn(w[0][m0], w12));
	}
}

// Writes the tile's faces of component c: out = value(li) for every face.
// Lanes run along x (8, 16 or 32 per row), the warps' row groups along y,
// planes one after the other: no division per face.
template <int DIMS, int NT, typename V>
__device__ __forceinline__ void write_tile(double* __restrict__ out, const CompGeom& cg, const int* lo, const int* e,
                                           int S1, int S2, V&& value)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int lpr = e[0] <= 8 ? 8 : (e[0] <= 16 ? 16 : 32);   // lanes per row
	const int rpw = 32 / lpr;                                 // rows per warp
	const int l0 = lane & (lpr - 1);
	const int rstep = (NT / 32) * rpw;                        // rows per CTA step
	const int planes = DIMS == 3 ? e[2] : 1;
	const size_t P0 = (size_t) cg.points[0];
	const size_t P01 = P0 * (size_t) cg.points[1];
	for (int l2 = 0; l2 < planes; ++l2) {
		const size_t pb = (size_t) lo[0] + P0 * (size_t) lo[1] + (DIMS == 3 ? P01 * (size_t) (lo[2] + l2) : 0);
		for (int l1 = warp * rpw + lane / lpr; l1 < e[1]; l1 += rstep) {
			double* o = out + pb + P0 * (size_t) l1;
			const int lb = (DIMS == 3 ? l2 * S2 : 0) + l1 * S1;
			for (int x0 = l0; x0 < e[0]; x0 += lpr) o[x0] = value(lb + x0);
		}
	}
}

// The folded FP32C form of a spread tile (tiles where a face may receive
// more terms than a 32-bit word holds): components c_lo .. c_hi - 1 one at a
// time (the folded kernel takes one component per item), kFoldChunk
// candidates per round, after each round the words added exactly into FP64
// totals (integers below 2^53) and cleared.  Every thread of the CTA calls
// it, after s_scale is set.
template <typename D, int DIMS, int NT>
__device__ __forceinline__ void spread_tile_folded(const GridGeom& g, const TileGeom& tg, int n,
                                                const double* __restrict__ fl, const PointRec* __restrict__ recs,
                                                int pbase, const RangeTable& rt, int ncand, const int* lo,
                                                const int* cells, const bool* wrap, bool wrap_any,
                                                unsigned acc_addr, const CompPtrs& fe,
                                                const float* s_scale, int c_lo, int c_hi)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const SpreadStrides ss = spread_strides(tg.T[0], tg.T[1], DIMS == 3 ? tg.T[2] : 1, DIMS);
	int* words = reinterpret_cast<int*>(smem_raw + 4 * kGuardWords);
	double* total = reinterpret_cast<double*>(words + ss.words);     // ss.words is a multiple of 4
	for (int c = c_lo; c < c_hi; ++c) {
		const CompGeom& cg = g.comp[c];
		int e[3] = {1, 1, 1};
#pragma unroll
		for (int d = 0; d < DIMS; ++d) e[d] = min(tg.T[d], cg.points[d] - lo[d]);
		for (int i = threadIdx.x; i < ss.words; i += NT) { words[i] = 0; total[i] = 0.0; }
		__syncthreads();
		const float sc = s_scale[c];
		if (sc != 0.0f) {
			int r = 0;
			for (int chunk = 0; chunk < ncand; chunk += kFoldChunk) {
				for (int it = chunk + threadIdx.x; it < min(ncand, chunk + kFoldChunk); it += NT) {
					const PointRec rec = load_rec(recs + range_walk(rt, r, it));
					const int sft = rt.shift[r];
					const int p = rec.p - pbase;
					int l[DIMS];
					float dl[DIMS];
#pragma unroll
					for (int d = 0; d < DIMS; ++d) {
						const bool own = tg.tag_mac && d == c;
						l[d] = rec_origin(rec.org, d) + unpack8(sft, d) + (own ? rec_own_shift(rec.org, d) : 0);
						dl[d] = own ? rec.dn[d] : rec.dh[d];
					}
					const float f = (float) (g.res * __ldg(fl + (size_t) c * n + p)) * sc;
					if (!wrap_any) {
						spread_fix<D, DIMS>(acc_addr, l, dl, f, e, ss.S1, ss.S2);
					} else {
						float w[DIMS][D::M];
#pragma unroll
						for (int d = 0; d < DIMS; ++d) weights32<D>(dl[d], w[d]);
						spread_wrapped<D, DIMS>(l, e, cells, wrap, ss.S1, ss.S2,
							[&](int li, int v) { red_shared(acc_addr + 4u * (unsigned) li, v); },
							[&](int m0, int m1, int m2) {
								const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
								return fix_term(w[0][m0] * f, w12);
							});
					}
				}
				__syncthreads();
				for (int i = threadIdx.x; i < ss.words; i += NT) {
					total[i] += (double) words[i];
					words[i] = 0;
				}
				__syncthreads();
			}
		}
		const double inv = sc != 0.0f ? 1.0 / (double) sc : 0.0;
		write_tile<DIMS, NT>(fe.p[c], cg, lo, e, ss.S1, ss.S2, [&](int li) { return total[li] * inv; });
		__syncthreads();
	}
}

// One spread tile; every thread of the CTA calls it.  comp < 0: every
// component (FP32C); else that component only (FP64).  Records carry point
// indices offset by pbase (a batch numbers the points of all its instances
// consecutively); off is this grid's bin table.
// Dense tiles (FP32C tiles where a face may receive more terms than a
// 32-bit word holds) are not summed by the one-pass kernel: it appends
// (defer_id << 2) | c for each component c to the deferral list and leaves
// the tile to the folded kernel, one component per item, which keeps the
// folded form out of the one-pass kernel's code.
struct Deferral {
	int* list;
	int* count;
};

template <typename D, int DIMS, int PREC, bool FOLDED = false, int NT = kTileThreads>
__device__ __forceinline__ void spread_tile(const GridGeom& g, const TileGeom& tg, int n, const double* __restrict__ x,
                                            const double* __restrict__ fl, const PointRec* __restrict__ recs, int pbase,
                                            const int* __restrict__ off, BinStatsView bs, const CompPtrs& fe,
                                            int tile, int comp, Deferral defer = Deferral{nullptr, nullptr},
                                            int defer_id = 0)
{
	using acc_t = typename SpreadAcc<PREC>::type;
	constexpr int M = D::M;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ RangeTable rt;
	__shared__ float s_scale[kMaxDims];

	const int T0 = tg.T[0], T1 = tg.T[1], T2 = DIMS == 3 ? tg.T[2] : 1;
	const SpreadStrides ss = spread_strides(T0, T1, T2, DIMS);
	const int c_lo = comp < 0 ? 0 : comp, c_hi = comp < 0 ? DIMS : comp + 1;
	acc_t* acc = reinterpret_cast<acc_t*>(smem_raw + 4 * kGuardWords);
	int tc[3] = {0, 0, 0};
	tile_coords(tg, tile, tc);
	int lo[3] = {0, 0, 0};
	bool wrap[3] = {false, false, false};
	bool wrap_any = false;
	int cells[3] = {1, 1, 1};
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		lo[d] = tc[d] * tg.T[d];
		cells[d] = tg.cells[d];
		wrap[d] = !g.solid[d] && tg.ntiles[d] == 1;
		wrap_any = wrap_any || wrap[d];
	}
	__shared__ unsigned s_fmax[kMaxDims];
	if constexpr (PREC == IBK_PRECISION_FP32C) build_ranges<DIMS>(g, tg, tc, off, rt, bs, s_fmax);
	else build_ranges<DIMS>(g, tg, tc, off, rt);
	const int ncand = rt.pref[rt.count];
	if (ncand == 0) {
		// no point reaches the tile: its faces are zero
		for (int c = c_lo; c < c_hi; ++c) {
			int e[3] = {1, 1, 1};
#pragma unroll
			for (int d = 0; d < DIMS; ++d) e[d] = min(tg.T[d], g.comp[c].points[d] - lo[d]);
			write_tile<DIMS, NT>(fe.p[c], g.comp[c], lo, e, ss.S1, ss.S2, [](int) { return 0.0; });
		}
		return;
	}
	const unsigned acc_addr = smem_addr(acc);
	if constexpr (PREC == IBK_PRECISION_FP32C && FOLDED) {
		if (threadIdx.x < kMaxDims) s_scale[threadIdx.x] = fix_scale(s_fmax[threadIdx.x], max_weight<D, DIMS>(), kFoldChunk);
		spread_tile_folded<D, DIMS, NT>(g, tg, n, fl, recs, pbase, rt, ncand, lo, cells, wrap, wrap_any, acc_addr,
		                                fe, s_scale, c_lo, c_hi);
		return;
	}
	if constexpr (PREC == IBK_PRECISION_FP32C && !FOLDED) {
		// one pass unless a face may receive more than 2 kFoldChunk terms (the
		// occupancy bound uses the accumulator memory before it is zeroed; a
		// tile that wraps a periodic axis counts every candidate)
		const int nmax = (ncand <= kFoldChunk || wrap_any)
			? ncand : window_occupancy<M, DIMS, NT>(g, tg, rt, ncand, recs, reinterpret_cast<int*>(acc));
		if (nmax > 2 * kFoldChunk) {
			// one deferred item per component: (defer_id << 2) | component
			if (threadIdx.x < DIMS) defer.list[atomicAdd(defer.count, 1)] = (defer_id << 2) | (int) threadIdx.x;
			return;
		}
		if (threadIdx.x < kMaxDims) s_scale[threadIdx.x] = fix_scale(s_fmax[threadIdx.x], max_weight<D, DIMS>(), nmax);
	}
	const int nwords = ss.words * (c_hi - c_lo);
	for (int i = threadIdx.x * 4; i < nwords; i += NT * 4) {
		if constexpr (PREC == IBK_PRECISION_FP32C) *reinterpret_cast<int4*>(acc + i) = make_int4(0, 0, 0, 0);
		else {
			*reinterpret_cast<double2*>(acc + i) = make_double2(0.0, 0.0);
			*reinterpret_cast<double2*>(acc + i + 2) = make_double2(0.0, 0.0);
		}
	}
	__syncthreads();

	int r = 0;
	for (int it = threadIdx.x; it < ncand; it += NT) {
		const int slot = range_walk(rt, r, it);
		const PointRec rec = load_rec(recs + slot);
		const int sft = rt.shift[r];
		const int p = rec.p - pbase;
		int lh[DIMS];
#pragma unroll
		for (int d = 0; d < DIMS; ++d) lh[d] = rec_origin(rec.org, d) + unpack8(sft, d);
#pragma unroll 1
		for (int c = c_lo; c < c_hi; ++c) {
			const CompGeom& cg = g.comp[c];
			int l[DIMS], e[DIMS];
#pragma unroll
			for (int d = 0; d < DIMS; ++d) {
				const bool own = tg.tag_mac && d == c;
				l[d] = lh[d] + (own ? rec_own_shift(rec.org, d) : 0);
				e[d] = min(tg.T[d], cg.points[d] - lo[d]);
			}
			if constexpr (PREC == IBK_PRECISION_FP32C) {
				const float sc = s_scale[c];
				if (sc == 0.0f) continue;
				const float f = (float) (g.res * __ldg(fl + (size_t) c * n + p)) * sc;
				float dl[DIMS];
#pragma unroll
				for (int d = 0; d < DIMS; ++d) dl[d] = (tg.tag_mac && d == c) ? rec.dn[d] : rec.dh[d];
				const unsigned a = acc_addr + 4u * (unsigned) (ss.words * (c - c_lo));
				if (!wrap_any) {
					spread_fix<D, DIMS>(a, l, dl, f, e, ss.S1, ss.S2);
				} else {
					float w[DIMS][M];
#pragma unroll
					for (int d = 0; d < DIMS; ++d) weights32<D>(dl[d], w[d]);
					spread_wrapped<D, DIMS>(l, e, cells, wrap, ss.S1, ss.S2,
						[&](int li, int v) { red_shared(a + 4u * (unsigned) li, v); },
						[&](int m0, int m1, int m2) {
							const float w12 = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
							return fix_term(w[0][m0] * f, w12);
						});
				}
			} else {
				const double f = __dmul_rn(g.res, __ldg(fl + (size_t) c * n + p));
				double dl[DIMS];
#pragma unroll
				for (int d = 0; d < DIMS; ++d) dl[d] = axis_step<M>(g, cg, d, __ldg(x + (size_t) d * n + p)).delta;
				double* a = reinterpret_cast<double*>(acc) + (size_t) ss.words * (c - c_lo);
				if (!wrap_any) {
					spread_f64<D, DIMS>(a, l, dl, f, e, ss.S1, ss.S2);
				} else {
					constexpr int sh = (M - 1) >> 1;
					double w[DIMS][M];
#pragma unroll
					for (int d = 0; d < DIMS; ++d)
#pragma unroll
						for (int m = 0; m < M; ++m) w[d][m] = D::phi64(__dadd_rn(dl[d], (double) (m - sh)));
					spread_wrapped<D, DIMS>(l, e, cells, wrap, ss.S1, ss.S2,
						[&](int li, double v) { atomicAdd(a + li, v); },
						[&](int m0, int m1, int m2) {
							const double w12 = DIMS == 3 ? __dmul_rn(w[1][m1], w[2][m2]) : w[1][m1];
							return __dmul_rn(__dmul_rn(w[0][m0], f), w12);
						});
				}
			}
		}
	}
	__syncthreads();

	// every face of the tile, written once
	for (int c = c_lo; c < c_hi; ++c) {
		int e[3] = {1, 1, 1};
#pragma unroll
		for (int d = 0; d < DIMS; ++d) e[d] = min(tg.T[d], g.comp[c].points[d] - lo[d]);
		const acc_t* ac = acc + (size_t) ss.words * (c - c_lo);
		if constexpr (PREC == IBK_PRECISION_FP64) {
			write_tile<DIMS, NT>(fe.p[c], g.comp[c], lo, e, ss.S1, ss.S2, [&](int li) { return ac[li]; });
		} else {
			const float sc = s_scale[c];
			const double inv = sc != 0.0f ? 1.0 / (double) sc : 0.0;
			write_tile<DIMS, NT>(fe.p[c], g.comp[c], lo, e, ss.S1, ss.S2,
			                     [&](int li) { return (double) ac[li] * inv; });
		}
	}
}

// Shared memory of a spread CTA: the accumulator words of the components it
// covers (FP32C: every component, 4 bytes per face, or the occupancy grid if
// larger; FP64: one component, 8 bytes per face), after the guard words.
__host__ __device__ inline size_t spread_smem_bytes(const GridGeom& g, const TileGeom& tg, int M, int precision)
{
	const int dims = g.dims;
	const size_t words = (size_t) spread_strides(tg.T[0], tg.T[1], tg.T[2], dims).words;
	if (precision != IBK_PRECISION_FP32C) return words * 8 + 4 * kGuardWords;
	// the region (accumulators, folded words and totals, or the occupancy
	// grid) and the guard words
	const size_t occ = occupancy_words_rt(g, tg, M), acc = words * 3;
	return ((acc > occ ? acc : occ) + kGuardWords) * 4;
}

// FP32C: 256-thread CTAs capped at 64 registers so that four fit on an SM
// (their accumulators take 54 KB each at 16^3 tiles); FP64 ones at 85 so
// that three fit.
template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads, PREC == IBK_PRECISION_FP32C ? 4 : 3)
spread_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const double* __restrict__ fl, const PointRec* __restrict__ recs,
                   const int* __restrict__ off, BinStatsView bs, CompPtrs fe, Deferral defer)
{
	// grid: tiles (FP32C) or (tile, component) (FP64)
	spread_tile<D, DIMS, PREC>(g, tg, n, x, fl, recs, 0, off, bs, fe, blockIdx.x,
	                           PREC == IBK_PRECISION_FP32C ? -1 : (int) blockIdx.y, defer, blockIdx.x);
}

// The deferred dense tiles of an FP32C spread, folded (see Deferral); the
// grid strides over the list, whose length the one-pass kernel left on the
// device.
template <typename D, int DIMS>
__global__ void __launch_bounds__(kTileThreads, 4)
spread_dense_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                    const double* __restrict__ fl, const PointRec* __restrict__ recs,
                    const int* __restrict__ off, BinStatsView bs, CompPtrs fe, const int* __restrict__ list,
                    const int* __restrict__ count)
{
	const int m = *count;
	for (int k = blockIdx.x; k < m; k += gridDim.x) {
		const int v = __ldg(list + k);
		spread_tile<D, DIMS, IBK_PRECISION_FP32C, true>(g, tg, n, x, fl, recs, 0, off, bs, fe, v >> 2, v & 3);
		__syncthreads();
	}
}

// ------------------------------------------------------------ interp ---

// Staged region of component c along one axis, relative to the tile's first
// cell: every node of every point of the tile lies in [lower, lower + extent)
// (own-axis origin shifts in [dlo, dhi]).  The x range starts on an even
// cell and has an even extent so a TMA box row is a multiple of 16 bytes.
template <int M>
__host__ __device__ inline void region_axis(int T, int dlo, int dhi, bool x_axis, int* lower, int* extent)
{
	constexpr int sh = (M - 1) >> 1;
	int lw = dlo - sh;
	const int up = T - 1 + dhi - sh + M - 1;
	if (x_axis) lw &= ~1;
	int ext = up - lw + 1;
	if (x_axis) ext = (ext + 1) & ~1;
	*lower = lw;
	*extent = ext;
}

template <int M>
__host__ __device__ inline void region_of(const GridGeom& g, const TileGeom& tg, int c, int* lower, int* extent)
{
	// axes at compile-time indices (the arrays stay in registers)
#pragma unroll
	for (int d = 0; d < kMaxDims; ++d) {
		lower[d] = 0;
		extent[d] = 1;
		if (d < g.dims) {
			int dlo, dhi;
			own_shift_range(g, tg.tag_mac, c, d, &dlo, &dhi);
			region_axis<M>(tg.T[d], dlo, dhi, d == 0, &lower[d], &extent[d]);
		}
	}
}

// Largest staged region of any component, in bytes, plus 128 bytes of slack
// for aligning the TMA destination by hand.
template <int M>
inline size_t interp_smem_bytes(const GridGeom& g, const TileGeom& tg)
{
	size_t best = 0;
	for (int c = 0; c < g.dims; ++c) {
		int lw[3], ex[3];
		region_of<M>(g, tg, c, lw, ex);
		best = std::max(best, (size_t) ex[0] * ex[1] * ex[2]);
	}
	return sizeof(double) * best + 128;
}

// Fold a region coordinate onto the grid: wrap periodic axes, clamp walls.
__device__ __forceinline__ int fold(const GridGeom& g, const CompGeom& cg, int d, int v)
{
	const int pd = cg.points[d];
	if (g.solid[d]) return v < 0 ? 0 : (v >= pd ? pd - 1 : v);
	if (v < 0 || v >= pd) v = wrap_index(v, cg.cells[d]);
	return v;
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

// Global gather of one point whose stencil leaves the staged region (points
// beyond a wall, whose clamped origin lies outside the tile's halo): node
// indices wrapped (periodic) or clamped (walls) as the reference clamps them
// (include/ib/interpolate.h:16-22), weights from the fractional offsets
// (the exact FP64 ones in the FP64 form), summed in the reference's pattern
// order.  b: stencil origin per axis in the component's index space
// (unwrapped); solid: bit d set for a wall axis.  Out of line: it is rare
// and its registers would otherwise weigh on the staged path.
template <typename D, int DIMS>
__device__ __noinline__ double interp_global(const double* __restrict__ u, int b0, int b1, int b2, double d0,
                                             double d1, double d2, int p0, int p1, int p2, int c0, int c1, int c2,
                                             int solid)
{
	using P = Pattern<D::M, DIMS, D::every_other>;
	constexpr int M = D::M, sh = (M - 1) >> 1;
	const int b[3] = {b0, b1, b2}, pts[3] = {p0, p1, p2}, cells[3] = {c0, c1, c2};
	const double dl[3] = {d0, d1, d2};
	int gidx[DIMS][M];
	double w[DIMS][M];
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
#pragma unroll
		for (int m = 0; m < M; ++m) {
			int j = b[d] + m - sh;
			if (!((solid >> d) & 1)) j = wrap_index(j, cells[d]);
			gidx[d][m] = j < 0 ? 0 : (j >= pts[d] ? pts[d] - 1 : j);
			w[d][m] = D::phi64(__dadd_rn(dl[d], (double) (m - sh)));
		}
	}
	double v = 0.0;
#pragma unroll
	for (int e = 0; e < P::V; ++e) {
		const int m0 = P::m(e, 0), m1 = P::m(e, 1);
		double wt;
		long long k;
		if constexpr (DIMS == 3) {
			const int m2 = P::m(e, 2);
			wt = __dmul_rn(w[0][m0], __dmul_rn(w[1][m1], w[2][m2]));
			k = gidx[0][m0] + (long long) p0 * (gidx[1][m1] + (long long) p1 * gidx[2][m2]);
		} else {
			wt = __dmul_rn(w[0][m0], w[1][m1]);
			k = gidx[0][m0] + (long long) p0 * gidx[1][m1];
		}
		v = __dadd_rn(v, __dmul_rn(wt, __ldg(u + k)));
	}
	return v;
}

// One (tile, component) of the interpolation; every thread of the CTA calls
// it.  maps/use_tma select TMA staging (maps_global: the maps live in global
// memory, written by a copy before the launch); epi, when not null, adds the
// serving-step epilogue; ul may then be null.  Returns false only when a
// bounded wait for the staging copy gave up (the status word records it and
// the CTA must stop).
template <typename D, int DIMS, int PREC>
__device__ __forceinline__ bool interp_tile(const GridGeom& g, const TileGeom& tg, int n, const double* __restrict__ x,
                                            const PointRec* __restrict__ recs, int pbase, const int* __restrict__ off,
                                            const ConstCompPtrs& ue, double* __restrict__ ul,
                                            const CUtensorMap* maps, int use_tma, bool maps_global, int* status,
                                            const StepEpilogue* epi, int t, int c)
{
	using P = Pattern<D::M, DIMS, D::every_other>;
	constexpr int M = D::M, sh = (M - 1) >> 1;
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
	int lower[3], E[3], rlo[3] = {0, 0, 0};
	region_of<M>(g, tg, c, lower, E);
	bool tma = use_tma != 0;        // stage with one bulk tensor copy
	bool interior = true;           // the region lies inside the grid
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		rlo[d] = tc[d] * tg.T[d] + lower[d];
		interior = interior && rlo[d] >= 0 && rlo[d] + E[d] <= cg.points[d];
	}
	// self-check of the TMA preconditions: 128-byte destination, x origin
	// on a 16-byte boundary; a violation is recorded and the region staged
	// by plain loads instead
	if (tma && (((smem_addr(reg) & 127u) != 0u) || (rlo[0] & 1) != 0)) {
		if (threadIdx.x == 0 && status) atomicExch(status, 2);
		tma = false;
	}
	// first record of this thread, fetched while the region is staged
	int it = start + threadIdx.x;
	PointRec rec_next{};
	if (it < end) rec_next = load_rec(recs + it);
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
			// out-of-range slabs: wrap periodic, clamp solid (interpolate.h:16-22);
			// the axis loop is unrolled so that the extents stay in registers
#pragma unroll
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
		const PointRec rec = rec_next;
		if (it + kTileThreads < end) rec_next = load_rec(recs + it + kTileThreads);   // prefetch the next point
		const int p = rec.p - pbase;
		int loc[DIMS];          // region index of the stencil's first node
		bool inside = true;
#pragma unroll
		for (int d = 0; d < DIMS; ++d) {
			const bool own = tg.tag_mac && d == c;
			const int l = rec_origin(rec.org, d) + (own ? rec_own_shift(rec.org, d) : 0);
			loc[d] = l - sh - lower[d];
			inside = inside && loc[d] >= 0 && loc[d] + M <= E[d];
		}
		double v;
		double zc = 0.0;
		if (PREC == IBK_PRECISION_FP64 || epi != nullptr) zc = __ldg(x + (size_t) c * n + p);
		// FP64: the exact fractional offsets of this component
		double dl64[DIMS];
		if constexpr (PREC == IBK_PRECISION_FP64) {
#pragma unroll
			for (int d = 0; d < DIMS; ++d)
				dl64[d] = axis_step<M>(g, cg, d, d == c ? zc : __ldg(x + (size_t) d * n + p)).delta;
		}
		if (inside) {
			const int base = DIMS == 3 ? (loc[2] * E[1] + loc[1]) * E[0] + loc[0] : loc[1] * E[0] + loc[0];
			if constexpr (PREC == IBK_PRECISION_FP64) {
				double w[DIMS][M];
#pragma unroll
				for (int d = 0; d < DIMS; ++d)
#pragma unroll
					for (int m = 0; m < M; ++m) w[d][m] = D::phi64(__dadd_rn(dl64[d], (double) (m - sh)));
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
				for (int d = 0; d < DIMS; ++d)
					weights32<D>((tg.tag_mac && d == c) ? rec.dn[d] : rec.dh[d], w32[d]);
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
			// stencil leaves the staged region: global gather
			int b[3] = {0, 0, 0}, sol = 0;
			double dd[3] = {0.0, 0.0, 0.0};
#pragma unroll
			for (int d = 0; d < DIMS; ++d) {
				b[d] = loc[d] + sh + lower[d] + tc[d] * tg.T[d];
				sol |= g.solid[d] << d;
				if constexpr (PREC == IBK_PRECISION_FP64) dd[d] = dl64[d];
				else dd[d] = (double) ((tg.tag_mac && d == c) ? rec.dn[d] : rec.dh[d]);
			}
			v = interp_global<D, DIMS>(u, b[0], b[1], b[2], dd[0], dd[1], dd[2], cg.points[0], cg.points[1],
			                           cg.points[2], cg.cells[0], cg.cells[1], cg.cells[2], sol);
		}
		const size_t i = (size_t) c * n + p;
		if (ul != nullptr) ul[i] = v;
		if (epi != nullptr) {
			const double xn = __dadd_rn(zc, __dmul_rn(epi->dt, v));
			epi->xn[i] = xn;
			epi->fl[i] = __dmul_rn(-epi->k, __dsub_rn(xn, __ldg(epi->xref + i)));
		}
	}
	return true;
}

template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads, D::M <= 4 ? 3 : 1)
interp_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const PointRec* __restrict__ recs, const int* __restrict__ off,
                   ConstCompPtrs ue, double* __restrict__ ul,
                   const __grid_constant__ TmaMaps maps, int use_tma, int* status)
{
	// grid: (tile, component)
	interp_tile<D, DIMS, PREC>(g, tg, n, x, recs, 0, off, ue, ul, maps.map, use_tma, false, status, nullptr,
	                           blockIdx.x, blockIdx.y);
}

} // namespace ibk
