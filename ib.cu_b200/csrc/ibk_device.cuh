// Device-side building blocks shared by every kernel of the IB coupling
// library: the reference's exact FP64 index step, its delta functions, its
// stencil orderings, and the per-component grid description.
//
// Exactness: the reference evaluates its index math as separate IEEE
// operations (no fused multiply-add on the host).  Every operation in this
// file that feeds a sort key, a stencil origin or an FP64 weight uses the
// explicitly rounded intrinsics (__dadd_rn, __dmul_rn, ...), which the
// compiler never contracts, so keys, origins and FP64 weights are bit-identical
// to the reference's host evaluation.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ibk {

constexpr int kMaxDims = 3;

// One MAC (or cell-centred) component grid: fd::discretization per dimension
// (include/fd/discretization.h:113-164).
struct CompGeom {
	int points[kMaxDims];      // grid points along d (fd::discretization::points)
	int cells[kMaxDims];       // cells along d (periodic wrap modulus)
	double shift[kMaxDims];    // discretization::shift()
	double s_over_r[kMaxDims]; // shift / resolution, one IEEE division on the host
	long long size;            // product of points
};

struct GridGeom {
	int dims;
	int solid[kMaxDims];
	double length[kMaxDims];
	double length_safe[kMaxDims]; // length * (1 - 2^-52): below it, t / length < 1
	double r;                  // resolution = refinement / domain unit
	double res;                // product of resolutions (1/h^dims), novel.h:101-103
	CompGeom comp[kMaxDims];
};

// Tile decomposition of the cell grid (shared by every component).
struct TileGeom {
	int T[kMaxDims];        // tile extent in cells
	int ntiles[kMaxDims];
	int cells[kMaxDims];
	int num_tiles;
	int nclass;             // 3^dims
	int num_bins;           // num_tiles * nclass
	int tag_mac;            // fd::mac (1) or fd::centered (0)
};

// Accumulator layout of a spread tile in shared memory: face (l0, l1, l2) at
// l2 * S2 + l1 * S1 + l0.  Rows are padded by one word and planes so that
// S2 = 24 (mod 32): the lanes of a warp, whose points lie close together,
// then spread their atomics over more banks (about 2.7 instead of 4
// wavefronts per instruction for 16^3 tiles on surface-sampled points).
struct SpreadStrides {
	int S1, S2, words;
};
__host__ __device__ inline SpreadStrides spread_strides(int T0, int T1, int T2, int dims)
{
	SpreadStrides st;
	st.S1 = T0 + 1;
	st.S2 = st.S1 * T1;
	st.S2 += (24 - st.S2 % 32 + 32) % 32;
	st.words = dims == 3 ? st.S2 * T2 : st.S1 * T1;
	st.words = (st.words + 3) & ~3;    // 16-byte multiples (vector zeroing)
	return st;
}

__host__ __device__ inline int ipow3(int d) { return d == 1 ? 3 : d == 2 ? 9 : 27; }

struct CompPtrs { double* p[kMaxDims]; };
struct ConstCompPtrs { const double* p[kMaxDims]; };

// ---------------------------------------------------------------- math ---

// util::math::floor (include/util/math.h:158-162):
//   (long) (x - (x < 0 && (-x != (long) -x)))
__device__ __forceinline__ double ref_floor(double x) {
	double nx = -x;
	double tn = __ll2double_rn(__double2ll_rz(nx));
	double adj = (x < 0.0 && nx != tn) ? 1.0 : 0.0;
	return __ll2double_rn(__double2ll_rz(__dsub_rn(x, adj)));
}

// util::math::modulo (include/util/math.h:164-168): x - s * floor(x / s)
__device__ __forceinline__ double ref_modulo(double x, double s) {
	return __dsub_rn(x, __dmul_rn(s, ref_floor(__ddiv_rn(x, s))));
}

// ------------------------------------------------------------ deltas ---
// Each delta: meshwidths M, stencil ordering, phi in FP64 (bit-exact with the
// reference) and a single-precision evaluation for the FP32C form.

enum DeltaKind { kBspline = 0, kPeskin = 1, kRoma = 2, kCosine = 3, kHat = 4 };

// bspline<n> (include/ib/bspline.h:13-27):
//   b = (n+1)/(2n); a = r/n; (b+a) f(r+1/2) + (b-a) f(r-1/2), f = bspline<n-1>
template <int n> struct BsplineFn {
	static __device__ __forceinline__ double eval64(double r) {
		constexpr double b = (n + 1.0) / (2.0 * n);
		double a;
		if constexpr (n == 1) a = r;                          // r / 1
		else if constexpr (n == 2) a = __dmul_rn(r, 0.5);      // r / 2, exact
		else if constexpr (n == 4) a = __dmul_rn(r, 0.25);     // r / 4, exact
		else a = __ddiv_rn(r, (double) n);
		double lo = BsplineFn<n - 1>::eval64(__dadd_rn(r, 0.5));
		double hi = BsplineFn<n - 1>::eval64(__dsub_rn(r, 0.5));
		return __dadd_rn(__dmul_rn(__dadd_rn(b, a), lo), __dmul_rn(__dsub_rn(b, a), hi));
	}
	static __device__ __forceinline__ float eval32(float r) {
		constexpr float b = (float) ((n + 1.0) / (2.0 * n));
		float a = r * (float) (1.0 / n);
		return (b + a) * BsplineFn<n - 1>::eval32(r + 0.5f) + (b - a) * BsplineFn<n - 1>::eval32(r - 0.5f);
	}
};
template <> struct BsplineFn<0> {
	static __device__ __forceinline__ double eval64(double r) { return (-0.5 <= r && r < 0.5) ? 1.0 : 0.0; }
	static __device__ __forceinline__ float eval32(float r) { return (-0.5f <= r && r < 0.5f) ? 1.0f : 0.0f; }
};

template <int KIND, int ORDER> struct Delta;

template <int ORDER> struct Delta<kBspline, ORDER> {
	static constexpr int M = ORDER + 1;
	static constexpr bool every_other = false;
	static __device__ __forceinline__ double phi64(double r) { return BsplineFn<ORDER>::eval64(r); }
	static __device__ __forceinline__ float phi32(float r) { return BsplineFn<ORDER>::eval32(r); }
};

// peskin (include/ib/peskin.h:6-14)
template <int ORDER> struct Delta<kPeskin, ORDER> {
	static constexpr int M = 4;
	static constexpr bool every_other = true;
	static __device__ __forceinline__ double phi64(double r) {
		double s = fabs(r);
		double s4 = __dmul_rn(4.0, s);
		if (s < 1.0) {
			double q = __dsub_rn(__dadd_rn(1.0, s4), __dmul_rn(s4, s));
			return __dmul_rn(__dadd_rn(__dsub_rn(3.0, __dmul_rn(2.0, s)), __dsqrt_rn(q)), 0.125);
		}
		double q = __dsub_rn(__dadd_rn(-7.0, __dmul_rn(12.0, s)), __dmul_rn(s4, s));
		return __dmul_rn(__dsub_rn(__dsub_rn(5.0, __dmul_rn(2.0, s)), __dsqrt_rn(q)), 0.125);
	}
	static __device__ __forceinline__ float phi32(float r) {
		float s = fabsf(r);
		if (s < 1.0f) return (3.0f - 2.0f * s + sqrtf(1.0f + 4.0f * s - 4.0f * s * s)) * 0.125f;
		return (5.0f - 2.0f * s - sqrtf(fmaxf(-7.0f + 12.0f * s - 4.0f * s * s, 0.0f))) * 0.125f;
	}
};

// roma (include/ib/roma.h:9-18)
template <int ORDER> struct Delta<kRoma, ORDER> {
	static constexpr int M = 3;
	static constexpr bool every_other = false;
	static __device__ __forceinline__ double phi64(double r) {
		double s = fabs(r);
		if (s >= 1.5) return 0.0;
		if (s < 0.5) {
			double q = __dsub_rn(1.0, __dmul_rn(__dmul_rn(3.0, s), s));
			return __ddiv_rn(__dadd_rn(1.0, __dsqrt_rn(q)), 3.0);
		}
		double t = __dsub_rn(1.0, s);
		double q = __dsub_rn(1.0, __dmul_rn(__dmul_rn(3.0, t), t));
		return __ddiv_rn(__dsub_rn(__dsub_rn(5.0, __dmul_rn(3.0, s)), __dsqrt_rn(q)), 6.0);
	}
	static __device__ __forceinline__ float phi32(float r) {
		float s = fabsf(r);
		if (s >= 1.5f) return 0.0f;
		if (s < 0.5f) return (1.0f + sqrtf(1.0f - 3.0f * s * s)) * (1.0f / 3.0f);
		float t = 1.0f - s;
		return (5.0f - 3.0f * s - sqrtf(fmaxf(1.0f - 3.0f * t * t, 0.0f))) * (1.0f / 6.0f);
	}
};

// cosine (include/ib/cosine.h:9-16).  cos() is CUDA's, so FP64 cosine
// weights agree with the host's libm to within its last-place error only.
template <int ORDER> struct Delta<kCosine, ORDER> {
	static constexpr int M = 4;
	static constexpr bool every_other = true;
	static __device__ __forceinline__ double phi64(double r) {
		const double pi_halves = 1.57079632679489661923;
		return __dmul_rn(0.25, __dadd_rn(1.0, cos(__dmul_rn(pi_halves, r))));
	}
	static __device__ __forceinline__ float phi32(float r) {
		return 0.25f * (1.0f + cospif(0.5f * r));
	}
};

// hat (include/ib/hat.h:9-16)
template <int ORDER> struct Delta<kHat, ORDER> {
	static constexpr int M = 2;
	static constexpr bool every_other = false;
	static __device__ __forceinline__ double phi64(double r) { return __dsub_rn(1.0, fabs(r)); }
	static __device__ __forceinline__ float phi32(float r) { return 1.0f - fabsf(r); }
};

// ---------------------------------------------------------- patterns ---
// standard_pattern / every_other_pattern (include/ib/delta.h:97-147): entry
// e of the stencil -> offset index m (0..M-1) along dimension j, where the
// grid offset is m - (M-1)/2.

__host__ __device__ constexpr int ipow_c(int b, int e) { return e == 0 ? 1 : b * ipow_c(b, e - 1); }

template <int M, int DIMS, bool EO>
struct Pattern {
	static constexpr int V = ipow_c(M, DIMS);
	static constexpr int shift = (M - 1) >> 1;
	// offset index (0..M-1) of entry e along dimension j
	__host__ __device__ static constexpr int m(int e, int j) {
		if constexpr (!EO) {
			int n = e;
			for (int k = 0; k < j; ++k) n /= M;
			return n % M;
		} else {
			constexpr int half = (M + 1) >> 1;
			constexpr int mod = ipow_c(half, DIMS);
			int x = e / mod, y = e % mod;
			for (int k = 0; k < j; ++k) { x /= 2; y /= half; }
			return x % 2 + 2 * (y % half);   // = s + shift
		}
	}
};

// ------------------------------------------------------ index step ---

// (i + cells) % cells, C remainder semantics (discretization.h:155), without
// an integer division for the indices that occur here (i in [-cells, 2 cells)).
__device__ __forceinline__ int wrap_index(int i, int cells) {
	if (i >= -cells && i < 2 * cells) {
		const int j = i + cells;
		return j >= 2 * cells ? j - 2 * cells : (j >= cells ? j - cells : j);
	}
	return (i + cells) % cells;
}

// Per point, per component: the reference's stencil origin ("base", from the
// clamped sort key, include/ib/indexing.h:10-33,239-250) and fractional offset
// (sweep::difference, include/ib/sweep.h:49-62), bit-exact.
template <int M>
struct AxisStep {
	int key;      // clamped sort-key digit along this axis, in [0, points+solid)
	int base;     // decompose(key) along this axis = key - solid
	double delta; // floor(u + rounding) - u
};

template <int M>
__device__ __forceinline__ AxisStep<M> axis_step(const GridGeom& g, const CompGeom& cg, int d, double x) {
	const double s = cg.shift[d];
	double t = __dsub_rn(x, cg.s_over_r[d]);                 // x - s / r
	// dimension::clamp.  For 0 <= t <= length*(1 - 2^-52) the quotient t/L
	// rounds below 1, floor gives 0 and modulo returns t itself: skip the
	// division there (same value, bit for bit).
	if (!g.solid[d] && !(t >= 0.0 && t <= g.length_safe[d])) t = ref_modulo(t, g.length[d]);
	double u = __dadd_rn(__dmul_rn(t, g.r), s);               // * r + s
	double diff = __dsub_rn(u, s);                             // units(x) - shift
	constexpr double rounding = 0.5 * (M & 1);
	int i = __double2int_rz(ref_floor(__dadd_rn(diff, rounding)));   // sweep::clamp
	AxisStep<M> a;
	a.delta = __dsub_rn((double) i, diff);
	int j = i;
	if (!g.solid[d]) j = wrap_index(i, cg.cells[d]);         // discretization::index
	const int solid = g.solid[d];
	const int w = cg.points[d] + solid;
	int k = j + solid;
	k = k < 0 ? 0 : (k >= w ? w - 1 : k);                    // clamped{j, -solid, points}
	a.key = k;
	a.base = k - solid;
	return a;
}

// discretization::index for a stencil node (include/fd/discretization.h:151-156)
__device__ __forceinline__ int node_index(const GridGeom& g, const CompGeom& cg, int d, int i) {
	if (g.solid[d]) return i;
	return wrap_index(i, cg.cells[d]);
}

} // namespace ibk
