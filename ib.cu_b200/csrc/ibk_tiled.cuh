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
//     FP32C: FP32 weights and products accumulated EXACTLY in 32-bit fixed
//            point with integer shared atomics.  The tile's scale is the
//            largest power of two for which a sure bound on every face sum
//            (sum over candidate points of max|w| * res * |F|) fits in 2^30,
//            so the sum is error-free and order-independent; the only
//            rounding is each product's quantisation.
//
// interp_tile_kernel  -- the CTA stages, per component, the tile plus its
//   stencil halo in shared memory (periodic halos wrapped, wall halos clamped
//   exactly as the reference clamps node indices), then every point of the
//   tile gathers its M^dims nodes from shared memory.
//     FP64:  FP64 staging, sums in the reference's pattern order (bit-exact).
//     FP32C: FP32 staging, FP32 weights, x-rows summed with FMA, the rows
//            combined with TwoProd/TwoSum compensation, FP64 result.
#pragma once
#include "ibk_device.cuh"
#include "ibk_bin.cuh"

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
};

template <int DIMS>
__device__ __forceinline__ void build_ranges(const GridGeom& g, const TileGeom& tg, const int* tc,
                                             const int* __restrict__ off, RangeTable& rt, bool neighbours)
{
	const int nent = neighbours ? (DIMS == 3 ? 125 : 25) : 1;
	const int tid = threadIdx.x;
	int len = 0, st = 0;
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
		}
		rt.start[tid] = st;
	}
	// block-wide exclusive scan of len over the first 128 threads
	__shared__ int warp_tot[4];
	const int lane = tid & 31, warp = tid >> 5;
	int incl = (tid < 128) ? len : 0;
	if (tid < 128) {
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int v = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o) incl += v;
		}
		if (lane == 31) warp_tot[warp] = incl;
	}
	__syncthreads();
	if (tid < 128) {
		int base = 0;
		for (int w = 0; w < warp; ++w) base += warp_tot[w];
		if (tid < nent) rt.pref[tid] = base + incl - len;
		if (tid == nent - 1) {
			rt.pref[nent] = base + incl;
			rt.count = nent;
		}
	}
	__syncthreads();
}

__device__ __forceinline__ int range_lookup(const RangeTable& rt, int item)
{
	int lo = 0, hi = rt.count - 1;
	while (lo < hi) {                   // largest r with pref[r] <= item
		int mid = (lo + hi + 1) >> 1;
		if (rt.pref[mid] <= item) lo = mid;
		else hi = mid - 1;
	}
	return rt.start[lo] + (item - rt.pref[lo]);
}

// ------------------------------------------------------------ spread ---

template <typename D, int DIMS, int PREC>
struct SpreadSmem;
template <typename D, int DIMS>
struct SpreadSmem<D, DIMS, IBK_PRECISION_FP64> { using acc_t = double; };
template <typename D, int DIMS>
struct SpreadSmem<D, DIMS, IBK_PRECISION_FP32C> { using acc_t = int; };

template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads)
spread_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const double* __restrict__ fl, const int* __restrict__ perm,
                   const int* __restrict__ off, CompPtrs fe)
{
	using acc_t = typename SpreadSmem<D, DIMS, PREC>::acc_t;
	constexpr int M = D::M, sh = (M - 1) >> 1;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ RangeTable rt;
	__shared__ float scale_s[kMaxDims];
	__shared__ float bound_part[kTileThreads / 32][kMaxDims];

	const int T0 = tg.T[0], T1 = tg.T[1], T2 = DIMS == 3 ? tg.T[2] : 1;
	const int TV = T0 * T1 * T2;
	acc_t* acc = reinterpret_cast<acc_t*>(smem_raw);     // [DIMS][TV]
	int tc[3] = {0, 0, 0};
	tile_coords(tg, blockIdx.x, tc);
	int lo[3], hi[3][3];   // hi[c][d]
#pragma unroll
	for (int d = 0; d < DIMS; ++d) {
		lo[d] = tc[d] * tg.T[d];
#pragma unroll
		for (int c = 0; c < DIMS; ++c) hi[c][d] = min(lo[d] + tg.T[d], g.comp[c].points[d]);
	}
	for (int i = threadIdx.x; i < DIMS * TV; i += kTileThreads) acc[i] = (acc_t) 0;
	build_ranges<DIMS>(g, tg, tc, off, rt, true);
	const int total = rt.pref[rt.count];

	float scale[kMaxDims] = {1.f, 1.f, 1.f};
	if constexpr (PREC == IBK_PRECISION_FP32C) {
		// Sure bound on every face sum of this tile, per component.
		float b[kMaxDims] = {0.f, 0.f, 0.f};
		for (int it = threadIdx.x; it < total; it += kTileThreads) {
			const int p = __ldg(perm + range_lookup(rt, it));
#pragma unroll
			for (int c = 0; c < DIMS; ++c) b[c] += fabsf((float) __ldg(fl + (size_t) c * n + p));
		}
#pragma unroll
		for (int c = 0; c < DIMS; ++c) {
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) b[c] += __shfl_xor_sync(0xffffffffu, b[c], o);
			if ((threadIdx.x & 31) == 0) bound_part[threadIdx.x >> 5][c] = b[c];
		}
		__syncthreads();
		if (threadIdx.x < DIMS) {
			float s = 0.f;
			for (int w = 0; w < kTileThreads / 32; ++w) s += bound_part[w][threadIdx.x];
			// bound on |face| in force units: max_w * res * sum|F| (+ slack for
			// the float sum and the per-term rounding)
			const float bound = s * 1.001f * max_weight<D, DIMS>() * (float) g.res + 1e-30f;
			int e;
			frexpf(bound, &e);                      // bound < 2^e
			// scale * bound <= 2^29, leaving room for n/2 rounding units
			scale_s[threadIdx.x] = ldexpf(1.0f, 29 - e);
		}
		__syncthreads();
#pragma unroll
		for (int c = 0; c < DIMS; ++c) scale[c] = scale_s[c];
	} else {
		__syncthreads();
	}

	for (int it = threadIdx.x; it < total; it += kTileThreads) {
		const int p = __ldg(perm + range_lookup(rt, it));
		double z[DIMS];
#pragma unroll
		for (int d = 0; d < DIMS; ++d) z[d] = __ldg(x + (size_t) d * n + p);
#pragma unroll 1
		for (int c = 0; c < DIMS; ++c) {
			const CompGeom& cg = g.comp[c];
			int loc[DIMS][M];
			unsigned mask[DIMS];
			double dl[DIMS];
			bool any = true;
#pragma unroll
			for (int d = 0; d < DIMS; ++d) {
				AxisStep<M> a = axis_step<M>(g, cg, d, z[d]);
				dl[d] = a.delta;
				unsigned mk = 0;
#pragma unroll
				for (int m = 0; m < M; ++m) {
					int j = node_index(g, cg, d, a.base + m - sh);
					// spread drops nodes outside [0, points) (errors_negative);
					// the tile owns [lo, hi)
					const bool in = j >= lo[d] && j < hi[c][d];
					loc[d][m] = j - lo[d];
					mk |= (unsigned) in << m;
				}
				mask[d] = mk;
				any = any && mk;
			}
			if (!any) continue;
			acc_t* A = acc + c * TV;
			if constexpr (PREC == IBK_PRECISION_FP64) {
				const double f = __dmul_rn(g.res, __ldg(fl + (size_t) c * n + p));
				double w[DIMS][M];
#pragma unroll
				for (int d = 0; d < DIMS; ++d)
#pragma unroll
					for (int m = 0; m < M; ++m)
						w[d][m] = (mask[d] >> m & 1u) ? D::phi64(__dadd_rn(dl[d], (double) (m - sh))) : 0.0;
				if constexpr (DIMS == 3) {
#pragma unroll
					for (int m2 = 0; m2 < M; ++m2) {
						if (!(mask[2] >> m2 & 1u)) continue;
#pragma unroll
						for (int m1 = 0; m1 < M; ++m1) {
							if (!(mask[1] >> m1 & 1u)) continue;
							const double w12 = __dmul_rn(w[1][m1], w[2][m2]);
							const int row = (loc[2][m2] * T1 + loc[1][m1]) * T0;
#pragma unroll
							for (int m0 = 0; m0 < M; ++m0)
								if (mask[0] >> m0 & 1u)
									atomicAdd(A + row + loc[0][m0], __dmul_rn(__dmul_rn(w[0][m0], w12), f));
						}
					}
				} else {
#pragma unroll
					for (int m1 = 0; m1 < M; ++m1) {
						if (!(mask[1] >> m1 & 1u)) continue;
						const int row = loc[1][m1] * T0;
#pragma unroll
						for (int m0 = 0; m0 < M; ++m0)
							if (mask[0] >> m0 & 1u)
								atomicAdd(A + row + loc[0][m0], __dmul_rn(__dmul_rn(w[0][m0], w[1][m1]), f));
					}
				}
			} else {
				const float f = (float) (g.res * __ldg(fl + (size_t) c * n + p)) * scale[c];
				float w[DIMS][M];
#pragma unroll
				for (int d = 0; d < DIMS; ++d) weights32<D>((float) dl[d], w[d]);
#pragma unroll
				for (int m0 = 0; m0 < M; ++m0) w[0][m0] *= f;
				if constexpr (DIMS == 3) {
#pragma unroll
					for (int m2 = 0; m2 < M; ++m2) {
						if (!(mask[2] >> m2 & 1u)) continue;
#pragma unroll
						for (int m1 = 0; m1 < M; ++m1) {
							if (!(mask[1] >> m1 & 1u)) continue;
							const float w12 = w[1][m1] * w[2][m2];
							const int row = (loc[2][m2] * T1 + loc[1][m1]) * T0;
#pragma unroll
							for (int m0 = 0; m0 < M; ++m0)
								if (mask[0] >> m0 & 1u)
									atomicAdd(A + row + loc[0][m0], __float2int_rn(w[0][m0] * w12));
						}
					}
				} else {
#pragma unroll
					for (int m1 = 0; m1 < M; ++m1) {
						if (!(mask[1] >> m1 & 1u)) continue;
						const int row = loc[1][m1] * T0;
#pragma unroll
						for (int m0 = 0; m0 < M; ++m0)
							if (mask[0] >> m0 & 1u)
								atomicAdd(A + row + loc[0][m0], __float2int_rn(w[0][m0] * w[1][m1]));
					}
				}
			}
		}
	}
	__syncthreads();

	// every face of the tile, written once
#pragma unroll 1
	for (int c = 0; c < DIMS; ++c) {
		const CompGeom& cg = g.comp[c];
		const acc_t* A = acc + c * TV;
		const int e0 = hi[c][0] - lo[0];
		const int e1 = hi[c][1] - lo[1];
		const int e2 = DIMS == 3 ? hi[c][2] - lo[2] : 1;
		const double inv = 1.0 / (double) scale[c];
		double* __restrict__ out = fe.p[c];
		const int rows = e1 * e2;
		for (int i = threadIdx.x; i < rows * T0; i += kTileThreads) {
			const int l0 = i % T0;
			const int r = i / T0;
			if (l0 >= e0) continue;
			const int l1 = r % e1, l2 = r / e1;
			const size_t gi = (size_t) (lo[0] + l0) + (size_t) cg.points[0] *
				((size_t) (lo[1] + l1) + (DIMS == 3 ? (size_t) cg.points[1] * (size_t) (lo[2] + l2) : 0));
			const acc_t v = A[(l2 * T1 + l1) * T0 + l0];
			if constexpr (PREC == IBK_PRECISION_FP64) out[gi] = v;
			else out[gi] = (double) v * inv;
		}
	}
}

// ------------------------------------------------------------ interp ---

template <int PREC> struct InterpStage;
template <> struct InterpStage<IBK_PRECISION_FP64> { using val_t = double; };
template <> struct InterpStage<IBK_PRECISION_FP32C> { using val_t = float; };

// Halo of the staged region around the tile, per side.
template <int M> struct Halo {
	static constexpr int lo = 1 + ((M - 1) >> 1);
	static constexpr int hi = 1 + M / 2;
};

template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads)
interp_tile_kernel(GridGeom g, TileGeom tg, int n, const double* __restrict__ x,
                   const int* __restrict__ perm, const int* __restrict__ off,
                   ConstCompPtrs ue, double* __restrict__ ul)
{
	using val_t = typename InterpStage<PREC>::val_t;
	using P = Pattern<D::M, DIMS, D::every_other>;
	constexpr int M = D::M, sh = (M - 1) >> 1;
	constexpr int HL = Halo<M>::lo, HH = Halo<M>::hi;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	val_t* reg = reinterpret_cast<val_t*>(smem_raw);

	const int t = blockIdx.x;
	const int start = __ldg(off + t * tg.nclass);
	const int end = __ldg(off + (t + 1) * tg.nclass);
	if (start == end) return;
	int tc[3] = {0, 0, 0};
	tile_coords(tg, t, tc);
	int rlo[3], E[3];
#pragma unroll
	for (int d = 0; d < 3; ++d) {
		rlo[d] = d < DIMS ? tc[d] * tg.T[d] - HL : 0;
		E[d] = d < DIMS ? tg.T[d] + HL + HH : 1;
	}
	const int EV = E[0] * E[1] * E[2];

#pragma unroll 1
	for (int c = 0; c < DIMS; ++c) {
		const CompGeom& cg = g.comp[c];
		const double* __restrict__ u = ue.p[c];
		// stage the region: wrap periodic, clamp solid (interpolate.h:16-22)
		for (int i = threadIdx.x; i < EV; i += kTileThreads) {
			int l0 = i % E[0];
			int r = i / E[0];
			int l1 = r % E[1], l2 = r / E[1];
			int gc[3] = {rlo[0] + l0, rlo[1] + l1, rlo[2] + l2};
			size_t gi = 0, stride = 1;
#pragma unroll
			for (int d = 0; d < DIMS; ++d) {
				int v = gc[d];
				const int pd = cg.points[d];
				if (g.solid[d]) v = v < 0 ? 0 : (v >= pd ? pd - 1 : v);
				else { v %= cg.cells[d]; if (v < 0) v += cg.cells[d]; }
				gi += (size_t) v * stride;
				stride *= (size_t) pd;
			}
			reg[i] = (val_t) __ldg(u + gi);
		}
		__syncthreads();
		for (int it = start + threadIdx.x; it < end; it += kTileThreads) {
			const int p = __ldg(perm + it);
			double z[DIMS];
#pragma unroll
			for (int d = 0; d < DIMS; ++d) z[d] = __ldg(x + (size_t) d * n + p);
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
					int diff = b - (rlo[d] + HL);
					if (2 * diff > cells) b -= cells;
					else if (2 * diff < -cells) b += cells;
				}
				const int l = b - sh - rlo[d];
				loc[d] = l;
				inside = inside && l >= 0 && l + M <= E[d];
			}
			double v;
			if (inside) {
				if constexpr (PREC == IBK_PRECISION_FP64) {
					double w[DIMS][M];
#pragma unroll
					for (int d = 0; d < DIMS; ++d)
#pragma unroll
						for (int m = 0; m < M; ++m) w[d][m] = D::phi64(__dadd_rn(dl[d], (double) (m - sh)));
					const int base = DIMS == 3 ? (loc[2] * E[1] + loc[1]) * E[0] + loc[0] : loc[1] * E[0] + loc[0];
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
						v = __dadd_rn(v, __dmul_rn(wt, (double) reg[k]));   // interpolate.h:71-72
					}
				} else {
					float w[DIMS][M];
#pragma unroll
					for (int d = 0; d < DIMS; ++d) weights32<D>((float) dl[d], w[d]);
					const int base = DIMS == 3 ? (loc[2] * E[1] + loc[1]) * E[0] + loc[0] : loc[1] * E[0] + loc[0];
					float s = 0.f, comp = 0.f;
					constexpr int R = DIMS == 3 ? M * M : M;
#pragma unroll
					for (int r = 0; r < R; ++r) {
						const int m1 = r % M, m2 = r / M;
						const float* row = reinterpret_cast<const float*>(reg) + base +
							(DIMS == 3 ? (m2 * E[1] + m1) * E[0] : m1 * E[0]);
						float rs = 0.f;
#pragma unroll
						for (int m0 = 0; m0 < M; ++m0) rs = fmaf(w[0][m0], row[m0], rs);
						const float wr = DIMS == 3 ? w[1][m1] * w[2][m2] : w[1][m1];
						// TwoProd (FMA) + TwoSum (Knuth)
						const float pr = wr * rs;
						const float pe = fmaf(wr, rs, -pr);
						float ns, se;
						two_sum(s, pr, ns, se);
						s = ns;
						comp += pe + se;
					}
					v = (double) s + (double) comp;
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
						int j = node_index(g, cg, d, a.base + m - sh);
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
			ul[(size_t) c * n + p] = v;
		}
		__syncthreads();
	}
}

} // namespace ibk
