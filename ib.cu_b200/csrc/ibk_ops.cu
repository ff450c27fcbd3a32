// Operator implementations and the (delta, dims, precision) dispatch table.
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <cuda.h>
#include "ibk_internal.h"
#include "ibk_direct.cuh"
#include "ibk_tiled.cuh"

namespace ibk {

namespace {

constexpr int kThreads = 128;

inline int blocks_for(long long n, int threads) { return (int) ((n + threads - 1) / threads); }

// Per-point kernels for degenerate grids (an axis with fewer cells than the
// stencil is wide, where one stencil would reach the same face twice).
template <typename D, int DIMS>
ibk_status spread_direct(Plan& plan, const OpArgs& a, const double* fl, CompPtrs fe)
{
	const GridGeom& g = *a.g;
	for (int c = 0; c < DIMS; ++c) {
		cudaError_t e = cudaMemsetAsync(fe.p[c], 0, sizeof(double) * (size_t) g.comp[c].size, a.stream);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
	}
	return launch(plan, "spread_direct_kernel", a.stream, [&] {
		spread_direct_kernel<D, DIMS><<<blocks_for(a.n, kThreads), kThreads, 0, a.stream>>>(g, a.n, a.x, fl, fe);
	});
}

template <typename D, int DIMS>
ibk_status interp_direct(Plan& plan, const OpArgs& a, ConstCompPtrs ue, double* ul)
{
	return launch(plan, "interp_direct_kernel", a.stream, [&] {
		interp_direct_kernel<D, DIMS><<<blocks_for(a.n, kThreads), kThreads, 0, a.stream>>>(*a.g, a.n, a.x, ue, ul);
	});
}

// Counting sort of the points by (tile, reach class): records in bin order
// and the bin offsets; with forces f (a spread follows) also the bins' force
// statistics for the FP32C scale.
template <int M, int DIMS>
ibk_status bin_points(Plan& plan, const OpArgs& a, const TileGeom& tg, const PointRec** recs_out,
                      const int** off_out, const double* f = nullptr, BinStatsView* stats_out = nullptr)
{
	ibk_status s;
	const int need = a.n > plan.reserved_points ? a.n : plan.reserved_points;
	if ((s = ensure_scratch(plan, kSlotCount, sizeof(int) * (size_t) tg.num_bins, a.stream, true)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotOffset, sizeof(int) * ((size_t) tg.num_bins + 1), a.stream)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotKeyRank, sizeof(int2) * (size_t) need, a.stream)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotRecs, sizeof(PointRec) * (size_t) need, a.stream)) != IBK_OK) return s;
	const int nchunks = (tg.num_bins + kScanChunk - 1) / kScanChunk;
	if ((s = ensure_scratch(plan, kSlotChunk, sizeof(int) * ((size_t) nchunks + 1), a.stream)) != IBK_OK) return s;
	int* count = static_cast<int*>(plan.scratch[kSlotCount].ptr);
	int* off = static_cast<int*>(plan.scratch[kSlotOffset].ptr);
	int2* kr = static_cast<int2*>(plan.scratch[kSlotKeyRank].ptr);
	PointRec* recs = static_cast<PointRec*>(plan.scratch[kSlotRecs].ptr);
	int* chunk = static_cast<int*>(plan.scratch[kSlotChunk].ptr);
	const GridGeom& g = *a.g;
	const int nb = blocks_for(a.n, 256);
	BinStats st{nullptr, g.res, nullptr};
	if (f) {
		const size_t nm = sizeof(unsigned) * kMaxDims * (size_t) tg.num_bins;
		if ((s = ensure_scratch(plan, kSlotBinMax, nm, a.stream)) != IBK_OK) return s;
		st.f = f;
		st.binmax = static_cast<unsigned*>(plan.scratch[kSlotBinMax].ptr);
		cudaError_t e = cudaMemsetAsync(st.binmax, 0, nm, a.stream);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
		*stats_out = BinStatsView{st.binmax};
	}
	if ((s = launch(plan, "bin_count_kernel", a.stream, [&] {
		bin_count_kernel<M, DIMS><<<nb, 256, 0, a.stream>>>(g, tg, a.n, a.x, count, kr, st);
	})) != IBK_OK) return s;
	if ((s = launch(plan, "bin_chunk_sum_kernel", a.stream, [&] {
		bin_chunk_sum_kernel<<<nchunks, kScanThreads, 0, a.stream>>>(count, chunk, tg.num_bins);
	})) != IBK_OK) return s;
	if ((s = launch(plan, "bin_scan_kernel", a.stream, [&] {
		bin_scan_kernel<<<nchunks, kScanThreads, 0, a.stream>>>(count, chunk, off, tg.num_bins, nchunks);
	})) != IBK_OK) return s;
	if ((s = launch(plan, "bin_scatter_kernel", a.stream, [&] {
		bin_scatter_kernel<M, DIMS><<<nb, 256, 0, a.stream>>>(g, tg, a.n, a.x, kr, off, recs);
	})) != IBK_OK) return s;
	*recs_out = recs;
	*off_out = off;
	return IBK_OK;
}

// Opt the kernel in to `bytes` of dynamic shared memory (static shared
// memory counts against the 48 KB default too, so this is always set).
template <typename K>
ibk_status set_smem(K kernel, size_t bytes)
{
	cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	return IBK_OK;
}

template <typename D, int DIMS, int PREC>
ibk_status launch_spread(Plan& plan, const OpArgs& a, const TileGeom& tg, const PointRec* recs, const int* off,
                         BinStatsView bs, const double* fl, CompPtrs fe)
{
	const size_t smem = spread_smem_bytes(*a.g, tg, D::M, PREC);
	auto kern = spread_tile_kernel<D, DIMS, PREC>;
	ibk_status s = set_smem(kern, smem);
	if (s != IBK_OK) return s;
	// FP32C: one CTA per tile for every component, dense tiles deferred to
	// the folded kernel; FP64: per (tile, component)
	Deferral defer{nullptr, nullptr};
	if constexpr (PREC == IBK_PRECISION_FP32C) {
		if ((s = ensure_scratch(plan, kSlotDefer, sizeof(int) * ((size_t) tg.num_tiles * DIMS + 4), a.stream)) != IBK_OK)
			return s;
		defer.count = static_cast<int*>(plan.scratch[kSlotDefer].ptr);
		defer.list = defer.count + 4;
		cudaError_t e = cudaMemsetAsync(defer.count, 0, sizeof(int), a.stream);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
	}
	const dim3 grid(tg.num_tiles, PREC == IBK_PRECISION_FP32C ? 1 : DIMS);
	if ((s = launch(plan, "spread_tile_kernel", a.stream, [&] {
		kern<<<grid, kTileThreads, smem, a.stream>>>(*a.g, tg, a.n, a.x, fl, recs, off, bs, fe, defer);
	})) != IBK_OK) return s;
	if constexpr (PREC == IBK_PRECISION_FP32C) {
		auto dense = spread_dense_kernel<D, DIMS>;
		if ((s = set_smem(dense, smem)) != IBK_OK) return s;
		const int gd = std::max(1, std::min(tg.num_tiles * DIMS, 4 * plan.num_sms));
		return launch(plan, "spread_dense_kernel", a.stream, [&] {
			dense<<<gd, kTileThreads, smem, a.stream>>>(*a.g, tg, a.n, a.x, fl, recs, off, bs, fe, defer.list,
			                                            defer.count);
		});
	}
	return IBK_OK;
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status spread_impl(Plan& plan, const OpArgs& a, const double* fl, CompPtrs fe)
{
	using D = Delta<KIND, ORDER>;
	if (!plan.tiled) return spread_direct<D, DIMS>(plan, a, fl, fe);
	const PointRec* recs = nullptr;
	const int* off = nullptr;
	BinStatsView bs{nullptr};
	constexpr bool fix = PREC == IBK_PRECISION_FP32C;
	ibk_status s = bin_points<D::M, DIMS>(plan, a, plan.spread_tiles, &recs, &off, fix ? fl : nullptr, &bs);
	if (s != IBK_OK) return s;
	return launch_spread<D, DIMS, PREC>(plan, a, plan.spread_tiles, recs, off, bs, fl, fe);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
	static EncodeTiledFn fn = [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
		    q != cudaDriverEntryPointSuccess) {
			cudaGetLastError();
			return (EncodeTiledFn) nullptr;
		}
		return reinterpret_cast<EncodeTiledFn>(p);
	}();
	return fn;
}

} // namespace

// Tensor map of one FP64 component grid with box `box` (elements per axis).
// False when the grid or box violates a TMA rule (16-byte base and strides,
// box rows a multiple of 16 bytes, at most 256 elements per box axis).
bool grid_tensor_map(CUtensorMap* map, const double* base, const CompGeom& cg, int dims, const int* box)
{
	EncodeTiledFn fn = encode_fn();
	if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
	if ((cg.points[0] * sizeof(double)) % 16 != 0 || (box[0] * sizeof(double)) % 16 != 0) return false;
	cuuint64_t gdim[3], gstride[2];
	cuuint32_t bdim[3], estride[3] = {1, 1, 1};
	cuuint64_t stride = sizeof(double);
	for (int d = 0; d < dims; ++d) {
		if (box[d] > 256 || box[d] > cg.points[d]) return false;
		gdim[d] = (cuuint64_t) cg.points[d];
		bdim[d] = (cuuint32_t) box[d];
		if (d > 0) gstride[d - 1] = stride;
		stride *= (cuuint64_t) cg.points[d];
	}
	CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t) dims, const_cast<double*>(base),
	                gdim, gstride, bdim, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
	                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
	                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	return r == CUDA_SUCCESS;
}

namespace {

template <typename D, int DIMS, int PREC>
ibk_status launch_interp(Plan& plan, const OpArgs& a, const TileGeom& tg, const PointRec* recs, const int* off,
                         ConstCompPtrs ue, double* ul)
{
	const GridGeom& g = *a.g;
	const size_t smem = interp_smem_bytes<D::M>(g, tg);
	// TMA needs every region's x origin on a 16-byte boundary: even tile
	// extents along x (the region's lower x offset is even by construction)
	TmaMaps maps{};
	int use_tma = tg.T[0] % 2 == 0;
	for (int c = 0; c < DIMS && use_tma; ++c) {
		int lower[3], box[3];
		region_of<D::M>(g, tg, c, lower, box);
		use_tma = grid_tensor_map(&maps.map[c], ue.p[c], g.comp[c], DIMS, box);
	}
	auto kern = interp_tile_kernel<D, DIMS, PREC>;
	ibk_status s = set_smem(kern, smem);
	if (s != IBK_OK) return s;
	return launch(plan, "interp_tile_kernel", a.stream, [&] {
		kern<<<dim3(tg.num_tiles, DIMS), kTileThreads, smem, a.stream>>>(g, tg, a.n, a.x, recs, off, ue, ul,
		                                                                   maps, use_tma, plan.d_status);
	});
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status interp_impl(Plan& plan, const OpArgs& a, ConstCompPtrs ue, double* ul)
{
	using D = Delta<KIND, ORDER>;
	if (!plan.tiled) return interp_direct<D, DIMS>(plan, a, ue, ul);
	const PointRec* recs = nullptr;
	const int* off = nullptr;
	ibk_status s = bin_points<D::M, DIMS>(plan, a, plan.tiles, &recs, &off);
	if (s != IBK_OK) return s;
	return launch_interp<D, DIMS, PREC>(plan, a, plan.tiles, recs, off, ue, ul);
}

bool same_tiles(const TileGeom& a, const TileGeom& b)
{
	return a.T[0] == b.T[0] && a.T[1] == b.T[1] && a.T[2] == b.T[2];
}

// Spread and interpolation at the same positions: one binning serves both
// when the plan's spread and interpolation tiles agree.
template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status both_impl(Plan& plan, const OpArgs& a, const double* fl, CompPtrs fe, ConstCompPtrs ue, double* ul)
{
	using D = Delta<KIND, ORDER>;
	if (!plan.tiled) {
		ibk_status s = spread_direct<D, DIMS>(plan, a, fl, fe);
		return s != IBK_OK ? s : interp_direct<D, DIMS>(plan, a, ue, ul);
	}
	const PointRec* recs = nullptr;
	const int* off = nullptr;
	BinStatsView bs{nullptr};
	constexpr bool fix = PREC == IBK_PRECISION_FP32C;
	ibk_status s = bin_points<D::M, DIMS>(plan, a, plan.spread_tiles, &recs, &off, fix ? fl : nullptr, &bs);
	if (s != IBK_OK) return s;
	if ((s = launch_spread<D, DIMS, PREC>(plan, a, plan.spread_tiles, recs, off, bs, fl, fe)) != IBK_OK) return s;
	if (!same_tiles(plan.spread_tiles, plan.tiles)) {
		if ((s = bin_points<D::M, DIMS>(plan, a, plan.tiles, &recs, &off)) != IBK_OK) return s;
	}
	return launch_interp<D, DIMS, PREC>(plan, a, plan.tiles, recs, off, ue, ul);
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
	               &keys_impl<KIND, ORDER, DIMS>, &both_impl<KIND, ORDER, DIMS, PREC>};
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
	IBK_DELTA_ENTRIES(2, IBK_PRECISION_FP32C),
	IBK_DELTA_ENTRIES(3, IBK_PRECISION_FP32C),
};

} // namespace

// Tile extent per axis: the preferred extent (by default 16 cells, or a
// quarter of a small axis, at least 8) where the last tile keeps at least M
// cells (a stencil can then reach at most one
// neighbour per side), otherwise the nearest size that does; an axis no
// longer than the preferred extent is one tile.
TileGeom make_tiles(const GridGeom& g, int tag, int M, const int* pref_extent)
{
	TileGeom tg{};
	tg.tag_mac = tag == IBK_TAG_MAC;
	tg.num_tiles = 1;
	const int minlast = M > 2 ? M : 2;
	for (int d = 0; d < kMaxDims; ++d) {
		if (d >= g.dims) { tg.T[d] = 1; tg.ntiles[d] = 1; tg.cells[d] = 1; continue; }
		const int cells = g.comp[0].cells[d];
		tg.cells[d] = cells;
		// default: 16 cells, but at least four tiles per axis on small grids
		// (extents of at least 8), so their work spreads over more CTAs
		const int want = pref_extent ? pref_extent[d] : std::min(16, std::max(8, cells / 4));
		int T = cells;
		if (cells > want) {
			static const int prefs[] = {16, 14, 18, 12, 20, 10, 8, 9, 11, 13, 15, 17, 19};
			T = 0;
			if (want != 16) {
				// the preferred extent, then its nearest neighbours (larger
				// first), then the regular ladder
				for (int dist = 0; dist <= 6 && T == 0; ++dist)
					for (int sgn = 1; sgn >= -1 && T == 0; sgn -= 2) {
						const int t = want + sgn * dist;
						if (t < minlast || t < 4 || t >= cells) continue;
						const int r = cells % t;
						if (r == 0 || r >= minlast) T = t;
					}
			}
			for (int i = 0; i < (int) (sizeof(prefs) / sizeof(prefs[0])) && T == 0; ++i) {
				const int r = cells % prefs[i];
				if (r == 0 || r >= minlast) T = prefs[i];
			}
			if (T == 0) T = 8;   // unreachable for M <= 6: some t in [8, 20] leaves r == 0 or r >= M
		}
		tg.T[d] = T;
		tg.ntiles[d] = (cells + T - 1) / T;
		tg.num_tiles *= tg.ntiles[d];
	}
	tg.nclass = ipow3(g.dims);
	tg.num_bins = tg.num_tiles * tg.nclass;
	return tg;
}

size_t spread_tile_bytes(const GridGeom& g, const TileGeom& tg, int M, int precision)
{
	return spread_smem_bytes(g, tg, M, precision);
}

void interp_region(const GridGeom& g, const TileGeom& tg, int M, int c, int* lower, int* extent)
{
	switch (M) {
	case 2: region_of<2>(g, tg, c, lower, extent); return;
	case 3: region_of<3>(g, tg, c, lower, extent); return;
	case 4: region_of<4>(g, tg, c, lower, extent); return;
	case 5: region_of<5>(g, tg, c, lower, extent); return;
	case 6: region_of<6>(g, tg, c, lower, extent); return;
	}
}

size_t interp_region_bytes(const GridGeom& g, const TileGeom& tg, int M)
{
	switch (M) {
	case 2: return interp_smem_bytes<2>(g, tg);
	case 3: return interp_smem_bytes<3>(g, tg);
	case 4: return interp_smem_bytes<4>(g, tg);
	case 5: return interp_smem_bytes<5>(g, tg);
	case 6: return interp_smem_bytes<6>(g, tg);
	}
	return 0;
}

const OpTable* find_ops(int kind, int order, int dims, int precision)
{
	if (kind != kBspline) order = 0;
	for (const Entry& e : kTable)
		if (e.kind == kind && e.order == order && e.dims == dims && e.prec == precision)
			return &e.ops;
	return nullptr;
}

} // namespace ibk
