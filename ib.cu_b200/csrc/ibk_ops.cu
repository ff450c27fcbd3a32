// Operator implementations and the (delta, dims, precision) dispatch table.
#include <cstdio>
#include "ibk_internal.h"
#include "ibk_direct.cuh"
#include "ibk_tiled.cuh"

namespace ibk {

namespace {

constexpr int kThreads = 128;

inline int blocks_for(long long n, int threads) { return (int) ((n + threads - 1) / threads); }

// Counting sort of the points by (tile, reach class): perm + bin offsets.
template <int M, int DIMS>
ibk_status bin_points(Plan& plan, const OpArgs& a, int** perm_out, int** off_out)
{
	const TileGeom& tg = plan.tiles;
	ibk_status s;
	const int need = a.n > plan.reserved_points ? a.n : plan.reserved_points;
	if ((s = ensure_scratch(plan, kSlotCount, sizeof(int) * (size_t) tg.num_bins, a.stream, true)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotOffset, sizeof(int) * ((size_t) tg.num_bins + 1), a.stream)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotKeyRank, sizeof(int2) * (size_t) need, a.stream)) != IBK_OK) return s;
	if ((s = ensure_scratch(plan, kSlotPerm, sizeof(int) * (size_t) need, a.stream)) != IBK_OK) return s;
	int* count = static_cast<int*>(plan.scratch[kSlotCount].ptr);
	int* off = static_cast<int*>(plan.scratch[kSlotOffset].ptr);
	int2* kr = static_cast<int2*>(plan.scratch[kSlotKeyRank].ptr);
	int* perm = static_cast<int*>(plan.scratch[kSlotPerm].ptr);
	const GridGeom& g = *a.g;
	const int nb = blocks_for(a.n, 256);
	if ((s = launch(plan, "bin_count_kernel", a.stream, [&] {
		bin_count_kernel<M, DIMS><<<nb, 256, 0, a.stream>>>(g, tg, a.n, a.x, count, kr);
	})) != IBK_OK) return s;
	if ((s = launch(plan, "bin_scan_kernel", a.stream, [&] {
		bin_scan_kernel<<<1, kScanThreads, 0, a.stream>>>(count, off, tg.num_bins);
	})) != IBK_OK) return s;
	if ((s = launch(plan, "bin_scatter_kernel", a.stream, [&] {
		bin_scatter_kernel<<<nb, 256, 0, a.stream>>>(a.n, kr, off, perm);
	})) != IBK_OK) return s;
	*perm_out = perm;
	*off_out = off;
	return IBK_OK;
}

template <typename K>
ibk_status set_smem(K kernel, size_t bytes)
{
	if (bytes > 48 * 1024) {
		cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	}
	return IBK_OK;
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status spread_impl(Plan& plan, const OpArgs& a, const double* fl, CompPtrs fe)
{
	using D = Delta<KIND, ORDER>;
	const GridGeom& g = *a.g;
	const TileGeom& tg = plan.tiles;
	int *perm = nullptr, *off = nullptr;
	ibk_status s = bin_points<D::M, DIMS>(plan, a, &perm, &off);
	if (s != IBK_OK) return s;
	using acc_t = typename SpreadSmem<D, DIMS, PREC>::acc_t;
	const size_t smem = sizeof(acc_t) * (size_t) DIMS * tg.T[0] * tg.T[1] * (DIMS == 3 ? tg.T[2] : 1);
	auto kern = spread_tile_kernel<D, DIMS, PREC>;
	if ((s = set_smem(kern, smem)) != IBK_OK) return s;
	return launch(plan, "spread_tile_kernel", a.stream, [&] {
		kern<<<tg.num_tiles, kTileThreads, smem, a.stream>>>(g, tg, a.n, a.x, fl, perm, off, fe);
	});
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status interp_impl(Plan& plan, const OpArgs& a, ConstCompPtrs ue, double* ul)
{
	using D = Delta<KIND, ORDER>;
	const GridGeom& g = *a.g;
	const TileGeom& tg = plan.tiles;
	int *perm = nullptr, *off = nullptr;
	ibk_status s = bin_points<D::M, DIMS>(plan, a, &perm, &off);
	if (s != IBK_OK) return s;
	using val_t = typename InterpStage<PREC>::val_t;
	constexpr int HL = Halo<D::M>::lo, HH = Halo<D::M>::hi;
	size_t ev = 1;
	for (int d = 0; d < DIMS; ++d) ev *= (size_t) (tg.T[d] + HL + HH);
	const size_t smem = sizeof(val_t) * ev;
	auto kern = interp_tile_kernel<D, DIMS, PREC>;
	if ((s = set_smem(kern, smem)) != IBK_OK) return s;
	return launch(plan, "interp_tile_kernel", a.stream, [&] {
		kern<<<tg.num_tiles, kTileThreads, smem, a.stream>>>(g, tg, a.n, a.x, perm, off, ue, ul);
	});
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
	               &keys_impl<KIND, ORDER, DIMS>};
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

// Tile extent per axis: 16 cells where the last tile keeps at least M cells
// (a stencil can then reach at most one neighbour per side), otherwise the
// nearest size in [8, 20] that does; axes of at most 16 cells are one tile.
TileGeom make_tiles(const GridGeom& g, int tag, int M)
{
	TileGeom tg{};
	tg.tag_mac = tag == IBK_TAG_MAC;
	tg.num_tiles = 1;
	const int minlast = M > 2 ? M : 2;
	for (int d = 0; d < kMaxDims; ++d) {
		if (d >= g.dims) { tg.T[d] = 1; tg.ntiles[d] = 1; tg.cells[d] = 1; continue; }
		const int cells = g.comp[0].cells[d];
		tg.cells[d] = cells;
		int T = cells;
		if (cells > 16) {
			// <= 20 keeps the FP64 staging region within shared memory
			static const int prefs[] = {16, 14, 18, 12, 20, 10, 8, 9, 11, 13, 15, 17, 19};
			T = 0;
			for (int t : prefs) {
				const int r = cells % t;
				if (r == 0 || r >= minlast) { T = t; break; }
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

const OpTable* find_ops(int kind, int order, int dims, int precision)
{
	if (kind != kBspline) order = 0;
	for (const Entry& e : kTable)
		if (e.kind == kind && e.order == order && e.dims == dims && e.prec == precision)
			return &e.ops;
	return nullptr;
}

} // namespace ibk
