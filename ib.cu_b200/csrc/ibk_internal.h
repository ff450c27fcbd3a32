// Host-side internals shared by the library's translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "ibk.h"
#include "ibk_device.cuh"

namespace ibk {

// Launch context handed to every operator implementation.
struct OpArgs {
	const GridGeom* g;
	int n;
	const double* x;
	cudaStream_t stream;
};

struct Plan;

// Implementation entry points (one instantiation per delta / dims / precision).
using SpreadFn = ibk_status (*)(Plan&, const OpArgs&, const double* fl, CompPtrs fe);
using InterpFn = ibk_status (*)(Plan&, const OpArgs&, ConstCompPtrs ue, double* ul);
using KeysFn = ibk_status (*)(Plan&, const OpArgs&, int comp, int* keys);
using BothFn = ibk_status (*)(Plan&, const OpArgs&, const double* fl, CompPtrs fe, ConstCompPtrs ue, double* ul);

struct OpTable {
	SpreadFn spread;
	InterpFn interp;
	KeysFn keys;
	BothFn both;             // spread and interpolation at the same positions
};

// Device scratch owned by a plan: grown on demand outside stream capture,
// released with the plan.
struct Scratch {
	void* ptr = nullptr;
	size_t bytes = 0;
};

struct TimedLaunch {
	int stat;            // index into Plan::stats
	cudaEvent_t start, stop;
};

struct Plan {
	GridGeom g{};
	TileGeom tiles{};          // interpolation tiles (halo staged in shared memory)
	TileGeom spread_tiles{};   // spread tiles (owner-computes accumulators); the
	                           // same as `tiles` unless set apart, so one binning serves both
	bool tiled = true;         // false: an axis has fewer cells than the stencil width
	ibk_grid_info info{};
	int delta_kind = 0, delta_order = 0, precision = 0, tag = 0;
	int device = 0;
	int num_sms = 0;
	int reserved_points = 0;
	OpTable ops{};
	Scratch scratch[8];
	int* d_status = nullptr;   // device-side error word written by kernel checks
	// instrumentation
	long long launches = 0;
	bool profiling = false;
	std::vector<ibk_kernel_stat> stats;
	std::vector<TimedLaunch> pending;
	std::vector<cudaEvent_t> event_pool;
};

// Bracket one kernel launch: counts it and, when profiling, records events.
ibk_status launch_begin(Plan& plan, const char* name, cudaStream_t stream, int& slot);
ibk_status launch_end(Plan& plan, const char* name, cudaStream_t stream, int slot);

template <typename F>
ibk_status launch(Plan& plan, const char* name, cudaStream_t stream, F&& body)
{
	int slot = -1;
	ibk_status s = launch_begin(plan, name, stream, slot);
	if (s != IBK_OK) return s;
	body();
	return launch_end(plan, name, stream, slot);
}

// Scratch slots of a plan.
enum { kSlotCount = 0, kSlotOffset = 1, kSlotKeyRank = 2, kSlotRecs = 3, kSlotChunk = 4, kSlotBinMax = 5,
       kSlotSums = 6, kSlotDefer = 7 };

// Largest tile extent in cells per axis (point records keep tile-relative
// origins in 8 bits).
constexpr int kMaxTileExtent = 64;

// Shared memory of a spread CTA for tiles tg, and of an interpolation CTA's
// staged region (largest component, stencil width M), in bytes.
size_t spread_tile_bytes(const GridGeom& g, const TileGeom& tg, int M, int precision);
size_t interp_region_bytes(const GridGeom& g, const TileGeom& tg, int M);
// Staged interpolation region of component c relative to a tile's first
// cell: lower corner and extent per axis (the TMA box).
void interp_region(const GridGeom& g, const TileGeom& tg, int M, int c, int* lower, int* extent);

// Tile decomposition of a plan's grid for stencil width M.
// pref_extent: preferred tile extent per axis (nullptr: 16 cells).
TileGeom make_tiles(const GridGeom& g, int tag, int M, const int* pref_extent = nullptr);

// Returns the table for (kind, order, dims, precision) or nullptr.
const OpTable* find_ops(int kind, int order, int dims, int precision);

// Grow scratch slot `slot` of the plan to at least `bytes`.
ibk_status ensure_scratch(Plan& plan, int slot, size_t bytes, cudaStream_t stream, bool zero = false);

// Stencil width M of a delta (1 + order for bspline<order>).
int meshwidths_of(int kind, int order);

// Validation of a domain / tag / refinement triple (status + message).
ibk_status check_domain(const ibk_domain* domain, int tag, int refinement);

// Geometry of every component grid of a validated domain.
ibk_status make_geometry(const ibk_domain* domain, int tag, int refinement, int meshwidths, GridGeom& g,
                         ibk_grid_info& info);

// Tensor map of one FP64 component grid for TMA boxes of `box` elements per
// axis; false when a TMA rule is violated (16-byte base and strides, box rows
// a multiple of 16 bytes, at most 256 elements per box axis).
bool grid_tensor_map(CUtensorMap* map, const double* base, const CompGeom& cg, int dims, const int* box);

ibk_status set_error(ibk_status s, const std::string& msg);
ibk_status check_launch(const char* what);

} // namespace ibk
