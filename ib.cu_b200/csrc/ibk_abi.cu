// C ABI of the library (declared in include/ibk.h): plans, geometry, errors.
//
// Plan geometry follows the reference's constexpr grid code, operation by
// operation, on the host (compiled with -ffp-contract=off):
//   fd::domain::unit      = foldl(algo::gcd, lengths)   include/fd/domain.h:30-32,
//                                                       include/algo/gcd.h:7-34
//   resolution            = refinement / unit           include/fd/grid.h:232-239
//   alignment             = 0 along the component's own axis for fd::mac,
//                           0.5 elsewhere / for fd::centered
//                                                       include/fd/cell.h:80-114,194-195
//   cells                 = (int) (length * r + 0.5)   include/fd/discretization.h:161
//   points                = cells - (on_boundary && solid)             :162
//   shift                 = alignment + (solid && on_boundary)         :113
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include "ibk_internal.h"

namespace ibk {

namespace {

thread_local std::string g_last_error;

double host_floor(double x)
{
	return (double) (long) (x - (double) (x < 0 && (-x != (double) (long) -x)));
}

double host_modulo(double x, double s) { return x - s * host_floor(x / s); }

double host_abs(double x) { return (double) ((x > 0) - (x < 0)) * x; }

double gcd_impl(double a, double b)
{
	double eps = DBL_EPSILON;
	while (host_abs(b) > eps) {
		if (a < b) { double t = a; a = b; b = t; }
		double c = a - host_floor(a / b) * b;
		a = b; b = c;
		eps *= 2;
	}
	return a;
}

double gcd_fp(double a, double b)
{
	if (a < b) { double t = a; a = b; b = t; }
	return gcd_impl(1.0, b / a) * a;
}

} // namespace

int meshwidths_of(int kind, int order)
{
	switch (kind) {
	case kBspline: return order + 1;
	case kPeskin: return 4;
	case kRoma: return 3;
	case kCosine: return 4;
	case kHat: return 2;
	}
	return 0;
}

ibk_status check_domain(const ibk_domain* domain, int tag, int refinement)
{
	const int dims = domain->dims;
	if (dims < 2 || dims > 3) return set_error(IBK_ERR_UNSUPPORTED, "dims must be 2 or 3");
	if (refinement <= 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "refinement must be positive");
	if (tag != IBK_TAG_MAC && tag != IBK_TAG_CENTERED) return set_error(IBK_ERR_INVALID_ARGUMENT, "unknown grid tag");
	for (int d = 0; d < dims; ++d)
		if (!(domain->length[d] > 0) || !(domain->length[d] < 1e300))
			return set_error(IBK_ERR_INVALID_ARGUMENT, "dimension lengths must be positive and finite");
	return IBK_OK;
}

// fd::domain / fd::grid / fd::discretization geometry of every component
// (include/fd/domain.h:30-32, include/algo/gcd.h:27-34, include/fd/grid.h:39-46,
// include/fd/discretization.h:113-164).  The domain is validated by the caller.
ibk_status make_geometry(const ibk_domain* domain, int tag, int refinement, int meshwidths, GridGeom& g,
                         ibk_grid_info& info)
{
	const int dims = domain->dims;
	g = GridGeom{};
	info = ibk_grid_info{};
	g.dims = dims;
	double unit = domain->length[0];
	for (int d = 1; d < dims; ++d) unit = gcd_fp(unit, domain->length[d]);
	const double r = (double) refinement / unit;
	g.r = r;
	double res = 1;
	for (int d = dims - 1; d >= 0; --d) res = r * res;
	g.res = res;
	for (int d = 0; d < dims; ++d) {
		g.length[d] = domain->length[d];
		g.length_safe[d] = domain->length[d] * (1.0 - 0x1p-52);
		g.solid[d] = domain->boundary[d] != IBK_PERIODIC;
	}
	info.dims = dims;
	info.meshwidths = meshwidths;
	info.unit = unit;
	info.resolution = r;
	for (int c = 0; c < dims; ++c) {
		CompGeom& cg = g.comp[c];
		long long size = 1;
		for (int d = 0; d < dims; ++d) {
			double al = (tag == IBK_TAG_MAC && c == d) ? host_modulo(0.5 + 0.5, 1.0) : 0.5;
			al = host_modulo(al, 1.0);
			const int on_boundary = !al;
			const double cells_f = domain->length[d] * r + 0.5;
			if (!(cells_f < 2147483647.0)) return set_error(IBK_ERR_INVALID_ARGUMENT, "grid too large");
			const int cells = (int) cells_f;
			const int points = cells - (on_boundary && g.solid[d]);
			if (points < 1) return set_error(IBK_ERR_INVALID_ARGUMENT, "grid has no points along a dimension");
			const double shift = al + (double) (g.solid[d] && on_boundary);
			cg.cells[d] = cells;
			cg.points[d] = points;
			cg.shift[d] = shift;
			cg.s_over_r[d] = shift / r;
			info.cells[c][d] = cells;
			info.points[c][d] = points;
			info.shift[c][d] = shift;
			size *= points;
		}
		if (size >= (1LL << 31)) return set_error(IBK_ERR_INVALID_ARGUMENT, "component grid exceeds 2^31 faces (32-bit reference indices)");
		cg.size = size;
		info.size[c] = size;
	}
	return IBK_OK;
}

ibk_status set_error(ibk_status s, const std::string& msg)
{
	g_last_error = msg;
	return s;
}

ibk_status check_launch(const char* what)
{
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess)
		return set_error(IBK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
	return IBK_OK;
}

ibk_status ensure_scratch(Plan& plan, int slot, size_t bytes, cudaStream_t stream, bool zero)
{
	Scratch& s = plan.scratch[slot];
	if (s.bytes >= bytes) return IBK_OK;
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(stream, &cap) == cudaSuccess && cap != cudaStreamCaptureStatusNone)
		return set_error(IBK_ERR_CAPACITY, "plan scratch must grow during stream capture; call ibk_plan_reserve first");
	// Round up to limit regrowth.
	size_t want = bytes + bytes / 4 + 4096;
	void* p = nullptr;
	cudaError_t e = cudaStreamSynchronize(stream);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
	if (s.ptr) cudaFree(s.ptr);
	s.ptr = nullptr;
	s.bytes = 0;
	e = cudaMalloc(&p, want);
	if (e != cudaSuccess) {
		cudaGetLastError();
		return set_error(IBK_ERR_OUT_OF_MEMORY, "cudaMalloc of plan scratch failed");
	}
	if (zero) {
		e = cudaMemset(p, 0, want);
		if (e != cudaSuccess) { cudaFree(p); return set_error(IBK_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e)); }
	}
	s.ptr = p;
	s.bytes = want;
	return IBK_OK;
}

namespace {

cudaEvent_t pooled_event(Plan& plan)
{
	if (!plan.event_pool.empty()) {
		cudaEvent_t e = plan.event_pool.back();
		plan.event_pool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}

int stat_index(Plan& plan, const char* name)
{
	for (size_t i = 0; i < plan.stats.size(); ++i)
		if (std::strncmp(plan.stats[i].name, name, sizeof(plan.stats[i].name)) == 0) return (int) i;
	ibk_kernel_stat st{};
	std::strncpy(st.name, name, sizeof(st.name) - 1);
	plan.stats.push_back(st);
	return (int) plan.stats.size() - 1;
}

ibk_status drain_pending(Plan& plan)
{
	for (TimedLaunch& t : plan.pending) {
		cudaError_t e = cudaEventSynchronize(t.stop);
		if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaEventSynchronize: ") + cudaGetErrorString(e));
		float ms = 0.f;
		cudaEventElapsedTime(&ms, t.start, t.stop);
		plan.stats[t.stat].total_ms += ms;
		plan.event_pool.push_back(t.start);
		plan.event_pool.push_back(t.stop);
	}
	plan.pending.clear();
	return IBK_OK;
}

} // namespace

ibk_status launch_begin(Plan& plan, const char* name, cudaStream_t stream, int& slot)
{
	slot = -1;
	if (!plan.profiling) return IBK_OK;
	TimedLaunch t;
	t.stat = stat_index(plan, name);
	t.start = pooled_event(plan);
	t.stop = pooled_event(plan);
	if (!t.start || !t.stop) return set_error(IBK_ERR_CUDA, "cudaEventCreate failed");
	cudaEventRecord(t.start, stream);
	plan.pending.push_back(t);
	slot = (int) plan.pending.size() - 1;
	return IBK_OK;
}

ibk_status launch_end(Plan& plan, const char* name, cudaStream_t stream, int slot)
{
	ibk_status s = check_launch(name);
	plan.launches++;
	if (slot >= 0) {
		cudaEventRecord(plan.pending[slot].stop, stream);
		plan.stats[plan.pending[slot].stat].launches++;
	}
	return s;
}

} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_plan_create(const ibk_domain* domain, int tag, int refinement, ibk_delta delta,
                           int precision, ibk_plan* out)
{
	if (!domain || !out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null domain or output pointer");
	*out = nullptr;
	ibk_status cs = check_domain(domain, tag, refinement);
	if (cs != IBK_OK) return cs;
	const int dims = domain->dims;
	const OpTable* ops = find_ops(delta.kind, delta.order, dims, precision);
	if (!ops) return set_error(IBK_ERR_UNSUPPORTED, "delta / dims / precision combination not built");

	Plan* plan = new (std::nothrow) Plan();
	if (!plan) return set_error(IBK_ERR_OUT_OF_MEMORY, "host allocation failed");
	plan->ops = *ops;
	plan->delta_kind = delta.kind;
	plan->delta_order = delta.kind == kBspline ? delta.order : 0;
	plan->precision = precision;
	cudaGetDevice(&plan->device);
	cudaDeviceGetAttribute(&plan->num_sms, cudaDevAttrMultiProcessorCount, plan->device);

	ibk_status gs = make_geometry(domain, tag, refinement, meshwidths_of(delta.kind, plan->delta_order),
	                              plan->g, plan->info);
	if (gs != IBK_OK) { delete plan; return gs; }
	const GridGeom& g = plan->g;
	const ibk_grid_info& info = plan->info;
	// both operators on the default tiles (16^3 cells, smaller on small
	// grids), so one binning serves a spread and an interpolation
	plan->tiles = make_tiles(g, tag, info.meshwidths);
	plan->spread_tiles = plan->tiles;
	plan->tag = tag;
	for (int d = 0; d < dims; ++d)
		if (g.comp[0].cells[d] < info.meshwidths) plan->tiled = false;
	cudaError_t e = cudaMalloc(&plan->d_status, sizeof(int) * 4);
	if (e != cudaSuccess) { cudaGetLastError(); delete plan; return set_error(IBK_ERR_OUT_OF_MEMORY, "cudaMalloc failed"); }
	cudaMemset(plan->d_status, 0, sizeof(int) * 4);
	*out = reinterpret_cast<ibk_plan>(plan);
	return IBK_OK;
}

ibk_status ibk_plan_destroy(ibk_plan handle)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return IBK_OK;
	drain_pending(*plan);
	for (cudaEvent_t e : plan->event_pool) cudaEventDestroy(e);
	for (Scratch& s : plan->scratch)
		if (s.ptr) cudaFree(s.ptr);
	if (plan->d_status) cudaFree(plan->d_status);
	delete plan;
	return IBK_OK;
}

ibk_status ibk_plan_info(ibk_plan handle, ibk_grid_info* info)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || !info) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or info");
	*info = plan->info;
	return IBK_OK;
}

ibk_status ibk_plan_set_tiles(ibk_plan handle, const int* spread_tile, const int* interp_tile)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	const int M = plan->info.meshwidths, dims = plan->g.dims;
	TileGeom ts = plan->spread_tiles, ti = plan->tiles;
	// extents up to 64 cells: records keep tile-relative origins in 8 bits
	if (spread_tile) {
		for (int d = 0; d < dims; ++d)
			if (spread_tile[d] < M || spread_tile[d] > kMaxTileExtent)
				return set_error(IBK_ERR_INVALID_ARGUMENT, "spread tile extents must lie in [M, 64]");
		ts = make_tiles(plan->g, plan->tag, M, spread_tile);
		if (spread_tile_bytes(plan->g, ts, M, plan->precision) > 200 * 1024)
			return set_error(IBK_ERR_UNSUPPORTED, "spread tile needs more than 200 KB of shared memory");
	}
	if (interp_tile) {
		for (int d = 0; d < dims; ++d)
			if (interp_tile[d] < M || interp_tile[d] > kMaxTileExtent)
				return set_error(IBK_ERR_INVALID_ARGUMENT, "interpolation tile extents must lie in [M, 64]");
		ti = make_tiles(plan->g, plan->tag, M, interp_tile);
		if (interp_region_bytes(plan->g, ti, M) > 200 * 1024)
			return set_error(IBK_ERR_UNSUPPORTED, "interpolation tile needs more than 200 KB of shared memory");
	}
	plan->spread_tiles = ts;
	plan->tiles = ti;
	return IBK_OK;
}

ibk_status ibk_plan_reserve(ibk_plan handle, int max_points)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || max_points < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or negative size");
	plan->reserved_points = max_points;
	return IBK_OK;
}

ibk_status ibk_spread(ibk_plan handle, int n, const double* x, const double* fl,
                      double* const* fe, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	if (n <= 0) return IBK_OK;                          // novel.h:201
	if (!x || !fl || !fe) return set_error(IBK_ERR_INVALID_ARGUMENT, "null array");
	CompPtrs out{};
	for (int c = 0; c < plan->g.dims; ++c) {
		if (!fe[c]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null grid component");
		out.p[c] = fe[c];
	}
	OpArgs a{&plan->g, n, x, (cudaStream_t) stream};
	return plan->ops.spread(*plan, a, fl, out);
}

ibk_status ibk_interpolate(ibk_plan handle, int n, const double* x, const double* const* ue,
                           double* ul, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	if (n <= 0) return IBK_OK;                          // interpolate.h:96
	if (!x || !ue || !ul) return set_error(IBK_ERR_INVALID_ARGUMENT, "null array");
	ConstCompPtrs in{};
	for (int c = 0; c < plan->g.dims; ++c) {
		if (!ue[c]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null grid component");
		in.p[c] = ue[c];
	}
	OpArgs a{&plan->g, n, x, (cudaStream_t) stream};
	return plan->ops.interp(*plan, a, in, ul);
}

ibk_status ibk_spread_interpolate(ibk_plan handle, int n, const double* x, const double* fl,
                                  double* const* fe, const double* const* ue, double* ul, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	if (n <= 0) return IBK_OK;                          // novel.h:201, interpolate.h:96
	if (!x || !fl || !fe || !ue || !ul) return set_error(IBK_ERR_INVALID_ARGUMENT, "null array");
	CompPtrs out{};
	ConstCompPtrs in{};
	for (int c = 0; c < plan->g.dims; ++c) {
		if (!fe[c] || !ue[c]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null grid component");
		out.p[c] = fe[c];
		in.p[c] = ue[c];
	}
	OpArgs a{&plan->g, n, x, (cudaStream_t) stream};
	return plan->ops.both(*plan, a, fl, out, in, ul);
}

ibk_status ibk_sort_keys(ibk_plan handle, int component, int n, const double* x, int* keys, void* stream)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	if (component < 0 || component >= plan->g.dims) return set_error(IBK_ERR_INVALID_ARGUMENT, "component out of range");
	if (n <= 0) return IBK_OK;
	if (!x || !keys) return set_error(IBK_ERR_INVALID_ARGUMENT, "null array");
	OpArgs a{&plan->g, n, x, (cudaStream_t) stream};
	return plan->ops.keys(*plan, a, component, keys);
}

ibk_status ibk_plan_set_profiling(ibk_plan handle, int enable)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	plan->profiling = enable != 0;
	return IBK_OK;
}

ibk_status ibk_plan_kernel_stats(ibk_plan handle, ibk_kernel_stat* out, int capacity, int* count)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || !count || (capacity > 0 && !out)) return set_error(IBK_ERR_INVALID_ARGUMENT, "null argument");
	ibk_status s = drain_pending(*plan);
	if (s != IBK_OK) return s;
	*count = (int) plan->stats.size();
	for (int i = 0; i < capacity && i < (int) plan->stats.size(); ++i) out[i] = plan->stats[i];
	return IBK_OK;
}

ibk_status ibk_plan_reset_stats(ibk_plan handle)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	ibk_status s = drain_pending(*plan);
	plan->stats.clear();
	return s;
}

ibk_status ibk_plan_launch_count(ibk_plan handle, long long* launches)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan || !launches) return set_error(IBK_ERR_INVALID_ARGUMENT, "null argument");
	*launches = plan->launches;
	return IBK_OK;
}

ibk_status ibk_plan_check(ibk_plan handle)
{
	Plan* plan = reinterpret_cast<Plan*>(handle);
	if (!plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan");
	int st[4] = {0, 0, 0, 0};
	cudaError_t e = cudaMemcpy(st, plan->d_status, sizeof(st), cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
	if (st[0] == 0) return IBK_OK;
	cudaMemset(plan->d_status, 0, sizeof(st));
	return set_error(IBK_ERR_DEVICE_CHECK, st[0] == 1 ? "a bounded device wait timed out" :
	                 "a TMA precondition failed on the device (staged by plain loads instead)");
}

const char* ibk_last_error(void) { return g_last_error.c_str(); }

const char* ibk_status_string(ibk_status s)
{
	switch (s) {
	case IBK_OK: return "ok";
	case IBK_ERR_INVALID_ARGUMENT: return "invalid argument";
	case IBK_ERR_UNSUPPORTED: return "unsupported configuration";
	case IBK_ERR_OUT_OF_MEMORY: return "out of device memory";
	case IBK_ERR_CUDA: return "CUDA error";
	case IBK_ERR_CAPACITY: return "scratch capacity exceeded during capture";
	case IBK_ERR_DEVICE_CHECK: return "device-side check failed";
	}
	return "unknown status";
}

int ibk_version(void) { return IBK_VERSION; }

} // extern "C"
