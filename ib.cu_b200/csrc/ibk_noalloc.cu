// ibk_interpolate_noalloc: interpolation for callers that must not allocate
// device memory.
//
// The regular entry points keep their scratch (point bins, offsets, the
// point permutation) in buffers that the plan grows with cudaMalloc on
// first use.  Some callers cannot allow that: code that runs while another
// component owns the device's memory pool, real-time loops where a
// cudaMalloc (which synchronises the device) would stall the step, or hosts
// that never hold a plan at all.  This entry point takes the grid
// description directly, allocates nothing, and keeps its scratch in one
// file-scope __device__ array of fixed size (kNoallocBytes, about 8 MB),
// which every GPU that loads this library holds until the process exits.
//
// Limits: at most kNoallocMaxPoints points and kNoallocMaxBins bins
// (tiles x 3^dims reach classes) per call; larger calls return
// IBK_ERR_CAPACITY.  Every call shares the one array: two calls whose
// kernels overlap on the GPU (different streams, or host threads) race and
// corrupt each other's results.  The first call on each device looks up
// the array's device address (cudaGetSymbolAddress); make that first call
// before any stream capture.
#include <cfloat>
#include <cstdint>
#include <mutex>
#include <string>
#include "ibk_internal.h"
#include "ibk_direct.cuh"
#include "ibk_tiled.cuh"

namespace ibk {
namespace {

constexpr int kNoallocMaxPoints = 1 << 19;      // 524,288 points per call
constexpr int kNoallocMaxBins = 1 << 18;        // 262,144 bins per call
constexpr int kNoallocMaxChunks = kNoallocMaxBins / kScanChunk + 2;

// Byte layout of the scratch array (every region 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffCount = 0;
constexpr size_t kOffOffset = kOffCount + align256(sizeof(int) * kNoallocMaxBins);
constexpr size_t kOffChunk = kOffOffset + align256(sizeof(int) * (kNoallocMaxBins + 1));
constexpr size_t kOffKeyRank = kOffChunk + align256(sizeof(int) * kNoallocMaxChunks);
constexpr size_t kOffPerm = kOffKeyRank + align256(sizeof(int2) * kNoallocMaxPoints);
constexpr size_t kOffStatus = kOffPerm + align256(sizeof(int) * kNoallocMaxPoints);
constexpr size_t kNoallocBytes = kOffStatus + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_lock;
unsigned char* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device.
ibk_status scratch_address(unsigned char** out)
{
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
	if (dev < 0 || dev >= kMaxDevices) return set_error(IBK_ERR_UNSUPPORTED, "device ordinal beyond 63");
	std::lock_guard<std::mutex> lock(g_addr_lock);
	if (!g_addr[dev]) {
		void* p = nullptr;
		e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess)
			return set_error(IBK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		g_addr[dev] = static_cast<unsigned char*>(p);
	}
	*out = g_addr[dev];
	return IBK_OK;
}

// Host geometry of fd::grid / fd::discretization, as ibk_plan_create
// computes it (include/fd/grid.h:232-239, include/fd/discretization.h:113-164,
// include/algo/gcd.h:7-34), into a caller-stack GridGeom.
double h_floor(double x) { return (double) (long) (x - (double) (x < 0 && (-x != (double) (long) -x))); }
double h_modulo(double x, double s) { return x - s * h_floor(x / s); }
double h_abs(double x) { return (double) ((x > 0) - (x < 0)) * x; }
double h_gcd(double a, double b)
{
	if (a < b) { double t = a; a = b; b = t; }
	double u = 1.0, v = b / a, eps = DBL_EPSILON;
	while (h_abs(v) > eps) {
		if (u < v) { double t = u; u = v; v = t; }
		double c = u - h_floor(u / v) * v;
		u = v; v = c;
		eps *= 2;
	}
	return u * a;
}

ibk_status geometry(const ibk_domain* domain, int tag, int refinement, int M, GridGeom& g)
{
	const int dims = domain->dims;
	if (dims < 2 || dims > 3) return set_error(IBK_ERR_UNSUPPORTED, "dims must be 2 or 3");
	if (refinement <= 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "refinement must be positive");
	if (tag != IBK_TAG_MAC && tag != IBK_TAG_CENTERED) return set_error(IBK_ERR_INVALID_ARGUMENT, "unknown grid tag");
	for (int d = 0; d < dims; ++d)
		if (!(domain->length[d] > 0) || !(domain->length[d] < 1e300))
			return set_error(IBK_ERR_INVALID_ARGUMENT, "dimension lengths must be positive and finite");
	g = GridGeom{};
	g.dims = dims;
	double unit = domain->length[0];
	for (int d = 1; d < dims; ++d) unit = h_gcd(unit, domain->length[d]);
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
	for (int c = 0; c < dims; ++c) {
		CompGeom& cg = g.comp[c];
		long long size = 1;
		for (int d = 0; d < dims; ++d) {
			double al = (tag == IBK_TAG_MAC && c == d) ? h_modulo(0.5 + 0.5, 1.0) : 0.5;
			al = h_modulo(al, 1.0);
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
			size *= points;
		}
		if (size >= (1LL << 31)) return set_error(IBK_ERR_INVALID_ARGUMENT, "component grid exceeds 2^31 faces");
		cg.size = size;
	}
	(void) M;
	return IBK_OK;
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status run(const GridGeom& g, int tag, int n, const double* x, ConstCompPtrs ue, double* ul,
               cudaStream_t stream)
{
	using D = Delta<KIND, ORDER>;
	constexpr int M = D::M;
	bool tiled = true;
	for (int d = 0; d < DIMS; ++d) if (g.comp[0].cells[d] < M) tiled = false;
	if (!tiled) {
		// degenerate grid: the per-point kernel needs no scratch
		interp_direct_kernel<D, DIMS><<<(n + 127) / 128, 128, 0, stream>>>(g, n, x, ue, ul);
		return check_launch("interp_direct_kernel");
	}
	const TileGeom tg = make_tiles(g, tag, M);
	if (n > kNoallocMaxPoints)
		return set_error(IBK_ERR_CAPACITY, "ibk_interpolate_noalloc: more than 524288 points");
	if (tg.num_bins > kNoallocMaxBins)
		return set_error(IBK_ERR_CAPACITY, "ibk_interpolate_noalloc: grid needs more than 262144 bins");
	unsigned char* base = nullptr;
	ibk_status s = scratch_address(&base);
	if (s != IBK_OK) return s;
	int* count = reinterpret_cast<int*>(base + kOffCount);
	int* off = reinterpret_cast<int*>(base + kOffOffset);
	int* chunk = reinterpret_cast<int*>(base + kOffChunk);
	int2* kr = reinterpret_cast<int2*>(base + kOffKeyRank);
	int* perm = reinterpret_cast<int*>(base + kOffPerm);
	int* status = reinterpret_cast<int*>(base + kOffStatus);
	// the array keeps the previous call's contents: clear what must start at 0
	cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * (size_t) tg.num_bins, stream);
	if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, 256, stream);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
	const int nb = (n + 255) / 256;
	const int nchunks = (tg.num_bins + kScanChunk - 1) / kScanChunk;
	bin_count_kernel<M, DIMS><<<nb, 256, 0, stream>>>(g, tg, n, x, count, kr, nullptr, nullptr);
	if ((s = check_launch("bin_count_kernel")) != IBK_OK) return s;
	bin_chunk_sum_kernel<<<nchunks, kScanThreads, 0, stream>>>(count, chunk, tg.num_bins);
	if ((s = check_launch("bin_chunk_sum_kernel")) != IBK_OK) return s;
	bin_scan_kernel<<<nchunks, kScanThreads, 0, stream>>>(count, chunk, off, tg.num_bins, nchunks);
	if ((s = check_launch("bin_scan_kernel")) != IBK_OK) return s;
	bin_scatter_kernel<<<nb, 256, 0, stream>>>(n, kr, off, perm);
	if ((s = check_launch("bin_scatter_kernel")) != IBK_OK) return s;
	size_t ev = 1;
	for (int d = 0; d < DIMS; ++d) ev *= (size_t) region_extent<M>(tg.T[d], d);
	const size_t smem = sizeof(double) * ev + 128;
	auto kern = interp_tile_kernel<D, DIMS, PREC>;
	e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	TmaMaps maps{};   // regions are staged with plain loads here (use_tma = 0)
	kern<<<dim3(tg.num_tiles, DIMS), kTileThreads, smem, stream>>>(g, tg, n, x, perm, off, ue, ul, maps, 0, status);
	return check_launch("interp_tile_kernel");
}

using RunFn = ibk_status (*)(const GridGeom&, int, int, const double*, ConstCompPtrs, double*, cudaStream_t);
struct RunEntry { int kind, order, dims, prec; RunFn fn; };

#define IBK_NA(K, O, DIM, PR) RunEntry{K, O, DIM, PR, &run<K, O, DIM, PR>}
#define IBK_NA_DELTAS(DIM, PR)                                                  \
	IBK_NA(kBspline, 1, DIM, PR), IBK_NA(kBspline, 2, DIM, PR),                  \
	IBK_NA(kBspline, 3, DIM, PR), IBK_NA(kBspline, 4, DIM, PR),                  \
	IBK_NA(kBspline, 5, DIM, PR), IBK_NA(kPeskin, 0, DIM, PR),                   \
	IBK_NA(kRoma, 0, DIM, PR), IBK_NA(kCosine, 0, DIM, PR), IBK_NA(kHat, 0, DIM, PR)

const RunEntry kRuns[] = {
	IBK_NA_DELTAS(2, IBK_PRECISION_FP64), IBK_NA_DELTAS(3, IBK_PRECISION_FP64),
	IBK_NA_DELTAS(2, IBK_PRECISION_FP32C), IBK_NA_DELTAS(3, IBK_PRECISION_FP32C),
};

int meshwidths(int kind, int order)
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

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" ibk_status ibk_interpolate_noalloc(const ibk_domain* domain, int tag, int refinement,
                                              ibk_delta delta, int precision, int n, const double* x,
                                              const double* const* ue, double* ul, void* stream)
{
	if (!domain) return set_error(IBK_ERR_INVALID_ARGUMENT, "null domain");
	const int order = delta.kind == kBspline ? delta.order : 0;
	RunFn fn = nullptr;
	for (const RunEntry& r : kRuns)
		if (r.kind == delta.kind && r.order == order && r.dims == domain->dims && r.prec == precision) fn = r.fn;
	if (!fn) return set_error(IBK_ERR_UNSUPPORTED, "delta / dims / precision combination not built");
	GridGeom g;
	ibk_status s = geometry(domain, tag, refinement, meshwidths(delta.kind, order), g);
	if (s != IBK_OK) return s;
	if (n <= 0) return IBK_OK;                       // interpolate.h:96
	if (!x || !ue || !ul) return set_error(IBK_ERR_INVALID_ARGUMENT, "null array");
	ConstCompPtrs in{};
	for (int c = 0; c < domain->dims; ++c) {
		if (!ue[c]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null grid component");
		in.p[c] = ue[c];
	}
	return fn(g, tag, n, x, in, ul, (cudaStream_t) stream);
}
