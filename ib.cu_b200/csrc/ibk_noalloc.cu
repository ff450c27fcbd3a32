// ibk_interpolate_noalloc: interpolation for callers that must not allocate
// device memory.
//
// The regular entry points keep their scratch (bin counts and offsets, the
// point records in bin order) in buffers that the plan grows with
// cudaMalloc on first use.  Some callers cannot allow that: code that runs
// while another component owns the device's memory pool, real-time loops
// where a cudaMalloc (which synchronises the device) would stall the step,
// or hosts that never hold a plan at all.  This entry point takes the grid
// description directly, allocates nothing, and keeps its scratch in one
// file-scope __device__ array of fixed size (kNoallocBytes, about 22 MB),
// which every GPU that loads this library holds until the process exits.
//
// Limits: at most kNoallocMaxPoints points and kNoallocMaxBins bins
// (tiles x 3^dims reach classes) per call; larger calls return
// IBK_ERR_CAPACITY.  Every call shares the one array: two calls whose
// kernels overlap on the GPU (different streams, or host threads) race and
// corrupt each other's results.  The first call in each CUDA context looks
// up the array's device address (cudaGetSymbolAddress); make that first
// call before any stream capture.
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
constexpr size_t kOffRecs = kOffKeyRank + align256(sizeof(int2) * kNoallocMaxPoints);
constexpr size_t kNoallocBytes = kOffRecs + align256(sizeof(PointRec) * kNoallocMaxPoints);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// cuCtxGetCurrent through the runtime's driver entry point (no link
// dependency on libcuda).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);

CtxGetCurrentFn ctx_get_current()
{
	static CtxGetCurrentFn fn = [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
		    q != cudaDriverEntryPointSuccess) {
			cudaGetLastError();
			return (CtxGetCurrentFn) nullptr;
		}
		return reinterpret_cast<CtxGetCurrentFn>(p);
	}();
	return fn;
}

// The array's device address is looked up per device and cached together
// with the context it was looked up in: a new primary context (after
// cudaDeviceReset, for instance) loads the module again and the array may
// move, so a changed context triggers a new lookup.
constexpr int kMaxDevices = 64;
std::mutex g_addr_lock;
struct AddrCache {
	CUcontext ctx = nullptr;
	unsigned char* addr = nullptr;
};
AddrCache g_addr[kMaxDevices];

ibk_status scratch_address(unsigned char** out)
{
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
	if (dev < 0 || dev >= kMaxDevices) return set_error(IBK_ERR_UNSUPPORTED, "device ordinal beyond 63");
	CtxGetCurrentFn get = ctx_get_current();
	CUcontext ctx = nullptr;
	if (get && get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
	std::lock_guard<std::mutex> lock(g_addr_lock);
	AddrCache& c = g_addr[dev];
	if (!c.addr || !ctx || c.ctx != ctx) {
		void* p = nullptr;
		e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess)
			return set_error(IBK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		// the lookup made the device's context current if none was
		if (get && get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
		c.addr = static_cast<unsigned char*>(p);
		c.ctx = ctx;
	}
	*out = c.addr;
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
	PointRec* recs = reinterpret_cast<PointRec*>(base + kOffRecs);
	// the array keeps the previous call's contents: clear what must start at 0
	// (the bin counts; everything else is written before it is read)
	cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * (size_t) tg.num_bins, stream);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
	const int nb = (n + 255) / 256;
	const int nchunks = (tg.num_bins + kScanChunk - 1) / kScanChunk;
	const BinStats no_stats{nullptr, g.res, nullptr};   // interpolation: no force statistics
	bin_count_kernel<M, DIMS><<<nb, 256, 0, stream>>>(g, tg, n, x, count, kr, no_stats);
	if ((s = check_launch("bin_count_kernel")) != IBK_OK) return s;
	bin_chunk_sum_kernel<<<nchunks, kScanThreads, 0, stream>>>(count, chunk, tg.num_bins);
	if ((s = check_launch("bin_chunk_sum_kernel")) != IBK_OK) return s;
	bin_scan_kernel<<<nchunks, kScanThreads, 0, stream>>>(count, chunk, off, tg.num_bins, nchunks);
	if ((s = check_launch("bin_scan_kernel")) != IBK_OK) return s;
	bin_scatter_kernel<M, DIMS><<<nb, 256, 0, stream>>>(g, tg, n, x, kr, off, recs);
	if ((s = check_launch("bin_scatter_kernel")) != IBK_OK) return s;
	const size_t smem = interp_smem_bytes<M>(g, tg);
	auto kern = interp_tile_kernel<D, DIMS, PREC>;
	e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	// regions are staged with plain loads here (use_tma = 0), so the kernel
	// has no device-side check to report and gets no status word
	TmaMaps maps{};
	kern<<<dim3(tg.num_tiles, DIMS), kTileThreads, smem, stream>>>(g, tg, n, x, recs, off, ue, ul, maps, 0, nullptr);
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
	// the plan's own validation and geometry (no second copy of the
	// bit-exact grid code), into caller-stack structures
	ibk_status s = check_domain(domain, tag, refinement);
	if (s != IBK_OK) return s;
	GridGeom g;
	ibk_grid_info info;
	s = make_geometry(domain, tag, refinement, meshwidths_of(delta.kind, order), g, info);
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
