// Batches: spread / interpolate / coupled step over many independent grids,
// one persistent kernel per operator.
//
// The reference builds one operator object per grid and runs its kernels
// grid by grid (include/ib/novel.h:197-227, include/ib/interpolate.h:92-115).
// Here every instance of a batch is binned into one global bin space
// (instance i owns bins [bin_base_i, bin_base_i + tiles_i * 3^dims)), the
// points of all instances are numbered consecutively (their records carry
// that number), and the tile kernels' bodies (spread_tile / interp_tile) run
// inside persistent CTAs that take work items from a device counter: FP32C
// spread items are (instance, tile), every component at once; FP64 spread
// and interpolation items are (instance, tile, component).  The work
// list is that of the instances bound with points: each bind uploads the
// list of active instances and the prefix sums of their item counts, and a
// CTA maps item k to (instance, tile, component) by a binary search.  Per
// item the CTA copies the instance's geometry and bound arrays into shared
// memory.  Nothing here waits on another CTA: a CTA only takes items until
// the list is exhausted.
//
// All device memory is allocated at create / configure time; a run launches
// a fixed sequence (a memset, four binning kernels and one persistent kernel
// per operator) whose grids depend only on the batch's capacity and
// configuration (the binning kernels stride over the bound points, the
// count kernel in per-instance chunks whose number the bound table holds),
// so it can be captured once as a CUDA graph and replayed with new bindings.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "ibk_internal.h"
#include "ibk_tiled.cuh"

namespace ibk {

// Static description of one instance (per configuration).
struct BatchInst {
	GridGeom g;
	TileGeom ts;            // spread tiles
	TileGeom ti;            // interpolation tiles
	int bin_s, bin_i;       // first bin of the instance in each bin space
};

// Bound arrays of one instance (per bind).
struct BatchIO {
	int n, pbase;           // points; index of the first point in the batch numbering
	const double* x;
	const double* fl;
	CompPtrs fe;            // kernels pass the shared copy by reference, so the
	ConstCompPtrs ue;       // component index never addresses a local array
	double* ul;
	double* xn;
	const double* xref;
	double* fs;
};

// Per-bind header of the device table.
struct BatchHeader {
	int total_points;       // bound points of all instances
	int num_active;         // instances bound with points
	int items_s, items_i;   // work items of the active instances
	int chunks;             // binning chunks (kBinThreads points of one instance)
};

// Device views of the bound table (all in one allocation).
struct BatchTable {
	const BatchHeader* hdr;
	const BatchIO* io;      // [count]
	const int* active;      // [num_active]: instances bound with points
	const int* spre;        // [num_active + 1]: prefix of their spread items
	const int* ipre;        // [num_active + 1]: prefix of their interpolation items
	const int* cpre;        // [num_active + 1]: prefix of their binning chunks
	const CUtensorMap* maps; // [count * 3]: velocity grids of the active instances
	const int* use_tma;     // [count]: 1 when the maps are valid for TMA staging
	int count;
};

namespace {

constexpr int kBinThreads = 256;
constexpr int kRing = 4;

// The last i in [0, count) with pre[i] <= k: the active instance holding
// work item k (pre = spre or ipre) or binning chunk k (pre = cpre).
__device__ __forceinline__ int find_instance(const int* __restrict__ pre, int count, int k)
{
	int lo = 0, hi = count - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (__ldg(pre + mid) <= k) lo = mid;
		else hi = mid - 1;
	}
	return lo;
}

// Copy a trivially copyable descriptor into shared memory, 4 bytes per thread.
template <typename T>
__device__ __forceinline__ void copy_to_shared(T* dst, const T* src)
{
	static_assert(sizeof(T) % 4 == 0, "descriptor size");
	const int* s = reinterpret_cast<const int*>(src);
	int* d = reinterpret_cast<int*>(dst);
	for (int i = threadIdx.x; i < (int) (sizeof(T) / 4); i += blockDim.x) d[i] = __ldg(s + i);
}

// Binning of every bound point of the batch.  The points of each active
// instance are cut into chunks of kBinThreads (cpre: prefix of the chunk
// counts) and each block iteration bins one chunk, so the instance is found
// by one search per chunk and its geometry read from a shared-memory copy.
// spread: bin by the spread tiles (else the interpolation tiles); moved:
// positions xn (else x); forces: 1 = fl, 2 = fs (the bins' force
// statistics for the FP32C scale, see BinStats), 0 = none.
template <int DIMS>
__device__ __forceinline__ void instance_forces(const BatchInst& si, const BatchIO& so, int forces, int p, float* a)
{
	const double* f = forces == 1 ? so.fl : so.fs;
#pragma unroll
	for (int c = 0; c < DIMS; ++c) a[c] = fabsf((float) (si.g.res * __ldg(f + (size_t) c * so.n + p)));
}

template <int M, int DIMS>
__global__ void __launch_bounds__(kBinThreads)
batch_bin_count_kernel(const BatchInst* __restrict__ insts, BatchTable t, int spread, int moved, int forces,
                       int* __restrict__ counts, int2* __restrict__ key_rank, unsigned* __restrict__ binmax)
{
	__shared__ int cur_inst, cur_chunk;
	__shared__ BatchInst si;
	__shared__ BatchIO so;
	const int nchunks = __ldg(&t.hdr->chunks), nact = __ldg(&t.hdr->num_active);
	for (int k = blockIdx.x; k < nchunks; k += gridDim.x) {
		if (threadIdx.x == 0) {
			const int j = find_instance(t.cpre, nact, k);
			cur_inst = __ldg(t.active + j);
			cur_chunk = k - __ldg(t.cpre + j);
		}
		__syncthreads();
		copy_to_shared(&si, insts + cur_inst);
		copy_to_shared(&so, t.io + cur_inst);
		__syncthreads();
		const int n = so.n;
		const int p = cur_chunk * kBinThreads + threadIdx.x;
		const bool active = p < n;
		int key = 0;
		float a[kMaxDims] = {0.0f, 0.0f, 0.0f};
		if (active) {
			// forces is uniform, and a bound instance with points has its force array
			if (forces) instance_forces<DIMS>(si, so, forces, p, a);
			const double* x = moved ? so.xn : so.x;
			key = spread ? si.bin_s + point_bin<M, DIMS>(si.g, si.ts, x, n, p, nullptr)
			             : si.bin_i + point_bin<M, DIMS>(si.g, si.ti, x, n, p, nullptr);
		}
		const unsigned mask = __ballot_sync(0xffffffffu, active);
		if (active) bin_rank<DIMS>(mask, key, counts, key_rank + so.pbase + p, forces ? a : nullptr, binmax);
		__syncthreads();            // the next chunk overwrites the shared copies
	}
}

// Records of every bound point at their sorted positions, by the same
// chunks as the count kernel.
template <int M, int DIMS>
__global__ void __launch_bounds__(kBinThreads)
batch_bin_scatter_kernel(const BatchInst* __restrict__ insts, BatchTable t, int spread, int moved,
                         const int2* __restrict__ key_rank, const int* __restrict__ offset,
                         PointRec* __restrict__ recs)
{
	__shared__ int cur_inst, cur_chunk;
	__shared__ BatchInst si;
	__shared__ BatchIO so;
	const int nchunks = __ldg(&t.hdr->chunks), nact = __ldg(&t.hdr->num_active);
	for (int k = blockIdx.x; k < nchunks; k += gridDim.x) {
		if (threadIdx.x == 0) {
			const int j = find_instance(t.cpre, nact, k);
			cur_inst = __ldg(t.active + j);
			cur_chunk = k - __ldg(t.cpre + j);
		}
		__syncthreads();
		copy_to_shared(&si, insts + cur_inst);
		copy_to_shared(&so, t.io + cur_inst);
		__syncthreads();
		const int p = cur_chunk * kBinThreads + threadIdx.x;
		if (p < so.n) {
			const int gp = so.pbase + p;
			const int2 kr = __ldg(key_rank + gp);
			PointRec r;
			point_bin<M, DIMS>(si.g, spread ? si.ts : si.ti, moved ? so.xn : so.x, so.n, p, &r);
			r.p = gp;
			store_rec(recs + __ldg(offset + kr.x) + kr.y, r);
		}
		__syncthreads();            // the next chunk overwrites the shared copies
	}
}

// Thread 0 takes the next work item of the active instances: instance and
// item index within it, or instance -1 when the list is exhausted.
__device__ __forceinline__ void next_item(int* next, int nitems, int nact, const int* __restrict__ pre,
                                          const int* __restrict__ active, int* inst, int* local, int* item = nullptr)
{
	const int k = atomicAdd(next, 1);
	if (item) *item = k;
	if (k >= nitems) { *inst = -1; *local = 0; return; }
	const int j = find_instance(pre, nact, k);
	*inst = __ldg(active + j);
	*local = k - __ldg(pre + j);
}

// Persistent spread over the active instances' items: tiles (FP32C, every
// component) or (tile, component) (FP64).
template <typename D, int DIMS, int PREC, int NT = kTileThreads>
__global__ void __launch_bounds__(NT, PREC == IBK_PRECISION_FP32C ? 1024 / NT : 3)
batch_spread_kernel(const BatchInst* __restrict__ insts, BatchTable t, int* __restrict__ next,
                    const PointRec* __restrict__ recs, const int* __restrict__ off, const unsigned* __restrict__ binmax,
                    int step, Deferral defer)
{
	__shared__ int cur_inst, cur_local, cur_item;
	__shared__ BatchInst si;
	__shared__ BatchIO so;
	const int nitems = __ldg(&t.hdr->items_s), nact = __ldg(&t.hdr->num_active);
	for (;;) {
		if (threadIdx.x == 0) next_item(next, nitems, nact, t.spre, t.active, &cur_inst, &cur_local, &cur_item);
		__syncthreads();
		const int inst = cur_inst, local = cur_local, item = cur_item;
		if (inst < 0) return;
		copy_to_shared(&si, insts + inst);
		copy_to_shared(&so, t.io + inst);
		__syncthreads();
		const CompPtrs& fe = so.fe;
		if constexpr (PREC == IBK_PRECISION_FP32C) {
			const BinStatsView bs{binmax + (size_t) si.bin_s * kMaxDims};
			// a dense tile is deferred by its work-item index
			spread_tile<D, DIMS, PREC, false, NT>(si.g, si.ts, so.n, step ? so.xn : so.x, step ? so.fs : so.fl, recs,
			                                      so.pbase, off + si.bin_s, bs, fe, local, -1, defer, item);
		} else {
			spread_tile<D, DIMS, PREC>(si.g, si.ts, so.n, step ? so.xn : so.x, step ? so.fs : so.fl, recs, so.pbase,
			                           off + si.bin_s, BinStatsView{nullptr}, fe, local / DIMS, local % DIMS);
		}
		__syncthreads();
	}
}

// The deferred dense tiles of an FP32C batch spread (see Deferral): work
// items in the deferral list, folded.
template <typename D, int DIMS>
__global__ void __launch_bounds__(kTileThreads, 4)
batch_spread_dense_kernel(const BatchInst* __restrict__ insts, BatchTable t, const PointRec* __restrict__ recs,
                          const int* __restrict__ off, const unsigned* __restrict__ binmax, int step,
                          const int* __restrict__ list, const int* __restrict__ count)
{
	__shared__ BatchInst si;
	__shared__ BatchIO so;
	__shared__ int cur_inst, cur_local;
	const int m = *count, nact = __ldg(&t.hdr->num_active);
	for (int q = blockIdx.x; q < m; q += gridDim.x) {
		__shared__ int cur_comp;
		if (threadIdx.x == 0) {
			const int v = __ldg(list + q);
			const int k = v >> 2;
			const int j = find_instance(t.spre, nact, k);
			cur_inst = __ldg(t.active + j);
			cur_local = k - __ldg(t.spre + j);
			cur_comp = v & 3;
		}
		__syncthreads();
		copy_to_shared(&si, insts + cur_inst);
		copy_to_shared(&so, t.io + cur_inst);
		__syncthreads();
		const CompPtrs& fe = so.fe;
		const BinStatsView bs{binmax + (size_t) si.bin_s * kMaxDims};
		spread_tile<D, DIMS, IBK_PRECISION_FP32C, true>(si.g, si.ts, so.n, step ? so.xn : so.x, step ? so.fs : so.fl,
		                                                recs, so.pbase, off + si.bin_s, bs, fe, cur_local, cur_comp);
		__syncthreads();
	}
}

// Persistent interpolation over the active instances' (tile, component)
// items (each tile's region staged by one TMA copy where the instance's grids
// allow it, else by plain loads); with step set, the serving epilogue
// (advection + spring force) is applied.
template <typename D, int DIMS, int PREC>
__global__ void __launch_bounds__(kTileThreads, D::M <= 4 ? 3 : 1)
batch_interp_kernel(const BatchInst* __restrict__ insts, BatchTable t, int* __restrict__ next,
                    const PointRec* __restrict__ recs, const int* __restrict__ off, int step, double dt, double k,
                    int* status)
{
	__shared__ int cur_inst, cur_local;
	__shared__ BatchInst si;
	__shared__ BatchIO so;
	__shared__ StepEpilogue epi;
	const int nitems = __ldg(&t.hdr->items_i), nact = __ldg(&t.hdr->num_active);
	for (;;) {
		if (threadIdx.x == 0) next_item(next, nitems, nact, t.ipre, t.active, &cur_inst, &cur_local);
		__syncthreads();
		const int inst = cur_inst, local = cur_local;
		if (inst < 0) return;
		copy_to_shared(&si, insts + inst);
		copy_to_shared(&so, t.io + inst);
		__syncthreads();
		if (step && threadIdx.x == 0) epi = StepEpilogue{so.xn, so.fs, so.xref, dt, k};
		__syncthreads();
		const ConstCompPtrs& ue = so.ue;
		const bool ok = interp_tile<D, DIMS, PREC>(si.g, si.ti, so.n, so.x, recs, so.pbase, off + si.bin_i, ue,
		                                           so.ul, t.maps + (size_t) inst * kMaxDims,
		                                           __ldg(t.use_tma + inst), true, status,
		                                           step ? &epi : nullptr, local / DIMS, local % DIMS);
		if (!ok) return;            // a staging copy never completed: stop this CTA
		__syncthreads();
	}
}

} // namespace

struct Batch;
using BatchRunFn = ibk_status (*)(Batch&, int op, cudaStream_t);
using BatchPrepFn = ibk_status (*)(Batch&);

struct BatchOps {
	BatchRunFn run;
	BatchPrepFn prepare;     // kernel attributes and persistent grid sizes
};

struct Batch {
	int device = 0, dims = 3, count = 0, M = 4, precision = 0;
	int delta_kind = 0, delta_order = 0;
	const BatchOps* ops = nullptr;
	std::vector<GridGeom> geo;
	std::vector<ibk_grid_info> info;
	std::vector<int> tag;
	ibk_batch_config config{};
	// configuration-derived
	std::vector<BatchInst> inst_h;
	int bins_s = 0, bins_i = 0;
	std::vector<int> nitem_s, nitem_i;  // work items per instance
	long long items_s = 0, items_i = 0; // of all instances
	size_t smem_s = 0, smem_i = 0;
	int grid_s = 0, grid_i = 0, grid_bin = 1;
	BatchInst* d_inst = nullptr;
	size_t bins_cap = 0;
	// bindings
	int capacity = 0;
	std::vector<BatchIO> io_h;
	unsigned char* d_table = nullptr; // header, io, active, spre, ipre, cpre
	size_t table_bytes = 0, off_io = 0, off_active = 0, off_spre = 0, off_ipre = 0, off_cpre = 0;
	size_t off_maps = 0, off_tma = 0;
	// tensor maps of the velocity grids, encoded on the host per instance and
	// component, reused while the bound pointer and the tile shape stay
	std::vector<CUtensorMap> map_cache;
	std::vector<const double*> map_ptr;     // grid the cached map describes
	std::vector<char> map_ok;
	unsigned char* h_ring[kRing] = {};
	cudaEvent_t ring_ev[kRing] = {};
	int ring_next = 0;
	bool bound = false;
	// scratch
	int *d_counts = nullptr, *d_off = nullptr, *d_chunk = nullptr, *d_next = nullptr;
	int* d_status = nullptr;
	int2* d_kr = nullptr;
	PointRec* d_recs = nullptr;
	unsigned* d_binmax = nullptr;               // spread bins' force maxima (FP32C)
	int* d_defer = nullptr;                     // deferred dense spread items: count, then the list
	size_t defer_cap = 0;
	// step parameters and graphs
	double dt = 0.0, k = 0.0;
	cudaStream_t cap_stream = nullptr;
	cudaGraphExec_t exec[5] = {};
	long long launches = 0;
	long long graph_kernels[5] = {};    // kernels in each captured graph
	int num_sms = 0;
};

namespace {

ibk_status cuda_check(cudaError_t e, const char* what)
{
	if (e == cudaSuccess) return IBK_OK;
	cudaGetLastError();
	return set_error(e == cudaErrorMemoryAllocation ? IBK_ERR_OUT_OF_MEMORY : IBK_ERR_CUDA,
	                 std::string(what) + ": " + cudaGetErrorString(e));
}

void drop_graphs(Batch& b)
{
	for (cudaGraphExec_t& e : b.exec)
		if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

inline int blocks_for(long long n, int threads) { return (int) ((n + threads - 1) / threads); }

BatchTable table_view(const Batch& b)
{
	BatchTable t;
	t.hdr = reinterpret_cast<const BatchHeader*>(b.d_table);
	t.io = reinterpret_cast<const BatchIO*>(b.d_table + b.off_io);
	t.active = reinterpret_cast<const int*>(b.d_table + b.off_active);
	t.spre = reinterpret_cast<const int*>(b.d_table + b.off_spre);
	t.ipre = reinterpret_cast<const int*>(b.d_table + b.off_ipre);
	t.cpre = reinterpret_cast<const int*>(b.d_table + b.off_cpre);
	t.maps = reinterpret_cast<const CUtensorMap*>(b.d_table + b.off_maps);
	t.use_tma = reinterpret_cast<const int*>(b.d_table + b.off_tma);
	t.count = b.count;
	return t;
}

// Binning of the bound points by the spread (spread = 1) or interpolation
// tiles, then the scan and the records in bin order.
template <int M, int DIMS>
ibk_status batch_bin(Batch& b, cudaStream_t s, int spread, int moved, int forces)
{
	const BatchTable t = table_view(b);
	const int nbins = spread ? b.bins_s : b.bins_i;
	if (forces) {
		ibk_status st = cuda_check(cudaMemsetAsync(b.d_binmax, 0, sizeof(unsigned) * kMaxDims * (size_t) nbins, s),
		                           "cudaMemsetAsync");
		if (st != IBK_OK) return st;
	}
	batch_bin_count_kernel<M, DIMS><<<b.grid_bin, kBinThreads, 0, s>>>(b.d_inst, t, spread, moved, forces,
	                                                                    b.d_counts, b.d_kr, b.d_binmax);
	const int nchunks = (nbins + kScanChunk - 1) / kScanChunk;
	bin_chunk_sum_kernel<<<nchunks, kScanThreads, 0, s>>>(b.d_counts, b.d_chunk, nbins);
	bin_scan_kernel<<<nchunks, kScanThreads, 0, s>>>(b.d_counts, b.d_chunk, b.d_off, nbins, nchunks);
	batch_bin_scatter_kernel<M, DIMS><<<b.grid_bin, kBinThreads, 0, s>>>(b.d_inst, t, spread, moved, b.d_kr,
	                                                                      b.d_off, b.d_recs);
	b.launches += 4;
	return check_launch("batch binning");
}

bool same_tiles(const ibk_batch_config& c)
{
	return c.spread_tile[0] == c.interp_tile[0] && c.spread_tile[1] == c.interp_tile[1] &&
	       c.spread_tile[2] == c.interp_tile[2];
}

template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status batch_run_impl(Batch& b, int op, cudaStream_t s)
{
	using D = Delta<KIND, ORDER>;
	const BatchTable t = table_view(b);
	ibk_status st;
	if ((st = cuda_check(cudaMemsetAsync(b.d_next, 0, sizeof(int) * 2, s), "cudaMemsetAsync")) != IBK_OK) return st;
	const bool step = op == IBK_OP_STEP;
	const bool both = op == IBK_OP_SPREAD_INTERPOLATE;
	auto interp = [&]() -> ibk_status {
		batch_interp_kernel<D, DIMS, PREC><<<b.grid_i, kTileThreads, b.smem_i, s>>>(
			b.d_inst, t, b.d_next + 1, b.d_recs, b.d_off, step ? 1 : 0, b.dt, b.k, b.d_status);
		b.launches += 1;
		return check_launch("batch_interp_kernel");
	};
	auto spread = [&]() -> ibk_status {
		Deferral defer{b.d_defer + 4, b.d_defer};
		if (PREC == IBK_PRECISION_FP32C) {
			ibk_status ds = cuda_check(cudaMemsetAsync(b.d_defer, 0, sizeof(int), s), "cudaMemsetAsync");
			if (ds != IBK_OK) return ds;
		}
		if (PREC == IBK_PRECISION_FP32C && b.config.spread_threads == 512)
			batch_spread_kernel<D, DIMS, PREC, 512><<<b.grid_s, 512, b.smem_s, s>>>(
				b.d_inst, t, b.d_next, b.d_recs, b.d_off, b.d_binmax, step ? 1 : 0, defer);
		else
			batch_spread_kernel<D, DIMS, PREC><<<b.grid_s, kTileThreads, b.smem_s, s>>>(
				b.d_inst, t, b.d_next, b.d_recs, b.d_off, b.d_binmax, step ? 1 : 0, defer);
		b.launches += 1;
		if (PREC == IBK_PRECISION_FP32C) {
			batch_spread_dense_kernel<D, DIMS><<<b.grid_s, kTileThreads, b.smem_s, s>>>(
				b.d_inst, t, b.d_recs, b.d_off, b.d_binmax, step ? 1 : 0, defer.list, defer.count);
			b.launches += 1;
		}
		return check_launch("batch_spread_kernel");
	};
	// FP32C spreads take the bins' force statistics from the binning
	const int forces = PREC == IBK_PRECISION_FP32C ? (step ? 2 : 1) : 0;
	if (op == IBK_OP_INTERPOLATE || step) {
		if ((st = batch_bin<D::M, DIMS>(b, s, 0, 0, 0)) != IBK_OK) return st;
		if ((st = interp()) != IBK_OK) return st;
	}
	if (op == IBK_OP_SPREAD || step || both) {
		if ((st = batch_bin<D::M, DIMS>(b, s, 1, step ? 1 : 0, forces)) != IBK_OK) return st;
		if ((st = spread()) != IBK_OK) return st;
	}
	if (both) {
		// the spread's records serve the interpolation when the tiles agree
		if (!same_tiles(b.config) && (st = batch_bin<D::M, DIMS>(b, s, 0, 0, 0)) != IBK_OK) return st;
		if ((st = interp()) != IBK_OK) return st;
	}
	return IBK_OK;
}

// Kernel attributes and persistent grid sizes for the current configuration.
template <int KIND, int ORDER, int DIMS, int PREC>
ibk_status batch_prepare_impl(Batch& b)
{
	using D = Delta<KIND, ORDER>;
	const bool wide = PREC == IBK_PRECISION_FP32C && b.config.spread_threads == 512;
	auto ks = wide ? batch_spread_kernel<D, DIMS, PREC, 512> : batch_spread_kernel<D, DIMS, PREC>;
	const int nts = wide ? 512 : kTileThreads;
	auto ki = batch_interp_kernel<D, DIMS, PREC>;
	ibk_status st;
	if constexpr (PREC == IBK_PRECISION_FP32C) {
		if ((st = cuda_check(cudaFuncSetAttribute(batch_spread_dense_kernel<D, DIMS>,
		                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) b.smem_s),
		                     "cudaFuncSetAttribute")) != IBK_OK) return st;
	}
	if ((st = cuda_check(cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) b.smem_s),
	                     "cudaFuncSetAttribute")) != IBK_OK) return st;
	if ((st = cuda_check(cudaFuncSetAttribute(ki, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) b.smem_i),
	                     "cudaFuncSetAttribute")) != IBK_OK) return st;
	int occ_s = 0, occ_i = 0;
	if ((st = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, ks, nts, b.smem_s),
	                     "cudaOccupancyMaxActiveBlocksPerMultiprocessor")) != IBK_OK) return st;
	if ((st = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_i, ki, kTileThreads, b.smem_i),
	                     "cudaOccupancyMaxActiveBlocksPerMultiprocessor")) != IBK_OK) return st;
	if (occ_s < 1 || occ_i < 1) return set_error(IBK_ERR_UNSUPPORTED, "batch tiles need more shared memory than an SM has");
	if (b.config.spread_ctas_per_sm > 0) occ_s = std::min(occ_s, b.config.spread_ctas_per_sm);
	if (b.config.interp_ctas_per_sm > 0) occ_i = std::min(occ_i, b.config.interp_ctas_per_sm);
	b.grid_s = (int) std::max(1LL, std::min(b.items_s, (long long) occ_s * b.num_sms));
	b.grid_i = (int) std::max(1LL, std::min(b.items_i, (long long) occ_i * b.num_sms));
	b.grid_bin = std::max(1, std::min(blocks_for(b.capacity, kBinThreads), 8 * b.num_sms));
	return IBK_OK;
}

template <int KIND, int ORDER, int DIMS, int PREC>
constexpr BatchOps make_batch_ops()
{
	return BatchOps{&batch_run_impl<KIND, ORDER, DIMS, PREC>, &batch_prepare_impl<KIND, ORDER, DIMS, PREC>};
}

struct BatchEntry { int kind, order, dims, prec; BatchOps ops; };

#define IBK_BENTRY(K, O, DIM, PR) BatchEntry{K, O, DIM, PR, make_batch_ops<K, O, DIM, PR>()}
#define IBK_BATCH_ENTRIES(DIM, PR)                                            \
	IBK_BENTRY(kBspline, 1, DIM, PR), IBK_BENTRY(kBspline, 2, DIM, PR),     \
	IBK_BENTRY(kBspline, 3, DIM, PR), IBK_BENTRY(kBspline, 4, DIM, PR),     \
	IBK_BENTRY(kBspline, 5, DIM, PR), IBK_BENTRY(kPeskin, 0, DIM, PR),      \
	IBK_BENTRY(kRoma, 0, DIM, PR), IBK_BENTRY(kCosine, 0, DIM, PR),         \
	IBK_BENTRY(kHat, 0, DIM, PR)

const BatchEntry kBatchTable[] = {
	IBK_BATCH_ENTRIES(2, IBK_PRECISION_FP64),
	IBK_BATCH_ENTRIES(3, IBK_PRECISION_FP64),
	IBK_BATCH_ENTRIES(2, IBK_PRECISION_FP32C),
	IBK_BATCH_ENTRIES(3, IBK_PRECISION_FP32C),
};

const BatchOps* find_batch_ops(int kind, int order, int dims, int precision)
{
	if (kind != kBspline) order = 0;
	for (const BatchEntry& e : kBatchTable)
		if (e.kind == kind && e.order == order && e.dims == dims && e.prec == precision) return &e.ops;
	return nullptr;
}

template <typename T>
ibk_status grow(T** ptr, size_t& cap, size_t want, const char* what)
{
	if (*ptr && cap >= want) return IBK_OK;
	if (*ptr) cudaFree(*ptr);
	*ptr = nullptr;
	cap = 0;
	ibk_status st = cuda_check(cudaMalloc(reinterpret_cast<void**>(ptr), std::max<size_t>(want, 1) * sizeof(T)), what);
	if (st == IBK_OK) cap = want;
	return st;
}

// Tensor maps of instance i's velocity grids for its interpolation regions,
// from the cache when the grid pointers are unchanged; false when any grid
// or box breaks a TMA rule (the instance is then staged by plain loads).
bool instance_maps(Batch& b, int i, const BatchIO& o)
{
	const BatchInst& bi = b.inst_h[i];
	if (bi.ti.T[0] & 1) return false;     // region x origins must stay even
	bool ok = true;
	for (int c = 0; c < b.dims; ++c) {
		const size_t k = (size_t) i * kMaxDims + c;
		if (b.map_ptr[k] != o.ue.p[c]) {
			int lower[3], box[3];
			interp_region(bi.g, bi.ti, b.M, c, lower, box);
			b.map_ok[k] = o.ue.p[c] && grid_tensor_map(&b.map_cache[k], o.ue.p[c], bi.g.comp[c], b.dims, box);
			b.map_ptr[k] = o.ue.p[c];
		}
		ok = ok && b.map_ok[k];
	}
	return ok;
}

// The table of a binding: header, io, active list, item and chunk prefixes and
// the active instances' tensor maps.
void build_table(Batch& b, const std::vector<BatchIO>& io, unsigned char* out)
{
	std::memset(out, 0, b.table_bytes);
	BatchHeader* h = reinterpret_cast<BatchHeader*>(out);
	int* active = reinterpret_cast<int*>(out + b.off_active);
	int* spre = reinterpret_cast<int*>(out + b.off_spre);
	int* ipre = reinterpret_cast<int*>(out + b.off_ipre);
	int* cpre = reinterpret_cast<int*>(out + b.off_cpre);
	std::memcpy(out + b.off_io, io.data(), sizeof(BatchIO) * io.size());
	CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(out + b.off_maps);
	int* use_tma = reinterpret_cast<int*>(out + b.off_tma);
	int total = 0, nact = 0, ns = 0, ni = 0, nc = 0;
	for (int i = 0; i < b.count; ++i) {
		total += io[i].n;
		if (io[i].n == 0) continue;
		if (instance_maps(b, i, io[i])) {
			use_tma[i] = 1;
			for (int c = 0; c < b.dims; ++c) maps[(size_t) i * kMaxDims + c] = b.map_cache[(size_t) i * kMaxDims + c];
		}
		active[nact] = i;
		spre[nact] = ns;
		ipre[nact] = ni;
		cpre[nact] = nc;
		nc += (io[i].n + kBinThreads - 1) / kBinThreads;
		ns += b.nitem_s[i];
		ni += b.nitem_i[i];
		++nact;
	}
	spre[nact] = ns;
	ipre[nact] = ni;
	cpre[nact] = nc;
	h->total_points = total;
	h->num_active = nact;
	h->items_s = ns;
	h->items_i = ni;
	h->chunks = nc;
}

// Tiles, bins, work items and shared-memory sizes of a configuration.
ibk_status configure(Batch& b, const ibk_batch_config& cfg)
{
	std::vector<BatchInst> inst(b.count);
	std::vector<int> nitem_s(b.count), nitem_i(b.count);
	long long bins_s = 0, bins_i = 0, items_s = 0, items_i = 0;
	size_t smem_max = 0, region_max = 0;
	for (int i = 0; i < b.count; ++i) {
		BatchInst& bi = inst[i];
		bi.g = b.geo[i];
		// small grids take smaller tiles (at least four per axis, extents of
		// at least 8 cells): the ensemble's small grids are its dense ones,
		// and their work then spreads over more CTAs
		int ext_s[3], ext_i[3];
		for (int d = 0; d < 3; ++d) {
			const int cells = d < b.dims ? bi.g.comp[0].cells[d] : 1;
			const int cap = std::max(8, cells / 4);
			ext_s[d] = std::min(cfg.spread_tile[d], cap);
			ext_i[d] = std::min(cfg.interp_tile[d], cap);
		}
		bi.ts = make_tiles(bi.g, b.tag[i], b.M, ext_s);
		bi.ti = make_tiles(bi.g, b.tag[i], b.M, ext_i);
		bi.bin_s = (int) bins_s;
		bi.bin_i = (int) bins_i;
		bins_s += bi.ts.num_bins;
		bins_i += bi.ti.num_bins;
		nitem_s[i] = bi.ts.num_tiles * (b.precision == IBK_PRECISION_FP32C ? 1 : b.dims);
		nitem_i[i] = bi.ti.num_tiles * b.dims;
		items_s += nitem_s[i];
		items_i += nitem_i[i];
		if (bins_s >= (1LL << 30) || bins_i >= (1LL << 30) || items_s >= (1LL << 30) || items_i >= (1LL << 30))
			return set_error(IBK_ERR_INVALID_ARGUMENT, "batch has too many tiles");
		smem_max = std::max(smem_max, spread_tile_bytes(bi.g, bi.ts, b.M, b.precision));
		region_max = std::max(region_max, interp_region_bytes(bi.g, bi.ti, b.M));
	}
	const size_t smem_s = smem_max;
	if (smem_s > 200 * 1024 || region_max > 200 * 1024)
		return set_error(IBK_ERR_UNSUPPORTED, "batch tile shape needs more than 200 KB of shared memory");
	ibk_status st;
	const size_t nb = (size_t) std::max(bins_s, bins_i);
	if (!b.d_counts || b.bins_cap < nb) {
		// bin arrays sized for the larger bin space (counts start zeroed and
		// every scan leaves them zeroed)
		void** bufs[] = {reinterpret_cast<void**>(&b.d_counts), reinterpret_cast<void**>(&b.d_off),
		                 reinterpret_cast<void**>(&b.d_chunk), reinterpret_cast<void**>(&b.d_binmax)};
		const size_t bytes[] = {sizeof(int) * nb, sizeof(int) * (nb + 1), sizeof(int) * (nb / kScanChunk + 2),
		                        sizeof(unsigned) * kMaxDims * nb};
		b.bins_cap = 0;
		for (int j = 0; j < 4; ++j) {
			if (*bufs[j]) cudaFree(*bufs[j]);
			*bufs[j] = nullptr;
		}
		for (int j = 0; j < 4; ++j)
			if ((st = cuda_check(cudaMalloc(bufs[j], bytes[j]), "cudaMalloc")) != IBK_OK) return st;
		if ((st = cuda_check(cudaMemset(b.d_counts, 0, bytes[0]), "cudaMemset")) != IBK_OK) return st;
		b.bins_cap = nb;
	}
	// deferred dense items: one per (tile, component)
	const size_t defer_want = (size_t) items_s * kMaxDims + 4;
	if (!b.d_defer || b.defer_cap < defer_want) {
		if (b.d_defer) cudaFree(b.d_defer);
		b.d_defer = nullptr;
		b.defer_cap = 0;
		if ((st = cuda_check(cudaMalloc(reinterpret_cast<void**>(&b.d_defer), sizeof(int) * defer_want),
		                     "cudaMalloc")) != IBK_OK) return st;
		b.defer_cap = defer_want;
	}
	size_t cap = 0;
	BatchInst* d_inst = nullptr;
	if ((st = grow(&d_inst, cap, (size_t) b.count, "cudaMalloc")) != IBK_OK) return st;
	st = cuda_check(cudaMemcpy(d_inst, inst.data(), sizeof(BatchInst) * b.count, cudaMemcpyHostToDevice), "cudaMemcpy");
	if (st != IBK_OK) { cudaFree(d_inst); return st; }
	// finish the work on the old configuration before replacing it
	if ((st = cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) != IBK_OK) { cudaFree(d_inst); return st; }
	if (b.d_inst) cudaFree(b.d_inst);
	b.d_inst = d_inst;
	b.inst_h = std::move(inst);
	b.nitem_s = std::move(nitem_s);
	b.nitem_i = std::move(nitem_i);
	b.bins_s = (int) bins_s;
	b.bins_i = (int) bins_i;
	b.items_s = items_s;
	b.items_i = items_i;
	b.smem_s = smem_s;
	b.smem_i = region_max;
	b.config = cfg;
	std::fill(b.map_ptr.begin(), b.map_ptr.end(), nullptr);   // boxes follow the tiles
	drop_graphs(b);
	if (b.bound) {
		// the bound table's item prefixes follow the tiles: rebuild it
		std::vector<unsigned char> tab(b.table_bytes);
		build_table(b, b.io_h, tab.data());
		if ((st = cuda_check(cudaMemcpy(b.d_table, tab.data(), b.table_bytes, cudaMemcpyHostToDevice), "cudaMemcpy")) != IBK_OK)
			return st;
	}
	return b.ops->prepare(b);
}

void destroy(Batch* b)
{
	drop_graphs(*b);
	for (int r = 0; r < kRing; ++r) {
		if (b->ring_ev[r]) { cudaEventSynchronize(b->ring_ev[r]); cudaEventDestroy(b->ring_ev[r]); }
		if (b->h_ring[r]) cudaFreeHost(b->h_ring[r]);
	}
	void* bufs[] = {b->d_inst, b->d_table, b->d_counts, b->d_off, b->d_chunk, b->d_recs,
	                b->d_next, b->d_status, b->d_kr, b->d_binmax, b->d_defer};
	for (void* p : bufs)
		if (p) cudaFree(p);
	if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
	delete b;
}

// Arrays an operation reads or writes for every instance with points.
ibk_status check_bound(const Batch& b, int op)
{
	if (!b.bound) return set_error(IBK_ERR_INVALID_ARGUMENT, "batch has no bound arrays");
	for (int i = 0; i < b.count; ++i) {
		const BatchIO& o = b.io_h[i];
		if (o.n == 0) continue;
		bool ok = o.x != nullptr;
		if (op == IBK_OP_SPREAD || op == IBK_OP_STEP)
			for (int c = 0; c < b.dims; ++c) ok = ok && o.fe.p[c] != nullptr;
		if (op == IBK_OP_SPREAD_INTERPOLATE)
			for (int c = 0; c < b.dims; ++c) ok = ok && o.fe.p[c] != nullptr;
		if (op == IBK_OP_SPREAD || op == IBK_OP_SPREAD_INTERPOLATE) ok = ok && o.fl != nullptr;
		if (op == IBK_OP_INTERPOLATE || op == IBK_OP_STEP || op == IBK_OP_SPREAD_INTERPOLATE)
			for (int c = 0; c < b.dims; ++c) ok = ok && o.ue.p[c] != nullptr;
		if (op == IBK_OP_INTERPOLATE || op == IBK_OP_SPREAD_INTERPOLATE) ok = ok && o.ul != nullptr;
		if (op == IBK_OP_STEP) ok = ok && o.xn && o.xref && o.fs;
		if (!ok)
			return set_error(IBK_ERR_INVALID_ARGUMENT,
			                 "instance " + std::to_string(i) + " lacks an array this operation needs");
	}
	return IBK_OK;
}

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_batch_create(int count, const ibk_instance_desc* instances, ibk_delta delta, int precision,
                            int max_points, ibk_batch* out)
{
	if (!out || !instances || count <= 0 || max_points < 0)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null pointer, no instances or negative capacity");
	*out = nullptr;
	const int dims = instances[0].domain.dims;
	for (int i = 0; i < count; ++i) {
		ibk_status cs = check_domain(&instances[i].domain, instances[i].tag, instances[i].refinement);
		if (cs != IBK_OK) return cs;
		if (instances[i].domain.dims != dims) return set_error(IBK_ERR_INVALID_ARGUMENT, "instances differ in dims");
	}
	const BatchOps* ops = find_batch_ops(delta.kind, delta.order, dims, precision);
	if (!ops) return set_error(IBK_ERR_UNSUPPORTED, "delta / dims / precision combination not built");
	Batch* b = new (std::nothrow) Batch();
	if (!b) return set_error(IBK_ERR_OUT_OF_MEMORY, "host allocation failed");
	b->ops = ops;
	b->dims = dims;
	b->count = count;
	b->precision = precision;
	b->delta_kind = delta.kind;
	b->delta_order = delta.kind == kBspline ? delta.order : 0;
	b->M = meshwidths_of(delta.kind, b->delta_order);
	b->capacity = max_points;
	cudaGetDevice(&b->device);
	cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
	b->geo.resize(count);
	b->info.resize(count);
	b->tag.resize(count);
	for (int i = 0; i < count; ++i) {
		ibk_status gs = make_geometry(&instances[i].domain, instances[i].tag, instances[i].refinement, b->M,
		                              b->geo[i], b->info[i]);
		if (gs != IBK_OK) { destroy(b); return gs; }
		b->tag[i] = instances[i].tag;
		for (int d = 0; d < dims; ++d)
			if (b->geo[i].comp[0].cells[d] < b->M) {
				destroy(b);
				return set_error(IBK_ERR_UNSUPPORTED, "instance " + std::to_string(i) +
				                 " has an axis with fewer cells than the stencil is wide (use a plan)");
			}
	}
	ibk_status st = IBK_OK;
	auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
	b->off_io = al(sizeof(BatchHeader));
	b->off_active = al(b->off_io + sizeof(BatchIO) * (size_t) count);
	b->off_spre = al(b->off_active + sizeof(int) * (size_t) count);
	b->off_ipre = al(b->off_spre + sizeof(int) * ((size_t) count + 1));
	b->off_cpre = al(b->off_ipre + sizeof(int) * ((size_t) count + 1));
	b->off_maps = al(b->off_cpre + sizeof(int) * ((size_t) count + 1));
	b->off_tma = al(b->off_maps + sizeof(CUtensorMap) * kMaxDims * (size_t) count);
	b->table_bytes = b->off_tma + sizeof(int) * (size_t) count;
	b->map_cache.resize((size_t) count * kMaxDims);
	b->map_ptr.assign((size_t) count * kMaxDims, nullptr);
	b->map_ok.assign((size_t) count * kMaxDims, 0);
	size_t cap = 0;
	if (st == IBK_OK) st = grow(&b->d_table, cap, b->table_bytes, "cudaMalloc");
	for (int r = 0; r < kRing && st == IBK_OK; ++r) {
		st = cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&b->h_ring[r]), b->table_bytes, cudaHostAllocDefault),
		                "cudaHostAlloc");
		if (st == IBK_OK) st = cuda_check(cudaEventCreateWithFlags(&b->ring_ev[r], cudaEventDisableTiming), "cudaEventCreate");
	}
	const size_t pts = (size_t) std::max(max_points, 1);
	cap = 0;
	if (st == IBK_OK) st = grow(&b->d_kr, cap, pts, "cudaMalloc");
	cap = 0;
	if (st == IBK_OK) st = grow(&b->d_recs, cap, pts, "cudaMalloc");
	cap = 0;
	if (st == IBK_OK) st = grow(&b->d_next, cap, 4, "cudaMalloc");
	cap = 0;
	if (st == IBK_OK) st = grow(&b->d_status, cap, 4, "cudaMalloc");
	if (st == IBK_OK) st = cuda_check(cudaMemset(b->d_status, 0, sizeof(int) * 4), "cudaMemset");
	if (st == IBK_OK) {
		// an empty binding: every instance idle
		std::vector<unsigned char> zero(b->table_bytes, 0);
		st = cuda_check(cudaMemcpy(b->d_table, zero.data(), b->table_bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
	}
	if (st == IBK_OK) st = cuda_check(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
	ibk_batch_config cfg{};
	for (int d = 0; d < 3; ++d) { cfg.spread_tile[d] = 16; cfg.interp_tile[d] = 16; }
	if (st == IBK_OK) st = configure(*b, cfg);
	if (st != IBK_OK) { destroy(b); return st; }
	*out = reinterpret_cast<ibk_batch>(b);
	return IBK_OK;
}

ibk_status ibk_batch_destroy(ibk_batch handle)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (b) destroy(b);
	return IBK_OK;
}

ibk_status ibk_batch_info(ibk_batch handle, int instance, ibk_grid_info* info)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || !info || instance < 0 || instance >= b->count)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or info, or instance out of range");
	*info = b->info[instance];
	return IBK_OK;
}

ibk_status ibk_batch_bind(ibk_batch handle, const ibk_instance_io* io, void* stream)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || !io) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or io");
	std::vector<BatchIO> tab(b->count);
	long long total = 0;
	for (int i = 0; i < b->count; ++i) {
		const ibk_instance_io& s = io[i];
		if (s.n < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "negative point count");
		BatchIO& t = tab[i];
		t.n = s.n;
		t.pbase = (int) total;
		t.x = s.x;
		t.fl = s.fl;
		for (int c = 0; c < kMaxDims; ++c) { t.fe.p[c] = s.fe[c]; t.ue.p[c] = s.ue[c]; }
		t.ul = s.ul;
		t.xn = s.xn;
		t.xref = s.xref;
		t.fs = s.fs;
		total += s.n;
		if (total > b->capacity)
			return set_error(IBK_ERR_CAPACITY, "bound points exceed the batch capacity of " +
			                 std::to_string(b->capacity));
	}
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const int r = b->ring_next;
	b->ring_next = (r + 1) % kRing;
	ibk_status st = cuda_check(cudaEventSynchronize(b->ring_ev[r]), "cudaEventSynchronize");
	if (st != IBK_OK) return st;
	build_table(*b, tab, b->h_ring[r]);
	if ((st = cuda_check(cudaMemcpyAsync(b->d_table, b->h_ring[r], b->table_bytes, cudaMemcpyHostToDevice, s),
	                     "cudaMemcpyAsync")) != IBK_OK) return st;
	if ((st = cuda_check(cudaEventRecord(b->ring_ev[r], s), "cudaEventRecord")) != IBK_OK) return st;
	b->io_h = std::move(tab);
	b->bound = true;
	return IBK_OK;
}

ibk_status ibk_batch_set_step(ibk_batch handle, double dt, double k)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch");
	if (dt != b->dt || k != b->k) {
		if (b->exec[IBK_OP_STEP]) { cudaGraphExecDestroy(b->exec[IBK_OP_STEP]); b->exec[IBK_OP_STEP] = nullptr; }
		b->dt = dt;
		b->k = k;
	}
	return IBK_OK;
}

ibk_status ibk_batch_run(ibk_batch handle, int op, void* stream)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || op < IBK_OP_SPREAD || op > IBK_OP_SPREAD_INTERPOLATE) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or unknown op");
	ibk_status st = check_bound(*b, op);
	if (st != IBK_OK) return st;
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	if (b->exec[op]) {
		b->launches += b->graph_kernels[op];
		return cuda_check(cudaGraphLaunch(b->exec[op], s), "cudaGraphLaunch");
	}
	return b->ops->run(*b, op, s);
}

ibk_status ibk_batch_capture(ibk_batch handle, int op)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || op < IBK_OP_SPREAD || op > IBK_OP_SPREAD_INTERPOLATE) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or unknown op");
	if (b->exec[op]) { cudaGraphExecDestroy(b->exec[op]); b->exec[op] = nullptr; }
	ibk_status st = cuda_check(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal),
	                           "cudaStreamBeginCapture");
	if (st != IBK_OK) return st;
	const long long before = b->launches;
	ibk_status rs = b->ops->run(*b, op, b->cap_stream);
	b->graph_kernels[op] = b->launches - before;
	b->launches = before;
	cudaGraph_t graph = nullptr;
	st = cuda_check(cudaStreamEndCapture(b->cap_stream, &graph), "cudaStreamEndCapture");
	if (rs != IBK_OK) { if (graph) cudaGraphDestroy(graph); return rs; }
	if (st != IBK_OK) return st;
	st = cuda_check(cudaGraphInstantiate(&b->exec[op], graph, 0), "cudaGraphInstantiate");
	cudaGraphDestroy(graph);
	return st;
}

ibk_status ibk_batch_configure(ibk_batch handle, const ibk_batch_config* config)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || !config) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or config");
	for (int d = 0; d < 3; ++d)
		if (config->spread_tile[d] < 2 || config->interp_tile[d] < 2 || config->spread_tile[d] > kMaxTileExtent ||
		    config->interp_tile[d] > kMaxTileExtent)
			return set_error(IBK_ERR_INVALID_ARGUMENT, "tile extents must lie in [2, 64]");
	if (config->spread_ctas_per_sm < 0 || config->interp_ctas_per_sm < 0)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "negative CTAs per SM");
	if (config->spread_threads != 0 && config->spread_threads != kTileThreads &&
	    !(config->spread_threads == 512 && b->precision == IBK_PRECISION_FP32C))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "spread threads per CTA: 256, or 512 with FP32C");
	const ibk_batch_config old = b->config;
	ibk_status st = configure(*b, *config);
	if (st != IBK_OK) configure(*b, old);
	return st;
}

ibk_status ibk_batch_get_config(ibk_batch handle, ibk_batch_config* config)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || !config) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or config");
	*config = b->config;
	return IBK_OK;
}

ibk_status ibk_batch_tune(ibk_batch handle, int op, void* stream, ibk_batch_config* best)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || op < IBK_OP_SPREAD || op > IBK_OP_SPREAD_INTERPOLATE) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or unknown op");
	ibk_status st = check_bound(*b, op);
	if (st != IBK_OK) return st;
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	// time one configuration: one warm-up run, then the mean of three
	auto time_cfg = [&](const ibk_batch_config& cfg, float& ms) -> ibk_status {
		ibk_status cs = configure(*b, cfg);
		if (cs != IBK_OK) return cs;
		if ((cs = b->ops->run(*b, op, s)) != IBK_OK) return cs;
		cudaEventRecord(e0, s);
		for (int r = 0; r < 3 && cs == IBK_OK; ++r) cs = b->ops->run(*b, op, s);
		cudaEventRecord(e1, s);
		if (cs != IBK_OK) return cs;
		if ((cs = cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize")) != IBK_OK) return cs;
		cudaEventElapsedTime(&ms, e0, e1);
		ms /= 3.0f;
		return IBK_OK;
	};
	static const int spread_shapes[][3] = {{16, 16, 16}, {32, 16, 16}, {16, 16, 8}, {32, 16, 8}, {32, 32, 8}, {8, 8, 8}};
	static const int interp_shapes[][3] = {{16, 16, 16}, {16, 16, 8}, {32, 16, 8}, {8, 8, 8}, {24, 16, 16}};
	ibk_batch_config cur = b->config;
	float best_ms = 0.0f;
	if ((st = time_cfg(cur, best_ms)) == IBK_OK) {
		const bool tune_s = op != IBK_OP_INTERPOLATE, tune_i = op != IBK_OP_SPREAD;
		for (int pass = 0; pass < 2 && st == IBK_OK; ++pass) {
			const bool spread_pass = pass == 0;
			if ((spread_pass && !tune_s) || (!spread_pass && !tune_i)) continue;
			const int nshape = spread_pass ? 6 : 5;
			for (int k = 0; k < nshape; ++k) {
				ibk_batch_config c = cur;
				int* ext = spread_pass ? c.spread_tile : c.interp_tile;
				const int* want = spread_pass ? spread_shapes[k] : interp_shapes[k];
				for (int d = 0; d < 3; ++d) ext[d] = want[d];
				float ms = 0.0f;
				ibk_status cs = time_cfg(c, ms);
				if (cs == IBK_ERR_UNSUPPORTED) continue;     // shape does not fit in shared memory
				if (cs != IBK_OK) { st = cs; break; }
				if (ms < best_ms) { best_ms = ms; cur = c; }
			}
			// threads per spread CTA (points of a tile shared by more threads)
			if (spread_pass && b->precision == IBK_PRECISION_FP32C && st == IBK_OK) {
				ibk_batch_config c = cur;
				c.spread_threads = cur.spread_threads == 512 ? kTileThreads : 512;
				float ms = 0.0f;
				ibk_status cs = time_cfg(c, ms);
				if (cs != IBK_OK && cs != IBK_ERR_UNSUPPORTED) st = cs;
				else if (cs == IBK_OK && ms < best_ms) { best_ms = ms; cur = c; }
			}
			// persistent CTAs per SM for the chosen shape
			for (int occ = 1; occ <= 4 && st == IBK_OK; ++occ) {
				ibk_batch_config c = cur;
				(spread_pass ? c.spread_ctas_per_sm : c.interp_ctas_per_sm) = occ;
				float ms = 0.0f;
				ibk_status cs = time_cfg(c, ms);
				if (cs != IBK_OK) { st = cs; break; }
				if (ms < best_ms) { best_ms = ms; cur = c; }
			}
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	ibk_status fs = configure(*b, cur);
	if (st == IBK_OK) st = fs;
	if (st == IBK_OK && best) *best = cur;
	return st;
}

ibk_status ibk_batch_launch_count(ibk_batch handle, long long* launches)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b || !launches) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch or output");
	*launches = b->launches;
	return IBK_OK;
}

ibk_status ibk_batch_check(ibk_batch handle)
{
	Batch* b = reinterpret_cast<Batch*>(handle);
	if (!b) return set_error(IBK_ERR_INVALID_ARGUMENT, "null batch");
	int st[4] = {0, 0, 0, 0};
	ibk_status s = cuda_check(cudaMemcpy(st, b->d_status, sizeof(st), cudaMemcpyDeviceToHost), "cudaMemcpy");
	if (s != IBK_OK) return s;
	if (st[0] == 0) return IBK_OK;
	cudaMemset(b->d_status, 0, sizeof(int) * 4);
	return set_error(IBK_ERR_DEVICE_CHECK, "device check tripped (code " + std::to_string(st[0]) + ")");
}

} // extern "C"
