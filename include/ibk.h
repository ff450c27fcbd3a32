/*
 * ibk.h -- C ABI of the B200 immersed-boundary coupling library.
 *
 * Drop-in replacement for sonwell/ib.cu's spread / interpolate operators
 * (header-only C++ templates in the reference).  Every entry point takes
 * plain pointers and sizes; no C++ or torch types cross this boundary.
 *
 * Conventions shared with the reference:
 *   - lengths and positions are in the reference's internal units
 *     (1 um == 0.1, include/units.h:16-18, 221-223);
 *   - point arrays are dims column blocks: x[d*n + p], fl[d*n + p],
 *     ul[d*n + p] (include/ib/novel.h:127-128, include/ib/interpolate.h:63-64);
 *   - grid component c is a flat FP64 vector, dimension 0 fastest:
 *     idx = i0 + p0*(i1 + p1*i2) (include/ib/indexing.h:27-33);
 *   - spread OVERWRITES every face of fe[c] (include/ib/novel.h:153-167),
 *     dropping stencil nodes outside a solid wall (indexing.h:35-62);
 *     interpolate OVERWRITES ul and clamps stencil nodes at walls
 *     (include/ib/interpolate.h:16-22);
 *   - n <= 0 returns immediately (novel.h:201, interpolate.h:96).
 * All device pointers are caller-owned device memory.  Calls are ordered on
 * the given CUDA stream (NULL = legacy default stream) and never synchronise
 * the host, except where noted.  A plan's scratch is shared by its calls:
 * use one stream per plan at a time.
 */
#ifndef IBK_H
#define IBK_H

#ifdef __cplusplus
extern "C" {
#endif

#define IBK_VERSION 100

typedef enum {
	IBK_OK = 0,
	IBK_ERR_INVALID_ARGUMENT = 1,   /* bad pointer, size or descriptor */
	IBK_ERR_UNSUPPORTED = 2,        /* delta / dims / precision not built */
	IBK_ERR_OUT_OF_MEMORY = 3,      /* device scratch could not be grown */
	IBK_ERR_CUDA = 4,               /* a CUDA call failed; see ibk_last_error() */
	IBK_ERR_CAPACITY = 5,           /* scratch must grow while a stream is capturing */
	IBK_ERR_DEVICE_CHECK = 6        /* a kernel's own bounds check tripped */
} ibk_status;

/* fd::boundary kinds (include/fd/boundary.h:31-42): only solidity matters to
 * the coupling operators, so dirichlet / neumann / robin are all SOLID. */
typedef enum { IBK_PERIODIC = 0, IBK_SOLID = 1 } ibk_boundary;

/* Grid tags: fd::mac (diagonally shifted cell-centred, the staggered MAC
 * grid) and fd::centered (include/fd/cell.h:194-196). */
typedef enum { IBK_TAG_MAC = 0, IBK_TAG_CENTERED = 1 } ibk_tag;

/* Delta kernels (include/ib/{bspline,peskin,roma,cosine,hat}.h).  For
 * IBK_DELTA_BSPLINE `order` is n of bspline<n> (1..5; bspline<3> is the
 * 4-point cubic used by every 3-D reference driver). */
typedef enum {
	IBK_DELTA_BSPLINE = 0,
	IBK_DELTA_PESKIN = 1,
	IBK_DELTA_ROMA = 2,
	IBK_DELTA_COSINE = 3,
	IBK_DELTA_HAT = 4
} ibk_delta_kind;

/* Arithmetic of the operators.  FP64: the reference's arithmetic (keys,
 * origins and weights bit-exact; interpolation sums in the reference's order;
 * spread differs from the reference only by summation order).  FP32C: the
 * same FP64 index step, FP32 weights and products, compensated (TwoSum)
 * accumulation; FP64 inputs and outputs. */
typedef enum { IBK_PRECISION_FP64 = 0, IBK_PRECISION_FP32C = 1 } ibk_precision;

/* fd::domain of fd::dimension{length, boundary} (include/fd/domain.h:15-33,
 * include/fd/dimension.h:32-80). */
typedef struct {
	int dims;               /* 2 or 3 */
	double length[3];       /* internal units */
	int boundary[3];        /* ibk_boundary */
} ibk_domain;

typedef struct {
	int kind;               /* ibk_delta_kind */
	int order;              /* bspline<order>; ignored otherwise */
} ibk_delta;

/* Geometry of each component grid, as fd::grid / fd::discretization compute
 * it (include/fd/grid.h:232-239, include/fd/discretization.h:113-164). */
typedef struct {
	int dims;
	int meshwidths;         /* stencil width M per dimension */
	double unit;            /* fd::domain::unit(): GCD of the lengths */
	double resolution;      /* refinement / unit */
	int points[3][3];       /* [component][dimension] */
	int cells[3][3];
	double shift[3][3];
	long long size[3];      /* faces per component */
} ibk_grid_info;

typedef struct ibk_plan_s* ibk_plan;

/* Plan = the reference's operator object: ib::spread{tag, domain, delta}
 * (include/ib/novel.h:193-195) and ib::interpolate{tag, domain, delta}
 * (include/ib/interpolate.h:88-90) share one plan.  `refinement` is
 * fd::mac{refinement}.  Binds the current CUDA device. */
ibk_status ibk_plan_create(const ibk_domain* domain, int tag, int refinement,
                           ibk_delta delta, int precision, ibk_plan* out);
ibk_status ibk_plan_destroy(ibk_plan plan);
ibk_status ibk_plan_info(ibk_plan plan, ibk_grid_info* info);

/* Pre-size the plan's device scratch for up to max_points points, so that
 * later calls allocate nothing (required before CUDA-graph capture). */
ibk_status ibk_plan_reserve(ibk_plan plan, int max_points);

/* ib::spread::operator()(n, x, fl, fe) (include/ib/novel.h:197-227):
 * fe[c][j] = sum_p res * w_pj * fl[c*n+p] over in-range nodes j; every face
 * of fe[c] is overwritten. x, fl: device, dims*n doubles; fe: host array of
 * dims device pointers, each ibk_grid_info.size[c] doubles. */
ibk_status ibk_spread(ibk_plan plan, int n, const double* x, const double* fl,
                      double* const* fe, void* stream);

/* ib::interpolate::operator()(n, x, ue, ul) (include/ib/interpolate.h:92-115):
 * ul[c*n+p] = sum_j w_pj * ue[c][clamp(j)].  ue: host array of dims device
 * pointers; ul: device, dims*n doubles. */
ibk_status ibk_interpolate(ibk_plan plan, int n, const double* x,
                           const double* const* ue, double* ul, void* stream);

/* ib::sweep::sort (include/ib/sweep.h:64-77): the reference's 32-bit sort key
 * of every point for component `component` (device output, n ints). */
ibk_status ibk_sort_keys(ibk_plan plan, int component, int n, const double* x,
                         int* keys, void* stream);

/* Instrumentation (no reference counterpart; the reference times with
 * cuda::timer, include/cuda/timer.h:9-19).  While profiling is enabled every
 * kernel launch of the plan is bracketed by CUDA events on its stream;
 * ibk_plan_kernel_stats synchronises on those events and returns, per kernel
 * name, the launch count and summed device time.  ibk_plan_launch_count
 * returns the number of kernels the plan has launched since creation. */
typedef struct {
	char name[48];
	long long launches;
	double total_ms;
} ibk_kernel_stat;

ibk_status ibk_plan_set_profiling(ibk_plan plan, int enable);
ibk_status ibk_plan_kernel_stats(ibk_plan plan, ibk_kernel_stat* out, int capacity, int* count);
ibk_status ibk_plan_reset_stats(ibk_plan plan);
ibk_status ibk_plan_launch_count(ibk_plan plan, long long* launches);

/* Reads (synchronising the device) and clears the plan's device status word,
 * which kernels set instead of faulting when one of their own checks trips
 * (a bounded wait that timed out, a copy precondition that failed).
 * IBK_OK when clean, IBK_ERR_DEVICE_CHECK otherwise. */
ibk_status ibk_plan_check(ibk_plan plan);

/* Interpolation that allocates no device memory (no counterpart in the
 * reference).  For callers that may not call cudaMalloc -- a component that
 * does not own the device's memory pool, a real-time loop where an
 * allocation would synchronise the device, a host that keeps no plan.  Same
 * arguments and result as ibk_interpolate, with the grid described directly
 * instead of by a plan.  Its scratch is one fixed array of about 8 MB that
 * every GPU loading this library holds until exit; calls beyond 524288
 * points, or grids needing more than 262144 bins (tiles x 3^dims), return
 * IBK_ERR_CAPACITY.  All calls share that array, so calls that overlap on the
 * GPU race.  The first call on a device looks up the array's address; make
 * it before any stream capture. */
ibk_status ibk_interpolate_noalloc(const ibk_domain* domain, int tag, int refinement,
                                   ibk_delta delta, int precision, int n, const double* x,
                                   const double* const* ue, double* ul, void* stream);

/* Human-readable text of the last error on the calling host thread. */
const char* ibk_last_error(void);
const char* ibk_status_string(ibk_status status);
int ibk_version(void);

#ifdef __cplusplus
}
#endif
#endif
