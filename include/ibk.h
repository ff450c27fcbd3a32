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
 * same FP64 index step (exact stencil origins) and FP32 weights; spread sums
 * the FP32 products exactly in a per-tile fixed point (order-independent, so
 * results do not depend on scheduling), interpolation applies the FP32
 * weights to the grid values rounded to FP32, with FP32 row sums and an FP64
 * total; FP64 inputs and outputs.  Forces must be finite. */
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

/* Preferred tile extents in cells per axis, in [M, 64], for the spread
 * (owner-computes accumulator tiles) and interpolation (staged halo regions)
 * kernels; either may be NULL to keep the current shape.  Each axis is
 * shrunk so its last tile keeps at least M cells.  Default for both: 16
 * cells per axis, but at least four tiles per axis on small grids (equal
 * shapes let ibk_spread_interpolate bin the points once).  Results do
 * not depend on the shape except through the FP32C fixed-point scale, which
 * is per tile. */
ibk_status ibk_plan_set_tiles(ibk_plan plan, const int* spread_tile, const int* interp_tile);

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

/* Spread and interpolation at the same positions, as the reference's time
 * step calls ib::spread and ib::interpolate on one x (include/ib/novel.h:
 * 197-227, include/ib/interpolate.h:92-115; test/ib-whole.cc:226-286 shows
 * the step).  The result is that of ibk_spread(plan, n, x, fl, fe, stream)
 * followed by ibk_interpolate(plan, n, x, ue, ul, stream); the points are
 * binned once when the plan's spread and interpolation tiles agree (the
 * default) instead of once per operator. */
ibk_status ibk_spread_interpolate(ibk_plan plan, int n, const double* x, const double* fl,
                                  double* const* fe, const double* const* ue, double* ul,
                                  void* stream);

/* ib::sweep::sort (include/ib/sweep.h:64-77): the reference's 32-bit sort key
 * of every point for component `component` (device output, n ints). */
ibk_status ibk_sort_keys(ibk_plan plan, int component, int n, const double* x,
                         int* keys, void* stream);

/* Conservation sums in FP64 with a fixed summation order (the same result on
 * every run).  ibk_force_moments: out[0..3) = sum_p F_p, out[3..6) = sum_p
 * x_p cross F_p (2-D: out[5] only).  ibk_grid_totals: out[c] = h^dims *
 * sum_j fe[c][j], the grid side of the force balance (equal to sum_p F_p,c in
 * periodic domains, where spreading conserves force).  out: device arrays of
 * 6 and dims doubles, written in stream order. */
ibk_status ibk_force_moments(ibk_plan plan, int n, const double* x, const double* fl, double* out,
                             void* stream);
ibk_status ibk_grid_totals(ibk_plan plan, double* const* fe, double* out, void* stream);

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
 * instead of by a plan.  Its scratch is one fixed array of about 22 MB that
 * every GPU loading this library holds until exit; calls beyond 524288
 * points, or grids needing more than 262144 bins (tiles x 3^dims), return
 * IBK_ERR_CAPACITY.  All calls share that array, so calls that overlap on the
 * GPU race.  The first call on a device looks up the array's address; make
 * it before any stream capture. */
ibk_status ibk_interpolate_noalloc(const ibk_domain* domain, int tag, int refinement,
                                   ibk_delta delta, int precision, int n, const double* x,
                                   const double* const* ue, double* ul, void* stream);

/* ---- Batches: many independent grids per launch --------------------------
 * No counterpart in the reference, which builds one operator object per grid
 * and launches its kernels grid by grid.  A batch holds `count` instances
 * (each its own domain, tag and refinement; one delta, precision and dims for
 * all) and runs spread, interpolate, or the coupled step below over all of
 * them with one persistent kernel per operator: CTAs take (instance, tile,
 * component) work items from a device-side counter, so uneven instances
 * balance across the SMs.  Instance i behaves exactly like a plan of its own
 * (same arrays, layouts, overwrite semantics; FP32C spread results are
 * bit-identical to a single plan's, FP64 ones equal up to summation order).
 * An instance whose bound point count is 0 is left untouched, as n <= 0 is
 * for a plan. */
typedef struct ibk_batch_s* ibk_batch;

typedef struct {
	ibk_domain domain;
	int tag;                /* ibk_tag */
	int refinement;
} ibk_instance_desc;

/* Device arrays of one instance for the next runs (reference layouts, as
 * ibk_spread / ibk_interpolate take them).  Pointers an operation does not
 * use may be NULL. */
typedef struct {
	int n;                  /* points (0: instance idle) */
	const double* x;        /* dims*n positions */
	const double* fl;       /* dims*n forces: IBK_OP_SPREAD input */
	double* fe[3];          /* force density per component: spread output */
	const double* ue[3];    /* velocity per component: interpolate input */
	double* ul;             /* dims*n velocities: interpolate output */
	double* xn;             /* dims*n: IBK_OP_STEP advected positions */
	const double* xref;     /* dims*n: IBK_OP_STEP spring rest positions */
	double* fs;             /* dims*n: IBK_OP_STEP spring forces */
} ibk_instance_io;

typedef enum {
	IBK_OP_SPREAD = 1,      /* fe <- spread(x, fl) */
	IBK_OP_INTERPOLATE = 2, /* ul <- interpolate(x, ue) */
	/* One coupled immersed-boundary step: U = interpolate(x, ue) (written to
	 * ul when ul is not NULL); xn = x + dt*U (forward Euler); fs = -k*(xn -
	 * xref) (linear spring to the rest shape); fe <- spread(xn, fs). */
	IBK_OP_STEP = 3,
	/* fe <- spread(x, fl) and ul <- interpolate(x, ue): the points are binned
	 * once when the spread and interpolation tiles agree. */
	IBK_OP_SPREAD_INTERPOLATE = 4
} ibk_batch_op;

/* Launch shape of a batch: preferred tile extents in cells per axis (shrunk
 * per instance so the last tile keeps at least M cells), persistent CTAs per
 * SM (0: as many as fit) and threads per spread CTA (0 or 256; 512 with
 * FP32C: the points of a tile shared by more threads, half as many CTAs per
 * SM). */
typedef struct {
	int spread_tile[3];
	int interp_tile[3];
	int spread_ctas_per_sm;
	int interp_ctas_per_sm;
	int spread_threads;
} ibk_batch_config;

/* max_points bounds the sum of the bound point counts; all scratch is
 * allocated here and by ibk_batch_configure, never by a run. */
ibk_status ibk_batch_create(int count, const ibk_instance_desc* instances, ibk_delta delta,
                            int precision, int max_points, ibk_batch* out);
ibk_status ibk_batch_destroy(ibk_batch batch);
ibk_status ibk_batch_info(ibk_batch batch, int instance, ibk_grid_info* info);

/* Binds the arrays of every instance (io[count]).  Stream-ordered: the table
 * is copied to the device on `stream` from a ring of pinned host buffers, so
 * a run queued after it on the same stream sees it; the host blocks only
 * when four binds are still in flight. */
ibk_status ibk_batch_bind(ibk_batch batch, const ibk_instance_io* io, void* stream);

/* dt and k of IBK_OP_STEP (internal units); drops a captured step graph. */
ibk_status ibk_batch_set_step(ibk_batch batch, double dt, double k);

/* Runs op over every instance with the bound arrays.  After
 * ibk_batch_capture(op) it replays the captured CUDA graph instead. */
ibk_status ibk_batch_run(ibk_batch batch, int op, void* stream);

/* Records op as one CUDA graph (on an internal stream) for later runs.  The
 * graph reads the arrays bound at run time, so binds stay outside it. */
ibk_status ibk_batch_capture(ibk_batch batch, int op);

ibk_status ibk_batch_configure(ibk_batch batch, const ibk_batch_config* config);
ibk_status ibk_batch_get_config(ibk_batch batch, ibk_batch_config* config);

/* Autotuner: times op (synchronising) over candidate tile shapes and CTAs per
 * SM on the bound arrays, keeps the fastest configuration and returns it. */
ibk_status ibk_batch_tune(ibk_batch batch, int op, void* stream, ibk_batch_config* best);

ibk_status ibk_batch_launch_count(ibk_batch batch, long long* launches);
/* As ibk_plan_check, for the batch's device status word. */
ibk_status ibk_batch_check(ibk_batch batch);

/* ---- Serving: continuous batching of coupled steps -------------------------
 * No counterpart in the reference.  A server holds the device-resident state
 * of many small simulations ("members": positions, spring rest shape, grid
 * velocity and grid force density) and takes IBK_OP_STEP requests for them as
 * they arrive.  Requests are packed into batched persistent launches on
 * `slots` CUDA streams: while one batch is on the GPU, requests that arrive
 * are launched on the next free slot, so their work overlaps on the device.
 * A member is stepped by at most one launch at a time (its requests run in
 * arrival order).  Admission allocates a member's state only while the total
 * stays within hbm_budget bytes and the device has the memory free.  With
 * FP32C a member's results do not depend on which other members share its
 * launches. */
typedef struct ibk_server_s* ibk_server;

typedef struct {
	ibk_delta delta;
	int precision;              /* ibk_precision */
	int slots;                  /* launches in flight at most (>= 1) */
	double dt, k;               /* IBK_OP_STEP parameters, internal units */
	long long hbm_budget;       /* bytes of member state admitted at most */
	int max_points;             /* points of all members together, at most */
} ibk_server_config;

typedef struct {
	long long requests;         /* completed requests */
	long long launches;         /* batched launches (graph replays) */
	long long points;           /* points stepped */
	double p50_ms, p99_ms, mean_ms, max_ms;   /* arrival -> completion seen */
	double wall_s;              /* first arrival -> last completion */
	long long admitted_bytes;
	double host_ms_per_launch;  /* host time to pack, bind and launch one step batch */
} ibk_server_stats;

ibk_status ibk_server_create(int members, const ibk_instance_desc* desc, const ibk_server_config* config,
                             ibk_server* out);
ibk_status ibk_server_destroy(ibk_server server);

/* Copies a member's initial positions (n points, host, x[d*n + p]; also its
 * spring rest shape) and grid velocity (host, one array per component) to
 * the device and zeroes its force grid.  IBK_ERR_CAPACITY when the member
 * would exceed hbm_budget or the device's free memory. */
ibk_status ibk_server_admit(ibk_server server, int member, int n, const double* x,
                            const double* const* ue);
/* Waits for the member's steps in flight, then releases its state. */
ibk_status ibk_server_retire(ibk_server server, int member);

/* Queues one step request; t_arrival in seconds on the server's clock
 * (ibk_server_clock), or < 0 for now. */
ibk_status ibk_server_submit(ibk_server server, int member, double t_arrival);
/* Non-blocking: completes finished launches and launches queued requests on
 * free slots.  *pending (optional) receives the requests not yet complete. */
ibk_status ibk_server_progress(ibk_server server, int* pending);
/* Progresses until every queued request is complete. */
ibk_status ibk_server_drain(ibk_server server);
double ibk_server_clock(ibk_server server);

/* Synchronising copy of a member's state to the host: positions (dims*n) and
 * force grid per component (either may be NULL). */
ibk_status ibk_server_read(ibk_server server, int member, double* x, double* const* fe);

ibk_status ibk_server_get_stats(ibk_server server, ibk_server_stats* stats);
ibk_status ibk_server_reset_stats(ibk_server server);

/* Open-loop load: `requests` step requests with Poisson arrivals at
 * rate_per_s, each for a member drawn uniformly from the admitted ones
 * (seeded); served as they arrive; returns the statistics of this run. */
ibk_status ibk_server_run_poisson(ibk_server server, double rate_per_s, int requests,
                                  unsigned long long seed, ibk_server_stats* stats);

/* Checkpoint of one member in the linalg::io binary format (below): its
 * positions and spring rest shape (matrices n x dims), grid velocity and grid
 * force density (one vector per component), in that order.  Synchronising.
 * ibk_server_admit_from admits a member from such a file. */
ibk_status ibk_server_save(ibk_server server, int member, const char* path);
ibk_status ibk_server_admit_from(ibk_server server, int member, const char* path);

/* ---- linalg::io binary containers (include/linalg/io.h:66-94, 425-533) ----
 * Each dense vector / matrix is a 32-bit magic number ('v','e' or 'm','a' |
 * 'd' dense | 'd' FP64 or 's' FP32), three 32-bit ints (rows, cols, values)
 * and the values column-major; scalars are raw bytes; objects follow each
 * other in one file.  Host arrays.  Writes are FP64; reads accept FP32 or
 * FP64 values and return FP64.  A sparse container ('s' layout;
 * io.h:432-470, 497-532) holds (rows, cols, nonzeros), then a matrix's CSR
 * row starts (rows + 1 ints, none when rows is 0), the nonzeros' column (or,
 * for a vector, row) indices and their values. */
typedef struct {
	int magic;
	int matrix;             /* 1: matrix, 0: vector */
	int rows, cols;
	int count;              /* dense: rows * cols; sparse: nonzeros */
} ibk_io_header;

ibk_status ibk_io_write_dense(const char* path, int append, int matrix, int rows, int cols,
                              const double* values);
ibk_status ibk_io_write_scalar(const char* path, int append, double value);
/* Reads the object at byte `offset`; values may be NULL to read the header
 * only; *next_offset (optional) receives the offset of the next object. */
ibk_status ibk_io_read_dense(const char* path, long long offset, ibk_io_header* header, double* values,
                             long long capacity, long long* next_offset);
ibk_status ibk_io_read_scalar(const char* path, long long offset, double* value, long long* next_offset);
/* Sparse vectors (matrix = 0, cols = 1, starts unused) and CSR matrices. */
ibk_status ibk_io_write_sparse(const char* path, int append, int matrix, int rows, int cols, int nonzeros,
                               const int* starts, const int* indices, const double* values);
/* starts / indices / values all NULL: the header only; else indices and
 * values of capacity >= nonzeros, and starts of rows + 1 for a matrix. */
ibk_status ibk_io_read_sparse(const char* path, long long offset, ibk_io_header* header, int* starts,
                              int* indices, double* values, long long capacity, long long* next_offset);

/* ---- Membrane forces on RBF surfaces ------------------------------------
 * The producers of the point forces that a spread takes: the surface geometry
 * of a family of shapes that share one set of RBF operators
 * (bases::geometry<2>::compute, include/bases/geometry.h:74-124) and the
 * in-plane tension of a hyperelastic membrane (forces::tension,
 * include/forces/tension.h:9-118) under the Skalak law
 * (include/forces/skalak.h:11-37), the neo-Hookean law
 * (include/forces/neohookean.h:10-37) or the Hookean law
 * (include/forces/hookean.h:11-35), the bending force, the viscous
 * dissipation, the tether and the wall repulsion.  FP64 throughout.  The
 * reference sums a shape's forces (forces::combine,
 * include/forces/combine.h:11-35: (f1 + f2) + f3 ...); the caller adds the
 * outputs in that order.
 *
 * Layout, as the reference's shape matrices: nc shapes of ns sample sites
 * (or nd data sites); a per-site vector quantity is 3 blocks of ns*nc values,
 * [component][shape][site] (the reference's column-major ns x 3nc matrix),
 * a scalar quantity one block of ns*nc values [shape][site]. */
typedef struct ibk_surface_plan_s* ibk_surface_plan;

/* Geometry at the sample sites (every pointer a caller-owned device array;
 * outputs may be NULL where noted). */
typedef struct {
	double* position;       /* 3*ns*nc; NULL: not computed */
	double* t[2];           /* tangents d/du, d/dv: 3*ns*nc each */
	double* tt[3];          /* second derivatives uu, uv, vv: 3*ns*nc each */
	double* normal;         /* t_u x t_v / |t_u x t_v|: 3*ns*nc; NULL: not computed */
	double* sigma;          /* patch areas weight * |t_u x t_v|: ns*nc */
} ibk_surface;

/* One shape family's operators (bases::operators<2>,
 * include/bases/operators.h:128-234): ops[0] evaluation, ops[1..2] first
 * derivatives (u, v), ops[3..5] second derivatives (uu, uv, vv), each a
 * column-major ns x nd device matrix; ops[0] may be NULL when the samples
 * are the data sites (ns == nd; the reference then copies the positions).
 * weights: ns quadrature weights.  The arrays are kept by pointer and must
 * outlive the plan.  Binds the current CUDA device.  A plan keeps per-call
 * device state (the batched products' pointer arrays, the bending and
 * dissipation scratch): calls that use one plan must be ordered, on one
 * stream or synchronised between streams. */
ibk_status ibk_surface_plan_create(int ns, int nd, const double* const* ops, const double* weights,
                                   ibk_surface_plan* out);
ibk_status ibk_surface_plan_destroy(ibk_surface_plan plan);

/* Geometry of nc shapes from their data-site positions x (3*nd*nc,
 * [component][shape][site]): position and derivatives are the operators
 * times x (FP64 library GEMMs), then per sample the normal and the patch area
 * (geometry.h:95-119).  Overwrites every non-NULL output of *out. */
ibk_status ibk_surface_geometry(ibk_surface_plan plan, int nc, const double* x, const ibk_surface* out,
                                void* stream);

/* Tension laws: w(I1, I2) and its second derivatives.  Hookean: w1 =
 * shear (1 - 1/sqrt(I1)), w11 = shear / (2 I1 sqrt(I1)), the rest 0 (bulk
 * unused). */
typedef enum { IBK_LAW_SKALAK = 0, IBK_LAW_NEOHOOKEAN = 1, IBK_LAW_HOOKEAN = 2 } ibk_tension_law;

/* Tension force at npoints sample sites (forces::tension::operator(),
 * tension.h:55-116): from the rest geometry (t, tt, sigma read) and the
 * current geometry (t, tt read), the strain invariants, the law's
 * derivatives and the divergence of the tension, times the rest patch area.
 * shear and bulk are energies per area in internal units (the reference's
 * skalak{shear, bulk} / neohookean{shear, bulk}).  Overwrites f (3*npoints,
 * [component][site]).  npoints <= 0 returns at once. */
ibk_status ibk_membrane_tension(int law, double shear, double bulk, int npoints, const ibk_surface* rest,
                                const ibk_surface* current, double* f, void* stream);

/* Bending force (forces::bending, include/forces/bending.h:10-229):
 * f = -4 kappa sigma (Lap H + 2 (H - H0)(H^2 - K + H H0)) n at every sample,
 * with H0 the rest shape's mean curvature when `preferred` is set (else 0).
 * The mean curvature is taken at the data sites from data_plan (that shape
 * family's operators at its own data sites: ns == nd, evaluation may be
 * NULL) and the positions x_rest / x_current (3*nd*nc; x_rest read only
 * with `preferred`), its surface Laplacian at the samples through
 * sample_plan's derivative operators and the current sample geometry
 * (t, tt, normal, sigma read); K and H at the samples from that geometry,
 * H0 there from the rest sample geometry (t, tt, normal read, with
 * `preferred`).  modulus: bending energy in internal units.  Overwrites f
 * (3*ns*nc).  Device scratch of about (21 nd + 5 ns) * nc doubles is kept by
 * sample_plan and grown on first use (not during stream capture). */
ibk_status ibk_membrane_bending(ibk_surface_plan data_plan, ibk_surface_plan sample_plan, double modulus,
                                int preferred, int nc, const double* x_rest, const double* x_current,
                                const ibk_surface* rest, const ibk_surface* current, double* f, void* stream);

/* Viscous dissipation (forces::dissipation, include/forces/dissipation.h:
 * 128-272): from the data-site velocity u (3*nd*nc, [component][shape][site])
 * its first and second derivatives at the samples through sample_plan's
 * derivative operators; with the current sample geometry (t, tt, sigma read)
 * the rate of change of the metric g' and of the Christoffel symbols, the
 * stress g^-1 g' adj(g) and its surface divergence, times modulus sigma /
 * det g.  modulus: surface viscosity in internal units (the reference's
 * dissipation{dyn s / cm}).  Overwrites f (3*ns*nc).  Device scratch of
 * 15 ns nc doubles is kept by sample_plan (shared with bending: calls on one
 * plan are ordered on one stream) and grown on first use. */
ibk_status ibk_membrane_dissipation(ibk_surface_plan sample_plan, double modulus, int nc, const double* u,
                                    const ibk_surface* current, double* f, void* stream);

/* Tether (forces::tether, include/forces/tether.h:9-26): f = modulus
 * (rest->position - current->position) at npoints samples (3*npoints). */
ibk_status ibk_membrane_tether(double modulus, int npoints, const ibk_surface* rest, const ibk_surface* current,
                               double* f, void* stream);

/* Wall repulsion (forces::repelling, include/forces/repelling.h:9-49): with
 * r = |height - y| / range at each sample (current->position's y), fy =
 * -log(r/2) exp(-4 / (4 - r^2)) for r < 2 (else 0) and f = -modulus (0, fy,
 * 0) sigma (current->sigma read).  The reference fixes height = 16 um and
 * range = 0.25 um (1.6 and 0.025 in its internal length unit of 10 um).
 * range must be positive. */
ibk_status ibk_membrane_repelling(double modulus, double height, double range, int npoints,
                                  const ibk_surface* current, double* f, void* stream);

/* ---- Curves in two-dimensional runs -------------------------------------
 * bases::geometry<1> (include/bases/geometry.h:74-124 with one tangent over
 * two components) and forces::tension1d (include/forces/tension.h:120-205)
 * under the skalak1d (include/forces/skalak.h:39-61) or hookean1d
 * (include/forces/hookean.h:38-60) law, as test/ib-platelet1d.cc uses them.
 * Layout: nc curves of ns samples (nd data sites), a vector quantity 2 blocks
 * of ns*nc values [component][curve][site]; ibk_surface's t[0], tt[0],
 * normal, sigma and position carry the tangent, the second derivative, the
 * normal (t1, -t0)/|t|, the segment lengths weight*|t| and the positions
 * (t[1], tt[1], tt[2] unused). */

/* ops[0] evaluation (NULL when ns == nd), ops[1] d/ds, ops[2] d2/ds2, each a
 * column-major ns x nd device matrix kept by pointer; weights: ns.  The plan
 * serves ibk_surface_geometry (x: 2*nd*nc) and is refused by the surface
 * forces (bending, dissipation). */
ibk_status ibk_curve_plan_create(int ns, int nd, const double* const* ops, const double* weights,
                                 ibk_surface_plan* out);

/* One-dimensional tension at npoints samples: i = |t|^2 / |t_rest|^2, its
 * derivative along the curve, the law's phi(i) and phi'(i), and f = sigma_rest
 * / |t_rest|^2 (phi t_ss - (|t_rest|^2)' / (2 |t_rest|^2) phi t_s + phi' i' t_s)
 * (tension.h:172-200).  law: IBK_LAW_SKALAK (skalak1d: phi = shear (i - 1) -
 * bulk i (i^2 - 1)) or IBK_LAW_HOOKEAN (hookean1d; bulk unused).  Reads rest
 * t[0], tt[0], sigma and current t[0], tt[0]; overwrites f (2*npoints). */
ibk_status ibk_curve_tension(int law, double shear, double bulk, int npoints, const ibk_surface* rest,
                             const ibk_surface* current, double* f, void* stream);

/* ---- The fluid step that consumes the spread: implicit diffusion --------
 * ins::diffusion (include/ins/diffusion.h:12-78) on one component grid of a
 * plan: with L the second-order finite-difference Laplacian and I~ the
 * boundary-corrected identity of that grid (fd::laplacian, fd::identity with
 * correction::second_order; include/fd/laplacian.h, identity.h,
 * discretization.h:47-80), each a Kronecker sum / product of 1-D operators,
 * a step with weight gamma (0.5 backward Euler, 1 Crank-Nicolson) is
 *     out = u + (I~ - lambda L)^-1 (k I~ f + k mu (L u + rhs)),
 *     k = gamma * timestep, lambda = timestep * mu / 2,
 * solved by preconditioned conjugate gradients on the device with the
 * reference's stopping rule: |d|_2 <= tolerance for the search direction d
 * (include/solvers/pcg.h:12-45).  Periodic axes wrap; on a solid axis each
 * side takes a Robin condition a u + b du/dn (Dirichlet {1, 0}, Neumann
 * {0, 1}; include/fd/boundary.h:31-42); the boundary data enter through rhs. */
typedef struct ibk_diffusion_s* ibk_diffusion;

/* robin[d][side][0..1]: (a, b) of the lower (side 0) and upper (side 1) wall
 * of axis d (ignored on periodic axes; a wall with a = b = 0 is rejected).
 * mu: diffusivity (viscosity / density) in internal units; timestep in
 * internal units; max_iterations bounds each solve.  Allocates the
 * component's working vectors; grids of 2^31 faces or more are
 * IBK_ERR_UNSUPPORTED. */
ibk_status ibk_diffusion_create(ibk_plan plan, int component, const double robin[3][2][2], double timestep,
                                double mu, double tolerance, int max_iterations, ibk_diffusion* out);

/* The solve's preconditioner.  IBK_PRECOND_CHEBYSHEV (the default, the
 * reference's solvers::chebpcg, include/solvers/chebpcg.h): z = p(H) r with
 * p the degree-4 polynomial of algo::chebyshev (include/algo/chebyshev.h:
 * 124-167) on the Gershgorin interval of H = I~ - lambda L
 * (include/algo/gershgorin.h), three operator applications per solve.
 * IBK_PRECOND_JACOBI: z = r / diag(H). */
typedef enum { IBK_PRECOND_CHEBYSHEV = 0, IBK_PRECOND_JACOBI = 1 } ibk_preconditioner;
ibk_status ibk_diffusion_set_preconditioner(ibk_diffusion d, int kind);
/* The Gershgorin interval {lower, upper} of H and the four Chebyshev
 * weights (either output may be NULL). */
ibk_status ibk_diffusion_info(ibk_diffusion d, double* bounds, double* weights);
ibk_status ibk_diffusion_destroy(ibk_diffusion d);

/* out = op(u) over the component grid: op 0 = L, 1 = I~, 2 = I~ - lambda L. */
ibk_status ibk_diffusion_apply(ibk_diffusion d, int op, const double* u, double* out, void* stream);

/* One step (ins::diffusion::operator(), diffusion.h:47-56): u, rhs, f and
 * out are component-grid vectors (ibk_grid_info.size[component] doubles;
 * out may alias u).  Synchronises the stream once per solver iteration to
 * test convergence; *iterations (optional) receives the iteration count.
 * IBK_ERR_DEVICE_CHECK when max_iterations pass without convergence. */
ibk_status ibk_diffusion_step(ibk_diffusion d, double gamma, const double* u, const double* rhs, const double* f,
                              double* out, int* iterations, void* stream);

/* Human-readable text of the last error on the calling host thread. */
const char* ibk_last_error(void);
const char* ibk_status_string(ibk_status status);
int ibk_version(void);

#ifdef __cplusplus
}
#endif
#endif
