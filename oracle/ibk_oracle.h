/*
 * CPU oracle for the immersed-boundary coupling operators (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of sonwell/ib.cu's spread / interpolate path,
 * used only as the checker by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline / --impl reference legs of bench.py.  The product path (the
 * CUDA library under ib.cu_b200/) never links or calls it.
 *
 * Every function cites the reference file:line it restates.  Parity of the
 * index / weight core is pinned against the reference's own headers compiled
 * on the host (oracle/ref_bridge.cc -> oracle/_ref/libibref.so) and against
 * the committed fixtures in tests/golden/.
 */
#ifndef IBK_ORACLE_H
#define IBK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { IBO_PERIODIC = 0, IBO_SOLID = 1 };
enum { IBO_TAG_MAC = 0, IBO_TAG_CENTERED = 1 };
enum { IBO_BSPLINE = 0, IBO_PESKIN = 1, IBO_ROMA = 2, IBO_COSINE = 3, IBO_HAT = 4 };
enum { IBO_STANDARD_PATTERN = 0, IBO_EVERY_OTHER_PATTERN = 1 };

typedef struct {
	int dims;                 /* 1..3 */
	int delta_kind, delta_order;
	int meshwidths;           /* M */
	int values;               /* V = M^dims */
	int pattern;              /* IBO_*_PATTERN */
	int per_sweep, sweeps;    /* include/ib/novel.h:33-45, :100 */
	double unit;              /* fd::domain::unit()  (GCD of lengths) */
	double resolution;        /* refinement / unit */
	double length[3];
	int solid[3];
	/* per component c, per dimension d */
	int cells[3][3];
	int points[3][3];
	double shift[3][3];
	long long size[3];        /* product of points over d */
} ibo_geom;

/* fd::grid / fd::discretization geometry (include/fd/grid.h:232-239,
 * include/fd/discretization.h:113-164, include/fd/domain.h:30-32). */
int ibo_geometry(int dims, const double* length, const int* solid, int tag,
                 int refinement, int delta_kind, int delta_order, ibo_geom* g);

/* delta functions phi(r) (include/ib/{bspline,peskin,roma,cosine,hat}.h) */
double ibo_phi(int delta_kind, int delta_order, double r);

/* stencil offset of entry `e` along each dimension (include/ib/delta.h:97-147) */
void ibo_pattern(const ibo_geom* g, int e, int* s);

/* ib::sweep::sort (include/ib/sweep.h:64-77): one sort key per point. */
void ibo_sort_keys(const ibo_geom* g, int comp, int n, const double* x, int* keys);

/* Per-point stencil data for component `comp`:
 *   base[p*dims+d]   = decompose(key) (include/ib/indexing.h:239-250)
 *   delta[p*dims+d]  = sweep::difference (include/ib/sweep.h:49-62)
 *   weights[p*V+e]   = sweep::values, entry order = pattern (sweep.h:98-112)
 *   sidx[p*V+e]      = spread grid index, -1 = dropped (errors_negative)
 *   iidx[p*V+e]      = interpolation grid index (clamped)
 * Any output pointer may be NULL. */
void ibo_stencil(const ibo_geom* g, int comp, int n, const double* x,
                 int* base, double* delta, double* weights, int* sidx, int* iidx);

/* ib::novel::spread::operator() (include/ib/novel.h:197-227): the reference
 * algorithm (stable sort by key, per-sweep segmented sums, per-sweep planes,
 * combine).  fe[c] is overwritten (or accumulated into when per_sweep == 1,
 * as the reference does).  fe_abs[c] (optional, may be NULL) receives the sum
 * of |contribution| per face, the scale of the rounding-error bound. */
int ibo_spread(const ibo_geom* g, int n, const double* x, const double* f,
               double* const* fe, double* const* fe_abs);

/* ib::interpolate::operator() (include/ib/interpolate.h:92-115): serial sum
 * in pattern order.  ul[c*n+p] is overwritten.  ul_abs optional. */
void ibo_interpolate(const ibo_geom* g, int n, const double* x,
                     const double* const* ue, double* ul, double* ul_abs);

/* Multi-threaded restatements of the same algorithms (CPU baseline only).
 * nthreads <= 0 uses every available host thread. */
int ibo_spread_mt(const ibo_geom* g, int n, const double* x, const double* f,
                  double* const* fe, int nthreads);
void ibo_interpolate_mt(const ibo_geom* g, int n, const double* x,
                        const double* const* ue, double* ul, int nthreads);
int ibo_max_threads(void);

/* Membrane forces (ibk_membrane_oracle.c).  Surface geometry of nc shapes:
 * ops[0..5] column-major ns x nd operators (ops[0] NULL: samples are the
 * data sites), x 3*nd*nc positions [component][shape][site]; out[0..7] =
 * position, tu, tv, tuu, tuv, tvv (3*ns*nc each), normal (3*ns*nc) and
 * sigma (ns*nc), NULL to skip (tu, tv and sigma required). */
void ibo_surface_geometry(int ns, int nd, int nc, const double* const* ops, const double* weights,
                          const double* x, double* const* out);
/* Tension force (law 0 Skalak, 1 neo-Hookean, 2 Hookean): rest[0..5] = tu,
 * tv, tuu, tuv, tvv, sigma; cur[0..4] = tu, tv, tuu, tuv, tvv; f 3*npoints. */
void ibo_membrane_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                          const double* const* cur, double* f);
/* Bending force: data_ops (nd x nd, evaluation NULL) with data_weights give
 * the curvature field at the data sites, sample_ops[1..5] (ns x nd) its
 * derivatives at the samples; rest[0..5] = tu, tv, tuu, tuv, tvv, normal
 * (read with preferred); cur[0..6] the same and sigma; f 3*ns*nc. */
void ibo_membrane_bending(int ns, int nd, int nc, const double* const* data_ops, const double* data_weights,
                          const double* const* sample_ops, double modulus, int preferred, const double* x_rest,
                          const double* x_cur, const double* const* rest, const double* const* cur, double* f);

/* Dissipation force: sample_ops[1..5] (ns x nd) give the derivatives of the
 * data-site velocity u (3*nd*nc) at the samples; cur[0..5] = tu, tv, tuu,
 * tuv, tvv, sigma of the current sample geometry; f 3*ns*nc. */
void ibo_membrane_dissipation(int ns, int nd, int nc, const double* const* sample_ops, double kappa,
                              const double* u, const double* const* cur, double* f);
/* Tether: f = modulus (x_rest - x_cur), 3*npoints values. */
void ibo_membrane_tether(double modulus, int npoints, const double* x_rest, const double* x_cur, double* f);
/* Wall repulsion at npoints samples: x 3*npoints positions, sigma npoints. */
void ibo_membrane_repelling(double modulus, double height, double range, int npoints, const double* x,
                            const double* sigma, double* f);

/* Curves (2 components): ops[0..2] = evaluation (NULL: samples are the data
 * sites), d/ds, d2/ds2 (ns x nd, column-major); x 2*nd*nc; out[0..4] =
 * position, t, tt (2*ns*nc each), normal (2*ns*nc) and sigma (ns*nc), NULL to
 * skip (t and sigma required).  ibo_curve_tension: law 0 skalak1d, 2
 * hookean1d; rest[0..2] = t, tt, sigma; cur[0..1] = t, tt; f 2*npoints. */
void ibo_curve_geometry(int ns, int nd, int nc, const double* const* ops, const double* weights,
                        const double* x, double* const* out);
void ibo_curve_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                       const double* const* cur, double* f);

/* Implicit diffusion step on one component grid (ibk_fluid_oracle.c):
 * points / periodic / shift per axis (dims of them), res the resolution,
 * robin[axis][side][2] the wall conditions (a, b).  ibo_wall_weights: out =
 * {interior, laplacian, boundary} weights of one wall (signed h). */
void ibo_wall_weights(const double* p, double h, double s_in, double* out);
void ibo_diffusion_apply(int dims, const int* points, const int* periodic, const double* shift, double res,
                         const double* robin, double lambda, int op, const double* u, double* out);
int ibo_diffusion_step(int dims, const int* points, const int* periodic, const double* shift, double res,
                       const double* robin, double timestep, double mu, double tolerance, int max_iterations,
                       double gamma, int precond, const double* u, const double* rhs, const double* f, double* out);
/* Chebyshev preconditioner pieces (precond 0 of the step; 1 is Jacobi): the
 * Gershgorin interval {lower, upper} of I~ - lambda L, and the four weights
 * of chebw<4>(a, b) (the step passes a = upper, b = lower). */
void ibo_gershgorin(int dims, const int* points, const int* periodic, const double* shift, double res,
                    const double* robin, double lambda, double* bounds);
void ibo_chebyshev_weights(double a, double b, double* w);

#ifdef __cplusplus
}
#endif
#endif
