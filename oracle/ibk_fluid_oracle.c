/*
 * CPU oracle for the implicit diffusion step (TEST INFRASTRUCTURE).
 *
 * Only tests/ use this file, and only as the checker.  It restates the
 * reference's diffusion step on one component grid,
 *     out = u + (I~ - lambda L)^-1 (k I~ f + k mu (L u + rhs)),
 * k = gamma * timestep, lambda = timestep * mu / 2 (include/ins/diffusion.h:
 * 12-56), with L and I~ the Kronecker sum / product of the 1-D operators
 * (include/fd/laplacian.h:18-46, include/fd/identity.h:22-47,
 * include/fd/combine.h:24-30, include/fd/discretization.h:15-80), solved by
 * the reference's preconditioned CG loop (include/solvers/pcg.h:12-45) with
 * the reference's preconditioner, a degree-4 Chebyshev polynomial in the
 * operator on its Gershgorin interval (include/solvers/chebpcg.h,
 * include/solvers/preconditioners/chebyshev.h, include/algo/chebyshev.h,
 * include/algo/gershgorin.h), or a Jacobi preconditioner.  Build with
 * -ffp-contract=off.
 *
 * The wall weights are checked against the reference's own discretization
 * through the bridge where it is built; the Laplacian and identity assembly
 * and the solver loop are restated from the text.
 */
#include "ibk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static double modulo1(double x) { return x - floor(x); }

void ibo_wall_weights(const double* p, double h, double s_in, double* out)
{
	const double s = 1 - modulo1(1 - s_in);
	const double denom = p[1] - p[0] * s * h;
	out[0] = (p[1] + p[0] * h * (1 - s)) / denom;                                   /* interior */
	out[1] = (-(p[1] * (1 - 2 * s) - p[0] * s * h * (1 - s))) / (2 * denom);        /* laplacian */
	out[2] = -h / denom;                                                             /* boundary */
}

typedef struct {
	int dims, P[3], periodic[3];
	double *lo[3], *dg[3], *hi[3], *id[3];
	long long size;
	double lambda;
} ops_t;

static void build(ops_t* o, int dims, const int* points, const int* periodic, const double* shift, double res,
                  const double* robin, double lambda)
{
	memset(o, 0, sizeof(*o));
	o->dims = dims;
	o->lambda = lambda;
	o->size = 1;
	for (int a = 0; a < 3; ++a) {
		const int P = a < dims ? points[a] : 1;
		o->P[a] = P;
		o->size *= P;
		o->lo[a] = calloc((size_t) P, sizeof(double));
		o->dg[a] = calloc((size_t) P, sizeof(double));
		o->hi[a] = calloc((size_t) P, sizeof(double));
		o->id[a] = calloc((size_t) P, sizeof(double));
		if (a >= dims) { o->id[a][0] = 1.0; continue; }
		const double scale = res * res;
		for (int i = 0; i < P; ++i) {
			o->lo[a][i] = i > 0 ? scale : 0.0;
			o->dg[a][i] = -2 * scale;
			o->hi[a][i] = i + 1 < P ? scale : 0.0;
			o->id[a][i] = 1.0;
		}
		o->periodic[a] = periodic[a];
		if (periodic[a]) {
			o->lo[a][0] = scale * 1.0;
			o->hi[a][P - 1] = scale * 1.0;
		} else {
			double wl[3], wu[3];
			const double h = 1 / res, al = modulo1(shift[a]);
			ibo_wall_weights(robin + 4 * a, h, al, wl);
			ibo_wall_weights(robin + 4 * a + 2, -h, 1 - al, wu);
			o->dg[a][0] += scale * wl[0];
			o->dg[a][P - 1] += scale * wu[0];
			o->id[a][0] += wl[1];
			o->id[a][P - 1] += wu[1];
		}
	}
}

static void release(ops_t* o)
{
	for (int a = 0; a < 3; ++a) { free(o->lo[a]); free(o->dg[a]); free(o->hi[a]); free(o->id[a]); }
}

static double axis_apply(const ops_t* o, int a, const double* u, long long idx, int i, long long stride)
{
	const int P = o->P[a];
	const double um = i > 0 ? u[idx - stride] : (o->periodic[a] ? u[idx + (long long) (P - 1) * stride] : 0.0);
	const double up = i + 1 < P ? u[idx + stride] : (o->periodic[a] ? u[idx - (long long) (P - 1) * stride] : 0.0);
	return o->lo[a][i] * um + o->dg[a][i] * u[idx] + o->hi[a][i] * up;
}

static void apply(const ops_t* o, int op, const double* u, double* out)
{
	const int P0 = o->P[0], P1 = o->P[1];
	for (long long idx = 0; idx < o->size; ++idx) {
		const int i = (int) (idx % P0);
		const long long r = idx / P0;
		const int j = (int) (r % P1);
		const int k = (int) (r / P1);
		const double ix = o->id[0][i], iy = o->dims > 1 ? o->id[1][j] : 1.0, iz = o->dims > 2 ? o->id[2][k] : 1.0;
		double v = 0.0;
		if (op != 1) {
			double l = iz * iy * axis_apply(o, 0, u, idx, i, 1);
			if (o->dims > 1) l += iz * axis_apply(o, 1, u, idx, j, P0) * ix;
			if (o->dims > 2) l += axis_apply(o, 2, u, idx, k, (long long) P0 * P1) * iy * ix;
			v = l;
		}
		if (op == 1) v = iz * iy * ix * u[idx];
		if (op == 2) v = iz * iy * ix * u[idx] - o->lambda * v;
		out[idx] = v;
	}
}

void ibo_diffusion_apply(int dims, const int* points, const int* periodic, const double* shift, double res,
                         const double* robin, double lambda, int op, const double* u, double* out)
{
	ops_t o;
	build(&o, dims, points, periodic, shift, res, robin, lambda);
	apply(&o, op, u, out);
	release(&o);
}

static double dot(const double* a, const double* b, long long n)
{
	double s = 0.0;
	for (long long i = 0; i < n; ++i) s += a[i] * b[i];
	return s;
}

/* Gershgorin interval of I~ - lambda L (algo/gershgorin.h:14-49): the
 * smallest diagonal minus the sum of |off-diagonal| entries and the largest
 * diagonal plus it, over the rows. */
static void gershgorin(const ops_t* o, double* lower, double* upper)
{
	const int P0 = o->P[0], P1 = o->P[1];
	double mn = INFINITY, mx = -INFINITY;
	for (long long idx = 0; idx < o->size; ++idx) {
		const int i = (int) (idx % P0);
		const long long r = idx / P0;
		const int j = (int) (r % P1);
		const int k = (int) (r / P1);
		const double ix = o->id[0][i], iy = o->dims > 1 ? o->id[1][j] : 1.0, iz = o->dims > 2 ? o->id[2][k] : 1.0;
		double l = iz * iy * o->dg[0][i];
		if (o->dims > 1) l += iz * o->dg[1][j] * ix;
		if (o->dims > 2) l += o->dg[2][k] * iy * ix;
		const double diag = iz * iy * ix - o->lambda * l;
		double off = fabs(o->lambda * (iz * iy * o->lo[0][i])) + fabs(o->lambda * (iz * iy * o->hi[0][i]));
		if (o->dims > 1) off += fabs(o->lambda * (iz * o->lo[1][j] * ix)) + fabs(o->lambda * (iz * o->hi[1][j] * ix));
		if (o->dims > 2) off += fabs(o->lambda * (o->lo[2][k] * iy * ix)) + fabs(o->lambda * (o->hi[2][k] * iy * ix));
		if (diag - off < mn) mn = diag - off;
		if (diag + off > mx) mx = diag + off;
	}
	*lower = mn;
	*upper = mx;
}

/* impl::polynomial (algo/chebyshev.h:48-65): sum_i c_i a^i b^(n-1-i). */
static double poly(const double* c, int n, double a, double b)
{
	double v = 0.0;
	for (int i = 0; i < n; ++i) v += c[i] * pow(a, i) * pow(b, n - 1 - i);
	return v;
}

void ibo_chebyshev_weights(double a, double b, double* w)
{
	/* impl::chebw<4> (algo/chebyshev.h:124-145) */
	static const double p1[] = {128}, p2[] = {256, 256}, p3[] = {160, 448, 160}, p4[] = {32, 224, 224, 32};
	static const double q[] = {1, 28, 70, 28, 1};
	const double qv = poly(q, 5, a, b);
	w[0] = poly(p1, 1, a, b) / qv;
	w[1] = poly(p2, 2, a, b) / qv;
	w[2] = poly(p3, 3, a, b) / qv;
	w[3] = poly(p4, 4, a, b) / qv;
}

void ibo_gershgorin(int dims, const int* points, const int* periodic, const double* shift, double res,
                    const double* robin, double lambda, double* bounds)
{
	ops_t o;
	build(&o, dims, points, periodic, shift, res, robin, lambda);
	gershgorin(&o, bounds, bounds + 1);
	release(&o);
}

/* chebyshev::polynomial (algo/chebyshev.h:152-167): s = w0 r, then
 * s = w_i r - H s for i = 1..3 (gemv(-1, H, s, w_i, t) with t = r); the
 * result in z, a and b scratch. */
static void chebyshev(const ops_t* o, const double* w, const double* r, double* z, double* a, double* b)
{
	const long long n = o->size;
	for (long long i = 0; i < n; ++i) a[i] = w[0] * r[i];
	apply(o, 2, a, b);
	for (long long i = 0; i < n; ++i) b[i] = w[1] * r[i] - b[i];
	apply(o, 2, b, a);
	for (long long i = 0; i < n; ++i) a[i] = w[2] * r[i] - a[i];
	apply(o, 2, a, z);
	for (long long i = 0; i < n; ++i) z[i] = w[3] * r[i] - z[i];
}

int ibo_diffusion_step(int dims, const int* points, const int* periodic, const double* shift, double res,
                       const double* robin, double timestep, double mu, double tolerance, int max_iterations,
                       double gamma, int precond, const double* u, const double* rhs, const double* f, double* out)
{
	ops_t o;
	build(&o, dims, points, periodic, shift, res, robin, timestep * mu / 2);
	const long long n = o.size;
	double* b = calloc((size_t) n, sizeof(double));
	double* lu = calloc((size_t) n, sizeof(double));
	double* idf = calloc((size_t) n, sizeof(double));
	double* diag = calloc((size_t) n, sizeof(double));
	double* x = calloc((size_t) n, sizeof(double));
	double* d = calloc((size_t) n, sizeof(double));
	double* q = calloc((size_t) n, sizeof(double));
	const double k = gamma * timestep;
	apply(&o, 0, u, lu);
	apply(&o, 1, f, idf);
	for (long long i = 0; i < n; ++i) b[i] = k * idf[i] + k * mu * (lu[i] + rhs[i]);
	/* Chebyshev weights on the Gershgorin interval (preconditioners/
	 * chebyshev.h:14-25: chebyshev(upper, lower, H)) */
	double lower = 0.0, upper = 0.0, w[4];
	gershgorin(&o, &lower, &upper);
	ibo_chebyshev_weights(upper, lower, w);
	/* Jacobi preconditioner: the reciprocal diagonal of I~ - lambda L */
	const int P0 = o.P[0], P1 = o.P[1];
	for (long long idx = 0; idx < n; ++idx) {
		const int i = (int) (idx % P0);
		const long long r = idx / P0;
		const int j = (int) (r % P1);
		const int kk = (int) (r / P1);
		const double ix = o.id[0][i], iy = dims > 1 ? o.id[1][j] : 1.0, iz = dims > 2 ? o.id[2][kk] : 1.0;
		double l = iz * iy * o.dg[0][i];
		if (dims > 1) l += iz * o.dg[1][j] * ix;
		if (dims > 2) l += o.dg[2][kk] * iy * ix;
		diag[idx] = 1.0 / (iz * iy * ix - o.lambda * l);      /* reciprocal */
	}
	double* rr = b;    /* the residual starts as b */
	/* z = M^-1 r into z: Chebyshev (precond 0) or Jacobi (1); lu, idf scratch */
#define PRECONDITION(r_, z_) do { \
		if (precond == 0) chebyshev(&o, w, (r_), (z_), lu, idf); \
		else for (long long i_ = 0; i_ < n; ++i_) (z_)[i_] = (r_)[i_] * diag[i_]; \
	} while (0)
	PRECONDITION(rr, d);
	double delta = dot(rr, d, n);
	int it = 0;
	while (sqrt(dot(d, d, n)) > tolerance) {
		if (it >= max_iterations) break;
		apply(&o, 2, d, q);
		const double nu = dot(d, q, n);
		if (fabs(nu) < tolerance * tolerance) break;
		const double alpha = delta / nu;
		for (long long i = 0; i < n; ++i) x[i] += alpha * d[i];
		for (long long i = 0; i < n; ++i) rr[i] -= alpha * q[i];
		PRECONDITION(rr, q);
		const double old = delta;
		delta = dot(rr, q, n);
		const double beta = delta / old;
		for (long long i = 0; i < n; ++i) d[i] = q[i] + beta * d[i];
		++it;
	}
#undef PRECONDITION
	for (long long i = 0; i < n; ++i) out[i] = x[i] + u[i];
	free(b); free(lu); free(idf); free(diag); free(x); free(d); free(q);
	release(&o);
	return it;
}
