/*
 * CPU oracle for sonwell/ib.cu's spread / interpolate (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this file,
 * and only as the checker / CPU baseline.  It restates the reference's
 * arithmetic operation by operation; build it with -ffp-contract=off so no
 * multiply-add is fused (the reference's host evaluation has none).
 *
 * Reference anchors (paths inside the sonwell/ib.cu tree):
 *   geometry  include/fd/domain.h:30-32, include/algo/gcd.h:7-34,
 *             include/fd/grid.h:232-239, include/fd/discretization.h:113-164,
 *             include/fd/cell.h:10-17,80-114,194-195, include/fd/dimension.h:52-57
 *   math      include/util/math.h:147-168 (sign, abs, floor, modulo)
 *   sweep     include/ib/sweep.h:38-125
 *   indexing  include/ib/indexing.h:10-122
 *   patterns  include/ib/delta.h:97-147
 *   deltas    include/ib/bspline.h:13-63, peskin.h:6-32, roma.h:9-35,
 *             cosine.h:9-34, hat.h:9-32
 *   spread    include/ib/novel.h:33-45,58-168,197-227
 *   interp    include/ib/interpolate.h:49-115
 */
#include "ibk_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- math --- */

/* util::math::floor (include/util/math.h:158-162): truncating cast with a
 * one-step fix for negative non-integers, evaluated as x - 1.0 in FP64. */
static double
ref_floor(double x)
{
	return (double) (long) (x - (double) (x < 0 && (-x != (double) (long) -x)));
}

/* util::math::modulo (include/util/math.h:164-168) */
static double
ref_modulo(double x, double s)
{
	return x - s * ref_floor(x / s);
}

/* util::math::abs = sign(x) * x (include/util/math.h:147-156) */
static double
ref_abs(double x)
{
	int sign = (x > 0) - (x < 0);
	return (double) sign * x;
}

/* algo::impl::gcd and algo::gcd for floating point (include/algo/gcd.h:7-34) */
static double
gcd_impl(double a, double b)
{
	double eps = DBL_EPSILON;
	while (ref_abs(b) > eps) {
		if (a < b) { double t = a; a = b; b = t; }
		double c = a - ref_floor(a / b) * b;
		a = b; b = c;
		eps *= 2;
	}
	return a;
}

static double
gcd_fp(double a, double b)
{
	if (a < b) { double t = a; a = b; b = t; }
	return gcd_impl(1.0, b / a) * a;
}

/* -------------------------------------------------------------- deltas --- */

/* bspline<n> (include/ib/bspline.h:13-27) */
static double
bspline(int n, double r)
{
	if (n == 0)
		return (-0.5 <= r && r < 0.5) ? 1.0 : 0.0;
	const double b = ((double) n + 1.0) / (2.0 * (double) n);
	double a = r / (double) n;
	return (b + a) * bspline(n - 1, r + 0.5) + (b - a) * bspline(n - 1, r - 0.5);
}

/* peskin (include/ib/peskin.h:6-14) */
static double
peskin(double r)
{
	double s = fabs(r);
	return s < 1 ?
		(3 - 2 * s + sqrt(1 + 4 * s - 4 * s * s)) / 8 :
		(5 - 2 * s - sqrt(-7 + 12 * s - 4 * s * s)) / 8;
}

/* roma (include/ib/roma.h:9-18) */
static double
roma(double r)
{
	double s = fabs(r);
	return s >= 1.5 ? 0 : s < 0.5 ?
		(1 + sqrt(1 - 3 * s * s)) / 3 :
		(5 - 3 * s - sqrt(1 - 3 * (1 - s) * (1 - s))) / 6;
}

/* cosine (include/ib/cosine.h:9-16) */
static double
cosine(double r)
{
	const double pi_halves = 1.57079632679489661923; /* M_PI_2 */
	return 0.25 * (1 + cos(pi_halves * r));
}

/* hat (include/ib/hat.h:9-16) */
static double
hat(double r)
{
	double s = fabs(r);
	return 1 - s;
}

double
ibo_phi(int kind, int order, double r)
{
	switch (kind) {
	case IBO_BSPLINE: return bspline(order, r);
	case IBO_PESKIN: return peskin(r);
	case IBO_ROMA: return roma(r);
	case IBO_COSINE: return cosine(r);
	case IBO_HAT: return hat(r);
	}
	return 0.0;
}

/* ------------------------------------------------------------ geometry --- */

static int
ipow(int b, int e)
{
	int r = 1;
	while (e-- > 0) r *= b;
	return r;
}

int
ibo_geometry(int dims, const double* length, const int* solid, int tag,
             int refinement, int kind, int order, ibo_geom* g)
{
	if (dims < 1 || dims > 3 || refinement <= 0) return -1;
	memset(g, 0, sizeof(*g));
	g->dims = dims;
	g->delta_kind = kind;
	g->delta_order = order;
	switch (kind) {
	case IBO_BSPLINE:
		if (order < 0 || order > 7) return -1;
		g->meshwidths = order + 1; g->pattern = IBO_STANDARD_PATTERN; break;
	case IBO_PESKIN: g->meshwidths = 4; g->pattern = IBO_EVERY_OTHER_PATTERN; break;
	case IBO_ROMA: g->meshwidths = 3; g->pattern = IBO_STANDARD_PATTERN; break;
	case IBO_COSINE: g->meshwidths = 4; g->pattern = IBO_EVERY_OTHER_PATTERN; break;
	case IBO_HAT: g->meshwidths = 2; g->pattern = IBO_STANDARD_PATTERN; break;
	default: return -1;
	}
	g->values = ipow(g->meshwidths, dims);
	/* spread::largest_divisor_under(10) (include/ib/novel.h:33-45) */
	{
		int v = g->values, ps = 1;
		if (10 >= v) ps = v;
		else for (int i = 10; i > 0; --i) if (v % i == 0) { ps = i; break; }
		g->per_sweep = ps;
		g->sweeps = (v + ps - 1) / ps;
	}
	/* fd::domain: base unit = foldl(gcd, lengths...) (include/fd/domain.h:30-32) */
	double unit = length[0];
	for (int d = 1; d < dims; ++d) unit = gcd_fp(unit, length[d]);
	g->unit = unit;
	/* fd::grid::construct: res = ref / base (include/fd/grid.h:232-239) */
	double r = (double) refinement / unit;
	g->resolution = r;
	for (int d = 0; d < dims; ++d) {
		g->length[d] = length[d];
		g->solid[d] = solid[d] ? 1 : 0;
	}
	for (int c = 0; c < dims; ++c) {
		long long size = 1;
		for (int d = 0; d < dims; ++d) {
			/* fd::mac = diagonally shifted cell-centred grid: component c has
			 * alignment 0 along d == c, 0.5 elsewhere (include/fd/cell.h:80-114,
			 * 194-195); fd::centered is 0.5 everywhere. */
			double al = (tag == IBO_TAG_MAC && c == d) ? ref_modulo(0.5 + 0.5, 1.0) : 0.5;
			al = ref_modulo(al, 1.0);                  /* alignment ctor, cell.h:15-16 */
			int on_boundary = !al;                        /* cell.h:11 */
			int cells = (int) (length[d] * r + 0.5);      /* discretization.h:161 */
			int points = cells - (on_boundary && g->solid[d]);
			double shift = al + (double) (g->solid[d] && on_boundary); /* :113 */
			g->cells[c][d] = cells;
			g->points[c][d] = points;
			g->shift[c][d] = shift;
			size *= points;
		}
		g->size[c] = size;
	}
	return 0;
}

/* discretization::units (include/fd/discretization.h:143-149) with
 * dimension::clamp (include/fd/dimension.h:52-57) */
static double
units(const ibo_geom* g, int c, int d, double x)
{
	double s = g->shift[c][d];
	double r = g->resolution;
	double t = x - s / r;
	if (!g->solid[d]) t = ref_modulo(t, g->length[d]);
	return t * r + s;
}

/* discretization::index (include/fd/discretization.h:151-156) */
static int
grid_index(const ibo_geom* g, int c, int d, int i)
{
	if (g->solid[d]) return i;
	int cells = g->cells[c][d];
	return (i + cells) % cells;
}

/* sweep::clamp (include/ib/sweep.h:38-44) */
static int
sweep_clamp(const ibo_geom* g, double r)
{
	const double rounding = 0.5 * (g->meshwidths & 1);
	return (int) ref_floor(r + rounding);
}

/* indexing::clamped::clamp (include/ib/indexing.h:11-16) */
static int
clamped(int index, int weight)
{
	return index < 0 ? 0 : index >= weight ? weight - 1 : index;
}

/* standard_pattern / every_other_pattern (include/ib/delta.h:97-147) */
void
ibo_pattern(const ibo_geom* g, int e, int* s)
{
	const int M = g->meshwidths, dims = g->dims;
	const int shift = (M - 1) >> 1;
	if (g->pattern == IBO_STANDARD_PATTERN) {
		int n = e;
		for (int j = 0; j < dims; ++j) {
			s[j] = n % M - shift;
			n /= M;
		}
	} else {
		const int half = (M + 1) >> 1;
		const int mod = ipow(half, dims);
		int x = e / mod, y = e % mod;
		for (int j = 0; j < dims; ++j) {
			s[j] = x % 2 + 2 * (y % half) - shift;
			x /= 2;
			y /= half;
		}
	}
}

/* sweep::sort (include/ib/sweep.h:64-77) folded by indexing::reduce with the
 * clamped combination rule (include/ib/indexing.h:10-33, 64-81). */
static int
sort_key(const ibo_geom* g, int c, const double* z)
{
	int index = 0, weight = 1;
	for (int d = 0; d < g->dims; ++d) {
		int solid = g->solid[d];
		double shift = g->shift[c][d];
		int i = sweep_clamp(g, units(g, c, d, z[d]) - shift);
		int j = grid_index(g, c, d, i);
		int points = g->points[c][d];
		/* clamped{j, -solid, points} */
		int w = points + solid;
		int k = clamped(j + solid, w);
		if (d == 0) { index = k; weight = w; }
		else {
			index = clamped(index + weight * k, weight * w);
			weight = weight * w;
		}
	}
	return index;
}

/* sorter::decompose (include/ib/indexing.h:239-250) */
static void
decompose(const ibo_geom* g, int c, int key, int* base)
{
	int i = key;
	for (int d = 0; d < g->dims; ++d) {
		int solid = g->solid[d];
		int weight = g->points[c][d] + solid;
		int index = clamped(0 + solid, weight);
		base[d] = i % weight - index;
		i /= weight;
	}
}

/* sweep::difference (include/ib/sweep.h:49-62) */
static void
difference(const ibo_geom* g, int c, const double* z, double* delta)
{
	for (int d = 0; d < g->dims; ++d) {
		double shift = g->shift[c][d];
		double diff = units(g, c, d, z[d]) - shift;
		delta[d] = (double) sweep_clamp(g, diff) - diff;
	}
}

/* sweep::values entry e (include/ib/sweep.h:104-110): right fold
 * phi(d0+s0) * (phi(d1+s1) * (phi(d2+s2) * 1)) */
static double
weight(const ibo_geom* g, const double* delta, const int* s)
{
	double w = 1;
	for (int d = g->dims - 1; d >= 0; --d)
		w = ibo_phi(g->delta_kind, g->delta_order, delta[d] + (double) s[d]) * w;
	return w;
}

/* sweep::grid with errors_negative (spread) or clamped (interpolate)
 * combination rules (include/ib/sweep.h:79-89, indexing.h:10-62,
 * interpolate.h:16-22). */
static int
grid_entry(const ibo_geom* g, int c, const int* base, const int* s, int is_spread)
{
	int index = 0, weight = 1;
	for (int d = 0; d < g->dims; ++d) {
		int points = g->points[c][d];
		int j = grid_index(g, c, d, base[d] + s[d]);
		int k;
		if (is_spread) k = (0 <= j && j < points) ? j : -1;
		else k = clamped(j, points);
		if (d == 0) { index = k; weight = points; continue; }
		if (is_spread)
			index = index < 0 ? -1 : index + weight * k;
		else
			index = clamped(index + weight * k, weight * points);
		weight *= points;
		if (is_spread && index < 0) index = -1;  /* errors_negative ctor */
	}
	return index;
}

void
ibo_sort_keys(const ibo_geom* g, int c, int n, const double* x, int* keys)
{
	for (int p = 0; p < n; ++p) {
		double z[3];
		for (int d = 0; d < g->dims; ++d) z[d] = x[(long) n * d + p];
		keys[p] = sort_key(g, c, z);
	}
}

void
ibo_stencil(const ibo_geom* g, int c, int n, const double* x,
            int* base_out, double* delta_out, double* w_out, int* sidx, int* iidx)
{
	const int dims = g->dims, V = g->values;
	for (int p = 0; p < n; ++p) {
		double z[3], delta[3];
		int base[3];
		for (int d = 0; d < dims; ++d) z[d] = x[(long) n * d + p];
		int key = sort_key(g, c, z);
		decompose(g, c, key, base);
		difference(g, c, z, delta);
		for (int d = 0; d < dims; ++d) {
			if (base_out) base_out[(long) p * dims + d] = base[d];
			if (delta_out) delta_out[(long) p * dims + d] = delta[d];
		}
		for (int e = 0; e < V; ++e) {
			int s[3];
			ibo_pattern(g, e, s);
			if (w_out) w_out[(long) p * V + e] = weight(g, delta, s);
			if (sidx) sidx[(long) p * V + e] = grid_entry(g, c, base, s, 1);
			if (iidx) iidx[(long) p * V + e] = grid_entry(g, c, base, s, 0);
		}
	}
}

/* ------------------------------------------------------------- sorting --- */

/* thrust::sort_by_key on (key, perm) is a stable radix sort: equal keys keep
 * ascending point order.  LSD radix sort, 8 bits per pass. */
static void
radix_sort_pairs(int n, int* keys, int* vals, int nthreads)
{
	int* k2 = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
	int* v2 = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
	unsigned maxkey = 0;
	for (int i = 0; i < n; ++i) if ((unsigned) keys[i] > maxkey) maxkey = (unsigned) keys[i];
	int T = nthreads > 0 ? nthreads : 1;
	size_t* hist = (size_t*) calloc((size_t) T * 256, sizeof(size_t));
	for (int shift = 0; shift < 32 && (maxkey >> shift); shift += 8) {
		memset(hist, 0, sizeof(size_t) * (size_t) T * 256);
		long chunk = ((long) n + T - 1) / T;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(static, 1)
#endif
		for (int t = 0; t < T; ++t) {
			long lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
			size_t* h = hist + (size_t) t * 256;
			for (long i = lo; i < hi; ++i) h[((unsigned) keys[i] >> shift) & 255]++;
		}
		size_t sum = 0;
		for (int b = 0; b < 256; ++b)
			for (int t = 0; t < T; ++t) {
				size_t c = hist[(size_t) t * 256 + b];
				hist[(size_t) t * 256 + b] = sum;
				sum += c;
			}
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(static, 1)
#endif
		for (int t = 0; t < T; ++t) {
			long lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
			size_t* h = hist + (size_t) t * 256;
			for (long i = lo; i < hi; ++i) {
				size_t dst = h[((unsigned) keys[i] >> shift) & 255]++;
				k2[dst] = keys[i];
				v2[dst] = vals[i];
			}
		}
		memcpy(keys, k2, sizeof(int) * (size_t) n);
		memcpy(vals, v2, sizeof(int) * (size_t) n);
	}
	free(hist);
	free(k2);
	free(v2);
}

/* -------------------------------------------------------------- spread --- */

static int
spread_impl(const ibo_geom* g, int n, const double* x, const double* f,
            double* const* fe, double* const* fe_abs, int nthreads)
{
	if (n <= 0) return 0;                               /* novel.h:201 */
	const int dims = g->dims, V = g->values;
	const int per_sweep = g->per_sweep, sweeps = g->sweeps;
	int T = nthreads > 0 ? nthreads : 1;
	(void) T;
	long long maxsize = 0;
	for (int c = 0; c < dims; ++c) if (g->size[c] > maxsize) maxsize = g->size[c];
	/* per_sweep planes (novel.h:180-191, 215); none when per_sweep == 1 */
	double* buf = NULL;
	if (per_sweep > 1) {
		buf = (double*) calloc((size_t) per_sweep * (size_t) maxsize, sizeof(double));
		if (!buf) return -1;
	}
	int* keys = (int*) malloc(sizeof(int) * (size_t) n);
	int* perm = (int*) malloc(sizeof(int) * (size_t) n);
	int* seg = (int*) malloc(sizeof(int) * ((size_t) n + 1));
	if (!keys || !perm || !seg) { free(buf); free(keys); free(perm); free(seg); return -1; }
	/* res = product of component resolutions (novel.h:101-103) */
	const double r = g->resolution;
	double res = 1;
	for (int d = dims - 1; d >= 0; --d) res = r * res;

	for (int c = 0; c < dims; ++c) {
		const double* fc = f + (long) n * c;            /* &fdata[n * i], :223 */
		const long long size = g->size[c];
		double* plane = per_sweep > 1 ? buf : fe[c];
		/* index(): keys + identity permutation, then sort (novel.h:68-90) */
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(static)
#endif
		for (int p = 0; p < n; ++p) {
			double z[3];
			for (int d = 0; d < dims; ++d) z[d] = x[(long) n * d + p];
			keys[p] = sort_key(g, c, z);
			perm[p] = p;
		}
		radix_sort_pairs(n, keys, perm, T);
		/* uniques(): segments of equal keys (novel.h:58-66) */
		int q = 0;
		for (int t = 0; t < n; ++t)
			if (t == 0 || keys[t] != keys[t - 1]) seg[q++] = t;
		seg[q] = n;
		/* reduce(): per sweep, segmented sum of weight*force, then scatter
		 * res * sum into plane i of the buffer (novel.h:92-151) */
		for (int sw = 0; sw < sweeps; ++sw) {
			const int offset = sw * per_sweep;
			const int count = offset + per_sweep >= V ? V - offset : per_sweep;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(dynamic, 256)
#endif
			for (int u = 0; u < q; ++u) {
				double v[16];
				int base[3];
				for (int i = 0; i < count; ++i) v[i] = 0.0;
				for (int t = seg[u]; t < seg[u + 1]; ++t) {
					int j = perm[t];
					double fv = fc[j];
					double z[3], delta[3];
					for (int d = 0; d < dims; ++d) z[d] = x[(long) n * d + j];
					difference(g, c, z, delta);
					for (int i = 0; i < count; ++i) {
						int s[3];
						ibo_pattern(g, offset + i, s);
						v[i] = v[i] + weight(g, delta, s) * fv;
					}
				}
				decompose(g, c, keys[seg[u]], base);
				for (int i = 0; i < count; ++i) {
					int s[3];
					ibo_pattern(g, offset + i, s);
					int j = grid_entry(g, c, base, s, 1);
					if (j >= 0) plane[(long long) i * size + j] += res * v[i];
				}
			}
		}
		/* combine planes into fe, re-zero the buffer (novel.h:153-167) */
		if (per_sweep > 1) {
			double* out = fe[c];
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(static)
#endif
			for (long long t = 0; t < size; ++t) {
				double acc = 0.0;
				for (int i = 0; i < per_sweep; ++i) {
					acc += buf[(long long) i * size + t];
					buf[(long long) i * size + t] = 0.0;
				}
				out[t] = acc;
			}
		}
		/* error-bound scale: sum of |res * w * F| per face (not part of the
		 * reference; used by the tests' tolerance) */
		if (fe_abs && fe_abs[c]) {
			double* a = fe_abs[c];
			memset(a, 0, sizeof(double) * (size_t) size);
			for (int p = 0; p < n; ++p) {
				double z[3], delta[3];
				int base[3];
				for (int d = 0; d < dims; ++d) z[d] = x[(long) n * d + p];
				int key = sort_key(g, c, z);
				decompose(g, c, key, base);
				difference(g, c, z, delta);
				for (int e = 0; e < V; ++e) {
					int s[3];
					ibo_pattern(g, e, s);
					int j = grid_entry(g, c, base, s, 1);
					if (j >= 0) a[j] += fabs(res * weight(g, delta, s) * fc[p]);
				}
			}
		}
	}
	free(buf);
	free(keys);
	free(perm);
	free(seg);
	return 0;
}

int
ibo_spread(const ibo_geom* g, int n, const double* x, const double* f,
           double* const* fe, double* const* fe_abs)
{
	return spread_impl(g, n, x, f, fe, fe_abs, 1);
}

int
ibo_spread_mt(const ibo_geom* g, int n, const double* x, const double* f,
              double* const* fe, int nthreads)
{
	if (nthreads <= 0) nthreads = ibo_max_threads();
	return spread_impl(g, n, x, f, fe, NULL, nthreads);
}

/* --------------------------------------------------------- interpolate --- */

static void
interp_point(const ibo_geom* g, int n, const double* x, const double* const* ue,
             double* ul, double* ul_abs, int p)
{
	const int dims = g->dims, V = g->values;
	double z[3];
	for (int d = 0; d < dims; ++d) z[d] = x[(long) n * d + p];
	for (int c = 0; c < dims; ++c) {
		int base[3];
		double delta[3];
		int key = sort_key(g, c, z);                       /* interpolate.h:66 */
		decompose(g, c, key, base);
		difference(g, c, z, delta);
		double v = 0.0, a = 0.0;
		for (int e = 0; e < V; ++e) {                      /* :70-72, pattern order */
			int s[3];
			ibo_pattern(g, e, s);
			int k = grid_entry(g, c, base, s, 0);
			double w = weight(g, delta, s);
			if (k >= 0) {
				v += w * ue[c][k];
				a += fabs(w * ue[c][k]);
			}
		}
		ul[(long) n * c + p] = v;                          /* &vdata[n * i], :112 */
		if (ul_abs) ul_abs[(long) n * c + p] = a;
	}
}

void
ibo_interpolate(const ibo_geom* g, int n, const double* x,
                const double* const* ue, double* ul, double* ul_abs)
{
	for (int p = 0; p < n; ++p) interp_point(g, n, x, ue, ul, ul_abs, p);
}

void
ibo_interpolate_mt(const ibo_geom* g, int n, const double* x,
                   const double* const* ue, double* ul, int nthreads)
{
	if (nthreads <= 0) nthreads = ibo_max_threads();
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
	for (int p = 0; p < n; ++p) interp_point(g, n, x, ue, ul, NULL, p);
}

int
ibo_max_threads(void)
{
#ifdef _OPENMP
	return omp_get_max_threads();
#else
	return 1;
#endif
}
