/*
 * CPU oracle for the membrane forces (TEST INFRASTRUCTURE).
 *
 * Only tests/ and bench.py's checks use this file, and only as the checker.
 * It restates, operation by operation, the reference's surface geometry at
 * the sample sites and its hyperelastic tension force; build it with
 * -ffp-contract=off (no fused multiply-add), as the library builds its
 * kernels for the same code.
 *
 * Reference anchors (paths inside the sonwell/ib.cu tree):
 *   geometry  include/bases/geometry.h:30-49 (operator products), 95-119
 *             (normal, patch area); include/algo/cross.h, include/algo/dot.h
 *   metric    include/forces/load.h:247-341 (metric, Christoffel symbols)
 *   tension   include/forces/tension.h:35-51 (helper), 71-112 (force)
 *   laws      include/forces/skalak.h:22-31, include/forces/neohookean.h:22-32,
 *             include/forces/hookean.h:19-30
 *   bending   include/forces/bending.h:46-74 (curvatures), 145-229 (force)
 *   dissipation include/forces/dissipation.h:57-127 (rates of the metric and
 *             the Christoffel symbols), 193-206 (helpers), 216-265 (force)
 *   tether    include/forces/tether.h:14-22
 *   repelling include/forces/repelling.h:15-45
 *   curves    include/bases/geometry.h:95-119 for one tangent (algo::cross,
 *             include/algo/cross.h, of one 2-vector: (t1, -t0));
 *             include/forces/tension.h:148-200 (tension1d),
 *             include/forces/skalak.h:49-55, include/forces/hookean.h:48-54
 *
 * Parity pinned: the reference's own force code (forces/skalak.h,
 * neohookean.h, hookean.h, bending.h, dissipation.h, tether.h and tension1d)
 * compiled on the host over shim containers (ref_forces.cc) gives the same
 * bits as this restatement on the same geometry.  The surface geometry (the
 * operator products, normal and patch area) is restated from the text and
 * checked against analytic tori; the wall repulsion too, since the
 * reference's repelling.h does not compile as written.
 */
#include "ibk_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>

typedef struct { double x, y, z; } v3;

static v3 ld3(const double* p, long long m, long long i) { v3 r = {p[i], p[m + i], p[2 * m + i]}; return r; }
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

void ibo_surface_geometry(int ns, int nd, int nc, const double* const* ops, const double* weights,
                          const double* x, double* const* out)
{
	const long long n = (long long) ns * nc;
	/* operator products: out_q(r, j) = sum_k op_q(r, k) x(k, j), column-major,
	 * j = component * nc + shape */
	for (int q = 0; q < 6; ++q) {
		double* y = out[q];
		if (!y) continue;
		if (q == 0 && !ops[0]) {
			for (long long i = 0; i < 3LL * nd * nc; ++i) y[i] = x[i];
			continue;
		}
		const double* op = ops[q];
		for (int j = 0; j < 3 * nc; ++j)
			for (int r = 0; r < ns; ++r) {
				double s = 0.0;
				for (int k = 0; k < nd; ++k) s += op[(size_t) k * ns + r] * x[(size_t) j * nd + k];
				y[(size_t) j * ns + r] = s;
			}
	}
	/* normal and patch area per sample (geometry.h:95-119) */
	for (long long p = 0; p < n; ++p) {
		const v3 a = ld3(out[1], n, p), b = ld3(out[2], n, p);
		const v3 c = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
		const double detf = sqrt(dot3(c, c));
		if (out[6]) {
			out[6][p] = c.x / detf;
			out[6][n + p] = c.y / detf;
			out[6][2 * n + p] = c.z / detf;
		}
		out[7][p] = weights[p % ns] * detf;
	}
}

typedef struct { double e, f, g, eu, fu, gu, ev, fv, gv, i, iu, iv; } metric_t;

/* tension.h:35-51 with g_ij = t_i . t_j and G_ij,k = t_ij . t_k */
static metric_t metric(v3 u, v3 v, v3 uu, v3 uv, v3 vv)
{
	metric_t m;
	m.e = dot3(u, u);
	m.f = dot3(u, v);
	m.g = dot3(v, v);
	const double uu_u = dot3(uu, u), uu_v = dot3(uu, v);
	const double uv_u = dot3(uv, u), uv_v = dot3(uv, v);
	const double vv_u = dot3(vv, u), vv_v = dot3(vv, v);
	m.eu = 2 * uu_u;
	m.fu = uu_v + uv_u;
	m.gu = 2 * uv_v;
	m.ev = 2 * uv_u;
	m.fv = uv_v + vv_u;
	m.gv = 2 * vv_v;
	m.i = m.e * m.g - m.f * m.f;
	m.iu = m.eu * m.g + m.e * m.gu - 2 * m.f * m.fu;
	m.iv = m.ev * m.g + m.e * m.gv - 2 * m.f * m.fv;
	return m;
}

void ibo_membrane_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                          const double* const* cur, double* f)
{
	const long long n = npoints;
	for (long long p = 0; p < n; ++p) {
		const metric_t o = metric(ld3(rest[0], n, p), ld3(rest[1], n, p), ld3(rest[2], n, p),
		                          ld3(rest[3], n, p), ld3(rest[4], n, p));
		const v3 u = ld3(cur[0], n, p), v = ld3(cur[1], n, p);
		const v3 uu = ld3(cur[2], n, p), uv = ld3(cur[3], n, p), vv = ld3(cur[4], n, p);
		const metric_t c = metric(u, v, uu, uv, vv);
		const double os = rest[5][p];

		const double i1 = (c.e * o.g + o.e * c.g - 2 * o.f * c.f) / o.i;
		const double i2 = c.i / o.i;
		const double i1u = (c.eu * o.g + c.e * o.gu + o.eu * c.g + o.e * c.gu - 2 * (o.fu * c.f + o.f * c.fu) - i1 * o.iu) / o.i;
		const double i1v = (c.ev * o.g + c.e * o.gv + o.ev * c.g + o.e * c.gv - 2 * (o.fv * c.f + o.f * c.fv) - i1 * o.iv) / o.i;
		const double i2u = (c.iu - i2 * o.iu) / o.i;
		const double i2v = (c.iv - i2 * o.iv) / o.i;

		double w1, w2, w11, w12, w22;
		if (law == 0) {                    /* Skalak */
			w1 = e * (i1 - 1);
			w2 = (kappa * (i2 - 1) - e);
			w11 = e;
			w12 = 0.0;
			w22 = kappa;
		} else if (law == 2) {             /* Hookean (hookean.h:19-30) */
			const double j = sqrt(i1);
			w1 = e * (1 - 1. / j);
			w2 = 0.0;
			w11 = e / (2 * i1 * j);
			w12 = 0.0;
			w22 = 0.0;
		} else {                           /* neo-Hookean */
			const double j = sqrt(i2);
			w1 = e / j;
			w2 = kappa * (1 - 1 / j) - 0.5 * w1 * i1 / i2;
			w11 = 0.0;
			w12 = -0.5 * w1 / i2;
			w22 = 0.75 * w1 * i1 / (i2 * i2) + 0.5 * kappa / (i2 * j);
		}
		const double w1u = w11 * i1u + w12 * i2u;
		const double w1v = w11 * i1v + w12 * i2v;
		const double w2u = w12 * i1u + w22 * i2u;
		const double w2v = w12 * i1v + w22 * i2v;

		const double uc[3] = {u.x, u.y, u.z}, vc[3] = {v.x, v.y, v.z};
		const double uuc[3] = {uu.x, uu.y, uu.z}, uvc[3] = {uv.x, uv.y, uv.z}, vvc[3] = {vv.x, vv.y, vv.z};
		for (int k = 0; k < 3; ++k)
			f[k * n + p] = os / o.i * (
					+     (w1 * o.g + w2 * c.g) * uuc[k]
					- 2 * (w1 * o.f + w2 * c.f) * uvc[k]
					+     (w1 * o.e + w2 * c.e) * vvc[k]
					- (w1 * o.g + w2 * c.g) * o.iu / (2 * o.i) * uc[k]
					+ (w1 * o.f + w2 * c.f) * o.iv / (2 * o.i) * uc[k]
					+ (w1 * o.f + w2 * c.f) * o.iu / (2 * o.i) * vc[k]
					- (w1 * o.e + w2 * c.e) * o.iv / (2 * o.i) * vc[k]
					+ (w1u * o.g + w1 * o.gu + w2u * c.g + w2 * c.gu) * uc[k]
					- (w1v * o.f + w1 * o.fv + w2v * c.f + w2 * c.fv) * uc[k]
					- (w1u * o.f + w1 * o.fu + w2u * c.f + w2 * c.fu) * vc[k]
					+ (w1v * o.e + w1 * o.ev + w2v * c.e + w2 * c.ev) * vc[k]
			);
	}
}

/* Mean and Gaussian curvature (include/forces/bending.h:46-74). */
static void curvatures(v3 u, v3 v, v3 uu, v3 uv, v3 vv, v3 n, double* h, double* k)
{
	const double e = dot3(u, u), f = dot3(u, v), g = dot3(v, v);
	const double l = dot3(uu, n), kk = dot3(uv, n), m = dot3(vv, n);
	*h = (l * g + m * e - 2 * kk * f) / (2 * (e * g - f * f));
	*k = (l * m - kk * kk) / (e * g - f * f);
}

static void curv_at(const double* const* s, long long n, long long p, double* h, double* k)
{
	curvatures(ld3(s[0], n, p), ld3(s[1], n, p), ld3(s[2], n, p), ld3(s[3], n, p), ld3(s[4], n, p),
	           ld3(s[5], n, p), h, k);
}

/* Bending force (include/forces/bending.h:145-229): mean curvature at the
 * data sites (data_ops, the shape family's operators at its data sites),
 * its derivatives at the samples (sample_ops[1..5]), the surface Laplacian
 * with the current sample metric, and -4 kappa sigma (Lap H + 2 (H - H0)
 * (H^2 - K + H H0)) along the normal.  rest / cur: tu, tv, tuu, tuv, tvv,
 * normal (cur also sigma) at the samples. */
void ibo_membrane_bending(int ns, int nd, int nc, const double* const* data_ops, const double* data_weights,
                          const double* const* sample_ops, double modulus, int preferred, const double* x_rest,
                          const double* x_cur, const double* const* rest, const double* const* cur, double* f)
{
	const long long m = (long long) nd * nc, n = (long long) ns * nc;
	double* geo = (double*) calloc((size_t) 19 * m, sizeof(double));
	double* h = (double*) calloc((size_t) m, sizeof(double));
	double* h0 = (double*) calloc((size_t) m, sizeof(double));
	double* hd = (double*) calloc((size_t) 5 * n, sizeof(double));
	double* out[8] = {NULL, geo, geo + 3 * m, geo + 6 * m, geo + 9 * m, geo + 12 * m, geo + 15 * m, geo + 18 * m};
	const double* dg[6] = {out[1], out[2], out[3], out[4], out[5], out[6]};
	double hh, kk;
	if (preferred) {
		ibo_surface_geometry(nd, nd, nc, data_ops, data_weights, x_rest, out);
		for (long long p = 0; p < m; ++p) { curv_at(dg, m, p, &hh, &kk); h0[p] = hh; }
	}
	ibo_surface_geometry(nd, nd, nc, data_ops, data_weights, x_cur, out);
	for (long long p = 0; p < m; ++p) {
		curv_at(dg, m, p, &hh, &kk);
		if (preferred) hh -= h0[p];
		h[p] = hh;
	}
	/* derivatives of the curvature field at the samples: ops (ns x nd) * h (nd x nc) */
	for (int q = 1; q < 6; ++q) {
		const double* op = sample_ops[q];
		double* y = hd + (q - 1) * n;
		for (int j = 0; j < nc; ++j)
			for (int r = 0; r < ns; ++r) {
				double s = 0.0;
				for (int k = 0; k < nd; ++k) s += op[(size_t) k * ns + r] * h[(size_t) j * nd + k];
				y[(size_t) j * ns + r] = s;
			}
	}
	for (long long p = 0; p < n; ++p) {
		const v3 u = ld3(cur[0], n, p), v = ld3(cur[1], n, p);
		const v3 uu = ld3(cur[2], n, p), uv = ld3(cur[3], n, p), vv = ld3(cur[4], n, p);
		const v3 nrm = ld3(cur[5], n, p);
		const metric_t x = metric(u, v, uu, uv, vv);
		const double hu = hd[p], hv = hd[n + p], huu = hd[2 * n + p], huv = hd[3 * n + p], hvv = hd[4 * n + p];
		const double lh = (((- x.iu * x.g + x.iv * x.f) / (2 * x.i) + x.gu - x.fv) / x.i * hu +
		                   ((+ x.iu * x.f - x.iv * x.e) / (2 * x.i) - x.fu + x.ev) / x.i * hv) +
		                  x.g / x.i * huu - 2 * x.f / x.i * huv + x.e / x.i * hvv;
		double hc, kc;
		curvatures(u, v, uu, uv, vv, nrm, &hc, &kc);
		double dh = hc, sh = hc * hc - kc;
		if (preferred) {
			double hr, kr;
			curv_at(rest, n, p, &hr, &kr);
			dh -= hr;
			sh += hc * hr;
		}
		const double b = lh + 2 * (dh * sh);
		const double mag = -4 * cur[6][p] * modulus * b;
		f[p] = mag * nrm.x;
		f[n + p] = mag * nrm.y;
		f[2 * n + p] = mag * nrm.z;
	}
	free(geo);
	free(h);
	free(h0);
	free(hd);
}

/* Operator products of the derivative operators ops[1..5] (ns x nd,
 * column-major) with y (nd x cols): out + (q - 1) * ns * cols, same loop as
 * ibo_surface_geometry. */
static void derivatives(int ns, int nd, int cols, const double* const* ops, const double* y, double* out)
{
	for (int q = 1; q < 6; ++q) {
		const double* op = ops[q];
		double* o = out + (size_t) (q - 1) * ns * cols;
		for (int j = 0; j < cols; ++j)
			for (int r = 0; r < ns; ++r) {
				double s = 0.0;
				for (int k = 0; k < nd; ++k) s += op[(size_t) k * ns + r] * y[(size_t) j * nd + k];
				o[(size_t) j * ns + r] = s;
			}
	}
}

void ibo_membrane_dissipation(int ns, int nd, int nc, const double* const* sample_ops, double kappa,
                              const double* u, const double* const* cur, double* f)
{
	const long long n = (long long) ns * nc;
	double* vd = (double*) malloc(sizeof(double) * 15 * (size_t) n);
	derivatives(ns, nd, 3 * nc, sample_ops, u, vd);
	for (long long p = 0; p < n; ++p) {
		const v3 tu = ld3(cur[0], n, p), tv = ld3(cur[1], n, p);
		const v3 tuu = ld3(cur[2], n, p), tuv = ld3(cur[3], n, p), tvv = ld3(cur[4], n, p);
		const v3 su = ld3(vd, n, p), sv = ld3(vd + 3 * n, n, p);
		const v3 suu = ld3(vd + 6 * n, n, p), suv = ld3(vd + 9 * n, n, p), svv = ld3(vd + 12 * n, n, p);
		const metric_t m = metric(tu, tv, tuu, tuv, tvv);
		const double e = m.e, ff = m.f, g = m.g, eu = m.eu, fu = m.fu, gu = m.gu, ev = m.ev, fv = m.fv, gv = m.gv;
		const double i = m.i, iu = m.iu, iv = m.iv;

		/* dot_metric (dissipation.h:57-79) */
		const double de = dot3(tu, su) + dot3(su, tu);
		const double df = dot3(tu, sv) + dot3(su, tv);
		const double dg = dot3(tv, sv) + dot3(sv, tv);
		/* dot_christoffel (dissipation.h:89-127) and dot_helper (193-206) */
		const double c00_0 = dot3(suu, tu) + dot3(tuu, su), c00_1 = dot3(suu, tv) + dot3(tuu, sv);
		const double c01_0 = dot3(suv, tu) + dot3(tuv, su), c01_1 = dot3(suv, tv) + dot3(tuv, sv);
		const double c11_0 = dot3(svv, tu) + dot3(tvv, su), c11_1 = dot3(svv, tv) + dot3(tvv, sv);
		const double deu = 2 * c00_0, dfu = c00_1 + c01_0, dgu = 2 * c01_1;
		const double dev = 2 * c01_0, dfv = c01_1 + c11_0, dgv = 2 * c11_1;

		/* dissipation.h:223-256 */
		double pig[4], pigu[4], pigv[4], pif[3], pifu[3], pifv[3];
		pig[0] = (g * de - ff * df) / i;
		pig[1] = (g * df - ff * dg) / i;
		pig[2] = (e * df - ff * de) / i;
		pig[3] = (e * dg - ff * df) / i;
		pigu[0] = (gu * de + g * deu - fu * df - ff * dfu - iu * pig[0]) / i;
		pigu[1] = (gu * df + g * dfu - fu * dg - ff * dgu - iu * pig[1]) / i;
		pigu[2] = (eu * df + e * dfu - fu * de - ff * deu - iu * pig[2]) / i;
		pigu[3] = (eu * dg + e * dgu - fu * df - ff * dfu - iu * pig[3]) / i;
		pigv[0] = (gv * de + g * dev - fv * df - ff * dfv - iv * pig[0]) / i;
		pigv[1] = (gv * df + g * dfv - fv * dg - ff * dgv - iv * pig[1]) / i;
		pigv[2] = (ev * df + e * dfv - fv * de - ff * dev - iv * pig[2]) / i;
		pigv[3] = (ev * dg + e * dgv - fv * df - ff * dfv - iv * pig[3]) / i;
		pif[0] = pig[0] * g - pig[1] * ff;
		pif[1] = 0.5 * (pig[1] * e + pig[2] * g - (pig[0] + pig[3]) * ff);
		pif[2] = pig[3] * e - pig[2] * ff;
		pifu[0] = pigu[0] * g + pig[0] * gu - pigu[1] * ff - pig[1] * fu;
		pifu[1] = 0.5 * (pigu[1] * e + pig[1] * eu + pigu[2] * g + pig[2] * gu
		                 - ((pigu[0] + pigu[3]) * ff + (pig[0] + pig[3]) * fu));
		pifu[2] = pigu[3] * e + pig[3] * eu - pigu[2] * ff - pig[2] * fu;
		pifv[0] = pigv[0] * g + pig[0] * gv - pigv[1] * ff - pig[1] * fv;
		pifv[1] = 0.5 * (pigv[1] * e + pig[1] * ev + pigv[2] * g + pig[2] * gv
		                 - ((pigv[0] + pigv[3]) * ff + (pig[0] + pig[3]) * fv));
		pifv[2] = pigv[3] * e + pig[3] * ev - pigv[2] * ff - pig[2] * fv;
		const double c0 = pifu[0] + pifv[1] - (iu * pif[0] + iv * pif[1]) / (2 * i);
		const double c1 = pifu[1] + pifv[2] - (iu * pif[1] + iv * pif[2]) / (2 * i);

		/* dissipation.h:258-264: fd = c0 t_u + c1 t_v + pif0 t_uu + 2 pif1 t_uv
		 * + pif2 t_vv, f = s kappa / i fd */
		const double uc[3] = {tu.x, tu.y, tu.z}, vc[3] = {tv.x, tv.y, tv.z};
		const double uuc[3] = {tuu.x, tuu.y, tuu.z}, uvc[3] = {tuv.x, tuv.y, tuv.z}, vvc[3] = {tvv.x, tvv.y, tvv.z};
		for (int k = 0; k < 3; ++k) {
			const double fd = c0 * uc[k] + c1 * vc[k] + pif[0] * uuc[k] + 2 * pif[1] * uvc[k] + pif[2] * vvc[k];
			f[k * n + p] = cur[5][p] * kappa / i * fd;
		}
	}
	free(vd);
}

void ibo_membrane_tether(double modulus, int npoints, const double* x_rest, const double* x_cur, double* f)
{
	for (long long p = 0; p < 3LL * npoints; ++p) f[p] = modulus * (x_rest[p] - x_cur[p]);
}

void ibo_membrane_repelling(double modulus, double height, double range, int npoints, const double* x,
                            const double* sigma, double* f)
{
	const long long n = npoints;
	for (long long p = 0; p < n; ++p) {
		const double r = fabs(height - x[n + p]) / range;
		const double fy = r < 2 ? -log(r / 2) * exp(-4 / (4 - r * r)) : 0.0;
		const double fc[3] = {0.0, fy, 0.0};
		for (int k = 0; k < 3; ++k) f[k * n + p] = -modulus * fc[k] * sigma[p];
	}
}

void ibo_curve_geometry(int ns, int nd, int nc, const double* const* ops, const double* weights,
                        const double* x, double* const* out)
{
	const long long n = (long long) ns * nc;
	/* out[0..2] = position, t, tt: ops[0..2] times x (2 nc columns) */
	for (int q = 0; q < 3; ++q) {
		double* y = out[q];
		if (!y) continue;
		if (q == 0 && !ops[0]) {
			for (long long i = 0; i < 2LL * nd * nc; ++i) y[i] = x[i];
			continue;
		}
		const double* op = ops[q];
		for (int j = 0; j < 2 * nc; ++j)
			for (int r = 0; r < ns; ++r) {
				double s = 0.0;
				for (int k = 0; k < nd; ++k) s += op[(size_t) k * ns + r] * x[(size_t) j * nd + k];
				y[(size_t) j * ns + r] = s;
			}
	}
	for (long long p = 0; p < n; ++p) {
		const double c0 = out[1][n + p], c1 = -out[1][p];
		const double detf = sqrt(c0 * c0 + c1 * c1);
		if (out[3]) {
			out[3][p] = c0 / detf;
			out[3][n + p] = c1 / detf;
		}
		out[4][p] = weights[p % ns] * detf;
	}
}

void ibo_curve_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                       const double* const* cur, double* f)
{
	const long long n = npoints;
	for (long long p = 0; p < n; ++p) {
		const double ou[2] = {rest[0][p], rest[0][n + p]}, ouu[2] = {rest[1][p], rest[1][n + p]};
		const double u[2] = {cur[0][p], cur[0][n + p]}, uu[2] = {cur[1][p], cur[1][n + p]};
		/* helper (tension.h:148-158): i = t . t, i' = 2 G_00,0 = 2 tt . t */
		const double oi = ou[0] * ou[0] + ou[1] * ou[1], odi = 2 * (ouu[0] * ou[0] + ouu[1] * ou[1]);
		const double ci = u[0] * u[0] + u[1] * u[1], cdi = 2 * (uu[0] * u[0] + uu[1] * u[1]);
		const double i = ci / oi;
		const double iu = (cdi - i * odi) / oi;
		double phi, phi1;
		if (law == 0) {                     /* skalak1d */
			phi = e * (i - 1) - kappa * i * (i * i - 1);
			phi1 = e - kappa * (3 * i * i - 1);
		} else {                            /* hookean1d */
			const double j = sqrt(i);
			phi = e * (1 - 1. / j);
			phi1 = e / (2 * i * j);
		}
		const double phiu = phi1 * iu;
		for (int k = 0; k < 2; ++k)
			f[k * n + p] = rest[2][p] / oi * (+ phi * uu[k] - odi / (2 * oi) * phi * u[k] + phiu * u[k]);
	}
}
