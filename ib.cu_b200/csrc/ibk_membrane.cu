// Membrane forces on RBF surfaces: the surface geometry of a family of
// shapes that share one set of RBF operators (bases::geometry<2>::compute,
// include/bases/geometry.h:74-124) and the in-plane tension of a
// hyperelastic membrane (forces::tension, include/forces/tension.h:9-118)
// under the Skalak (include/forces/skalak.h:11-37), neo-Hookean
// (include/forces/neohookean.h:10-37) and Hookean
// (include/forces/hookean.h:11-35) laws, the bending force (forces::bending,
// include/forces/bending.h:10-229), the viscous dissipation
// (forces::dissipation, include/forces/dissipation.h:128-272), the tether
// (include/forces/tether.h:9-26) and the wall repulsion
// (include/forces/repelling.h:9-49); for curves in two-dimensional runs the
// geometry and the one-dimensional tension (forces::tension1d,
// include/forces/tension.h:120-205) under the skalak1d and hookean1d laws.
// These produce the point forces that a spread takes.
//
// Arithmetic: FP64.  Every per-sample expression is evaluated in the order
// the reference writes it, with no contraction (the build compiles this file
// with -fmad=false), so a plain C restatement compiled without contraction
// gives the same bits.  The operator products (dense ns x nd operators times
// every shape's positions) are FP64 library GEMMs.
#include <cublas_v2.h>
#include <string>
#include "ibk_internal.h"

struct ibk_surface_plan_s {
	int ns = 0, nd = 0, device = 0;
	int dims = 2;                   // 2: surfaces in 3-D; 1: curves in 2-D (ops[0], ops[1], ops[3] only)
	const double* ops[6] = {};
	const double* weights = nullptr;
	cublasHandle_t blas = nullptr;
	double* scratch = nullptr;      // bending's intermediate fields, grown on use
	size_t scratch_bytes = 0;
	const double** gemm_ptrs = nullptr;   // device pointer arrays of a batched product: A[6], B[6], C[6]
};

namespace ibk {
namespace {

constexpr int kMembraneThreads = 256;

struct V3 { double x, y, z; };

// Vector quantity of sample i in [component][site] blocks of m values.
__device__ __forceinline__ V3 load3(const double* __restrict__ p, long long m, long long i)
{
	return {__ldg(p + i), __ldg(p + m + i), __ldg(p + 2 * m + i)};
}

// algo::dot (include/algo/dot.h:8-14): a left fold of the products.
__device__ __forceinline__ double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Metric, its derivatives and the area element of one configuration
// (tension.h:35-51): g_ij = t_i . t_j; with the Christoffel symbols of the
// first kind G_ij,k = t_ij . t_k (include/forces/load.h:311-341),
// g_ij,k = G_ik,j + G_kj,i.
struct Metric {
	double e, f, g;
	double eu, fu, gu, ev, fv, gv;
	double i, iu, iv;
};

__device__ __forceinline__ Metric metric(const V3& u, const V3& v, const V3& uu, const V3& uv, const V3& vv)
{
	Metric m;
	m.e = dot(u, u);
	m.f = dot(u, v);
	m.g = dot(v, v);
	const double uu_u = dot(uu, u), uu_v = dot(uu, v);
	const double uv_u = dot(uv, u), uv_v = dot(uv, v);
	const double vv_u = dot(vv, u), vv_v = dot(vv, v);
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

// Strain energy density derivatives w1, w2, w11, w12, w22 of a law at the
// invariants (i1, i2).
struct LawValues { double w1, w2, w11, w12, w22; };

template <int LAW>
__device__ __forceinline__ LawValues law_values(double e, double kappa, double i1, double i2)
{
	if constexpr (LAW == IBK_LAW_SKALAK) {
		// skalak.h:22-31
		return {e * (i1 - 1), (kappa * (i2 - 1) - e), e, 0.0, kappa};
	} else if constexpr (LAW == IBK_LAW_HOOKEAN) {
		// hookean.h:19-30: a function of i1 alone; kappa unused
		const double j = sqrt(i1);
		return {e * (1 - 1. / j), 0.0, e / (2 * i1 * j), 0.0, 0.0};
	} else {
		// neohookean.h:22-32
		const double j = sqrt(i2);
		const double w1 = e / j;
		const double w2 = kappa * (1 - 1 / j) - 0.5 * w1 * i1 / i2;
		const double w12 = -0.5 * w1 / i2;
		const double w22 = 0.75 * w1 * i1 / (i2 * i2) + 0.5 * kappa / (i2 * j);
		return {w1, w2, 0.0, w12, w22};
	}
}

struct SurfaceIn {
	const double* t[2];
	const double* tt[3];
	const double* sigma;
};

// tension.h:71-112, one thread per sample site.
template <int LAW>
__global__ void __launch_bounds__(kMembraneThreads)
tension_kernel(long long n, SurfaceIn rest, SurfaceIn cur, double e, double kappa, double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const Metric o = metric(load3(rest.t[0], n, p), load3(rest.t[1], n, p), load3(rest.tt[0], n, p),
	                        load3(rest.tt[1], n, p), load3(rest.tt[2], n, p));
	const V3 u = load3(cur.t[0], n, p), v = load3(cur.t[1], n, p);
	const V3 uu = load3(cur.tt[0], n, p), uv = load3(cur.tt[1], n, p), vv = load3(cur.tt[2], n, p);
	const Metric c = metric(u, v, uu, uv, vv);
	const double os = __ldg(rest.sigma + p);

	// invariants and their derivatives
	const double i1 = (c.e * o.g + o.e * c.g - 2 * o.f * c.f) / o.i;
	const double i2 = c.i / o.i;
	const double i1u = (c.eu * o.g + c.e * o.gu + o.eu * c.g + o.e * c.gu - 2 * (o.fu * c.f + o.f * c.fu) - i1 * o.iu) / o.i;
	const double i1v = (c.ev * o.g + c.e * o.gv + o.ev * c.g + o.e * c.gv - 2 * (o.fv * c.f + o.f * c.fv) - i1 * o.iv) / o.i;
	const double i2u = (c.iu - i2 * o.iu) / o.i;
	const double i2v = (c.iv - i2 * o.iv) / o.i;

	const LawValues w = law_values<LAW>(e, kappa, i1, i2);
	const double w1u = w.w11 * i1u + w.w12 * i2u;
	const double w1v = w.w11 * i1v + w.w12 * i2v;
	const double w2u = w.w12 * i1u + w.w22 * i2u;
	const double w2v = w.w12 * i1v + w.w22 * i2v;

	// the per-sample factors the reference repeats in each component's sum
	const double ag = w.w1 * o.g + w.w2 * c.g;
	const double af = w.w1 * o.f + w.w2 * c.f;
	const double ae = w.w1 * o.e + w.w2 * c.e;
	const double oi2 = 2 * o.i;
	const double kgu = ag * o.iu / oi2, kfv = af * o.iv / oi2, kfu = af * o.iu / oi2, kev = ae * o.iv / oi2;
	const double du = w1u * o.g + w.w1 * o.gu + w2u * c.g + w.w2 * c.gu;
	const double dv1 = w1v * o.f + w.w1 * o.fv + w2v * c.f + w.w2 * c.fv;
	const double du1 = w1u * o.f + w.w1 * o.fu + w2u * c.f + w.w2 * c.fu;
	const double dv = w1v * o.e + w.w1 * o.ev + w2v * c.e + w.w2 * c.ev;
	const double scale = os / o.i;
	const double uc[3] = {u.x, u.y, u.z}, vc[3] = {v.x, v.y, v.z};
	const double uuc[3] = {uu.x, uu.y, uu.z}, uvc[3] = {uv.x, uv.y, uv.z}, vvc[3] = {vv.x, vv.y, vv.z};
#pragma unroll
	for (int k = 0; k < 3; ++k) {
		f[k * n + p] = scale * (
			+ ag * uuc[k]
			- 2 * af * uvc[k]
			+ ae * vvc[k]
			- kgu * uc[k]
			+ kfv * uc[k]
			+ kfu * vc[k]
			- kev * vc[k]
			+ du * uc[k]
			- dv1 * uc[k]
			- du1 * vc[k]
			+ dv * vc[k]);
	}
}

// geometry.h:95-119: the normal t_u x t_v / |t_u x t_v| (algo::cross of the
// two tangents) and the patch area weight * |t_u x t_v| of every sample.
__global__ void __launch_bounds__(kMembraneThreads)
surface_metrics_kernel(long long n, int ns, const double* __restrict__ tu, const double* __restrict__ tv,
                       const double* __restrict__ weights, double* __restrict__ normal, double* __restrict__ sigma)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const V3 a = load3(tu, n, p), b = load3(tv, n, p);
	const V3 c = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
	const double detf = sqrt(dot(c, c));
	if (normal) {
		normal[p] = c.x / detf;
		normal[n + p] = c.y / detf;
		normal[2 * n + p] = c.z / detf;
	}
	sigma[p] = __ldg(weights + p % ns) * detf;
}

// Mean and Gaussian curvature of a sample (bending.h:46-74): metric
// (e, f, g) and second fundamental form (l, k, m) = t_ij . n.
struct Curvatures { double h, k; };

__device__ __forceinline__ Curvatures curvatures(const V3& u, const V3& v, const V3& uu, const V3& uv, const V3& vv,
                                                 const V3& n)
{
	const double e = dot(u, u), f = dot(u, v), g = dot(v, v);
	const double l = dot(uu, n), k = dot(uv, n), m = dot(vv, n);
	return {(l * g + m * e - 2 * k * f) / (2 * (e * g - f * f)), (l * m - k * k) / (e * g - f * f)};
}

struct SurfaceFull {
	const double* t[2];
	const double* tt[3];
	const double* normal;
	const double* sigma;
};

__device__ __forceinline__ Curvatures curvatures_at(const SurfaceFull& s, long long n, long long p)
{
	return curvatures(load3(s.t[0], n, p), load3(s.t[1], n, p), load3(s.tt[0], n, p), load3(s.tt[1], n, p),
	                  load3(s.tt[2], n, p), load3(s.normal, n, p));
}

// Mean curvature field at the data sites (bending.h:151-158): H of the
// current shape, minus H of the rest shape (h0) when one is given.
__global__ void __launch_bounds__(kMembraneThreads)
mean_curvature_kernel(long long n, SurfaceFull s, const double* __restrict__ h0, double* __restrict__ h)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	double v = curvatures_at(s, n, p).h;
	if (h0) v -= h0[p];
	h[p] = v;
}

// Bending force at the samples (bending.h:164-181 and 186-224): the surface
// Laplacian of the mean-curvature field from its derivatives (hd: u, v, uu,
// uv, vv) and the current metric, plus 2 (H - H0)(H^2 - K + H H0), times
// -4 kappa sigma along the normal.
__global__ void __launch_bounds__(kMembraneThreads)
bending_kernel(long long n, SurfaceFull cur, SurfaceFull rest, int preferred, const double* __restrict__ hd,
               double modulus, double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const V3 u = load3(cur.t[0], n, p), v = load3(cur.t[1], n, p);
	const V3 uu = load3(cur.tt[0], n, p), uv = load3(cur.tt[1], n, p), vv = load3(cur.tt[2], n, p);
	const V3 nrm = load3(cur.normal, n, p);
	const Metric x = metric(u, v, uu, uv, vv);
	const double hu = hd[p], hv = hd[n + p], huu = hd[2 * n + p], huv = hd[3 * n + p], hvv = hd[4 * n + p];
	const double lh = (((- x.iu * x.g + x.iv * x.f) / (2 * x.i) + x.gu - x.fv) / x.i * hu +
	                   ((+ x.iu * x.f - x.iv * x.e) / (2 * x.i) - x.fu + x.ev) / x.i * hv) +
	                  x.g / x.i * huu - 2 * x.f / x.i * huv + x.e / x.i * hvv;
	const Curvatures c = curvatures(u, v, uu, uv, vv, nrm);
	double dh = c.h;
	double sh = c.h * c.h - c.k;
	if (preferred) {
		const double h0 = curvatures_at(rest, n, p).h;
		dh -= h0;
		sh += c.h * h0;
	}
	const double b = lh + 2 * (dh * sh);
	const double mag = -4 * __ldg(cur.sigma + p) * modulus * b;
	f[p] = mag * nrm.x;
	f[n + p] = mag * nrm.y;
	f[2 * n + p] = mag * nrm.z;
}

// Curves in two-dimensional runs: bases::geometry<1> (geometry.h:74-124 with
// one tangent over two components, whose algo::cross is (t1, -t0)) and
// forces::tension1d (tension.h:120-205).
__device__ __forceinline__ double dot2(double a0, double a1, double b0, double b1) { return a0 * b0 + a1 * b1; }

__global__ void __launch_bounds__(kMembraneThreads)
curve_metrics_kernel(long long n, int ns, const double* __restrict__ t, const double* __restrict__ weights,
                     double* __restrict__ normal, double* __restrict__ sigma)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const double c0 = __ldg(t + n + p), c1 = -__ldg(t + p);
	const double detf = sqrt(dot2(c0, c1, c0, c1));
	if (normal) {
		normal[p] = c0 / detf;
		normal[n + p] = c1 / detf;
	}
	sigma[p] = __ldg(weights + p % ns) * detf;
}

// tension.h:172-200 with the skalak1d (skalak.h:49-55) or hookean1d
// (hookean.h:48-54) law of the stretch invariant i = |t|^2 / |t0|^2.
template <int LAW>
__global__ void __launch_bounds__(kMembraneThreads)
curve_tension_kernel(long long n, SurfaceIn rest, SurfaceIn cur, double e, double kappa, double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const double ou0 = __ldg(rest.t[0] + p), ou1 = __ldg(rest.t[0] + n + p);
	const double ouu0 = __ldg(rest.tt[0] + p), ouu1 = __ldg(rest.tt[0] + n + p);
	const double u0 = __ldg(cur.t[0] + p), u1 = __ldg(cur.t[0] + n + p);
	const double uu0 = __ldg(cur.tt[0] + p), uu1 = __ldg(cur.tt[0] + n + p);
	const double oi = dot2(ou0, ou1, ou0, ou1), odi = 2 * dot2(ouu0, ouu1, ou0, ou1);
	const double ci = dot2(u0, u1, u0, u1), cdi = 2 * dot2(uu0, uu1, u0, u1);
	const double i = ci / oi;
	const double iu = (cdi - i * odi) / oi;
	double phi, phi1;
	if constexpr (LAW == IBK_LAW_SKALAK) {
		phi = e * (i - 1) - kappa * i * (i * i - 1);
		phi1 = e - kappa * (3 * i * i - 1);
	} else {
		const double j = sqrt(i);
		phi = e * (1 - 1. / j);
		phi1 = e / (2 * i * j);
	}
	const double phiu = phi1 * iu;
	const double scale = __ldg(rest.sigma + p) / oi;
	const double uc[2] = {u0, u1}, uuc[2] = {uu0, uu1};
#pragma unroll
	for (int k = 0; k < 2; ++k)
		f[k * n + p] = scale * (+ phi * uuc[k] - odi / (2 * oi) * phi * uc[k] + phiu * uc[k]);
}

// Viscous dissipation at the samples (dissipation.h:216-265): the rate of
// change of the metric and of the Christoffel symbols from the velocity's
// derivatives (vd: u, v, uu, uv, vv, each 3n values [component][site]) and
// the current geometry, the in-plane stress g^-1 g' adj(g) they give and its
// surface divergence, times kappa sigma / det g.
__global__ void __launch_bounds__(kMembraneThreads)
dissipation_kernel(long long n, SurfaceIn cur, const double* __restrict__ vd, double kappa, double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const V3 tu = load3(cur.t[0], n, p), tv = load3(cur.t[1], n, p);
	const V3 tuu = load3(cur.tt[0], n, p), tuv = load3(cur.tt[1], n, p), tvv = load3(cur.tt[2], n, p);
	const V3 su = load3(vd, n, p), sv = load3(vd + 3 * n, n, p);
	const V3 suu = load3(vd + 6 * n, n, p), suv = load3(vd + 9 * n, n, p), svv = load3(vd + 12 * n, n, p);
	const Metric m = metric(tu, tv, tuu, tuv, tvv);
	const double e = m.e, ff = m.f, g = m.g, eu = m.eu, fu = m.fu, gu = m.gu, ev = m.ev, fv = m.fv, gv = m.gv;
	const double i = m.i, iu = m.iu, iv = m.iv;

	// dot_metric: g'_ij = t_i . u_j + u_i . t_j (dissipation.h:57-79)
	const double de = dot(tu, su) + dot(su, tu);
	const double df = dot(tu, sv) + dot(su, tv);
	const double dg = dot(tv, sv) + dot(sv, tv);
	// dot_christoffel: G'_ij,k = u_ij . t_k + t_ij . u_k (dissipation.h:89-127),
	// and g'_ij,k = G'_ik,j + G'_kj,i (dissipation.h:193-206)
	const double c00_0 = dot(suu, tu) + dot(tuu, su), c00_1 = dot(suu, tv) + dot(tuu, sv);
	const double c01_0 = dot(suv, tu) + dot(tuv, su), c01_1 = dot(suv, tv) + dot(tuv, sv);
	const double c11_0 = dot(svv, tu) + dot(tvv, su), c11_1 = dot(svv, tv) + dot(tvv, sv);
	const double deu = 2 * c00_0, dfu = c00_1 + c01_0, dgu = 2 * c01_1;
	const double dev = 2 * c01_0, dfv = c01_1 + c11_0, dgv = 2 * c11_1;

	const double pig[4] = {(g * de - ff * df) / i, (g * df - ff * dg) / i,
	                       (e * df - ff * de) / i, (e * dg - ff * df) / i};
	const double pigu[4] = {
		(gu * de + g * deu - fu * df - ff * dfu - iu * pig[0]) / i,
		(gu * df + g * dfu - fu * dg - ff * dgu - iu * pig[1]) / i,
		(eu * df + e * dfu - fu * de - ff * deu - iu * pig[2]) / i,
		(eu * dg + e * dgu - fu * df - ff * dfu - iu * pig[3]) / i};
	const double pigv[4] = {
		(gv * de + g * dev - fv * df - ff * dfv - iv * pig[0]) / i,
		(gv * df + g * dfv - fv * dg - ff * dgv - iv * pig[1]) / i,
		(ev * df + e * dfv - fv * de - ff * dev - iv * pig[2]) / i,
		(ev * dg + e * dgv - fv * df - ff * dfv - iv * pig[3]) / i};
	const double pif[3] = {
		pig[0] * g - pig[1] * ff,
		0.5 * (pig[1] * e + pig[2] * g - (pig[0] + pig[3]) * ff),
		pig[3] * e - pig[2] * ff};
	const double pifu[3] = {
		pigu[0] * g + pig[0] * gu - pigu[1] * ff - pig[1] * fu,
		0.5 * (pigu[1] * e + pig[1] * eu + pigu[2] * g + pig[2] * gu
		       - ((pigu[0] + pigu[3]) * ff + (pig[0] + pig[3]) * fu)),
		pigu[3] * e + pig[3] * eu - pigu[2] * ff - pig[2] * fu};
	const double pifv[3] = {
		pigv[0] * g + pig[0] * gv - pigv[1] * ff - pig[1] * fv,
		0.5 * (pigv[1] * e + pig[1] * ev + pigv[2] * g + pig[2] * gv
		       - ((pigv[0] + pigv[3]) * ff + (pig[0] + pig[3]) * fv)),
		pigv[3] * e + pig[3] * ev - pigv[2] * ff - pig[2] * fv};
	const double c0 = pifu[0] + pifv[1] - (iu * pif[0] + iv * pif[1]) / (2 * i);
	const double c1 = pifu[1] + pifv[2] - (iu * pif[1] + iv * pif[2]) / (2 * i);

	const double scale = __ldg(cur.sigma + p) * kappa / i;
	const double two_pif1 = 2 * pif[1];
	const double uc[3] = {tu.x, tu.y, tu.z}, vc[3] = {tv.x, tv.y, tv.z};
	const double uuc[3] = {tuu.x, tuu.y, tuu.z}, uvc[3] = {tuv.x, tuv.y, tuv.z}, vvc[3] = {tvv.x, tvv.y, tvv.z};
#pragma unroll
	for (int k = 0; k < 3; ++k)
		f[k * n + p] = scale * (c0 * uc[k] + c1 * vc[k] + pif[0] * uuc[k] + two_pif1 * uvc[k] + pif[2] * vvc[k]);
}

// Tether (tether.h:14-22): modulus (x_rest - x_current), element by element
// over 3n values.
__global__ void __launch_bounds__(kMembraneThreads)
tether_kernel(long long m, const double* __restrict__ xr, const double* __restrict__ xc, double modulus,
              double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= m) return;
	f[p] = modulus * (__ldg(xr + p) - __ldg(xc + p));
}

// Wall repulsion (repelling.h:15-45): r = |height - y| / range and, inside
// r < 2, fy = -log(r / 2) exp(-4 / (4 - r^2)); f = -modulus (0, fy, 0) sigma.
__global__ void __launch_bounds__(kMembraneThreads)
repelling_kernel(long long n, const double* __restrict__ x, const double* __restrict__ sigma, double modulus,
                 double height, double range, double* __restrict__ f)
{
	const long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	const double r = fabs(height - __ldg(x + n + p)) / range;
	const double fy = r < 2 ? -log(r / 2) * exp(-4 / (4 - r * r)) : 0.0;
	const double fc[3] = {0.0, fy, 0.0};
	const double s = __ldg(sigma + p);
#pragma unroll
	for (int k = 0; k < 3; ++k) f[k * n + p] = -modulus * fc[k] * s;
}

ibk_status blas_check(cublasStatus_t st, const char* what)
{
	if (st == CUBLAS_STATUS_SUCCESS) return IBK_OK;
	return set_error(IBK_ERR_CUDA, std::string(what) + ": cuBLAS status " + std::to_string((int) st));
}

int blocks_of(long long n) { return (int) ((n + kMembraneThreads - 1) / kMembraneThreads); }

// Pointer arrays of one batched product, written on the stream (so a call
// needs no host-to-device copy and stays in stream order).
struct GemmPtrs {
	const double* a[6];
	const double* b;
	double* c[6];
	int count;
};

__global__ void gemm_ptrs_kernel(GemmPtrs g, const double** dst)
{
	const int i = threadIdx.x;
	if (i < g.count) {
		dst[i] = g.a[i];
		dst[6 + i] = g.b;
		dst[12 + i] = g.c[i];
	}
}

// Operator products of one plan: out[q] = ops[q] (ns x nd) * y (nd x cols),
// column-major, for the q with out[q] set (q = 0: evaluation, a copy when
// the plan has none).  The products go to the library as one batched call:
// one product of ns x cols outputs fills only part of the GPU's last wave of
// tiles, several together fill it.
ibk_status apply_ops(ibk_surface_plan_s& plan, int cols, const double* y, double* const* out, cudaStream_t s)
{
	ibk_status st = blas_check(cublasSetStream(plan.blas, s), "cublasSetStream");
	if (st != IBK_OK) return st;
	const double one = 1.0, zero = 0.0;
	GemmPtrs g{};
	g.b = y;
	for (int q = 0; q < 6; ++q) {
		if (!out[q]) continue;
		if (q == 0 && !plan.ops[0]) {
			// samples are the data sites: the values themselves (geometry.h:43-49)
			const cudaError_t e = cudaMemcpyAsync(out[0], y, sizeof(double) * (size_t) plan.nd * cols,
			                                      cudaMemcpyDeviceToDevice, s);
			if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
			continue;
		}
		g.a[g.count] = plan.ops[q];
		g.c[g.count] = out[q];
		++g.count;
	}
	if (g.count == 0) return IBK_OK;
	if (g.count == 1)
		return blas_check(cublasDgemm(plan.blas, CUBLAS_OP_N, CUBLAS_OP_N, plan.ns, cols, plan.nd, &one, g.a[0],
		                              plan.ns, y, plan.nd, &zero, g.c[0], plan.ns), "cublasDgemm");
	gemm_ptrs_kernel<<<1, 32, 0, s>>>(g, plan.gemm_ptrs);
	if ((st = check_launch("gemm_ptrs_kernel")) != IBK_OK) return st;
	return blas_check(cublasDgemmBatched(plan.blas, CUBLAS_OP_N, CUBLAS_OP_N, plan.ns, cols, plan.nd, &one,
	                                     plan.gemm_ptrs, plan.ns, plan.gemm_ptrs + 6, plan.nd, &zero,
	                                     const_cast<double**>(plan.gemm_ptrs + 12), plan.ns, g.count),
	                  "cublasDgemmBatched");
}

ibk_status geometry_impl(ibk_surface_plan_s& plan, int nc, const double* x, const ibk_surface& out, cudaStream_t s)
{
	if (plan.dims == 1) {
		double* outs[6] = {out.position, out.t[0], nullptr, out.tt[0], nullptr, nullptr};
		const ibk_status st = apply_ops(plan, 2 * nc, x, outs, s);
		if (st != IBK_OK) return st;
		const long long n = (long long) plan.ns * nc;
		curve_metrics_kernel<<<blocks_of(n), kMembraneThreads, 0, s>>>(n, plan.ns, out.t[0], plan.weights,
		                                                               out.normal, out.sigma);
		return check_launch("curve_metrics_kernel");
	}
	double* outs[6] = {out.position, out.t[0], out.t[1], out.tt[0], out.tt[1], out.tt[2]};
	const ibk_status st = apply_ops(plan, 3 * nc, x, outs, s);
	if (st != IBK_OK) return st;
	const long long n = (long long) plan.ns * nc;
	surface_metrics_kernel<<<blocks_of(n), kMembraneThreads, 0, s>>>(n, plan.ns, out.t[0], out.t[1], plan.weights,
	                                                                 out.normal, out.sigma);
	return check_launch("surface_metrics_kernel");
}

ibk_status grow_scratch(ibk_surface_plan_s& plan, size_t bytes, cudaStream_t s)
{
	if (plan.scratch_bytes >= bytes) return IBK_OK;
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap != cudaStreamCaptureStatusNone)
		return set_error(IBK_ERR_CAPACITY, "surface plan scratch must grow during stream capture");
	cudaError_t e = cudaStreamSynchronize(s);
	if (e != cudaSuccess) return set_error(IBK_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
	if (plan.scratch) cudaFree(plan.scratch);
	plan.scratch = nullptr;
	plan.scratch_bytes = 0;
	e = cudaMalloc(reinterpret_cast<void**>(&plan.scratch), bytes);
	if (e != cudaSuccess) {
		cudaGetLastError();
		plan.scratch = nullptr;
		return set_error(IBK_ERR_OUT_OF_MEMORY, "cudaMalloc of surface plan scratch failed");
	}
	plan.scratch_bytes = bytes;
	return IBK_OK;
}

// cuBLAS handle and the batched products' pointer arrays of a new plan.
ibk_status finish_plan(ibk_surface_plan_s* plan, ibk_surface_plan* out)
{
	cudaGetDevice(&plan->device);
	ibk_status st = blas_check(cublasCreate(&plan->blas), "cublasCreate");
	if (st == IBK_OK && cudaMalloc(reinterpret_cast<void**>(&plan->gemm_ptrs), 18 * sizeof(double*)) != cudaSuccess) {
		cudaGetLastError();
		plan->gemm_ptrs = nullptr;
		st = set_error(IBK_ERR_OUT_OF_MEMORY, "cudaMalloc of the product pointer arrays failed");
	}
	if (st != IBK_OK) {
		if (plan->blas) cublasDestroy(plan->blas);
		delete plan;
		return st;
	}
	*out = plan;
	return IBK_OK;
}

SurfaceFull full(const ibk_surface& g)
{
	return SurfaceFull{{g.t[0], g.t[1]}, {g.tt[0], g.tt[1], g.tt[2]}, g.normal, g.sigma};
}

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_surface_plan_create(int ns, int nd, const double* const* ops, const double* weights,
                                   ibk_surface_plan* out)
{
	if (!out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null output handle");
	*out = nullptr;
	if (ns <= 0 || nd <= 0 || !ops || !weights)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "sizes must be positive, operators and weights given");
	for (int q = 1; q < 6; ++q)
		if (!ops[q]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null derivative operator");
	if (!ops[0] && ns != nd)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "without an evaluation operator the samples are the data sites (ns == nd)");
	auto* plan = new ibk_surface_plan_s;
	plan->ns = ns;
	plan->nd = nd;
	for (int q = 0; q < 6; ++q) plan->ops[q] = ops[q];
	plan->weights = weights;
	return finish_plan(plan, out);
}

ibk_status ibk_curve_plan_create(int ns, int nd, const double* const* ops, const double* weights,
                                 ibk_surface_plan* out)
{
	if (!out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null output handle");
	*out = nullptr;
	if (ns <= 0 || nd <= 0 || !ops || !weights)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "sizes must be positive, operators and weights given");
	if (!ops[1] || !ops[2]) return set_error(IBK_ERR_INVALID_ARGUMENT, "null derivative operator");
	if (!ops[0] && ns != nd)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "without an evaluation operator the samples are the data sites (ns == nd)");
	auto* plan = new ibk_surface_plan_s;
	plan->ns = ns;
	plan->nd = nd;
	plan->dims = 1;
	plan->ops[0] = ops[0];
	plan->ops[1] = ops[1];
	plan->ops[3] = ops[2];
	plan->weights = weights;
	return finish_plan(plan, out);
}

ibk_status ibk_surface_plan_destroy(ibk_surface_plan plan)
{
	if (!plan) return IBK_OK;
	int dev = 0;
	cudaGetDevice(&dev);
	cudaSetDevice(plan->device);
	if (plan->blas) cublasDestroy(plan->blas);
	if (plan->scratch) cudaFree(plan->scratch);
	if (plan->gemm_ptrs) cudaFree(plan->gemm_ptrs);
	cudaSetDevice(dev);
	delete plan;
	return IBK_OK;
}

ibk_status ibk_surface_geometry(ibk_surface_plan plan, int nc, const double* x, const ibk_surface* out, void* stream)
{
	if (!plan || !out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or output");
	if (nc < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "negative shape count");
	if (nc == 0) return IBK_OK;
	if (plan->dims == 1) {
		if (!x || !out->t[0] || !out->tt[0] || !out->sigma)
			return set_error(IBK_ERR_INVALID_ARGUMENT, "null positions, tangent, second derivative or lengths");
		return geometry_impl(*plan, nc, x, *out, static_cast<cudaStream_t>(stream));
	}
	if (!x || !out->t[0] || !out->t[1] || !out->tt[0] || !out->tt[1] || !out->tt[2] || !out->sigma)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null positions, tangents, second derivatives or areas");
	return geometry_impl(*plan, nc, x, *out, static_cast<cudaStream_t>(stream));
}

ibk_status ibk_membrane_tension(int law, double shear, double bulk, int npoints, const ibk_surface* rest,
                                const ibk_surface* current, double* f, void* stream)
{
	if (law != IBK_LAW_SKALAK && law != IBK_LAW_NEOHOOKEAN && law != IBK_LAW_HOOKEAN)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "unknown tension law");
	if (npoints <= 0) return IBK_OK;
	if (!rest || !current || !f) return set_error(IBK_ERR_INVALID_ARGUMENT, "null geometry or force array");
	const ibk_surface* g[2] = {rest, current};
	for (const ibk_surface* q : g)
		if (!q->t[0] || !q->t[1] || !q->tt[0] || !q->tt[1] || !q->tt[2])
			return set_error(IBK_ERR_INVALID_ARGUMENT, "null tangents or second derivatives");
	if (!rest->sigma) return set_error(IBK_ERR_INVALID_ARGUMENT, "null rest patch areas");
	SurfaceIn r{{rest->t[0], rest->t[1]}, {rest->tt[0], rest->tt[1], rest->tt[2]}, rest->sigma};
	SurfaceIn c{{current->t[0], current->t[1]}, {current->tt[0], current->tt[1], current->tt[2]}, nullptr};
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const long long n = npoints;
	if (law == IBK_LAW_SKALAK)
		tension_kernel<IBK_LAW_SKALAK><<<blocks_of(n), kMembraneThreads, 0, s>>>(n, r, c, shear, bulk, f);
	else if (law == IBK_LAW_NEOHOOKEAN)
		tension_kernel<IBK_LAW_NEOHOOKEAN><<<blocks_of(n), kMembraneThreads, 0, s>>>(n, r, c, shear, bulk, f);
	else
		tension_kernel<IBK_LAW_HOOKEAN><<<blocks_of(n), kMembraneThreads, 0, s>>>(n, r, c, shear, bulk, f);
	return check_launch("tension_kernel");
}

ibk_status ibk_curve_tension(int law, double shear, double bulk, int npoints, const ibk_surface* rest,
                             const ibk_surface* current, double* f, void* stream)
{
	if (law != IBK_LAW_SKALAK && law != IBK_LAW_HOOKEAN)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "curves take the Skalak or Hookean law");
	if (npoints <= 0) return IBK_OK;
	if (!rest || !current || !f) return set_error(IBK_ERR_INVALID_ARGUMENT, "null geometry or force array");
	if (!rest->t[0] || !rest->tt[0] || !rest->sigma || !current->t[0] || !current->tt[0])
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null tangent, second derivative or rest lengths");
	SurfaceIn r{{rest->t[0], nullptr}, {rest->tt[0], nullptr, nullptr}, rest->sigma};
	SurfaceIn c{{current->t[0], nullptr}, {current->tt[0], nullptr, nullptr}, nullptr};
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const long long n = npoints;
	if (law == IBK_LAW_SKALAK)
		curve_tension_kernel<IBK_LAW_SKALAK><<<blocks_of(n), kMembraneThreads, 0, s>>>(n, r, c, shear, bulk, f);
	else
		curve_tension_kernel<IBK_LAW_HOOKEAN><<<blocks_of(n), kMembraneThreads, 0, s>>>(n, r, c, shear, bulk, f);
	return check_launch("curve_tension_kernel");
}

ibk_status ibk_membrane_dissipation(ibk_surface_plan sample_plan, double modulus, int nc, const double* u,
                                    const ibk_surface* current, double* f, void* stream)
{
	if (!sample_plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null surface plan");
	if (sample_plan->dims != 2) return set_error(IBK_ERR_INVALID_ARGUMENT, "dissipation acts on surfaces, not curves");
	if (nc < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "negative shape count");
	if (nc == 0) return IBK_OK;
	if (!u || !current || !f) return set_error(IBK_ERR_INVALID_ARGUMENT, "null velocity, geometry or force array");
	if (!current->t[0] || !current->t[1] || !current->tt[0] || !current->tt[1] || !current->tt[2] || !current->sigma)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null sample tangents, second derivatives or patch areas");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const long long n = (long long) sample_plan->ns * nc;
	// scratch: the velocity's five derivatives at the samples (dissipation.h:41-53)
	ibk_status st = grow_scratch(*sample_plan, sizeof(double) * (size_t) (15 * n), s);
	if (st != IBK_OK) return st;
	double* vd = sample_plan->scratch;
	double* outs[6] = {nullptr, vd, vd + 3 * n, vd + 6 * n, vd + 9 * n, vd + 12 * n};
	if ((st = apply_ops(*sample_plan, 3 * nc, u, outs, s)) != IBK_OK) return st;
	SurfaceIn c{{current->t[0], current->t[1]}, {current->tt[0], current->tt[1], current->tt[2]}, current->sigma};
	dissipation_kernel<<<blocks_of(n), kMembraneThreads, 0, s>>>(n, c, vd, modulus, f);
	return check_launch("dissipation_kernel");
}

ibk_status ibk_membrane_tether(double modulus, int npoints, const ibk_surface* rest, const ibk_surface* current,
                               double* f, void* stream)
{
	if (npoints <= 0) return IBK_OK;
	if (!rest || !current || !rest->position || !current->position || !f)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null positions or force array");
	const long long m = 3LL * npoints;
	tether_kernel<<<blocks_of(m), kMembraneThreads, 0, static_cast<cudaStream_t>(stream)>>>(
		m, rest->position, current->position, modulus, f);
	return check_launch("tether_kernel");
}

ibk_status ibk_membrane_repelling(double modulus, double height, double range, int npoints,
                                  const ibk_surface* current, double* f, void* stream)
{
	if (npoints <= 0) return IBK_OK;
	if (!current || !current->position || !current->sigma || !f)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null positions, patch areas or force array");
	if (!(range > 0)) return set_error(IBK_ERR_INVALID_ARGUMENT, "the repulsion range must be positive");
	const long long n = npoints;
	repelling_kernel<<<blocks_of(n), kMembraneThreads, 0, static_cast<cudaStream_t>(stream)>>>(
		n, current->position, current->sigma, modulus, height, range, f);
	return check_launch("repelling_kernel");
}

ibk_status ibk_membrane_bending(ibk_surface_plan data_plan, ibk_surface_plan sample_plan, double modulus,
                                int preferred, int nc, const double* x_rest, const double* x_current,
                                const ibk_surface* rest, const ibk_surface* current, double* f, void* stream)
{
	if (!data_plan || !sample_plan) return set_error(IBK_ERR_INVALID_ARGUMENT, "null surface plan");
	if (nc < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "negative shape count");
	if (nc == 0) return IBK_OK;
	if (data_plan->dims != 2 || sample_plan->dims != 2)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "bending acts on surfaces, not curves");
	if (data_plan->ns != data_plan->nd || sample_plan->nd != data_plan->nd)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "the data plan must map the data sites to themselves, "
		                                           "and both plans must share them");
	if (!x_current || !current || !f || (preferred && (!x_rest || !rest)))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null positions, geometry or force array");
	const ibk_surface* need[2] = {current, preferred ? rest : current};
	for (const ibk_surface* q : need)
		if (!q->t[0] || !q->t[1] || !q->tt[0] || !q->tt[1] || !q->tt[2] || !q->normal)
			return set_error(IBK_ERR_INVALID_ARGUMENT, "null sample tangents, second derivatives or normals");
	if (!current->sigma) return set_error(IBK_ERR_INVALID_ARGUMENT, "null current patch areas");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const long long nd = data_plan->nd, ns = sample_plan->ns;
	const size_t doubles = (size_t) (21 * nd + 5 * ns) * nc;
	ibk_status st = grow_scratch(*sample_plan, sizeof(double) * doubles, s);
	if (st != IBK_OK) return st;
	// scratch: data geometry (t, tt, normal: 3 nd nc each; sigma), h, h0, h's
	// derivatives at the samples
	double* w = sample_plan->scratch;
	const long long m = nd * nc;
	ibk_surface dg{};
	dg.t[0] = w; dg.t[1] = w + 3 * m;
	dg.tt[0] = w + 6 * m; dg.tt[1] = w + 9 * m; dg.tt[2] = w + 12 * m;
	dg.normal = w + 15 * m;
	dg.sigma = w + 18 * m;
	double* h = w + 19 * m;
	double* h0 = w + 20 * m;
	double* hd = w + 21 * m;
	if (preferred) {
		if ((st = geometry_impl(*data_plan, nc, x_rest, dg, s)) != IBK_OK) return st;
		mean_curvature_kernel<<<blocks_of(m), kMembraneThreads, 0, s>>>(m, full(dg), nullptr, h0);
		if ((st = check_launch("mean_curvature_kernel")) != IBK_OK) return st;
	}
	if ((st = geometry_impl(*data_plan, nc, x_current, dg, s)) != IBK_OK) return st;
	mean_curvature_kernel<<<blocks_of(m), kMembraneThreads, 0, s>>>(m, full(dg), preferred ? h0 : nullptr, h);
	if ((st = check_launch("mean_curvature_kernel")) != IBK_OK) return st;
	// derivatives of the curvature field at the samples (bending.h:100-124)
	const long long n = ns * nc;
	double* outs[6] = {nullptr, hd, hd + n, hd + 2 * n, hd + 3 * n, hd + 4 * n};
	if ((st = apply_ops(*sample_plan, nc, h, outs, s)) != IBK_OK) return st;
	bending_kernel<<<blocks_of(n), kMembraneThreads, 0, s>>>(n, full(*current), full(preferred ? *rest : *current),
	                                                         preferred, hd, modulus, f);
	return check_launch("bending_kernel");
}

} // extern "C"
