// The fluid step that consumes the spread's force density: one implicit
// diffusion step of a component grid (ins::diffusion,
// include/ins/diffusion.h:12-78),
//     out = u + (I~ - lambda L)^-1 (k I~ f + k mu (L u + rhs)),
// with L the second-order finite-difference Laplacian and I~ the
// boundary-corrected identity (fd::laplacian, fd::identity with
// correction::second_order).  Both are Kronecker sums / products of 1-D
// operators (include/fd/combine.h:24-30): along an axis L_d is the 3-point
// Laplacian res^2 (1, -2, 1) with a wrap entry per corner on a periodic axis,
// or on a solid axis the ghost-point weight of each wall added to its corner
// diagonal, and I~_d is the identity plus each wall's second-order error
// coefficient on its corner (include/fd/laplacian.h:18-46,
// include/fd/identity.h:22-47, include/fd/discretization.h:47-80).  So
//     (L u)_ijk = Iz Iy (Lx u) + Iz (Ly u) Ix + (Lz u) Iy Ix,   I~ = Iz Iy Ix,
// a 7-point stencil whose coefficients differ from the interior only at the
// walls: applied matrix-free here.  The solve is the reference's
// preconditioned CG loop (include/solvers/pcg.h:12-45: stop when |d|_2 <=
// tolerance for the search direction d, bail out when <d, H d> is below
// tolerance^2) with the reference's preconditioner, a degree-4 Chebyshev
// polynomial in H = I~ - lambda L on its Gershgorin interval
// (include/solvers/chebpcg.h, include/solvers/preconditioners/chebyshev.h,
// include/algo/chebyshev.h, include/algo/gershgorin.h), or, selectable, a
// Jacobi preconditioner.  FP64, compiled without contraction.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>
#include "ibk_internal.h"

namespace ibk {
namespace {

constexpr int kFluidThreads = 256;
constexpr int kFluidBlocks = 1184;          // 8 CTAs per SM on 148 SMs: fixed, so sums have one order

// 1-D operators of one axis: L (lo, diag, hi; lo[0] / hi[P-1] wrap on a
// periodic axis, else 0) and the corrected identity id.
struct AxisOps {
	const double* lo;
	const double* diag;
	const double* hi;
	const double* id;
	int P;
	int periodic;
};

struct FluidOps {
	AxisOps ax[3];
	int dims;
	long long size;
	double lambda;
};

// Axis coordinates of face idx (x fastest); 32-bit arithmetic below 2^31 faces.
__device__ __forceinline__ void face_coords(long long idx, int P0, int P1, int& i, int& j, int& k)
{
	if (idx < 0x7fffffffLL) {
		const unsigned u = (unsigned) idx, r = u / (unsigned) P0;
		i = (int) (u - r * (unsigned) P0);
		j = (int) (r % (unsigned) P1);
		k = (int) (r / (unsigned) P1);
	} else {
		i = (int) (idx % P0);
		const long long r = idx / P0;
		j = (int) (r % P1);
		k = (int) (r / P1);
	}
}

// op 0: L u, 1: I~ u, 2: H u with H = I~ - lambda L, 3: wa r - H u, 4: wa r -
// H (wb r) with u = r (the steps of the Chebyshev preconditioner, whose
// first step's wb r is formed per loaded value instead of stored), per face
//     (L u) = Iz Iy (Lx u) + Iz (Ly u) Ix + (Lz u) Iy Ix
// with (L_d u) = lo u[-1] + diag u + hi u[+1] along axis d (wrapping on a
// periodic axis).  Each thread marches along z through kMarchZ planes of one
// (x, y) column: its x and y coefficients and neighbour offsets are taken
// once, the z neighbours move through registers (one new load per face), and
// no face needs a division for its coordinates.  A block is 32 columns along
// x (one warp, coalesced) by 8 along y.  With dot != nullptr the per-block
// partial sums of u . out (ops 0-2) or r . out (ops 3, 4) go to dot[block]
// (fixed order).
constexpr int kMarchX = 32, kMarchY = 8, kMarchZ = 16;

template <int OP, int DIMS>
__global__ void __launch_bounds__(kMarchX * kMarchY, 5)
march_apply_kernel(FluidOps o, const double* __restrict__ u, double* __restrict__ out, double* __restrict__ dot,
                   const double* __restrict__ rr, double wa, double wb)
{
	constexpr int op = OP;
	// a loaded value of the operand: wb r for op 4, else u itself
	auto ld = [wb](const double* p) { return OP == 4 ? wb * *p : *p; };
	__shared__ double red[kMarchY];
	const int P0 = o.ax[0].P;
	const int P1 = DIMS > 1 ? o.ax[1].P : 1;
	const int P2 = DIMS > 2 ? o.ax[2].P : 1;
	const int i = blockIdx.x * kMarchX + threadIdx.x;
	const int j = blockIdx.y * kMarchY + threadIdx.y;
	const int k0 = blockIdx.z * kMarchZ;
	const int k1 = min(k0 + kMarchZ, P2);
	double acc = 0.0;
	if (i < P0 && j < P1) {
		// 32-bit offsets: the plan's grids hold fewer than 2^31 faces
		const int sy = P0, sz = P0 * P1;
		const AxisOps& X = o.ax[0];
		const double ix = X.id[i], xl = X.lo[i], xd = X.diag[i], xh = X.hi[i];
		const bool has_xm = i > 0 || X.periodic, has_xp = i + 1 < P0 || X.periodic;
		const int dxm = i > 0 ? -1 : P0 - 1, dxp = i + 1 < P0 ? 1 : 1 - P0;
		double iy = 1.0, yl = 0.0, yd = 0.0, yh = 0.0;
		bool has_ym = false, has_yp = false;
		int dym = 0, dyp = 0;
		if (DIMS > 1) {
			const AxisOps& Y = o.ax[1];
			iy = Y.id[j]; yl = Y.lo[j]; yd = Y.diag[j]; yh = Y.hi[j];
			has_ym = j > 0 || Y.periodic;
			has_yp = j + 1 < P1 || Y.periodic;
			dym = j > 0 ? -sy : (P1 - 1) * sy;
			dyp = j + 1 < P1 ? sy : (1 - P1) * sy;
		}
		// z coefficients from one base: lo, diag, hi and id lie P2 apart
		const double* __restrict__ zc = o.ax[2].lo;
		const bool zper = o.ax[2].periodic;
		const int base = i + j * sy + k0 * sz;
		const double* __restrict__ pu = u + base;      // this column at plane k
		const double* __restrict__ pr = OP == 3 ? rr + base : nullptr;   // op 4: r is u itself
		double* __restrict__ po = out + base;
		// register window along z: uzm, uc, uzp = planes k - 1, k, k + 1 (wrapped
		// on a periodic axis, 0 past a wall), and the plane after next loaded
		// one iteration ahead
		double uc = ld(pu);
		double uzm = 0.0, uzp = 0.0;
		if (DIMS > 2) {
			uzm = k0 > 0 ? ld(pu - sz) : (zper ? ld(pu + (P2 - 1) * sz) : 0.0);
			uzp = k0 + 1 < P2 ? ld(pu + sz) : (zper ? ld(pu + (1 - P2) * sz) : 0.0);
		}
		for (int k = k0; k < k1; ++k) {
			double unx = 0.0;
			if (DIMS > 2 && k + 1 < k1)      // k + 2 <= P2: plane k + 2, or plane 0 past a periodic end
				unx = k + 2 < P2 ? ld(pu + 2 * sz) : (zper ? ld(pu + (2 - P2) * sz) : 0.0);
			const double iz = DIMS > 2 ? zc[3 * P2 + k] : 1.0;
			double v = 0.0;
			if (op != 1) {
				const double um = has_xm ? ld(pu + dxm) : 0.0, up = has_xp ? ld(pu + dxp) : 0.0;
				double l = iz * iy * (xl * um + xd * uc + xh * up);
				if (DIMS > 1) {
					const double vm = has_ym ? ld(pu + dym) : 0.0, vp = has_yp ? ld(pu + dyp) : 0.0;
					l += iz * (yl * vm + yd * uc + yh * vp) * ix;
				}
				if (DIMS > 2) l += (zc[k] * uzm + zc[P2 + k] * uc + zc[2 * P2 + k] * uzp) * iy * ix;
				v = l;
			}
			if (op == 1) v = iz * iy * ix * uc;
			if (op >= 2) v = iz * iy * ix * uc - o.lambda * v;
			if constexpr (OP >= 3) {
				// gemv(-1, H, s, w, t) with t = r: -(H s) + w r
				const double rc = OP == 3 ? *pr : *pu;
				v = wa * rc - v;
				if (dot) acc += rc * v;
				if (OP == 3) pr += sz;
			} else {
				if (dot) acc += uc * v;
			}
			*po = v;
			uzm = uc;
			uc = uzp;
			uzp = unx;
			pu += sz;
			po += sz;
		}
	}
	if (!dot) return;
	for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
	if (threadIdx.x == 0) red[threadIdx.y] = acc;
	__syncthreads();
	if (threadIdx.x == 0 && threadIdx.y == 0) {
		double t = 0.0;
		for (int w = 0; w < kMarchY; ++w) t += red[w];
		dot[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
	}
}

template <int OP>
void launch_march_dims(const FluidOps& o, dim3 grid, const double* u, double* out, double* dot, const double* r,
                       double wa, double wb, cudaStream_t s)
{
	if (o.dims == 3) march_apply_kernel<OP, 3><<<grid, dim3(kMarchX, kMarchY), 0, s>>>(o, u, out, dot, r, wa, wb);
	else march_apply_kernel<OP, 2><<<grid, dim3(kMarchX, kMarchY), 0, s>>>(o, u, out, dot, r, wa, wb);
}

void launch_march(const FluidOps& o, int op, dim3 grid, const double* u, double* out, double* dot, cudaStream_t s,
                  const double* r = nullptr, double wa = 0.0, double wb = 0.0)
{
	switch (op) {
	case 0: launch_march_dims<0>(o, grid, u, out, dot, r, wa, wb, s); break;
	case 1: launch_march_dims<1>(o, grid, u, out, dot, r, wa, wb, s); break;
	case 2: launch_march_dims<2>(o, grid, u, out, dot, r, wa, wb, s); break;
	case 3: launch_march_dims<3>(o, grid, u, out, dot, r, wa, wb, s); break;
	default: launch_march_dims<4>(o, grid, u, out, dot, r, wa, wb, s); break;
	}
}

// Gershgorin interval of H = I~ - lambda L (algo/gershgorin.h:14-49): per
// block the smallest diagonal - sum |off-diagonal| and the largest diagonal
// + sum |off-diagonal| of its rows (minimum and maximum are exact in any
// order).  part: 2 per block.
__global__ void __launch_bounds__(kFluidThreads)
gershgorin_kernel(FluidOps o, double* __restrict__ part)
{
	__shared__ double smin[kFluidThreads], smax[kFluidThreads];
	double mn = INFINITY, mx = -INFINITY;
	const int P0 = o.ax[0].P, P1 = o.ax[1].P;
	for (long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x; idx < o.size;
	     idx += (long long) gridDim.x * blockDim.x) {
		int i, j, k;
		face_coords(idx, P0, P1, i, j, k);
		const double ix = o.ax[0].id[i], iy = o.dims > 1 ? o.ax[1].id[j] : 1.0;
		const double iz = o.dims > 2 ? o.ax[2].id[k] : 1.0;
		double l = iz * iy * o.ax[0].diag[i];
		if (o.dims > 1) l += iz * o.ax[1].diag[j] * ix;
		if (o.dims > 2) l += o.ax[2].diag[k] * iy * ix;
		const double diag = iz * iy * ix - o.lambda * l;
		double off = fabs(o.lambda * (iz * iy * o.ax[0].lo[i])) + fabs(o.lambda * (iz * iy * o.ax[0].hi[i]));
		if (o.dims > 1)
			off += fabs(o.lambda * (iz * o.ax[1].lo[j] * ix)) + fabs(o.lambda * (iz * o.ax[1].hi[j] * ix));
		if (o.dims > 2)
			off += fabs(o.lambda * (o.ax[2].lo[k] * iy * ix)) + fabs(o.lambda * (o.ax[2].hi[k] * iy * ix));
		mn = fmin(mn, diag - off);
		mx = fmax(mx, diag + off);
	}
	smin[threadIdx.x] = mn;
	smax[threadIdx.x] = mx;
	__syncthreads();
	for (int w = kFluidThreads / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w) {
			smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + w]);
			smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + w]);
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		part[2 * blockIdx.x] = smin[0];
		part[2 * blockIdx.x + 1] = smax[0];
	}
}

// Reciprocal of the diagonal of I~ - lambda L (the Jacobi preconditioner).
__global__ void __launch_bounds__(kFluidThreads)
diagonal_kernel(FluidOps o, double* __restrict__ diag)
{
	const int P0 = o.ax[0].P, P1 = o.ax[1].P;
	for (long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x; idx < o.size;
	     idx += (long long) gridDim.x * blockDim.x) {
		int i, j, k;
		face_coords(idx, P0, P1, i, j, k);
		const double ix = o.ax[0].id[i], iy = o.dims > 1 ? o.ax[1].id[j] : 1.0;
		const double iz = o.dims > 2 ? o.ax[2].id[k] : 1.0;
		double l = iz * iy * o.ax[0].diag[i];
		if (o.dims > 1) l += iz * o.ax[1].diag[j] * ix;
		if (o.dims > 2) l += o.ax[2].diag[k] * iy * ix;
		diag[idx] = 1.0 / (iz * iy * ix - o.lambda * l);   // the preconditioner's reciprocal
	}
}

__device__ __forceinline__ void block_partial(double acc, double* __restrict__ out)
{
	__shared__ double red[kFluidThreads / 32];
	for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < kFluidThreads / 32; ++w) t += red[w];
		out[blockIdx.x] = t;
	}
}

// Sum of n per-block partials by one block of kSumThreads threads in a
// fixed order (strided per-thread sums, then a fixed tree); every thread
// returns the total.
constexpr int kSumThreads = 256;

__device__ __forceinline__ double sum_partials(const double* __restrict__ partial, int n)
{
	__shared__ double s[kSumThreads];
	double t = 0.0;
	for (int b = threadIdx.x; b < n; b += kSumThreads) t += partial[b];
	s[threadIdx.x] = t;
	__syncthreads();
	for (int w = kSumThreads / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
		__syncthreads();
	}
	return s[0];
}

__global__ void __launch_bounds__(kSumThreads) sum_kernel(const double* __restrict__ partial, int n,
                                                          double* __restrict__ out)
{
	const double t = sum_partials(partial, n);
	if (threadIdx.x == 0) *out = t;
}

// rhs = k I~ f + k mu (L u + rhs0): the right-hand side of the solve
// (diffusion.h:51-53: gemv(1, L, u, 1, rhs), then gemv(k, I~, f, k mu, rhs)).
__global__ void __launch_bounds__(kFluidThreads)
rhs_kernel(long long n, double k, double kmu, const double* __restrict__ lu, const double* __restrict__ rhs0,
           const double* __restrict__ idf, double* __restrict__ b)
{
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
		b[i] = k * idf[i] + kmu * (lu[i] + rhs0[i]);
}

// Start of the loop: x = 0, d = M^-1 r (dinv: the reciprocal diagonal),
// partials of r . d and d . d.
__global__ void __launch_bounds__(kFluidThreads)
start_kernel(long long n, const double* __restrict__ r, const double* __restrict__ diag, double* __restrict__ x,
             double* __restrict__ d, double* __restrict__ rd, double* __restrict__ dd)
{
	double a = 0.0, b = 0.0;
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		const double z = r[i] * diag[i];
		x[i] = 0.0;
		d[i] = z;
		a += r[i] * z;
		b += z * z;
	}
	block_partial(a, rd);
	__syncthreads();
	block_partial(b, dd);
}

// Device scalars of the loop (sc): [0] delta = r . M^-1 r, [1] nu = d . H d,
// [2] |d|^2, [3] alpha, [4] beta, [5] stop (1 when nu fell below tol^2).

// nu from its partials; alpha = delta / nu, or stop (pcg.h:23-31).
__global__ void __launch_bounds__(kSumThreads) alpha_kernel(const double* __restrict__ partial, int n, double tol2,
                                                            double* __restrict__ sc)
{
	const double t = sum_partials(partial, n);
	if (threadIdx.x != 0) return;
	sc[1] = t;
	if (fabs(t) < tol2) { sc[5] = 1.0; sc[3] = 0.0; return; }
	sc[3] = sc[0] / t;
}

// delta_new from its partials; beta = delta_new / delta (pcg.h:36-39).
__global__ void __launch_bounds__(kSumThreads) beta_kernel(const double* __restrict__ partial, int n,
                                                           double* __restrict__ sc)
{
	if (sc[5] != 0.0) return;
	const double t = sum_partials(partial, n);
	if (threadIdx.x != 0) return;
	sc[4] = t / sc[0];
	sc[0] = t;
}

// x += alpha d, r -= alpha q, q = M^-1 r; partial sums of r . q.  Does
// nothing once the loop has stopped.
__global__ void __launch_bounds__(kFluidThreads, 8)
update_kernel(long long n, const double* __restrict__ sc, const double* __restrict__ d, double* __restrict__ q,
              double* __restrict__ x, double* __restrict__ r, const double* __restrict__ dinv, double* __restrict__ rq)
{
	if (sc[5] != 0.0) return;
	const double alpha = sc[3];
	double a = 0.0;
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		x[i] += alpha * d[i];
		const double ri = r[i] - alpha * q[i];
		r[i] = ri;
		const double z = ri * dinv[i];
		q[i] = z;
		a += ri * z;
	}
	block_partial(a, rq);
}

// x += alpha d, r -= alpha q (the Chebyshev preconditioner and the r . z
// partials follow in the operator kernel).  Does nothing once the loop has
// stopped.
__global__ void __launch_bounds__(kFluidThreads, 8)
update_xr_kernel(long long n, const double* __restrict__ sc, const double* __restrict__ d,
                 const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r)
{
	if (sc[5] != 0.0) return;
	const double alpha = sc[3];
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		x[i] += alpha * d[i];
		r[i] = r[i] - alpha * q[i];
	}
}

// |d|^2 partials (the start of the loop under the Chebyshev preconditioner).
__global__ void __launch_bounds__(kFluidThreads)
norm_kernel(long long n, const double* __restrict__ d, double* __restrict__ dd)
{
	double a = 0.0;
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
		a += d[i] * d[i];
	block_partial(a, dd);
}

// d = q + beta d; partial sums of d . d.
__global__ void __launch_bounds__(kFluidThreads)
direction_kernel(long long n, const double* __restrict__ sc, const double* __restrict__ q, double* __restrict__ d,
                 double* __restrict__ dd)
{
	if (sc[5] != 0.0) return;
	const double beta = sc[4];
	double a = 0.0;
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		const double v = q[i] + beta * d[i];
		d[i] = v;
		a += v * v;
	}
	block_partial(a, dd);
}

// out = u + x
__global__ void __launch_bounds__(kFluidThreads)
finish_kernel(long long n, const double* __restrict__ u, const double* __restrict__ x, double* __restrict__ out)
{
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
		out[i] = x[i] + u[i];
}

// util::math::modulo for the non-negative arguments met here
double modulo1(double x) { return x - std::floor(x); }

// Ghost-point weights of one wall (fd::__1::coefficients,
// include/fd/discretization.h:47-80): Robin condition a u + b du/dn, signed
// mesh width h, alignment s of the grid against the wall.
struct WallWeights { double interior, laplacian; };

WallWeights wall_weights(const double* p, double h, double s_in)
{
	const double s = 1 - modulo1(1 - s_in);
	const double denom = p[1] - p[0] * s * h;
	return {(p[1] + p[0] * h * (1 - s)) / denom, (-(p[1] * (1 - 2 * s) - p[0] * s * h * (1 - s))) / (2 * denom)};
}

// impl::polynomial and impl::chebw<4> (algo/chebyshev.h:48-65, 124-145):
// p(a, b) = sum_i c_i a^i b^(n-1-i), evaluated as the reference does.
double cheb_poly(const double* c, int n, double a, double b)
{
	double v = 0.0;
	for (int i = 0; i < n; ++i) v += c[i] * std::pow(a, i) * std::pow(b, n - 1 - i);
	return v;
}

void chebyshev_weights(double a, double b, double* w)
{
	static const double p1[] = {128}, p2[] = {256, 256}, p3[] = {160, 448, 160}, p4[] = {32, 224, 224, 32};
	static const double q[] = {1, 28, 70, 28, 1};
	const double qv = cheb_poly(q, 5, a, b);
	w[0] = cheb_poly(p1, 1, a, b) / qv;
	w[1] = cheb_poly(p2, 2, a, b) / qv;
	w[2] = cheb_poly(p3, 3, a, b) / qv;
	w[3] = cheb_poly(p4, 4, a, b) / qv;
}

ibk_status cuda_fail(cudaError_t e, const char* what)
{
	return set_error(IBK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace
} // namespace ibk

using namespace ibk;

struct ibk_diffusion_s {
	int device = 0;
	FluidOps ops{};
	double mu = 0.0, timestep = 0.0, tolerance = 0.0;
	int max_iterations = 0;
	double* coef = nullptr;        // per axis: lo, diag, hi, id (4 P_d doubles)
	double* work = nullptr;        // b, r, d, q, x, diag, tmp, tmp2 (8 size doubles)
	int precond = IBK_PRECOND_CHEBYSHEV;
	double cheb_w[4] = {};         // chebw<4> on the Gershgorin interval
	double bounds[2] = {};         // that interval (lower, upper)
	double* partial = nullptr;     // partial sums: max(march blocks, kFluidBlocks) + kFluidBlocks
	dim3 march_grid;               // march_apply_kernel's grid
	int march_blocks = 0;
	double* scalars = nullptr;     // device scalars of the loop (see alpha_kernel)
};

extern "C" {

ibk_status ibk_diffusion_create(ibk_plan plan, int component, const double robin[3][2][2], double timestep,
                                double mu, double tolerance, int max_iterations, ibk_diffusion* out)
{
	if (!out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null output handle");
	*out = nullptr;
	Plan* p = reinterpret_cast<Plan*>(plan);
	if (!p || !robin) return set_error(IBK_ERR_INVALID_ARGUMENT, "null plan or boundary conditions");
	const GridGeom& g = p->g;
	if (component < 0 || component >= g.dims) return set_error(IBK_ERR_INVALID_ARGUMENT, "component out of range");
	if (!(timestep > 0.0) || !(mu >= 0.0) || !(tolerance > 0.0) || max_iterations < 1)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "timestep and tolerance must be positive, mu non-negative");
	for (int a = 0; a < g.dims; ++a)
		for (int side = 0; side < 2 && g.solid[a]; ++side)
			if (robin[a][side][0] == 0.0 && robin[a][side][1] == 0.0)
				return set_error(IBK_ERR_INVALID_ARGUMENT, "a wall's Robin condition needs a or b nonzero");
	const CompGeom& cg = g.comp[component];
	auto* d = new ibk_diffusion_s;
	cudaGetDevice(&d->device);
	d->mu = mu;
	d->timestep = timestep;
	d->tolerance = tolerance;
	d->max_iterations = max_iterations;
	d->ops.dims = g.dims;
	d->ops.lambda = timestep * mu / 2;       // diffusion.h:21-25
	long long size = 1;
	int total = 0;
	for (int a = 0; a < 3; ++a) {
		d->ops.ax[a].P = a < g.dims ? cg.points[a] : 1;
		size *= d->ops.ax[a].P;
		total += 4 * d->ops.ax[a].P;
	}
	d->ops.size = size;
	std::vector<double> host((size_t) total, 0.0);
	int off = 0;
	for (int a = 0; a < g.dims; ++a) {
		const int P = cg.points[a];
		if (P < 3) {
			delete d;
			return set_error(IBK_ERR_INVALID_ARGUMENT, "each axis needs at least 3 points");
		}
		double* lo = host.data() + off;
		double* dg = lo + P;
		double* hi = dg + P;
		double* id = hi + P;
		const double scale = g.r * g.r;          // laplacian.h:25-26
		for (int i = 0; i < P; ++i) {
			lo[i] = i > 0 ? scale : 0.0;
			dg[i] = -2 * scale;
			hi[i] = i + 1 < P ? scale : 0.0;
			id[i] = 1.0;
		}
		const int periodic = !g.solid[a];
		if (periodic) {
			// wrap entries (discretization.h:94-100: {!lower, lower, 1})
			lo[0] = scale * 1.0;
			hi[P - 1] = scale * 1.0;
		} else {
			// ghost-point weights of each wall on the corner diagonals, and the
			// second-order error coefficients on the identity's corners
			const double h = 1 / g.r;
			const double al = modulo1(cg.shift[a]);
			const WallWeights wl = wall_weights(robin[a][0], h, al);
			const WallWeights wu = wall_weights(robin[a][1], -h, 1 - al);
			dg[0] += scale * wl.interior;
			dg[P - 1] += scale * wu.interior;
			id[0] += wl.laplacian;
			id[P - 1] += wu.laplacian;
		}
		d->ops.ax[a].periodic = periodic;
		off += 4 * P;
	}
	d->march_grid = dim3((unsigned) ((d->ops.ax[0].P + kMarchX - 1) / kMarchX),
	                     (unsigned) ((d->ops.ax[1].P + kMarchY - 1) / kMarchY),
	                     (unsigned) ((d->ops.ax[2].P + kMarchZ - 1) / kMarchZ));
	d->march_blocks = (int) (d->march_grid.x * d->march_grid.y * d->march_grid.z);
	if (d->march_grid.y > 65535u || d->march_grid.z > 65535u || size >= (1LL << 31)) {
		delete d;
		return set_error(IBK_ERR_UNSUPPORTED, "grid too large for the operator kernel (2^31 faces)");
	}
	const int first_partials = std::max(d->march_blocks, kFluidBlocks);
	cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d->coef), sizeof(double) * (size_t) total);
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d->work), sizeof(double) * 8 * (size_t) size);
	if (e == cudaSuccess)
		e = cudaMalloc(reinterpret_cast<void**>(&d->partial), sizeof(double) * (size_t) (first_partials + kFluidBlocks));
	if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d->scalars), sizeof(double) * 8);
	if (e == cudaSuccess) e = cudaMemcpy(d->coef, host.data(), sizeof(double) * (size_t) total, cudaMemcpyHostToDevice);
	if (e != cudaSuccess) {
		cudaGetLastError();
		ibk_diffusion_destroy(d);
		return set_error(IBK_ERR_OUT_OF_MEMORY, std::string("diffusion set-up: ") + cudaGetErrorString(e));
	}
	off = 0;
	for (int a = 0; a < 3; ++a) {
		AxisOps& ax = d->ops.ax[a];
		if (a < g.dims) {
			ax.lo = d->coef + off;
			ax.diag = ax.lo + ax.P;
			ax.hi = ax.diag + ax.P;
			ax.id = ax.hi + ax.P;
			off += 4 * ax.P;
		} else {
			ax.lo = ax.diag = ax.hi = ax.id = d->coef;    // never read (dims < 3)
			ax.periodic = 0;
		}
	}
	// the Jacobi preconditioner's reciprocal diagonal, kept in work slot 5, and
	// the Gershgorin interval of the Chebyshev preconditioner (through the
	// partial-sum buffer, 2 per block)
	diagonal_kernel<<<kFluidBlocks, kFluidThreads>>>(d->ops, d->work + 5 * size);
	gershgorin_kernel<<<kFluidBlocks, kFluidThreads>>>(d->ops, d->partial);
	ibk_status st = check_launch("diffusion set-up kernels");
	std::vector<double> part(2 * kFluidBlocks);
	if (st == IBK_OK && (e = cudaMemcpy(part.data(), d->partial, sizeof(double) * part.size(),
	                                    cudaMemcpyDeviceToHost)) != cudaSuccess)
		st = cuda_fail(e, "diffusion set-up");
	if (st != IBK_OK) {
		ibk_diffusion_destroy(d);
		return st;
	}
	double lower = INFINITY, upper = -INFINITY;
	for (int b = 0; b < kFluidBlocks; ++b) {
		lower = std::min(lower, part[2 * b]);
		upper = std::max(upper, part[2 * b + 1]);
	}
	d->bounds[0] = lower;
	d->bounds[1] = upper;
	chebyshev_weights(upper, lower, d->cheb_w);     // chebyshev(upper, lower, H): preconditioners/chebyshev.h:14-25
	*out = d;
	return IBK_OK;
}

ibk_status ibk_diffusion_set_preconditioner(ibk_diffusion d, int kind)
{
	if (!d) return set_error(IBK_ERR_INVALID_ARGUMENT, "null diffusion handle");
	if (kind != IBK_PRECOND_CHEBYSHEV && kind != IBK_PRECOND_JACOBI)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "unknown preconditioner");
	d->precond = kind;
	return IBK_OK;
}

ibk_status ibk_diffusion_info(ibk_diffusion d, double* bounds, double* weights)
{
	if (!d) return set_error(IBK_ERR_INVALID_ARGUMENT, "null diffusion handle");
	if (bounds) { bounds[0] = d->bounds[0]; bounds[1] = d->bounds[1]; }
	if (weights) for (int q = 0; q < 4; ++q) weights[q] = d->cheb_w[q];
	return IBK_OK;
}

ibk_status ibk_diffusion_destroy(ibk_diffusion d)
{
	if (!d) return IBK_OK;
	int dev = 0;
	cudaGetDevice(&dev);
	cudaSetDevice(d->device);
	cudaFree(d->coef);
	cudaFree(d->work);
	cudaFree(d->partial);
	cudaFree(d->scalars);
	cudaSetDevice(dev);
	delete d;
	return IBK_OK;
}

ibk_status ibk_diffusion_apply(ibk_diffusion d, int op, const double* u, double* out, void* stream)
{
	if (!d || !u || !out || op < 0 || op > 2) return set_error(IBK_ERR_INVALID_ARGUMENT, "null arrays or unknown operator");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	launch_march(d->ops, op, d->march_grid, u, out, nullptr, s);
	return check_launch("march_apply_kernel");
}

ibk_status ibk_diffusion_step(ibk_diffusion d, double gamma, const double* u, const double* rhs, const double* f,
                              double* out, int* iterations, void* stream)
{
	if (!d || !u || !rhs || !f || !out) return set_error(IBK_ERR_INVALID_ARGUMENT, "null arrays");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const long long n = d->ops.size;
	double* b = d->work;
	double* r = b + n;
	double* dv = r + n;
	double* q = dv + n;
	double* x = q + n;
	double* diag = x + n;
	double* tmp = diag + n;
	double* tmp2 = tmp + n;
	double* pa = d->partial;                                            // march_blocks or kFluidBlocks
	double* pb = d->partial + std::max(d->march_blocks, kFluidBlocks);   // kFluidBlocks
	double* sc = d->scalars;
	const double k = gamma * d->timestep;
	const bool cheb = d->precond == IBK_PRECOND_CHEBYSHEV;
	const double* w = d->cheb_w;
	// rhs of the solve: k I~ f + k mu (L u + rhs)
	const dim3 mg = d->march_grid;
	launch_march(d->ops, 0, mg, u, tmp, nullptr, s);
	launch_march(d->ops, 1, mg, f, q, nullptr, s);
	rhs_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, k, k * d->mu, tmp, rhs, q, b);
	cudaError_t e = cudaMemcpyAsync(r, b, sizeof(double) * (size_t) n, cudaMemcpyDeviceToDevice, s);
	if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
	// z = M^-1 r with the r . z partials in pa: the Chebyshev polynomial
	// (algo/chebyshev.h:152-167: s = w0 r, then s = w_i r - H s, i = 1..3)
	auto chebyshev = [&](double* z) {
		launch_march(d->ops, 4, mg, r, tmp, nullptr, s, r, w[1], w[0]);
		launch_march(d->ops, 3, mg, tmp, tmp2, nullptr, s, r, w[2]);
		launch_march(d->ops, 3, mg, tmp2, z, pa, s, r, w[3]);
	};
	int za = kFluidBlocks;       // the count of r . z partials
	if (cheb) {
		// pcg.h:14-18: x = 0, d = M^-1 r, delta = r . d
		e = cudaMemsetAsync(x, 0, sizeof(double) * (size_t) n, s);
		if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
		chebyshev(dv);
		norm_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, dv, pb);
		za = d->march_blocks;
	} else {
		start_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, r, diag, x, dv, pa, pb);
	}
	sum_kernel<<<1, kSumThreads, 0, s>>>(pa, za, sc + 0);
	sum_kernel<<<1, kSumThreads, 0, s>>>(pb, kFluidBlocks, sc + 2);
	ibk_status st = check_launch("diffusion set-up kernels");
	if (st != IBK_OK) return st;
	e = cudaMemsetAsync(sc + 5, 0, sizeof(double), s);
	if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
	const double tol = d->tolerance;
	int it = 0;
	double hs[6];
	for (;;) {
		// the loop test of pcg.h:21 (|d| > tol) and its bail-out, read back once
		// per iteration; alpha and beta stay on the device
		e = cudaMemcpyAsync(hs, sc, sizeof(double) * 6, cudaMemcpyDeviceToHost, s);
		if (e == cudaSuccess) e = cudaStreamSynchronize(s);
		if (e != cudaSuccess) return cuda_fail(e, "diffusion residual read");
		if (hs[5] != 0.0 || !(std::sqrt(hs[2]) > tol)) break;
		if (it >= d->max_iterations) {
			if (iterations) *iterations = it;
			return set_error(IBK_ERR_DEVICE_CHECK, "diffusion solve did not converge within max_iterations");
		}
		launch_march(d->ops, 2, mg, dv, q, pa, s);
		alpha_kernel<<<1, kSumThreads, 0, s>>>(pa, d->march_blocks, tol * tol, sc);
		if (cheb) {
			// x += alpha d, r -= alpha q, q = M^-1 r (a bail-out leaves x and r as
			// they are; the polynomial of the unchanged r is then not used)
			update_xr_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, sc, dv, q, x, r);
			chebyshev(q);
		} else {
			update_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, sc, dv, q, x, r, diag, pa);
		}
		beta_kernel<<<1, kSumThreads, 0, s>>>(pa, za, sc);
		direction_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, sc, q, dv, pb);
		sum_kernel<<<1, kSumThreads, 0, s>>>(pb, kFluidBlocks, sc + 2);
		if ((st = check_launch("diffusion iteration kernels")) != IBK_OK) return st;
		++it;
	}
	// a bail-out leaves the last iteration's update undone, as pcg.h does
	if (hs[5] != 0.0 && it > 0) --it;
	finish_kernel<<<kFluidBlocks, kFluidThreads, 0, s>>>(n, u, x, out);
	if (iterations) *iterations = it;
	return check_launch("finish_kernel");
}

} // extern "C"
