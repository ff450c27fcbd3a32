/*
 * Reference bridge (TEST INFRASTRUCTURE): builds sonwell/ib.cu's own host
 * constexpr headers, unmodified, into oracle/_ref/libibref.so so that the
 * plain-C oracle (ibk_oracle.c) and the golden fixtures can be pinned to the
 * reference's arithmetic.
 *
 * Compiled from the reference sources where they lie (see oracle/Makefile):
 *   fd::dimension / fd::domain / fd::grid / fd::discretization   (geometry)
 *   util::math::floor                                           (index step)
 *   ib::indexing::{clamped, errors_negative, reduce, sorter}     (keys, indices)
 *   ib::delta::{standard,every_other}_pattern                     (entry order)
 *   ib::delta::{bspline<n>, peskin, roma, cosine, hat}            (weights)
 *
 * include/ib/sweep.h itself does not compile with g++ (a constexpr static
 * member without an initializer at include/ib/sweep.h:34), so the four short
 * sweep methods that glue those pieces together -- clamp (:38-44), difference
 * (:49-62), sort (:64-77), grid (:79-89), values (:98-112), indices (:114-125)
 * -- are restated below line by line on top of the reference's own types.
 */
#include "fd/boundary.h"
#include "fd/dimension.h"
#include "fd/domain.h"
#include "fd/discretization.h"
#include "fd/grid.h"
#include "fd/cell.h"
#include "ib/indexing.h"
#include "ib/delta.h"
#include "ib/bspline.h"
#include "ib/peskin.h"
#include "ib/roma.h"
#include "ib/cosine.h"
#include "ib/hat.h"
#include "ib/types.h"

#include <array>
#include <utility>

namespace {

using periodic_t = std::remove_cv_t<decltype(fd::boundary::periodic)>;
using dirichlet_t = std::remove_cv_t<decltype(fd::boundary::dirichlet)>;

template <typename B> constexpr B boundary_value() { return B{}; }

/* Three separate construction sites so each dimension gets its own
 * util::unique_id (the grid identifies components by dimension identity). */
template <typename B> auto make_dim0(double L) { return fd::dimension{L, boundary_value<B>()}; }
template <typename B> auto make_dim1(double L) { return fd::dimension{L, boundary_value<B>()}; }
template <typename B> auto make_dim2(double L) { return fd::dimension{L, boundary_value<B>()}; }

struct outputs {
	int* keys; int* base; double* delta; double* weights; int* sidx; int* iidx;
};

/* One delta type: pattern + phi from the reference's headers. */
template <typename delta_type, std::size_t dims>
struct delta_ops {
	using traits = ib::delta::traits<delta_type>;
	static constexpr int meshwidths = traits::meshwidths;
	static ib::shift<dims> pattern(int offset, int i)
	{
		typename traits::template pattern<dims> p{};
		return p(offset, i);
	}
	static double phi(double r) { return delta_type{}(r); }
};

template <typename grid_type, typename ops, std::size_t dims>
void
run_grid(const grid_type& grid, int n, const double* x, const outputs& o)
{
	using point = ib::point<dims>;
	using indices = ib::indices<dims>;
	constexpr int M = ops::meshwidths;
	constexpr int V = [] { int v = 1; for (std::size_t d = 0; d < dims; ++d) v *= M; return v; }();
	ib::indexing::sorter<grid_type> idx{grid};
	ib::indexing::sorter<grid_type> iidx_sorter{grid};

	/* sweep::clamp (sweep.h:38-44) */
	auto clamp = [] (double r) -> int {
		using util::math::floor;
		constexpr double rounding = 0.5 * (M & 1);
		return floor(r + rounding);
	};

	for (int p = 0; p < n; ++p) {
		point z;
		for (std::size_t d = 0; d < dims; ++d) z[d] = x[(long) n * d + p];

		/* sweep::sort (sweep.h:64-77) */
		auto ks = [&] (double xv, const auto& comp) {
			auto solid = comp.solid_boundary;
			auto shift = comp.shift();
			int i = clamp(comp.units(xv) - shift);
			int j = comp.index(i);
			return ib::indexing::clamped{j, -solid, comp.points()};
		};
		int key = (int) ib::indexing::reduce(ks, z, idx);
		if (o.keys) o.keys[p] = key;

		/* sorter::decompose (indexing.h:239-250) */
		indices dec = idx.decompose(key);
		if (o.base) for (std::size_t d = 0; d < dims; ++d) o.base[(long) p * dims + d] = dec[d];

		/* sweep::difference (sweep.h:49-62) */
		std::array<double, dims> diff{};
		{
			auto comps = fd::components(grid);
			std::size_t d = 0;
			std::apply([&] (const auto& ... comp) {
				((diff[d] = [&] {
					auto shift = comp.shift();
					auto dd = comp.units(z[d]) - shift;
					return clamp(dd) - dd;
				}(), ++d), ...);
			}, comps);
		}
		if (o.delta) for (std::size_t d = 0; d < dims; ++d) o.delta[(long) p * dims + d] = diff[d];

		for (int e = 0; e < V; ++e) {
			auto s = ops::pattern(0, e);
			/* sweep::values (sweep.h:104-110): right fold of phi(r + s) */
			if (o.weights) {
				double w = 1;
				for (int d = (int) dims - 1; d >= 0; --d) w = ops::phi(diff[d] + s[d]) * w;
				o.weights[(long) p * V + e] = w;
			}
			/* sweep::indices + sweep::grid (sweep.h:79-89, 114-125) */
			indices target = dec + s;
			if (o.sidx) {
				auto kg = [] (int i, const auto& comp) {
					auto j = comp.index(i);
					return ib::indexing::errors_negative{j, 0, comp.points()};
				};
				o.sidx[(long) p * V + e] = (int) ib::indexing::reduce(kg, target, idx);
			}
			if (o.iidx) {
				auto kg = [] (int i, const auto& comp) {
					auto j = comp.index(i);
					return ib::indexing::clamped{j, 0, comp.points()};
				};
				o.iidx[(long) p * V + e] = (int) ib::indexing::reduce(kg, target, iidx_sorter);
			}
		}
	}
}

template <typename domain_type, typename tag_type, typename ops>
int
run_domain(const domain_type& domain, const tag_type& tag, int comp, int n,
           const double* x, const outputs& o, double* geo)
{
	constexpr std::size_t dims = domain_type::dimensions;
	const auto& comps = fd::components(domain);
	auto go = [&] (const auto& dimension) {
		fd::grid grid{tag, domain, dimension};
		if (geo) {
			geo[0] = domain.unit();
			geo[1] = grid.resolution();
			auto cs = grid.components();
			std::size_t d = 0;
			std::apply([&] (const auto& ... c) {
				((geo[2 + 3 * d] = c.cells(), geo[3 + 3 * d] = c.points(),
				  geo[4 + 3 * d] = c.shift(), ++d), ...);
			}, cs);
		}
		run_grid<decltype(grid), ops, dims>(grid, n, x, o);
		return 0;
	};
	if (comp == 0) return go(std::get<0>(comps));
	if constexpr (dims > 1) if (comp == 1) return go(std::get<1>(comps));
	if constexpr (dims > 2) if (comp == 2) return go(std::get<2>(comps));
	return -1;
}

template <typename ops, typename domain_type>
int
run_tag(const domain_type& domain, int tag, int ref, int comp, int n,
        const double* x, const outputs& o, double* geo)
{
	if (tag == 0) return run_domain<domain_type, fd::mac, ops>(domain, fd::mac{ref}, comp, n, x, o, geo);
	return run_domain<domain_type, fd::centered, ops>(domain, fd::centered{ref}, comp, n, x, o, geo);
}

template <std::size_t dims, typename ops>
int
run_boundaries(const double* L, const int* solid, int tag, int ref, int comp,
               int n, const double* x, const outputs& o, double* geo)
{
	auto d0 = [&] (auto b0) {
		using B0 = decltype(b0);
		auto x0 = make_dim0<B0>(L[0]);
		if constexpr (dims == 1) {
			fd::domain dom{x0};
			return run_tag<ops>(dom, tag, ref, comp, n, x, o, geo);
		} else {
			auto d1 = [&] (auto b1) {
				using B1 = decltype(b1);
				auto x1 = make_dim1<B1>(L[1]);
				if constexpr (dims == 2) {
					fd::domain dom{x0, x1};
					return run_tag<ops>(dom, tag, ref, comp, n, x, o, geo);
				} else {
					auto d2 = [&] (auto b2) {
						using B2 = decltype(b2);
						auto x2 = make_dim2<B2>(L[2]);
						fd::domain dom{x0, x1, x2};
						return run_tag<ops>(dom, tag, ref, comp, n, x, o, geo);
					};
					return solid[2] ? d2(dirichlet_t{}) : d2(periodic_t{});
				}
			};
			return solid[1] ? d1(dirichlet_t{}) : d1(periodic_t{});
		}
	};
	return solid[0] ? d0(dirichlet_t{}) : d0(periodic_t{});
}

template <std::size_t dims>
int
run_delta(int kind, int order, const double* L, const int* solid, int tag,
          int ref, int comp, int n, const double* x, const outputs& o, double* geo)
{
	using namespace ib::delta;
	switch (kind) {
	case 0:
		switch (order) {
		case 1: return run_boundaries<dims, delta_ops<bspline<1>, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
		case 2: return run_boundaries<dims, delta_ops<bspline<2>, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
		case 3: return run_boundaries<dims, delta_ops<bspline<3>, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
		case 4: return run_boundaries<dims, delta_ops<bspline<4>, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
		case 5: return run_boundaries<dims, delta_ops<bspline<5>, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
		}
		return -2;
	case 1: return run_boundaries<dims, delta_ops<peskin, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
	case 2: return run_boundaries<dims, delta_ops<roma, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
	case 3: return run_boundaries<dims, delta_ops<cosine, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
	case 4: return run_boundaries<dims, delta_ops<hat, dims>>(L, solid, tag, ref, comp, n, x, o, geo);
	}
	return -2;
}

} // namespace

extern "C" {

/* Per-point stencil data of component `comp`, computed by the reference's
 * own headers.  geo (optional, 2 + 3*dims doubles) receives unit,
 * resolution, then cells/points/shift per dimension of that component. */
int
ibref_stencil(int dims, const double* length, const int* solid, int tag,
              int refinement, int delta_kind, int delta_order, int comp,
              int n, const double* x, int* keys, int* base, double* delta,
              double* weights, int* sidx, int* iidx, double* geo)
{
	outputs o{keys, base, delta, weights, sidx, iidx};
	switch (dims) {
	case 2: return run_delta<2>(delta_kind, delta_order, length, solid, tag, refinement, comp, n, x, o, geo);
	case 3: return run_delta<3>(delta_kind, delta_order, length, solid, tag, refinement, comp, n, x, o, geo);
	}
	return -1;
}

/* phi(r) of the reference's delta functors. */
double
ibref_phi(int kind, int order, double r)
{
	using namespace ib::delta;
	switch (kind) {
	case 0:
		switch (order) {
		case 1: return bspline<1>{}(r);
		case 2: return bspline<2>{}(r);
		case 3: return bspline<3>{}(r);
		case 4: return bspline<4>{}(r);
		case 5: return bspline<5>{}(r);
		}
		return 0;
	case 1: return peskin{}(r);
	case 2: return roma{}(r);
	case 3: return cosine{}(r);
	case 4: return hat{}(r);
	}
	return 0;
}

/* Wall weights of the reference's fd::discretization over Robin walls
 * (include/fd/discretization.h:47-80, 159-164): out = {lower interior, lower
 * laplacian (second-order correction), lower boundary, the same for the
 * upper wall}. */
void
ibref_wall_weights(double length, double resolution, double shift, double la, double lb, double ua, double ub,
                   double* out)
{
	using robin_t = fd::boundary::robin;
	fd::dimension<robin_t, robin_t> dim{length, robin_t(la, lb), robin_t(ua, ub)};
	fd::discretization<fd::dimension<robin_t, robin_t>> disc{dim, fd::alignment{shift}, resolution};
	const auto in = disc.interior();
	const auto bd = disc.boundary();
	const auto lp = disc.coefficient(fd::correction::second_order);
	out[0] = in.lower; out[1] = lp.lower; out[2] = bd.lower;
	out[3] = in.upper; out[4] = lp.upper; out[5] = bd.upper;
}

/* fd::domain::unit(): GCD of the dimension lengths (include/fd/domain.h:30-32) */
double
ibref_domain_unit(int dims, const double* length)
{
	if (dims == 1) return fd::domain{make_dim0<periodic_t>(length[0])}.unit();
	if (dims == 2) return fd::domain{make_dim0<periodic_t>(length[0]), make_dim1<periodic_t>(length[1])}.unit();
	return fd::domain{make_dim0<periodic_t>(length[0]), make_dim1<periodic_t>(length[1]),
	                  make_dim2<periodic_t>(length[2])}.unit();
}

}
