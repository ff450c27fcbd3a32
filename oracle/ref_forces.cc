/*
 * The reference's own membrane-force code, compiled on the host (TEST
 * INFRASTRUCTURE: only oracle.py loads it, to check the oracle's restatement).
 *
 * include/forces/{skalak,neohookean,hookean,bending,dissipation,tether}.h
 * are compiled as they are, with -Iref_shim_forces standing in
 * for the CUDA linalg layer (a host column-major matrix), bases/geometry.h
 * (the geometry and operator containers, the reference / current tags and a
 * host util::transform) and cublas/handle.h.  The caller supplies the
 * geometry and the operators; the force formulas are the reference's.
 * (include/forces/repelling.h does not compile as written: `loader
 * deformed{curr}` has no deduction guide and `deformed(tid)` no call
 * operator; no driver of the reference uses it.)
 * Built by `make -C oracle ref REF=<sonwell/ib.cu tree>`.
 */
#include <cstring>
#include "forces/skalak.h"
#include "forces/neohookean.h"
#include "forces/hookean.h"
#include "forces/bending.h"
#include "forces/dissipation.h"
#include "forces/tether.h"

namespace {

using M = bases::matrix;

M from(const double* p, int rows, int cols)
{
	M m(rows, cols);
	if (p) std::memcpy(m.values(), p, sizeof(double) * (std::size_t) rows * cols);
	return m;
}

void to(const M& m, double* out) { std::memcpy(out, m.values(), sizeof(double) * m.v.size()); }

/* a shape family's geometry and operators, as object.geometry(tag).sample /
 * .data and object.operators().sample / .data */
struct family {
	struct geometries { bases::geometry<2> data, sample; };
	struct operator_sets { bases::operators<2> data, sample; };
	geometries ref, cur;
	operator_sets ops;
	const geometries& geometry(decltype(bases::reference)) const { return ref; }
	const geometries& geometry(decltype(bases::current)) const { return cur; }
	const operator_sets& operators() const { return ops; }
};

/* geometry of n sites x nc shapes from [tu, tv, tuu, tuv, tvv, normal, sigma,
 * position] arrays (NULL entries stay empty) */
void fill(bases::geometry<2>& g, int n, int nc, const double* const* a, int count)
{
	const int cols = 3 * nc;
	if (count > 0 && a[0]) g.tangents[0] = from(a[0], n, cols);
	if (count > 1 && a[1]) g.tangents[1] = from(a[1], n, cols);
	for (int q = 0; q < 3; ++q)
		if (count > 2 + q && a[2 + q]) g.second_derivatives[q] = from(a[2 + q], n, cols);
	if (count > 5 && a[5]) g.normal = from(a[5], n, cols);
	if (count > 6 && a[6]) g.sigma = from(a[6], n, nc);
	if (count > 7 && a[7]) g.position = from(a[7], n, cols);
}

void ops(bases::operators<2>& o, int ns, int nd, const double* const* p)
{
	o.sample_sites = ns;
	o.data_sites = nd;
	for (int q = 0; q < 2; ++q) o.first_derivatives[q] = from(p[1 + q], ns, nd);
	for (int q = 0; q < 3; ++q) o.second_derivatives[q] = from(p[3 + q], ns, nd);
}

} // namespace

extern "C" {

/* law 0 skalak, 1 neohookean, 2 hookean; rest = tu, tv, tuu, tuv, tvv, sigma;
 * cur = tu, tv, tuu, tuv, tvv; npoints sites of one shape */
void ibref_membrane_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                            const double* const* cur, double* f)
{
	family obj;
	const double* r[8] = {rest[0], rest[1], rest[2], rest[3], rest[4], nullptr, rest[5], nullptr};
	// the current geometry's loader reads a patch area too (tension.h:16-33),
	// which the force does not use: the rest areas stand in
	const double* c[8] = {cur[0], cur[1], cur[2], cur[3], cur[4], nullptr, rest[5], nullptr};
	fill(obj.ref.sample, npoints, 1, r, 8);
	fill(obj.cur.sample, npoints, 1, c, 8);
	obj.cur.sample.position = M(npoints, 3);
	M out;
	if (law == 0) out = forces::skalak{e, kappa}(obj, M{});
	else if (law == 1) out = forces::neohookean{e, kappa}(obj, M{});
	else out = forces::hookean{e}(obj);
	to(out, f);
}

/* data geometries (rest, current) at the data sites and sample geometries,
 * each tu, tv, tuu, tuv, tvv, normal, sigma; sample_ops[1..5] ns x nd */
void ibref_membrane_bending(int ns, int nd, int nc, const double* const* sample_ops, double modulus, int preferred,
                            const double* const* data_rest, const double* const* data_cur,
                            const double* const* rest, const double* const* cur, double* f)
{
	family obj;
	fill(obj.ref.data, nd, nc, data_rest, 7);
	fill(obj.cur.data, nd, nc, data_cur, 7);
	fill(obj.ref.sample, ns, nc, rest, 7);
	fill(obj.cur.sample, ns, nc, cur, 7);
	// the fields are sized from the positions (bending.h:127, 162, 212), whose
	// values the force does not read
	obj.cur.sample.position = M(ns, 3 * nc);
	obj.ref.sample.position = M(ns, 3 * nc);
	obj.cur.data.position = M(nd, 3 * nc);
	obj.ref.data.position = M(nd, 3 * nc);
	ops(obj.ops.sample, ns, nd, sample_ops);
	const M out = forces::bending{modulus, preferred != 0}(obj, M{});
	to(out, f);
}

/* cur = tu, tv, tuu, tuv, tvv, sigma at the samples; u the data-site velocity */
void ibref_membrane_dissipation(int ns, int nd, int nc, const double* const* sample_ops, double kappa,
                                const double* u, const double* const* cur, double* f)
{
	family obj;
	const double* c[8] = {cur[0], cur[1], cur[2], cur[3], cur[4], nullptr, cur[5], nullptr};
	fill(obj.cur.sample, ns, nc, c, 8);
	obj.cur.sample.position = M(ns, 3 * nc);
	ops(obj.ops.sample, ns, nd, sample_ops);
	const M out = forces::dissipation{kappa}(obj, from(u, nd, 3 * nc));
	to(out, f);
}

/* curves: law 0 skalak1d, 2 hookean1d; rest = t, tt, sigma; cur = t, tt
 * (2 components each) */
void ibref_curve_tension(int law, double e, double kappa, int npoints, const double* const* rest,
                         const double* const* cur, double* f)
{
	struct curve_family {
		struct geometries { bases::geometry<1> data, sample; };
		geometries ref, cur;
		const geometries& geometry(decltype(bases::reference)) const { return ref; }
		const geometries& geometry(decltype(bases::current)) const { return cur; }
	} obj;
	obj.ref.sample.tangents[0] = from(rest[0], npoints, 2);
	obj.ref.sample.second_derivatives[0] = from(rest[1], npoints, 2);
	obj.ref.sample.sigma = from(rest[2], npoints, 1);
	obj.cur.sample.tangents[0] = from(cur[0], npoints, 2);
	obj.cur.sample.second_derivatives[0] = from(cur[1], npoints, 2);
	obj.cur.sample.sigma = from(rest[2], npoints, 1);      // read by the loader, not by the force
	obj.cur.sample.position = M(npoints, 2);
	const M out = law == 0 ? forces::skalak1d{e, kappa}(obj, M{}) : forces::hookean1d{e}(obj);
	to(out, f);
}

void ibref_membrane_tether(double modulus, int npoints, const double* x_rest, const double* x_cur, double* f)
{
	family obj;
	obj.ref.sample.position = from(x_rest, npoints, 3);
	obj.cur.sample.position = from(x_cur, npoints, 3);
	to(forces::tether{modulus}(obj, M{}), f);
}

} // extern "C"
