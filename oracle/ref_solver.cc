/*
 * The reference's own preconditioned CG and Chebyshev preconditioner,
 * compiled on the host (TEST INFRASTRUCTURE: only oracle.py loads it, to check
 * the oracle's restatement of the diffusion solve).
 *
 * include/solvers/pcg.h and algo/chebyshev.h are compiled as they are, with
 * -Iref_shim_solver standing in for the CUDA linalg layer (a host vector, the
 * reductions as plain sums in index order) and for what algo/gershgorin.h
 * names from thrust and the launcher.  The preconditioner is built here as
 * solvers/preconditioners/chebyshev.h builds it, algo::chebyshev(upper,
 * lower, H), from the caller's Gershgorin interval; the operator is the
 * caller's, through a callback.  Built by `make -C oracle ref
 * REF=<sonwell/ib.cu tree>`.
 */
#include <cstring>
#include "algo/chebyshev.h"
#include "solvers/pcg.h"

namespace {

// preconditioners::chebyshev (solvers/preconditioners/chebyshev.h:9-26) with
// its interval given: algo::chebyshev(range.second, range.first, H)
struct chebyshev_pr : algo::chebyshev, solvers::preconditioner {
	chebyshev_pr(double lower, double upper, algo::matrix m) : algo::chebyshev(upper, lower, std::move(m)) {}
	solvers::dense::vector operator()(solvers::dense::vector b) const override
	{
		return algo::chebyshev::operator()(std::move(b));
	}
};

struct counted {
	linalg::apply_fn apply;
	void* ctx;
	long long calls = 0;
};

void count_apply(const double* in, double* out, void* ctx)
{
	auto* c = static_cast<counted*>(ctx);
	++c->calls;
	c->apply(in, out, c->ctx);
}

} // namespace

extern "C" {

/* x = H^-1 b by solvers::pcg with the Chebyshev preconditioner, as
 * solvers::chebpcg{H, tol} solves; returns the operator applications */
long long ibref_chebpcg(int n, linalg::apply_fn apply, void* ctx, double lower, double upper, const double* b,
                        double tol, double* x)
{
	counted c{apply, ctx};
	linalg::matrix<linalg::sparse<double>> h;
	h.apply = count_apply;
	h.ctx = &c;
	h.n = n;
	const chebyshev_pr pr(lower, upper, h);
	linalg::dvec rhs(n);
	std::memcpy(rhs.values(), b, sizeof(double) * (std::size_t) n);
	const linalg::dvec out = solvers::pcg(pr, h, std::move(rhs), tol);      // chebpcg.h:16-19
	std::memcpy(x, out.values(), sizeof(double) * (std::size_t) n);
	return c.calls;
}

/* impl::chebw<4>(a, b).weights (algo/chebyshev.h:124-145) */
void ibref_chebyshev_weights(double a, double b, double* w)
{
	const algo::impl::chebw<4> cw(a, b);
	for (int i = 0; i < 4; ++i) w[i] = cw.weights[i];
}

} // extern "C"
