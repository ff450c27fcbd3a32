// ibk.hpp -- C++ adapter over the C ABI (ibk.h) with the reference's call
// surface, so an ib::solver-style step can swap its operators:
//
//   reference (include/ib/novel.h:193-250, include/ib/interpolate.h:88-138):
//     ib::spread      spread{fd::mac{64}, domain, ib::delta::bspline<3>{}};
//     ib::interpolate interp{fd::mac{64}, domain, ib::delta::bspline<3>{}};
//     spread(n, x, fl, fe);     interp(n, x, ue, ul);
//   this library:
//     ibk::spread      spread{ibk::mac{64}, domain, ibk::bspline<3>{}};
//     ibk::interpolate interp{ibk::mac{64}, domain, ibk::bspline<3>{}};
//     spread(n, x, fl, fe);     interp(n, x, ue, ul);
//
// Arrays are raw device pointers with the reference's layouts (x[d*n+p];
// grid components x-fastest).  Errors throw ibk::error, as the reference
// throws cuda::exception (include/cuda/exceptions.h:34-46); n <= 0 returns
// at once (include/ib/novel.h:201).
#pragma once
#include <array>
#include <stdexcept>
#include <string>
#include "ibk.h"

namespace ibk {

struct error : std::runtime_error {
	ibk_status status;
	error(ibk_status s, const char* what) : std::runtime_error(std::string(ibk_status_string(s)) + ": " + what), status(s) {}
};

inline void check(ibk_status s)
{
	if (s != IBK_OK) throw error(s, ibk_last_error());
}

// fd::boundary (include/fd/boundary.h:31-42)
struct periodic_t { static constexpr int kind = IBK_PERIODIC; };
struct solid_t { static constexpr int kind = IBK_SOLID; };
inline constexpr periodic_t periodic{};
inline constexpr solid_t dirichlet{}, neumann{}, robin{};

// fd::dimension / fd::domain (include/fd/dimension.h, include/fd/domain.h)
struct dimension {
	double length;
	int boundary;
	template <typename B> constexpr dimension(double l, B) : length(l), boundary(B::kind) {}
};

struct domain {
	ibk_domain d{};
	template <typename... Ds> explicit domain(const Ds&... dims)
	{
		const dimension ds[] = {dims...};
		d.dims = (int) sizeof...(Ds);
		for (int i = 0; i < d.dims; ++i) { d.length[i] = ds[i].length; d.boundary[i] = ds[i].boundary; }
	}
};

// fd::mac / fd::centered (include/fd/cell.h:194-196)
struct mac { int refinement; static constexpr int tag = IBK_TAG_MAC; };
struct centered { int refinement; static constexpr int tag = IBK_TAG_CENTERED; };

// ib::delta kernels (include/ib/{bspline,peskin,roma,cosine,hat}.h)
template <int n> struct bspline { static constexpr ibk_delta value{IBK_DELTA_BSPLINE, n}; };
struct peskin { static constexpr ibk_delta value{IBK_DELTA_PESKIN, 0}; };
struct roma { static constexpr ibk_delta value{IBK_DELTA_ROMA, 0}; };
struct cosine { static constexpr ibk_delta value{IBK_DELTA_COSINE, 0}; };
struct hat { static constexpr ibk_delta value{IBK_DELTA_HAT, 0}; };

class plan {
public:
	template <typename Tag, typename Delta>
	plan(const Tag& tag, const domain& dom, Delta, int precision = IBK_PRECISION_FP64)
	{
		check(ibk_plan_create(&dom.d, Tag::tag, tag.refinement, Delta::value, precision, &h_));
		check(ibk_plan_info(h_, &info_));
	}
	plan(const plan&) = delete;
	plan& operator=(const plan&) = delete;
	~plan() { ibk_plan_destroy(h_); }
	const ibk_grid_info& info() const { return info_; }
	ibk_plan handle() const { return h_; }
protected:
	ibk_plan h_ = nullptr;
	ibk_grid_info info_{};
};

// ib::spread (include/ib/novel.h:197-227): overwrites every face of fe.
class spread : public plan {
public:
	using plan::plan;
	void operator()(int n, const double* x, const double* fl, const std::array<double*, 3>& fe,
	                void* stream = nullptr) const
	{
		if (n <= 0) return;
		check(ibk_spread(h_, n, x, fl, fe.data(), stream));
	}
};

// ib::interpolate (include/ib/interpolate.h:92-115): overwrites ul.
class interpolate : public plan {
public:
	using plan::plan;
	void operator()(int n, const double* x, const std::array<const double*, 3>& ue, double* ul,
	                void* stream = nullptr) const
	{
		if (n <= 0) return;
		check(ibk_interpolate(h_, n, x, ue.data(), ul, stream));
	}
};

} // namespace ibk
