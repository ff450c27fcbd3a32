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
#include <utility>
#include <vector>
#include <cuda_runtime.h>
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

// Device array returned by the allocating overloads (the reference returns
// linalg vectors allocated by util::memory, include/ib/novel.h:236-244 and
// include/ib/interpolate.h:124-131).
class device_vector {
public:
	device_vector() = default;
	explicit device_vector(long long n) : n_(n)
	{
		if (n <= 0) return;
		cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p_), sizeof(double) * (size_t) n);
		if (e != cudaSuccess) throw error(IBK_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
		e = cudaMemset(p_, 0, sizeof(double) * (size_t) n);
		if (e != cudaSuccess) throw error(IBK_ERR_CUDA, cudaGetErrorString(e));
	}
	device_vector(const device_vector&) = delete;
	device_vector& operator=(const device_vector&) = delete;
	device_vector(device_vector&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
	device_vector& operator=(device_vector&& o) noexcept
	{
		std::swap(p_, o.p_);
		std::swap(n_, o.n_);
		return *this;
	}
	~device_vector() { if (p_) cudaFree(p_); }
	double* values() { return p_; }
	const double* values() const { return p_; }
	long long size() const { return n_; }
private:
	double* p_ = nullptr;
	long long n_ = 0;
};

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
	// (n, x, fl): new zeroed grid vectors, then spread (include/ib/novel.h:236-244)
	std::array<device_vector, 3> operator()(int n, const double* x, const double* fl, void* stream = nullptr) const
	{
		std::array<device_vector, 3> fe;
		std::array<double*, 3> ptrs{nullptr, nullptr, nullptr};
		for (int c = 0; c < info_.dims; ++c) {
			fe[c] = device_vector(info_.size[c]);
			ptrs[c] = fe[c].values();
		}
		(*this)(n, x, fl, ptrs, stream);
		return fe;
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
	// (n, x, ue): a new dims*n vector (include/ib/interpolate.h:124-131)
	device_vector operator()(int n, const double* x, const std::array<const double*, 3>& ue,
	                         void* stream = nullptr) const
	{
		device_vector ul((long long) info_.dims * (n > 0 ? n : 0));
		(*this)(n, x, ue, ul.values(), stream);
		return ul;
	}
};

// Many grids per launch (no reference counterpart): see ibk_batch_* in ibk.h.
class batch {
public:
	template <typename Tag>
	batch(const std::vector<std::pair<Tag, domain>>& instances, ibk_delta delta, int precision, int max_points)
	{
		std::vector<ibk_instance_desc> d(instances.size());
		for (size_t i = 0; i < instances.size(); ++i)
			d[i] = ibk_instance_desc{instances[i].second.d, Tag::tag, instances[i].first.refinement};
		check(ibk_batch_create((int) d.size(), d.data(), delta, precision, max_points, &h_));
	}
	batch(const batch&) = delete;
	batch& operator=(const batch&) = delete;
	~batch() { ibk_batch_destroy(h_); }
	void bind(const std::vector<ibk_instance_io>& io, void* stream = nullptr) { check(ibk_batch_bind(h_, io.data(), stream)); }
	void run(int op, void* stream = nullptr) { check(ibk_batch_run(h_, op, stream)); }
	void capture(int op) { check(ibk_batch_capture(h_, op)); }
	void set_step(double dt, double k) { check(ibk_batch_set_step(h_, dt, k)); }
	ibk_batch_config tune(int op, void* stream = nullptr)
	{
		ibk_batch_config c{};
		check(ibk_batch_tune(h_, op, stream, &c));
		return c;
	}
	ibk_batch handle() const { return h_; }
private:
	ibk_batch h_ = nullptr;
};

} // namespace ibk
