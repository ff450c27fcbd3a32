// Runs the C++ adapter (include/ibk.hpp) on the GPU in the reference's call
// forms and writes inputs and outputs for the Python test to compare with
// the oracle.  Cases:
//   0: the reference's test/grid.cc:28-57 setup -- a periodic 10 um cube,
//      fd::mac{16}, two points at (5, 5, 5) um, unit forces and velocities;
//   1: a walled channel (3.2 x 1.6 x 3.2 units, walls in y, fd::mac{64})
//      with seeded points, forces and velocities.
// Per case the file holds: dims, n, lengths[3], boundaries[3], refinement,
// x (3n), fl (3n), then for each component its size and ue, then the outputs
// of spread(n, x, fl), spread(n, x, fl, fe), interp(n, x, ue, ul) and
// interp(n, x, ue).  Usage: adapter_run <output file>
#include <cstdint>
#include <cstdio>
#include <vector>
#include "ibk.hpp"

namespace {

void put(FILE* out, const void* p, size_t bytes) { fwrite(p, 1, bytes, out); }

std::vector<double> host(const double* d, long long n)
{
	std::vector<double> h((size_t) n);
	if (cudaMemcpy(h.data(), d, sizeof(double) * (size_t) n, cudaMemcpyDeviceToHost) != cudaSuccess)
		throw ibk::error(IBK_ERR_CUDA, "cudaMemcpy");
	return h;
}

double* device(const std::vector<double>& h)
{
	double* d = nullptr;
	if (cudaMalloc(reinterpret_cast<void**>(&d), sizeof(double) * h.size()) != cudaSuccess ||
	    cudaMemcpy(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
		throw ibk::error(IBK_ERR_CUDA, "cudaMalloc / cudaMemcpy");
	return d;
}

struct Lcg {
	uint64_t s;
	double next() { s = s * 6364136223846793005ull + 1442695040888963407ull; return (double) (s >> 11) * 0x1p-53; }
};

void run_case(FILE* out, const ibk::domain& dom, int refinement, const std::vector<double>& x,
              const std::vector<double>& fl, Lcg& rng)
{
	const int n = (int) (x.size() / 3);
	ibk::spread spread{ibk::mac{refinement}, dom, ibk::bspline<3>{}};
	ibk::interpolate interp{ibk::mac{refinement}, dom, ibk::bspline<3>{}};
	const ibk_grid_info& info = spread.info();
	const int dims = info.dims;
	put(out, &dims, sizeof dims);
	put(out, &n, sizeof n);
	put(out, dom.d.length, sizeof dom.d.length);
	put(out, dom.d.boundary, sizeof dom.d.boundary);
	put(out, &refinement, sizeof refinement);
	put(out, x.data(), sizeof(double) * x.size());
	put(out, fl.data(), sizeof(double) * fl.size());
	std::vector<std::vector<double>> ue(3);
	std::array<const double*, 3> ued{nullptr, nullptr, nullptr};
	for (int c = 0; c < dims; ++c) {
		ue[c].resize((size_t) info.size[c]);
		for (double& v : ue[c]) v = refinement == 16 ? 1.0 : 2.0 * rng.next() - 1.0;
		ued[c] = device(ue[c]);
		const long long sz = info.size[c];
		put(out, &sz, sizeof sz);
		put(out, ue[c].data(), sizeof(double) * ue[c].size());
	}
	double* xd = device(x);
	double* fd = device(fl);
	// spread(n, x, fl): new zeroed vectors (include/ib/novel.h:236-244)
	auto fe_new = spread(n, xd, fd);
	// spread(n, x, fl, fe): overwrites every face of NaN-filled vectors
	std::array<double*, 3> fe{nullptr, nullptr, nullptr};
	for (int c = 0; c < dims; ++c)
		fe[c] = device(std::vector<double>((size_t) info.size[c], 0.0 / 0.0));
	spread(n, xd, fd, fe);
	// interp(n, x, ue, ul) and interp(n, x, ue)
	double* ul = device(std::vector<double>((size_t) dims * n, 0.0 / 0.0));
	interp(n, xd, ued, ul);
	auto ul_new = interp(n, xd, ued);
	for (int c = 0; c < dims; ++c) {
		auto a = host(fe_new[c].values(), info.size[c]);
		auto b = host(fe[c], info.size[c]);
		put(out, a.data(), sizeof(double) * a.size());
		put(out, b.data(), sizeof(double) * b.size());
	}
	auto u1 = host(ul, (long long) dims * n);
	auto u2 = host(ul_new.values(), ul_new.size());
	put(out, u1.data(), sizeof(double) * u1.size());
	put(out, u2.data(), sizeof(double) * u2.size());
	for (int c = 0; c < dims; ++c) { cudaFree(fe[c]); cudaFree(const_cast<double*>(ued[c])); }
	cudaFree(ul);
	cudaFree(xd);
	cudaFree(fd);
}

} // namespace

int main(int argc, char** argv)
{
	if (argc != 2) { fprintf(stderr, "usage: adapter_run <output file>\n"); return 2; }
	FILE* out = fopen(argv[1], "wb");
	if (!out) { perror("fopen"); return 2; }
	try {
		Lcg rng{12345};
		// case 0: test/grid.cc (units: 1 um = 0.1)
		{
			ibk::domain dom{ibk::dimension{1.0, ibk::periodic}, ibk::dimension{1.0, ibk::periodic},
			                ibk::dimension{1.0, ibk::periodic}};
			const int n = 2;
			std::vector<double> x(3 * n, 0.5), fl(3 * n, 1.0);
			run_case(out, dom, 16, x, fl, rng);
		}
		// case 1: a walled channel with seeded points (some beyond the walls)
		{
			ibk::domain dom{ibk::dimension{3.2, ibk::periodic}, ibk::dimension{1.6, ibk::dirichlet},
			                ibk::dimension{3.2, ibk::periodic}};
			const int n = 5000;
			const double L[3] = {3.2, 1.6, 3.2};
			std::vector<double> x(3 * n), fl(3 * n);
			for (int d = 0; d < 3; ++d)
				for (int p = 0; p < n; ++p) x[(size_t) d * n + p] = (1.1 * rng.next() - 0.05) * L[d];
			for (double& v : fl) v = 2.0 * rng.next() - 1.0;
			run_case(out, dom, 64, x, fl, rng);
		}
	} catch (const std::exception& e) {
		fprintf(stderr, "adapter_run: %s\n", e.what());
		fclose(out);
		return 1;
	}
	fclose(out);
	return 0;
}
