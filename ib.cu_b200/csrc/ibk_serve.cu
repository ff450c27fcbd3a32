// Serving: continuous batching of coupled immersed-boundary steps.
//
// No counterpart in the reference (its solver steps one simulation at a
// time).  The server keeps every admitted member's state resident on the
// device -- positions (two buffers, swapped by each step), the spring rest
// shape, spring forces, grid velocity and grid force density -- and serves
// step requests (IBK_OP_STEP: interpolate, forward Euler advection, linear
// spring force, spread) as they arrive.
//
// Each of `slots` CUDA streams owns one batch over all members, with the
// step captured once as a CUDA graph.  progress() reaps finished slots and,
// for every free slot, packs the queued requests whose members are idle into
// one launch: it binds those members (the others idle) and replays the
// slot's graph.  Requests that arrive while launches are on the GPU go to the
// next free slot, so launches overlap on the device.  A member is stepped by
// one launch at a time, in arrival order.  Only host-side work (table
// building, event queries) is on the launch path; nothing synchronises the
// device except an explicit read, retire or destroy.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <new>
#include <random>
#include <string>
#include <thread>
#include <vector>
#include "ibk_internal.h"

namespace ibk {
namespace {

struct Member {
	bool admitted = false, busy = false;
	int n = 0, cur = 0;
	double* x[2] = {nullptr, nullptr};
	double* xref = nullptr;
	double* fs = nullptr;
	double* ue[kMaxDims] = {};
	double* fe[kMaxDims] = {};
	long long bytes = 0;
	long long sizes[kMaxDims] = {};
};

struct Request {
	int member;
	double t_arrival;
};

struct Slot {
	ibk_batch batch = nullptr;
	cudaStream_t stream = nullptr;
	cudaEvent_t done = nullptr;
	bool busy = false;
	std::vector<Request> reqs;
	long long points = 0;
};

} // namespace

struct Server {
	ibk_server_config cfg{};
	int dims = 3;
	std::vector<ibk_instance_desc> desc;
	std::vector<ibk_grid_info> info;
	std::vector<Member> members;
	std::vector<Slot> slots;
	std::deque<Request> queue;
	std::vector<ibk_instance_io> io;      // binding scratch
	std::vector<char> chosen;
	long long admitted_bytes = 0, admitted_points = 0;
	std::chrono::steady_clock::time_point t0;
	// statistics
	std::vector<double> latency_ms;
	long long launches = 0, points = 0;
	double first_arrival = -1.0, last_done = 0.0;
	double launch_host_s = 0.0;           // host time spent in launches
};

namespace {

double now_s(const Server& s)
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now() - s.t0).count();
}

ibk_status cuda_ok(cudaError_t e, const char* what)
{
	if (e == cudaSuccess) return IBK_OK;
	cudaGetLastError();
	return set_error(e == cudaErrorMemoryAllocation ? IBK_ERR_OUT_OF_MEMORY : IBK_ERR_CUDA,
	                 std::string(what) + ": " + cudaGetErrorString(e));
}

void free_member(Member& m)
{
	double* bufs[] = {m.x[0], m.x[1], m.xref, m.fs, m.ue[0], m.ue[1], m.ue[2], m.fe[0], m.fe[1], m.fe[2]};
	for (double* p : bufs)
		if (p) cudaFree(p);
	Member fresh;
	m = fresh;
}

// Completes the finished launches of busy slots.
ibk_status reap(Server& s)
{
	for (Slot& sl : s.slots) {
		if (!sl.busy) continue;
		cudaError_t q = cudaEventQuery(sl.done);
		if (q == cudaErrorNotReady) continue;
		if (q != cudaSuccess) return cuda_ok(q, "cudaEventQuery");
		const double t = now_s(s);
		for (const Request& r : sl.reqs) {
			s.latency_ms.push_back(1000.0 * (t - r.t_arrival));
			s.members[r.member].busy = false;
		}
		s.points += sl.points;
		s.last_done = t;
		sl.reqs.clear();
		sl.busy = false;
	}
	return IBK_OK;
}

// Launches the queued requests of idle members on one free slot.
ibk_status launch(Server& s, Slot& sl)
{
	const double t_start = now_s(s);
	std::fill(s.chosen.begin(), s.chosen.end(), 0);
	sl.reqs.clear();
	sl.points = 0;
	for (auto it = s.queue.begin(); it != s.queue.end();) {
		Member& m = s.members[it->member];
		if (m.busy || s.chosen[it->member]) { ++it; continue; }
		s.chosen[it->member] = 1;
		sl.reqs.push_back(*it);
		it = s.queue.erase(it);
	}
	if (sl.reqs.empty()) return IBK_OK;
	for (size_t i = 0; i < s.members.size(); ++i) {
		ibk_instance_io& e = s.io[i];
		std::memset(&e, 0, sizeof(e));
		if (!s.chosen[i]) continue;
		Member& m = s.members[i];
		e.n = m.n;
		e.x = m.x[m.cur];
		e.xn = m.x[m.cur ^ 1];
		e.xref = m.xref;
		e.fs = m.fs;
		for (int c = 0; c < s.dims; ++c) { e.ue[c] = m.ue[c]; e.fe[c] = m.fe[c]; }
		sl.points += m.n;
	}
	ibk_status st = ibk_batch_bind(sl.batch, s.io.data(), sl.stream);
	if (st == IBK_OK) st = ibk_batch_run(sl.batch, IBK_OP_STEP, sl.stream);
	if (st == IBK_OK) st = cuda_ok(cudaEventRecord(sl.done, sl.stream), "cudaEventRecord");
	if (st != IBK_OK) {
		// give the requests back in their order
		for (auto r = sl.reqs.rbegin(); r != sl.reqs.rend(); ++r) s.queue.push_front(*r);
		sl.reqs.clear();
		return st;
	}
	for (const Request& r : sl.reqs) {
		Member& m = s.members[r.member];
		m.busy = true;
		m.cur ^= 1;          // the step writes the next positions
	}
	sl.busy = true;
	++s.launches;
	s.launch_host_s += now_s(s) - t_start;
	return IBK_OK;
}

ibk_status progress(Server& s, int* pending)
{
	ibk_status st = reap(s);
	if (st != IBK_OK) return st;
	for (Slot& sl : s.slots) {
		if (s.queue.empty()) break;
		if (sl.busy) continue;
		if ((st = launch(s, sl)) != IBK_OK) return st;
	}
	if (pending) {
		int p = (int) s.queue.size();
		for (const Slot& sl : s.slots) p += (int) sl.reqs.size();
		*pending = p;
	}
	return IBK_OK;
}

// Waits (progressing) until member m has no step in flight or queued.
ibk_status wait_member(Server& s, int m)
{
	for (;;) {
		bool queued = false;
		for (const Request& r : s.queue) queued = queued || r.member == m;
		if (!queued && !s.members[m].busy) return IBK_OK;
		ibk_status st = progress(s, nullptr);
		if (st != IBK_OK) return st;
		std::this_thread::yield();
	}
}

void fill_stats(const Server& s, ibk_server_stats* out)
{
	std::memset(out, 0, sizeof(*out));
	out->requests = (long long) s.latency_ms.size();
	out->launches = s.launches;
	out->points = s.points;
	out->admitted_bytes = s.admitted_bytes;
	out->host_ms_per_launch = s.launches ? 1e3 * s.launch_host_s / (double) s.launches : 0.0;
	if (s.latency_ms.empty()) return;
	std::vector<double> v(s.latency_ms);
	std::sort(v.begin(), v.end());
	auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t) (q * (double) (v.size() - 1) + 0.5))]; };
	out->p50_ms = pct(0.50);
	out->p99_ms = pct(0.99);
	out->max_ms = v.back();
	double sum = 0.0;
	for (double x : v) sum += x;
	out->mean_ms = sum / (double) v.size();
	out->wall_s = s.first_arrival >= 0.0 ? s.last_done - s.first_arrival : 0.0;
}

void destroy(Server* s)
{
	for (Slot& sl : s->slots) {
		if (sl.stream) cudaStreamSynchronize(sl.stream);
		if (sl.batch) ibk_batch_destroy(sl.batch);
		if (sl.done) cudaEventDestroy(sl.done);
		if (sl.stream) cudaStreamDestroy(sl.stream);
	}
	for (Member& m : s->members) free_member(m);
	delete s;
}

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_server_create(int members, const ibk_instance_desc* desc, const ibk_server_config* config,
                             ibk_server* out)
{
	if (!out || !desc || !config || members <= 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "null pointer or no members");
	*out = nullptr;
	if (config->slots < 1 || config->slots > 16) return set_error(IBK_ERR_INVALID_ARGUMENT, "slots must lie in [1, 16]");
	if (config->hbm_budget < 0 || config->max_points < 0)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "negative budget or capacity");
	Server* s = new (std::nothrow) Server();
	if (!s) return set_error(IBK_ERR_OUT_OF_MEMORY, "host allocation failed");
	s->cfg = *config;
	s->t0 = std::chrono::steady_clock::now();
	s->desc.assign(desc, desc + members);
	s->dims = desc[0].domain.dims;
	s->members.resize(members);
	s->io.resize(members);
	s->chosen.resize(members);
	s->slots.resize(config->slots);
	ibk_status st = IBK_OK;
	for (Slot& sl : s->slots) {
		if ((st = ibk_batch_create(members, desc, config->delta, config->precision, config->max_points, &sl.batch)) != IBK_OK)
			break;
		if ((st = cuda_ok(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate")) != IBK_OK)
			break;
		if ((st = cuda_ok(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "cudaEventCreate")) != IBK_OK)
			break;
		if ((st = ibk_batch_set_step(sl.batch, config->dt, config->k)) != IBK_OK) break;
		// the step graph, captured on an all-idle binding: it reads the
		// binding made before each replay
		std::vector<ibk_instance_io> idle(members);
		std::memset(idle.data(), 0, sizeof(ibk_instance_io) * members);
		if ((st = ibk_batch_bind(sl.batch, idle.data(), sl.stream)) != IBK_OK) break;
		if ((st = ibk_batch_capture(sl.batch, IBK_OP_STEP)) != IBK_OK) break;
	}
	if (st == IBK_OK) {
		s->info.resize(members);
		for (int i = 0; i < members && st == IBK_OK; ++i) st = ibk_batch_info(s->slots[0].batch, i, &s->info[i]);
	}
	if (st != IBK_OK) { destroy(s); return st; }
	*out = reinterpret_cast<ibk_server>(s);
	return IBK_OK;
}

ibk_status ibk_server_destroy(ibk_server handle)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (s) destroy(s);
	return IBK_OK;
}

ibk_status ibk_server_admit(ibk_server handle, int member, int n, const double* x, const double* const* ue)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || member < 0 || member >= (int) s->members.size() || n < 0 || (n > 0 && !x) || !ue)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or arrays, bad member or count");
	Member& m = s->members[member];
	if (m.admitted) return set_error(IBK_ERR_INVALID_ARGUMENT, "member already admitted");
	const ibk_grid_info& gi = s->info[member];
	long long bytes = 4LL * s->dims * n * (long long) sizeof(double);
	for (int c = 0; c < s->dims; ++c) bytes += 2LL * gi.size[c] * (long long) sizeof(double);
	if (s->admitted_points + n > s->cfg.max_points)
		return set_error(IBK_ERR_CAPACITY, "members' points exceed the server's max_points");
	if (s->admitted_bytes + bytes > s->cfg.hbm_budget)
		return set_error(IBK_ERR_CAPACITY, "member state exceeds the HBM budget (" + std::to_string(s->cfg.hbm_budget) +
		                 " bytes)");
	size_t free_b = 0, total_b = 0;
	ibk_status st = cuda_ok(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
	if (st != IBK_OK) return st;
	if ((long long) free_b < bytes + (256LL << 20))
		return set_error(IBK_ERR_CAPACITY, "device has too little free memory for the member");
	const size_t pbytes = sizeof(double) * (size_t) s->dims * (size_t) std::max(n, 1);
	double** pts[] = {&m.x[0], &m.x[1], &m.xref, &m.fs};
	for (double** p : pts)
		if (st == IBK_OK) st = cuda_ok(cudaMalloc(reinterpret_cast<void**>(p), pbytes), "cudaMalloc");
	for (int c = 0; c < s->dims && st == IBK_OK; ++c) {
		m.sizes[c] = gi.size[c];
		const size_t gb = sizeof(double) * (size_t) gi.size[c];
		st = cuda_ok(cudaMalloc(reinterpret_cast<void**>(&m.ue[c]), gb), "cudaMalloc");
		if (st == IBK_OK) st = cuda_ok(cudaMalloc(reinterpret_cast<void**>(&m.fe[c]), gb), "cudaMalloc");
		if (st == IBK_OK) st = cuda_ok(cudaMemcpy(m.ue[c], ue[c], gb, cudaMemcpyHostToDevice), "cudaMemcpy");
		if (st == IBK_OK) st = cuda_ok(cudaMemset(m.fe[c], 0, gb), "cudaMemset");
	}
	const size_t xb = sizeof(double) * (size_t) s->dims * (size_t) n;
	if (st == IBK_OK && n > 0) st = cuda_ok(cudaMemcpy(m.x[0], x, xb, cudaMemcpyHostToDevice), "cudaMemcpy");
	if (st == IBK_OK && n > 0) st = cuda_ok(cudaMemcpy(m.xref, x, xb, cudaMemcpyHostToDevice), "cudaMemcpy");
	if (st == IBK_OK) st = cuda_ok(cudaMemset(m.fs, 0, pbytes), "cudaMemset");
	if (st == IBK_OK) st = cuda_ok(cudaMemset(m.x[1], 0, pbytes), "cudaMemset");
	if (st != IBK_OK) { free_member(m); return st; }
	m.admitted = true;
	m.n = n;
	m.cur = 0;
	m.bytes = bytes;
	s->admitted_bytes += bytes;
	s->admitted_points += n;
	return IBK_OK;
}

ibk_status ibk_server_retire(ibk_server handle, int member)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || member < 0 || member >= (int) s->members.size() || !s->members[member].admitted)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or member not admitted");
	ibk_status st = wait_member(*s, member);
	if (st != IBK_OK) return st;
	s->admitted_bytes -= s->members[member].bytes;
	s->admitted_points -= s->members[member].n;
	free_member(s->members[member]);
	return IBK_OK;
}

ibk_status ibk_server_submit(ibk_server handle, int member, double t_arrival)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || member < 0 || member >= (int) s->members.size() || !s->members[member].admitted)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or member not admitted");
	const double t = t_arrival < 0.0 ? now_s(*s) : t_arrival;
	if (s->first_arrival < 0.0 || t < s->first_arrival) s->first_arrival = t;
	s->queue.push_back(Request{member, t});
	return IBK_OK;
}

ibk_status ibk_server_progress(ibk_server handle, int* pending)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s) return set_error(IBK_ERR_INVALID_ARGUMENT, "null server");
	return progress(*s, pending);
}

ibk_status ibk_server_drain(ibk_server handle)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s) return set_error(IBK_ERR_INVALID_ARGUMENT, "null server");
	for (;;) {
		int pending = 0;
		ibk_status st = progress(*s, &pending);
		if (st != IBK_OK) return st;
		if (pending == 0) return IBK_OK;
		std::this_thread::yield();
	}
}

double ibk_server_clock(ibk_server handle)
{
	Server* s = reinterpret_cast<Server*>(handle);
	return s ? now_s(*s) : 0.0;
}

ibk_status ibk_server_read(ibk_server handle, int member, double* x, double* const* fe)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || member < 0 || member >= (int) s->members.size() || !s->members[member].admitted)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or member not admitted");
	ibk_status st = wait_member(*s, member);
	if (st != IBK_OK) return st;
	Member& m = s->members[member];
	if ((st = cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) != IBK_OK) return st;
	if (x && m.n > 0)
		st = cuda_ok(cudaMemcpy(x, m.x[m.cur], sizeof(double) * s->dims * (size_t) m.n, cudaMemcpyDeviceToHost),
		             "cudaMemcpy");
	for (int c = 0; fe && c < s->dims && st == IBK_OK; ++c)
		if (fe[c])
			st = cuda_ok(cudaMemcpy(fe[c], m.fe[c], sizeof(double) * (size_t) m.sizes[c], cudaMemcpyDeviceToHost),
			             "cudaMemcpy");
	return st;
}

ibk_status ibk_server_save(ibk_server handle, int member, const char* path)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || !path || member < 0 || member >= (int) s->members.size() || !s->members[member].admitted)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or path, or member not admitted");
	ibk_status st = wait_member(*s, member);
	if (st != IBK_OK) return st;
	Member& m = s->members[member];
	if ((st = cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) != IBK_OK) return st;
	const size_t pn = (size_t) s->dims * (size_t) m.n;
	std::vector<double> buf(pn);
	const double* pts[2] = {m.x[m.cur], m.xref};
	for (int k = 0; k < 2 && st == IBK_OK; ++k) {
		if (pn) st = cuda_ok(cudaMemcpy(buf.data(), pts[k], sizeof(double) * pn, cudaMemcpyDeviceToHost), "cudaMemcpy");
		if (st == IBK_OK) st = ibk_io_write_dense(path, k, 1, m.n, s->dims, buf.data());
	}
	for (int pass = 0; pass < 2 && st == IBK_OK; ++pass)
		for (int c = 0; c < s->dims && st == IBK_OK; ++c) {
			std::vector<double> g((size_t) m.sizes[c]);
			st = cuda_ok(cudaMemcpy(g.data(), pass == 0 ? m.ue[c] : m.fe[c], sizeof(double) * g.size(),
			                        cudaMemcpyDeviceToHost), "cudaMemcpy");
			if (st == IBK_OK) st = ibk_io_write_dense(path, 1, 0, (int) g.size(), 1, g.data());
		}
	return st;
}

ibk_status ibk_server_admit_from(ibk_server handle, int member, const char* path)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || !path || member < 0 || member >= (int) s->members.size())
		return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or path, or bad member");
	long long off = 0;
	ibk_io_header h{};
	std::vector<double> x, xref;
	std::vector<std::vector<double>> grids(2 * s->dims);
	ibk_status st = IBK_OK;
	for (int k = 0; k < 2 && st == IBK_OK; ++k) {
		std::vector<double>& dst = k == 0 ? x : xref;
		if ((st = ibk_io_read_dense(path, off, &h, nullptr, 0, nullptr)) != IBK_OK) break;
		if (!h.matrix || h.cols != s->dims) { st = set_error(IBK_ERR_INVALID_ARGUMENT, "checkpoint positions are not n x dims"); break; }
		dst.resize((size_t) h.count);
		st = ibk_io_read_dense(path, off, &h, dst.data(), h.count, &off);
	}
	if (st == IBK_OK && xref.size() != x.size()) st = set_error(IBK_ERR_INVALID_ARGUMENT, "checkpoint shapes differ");
	for (int j = 0; j < 2 * s->dims && st == IBK_OK; ++j) {
		const int c = j % s->dims;
		if ((st = ibk_io_read_dense(path, off, &h, nullptr, 0, nullptr)) != IBK_OK) break;
		if (h.count != s->info[member].size[c]) { st = set_error(IBK_ERR_INVALID_ARGUMENT, "checkpoint grid size differs from the member's grid"); break; }
		grids[j].resize((size_t) h.count);
		st = ibk_io_read_dense(path, off, &h, grids[j].data(), h.count, &off);
	}
	if (st != IBK_OK) return st;
	const int n = (int) (x.size() / (size_t) s->dims);
	const double* ue[kMaxDims] = {nullptr, nullptr, nullptr};
	for (int c = 0; c < s->dims; ++c) ue[c] = grids[c].data();
	if ((st = ibk_server_admit(handle, member, n, x.data(), ue)) != IBK_OK) return st;
	Member& m = s->members[member];
	if (n > 0) st = cuda_ok(cudaMemcpy(m.xref, xref.data(), sizeof(double) * xref.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
	for (int c = 0; c < s->dims && st == IBK_OK; ++c)
		st = cuda_ok(cudaMemcpy(m.fe[c], grids[s->dims + c].data(), sizeof(double) * grids[s->dims + c].size(),
		                        cudaMemcpyHostToDevice), "cudaMemcpy");
	if (st != IBK_OK) {
		// a member restored only in part is not left admitted: release it as
		// retire does (nothing of it is in flight yet) and report the error
		const std::string msg = ibk_last_error();
		s->admitted_bytes -= m.bytes;
		s->admitted_points -= m.n;
		free_member(m);
		return set_error(st, msg);
	}
	return IBK_OK;
}

ibk_status ibk_server_get_stats(ibk_server handle, ibk_server_stats* stats)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || !stats) return set_error(IBK_ERR_INVALID_ARGUMENT, "null server or stats");
	fill_stats(*s, stats);
	return IBK_OK;
}

ibk_status ibk_server_reset_stats(ibk_server handle)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s) return set_error(IBK_ERR_INVALID_ARGUMENT, "null server");
	s->latency_ms.clear();
	s->launches = 0;
	s->points = 0;
	s->first_arrival = -1.0;
	s->last_done = 0.0;
	s->launch_host_s = 0.0;
	return IBK_OK;
}

ibk_status ibk_server_run_poisson(ibk_server handle, double rate_per_s, int requests, unsigned long long seed,
                                  ibk_server_stats* stats)
{
	Server* s = reinterpret_cast<Server*>(handle);
	if (!s || !(rate_per_s > 0.0) || requests < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "null server, bad rate or count");
	std::vector<int> live;
	for (int i = 0; i < (int) s->members.size(); ++i)
		if (s->members[i].admitted) live.push_back(i);
	if (live.empty()) return set_error(IBK_ERR_INVALID_ARGUMENT, "no admitted members");
	ibk_status st = ibk_server_drain(handle);
	if (st != IBK_OK) return st;
	ibk_server_reset_stats(handle);
	std::mt19937_64 rng(seed);
	std::exponential_distribution<double> gap(rate_per_s);
	std::uniform_int_distribution<int> pick(0, (int) live.size() - 1);
	std::vector<Request> arrivals(requests);
	double t = now_s(*s) + 1e-3;
	for (Request& r : arrivals) {
		t += gap(rng);
		r = Request{live[pick(rng)], t};
	}
	size_t next = 0;
	for (;;) {
		const double now = now_s(*s);
		while (next < arrivals.size() && arrivals[next].t_arrival <= now) {
			s->queue.push_back(arrivals[next]);
			if (s->first_arrival < 0.0) s->first_arrival = arrivals[next].t_arrival;
			++next;
		}
		int pending = 0;
		if ((st = progress(*s, &pending)) != IBK_OK) return st;
		if (pending == 0 && next == arrivals.size()) break;
		if (pending == 0) {
			// idle until the next arrival (sleep through long gaps)
			const double wait = arrivals[next].t_arrival - now_s(*s);
			if (wait > 2e-3) std::this_thread::sleep_for(std::chrono::duration<double>(wait - 1e-3));
		}
	}
	if (stats) fill_stats(*s, stats);
	return IBK_OK;
}

} // extern "C"
