/*
 * Serving loop: continuous batching of queries over HBM-resident tables.
 *
 * The reference executes one query at a time, each as its own launch
 * sequence (src/vm/execute.c:85-86, src/vm/vm_gpu.cu:474-565).  Here a
 * scheduler thread keeps one persistent VM kernel running (a "session") and
 * folds arriving queries into it while it runs:
 *
 *  - admission: queries are admitted in arrival order while the result
 *    arena (the result budget, one device allocation) has room for their
 *    estimated result size and the session has descriptor slots left.  The
 *    estimate is the caller's, else the rows the same program last returned
 *    on the same table, else the share of the table's host row sample its
 *    filter keeps (estimate.cpp), each with a margin, else the bound (the
 *    table's rows); a query whose rows exceed its reservation is admitted
 *    again with exactly its row count;
 *  - folding in: the scheduler writes the admitted queries' descriptors to
 *    device memory on an upload stream, waits for that copy, then publishes
 *    the new query and work counts through a doorbell word in host-mapped
 *    memory.  The kernel's producer warps poll the doorbell when they run
 *    out of published work, so new chunks are claimed as soon as CTAs free
 *    up, interleaved with the chunks of queries already running;
 *  - completion: after a chunk's rows are stored, the last compute warp of
 *    its CTA to finish counts it; the chunk that completes a query writes
 *    the query's row count and sequence number to a completion record in
 *    host-mapped memory, which the scheduler polls;
 *  - sessions end when the loop is idle, when the session's descriptor
 *    slots are used up or when its work numbering nears 2^31; the next
 *    admission starts a new one.
 *
 * Look-back words are a ring of kStatusRing words tagged by lap, since a
 * session's work list has no fixed length.  Every wait in the kernel is
 * bounded by the session's wait limit.
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "virginian_b200.h"
#include "vgpu_engine.h"
#include "vgpu_util.h"
#include "engine_internal.h"

using namespace vgpu;

#define CUDA_OK(call, what)                                                   \
	do {                                                                      \
		cudaError_t e_ = (call);                                              \
		if (e_ != cudaSuccess)                                                \
			VGPU_FAIL("%s: %s", what, cudaGetErrorString(e_));                 \
	} while (0)

namespace {

constexpr unsigned kStatusRingBits = 22;  /* 4M look-back words, 32 MB */
constexpr uint64_t kStatusRing = 1ull << kStatusRingBits;
constexpr uint64_t kSessionWorkLimit = 1ull << 31;
/* (program, table) pairs whose last result size is remembered */
constexpr size_t kHistoryLimit = 1 << 16;
constexpr size_t kChunkPoolWords = 4u << 20;  /* segment chunk prefixes per session */
constexpr uint32_t kServeChunkRows = kMaxChunkRows;  /* the bound; each query's chunk fills its buffers */

using Clock = std::chrono::steady_clock;

double since_us(Clock::time_point a, Clock::time_point b)
{
	return std::chrono::duration<double, std::micro>(b - a).count();
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

/* first-fit allocator over [0, size) */
struct Arena {
	std::map<size_t, size_t> free_;  /* offset -> size */
	size_t size = 0, used = 0;
	void reset(size_t n)
	{
		free_.clear();
		free_[0] = n;
		size = n;
		used = 0;
	}
	bool alloc(size_t n, size_t *off)
	{
		for (auto it = free_.begin(); it != free_.end(); ++it)
			if (it->second >= n) {
				*off = it->first;
				const size_t rest = it->second - n;
				const size_t at = it->first + n;
				free_.erase(it);
				if (rest)
					free_[at] = rest;
				used += n;
				return true;
			}
		return false;
	}
	void release(size_t off, size_t n)
	{
		used -= n;
		auto it = free_.emplace(off, n).first;
		auto nx = std::next(it);
		if (nx != free_.end() && it->first + it->second == nx->first) {
			it->second += nx->second;
			free_.erase(nx);
		}
		if (it != free_.begin()) {
			auto pv = std::prev(it);
			if (pv->first + pv->second == it->first) {
				pv->second += it->second;
				free_.erase(it);
			}
		}
	}
};

}  // namespace

struct virg_serve {
	virg_gpu_engine *e = nullptr;
	virg_serve_config cfg{};
	/* the session's launch geometry (one for every query it takes): the
	 * wide layout holds every program the bounds admit; the narrow one,
	 * when it has larger data buffers, holds programs with fewer vector
	 * bytes.  A session runs one of them; a query at the head of the queue
	 * that the running session's layout does not match ends it once its
	 * queries are done, and the next session takes the other layout */
	Geom geom{};
	Geom geom_wide{}, geom_narrow{};
	bool have_narrow = false, session_narrow = false;
	unsigned narrow_row = 0, narrow_sel = 0;
	unsigned grid = 0;
	cudaStream_t kstream = nullptr, ustream = nullptr;
	/* device memory */
	QDesc *d_queries = nullptr;
	uint64_t *d_prefix = nullptr;
	uint32_t *d_chunks = nullptr;
	uint64_t *d_status = nullptr;
	unsigned *d_done = nullptr;
	unsigned long long *d_totals = nullptr;
	unsigned *d_ctrl = nullptr;  /* [0] work counter, [1] error word */
	unsigned char *d_arena = nullptr;
	/* host-mapped memory */
	ServeCtl *h_ctl = nullptr, *d_ctl = nullptr;
	ServeRec *h_recs = nullptr, *d_recs = nullptr;
	/* pinned staging for descriptor uploads */
	QDesc *h_qstage = nullptr;
	uint64_t *h_pstage = nullptr;
	uint32_t *h_cstage = nullptr;

	struct Query {
		uint64_t ticket;
		const virg_gpu_program *p;
		virg_gpu_table *t;
		uint64_t estimate_rows;
		Clock::time_point submitted, admitted, completed;
		/* while in flight */
		uint32_t qi = 0;
		uint64_t nchunks = 0;
		size_t arena_off = 0, arena_bytes = 0;
		uint64_t capacity = 0;
		void *out[kMaxRegs] = {nullptr};
		uint64_t rows = 0;
		int state = 0;  /* 0 pending, 1 in flight, 2 done, 3 failed */
		std::string error;  /* why it failed */
		unsigned readmits = 0;
		bool narrow = false;  /* fits the narrow layout */
	};
	std::map<uint64_t, Query> queries;
	std::deque<uint64_t> pending;
	std::vector<uint64_t> inflight;  /* tickets, in admission order */
	uint64_t next_ticket = 1;
	Arena arena;

	/* session state */
	bool running = false;
	uint32_t nq = 0;
	uint64_t work = 0;
	size_t chunk_words = 0;  /* segment chunk prefixes written this session */
	Clock::time_point idle_since;
	unsigned sessions = 0;
	unsigned long long launches = 0, admitted_total = 0, readmitted = 0, restarts = 0;
	unsigned device_error = 0;

	std::mutex mu;
	std::condition_variable cv;  /* completions, for waiters */
	std::thread sched;
	std::atomic<bool> quit{false};
	std::atomic<unsigned long long> sampled{0};  /* submissions estimated from a table sample */
	std::string fail;
	/* result rows each (program, table) pair last had, with the table's rows
	 * then: the default estimate of its next submission */
	std::map<std::pair<const virg_gpu_program *, const virg_gpu_table *>, std::pair<uint64_t, uint64_t>> history;
};

namespace {

int serve_layout(virg_serve *s)
{
	virg_gpu_engine *e = s->e;
	/* eight compute warps, one CTA per SM, the largest data buffers (48 KB
	 * down to 8 KB, each holding a group of blocks of the widest staging the session
	 * admits) of which at least two fit beside the warps' vector areas.  The
	 * session's full phase reads staged tiles in place (no gather area). */
	const unsigned min_kb = (kCountGroup * kBlockRows * s->cfg.max_load_bytes_per_row + 1023) / 1024;
	bool fit = false;
	for (unsigned min_stages : {3u, 2u}) {
		for (unsigned kb : {48u, 40u, 32u, 24u, 16u, 8u}) {
			Shape sh = {256, std::max(kb, min_kb), 0, 1, kServeChunkRows, 0};
			if (geom_make(sh, s->cfg.max_sel_vector_bytes, s->cfg.max_row_vector_bytes, 0u, e->smem_optin,
					e->smem_sm, &s->geom, 1) && s->geom.shape.stages >= min_stages) {
				fit = true;
				break;
			}
		}
		if (fit)
			break;
	}
	VGPU_CHECK(fit, "serving layout does not fit shared memory (vectors of %u + %u bytes per row)",
		s->cfg.max_sel_vector_bytes, s->cfg.max_row_vector_bytes);
	s->geom_wide = s->geom;
	/* the narrow layout: three 48 KB buffers for programs of at most 8
	 * filter-vector and 20 projection-vector bytes per row (within the
	 * bounds), if that beats the wide layout's buffers */
	s->narrow_row = std::min(s->cfg.max_row_vector_bytes, 8u);
	s->narrow_sel = std::min(s->cfg.max_sel_vector_bytes, 20u);
	{
		Shape sh = {256, std::max(48u, min_kb), 3, 1, kServeChunkRows, 0};
		Geom g;
		s->have_narrow = sh.stage_kb > s->geom_wide.shape.stage_kb &&
			geom_make(sh, s->narrow_sel, s->narrow_row, 0u, e->smem_optin, e->smem_sm, &g, 1);
		if (s->have_narrow) {
			int n = 0;
			s->have_narrow = occupancy(g.shape, g.smem, &n) && n >= 1;
			s->geom_narrow = g;
		}
		set_error("%s", "");
	}
	int per_sm = 0;
	if (!occupancy(s->geom.shape, s->geom.smem, &per_sm))
		VGPU_FAIL("occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
	VGPU_CHECK(per_sm >= 1, "the serving kernel cannot be resident");
	s->grid = (unsigned)e->nsm;
	return 1;
}

/* does a program fit the narrow layout */
bool fits_narrow(const virg_serve *s, const Program &P)
{
	if (!s->have_narrow)
		return false;
	ProgPlan pp;
	plan_program(P, pp);
	return pp.row_bpr <= s->narrow_row && pp.sel_bpr <= s->narrow_sel;
}

/* does a program fit the session's layout */
int program_fits(const virg_serve *s, const Program &P, const char **why)
{
	ProgPlan pp;
	plan_program(P, pp);
	if (pp.count_bpr > s->cfg.max_load_bytes_per_row || pp.full_bpr > s->cfg.max_load_bytes_per_row) {
		*why = "the program stages more bytes per row than the serving layout holds";
		return 0;
	}
	if (pp.row_bpr > s->cfg.max_row_vector_bytes || pp.sel_bpr > s->cfg.max_sel_vector_bytes) {
		*why = "the program needs more register-vector bytes than the serving layout holds";
		return 0;
	}
	return 1;
}

size_t arena_need(const Program &P, uint64_t cap)
{
	size_t b = 0;
	for (unsigned j = 0; j < P.nout; j++)
		b += align_up(std::max<uint64_t>(cap, 1) * P.out_stride[j], 256);
	return std::max<size_t>(b, 256);
}

uint64_t query_chunks(const virg_gpu_table *t, uint32_t chunk_rows)
{
	return chunk_prefix(t->seg_rows.data(), (uint32_t)t->seg_rows.size(), chunk_rows, nullptr);
}

/* does the query at the head of the queue need the other layout than the
 * running session's */
bool head_mismatch(const virg_serve *s)
{
	if (!s->have_narrow || s->pending.empty())
		return false;
	return s->queries.at(s->pending.front()).narrow != s->session_narrow;
}

/* start a session: clear its counters and look-back ring, launch the kernel
 * with the layout the query at the head of the queue needs */
int session_start(virg_serve *s)
{
	s->session_narrow = s->have_narrow && !s->pending.empty() && s->queries.at(s->pending.front()).narrow;
	s->geom = s->session_narrow ? s->geom_narrow : s->geom_wide;
	CUDA_OK(cudaMemsetAsync(s->d_ctrl, 0, 2 * sizeof(unsigned), s->kstream), "session reset");
	CUDA_OK(cudaMemsetAsync(s->d_status, 0, kStatusRing * sizeof(uint64_t), s->kstream), "status reset");
	CUDA_OK(cudaMemsetAsync(s->d_done, 0, s->cfg.max_queries * sizeof(unsigned), s->kstream), "done reset");
	s->h_ctl->avail = 0;
	s->h_ctl->stop = 0;
	memset(s->h_recs, 0, s->cfg.max_queries * sizeof(ServeRec));
	std::atomic_thread_fence(std::memory_order_seq_cst);
	KParams kp = geom_params(s->geom);
	kp.queries = s->d_queries;
	kp.q_work_prefix = s->d_prefix;
	kp.nq = 0;
	kp.total_work = 0xffffffffu;
	kp.counter = s->d_ctrl;
	kp.status = s->d_status;
	kp.error = s->d_ctrl + 1;
	kp.epoch = 1;
	kp.status_mask = kStatusRing - 1;
	kp.status_shift = kStatusRingBits;
	kp.wait_limit_ms = s->cfg.wait_limit_ms;
	kp.serve = s->d_ctl;
	kp.recs = s->d_recs;
	kp.done_chunks = s->d_done;
	if (!launch_vm(s->geom.shape, kp, s->grid, s->geom.smem, s->kstream))
		VGPU_FAIL("serving kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
	s->running = true;
	s->nq = 0;
	s->work = 0;
	s->chunk_words = 0;
	s->sessions++;
	s->launches++;
	s->idle_since = Clock::now();
	return 1;
}

/* stop the session: the kernel finishes what it holds and exits */
int session_stop(virg_serve *s)
{
	if (!s->running)
		return 1;
	std::atomic_thread_fence(std::memory_order_seq_cst);
	s->h_ctl->stop = 1;
	std::atomic_thread_fence(std::memory_order_seq_cst);
	const cudaError_t ce = cudaStreamSynchronize(s->kstream);
	s->running = false;
	VGPU_CHECK(ce == cudaSuccess, "serving session: %s", cudaGetErrorString(ce));
	unsigned err = 0;
	CUDA_OK(cudaMemcpy(&err, s->d_ctrl + 1, sizeof(err), cudaMemcpyDeviceToHost), "session error read");
	if (err && !s->device_error)
		s->device_error = err;
	return 1;
}

/* admit pending queries into the running session: descriptors, upload,
 * doorbell.  Returns the number admitted. */
unsigned admit(virg_serve *s)
{
	std::vector<uint64_t> batch;
	const uint32_t nq0 = s->nq;
	uint64_t work = s->work;
	size_t chunk_words = s->chunk_words;
	while (!s->pending.empty() && nq0 + batch.size() < s->cfg.max_queries && !head_mismatch(s)) {
		auto &q = s->queries[s->pending.front()];
		const Program &P = q.p->prog;
		/* descriptor (its chunking depends on the program's staging) */
		const uint32_t qi = nq0 + (uint32_t)batch.size();
		QDesc &d = s->h_qstage[batch.size()];
		memset(&d, 0, sizeof(d));
		ProgPlan pp;
		plan_program(P, pp);
		if (!desc_fill(d, P, pp, s->geom, kServeChunkRows)) {
			s->fail = last_error();
			return 0;
		}
		const uint32_t nsegs = (uint32_t)q.t->segs.size();
		const uint64_t nchunks = query_chunks(q.t, d.chunk_rows);
		if (work + nchunks >= kSessionWorkLimit || chunk_words + nsegs + 1 > kChunkPoolWords)
			break;
		const uint64_t cap = std::min<uint64_t>(q.estimate_rows, q.t->rows);
		const size_t need = arena_need(P, cap);
		size_t off;
		if (!s->arena.alloc(need, &off))
			break;
		q.arena_off = off;
		q.arena_bytes = need;
		q.capacity = cap;
		unsigned char *p = s->d_arena + off;
		for (unsigned j = 0; j < P.nout; j++) {
			q.out[j] = p;
			p += align_up(std::max<uint64_t>(cap, 1) * P.out_stride[j], 256);
		}
		d.segs = q.t->d_segs;
		d.nsegs = nsegs;
		d.seg_chunk_prefix = s->d_chunks + chunk_words;
		chunk_prefix(q.t->seg_rows.data(), nsegs, d.chunk_rows, s->h_cstage + chunk_words);
		chunk_words += nsegs + 1;
		d.work_first = work;
		d.nchunks = nchunks;
		for (unsigned j = 0; j < P.nout; j++)
			d.out_ptr[j] = q.out[j];
		d.capacity = cap;
		d.total_out = s->d_totals + qi;
		d.block_counts = nullptr;
		d.base_in = nullptr;
		s->h_pstage[batch.size()] = work;
		work += nchunks;
		q.qi = qi;
		q.nchunks = nchunks;
		q.state = 1;
		q.admitted = Clock::now();
		batch.push_back(q.ticket);
		s->pending.pop_front();
	}
	if (batch.empty())
		return 0;
	const size_t b = batch.size();
	const size_t c0 = s->chunk_words;
	cudaError_t ce = cudaMemcpyAsync(s->d_queries + nq0, s->h_qstage, b * sizeof(QDesc), cudaMemcpyHostToDevice,
		s->ustream);
	if (ce == cudaSuccess)
		ce = cudaMemcpyAsync(s->d_prefix + nq0, s->h_pstage, b * sizeof(uint64_t), cudaMemcpyHostToDevice,
			s->ustream);
	if (ce == cudaSuccess)
		ce = cudaMemcpyAsync(s->d_chunks + c0, s->h_cstage + c0, (chunk_words - c0) * sizeof(uint32_t),
			cudaMemcpyHostToDevice, s->ustream);
	if (ce == cudaSuccess)
		ce = cudaStreamSynchronize(s->ustream);
	if (ce != cudaSuccess) {
		s->fail = std::string("descriptor upload: ") + cudaGetErrorString(ce);
		return 0;
	}
	s->nq = nq0 + (uint32_t)b;
	s->work = work;
	s->chunk_words = chunk_words;
	/* the doorbell: descriptors are in device memory before they are counted */
	std::atomic_thread_fence(std::memory_order_seq_cst);
	s->h_ctl->avail = ((unsigned long long)s->nq << 40) | (s->work & kAvailWorkMask);
	std::atomic_thread_fence(std::memory_order_seq_cst);
	/* queries without rows complete at once */
	for (uint64_t tk : batch) {
		auto &q = s->queries[tk];
		s->admitted_total++;
		if (q.nchunks == 0) {
			q.rows = 0;
			q.state = 2;
			q.completed = Clock::now();
		} else {
			s->inflight.push_back(tk);
		}
	}
	return (unsigned)b;
}

/* completion records of the running session */
unsigned harvest(virg_serve *s)
{
	unsigned n = 0;
	std::vector<uint64_t> keep;
	keep.reserve(s->inflight.size());
	for (uint64_t tk : s->inflight) {
		auto &q = s->queries[tk];
		volatile ServeRec *r = s->h_recs + q.qi;
		if (r->seq != (unsigned long long)q.qi + 1ull) {
			keep.push_back(tk);
			continue;
		}
		std::atomic_thread_fence(std::memory_order_acquire);
		const uint64_t rows = r->rows;
		n++;
		if (rows > q.capacity) {
			/* more rows than reserved: again, with exactly that many, unless
			 * that many can never fit the result budget */
			s->arena.release(q.arena_off, q.arena_bytes);
			q.arena_bytes = 0;
			if (arena_need(q.p->prog, rows) > s->cfg.result_budget_bytes) {
				char buf[160];
				snprintf(buf, sizeof(buf), "the query's %llu result rows need %zu bytes, more than the result budget",
					(unsigned long long)rows, arena_need(q.p->prog, rows));
				q.error = buf;
				q.state = 3;
				q.completed = Clock::now();
				continue;
			}
			q.estimate_rows = rows;
			q.state = 0;
			q.readmits++;
			s->readmitted++;
			s->pending.push_front(tk);
			continue;
		}
		q.rows = rows;
		q.state = 2;
		q.completed = Clock::now();
		if (s->history.size() >= kHistoryLimit)
			s->history.clear();
		s->history[{q.p, q.t}] = {rows, q.t->rows};
	}
	s->inflight.swap(keep);
	return n;
}

void scheduler(virg_serve *s)
{
	cudaSetDevice(s->e->device);
	while (!s->quit.load()) {
		bool busy = false;
		{
			std::unique_lock<std::mutex> lk(s->mu);
			if (s->running && !s->inflight.empty() && harvest(s))
				busy = true;
			/* a session kernel that ended by itself (a bounded wait ran out:
			 * the device error word says which) is over: its finished
			 * queries keep their results, the others are admitted again
			 * into a new session */
			if (s->running && cudaStreamQuery(s->kstream) != cudaErrorNotReady) {
				harvest(s);
				if (!session_stop(s))
					s->fail = last_error();
				for (auto it = s->inflight.rbegin(); it != s->inflight.rend(); ++it) {
					auto &q = s->queries[*it];
					s->arena.release(q.arena_off, q.arena_bytes);
					q.arena_bytes = 0;
					q.state = 0;
					q.readmits++;
					s->readmitted++;
					s->pending.push_front(*it);
				}
				s->inflight.clear();
				s->restarts++;
				busy = true;
			}
			/* a session that cannot take the next query ends once drained */
			if (s->running && !s->pending.empty() && s->inflight.empty() &&
				(s->nq >= s->cfg.max_queries || s->work >= kSessionWorkLimit / 2 ||
				 s->chunk_words > kChunkPoolWords / 2 || head_mismatch(s))) {
				if (!session_stop(s))
					s->fail = last_error();
			}
			if (!s->pending.empty()) {
				if (!s->running && s->fail.empty() && !session_start(s))
					s->fail = last_error();
				if (s->running && admit(s))
					busy = true;
			}
			if (busy || !s->inflight.empty() || !s->pending.empty())
				s->idle_since = Clock::now();
			else if (s->running && since_us(s->idle_since, Clock::now()) > s->cfg.idle_us) {
				if (!session_stop(s))
					s->fail = last_error();
			}
			if (busy)
				s->cv.notify_all();
		}
		if (!busy)
			std::this_thread::sleep_for(std::chrono::microseconds(s->inflight.empty() ? 50 : 5));
	}
	std::unique_lock<std::mutex> lk(s->mu);
	session_stop(s);
	s->cv.notify_all();
}

}  // namespace

extern "C" int virg_serve_create(virg_gpu_engine *e, const virg_serve_config *cfg, virg_serve **out)
{
	VGPU_CHECK(e != nullptr && out != nullptr, "null argument");
	*out = nullptr;
	CUDA_OK(cudaSetDevice(e->device), "set device");
	virg_serve *s = new virg_serve();
	s->e = e;
	if (cfg)
		s->cfg = *cfg;
	auto &c = s->cfg;
	if (!c.result_budget_bytes)
		c.result_budget_bytes = 20ull << 30;
	if (!c.max_queries)
		c.max_queries = 4096;
	if (!c.idle_us)
		c.idle_us = 50000;
	if (!c.max_load_bytes_per_row)
		c.max_load_bytes_per_row = 32;
	/* the default vector bounds (12 and 20 bytes per row) leave three
	 * 40 KB data buffers beside eight compute warps' areas */
	if (!c.max_row_vector_bytes)
		c.max_row_vector_bytes = 12;
	if (!c.max_sel_vector_bytes)
		c.max_sel_vector_bytes = 20;
	if (!c.wait_limit_ms)
		c.wait_limit_ms = 60000;
	auto fail = [&](const char *what, cudaError_t ce) {
		set_error("%s: %s", what, cudaGetErrorString(ce));
		virg_serve_destroy(s);
		return 0;
	};
	if (!serve_layout(s)) {
		delete s;
		return 0;
	}
	cudaError_t ce;
	if ((ce = cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking)) != cudaSuccess)
		return fail("stream", ce);
	if ((ce = cudaStreamCreateWithFlags(&s->ustream, cudaStreamNonBlocking)) != cudaSuccess)
		return fail("stream", ce);
	const size_t nqc = c.max_queries;
	if ((ce = cudaMalloc((void **)&s->d_queries, nqc * sizeof(QDesc))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_prefix, (nqc + 1) * sizeof(uint64_t))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_chunks, kChunkPoolWords * sizeof(uint32_t))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_status, kStatusRing * sizeof(uint64_t))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_done, nqc * sizeof(unsigned))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_totals, nqc * sizeof(unsigned long long))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_ctrl, 2 * sizeof(unsigned))) != cudaSuccess ||
		(ce = cudaMalloc((void **)&s->d_arena, c.result_budget_bytes)) != cudaSuccess)
		return fail("serving device memory", ce);
	if ((ce = cudaHostAlloc((void **)&s->h_ctl, sizeof(ServeCtl), cudaHostAllocMapped)) != cudaSuccess ||
		(ce = cudaHostAlloc((void **)&s->h_recs, nqc * sizeof(ServeRec), cudaHostAllocMapped)) != cudaSuccess ||
		(ce = cudaHostGetDevicePointer((void **)&s->d_ctl, s->h_ctl, 0)) != cudaSuccess ||
		(ce = cudaHostGetDevicePointer((void **)&s->d_recs, s->h_recs, 0)) != cudaSuccess)
		return fail("serving mapped memory", ce);
	if ((ce = cudaMallocHost((void **)&s->h_qstage, nqc * sizeof(QDesc))) != cudaSuccess ||
		(ce = cudaMallocHost((void **)&s->h_pstage, (nqc + 1) * sizeof(uint64_t))) != cudaSuccess ||
		(ce = cudaMallocHost((void **)&s->h_cstage, kChunkPoolWords * sizeof(uint32_t))) != cudaSuccess)
		return fail("serving staging memory", ce);
	memset(s->h_ctl, 0, sizeof(ServeCtl));
	s->arena.reset(c.result_budget_bytes);
	s->sched = std::thread(scheduler, s);
	*out = s;
	return 1;
}

extern "C" int virg_serve_submit(virg_serve *s, const virg_gpu_program *p, virg_gpu_table *t,
	uint64_t estimated_rows, uint64_t *ticket)
{
	VGPU_CHECK(s != nullptr && p != nullptr && t != nullptr && ticket != nullptr, "null argument");
	VGPU_CHECK(t->e == s->e, "table belongs to another engine");
	const Program &P = p->prog;
	const char *why = nullptr;
	VGPU_CHECK(program_fits(s, P, &why), "%s", why);
	for (unsigned i = 0; i < P.nload; i++) {
		if (P.load_src[i] == kKeySlot)
			VGPU_CHECK(t->segs_without_key == 0 && P.load_stride[i] == 4,
				"program reads the key column, which the table does not hold with that type");
		else
			VGPU_CHECK(P.load_src[i] < t->schema.ncols && t->schema.col_type[P.load_src[i]] == (int)P.load_type[i],
				"program column %u does not match the table schema", P.load_src[i]);
	}
	{
		std::lock_guard<std::mutex> elk(s->e->mu);
		if (!table_sync_desc(t))
			return 0;
	}
	const uint64_t bound = t->rows;
	uint64_t est = estimated_rows ? std::min(estimated_rows, bound) : bound;
	if (!estimated_rows) {
		/* the selectivity this program last had on this table, else the
		 * fraction of the table's host sample its filter keeps, with a
		 * margin; a short estimate is admitted again with its exact rows */
		bool known = false;
		{
			std::lock_guard<std::mutex> lk(s->mu);
			auto h = s->history.find({p, t});
			if (h != s->history.end() && h->second.second == bound) {
				est = std::min<uint64_t>(bound, h->second.first + h->second.first / 4 + 1024);
				known = true;
			}
		}
		const double sel = known ? -1.0 : sample_selectivity(P, t);
		if (sel >= 0.0) {
			est = std::min<uint64_t>(bound, (uint64_t)(sel * 1.25 * (double)bound) + 4096);
			s->sampled.fetch_add(1);
		}
	}
	VGPU_CHECK(arena_need(P, est) <= s->cfg.result_budget_bytes,
		"the query's result reservation (%zu bytes) exceeds the result budget", arena_need(P, est));
	std::lock_guard<std::mutex> lk(s->mu);
	VGPU_CHECK(s->fail.empty(), "serving loop failed: %s", s->fail.c_str());
	virg_serve::Query q;
	q.ticket = s->next_ticket++;
	q.p = p;
	q.t = t;
	q.estimate_rows = est;
	q.narrow = fits_narrow(s, P);
	q.submitted = Clock::now();
	s->queries.emplace(q.ticket, q);
	s->pending.push_back(q.ticket);
	*ticket = q.ticket;
	return 1;
}

extern "C" int virg_serve_poll(virg_serve *s, uint64_t ticket, int wait_ms, virg_serve_status *st)
{
	VGPU_CHECK(s != nullptr && st != nullptr, "null argument");
	std::unique_lock<std::mutex> lk(s->mu);
	auto it = s->queries.find(ticket);
	VGPU_CHECK(it != s->queries.end(), "unknown ticket %llu", (unsigned long long)ticket);
	if (wait_ms != 0) {
		auto pred = [&] { return it->second.state >= 2 || !s->fail.empty(); };
		if (wait_ms < 0)
			s->cv.wait(lk, pred);
		else
			s->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
	}
	VGPU_CHECK(s->fail.empty(), "serving loop failed: %s", s->fail.c_str());
	const auto &q = it->second;
	VGPU_CHECK(q.state != 3, "query %llu failed: %s", (unsigned long long)ticket, q.error.c_str());
	st->done = q.state == 2;
	st->rows = q.rows;
	st->readmits = q.readmits;
	st->queue_us = q.state >= 1 ? since_us(q.submitted, q.admitted) : 0.0;
	st->latency_us = q.state == 2 ? since_us(q.submitted, q.completed) : 0.0;
	return 1;
}

extern "C" int virg_serve_download(virg_serve *s, uint64_t ticket, void *const *host_cols)
{
	VGPU_CHECK(s != nullptr && host_cols != nullptr, "null argument");
	/* the columns' places under the lock; the copies without it, so that
	 * submissions and the scheduler go on during a long download (a
	 * completed result stays where it is until its ticket is released) */
	const void *src[kMaxRegs];
	size_t bytes[kMaxRegs];
	unsigned nout = 0;
	{
		std::lock_guard<std::mutex> lk(s->mu);
		auto it = s->queries.find(ticket);
		VGPU_CHECK(it != s->queries.end(), "unknown ticket %llu", (unsigned long long)ticket);
		const auto &q = it->second;
		VGPU_CHECK(q.state == 2, "query %llu has not completed", (unsigned long long)ticket);
		const Program &P = q.p->prog;
		nout = q.rows ? P.nout : 0u;
		for (unsigned j = 0; j < nout; j++) {
			src[j] = q.out[j];
			bytes[j] = q.rows * P.out_stride[j];
		}
	}
	for (unsigned j = 0; j < nout; j++)
		CUDA_OK(cudaMemcpy(host_cols[j], src[j], bytes[j], cudaMemcpyDeviceToHost), "result download");
	return 1;
}

extern "C" const void *virg_serve_column(virg_serve *s, uint64_t ticket, unsigned c)
{
	if (!s)
		return nullptr;
	std::lock_guard<std::mutex> lk(s->mu);
	auto it = s->queries.find(ticket);
	if (it == s->queries.end() || it->second.state != 2 || c >= it->second.p->prog.nout)
		return nullptr;
	return it->second.out[c];
}

extern "C" int virg_serve_release(virg_serve *s, uint64_t ticket)
{
	VGPU_CHECK(s != nullptr, "null argument");
	std::lock_guard<std::mutex> lk(s->mu);
	auto it = s->queries.find(ticket);
	VGPU_CHECK(it != s->queries.end(), "unknown ticket %llu", (unsigned long long)ticket);
	VGPU_CHECK(it->second.state >= 2, "query %llu has not completed", (unsigned long long)ticket);
	if (it->second.arena_bytes)
		s->arena.release(it->second.arena_off, it->second.arena_bytes);
	s->queries.erase(it);
	return 1;
}

extern "C" int virg_serve_stats(virg_serve *s, virg_serve_counters *c)
{
	VGPU_CHECK(s != nullptr && c != nullptr, "null argument");
	std::lock_guard<std::mutex> lk(s->mu);
	c->sessions = s->sessions;
	c->admitted = s->admitted_total;
	c->readmitted = s->readmitted;
	c->pending = s->pending.size();
	c->inflight = s->inflight.size();
	c->arena_used = s->arena.used;
	c->device_error = s->device_error;
	c->restarts = s->restarts;
	c->work_items = s->work;
	c->sampled = s->sampled.load();
	c->status_ring = kStatusRing;
	c->shape[0] = s->geom.shape.threads;
	c->shape[1] = s->geom.shape.stage_kb;
	c->shape[2] = s->geom.shape.stages;
	c->shape[3] = s->grid;
	return 1;
}

extern "C" void virg_serve_destroy(virg_serve *s)
{
	if (!s)
		return;
	cudaSetDevice(s->e->device);
	if (s->sched.joinable()) {
		s->quit.store(true);
		s->sched.join();
	}
	if (s->kstream)
		cudaStreamSynchronize(s->kstream);
	cudaFree(s->d_queries);
	cudaFree(s->d_prefix);
	cudaFree(s->d_chunks);
	cudaFree(s->d_status);
	cudaFree(s->d_done);
	cudaFree(s->d_totals);
	cudaFree(s->d_ctrl);
	cudaFree(s->d_arena);
	if (s->h_ctl)
		cudaFreeHost(s->h_ctl);
	if (s->h_recs)
		cudaFreeHost(s->h_recs);
	if (s->h_qstage)
		cudaFreeHost(s->h_qstage);
	if (s->h_pstage)
		cudaFreeHost(s->h_pstage);
	if (s->h_cstage)
		cudaFreeHost(s->h_cstage);
	if (s->kstream)
		cudaStreamDestroy(s->kstream);
	if (s->ustream)
		cudaStreamDestroy(s->ustream);
	delete s;
}
