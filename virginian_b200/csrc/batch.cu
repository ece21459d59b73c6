/*
 * Batched persistent execution: many queries over many resident tables in
 * one launch of the VM kernel.
 *
 * The reference runs one query at a time: one launch sequence per data
 * tablet with a blocking copy of its result count after each
 * (src/vm/vm_gpu.cu:474-565).  A batch numbers the chunks of all its queries
 * into one work list; persistent CTAs claim chunks in order, so small and
 * large tables share the machine and a query's ordered look-back chain only
 * waits on that query's earlier chunks.  A batch owns its descriptors,
 * look-back words, work counter and result counters, so its launch (counter
 * and status reset, kernel, count read-back) can be captured once in a CUDA
 * graph and replayed.  The launch shape (compute warps, stage size and
 * count, CTAs per SM, chunk size) can be tuned by timing the candidates on
 * the batch itself; the winner is cached in the engine per program-shape
 * key.
 */
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

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

/* epoch reserved for graph-replayed batches: their status words are cleared
 * before every replay, so a fixed epoch is safe */
constexpr uint32_t kBatchEpoch = kEpochMask;

/* programs whose table sample says they keep at least this share of the
 * rows form their own part of a batch */
constexpr double kDensePartSel = 0.5;

}  // namespace

struct virg_gpu_batch {
	virg_gpu_engine *e = nullptr;
	struct Item {
		const virg_gpu_program *p;
		virg_gpu_table *t;
		virg_gpu_result *r;
	};
	std::vector<Item> items;
	/* one launch per part: the programs whose compute warps' vector areas
	 * leave three 48 KB data buffers, and the others (a launch's areas are
	 * sized for its widest program, so one wide program would shrink every
	 * query's buffers) */
	struct Part {
		std::vector<size_t> items;
		Plan plan;
		unsigned char *d_blob = nullptr;
		uint64_t *d_status = nullptr;
	};
	std::vector<Part> parts;
	bool built = false;
	unsigned *d_ctrl = nullptr;            /* per part p: [2p] work counter, [2p + 1] error */
	unsigned long long *d_totals = nullptr;
	unsigned long long *h_totals = nullptr;  /* pinned */
	unsigned *h_ctrl = nullptr;              /* pinned copy of d_ctrl */
	cudaGraphExec_t gexec = nullptr;
	cudaEvent_t done = nullptr;
	bool ran = false;
	bool tune = false;
	double last_ms = 0;
};

namespace {

void batch_release(virg_gpu_batch *b)
{
	cudaStream_t s = b->e->stream;
	cudaStreamSynchronize(s);
	if (b->gexec)
		cudaGraphExecDestroy(b->gexec);
	b->gexec = nullptr;
	for (auto &it : b->items)
		if (it.r) {
			virg_gpu_result_destroy(it.r);
			it.r = nullptr;
		}
	for (auto &pt : b->parts) {
		if (pt.d_blob) cudaFree(pt.d_blob);
		if (pt.d_status) cudaFree(pt.d_status);
	}
	b->parts.clear();
	if (b->d_ctrl) cudaFree(b->d_ctrl);
	if (b->d_totals) cudaFree(b->d_totals);
	if (b->h_totals) cudaFreeHost(b->h_totals);
	if (b->h_ctrl) cudaFreeHost(b->h_ctrl);
	b->d_ctrl = nullptr;
	b->d_totals = nullptr;
	b->h_totals = nullptr;
	b->h_ctrl = nullptr;
	b->built = false;
	b->ran = false;
}

std::vector<QueryLaunch> launches_of(virg_gpu_batch *b, size_t part)
{
	std::vector<QueryLaunch> qs;
	for (size_t i : b->parts[part].items) {
		auto &it = b->items[i];
		QueryLaunch q;
		q.prog = &it.p->prog;
		q.d_segs = it.t->d_segs;
		q.nsegs = (uint32_t)it.t->segs.size();
		q.seg_rows = it.t->seg_rows.data();
		for (unsigned j = 0; j < it.p->prog.nout; j++)
			q.out[j] = it.r->out[j];
		q.capacity = it.t->rows;
		q.d_total = b->d_totals + i;
		q.block_counts = nullptr;
		qs.push_back(q);
	}
	return qs;
}

/* the launch sequence (captured into the graph, or issued directly) */
int issue(virg_gpu_batch *b)
{
	virg_gpu_engine *e = b->e;
	cudaStream_t s = e->stream;
	const size_t np = b->parts.size();
	CUDA_OK(cudaMemsetAsync(b->d_ctrl, 0, 2 * np * sizeof(unsigned), s), "batch counter reset");
	CUDA_OK(cudaMemsetAsync(b->d_totals, 0, b->items.size() * sizeof(unsigned long long), s),
		"batch totals reset");
	for (size_t p = 0; p < np; p++) {
		const auto &pt = b->parts[p];
		const Plan &plan = pt.plan;
		if (!plan.work)
			continue;
		CUDA_OK(cudaMemsetAsync(pt.d_status, 0, plan.work * sizeof(uint64_t), s), "batch status reset");
		const KParams kp = plan_params(plan, pt.d_blob, b->d_ctrl + 2 * p, pt.d_status, b->d_ctrl + 2 * p + 1,
			kBatchEpoch);
		if (!launch_vm(plan.geom.shape, kp, plan.grid, plan.geom.smem, s))
			VGPU_FAIL("batch kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
	}
	CUDA_OK(cudaMemcpyAsync(b->h_totals, b->d_totals, b->items.size() * sizeof(unsigned long long),
		cudaMemcpyDeviceToHost, s), "batch totals read");
	CUDA_OK(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, 2 * np * sizeof(unsigned), cudaMemcpyDeviceToHost, s),
		"batch error read");
	return 1;
}

/* the first part's device error, once the batch's copies have landed */
unsigned batch_error(const virg_gpu_batch *b)
{
	for (size_t p = 0; p < b->parts.size(); p++)
		if (b->h_ctrl[2 * p + 1])
			return b->h_ctrl[2 * p + 1];
	return 0;
}

/* the part with the most work (its shape is the batch's reported shape) */
size_t main_part(const virg_gpu_batch *b)
{
	size_t m = 0;
	for (size_t p = 1; p < b->parts.size(); p++)
		if (b->parts[p].plan.work > b->parts[m].plan.work)
			m = p;
	return m;
}

int build_with(virg_gpu_batch *b, size_t part, const Shape *forced)
{
	virg_gpu_engine *e = b->e;
	auto &pt = b->parts[part];
	std::vector<QueryLaunch> qs = launches_of(b, part);
	size_t off_prefix, off_chunks;
	const size_t bytes = plan_blob_bytes(qs, &off_prefix, &off_chunks);
	if (!pt.d_blob)
		CUDA_OK(cudaMalloc((void **)&pt.d_blob, bytes), "batch descriptor alloc");
	Plan plan;
	if (!plan_build(e, qs, forced, pt.d_blob, plan))
		return 0;
	CUDA_OK(cudaMemcpy(pt.d_blob, plan.blob.data(), plan.blob.size(), cudaMemcpyHostToDevice),
		"batch descriptor copy");
	if (pt.d_status && pt.plan.work < plan.work) {
		cudaFree(pt.d_status);
		pt.d_status = nullptr;
	}
	if (!pt.d_status)
		CUDA_OK(cudaMalloc((void **)&pt.d_status, std::max<uint64_t>(plan.work, 1) * sizeof(uint64_t)),
			"batch status alloc");
	pt.plan = std::move(plan);
	if (b->gexec) {
		cudaGraphExecDestroy(b->gexec);
		b->gexec = nullptr;
	}
	return 1;
}

float time_once(virg_gpu_batch *b)
{
	virg_gpu_engine *e = b->e;
	cudaEvent_t a, z;
	cudaEventCreate(&a);
	cudaEventCreate(&z);
	cudaEventRecord(a, e->stream);
	int ok = issue(b);
	cudaEventRecord(z, e->stream);
	cudaEventSynchronize(z);
	float ms = -1;
	if (ok)
		cudaEventElapsedTime(&ms, a, z);
	cudaEventDestroy(a);
	cudaEventDestroy(z);
	return ok && batch_error(b) == 0 ? ms : -1.0f;
}

/* tune each part in turn (the others at their current shapes), timing the
 * whole batch; the winner is cached per part's program-shape key */
int autotune_part(virg_gpu_batch *b, size_t part)
{
	virg_gpu_engine *e = b->e;
	const std::string key = shape_key(launches_of(b, part));
	auto hit = e->tuned.find(key);
	if (hit != e->tuned.end())
		return build_with(b, part, &hit->second);
	float best = 1e30f;
	Shape best_shape = {0, 0, 0, 0, 0, 0};
	for (const Shape &c : tune_candidates()) {
		set_error("%s", "");
		if (!build_with(b, part, &c))
			continue;  /* does not fit shared memory */
		float t = 1e30f;
		for (int rep = 0; rep < 3; rep++) {
			float ms = time_once(b);
			if (ms < 0)
				VGPU_FAIL("autotune run failed");
			t = std::min(t, ms);
		}
		if (t < best) {
			best = t;
			best_shape = b->parts[part].plan.geom.shape;
		}
	}
	VGPU_CHECK(best_shape.threads != 0, "no launch shape fits this batch");
	tune_remember(e, key, best_shape);
	return build_with(b, part, &best_shape);
}

/* split the items into parts.  A launch's warp areas hold its largest
 * selection, row and gather vectors (possibly of different programs), so
 * the first part is the set of programs under a pair of limits (row vector
 * bytes r, selection vector bytes s) whose combined layout leaves three
 * 48 KB data buffers beside eight compute warps, chosen to cover the most
 * table rows; the others form the second part (one part if either is
 * empty).  Item order is kept within a part. */
void make_parts(virg_gpu_batch *b)
{
	virg_gpu_engine *e = b->e;
	const size_t n = b->items.size();
	std::vector<ProgPlan> pp(n);
	std::vector<uint32_t> rows_opts, sel_opts;
	for (size_t i = 0; i < n; i++) {
		plan_program(b->items[i].p->prog, pp[i], e->pref.full_mode);
		rows_opts.push_back(pp[i].row_bpr);
		sel_opts.push_back(pp[i].sel_bpr);
	}
	std::sort(rows_opts.begin(), rows_opts.end());
	rows_opts.erase(std::unique(rows_opts.begin(), rows_opts.end()), rows_opts.end());
	std::sort(sel_opts.begin(), sel_opts.end());
	sel_opts.erase(std::unique(sel_opts.begin(), sel_opts.end()), sel_opts.end());
	const Shape s = {256, 48, 3, 1, 0, e->pref.full_mode};
	auto fits = [&](uint32_t sel, uint32_t row, uint32_t gat) {
		Geom g;
		return geom_make(s, sel, row, gat, e->smem_optin, e->smem_sm, &g, 1) != 0;
	};
	uint64_t best_w = 0;
	uint32_t best_r = 0, best_s = 0;
	bool have = false;
	for (uint32_t r : rows_opts) {
		for (auto it = sel_opts.rbegin(); it != sel_opts.rend(); ++it) {
			uint32_t gat = 0;
			uint64_t w = 0;
			for (size_t i = 0; i < n; i++)
				if (pp[i].row_bpr <= r && pp[i].sel_bpr <= *it) {
					gat = std::max(gat, pp[i].gather_bpr);
					w += b->items[i].t->rows + 1;
				}
			if (!fits(*it, r, gat))
				continue;
			if (!have || w > best_w) {
				have = true;
				best_w = w;
				best_r = r;
				best_s = *it;
			}
			break;  /* the largest selection limit that fits for this r */
		}
	}
	/* the narrow programs split again by the share of their table's row
	 * sample their filter keeps: a part of mostly-kept rows can take the
	 * shape and full-phase mode (dense) that suit it */
	std::vector<size_t> sparse, dense, wide;
	for (size_t i = 0; i < n; i++) {
		if (!(have && pp[i].row_bpr <= best_r && pp[i].sel_bpr <= best_s)) {
			wide.push_back(i);
			continue;
		}
		const double sel = sample_selectivity(b->items[i].p->prog, b->items[i].t);
		(sel >= kDensePartSel ? dense : sparse).push_back(i);
	}
	set_error("%s", "");
	b->parts.clear();
	for (auto *set : {&sparse, &dense, &wide})
		if (!set->empty()) {
			b->parts.emplace_back();
			b->parts.back().items = *set;
		}
}

}  // namespace

extern "C" int virg_gpu_batch_create(virg_gpu_engine *e, virg_gpu_batch **out)
{
	VGPU_CHECK(e != nullptr && out != nullptr, "null argument");
	virg_gpu_batch *b = new virg_gpu_batch();
	b->e = e;
	*out = b;
	return 1;
}

extern "C" int virg_gpu_batch_add(virg_gpu_batch *b, const virg_gpu_program *p,
	virg_gpu_table *t, unsigned *slot)
{
	VGPU_CHECK(b != nullptr && p != nullptr && t != nullptr, "null argument");
	VGPU_CHECK(t->e == b->e, "table belongs to another engine");
	const Program &P = p->prog;
	for (unsigned i = 0; i < P.nload; i++) {
		if (P.load_src[i] == kKeySlot)
			VGPU_CHECK(t->segs_without_key == 0, "program reads the key column the table lacks");
		else
			VGPU_CHECK(P.load_src[i] < t->schema.ncols &&
				t->schema.col_type[P.load_src[i]] == (int)P.load_type[i],
				"program column %u does not match the table schema", P.load_src[i]);
	}
	if (b->built)
		batch_release(b);
	b->items.push_back({p, t, nullptr});
	if (slot)
		*slot = (unsigned)b->items.size() - 1;
	return 1;
}

extern "C" int virg_gpu_batch_set_autotune(virg_gpu_batch *b, int enable)
{
	VGPU_CHECK(b != nullptr, "null batch");
	if (b->built && (enable != 0) != b->tune)
		batch_release(b);
	b->tune = enable != 0;
	return 1;
}

static int batch_build(virg_gpu_batch *b)
{
	virg_gpu_engine *e = b->e;
	VGPU_CHECK(!b->items.empty(), "empty batch");
	for (auto &it : b->items) {
		if (!table_sync_desc(it.t))
			return 0;
		if (!result_alloc(e, it.p->prog, it.t->rows, false, 0, &it.r))
			return 0;
	}
	const size_t nq = b->items.size();
	make_parts(b);
	const size_t np = b->parts.size();
	CUDA_OK(cudaMalloc((void **)&b->d_ctrl, 2 * np * sizeof(unsigned)), "batch control alloc");
	CUDA_OK(cudaMalloc((void **)&b->d_totals, nq * sizeof(unsigned long long)), "batch totals alloc");
	CUDA_OK(cudaHostAlloc((void **)&b->h_totals, nq * sizeof(unsigned long long), cudaHostAllocDefault),
		"batch pinned totals");
	CUDA_OK(cudaHostAlloc((void **)&b->h_ctrl, 2 * np * sizeof(unsigned), cudaHostAllocDefault),
		"batch pinned control");
	CUDA_OK(cudaStreamSynchronize(e->stream), "batch result alloc");
	for (size_t p = 0; p < np; p++)
		if (!build_with(b, p, nullptr))
			return 0;
	if (b->tune)
		for (size_t p = 0; p < np; p++)
			if (!autotune_part(b, p))
				return 0;
	for (size_t i = 0; i < nq; i++)
		b->items[i].r->d_total = b->d_totals + i;
	if (!b->done)
		CUDA_OK(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch event");
	b->built = true;
	return 1;
}

extern "C" int virg_gpu_batch_run(virg_gpu_batch *b, int use_graph)
{
	VGPU_CHECK(b != nullptr, "null batch");
	virg_gpu_engine *e = b->e;
	std::lock_guard<std::mutex> lk(e->mu);
	CUDA_OK(cudaSetDevice(e->device), "set device");
	if (!b->built && !batch_build(b))
		return 0;
	cudaStream_t s = e->stream;
	if (use_graph) {
		if (!b->gexec) {
			/* one direct run first: sets kernel attributes outside capture */
			if (!issue(b))
				return 0;
			CUDA_OK(cudaStreamSynchronize(s), "batch warm run");
			cudaGraph_t g;
			CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
			int ok = issue(b);
			cudaError_t ce = cudaStreamEndCapture(s, &g);
			VGPU_CHECK(ok && ce == cudaSuccess, "graph capture failed: %s", cudaGetErrorString(ce));
			ce = cudaGraphInstantiate(&b->gexec, g, 0);
			cudaGraphDestroy(g);
			VGPU_CHECK(ce == cudaSuccess, "graph instantiate failed: %s", cudaGetErrorString(ce));
		}
		CUDA_OK(cudaGraphLaunch(b->gexec, s), "graph launch");
	} else if (!issue(b)) {
		return 0;
	}
	CUDA_OK(cudaEventRecord(b->done, s), "batch event record");
	for (const auto &pt : b->parts)
		e->launches += pt.plan.work ? 1 : 0;
	const Plan &mp = b->parts[main_part(b)].plan;
	e->last_shape = mp.geom.shape;
	e->last_grid = mp.grid;
	e->last_smem = mp.geom.smem;
	b->ran = true;
	return 1;
}

extern "C" int virg_gpu_batch_wait(virg_gpu_batch *b)
{
	VGPU_CHECK(b != nullptr && b->ran, "batch has not run");
	CUDA_OK(cudaEventSynchronize(b->done), "batch wait");
	const unsigned err = batch_error(b);
	VGPU_CHECK(err == 0, "batch failed on the device: %s", device_error_text(err));
	for (size_t i = 0; i < b->items.size(); i++) {
		virg_gpu_result *r = b->items[i].r;
		r->rows = b->h_totals[i];
		r->have_rows = true;
	}
	return 1;
}

extern "C" int virg_gpu_batch_rows(virg_gpu_batch *b, unsigned slot, uint64_t *rows)
{
	VGPU_CHECK(b != nullptr && rows != nullptr && slot < b->items.size(), "bad argument");
	VGPU_CHECK(b->ran, "batch has not run");
	if (!b->items[slot].r->have_rows && !virg_gpu_batch_wait(b))
		return 0;
	*rows = b->items[slot].r->rows;
	return 1;
}

extern "C" const void *virg_gpu_batch_column(const virg_gpu_batch *b, unsigned slot, unsigned c)
{
	if (!b || slot >= b->items.size() || !b->items[slot].r)
		return nullptr;
	return virg_gpu_result_column(b->items[slot].r, c);
}

extern "C" int virg_gpu_batch_download(virg_gpu_batch *b, unsigned slot, void *const *host_cols,
	uint64_t first, uint64_t count)
{
	uint64_t rows;
	if (!virg_gpu_batch_rows(b, slot, &rows))
		return 0;
	return virg_gpu_result_download(b->items[slot].r, host_cols, first, count);
}

extern "C" int virg_gpu_batch_shape(const virg_gpu_batch *b, unsigned *shape4, uint64_t *work)
{
	VGPU_CHECK(b != nullptr && b->built, "batch not built");
	const Plan &mp = b->parts[main_part(b)].plan;
	if (shape4) {
		shape4[0] = mp.geom.shape.threads;
		shape4[1] = mp.geom.shape.stage_kb;
		shape4[2] = mp.geom.shape.stages;
		shape4[3] = mp.grid;
	}
	if (work) {
		*work = 0;
		for (const auto &pt : b->parts)
			*work += pt.plan.work;
	}
	return 1;
}

extern "C" void virg_gpu_batch_destroy(virg_gpu_batch *b)
{
	if (!b)
		return;
	cudaSetDevice(b->e->device);
	batch_release(b);
	if (b->done)
		cudaEventDestroy(b->done);
	delete b;
}
