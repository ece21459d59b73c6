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

}  // namespace

struct virg_gpu_batch {
	virg_gpu_engine *e = nullptr;
	struct Item {
		const virg_gpu_program *p;
		virg_gpu_table *t;
		virg_gpu_result *r;
	};
	std::vector<Item> items;
	bool built = false;
	Plan plan;
	unsigned char *d_blob = nullptr;
	uint64_t *d_status = nullptr;
	unsigned *d_ctrl = nullptr;            /* [0] work counter, [1] error */
	unsigned long long *d_totals = nullptr;
	unsigned long long *h_totals = nullptr;  /* pinned */
	unsigned *h_err = nullptr;               /* pinned */
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
	if (b->d_blob) cudaFree(b->d_blob);
	if (b->d_status) cudaFree(b->d_status);
	if (b->d_ctrl) cudaFree(b->d_ctrl);
	if (b->d_totals) cudaFree(b->d_totals);
	if (b->h_totals) cudaFreeHost(b->h_totals);
	if (b->h_err) cudaFreeHost(b->h_err);
	b->d_blob = nullptr;
	b->d_status = nullptr;
	b->d_ctrl = nullptr;
	b->d_totals = nullptr;
	b->h_totals = nullptr;
	b->h_err = nullptr;
	b->built = false;
	b->ran = false;
}

std::vector<QueryLaunch> launches_of(virg_gpu_batch *b)
{
	std::vector<QueryLaunch> qs;
	for (size_t i = 0; i < b->items.size(); i++) {
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
	const Plan &plan = b->plan;
	CUDA_OK(cudaMemsetAsync(b->d_ctrl, 0, 2 * sizeof(unsigned), s), "batch counter reset");
	CUDA_OK(cudaMemsetAsync(b->d_totals, 0, b->items.size() * sizeof(unsigned long long), s),
		"batch totals reset");
	if (plan.work) {
		CUDA_OK(cudaMemsetAsync(b->d_status, 0, plan.work * sizeof(uint64_t), s), "batch status reset");
		const KParams kp = plan_params(plan, b->d_blob, b->d_ctrl, b->d_status, b->d_ctrl + 1,
			kBatchEpoch);
		if (!launch_vm(plan.geom.shape, kp, plan.grid, plan.geom.smem, s))
			VGPU_FAIL("batch kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
	}
	CUDA_OK(cudaMemcpyAsync(b->h_totals, b->d_totals, b->items.size() * sizeof(unsigned long long),
		cudaMemcpyDeviceToHost, s), "batch totals read");
	CUDA_OK(cudaMemcpyAsync(b->h_err, b->d_ctrl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s),
		"batch error read");
	return 1;
}

int build_with(virg_gpu_batch *b, const Shape *forced)
{
	virg_gpu_engine *e = b->e;
	std::vector<QueryLaunch> qs = launches_of(b);
	size_t off_prefix, off_chunks;
	const size_t bytes = plan_blob_bytes(qs, &off_prefix, &off_chunks);
	if (!b->d_blob)
		CUDA_OK(cudaMalloc((void **)&b->d_blob, bytes), "batch descriptor alloc");
	Plan plan;
	if (!plan_build(e, qs, forced, b->d_blob, plan))
		return 0;
	CUDA_OK(cudaMemcpy(b->d_blob, plan.blob.data(), plan.blob.size(), cudaMemcpyHostToDevice),
		"batch descriptor copy");
	if (b->d_status && b->plan.work < plan.work) {
		cudaFree(b->d_status);
		b->d_status = nullptr;
	}
	if (!b->d_status)
		CUDA_OK(cudaMalloc((void **)&b->d_status, std::max<uint64_t>(plan.work, 1) * sizeof(uint64_t)),
			"batch status alloc");
	b->plan = std::move(plan);
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
	return ok && *b->h_err == 0 ? ms : -1.0f;
}

int autotune(virg_gpu_batch *b)
{
	virg_gpu_engine *e = b->e;
	const std::string key = shape_key(launches_of(b));
	auto hit = e->tuned.find(key);
	if (hit != e->tuned.end())
		return build_with(b, &hit->second);
	float best = 1e30f;
	Shape best_shape = {0, 0, 0, 0, 0, 0};
	for (const Shape &c : tune_candidates()) {
		set_error("%s", "");
		if (!build_with(b, &c))
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
			best_shape = b->plan.geom.shape;
		}
	}
	VGPU_CHECK(best_shape.threads != 0, "no launch shape fits this batch");
	tune_remember(e, key, best_shape);
	return build_with(b, &best_shape);
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
	CUDA_OK(cudaMalloc((void **)&b->d_ctrl, 2 * sizeof(unsigned)), "batch control alloc");
	CUDA_OK(cudaMalloc((void **)&b->d_totals, nq * sizeof(unsigned long long)), "batch totals alloc");
	CUDA_OK(cudaHostAlloc((void **)&b->h_totals, nq * sizeof(unsigned long long), cudaHostAllocDefault),
		"batch pinned totals");
	CUDA_OK(cudaHostAlloc((void **)&b->h_err, sizeof(unsigned), cudaHostAllocDefault),
		"batch pinned error");
	CUDA_OK(cudaStreamSynchronize(e->stream), "batch result alloc");
	int ok = b->tune ? autotune(b) : build_with(b, nullptr);
	if (!ok)
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
	e->launches += b->plan.work ? 1 : 0;
	e->last_shape = b->plan.geom.shape;
	e->last_grid = b->plan.grid;
	e->last_smem = b->plan.geom.smem;
	b->ran = true;
	return 1;
}

extern "C" int virg_gpu_batch_wait(virg_gpu_batch *b)
{
	VGPU_CHECK(b != nullptr && b->ran, "batch has not run");
	CUDA_OK(cudaEventSynchronize(b->done), "batch wait");
	VGPU_CHECK(*b->h_err == 0, "batch failed on the device: %s", device_error_text(*b->h_err));
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
	if (shape4) {
		shape4[0] = b->plan.geom.shape.threads;
		shape4[1] = b->plan.geom.shape.stage_kb;
		shape4[2] = b->plan.geom.shape.stages;
		shape4[3] = b->plan.grid;
	}
	if (work)
		*work = b->plan.work;
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
