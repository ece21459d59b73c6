/*
 * Drop-in replacement of the reference's GPU VM entry points
 * (src/virginian.h:620-622, src/vm/vm_gpu.cu:27-30 and :107-578).
 *
 * virg_vm_execute (src/vm/execute.c:77-90) calls virg_vm_gpu at OP_Parallel
 * with tab[0] = the table's first tablet and res[0] = a result tablet whose
 * columns were added and grown to its maximum row count.  This version:
 *
 *  1. decodes the program's data-parallel section once (program.cpp);
 *  2. for each data tablet of the chain, copies the columns the program reads
 *     from the tablet's host slot to HBM, runs the VM kernel (one launch per
 *     tablet; rows come back in original order) and reads back the row count
 *     and the valid-row count of every 64-row block;
 *  3. replays the single-core CPU VM's result-tablet roll-over rule on those
 *     block counts (src/vm/virginia.c:516-527: roll when
 *     rows + block_rows >= possible_rows - 300) and copies each run of result
 *     rows straight from HBM into its result tablet, so the result chain is
 *     the one virginia_single builds, tablet by tablet.
 *
 * Host library calls (virg_db_loadnext, virg_vm_allocresult,
 * virg_tablet_unlock) bind to the reference library this one is linked or
 * loaded with.  Locks follow the reference GPU VM (src/vm/vm_gpu.cu:555-564):
 * on return tab[0] and res[0] hold one lock each; superseded result tablets
 * hold none.
 */
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "vgpu_engine.h"
#include "vgpu_util.h"
#include "engine_internal.h"

extern "C" {
int virg_db_loadnext(virginian *v, virg_tablet_meta **tab) __attribute__((weak));
int virg_vm_allocresult(virginian *v, virg_vm *vm, virg_tablet_meta **meta,
	virg_tablet_meta *template_) __attribute__((weak));
int virg_tablet_unlock(virginian *v, unsigned tablet_id) __attribute__((weak));
}

namespace {

using namespace vgpu;

struct HostApi {
	int (*loadnext)(virginian *, virg_tablet_meta **);
	int (*allocresult)(virginian *, virg_vm *, virg_tablet_meta **, virg_tablet_meta *);
	int (*unlock)(virginian *, unsigned);
};

/* bind to the reference host library: direct weak references when it is
 * linked in, else the global symbol scope of the process */
bool resolve(HostApi &h)
{
	h.loadnext = &virg_db_loadnext ? virg_db_loadnext
		: (int (*)(virginian *, virg_tablet_meta **))dlsym(RTLD_DEFAULT, "virg_db_loadnext");
	h.allocresult = &virg_vm_allocresult ? virg_vm_allocresult
		: (int (*)(virginian *, virg_vm *, virg_tablet_meta **, virg_tablet_meta *))dlsym(
			RTLD_DEFAULT, "virg_vm_allocresult");
	h.unlock = &virg_tablet_unlock ? virg_tablet_unlock
		: (int (*)(virginian *, unsigned))dlsym(RTLD_DEFAULT, "virg_tablet_unlock");
	return h.loadnext && h.allocresult && h.unlock;
}

std::mutex g_mu;
virg_gpu_engine *g_engine = nullptr;

/* Residency cache of data tablets in HBM (off unless a capacity is set):
 * every column and the key of a tablet, in the engine's device layout,
 * keyed by tablet id and checked against the tablet's row count and host
 * slot, least recently used evicted first.  The reference's tables only
 * grow by appends (a changed row count is a miss); a caller that rebuilds a
 * table under the same tablet ids clears the cache (capacity 0). */
struct CachedTablet {
	uint64_t rows = 0;
	const void *slot = nullptr;
	void *mem = nullptr;
	size_t bytes = 0;
	const void *col[kMaxLoads] = {};
	uint64_t last_use = 0;
};
std::map<unsigned, CachedTablet> g_cache;
size_t g_cache_cap = 0, g_cache_bytes = 0;
uint64_t g_cache_clock = 0, g_cache_hits = 0, g_cache_misses = 0;

void cache_drop(std::map<unsigned, CachedTablet>::iterator it)
{
	cudaFree(it->second.mem);
	g_cache_bytes -= it->second.bytes;
	g_cache.erase(it);
}

/* the tablet's device copy from the cache, or a new one (all columns and the
 * key); nullptr if it cannot be cached (too big, or a copy failed) */
const CachedTablet *cache_get(const virg_tablet_meta *t, const virg_gpu_schema &schema, cudaStream_t st)
{
	auto it = g_cache.find(t->id);
	if (it != g_cache.end()) {
		if (it->second.rows == t->rows && it->second.slot == (const void *)t) {
			it->second.last_use = ++g_cache_clock;
			g_cache_hits++;
			return &it->second;
		}
		cache_drop(it);
	}
	g_cache_misses++;
	const uint32_t pr = (uint32_t)((t->rows + 63) / 64 * 64 + 16);
	size_t bytes = 0;
	for (unsigned c = 0; c < schema.ncols; c++)
		bytes += (pr * (size_t)t->fixed_stride[c] + 255) / 256 * 256;
	bytes += (pr * (size_t)t->key_stride + 255) / 256 * 256;
	if (bytes > g_cache_cap)
		return nullptr;
	while (g_cache_bytes + bytes > g_cache_cap && !g_cache.empty()) {
		auto lru = g_cache.begin();
		for (auto i = g_cache.begin(); i != g_cache.end(); ++i)
			if (i->second.last_use < lru->second.last_use)
				lru = i;
		cache_drop(lru);
	}
	CachedTablet ct;
	if (cudaMalloc(&ct.mem, bytes) != cudaSuccess) {
		cudaGetLastError();
		return nullptr;
	}
	ct.rows = t->rows;
	ct.slot = t;
	ct.bytes = bytes;
	ct.last_use = ++g_cache_clock;
	unsigned char *p = static_cast<unsigned char *>(ct.mem);
	bool ok = true;
	for (unsigned c = 0; c < schema.ncols; c++) {
		const size_t sz = t->fixed_stride[c];
		ok = ok && cudaMemcpyAsync(p, (const char *)t + t->fixed_block + t->fixed_offset[c], t->rows * sz,
			cudaMemcpyHostToDevice, st) == cudaSuccess;
		ct.col[c] = p;
		p += (pr * sz + 255) / 256 * 256;
	}
	ok = ok && cudaMemcpyAsync(p, (const char *)t + t->key_block, t->rows * (size_t)t->key_stride,
		cudaMemcpyHostToDevice, st) == cudaSuccess;
	ct.col[kKeySlot] = p;
	if (!ok) {
		cudaStreamSynchronize(st);
		cudaFree(ct.mem);
		return nullptr;
	}
	g_cache_bytes += bytes;
	return &(g_cache[t->id] = ct);
}

/* VIRG_CUDADEVICE (src/virginian.h:103) */
constexpr int kDevice = 0;

int fail(const char *msg)
{
	fprintf(stderr, "::: Virginian B200 VM error :: %s\n", msg);
	return VIRG_FAIL;
}

struct Timers {
	cudaEvent_t a, b, c, d;
	float h2d = 0, kern = 0, d2h = 0;
};

}  // namespace

extern "C" int virg_gpu_dropin_cache(uint64_t bytes)
{
	std::lock_guard<std::mutex> glk(g_mu);
	g_cache_cap = (size_t)bytes;
	while (g_cache_bytes > g_cache_cap && !g_cache.empty()) {
		auto lru = g_cache.begin();
		for (auto i = g_cache.begin(); i != g_cache.end(); ++i)
			if (i->second.last_use < lru->second.last_use)
				lru = i;
		cache_drop(lru);
	}
	return 1;
}

extern "C" int virg_gpu_dropin_cache_stats(uint64_t *hits, uint64_t *misses, uint64_t *bytes)
{
	std::lock_guard<std::mutex> glk(g_mu);
	if (hits)
		*hits = g_cache_hits;
	if (misses)
		*misses = g_cache_misses;
	if (bytes)
		*bytes = g_cache_bytes;
	return 1;
}

extern "C" const size_t *virg_gpu_getsizes(void)
{
	/* virg_testsizes order, src/virginian.h:553-569 */
	static const size_t sizes[15] = {sizeof(int), sizeof(float), sizeof(long long int),
		sizeof(double), sizeof(char), sizeof(virg_tablet_meta), sizeof(virg_tablet_info),
		sizeof(virg_var), sizeof(virg_vm), sizeof(virg_op), sizeof(virg_result_node),
		sizeof(virg_db), sizeof(virg_reader), sizeof(virg_vm_arg), sizeof(virginian)};
	return sizes;
}

extern "C" int virg_vm_gpu(virginian *v, virg_vm *vm, virg_tablet_meta **tab,
	virg_tablet_meta **res, unsigned num_tablets)
{
	HostApi host;
	if (!resolve(host))
		return fail("virg_db_loadnext/virg_vm_allocresult/virg_tablet_unlock not found; "
			"link or load the Virginian host library first");
	if (!v || !vm || !tab || !tab[0] || !res || !res[0])
		return fail("null argument");

	std::lock_guard<std::mutex> glk(g_mu);
	if (!g_engine && !virg_gpu_engine_create(kDevice, &g_engine))
		return fail(vgpu::last_error());
	virg_gpu_engine *e = g_engine;
	cudaSetDevice(e->device);

	/* the table's schema, from its first tablet */
	virg_gpu_schema schema;
	memset(&schema, 0, sizeof(schema));
	schema.key_type = tab[0]->key_type;
	schema.ncols = tab[0]->fixed_columns;
	for (unsigned c = 0; c < schema.ncols && c < VIRG_MAX_COLUMNS; c++)
		schema.col_type[c] = tab[0]->fixed_type[c];
	virg_gpu_program prog;
	if (!decode_program(vm->stmt, vm->num_ops, vm->pc, schema, prog.prog, prog.extra))
		return fail(vgpu::last_error());
	prog.schema = schema;
	const Program &P = prog.prog;
	if (P.nout > res[0]->fixed_columns)
		return fail("Result writes more registers than the result tablet has columns");

	Timers tm;
	cudaEventCreate(&tm.a);
	cudaEventCreate(&tm.b);
	cudaEventCreate(&tm.c);
	cudaEventCreate(&tm.d);
	int ok = 1;
	unsigned proced = 0;
	std::vector<uint8_t> counts;
	std::lock_guard<std::mutex> elk(e->mu);

	while (ok) {
		virg_tablet_meta *t = tab[0];
		if (t->fixed_columns != schema.ncols) {
			ok = fail("tablet column layout differs within the table");
			break;
		}
		/* this tablet's columns, as plain pointers into its host slot */
		virg_gpu_segment seg;
		memset(&seg, 0, sizeof(seg));
		seg.rows = t->rows;
		seg.key = (const char *)t + t->key_block;
		for (unsigned c = 0; c < schema.ncols; c++)
			seg.col[c] = (const char *)t + t->fixed_block + t->fixed_offset[c];

		virg_gpu_table stage;
		stage.e = e;
		stage.schema = schema;
		stage.transient = true;
		bool want[VIRG_MAX_COLUMNS] = {false};
		bool want_key = false;
		for (unsigned i = 0; i < P.nload; i++) {
			if (P.load_src[i] == kKeySlot)
				want_key = true;
			else
				want[P.load_src[i]] = true;
		}
		cudaEventRecord(tm.a, e->stream);
		virg_gpu_result *r = nullptr;
		const uint64_t nblocks = (t->rows + 63) / 64;
		/* the tablet's columns in HBM: from the residency cache when it is
		 * on, else copied for this query only */
		const CachedTablet *ct = g_cache_cap && t->rows ? cache_get(t, schema, e->stream) : nullptr;
		if (ct) {
			SegDesc d;
			memset(&d, 0, sizeof(d));
			d.rows = t->rows;
			d.block_base = 0;
			for (unsigned c = 0; c < kMaxLoads; c++)
				d.col[c] = ct->col[c];
			stage.segs.push_back(d);
			stage.seg_rows.push_back((uint32_t)t->rows);
			stage.rows = t->rows;
			stage.blocks = nblocks;
			stage.dirty = true;
			ok = table_sync_desc(&stage);
		} else {
			ok = table_add_segments(&stage, &seg, 1, want, want_key, e->stream) && table_sync_desc(&stage);
		}
		ok = ok && result_alloc(e, P, t->rows, true, nblocks, &r);
		cudaEventRecord(tm.b, e->stream);
		if (ok && t->rows) {
			QueryLaunch q;
			q.prog = &P;
			q.d_segs = stage.d_segs;
			q.nsegs = 1;
			q.seg_rows = stage.seg_rows.data();
			for (unsigned j = 0; j < P.nout; j++)
				q.out[j] = r->out[j];
			q.capacity = t->rows;
			q.d_total = r->d_total;
			q.block_counts = r->block_counts;
			ok = run_queries(e, std::vector<QueryLaunch>(1, q), nullptr);
		}
		cudaEventRecord(tm.c, e->stream);
		uint64_t total = 0;
		if (ok && t->rows) {
			counts.resize(nblocks);
			ok = virg_gpu_result_rows(r, &total) &&
				cudaMemcpyAsync(counts.data(), r->block_counts, nblocks, cudaMemcpyDeviceToHost,
					e->stream) == cudaSuccess &&
				cudaStreamSynchronize(e->stream) == cudaSuccess;
			if (!ok && vgpu::last_error()[0])
				fail(vgpu::last_error());
		}

		/* distribute the ordered rows over result tablets like the CPU VM */
		uint64_t done = 0;
		for (uint64_t b = 0; ok && b < nblocks; b++) {
			const unsigned simd_rows = (unsigned)std::min<uint64_t>(64, t->rows - b * 64);
			virg_tablet_meta *rt = res[0];
			if (rt->rows + simd_rows >= rt->possible_rows - 300) {
				/* roll over: the current tablet is complete, so release it
				 * once the copies into it have landed */
				if (cudaStreamSynchronize(e->stream) != cudaSuccess)
					ok = fail("result copy sync failed");
				virg_tablet_meta *old = rt;
				host.allocresult(v, vm, res, res[0]);
				host.unlock(v, old->id);
				rt = res[0];
			}
			/* gather this block's rows with the following blocks that stay in
			 * the same result tablet, then copy the run at once */
			uint64_t run = counts[b];
			uint64_t b2 = b + 1;
			unsigned rows_after = rt->rows + counts[b];
			while (b2 < nblocks) {
				const unsigned sr = (unsigned)std::min<uint64_t>(64, t->rows - b2 * 64);
				if (rows_after + sr >= rt->possible_rows - 300)
					break;
				run += counts[b2];
				rows_after += counts[b2];
				b2++;
			}
			if (rt->rows + run > rt->possible_rows) {
				ok = fail("result tablet overflow");
				break;
			}
			/* result tablets live in pinned host slots (src/init.c:57-58), so
			 * the copies run asynchronously; the tablet's last copy is waited
			 * for before it is released or the data tablet is done */
			for (unsigned j = 0; j < P.nout && run; j++) {
				char *dst = (char *)rt + rt->fixed_block + rt->fixed_offset[j] +
					(size_t)P.out_stride[j] * rt->rows;
				const char *src = (const char *)r->out[j] + (size_t)P.out_stride[j] * done;
				if (cudaMemcpyAsync(dst, src, run * P.out_stride[j], cudaMemcpyDeviceToHost,
						e->stream) != cudaSuccess)
					ok = fail("result copy failed");
			}
			rt->rows += (unsigned)run;
			done += run;
			b = b2 - 1;
		}
		if (cudaStreamSynchronize(e->stream) != cudaSuccess)
			ok = fail("result copy sync failed");
		if (ok && done != total)
			ok = fail("result row count mismatch");
		cudaEventRecord(tm.d, e->stream);
		cudaEventSynchronize(tm.d);
		float f;
		if (cudaEventElapsedTime(&f, tm.a, tm.b) == cudaSuccess) tm.h2d += f;
		if (cudaEventElapsedTime(&f, tm.b, tm.c) == cudaSuccess) tm.kern += f;
		if (cudaEventElapsedTime(&f, tm.c, tm.d) == cudaSuccess) tm.d2h += f;

		if (r)
			virg_gpu_result_destroy(r);
		for (void *m : stage.allocs)
			cudaFreeAsync(m, e->stream);
		if (stage.d_segs)
			cudaFreeAsync(stage.d_segs, e->stream);
		stage.allocs.clear();
		stage.d_segs = nullptr;
		if (!ok)
			break;

		proced++;
		if (t->last_tablet || (num_tablets != 0 && proced >= num_tablets))
			break;
		host.loadnext(v, tab);
	}
	cudaStreamSynchronize(e->stream);
	cudaEventDestroy(tm.a);
	cudaEventDestroy(tm.b);
	cudaEventDestroy(tm.c);
	cudaEventDestroy(tm.d);
	vm->timing1 = tm.h2d / 1000.0f;
	vm->timing2 = tm.kern / 1000.0f;
	vm->timing3 = tm.d2h / 1000.0f;
	return ok ? VIRG_SUCCESS : VIRG_FAIL;
}
