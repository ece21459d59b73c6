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
 *     and the valid-row count of every 64-row block, two tablets in flight;
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
cudaStream_t g_h2d = nullptr;  /* tablet copies, beside the engine's kernel and copy streams */

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
const CachedTablet *cache_get(const virg_tablet_meta *t, const virg_gpu_schema &schema, cudaStream_t st,
	cudaStream_t kst)
{
	/* a tablet about to be evicted may still be read by a kernel in flight */
	auto quiesce = [&]() {
		cudaStreamSynchronize(kst);
		cudaStreamSynchronize(st);
	};
	auto it = g_cache.find(t->id);
	if (it != g_cache.end()) {
		if (it->second.rows == t->rows && it->second.slot == (const void *)t) {
			it->second.last_use = ++g_cache_clock;
			g_cache_hits++;
			return &it->second;
		}
		quiesce();
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
	if (g_cache_bytes + bytes > g_cache_cap && !g_cache.empty())
		quiesce();
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

/* One data tablet in flight.  Tablet k's columns are copied in and its
 * kernel queued before tablet k-1's result rows are spread over the result
 * tablets, so the host's work on one tablet (reading back its counts,
 * placing its rows, loading the next tablet into a host slot) overlaps the
 * device's work on the next.  A pinned buffer per flight carries the
 * segment descriptor to the device and brings the row total and the
 * per-block counts back in one wait. */
struct Flight {
	virg_gpu_table stage;
	virg_gpu_result *r = nullptr;
	uint64_t rows = 0, nblocks = 0;
	bool busy = false, timed = false;
	cudaEvent_t a = nullptr, b = nullptr, c0 = nullptr, c = nullptr, counted = nullptr, d0 = nullptr,
		d1 = nullptr;
};
/* pinned buffer layout: SegDesc | u64 total | u8 counts[nblocks] */
constexpr size_t kPinTotal = (sizeof(SegDesc) + 63) / 64 * 64;
constexpr size_t kPinCounts = kPinTotal + 64;
unsigned char *g_pin[2] = {nullptr, nullptr};
size_t g_pin_cap[2] = {0, 0};

bool pin_reserve(unsigned i, size_t bytes)
{
	if (g_pin_cap[i] >= bytes)
		return true;
	if (g_pin[i])
		cudaFreeHost(g_pin[i]);
	g_pin[i] = nullptr;
	g_pin_cap[i] = 0;
	const size_t want = std::max<size_t>(bytes, 64 << 10);
	if (cudaHostAlloc((void **)&g_pin[i], want, cudaHostAllocDefault) != cudaSuccess) {
		cudaGetLastError();
		g_pin[i] = nullptr;
		return false;
	}
	g_pin_cap[i] = want;
	return true;
}

struct Times {
	float h2d = 0, kern = 0, d2h = 0;
};

/* the stage times of a flight's last tablet, once its copies are done */
void flight_times(Flight &f, Times &tm)
{
	if (!f.timed)
		return;
	cudaEventSynchronize(f.d1);
	float x;
	if (cudaEventElapsedTime(&x, f.a, f.b) == cudaSuccess)
		tm.h2d += x;
	if (cudaEventElapsedTime(&x, f.c0, f.c) == cudaSuccess)
		tm.kern += x;
	if (cudaEventElapsedTime(&x, f.d0, f.d1) == cudaSuccess)
		tm.d2h += x;
	f.timed = false;
}

/* release a flight's staged columns (queued after its kernel) */
void flight_unstage(Flight &f, cudaStream_t st)
{
	for (void *m : f.stage.allocs)
		cudaFreeAsync(m, st);
	if (f.stage.d_segs)
		cudaFreeAsync(f.stage.d_segs, st);
	f.stage.allocs.clear();
	f.stage.segs.clear();
	f.stage.seg_rows.clear();
	f.stage.d_segs = nullptr;
}

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
	if (!g_h2d && cudaStreamCreateWithFlags(&g_h2d, cudaStreamNonBlocking) != cudaSuccess) {
		g_h2d = nullptr;
		return fail("copy stream create failed");
	}

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

	std::lock_guard<std::mutex> elk(e->mu);
	Flight fl[2];
	cudaEvent_t roll = nullptr;
	bool events = cudaEventCreateWithFlags(&roll, cudaEventDisableTiming) == cudaSuccess;
	for (Flight &f : fl) {
		for (cudaEvent_t *ev : {&f.a, &f.b, &f.c0, &f.c, &f.d0, &f.d1})
			events = events && cudaEventCreate(ev) == cudaSuccess;
		events = events && cudaEventCreateWithFlags(&f.counted, cudaEventDisableTiming) == cudaSuccess;
		f.stage.e = e;
		f.stage.schema = schema;
		f.stage.transient = true;
	}
	int ok = events ? 1 : fail("event create failed");
	Times tm;
	bool want[VIRG_MAX_COLUMNS] = {false};
	bool want_key = false;
	for (unsigned i = 0; i < P.nload; i++) {
		if (P.load_src[i] == kKeySlot)
			want_key = true;
		else
			want[P.load_src[i]] = true;
	}

	/* spread a finished tablet's ordered rows over result tablets like the
	 * CPU VM: roll when rows + block_rows >= possible_rows - 300
	 * (src/vm/virginia.c:516-527), copying each run of rows that stays in
	 * one result tablet straight from HBM on the copy stream */
	auto finish = [&](Flight &f) -> int {
		f.busy = false;
		if (cudaEventSynchronize(f.counted) != cudaSuccess)
			return fail("result count read failed");
		const unsigned char *pin = g_pin[&f - fl];
		uint64_t total = 0, sum = 0;
		if (f.rows) {
			memcpy(&total, pin + kPinTotal, sizeof(total));
			for (uint64_t b = 0; b < f.nblocks; b++)
				sum += pin[kPinCounts + b];
		}
		if (sum != total || total > f.rows) {
			unsigned err = 0;
			if (read_device_error(e, &err) && err)
				return fail(device_error_text(err));
			return fail("result row count mismatch");
		}
		const unsigned char *counts = pin + kPinCounts;
		cudaStreamWaitEvent(e->copy_stream, f.counted, 0);
		cudaEventRecord(f.d0, e->copy_stream);
		int good = 1;
		uint64_t done = 0;
		for (uint64_t b = 0; good && b < f.nblocks; b++) {
			virg_tablet_meta *rt = res[0];
			const unsigned simd_rows = (unsigned)std::min<uint64_t>(64, f.rows - b * 64);
			if (rt->rows + simd_rows >= rt->possible_rows - 300) {
				/* roll over: the current tablet is complete, so release it
				 * once the copies into it have landed */
				if (cudaEventRecord(roll, e->copy_stream) != cudaSuccess ||
					cudaEventSynchronize(roll) != cudaSuccess) {
					good = fail("result copy sync failed");
					break;
				}
				virg_tablet_meta *old = rt;
				host.allocresult(v, vm, res, res[0]);
				host.unlock(v, old->id);
				rt = res[0];
			}
			/* this block's rows with the following blocks that stay in the
			 * same result tablet, copied as one run */
			uint64_t run = counts[b];
			uint64_t b2 = b + 1;
			unsigned rows_after = rt->rows + counts[b];
			while (b2 < f.nblocks) {
				const unsigned sr = (unsigned)std::min<uint64_t>(64, f.rows - b2 * 64);
				if (rows_after + sr >= rt->possible_rows - 300)
					break;
				run += counts[b2];
				rows_after += counts[b2];
				b2++;
			}
			if (rt->rows + run > rt->possible_rows) {
				good = fail("result tablet overflow");
				break;
			}
			/* result tablets live in pinned host slots (src/init.c:57-58), so
			 * the copies run asynchronously */
			for (unsigned j = 0; j < P.nout && run; j++) {
				char *dst = (char *)rt + rt->fixed_block + rt->fixed_offset[j] +
					(size_t)P.out_stride[j] * rt->rows;
				const char *src = (const char *)f.r->out[j] + (size_t)P.out_stride[j] * done;
				if (cudaMemcpyAsync(dst, src, run * P.out_stride[j], cudaMemcpyDeviceToHost,
						e->copy_stream) != cudaSuccess)
					good = fail("result copy failed");
			}
			rt->rows += (unsigned)run;
			done += run;
			b = b2 - 1;
		}
		cudaEventRecord(f.d1, e->copy_stream);
		/* the result buffers are freed on the engine stream after the copies */
		cudaStreamWaitEvent(e->stream, f.d1, 0);
		virg_gpu_result_destroy(f.r);
		f.r = nullptr;
		f.timed = true;
		return good;
	};

	unsigned proced = 0;
	for (uint64_t k = 0; ok; k++) {
		virg_tablet_meta *t = tab[0];
		if (t->fixed_columns != schema.ncols) {
			ok = fail("tablet column layout differs within the table");
			break;
		}
		Flight &f = fl[k & 1];
		flight_times(f, tm);
		f.rows = t->rows;
		f.nblocks = (t->rows + 63) / 64;
		if (!pin_reserve((unsigned)(k & 1), kPinCounts + f.nblocks)) {
			ok = fail("pinned count buffer alloc failed");
			break;
		}
		unsigned char *pin = g_pin[k & 1];
		/* the tablet's columns in HBM, on the copy-in stream (so they
		 * overlap the previous tablet's kernel): from the residency cache
		 * when it is on, else copied from its host slot for this query only */
		cudaEventRecord(f.a, g_h2d);
		const CachedTablet *ct = g_cache_cap && t->rows ? cache_get(t, schema, g_h2d, e->stream) : nullptr;
		SegDesc d;
		memset(&d, 0, sizeof(d));
		if (ct) {
			d.rows = t->rows;
			for (unsigned c = 0; c < kMaxLoads; c++)
				d.col[c] = ct->col[c];
		} else if (t->rows) {
			virg_gpu_segment seg;
			memset(&seg, 0, sizeof(seg));
			seg.rows = t->rows;
			seg.key = (const char *)t + t->key_block;
			for (unsigned c = 0; c < schema.ncols; c++)
				seg.col[c] = (const char *)t + t->fixed_block + t->fixed_offset[c];
			f.stage.rows = f.stage.blocks = 0;
			ok = table_add_segments(&f.stage, &seg, 1, want, want_key, g_h2d);
			if (ok)
				d = f.stage.segs[0];
		}
		if (ok && t->rows) {
			memcpy(pin, &d, sizeof(d));
			ok = cudaMallocAsync((void **)&f.stage.d_segs, sizeof(SegDesc), g_h2d) == cudaSuccess &&
				cudaMemcpyAsync(f.stage.d_segs, pin, sizeof(SegDesc), cudaMemcpyHostToDevice, g_h2d) ==
					cudaSuccess;
			if (!ok)
				fail("segment descriptor copy failed");
			f.stage.seg_rows.assign(1, (uint32_t)t->rows);
		}
		cudaEventRecord(f.b, g_h2d);
		cudaStreamWaitEvent(e->stream, f.b, 0);
		ok = ok && result_alloc(e, P, t->rows, true, f.nblocks, &f.r);
		cudaEventRecord(f.c0, e->stream);
		if (ok && t->rows) {
			QueryLaunch q;
			q.prog = &P;
			q.d_segs = f.stage.d_segs;
			q.nsegs = 1;
			q.seg_rows = f.stage.seg_rows.data();
			for (unsigned j = 0; j < P.nout; j++)
				q.out[j] = f.r->out[j];
			q.capacity = t->rows;
			q.d_total = f.r->d_total;
			q.block_counts = f.r->block_counts;
			ok = run_queries(e, std::vector<QueryLaunch>(1, q), nullptr);
			if (!ok)
				fail(vgpu::last_error());
		}
		cudaEventRecord(f.c, e->stream);
		if (ok && t->rows) {
			ok = cudaMemcpyAsync(pin + kPinTotal, f.r->d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost,
					e->stream) == cudaSuccess &&
				cudaMemcpyAsync(pin + kPinCounts, f.r->block_counts, f.nblocks, cudaMemcpyDeviceToHost,
					e->stream) == cudaSuccess;
			if (!ok)
				fail("result count read failed");
		}
		cudaEventRecord(f.counted, e->stream);
		flight_unstage(f, e->stream);
		f.busy = ok != 0;
		/* the previous tablet's rows go out while this one runs */
		Flight &prev = fl[(k + 1) & 1];
		if (prev.busy && !finish(prev))
			ok = 0;
		if (!ok)
			break;
		proced++;
		if (t->last_tablet || (num_tablets != 0 && proced >= num_tablets)) {
			ok = finish(f);
			break;
		}
		/* the host slot may be reused once its columns are in HBM */
		if (cudaEventSynchronize(f.b) != cudaSuccess) {
			ok = fail("tablet copy failed");
			break;
		}
		host.loadnext(v, tab);
	}
	cudaStreamSynchronize(g_h2d);
	cudaStreamSynchronize(e->copy_stream);
	cudaStreamSynchronize(e->stream);
	for (Flight &f : fl) {
		if (f.r)
			virg_gpu_result_destroy(f.r);
		f.r = nullptr;
		flight_unstage(f, e->stream);
		flight_times(f, tm);
	}
	if (ok) {
		unsigned err = 0;
		if (!read_device_error(e, &err))
			ok = fail(vgpu::last_error());
		else if (err)
			ok = fail(device_error_text(err));
	}
	cudaStreamSynchronize(e->stream);
	for (Flight &f : fl)
		for (cudaEvent_t ev : {f.a, f.b, f.c0, f.c, f.counted, f.d0, f.d1})
			if (ev)
				cudaEventDestroy(ev);
	if (roll)
		cudaEventDestroy(roll);
	vm->timing1 = tm.h2d / 1000.0f;
	vm->timing2 = tm.kern / 1000.0f;
	vm->timing3 = tm.d2h / 1000.0f;
	return ok ? VIRG_SUCCESS : VIRG_FAIL;
}
