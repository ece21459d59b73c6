/*
 * Host runtime of the B200 query VM: engines, HBM-resident tables, launch
 * planning and results.
 *
 * Device layout.  The reference keeps tablets as 8 MB self-describing blocks
 * (key column, key-pointer column, fixed columns; src/virginian.h:251-302)
 * and copies a whole tablet per kernel in its serial mode
 * (src/vm/vm_gpu.cu:166-168).  Here every resident segment (one tablet's
 * rows) keeps each column in its own 256-byte-aligned device array padded to
 * a multiple of 64 rows plus 16, so a tile of any column is one aligned bulk
 * copy and the 8-byte key-pointer column never crosses the bus.
 *
 * Launch planning.  One launch runs any number of queries: their tiles are
 * numbered query by query, CTAs claim tiles in order, and each query's tiles
 * chain their look-back through the engine's status words, which carry a
 * per-launch epoch so the array never needs clearing between launches.
 */
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vgpu_engine.h"
#include "vgpu_util.h"
#include "engine_internal.h"

namespace vgpu {

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

static int type_bytes(int t)
{
	switch (t) {
	case VT_INT: case VT_FLOAT: return 4;
	case VT_INT64: case VT_DOUBLE: return 8;
	case VT_CHAR: return 1;
	default: return 0;
	}
}

#define CUDA_OK(call, what)                                                        \
	do {                                                                           \
		cudaError_t e_ = (call);                                                   \
		if (e_ != cudaSuccess)                                                     \
			VGPU_FAIL("%s: %s", what, cudaGetErrorString(e_));                      \
	} while (0)

/* smem bytes a program needs per stage and for its register vectors.
 * Vectors indexed by tile row (written by the filter) get kSlots slots, one
 * per tile in flight between filter and stores; vectors indexed by
 * selection position (written and read only by the projection warps) get
 * one.  The vector region of a launch is [row slots | selection vectors],
 * sized for the largest of its programs, so that one query's row slot never
 * overlaps another's selection vectors. */
void program_layout(const Program &P, unsigned tile, uint32_t *load_off, uint32_t *stage_bytes,
	uint32_t *row_bytes, uint32_t *sel_bytes)
{
	/* a stage: query descriptor + tile info header, then the columns */
	uint32_t off = kStageHdr;
	for (unsigned i = 0; i < P.nload; i++) {
		if (load_off)
			load_off[i] = off;
		off += (uint32_t)align_up((size_t)tile * P.load_stride[i], 128);
	}
	*stage_bytes = off;
	uint32_t row = 0, sel = 0;
	for (unsigned i = 0; i < P.nvec; i++) {
		const uint32_t sz = (uint32_t)align_up((size_t)tile * P.vec_stride[i], 128);
		if (P.vec_compact[i])
			sel += sz;
		else
			row += sz;
	}
	*row_bytes = row;
	*sel_bytes = sel;
}

/* offsets of a program's vectors in a launch's vector region whose row slots
 * are row_slot bytes apart */
void vec_offsets(const Program &P, unsigned tile, uint32_t row_slot, uint32_t *vec_off)
{
	uint32_t r = 0, s = kSlots * row_slot;
	for (unsigned i = 0; i < P.nvec; i++) {
		const uint32_t sz = (uint32_t)align_up((size_t)tile * P.vec_stride[i], 128);
		if (P.vec_compact[i]) {
			vec_off[i] = s;
			s += sz;
		} else {
			vec_off[i] = r;
			r += sz;
		}
	}
}

/* stage bytes, row-slot bytes and vector-region bytes of a launch */
void launch_layout(const std::vector<const Program *> &progs, unsigned tile, uint32_t *stage_bytes,
	uint32_t *row_slot, uint32_t *vec_bytes)
{
	uint32_t stage = 0, row = 0, sel = 0;
	for (const Program *P : progs) {
		uint32_t sb, rb, vb;
		program_layout(*P, tile, nullptr, &sb, &rb, &vb);
		stage = std::max(stage, sb);
		row = std::max(row, rb);
		sel = std::max(sel, vb);
	}
	*stage_bytes = (uint32_t)align_up(std::max<uint32_t>(stage, 128), 128);
	*row_slot = row;
	*vec_bytes = kSlots * row + sel;
}

/* header | stages x stage bytes | register vectors | selection lists */
size_t smem_for(const Shape &s, uint32_t stage_bytes, uint32_t vec_bytes)
{
	/* a selection list (a tile row per selected row) per slot: a tile's list
	 * is built while earlier tiles' are projected */
	return kSmemHeader + (size_t)s.stages * stage_bytes + (size_t)vec_bytes +
		kSlots * align_up((size_t)s.tile() * sizeof(uint16_t), 128);
}

int choose_shape(virg_gpu_engine *e, const std::vector<const Program *> &progs, Shape *out,
	size_t *smem_out, uint32_t *stage_out, uint32_t *vec_out)
{
	/* first choice: one CTA per SM with 2048-row tiles and three stages (a
	 * tile's fixed costs - claim, look-back, barriers - spread over many
	 * rows, and loads in flight while two tiles are processed); then
	 * smaller tiles for programs whose staging does not fit */
	static const unsigned cand[][2] = {{512, 4}, {256, 8}, {256, 4}, {128, 8}};
	const size_t limit = (size_t)e->smem_optin;
	for (int pass = 1; pass < 2; pass++)
	for (auto &c : cand) {
		Shape s;
		s.threads = e->pref.threads ? e->pref.threads : c[0];
		s.rows_per_thread = e->pref.rows_per_thread ? e->pref.rows_per_thread : c[1];
		if (!shape_supported(s))
			VGPU_FAIL("unsupported launch shape %u threads x %u rows", s.threads, s.rows_per_thread);
		uint32_t stage, row_slot, vec;
		launch_layout(progs, s.tile(), &stage, &row_slot, &vec);
		/* a requested stage count is kept, at one CTA per SM if need be */
		const unsigned st_list[] = {e->pref.stages ? e->pref.stages : 3u, e->pref.stages ? 0u : 2u};
		for (unsigned st : st_list) {
			if (st == 0)
				continue;
			s.stages = std::min(st, kMaxStages);
			size_t smem = smem_for(s, stage, vec);
			/* 1 KB of the SM's shared memory is reserved per resident CTA */
			if (smem <= (pass == 0 ? limit / 2 - 1024 : limit)) {
				s.ctas_per_sm = e->pref.ctas_per_sm;
				*out = s;
				*smem_out = smem;
				*stage_out = stage;
				*vec_out = vec;
				return 1;
			}
		}
		if (e->pref.threads || e->pref.rows_per_thread)
			break;
	}
	VGPU_FAIL("program needs more shared memory than the device offers");
}

static int ensure_status(virg_gpu_engine *e, size_t n)
{
	if (n <= e->status_cap)
		return 1;
	if (e->status)
		cudaFreeAsync(e->status, e->stream);
	size_t cap = std::max<size_t>(n, 1 << 16);
	CUDA_OK(cudaMallocAsync((void **)&e->status, cap * sizeof(uint64_t), e->stream), "status alloc");
	CUDA_OK(cudaMemsetAsync(e->status, 0, cap * sizeof(uint64_t), e->stream), "status clear");
	e->status_cap = cap;
	return 1;
}

static int ensure_blob(virg_gpu_engine *e, size_t n)
{
	if (n <= e->blob_cap)
		return 1;
	if (e->blob)
		cudaFreeAsync(e->blob, e->stream);
	size_t cap = std::max<size_t>(align_up(n, 4096), 1 << 16);
	CUDA_OK(cudaMallocAsync(&e->blob, cap, e->stream), "descriptor alloc");
	e->blob_cap = cap;
	return 1;
}

/* the head word of a uop's record (one-hot kind, type and operator) */
static uint32_t op_head(const UOp &u)
{
	uint32_t kind = 0;
	switch (u.kind) {
	case UK_CMP: kind = OK_CMP; break;
	case UK_MATH: kind = OK_MATH; break;
	case UK_NOT: kind = OK_NOT; break;
	case UK_INVALID: kind = OK_INVALID; break;
	case UK_SETCONST: kind = OK_SETCONST; break;
	case UK_COPYCOL: kind = OK_COPY; break;
	default: break;
	}
	const bool has_op = u.kind == UK_CMP || u.kind == UK_MATH;
	return kind | (1u << (OT_SHIFT + u.type)) | (has_op ? 1u << (OO_SHIFT + u.sub) : 0u) |
		((uint32_t)(u.tslot & 7u) << OPH_SLOT_SHIFT) | (u.vjump ? OPH_VJUMP : 0u) |
		((u.flags & UF_SINGLE_DEF) ? OPH_SINGLE_DEF : 0u) | ((uint32_t)u.join << OPH_JOIN_SHIFT);
}

/* operand descriptors of a query descriptor whose program, load_off and
 * vec_off are set, for register vectors starting at vec_area */
void fill_operands(QDesc &d, uint32_t vec_area)
{
	const Program &P = d.prog;
	/* the kernel's view of the program, in the staged prefix */
	for (unsigned i = 0; i < kMaxRegs; i++) {
		d.consts[i] = P.consts[i];
		d.out_stride[i] = P.out_stride[i];
	}
	d.nfilter = P.nfilter;
	d.nuops = P.nuops;
	d.nout = P.nout;
	auto od = [&](uint8_t cls, uint8_t idx) -> uint32_t {
		if (cls == OC_COL)
			return OD_STAGE | (uint32_t)(kSmemHeader + d.load_off[idx]);
		if (cls == OC_VEC)
			return (P.vec_compact[idx] ? OD_SELVEC : OD_ROWVEC) | (vec_area + d.vec_off[idx]);
		/* scalars are read from the stage's copy of the descriptor */
		return OD_SCALAR |
			(uint32_t)(kSmemHeader + offsetof(QDesc, consts) + idx * 8u);
	};
	for (uint32_t k = 0; k < P.nuops; k++) {
		const UOp &u = P.uops[k];
		OpRec &r = d.ops[k];
		r.head = op_head(u);
		r.a = od(u.a_cls, u.a_idx);
		r.b = od(u.b_cls, u.b_idx);
		r.d = od(OC_VEC, u.dst);
	}
	for (uint32_t j = 0; j < P.nout; j++)
		d.od_out[j] = od(P.out_cls[j], P.out_idx[j]);
}

size_t plan_blob_bytes(const std::vector<QueryLaunch> &qs, size_t *off_prefix, size_t *off_tiles)
{
	const size_t nq = qs.size();
	*off_prefix = align_up(nq * sizeof(QDesc), 16);
	*off_tiles = align_up(*off_prefix + (nq + 1) * sizeof(uint64_t), 16);
	size_t words = 0;
	for (const QueryLaunch &q : qs)
		words += q.nsegs + 1;
	return *off_tiles + words * sizeof(uint32_t);
}

/* descriptor blob: QDesc[nq] | q_work_prefix[nq+1] | seg_tile_prefix...,
 * built in host memory with pointers into the device copy at `db` */
int plan_build(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, const Shape *forced,
	unsigned char *db, Plan &plan)
{
	VGPU_CHECK(!qs.empty(), "no queries");
	std::vector<const Program *> progs;
	for (const QueryLaunch &q : qs)
		progs.push_back(q.prog);
	if (forced) {
		plan.shape = *forced;
		uint32_t forced_slot;
		launch_layout(progs, forced->tile(), &plan.stage_bytes, &forced_slot, &plan.vec_bytes);
		plan.smem = smem_for(plan.shape, plan.stage_bytes, plan.vec_bytes);
		VGPU_CHECK(plan.smem <= (size_t)e->smem_optin, "shape does not fit shared memory");
	} else if (!choose_shape(e, progs, &plan.shape, &plan.smem, &plan.stage_bytes, &plan.vec_bytes)) {
		return 0;
	}
	const unsigned tile = plan.shape.tile();
	const size_t nq = qs.size();
	uint32_t stage_all, row_slot, vec_all;
	launch_layout(progs, tile, &stage_all, &row_slot, &vec_all);
	size_t off_prefix, off_tiles;
	const size_t blob_bytes = plan_blob_bytes(qs, &off_prefix, &off_tiles);
	plan.blob.assign(blob_bytes, 0);
	plan.off_prefix = off_prefix;
	unsigned char *hb = plan.blob.data();
	QDesc *hq = reinterpret_cast<QDesc *>(hb);
	uint64_t *hprefix = reinterpret_cast<uint64_t *>(hb + off_prefix);
	uint32_t *htiles = reinterpret_cast<uint32_t *>(hb + off_tiles);
	uint64_t work = 0;
	size_t tw = 0;
	for (size_t i = 0; i < nq; i++) {
		const QueryLaunch &q = qs[i];
		QDesc &d = hq[i];
		d.prog = *q.prog;
		uint32_t sb, rb, vb;
		program_layout(*q.prog, tile, d.load_off, &sb, &rb, &vb);
		vec_offsets(*q.prog, tile, row_slot, d.vec_off);
		d.vec_slot = row_slot;
		d.stage_bytes = sb;
		d.segs = q.d_segs;
		d.nsegs = q.nsegs;
		d.seg_tile_prefix = reinterpret_cast<const uint32_t *>(db + off_tiles + tw * sizeof(uint32_t));
		uint32_t *pre = htiles + tw;
		uint64_t t = 0;
		for (uint32_t s = 0; s < q.nsegs; s++) {
			pre[s] = (uint32_t)t;
			t += (q.seg_rows[s] + tile - 1) / tile;
		}
		pre[q.nsegs] = (uint32_t)t;
		tw += q.nsegs + 1;
		d.work_first = work;
		d.ntiles = t;
		hprefix[i] = work;
		work += t;
		for (unsigned j = 0; j < q.prog->nout; j++)
			d.out_ptr[j] = q.out[j];
		d.capacity = q.capacity;
		d.total_out = q.d_total;
		d.block_counts = q.block_counts;
		d.base_in = q.base_in;
		fill_operands(d, (uint32_t)(kSmemHeader + (size_t)plan.shape.stages * plan.stage_bytes));
	}
	hprefix[nq] = work;
	VGPU_CHECK(work < 0xFFFFFFF0ull, "too many tiles in one launch (%llu)", (unsigned long long)work);
	plan.work = work;
	plan.nq = (uint32_t)nq;

	int per_sm = (int)plan.shape.ctas_per_sm;
	if (per_sm == 0 && !occupancy(plan.shape, plan.smem, &per_sm))
		VGPU_FAIL("occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
	per_sm = std::max(per_sm, 1);
	plan.grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(work, 1), (uint64_t)per_sm * e->nsm);
	return 1;
}

KParams plan_params(const Plan &plan, const unsigned char *db, unsigned *counter, uint64_t *status,
	unsigned *error, uint32_t epoch)
{
	KParams kp;
	kp.queries = reinterpret_cast<const QDesc *>(db);
	kp.q_work_prefix = reinterpret_cast<const uint64_t *>(db + plan.off_prefix);
	kp.nq = plan.nq;
	kp.total_work = (uint32_t)plan.work;
	kp.counter = counter;
	kp.status = status;
	kp.error = error;
	kp.epoch = epoch;
	kp.nstages = plan.shape.stages;
	kp.stage_bytes = plan.stage_bytes;
	kp.stage_area = kSmemHeader;
	kp.vec_area = (uint32_t)(kSmemHeader + (size_t)plan.shape.stages * plan.stage_bytes);
	kp.vec_bytes = plan.vec_bytes;
	kp.sel_area = kp.vec_area + plan.vec_bytes;
	return kp;
}

/* the key a tuned launch shape is cached under: the largest per-row staging
 * and register-vector bytes and program length of the launch's queries, the
 * number of queries and the size class of the rows they scan */
std::string shape_key(const std::vector<QueryLaunch> &qs)
{
	unsigned ld = 0, vec = 0, nuops = 0, nout = 0;
	uint64_t rows = 0;
	for (const QueryLaunch &q : qs) {
		const Program &P = *q.prog;
		unsigned l = 0, v = 0;
		for (unsigned i = 0; i < P.nload; i++)
			l += P.load_stride[i];
		for (unsigned i = 0; i < P.nvec; i++)
			v += P.vec_stride[i];
		ld = std::max(ld, l);
		vec = std::max(vec, v);
		nuops = std::max(nuops, P.nuops);
		nout = std::max(nout, P.nout);
		for (uint32_t s = 0; s < q.nsegs; s++)
			rows += q.seg_rows[s];
	}
	unsigned size_class = 0;
	while ((1ull << size_class) < rows && size_class < 63)
		size_class++;
	char buf[96];
	snprintf(buf, sizeof(buf), "l%u-v%u-u%u-o%u-q%zu-r%u", ld, vec, nuops, nout, qs.size(), size_class);
	return buf;
}

int run_queries(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, LaunchTiming *timing)
{
	size_t off_prefix, off_tiles;
	if (!ensure_blob(e, plan_blob_bytes(qs, &off_prefix, &off_tiles)))
		return 0;
	unsigned char *db = static_cast<unsigned char *>(e->blob);
	Plan plan;
	const Shape *forced = e->force.threads ? &e->force : nullptr;
	if (!forced && !e->tuned.empty() && !e->pref.threads) {
		auto hit = e->tuned.find(shape_key(qs));
		if (hit != e->tuned.end())
			forced = &hit->second;
	}
	if (!plan_build(e, qs, forced, db, plan))
		return 0;
	e->launches_last = 0;
	if (plan.work == 0)
		return 1;
	if (!ensure_status(e, plan.work))
		return 0;
	e->epoch = (e->epoch + 1) & kEpochMask;
	if (e->epoch == 0 || e->epoch == kEpochMask) {
		/* epoch wrapped: stale words could alias the new epoch; kEpochMask is
		 * reserved for graph-captured batches */
		CUDA_OK(cudaMemsetAsync(e->status, 0, e->status_cap * sizeof(uint64_t), e->stream), "status");
		e->epoch = 1;
	}
	CUDA_OK(cudaMemcpyAsync(db, plan.blob.data(), plan.blob.size(), cudaMemcpyHostToDevice, e->stream),
		"descriptor copy");
	CUDA_OK(cudaMemsetAsync(e->ctrl, 0, sizeof(unsigned), e->stream), "counter reset");
	const KParams kp = plan_params(plan, db, e->ctrl, e->status, e->ctrl + 1, e->epoch);
	const Shape shape = plan.shape;
	const size_t smem = plan.smem;
	const unsigned grid = plan.grid;

	if (timing && timing->start)
		cudaEventRecord(timing->start, e->stream);
	const size_t nring = e->ring_start.size();
	if (nring)
		cudaEventRecord(e->ring_start[e->ring_count % nring], e->stream);
	if (!launch_vm(shape, kp, grid, smem, e->stream))
		VGPU_FAIL("kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
	if (nring)
		cudaEventRecord(e->ring_stop[e->ring_count++ % nring], e->stream);
	if (timing && timing->stop)
		cudaEventRecord(timing->stop, e->stream);
	e->launches++;
	e->launches_last = 1;
	e->last_shape = shape;
	e->last_grid = grid;
	e->last_smem = smem;
	return 1;
}

int read_device_error(virg_gpu_engine *e, unsigned *err)
{
	unsigned h = 0;
	CUDA_OK(cudaMemcpyAsync(&h, e->ctrl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream),
		"error read");
	CUDA_OK(cudaStreamSynchronize(e->stream), "stream sync");
	if (h)
		CUDA_OK(cudaMemsetAsync(e->ctrl + 1, 0, sizeof(unsigned), e->stream), "error clear");
	*err = h;
	return 1;
}

const char *device_error_text(unsigned code)
{
	switch (code) {
	case DE_LOOKBACK_TIMEOUT: return "look-back wait timed out";
	case DE_STAGE_TIMEOUT: return "column staging wait timed out";
	case DE_OUTPUT_OVERFLOW: return "result buffer overflow";
	case DE_BAD_WORK: return "bad work item";
	default: return "unknown device error";
	}
}

}  // namespace vgpu

using namespace vgpu;

/* ---- engine ------------------------------------------------------------ */

extern "C" int virg_gpu_engine_create(int device, virg_gpu_engine **out)
{
	VGPU_CHECK(out != nullptr, "null argument");
	*out = nullptr;
	int ndev = 0;
	CUDA_OK(cudaGetDeviceCount(&ndev), "no CUDA device");
	VGPU_CHECK(device >= 0 && device < ndev, "device %d not present (%d devices)", device, ndev);
	CUDA_OK(cudaSetDevice(device), "set device");
	cudaDeviceProp prop;
	CUDA_OK(cudaGetDeviceProperties(&prop, device), "device properties");
	VGPU_CHECK(prop.major == 10, "device %d is sm_%d%d; this library is built for sm_100a", device,
		prop.major, prop.minor);
	virg_gpu_engine *e = new virg_gpu_engine();
	e->device = device;
	e->nsm = prop.multiProcessorCount;
	e->smem_optin = (int)prop.sharedMemPerBlockOptin;
	if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaMalloc((void **)&e->ctrl, 64) != cudaSuccess || cudaMemset(e->ctrl, 0, 64) != cudaSuccess) {
		delete e;
		VGPU_FAIL("engine setup failed: %s", cudaGetErrorString(cudaGetLastError()));
	}
	/* keep freed stream-ordered blocks cached instead of returning them */
	cudaMemPool_t pool;
	if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
		uint64_t thr = UINT64_MAX;
		cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
	}
	*out = e;
	return 1;
}

static void ring_free(virg_gpu_engine *e)
{
	for (cudaEvent_t ev : e->ring_start)
		cudaEventDestroy(ev);
	for (cudaEvent_t ev : e->ring_stop)
		cudaEventDestroy(ev);
	e->ring_start.clear();
	e->ring_stop.clear();
	e->ring_count = 0;
}

extern "C" int virg_gpu_engine_timing(virg_gpu_engine *e, unsigned slots)
{
	VGPU_CHECK(e != nullptr, "null engine");
	std::lock_guard<std::mutex> lk(e->mu);
	CUDA_OK(cudaSetDevice(e->device), "set device");
	CUDA_OK(cudaStreamSynchronize(e->stream), "stream sync");
	ring_free(e);
	for (unsigned i = 0; i < slots; i++) {
		cudaEvent_t a, b;
		CUDA_OK(cudaEventCreate(&a), "event create");
		CUDA_OK(cudaEventCreate(&b), "event create");
		e->ring_start.push_back(a);
		e->ring_stop.push_back(b);
	}
	return 1;
}

extern "C" int virg_gpu_engine_kernel_times(virg_gpu_engine *e, float *ms, unsigned n, unsigned *got)
{
	VGPU_CHECK(e != nullptr && ms != nullptr && got != nullptr, "null argument");
	std::lock_guard<std::mutex> lk(e->mu);
	const size_t nring = e->ring_start.size();
	unsigned have = (unsigned)std::min<unsigned long long>(e->ring_count, nring);
	have = std::min(have, n);
	*got = 0;
	if (have == 0)
		return 1;
	CUDA_OK(cudaEventSynchronize(e->ring_stop[(e->ring_count - 1) % nring]), "event sync");
	for (unsigned i = 0; i < have; i++) {
		const unsigned long long k = e->ring_count - have + i;
		CUDA_OK(cudaEventElapsedTime(&ms[i], e->ring_start[k % nring], e->ring_stop[k % nring]),
			"event elapsed");
	}
	*got = have;
	return 1;
}

extern "C" void virg_gpu_engine_destroy(virg_gpu_engine *e)
{
	if (!e)
		return;
	cudaSetDevice(e->device);
	cudaStreamSynchronize(e->stream);
	ring_free(e);
	if (e->status)
		cudaFree(e->status);
	if (e->blob)
		cudaFree(e->blob);
	for (auto &kv : e->scratch)
		if (kv.second.ptr)
			cudaFree(kv.second.ptr);
	cudaFree(e->ctrl);
	cudaStreamDestroy(e->stream);
	cudaStreamDestroy(e->copy_stream);
	delete e;
}

extern "C" void *virg_gpu_engine_stream(virg_gpu_engine *e) { return e ? (void *)e->stream : nullptr; }

extern "C" int virg_gpu_query_tune(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_table *t, unsigned *shape4)
{
	VGPU_CHECK(e != nullptr && p != nullptr && t != nullptr, "null argument");
	static const unsigned cand[][2] = {{128, 4}, {128, 8}, {128, 16}, {256, 4}, {256, 8}, {256, 16}, {512, 4},
		{512, 8}};
	cudaEvent_t a, z;
	CUDA_OK(cudaEventCreate(&a), "event");
	CUDA_OK(cudaEventCreate(&z), "event");
	float best = 1e30f;
	Shape best_shape = {0, 0, 0, 0};
	std::string key;
	for (auto &c : cand)
		for (unsigned st = 2; st <= 4; st++) {
			e->force = Shape{c[0], c[1], st, 0};
			float t_best = 1e30f;
			bool ran = true;
			for (int rep = 0; rep < 3 && ran; rep++) {
				virg_gpu_result *r = nullptr;
				cudaEventRecord(a, e->stream);
				if (!virg_gpu_query(e, p, t, &r)) {
					ran = false;  /* shape does not fit this program */
					break;
				}
				cudaEventRecord(z, e->stream);
				uint64_t rows;
				ran = virg_gpu_result_rows(r, &rows);
				float ms = 0;
				cudaEventElapsedTime(&ms, a, z);
				virg_gpu_result_destroy(r);
				t_best = std::min(t_best, ms);
			}
			if (ran && t_best < best) {
				best = t_best;
				best_shape = e->force;
			}
		}
	e->force = Shape{0, 0, 0, 0};
	cudaEventDestroy(a);
	cudaEventDestroy(z);
	VGPU_CHECK(best_shape.threads != 0, "no launch shape fits this program");
	/* the key of this launch */
	QueryLaunch q;
	q.prog = &p->prog;
	q.nsegs = (uint32_t)t->seg_rows.size();
	q.seg_rows = t->seg_rows.data();
	e->tuned[shape_key(std::vector<QueryLaunch>(1, q))] = best_shape;
	if (shape4) {
		shape4[0] = best_shape.threads;
		shape4[1] = best_shape.rows_per_thread;
		shape4[2] = best_shape.stages;
		shape4[3] = 0;
	}
	set_error("%s", "");
	return 1;
}

extern "C" int virg_gpu_engine_check(virg_gpu_engine *e, unsigned *device_error)
{
	VGPU_CHECK(e != nullptr, "null engine");
	unsigned err = 0;
	if (!read_device_error(e, &err))
		return 0;
	if (device_error)
		*device_error = err;
	return 1;
}

extern "C" int virg_gpu_engine_set_shape(virg_gpu_engine *e, unsigned threads,
	unsigned rows_per_thread, unsigned stages, unsigned ctas_per_sm)
{
	VGPU_CHECK(e != nullptr, "null engine");
	if (threads || rows_per_thread) {
		Shape s;
		s.threads = threads ? threads : 256;
		s.rows_per_thread = rows_per_thread ? rows_per_thread : 4;
		VGPU_CHECK(shape_supported(s), "unsupported shape %u x %u", s.threads, s.rows_per_thread);
	}
	VGPU_CHECK(stages <= kMaxStages, "at most %u stages", kMaxStages);
	e->pref.threads = threads;
	e->pref.rows_per_thread = rows_per_thread;
	e->pref.stages = stages;
	e->pref.ctas_per_sm = ctas_per_sm;
	return 1;
}

extern "C" unsigned long long virg_gpu_engine_launches(virg_gpu_engine *e)
{
	return e ? e->launches : 0;
}

extern "C" int virg_gpu_engine_last_launch(virg_gpu_engine *e, unsigned *shape4, unsigned *grid,
	unsigned *smem)
{
	VGPU_CHECK(e != nullptr, "null engine");
	if (shape4) {
		shape4[0] = e->last_shape.threads;
		shape4[1] = e->last_shape.rows_per_thread;
		shape4[2] = e->last_shape.stages;
		shape4[3] = e->last_shape.ctas_per_sm;
	}
	if (grid)
		*grid = e->last_grid;
	if (smem)
		*smem = (unsigned)e->last_smem;
	return 1;
}

/* ---- resident tables --------------------------------------------------- */

extern "C" int virg_gpu_table_create(virg_gpu_engine *e, const virg_gpu_schema *schema,
	virg_gpu_table **out)
{
	VGPU_CHECK(e != nullptr && schema != nullptr && out != nullptr, "null argument");
	VGPU_CHECK(schema->ncols <= (unsigned)kMaxCols, "too many columns");
	for (unsigned c = 0; c < schema->ncols; c++)
		VGPU_CHECK(type_bytes(schema->col_type[c]) > 0, "column %u: unsupported type %d", c,
			schema->col_type[c]);
	virg_gpu_table *t = new virg_gpu_table();
	t->e = e;
	t->schema = *schema;
	*out = t;
	return 1;
}

namespace vgpu {

/* rows of device padding per segment column: bulk copies read whole 16-byte
 * chunks, up to 15 bytes past the last row */
uint32_t padded_rows(uint32_t rows) { return (uint32_t)align_up(rows, 64) + 16; }

int table_add_segments(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned n,
	const bool *want_col, bool want_key, cudaStream_t stream)
{
	for (unsigned i = 0; i < n; i++) {
		const virg_gpu_segment &g = segs[i];
		SegDesc d;
		memset(&d, 0, sizeof(d));
		d.rows = g.rows;
		d.block_base = t->blocks;
		size_t bytes = 0;
		const uint32_t pr = padded_rows(g.rows);
		for (unsigned c = 0; c < t->schema.ncols; c++)
			if (!want_col || want_col[c])
				bytes += align_up((size_t)pr * type_bytes(t->schema.col_type[c]), 256);
		bool key = (want_key || !want_col) && g.key != nullptr;
		if (key)
			bytes += align_up((size_t)pr * type_bytes(t->schema.key_type), 256);
		void *mem = nullptr;
		if (bytes) {
			if (t->transient)
				CUDA_OK(cudaMallocAsync(&mem, bytes, stream), "segment alloc");
			else
				CUDA_OK(cudaMalloc(&mem, bytes), "segment alloc");
			t->allocs.push_back(mem);
		}
		unsigned char *p = static_cast<unsigned char *>(mem);
		for (unsigned c = 0; c < t->schema.ncols; c++) {
			if (want_col && !want_col[c])
				continue;
			const size_t sz = type_bytes(t->schema.col_type[c]);
			VGPU_CHECK(g.rows == 0 || g.col[c] != nullptr, "segment %u: column %u missing", i, c);
			if (g.rows)
				CUDA_OK(cudaMemcpyAsync(p, g.col[c], (size_t)g.rows * sz, cudaMemcpyDefault, stream),
					"segment copy");
			d.col[c] = p;
			p += align_up((size_t)pr * sz, 256);
		}
		if (key) {
			const size_t sz = type_bytes(t->schema.key_type);
			if (g.rows)
				CUDA_OK(cudaMemcpyAsync(p, g.key, (size_t)g.rows * sz, cudaMemcpyDefault, stream),
					"segment key copy");
			d.col[kKeySlot] = p;
		} else if (g.rows) {
			t->segs_without_key++;
		}
		t->segs.push_back(d);
		t->rows += g.rows;
		t->bytes += bytes;
		t->blocks += (g.rows + 63) / 64;
	}
	t->dirty = true;
	return 1;
}

int table_sync_desc(virg_gpu_table *t)
{
	if (!t->dirty)
		return 1;
	virg_gpu_engine *e = t->e;
	if (t->d_segs)
		cudaFreeAsync(t->d_segs, e->stream);
	t->d_segs = nullptr;
	if (!t->segs.empty()) {
		CUDA_OK(cudaMallocAsync((void **)&t->d_segs, t->segs.size() * sizeof(SegDesc), e->stream),
			"segment table alloc");
		CUDA_OK(cudaMemcpyAsync(t->d_segs, t->segs.data(), t->segs.size() * sizeof(SegDesc),
			cudaMemcpyHostToDevice, e->stream), "segment table copy");
		CUDA_OK(cudaStreamSynchronize(e->stream), "segment table sync");
	}
	t->seg_rows.resize(t->segs.size());
	for (size_t i = 0; i < t->segs.size(); i++)
		t->seg_rows[i] = t->segs[i].rows;
	t->dirty = false;
	return 1;
}

}  // namespace vgpu

extern "C" int virg_gpu_table_append(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned nsegs)
{
	VGPU_CHECK(t != nullptr && (segs != nullptr || nsegs == 0), "null argument");
	CUDA_OK(cudaSetDevice(t->e->device), "set device");
	if (!table_add_segments(t, segs, nsegs, nullptr, true, t->e->stream))
		return 0;
	CUDA_OK(cudaStreamSynchronize(t->e->stream), "table copy");
	return table_sync_desc(t);
}

extern "C" uint64_t virg_gpu_table_rows(const virg_gpu_table *t) { return t ? t->rows : 0; }
extern "C" uint64_t virg_gpu_table_bytes(const virg_gpu_table *t) { return t ? t->bytes : 0; }

extern "C" void virg_gpu_table_destroy(virg_gpu_table *t)
{
	if (!t)
		return;
	cudaSetDevice(t->e->device);
	cudaStreamSynchronize(t->e->stream);
	for (void *p : t->allocs)
		cudaFree(p);
	if (t->d_segs)
		cudaFree(t->d_segs);
	delete t;
}

/* ---- results ----------------------------------------------------------- */

namespace vgpu {

int result_alloc(virg_gpu_engine *e, const Program &P, uint64_t capacity, bool block_counts,
	uint64_t nblocks, virg_gpu_result **out)
{
	virg_gpu_result *r = new virg_gpu_result();
	r->e = e;
	r->nout = P.nout;
	r->capacity = capacity;
	size_t bytes = 256;  /* total counter */
	for (unsigned j = 0; j < P.nout; j++) {
		r->stride[j] = P.out_stride[j];
		r->type[j] = P.out_type[j];
		bytes += align_up(std::max<uint64_t>(capacity, 1) * P.out_stride[j], 256);
	}
	if (block_counts)
		bytes += align_up(std::max<uint64_t>(nblocks, 1), 256);
	if (cudaMallocAsync(&r->mem, bytes, e->stream) != cudaSuccess) {
		delete r;
		VGPU_FAIL("result alloc of %zu bytes failed: %s", bytes, cudaGetErrorString(cudaGetLastError()));
	}
	unsigned char *p = static_cast<unsigned char *>(r->mem);
	r->d_total = reinterpret_cast<unsigned long long *>(p);
	p += 256;
	for (unsigned j = 0; j < P.nout; j++) {
		r->out[j] = p;
		p += align_up(std::max<uint64_t>(capacity, 1) * P.out_stride[j], 256);
	}
	r->block_counts = block_counts ? p : nullptr;
	r->nblocks = nblocks;
	*out = r;
	return 1;
}

}  // namespace vgpu

extern "C" int virg_gpu_query(virg_gpu_engine *e, const virg_gpu_program *p, const virg_gpu_table *t,
	virg_gpu_result **out)
{
	VGPU_CHECK(e != nullptr && p != nullptr && t != nullptr && out != nullptr, "null argument");
	VGPU_CHECK(t->e == e, "table belongs to another engine");
	*out = nullptr;
	CUDA_OK(cudaSetDevice(e->device), "set device");
	virg_gpu_table *tm = const_cast<virg_gpu_table *>(t);
	if (!table_sync_desc(tm))
		return 0;
	const Program &P = p->prog;
	for (unsigned i = 0; i < P.nload; i++) {
		if (P.load_src[i] == kKeySlot)
			VGPU_CHECK(t->segs_without_key == 0 && type_bytes(t->schema.key_type) == P.load_stride[i],
				"program reads the key column, which the table does not hold with that type");
		else
			VGPU_CHECK(P.load_src[i] < t->schema.ncols &&
				t->schema.col_type[P.load_src[i]] == (int)P.load_type[i],
				"program column %u does not match the table schema", P.load_src[i]);
	}
	std::lock_guard<std::mutex> lk(e->mu);
	virg_gpu_result *r;
	if (!result_alloc(e, P, t->rows, false, 0, &r))
		return 0;
	QueryLaunch q;
	q.prog = &P;
	q.d_segs = t->d_segs;
	q.nsegs = (uint32_t)t->segs.size();
	q.seg_rows = t->seg_rows.data();
	for (unsigned j = 0; j < P.nout; j++)
		q.out[j] = r->out[j];
	q.capacity = t->rows;
	q.d_total = r->d_total;
	q.block_counts = nullptr;
	std::vector<QueryLaunch> qs(1, q);
	LaunchTiming lt = {e->ev_start, e->ev_stop};
	if (!run_queries(e, qs, e->timing_enabled ? &lt : nullptr)) {
		virg_gpu_result_destroy(r);
		return 0;
	}
	r->ntiles_zero = (t->rows == 0);
	*out = r;
	return 1;
}

extern "C" int virg_gpu_result_rows(virg_gpu_result *r, uint64_t *rows)
{
	VGPU_CHECK(r != nullptr && rows != nullptr, "null argument");
	if (!r->have_rows) {
		virg_gpu_engine *e = r->e;
		unsigned long long h = 0;
		if (!r->ntiles_zero)
			CUDA_OK(cudaMemcpyAsync(&h, r->d_total, sizeof(h), cudaMemcpyDeviceToHost, e->stream),
				"result count read");
		unsigned err = 0;
		if (!read_device_error(e, &err))
			return 0;
		VGPU_CHECK(err == 0, "query failed on the device: %s", device_error_text(err));
		r->rows = h;
		r->have_rows = true;
	}
	*rows = r->rows;
	return 1;
}

extern "C" const void *virg_gpu_result_column(const virg_gpu_result *r, unsigned c)
{
	return (r && c < r->nout) ? r->out[c] : nullptr;
}

extern "C" int virg_gpu_result_download(virg_gpu_result *r, void *const *host_cols, uint64_t first,
	uint64_t count)
{
	uint64_t rows;
	if (!virg_gpu_result_rows(r, &rows))
		return 0;
	VGPU_CHECK(first + count <= rows, "rows %llu..%llu past the result (%llu rows)",
		(unsigned long long)first, (unsigned long long)(first + count), (unsigned long long)rows);
	virg_gpu_engine *e = r->e;
	for (unsigned j = 0; j < r->nout; j++)
		if (count)
			CUDA_OK(cudaMemcpyAsync(host_cols[j], static_cast<unsigned char *>(r->out[j]) + first * r->stride[j],
				count * r->stride[j], cudaMemcpyDeviceToHost, e->stream), "result download");
	CUDA_OK(cudaStreamSynchronize(e->stream), "result download sync");
	return 1;
}

extern "C" void virg_gpu_result_destroy(virg_gpu_result *r)
{
	if (!r)
		return;
	if (r->mem)
		cudaFreeAsync(r->mem, r->e->stream);
	delete r;
}

/* ---- end to end from host buffers -------------------------------------- */

extern "C" int virg_gpu_query_host(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_segment *segs, unsigned nsegs, void *const *out_cols, uint64_t capacity,
	uint64_t *out_rows)
{
	VGPU_CHECK(e != nullptr && p != nullptr && (segs != nullptr || nsegs == 0) && out_rows != nullptr,
		"null argument");
	CUDA_OK(cudaSetDevice(e->device), "set device");
	const Program &P = p->prog;
	/* stage only the columns the program reads */
	virg_gpu_table tmp;
	tmp.e = e;
	tmp.schema = p->schema;
	tmp.transient = true;
	bool want[kMaxCols] = {false};
	bool want_key = false;
	for (unsigned i = 0; i < P.nload; i++) {
		if (P.load_src[i] == kKeySlot)
			want_key = true;
		else
			want[P.load_src[i]] = true;
	}
	for (unsigned s = 0; s < nsegs; s++)
		if (want_key)
			VGPU_CHECK(segs[s].key != nullptr || segs[s].rows == 0, "segment %u has no key column", s);
	std::lock_guard<std::mutex> lk(e->mu);
	int ok = table_add_segments(&tmp, segs, nsegs, want, want_key, e->stream) && table_sync_desc(&tmp);
	virg_gpu_result *r = nullptr;
	if (ok)
		ok = result_alloc(e, P, tmp.rows, false, 0, &r);
	if (ok) {
		QueryLaunch q;
		q.prog = &P;
		q.d_segs = tmp.d_segs;
		q.nsegs = (uint32_t)tmp.segs.size();
		q.seg_rows = tmp.seg_rows.data();
		for (unsigned j = 0; j < P.nout; j++)
			q.out[j] = r->out[j];
		q.capacity = tmp.rows;
		q.d_total = r->d_total;
		q.block_counts = nullptr;
		std::vector<QueryLaunch> qs(1, q);
		ok = run_queries(e, qs, nullptr);
		r->ntiles_zero = (tmp.rows == 0);
	}
	uint64_t rows = 0;
	if (ok)
		ok = virg_gpu_result_rows(r, &rows);
	if (ok) {
		*out_rows = rows;
		uint64_t n = std::min(rows, capacity);
		for (unsigned j = 0; j < P.nout && n; j++) {
			cudaError_t ce = cudaMemcpyAsync(out_cols[j], r->out[j], n * r->stride[j],
				cudaMemcpyDeviceToHost, e->stream);
			if (ce != cudaSuccess) {
				set_error("result copy: %s", cudaGetErrorString(ce));
				ok = 0;
			}
		}
		if (ok && cudaStreamSynchronize(e->stream) != cudaSuccess) {
			set_error("result copy sync failed");
			ok = 0;
		}
		if (ok && rows > capacity) {
			set_error("result has %llu rows, the buffers hold %llu", (unsigned long long)rows,
				(unsigned long long)capacity);
			ok = 0;
		}
	}
	if (r)
		virg_gpu_result_destroy(r);
	for (void *m : tmp.allocs)
		cudaFreeAsync(m, e->stream);
	tmp.allocs.clear();
	if (tmp.d_segs)
		cudaFreeAsync(tmp.d_segs, e->stream);
	tmp.d_segs = nullptr;
	return ok;
}
