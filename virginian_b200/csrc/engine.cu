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
 * Launch planning.  One launch runs any number of queries: their chunks are
 * numbered query by query, CTAs claim chunks in order, and each query's
 * chunks chain their look-back through the engine's status words, which
 * carry a per-launch epoch so the array never needs clearing between
 * launches.  With shared scans on, queries over the same table sit side by
 * side and claim their chunks interleaved, so each chunk of the table is
 * read from HBM once and from L2 by the group's other queries.
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

/* ---- launch planning --------------------------------------------------- */

/* The staging plan of a program, independent of the launch geometry.  The
 * count phase stages the columns the filter uops read; the full phase the
 * columns the projection uops and result columns read.  If the projection
 * or a result column touches a register vector the filter wrote (a
 * register indexed by block row), the full phase runs the filter again and
 * stages every column the program reads. */
/* which operand fields a uop reads, and whether it writes its destination */
static bool uses_a(const UOp &u)
{
	return u.kind == UK_CMP || u.kind == UK_NOT || u.kind == UK_MATH || u.kind == UK_SETCONST ||
		u.kind == UK_COPYCOL;
}
static bool uses_b(const UOp &u) { return u.kind == UK_CMP || u.kind == UK_MATH; }
static bool writes_d(const UOp &u) { return u.kind == UK_MATH || u.kind == UK_SETCONST || u.kind == UK_COPYCOL; }

void plan_program(const Program &P, ProgPlan &pp, unsigned full_mode)
{
	memset(&pp, 0, sizeof(pp));
	bool in_count[kMaxLoads] = {false}, in_proj[kMaxLoads] = {false};
	bool refilter = false;
	const uint32_t nproj_end = P.nuops ? P.nuops - 1 : 0;
	auto col_of = [&](uint8_t cls, uint8_t idx, bool *set) {
		if (cls == OC_COL)
			set[idx] = true;
	};
	auto rowvec = [&](uint8_t cls, uint8_t idx) { return cls == OC_VEC && !P.vec_compact[idx]; };
	for (uint32_t k = 0; k < P.nfilter; k++) {
		const UOp &u = P.uops[k];
		if (uses_a(u))
			col_of(u.a_cls, u.a_idx, in_count);
		if (uses_b(u))
			col_of(u.b_cls, u.b_idx, in_count);
	}
	for (uint32_t k = P.nfilter; k < nproj_end; k++) {
		const UOp &u = P.uops[k];
		if (uses_a(u))
			col_of(u.a_cls, u.a_idx, in_proj);
		if (uses_b(u))
			col_of(u.b_cls, u.b_idx, in_proj);
		if ((uses_a(u) && rowvec(u.a_cls, u.a_idx)) || (uses_b(u) && rowvec(u.b_cls, u.b_idx)) ||
			(writes_d(u) && !P.vec_compact[u.dst]))
			refilter = true;
	}
	for (uint32_t j = 0; j < P.nout; j++) {
		col_of(P.out_cls[j], P.out_idx[j], in_proj);
		if (rowvec(P.out_cls[j], P.out_idx[j]))
			refilter = true;
	}
	pp.mode = refilter ? FM_REFILTER : FM_BITMAP;
	for (uint32_t i = 0; i < P.nload; i++) {
		if (in_count[i]) {
			pp.count_cols[pp.ncount++] = (uint8_t)i;
			pp.count_bpr += P.load_stride[i];
		}
		if (in_proj[i] || (refilter && in_count[i])) {
			pp.full_cols[pp.nfull++] = (uint8_t)i;
			pp.full_bpr += P.load_stride[i];
		}
	}
	/* full_mode 1: the full phase gathers the selected rows' values from
	 * device memory into each compute warp's area, unless they are many
	 * bytes per row; full_mode 2: it runs the projection over whole groups */
	if (pp.mode == FM_BITMAP && pp.full_bpr <= kGatherMaxBpr && full_mode == 1) {
		pp.mode = FM_GATHER;
		pp.gather_bpr = pp.full_bpr;
	}
	if (pp.mode == FM_BITMAP && full_mode == 2) {
		uint32_t dense_row = 0;
		for (uint32_t i = 0; i < P.nvec; i++)
			dense_row += P.vec_stride[i];
		if (dense_row <= kDenseMaxRowBpr)
			pp.mode = FM_DENSE;
	}
	/* selection vectors hold a projection batch's entries, row vectors a
	 * count group's rows (every vector is a row vector in FM_DENSE) */
	uint32_t sel = 0, row = 0;
	for (uint32_t i = 0; i < P.nvec; i++) {
		if (P.vec_compact[i] && pp.mode != FM_DENSE) {
			pp.vec_off[i] = sel;  /* re-laid by desc_fill for the launch's unit size */
			sel += kUnitE * P.vec_stride[i];
		} else {
			pp.vec_off[i] = row;
			row += kCountGroup * kBlockRows * P.vec_stride[i];
		}
		(P.vec_compact[i] && pp.mode != FM_DENSE ? pp.sel_bpr : pp.row_bpr) += P.vec_stride[i];
	}
}

/* geom_make for units of `ub` batches */
static int geom_make1(const Shape &s0, uint32_t sel_bpr, uint32_t row_bpr, uint32_t gather_bpr, int smem_block,
	int smem_sm, uint32_t ub, Geom *g)
{
	Shape s = s0;
	VGPU_CHECK(shape_supported(s), "unsupported launch shape: %u compute threads", s.threads);
	VGPU_CHECK(s.stage_kb >= 1 && s.stage_kb <= 192, "stage size %u KB out of range", s.stage_kb);
	g->ub = ub;
	g->wl = warp_layout(sel_bpr, row_bpr, gather_bpr, ub);
	g->stage_area = (uint32_t)align_up(kWarpArea + (size_t)s.warps() * g->wl.bytes, 128);
	const unsigned ctas = s.ctas_per_sm ? s.ctas_per_sm : 1;
	/* 1 KB of an SM's shared memory is reserved per resident CTA */
	const size_t budget = std::min<size_t>((size_t)smem_block, (size_t)smem_sm / ctas - 1024);
	if (budget <= g->stage_area)
		return 0;
	const size_t fit = (budget - g->stage_area) / s.stage_bytes();
	if (s.stages == 0)
		s.stages = (unsigned)std::min<size_t>(fit, kMaxStages);
	if (s.stages < 2 || s.stages > kMaxStages || s.stages > fit)
		return 0;
	g->shape = s;
	g->smem = g->stage_area + (size_t)s.stages * s.stage_bytes();
	return 1;
}

/* the launch geometry of a shape whose compute warps hold sel_bpr and
 * row_bpr bytes of vectors per row; stages == 0 takes as many stages as fit
 * the shared memory left per CTA */
int geom_make(const Shape &s, uint32_t sel_bpr, uint32_t row_bpr, uint32_t gather_bpr, int smem_block, int smem_sm,
	Geom *g, uint32_t ub_max)
{
	Geom one;
	if (!geom_make1(s, sel_bpr, row_bpr, gather_bpr, smem_block, smem_sm, 1, &one))
		return 0;
	*g = one;
	Geom two;
	if (ub_max >= 2 && geom_make1(s, sel_bpr, row_bpr, gather_bpr, smem_block, smem_sm, 2, &two) &&
		(two.shape.stages >= one.shape.stages || two.shape.stages >= 3))
		*g = two;
	return 1;
}

/* a phase's staged columns for tiles of `rows` rows */
/* (group rows: a staged tile's column is laid out for whole groups of
 * kCountGroup blocks, since a group's lanes read all of its rows, valid or
 * not; 0 for a gather area) */
static void load_set(LoadSet &ls, const Program &P, const uint8_t *cols, uint32_t n, uint32_t rows,
	uint32_t group_rows = kCountGroup * kBlockRows)
{
	memset(&ls, 0, sizeof(ls));
	ls.n = n;
	ls.rows = rows;
	const uint32_t laid = group_rows ? (rows + group_rows - 1) / group_rows * group_rows : rows;
	uint32_t off = 0;
	for (uint32_t i = 0; i < n; i++) {
		const uint32_t slot = cols[i];
		ls.src[i] = P.load_src[slot];
		ls.stride[i] = P.load_stride[slot];
		ls.off[i] = off;
		ls.bytes_per_row += P.load_stride[slot];
		off += (uint32_t)align_up((size_t)laid * P.load_stride[slot], 128);
	}
}

/* tile rows of a phase staging bpr bytes per row in a stage of `stage`
 * bytes (whole blocks, at most `cap` rows); 0 if not one block fits */
static uint32_t tile_rows(uint32_t bpr, uint32_t stage, uint32_t cap)
{
	if (bpr == 0)
		return cap;
	/* whole groups of kCountGroup blocks (a tile's columns are laid out for
	 * whole groups); 0 if not one group fits */
	constexpr uint32_t kGroupRows = kCountGroup * kBlockRows;
	return std::min<uint32_t>(cap, stage / bpr / kGroupRows * kGroupRows);
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

int desc_fill(QDesc &d, const Program &P, const ProgPlan &pp, const Geom &g, uint32_t chunk_cap)
{
	const uint32_t stage = g.shape.stage_bytes();
	chunk_cap = std::max<uint32_t>(kBlockRows, std::min<uint32_t>(chunk_cap, kMaxChunkRows) / kBlockRows * kBlockRows);
	const uint32_t tf = tile_rows(pp.full_bpr, stage, chunk_cap);
	VGPU_CHECK(tf >= kBlockRows, "a %u KB stage cannot hold %u rows of the %u bytes per row the results read",
		g.shape.stage_kb, kCountGroup * kBlockRows, pp.full_bpr);
	/* the chunk: a multiple of the full tile, at most the cap, whose count
	 * and full tiles fill their data buffers best (a short last tile still
	 * takes a whole buffer, and every buffer use costs the same issue and
	 * claim work): the most rows per buffer use, ties to the larger chunk */
	uint32_t chunk = tf;
	uint64_t best_num = 0, best_den = 1;
	for (uint32_t c = tf; c <= std::max(tf, chunk_cap); c += tf) {
		const uint32_t t = tile_rows(pp.count_bpr, stage, c);
		if (t < kBlockRows)
			break;
		const uint64_t uses = (c + t - 1) / t + (pp.mode == FM_GATHER ? 0u : c / tf);
		if ((uint64_t)c * best_den >= best_num * uses) {
			best_num = c;
			best_den = uses;
			chunk = c;
		}
	}
	const uint32_t tc = tile_rows(pp.count_bpr, stage, chunk);
	VGPU_CHECK(tc >= kBlockRows, "a %u KB stage cannot hold %u rows of the %u bytes per row the filter reads",
		g.shape.stage_kb, kCountGroup * kBlockRows, pp.count_bpr);
	d.prog = P;
	load_set(d.count_set, P, pp.count_cols, pp.ncount, tc);
	if (pp.mode == FM_GATHER) {
		/* one full entry per chunk; the staged columns of a batch are its
		 * 32 kBatchE gathered entries, in the warp's gather area.  The
		 * chunk is a whole number of count tiles, so every count buffer
		 * use is full */
		const uint32_t tcap = tile_rows(pp.count_bpr, stage, chunk_cap);
		const uint32_t gchunk = tcap >= kBlockRows ? std::max(tcap, chunk_cap / tcap * tcap) : chunk_cap;
		load_set(d.full_set, P, pp.full_cols, pp.nfull, kBatchRows * g.ub, 0);
		d.full_set.rows = gchunk;
		d.chunk_rows = gchunk;
		load_set(d.count_set, P, pp.count_cols, pp.ncount, tile_rows(pp.count_bpr, stage, gchunk));
		VGPU_CHECK(d.count_set.rows >= kBlockRows, "a %u KB stage cannot hold %u rows of the %u bytes per row the filter reads",
			g.shape.stage_kb, kCountGroup * kBlockRows, pp.count_bpr);
		d.gather_n = d.full_set.n;
		for (uint32_t i = 0; i < d.full_set.n; i++) {
			d.gather_stride[i] = d.full_set.stride[i];
			d.gather_off[i] = d.full_set.off[i];
		}
	} else {
		load_set(d.full_set, P, pp.full_cols, pp.nfull, tf);
		d.chunk_rows = chunk;
	}
	const LoadSet &rset = d.full_set;
	d.full_mode = pp.mode;
	for (unsigned i = 0; i < kMaxRegs; i++) {
		d.consts[i] = P.consts[i];
		d.out_stride[i] = P.out_stride[i];
	}
	d.nfilter = P.nfilter;
	d.nuops = P.nuops;
	d.nout = P.nout;
	/* selection-indexed vectors over the launch's unit size */
	uint32_t sel_off[kMaxRegs] = {0};
	const bool dense = pp.mode == FM_DENSE;
	for (uint32_t i = 0, at = 0; i < P.nvec; i++)
		if (P.vec_compact[i] && !dense) {
			sel_off[i] = at;
			at += kBatchRows * g.ub * P.vec_stride[i];
		}
	/* operand descriptors over one phase's layout (bad: a column the phase
	 * does not stage, never read in that phase) */
	auto od = [&](uint8_t cls, uint8_t idx, const LoadSet &ls, const uint8_t *cols, uint32_t n, bool *bad) -> uint32_t {
		if (cls == OC_COL) {
			for (uint32_t i = 0; i < n; i++)
				if (cols[i] == idx)
					return OD_STAGE | ls.off[i];
			*bad = true;
			return OD_STAGE;
		}
		if (cls == OC_VEC)
			return P.vec_compact[idx] && !dense ? (OD_SELVEC | sel_off[idx]) : (OD_ROWVEC | pp.vec_off[idx]);
		return OD_SCALAR | (uint32_t)(offsetof(QDesc, consts) + idx * 8u);
	};
	/* a record over one phase's layout; operand fields the uop does not use
	 * stay 0 */
	auto rec = [&](const UOp &u, const LoadSet &ls, const uint8_t *cols, uint32_t n, bool *bad) {
		OpRec r;
		r.head = op_head(u);
		r.a = uses_a(u) ? od(u.a_cls, u.a_idx, ls, cols, n, bad) : 0u;
		r.b = uses_b(u) ? od(u.b_cls, u.b_idx, ls, cols, n, bad) : 0u;
		r.d = writes_d(u) ? od(OC_VEC, u.dst, ls, cols, n, bad) : 0u;
		return r;
	};
	bool bad = false;
	for (uint32_t k = 0; k < P.nfilter; k++)
		d.ops_count[k] = rec(P.uops[k], d.count_set, pp.count_cols, pp.ncount, &bad);
	VGPU_CHECK(!bad, "internal: a filter operand is not staged in the count phase");
	for (uint32_t k = 0; k < P.nuops; k++) {
		/* the full phase runs filter uops only when it runs the filter again */
		if (k < P.nfilter && pp.mode != FM_REFILTER) {
			d.ops_full[k] = OpRec{op_head(P.uops[k]), 0u, 0u, 0u};
			continue;
		}
		d.ops_full[k] = rec(P.uops[k], rset, pp.full_cols, pp.nfull, &bad);
	}
	for (uint32_t j = 0; j < P.nout; j++)
		d.od_out[j] = od(P.out_cls[j], P.out_idx[j], rset, pp.full_cols, pp.nfull, &bad);
	VGPU_CHECK(!bad, "internal: a result operand is not staged in the full phase");
	return 1;
}

uint64_t chunk_prefix(const uint32_t *seg_rows, uint32_t nsegs, uint32_t chunk_rows, uint32_t *pre)
{
	uint64_t t = 0;
	for (uint32_t s = 0; s < nsegs; s++) {
		if (pre)
			pre[s] = (uint32_t)t;
		t += (seg_rows[s] + chunk_rows - 1) / chunk_rows;
	}
	if (pre)
		pre[nsegs] = (uint32_t)t;
	return t;
}

KParams geom_params(const Geom &g)
{
	KParams kp;
	kp.queries = nullptr;
	kp.q_work_prefix = nullptr;
	kp.nq = 0;
	kp.total_work = 0;
	kp.counter = nullptr;
	kp.status = nullptr;
	kp.error = nullptr;
	kp.epoch = 1;
	kp.nstages = g.shape.stages;
	kp.stage_bytes = g.shape.stage_bytes();
	kp.stage_area = g.stage_area;
	kp.warp_bytes = g.wl.bytes;
	kp.sel_off = g.wl.sel_off;
	kp.gat_off = g.wl.gat_off;
	kp.row_off = g.wl.row_off;
	kp.unit_batches = g.ub;
	return kp;
}

/* the widest vector areas and staging of a launch's programs */
static void launch_needs(const std::vector<QueryLaunch> &qs, unsigned full_mode, uint32_t *sel, uint32_t *row,
	uint32_t *gat, uint32_t *bpr)
{
	*sel = *row = *gat = *bpr = 0;
	for (const QueryLaunch &q : qs) {
		ProgPlan pp;
		plan_program(*q.prog, pp, full_mode);
		*sel = std::max(*sel, pp.sel_bpr);
		*row = std::max(*row, pp.row_bpr);
		*gat = std::max(*gat, pp.gather_bpr);
		*bpr = std::max({*bpr, pp.count_bpr, pp.mode == FM_GATHER ? 0u : pp.full_bpr});
	}
}

int choose_shape(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, Geom *g)
{
	uint32_t sel, row, gat, bpr;
	launch_needs(qs, e->pref.full_mode, &sel, &row, &gat, &bpr);
	Shape s;
	s.full_mode = e->pref.full_mode;
	s.threads = e->pref.threads ? e->pref.threads : 256;
	s.stage_kb = e->pref.stage_kb ? e->pref.stage_kb : 32;
	s.stages = e->pref.stages;
	s.ctas_per_sm = e->pref.ctas_per_sm;
	s.chunk_rows = e->pref.chunk_rows;
	/* a stage holds at least one group of kCountGroup blocks of the widest
	 * phase; without a preference, the largest data buffers of which three
	 * fit beside the warps' areas (fewer, fuller buffer uses per row: each
	 * use costs the same issue, claim and release work), else the smallest
	 * size that fits at all */
	const unsigned min_kb = (kCountGroup * kBlockRows * bpr + 1023) / 1024;
	if (!e->pref.stage_kb) {
		s.stage_kb = std::max<unsigned>(32, min_kb);
		for (unsigned kb : {48u, 40u, 32u, 24u}) {
			Shape t = s;
			t.stage_kb = std::max(kb, min_kb);
			Geom gt;
			if (geom_make(t, sel, row, gat, e->smem_optin, e->smem_sm, &gt) && gt.shape.stages >= 3) {
				*g = gt;
				return 1;
			}
		}
	}
	if (geom_make(s, sel, row, gat, e->smem_optin, e->smem_sm, g))
		return 1;
	/* a dense full phase whose row vectors leave no room for two stages
	 * falls back to the in-place one */
	if (s.full_mode == 2) {
		s.full_mode = 0;
		launch_needs(qs, 0, &sel, &row, &gat, &bpr);
		if (geom_make(s, sel, row, gat, e->smem_optin, e->smem_sm, g))
			return 1;
	}
	VGPU_FAIL("launch shape (%u threads, %u KB x %u stages, %u CTAs per SM) does not fit shared memory",
		s.threads, s.stage_kb, s.stages, s.ctas_per_sm);
}

size_t plan_blob_bytes(const std::vector<QueryLaunch> &qs, size_t *off_prefix, size_t *off_chunks)
{
	const size_t nq = qs.size();
	*off_prefix = align_up(nq * sizeof(QDesc), 16);
	*off_chunks = align_up(*off_prefix + (nq + 1) * sizeof(uint64_t), 16);
	size_t words = 0;
	for (const QueryLaunch &q : qs)
		words += q.nsegs + 1;
	return *off_chunks + words * sizeof(uint32_t);
}

/* the automatic chunk bound: kMaxChunkRows, smaller (down to 1024) when
 * the launch has too few rows to give every CTA a few chunks (each query's
 * chunk is then the multiple of its tiles below the bound that fills its
 * buffers best) */
static uint32_t auto_chunk(uint64_t rows, unsigned ctas)
{
	const uint64_t want = rows / (4ull * std::max(ctas, 1u));
	return (uint32_t)std::max<uint64_t>(1024, std::min<uint64_t>(kMaxChunkRows, want / kBlockRows * kBlockRows));
}

/* descriptor blob: QDesc[nq] | q_work_prefix[nq+1] | seg_chunk_prefix...,
 * built in host memory with pointers into the device copy at `db` */
int plan_build(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, const Shape *forced,
	unsigned char *db, Plan &plan)
{
	VGPU_CHECK(!qs.empty(), "no queries");
	if (forced) {
		uint32_t sel, row, gat, bpr;
		launch_needs(qs, forced->full_mode, &sel, &row, &gat, &bpr);
		VGPU_CHECK(geom_make(*forced, sel, row, gat, e->smem_optin, e->smem_sm, &plan.geom),
			"shape does not fit shared memory");
	} else if (!choose_shape(e, qs, &plan.geom)) {
		return 0;
	}
	const Geom &g = plan.geom;
	/* resident CTAs per SM: the shape's request, capped by what its shared
	 * memory and registers allow */
	int per_sm = 0;
	if (!occupancy(g.shape, g.smem, &per_sm))
		VGPU_FAIL("occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
	if (g.shape.ctas_per_sm)
		per_sm = std::min(per_sm, (int)g.shape.ctas_per_sm);
	per_sm = std::max(per_sm, 1);
	const unsigned slots = (unsigned)per_sm * (unsigned)e->nsm;
	uint64_t all_rows = 0;
	for (const QueryLaunch &q : qs)
		for (uint32_t s = 0; s < q.nsegs; s++)
			all_rows += q.seg_rows[s];
	const uint32_t cap = g.shape.chunk_rows ? g.shape.chunk_rows : auto_chunk(all_rows, slots);

	const size_t nq = qs.size();
	size_t off_prefix, off_chunks;
	const size_t blob_bytes = plan_blob_bytes(qs, &off_prefix, &off_chunks);
	plan.blob.assign(blob_bytes, 0);
	plan.off_prefix = off_prefix;
	unsigned char *hb = plan.blob.data();
	QDesc *hq = reinterpret_cast<QDesc *>(hb);
	uint64_t *hprefix = reinterpret_cast<uint64_t *>(hb + off_prefix);
	uint32_t *hchunks = reinterpret_cast<uint32_t *>(hb + off_chunks);
	/* descriptors in work-list order: the queries over one table (the same
	 * segments, chunked alike) side by side as a shared scan whose chunks
	 * are claimed interleaved (QDesc::grp_size), the groups in the order of
	 * their first query.  Nothing outside the blob refers to a
	 * descriptor's place: results, counts and look-back words go through
	 * its own pointers and work range. */
	std::vector<QDesc> descs(nq);
	std::vector<size_t> order;
	order.reserve(nq);
	{
		std::map<std::pair<const void *, uint32_t>, std::vector<size_t>> groups;
		std::vector<std::pair<const void *, uint32_t>> keys;
		for (size_t i = 0; i < nq; i++) {
			const QueryLaunch &q = qs[i];
			QDesc &d = descs[i];
			memset(&d, 0, sizeof(d));
			ProgPlan pp;
			plan_program(*q.prog, pp, g.shape.full_mode);
			if (!desc_fill(d, *q.prog, pp, g, cap))
				return 0;
			/* a query continuing an earlier launch's result scans alone */
			const auto key = std::make_pair(e->shared_scan && !q.base_in ? (const void *)q.d_segs : (const void *)&qs[i],
				d.chunk_rows);
			auto it = groups.find(key);
			if (it == groups.end()) {
				keys.push_back(key);
				it = groups.emplace(key, std::vector<size_t>()).first;
			}
			it->second.push_back(i);
		}
		for (const auto &k : keys)
			for (size_t i : groups[k])
				order.push_back(i);
	}
	uint64_t work = 0;
	size_t cw = 0;
	for (size_t p = 0; p < nq; p++) {
		const size_t i = order[p];
		const QueryLaunch &q = qs[i];
		QDesc &d = hq[p];
		d = descs[i];
		d.segs = q.d_segs;
		d.nsegs = q.nsegs;
		d.seg_chunk_prefix = reinterpret_cast<const uint32_t *>(db + off_chunks + cw * sizeof(uint32_t));
		const uint64_t nch = chunk_prefix(q.seg_rows, q.nsegs, d.chunk_rows, hchunks + cw);
		cw += q.nsegs + 1;
		d.work_first = work;
		d.nchunks = nch;
		hprefix[p] = work;
		work += nch;
		for (unsigned j = 0; j < q.prog->nout; j++)
			d.out_ptr[j] = q.out[j];
		d.capacity = q.capacity;
		d.total_out = q.d_total;
		d.block_counts = q.block_counts;
		d.base_in = q.base_in;
	}
	hprefix[nq] = work;
	/* mark the shared scans: runs of two or more descriptors over the same
	 * segments with the same chunking (so the same number of chunks) */
	for (size_t p = 0; p < nq;) {
		size_t r = p + 1;
		while (r < nq && e->shared_scan && hq[r].segs == hq[p].segs && hq[r].nsegs == hq[p].nsegs &&
			hq[r].chunk_rows == hq[p].chunk_rows && hq[r].nchunks == hq[p].nchunks && hq[p].nchunks &&
			!hq[r].base_in && !hq[p].base_in)
			r++;
		if (r - p >= 2)
			for (size_t x = p; x < r; x++) {
				hq[x].grp_size = (uint32_t)(r - p);
				hq[x].grp_q0 = (uint32_t)p;
				hq[x].grp_first = (uint32_t)hq[p].work_first;
			}
		p = r;
	}
	VGPU_CHECK(work < 0xFFFFFFF0ull, "too many chunks in one launch (%llu)", (unsigned long long)work);
	plan.work = work;
	plan.nq = (uint32_t)nq;
	plan.grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(work, 1), slots);
	return 1;
}

KParams plan_params(const Plan &plan, const unsigned char *db, unsigned *counter, uint64_t *status,
	unsigned *error, uint32_t epoch)
{
	KParams kp = geom_params(plan.geom);
	kp.queries = reinterpret_cast<const QDesc *>(db);
	kp.q_work_prefix = reinterpret_cast<const uint64_t *>(db + plan.off_prefix);
	kp.nq = plan.nq;
	kp.total_work = (uint32_t)plan.work;
	kp.counter = counter;
	kp.status = status;
	kp.error = error;
	kp.epoch = epoch;
	return kp;
}

/* the key a tuned launch shape is cached under: the largest per-row staging
 * of a phase and register-vector bytes, program length and result columns
 * of the launch's queries, the number of queries and the size class of the
 * rows they scan */
std::string shape_key(const std::vector<QueryLaunch> &qs)
{
	unsigned cb = 0, fb = 0, vec = 0, nuops = 0, nout = 0;
	uint64_t rows = 0;
	for (const QueryLaunch &q : qs) {
		ProgPlan pp;
		plan_program(*q.prog, pp);
		cb = std::max(cb, pp.count_bpr);
		fb = std::max(fb, pp.full_bpr);
		vec = std::max(vec, pp.sel_bpr + pp.row_bpr);
		nuops = std::max(nuops, q.prog->nuops);
		nout = std::max(nout, q.prog->nout);
		for (uint32_t s = 0; s < q.nsegs; s++)
			rows += q.seg_rows[s];
	}
	unsigned size_class = 0;
	while ((1ull << size_class) < rows && size_class < 63)
		size_class++;
	char buf[96];
	snprintf(buf, sizeof(buf), "c%u-f%u-v%u-u%u-o%u-q%zu-r%u", cb, fb, vec, nuops, nout, qs.size(), size_class);
	return buf;
}

int run_queries(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, LaunchTiming *timing)
{
	size_t off_prefix, off_chunks;
	if (!ensure_blob(e, plan_blob_bytes(qs, &off_prefix, &off_chunks)))
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
	const Shape shape = plan.geom.shape;
	const size_t smem = plan.geom.smem;
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
	e->smem_sm = (int)prop.sharedMemPerMultiprocessor;
	e->device_name = prop.name;
	if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaMalloc((void **)&e->ctrl, 64) != cudaSuccess || cudaMemset(e->ctrl, 0, 64) != cudaSuccess ||
		cudaHostAlloc((void **)&e->h_words, 2 * sizeof(unsigned long long), cudaHostAllocDefault) != cudaSuccess) {
		delete e;
		VGPU_FAIL("engine setup failed: %s", cudaGetErrorString(cudaGetLastError()));
	}
	/* keep freed stream-ordered blocks cached instead of returning them */
	cudaMemPool_t pool;
	if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
		uint64_t thr = UINT64_MAX;
		cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
	}
	tune_cache_load(e);
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
	host_ring_free(e);
	if (e->status)
		cudaFree(e->status);
	if (e->blob)
		cudaFree(e->blob);
	for (auto &kv : e->scratch)
		if (kv.second.ptr)
			cudaFree(kv.second.ptr);
	cudaFree(e->ctrl);
	if (e->h_words)
		cudaFreeHost(e->h_words);
	cudaStreamDestroy(e->stream);
	cudaStreamDestroy(e->copy_stream);
	delete e;
}

extern "C" void *virg_gpu_engine_stream(virg_gpu_engine *e) { return e ? (void *)e->stream : nullptr; }

/* the launch shapes the tuners try: compute warps, stage size, CTAs per SM
 * and chunk bound (each with as many stages as fit) */
namespace vgpu {
std::vector<Shape> tune_candidates()
{
	std::vector<Shape> c;
	for (unsigned threads : {256u, 320u, 448u})
		for (unsigned kb : {24u, 32u, 40u, 48u})
			for (unsigned chunk : {4096u, 8192u})
				for (unsigned mode : {0u, 2u})
					c.push_back(Shape{threads, kb, 0, 1, chunk, mode});
	for (unsigned kb : {16u, 32u})
		c.push_back(Shape{256, kb, 0, 1, 8192, 1});
	/* two CTAs of four compute warps per SM: two producers and look-back
	 * warps per SM */
	for (unsigned kb : {24u, 32u})
		for (unsigned chunk : {4096u, 8192u})
			for (unsigned mode : {0u, 2u})
				c.push_back(Shape{128, kb, 0, 2, chunk, mode});
	return c;
}
}  // namespace vgpu

extern "C" int virg_gpu_query_tune(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_table *t, unsigned *shape4)
{
	VGPU_CHECK(e != nullptr && p != nullptr && t != nullptr, "null argument");
	cudaEvent_t a, z;
	CUDA_OK(cudaEventCreate(&a), "event");
	CUDA_OK(cudaEventCreate(&z), "event");
	float best = 1e30f;
	Shape best_shape = {0, 0, 0, 0, 0, 0};
	for (const Shape &c : tune_candidates()) {
		e->force = c;
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
			best_shape = e->last_shape;
		}
	}
	e->force = Shape{0, 0, 0, 0, 0, 0};
	cudaEventDestroy(a);
	cudaEventDestroy(z);
	VGPU_CHECK(best_shape.threads != 0, "no launch shape fits this program");
	/* the key of this launch */
	QueryLaunch q;
	q.prog = &p->prog;
	q.nsegs = (uint32_t)t->seg_rows.size();
	q.seg_rows = t->seg_rows.data();
	tune_remember(e, shape_key(std::vector<QueryLaunch>(1, q)), best_shape);
	if (shape4) {
		shape4[0] = best_shape.threads;
		shape4[1] = best_shape.stage_kb;
		shape4[2] = best_shape.stages;
		shape4[3] = best_shape.ctas_per_sm;
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
	unsigned stage_kb, unsigned stages, unsigned ctas_per_sm)
{
	VGPU_CHECK(e != nullptr, "null engine");
	if (threads) {
		Shape s = {threads, 32, 2, 1, 0, 0};
		VGPU_CHECK(shape_supported(s), "unsupported shape: %u compute threads (128, 256, 320, 448 or 512)", threads);
	}
	VGPU_CHECK(stage_kb <= 192, "stage size %u KB out of range", stage_kb);
	VGPU_CHECK(stages <= kMaxStages, "at most %u stages", kMaxStages);
	e->pref.threads = threads;
	e->pref.stage_kb = stage_kb;
	e->pref.stages = stages;
	e->pref.ctas_per_sm = ctas_per_sm;
	return 1;
}

extern "C" int virg_gpu_engine_set_full_mode(virg_gpu_engine *e, unsigned mode)
{
	VGPU_CHECK(e != nullptr, "null engine");
	VGPU_CHECK(mode <= 2, "full-phase mode %u: 0 in place, 1 gather, 2 dense", mode);
	e->pref.full_mode = mode;
	return 1;
}

extern "C" int virg_gpu_engine_set_shared_scan(virg_gpu_engine *e, int enable)
{
	VGPU_CHECK(e != nullptr, "null engine");
	std::lock_guard<std::mutex> lk(e->mu);
	e->shared_scan = enable != 0;
	return 1;
}

extern "C" int virg_gpu_engine_set_chunk_rows(virg_gpu_engine *e, unsigned rows)
{
	VGPU_CHECK(e != nullptr, "null engine");
	VGPU_CHECK(rows == 0 || (rows >= kBlockRows && rows <= kMaxChunkRows && rows % kBlockRows == 0),
		"chunk rows must be 0 or a multiple of %u in [%u, %u]", kBlockRows, kBlockRows, kMaxChunkRows);
	e->pref.chunk_rows = rows;
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
		shape4[1] = e->last_shape.stage_kb;
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
	table_sample(t, segs, nsegs);
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
		/* the row count and the engine's error word in one pinned copy
		 * pair and one wait */
		virg_gpu_engine *e = r->e;
		unsigned long long h = 0;
		unsigned err = 0;
		{
			std::lock_guard<std::mutex> lk(e->words_mu);
			e->h_words[0] = 0;
			e->h_words[1] = 0;
			if (!r->ntiles_zero)
				CUDA_OK(cudaMemcpyAsync(&e->h_words[0], r->d_total, sizeof(unsigned long long),
					cudaMemcpyDeviceToHost, e->stream), "result count read");
			CUDA_OK(cudaMemcpyAsync(&e->h_words[1], e->ctrl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
				e->stream), "error read");
			CUDA_OK(cudaStreamSynchronize(e->stream), "stream sync");
			h = e->h_words[0];
			err = (unsigned)e->h_words[1];
		}
		if (err)
			CUDA_OK(cudaMemsetAsync(e->ctrl + 1, 0, sizeof(unsigned), e->stream), "error clear");
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

