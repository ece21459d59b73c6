/* Host-side engine structures (not part of the C ABI). */
#ifndef VGPU_ENGINE_INTERNAL_H
#define VGPU_ENGINE_INTERNAL_H

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vgpu_engine.h"

namespace vgpu {

struct ScratchBuf {
	void *ptr = nullptr;
	size_t cap = 0;
};

/* a host sample of a resident table's rows: runs of consecutive rows from
 * segments spread over each append, per column (index kKeySlot: the key) */
struct TableSample {
	uint32_t rows = 0, runs = 0;
	std::vector<unsigned char> col[kMaxLoads];
};

/* the engine's staging ring for rows read from host memory: device buffers
 * and events kept across calls, grown when a call needs more */
struct HostRing {
	static constexpr unsigned kBufs = 3;
	unsigned char *mem[kBufs] = {};
	size_t bytes = 0;                    /* each buffer */
	SegDesc *d_segs[kBufs] = {};
	size_t seg_cap = 0;                  /* descriptors each buffer holds */
	cudaEvent_t copied[kBufs] = {}, freed[kBufs] = {}, c0[kBufs] = {}, c1[kBufs] = {};
	unsigned long long *d_totals = nullptr;  /* running result counts, two alternating words */
	bool ready = false;
};

}  // namespace vgpu

struct virg_gpu_engine {
	int device = 0;
	int nsm = 0;
	int smem_optin = 0;                  /* shared memory per CTA (opt-in limit) */
	int smem_sm = 0;                     /* shared memory per SM */
	cudaStream_t stream = nullptr;       /* launches, descriptor and result copies */
	cudaStream_t copy_stream = nullptr;  /* streamed tablet uploads */
	unsigned *ctrl = nullptr;            /* [0] work counter, [1] error word */
	/* pinned: a result's row count and the error word, read back together */
	unsigned long long *h_words = nullptr;
	std::mutex words_mu;
	uint64_t *status = nullptr;          /* look-back words */
	size_t status_cap = 0;
	uint32_t epoch = 0;
	void *blob = nullptr;                /* per-launch descriptors */
	size_t blob_cap = 0;
	std::vector<unsigned char> host_blob;
	std::map<int, vgpu::ScratchBuf> scratch;
	vgpu::HostRing hring;
	vgpu::Shape pref = {0, 0, 0, 0, 0, 0};
	vgpu::Shape last_shape = {0, 0, 0, 0, 0, 0};
	unsigned last_grid = 0;
	size_t last_smem = 0;
	unsigned long long launches = 0;
	int launches_last = 0;
	bool timing_enabled = false;
	cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
	/* ring of (start, stop) events recorded around each kernel launch */
	std::vector<cudaEvent_t> ring_start, ring_stop;
	unsigned long long ring_count = 0;
	/* launch shapes found by autotuning, per program-shape key */
	std::map<std::string, vgpu::Shape> tuned;
	std::string device_name;             /* keys the persistent tuned-shape cache */
	vgpu::Shape force = {0, 0, 0, 0, 0, 0};  /* shape under trial while tuning */
	bool shared_scan = false;            /* queries over one table claim their chunks interleaved */
	std::mutex mu;
};

struct virg_gpu_table {
	virg_gpu_engine *e = nullptr;
	virg_gpu_schema schema;
	std::vector<vgpu::SegDesc> segs;     /* device pointers, host copy */
	std::vector<uint32_t> seg_rows;
	std::vector<void *> allocs;
	vgpu::SegDesc *d_segs = nullptr;
	bool dirty = false;
	uint32_t segs_without_key = 0;       /* non-empty segments lacking a key */
	bool transient = false;              /* stream-ordered allocations */
	uint64_t rows = 0;
	uint64_t bytes = 0;
	uint32_t blocks = 0;                 /* 64-row blocks so far */
	vgpu::TableSample sample;            /* for result-size estimates */
};

struct virg_gpu_result {
	virg_gpu_engine *e = nullptr;
	unsigned nout = 0;
	void *out[vgpu::kMaxRegs] = {nullptr};
	unsigned stride[vgpu::kMaxRegs] = {0};
	unsigned type[vgpu::kMaxRegs] = {0};
	uint64_t capacity = 0;
	unsigned long long *d_total = nullptr;
	uint8_t *block_counts = nullptr;
	uint64_t nblocks = 0;
	void *mem = nullptr;
	uint64_t rows = 0;
	bool have_rows = false;
	bool ntiles_zero = false;
};

namespace vgpu {

struct QueryLaunch {
	const Program *prog = nullptr;
	const SegDesc *d_segs = nullptr;
	uint32_t nsegs = 0;
	const uint32_t *seg_rows = nullptr;
	void *out[kMaxRegs] = {nullptr};
	uint64_t capacity = 0;
	unsigned long long *d_total = nullptr;
	uint8_t *block_counts = nullptr;
	const unsigned long long *base_in = nullptr;
};

struct LaunchTiming {
	cudaEvent_t start;
	cudaEvent_t stop;
};

/* the staging plan of a program, independent of the launch geometry:
 * which load slots each phase stages, how the full phase gets validity and
 * where the program's register vectors sit in a compute warp's areas */
struct ProgPlan {
	uint8_t count_cols[kMaxLoads], full_cols[kMaxLoads];
	uint32_t ncount, nfull;
	uint32_t count_bpr, full_bpr;  /* staged bytes per row of each phase */
	uint32_t mode;                 /* FM_GATHER, FM_BITMAP or FM_REFILTER */
	uint32_t sel_bpr, row_bpr;     /* register-vector bytes per row */
	uint32_t gather_bpr;           /* bytes per row in a warp's gather area (FM_GATHER) */
	uint32_t vec_off[kMaxRegs];    /* offset in the selection or row-vector area */
};

/* a launch geometry: its shape and the shared-memory layout that every
 * query of the launch fits */
struct Geom {
	Shape shape;
	WarpLayout wl;
	uint32_t ub;                  /* batches a full-phase unit may hold */
	uint32_t stage_area;
	size_t smem;
};

/* a launch of one or more queries, ready to issue */
struct Plan {
	Geom geom;
	std::vector<unsigned char> blob;  /* host copy of the device descriptors */
	size_t off_prefix = 0;
	uint64_t work = 0;                /* chunks */
	uint32_t nq = 0;
	unsigned grid = 0;
};

/* full_mode: as Shape::full_mode (1: gather from device memory where the
 * program allows it) */
void plan_program(const Program &P, ProgPlan &pp, unsigned full_mode = 0);
/* ub_max: the most batches a full-phase unit may hold (two-batch units are
 * taken when the warp areas for them leave as many data buffers, or three) */
int geom_make(const Shape &s, uint32_t sel_bpr, uint32_t row_bpr, uint32_t gather_bpr, int smem_block, int smem_sm,
	Geom *g, uint32_t ub_max = kUnitBatches);
int desc_fill(QDesc &d, const Program &P, const ProgPlan &pp, const Geom &g, uint32_t chunk_cap);
uint64_t chunk_prefix(const uint32_t *seg_rows, uint32_t nsegs, uint32_t chunk_rows, uint32_t *pre);
KParams geom_params(const Geom &g);
size_t plan_blob_bytes(const std::vector<QueryLaunch> &qs, size_t *off_prefix, size_t *off_chunks);
int plan_build(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, const Shape *forced,
	unsigned char *db, Plan &plan);
KParams plan_params(const Plan &plan, const unsigned char *db, unsigned *counter, uint64_t *status,
	unsigned *error, uint32_t epoch);
int run_queries(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, LaunchTiming *timing);
/* one program over rows in host memory, through the engine's staging ring:
 * contiguous host rows are merged into pieces, pieces into chunks of at most
 * chunk_rows rows; each chunk is copied on the copy stream and scanned by
 * one launch that appends to result r.  The caller holds the engine's lock. */
int host_pipeline(virg_gpu_engine *e, const Program &P, const virg_gpu_segment *segs, unsigned nsegs,
	uint64_t chunk_rows, virg_gpu_result *r, virg_gpu_stream_stats *stats);
void host_ring_free(virg_gpu_engine *e);
/* the persistent tuned-shape cache: loaded when an engine is created, and
 * a newly tuned shape recorded in the engine and appended to it */
void tune_cache_load(virg_gpu_engine *e);
/* the table's host sample, extended by appended segments; the fraction of
 * sample rows a program's filter keeps (negative: no usable sample) */
void table_sample(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned n);
double sample_selectivity(const Program &P, const virg_gpu_table *t);
void tune_remember(virg_gpu_engine *e, const std::string &key, const Shape &s);
std::string shape_key(const std::vector<QueryLaunch> &qs);
int read_device_error(virg_gpu_engine *e, unsigned *err);
const char *device_error_text(unsigned code);
uint32_t padded_rows(uint32_t rows);
int table_add_segments(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned n,
	const bool *want_col, bool want_key, cudaStream_t stream);
int table_sync_desc(virg_gpu_table *t);
int result_alloc(virg_gpu_engine *e, const Program &P, uint64_t capacity, bool block_counts,
	uint64_t nblocks, virg_gpu_result **out);
int choose_shape(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, Geom *g);
/* the launch shapes the autotuners time */
std::vector<Shape> tune_candidates();

}  // namespace vgpu

#endif
