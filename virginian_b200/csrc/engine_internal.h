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

}  // namespace vgpu

struct virg_gpu_engine {
	int device = 0;
	int nsm = 0;
	int smem_optin = 0;
	cudaStream_t stream = nullptr;       /* launches, descriptor and result copies */
	cudaStream_t copy_stream = nullptr;  /* streamed tablet uploads */
	unsigned *ctrl = nullptr;            /* [0] work counter, [1] error word */
	uint64_t *status = nullptr;          /* look-back words */
	size_t status_cap = 0;
	uint32_t epoch = 0;
	void *blob = nullptr;                /* per-launch descriptors */
	size_t blob_cap = 0;
	std::vector<unsigned char> host_blob;
	std::map<int, vgpu::ScratchBuf> scratch;
	vgpu::Shape pref = {0, 0, 0, 0};
	vgpu::Shape last_shape = {0, 0, 0, 0};
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
	vgpu::Shape force = {0, 0, 0, 0};  /* shape under trial while tuning */
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

/* a launch of one or more queries, ready to issue */
struct Plan {
	Shape shape;
	size_t smem = 0;
	uint32_t stage_bytes = 0, vec_bytes = 0;
	std::vector<unsigned char> blob;  /* host copy of the device descriptors */
	size_t off_prefix = 0;
	uint64_t work = 0;
	uint32_t nq = 0;
	unsigned grid = 0;
};

void program_layout(const Program &P, unsigned tile, uint32_t *load_off, uint32_t *stage_bytes,
	uint32_t *row_bytes, uint32_t *sel_bytes);
void vec_offsets(const Program &P, unsigned tile, uint32_t row_slot, uint32_t *vec_off);
void launch_layout(const std::vector<const Program *> &progs, unsigned tile, uint32_t *stage_bytes,
	uint32_t *row_slot, uint32_t *vec_bytes);
size_t smem_for(const Shape &s, uint32_t stage_bytes, uint32_t vec_bytes);
void fill_operands(QDesc &d, uint32_t vec_area);
size_t plan_blob_bytes(const std::vector<QueryLaunch> &qs, size_t *off_prefix, size_t *off_tiles);
int plan_build(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, const Shape *forced,
	unsigned char *db, Plan &plan);
KParams plan_params(const Plan &plan, const unsigned char *db, unsigned *counter, uint64_t *status,
	unsigned *error, uint32_t epoch);
int run_queries(virg_gpu_engine *e, const std::vector<QueryLaunch> &qs, LaunchTiming *timing);
std::string shape_key(const std::vector<QueryLaunch> &qs);
int read_device_error(virg_gpu_engine *e, unsigned *err);
const char *device_error_text(unsigned code);
uint32_t padded_rows(uint32_t rows);
int table_add_segments(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned n,
	const bool *want_col, bool want_key, cudaStream_t stream);
int table_sync_desc(virg_gpu_table *t);
int result_alloc(virg_gpu_engine *e, const Program &P, uint64_t capacity, bool block_counts,
	uint64_t nblocks, virg_gpu_result **out);
int choose_shape(virg_gpu_engine *e, const std::vector<const Program *> &progs, Shape *out,
	size_t *smem_out, uint32_t *stage_out, uint32_t *vec_out);

}  // namespace vgpu

#endif
