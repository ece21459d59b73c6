/* Engine internals shared by the host-side translation units. */
#ifndef VGPU_ENGINE_H
#define VGPU_ENGINE_H

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/virginian_b200.h"
#include "vgpu_program.h"

namespace vgpu {

struct ProgramExtra {
	int maybe_undefined;  /* some row may read a register its path never set */
	int result_k;         /* program index of the Result op */
	int converge_k;       /* program index of the Converge op */
	int split_k;          /* first op of the projection (== result_k if none) */
};

int decode_program(const virg_op *ops, unsigned num_ops, unsigned pc,
	const virg_gpu_schema &schema, Program &P, ProgramExtra &X);

/* launch shape: CTA width, rows per thread, staging depth, CTAs per SM */
struct Shape {
	unsigned threads;
	unsigned rows_per_thread;
	unsigned stages;
	unsigned ctas_per_sm;
	unsigned tile() const { return threads * rows_per_thread; }
};

/* fixed smem header of the kernel: QDesc copy, barriers, per-stage work
 * info and the result-scan scratch */
/* (the kernel's fixed header: barriers, tile offsets, scan scratch) */
constexpr unsigned kMaxStages = 8;
constexpr unsigned kSmemHeader = 2048;

/* per-stage work item, decoded by the issuing thread */
struct StageInfo {
	uint32_t work;      /* global work index, >= total when empty */
	uint32_t query;
	uint32_t seg;
	uint32_t row0;
	uint32_t nrows;
	uint32_t pad[3];
};

/* every stage starts with a copy of its tile's query descriptor and the tile's
 * StageInfo, then the staged columns */
/* tiles in flight between the filter and the stores of a CTA: slots of the
 * selection lists, row vectors, counts and offsets */
constexpr unsigned kSlots = 3;

constexpr unsigned kStageHdr = (unsigned)((kQDescStaged + sizeof(StageInfo) + 127) / 128 * 128);

/* serving-session control, in host-mapped memory written by the host:
 * published queries and work items (a query's descriptor is complete before
 * it is counted here) and the stop request */
struct ServeCtl {
	unsigned long long avail;  /* (queries << 40) | work items */
	unsigned stop;             /* no more work after `avail` */
	unsigned pad;
};
constexpr unsigned long long kAvailWorkMask = (1ull << 40) - 1;

/* per-query completion record, in host-mapped memory: rows, then `seq`
 * (the query's index + 1) once every tile's rows are stored */
struct ServeRec {
	unsigned long long rows;
	unsigned long long seq;
};

/* kernel arguments */
struct KParams {
	const QDesc *queries;
	const uint64_t *q_work_prefix;  /* nq + 1 */
	uint32_t nq;
	uint32_t total_work;
	unsigned *counter;              /* work claim counter, zeroed per launch */
	uint64_t *status;               /* look-back words, one per work item */
	unsigned *error;                /* first device error of the launch */
	uint32_t epoch;
	uint32_t nstages;
	uint32_t stage_bytes;           /* stride between stages */
	uint32_t stage_area;            /* smem offset of stage 0 */
	uint32_t vec_area;              /* smem offset of the register-vector region */
	uint32_t vec_bytes;             /* its size (the largest of the launch's queries) */
	uint32_t sel_area;              /* smem offset of the selection lists (2 slots) */
	/* look-back words: word idx & status_mask, tagged epoch + (idx >> status_shift);
	 * a launch with a word per work item uses ~0 and 63 (one tag) */
	unsigned long long status_mask = ~0ull;
	uint32_t status_shift = 63;
	uint32_t wait_limit_ms = 1000;  /* bound of every wait of the kernel's warps */
	/* serving sessions only (null otherwise): the work list grows while the
	 * kernel runs; finished queries are reported in recs */
	const ServeCtl *serve = nullptr;
	ServeRec *recs = nullptr;
	unsigned *done_tiles = nullptr; /* stored tiles per query */
};

/* host-side launcher implemented in vm_kernel.cu */
int launch_vm(const Shape &shape, const KParams &kp, unsigned grid, size_t smem,
	void *stream);
/* largest dynamic shared memory and resident CTAs for a shape */
int shape_supported(const Shape &shape);
int occupancy(const Shape &shape, size_t smem, int *ctas_per_sm);

}  // namespace vgpu

struct virg_gpu_program {
	vgpu::Program prog;
	vgpu::ProgramExtra extra;
	virg_gpu_schema schema;
};

#endif
