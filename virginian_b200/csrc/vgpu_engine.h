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

/* launch shape: compute warps, stage size and count, CTAs per SM and the
 * chunk size bound (0 in a field: the planner's choice) */
struct Shape {
	unsigned threads;      /* compute threads per CTA: 32 x compute warps */
	unsigned stage_kb;     /* data bytes per stage, in KB */
	unsigned stages;
	unsigned ctas_per_sm;  /* 0: as many as fit */
	unsigned chunk_rows;   /* upper bound on rows per chunk; 0: automatic */
	unsigned full_mode;    /* full phase of programs whose results read few bytes per row: 0 reads staged
	                        * tiles in place, 1 gathers the selected rows from device memory */
	unsigned warps() const { return threads / 32; }
	unsigned stage_bytes() const { return stage_kb * 1024u; }
};

/* shared memory of a CTA:
 *   header | chunk slots | compute warps' private areas | data buffers
 * header: mbarriers, flags, the ring of entries (tile info) and per-slot
 * chunk info; chunk slot: the chunk's query descriptor view, validity
 * bitmap, per-block counts and offsets, gathered columns' addresses; warp
 * area: a group's selection list, selection vectors and gathered columns
 * of a projection batch, row vectors of a count group.
 *
 * Entries announce the pipeline's work in order (a count tile, a full tile
 * or a chunk's gathering full phase, or the end); an entry that stages
 * data also holds one of the data buffers ("stages") until its groups are
 * done. */
constexpr unsigned kMaxStages = 12;   /* data buffers */
constexpr unsigned kEntries = 16;     /* ring of entries */
constexpr unsigned kChunkSlots = 6;
/* chunks whose count phase the producer issues before a chunk's full
 * phase, so the chunk's offset is resolved by the time its full tiles run */
#ifndef VGPU_COUNT_AHEAD
#define VGPU_COUNT_AHEAD 2
#endif
constexpr unsigned kCountAhead = VGPU_COUNT_AHEAD;
static_assert(kChunkSlots >= kCountAhead + 2, "slots for the chunks in flight");

/* blocks a compute warp filters at once (16 rows per lane; also the rows a
 * re-filtering or dense full phase takes at once), and selection entries
 * per lane in a projection batch */
#ifndef VGPU_COUNT_GROUP
#define VGPU_COUNT_GROUP 2
#endif
#ifndef VGPU_BATCH_E
#define VGPU_BATCH_E 4
#endif
constexpr unsigned kCountGroup = VGPU_COUNT_GROUP;
constexpr unsigned kBatchE = VGPU_BATCH_E;
/* a full-phase unit: one or (at most) kUnitBatches batches of 32 kBatchE
 * selected rows, each op run over all of them before the next op; a launch
 * whose warp areas hold two batches' vectors uses two-batch units for
 * entries with more than one batch of selected rows */
constexpr unsigned kUnitBatches = 2;
constexpr unsigned kBatchRows = 32 * kBatchE;
constexpr unsigned kUnitE = kBatchRows * kUnitBatches;
static_assert(32 * kBatchE <= kCountGroup * kBlockRows, "a batch within a group");
/* a compute warp's selection list: a 16-bit row per entry, for a
 * re-filtered group's valid rows or a unit's entries */
constexpr unsigned kListBytes = 2 * kCountGroup * kBlockRows;
static_assert(kUnitE * 2 <= kListBytes, "a unit's list within the list area");

/* per-stage tile, written by the producer before the stage's data lands */
struct StageInfo {
	uint32_t kind;       /* SK_* */
	uint32_t slot;       /* chunk slot */
	uint32_t chunk_seq;  /* the CTA's ordinal of the chunk (barrier phases) */
	uint32_t row0;       /* first row of the tile within its chunk */
	uint32_t nrows;
	uint32_t last;       /* the last tile of its phase for the chunk */
	uint32_t buf;        /* data buffer, or kNoBuf (a gathering full phase, the end) */
	uint32_t pad;
};
constexpr uint32_t kNoBuf = ~0u;
constexpr uint32_t SK_COUNT = 1, SK_FULL = 2, SK_END = 3;

/* per-slot chunk, written by the producer when it claims the chunk */
struct ChunkInfo {
	uint32_t valid;      /* 0: no more chunks (the pipeline's end) */
	uint32_t query;
	uint64_t work;       /* global work index */
	uint32_t rows;
	uint32_t block_base; /* the chunk's first 64-row block in its table */
	uint32_t ncount;     /* the chunk's count entries */
	uint32_t nfull;      /* the chunk's full entries */
};

constexpr unsigned kOffFull = 0;                                   /* u64[kEntries]: data landed */
constexpr unsigned kOffEmpty = kOffFull + 8 * kEntries;            /* u64[kEntries]: entry done */
constexpr unsigned kOffAnn = kOffEmpty + 8 * kEntries;             /* u64[kEntries]: info written */
constexpr unsigned kOffBfree = kOffAnn + 8 * kEntries;             /* u64[kMaxStages]: buffer free */
constexpr unsigned kOffCounted = kOffBfree + 8 * kMaxStages;       /* u64[kChunkSlots] */
constexpr unsigned kOffBased = kOffCounted + 8 * kChunkSlots;      /* u64[kChunkSlots] */
constexpr unsigned kOffDone = kOffBased + 8 * kChunkSlots;         /* u64[kChunkSlots] */
constexpr unsigned kOffDesc = kOffDone + 8 * kChunkSlots;          /* u64[kChunkSlots]: the slot's descriptor view landed */
constexpr unsigned kOffFlags = kOffDesc + 8 * kChunkSlots;         /* u32[8] */
constexpr unsigned kOffCfin = kOffFlags + 32;                      /* u32[kChunkSlots]: count entries finished */
constexpr unsigned kOffFfin = kOffCfin + 4 * kChunkSlots;          /* u32[kChunkSlots]: full entries finished */
constexpr unsigned kOffHeld = kOffFfin + 4 * kChunkSlots;          /* u32[kChunkSlots] */
constexpr unsigned kOffClaim = kOffHeld + 4 * kChunkSlots;         /* u32[kEntries]: entry tag << 16 | units taken */
constexpr unsigned kOffFin = kOffClaim + 4 * kEntries;             /* u32[kEntries]: units finished */
constexpr unsigned kOffCur = kOffFin + 4 * kEntries;               /* u32: the entry units are claimed from */
constexpr unsigned kOffStageInfo = (kOffCur + 4 + 31) / 32 * 32;
constexpr unsigned kOffChunkInfo = kOffStageInfo + (unsigned)sizeof(StageInfo) * kEntries;
constexpr unsigned kHdrBytes = (kOffChunkInfo + (unsigned)sizeof(ChunkInfo) * kChunkSlots + 127) / 128 * 128;
/* flag words */
constexpr unsigned kFAbort = 0, kFWaitMs = 1;

/* a chunk slot */
constexpr unsigned kSlotBitmap = kQDescView;                        /* u32[kChunkWords] */
constexpr unsigned kSlotBlockCnt = kSlotBitmap + 4 * kChunkWords;   /* u32[kMaxChunkBlocks] */
constexpr unsigned kSlotBlockOff = kSlotBlockCnt + 4 * kMaxChunkBlocks;  /* u64[kMaxChunkBlocks] */
constexpr unsigned kSlotColPtr = kSlotBlockOff + 8 * kMaxChunkBlocks;   /* u64[kMaxLoads]: gathered columns at the chunk's row 0 */
constexpr unsigned kSlotBytes = (kSlotColPtr + 8 * kMaxLoads + 127) / 128 * 128;
constexpr unsigned kSlotArea = kHdrBytes;
constexpr unsigned kWarpArea = kSlotArea + kChunkSlots * kSlotBytes;

/* a compute warp's private area: the selection list of a full-phase unit
 * (a 16-bit row per entry), selection vectors and gathered columns of a
 * projection batch, row vectors of a count group */
struct WarpLayout {
	uint32_t sel_off, gat_off, row_off, bytes;
};
inline WarpLayout warp_layout(unsigned sel_bytes_per_row, unsigned row_bytes_per_row, unsigned gather_bytes_per_row,
	unsigned unit_batches)
{
	WarpLayout w;
	const unsigned ue = kBatchRows * unit_batches;
	w.sel_off = kListBytes;
	w.gat_off = w.sel_off + (ue * sel_bytes_per_row + 127u) / 128u * 128u;
	w.row_off = w.gat_off + (ue * gather_bytes_per_row + 127u) / 128u * 128u;
	w.bytes = w.row_off + (kCountGroup * kBlockRows * row_bytes_per_row + 127u) / 128u * 128u;
	return w;
}

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
 * (the query's index + 1) once every chunk's rows are stored */
struct ServeRec {
	unsigned long long rows;
	unsigned long long seq;
};

/* kernel arguments */
struct KParams {
	const QDesc *queries;
	const uint64_t *q_work_prefix;  /* nq + 1 */
	uint32_t nq;
	uint32_t total_work;            /* chunks */
	unsigned *counter;              /* work claim counter, zeroed per launch */
	uint64_t *status;               /* look-back words, one per work item */
	unsigned *error;                /* first device error of the launch */
	uint32_t epoch;
	uint32_t nstages;               /* data buffers */
	uint32_t stage_bytes;           /* stride between data buffers */
	uint32_t stage_area;            /* smem offset of buffer 0 */
	uint32_t warp_bytes;            /* stride between compute warps' areas */
	uint32_t sel_off, gat_off, row_off;  /* areas within a compute warp's area */
	uint32_t unit_batches = 1;      /* batches the warp areas hold (1 or kUnitBatches) */
	/* look-back words: word idx & status_mask, tagged epoch + (idx >> status_shift);
	 * a launch with a word per work item uses ~0 and 63 (one tag) */
	unsigned long long status_mask = ~0ull;
	uint32_t status_shift = 63;
	uint32_t wait_limit_ms = 1000;  /* bound of every wait of the kernel's warps */
	/* serving sessions only (null otherwise): the work list grows while the
	 * kernel runs; finished queries are reported in recs */
	const ServeCtl *serve = nullptr;
	ServeRec *recs = nullptr;
	unsigned *done_chunks = nullptr; /* stored chunks per query */
};

/* host-side launcher implemented in vm_kernel.cu (launch shapes differ in
 * the number of compute warps) */
int launch_vm(const Shape &shape, const KParams &kp, unsigned grid, size_t smem,
	void *stream);
int shape_supported(const Shape &shape);
/* resident CTAs per SM of a shape at a dynamic shared memory size */
int occupancy(const Shape &shape, size_t smem, int *ctas_per_sm);

}  // namespace vgpu

struct virg_gpu_program {
	vgpu::Program prog;
	vgpu::ProgramExtra extra;
	virg_gpu_schema schema;
};

#endif
