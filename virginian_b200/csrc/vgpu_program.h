/*
 * Decoded form of a Virginian data-parallel section, shared by the host-side
 * decoder (program.cpp) and the sm_100a kernel (vm_kernel.cu).
 *
 * The reference executes the opcode program (virg_op, src/virginian.h:327-333)
 * once per 64-row block on the CPU (src/vm/virginia.c:352-877) or once per
 * row on the GPU (src/vm/vm_gpu.cu:1152-1225).  Here the program is decoded
 * once on the host into "uops" that keep the semantics of the single-core CPU
 * VM, which is the reference for results:
 *
 *  - a row is active at the op with program counter k when its pending jump
 *    target is <= k (the CPU keeps row_pc[i] == pc for active rows and
 *    row_pc[i] > pc for rows that jumped ahead, src/vm/virginia.c:57-66);
 *  - Column/Rowid read the whole block regardless of row pc
 *    (src/vm/virginia.c:442-474), so a register defined only by loads of one
 *    column aliases that column's staged tile and costs no device op;
 *  - a register defined only by Integer/Float ops of one value is a scalar;
 *  - every other register definition is an interpreted op writing a per-row
 *    register vector, and only for active rows, as the CPU does.
 */
#ifndef VGPU_PROGRAM_H
#define VGPU_PROGRAM_H

#include <stddef.h>
#include <stdint.h>

namespace vgpu {

constexpr int kMaxOps = 32;      /* VIRG_OPS, src/virginian.h:100 */
constexpr int kMaxRegs = 16;     /* VIRG_REGS, src/virginian.h:96 */
constexpr int kMaxCols = 16;     /* VIRG_MAX_COLUMNS, src/virginian.h:72 */
constexpr int kKeySlot = 16;     /* segment column index of the key column */
constexpr int kMaxLoads = 17;    /* 16 fixed columns + key */

/* value types, same numbering as virg_t (src/virginian.h:196-204) */
enum VType : uint8_t { VT_INT = 0, VT_INT64 = 1, VT_FLOAT = 2, VT_DOUBLE = 3, VT_CHAR = 4 };

enum UKind : uint8_t {
	UK_CMP = 1,      /* Le..Neq, And, Or: jump to target when true */
	UK_NOT = 2,      /* Not: jump when the value is zero */
	UK_MATH = 3,     /* Add/Sub/Mul/Div into a register vector */
	UK_INVALID = 4,  /* Invalid: clear validity of active rows */
	UK_SETCONST = 5, /* Integer/Float into a register vector */
	UK_COPYCOL = 6,  /* Column/Rowid into a register vector */
	UK_RESULT = 7    /* Result: ordered append of valid rows */
};

enum CmpOp : uint8_t { CO_LE = 0, CO_LT, CO_GE, CO_GT, CO_EQ, CO_NEQ, CO_AND, CO_OR };
enum MathOp : uint8_t { MO_ADD = 0, MO_SUB, MO_MUL, MO_DIV };

/* operand classes */
enum OClass : uint8_t { OC_COL = 0, OC_VEC = 1, OC_CONST = 2 };

struct UOp {
	uint8_t kind;
	uint8_t sub;      /* CmpOp / MathOp */
	uint8_t type;     /* VType of the operands */
	uint8_t dst;      /* vector slot written (MATH/SETCONST/COPYCOL) */
	uint8_t a_cls, a_idx;
	uint8_t b_cls, b_idx;
	uint8_t pc;       /* program counter of the source op */
	uint8_t target;   /* jump target (CMP/NOT) */
	uint8_t vjump;    /* validity kept on jump: p4.i != 0 */
	uint8_t tslot;    /* pending-target slot the jump parks rows in */
	uint8_t join;     /* slots whose rows become active again at this op */
	uint8_t flags;    /* UF_* */
	uint8_t pad0, pad1;
};

/* the destination register has this single definition, so rows that skip
 * the op never read it and the store need not be predicated */
constexpr uint8_t UF_SINGLE_DEF = 1;
constexpr int kMaxSlots = 8;     /* pending jump targets at any one time */

/* what a decoded program needs; independent of the launch shape */
struct Program {
	UOp uops[kMaxOps];
	uint32_t nuops;
	/* staged columns: source column index or kKeySlot, and stride */
	uint32_t nload;
	uint8_t load_src[kMaxLoads];
	uint8_t load_stride[kMaxLoads];
	uint8_t load_type[kMaxLoads];
	/* register vectors */
	uint32_t nvec;
	uint8_t vec_stride[kMaxRegs];
	/* scalar registers */
	uint32_t nconst;
	uint64_t consts[kMaxRegs];
	/* result columns */
	uint32_t nout;
	uint8_t out_cls[kMaxRegs], out_idx[kMaxRegs], out_type[kMaxRegs], out_stride[kMaxRegs];
	/* uops [0, nfilter) run on every row of a tile (the filter); uops
	 * [nfilter, nuops - 1) only on the rows still valid (the projection);
	 * uops[nuops - 1] is the Result */
	uint32_t nfilter;
	/* register vectors written only by projection uops are indexed by a
	 * row's position in its warp's selection list, not by its tile row */
	uint8_t vec_compact[kMaxRegs];
};

/* operand descriptor resolved for a launch layout: bits [0,30) are a byte
 * offset, bits [30,32) the kind.  The kernel adds the base the kind names:
 * the stage holding the tile (staged columns), the warp's row-vector or
 * selection-vector area, or the chunk slot's descriptor copy (scalars). */
constexpr uint32_t OD_STAGE = 0u << 30;    /* staged column, indexed by tile row */
constexpr uint32_t OD_ROWVEC = 1u << 30;   /* register vector, indexed by block row */
constexpr uint32_t OD_SELVEC = 2u << 30;   /* register vector, indexed by selection entry */
constexpr uint32_t OD_SCALAR = 3u << 30;   /* scalar register */
constexpr uint32_t OD_OFFSET = (1u << 30) - 1;

/* one interpreted op as the kernel reads it: a single 16-byte record, so a
 * warp fetches everything an op needs with one shared-memory load */
struct alignas(16) OpRec {
	uint32_t head;
	uint32_t a, b, d;  /* operand descriptors: source a, source b, destination */
};

/* The head's fields are one-hot, so the kernel picks an op's code with a few
 * uniform bit-test branches instead of an indirect jump through a table:
 * bits [0,6) kind, [6,11) operand type (bit OT_SHIFT + VType), [11,19)
 * operator (bit OO_SHIFT + CmpOp or MathOp), [19,22) pending-target slot,
 * bit 22 validity kept on jump, bit 23 single definition, [24,32) slots
 * joined at this op. */
constexpr uint32_t OK_CMP = 1u << 0;       /* Le..Neq, And, Or */
constexpr uint32_t OK_MATH = 1u << 1;      /* Add/Sub/Mul/Div */
constexpr uint32_t OK_NOT = 1u << 2;
constexpr uint32_t OK_INVALID = 1u << 3;
constexpr uint32_t OK_SETCONST = 1u << 4;  /* 4-byte Integer/Float */
constexpr uint32_t OK_COPY = 1u << 5;      /* Column/Rowid into a register vector */
constexpr uint32_t OT_SHIFT = 6;
constexpr uint32_t OO_SHIFT = 11;
constexpr uint32_t OPH_SLOT_SHIFT = 19;
constexpr uint32_t OPH_VJUMP = 1u << 22;
constexpr uint32_t OPH_SINGLE_DEF = 1u << 23;
constexpr uint32_t OPH_JOIN_SHIFT = 24;

/* one resident segment (tablet) on the device */
struct SegDesc {
	const void *col[kMaxLoads];  /* fixed columns 0..15, key at kKeySlot */
	uint32_t rows;
	uint32_t block_base;         /* first 64-row block of this segment */
};

/* Rows are processed in blocks of kBlockRows (8 words of 32 rows; lane l of
 * a warp holds rows l, l + 32, ..., l + 224 of its block) and scanned in
 * chunks of at most kMaxChunkRows rows that lie inside one segment.  A chunk
 * is the unit of claiming and of ordered placement: its count phase stages
 * the columns the filter reads and leaves one validity bit per row, its full
 * phase stages the columns the results need and stores the selected rows at
 * the chunk's offset. */
constexpr unsigned kBlockRows = 256;
constexpr unsigned kMaxChunkRows = 8192;
constexpr unsigned kMaxChunkBlocks = kMaxChunkRows / kBlockRows;  /* 32: one lane each */
constexpr unsigned kChunkWords = kMaxChunkRows / 32;

/* how the full phase gets its rows.  FM_BITMAP and FM_GATHER take the rows'
 * validity from the count phase's bitmap (the results read only columns,
 * constants and vectors computed after the filter) and split an entry's
 * selected rows into batches of up to 32 kBatchE rows, each a unit of work:
 *  - FM_BITMAP stages full tiles of the columns the results read and reads
 *    the selected rows in place;
 *  - FM_GATHER stages nothing: it loads the selected rows' values straight
 *    from device memory into the compute warp's own area.
 * FM_REFILTER stages full tiles of every column and runs the filter again
 * over groups of kCountGroup blocks (the results read register vectors the
 * filter computed).  FM_DENSE stages full tiles and runs the projection over
 * every row of a group of kCountGroup blocks, as the filter runs (rows held
 * by lanes, register vectors indexed by row), then stores the valid rows at
 * their ranks: no selection list and no indirect operand addresses, for
 * programs whose rows mostly pass the filter (a tuning choice). */
constexpr uint32_t FM_BITMAP = 0;
constexpr uint32_t FM_REFILTER = 1;
constexpr uint32_t FM_GATHER = 2;
constexpr uint32_t FM_DENSE = 3;
/* the largest bytes per row a gathering full phase moves into a compute
 * warp's area */
constexpr uint32_t kGatherMaxBpr = 32;
/* the largest bytes per row of register vectors a dense full phase keeps
 * for a whole count group in a compute warp's area (wider programs keep
 * the in-place full phase) */
constexpr uint32_t kDenseMaxRowBpr = 16;

/* the staged columns of one phase: which segment columns, where in a stage */
struct LoadSet {
	uint32_t n;
	uint32_t rows;                /* rows per tile of this phase (multiple of kBlockRows) */
	uint32_t bytes_per_row;
	uint32_t pad;
	uint8_t src[kMaxLoads];       /* segment column index, kKeySlot for the key */
	uint8_t stride[kMaxLoads];
	uint8_t pad2[14];
	uint32_t off[kMaxLoads];      /* byte offset of the column in the stage */
	uint32_t pad3[3];
};

/* per-query launch descriptor, in device memory */
struct alignas(16) QDesc {
	/* ---- the kernel's view: the producer copies everything up to `segs`
	 * into the chunk slot of each chunk it claims (unless the slot holds the
	 * same query already); compute and look-back warps read only that copy */
	uint64_t consts[kMaxRegs];     /* scalar registers (OD_SCALAR offsets point here) */
	uint32_t nfilter;              /* uops [0, nfilter) are the filter */
	uint32_t nuops;                /* uops [nfilter, nuops - 1) the projection, then Result */
	uint32_t nout;
	uint32_t full_mode;            /* FM_BITMAP, FM_REFILTER or FM_GATHER */
	uint32_t chunk_rows;           /* rows per chunk (a multiple of both tile sizes) */
	uint32_t pad0[3];
	uint8_t out_stride[kMaxRegs];
	/* the filter over the count phase's staged columns, and every uop over
	 * the full phase's (the filter part only used by FM_REFILTER) */
	OpRec ops_count[kMaxOps];
	OpRec ops_full[kMaxOps];
	uint32_t od_out[kMaxRegs];     /* result columns, over the full phase's layout */
	/* FM_GATHER: the columns the results read (the full set) and where a
	 * batch of them sits in a compute warp's gather area */
	uint32_t gather_n;
	uint8_t gather_stride[kMaxLoads];
	uint8_t pad3[3];
	uint32_t gather_off[kMaxLoads];
	uint32_t pad4;
	void *out_ptr[kMaxRegs];
	uint64_t capacity;             /* rows each out column can hold */
	unsigned long long *total_out; /* the query's row count, written with its last chunk's offset */
	uint8_t *block_counts;         /* optional: valid rows per 64-row block */
	/* optional: result rows already written by earlier launches of the same
	 * query; its first chunk starts there */
	const unsigned long long *base_in;
	uint64_t work_first;           /* global work index of the query's chunk 0 */
	uint64_t nchunks;
	/* ---- the producer's view, read from device memory */
	const SegDesc *segs;
	const uint32_t *seg_chunk_prefix;  /* nsegs + 1 entries */
	uint32_t nsegs;
	/* a shared scan: grp_size queries over the same segments with the same
	 * chunking (descriptors grp_q0, grp_q0 + 1, ...) hold consecutive places
	 * in the work list from grp_first on, and their chunks are claimed
	 * interleaved (claim grp_first + t * grp_size + g is chunk t of query
	 * grp_q0 + g), so one chunk of the table is read by all of them within
	 * a few claims; grp_size 0 or 1: claims are work items */
	uint32_t grp_size;
	uint32_t grp_q0;
	uint32_t grp_first;
	LoadSet count_set, full_set;
	Program prog;
};

/* bytes of a descriptor that a chunk slot holds (the kernel's view), and the
 * slot area that holds them */
constexpr unsigned kQDescCopy = (unsigned)offsetof(QDesc, segs);
constexpr unsigned kQDescView = (kQDescCopy + 127) / 128 * 128;
static_assert(kQDescCopy % 16 == 0, "the view is copied in 16-byte units");

/* device error codes (written once per launch to the error word) */
enum DevError : unsigned {
	DE_NONE = 0,
	DE_LOOKBACK_TIMEOUT = 1,
	DE_STAGE_TIMEOUT = 2,
	DE_OUTPUT_OVERFLOW = 3,
	DE_BAD_WORK = 4
};

/* look-back status word: [63:44] epoch, [43:42] flag, [41:0] count */
constexpr int kStatusEpochShift = 44;
constexpr int kStatusFlagShift = 42;
constexpr uint64_t kStatusValueMask = (1ull << 42) - 1;
constexpr uint64_t kFlagAggregate = 1;
constexpr uint64_t kFlagPrefix = 2;
constexpr uint32_t kEpochMask = (1u << 20) - 1;

}  // namespace vgpu

#endif
