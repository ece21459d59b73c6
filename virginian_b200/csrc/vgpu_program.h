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

/* operand descriptor resolved for a launch shape: bits [0,30) are a shared
 * memory byte offset, bits [30,32) the kind */
constexpr uint32_t OD_STAGE = 0u << 30;    /* staged column, + stage offset */
constexpr uint32_t OD_ROWVEC = 1u << 30;   /* register vector by tile row */
constexpr uint32_t OD_SELVEC = 2u << 30;   /* register vector by selection index */
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

/* per-query launch descriptor, in device memory */
struct alignas(16) QDesc {
	/* Everything before `prog` is what the kernel reads from a stage's copy
	 * of the descriptor (the stage holds only that prefix); the decoded
	 * program itself is read from device memory by the producer (its loads)
	 * and is host-side otherwise. */
	/* the program's constants, split point, op count and result columns */
	uint64_t consts[kMaxRegs];
	uint32_t nfilter;
	uint32_t nuops;
	uint32_t nout;
	uint8_t out_stride[kMaxRegs];
	/* smem layout for this launch shape */
	uint32_t load_off[kMaxLoads];
	uint32_t stage_bytes;
	uint32_t vec_off[kMaxRegs];
	/* the uops as records (handler, operands) and the result columns'
	 * operand descriptors */
	OpRec ops[kMaxOps];
	uint32_t od_out[kMaxRegs];
	/* inputs */
	const SegDesc *segs;
	const uint32_t *seg_tile_prefix;  /* nsegs + 1 entries */
	uint32_t nsegs;
	uint32_t vec_slot;                /* distance between the two row-vector slots */
	uint64_t work_first;              /* global work index of tile 0 */
	uint64_t ntiles;
	/* outputs */
	void *out_ptr[kMaxRegs];
	uint64_t capacity;                /* rows each out column can hold */
	unsigned long long *total_out;    /* written by the last tile */
	uint8_t *block_counts;            /* optional: valid rows per 64-row block */
	/* optional: result rows already written by earlier launches of the same
	 * query; its first tile starts there */
	const unsigned long long *base_in;
	uint64_t pad1;
	Program prog;
};

/* bytes of a descriptor that a stage holds (the kernel's view) */
constexpr unsigned kQDescStaged = (unsigned)((offsetof(QDesc, prog) + 15) / 16 * 16);

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
