/*
 * The sm_100a data-parallel VM kernel.
 *
 * Replaces the reference's virginia_gpu (src/vm/vm_gpu.cu:1152-1225), which
 * runs one thread per row with a 16-entry register file in local memory, a
 * switch dispatch per op per thread and atomics for (unordered) result
 * placement.  Here persistent CTAs claim chunks of rows (at most
 * kMaxChunkRows rows of one segment of one query) in order and run each
 * chunk in two phases through a ring of shared-memory stages:
 *
 *  - count phase: the producer warp bulk-copies (cp.async.bulk, completing
 *    on the stage's mbarrier) only the columns the filter reads; compute
 *    warps run the filter ops over 256-row blocks (a lane holds rows l,
 *    l + 32, ..., l + 224 as bits of its row masks) and leave one validity
 *    bit per row in the chunk slot's bitmap and a count per block;
 *  - the look-back warp sums the chunk's block counts, publishes them to the
 *    query's look-back words and resolves the chunk's place in the query's
 *    result with a decoupled look-back over earlier chunks, then writes
 *    each block's result offset;
 *  - full phase: the producer stages the columns the result columns need;
 *    compute warps build each block's selection list from the bitmap, run
 *    the projection ops on the selected rows 32 at a time and store them
 *    at the block's offset (coalesced, original row order).
 *
 * The producer takes the data buffer in turn if it is free, else the next
 * one released (tiles release out of order), and issues a chunk's count
 * phase kCountAhead chunks before its full phase, so a chunk's offset is
 * resolved while the CTA counts the next chunks: no stage waits for another
 * CTA, and a column both phases read is read from HBM once and found in L2
 * the second time.
 *
 * Each op is one 16-byte record read with one shared-memory load and
 * dispatched by bit tests on its head; operands are read and written by
 * 32-bit shared-memory address.  Rows land in the single-core CPU VM's
 * order (src/vm/virginia.c:476-578) with plain stores; no output atomics.
 * Arithmetic matches the CPU VM bit for bit: float/double use the _rn
 * intrinsics (no FMA contraction, IEEE division) and x86 NaN results,
 * integers wrap as on x86.  Every wait is bounded; on expiry the kernel
 * records an error code and stops instead of hanging.
 */
#include <cstddef>
#include <cstdint>
#include <climits>

#include <cuda_runtime.h>

#include "vgpu_engine.h"

namespace vgpu {

/* bounded waits: a stage, slot or offset wait gives up after the launch's
 * limit (a second by default), far beyond any real wait; look-back polls
 * after 2^24 rounds of 32-256 ns */
constexpr uint32_t kSuspendHintNs = 20000;
/* 1 (default): the producer gives a tile the buffer in turn if it is free,
 * else the next released one (entries release their buffers out of order:
 * a count tile keeps its buffer for a dozen groups, a sparse projection
 * tile for a unit or two); 0: buffers strictly in turn */
#ifndef VGPU_BUF_FREELIST
#define VGPU_BUF_FREELIST 1
#endif
constexpr unsigned kLookbackSpinLimit = 1u << 24;

/* where the fields the kernel's warps read sit in a slot's descriptor copy */
constexpr uint32_t kQNFilter = (uint32_t)offsetof(QDesc, nfilter);
constexpr uint32_t kQNUops = (uint32_t)offsetof(QDesc, nuops);
constexpr uint32_t kQNOut = (uint32_t)offsetof(QDesc, nout);
constexpr uint32_t kQFullMode = (uint32_t)offsetof(QDesc, full_mode);
constexpr uint32_t kQOutStride = (uint32_t)offsetof(QDesc, out_stride);
constexpr uint32_t kQOpsCount = (uint32_t)offsetof(QDesc, ops_count);
constexpr uint32_t kQOpsFull = (uint32_t)offsetof(QDesc, ops_full);
constexpr uint32_t kQOdOut = (uint32_t)offsetof(QDesc, od_out);
constexpr uint32_t kQOutPtr = (uint32_t)offsetof(QDesc, out_ptr);
constexpr uint32_t kQCapacity = (uint32_t)offsetof(QDesc, capacity);
constexpr uint32_t kQTotalOut = (uint32_t)offsetof(QDesc, total_out);
constexpr uint32_t kQBlockCounts = (uint32_t)offsetof(QDesc, block_counts);
constexpr uint32_t kQBaseIn = (uint32_t)offsetof(QDesc, base_in);
constexpr uint32_t kQWorkFirst = (uint32_t)offsetof(QDesc, work_first);
constexpr uint32_t kQNChunks = (uint32_t)offsetof(QDesc, nchunks);
constexpr uint32_t kQGatherN = (uint32_t)offsetof(QDesc, gather_n);
constexpr uint32_t kQGatherStride = (uint32_t)offsetof(QDesc, gather_stride);
constexpr uint32_t kQGatherOff = (uint32_t)offsetof(QDesc, gather_off);
static_assert(kQOpsCount % 16 == 0 && kQOpsFull % 16 == 0, "op records are read 16 bytes at a time");
static_assert(kSlotBitmap % 16 == 0 && kSlotBlockOff % 8 == 0, "slot layout");
static_assert(kOffStageInfo % 16 == 0 && sizeof(StageInfo) == 32, "stage info is read as two 16-byte words");

/* ---- PTX wrappers ---------------------------------------------------- */

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
		: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(bar), "r"(phase)
		: "memory");
	return ok != 0;
}

/* try_wait that suspends the thread until the phase completes or about
 * hint_ns pass, so a waiting warp takes no issue slots meanwhile */
__device__ __forceinline__ bool mbar_try_wait_hint(uint32_t bar, uint32_t phase, uint32_t hint_ns)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(bar), "r"(phase), "r"(hint_ns)
		: "memory");
	return ok != 0;
}

/* global -> shared bulk copy completing on an mbarrier; dst, src and bytes
 * are multiples of 16 */
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
	asm volatile(
		"cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
		::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
		: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* Look-back status words carry epoch, flag and count in one aligned 64-bit
 * word, and no other data is published with them, so relaxed (single-copy
 * atomic) accesses suffice. */
__device__ __forceinline__ uint64_t ld_status(const uint64_t *p)
{
	uint64_t v;
	asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void st_status(uint64_t *p, uint64_t v)
{
	asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

/* the serving doorbell, with acquire semantics: descriptors and prefixes the
 * host wrote before ringing it are seen by every later load of this CTA
 * (ordered through its mbarriers), even where a load of a neighbouring entry
 * had cached their lines before the host wrote them */
__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long *p)
{
	unsigned long long v;
	asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void report(unsigned *error, unsigned code)
{
	atomicCAS(error, 0u, code);
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

/* ---- shared-memory access by 32-bit shared address --------------------- */

__device__ __forceinline__ uint32_t lds_u8(uint32_t a)
{
	uint32_t v;
	asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
	return v;
}

__device__ __forceinline__ uint32_t lds_u32(uint32_t a)
{
	uint32_t v;
	asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
	return v;
}

__device__ __forceinline__ uint64_t lds_u64(uint32_t a)
{
	uint64_t v;
	asm volatile("ld.shared.b64 %0, [%1];" : "=l"(v) : "r"(a));
	return v;
}

__device__ __forceinline__ uint4 lds_v4(uint32_t a)
{
	uint4 v;
	asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
		: "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
	return v;
}

__device__ __forceinline__ void sts_u8(uint32_t a, uint32_t v)
{
	asm volatile("st.shared.u8 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v)
{
	asm volatile("st.shared.b32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

__device__ __forceinline__ void sts_u64(uint32_t a, uint64_t v)
{
	asm volatile("st.shared.b64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}

__device__ __forceinline__ void sts_v4(uint32_t a, uint4 v)
{
	asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
		: "memory");
}

/* bounded wait for an mbarrier phase; false on timeout or when the CTA's
 * abort flag is set.  The bound is the launch's wait limit, which the CTA
 * keeps in its flag words. */
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t phase)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(bar), "r"(phase)
		: "memory");
	return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, uint32_t flags)
{
	if (mbar_try_wait(bar, phase))
		return true;
	const uint64_t limit_ns = (uint64_t)lds_u32(flags + 4 * kFWaitMs) * 1000000ull;
	const uint64_t t0 = globaltimer_ns();
	for (;;) {
#ifdef VGPU_SPIN_WAIT
		if (mbar_test(bar, phase))
			return true;
#else
		if (mbar_try_wait_hint(bar, phase, kSuspendHintNs))
			return true;
#endif
		uint32_t v;
		asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(flags + 4 * kFAbort));
		if (v)
			return false;
		if (globaltimer_ns() - t0 > limit_ns)
			return false;
	}
}

/* a failed wait: record the error (unless another warp already aborted the
 * CTA for its own reason) and make every other wait of the CTA give up */
__device__ __forceinline__ void abort_cta(const KParams &kp, uint32_t flags, unsigned code)
{
	uint32_t v;
	asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(flags + 4 * kFAbort));
	if (!v)
		report(kp.error, code);
	asm volatile("st.volatile.shared.u32 [%0], %1;" ::"r"(flags + 4 * kFAbort), "r"(1u) : "memory");
}

/* typed element access */
template <typename T>
struct SM;
template <>
struct SM<int32_t> {
	static __device__ __forceinline__ int32_t ld(uint32_t a) { return (int32_t)lds_u32(a); }
	static __device__ __forceinline__ void st(uint32_t a, int32_t v) { sts_u32(a, (uint32_t)v); }
};
template <>
struct SM<uint32_t> {
	static __device__ __forceinline__ uint32_t ld(uint32_t a) { return lds_u32(a); }
	static __device__ __forceinline__ void st(uint32_t a, uint32_t v) { sts_u32(a, v); }
};
template <>
struct SM<float> {
	static __device__ __forceinline__ float ld(uint32_t a) { return __uint_as_float(lds_u32(a)); }
	static __device__ __forceinline__ void st(uint32_t a, float v) { sts_u32(a, __float_as_uint(v)); }
};
template <>
struct SM<long long> {
	static __device__ __forceinline__ long long ld(uint32_t a) { return (long long)lds_u64(a); }
	static __device__ __forceinline__ void st(uint32_t a, long long v) { sts_u64(a, (uint64_t)v); }
};
template <>
struct SM<unsigned long long> {
	static __device__ __forceinline__ unsigned long long ld(uint32_t a) { return lds_u64(a); }
	static __device__ __forceinline__ void st(uint32_t a, unsigned long long v) { sts_u64(a, v); }
};
template <>
struct SM<double> {
	static __device__ __forceinline__ double ld(uint32_t a) { return __longlong_as_double((long long)lds_u64(a)); }
	static __device__ __forceinline__ void st(uint32_t a, double v) { sts_u64(a, (uint64_t)__double_as_longlong(v)); }
};
template <>
struct SM<signed char> {
	static __device__ __forceinline__ signed char ld(uint32_t a) { return (signed char)lds_u8(a); }
	static __device__ __forceinline__ void st(uint32_t a, signed char v) { sts_u8(a, (uint32_t)(unsigned char)v); }
};
template <>
struct SM<unsigned char> {
	static __device__ __forceinline__ unsigned char ld(uint32_t a) { return (unsigned char)lds_u8(a); }
	static __device__ __forceinline__ void st(uint32_t a, unsigned char v) { sts_u8(a, v); }
};

/* ---- operands ----------------------------------------------------------- */

/* the bases of one block's operands: the stage holding its tile (and the
 * block's first tile row), the warp's vector areas and the chunk slot */
struct Bases {
	uint32_t stage;
	uint32_t blk_row0;
	uint32_t rowv;
	uint32_t selv;
	uint32_t slot;
};

/* an operand resolved for one block: element i at addr + i * step (step 0
 * for a scalar), indexed by selection entry instead of block row when sel */
struct Opnd {
	uint32_t addr;
	uint32_t step;
	bool sel;
};

template <int SIZE>
__device__ __forceinline__ Opnd opnd(uint32_t od, const Bases &b)
{
	const uint32_t kind = od >> 30;
	const uint32_t off = od & OD_OFFSET;
	Opnd o;
	o.addr = off + (kind == (OD_STAGE >> 30) ? b.stage + b.blk_row0 * (uint32_t)SIZE
		: kind == (OD_ROWVEC >> 30) ? b.rowv
		: kind == (OD_SELVEC >> 30) ? b.selv : b.slot);
	o.step = kind == (OD_SCALAR >> 30) ? 0u : (uint32_t)SIZE;
	o.sel = kind == (OD_SELVEC >> 30);
	return o;
}

/* ---- op semantics (src/vm/virginia.c:48-194, :598-680) ------------------ */

template <typename T, int OP>
__device__ __forceinline__ bool cmp_eval(T a, T b)
{
	if (OP == CO_LE) return a <= b;
	if (OP == CO_LT) return a < b;
	if (OP == CO_GE) return a >= b;
	if (OP == CO_GT) return a > b;
	if (OP == CO_EQ) return a == b;
	if (OP == CO_NEQ) return a != b;
	if (OP == CO_AND) return (a != T(0)) && (b != T(0));
	return (a != T(0)) || (b != T(0));
}

template <typename T, int OP>
struct Math;

/* NaN results as x86 SSE produces them (the CPU VM's arithmetic): a NaN
 * operand propagates quieted, the first operand's first; an invalid
 * operation on non-NaN operands (0/0, inf-inf, 0*inf) gives the "default
 * NaN" with the sign bit set.  The GPU's own NaN results are canonical
 * positive NaNs, so only the NaN case is patched. */
__device__ __forceinline__ float x86_nan(float r, float a, float b)
{
	if (!isnan(r))
		return r;
	if (isnan(a))
		return __int_as_float(__float_as_int(a) | 0x00400000);
	if (isnan(b))
		return __int_as_float(__float_as_int(b) | 0x00400000);
	return __int_as_float((int)0xffc00000u);
}

__device__ __forceinline__ double x86_nan(double r, double a, double b)
{
	if (!isnan(r))
		return r;
	if (isnan(a))
		return __longlong_as_double(__double_as_longlong(a) | 0x0008000000000000ll);
	if (isnan(b))
		return __longlong_as_double(__double_as_longlong(b) | 0x0008000000000000ll);
	return __longlong_as_double((long long)0xfff8000000000000ull);
}

template <int OP>
struct Math<float, OP> {
	static __device__ __forceinline__ float eval(float a, float b)
	{
		float r;
		if (OP == MO_ADD) r = __fadd_rn(a, b);
		else if (OP == MO_SUB) r = __fsub_rn(a, b);
		else if (OP == MO_MUL) r = __fmul_rn(a, b);
		else r = __fdiv_rn(a, b);
		return x86_nan(r, a, b);
	}
};

template <int OP>
struct Math<double, OP> {
	static __device__ __forceinline__ double eval(double a, double b)
	{
		double r;
		if (OP == MO_ADD) r = __dadd_rn(a, b);
		else if (OP == MO_SUB) r = __dsub_rn(a, b);
		else if (OP == MO_MUL) r = __dmul_rn(a, b);
		else r = __ddiv_rn(a, b);
		return x86_nan(r, a, b);
	}
};

/* integer division by zero traps in the CPU VM (SIGFPE); here it yields 0 */
template <int OP>
struct Math<int32_t, OP> {
	static __device__ __forceinline__ int32_t eval(int32_t a, int32_t b)
	{
		if (OP == MO_ADD) return (int32_t)((uint32_t)a + (uint32_t)b);
		if (OP == MO_SUB) return (int32_t)((uint32_t)a - (uint32_t)b);
		if (OP == MO_MUL) return (int32_t)((uint32_t)a * (uint32_t)b);
		if (b == 0) return 0;
		if (a == INT_MIN && b == -1) return INT_MIN;
		return a / b;
	}
};

template <int OP>
struct Math<long long, OP> {
	static __device__ __forceinline__ long long eval(long long a, long long b)
	{
		if (OP == MO_ADD) return (long long)((unsigned long long)a + (unsigned long long)b);
		if (OP == MO_SUB) return (long long)((unsigned long long)a - (unsigned long long)b);
		if (OP == MO_MUL) return (long long)((unsigned long long)a * (unsigned long long)b);
		if (b == 0) return 0;
		if (a == LLONG_MIN && b == -1) return LLONG_MIN;
		return a / b;
	}
};

/* char arithmetic is done in int and narrowed, as C does on the CPU */
template <int OP>
struct Math<signed char, OP> {
	static __device__ __forceinline__ signed char eval(signed char a, signed char b)
	{
		int x = a, y = b, z;
		if (OP == MO_ADD) z = x + y;
		else if (OP == MO_SUB) z = x - y;
		else if (OP == MO_MUL) z = x * y;
		else z = (y == 0) ? 0 : x / y;
		return (signed char)z;
	}
};

/* operand type and operator tests on a record head */
__device__ __forceinline__ bool h_type(uint32_t h, int t) { return (h >> (OT_SHIFT + t)) & 1u; }
__device__ __forceinline__ bool h_op(uint32_t h, int o) { return (h >> (OO_SHIFT + o)) & 1u; }

/* ---- filter: every row of a group, row state in bit masks ---------------
 * A count group is kCountGroup blocks; lane l holds its rows l, l + 32, ...,
 * as bits 0, 1, ... of its row masks, so a ballot of bit u is the group's
 * validity word u. */

struct RowState {
	uint32_t valid;
	uint32_t active;
	uint32_t pend[kMaxSlots];
};

/* rows in `jumped` leave the active set, park in the op's target slot and,
 * for a jump with p4 == 0, stop being valid (src/vm/virginia.c:59-63).  The
 * code generator's programs park rows in the first two slots. */
__device__ __forceinline__ void take_jump(RowState &st, uint32_t head, uint32_t jumped)
{
	st.active &= ~jumped;
	if (!(head & OPH_VJUMP))
		st.valid &= ~jumped;
	const uint32_t slot = (head >> OPH_SLOT_SHIFT) & 7u;
	if (slot == 0) {
		st.pend[0] |= jumped;
	} else if (slot == 1) {
		st.pend[1] |= jumped;
	} else {
#pragma unroll
		for (int s = 2; s < kMaxSlots; s++)
			if (slot == (uint32_t)s)
				st.pend[s] |= jumped;
	}
}

/* the operand's elements for this lane's U rows of the group */
template <typename T, int U>
__device__ __forceinline__ void load_rows(const Opnd &o, int lane, T (&v)[U])
{
	if (o.step == 0) {
		const T x = SM<T>::ld(o.addr);
#pragma unroll
		for (int u = 0; u < U; u++)
			v[u] = x;
	} else {
#pragma unroll
		for (int u = 0; u < U; u++)
			v[u] = SM<T>::ld(o.addr + (uint32_t)(32 * u + lane) * (uint32_t)sizeof(T));
	}
}

/* store the rows whose bit is set in `mask` */
template <typename T, int U>
__device__ __forceinline__ void store_rows(uint32_t addr, int lane, const T (&v)[U], uint32_t mask)
{
#pragma unroll
	for (int u = 0; u < U; u++)
		if ((mask >> u) & 1u)
			SM<T>::st(addr + (uint32_t)(32 * u + lane) * (uint32_t)sizeof(T), v[u]);
}

/* an operand seen from row 32 h0 + lane onward */
__device__ __forceinline__ Opnd shifted(Opnd o, int h0)
{
	o.addr += (uint32_t)(32 * h0) * o.step;
	return o;
}

/* The op handlers of the 4-byte types run inline, fully unrolled over the
 * lane's U rows; those of the 8-byte and char types run out of line, over
 * chunks of four rows, with every argument passed by value, so that the
 * kernel's hot code (the 4-byte paths) stays small enough for the
 * instruction cache.  A handler computes a row mask (compares and Not) or
 * writes a register vector (arithmetic and copies); the caller applies the
 * mask to the row state. */

/* row mask of a compare (OP) or, for OP = -1, of Not (the value is zero) */
template <typename T, int OP>
__device__ __forceinline__ bool test_eval(T x, T y)
{
	if constexpr (OP < 0)
		return x == T(0);
	else
		return cmp_eval<T, OP>(x, y);
}

template <typename T, int OP, int U>
__device__ __forceinline__ uint32_t bits_rows(const uint4 &rec, const Bases &b, int lane)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b);
	T x[U], y[U];
	load_rows<T, U>(oa, lane, x);
	if constexpr (OP >= 0)
		load_rows<T, U>(ob, lane, y);
	uint32_t acc[4] = {0u, 0u, 0u, 0u};  /* four independent chains */
#pragma unroll
	for (int u = 0; u < U; u++)
		acc[u & 3] |= (uint32_t)test_eval<T, OP>(x[u], OP >= 0 ? y[u] : x[u]) << u;
	return (acc[0] | acc[1]) | (acc[2] | acc[3]);
}

/* the same over chunks of four rows, a loop the compiler keeps rolled */
template <typename T, int OP, int U>
__device__ __forceinline__ uint32_t bits_chunked(const uint4 &rec, const Bases &b, int lane)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b);
	uint32_t bits = 0;
#pragma unroll 1
	for (int c = 0; c < U / 4; c++) {
		T x[4], y[4];
		load_rows<T, 4>(shifted(oa, 4 * c), lane, x);
		if constexpr (OP >= 0)
			load_rows<T, 4>(shifted(ob, 4 * c), lane, y);
#pragma unroll
		for (int u = 0; u < 4; u++)
			bits |= (uint32_t)test_eval<T, OP>(x[u], OP >= 0 ? y[u] : x[u]) << (4 * c + u);
	}
	return bits;
}

template <typename T, int U, bool CHUNKED>
__device__ __forceinline__ uint32_t bits_any(const uint4 &rec, const Bases &b, int lane)
{
	const uint32_t h = rec.x;
#define VGPU_BITS(OP) (CHUNKED ? bits_chunked<T, OP, U>(rec, b, lane) : bits_rows<T, OP, U>(rec, b, lane))
	if (h & OK_NOT) return VGPU_BITS(-1);
	if (h_op(h, CO_LT)) return VGPU_BITS(CO_LT);
	if (h_op(h, CO_GT)) return VGPU_BITS(CO_GT);
	if (h_op(h, CO_LE)) return VGPU_BITS(CO_LE);
	if (h_op(h, CO_GE)) return VGPU_BITS(CO_GE);
	if (h_op(h, CO_EQ)) return VGPU_BITS(CO_EQ);
	if (h_op(h, CO_NEQ)) return VGPU_BITS(CO_NEQ);
	if (h_op(h, CO_AND)) return VGPU_BITS(CO_AND);
	return VGPU_BITS(CO_OR);
#undef VGPU_BITS
}

/* arithmetic (OP) or, for OP = -1, a copy of operand a into a register
 * vector, for the rows in `mask` */
template <typename T, int OP, int U>
__device__ __forceinline__ void vec_rows(const uint4 &rec, const Bases &b, int lane, uint32_t mask)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b), od = opnd<sizeof(T)>(rec.w, b);
	T x[U], y[U];
	load_rows<T, U>(oa, lane, x);
	if constexpr (OP >= 0) {
		load_rows<T, U>(ob, lane, y);
#pragma unroll
		for (int u = 0; u < U; u++)
			x[u] = Math<T, OP>::eval(x[u], y[u]);
	}
	store_rows<T, U>(od.addr, lane, x, mask);
}

template <typename T, int OP, int U>
__device__ __forceinline__ void vec_chunked(const uint4 &rec, const Bases &b, int lane, uint32_t mask)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b), od = opnd<sizeof(T)>(rec.w, b);
#pragma unroll 1
	for (int c = 0; c < U / 4; c++) {
		T x[4], y[4];
		load_rows<T, 4>(shifted(oa, 4 * c), lane, x);
		if constexpr (OP >= 0) {
			load_rows<T, 4>(shifted(ob, 4 * c), lane, y);
#pragma unroll
			for (int u = 0; u < 4; u++)
				x[u] = Math<T, OP>::eval(x[u], y[u]);
		}
		store_rows<T, 4>(shifted(od, 4 * c).addr, lane, x, mask >> (4 * c));
	}
}

template <typename T, int U, bool CHUNKED>
__device__ __forceinline__ void vec_any(const uint4 &rec, const Bases &b, int lane, uint32_t mask)
{
	const uint32_t h = rec.x;
#define VGPU_VEC(OP) { if (CHUNKED) vec_chunked<T, OP, U>(rec, b, lane, mask); else vec_rows<T, OP, U>(rec, b, lane, mask); return; }
	if (h & OK_COPY) VGPU_VEC(-1);
	if (h_op(h, MO_ADD)) VGPU_VEC(MO_ADD);
	if (h_op(h, MO_SUB)) VGPU_VEC(MO_SUB);
	if (h_op(h, MO_MUL)) VGPU_VEC(MO_MUL);
	VGPU_VEC(MO_DIV);
#undef VGPU_VEC
}

/* compares and Not over 8-byte and char values, out of line */
template <int U>
__device__ __noinline__ uint32_t bits_rare(uint4 rec, Bases b, int lane)
{
	const uint32_t h = rec.x;
	if (h_type(h, VT_DOUBLE)) return bits_any<double, U, true>(rec, b, lane);
	if (h_type(h, VT_INT64)) return bits_any<long long, U, true>(rec, b, lane);
	return bits_any<signed char, U, true>(rec, b, lane);
}

/* arithmetic and copies over 8-byte and char values, out of line */
template <int U>
__device__ __noinline__ void vec_rare(uint4 rec, Bases b, int lane, uint32_t mask)
{
	const uint32_t h = rec.x;
	if (h_type(h, VT_DOUBLE)) vec_any<double, U, true>(rec, b, lane, mask);
	else if (h_type(h, VT_INT64)) vec_any<long long, U, true>(rec, b, lane, mask);
	else if (h & OK_COPY) {
		if (h_type(h, VT_CHAR)) vec_chunked<unsigned char, -1, U>(rec, b, lane, mask);
	} else vec_any<signed char, U, true>(rec, b, lane, mask);
}

#ifndef VGPU_HOT_CHUNKED
#define VGPU_HOT_CHUNKED 0
#endif
constexpr bool kHotChunked = VGPU_HOT_CHUNKED != 0;

/* one filter op: kind, then type, then operator, each by bit tests */
template <int U>
__device__ __forceinline__ void filter_op(const uint4 &rec, const Bases &b, int lane, RowState &st)
{
	const uint32_t h = rec.x;
	const uint32_t join = h >> OPH_JOIN_SHIFT;
	if (join) {
#pragma unroll
		for (int s = 0; s < kMaxSlots; s++)
			if ((join >> s) & 1u) {
				st.active |= st.pend[s];
				st.pend[s] = 0;
			}
	}
	if (h & (OK_CMP | OK_NOT)) {
		uint32_t bits;
		if (h_type(h, VT_FLOAT)) bits = bits_any<float, U, kHotChunked>(rec, b, lane);
		else if (h_type(h, VT_INT)) bits = bits_any<int32_t, U, kHotChunked>(rec, b, lane);
		else bits = bits_rare<U>(rec, b, lane);
		take_jump(st, h, st.active & bits);
	} else if (h & OK_INVALID) {
		st.valid &= ~st.active;
	} else if (h & (OK_MATH | OK_COPY)) {
		/* arithmetic writes the active rows (every row if this is the
		 * register's single definition); a Column/Rowid copy writes every
		 * row (the CPU copies the whole block, src/vm/virginia.c:448) */
		const uint32_t mask = (h & OK_COPY) || (h & OPH_SINGLE_DEF) ? 0xffffffffu : st.active;
		if (h & OK_COPY) {
			if (h_type(h, VT_INT) || h_type(h, VT_FLOAT)) {
				if (kHotChunked) vec_chunked<uint32_t, -1, U>(rec, b, lane, mask);
				else vec_rows<uint32_t, -1, U>(rec, b, lane, mask);
			} else {
				vec_rare<U>(rec, b, lane, mask);
			}
		} else if (h_type(h, VT_FLOAT)) {
			vec_any<float, U, kHotChunked>(rec, b, lane, mask);
		} else if (h_type(h, VT_INT)) {
			vec_any<int32_t, U, kHotChunked>(rec, b, lane, mask);
		} else {
			vec_rare<U>(rec, b, lane, mask);
		}
	} else if (h & OK_SETCONST) {
		/* Integer/Float into a register vector: active rows only */
		if (kHotChunked) vec_chunked<uint32_t, -1, U>(rec, b, lane, st.active);
		else vec_rows<uint32_t, -1, U>(rec, b, lane, st.active);
	}
}

/* the filter ops [0, nf) of a record array over one group; returns the
 * lane's validity bits (rows at or past nrows start invalid).  Out of line
 * (one copy for the count phase and the re-filtering full phase), its
 * arguments by value. */
template <int U>
__device__ __noinline__ uint32_t run_filter(uint32_t ops, uint32_t nf, Bases b, uint32_t nrows, int lane)
{
	RowState st;
	st.valid = 0;
#pragma unroll
	for (int u = 0; u < U; u++)
		if ((uint32_t)(32 * u + lane) < nrows)
			st.valid |= 1u << u;
	st.active = st.valid;
#pragma unroll
	for (int s = 0; s < kMaxSlots; s++)
		st.pend[s] = 0;
	uint4 rec = lds_v4(ops);
	for (uint32_t k = 0; k < nf; k++) {
		const uint4 cur = rec;
		/* the next record's load overlaps this op */
		rec = lds_v4(ops + 16u * min(k + 1u, (uint32_t)kMaxOps - 1u));
		filter_op<U>(cur, b, lane, st);
	}
	return st.valid;
}

/* ---- projection: the batches of a unit, op by op -------------------------
 * A unit is kUnitBatches batches of 32 kBatchE selected rows; entry i of
 * batch s of a lane is unit entry 32 kBatchE s + 32 i + lane, at row
 * row[s][i] of the staged tile (or the warp's gather area).  Each op runs
 * over every batch of the unit before the next op, so an op's record is
 * read and dispatched once per unit.  Register vectors indexed by selection
 * entry use the unit entry. */

struct UnitRows {
	uint32_t row[kUnitBatches][kBatchE];
	uint32_t act[kUnitBatches];  /* entries that exist */
	uint32_t nb;                 /* batches in use (1 or kUnitBatches) */
};

template <typename T, int OP, int NB>
__device__ __forceinline__ void p_math(const uint4 &rec, const Bases &b, const UnitRows &u, int lane)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b), od = opnd<sizeof(T)>(rec.w, b);
	T x[NB][kBatchE], y[NB][kBatchE];
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++) {
			const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
			x[s][i] = SM<T>::ld(oa.addr + (oa.sel ? e : u.row[s][i]) * oa.step);
			y[s][i] = SM<T>::ld(ob.addr + (ob.sel ? e : u.row[s][i]) * ob.step);
		}
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++)
			if ((u.act[s] >> i) & 1u) {
				const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
				SM<T>::st(od.addr + (od.sel ? e : u.row[s][i]) * od.step, Math<T, OP>::eval(x[s][i], y[s][i]));
			}
}

template <typename T, int NB>
__device__ __forceinline__ void p_copy(const uint4 &rec, const Bases &b, const UnitRows &u, int lane)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), od = opnd<sizeof(T)>(rec.w, b);
	T x[NB][kBatchE];
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++) {
			const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
			x[s][i] = SM<T>::ld(oa.addr + (oa.sel ? e : u.row[s][i]) * oa.step);
		}
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++)
			if ((u.act[s] >> i) & 1u) {
				const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
				SM<T>::st(od.addr + (od.sel ? e : u.row[s][i]) * od.step, x[s][i]);
			}
}

template <typename T, int NB>
__device__ __forceinline__ void p_math_any(const uint4 &rec, const Bases &b, const UnitRows &u, int lane)
{
	const uint32_t h = rec.x;
	if (h_op(h, MO_ADD)) p_math<T, MO_ADD, NB>(rec, b, u, lane);
	else if (h_op(h, MO_SUB)) p_math<T, MO_SUB, NB>(rec, b, u, lane);
	else if (h_op(h, MO_MUL)) p_math<T, MO_MUL, NB>(rec, b, u, lane);
	else p_math<T, MO_DIV, NB>(rec, b, u, lane);
}

/* one batch of a projection op over 8-byte and char values, out of line,
 * arguments by value (rows: the batch's four rows of this lane; e0: the
 * batch's first unit entry) */
template <typename T, int OP>
__device__ __forceinline__ void p_math1(const uint4 &rec, const Bases &b, const uint32_t (&row)[kBatchE], uint32_t act,
	uint32_t e0, int lane)
{
	const Opnd oa = opnd<sizeof(T)>(rec.y, b), ob = opnd<sizeof(T)>(rec.z, b), od = opnd<sizeof(T)>(rec.w, b);
#pragma unroll
	for (int i = 0; i < kBatchE; i++) {
		const uint32_t e = e0 + 32u * i + (uint32_t)lane;
		const T x = SM<T>::ld(oa.addr + (oa.sel ? e : row[i]) * oa.step);
		if constexpr (OP < 0) {
			if ((act >> i) & 1u)
				SM<T>::st(od.addr + (od.sel ? e : row[i]) * od.step, x);
		} else {
			const T y = SM<T>::ld(ob.addr + (ob.sel ? e : row[i]) * ob.step);
			if ((act >> i) & 1u)
				SM<T>::st(od.addr + (od.sel ? e : row[i]) * od.step, Math<T, OP>::eval(x, y));
		}
	}
}

template <typename T>
__device__ __forceinline__ void p_math1_any(const uint4 &rec, const Bases &b, const uint32_t (&row)[kBatchE],
	uint32_t act, uint32_t e0, int lane)
{
	const uint32_t h = rec.x;
	if (h_op(h, MO_ADD)) p_math1<T, MO_ADD>(rec, b, row, act, e0, lane);
	else if (h_op(h, MO_SUB)) p_math1<T, MO_SUB>(rec, b, row, act, e0, lane);
	else if (h_op(h, MO_MUL)) p_math1<T, MO_MUL>(rec, b, row, act, e0, lane);
	else p_math1<T, MO_DIV>(rec, b, row, act, e0, lane);
}

__device__ __noinline__ void project_rare(uint4 rec, Bases b, uint4 rows, uint32_t act, uint32_t e0, int lane)
{
	const uint32_t row[kBatchE] = {rows.x, rows.y, rows.z, rows.w};
	const uint32_t h = rec.x;
	if (h & OK_MATH) {
		if (h_type(h, VT_DOUBLE)) p_math1_any<double>(rec, b, row, act, e0, lane);
		else if (h_type(h, VT_INT64)) p_math1_any<long long>(rec, b, row, act, e0, lane);
		else p_math1_any<signed char>(rec, b, row, act, e0, lane);
	} else if (h & OK_COPY) {
		if (h_type(h, VT_CHAR)) p_math1<unsigned char, -1>(rec, b, row, act, e0, lane);
		else p_math1<unsigned long long, -1>(rec, b, row, act, e0, lane);
	}
}

/* one projection op over the unit: arithmetic, or a copy (every listed row
 * is active here, so constants and columns are copies) */
template <int NB>
__device__ __forceinline__ void project_op(const uint4 &rec, const Bases &b, const UnitRows &u, int lane)
{
	static_assert(kBatchE == 4, "project_rare passes a batch's rows as a uint4");
	const uint32_t h = rec.x;
	if (h & OK_SETCONST) {
		p_copy<uint32_t, NB>(rec, b, u, lane);
	} else if (!(h_type(h, VT_FLOAT) || h_type(h, VT_INT))) {
#pragma unroll
		for (int s = 0; s < NB; s++)
			project_rare(rec, b, make_uint4(u.row[s][0], u.row[s][1], u.row[s][2], u.row[s][3]), u.act[s],
				kBatchRows * s, lane);
	} else if (h & OK_MATH) {
		if (h_type(h, VT_FLOAT)) p_math_any<float, NB>(rec, b, u, lane);
		else p_math_any<int32_t, NB>(rec, b, u, lane);
	} else if (h & OK_COPY) {
		p_copy<uint32_t, NB>(rec, b, u, lane);
	}
}

/* one result column of the unit: entries whose bit is set in in[s] are
 * stored at pos0 + their unit entry */
template <typename T, int NB>
__device__ __forceinline__ void p_store(uint32_t od, const Bases &b, const UnitRows &u, const uint32_t (&in)[kUnitBatches],
	T *out, uint64_t pos0, int lane)
{
	const Opnd o = opnd<sizeof(T)>(od, b);
	T v[NB][kBatchE];
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++) {
			const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
			v[s][i] = SM<T>::ld(o.addr + (o.sel ? e : u.row[s][i]) * o.step);
		}
#pragma unroll
	for (int s = 0; s < NB; s++)
#pragma unroll
		for (int i = 0; i < kBatchE; i++)
			if ((in[s] >> i) & 1u)
				out[pos0 + (uint64_t)(kBatchRows * s + 32u * i + (uint32_t)lane)] = v[s][i];
}

/* one batch of a result column of 8-byte or char values, out of line, by value */
__device__ __noinline__ void p_store_rare(uint32_t od, Bases b, uint4 rows, uint32_t in, void *out, uint64_t pos0,
	uint32_t e0, uint32_t stride, int lane)
{
	const uint32_t row[kBatchE] = {rows.x, rows.y, rows.z, rows.w};
	const Opnd o = stride == 8 ? opnd<8>(od, b) : opnd<1>(od, b);
#pragma unroll
	for (int i = 0; i < kBatchE; i++) {
		const uint32_t e = e0 + 32u * i + (uint32_t)lane;
		const uint32_t a = o.addr + (o.sel ? e : row[i]) * o.step;
		if ((in >> i) & 1u) {
			if (stride == 8)
				static_cast<unsigned long long *>(out)[pos0 + e] = SM<unsigned long long>::ld(a);
			else
				static_cast<unsigned char *>(out)[pos0 + e] = SM<unsigned char>::ld(a);
		}
	}
}

/* ---- groups ------------------------------------------------------------- */

/* count phase: the filter over one group of up to kCountGroup blocks (its
 * first block is chunk block blk, nblk of them exist); its validity words
 * go to the chunk's bitmap and a count per block to the block counts */
__device__ __forceinline__ void count_group(const Bases &b, uint32_t blk, uint32_t nblk, uint32_t nrows, int lane)
{
	constexpr int U = kCountGroup * kBlockRows / 32;
	const uint32_t valid = run_filter<U>(b.slot + kQOpsCount, lds_u32(b.slot + kQNFilter), b, nrows, lane);
	uint32_t w[U];
#pragma unroll
	for (int u = 0; u < U; u++)
		w[u] = __ballot_sync(0xffffffffu, (valid >> u) & 1u);
	if (lane == 0) {
		const uint32_t bm = b.slot + kSlotBitmap + 32u * blk;
#pragma unroll
		for (int k = 0; k < kCountGroup; k++)
			if ((uint32_t)k < nblk) {
				sts_v4(bm + 32 * k, make_uint4(w[8 * k], w[8 * k + 1], w[8 * k + 2], w[8 * k + 3]));
				sts_v4(bm + 32 * k + 16, make_uint4(w[8 * k + 4], w[8 * k + 5], w[8 * k + 6], w[8 * k + 7]));
				uint32_t n = 0;
#pragma unroll
				for (int u = 0; u < 8; u++)
					n += __popc(w[8 * k + u]);
				sts_u32(b.slot + kSlotBlockCnt + 4u * (blk + k), n);
			}
	}
}

/* one value of a gathered column, read through the non-coherent path (the
 * tables do not change while a launch runs) */
__device__ __forceinline__ uint64_t ldg_val(const unsigned char *p, uint32_t stride)
{
	if (stride == 4) {
		uint32_t v;
		asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(v) : "l"(p));
		return v;
	}
	if (stride == 8) {
		uint64_t v;
		asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(p));
		return v;
	}
	uint32_t v;
	asm volatile("ld.global.nc.u8 %0, [%1];" : "=r"(v) : "l"(p));
	return v;
}

/* FM_GATHER: one batch's selected rows of every gathered column, from
 * device memory into the warp's gather area (unit entry e0 + 32 i + lane at
 * row grow[i] of the chunk); four columns' loads in flight at a time */
__device__ __forceinline__ void gather_batch(const Bases &b, const uint32_t (&grow)[kBatchE], uint32_t e0, int lane)
{
	const uint32_t n = lds_u32(b.slot + kQGatherN);
	for (uint32_t c0 = 0; c0 < n; c0 += 4) {
		uint64_t v[4][kBatchE];
		uint32_t st[4];
#pragma unroll
		for (int cc = 0; cc < 4; cc++) {
			st[cc] = c0 + cc < n ? lds_u8(b.slot + kQGatherStride + c0 + cc) : 0u;
			if (st[cc]) {
				const unsigned char *col =
					reinterpret_cast<const unsigned char *>(lds_u64(b.slot + kSlotColPtr + 8 * (c0 + cc)));
#pragma unroll
				for (int i = 0; i < kBatchE; i++)
					v[cc][i] = ldg_val(col + (size_t)grow[i] * st[cc], st[cc]);
			}
		}
#pragma unroll
		for (int cc = 0; cc < 4; cc++)
			if (st[cc]) {
				const uint32_t dst = b.stage + lds_u32(b.slot + kQGatherOff + 4 * (c0 + cc));
#pragma unroll
				for (int i = 0; i < kBatchE; i++) {
					const uint32_t a = dst + (e0 + (uint32_t)(32 * i + lane)) * st[cc];
					if (st[cc] == 4)
						sts_u32(a, (uint32_t)v[cc][i]);
					else if (st[cc] == 8)
						sts_u64(a, v[cc][i]);
					else
						sts_u8(a, (uint32_t)v[cc][i]);
				}
			}
	}
}

/* the projection and stores of a unit of NB batches (see UnitRows);
 * entries in in[s] fit the output and are stored at pos0 + their unit entry */
template <int NB>
__device__ __forceinline__ void unit_out_n(const Bases &b, const UnitRows &u, const uint32_t (&in)[kUnitBatches],
	uint64_t pos0, int lane)
{
	const uint32_t ops = b.slot + kQOpsFull;
	const uint32_t nf = lds_u32(b.slot + kQNFilter);
	const uint32_t nu = lds_u32(b.slot + kQNUops) - 1u;
	const uint32_t nout = lds_u32(b.slot + kQNOut);
	for (uint32_t k = nf; k < nu; k++)
		project_op<NB>(lds_v4(ops + 16u * k), b, u, lane);
	for (uint32_t j = 0; j < nout; j++) {
		const uint32_t od = lds_u32(b.slot + kQOdOut + 4 * j);
		void *out = reinterpret_cast<void *>(lds_u64(b.slot + kQOutPtr + 8 * j));
		const uint32_t stride = lds_u8(b.slot + kQOutStride + j);
		if (stride == 4) {
			p_store<uint32_t, NB>(od, b, u, in, static_cast<uint32_t *>(out), pos0, lane);
		} else {
#pragma unroll
			for (int s2 = 0; s2 < NB; s2++)
				p_store_rare(od, b, make_uint4(u.row[s2][0], u.row[s2][1], u.row[s2][2], u.row[s2][3]), in[s2], out,
					pos0, kBatchRows * s2, stride, lane);
		}
	}
}

__device__ __forceinline__ void unit_out(const Bases &b, const UnitRows &u, const uint32_t (&in)[kUnitBatches],
	uint64_t pos0, int lane)
{
	if (u.nb == 1)
		unit_out_n<1>(b, u, in, pos0, lane);
	else
		unit_out_n<kUnitBatches>(b, u, in, pos0, lane);
}

/* a unit's rows from its selection list (list entry e: the row of unit
 * entry e), the first cnt existing (at most kBatchRows nb); in[s]: those
 * below the output capacity */
__device__ __forceinline__ void unit_rows(uint32_t list, uint32_t cnt, uint32_t nb, uint64_t pos0, uint64_t cap,
	UnitRows &u, uint32_t (&in)[kUnitBatches], int lane)
{
	u.nb = nb;
#pragma unroll
	for (int s = 0; s < (int)kUnitBatches; s++) {
		u.act[s] = 0;
		in[s] = 0;
#pragma unroll
		for (int i = 0; i < kBatchE; i++) {
			const uint32_t e = kBatchRows * s + 32u * i + (uint32_t)lane;
			const bool a = e < cnt;
			u.row[s][i] = 0;
			if (a) {
				uint16_t r;
				asm volatile("ld.shared.u16 %0, [%1];" : "=h"(r) : "r"(list + 2 * e));
				u.row[s][i] = r;
			}
			u.act[s] |= (a ? 1u : 0u) << i;
			if (a && pos0 + e < cap)
				in[s] |= 1u << i;
		}
	}
}

/* FM_REFILTER full phase: one group's selected rows (up to kCountGroup
 * blocks from chunk block blk, nrows rows), in row order, with the filter
 * run again for the register vectors the results read; b.stage is the
 * staged tile and b.blk_row0 the group's first tile row.  Returns false on
 * an output overflow. */
__device__ __forceinline__ bool refilter_group(const Bases &b, uint32_t list, uint32_t blk, uint32_t nrows, uint32_t ub,
	int lane)
{
	/* lane l holds validity word l of the group (32 rows) */
	const uint32_t nw = (nrows + 31) / 32;
	const uint32_t word = (uint32_t)lane < nw ? lds_u32(b.slot + kSlotBitmap + 32u * blk + 4u * lane) : 0u;
	const uint32_t cnt = __popc(word);
	uint32_t incl = cnt;
#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
		if (lane >= d)
			incl += v;
	}
	const uint32_t n = __shfl_sync(0xffffffffu, incl, 31);
	if (n == 0)
		return true;
	(void)run_filter<kCountGroup * kBlockRows / 32>(b.slot + kQOpsFull, lds_u32(b.slot + kQNFilter), b, nrows,
		lane);  /* the filter's register vectors */
	/* the selection list: entry i is the group row of the group's i-th
	 * selected row; each lane lists its own word's rows */
	{
		uint32_t pos = incl - cnt, w = word;
		while (w) {
			const uint32_t bit = __ffs(w) - 1;
			asm volatile("st.shared.u16 [%0], %1;" ::"r"(list + 2 * pos), "h"((uint16_t)(32 * lane + bit)) : "memory");
			pos++;
			w &= w - 1;
		}
	}
	__syncwarp();
	const uint64_t off = lds_u64(b.slot + kSlotBlockOff + 8u * blk);
	const uint64_t cap = lds_u64(b.slot + kQCapacity);
	bool ok = true;
	for (uint32_t base = 0, step = 0; base < n; base += step) {
		const uint32_t nb = ub > 1 && n - base >= kUnitE ? kUnitBatches : 1u;
		step = kBatchRows * nb;
		UnitRows u;
		uint32_t in[kUnitBatches];
		unit_rows(list + 2 * base, min(n - base, step), nb, off + base, cap, u, in, lane);
#pragma unroll
		for (int s2 = 0; s2 < (int)kUnitBatches; s2++)
			ok = ok && u.act[s2] == in[s2];
		unit_out(b, u, in, off + base, lane);
	}
	__syncwarp();
	return ok;
}

/* FM_DENSE: one result column over a group's rows held by lanes (row
 * 32 u + lane in element u; `mine`: the group's validity word `lane`, so
 * word u is lane u's); valid rows go to pos0 + their rank among the group's
 * valid rows (the valid rows of earlier words and of lower lanes in word u);
 * false if a row falls past cap */
template <typename T>
__device__ __forceinline__ bool dense_store(uint32_t od, const Bases &b, uint32_t mine, uint32_t vb, T *out,
	uint64_t pos0, uint64_t cap, int lane)
{
	constexpr int U = kCountGroup * kBlockRows / 32;
	const Opnd o = opnd<sizeof(T)>(od, b);
	T v[U];
	load_rows<T, U>(o, lane, v);
	const uint32_t below = (1u << lane) - 1u;
	uint32_t base = 0;
	bool ok = true;
#pragma unroll
	for (int u = 0; u < U; u++) {
		const uint32_t wu = __shfl_sync(0xffffffffu, mine, u);
		if ((vb >> u) & 1u) {
			const uint64_t pos = pos0 + base + __popc(wu & below);
			if (pos < cap)
				out[pos] = v[u];
			else
				ok = false;
		}
		base += __popc(wu);
	}
	return ok;
}

/* 8-byte and char result columns of a dense group, out of line, by value */
__device__ __noinline__ bool dense_store_rare(uint32_t od, Bases b, uint32_t mine, uint32_t vb, void *out,
	uint64_t pos0, uint64_t cap, uint32_t stride, int lane)
{
	if (stride == 8)
		return dense_store<unsigned long long>(od, b, mine, vb, static_cast<unsigned long long *>(out), pos0, cap, lane);
	return dense_store<unsigned char>(od, b, mine, vb, static_cast<unsigned char *>(out), pos0, cap, lane);
}

/* FM_DENSE full phase: one group (up to kCountGroup blocks from chunk
 * block blk, nrows rows) with the projection run over every valid row as
 * vector ops (b.stage the staged tile, b.blk_row0 the group's first tile
 * row), then each result column's valid rows stored in row order.  Returns
 * false on an output overflow. */
__device__ __forceinline__ bool dense_group(const Bases &b, uint32_t blk, uint32_t nrows, int lane)
{
	constexpr int U = kCountGroup * kBlockRows / 32;
	const uint32_t nw = (nrows + 31) / 32;
	const uint32_t mine = (uint32_t)lane < nw ? lds_u32(b.slot + kSlotBitmap + 32u * blk + 4u * lane) : 0u;
	uint32_t vb = 0;
#pragma unroll
	for (int u = 0; u < U; u++)
		vb |= ((__shfl_sync(0xffffffffu, mine, u) >> lane) & 1u) << u;
	if (!__any_sync(0xffffffffu, vb != 0))
		return true;
	const uint32_t ops = b.slot + kQOpsFull;
	const uint32_t nf = lds_u32(b.slot + kQNFilter);
	const uint32_t nu = lds_u32(b.slot + kQNUops) - 1u;
	const uint32_t nout = lds_u32(b.slot + kQNOut);
	for (uint32_t k = nf; k < nu; k++) {
		const uint4 rec = lds_v4(ops + 16u * k);
		const uint32_t h = rec.x;
		if (h & (OK_SETCONST | OK_COPY)) {
			if (h_type(h, VT_INT) || h_type(h, VT_FLOAT)) vec_rows<uint32_t, -1, U>(rec, b, lane, vb);
			else vec_rare<U>(rec, b, lane, vb);
		} else if (h & OK_MATH) {
			if (h_type(h, VT_FLOAT)) vec_any<float, U, false>(rec, b, lane, vb);
			else if (h_type(h, VT_INT)) vec_any<int32_t, U, false>(rec, b, lane, vb);
			else vec_rare<U>(rec, b, lane, vb);
		}
	}
	const uint64_t off = lds_u64(b.slot + kSlotBlockOff + 8u * blk);
	const uint64_t cap = lds_u64(b.slot + kQCapacity);
	bool ok = true;
	for (uint32_t j = 0; j < nout; j++) {
		const uint32_t od = lds_u32(b.slot + kQOdOut + 4 * j);
		void *out = reinterpret_cast<void *>(lds_u64(b.slot + kQOutPtr + 8 * j));
		const uint32_t stride = lds_u8(b.slot + kQOutStride + j);
		if (stride == 4)
			ok = dense_store<uint32_t>(od, b, mine, vb, static_cast<uint32_t *>(out), off, cap, lane) && ok;
		else
			ok = dense_store_rare(od, b, mine, vb, out, off, cap, stride, lane) && ok;
	}
	__syncwarp();
	return ok;
}

/* the selected rows of one full entry (chunk blocks [blk0, blk0 + nblk),
 * up to 32 of them): how many, and the output position of the first */
__device__ __forceinline__ uint32_t entry_selected(uint32_t slot, uint32_t blk0, uint32_t nblk, uint64_t *off0)
{
	const uint64_t first = lds_u64(slot + kSlotBlockOff + 8u * blk0);
	const uint32_t last = blk0 + nblk - 1;
	*off0 = first;
	return (uint32_t)(lds_u64(slot + kSlotBlockOff + 8u * last) + lds_u32(slot + kSlotBlockCnt + 4u * last) - first);
}

/* FM_BITMAP / FM_GATHER full phase: unit j of an entry's selected rows
 * (ranks [urows j, ...) of the nsel rows of chunk blocks
 * [blk0, blk0 + nblk), whose first is stored at off0).  The warp lists the
 * unit's rows from the bitmap, starting at the block that holds its first
 * rank, then reads them from the staged tile in place (b.stage the tile,
 * rows counted from its first row) or gathers them from device memory into
 * the warp's gather area.  Returns false on an output overflow. */
__device__ __forceinline__ bool full_unit(Bases b, uint32_t list, uint32_t gat, uint32_t blk0, uint32_t nblk,
	uint32_t j, uint32_t urows, uint32_t nsel, uint64_t off0, uint32_t mode, int lane)
{
	const uint32_t nb = urows > kBatchRows ? kUnitBatches : 1u;
	const uint32_t r0 = urows * j;
	if (r0 >= nsel)
		return true;  /* an entry with no selected rows: nothing to do */
	const uint32_t cnt = min(urows, nsel - r0);
	/* the block holding rank r0: lane l looks at block blk0 + l */
	uint32_t bo = 0, bc = 0;
	if ((uint32_t)lane < nblk) {
		bo = (uint32_t)(lds_u64(b.slot + kSlotBlockOff + 8u * (blk0 + lane)) - off0);
		bc = lds_u32(b.slot + kSlotBlockCnt + 4u * (blk0 + lane));
	}
	const uint32_t hit = __ballot_sync(0xffffffffu, (uint32_t)lane < nblk && bo <= r0 && r0 < bo + bc);
	if (hit == 0)
		return false;  /* counts and offsets disagree: stores nothing, reports an error */
	const int bsel = __ffs(hit) - 1;
	uint32_t rank = __shfl_sync(0xffffffffu, bo, bsel);  /* rank of the block's first selected row */
	/* words of 32 rows from that block on, 32 at a time, until the batch's
	 * last rank is listed */
	const uint32_t nwords = 8u * nblk;
	const uint32_t bm = b.slot + kSlotBitmap + 32u * blk0;
	for (uint32_t w0 = 8u * (uint32_t)bsel; w0 < nwords && rank < r0 + cnt; w0 += 32) {
		const uint32_t wi = w0 + (uint32_t)lane;
		const uint32_t word = wi < nwords ? lds_u32(bm + 4u * wi) : 0u;
		const uint32_t c = __popc(word);
		uint32_t incl = c;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
			if (lane >= d)
				incl += v;
		}
		uint32_t rr = rank + incl - c, x = word;
		const bool part = rr + c > r0 && rr < r0 + cnt;  /* this word holds ranks of the batch */
		const uint32_t parts = __ballot_sync(0xffffffffu, part);
		if (__popc(parts) <= 8) {
			/* dense rows: the batch lies in a few words, so the warp lists
			 * each of them together, lane j taking bit j */
			for (uint32_t m = parts; m; m &= m - 1) {
				const int src = __ffs(m) - 1;
				const uint32_t wx = __shfl_sync(0xffffffffu, word, src);
				const uint32_t rx = __shfl_sync(0xffffffffu, rr, src) + __popc(wx & ((1u << lane) - 1u));
				if (((wx >> lane) & 1u) && rx >= r0 && rx < r0 + cnt)
					asm volatile("st.shared.u16 [%0], %1;" ::"r"(list + 2 * (rx - r0)),
						"h"((uint16_t)(32 * (w0 + (uint32_t)src) + (uint32_t)lane)) : "memory");
			}
		} else if (part) {
			/* sparse rows: each lane lists its own word's few rows */
			while (rr < r0) {  /* ranks before the batch */
				x &= x - 1;
				rr++;
			}
			while (x && rr < r0 + cnt) {
				const uint32_t bit = __ffs(x) - 1;
				asm volatile("st.shared.u16 [%0], %1;" ::"r"(list + 2 * (rr - r0)), "h"((uint16_t)(32 * wi + bit))
					: "memory");
				rr++;
				x &= x - 1;
			}
		}
		rank += __shfl_sync(0xffffffffu, incl, 31);
	}
	__syncwarp();
	const uint64_t cap = lds_u64(b.slot + kQCapacity);
	const uint64_t pos0 = off0 + r0;
	UnitRows u;
	uint32_t in[kUnitBatches];
	unit_rows(list, cnt, nb, pos0, cap, u, in, lane);
	b.blk_row0 = 0;
	if (mode == FM_GATHER) {
		/* gathered values are indexed by unit entry; the chunk row of an
		 * entry is the entry's first row plus its row */
		b.stage = gat;
#pragma unroll
		for (int s2 = 0; s2 < (int)kUnitBatches; s2++) {
			if ((uint32_t)s2 >= nb)
				break;
			uint32_t grow[kBatchE];
#pragma unroll
			for (int i = 0; i < kBatchE; i++) {
				grow[i] = blk0 * kBlockRows + u.row[s2][i];
				u.row[s2][i] = kBatchRows * s2 + 32u * i + (uint32_t)lane;
			}
			gather_batch(b, grow, kBatchRows * s2, lane);
		}
		__syncwarp();
	}
	unit_out(b, u, in, pos0, lane);
	__syncwarp();  /* the list and gather area are this warp's next unit's */
	bool ok = true;
#pragma unroll
	for (int s2 = 0; s2 < (int)kUnitBatches; s2++)
		ok = ok && u.act[s2] == in[s2];
	return ok;
}

/* ---- ordered placement ------------------------------------------------- */

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
	for (int d = 16; d > 0; d >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, d);
	return v;
}

/* a work item's look-back word and the tag its words carry in this launch */
__device__ __forceinline__ uint64_t *status_at(const KParams &kp, uint64_t idx)
{
	return kp.status + (idx & kp.status_mask);
}

__device__ __forceinline__ uint64_t status_tag(const KParams &kp, uint64_t idx)
{
	return (uint64_t)((kp.epoch + (uint32_t)(idx >> kp.status_shift)) & kEpochMask);
}

__device__ __forceinline__ void publish(const KParams &kp, uint64_t g, uint64_t flag, uint64_t value)
{
	st_status(status_at(kp, g), (status_tag(kp, g) << kStatusEpochShift) | (flag << kStatusFlagShift) |
		(value & kStatusValueMask));
}

/* Rows written by the query's chunks before chunk g (its exclusive prefix):
 * walks back over earlier chunks' status words, kLookbackPerLane per lane
 * per round, summing aggregates up to the nearest inclusive prefix.  The
 * caller's own latest chunk of the query (index `known` with inclusive
 * prefix `known_end`, or none when known < first) is a prefix that needs no
 * load, so the walk never passes it.  Returns false if a predecessor never
 * published (bounded wait). */
constexpr int kLookbackPerLane = 4;

__device__ bool lookback_excl(const KParams &kp, int64_t first, uint64_t g, int64_t known, uint64_t known_end,
	int lane, uint64_t *excl_out)
{
	constexpr int W = 32 * kLookbackPerLane;
	/* indices below `floor` are not read: the query's start, or the known
	 * prefix (read as a stop) */
	const int64_t floor = known >= first ? known : first;
	uint64_t excl = 0;
	int64_t j = (int64_t)g - 1;
	unsigned spins = 0;
	while (true) {
		uint64_t v[kLookbackPerLane];
		uint32_t stopbits = 0, wait = 0;
#pragma unroll
		for (int x = 0; x < kLookbackPerLane; x++) {
			const int64_t idx = j - (lane * kLookbackPerLane + x);
			if (idx < floor || idx == known) {
				v[x] = (idx == known) ? (known_end & kStatusValueMask) : 0ull;
				stopbits |= 1u << x;
			} else {
				v[x] = ld_status(status_at(kp, (uint64_t)idx));
			}
		}
		/* wait until every loaded word carries this launch's tag and a flag */
		while (true) {
			wait = 0;
#pragma unroll
			for (int x = 0; x < kLookbackPerLane; x++)
				if (!((stopbits >> x) & 1u)) {
					const uint64_t idx = (uint64_t)(j - (lane * kLookbackPerLane + x));
					const bool rx = (v[x] >> kStatusEpochShift) == status_tag(kp, idx) &&
						((v[x] >> kStatusFlagShift) & 3u);
					if (!rx)
						wait |= 1u << x;
					else if (((v[x] >> kStatusFlagShift) & 3u) == kFlagPrefix)
						stopbits |= 1u << x;
				}
			/* only words before the window's nearest stop are needed */
			const uint32_t sm = __ballot_sync(0xffffffffu, stopbits != 0);
			const int stop_lane = sm ? __ffs(sm) - 1 : 32;
			const uint32_t need = lane < stop_lane ? 0xffffffffu
				: lane == stop_lane ? ((stopbits & (0u - stopbits)) - 1u) : 0u;
			const uint32_t blocking = wait & need;
			if (__all_sync(0xffffffffu, blocking == 0))
				break;
			if (++spins > kLookbackSpinLimit)
				return false;
			__nanosleep(spins < 64 ? 32 : 256);
#pragma unroll
			for (int x = 0; x < kLookbackPerLane; x++)
				if ((blocking >> x) & 1u)
					v[x] = ld_status(status_at(kp, (uint64_t)(j - (lane * kLookbackPerLane + x))));
		}
		/* the nearest stop over the whole window: the first lane with one,
		 * then that lane's first */
		const int xs = stopbits ? __ffs(stopbits) - 1 : kLookbackPerLane;
		const uint32_t pm = __ballot_sync(0xffffffffu, stopbits != 0);
		uint64_t part = 0;
		if (pm) {
			const int stop = __ffs(pm) - 1;
			const int xstop = __shfl_sync(0xffffffffu, xs, stop);
#pragma unroll
			for (int x = 0; x < kLookbackPerLane; x++)
				if (lane < stop || (lane == stop && x <= xstop))
					part += v[x] & kStatusValueMask;
			excl += warp_sum_u64(part);
			break;
		}
#pragma unroll
		for (int x = 0; x < kLookbackPerLane; x++)
			part += v[x] & kStatusValueMask;
		excl += warp_sum_u64(part);
		j -= W;
	}
	*excl_out = excl;
	return true;
}

/* ---- look-back warp: chunk counts -> block offsets ----------------------- */

__device__ void lookback_warp(const KParams &kp, unsigned char *smem, int lane)
{
	const uint32_t sbase = smem_addr(smem);
	const uint32_t flags = sbase + kOffFlags;
	/* the CTA's previous chunk: one that directly follows it in the same
	 * query starts where it ended, with no look-back */
	uint64_t prev_work = ~0ull, prev_end = 0;
	for (uint32_t i = 0;; i++) {
		const uint32_t s = i % kChunkSlots;
		if (!mbar_wait(sbase + kOffCounted + 8 * s, (i / kChunkSlots) & 1u, flags)) {
			abort_cta(kp, flags, DE_STAGE_TIMEOUT);
			return;
		}
		const uint32_t ci = sbase + kOffChunkInfo + (uint32_t)sizeof(ChunkInfo) * s;
		if (!lds_u32(ci + offsetof(ChunkInfo, valid)))
			return;
		/* the chunk's descriptor view (landed before any count group ran) */
		if (!mbar_wait(sbase + kOffDesc + 8 * s, (i / kChunkSlots) & 1u, flags)) {
			abort_cta(kp, flags, DE_STAGE_TIMEOUT);
			return;
		}
		const uint32_t slot = sbase + kSlotArea + s * kSlotBytes;
		const uint64_t g = lds_u64(ci + offsetof(ChunkInfo, work));
		const uint32_t rows = lds_u32(ci + offsetof(ChunkInfo, rows));
		const uint64_t first = lds_u64(slot + kQWorkFirst);
		const uint64_t nchunks = lds_u64(slot + kQNChunks);
		/* the chunk's count: a scan of its block counts, one per lane */
		const uint32_t nblk = (rows + kBlockRows - 1) / kBlockRows;
		const uint32_t cnt = (uint32_t)lane < nblk ? lds_u32(slot + kSlotBlockCnt + 4 * lane) : 0u;
		uint32_t incl = cnt;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
			if (lane >= d)
				incl += v;
		}
		const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
		uint64_t excl = 0;
		bool ok = true;
		if (g == first) {
			const unsigned long long *base_in =
				reinterpret_cast<const unsigned long long *>(lds_u64(slot + kQBaseIn));
			excl = base_in != nullptr ? *base_in : 0ull;
		} else if (g == prev_work + 1) {
			excl = prev_end;
		} else {
			/* the count first, so other CTAs' look-backs see it at once */
			if (lane == 0)
				publish(kp, g, kFlagAggregate, total);
			ok = lookback_excl(kp, (int64_t)first, g,
				prev_work != ~0ull && prev_work >= first && prev_work < g ? (int64_t)prev_work : -1, prev_end,
				lane, &excl);
		}
		if (!ok) {
			if (lane == 0)
				abort_cta(kp, flags, DE_LOOKBACK_TIMEOUT);
			return;
		}
		if (lane == 0) {
			publish(kp, g, kFlagPrefix, excl + total);
			if (g == first + nchunks - 1)
				*reinterpret_cast<unsigned long long *>(lds_u64(slot + kQTotalOut)) = excl + total;
		}
		if ((uint32_t)lane < nblk)
			sts_u64(slot + kSlotBlockOff + 8 * lane, excl + incl - cnt);
		/* valid rows per 64-row block, for result-tablet splitting on the
		 * host (the chunk starts on a 64-row block of its segment) */
		uint8_t *bc = reinterpret_cast<uint8_t *>(lds_u64(slot + kQBlockCounts));
		if (bc != nullptr) {
			const uint32_t base = lds_u32(ci + offsetof(ChunkInfo, block_base));
			for (uint32_t k = (uint32_t)lane; 64 * k < rows; k += 32)
				bc[base + k] = (uint8_t)(__popc(lds_u32(slot + kSlotBitmap + 8 * k)) +
					__popc(lds_u32(slot + kSlotBitmap + 8 * k + 4)));
		}
		__syncwarp();
		if (lane == 0)
			mbar_arrive(sbase + kOffBased + 8 * s);
		prev_work = g;
		prev_end = excl + total;
	}
}

/* ---- producer: claims chunks and stages their columns -------------------- */

/* last index i in [lo, hi) with a[i] <= t, given a[lo] <= t: a k-ary
 * search in which each of the warp's 32 lanes tests one probe per round, so
 * a few hundred entries take two dependent loads instead of eight */
template <typename T>
__device__ __forceinline__ uint32_t warp_search(const T *a, uint32_t lo, uint32_t hi, uint64_t t,
	int lane)
{
	while (hi - lo > 1) {
		const uint32_t step = (hi - lo + 31) / 32;
		const uint32_t i = lo + (uint32_t)lane * step;
		const bool le = i < hi && (uint64_t)a[i] <= t;
		const uint32_t m = __ballot_sync(0xffffffffu, le);  /* lane 0 (a[lo]) is set */
		lo += (uint32_t)(31 - __clz(m)) * step;
		hi = min(lo + step, hi);
	}
	return lo;
}

/* one phase's column for this lane (lane i < n holds column i of the set) */
struct LaneCol {
	uint32_t src, stride, off;
	bool has;
};

__device__ __forceinline__ LaneCol lane_col(const LoadSet &ls, int lane)
{
	LaneCol c;
	c.has = (uint32_t)lane < ls.n;
	c.src = c.has ? ls.src[lane] : 0u;
	c.stride = c.has ? ls.stride[lane] : 0u;
	c.off = c.has ? ls.off[lane] : 0u;
	return c;
}

/* the producer's copy of the current query's fields (every lane) */
struct ProdQuery {
	const QDesc *Q;
	uint64_t first, end;          /* the query's work items */
	const SegDesc *segs;
	const uint32_t *chunk_prefix;
	uint32_t nsegs, qi, seg_hint, chunk_rows;
	uint32_t count_tile, full_tile;
	uint32_t grp_size, grp_q0, grp_first;  /* the query's shared scan, if any */
	bool gather;                  /* the full phase gathers (FM_GATHER) */
	LaneCol cc, fc;               /* this lane's count and full column */
	/* the current segment: its chunks [seg_c0, seg_c1) of the query, rows,
	 * first 64-row block and this lane's columns in it; seg ~0 when none */
	uint32_t seg, seg_c0, seg_c1, seg_rows, seg_block;
	const unsigned char *ccol, *fcol;
};

/* a claimed chunk, as the producer issues its phases */
struct ProdChunk {
	uint32_t w, slot, seq, rows, row0, qi, block_base;
	uint32_t count_tile, full_tile;
	bool gather;
	LaneCol cc, fc;
	const unsigned char *ccol, *fcol;  /* this lane's columns at the chunk's first row */
};

/* the producer's copy of query qi's fields */
__device__ __forceinline__ void load_query(const KParams &kp, uint32_t qi, ProdQuery &pq, int lane)
{
	const QDesc *Q = kp.queries + qi;
	pq.Q = Q;
	pq.qi = qi;
	pq.first = Q->work_first;
	pq.end = pq.first + Q->nchunks;
	pq.segs = Q->segs;
	pq.chunk_prefix = Q->seg_chunk_prefix;
	pq.nsegs = Q->nsegs;
	pq.chunk_rows = Q->chunk_rows;
	pq.count_tile = Q->count_set.rows;
	pq.full_tile = Q->full_set.rows;
	pq.grp_size = Q->grp_size;
	pq.grp_q0 = Q->grp_q0;
	pq.grp_first = Q->grp_first;
	pq.gather = Q->full_mode == FM_GATHER;
	pq.cc = lane_col(Q->count_set, lane);
	pq.fc = lane_col(Q->full_set, lane);
	pq.seg_hint = 0;
	pq.seg = ~0u;
}

/* decode claim `cl` with the whole producer warp: the work item it names
 * (itself, or in a shared scan the chunk of one of the group's queries; see
 * QDesc::grp_size) and that chunk's query, segment and columns.  A CTA's
 * claims increase, so a search starts at the previous claim's query when it
 * can; a claim in the previous claim's group needs no search at all. */
__device__ __forceinline__ void decode_chunk(const KParams &kp, uint32_t cl, uint32_t nq, ProdQuery &pq,
	ProdChunk &c, int lane)
{
	const bool in_group = pq.Q != nullptr && pq.grp_size > 1 && cl >= pq.grp_first &&
		cl - pq.grp_first < pq.grp_size * (uint32_t)(pq.end - pq.first);
	if (!in_group && (pq.Q == nullptr || cl < pq.first || cl >= pq.end)) {
		const uint32_t lo = pq.Q != nullptr && cl >= pq.first ? pq.qi : 0u;
		load_query(kp, warp_search(kp.q_work_prefix, lo, nq, cl, lane), pq, lane);
	}
	uint32_t w = cl;
	if (pq.grp_size > 1) {
		const uint32_t local = cl - pq.grp_first;
		const uint32_t qi = pq.grp_q0 + local % pq.grp_size;
		if (qi != pq.qi)
			load_query(kp, qi, pq, lane);
		w = (uint32_t)pq.first + local / pq.grp_size;
	}
	/* a chunk in the previous chunk's segment needs no load at all */
	const uint32_t t = (uint32_t)(w - pq.first);
	if (pq.seg == ~0u || t >= pq.seg_c1) {
		const uint32_t s = warp_search(pq.chunk_prefix, pq.seg_hint, pq.nsegs, t, lane);
		const SegDesc *sd = pq.segs + s;
		pq.seg_hint = s;
		pq.seg = s;
		pq.seg_c0 = pq.chunk_prefix[s];
		pq.seg_c1 = pq.chunk_prefix[s + 1];
		pq.seg_rows = sd->rows;
		pq.seg_block = sd->block_base;
		pq.ccol = pq.cc.has ? static_cast<const unsigned char *>(sd->col[pq.cc.src]) : nullptr;
		pq.fcol = pq.fc.has ? static_cast<const unsigned char *>(sd->col[pq.fc.src]) : nullptr;
	}
	c.w = w;
	c.qi = pq.qi;
	c.row0 = (t - pq.seg_c0) * pq.chunk_rows;
	c.rows = min(pq.chunk_rows, pq.seg_rows - c.row0);
	c.block_base = pq.seg_block + c.row0 / 64u;
	c.count_tile = pq.count_tile;
	c.full_tile = pq.full_tile;
	c.gather = pq.gather;
	c.cc = pq.cc;
	c.fc = pq.fc;
	c.ccol = pq.ccol ? pq.ccol + (size_t)c.row0 * pq.cc.stride : nullptr;
	c.fcol = pq.fcol ? pq.fcol + (size_t)c.row0 * pq.fc.stride : nullptr;
}

/* The producer warp fills the ring of stages.  For each chunk it claims (in
 * order, with the next claim's atomic in flight) it waits until the chunk's
 * slot is free, writes the chunk's info, copies the query's descriptor view
 * into the slot if the slot held another query, and issues the chunk's
 * count tiles; then it issues the full tiles of the chunk claimed
 * kCountAhead chunks earlier.  Lane i
 * copies column i of a tile; the bytes of a column past its last 16-byte
 * boundary (a segment's end) are copied with plain loads before the tile is
 * announced, so no copy reads past a column.  After the last chunk it
 * announces the end on the next slot and stage.
 *
 * In a serving session the work list grows: a claim past the published
 * work first issues the pending chunks' full tiles (so queries complete),
 * then waits (bounded) for the host's doorbell or its stop request. */
__device__ void producer(const KParams &kp, unsigned char *smem, int lane)
{
	const uint32_t sbase = smem_addr(smem);
	const uint32_t flags = sbase + kOffFlags;
	const uint32_t nst = kp.nstages;
	const bool serving = kp.serve != nullptr;
	uint64_t total = serving ? 0ull : kp.total_work;
	uint32_t nq = serving ? 0u : kp.nq;
	ProdQuery pq;
	pq.Q = nullptr;
	pq.qi = 0;
	uint32_t k = 0;   /* entries issued */
	uint32_t nb = 0;  /* data buffers taken */
#if VGPU_BUF_FREELIST
	/* buffer lane's uses so far (lanes below nst): a tile takes whichever
	 * buffer was released first, not the next in turn */
	uint32_t buses = 0;
#endif
	uint32_t i = 0;   /* chunks set up (and the end) */
	bool failed = false;

	/* claims: one atomic in flight (lane 0) while the previous claim's chunk
	 * is issued, so its round trip is off the per-chunk path */
	uint32_t inflight = 0;
	bool have = false;
	auto claim = [&]() -> uint32_t {
		uint32_t v = 0;
		if (lane == 0) {
			if (!have) {
				inflight = atomicAdd(kp.counter, 1u);
				have = true;
			}
			v = inflight;
			inflight = atomicAdd(kp.counter, 1u);
		}
		return __shfl_sync(0xffffffffu, v, 0);
	};

	/* one entry: wait for its ring place (and, if it stages data, for a data
	 * buffer), announce it, copy this lane's column */
	auto issue = [&](uint32_t kind, const ProdChunk &c, uint32_t row0, uint32_t nrows, bool last,
		const LaneCol &col, const unsigned char *src, bool staged) -> bool {
		const uint32_t s = k % kEntries;
		const uint32_t full = sbase + kOffFull + 8 * s;
#if VGPU_BUF_FREELIST
		uint32_t bf = kNoBuf;
#else
		const uint32_t bf = staged ? nb % nst : kNoBuf;
#endif
		int ok = 1;
		if (lane == 0) {
			if (k >= kEntries)
				ok = mbar_wait(sbase + kOffEmpty + 8 * s, ((k / kEntries) - 1) & 1u, flags);
#if !VGPU_BUF_FREELIST
			if (ok && staged && nb >= nst)
				ok = mbar_wait(sbase + kOffBfree + 8 * bf, ((nb / nst) - 1) & 1u, flags);
#endif
		}
		if (!__shfl_sync(0xffffffffu, ok, 0))
			return false;
#if VGPU_BUF_FREELIST
		if (staged) {
			/* buffer b is free once its releases equal its uses: the phase
			 * of its last use has completed (or it has none).  The buffer
			 * in turn if it is free, else the next free one after it; with
			 * none free, sleep on the one in turn (hardware-suspended,
			 * woken by its release) and look again */
			const uint32_t turn = nb % nst;
			const uint32_t tuses = __shfl_sync(0xffffffffu, buses, (int)turn);
			uint64_t t0 = 0;
			for (uint32_t spin = 0;; spin++) {
				const bool fr = (uint32_t)lane < nst &&
					(buses == 0 || mbar_test(sbase + kOffBfree + 8 * (uint32_t)lane, (buses - 1) & 1u));
				const uint32_t m = __ballot_sync(0xffffffffu, fr);
				if (m) {
					const uint32_t after = m & (0xffffffffu << turn);
					bf = (uint32_t)(__ffs(after ? after : m) - 1);
					break;
				}
				if (lane == 0 && tuses)
					mbar_try_wait_hint(sbase + kOffBfree + 8 * turn, (tuses - 1) & 1u, 2000);
				__syncwarp();
				if ((spin & 63u) == 63u) {
					int give_up = 0;
					if (lane == 0) {
						const uint64_t now = globaltimer_ns();
						if (t0 == 0)
							t0 = now;
						else {
							uint32_t ab;
							asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(ab) : "r"(flags + 4 * kFAbort));
							if (ab || now - t0 > (uint64_t)lds_u32(flags + 4 * kFWaitMs) * 1000000ull)
								give_up = 1;
						}
					}
					if (__shfl_sync(0xffffffffu, give_up, 0))
						return false;
				}
			}
			if ((uint32_t)lane == bf)
				buses++;
		}
#endif
		const uint32_t data = sbase + kp.stage_area + (staged ? bf : 0u) * kp.stage_bytes;
		uint32_t bulk = 0;
		if (staged && col.has && nrows) {
			const uint32_t bytes = nrows * col.stride;
			bulk = bytes & ~15u;
			/* the column's last bytes past a 16-byte boundary, with plain
			 * stores; this lane's later bulk copies into the same stage
			 * bytes are ordered after them by the proxy fence */
			if (bulk < bytes) {
				const unsigned char *p = src + (size_t)row0 * col.stride;
				for (uint32_t b = bulk; b < bytes; b++)
					sts_u8(data + col.off + b, *(p + b));
				fence_proxy_async_smem();
			}
		}
		const uint32_t tx = __reduce_add_sync(0xffffffffu, bulk);
		if (lane == 0) {
			const uint32_t si = sbase + kOffStageInfo + (uint32_t)sizeof(StageInfo) * s;
			sts_v4(si, make_uint4(kind, c.slot, c.seq, row0));
			sts_v4(si + 16, make_uint4(nrows, last ? 1u : 0u, bf, 0u));
			sts_u32(sbase + kOffFin + 4 * s, 0u);
			/* the entry's tag, after its info: compute warps claim its
			 * units from here on */
			__threadfence_block();
			asm volatile("st.volatile.shared.u32 [%0], %1;" ::"r"(sbase + kOffClaim + 4 * s), "r"((k & 0xffffu) << 16)
				: "memory");
		}
		__syncwarp();
		if (lane == 0) {
			mbar_arrive_expect_tx(full, tx);
			/* the tile's info is readable now; its data lands later */
			mbar_arrive(sbase + kOffAnn + 8 * s);
		}
		__syncwarp();
		if (bulk)
			bulk_load(data + col.off, src + (size_t)row0 * col.stride, bulk, full);
		k++;
		if (staged)
			nb++;
		return true;
	};

	/* the full phase of a chunk whose count tiles were issued: one entry
	 * without data when it gathers, else its full tiles */
	auto issue_full = [&](const ProdChunk &c) -> bool {
		if (c.gather)
			return issue(SK_FULL, c, 0, c.rows, true, c.fc, nullptr, false);
		for (uint32_t r = 0; r < c.rows; r += c.full_tile)
			if (!issue(SK_FULL, c, r, min(c.full_tile, c.rows - r), r + c.full_tile >= c.rows, c.fc, c.fcol, true))
				return false;
		return true;
	};

	/* wait until slot i % kChunkSlots no longer holds chunk i - kChunkSlots */
	auto slot_free = [&](uint32_t n) -> bool {
		if (n < kChunkSlots)
			return true;
		int ok = 1;
		if (lane == 0)
			ok = mbar_wait(sbase + kOffDone + 8 * (n % kChunkSlots), ((n - kChunkSlots) / kChunkSlots) & 1u, flags);
		return __shfl_sync(0xffffffffu, ok, 0) != 0;
	};

	/* chunks whose count tiles are issued and full tiles are not, oldest
	 * first */
	ProdChunk pend[kCountAhead];
	uint32_t npend = 0;
	auto flush_one = [&]() -> bool {
		const bool ok = issue_full(pend[0]);
#pragma unroll
		for (uint32_t x = 0; x + 1 < kCountAhead; x++)
			pend[x] = pend[x + 1];
		npend--;
		return ok;
	};
	for (;;) {
		uint32_t w = claim();
		if (serving && w >= total) {
			/* nothing published to claim yet: finish the pending chunks, then
			 * wait (bounded) for the doorbell */
			while (npend && !failed)
				failed = !flush_one();
			if (failed)
				break;
			uint64_t t0 = 0;
			unsigned nap = 1000;  /* ns between doorbell polls, growing while idle */
			bool stop = false;
			for (;;) {
				unsigned long long a = 0;
				unsigned st = 0;
				if (lane == 0) {
					a = ld_acquire_sys(&kp.serve->avail);
					st = *reinterpret_cast<const volatile unsigned *>(&kp.serve->stop);
				}
				a = __shfl_sync(0xffffffffu, a, 0);
				st = __shfl_sync(0xffffffffu, st, 0);
				total = a & kAvailWorkMask;
				nq = (uint32_t)(a >> 40);
				if (w < total)
					break;
				if (st || lds_u32(flags + 4 * kFAbort)) {
					stop = true;
					break;
				}
				if (t0 == 0) {
					t0 = globaltimer_ns();
				} else if (globaltimer_ns() - t0 > (uint64_t)kp.wait_limit_ms * 1000000ull) {
					if (lane == 0)
						report(kp.error, DE_STAGE_TIMEOUT);
					stop = true;
					break;
				}
				__nanosleep(nap);
				nap = nap < 16000 ? nap * 2 : nap;
			}
			if (stop)
				w = ~0u;
		}
		if (w >= total) {
			/* the end: the pending chunks' full tiles, then the end marker */
			while (npend && !failed)
				failed = !flush_one();
			if (failed || !slot_free(i)) {
				failed = true;
				break;
			}
			ProdChunk e;
			e.slot = i % kChunkSlots;
			e.seq = i;
			e.qi = 0;
			e.gather = false;
			if (lane == 0) {
				sts_u32(sbase + kOffChunkInfo + (uint32_t)sizeof(ChunkInfo) * e.slot + offsetof(ChunkInfo, valid), 0u);
				/* the look-back warp finds the end in this slot */
				mbar_arrive(sbase + kOffCounted + 8 * e.slot);
			}
			LaneCol none;
			none.has = false;
			none.src = none.stride = none.off = 0;
			if (!issue(SK_END, e, 0, 0, true, none, nullptr, false))
				failed = true;
			break;
		}
		ProdChunk c;
		decode_chunk(kp, w, nq, pq, c, lane);
		c.slot = i % kChunkSlots;
		c.seq = i;
		if (!slot_free(i)) {
			failed = true;
			break;
		}
		/* a gathering full phase reads the full set's columns of this chunk
		 * from device memory: their addresses at the chunk's first row */
		if (c.gather && c.fc.has)
			sts_u64(sbase + kSlotArea + c.slot * kSlotBytes + kSlotColPtr + 8 * lane,
				reinterpret_cast<uint64_t>(c.fcol));
		bool desc = false;
		if (lane == 0) {
			const uint32_t ci = sbase + kOffChunkInfo + (uint32_t)sizeof(ChunkInfo) * c.slot;
			sts_v4(ci, make_uint4(1u, c.qi, (uint32_t)c.w, 0u));
			sts_v4(ci + 16, make_uint4(c.rows, c.block_base, (c.rows + c.count_tile - 1) / c.count_tile,
				c.gather ? 1u : (c.rows + c.full_tile - 1) / c.full_tile));
			const uint32_t held = sbase + kOffHeld + 4 * c.slot;
			desc = lds_u32(held) != c.qi;
			sts_u32(held, c.qi);
		}
		desc = __shfl_sync(0xffffffffu, desc ? 1 : 0, 0) != 0;
		/* the slot's descriptor barrier completes once per chunk, when the
		 * query's descriptor view has landed in the slot (at once if the slot
		 * holds that query's view already) */
		const uint32_t dbar = sbase + kOffDesc + 8 * c.slot;
		if (lane == 0) {
			if (desc)
				mbar_arrive_expect_tx(dbar, kQDescCopy);
			else
				mbar_arrive(dbar);
		}
		__syncwarp();
		if (desc && lane == 0)
			bulk_load(sbase + kSlotArea + c.slot * kSlotBytes, kp.queries + c.qi, kQDescCopy, dbar);
		bool ok = true;
		for (uint32_t r = 0; ok && r < c.rows; r += c.count_tile)
			ok = issue(SK_COUNT, c, r, min(c.count_tile, c.rows - r), r + c.count_tile >= c.rows, c.cc, c.ccol,
				true);
		if (ok && npend == kCountAhead)
			ok = flush_one();
		if (!ok) {
			failed = true;
			break;
		}
		pend[npend++] = c;
		i++;
	}
	if (failed) {
		if (lane == 0) {
			abort_cta(kp, flags, DE_STAGE_TIMEOUT);
			/* wait (bounded) for the copies already issued so none lands
			 * after the CTA exits (entries without data complete at once) */
			const uint32_t first = k > kEntries ? k - kEntries : 0;
			for (uint32_t kk = first; kk < k; kk++) {
				const uint32_t bar = sbase + kOffFull + 8 * (kk % kEntries);
				const uint64_t t0 = globaltimer_ns();
				while (!mbar_try_wait_hint(bar, (kk / kEntries) & 1u, kSuspendHintNs) &&
					globaltimer_ns() - t0 < 1000000000ull) {
				}
			}
		}
	}
}

/* ---- compute warps ------------------------------------------------------- */

__device__ __forceinline__ uint32_t ldv_u32(uint32_t a)
{
	uint32_t v;
	asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
	return v;
}

__device__ __forceinline__ void stv_u32(uint32_t a, uint32_t v)
{
	asm volatile("st.volatile.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t atom_cas_shared(uint32_t a, uint32_t cmp, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.shared.cas.b32 %0, [%1], %2, %3;" : "=r"(old) : "r"(a), "r"(cmp), "r"(v) : "memory");
	return old;
}

/* finish counters: each finisher's release orders its warp's work before
 * the count, and the last one's acquire makes all of it visible to it (and,
 * through its barrier arrivals, to the warps that wait on them) */
__device__ __forceinline__ uint32_t atom_add_acq_rel_shared(uint32_t a, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.acq_rel.cta.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(v) : "memory");
	return old;
}

/* Compute warps claim units of work from the entries in ring order: a count
 * entry's units are its groups of kCountGroup blocks; a full entry's are
 * batches of up to 32 kBatchE of its selected rows (groups of kCountGroup
 * blocks when it runs the filter again).  The claim word of an entry holds
 * the entry's ordinal (low 16 bits, written by the producer when it
 * announces the entry) and the units taken; a warp takes a unit with a
 * compare-and-swap on it, the warp that takes an entry's last unit moves the
 * cursor to the next entry, and the warp that finishes an entry's last unit
 * releases the entry and its data buffer and, after a chunk's last count or
 * full entry, arrives on the chunk's counted or done barrier.  So idle warps
 * always take the oldest work, however uneven an entry's units are, and no
 * warp waits for another to pass an entry.  A full entry's unit count needs
 * the chunk's offsets, so a warp waits for them before it counts. */
template <int W>
__device__ void compute_warp(const KParams &kp, unsigned char *smem, int w, int lane)
{
	const uint32_t sbase = smem_addr(smem);
	const uint32_t flags = sbase + kOffFlags;
	const uint32_t warp_base = sbase + kWarpArea + (uint32_t)w * kp.warp_bytes;
	const uint32_t list = warp_base;
	const uint32_t gat = warp_base + kp.gat_off;
	Bases b;
	b.rowv = warp_base + kp.row_off;
	b.selv = warp_base + kp.sel_off;
	uint32_t based_seq = ~0u;    /* the chunk whose offsets this warp waited for */
	uint32_t desc_seq = ~0u;     /* the chunk whose descriptor view this warp waited for */
	/* the chunk's descriptor view in its slot: a warp waits for it before it
	 * first reads the slot for that chunk */
	auto wait_desc = [&](uint32_t slot, uint32_t seq) -> bool {
		if (desc_seq == seq)
			return true;
		desc_seq = seq;
		return mbar_wait(sbase + kOffDesc + 8 * slot, (seq / kChunkSlots) & 1u, flags);
	};
	auto wait_based = [&](uint32_t slot, uint32_t seq) -> bool {
		if (based_seq == seq)
			return true;
		based_seq = seq;
		return mbar_wait(sbase + kOffBased + 8 * slot, (seq / kChunkSlots) & 1u, flags);
	};
	/* the entry of the warp's last unit, kept for the fast claim below */
	uint32_t k = 0, n = 0, kind = 0, slot = 0, seq = 0, row0 = 0, nrows = 0, buf = 0, mode = FM_BITMAP;
	uint32_t nsel = 0, urows = kBatchRows;
	uint64_t off0 = 0;
	bool have = false;
	for (;;) {
		/* ---- claim a unit */
		uint32_t j = 0;
		bool fail = false, fast = false;
		uint64_t t0 = 0;
		if (have) {
			/* fast path: the next unit of the entry of the warp's last unit.
			 * The entry's info is still the warp's while its claim word
			 * carries its tag and units remain (a recycled entry has a new
			 * tag, so the swap fails) */
			uint32_t got = 0, taken = 0;
			if (lane == 0) {
				const uint32_t cw = sbase + kOffClaim + 4 * (k % kEntries);
				const uint32_t c = ldv_u32(cw);
				taken = c & 0xffffu;
				if ((c >> 16) == (k & 0xffffu) && taken < n) {
					got = atom_cas_shared(cw, c, c + 1) == c;
					if (got && taken + 1 == n)
						stv_u32(sbase + kOffCur, k + 1);
				}
			}
			fast = __shfl_sync(0xffffffffu, got, 0) != 0;
			j = __shfl_sync(0xffffffffu, taken, 0);
		}
		for (uint32_t spin = 0; !fast; spin++) {
			/* bounded: a claim that makes no progress for the wait limit
			 * (or after another warp aborted the CTA) gives up */
			if ((spin & 255u) == 255u) {
				const uint64_t now = globaltimer_ns();
				if (t0 == 0) {
					t0 = now;
				} else if (ldv_u32(flags + 4 * kFAbort) ||
					now - t0 > (uint64_t)lds_u32(flags + 4 * kFWaitMs) * 1000000ull) {
					fail = true;
					break;
				}
			}
			uint32_t kk = 0, c = 0;
			if (lane == 0) {
				kk = ldv_u32(sbase + kOffCur);
				c = ldv_u32(sbase + kOffClaim + 4 * (kk % kEntries));
			}
			kk = __shfl_sync(0xffffffffu, kk, 0);
			c = __shfl_sync(0xffffffffu, c, 0);
			const uint32_t s = kk % kEntries;
			const uint32_t tag = c >> 16;
			if (tag != (kk & 0xffffu)) {
				/* not announced yet (the slot still holds the entry a lap
				 * earlier), or the cursor moved on meanwhile */
				if (tag == ((kk - kEntries) & 0xffffu) &&
					!mbar_wait(sbase + kOffAnn + 8 * s, (kk / kEntries) & 1u, flags)) {
					fail = true;
					break;
				}
				continue;
			}
			__threadfence_block();  /* the entry's info after its tag */
			const uint32_t sia = sbase + kOffStageInfo + (uint32_t)sizeof(StageInfo) * s;
			const uint4 s0 = lds_v4(sia), s1 = lds_v4(sia + 16);
			__threadfence_block();
			uint32_t c2 = 0;
			if (lane == 0)
				c2 = ldv_u32(sbase + kOffClaim + 4 * s);
			if (__shfl_sync(0xffffffffu, c2, 0) != c)
				continue;  /* claimed or recycled meanwhile: the info may be torn */
			kind = s0.x;
			slot = s0.y;
			seq = s0.z;
			row0 = s0.w;
			nrows = s1.x;
			buf = s1.z;
			if (kind == SK_END)
				return;  /* every unit before the end is claimed */
			const uint32_t nblk = (nrows + kBlockRows - 1) / kBlockRows;
			if (kind == SK_COUNT) {
				n = (nblk + kCountGroup - 1) / kCountGroup;
			} else {
				if (!wait_desc(slot, seq) || !wait_based(slot, seq)) {
					fail = true;
					break;
				}
				b.slot = sbase + kSlotArea + slot * kSlotBytes;
				mode = lds_u32(b.slot + kQFullMode);
				if (mode == FM_REFILTER || mode == FM_DENSE) {
					n = (nblk + kCountGroup - 1) / kCountGroup;
				} else {
					nsel = entry_selected(b.slot, row0 / kBlockRows, nblk, &off0);
					/* two-batch units for entries with at least two such
					 * units of rows (dense entries: the op dispatch is shared
					 * by twice the rows, and units still run in parallel),
					 * where the launch's warp areas hold them */
					urows = kp.unit_batches > 1 && nsel >= 2 * kUnitE ? kUnitE : kBatchRows;
					n = max(1u, (nsel + urows - 1) / urows);
				}
			}
			const uint32_t taken = c & 0xffffu;
			if (taken < n) {
				uint32_t got = 0;
				if (lane == 0) {
					got = atom_cas_shared(sbase + kOffClaim + 4 * s, c, c + 1) == c;
					if (got && taken + 1 == n)
						stv_u32(sbase + kOffCur, kk + 1);
				}
				if (__shfl_sync(0xffffffffu, got, 0)) {
					k = kk;
					j = taken;
					have = true;
					break;
				}
				continue;
			}
			/* every unit taken: the last taker is moving the cursor */
		}
		if (fail || (kind == SK_COUNT && !wait_desc(slot, seq)) ||
			!mbar_wait(sbase + kOffFull + 8 * (k % kEntries), (k / kEntries) & 1u, flags)) {
			if (lane == 0)
				abort_cta(kp, flags, DE_STAGE_TIMEOUT);
			return;
		}
		/* ---- run it */
		b.slot = sbase + kSlotArea + slot * kSlotBytes;
		const uint32_t tile = buf != kNoBuf ? sbase + kp.stage_area + buf * kp.stage_bytes : 0u;
		const uint32_t nblk = (nrows + kBlockRows - 1) / kBlockRows;
		const uint32_t blk0 = row0 / kBlockRows;
		bool ok = true;
		if (kind == SK_COUNT || mode == FM_REFILTER || mode == FM_DENSE) {
			const uint32_t r = j * kCountGroup * kBlockRows;
			b.stage = tile;
			b.blk_row0 = r;
			if (kind == SK_COUNT)
				count_group(b, blk0 + j * kCountGroup, min((uint32_t)kCountGroup, nblk - j * kCountGroup),
					min((uint32_t)(kCountGroup * kBlockRows), nrows - r), lane);
			else if (mode == FM_DENSE)
				ok = dense_group(b, blk0 + j * kCountGroup, min((uint32_t)(kCountGroup * kBlockRows), nrows - r), lane);
			else
				ok = refilter_group(b, list, blk0 + j * kCountGroup, min((uint32_t)(kCountGroup * kBlockRows), nrows - r),
					kp.unit_batches, lane);
		} else {
			b.stage = tile;
			ok = full_unit(b, list, gat, blk0, nblk, j, urows, nsel, off0, mode, lane);
		}
		/* a serving session reports rows beyond capacity in the query's
		 * completion record instead */
		if (!__all_sync(0xffffffffu, ok) && lane == 0 && kp.serve == nullptr)
			report(kp.error, DE_OUTPUT_OVERFLOW);
		const bool serving_full = kind == SK_FULL && kp.serve != nullptr;
		if (serving_full)
			__threadfence();  /* this unit's result rows before the chunk counts as stored */
		__syncwarp();
		/* ---- finish it */
		if (lane == 0 && atom_add_acq_rel_shared(sbase + kOffFin + 4 * (k % kEntries), 1u) + 1u == n) {
			/* the entry's last unit: its buffer is free, and the chunk's
			 * phase is done once all its entries of this kind are */
			if (buf != kNoBuf)
				mbar_arrive(sbase + kOffBfree + 8 * buf);
			const uint32_t ci = sbase + kOffChunkInfo + (uint32_t)sizeof(ChunkInfo) * slot;
			const uint32_t cf = sbase + (kind == SK_COUNT ? kOffCfin : kOffFfin) + 4 * slot;
			const uint32_t need = lds_u32(ci + (kind == SK_COUNT ? offsetof(ChunkInfo, ncount) : offsetof(ChunkInfo, nfull)));
			if (atom_add_acq_rel_shared(cf, 1u) + 1u == need) {
				stv_u32(cf, 0u);
				if (kind == SK_COUNT) {
					mbar_arrive(sbase + kOffCounted + 8 * slot);
				} else {
					if (serving_full) {
						/* the chunk that completes its query writes the
						 * query's completion record */
						const uint32_t qi = lds_u32(ci + offsetof(ChunkInfo, query));
						const uint64_t nch = lds_u64(b.slot + kQNChunks);
						unsigned long long *tot = reinterpret_cast<unsigned long long *>(lds_u64(b.slot + kQTotalOut));
						__threadfence();
						const unsigned done = atomicAdd(&kp.done_chunks[qi], 1u) + 1u;
						if (done == (unsigned)nch) {
							__threadfence();
							const unsigned long long nrow = *reinterpret_cast<volatile unsigned long long *>(tot);
							volatile ServeRec *r = kp.recs + qi;
							r->rows = nrow;
							__threadfence_system();
							r->seq = (unsigned long long)qi + 1ull;
						}
					}
					mbar_arrive(sbase + kOffDone + 8 * slot);
				}
			}
			mbar_arrive(sbase + kOffEmpty + 8 * (k % kEntries));
		}
		__syncwarp();
	}
}

template <int W>
__global__ void __launch_bounds__(32 * (W + 2), 1) vm_kernel(const KParams kp)
{
	extern __shared__ __align__(128) unsigned char smem[];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	if (tid == 0) {
		const uint32_t sbase = smem_addr(smem);
		/* entries, buffers and chunk phases are released once, by the
		 * warp that finishes their last unit */
		for (uint32_t s = 0; s < kEntries; s++) {
			mbar_init(sbase + kOffFull + 8 * s, 1);
			mbar_init(sbase + kOffEmpty + 8 * s, 1);
			mbar_init(sbase + kOffAnn + 8 * s, 1);
			/* the slot holds "entry s - kEntries" until entry s is announced */
			sts_u32(sbase + kOffClaim + 4 * s, ((s - kEntries) & 0xffffu) << 16);
			sts_u32(sbase + kOffFin + 4 * s, 0u);
		}
		sts_u32(sbase + kOffCur, 0u);
		for (uint32_t s = 0; s < kp.nstages; s++)
			mbar_init(sbase + kOffBfree + 8 * s, 1);
		for (uint32_t q = 0; q < kChunkSlots; q++) {
			mbar_init(sbase + kOffCounted + 8 * q, 1);
			mbar_init(sbase + kOffBased + 8 * q, 1);
			mbar_init(sbase + kOffDone + 8 * q, 1);
			mbar_init(sbase + kOffDesc + 8 * q, 1);
			sts_u32(sbase + kOffCfin + 4 * q, 0u);
			sts_u32(sbase + kOffFfin + 4 * q, 0u);
			sts_u32(sbase + kOffHeld + 4 * q, ~0u);
		}
		for (int x = 0; x < 8; x++)
			sts_u32(sbase + kOffFlags + 4 * x, 0u);
		sts_u32(sbase + kOffFlags + 4 * kFWaitMs, kp.wait_limit_ms);
		fence_mbar_init();
	}
	__syncthreads();
	if (warp == W)
		producer(kp, smem, lane);
	else if (warp == W + 1)
		lookback_warp(kp, smem, lane);
	else
		compute_warp<W>(kp, smem, warp, lane);
}

/* ---- host-side launcher ------------------------------------------------ */

/* The kernel's dynamic shared-memory bound is always set to the device's
 * opt-in maximum, never to one launch's size: host threads launching
 * different shapes of the same kernel (a serving session beside single
 * queries) would otherwise lower the bound under one another's launches. */
static int allow_smem(const void *fn)
{
	int dev = 0, optin = 0;
	if (cudaGetDevice(&dev) != cudaSuccess ||
		cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
		return 0;
	return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) == cudaSuccess;
}

template <int W>
static int launch_t(const KParams &kp, unsigned grid, size_t smem, cudaStream_t stream)
{
	auto fn = vm_kernel<W>;
	if (!allow_smem((const void *)fn))
		return 0;
	/* W compute warps, the producer and the look-back warp; a failed launch
	 * leaves its error for the caller's message */
	fn<<<grid, 32 * (W + 2), smem, stream>>>(kp);
	return cudaPeekAtLastError() == cudaSuccess;
}

template <int W>
static int occ_t(size_t smem, int *ctas)
{
	auto fn = vm_kernel<W>;
	if (!allow_smem((const void *)fn))
		return 0;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, 32 * (W + 2), smem) == cudaSuccess;
}

#define VGPU_WARPS(X) X(4) X(8) X(10) X(14) X(16)

int shape_supported(const Shape &s)
{
#define X(W) if (s.threads == 32 * W) return 1;
	VGPU_WARPS(X)
#undef X
	return 0;
}

int launch_vm(const Shape &s, const KParams &kp, unsigned grid, size_t smem, void *stream)
{
#define X(W) if (s.threads == 32 * W) return launch_t<W>(kp, grid, smem, (cudaStream_t)stream);
	VGPU_WARPS(X)
#undef X
	return 0;
}

int occupancy(const Shape &s, size_t smem, int *ctas)
{
#define X(W) if (s.threads == 32 * W) return occ_t<W>(smem, ctas);
	VGPU_WARPS(X)
#undef X
	return 0;
}

}  // namespace vgpu
