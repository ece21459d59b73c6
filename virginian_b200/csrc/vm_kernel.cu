/*
 * The sm_100a data-parallel VM kernel.
 *
 * Replaces the reference's virginia_gpu (src/vm/vm_gpu.cu:1152-1225), which
 * runs one thread per row with a 16-entry register file in local memory, a
 * switch dispatch per op per thread and atomics for (unordered) result
 * placement.  Here a CTA is a pipeline over tiles of TILE = THREADS x R
 * rows, tied together by mbarriers, with four roles:
 *
 *  - producer warp: claims work items (one tile of one segment of one query)
 *    from a global counter, in order, decodes them warp-wide and copies the
 *    tile's columns (plus the query's descriptor when the stage does not hold
 *    it) into a ring of shared-memory stages with TMA bulk copies
 *    (cp.async.bulk completing on the stage's full barrier);
 *  - filter warps (THREADS threads): run the filter ops over every row of the
 *    tile (row state as bit masks: valid, active, and rows parked at pending
 *    jump targets; each lane holds R rows in chunks of 4 consecutive rows),
 *    count valid rows per 64 rows with bit-plane ballots, scan the counts and
 *    write the tile's selected rows, in row order, to a shared list, then
 *    publish the tile's count to the query's look-back words;
 *  - look-back warp: resolves the tile's position in the query's result with
 *    a warp-wide decoupled look-back over earlier tiles (32 status words per
 *    round); a tile that directly follows the CTA's previous tile of the same
 *    query starts where that one ended, with no look-back;
 *  - projection warps: run the projection ops over the tile's list in
 *    32-entry batches and write each result row to the tile's offset plus
 *    its list position (coalesced stores), then release the stage.
 *
 * Each op is one 16-byte record fetched with a single shared-memory load and
 * dispatched on one handler code; operands are read and written by 32-bit
 * shared-memory address.  Rows land in original row order (the single-core
 * CPU VM's order, src/vm/virginia.c:476-578) with plain stores; no output
 * atomics.  Arithmetic matches the CPU VM bit for bit: float/double use the
 * _rn intrinsics (no FMA contraction, IEEE division) and x86 NaN results,
 * integers wrap as on x86.  Every wait is bounded; on expiry the kernel
 * records an error code and stops instead of hanging.
 */
#include <cstddef>
#include <cstdint>
#include <climits>

#include <cuda_runtime.h>

#include "vgpu_engine.h"

namespace vgpu {

/* bounded waits: a stage or offset wait gives up after the launch's limit
 * (a second by default), far beyond any real wait; look-back polls after
 * 2^24 rounds of 32-256 ns */
constexpr uint32_t kSuspendHintNs = 20000;

/* flag words of a CTA: ok per slot, then abort, end tile, -, wait limit */
constexpr unsigned kFAbortSlot = 4;
constexpr unsigned kLookbackSpinLimit = 1u << 24;

/* shared memory header (kSmemHeader bytes) */
constexpr unsigned kMaxGroups = 128;  /* R x warps */
constexpr unsigned kOffFull = 0;                            /* mbarrier[kMaxStages] */
constexpr unsigned kOffEmpty = kOffFull + 8 * kMaxStages;   /* mbarrier[kMaxStages] */
constexpr unsigned kOffLready = kOffEmpty + 8 * kMaxStages; /* mbarrier[kSlots]: list and count ready */
constexpr unsigned kOffOready = kOffLready + 8 * kSlots;     /* mbarrier[kSlots]: offset ready */
constexpr unsigned kOffLfree = kOffOready + 8 * kSlots;      /* mbarrier[kSlots]: projection done */
constexpr unsigned kOffCdone = kOffLfree + 8 * kSlots;       /* mbarrier[kSlots]: all counts written */
constexpr unsigned kOffOff = kOffCdone + 8 * kSlots;         /* uint64[kSlots]: tile offsets */
constexpr unsigned kOffFlags = kOffOff + 8 * kSlots;         /* uint32[8]: ok[kSlots], abort, end tile */
constexpr unsigned kOffTot = kOffFlags + 32;                 /* uint32[kSlots]: tile totals */
constexpr unsigned kOffHeld = kOffTot + 4 * kSlots;          /* uint32[kMaxStages]: query per stage */
constexpr unsigned kOffTready = 328;                          /* mbarrier[kSlots]: tile count ready */
constexpr unsigned kOffCnt = 512;                            /* uint32[kSlots][kMaxGroups]: per 64 rows */
constexpr unsigned kFAbort = kFAbortSlot, kFEnd = 5, kFWaitMs = 7;  /* flag words */
static_assert(kSlots <= kFAbort, "ok flags per slot");
static_assert(kOffHeld + 4 * kMaxStages <= kOffTready, "smem header layout");
static_assert(kOffTready + 8 * kSlots <= kOffCnt, "smem header layout");
static_assert(kOffCnt + 4 * kSlots * kMaxGroups <= kSmemHeader, "smem header overflow");
static_assert(kQDescStaged % 16 == 0 && kQDescStaged <= sizeof(QDesc), "descriptor copies in 16-byte chunks");
static_assert(kStageHdr >= kQDescStaged + sizeof(StageInfo), "stage header too small");
static_assert(offsetof(QDesc, ops) % 16 == 0, "op records are read 16 bytes at a time");

/* where the fields the compute warps read sit in a stage's descriptor copy */
constexpr uint32_t kQOps = (uint32_t)offsetof(QDesc, ops);
constexpr uint32_t kQNFilter = (uint32_t)offsetof(QDesc, nfilter);
constexpr uint32_t kQNUops = (uint32_t)offsetof(QDesc, nuops);
constexpr uint32_t kQNOut = (uint32_t)offsetof(QDesc, nout);
constexpr uint32_t kQOutStride = (uint32_t)offsetof(QDesc, out_stride);
constexpr uint32_t kQOdOut = (uint32_t)offsetof(QDesc, od_out);
constexpr uint32_t kQOutPtr = (uint32_t)offsetof(QDesc, out_ptr);
constexpr uint32_t kQCapacity = (uint32_t)offsetof(QDesc, capacity);
constexpr uint32_t kQVecSlot = (uint32_t)offsetof(QDesc, vec_slot);

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
 * atomic) accesses suffice: an acquire or release here would fence the
 * warp's outstanding result stores on every tile. */
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

/* the serving doorbell, with acquire semantics: descriptors, work prefixes
 * and tile prefixes the host wrote before ringing it are seen by every
 * later load of this CTA (ordered through its mbarriers), even where a load
 * of a neighbouring entry had cached their lines before the host wrote them */
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

/* bounded wait for an mbarrier phase; false on timeout or when the CTA's
 * abort flag (a shared-memory word, if given) is set.  The bound is the
 * launch's wait limit, which the CTA keeps in the last of its flag words
 * (the abort flag's neighbours); a second without an abort flag. */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, const volatile uint32_t *abort)
{
	if (mbar_try_wait(bar, phase))
		return true;
	const uint32_t abort_addr = abort ? smem_addr(const_cast<const uint32_t *>(abort)) : 0u;
	uint64_t limit_ns = 1000000000ull;
	if (abort_addr) {
		uint32_t ms;
		asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(ms) : "r"(abort_addr + 4 * (7 - kFAbortSlot)));
		limit_ns = (uint64_t)ms * 1000000ull;
	}
	const uint64_t t0 = globaltimer_ns();
	for (;;) {
		if (mbar_try_wait_hint(bar, phase, kSuspendHintNs))
			return true;
		if (abort_addr) {
			uint32_t v;
			asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(abort_addr));
			if (v)
				return false;
		}
		if (globaltimer_ns() - t0 > limit_ns)
			return false;
	}
}

/* ---- shared-memory access by 32-bit shared address ---------------------
 * Every tile, register-vector and descriptor access of the compute warps
 * goes through these, so each is one ld/st.shared.  They are volatile asm:
 * the compiler keeps them in program order, and the hardware still
 * pipelines consecutive independent loads. */

__device__ __forceinline__ uint32_t lds_u8(uint32_t a)
{
	uint32_t v;
	asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
	return v;
}

__device__ __forceinline__ uint32_t lds_u16(uint32_t a)
{
	uint16_t v;
	asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
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

__device__ __forceinline__ void sts_u16(uint32_t a, uint32_t v)
{
	asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"((uint16_t)v) : "memory");
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

/* an operand resolved for one tile: element i at addr + i * step (step 0 for
 * a scalar), indexed by selection position instead of tile row when sel */
struct Opnd {
	uint32_t addr;
	uint32_t step;
	bool sel;
};

/* staged columns and scalars (the descriptor's constant table) live in the
 * tile's stage, row vectors in the tile's row-vector slot, selection
 * vectors in their single area */
template <int SIZE>
__device__ __forceinline__ Opnd opnd(uint32_t od, uint32_t sbase, uint32_t sdelta, uint32_t vdelta)
{
	const uint32_t kind = od >> 30;
	Opnd o;
	o.addr = sbase + (od & OD_OFFSET) +
		((kind == (OD_STAGE >> 30) || kind == (OD_SCALAR >> 30)) ? sdelta
			: kind == (OD_ROWVEC >> 30) ? vdelta : 0u);
	o.step = kind == (OD_SCALAR >> 30) ? 0u : (uint32_t)SIZE;
	o.sel = kind == (OD_SELVEC >> 30);
	return o;
}

/* Rows of a tile: thread tid holds R = 4 C rows, in C chunks of 4
 * consecutive rows; chunk c of thread tid starts at tile row
 * c * 4 * THREADS + 4 * tid, and row k of the chunk is bit 4 c + k of the
 * thread's row masks.  One 16-byte shared load fetches a chunk of a 4-byte
 * column. */
template <int THREADS>
__device__ __forceinline__ uint32_t chunk_row(int c, int tid)
{
	return (uint32_t)(c * 4 * THREADS + 4 * tid);
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

/* ---- filter: every row of the tile, row state in bit masks --------------- */

struct RowState {
	uint32_t valid;
	uint32_t active;
	uint32_t pend[kMaxSlots];
};

/* rows in `jumped` leave the active set, park in the op's target slot and,
 * for a jump with p4 == 0, stop being valid (src/vm/virginia.c:59-63) */
__device__ __forceinline__ void take_jump(RowState &st, uint32_t head, uint32_t jumped)
{
	st.active &= ~jumped;
	if (!(head & OPH_VJUMP))
		st.valid &= ~jumped;
	const uint32_t slot = (head >> OPH_SLOT_SHIFT) & 7u;
#pragma unroll
	for (int s = 0; s < kMaxSlots; s++)
		if (slot == (uint32_t)s)
			st.pend[s] |= jumped;
}

/* element bits <-> values */
template <typename T>
__device__ __forceinline__ T from_bits(uint64_t b)
{
	if constexpr (sizeof(T) == 8) {
		const long long v = (long long)b;
		return *reinterpret_cast<const T *>(&v);
	} else if constexpr (sizeof(T) == 4) {
		const uint32_t v = (uint32_t)b;
		return *reinterpret_cast<const T *>(&v);
	} else {
		const unsigned char v = (unsigned char)b;
		return *reinterpret_cast<const T *>(&v);
	}
}

template <typename T>
__device__ __forceinline__ uint64_t to_bits(T x)
{
	if constexpr (sizeof(T) == 8)
		return *reinterpret_cast<const unsigned long long *>(&x);
	else if constexpr (sizeof(T) == 4)
		return *reinterpret_cast<const uint32_t *>(&x);
	else
		return *reinterpret_cast<const unsigned char *>(&x);
}

/* one chunk (4 consecutive rows) of a column or row vector */
template <typename T>
__device__ __forceinline__ void ld_chunk(uint32_t a, T *v)
{
	if constexpr (sizeof(T) == 4) {
		const uint4 q = lds_v4(a);
		v[0] = from_bits<T>(q.x); v[1] = from_bits<T>(q.y); v[2] = from_bits<T>(q.z); v[3] = from_bits<T>(q.w);
	} else if constexpr (sizeof(T) == 8) {
		const uint4 q0 = lds_v4(a), q1 = lds_v4(a + 16);
		v[0] = from_bits<T>((uint64_t)q0.y << 32 | q0.x);
		v[1] = from_bits<T>((uint64_t)q0.w << 32 | q0.z);
		v[2] = from_bits<T>((uint64_t)q1.y << 32 | q1.x);
		v[3] = from_bits<T>((uint64_t)q1.w << 32 | q1.z);
	} else {
		const uint32_t w = lds_u32(a);
		v[0] = from_bits<T>(w & 0xffu); v[1] = from_bits<T>((w >> 8) & 0xffu);
		v[2] = from_bits<T>((w >> 16) & 0xffu); v[3] = from_bits<T>(w >> 24);
	}
}

template <typename T>
__device__ __forceinline__ void st_chunk(uint32_t a, const T *v)
{
	if constexpr (sizeof(T) == 4) {
		sts_v4(a, make_uint4((uint32_t)to_bits(v[0]), (uint32_t)to_bits(v[1]), (uint32_t)to_bits(v[2]),
			(uint32_t)to_bits(v[3])));
	} else if constexpr (sizeof(T) == 8) {
		const uint64_t b0 = to_bits(v[0]), b1 = to_bits(v[1]), b2 = to_bits(v[2]), b3 = to_bits(v[3]);
		sts_v4(a, make_uint4((uint32_t)b0, (uint32_t)(b0 >> 32), (uint32_t)b1, (uint32_t)(b1 >> 32)));
		sts_v4(a + 16, make_uint4((uint32_t)b2, (uint32_t)(b2 >> 32), (uint32_t)b3, (uint32_t)(b3 >> 32)));
	} else {
		sts_u32(a, (uint32_t)(to_bits(v[0]) | to_bits(v[1]) << 8 | to_bits(v[2]) << 16 | to_bits(v[3]) << 24));
	}
}

/* the operand's elements for this thread's R rows */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void load_rows(const Opnd &o, int tid, T (&v)[R])
{
	if (o.step == 0) {
		const T x = SM<T>::ld(o.addr);
#pragma unroll
		for (int r = 0; r < R; r++)
			v[r] = x;
	} else {
#pragma unroll
		for (int c = 0; c < R / 4; c++)
			ld_chunk<T>(o.addr + chunk_row<THREADS>(c, tid) * (uint32_t)sizeof(T), v + 4 * c);
	}
}

/* store the rows whose bit is set in `mask` (whole chunks at once) */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void store_rows(uint32_t addr, int tid, const T (&v)[R], uint32_t mask)
{
#pragma unroll
	for (int c = 0; c < R / 4; c++) {
		const uint32_t a = addr + chunk_row<THREADS>(c, tid) * (uint32_t)sizeof(T);
		const uint32_t m = (mask >> (4 * c)) & 0xfu;
		if (m == 0xfu) {
			st_chunk<T>(a, v + 4 * c);
		} else if (m) {
#pragma unroll
			for (int k = 0; k < 4; k++)
				if ((m >> k) & 1u)
					SM<T>::st(a + k * (uint32_t)sizeof(T), v[4 * c + k]);
		}
	}
}

/* per-op arguments of the filter */
struct FArgs {
	uint32_t sbase, sd, vd;
	int tid;
};

template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void f_cmp(const uint4 &rec, const FArgs &f, RowState &st)
{
	T x[R], y[R];
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.y, f.sbase, f.sd, f.vd), f.tid, x);
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.z, f.sbase, f.sd, f.vd), f.tid, y);
	uint32_t bits = 0;
#pragma unroll
	for (int r = 0; r < R; r++)
		bits |= (uint32_t)cmp_eval<T, OP>(x[r], y[r]) << r;
	take_jump(st, rec.x, st.active & bits);
}

template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_not(const uint4 &rec, const FArgs &f, RowState &st)
{
	T x[R];
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.y, f.sbase, f.sd, f.vd), f.tid, x);
	uint32_t bits = 0;
#pragma unroll
	for (int r = 0; r < R; r++)
		bits |= (uint32_t)(x[r] == T(0)) << r;
	take_jump(st, rec.x, st.active & bits);
}

/* arithmetic into a register vector: active rows only, unless the register
 * has this single definition (then no row that skips it reads it) */
template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void f_math(const uint4 &rec, const FArgs &f, const RowState &st)
{
	T x[R], y[R];
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.y, f.sbase, f.sd, f.vd), f.tid, x);
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.z, f.sbase, f.sd, f.vd), f.tid, y);
#pragma unroll
	for (int r = 0; r < R; r++)
		x[r] = Math<T, OP>::eval(x[r], y[r]);
	store_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.w, f.sbase, f.sd, f.vd).addr, f.tid, x,
		(rec.x & OPH_SINGLE_DEF) ? 0xffffffffu : st.active);
}

/* Integer/Float into a register vector: active rows only */
template <int THREADS, int R>
__device__ __forceinline__ void f_setconst(const uint4 &rec, const FArgs &f, const RowState &st)
{
	uint32_t v[R];
	load_rows<uint32_t, THREADS, R>(opnd<4>(rec.y, f.sbase, f.sd, f.vd), f.tid, v);
	store_rows<uint32_t, THREADS, R>(opnd<4>(rec.w, f.sbase, f.sd, f.vd).addr, f.tid, v, st.active);
}

/* Column/Rowid into a register vector: every row (the CPU copies the whole
 * block, src/vm/virginia.c:448) */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_copy(const uint4 &rec, const FArgs &f)
{
	T x[R];
	load_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.y, f.sbase, f.sd, f.vd), f.tid, x);
	store_rows<T, THREADS, R>(opnd<sizeof(T)>(rec.w, f.sbase, f.sd, f.vd).addr, f.tid, x, 0xffffffffu);
}

/* operand type and operator tests on a record head */
__device__ __forceinline__ bool h_type(uint32_t h, int t) { return (h >> (OT_SHIFT + t)) & 1u; }
__device__ __forceinline__ bool h_op(uint32_t h, int o) { return (h >> (OO_SHIFT + o)) & 1u; }

template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_cmp_any(const uint4 &rec, const FArgs &f, RowState &st)
{
	const uint32_t h = rec.x;
	if (h_op(h, CO_LT)) f_cmp<T, CO_LT, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_GT)) f_cmp<T, CO_GT, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_LE)) f_cmp<T, CO_LE, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_GE)) f_cmp<T, CO_GE, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_EQ)) f_cmp<T, CO_EQ, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_NEQ)) f_cmp<T, CO_NEQ, THREADS, R>(rec, f, st);
	else if (h_op(h, CO_AND)) f_cmp<T, CO_AND, THREADS, R>(rec, f, st);
	else f_cmp<T, CO_OR, THREADS, R>(rec, f, st);
}

template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_math_any(const uint4 &rec, const FArgs &f, const RowState &st)
{
	const uint32_t h = rec.x;
	if (h_op(h, MO_ADD)) f_math<T, MO_ADD, THREADS, R>(rec, f, st);
	else if (h_op(h, MO_SUB)) f_math<T, MO_SUB, THREADS, R>(rec, f, st);
	else if (h_op(h, MO_MUL)) f_math<T, MO_MUL, THREADS, R>(rec, f, st);
	else f_math<T, MO_DIV, THREADS, R>(rec, f, st);
}

/* one filter op: kind, then type, then operator, each by bit tests */
template <int THREADS, int R>
__device__ __forceinline__ void filter_op(const uint4 &rec, const FArgs &f, RowState &st)
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
	if (h & OK_CMP) {
		if (h_type(h, VT_FLOAT)) f_cmp_any<float, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT)) f_cmp_any<int32_t, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_DOUBLE)) f_cmp_any<double, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT64)) f_cmp_any<long long, THREADS, R>(rec, f, st);
		else f_cmp_any<signed char, THREADS, R>(rec, f, st);
	} else if (h & OK_INVALID) {
		st.valid &= ~st.active;
	} else if (h & OK_MATH) {
		if (h_type(h, VT_FLOAT)) f_math_any<float, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT)) f_math_any<int32_t, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_DOUBLE)) f_math_any<double, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT64)) f_math_any<long long, THREADS, R>(rec, f, st);
		else f_math_any<signed char, THREADS, R>(rec, f, st);
	} else if (h & OK_NOT) {
		if (h_type(h, VT_FLOAT)) f_not<float, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT)) f_not<int32_t, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_DOUBLE)) f_not<double, THREADS, R>(rec, f, st);
		else if (h_type(h, VT_INT64)) f_not<long long, THREADS, R>(rec, f, st);
		else f_not<signed char, THREADS, R>(rec, f, st);
	} else if (h & OK_SETCONST) {
		f_setconst<THREADS, R>(rec, f, st);
	} else if (h & OK_COPY) {
		if (h_type(h, VT_INT64) || h_type(h, VT_DOUBLE)) f_copy<unsigned long long, THREADS, R>(rec, f);
		else if (h_type(h, VT_CHAR)) f_copy<unsigned char, THREADS, R>(rec, f);
		else f_copy<uint32_t, THREADS, R>(rec, f);
	}
}

/* ---- projection: the tile's selected rows, in row order ------------------
 * The projection warps share the tile's list: warp p takes the 32-entry
 * batches p, p + P, p + 2 P, ...; entry e is selection index e and its
 * result row lands at the tile's offset + e. */

struct PArgs {
	uint32_t sbase, sd, vd;
	uint32_t list;   /* smem address of the tile's list of tile rows (u16) */
	uint32_t n;      /* entries */
	uint32_t e0;     /* this lane's first entry */
	uint32_t step;   /* entries between this lane's entries: 32 P */
};

/* element address of a list entry */
__device__ __forceinline__ uint32_t p_addr(const Opnd &o, uint32_t row, uint32_t e)
{
	return o.addr + (o.sel ? e : row) * o.step;
}

template <typename T, int OP>
__device__ __forceinline__ void p_math(const uint4 &rec, const PArgs &c)
{
	const Opnd a = opnd<sizeof(T)>(rec.y, c.sbase, c.sd, c.vd);
	const Opnd b = opnd<sizeof(T)>(rec.z, c.sbase, c.sd, c.vd);
	const Opnd d = opnd<sizeof(T)>(rec.w, c.sbase, c.sd, c.vd);
	for (uint32_t e = c.e0; e < c.n; e += c.step) {
		const uint32_t row = lds_u16(c.list + 2 * e);
		const T x = SM<T>::ld(p_addr(a, row, e));
		const T y = SM<T>::ld(p_addr(b, row, e));
		SM<T>::st(p_addr(d, row, e), Math<T, OP>::eval(x, y));
	}
}

template <typename T>
__device__ __forceinline__ void p_copy(const uint4 &rec, const PArgs &c)
{
	const Opnd a = opnd<sizeof(T)>(rec.y, c.sbase, c.sd, c.vd);
	const Opnd d = opnd<sizeof(T)>(rec.w, c.sbase, c.sd, c.vd);
	for (uint32_t e = c.e0; e < c.n; e += c.step) {
		const uint32_t row = lds_u16(c.list + 2 * e);
		SM<T>::st(p_addr(d, row, e), SM<T>::ld(p_addr(a, row, e)));
	}
}

template <typename T>
__device__ __forceinline__ void p_math_any(const uint4 &rec, const PArgs &c)
{
	const uint32_t h = rec.x;
	if (h_op(h, MO_ADD)) p_math<T, MO_ADD>(rec, c);
	else if (h_op(h, MO_SUB)) p_math<T, MO_SUB>(rec, c);
	else if (h_op(h, MO_MUL)) p_math<T, MO_MUL>(rec, c);
	else p_math<T, MO_DIV>(rec, c);
}

/* one projection op: arithmetic, or a copy (every listed row is active
 * here, so constants and columns are copies) */
__device__ __forceinline__ void project_op(const uint4 &rec, const PArgs &c)
{
	const uint32_t h = rec.x;
	if (h & OK_MATH) {
		if (h_type(h, VT_FLOAT)) p_math_any<float>(rec, c);
		else if (h_type(h, VT_INT)) p_math_any<int32_t>(rec, c);
		else if (h_type(h, VT_DOUBLE)) p_math_any<double>(rec, c);
		else if (h_type(h, VT_INT64)) p_math_any<long long>(rec, c);
		else p_math_any<signed char>(rec, c);
	} else if (h & OK_SETCONST) {
		p_copy<uint32_t>(rec, c);
	} else if (h & OK_COPY) {
		if (h_type(h, VT_INT64) || h_type(h, VT_DOUBLE)) p_copy<unsigned long long>(rec, c);
		else if (h_type(h, VT_CHAR)) p_copy<unsigned char>(rec, c);
		else p_copy<uint32_t>(rec, c);
	}
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

/* rows the query wrote before its first tile: nonzero only for a query
 * continued from an earlier launch */
__device__ __forceinline__ uint64_t query_base(const QDesc &Q)
{
	return Q.base_in != nullptr ? *Q.base_in : 0ull;
}

/* the tile's own count, published by the last compute warp to finish its
 * ballots: an aggregate, or at once an inclusive prefix for a query's first
 * tile.  Publishing here, not in the sequencer, keeps one CTA's look-back
 * from delaying the counts that other CTAs' look-backs wait for. */
__device__ __forceinline__ void publish_count(const KParams &kp, const QDesc &Q, uint64_t g,
	uint32_t tile_total)
{
	const uint64_t ep = status_tag(kp, g) << kStatusEpochShift;
	if (g == Q.work_first)
		st_status(status_at(kp, g), ep | (kFlagPrefix << kStatusFlagShift) |
			((query_base(Q) + tile_total) & kStatusValueMask));
	else
		st_status(status_at(kp, g), ep | (kFlagAggregate << kStatusFlagShift) | tile_total);
}

/* Rows written by the query's tiles before tile g (its exclusive prefix):
 * walks back over earlier tiles' status words, kLookbackPerLane per lane
 * per round, summing aggregates up to the nearest inclusive prefix.  The
 * caller's own latest tile of the query (known, the index `known` with
 * inclusive prefix `known_end`, or none when known < the query's first
 * tile) is a prefix that needs no load, so the walk never passes it.  It
 * needs only the predecessors, so it runs while tile g itself is still being
 * filtered.  Returns false if a predecessor never published (bounded wait). */
constexpr int kLookbackPerLane = 4;

__device__ bool lookback_excl(const KParams &kp, const QDesc &Q, uint64_t g, int64_t known, uint64_t known_end,
	int lane, uint64_t *excl_out)
{
	constexpr int W = 32 * kLookbackPerLane;
	const int64_t first = (int64_t)Q.work_first;
	if ((int64_t)g == first) {
		*excl_out = query_base(Q);
		return true;
	}
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
				/* a stop: the known prefix, or nothing before the query */
				v[x] = (idx == known) ? (known_end & kStatusValueMask) : 0ull;
				stopbits |= 1u << x;
			} else {
				v[x] = ld_status(status_at(kp, (uint64_t)idx));
			}
		}
		/* wait until every loaded word carries this launch's epoch and a flag */
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

/* ---- producer: claims work items and stages their columns ---------------- */

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

/* the producer's copy of the current query's fields (every lane) and of one
 * staged column (lane i < nload holds column i) */
struct ProdQuery {
	const QDesc *Q;
	uint64_t first, end;         /* the query's work items */
	const SegDesc *segs;
	const uint32_t *tile_prefix;
	uint32_t nsegs, nload, qi, seg_hint;
	uint32_t src, stride, off;   /* this lane's column */
	/* the current segment: its tiles [seg_t0, seg_t1) of the query, rows,
	 * and this lane's column in it; seg ~0 when none */
	uint32_t seg, seg_t0, seg_t1, seg_rows;
	const unsigned char *colp;
};

/* one decoded work item; src and bytes are this lane's column copy */
struct ProdItem {
	uint32_t w, seg, row0, nrows;
	const unsigned char *src;
	uint32_t bytes;
};

/* decode work item w with the whole producer warp.  A CTA claims work items
 * in increasing order, so the query and segment searches start at the
 * previous item's. */
template <int TILE>
__device__ __forceinline__ void decode_item(const KParams &kp, uint32_t w, uint64_t total, uint32_t nq,
	ProdQuery &pq, ProdItem &it, int lane)
{
	it.w = w;
	it.bytes = 0;
	it.src = nullptr;
	if (w >= total)
		return;
	if (pq.Q == nullptr || w >= pq.end) {
		const uint32_t qi = warp_search(kp.q_work_prefix, pq.Q ? pq.qi : 0u, nq, w, lane);
		const QDesc *Q = kp.queries + qi;
		pq.Q = Q;
		pq.qi = qi;
		pq.first = Q->work_first;
		pq.end = pq.first + Q->ntiles;
		pq.segs = Q->segs;
		pq.tile_prefix = Q->seg_tile_prefix;
		pq.nsegs = Q->nsegs;
		pq.nload = Q->prog.nload;
		pq.seg_hint = 0;
		pq.seg = ~0u;
		if (lane < kMaxLoads) {
			pq.src = Q->prog.load_src[lane];
			pq.stride = Q->prog.load_stride[lane];
			pq.off = Q->load_off[lane];
		}
	}
	/* an item in the previous item's segment needs no load at all */
	const uint32_t t = (uint32_t)(w - pq.first);
	if (pq.seg == ~0u || t >= pq.seg_t1) {
		const uint32_t s = warp_search(pq.tile_prefix, pq.seg_hint, pq.nsegs, t, lane);
		const SegDesc *sd = pq.segs + s;
		pq.seg_hint = s;
		pq.seg = s;
		pq.seg_t0 = pq.tile_prefix[s];
		pq.seg_t1 = pq.tile_prefix[s + 1];
		pq.seg_rows = sd->rows;
		if ((uint32_t)lane < pq.nload)
			pq.colp = static_cast<const unsigned char *>(sd->col[pq.src]);
	}
	const uint32_t row0 = (t - pq.seg_t0) * TILE;
	it.seg = pq.seg;
	it.row0 = row0;
	it.nrows = min((uint32_t)TILE, pq.seg_rows - row0);
	if ((uint32_t)lane < pq.nload) {
		it.src = pq.colp + (size_t)row0 * pq.stride;
		it.bytes = (it.nrows * pq.stride + 15u) & ~15u;
	}
}

/* The producer warp fills the ring of stages.  Once the compute warps
 * released a stage it announces the decoded work item and issues its copies
 * (lane i copies column i; the query descriptor only when the stage does
 * not hold it already), then takes the next claim (in order, with the one
 * after it already in flight) and decodes it while those copies run.
 * Claiming a couple of items ahead, not a whole ring ahead, keeps claimed
 * tiles from idling while other CTAs' look-backs wait for their counts.
 * The claim and decode are the producer's serial path per tile, so the
 * claim's atomic round trip is overlapped and an item in the previous
 * item's segment is decoded without loads.  An invalid claim (past the end of the
 * work list) is announced without data and ends the CTA's pipeline.
 *
 * In a serving session the work list grows: a claim past the published
 * work waits for the host's doorbell (or its stop request), and each
 * released stage counts its tile as stored; the tile that completes a
 * query writes the query's completion record. */
template <int TILE>
__device__ void producer(const KParams &kp, unsigned char *smem, int lane)
{
	const volatile uint32_t *abort = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags) + kFAbort;
	uint32_t *held = reinterpret_cast<uint32_t *>(smem + kOffHeld);
	const uint32_t nst = kp.nstages;
	const bool serving = kp.serve != nullptr;
	/* published work and queries: fixed for a launch, growing (from none)
	 * in a serving session, whose kp.total_work only marks the end item */
	uint64_t total = serving ? 0ull : kp.total_work;
	uint32_t nq = serving ? 0u : kp.nq;
	uint32_t pend = 0;  /* serving: stages whose tile is issued but not yet counted */
	ProdQuery pq;
	pq.Q = nullptr;
	pq.qi = 0;
	/* claims: one atomic in flight (lane 0) while the previous claim's item
	 * is decoded and issued, so its round trip is off the per-tile path */
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
	/* serving: the tile of stage s is stored; the query's last one reports */
	auto count_stored = [&](uint32_t s) {
		const uint32_t qi = held[s];
		__threadfence();
		const unsigned done = atomicAdd(&kp.done_tiles[qi], 1u) + 1u;
		const QDesc *Q = kp.queries + qi;
		if (done == (unsigned)Q->ntiles) {
			__threadfence();
			const unsigned long long rows = *reinterpret_cast<volatile unsigned long long *>(Q->total_out);
			volatile ServeRec *r = kp.recs + qi;
			r->rows = rows;
			__threadfence_system();
			r->seq = (unsigned long long)qi + 1ull;
		}
	};
	/* serving: wait for the tiles issued in iterations lo..hi to be stored
	 * and count them (lane 0) */
	auto drain = [&](uint32_t lo, uint32_t hi) {
		for (uint32_t kk = lo; kk <= hi; kk++) {
			const uint32_t s = kk % nst;
			if ((pend >> s) & 1u) {
				if (!mbar_wait(smem_addr(smem + kOffEmpty + 8 * s), (kk / nst) & 1u, abort))
					return false;
				count_stored(s);
				pend &= ~(1u << s);
			}
		}
		return true;
	};
	/* the next work item: in a serving session a claim past the published
	 * work waits (bounded) for the doorbell; ~0 ends the pipeline */
	auto next_item = [&](uint32_t issued_k) -> uint32_t {
		const uint32_t w = claim();
		if (!serving || w < total)
			return w;
		uint64_t t0 = 0;
		int ok = 1;
		unsigned nap = 1000;  /* ns between doorbell polls, growing while idle */
		for (;;) {
			unsigned long long a = 0;
			unsigned stop = 0;
			if (lane == 0) {
				if (issued_k != ~0u && pend)
					ok = drain(issued_k + 1 > nst ? issued_k + 1 - nst : 0u, issued_k) ? 1 : 0;
				a = ld_acquire_sys(&kp.serve->avail);
				stop = *reinterpret_cast<const volatile unsigned *>(&kp.serve->stop);
			}
			ok = __shfl_sync(0xffffffffu, ok, 0);
			a = __shfl_sync(0xffffffffu, a, 0);
			stop = __shfl_sync(0xffffffffu, stop, 0);
			total = a & kAvailWorkMask;
			nq = (uint32_t)(a >> 40);
			if (w < total)
				return w;
			if (stop || !ok)
				return ~0u;
			if (t0 == 0)
				t0 = globaltimer_ns();
			else if (globaltimer_ns() - t0 > (uint64_t)kp.wait_limit_ms * 1000000ull) {
				if (lane == 0)
					report(kp.error, DE_STAGE_TIMEOUT);
				return ~0u;
			}
			__nanosleep(nap);
			nap = nap < 16000 ? nap * 2 : nap;
		}
	};
	ProdItem it;
	{
		/* claim first: next_item updates total and nq */
		const uint32_t w = next_item(~0u);
		decode_item<TILE>(kp, w, total, nq, pq, it, lane);
	}
	uint32_t k = 0;
	for (;; k++) {
		const uint32_t s = k % nst, j = k / nst;
		const uint32_t full = smem_addr(smem + kOffFull + 8 * s);
		const uint32_t empty = smem_addr(smem + kOffEmpty + 8 * s);
		if (j >= 1) {
			int ok = 1;
			if (lane == 0) {
				ok = mbar_wait(empty, (j - 1) & 1u, abort);
				if (!ok && !*abort)
					report(kp.error, DE_STAGE_TIMEOUT);
				if (ok && serving && ((pend >> s) & 1u)) {
					count_stored(s);
					pend &= ~(1u << s);
				}
			}
			if (!__shfl_sync(0xffffffffu, ok, 0))
				break;
		}
		unsigned char *hdr = smem + kp.stage_area + s * kp.stage_bytes;
		bool end = it.w >= total;
		if (!end && pq.Q == nullptr) {
			/* a work item without a decoded query: never copy from it */
			if (lane == 0)
				report(kp.error, DE_BAD_WORK);
			end = true;
		}
		if (lane == 0) {
			StageInfo si;
			si.work = end ? ~0u : it.w;
			si.query = pq.qi;
			si.seg = it.seg;
			si.row0 = it.row0;
			si.nrows = it.nrows;
			*reinterpret_cast<StageInfo *>(hdr + kQDescStaged) = si;
		}
		if (end) {
			/* serving: every issued tile is counted before the CTA ends */
			if (serving && lane == 0 && k > 0)
				drain(k > nst ? k - nst : 0u, k - 1);
			__syncwarp();
			if (lane == 0)
				mbar_arrive(full);
			return;
		}
		const bool copy_desc = held[s] != pq.qi;
		const uint32_t bytes = __reduce_add_sync(0xffffffffu, it.bytes) +
			(copy_desc ? (uint32_t)kQDescStaged : 0u);
		__syncwarp();
		if (lane == 0) {
			held[s] = pq.qi;
			pend |= 1u << s;
			fence_proxy_async_smem();
			mbar_arrive_expect_tx(full, bytes);
		}
		pend = __shfl_sync(0xffffffffu, pend, 0);
		__syncwarp();
		const uint32_t base = smem_addr(hdr);
		if (it.bytes)
			bulk_load(base + pq.off, it.src, it.bytes, full);
		if (copy_desc && lane == 31)
			bulk_load(base, pq.Q, (uint32_t)kQDescStaged, full);
		const uint32_t w = next_item(k);
		decode_item<TILE>(kp, w, total, nq, pq, it, lane);
	}
	/* abandoned: wait (bounded) for the copies already issued so none lands
	 * after the CTA exits */
	if (lane == 0) {
		const uint32_t first = k > nst ? k - nst : 0;
		for (uint32_t kk = first; kk < k; kk++)
			mbar_wait(smem_addr(smem + kOffFull + 8 * (kk % nst)), (kk / nst) & 1u, nullptr);
	}
}

/* ---- look-back warp: tile totals -> result offsets ----------------------- */

template <int THREADS, int R>
__device__ void lookback_warp(const KParams &kp, unsigned char *smem, int lane)
{
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	const volatile uint32_t *tot = reinterpret_cast<const volatile uint32_t *>(smem + kOffTot);
	uint64_t *offs = reinterpret_cast<uint64_t *>(smem + kOffOff);
	const uint32_t nst = kp.nstages;
	/* the previous tile of this CTA: a tile that directly follows it in the
	 * same query starts where it ended, with no look-back */
	uint64_t prev_work = ~0ull, prev_end = 0;
	for (uint32_t i = 0;; i++) {
		const uint32_t s = i % nst, q = i % kSlots;
		/* the tile's data has landed: its work item is known, so the walk
		 * over earlier tiles starts while the filter warps run */
		if (!mbar_wait(smem_addr(smem + kOffFull + 8 * s), (i / nst) & 1u, flags + kFAbort))
			return;
		/* the stage holds tile i until the tile's stores, which wait for
		 * this warp */
		const unsigned char *hdr = smem + kp.stage_area + s * kp.stage_bytes;
		const QDesc &Q = *reinterpret_cast<const QDesc *>(hdr);
		const StageInfo si = *reinterpret_cast<const StageInfo *>(hdr + kQDescStaged);
		if (si.work >= kp.total_work)
			return;
		uint64_t excl = 0;
		bool ok = true;
		const bool follows = si.work == prev_work + 1 && si.work != Q.work_first;
		if (follows)
			excl = prev_end;
		else
			ok = lookback_excl(kp, Q, si.work, prev_work == ~0ull ? -1 : (int64_t)prev_work, prev_end, lane, &excl);
		/* the tile's own count */
		if (ok && !mbar_wait(smem_addr(smem + kOffTready + 8 * q), (i / kSlots) & 1u, flags + kFAbort))
			return;
		const uint32_t tile_total = ok ? tot[q] : 0u;
		prev_work = si.work;
		prev_end = excl + tile_total;
		__syncwarp();
		if (lane == 0) {
			if (!ok) {
				report(kp.error, DE_LOOKBACK_TIMEOUT);
			} else {
				/* the inclusive prefix (a query's first tile published its own) */
				if (si.work != Q.work_first)
					st_status(status_at(kp, si.work),
						(status_tag(kp, si.work) << kStatusEpochShift) | (kFlagPrefix << kStatusFlagShift) |
						((excl + tile_total) & kStatusValueMask));
				if (si.work == Q.work_first + Q.ntiles - 1)
					*Q.total_out = excl + tile_total;
			}
			offs[q] = excl;
			flags[q] = ok ? 1u : 0u;
			if (!ok)
				flags[kFAbort] = 1u;
			mbar_arrive(smem_addr(smem + kOffOready + 8 * q));
		}
		if (!ok)
			return;
	}
}

/* ---- projection warps: projection and ordered stores of each tile -------- */

template <int THREADS, int R, int P>
__device__ void proj_warps(const KParams &kp, unsigned char *smem, int pw, int lane)
{
	constexpr int TILE = THREADS * R;
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	const uint32_t sbase = smem_addr(smem);
	const uint32_t nst = kp.nstages;
	for (uint32_t i = 0;; i++) {
		const uint32_t s = i % nst, q = i % kSlots;
		if (!mbar_wait(smem_addr(smem + kOffLready + 8 * q), (i / kSlots) & 1u, flags + kFAbort)) {
			if (lane == 0 && !flags[kFAbort]) {
				report(kp.error, DE_STAGE_TIMEOUT);
				flags[kFAbort] = 1u;
			}
			return;
		}
		if (flags[kFEnd] == i)
			return;
		const uint32_t sd = s * kp.stage_bytes;
		const uint32_t qd = sbase + kp.stage_area + sd;
		PArgs c;
		c.sbase = sbase;
		c.sd = sd;
		c.vd = q * lds_u32(qd + kQVecSlot);
		c.list = sbase + kp.sel_area + q * TILE * 2;
		c.n = lds_u32(sbase + kOffTot + 4 * q);
		c.e0 = 32u * (uint32_t)pw + (uint32_t)lane;
		c.step = 32u * P;
		const uint32_t ops = qd + kQOps;
		if (c.e0 - (uint32_t)lane < c.n) {
			const uint32_t nu = lds_u32(qd + kQNUops) - 1u;
			for (uint32_t k = lds_u32(qd + kQNFilter); k < nu; k++)
				project_op(lds_v4(ops + 16u * k), c);
		}

		/* ---- stores at the tile's offset, once the look-back resolved it */
		if (!mbar_wait(smem_addr(smem + kOffOready + 8 * q), (i / kSlots) & 1u, flags + kFAbort))
			return;
		if (!flags[q])
			return;
		const uint64_t off = lds_u64(sbase + kOffOff + 8 * q);
		if (c.e0 - (uint32_t)lane < c.n) {
			const uint64_t cap = lds_u64(qd + kQCapacity);
			bool overflow = false;
			const uint32_t nout = lds_u32(qd + kQNOut);
			for (uint32_t j = 0; j < nout; j++) {
				const uint32_t od = lds_u32(qd + kQOdOut + 4 * j);
				unsigned char *out = reinterpret_cast<unsigned char *>(lds_u64(qd + kQOutPtr + 8 * j));
				const uint32_t stride = lds_u8(qd + kQOutStride + j);
				const Opnd a = stride == 8 ? opnd<8>(od, sbase, sd, c.vd)
					: stride == 4 ? opnd<4>(od, sbase, sd, c.vd) : opnd<1>(od, sbase, sd, c.vd);
				uint32_t e0 = c.e0;
				if (stride == 4) {
					/* four entries per lane in flight: their list and value
					 * loads overlap */
					uint32_t *o32 = reinterpret_cast<uint32_t *>(out);
					for (; e0 + 3 * c.step < c.n && off + e0 + 3 * c.step < cap; e0 += 4 * c.step) {
						const uint32_t e1 = e0 + c.step, e2 = e1 + c.step, e3 = e2 + c.step;
						const uint32_t r0 = lds_u16(c.list + 2 * e0), r1 = lds_u16(c.list + 2 * e1);
						const uint32_t r2 = lds_u16(c.list + 2 * e2), r3 = lds_u16(c.list + 2 * e3);
						const uint32_t v0 = lds_u32(p_addr(a, r0, e0)), v1 = lds_u32(p_addr(a, r1, e1));
						const uint32_t v2 = lds_u32(p_addr(a, r2, e2)), v3 = lds_u32(p_addr(a, r3, e3));
						o32[off + e0] = v0;
						o32[off + e1] = v1;
						o32[off + e2] = v2;
						o32[off + e3] = v3;
					}
				}
				for (uint32_t e = e0; e < c.n; e += c.step) {
					const uint64_t pos = off + e;
					if (pos >= cap) {
						overflow = true;
						break;
					}
					const uint32_t at = p_addr(a, lds_u16(c.list + 2 * e), e);
					if (stride == 4)
						reinterpret_cast<uint32_t *>(out)[pos] = lds_u32(at);
					else if (stride == 8)
						reinterpret_cast<unsigned long long *>(out)[pos] = lds_u64(at);
					else
						out[pos] = (unsigned char)lds_u8(at);
				}
			}
			/* a serving session reports rows beyond capacity in the
			 * query's completion record instead */
			if (overflow && kp.serve == nullptr)
				report(kp.error, DE_OUTPUT_OVERFLOW);
		}
		__syncwarp();
		if (lane == 0) {
			mbar_arrive(smem_addr(smem + kOffEmpty + 8 * s));
			mbar_arrive(smem_addr(smem + kOffLfree + 8 * q));
		}
	}
}

/* projection warps per CTA: half the filter warps, 1 to 4 */
template <int THREADS>
struct ProjWarps {
	static constexpr int value = THREADS / 64 < 1 ? 1 : THREADS / 64 > 4 ? 4 : THREADS / 64;
};

template <int THREADS, int R>
__global__ void __launch_bounds__(THREADS + 32 * (2 + ProjWarps<THREADS>::value)) vm_kernel(const KParams kp)
{
	constexpr int TILE = THREADS * R;
	constexpr int NW = THREADS / 32;
	constexpr int C = R / 4;
	constexpr int P = ProjWarps<THREADS>::value;
	constexpr int G = 2 * C * NW;          /* 64-row groups per tile */
	constexpr int PER = (G + 31) / 32;
	static_assert(R % 4 == 0 && R <= 32, "rows per thread: whole 4-row chunks, 32-bit row masks");
	static_assert(G <= (int)kMaxGroups, "64-row groups per tile");
	static_assert(TILE <= 65536, "tile rows are 16-bit in the selection lists");
	extern __shared__ __align__(128) unsigned char smem[];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	const uint32_t nst = kp.nstages;

	if (tid == 0) {
		for (uint32_t s = 0; s < nst; s++) {
			mbar_init(smem_addr(smem + kOffFull + 8 * s), 1);
			mbar_init(smem_addr(smem + kOffEmpty + 8 * s), P);
		}
		for (uint32_t q = 0; q < kSlots; q++) {
			mbar_init(smem_addr(smem + kOffLready + 8 * q), NW);
			mbar_init(smem_addr(smem + kOffTready + 8 * q), 1);
			mbar_init(smem_addr(smem + kOffOready + 8 * q), 1);
			mbar_init(smem_addr(smem + kOffLfree + 8 * q), P);
			mbar_init(smem_addr(smem + kOffCdone + 8 * q), NW);
		}
		for (int x = 0; x < 8; x++)
			flags[x] = 0;
		flags[kFEnd] = ~0u;
		flags[kFWaitMs] = kp.wait_limit_ms;
		for (uint32_t s = 0; s < kMaxStages; s++)
			reinterpret_cast<uint32_t *>(smem + kOffHeld)[s] = ~0u;
		fence_mbar_init();
	}
	__syncthreads();
	if (warp == NW) {
		producer<TILE>(kp, smem, lane);
		return;
	}
	if (warp == NW + 1) {
		lookback_warp<THREADS, R>(kp, smem, lane);
		return;
	}
	if (warp >= NW + 2) {
		proj_warps<THREADS, R, P>(kp, smem, warp - (NW + 2), lane);
		return;
	}

	/* filter warps */
	const uint32_t sbase = smem_addr(smem);
	for (uint32_t i = 0;; i++) {
		const uint32_t s = i % nst, q = i % kSlots;
		/* the list and row-vector slot q are free once the projection of
		 * tile i - kSlots is done */
		bool ok = i < kSlots ||
			mbar_wait(smem_addr(smem + kOffLfree + 8 * q), ((i - kSlots) / kSlots) & 1u, flags + kFAbort);
		ok = ok && mbar_wait(smem_addr(smem + kOffFull + 8 * s), (i / nst) & 1u, flags + kFAbort);
		if (!ok) {
			if (lane == 0 && !flags[kFAbort]) {
				report(kp.error, DE_STAGE_TIMEOUT);
				flags[kFAbort] = 1u;
			}
			return;
		}
		const uint32_t sd = s * kp.stage_bytes;
		const uint32_t qd = sbase + kp.stage_area + sd;
		const uint32_t sinfo = qd + (uint32_t)kQDescStaged;
		if (lds_u32(sinfo + offsetof(StageInfo, work)) >= kp.total_work) {
			/* no more tiles: tell the look-back and projection warps */
			__syncwarp();
			if (lane == 0) {
				flags[kFEnd] = i;
				mbar_arrive(smem_addr(smem + kOffLready + 8 * q));
			}
			return;
		}
		const uint32_t nrows = lds_u32(sinfo + offsetof(StageInfo, nrows));
		const uint32_t vd = q * lds_u32(qd + kQVecSlot);

		/* ---- filter over every row */
		RowState st;
		st.valid = 0;
#pragma unroll
		for (int c = 0; c < C; c++)
#pragma unroll
			for (int k = 0; k < 4; k++)
				if (chunk_row<THREADS>(c, tid) + k < nrows)
					st.valid |= 1u << (4 * c + k);
		st.active = st.valid;
#pragma unroll
		for (int sl = 0; sl < kMaxSlots; sl++)
			st.pend[sl] = 0;
		{
			const uint32_t ops = qd + kQOps;
			const uint32_t nf = lds_u32(qd + kQNFilter);
			const FArgs f{sbase, sd, vd, tid};
			uint4 rec = lds_v4(ops);
			for (uint32_t k = 0; k < nf; k++) {
				const uint4 cur = rec;
				/* the next record's load overlaps this op */
				rec = lds_v4(ops + 16u * min(k + 1u, (uint32_t)kMaxOps - 1u));
				filter_op<THREADS, R>(cur, f, st);
			}
		}

		/* ---- counts per 64 rows, from four bit-plane ballots per 128-row
		 * chunk of the warp (row k of each lane's 4) */
		const uint32_t cnt = sbase + kOffCnt + q * kMaxGroups * 4;
		const uint32_t lt = (1u << lane) - 1u;
		uint32_t rank[C], total[C];
#pragma unroll
		for (int c = 0; c < C; c++) {
			const uint32_t m = (st.valid >> (4 * c)) & 0xfu;
			const uint32_t b0 = __ballot_sync(0xffffffffu, m & 1u);
			const uint32_t b1 = __ballot_sync(0xffffffffu, m & 2u);
			const uint32_t b2 = __ballot_sync(0xffffffffu, m & 4u);
			const uint32_t b3 = __ballot_sync(0xffffffffu, m & 8u);
			total[c] = __popc(b0) + __popc(b1) + __popc(b2) + __popc(b3);
			rank[c] = __popc(b0 & lt) + __popc(b1 & lt) + __popc(b2 & lt) + __popc(b3 & lt);
			if (lane == 0) {
				/* lanes 0-15 hold the chunk's first 64 rows */
				const uint32_t h0 = __popc(b0 & 0xffffu) + __popc(b1 & 0xffffu) + __popc(b2 & 0xffffu) +
					__popc(b3 & 0xffffu);
				sts_u32(cnt + 8 * (c * NW + warp), h0);
				sts_u32(cnt + 8 * (c * NW + warp) + 4, total[c] - h0);
			}
		}
		__syncwarp();
		if (lane == 0)
			mbar_arrive(smem_addr(smem + kOffCdone + 8 * q));
		if (!mbar_wait(smem_addr(smem + kOffCdone + 8 * q), (i / kSlots) & 1u, flags + kFAbort)) {
			if (lane == 0 && !flags[kFAbort]) {
				report(kp.error, DE_STAGE_TIMEOUT);
				flags[kFAbort] = 1u;
			}
			return;
		}

		/* ---- every warp scans the tile's counts: (chunk, warp, half) is row
		 * order, so a chunk's rows start at the sum of the counts before it */
		uint32_t loc[PER], lane_pre[PER];
		uint32_t sum = 0;
#pragma unroll
		for (int x = 0; x < PER; x++) {
			const int g = lane * PER + x;
			loc[x] = g < G ? lds_u32(cnt + 4 * g) : 0u;
			lane_pre[x] = sum;
			sum += loc[x];
		}
		uint32_t incl = sum;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
			if (lane >= d)
				incl += v;
		}
		const uint32_t ex = incl - sum;
		const uint32_t tile_total = __shfl_sync(0xffffffffu, incl, 31);

		/* ---- the tile's count: to the look-back words (before the list, so
		 * that other CTAs' look-backs see it as early as possible) and the
		 * other roles */
		if (warp == 0) {
			const unsigned char *hdr = smem + kp.stage_area + sd;
			const QDesc &Q = *reinterpret_cast<const QDesc *>(hdr);
			if (lane == 0) {
				publish_count(kp, Q, lds_u32(sinfo + offsetof(StageInfo, work)), tile_total);
				sts_u32(sbase + kOffTot + 4 * q, tile_total);
				mbar_arrive(smem_addr(smem + kOffTready + 8 * q));
			}
			/* valid rows per 64-row block, for result-tablet splitting on the
			 * host: group g covers tile rows 64 g .. 64 g + 63 */
			if (Q.block_counts != nullptr) {
				const StageInfo si = *reinterpret_cast<const StageInfo *>(hdr + kQDescStaged);
				for (int g = lane; g < G; g += 32)
					if (64u * (uint32_t)g < si.nrows)
						Q.block_counts[(uint64_t)Q.segs[si.seg].block_base + (si.row0 + 64u * g) / 64] =
							(uint8_t)lds_u32(cnt + 4 * g);
			}
		}
		/* ---- the tile-ordered list of selected rows */
		const uint32_t list = sbase + kp.sel_area + q * TILE * 2;
#pragma unroll
		for (int c = 0; c < C; c++) {
			const uint32_t g = 2u * (uint32_t)(c * NW + warp);
			uint32_t v = 0;
#pragma unroll
			for (int x = 0; x < PER; x++)
				if ((uint32_t)x == g % PER)
					v = ex + lane_pre[x];
			const uint32_t base = __shfl_sync(0xffffffffu, v, (int)(g / PER));
			if (total[c]) {
				const uint32_t m = (st.valid >> (4 * c)) & 0xfu;
				uint32_t at = base + rank[c];
				const uint32_t row0 = chunk_row<THREADS>(c, tid);
#pragma unroll
				for (int k = 0; k < 4; k++)
					if ((m >> k) & 1u)
						sts_u16(list + 2 * at++, row0 + k);
			}
		}

		__syncwarp();
		if (lane == 0)
			mbar_arrive(smem_addr(smem + kOffLready + 8 * q));
	}
}

/* ---- host-side launcher ------------------------------------------------ */

template <int THREADS, int R>
static int launch_t(const KParams &kp, unsigned grid, size_t smem, cudaStream_t stream)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	/* THREADS filter threads, the producer and look-back warps and the projection warps */
	fn<<<grid, THREADS + 32 * (2 + ProjWarps<THREADS>::value), smem, stream>>>(kp);
	return cudaGetLastError() == cudaSuccess;
}

template <int THREADS, int R>
static int occ_t(size_t smem, int *ctas)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, THREADS + 32 * (2 + ProjWarps<THREADS>::value), smem) == cudaSuccess;
}

#define VGPU_SHAPES(X) X(128, 4) X(128, 8) X(128, 16) X(256, 4) X(256, 8) X(256, 16) X(512, 4) X(512, 8)

int shape_supported(const Shape &s)
{
#define X(T, R) if (s.threads == T && s.rows_per_thread == R) return 1;
	VGPU_SHAPES(X)
#undef X
	return 0;
}

int launch_vm(const Shape &s, const KParams &kp, unsigned grid, size_t smem, void *stream)
{
#define X(T, R) \
	if (s.threads == T && s.rows_per_thread == R) return launch_t<T, R>(kp, grid, smem, (cudaStream_t)stream);
	VGPU_SHAPES(X)
#undef X
	return 0;
}

int occupancy(const Shape &s, size_t smem, int *ctas)
{
#define X(T, R) if (s.threads == T && s.rows_per_thread == R) return occ_t<T, R>(smem, ctas);
	VGPU_SHAPES(X)
#undef X
	return 0;
}

}  // namespace vgpu
