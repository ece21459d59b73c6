/*
 * The sm_100a data-parallel VM kernel.
 *
 * Replaces the reference's virginia_gpu (src/vm/vm_gpu.cu:1152-1225), which
 * runs one thread per row with a 16-entry register file in local memory, a
 * switch dispatch per op per thread and atomics for (unordered) result
 * placement.  Here a CTA is a three-role pipeline over tiles of
 * TILE = THREADS x R rows, tied together by mbarriers:
 *
 *  - producer warp: claims work items (one tile of one segment of one query)
 *    from a global counter, in order, and copies the tile's columns plus the
 *    query's descriptor into a ring of shared-memory stages with TMA bulk
 *    copies (cp.async.bulk completing on the stage's full barrier);
 *  - compute warps: filter every row of the tile (row state as bit masks:
 *    valid, active, and rows parked at pending jump targets), compact each
 *    warp's valid rows into a selection list (__ballot_sync/__popc), run the
 *    projection (result expressions) on listed rows only, then store the
 *    previous tile's rows at their final positions and release its stage;
 *  - sequencer warp: for each tile, scans the (row group, warp) counts and
 *    resolves the tile's position in the query's result with a warp-wide
 *    decoupled look-back over earlier tiles (32 status words per round),
 *    one tile ahead of the stores, so cross-CTA waits overlap computation.
 *
 * Rows land in original row order (the single-core CPU VM's order,
 * src/vm/virginia.c:476-578) with plain stores; no output atomics.
 * Arithmetic matches the CPU VM bit for bit: float/double use the _rn
 * intrinsics (no FMA contraction, IEEE division) and x86 NaN results,
 * integers wrap as on x86.  Every wait is bounded; on expiry the kernel
 * records an error code and stops instead of hanging.
 */
#include <cstdint>
#include <climits>

#include <cuda_runtime.h>

#include "vgpu_engine.h"

namespace vgpu {

/* bounded waits: iterations of ~100 ns and more, far beyond any real wait */
constexpr unsigned kStageSpinLimit = 1u << 24;
constexpr unsigned kLookbackSpinLimit = 1u << 24;

/* work items claimed per atomic by the producer */
constexpr unsigned kClaim = 1;

/* shared memory header (kSmemHeader bytes) */
constexpr unsigned kMaxGroups = 128;  /* R x warps */
constexpr unsigned kOffFull = 0;                           /* mbarrier[kMaxStages] */
constexpr unsigned kOffEmpty = kOffFull + 8 * kMaxStages;  /* mbarrier[kMaxStages] */
constexpr unsigned kOffCready = kOffEmpty + 8 * kMaxStages; /* mbarrier[2]: counts ready */
constexpr unsigned kOffOready = kOffCready + 16;           /* mbarrier[2]: offsets ready */
constexpr unsigned kOffOff = kOffOready + 16;              /* uint64[2]: tile offsets */
constexpr unsigned kOffFlags = kOffOff + 16;               /* uint32[4]: ok[2], abort */
constexpr unsigned kOffAgg = kOffFlags + 16;               /* uint64[2]: warps arrived | count */
constexpr unsigned kOffHeld = kOffAgg + 16;                /* uint32[kMaxStages]: query per stage */
constexpr unsigned kOffCnt = 256;                          /* uint32[2][kMaxGroups] */
constexpr unsigned kOffPre = kOffCnt + 8 * kMaxGroups;     /* uint32[2][kMaxGroups] */
static_assert(kOffHeld + 4 * kMaxStages <= kOffCnt, "smem header layout");
static_assert(kOffPre + 8 * kMaxGroups <= kSmemHeader, "smem header overflow");
static_assert(sizeof(QDesc) % 16 == 0, "QDesc copies in 16-byte chunks");
static_assert(kStageHdr >= sizeof(QDesc) + sizeof(StageInfo), "stage header too small");

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

__device__ __forceinline__ void report(unsigned *error, unsigned code)
{
	atomicCAS(error, 0u, code);
}

/* bounded wait for an mbarrier phase; false on timeout or when the CTA's
 * abort flag is set */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, const volatile uint32_t *abort)
{
	for (unsigned i = 0; i < kStageSpinLimit; i++) {
		if (mbar_try_wait(bar, phase))
			return true;
		if (abort && *abort)
			return false;
		if (i > 8)
			__nanosleep(i < 64 ? 32 : 128);
	}
	return false;
}

/* ---- operand access ---------------------------------------------------- */

/* element i of an operand is at p + i * step (step 0: a broadcast scalar) */
struct Acc {
	unsigned char *p;
	uint32_t step;
	bool sel;  /* indexed by selection position instead of tile row */
};

/* staged columns and the scalar table live in the stage; register vectors
 * in the tile's vector slot */
template <typename T>
__device__ __forceinline__ Acc acc_of(unsigned char *smem, uint32_t od, uint32_t stage_delta,
	uint32_t vec_delta)
{
	Acc a;
	const uint32_t kind = od & ~OD_OFFSET;
	const bool in_stage = kind == OD_STAGE || kind == OD_SCALAR;
	a.p = smem + (od & OD_OFFSET) + (in_stage ? stage_delta : vec_delta);
	a.step = kind == OD_SCALAR ? 0u : (uint32_t)sizeof(T);
	a.sel = kind == OD_SELVEC;
	return a;
}

template <typename T>
__device__ __forceinline__ T ld_at(const Acc &a, uint32_t i)
{
	return *reinterpret_cast<const T *>(a.p + i * a.step);
}

template <typename T>
__device__ __forceinline__ void st_at(const Acc &a, uint32_t i, T v)
{
	*reinterpret_cast<T *>(a.p + i * a.step) = v;
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

struct FCtx {
	unsigned char *smem;
	const QDesc *Q;
	uint32_t stage_delta;
	uint32_t vec_delta;
	int tid;
};

/* rows in `jumped` leave the active set, park in the op's target slot and,
 * for a jump with p4 == 0, stop being valid (src/vm/virginia.c:59-63) */
__device__ __forceinline__ void take_jump(RowState &st, const UOp &u, uint32_t jumped)
{
	st.active &= ~jumped;
	if (!u.vjump)
		st.valid &= ~jumped;
#pragma unroll
	for (int s = 0; s < kMaxSlots; s++)
		if (u.tslot == s)
			st.pend[s] |= jumped;
}

template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void f_cmp(const FCtx &c, const UOp &u, uint32_t k, RowState &st)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc b = acc_of<T>(c.smem, c.Q->od_b[k], c.stage_delta, c.vec_delta);
	uint32_t bits = 0;
	if (b.step == 0) {
		/* column or vector against a scalar: the common WHERE shape */
		const T y = ld_at<T>(b, 0);
#pragma unroll
		for (int r = 0; r < R; r++)
			bits |= (uint32_t)cmp_eval<T, OP>(ld_at<T>(a, r * THREADS + c.tid), y) << r;
	} else {
#pragma unroll
		for (int r = 0; r < R; r++) {
			const uint32_t row = r * THREADS + c.tid;
			bits |= (uint32_t)cmp_eval<T, OP>(ld_at<T>(a, row), ld_at<T>(b, row)) << r;
		}
	}
	take_jump(st, u, st.active & bits);
}

template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_not(const FCtx &c, const UOp &u, uint32_t k, RowState &st)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	uint32_t bits = 0;
#pragma unroll
	for (int r = 0; r < R; r++)
		bits |= (uint32_t)(ld_at<T>(a, r * THREADS + c.tid) == T(0)) << r;
	take_jump(st, u, st.active & bits);
}

template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void f_math(const FCtx &c, const UOp &u, uint32_t k, const RowState &st)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc b = acc_of<T>(c.smem, c.Q->od_b[k], c.stage_delta, c.vec_delta);
	const Acc d = acc_of<T>(c.smem, c.Q->od_d[k], c.stage_delta, c.vec_delta);
	const uint32_t store = (u.flags & UF_SINGLE_DEF) ? 0xffffffffu : st.active;
#pragma unroll
	for (int r = 0; r < R; r++) {
		const uint32_t row = r * THREADS + c.tid;
		const T z = Math<T, OP>::eval(ld_at<T>(a, row), ld_at<T>(b, row));
		if ((store >> r) & 1u)
			st_at<T>(d, row, z);
	}
}

/* Integer/Float into a vector register: active rows only */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_setconst(const FCtx &c, uint32_t k, const RowState &st)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc d = acc_of<T>(c.smem, c.Q->od_d[k], c.stage_delta, c.vec_delta);
	const T v = ld_at<T>(a, 0);
#pragma unroll
	for (int r = 0; r < R; r++)
		if ((st.active >> r) & 1u)
			st_at<T>(d, r * THREADS + c.tid, v);
}

/* Column/Rowid into a vector register: every row (the CPU copies the whole
 * block, src/vm/virginia.c:448) */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void f_copycol(const FCtx &c, uint32_t k)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc d = acc_of<T>(c.smem, c.Q->od_d[k], c.stage_delta, c.vec_delta);
#pragma unroll
	for (int r = 0; r < R; r++) {
		const uint32_t row = r * THREADS + c.tid;
		st_at<T>(d, row, ld_at<T>(a, row));
	}
}

template <int THREADS, int R>
__device__ __forceinline__ void filter_op(const FCtx &c, const UOp &u, uint32_t k, RowState &st)
{
	if (u.join) {
#pragma unroll
		for (int s = 0; s < kMaxSlots; s++)
			if ((u.join >> s) & 1u) {
				st.active |= st.pend[s];
				st.pend[s] = 0;
			}
	}
#define VGPU_CMP_CASES(T, TY)                                                        \
	case TY * 8 + CO_LE: f_cmp<T, CO_LE, THREADS, R>(c, u, k, st); break;           \
	case TY * 8 + CO_LT: f_cmp<T, CO_LT, THREADS, R>(c, u, k, st); break;           \
	case TY * 8 + CO_GE: f_cmp<T, CO_GE, THREADS, R>(c, u, k, st); break;           \
	case TY * 8 + CO_GT: f_cmp<T, CO_GT, THREADS, R>(c, u, k, st); break;           \
	case TY * 8 + CO_EQ: f_cmp<T, CO_EQ, THREADS, R>(c, u, k, st); break;           \
	case TY * 8 + CO_NEQ: f_cmp<T, CO_NEQ, THREADS, R>(c, u, k, st); break;         \
	case TY * 8 + CO_AND: f_cmp<T, CO_AND, THREADS, R>(c, u, k, st); break;         \
	case TY * 8 + CO_OR: f_cmp<T, CO_OR, THREADS, R>(c, u, k, st); break;
#define VGPU_MATH_CASES(T, TY)                                                 \
	case TY * 8 + MO_ADD: f_math<T, MO_ADD, THREADS, R>(c, u, k, st); break;  \
	case TY * 8 + MO_SUB: f_math<T, MO_SUB, THREADS, R>(c, u, k, st); break;  \
	case TY * 8 + MO_MUL: f_math<T, MO_MUL, THREADS, R>(c, u, k, st); break;  \
	case TY * 8 + MO_DIV: f_math<T, MO_DIV, THREADS, R>(c, u, k, st); break;
	switch (u.kind) {
	case UK_CMP:
		switch (u.type * 8 + u.sub) {
			VGPU_CMP_CASES(int32_t, VT_INT)
			VGPU_CMP_CASES(long long, VT_INT64)
			VGPU_CMP_CASES(float, VT_FLOAT)
			VGPU_CMP_CASES(double, VT_DOUBLE)
			VGPU_CMP_CASES(signed char, VT_CHAR)
		default: break;
		}
		break;
	case UK_MATH:
		switch (u.type * 8 + u.sub) {
			VGPU_MATH_CASES(int32_t, VT_INT)
			VGPU_MATH_CASES(long long, VT_INT64)
			VGPU_MATH_CASES(float, VT_FLOAT)
			VGPU_MATH_CASES(double, VT_DOUBLE)
			VGPU_MATH_CASES(signed char, VT_CHAR)
		default: break;
		}
		break;
	case UK_NOT:
		switch (u.type) {
		case VT_INT: f_not<int32_t, THREADS, R>(c, u, k, st); break;
		case VT_INT64: f_not<long long, THREADS, R>(c, u, k, st); break;
		case VT_FLOAT: f_not<float, THREADS, R>(c, u, k, st); break;
		case VT_DOUBLE: f_not<double, THREADS, R>(c, u, k, st); break;
		default: f_not<signed char, THREADS, R>(c, u, k, st); break;
		}
		break;
	case UK_INVALID:
		st.valid &= ~st.active;
		break;
	case UK_SETCONST:
		f_setconst<uint32_t, THREADS, R>(c, k, st);
		break;
	case UK_COPYCOL:
		switch (u.type) {
		case VT_INT64:
		case VT_DOUBLE: f_copycol<unsigned long long, THREADS, R>(c, k); break;
		case VT_CHAR: f_copycol<unsigned char, THREADS, R>(c, k); break;
		default: f_copycol<uint32_t, THREADS, R>(c, k); break;
		}
		break;
	default:
		break;
	}
#undef VGPU_CMP_CASES
#undef VGPU_MATH_CASES
}

/* ---- projection: only the rows in the warp's selection list ------------- */

/* lane `lane` of a warp handles the warp's selection entries lane + 32 i,
 * i < R; their tile rows are held in registers for the whole projection */
template <int R>
struct PCtx {
	unsigned char *smem;
	const QDesc *Q;
	uint32_t stage_delta;
	uint32_t vec_delta;
	uint32_t n;            /* entries in the warp's list */
	uint32_t sel_base;     /* this warp's first selection-vector index */
	int lane;
	uint32_t row[R];       /* tile rows of this lane's entries */
};

template <typename T>
__device__ __forceinline__ T p_ld(const Acc &a, uint32_t row, uint32_t sidx)
{
	return ld_at<T>(a, a.sel ? sidx : row);
}

template <typename T>
__device__ __forceinline__ void p_st(const Acc &a, uint32_t row, uint32_t sidx, T v)
{
	st_at<T>(a, a.sel ? sidx : row, v);
}

template <typename T, int OP, int R>
__device__ __forceinline__ void p_math(const PCtx<R> &c, uint32_t k)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc b = acc_of<T>(c.smem, c.Q->od_b[k], c.stage_delta, c.vec_delta);
	const Acc d = acc_of<T>(c.smem, c.Q->od_d[k], c.stage_delta, c.vec_delta);
#pragma unroll
	for (int i = 0; i < R; i++) {
		const uint32_t e = c.lane + 32 * i;
		if (32 * i >= c.n)
			break;
		if (e < c.n) {
			const uint32_t si = c.sel_base + e;
			p_st<T>(d, c.row[i], si,
				Math<T, OP>::eval(p_ld<T>(a, c.row[i], si), p_ld<T>(b, c.row[i], si)));
		}
	}
}

template <typename T, int R>
__device__ __forceinline__ void p_copy(const PCtx<R> &c, uint32_t k)
{
	const Acc a = acc_of<T>(c.smem, c.Q->od_a[k], c.stage_delta, c.vec_delta);
	const Acc d = acc_of<T>(c.smem, c.Q->od_d[k], c.stage_delta, c.vec_delta);
#pragma unroll
	for (int i = 0; i < R; i++) {
		const uint32_t e = c.lane + 32 * i;
		if (32 * i >= c.n)
			break;
		if (e < c.n) {
			const uint32_t si = c.sel_base + e;
			p_st<T>(d, c.row[i], si, p_ld<T>(a, c.row[i], si));
		}
	}
}

template <int R>
__device__ __forceinline__ void project_op(const PCtx<R> &c, const UOp &u, uint32_t k)
{
#define VGPU_PMATH_CASES(T, TY)                                      \
	case TY * 8 + MO_ADD: p_math<T, MO_ADD, R>(c, k); break;        \
	case TY * 8 + MO_SUB: p_math<T, MO_SUB, R>(c, k); break;        \
	case TY * 8 + MO_MUL: p_math<T, MO_MUL, R>(c, k); break;        \
	case TY * 8 + MO_DIV: p_math<T, MO_DIV, R>(c, k); break;
	switch (u.kind) {
	case UK_MATH:
		switch (u.type * 8 + u.sub) {
			VGPU_PMATH_CASES(int32_t, VT_INT)
			VGPU_PMATH_CASES(long long, VT_INT64)
			VGPU_PMATH_CASES(float, VT_FLOAT)
			VGPU_PMATH_CASES(double, VT_DOUBLE)
			VGPU_PMATH_CASES(signed char, VT_CHAR)
		default: break;
		}
		break;
	case UK_SETCONST:
	case UK_COPYCOL:
		/* every listed row is active here, so both copy their source */
		switch (u.type) {
		case VT_INT64:
		case VT_DOUBLE: p_copy<unsigned long long, R>(c, k); break;
		case VT_CHAR: p_copy<unsigned char, R>(c, k); break;
		default: p_copy<uint32_t, R>(c, k); break;
		}
		break;
	default:
		break;
	}
#undef VGPU_PMATH_CASES
}

/* ---- ordered placement ------------------------------------------------- */

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
	for (int d = 16; d > 0; d >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, d);
	return v;
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
	const uint64_t ep = (uint64_t)kp.epoch << kStatusEpochShift;
	if (g == Q.work_first)
		st_status(&kp.status[g], ep | (kFlagPrefix << kStatusFlagShift) |
			((query_base(Q) + tile_total) & kStatusValueMask));
	else
		st_status(&kp.status[g], ep | (kFlagAggregate << kStatusFlagShift) | tile_total);
}

/* find the rows written by the query's earlier tiles and publish this
 * tile's inclusive prefix.  Each round reads 32 predecessors' status words;
 * it stops at the nearest one that carries an inclusive prefix.  Returns
 * false if a predecessor never published (bounded wait). */
__device__ bool lookback(const KParams &kp, const QDesc &Q, uint64_t g, uint32_t tile_total,
	int lane, uint64_t *excl_out)
{
	const uint64_t first = Q.work_first;
	const uint64_t ep = (uint64_t)kp.epoch << kStatusEpochShift;
	if (g == first) {
		*excl_out = query_base(Q);
		return true;
	}
	uint64_t excl = 0;
	int64_t j = (int64_t)g - 1;
	unsigned spins = 0;
	while (true) {
		const int64_t idx = j - lane;
		const bool inrange = idx >= (int64_t)first;
		uint64_t v = 0;
		bool ready = !inrange;
		if (inrange) {
			v = ld_status(&kp.status[idx]);
			ready = (v >> kStatusEpochShift) == kp.epoch && ((v >> kStatusFlagShift) & 3u);
		}
		while (!__all_sync(0xffffffffu, ready)) {
			if (++spins > kLookbackSpinLimit)
				return false;
			__nanosleep(spins < 64 ? 32 : 256);
			if (!ready) {
				v = ld_status(&kp.status[idx]);
				ready = (v >> kStatusEpochShift) == kp.epoch && ((v >> kStatusFlagShift) & 3u);
			}
		}
		const bool is_prefix = !inrange || ((v >> kStatusFlagShift) & 3u) == kFlagPrefix;
		const uint32_t pm = __ballot_sync(0xffffffffu, is_prefix);
		const uint64_t val = inrange ? (v & kStatusValueMask) : 0ull;
		if (pm) {
			const int stop = __ffs(pm) - 1;
			excl += warp_sum_u64(lane <= stop ? val : 0ull);
			break;
		}
		excl += warp_sum_u64(val);
		j -= 32;
	}
	if (lane == 0)
		st_status(&kp.status[g],
			ep | (kFlagPrefix << kStatusFlagShift) | ((excl + tile_total) & kStatusValueMask));
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
__device__ __forceinline__ void decode_item(const KParams &kp, uint32_t w, ProdQuery &pq, ProdItem &it,
	int lane)
{
	it.w = w;
	it.bytes = 0;
	it.src = nullptr;
	if (w >= kp.total_work)
		return;
	if (pq.Q == nullptr || w >= pq.end) {
		const uint32_t qi = warp_search(kp.q_work_prefix, pq.Q ? pq.qi : 0u, kp.nq, w, lane);
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
		if (lane < kMaxLoads) {
			pq.src = Q->prog.load_src[lane];
			pq.stride = Q->prog.load_stride[lane];
			pq.off = Q->load_off[lane];
		}
	}
	const uint64_t t = w - pq.first;
	const uint32_t s = warp_search(pq.tile_prefix, pq.seg_hint, pq.nsegs, t, lane);
	pq.seg_hint = s;
	const SegDesc *sd = pq.segs + s;
	const uint32_t row0 = (uint32_t)(t - pq.tile_prefix[s]) * TILE;
	it.seg = s;
	it.row0 = row0;
	it.nrows = min((uint32_t)TILE, sd->rows - row0);
	if ((uint32_t)lane < pq.nload) {
		it.src = static_cast<const unsigned char *>(sd->col[pq.src]) + (size_t)row0 * pq.stride;
		it.bytes = (it.nrows * pq.stride + 15u) & ~15u;
	}
}

/* The producer warp fills the ring of stages.  Once the compute warps
 * released a stage it announces the decoded work item and issues its copies
 * (lane i copies column i; the query descriptor only when the stage does
 * not hold it already), then claims (kClaim per atomic, in order) and
 * decodes the next item while those copies run.  Claiming one item ahead,
 * not a whole ring ahead, keeps claimed tiles from idling while other CTAs'
 * look-backs wait for their counts.  An invalid claim (past the end of the
 * work list) is announced without data and ends the CTA's pipeline. */
template <int TILE>
__device__ void producer(const KParams &kp, unsigned char *smem, int lane)
{
	const volatile uint32_t *abort = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags) + 2;
	uint32_t *held = reinterpret_cast<uint32_t *>(smem + kOffHeld);
	const uint32_t nst = kp.nstages;
	ProdQuery pq;
	pq.Q = nullptr;
	pq.qi = 0;
	uint32_t next = 0, left = 0;
	auto claim = [&]() -> uint32_t {
		if (left == 0) {
			uint32_t v = 0;
			if (lane == 0)
				v = atomicAdd(kp.counter, kClaim);
			next = __shfl_sync(0xffffffffu, v, 0);
			left = kClaim;
		}
		left--;
		return next++;
	};
	ProdItem it;
	decode_item<TILE>(kp, claim(), pq, it, lane);
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
			}
			if (!__shfl_sync(0xffffffffu, ok, 0))
				break;
		}
		unsigned char *hdr = smem + kp.stage_area + s * kp.stage_bytes;
		if (lane == 0) {
			StageInfo si;
			si.work = it.w;
			si.query = pq.qi;
			si.seg = it.seg;
			si.row0 = it.row0;
			si.nrows = it.nrows;
			*reinterpret_cast<StageInfo *>(hdr + sizeof(QDesc)) = si;
		}
		if (it.w >= kp.total_work) {
			__syncwarp();
			if (lane == 0)
				mbar_arrive(full);
			return;
		}
		const bool copy_desc = held[s] != pq.qi;
		const uint32_t total = __reduce_add_sync(0xffffffffu, it.bytes) +
			(copy_desc ? (uint32_t)sizeof(QDesc) : 0u);
		__syncwarp();
		if (lane == 0) {
			held[s] = pq.qi;
			fence_proxy_async_smem();
			mbar_arrive_expect_tx(full, total);
		}
		__syncwarp();
		const uint32_t base = smem_addr(hdr);
		if (it.bytes)
			bulk_load(base + pq.off, it.src, it.bytes, full);
		if (copy_desc && lane == 31)
			bulk_load(base, pq.Q, (uint32_t)sizeof(QDesc), full);
		decode_item<TILE>(kp, claim(), pq, it, lane);
	}
	/* abandoned: wait (bounded) for the copies already issued so none lands
	 * after the CTA exits */
	if (lane == 0) {
		const uint32_t first = k > nst ? k - nst : 0;
		for (uint32_t kk = first; kk < k; kk++)
			mbar_wait(smem_addr(smem + kOffFull + 8 * (kk % nst)), (kk / nst) & 1u, nullptr);
	}
}

/* ---- sequencer: counts -> tile offsets ----------------------------------- */

template <int THREADS, int R>
__device__ void sequencer(const KParams &kp, unsigned char *smem, int lane)
{
	constexpr int NW = THREADS / 32;
	constexpr int G = R * NW;
	constexpr int PER = (G + 31) / 32;
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	uint64_t *offs = reinterpret_cast<uint64_t *>(smem + kOffOff);
	const uint32_t nst = kp.nstages;
	/* the previous tile of this CTA: a tile that directly follows it in the
	 * same query starts where it ended, with no look-back */
	uint64_t prev_work = ~0ull, prev_end = 0;
	for (uint32_t i = 0;; i++) {
		const uint32_t s = i % nst, q = i & 1u;
		if (!mbar_wait(smem_addr(smem + kOffFull + 8 * s), (i / nst) & 1u, flags + 2))
			return;
		const unsigned char *hdr = smem + kp.stage_area + s * kp.stage_bytes;
		const QDesc &Q = *reinterpret_cast<const QDesc *>(hdr);
		const StageInfo si = *reinterpret_cast<const StageInfo *>(hdr + sizeof(QDesc));
		if (si.work >= kp.total_work)
			return;
		if (!mbar_wait(smem_addr(smem + kOffCready + 8 * q), (i >> 1) & 1u, flags + 2))
			return;
		const uint32_t *cnt = reinterpret_cast<const uint32_t *>(smem + kOffCnt) + q * kMaxGroups;
		uint32_t *pre = reinterpret_cast<uint32_t *>(smem + kOffPre) + q * kMaxGroups;
		/* exclusive scan over groups in (row group, warp) = row order */
		uint32_t local[PER];
		uint32_t sum = 0;
#pragma unroll
		for (int x = 0; x < PER; x++) {
			const int gi = lane * PER + x;
			local[x] = gi < G ? cnt[gi] : 0u;
			sum += local[x];
		}
		uint32_t incl = sum;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
			if (lane >= d)
				incl += v;
		}
		uint32_t run = incl - sum;
#pragma unroll
		for (int x = 0; x < PER; x++) {
			const int gi = lane * PER + x;
			if (gi < G)
				pre[gi] = run;
			run += local[x];
		}
		const uint32_t tile_total = __shfl_sync(0xffffffffu, incl, 31);
		uint64_t excl = 0;
		bool ok = true;
		if (si.work == prev_work + 1 && si.work != Q.work_first) {
			excl = prev_end;
			if (lane == 0)
				st_status(&kp.status[si.work],
					((uint64_t)kp.epoch << kStatusEpochShift) | (kFlagPrefix << kStatusFlagShift) |
					((excl + tile_total) & kStatusValueMask));
		} else {
			ok = lookback(kp, Q, si.work, tile_total, lane, &excl);
		}
		prev_work = si.work;
		prev_end = excl + tile_total;
		/* valid rows per 64-row block, for result-tablet splitting on the host */
		if (Q.block_counts != nullptr) {
			for (int b = lane; b < R * (THREADS / 64); b += 32) {
				const int r = b / (THREADS / 64), m = b % (THREADS / 64);
				const uint32_t local_row = r * THREADS + m * 64;
				if (local_row < si.nrows) {
					const uint64_t blk =
						(uint64_t)Q.segs[si.seg].block_base + (si.row0 + local_row) / 64;
					Q.block_counts[blk] = (uint8_t)(cnt[r * NW + 2 * m] + cnt[r * NW + 2 * m + 1]);
				}
			}
		}
		__syncwarp();
		if (lane == 0) {
			if (!ok)
				report(kp.error, DE_LOOKBACK_TIMEOUT);
			else if (si.work == Q.work_first + Q.ntiles - 1)
				*Q.total_out = excl + tile_total;
			offs[q] = excl;
			flags[q] = ok ? 1u : 0u;
			if (!ok)
				flags[2] = 1u;
			mbar_arrive(smem_addr(smem + kOffOready + 8 * q));
		}
		if (!ok)
			return;
	}
}

/* ---- compute warps: stores of a finished tile ---------------------------- */

template <int THREADS, int R>
__device__ __forceinline__ bool store_tile(const KParams &kp, unsigned char *smem, uint32_t p,
	uint32_t nsel, int warp, int lane)
{
	constexpr int NW = THREADS / 32;
	constexpr int TILE = THREADS * R;
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	const uint32_t s = p % kp.nstages, q = p & 1u;
	if (!mbar_wait(smem_addr(smem + kOffOready + 8 * q), (p >> 1) & 1u, flags + 2))
		return false;
	if (!flags[q])
		return false;
	const uint64_t off = reinterpret_cast<const uint64_t *>(smem + kOffOff)[q];
	const uint32_t *pre = reinterpret_cast<const uint32_t *>(smem + kOffPre) + q * kMaxGroups;
	const uint32_t stage_delta = s * kp.stage_bytes, vec_delta = q * kp.vec_bytes;
	const QDesc &Q = *reinterpret_cast<const QDesc *>(smem + kp.stage_area + stage_delta);
	const uint16_t *list = reinterpret_cast<const uint16_t *>(smem + kp.sel_area) + q * 2 * TILE +
		warp * 32 * R;
	const uint16_t *tag = list + TILE;
	uint32_t row[R];
	uint64_t pos[R];
	bool overflow = false;
#pragma unroll
	for (int i = 0; i < R; i++) {
		const uint32_t e = lane + 32 * i;
		pos[i] = ~0ull;
		row[i] = 0;
		if (e < nsel) {
			row[i] = list[e];
			const uint32_t t = tag[e];
			pos[i] = off + pre[(t >> 5) * NW + warp] + (t & 31u);
			if (pos[i] >= Q.capacity) {
				overflow = true;
				pos[i] = ~0ull;
			}
		}
	}
	const uint32_t sel_base = warp * 32 * R;
	const uint32_t nout = Q.prog.nout;
	for (uint32_t j = 0; j < nout; j++) {
		const uint32_t od = Q.od_out[j];
		void *out = Q.out_ptr[j];
		switch (Q.prog.out_stride[j]) {
		case 4: {
			const Acc a = acc_of<uint32_t>(smem, od, stage_delta, vec_delta);
#pragma unroll
			for (int i = 0; i < R; i++)
				if (pos[i] != ~0ull)
					reinterpret_cast<uint32_t *>(out)[pos[i]] =
						p_ld<uint32_t>(a, row[i], sel_base + lane + 32 * i);
			break;
		}
		case 8: {
			const Acc a = acc_of<unsigned long long>(smem, od, stage_delta, vec_delta);
#pragma unroll
			for (int i = 0; i < R; i++)
				if (pos[i] != ~0ull)
					reinterpret_cast<unsigned long long *>(out)[pos[i]] =
						p_ld<unsigned long long>(a, row[i], sel_base + lane + 32 * i);
			break;
		}
		default: {
			const Acc a = acc_of<unsigned char>(smem, od, stage_delta, vec_delta);
#pragma unroll
			for (int i = 0; i < R; i++)
				if (pos[i] != ~0ull)
					reinterpret_cast<unsigned char *>(out)[pos[i]] =
						p_ld<unsigned char>(a, row[i], sel_base + lane + 32 * i);
			break;
		}
		}
	}
	if (overflow)
		report(kp.error, DE_OUTPUT_OVERFLOW);
	__syncwarp();
	if (lane == 0)
		mbar_arrive(smem_addr(smem + kOffEmpty + 8 * s));
	return true;
}

template <int THREADS, int R>
__global__ void __launch_bounds__(THREADS + 64) vm_kernel(const KParams kp)
{
	constexpr int TILE = THREADS * R;
	constexpr int NW = THREADS / 32;
	constexpr int G = R * NW;
	static_assert(R <= 32 && G <= (int)kMaxGroups, "row masks are 32-bit");
	extern __shared__ __align__(128) unsigned char smem[];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	volatile uint32_t *flags = reinterpret_cast<volatile uint32_t *>(smem + kOffFlags);
	const uint32_t nst = kp.nstages;

	if (tid == 0) {
		for (uint32_t s = 0; s < nst; s++) {
			mbar_init(smem_addr(smem + kOffFull + 8 * s), 1);
			mbar_init(smem_addr(smem + kOffEmpty + 8 * s), NW);
		}
		for (uint32_t q = 0; q < 2; q++) {
			mbar_init(smem_addr(smem + kOffCready + 8 * q), NW);
			mbar_init(smem_addr(smem + kOffOready + 8 * q), 1);
		}
		flags[0] = flags[1] = flags[2] = 0;
		reinterpret_cast<unsigned long long *>(smem + kOffAgg)[0] = 0ull;
		reinterpret_cast<unsigned long long *>(smem + kOffAgg)[1] = 0ull;
		for (uint32_t s = 0; s < kMaxStages; s++)
			reinterpret_cast<uint32_t *>(smem + kOffHeld)[s] = ~0u;
		fence_mbar_init();
	}
	__syncthreads();
	if (warp == NW + 1) {
		producer<TILE>(kp, smem, lane);
		return;
	}
	if (warp == NW) {
		sequencer<THREADS, R>(kp, smem, lane);
		return;
	}

	/* compute warps */
	uint32_t prev_nsel = 0;
	uint32_t i = 0;
	for (;; i++) {
		const uint32_t s = i % nst, q = i & 1u;
		if (!mbar_wait(smem_addr(smem + kOffFull + 8 * s), (i / nst) & 1u, flags + 2)) {
			if (lane == 0 && !flags[2]) {
				report(kp.error, DE_STAGE_TIMEOUT);
				flags[2] = 1u;
			}
			return;
		}
		const uint32_t stage_delta = s * kp.stage_bytes, vec_delta = q * kp.vec_bytes;
		unsigned char *hdr = smem + kp.stage_area + stage_delta;
		const QDesc *Q = reinterpret_cast<const QDesc *>(hdr);
		const StageInfo si = *reinterpret_cast<const StageInfo *>(hdr + sizeof(QDesc));
		if (si.work >= kp.total_work)
			break;

		/* ---- filter over every row */
		RowState st;
		st.valid = 0;
#pragma unroll
		for (int r = 0; r < R; r++)
			if ((uint32_t)(r * THREADS + tid) < si.nrows)
				st.valid |= 1u << r;
		st.active = st.valid;
#pragma unroll
		for (int sl = 0; sl < kMaxSlots; sl++)
			st.pend[sl] = 0;
		{
			FCtx fc{smem, Q, stage_delta, vec_delta, tid};
			const uint32_t nf = Q->prog.nfilter;
			for (uint32_t k = 0; k < nf; k++)
				filter_op<THREADS, R>(fc, Q->prog.uops[k], k, st);
		}

		/* ---- selection: ballots, this warp's list of valid rows */
		uint16_t *list = reinterpret_cast<uint16_t *>(smem + kp.sel_area) + q * 2 * TILE +
			warp * 32 * R;
		uint16_t *tag = list + TILE;
		uint32_t *cnt = reinterpret_cast<uint32_t *>(smem + kOffCnt) + q * kMaxGroups;
		uint32_t nsel = 0;
		{
			const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
			for (int r = 0; r < R; r++) {
				const uint32_t bal = __ballot_sync(0xffffffffu, (st.valid >> r) & 1u);
				if ((st.valid >> r) & 1u) {
					const uint32_t rank = __popc(bal & lt);
					list[nsel + rank] = (uint16_t)(r * THREADS + tid);
					/* group and rank: the entry's place in the result */
					tag[nsel + rank] = (uint16_t)(r * 32 + rank);
				}
				nsel += __popc(bal);
				if (lane == 0)
					cnt[r * NW + warp] = __popc(bal);
			}
		}
		__syncwarp();
		if (lane == 0) {
			/* the last warp to add its count publishes the tile's total; the
			 * counter is next used two tiles on, after the sequencer has
			 * consumed this tile, so the last warp can clear it */
			unsigned long long *agg = reinterpret_cast<unsigned long long *>(smem + kOffAgg) + q;
			const unsigned long long old = atomicAdd(agg, (1ull << 32) | nsel);
			if ((uint32_t)(old >> 32) == NW - 1) {
				*agg = 0ull;
				publish_count(kp, *Q, si.work, (uint32_t)old + nsel);
			}
			mbar_arrive(smem_addr(smem + kOffCready + 8 * q));
		}

		/* ---- projection over this warp's selection list */
		{
			PCtx<R> pc{smem, Q, stage_delta, vec_delta, nsel, (uint32_t)(warp * 32 * R), lane, {}};
#pragma unroll
			for (int x = 0; x < R; x++) {
				const uint32_t e = lane + 32 * x;
				pc.row[x] = e < nsel ? list[e] : 0u;
			}
			const uint32_t nu = Q->prog.nuops - 1;
			for (uint32_t k = Q->prog.nfilter; k < nu; k++)
				project_op<R>(pc, Q->prog.uops[k], k);
		}
		__syncwarp();

		/* ---- stores of the previous tile, whose offset is resolved by now */
		if (i > 0 && !store_tile<THREADS, R>(kp, smem, i - 1, prev_nsel, warp, lane))
			return;
		prev_nsel = nsel;
	}
	if (i > 0)
		store_tile<THREADS, R>(kp, smem, i - 1, prev_nsel, warp, lane);
}

/* ---- host-side launcher ------------------------------------------------ */

template <int THREADS, int R>
static int launch_t(const KParams &kp, unsigned grid, size_t smem, cudaStream_t stream)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	/* THREADS compute threads, the sequencer warp and the producer warp */
	fn<<<grid, THREADS + 64, smem, stream>>>(kp);
	return cudaGetLastError() == cudaSuccess;
}

template <int THREADS, int R>
static int occ_t(size_t smem, int *ctas)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, THREADS + 64, smem) == cudaSuccess;
}

#define VGPU_SHAPES(X) X(128, 8) X(128, 16) X(256, 4) X(256, 8) X(256, 16) X(512, 4) X(512, 8)

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
