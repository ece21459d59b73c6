/*
 * The sm_100a data-parallel VM kernel.
 *
 * Replaces the reference's virginia_gpu (src/vm/vm_gpu.cu:1152-1225), which
 * runs one thread per row with a 16-entry register file in local memory, a
 * switch dispatch per op per thread and atomics for (unordered) result
 * placement.  Design here:
 *
 *  - persistent CTAs pull work items (one tile of TILE = THREADS x R rows of
 *    one segment of one query) from a global counter, so look-back
 *    predecessors are always held by running CTAs;
 *  - the columns a program reads are staged tile by tile into shared memory
 *    with TMA bulk copies (cp.async.bulk + mbarrier transaction counts) in a
 *    ring of `nstages` buffers, so the next tiles stream from HBM while the
 *    current one is interpreted;
 *  - each thread owns rows tid, tid + THREADS, ... of the tile and keeps
 *    their pending jump targets and validity bits in registers; the program
 *    (decoded uops, in shared memory) is interpreted warp-uniformly, so
 *    dispatch costs are paid once per R rows; column registers alias the
 *    staged tile, scalar registers are broadcast from shared memory and other
 *    registers are per-row vectors in shared memory;
 *  - Result: valid rows are ranked with __ballot_sync/__popc, a block scan
 *    over (row group, warp) orders them, and a decoupled look-back over the
 *    query's earlier tiles gives the tile's global offset, so rows land in
 *    original order (the single-core CPU VM's order, src/vm/virginia.c:476-578)
 *    with no atomics on the output.
 *
 * Arithmetic matches the CPU VM bit for bit: float/double use the _rn
 * intrinsics (no FMA contraction, IEEE division), integers wrap as on x86.
 * Every wait (stage barrier, look-back flag) is bounded; on expiry the kernel
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

/* shared memory header layout (kSmemHeader bytes) */
constexpr unsigned kOffMbar = 2048;
constexpr unsigned kOffStage = kOffMbar + 8 * kMaxStages;
constexpr unsigned kOffCnt = kOffStage + sizeof(StageInfo) * kMaxStages;
constexpr unsigned kMaxGroups = 128;  /* R x warps */
constexpr unsigned kOffPre = kOffCnt + 4 * kMaxGroups;
constexpr unsigned kOffBcast = kOffPre + 4 * kMaxGroups;
static_assert(sizeof(QDesc) <= kOffMbar, "QDesc must fit the smem header");
static_assert(sizeof(QDesc) % 16 == 0, "QDesc copies in 16-byte chunks");
static_assert(kOffBcast + 64 <= kSmemHeader, "smem header overflow");

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

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t *p)
{
	uint64_t v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void st_release_u64(uint64_t *p, uint64_t v)
{
	asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void report(unsigned *error, unsigned code)
{
	atomicCAS(error, 0u, code);
}

/* ---- operand access ---------------------------------------------------- */

struct Ctx {
	unsigned char *stage;  /* current stage buffer */
	unsigned char *vec;    /* register vectors */
	const QDesc *Q;        /* shared-memory copy of the query descriptor */
};

/* element `row` of an operand is p[row * step]: step 0 broadcasts a scalar
 * register (little-endian low bytes of its 8-byte slot) */
template <typename T>
struct Src {
	const T *p;
	int step;
};

template <typename T>
__device__ __forceinline__ Src<T> src_of(const Ctx &c, uint8_t cls, uint8_t idx)
{
	Src<T> s;
	if (cls == OC_COL) {
		s.p = reinterpret_cast<const T *>(c.stage + c.Q->load_off[idx]);
		s.step = 1;
	} else if (cls == OC_VEC) {
		s.p = reinterpret_cast<const T *>(c.vec + c.Q->vec_off[idx]);
		s.step = 1;
	} else {
		s.p = reinterpret_cast<const T *>(&c.Q->prog.consts[idx]);
		s.step = 0;
	}
	return s;
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

template <int OP>
struct Math<float, OP> {
	static __device__ __forceinline__ float eval(float a, float b)
	{
		if (OP == MO_ADD) return __fadd_rn(a, b);
		if (OP == MO_SUB) return __fsub_rn(a, b);
		if (OP == MO_MUL) return __fmul_rn(a, b);
		return __fdiv_rn(a, b);
	}
};

template <int OP>
struct Math<double, OP> {
	static __device__ __forceinline__ double eval(double a, double b)
	{
		if (OP == MO_ADD) return __dadd_rn(a, b);
		if (OP == MO_SUB) return __dsub_rn(a, b);
		if (OP == MO_MUL) return __dmul_rn(a, b);
		return __ddiv_rn(a, b);
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

template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void run_cmp(const Ctx &c, const UOp &u, int tid, uint8_t (&wait)[R],
	uint32_t &vmask)
{
	const Src<T> a = src_of<T>(c, u.a_cls, u.a_idx);
	const Src<T> b = src_of<T>(c, u.b_cls, u.b_idx);
	T x[R], y[R];
#pragma unroll
	for (int r = 0; r < R; r++) {
		const int row = r * THREADS + tid;
		x[r] = a.p[row * a.step];
		y[r] = b.p[row * b.step];
	}
#pragma unroll
	for (int r = 0; r < R; r++) {
		if (wait[r] <= u.pc && cmp_eval<T, OP>(x[r], y[r])) {
			if (!u.vjump)
				vmask &= ~(1u << r);
			wait[r] = u.target;
		}
	}
}

template <typename T, int OP, int THREADS, int R>
__device__ __forceinline__ void run_math(const Ctx &c, const UOp &u, int tid, const uint8_t (&wait)[R])
{
	const Src<T> a = src_of<T>(c, u.a_cls, u.a_idx);
	const Src<T> b = src_of<T>(c, u.b_cls, u.b_idx);
	T *d = reinterpret_cast<T *>(c.vec + c.Q->vec_off[u.dst]);
	T x[R], y[R];
#pragma unroll
	for (int r = 0; r < R; r++) {
		const int row = r * THREADS + tid;
		x[r] = a.p[row * a.step];
		y[r] = b.p[row * b.step];
	}
#pragma unroll
	for (int r = 0; r < R; r++) {
		const T z = Math<T, OP>::eval(x[r], y[r]);
		if (wait[r] <= u.pc)
			d[r * THREADS + tid] = z;
	}
}

template <typename T, int THREADS, int R>
__device__ __forceinline__ void run_not(const Ctx &c, const UOp &u, int tid, uint8_t (&wait)[R],
	uint32_t &vmask)
{
	const Src<T> a = src_of<T>(c, u.a_cls, u.a_idx);
#pragma unroll
	for (int r = 0; r < R; r++) {
		const T x = a.p[(r * THREADS + tid) * a.step];
		if (wait[r] <= u.pc && x == T(0)) {
			if (!u.vjump)
				vmask &= ~(1u << r);
			wait[r] = u.target;
		}
	}
}

/* Integer/Float into a vector register: active rows only */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void run_setconst(const Ctx &c, const UOp &u, int tid, const uint8_t (&wait)[R])
{
	const T v = *reinterpret_cast<const T *>(&c.Q->prog.consts[u.a_idx]);
	T *d = reinterpret_cast<T *>(c.vec + c.Q->vec_off[u.dst]);
#pragma unroll
	for (int r = 0; r < R; r++)
		if (wait[r] <= u.pc)
			d[r * THREADS + tid] = v;
}

/* Column/Rowid into a vector register: every row (the CPU copies the whole
 * block, src/vm/virginia.c:448) */
template <typename T, int THREADS, int R>
__device__ __forceinline__ void run_copycol(const Ctx &c, const UOp &u, int tid)
{
	const T *s = reinterpret_cast<const T *>(c.stage + c.Q->load_off[u.a_idx]);
	T *d = reinterpret_cast<T *>(c.vec + c.Q->vec_off[u.dst]);
#pragma unroll
	for (int r = 0; r < R; r++)
		d[r * THREADS + tid] = s[r * THREADS + tid];
}

template <int THREADS, int R>
__device__ __forceinline__ void dispatch(const Ctx &c, const UOp &u, int tid, uint8_t (&wait)[R],
	uint32_t &vmask)
{
#define VGPU_CMP_CASES(T, TY)                                                           \
	case TY * 8 + CO_LE: run_cmp<T, CO_LE, THREADS, R>(c, u, tid, wait, vmask); break;   \
	case TY * 8 + CO_LT: run_cmp<T, CO_LT, THREADS, R>(c, u, tid, wait, vmask); break;   \
	case TY * 8 + CO_GE: run_cmp<T, CO_GE, THREADS, R>(c, u, tid, wait, vmask); break;   \
	case TY * 8 + CO_GT: run_cmp<T, CO_GT, THREADS, R>(c, u, tid, wait, vmask); break;   \
	case TY * 8 + CO_EQ: run_cmp<T, CO_EQ, THREADS, R>(c, u, tid, wait, vmask); break;   \
	case TY * 8 + CO_NEQ: run_cmp<T, CO_NEQ, THREADS, R>(c, u, tid, wait, vmask); break; \
	case TY * 8 + CO_AND: run_cmp<T, CO_AND, THREADS, R>(c, u, tid, wait, vmask); break; \
	case TY * 8 + CO_OR: run_cmp<T, CO_OR, THREADS, R>(c, u, tid, wait, vmask); break;
#define VGPU_MATH_CASES(T, TY)                                                   \
	case TY * 8 + MO_ADD: run_math<T, MO_ADD, THREADS, R>(c, u, tid, wait); break; \
	case TY * 8 + MO_SUB: run_math<T, MO_SUB, THREADS, R>(c, u, tid, wait); break; \
	case TY * 8 + MO_MUL: run_math<T, MO_MUL, THREADS, R>(c, u, tid, wait); break; \
	case TY * 8 + MO_DIV: run_math<T, MO_DIV, THREADS, R>(c, u, tid, wait); break;

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
		case VT_INT: run_not<int32_t, THREADS, R>(c, u, tid, wait, vmask); break;
		case VT_INT64: run_not<long long, THREADS, R>(c, u, tid, wait, vmask); break;
		case VT_FLOAT: run_not<float, THREADS, R>(c, u, tid, wait, vmask); break;
		case VT_DOUBLE: run_not<double, THREADS, R>(c, u, tid, wait, vmask); break;
		default: run_not<signed char, THREADS, R>(c, u, tid, wait, vmask); break;
		}
		break;
	case UK_INVALID:
#pragma unroll
		for (int r = 0; r < R; r++)
			if (wait[r] <= u.pc)
				vmask &= ~(1u << r);
		break;
	case UK_SETCONST:
		if (u.type == VT_INT || u.type == VT_FLOAT)
			run_setconst<uint32_t, THREADS, R>(c, u, tid, wait);
		break;
	case UK_COPYCOL:
		switch (u.type) {
		case VT_INT64:
		case VT_DOUBLE: run_copycol<unsigned long long, THREADS, R>(c, u, tid); break;
		case VT_CHAR: run_copycol<unsigned char, THREADS, R>(c, u, tid); break;
		default: run_copycol<uint32_t, THREADS, R>(c, u, tid); break;
		}
		break;
	default:
		break;
	}
#undef VGPU_CMP_CASES
#undef VGPU_MATH_CASES
}

/* ---- ordered result emission ----------------------------------------- */

template <int THREADS, int R>
__device__ __forceinline__ bool emit_result(const Ctx &c, const KParams &kp, const StageInfo &si,
	uint32_t vmask, unsigned char *smem, int tid)
{
	constexpr int NW = THREADS / 32;
	const QDesc &Q = *c.Q;
	const int lane = tid & 31, warp = tid >> 5;
	uint32_t *cnt = reinterpret_cast<uint32_t *>(smem + kOffCnt);
	uint32_t *pre = reinterpret_cast<uint32_t *>(smem + kOffPre);
	volatile uint32_t *bc = reinterpret_cast<volatile uint32_t *>(smem + kOffBcast);

	uint32_t bal[R];
#pragma unroll
	for (int r = 0; r < R; r++) {
		bal[r] = __ballot_sync(0xffffffffu, (vmask >> r) & 1u);
		if (lane == 0)
			cnt[r * NW + warp] = __popc(bal[r]);
	}
	__syncthreads();

	/* exclusive scan over groups in (row group, warp) order = row order */
	constexpr int G = R * NW;
	constexpr int PER = (G + 31) / 32;
	if (warp == 0) {
		uint32_t local[PER];
		uint32_t sum = 0;
#pragma unroll
		for (int i = 0; i < PER; i++) {
			const int g = lane * PER + i;
			local[i] = g < G ? cnt[g] : 0u;
			sum += local[i];
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
		for (int i = 0; i < PER; i++) {
			const int g = lane * PER + i;
			if (g < G)
				pre[g] = run;
			run += local[i];
		}
		if (lane == 31)
			bc[0] = incl;
	}
	__syncthreads();
	const uint32_t tile_total = bc[0];

	/* decoupled look-back over this query's earlier tiles */
	if (tid == 0) {
		const uint64_t g = si.work;
		const uint64_t first = Q.work_first;
		const uint64_t ep = (uint64_t)kp.epoch << kStatusEpochShift;
		uint64_t excl = 0;
		bool ok = true;
		if (g == first) {
			/* a query continued from an earlier launch starts at its row count */
			if (Q.base_in != nullptr)
				excl = *Q.base_in;
			st_release_u64(&kp.status[g],
				ep | (kFlagPrefix << kStatusFlagShift) | ((excl + tile_total) & kStatusValueMask));
		} else {
			st_release_u64(&kp.status[g], ep | (kFlagAggregate << kStatusFlagShift) | tile_total);
			uint64_t j = g - 1;
			while (true) {
				uint64_t v = 0;
				unsigned spins = 0;
				while (true) {
					v = ld_acquire_u64(&kp.status[j]);
					if ((v >> kStatusEpochShift) == kp.epoch && ((v >> kStatusFlagShift) & 3u))
						break;
					if (++spins > kLookbackSpinLimit) {
						ok = false;
						break;
					}
					__nanosleep(spins < 64 ? 32 : 256);
				}
				if (!ok)
					break;
				excl += v & kStatusValueMask;
				if (((v >> kStatusFlagShift) & 3u) == kFlagPrefix || j == first)
					break;
				j--;
			}
			if (ok)
				st_release_u64(&kp.status[g],
					ep | (kFlagPrefix << kStatusFlagShift) | ((excl + tile_total) & kStatusValueMask));
			else
				report(kp.error, DE_LOOKBACK_TIMEOUT);
		}
		if (ok && g == first + Q.ntiles - 1)
			*Q.total_out = excl + tile_total;
		bc[1] = (uint32_t)excl;
		bc[2] = (uint32_t)(excl >> 32);
		bc[3] = ok ? 1u : 0u;
	}
	__syncthreads();
	const bool ok = bc[3] != 0;
	const uint64_t off = (uint64_t)bc[1] | ((uint64_t)bc[2] << 32);

	/* valid rows per 64-row block, for result-tablet splitting on the host */
	if (Q.block_counts != nullptr && tid < R * (THREADS / 64)) {
		const int r = tid / (THREADS / 64), m = tid % (THREADS / 64);
		const uint32_t local_row = r * THREADS + m * 64;
		if (local_row < si.nrows) {
			const SegDesc *sd = Q.segs + si.seg;
			const uint64_t blk = (uint64_t)sd->block_base + (si.row0 + local_row) / 64;
			Q.block_counts[blk] = (uint8_t)(cnt[r * NW + 2 * m] + cnt[r * NW + 2 * m + 1]);
		}
	}
	if (!ok)
		return false;

	const uint32_t lt_mask = (1u << lane) - 1u;
	bool overflow = false;
#pragma unroll
	for (int r = 0; r < R; r++) {
		if (!((vmask >> r) & 1u))
			continue;
		const uint64_t pos = off + pre[r * NW + warp] + __popc(bal[r] & lt_mask);
		if (pos >= Q.capacity) {
			overflow = true;
			continue;
		}
		const int row = r * THREADS + tid;
		for (uint32_t j = 0; j < Q.prog.nout; j++) {
			const uint8_t cls = Q.prog.out_cls[j], idx = Q.prog.out_idx[j];
			switch (Q.prog.out_stride[j]) {
			case 4: {
				const Src<uint32_t> s = src_of<uint32_t>(c, cls, idx);
				reinterpret_cast<uint32_t *>(Q.out_ptr[j])[pos] = s.p[row * s.step];
				break;
			}
			case 8: {
				const Src<unsigned long long> s = src_of<unsigned long long>(c, cls, idx);
				reinterpret_cast<unsigned long long *>(Q.out_ptr[j])[pos] = s.p[row * s.step];
				break;
			}
			default: {
				const Src<unsigned char> s = src_of<unsigned char>(c, cls, idx);
				reinterpret_cast<unsigned char *>(Q.out_ptr[j])[pos] = s.p[row * s.step];
				break;
			}
			}
		}
	}
	if (overflow)
		report(kp.error, DE_OUTPUT_OVERFLOW);
	return true;
}

/* ---- work decoding and staging (one thread) --------------------------- */

template <int TILE>
__device__ void claim_and_issue(const KParams &kp, unsigned char *smem, int s)
{
	StageInfo *st = reinterpret_cast<StageInfo *>(smem + kOffStage) + s;
	const uint32_t w = atomicAdd(kp.counter, 1u);
	st->work = w;
	if (w >= kp.total_work)
		return;
	/* query: last q with q_work_prefix[q] <= w */
	uint32_t lo = 0, hi = kp.nq;
	while (hi - lo > 1) {
		const uint32_t mid = (lo + hi) / 2;
		if (kp.q_work_prefix[mid] <= w) lo = mid; else hi = mid;
	}
	const QDesc *Q = kp.queries + lo;
	const uint64_t t = w - Q->work_first;
	/* segment: last s with seg_tile_prefix[s] <= t */
	uint32_t slo = 0, shi = Q->nsegs;
	while (shi - slo > 1) {
		const uint32_t mid = (slo + shi) / 2;
		if (Q->seg_tile_prefix[mid] <= t) slo = mid; else shi = mid;
	}
	const SegDesc *sd = Q->segs + slo;
	const uint32_t row0 = (uint32_t)(t - Q->seg_tile_prefix[slo]) * TILE;
	const uint32_t nrows = min((uint32_t)TILE, sd->rows - row0);
	st->query = lo;
	st->seg = slo;
	st->row0 = row0;
	st->nrows = nrows;

	const uint32_t bar = smem_addr(smem + kOffMbar + 8 * s);
	const uint32_t base = smem_addr(smem + kp.stage_area + (uint32_t)s * kp.stage_bytes);
	uint32_t total = 0;
	const uint32_t nload = Q->prog.nload;
	for (uint32_t i = 0; i < nload; i++)
		total += (nrows * Q->prog.load_stride[i] + 15u) & ~15u;
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(bar, total);
	for (uint32_t i = 0; i < nload; i++) {
		const uint32_t stride = Q->prog.load_stride[i];
		const unsigned char *src =
			static_cast<const unsigned char *>(sd->col[Q->prog.load_src[i]]) + (size_t)row0 * stride;
		bulk_load(base + Q->load_off[i], src, (nrows * stride + 15u) & ~15u, bar);
	}
}

/* after an abort at iteration `it`, wait (bounded) for the bulk copies the
 * CTA already issued into the other stages so none lands after exit */
__device__ void drain_stages(const KParams &kp, unsigned char *smem, uint32_t it)
{
	const StageInfo *stage_info = reinterpret_cast<const StageInfo *>(smem + kOffStage);
	const uint32_t nst = kp.nstages;
	for (uint32_t d = 1; d < nst; d++) {
		const uint32_t it2 = it + d, s2 = it2 % nst;
		if (stage_info[s2].work >= kp.total_work)
			continue;
		const uint32_t bar = smem_addr(smem + kOffMbar + 8 * s2);
		for (unsigned i = 0; i < kStageSpinLimit; i++) {
			if (mbar_try_wait(bar, (it2 / nst) & 1u))
				break;
			__nanosleep(64);
		}
	}
}

template <int THREADS, int R>
__global__ void __launch_bounds__(THREADS) vm_kernel(const KParams kp)
{
	constexpr int TILE = THREADS * R;
	extern __shared__ __align__(128) unsigned char smem[];
	const int tid = threadIdx.x;
	QDesc *Q = reinterpret_cast<QDesc *>(smem + kSmemQDesc);
	StageInfo *stage_info = reinterpret_cast<StageInfo *>(smem + kOffStage);
	const uint32_t nst = kp.nstages;

	if (tid == 0) {
		for (uint32_t s = 0; s < nst; s++)
			mbar_init(smem_addr(smem + kOffMbar + 8 * s), 1);
		fence_mbar_init();
	}
	__syncthreads();
	if (tid == 0)
		for (uint32_t s = 0; s < nst; s++)
			claim_and_issue<TILE>(kp, smem, (int)s);
	__syncthreads();

	uint32_t qcur = 0xffffffffu;
	for (uint32_t it = 0;; it++) {
		const uint32_t s = it % nst;
		const uint32_t phase = (it / nst) & 1u;
		const StageInfo si = stage_info[s];
		if (si.work >= kp.total_work)
			break;
		if (si.query != qcur) {
			const uint4 *src = reinterpret_cast<const uint4 *>(kp.queries + si.query);
			uint4 *dst = reinterpret_cast<uint4 *>(Q);
			for (int i = tid; i < (int)(sizeof(QDesc) / 16); i += THREADS)
				dst[i] = src[i];
			qcur = si.query;
			__syncthreads();
		}

		/* wait for this stage's columns */
		const uint32_t bar = smem_addr(smem + kOffMbar + 8 * s);
		bool timed_out = true;
		for (unsigned i = 0; i < kStageSpinLimit; i++) {
			if (mbar_try_wait(bar, phase)) {
				timed_out = false;
				break;
			}
			if (i > 16)
				__nanosleep(64);
		}
		if (__syncthreads_or(timed_out)) {
			if (tid == 0) {
				report(kp.error, DE_STAGE_TIMEOUT);
				/* give copies still in flight one more bounded wait */
				for (unsigned i = 0; i < kStageSpinLimit; i++) {
					if (mbar_try_wait(bar, phase))
						break;
					__nanosleep(64);
				}
				drain_stages(kp, smem, it);
			}
			__syncthreads();
			break;
		}

		Ctx c;
		c.stage = smem + kp.stage_area + s * kp.stage_bytes;
		c.vec = smem + kp.vec_area;
		c.Q = Q;

		uint32_t vmask = 0;
		uint8_t wait[R];
#pragma unroll
		for (int r = 0; r < R; r++) {
			wait[r] = 0;
			if ((uint32_t)(r * THREADS + tid) < si.nrows)
				vmask |= 1u << r;
		}
		const uint32_t nuops = Q->prog.nuops;
		bool aborted = false;
		for (uint32_t k = 0; k < nuops; k++) {
			const UOp u = Q->prog.uops[k];
			if (u.kind == UK_RESULT) {
				if (!emit_result<THREADS, R>(c, kp, si, vmask, smem, tid))
					aborted = true;
				break;
			}
			dispatch<THREADS, R>(c, u, tid, wait, vmask);
		}

		__syncthreads();  /* everyone is done with stage s */
		if (aborted) {
			if (tid == 0)
				drain_stages(kp, smem, it);
			break;
		}
		if (tid == 0)
			claim_and_issue<TILE>(kp, smem, (int)s);
		__syncthreads();
	}
}

/* ---- host-side launcher ------------------------------------------------ */

template <int THREADS, int R>
static int launch_t(const KParams &kp, unsigned grid, size_t smem, cudaStream_t stream)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	fn<<<grid, THREADS, smem, stream>>>(kp);
	return cudaGetLastError() == cudaSuccess;
}

template <int THREADS, int R>
static int occ_t(size_t smem, int *ctas)
{
	auto fn = vm_kernel<THREADS, R>;
	if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return 0;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, THREADS, smem) == cudaSuccess;
}

#define VGPU_SHAPES(X) X(128, 4) X(128, 8) X(256, 2) X(256, 4) X(256, 8) X(512, 2) X(512, 4)

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
