/*
 * Read-bandwidth ceiling of a resident table: kernels that only read the
 * columns a query reads, for comparison with the VM kernel on the same
 * bytes (no reference counterpart; a measurement aid).
 *
 *  - mode 0: every thread streams 16-byte loads (ld.global.nc.v4) over the
 *    column pieces and folds them into a checksum;
 *  - modes 1-3: persistent CTAs copy 32 KB tiles of the pieces into a ring
 *    of 4, 6 or 2 shared-memory stages with cp.async.bulk (the VM kernel's
 *    staging path), as many CTAs per SM as fit, and one warp folds one word
 *    per 256 bytes of each landed tile.
 *
 * Both write the checksum (so no load can be dropped) and report the
 * device time of the best of `reps` launches, timed with CUDA events on the
 * engine's stream.
 */
#include <algorithm>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "virginian_b200.h"
#include "engine_internal.h"
#include "vgpu_util.h"

using namespace vgpu;

namespace {

/* a 32 KB tile of a column piece (the last tile of a piece may be shorter;
 * bytes are a multiple of 16) */
struct Tile {
	const unsigned char *p;
	uint32_t bytes;
	uint32_t pad;
};

constexpr uint32_t kTile = 32768;

__device__ __forceinline__ uint4 ldg_nc_v4(const void *p)
{
	uint4 v;
	asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
		: "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
	return v;
}

/* mode 0: a CTA of 512 threads reads a whole tile per step, 64 bytes per
 * thread in four 16-byte loads */
__global__ void __launch_bounds__(512) read_ld(const Tile *tiles, uint32_t ntiles, unsigned long long *sum)
{
	uint32_t acc = 0;
	for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const Tile tl = tiles[t];
		const uint32_t at = 64u * threadIdx.x;
		uint4 v[4];
#pragma unroll
		for (int k = 0; k < 4; k++)
			v[k] = at + 16u * k < tl.bytes ? ldg_nc_v4(tl.p + at + 16u * k) : make_uint4(0, 0, 0, 0);
#pragma unroll
		for (int k = 0; k < 4; k++)
			acc ^= v[k].x ^ v[k].y ^ v[k].z ^ v[k].w;
	}
	if (acc)
		atomicAdd(sum, (unsigned long long)acc);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t phase)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 20000;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
	return ok != 0;
}

/* bounded wait (a second); false if it ran out */
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t phase)
{
	uint64_t t0, t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
	while (!try_wait(bar, phase)) {
		asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
		if (t - t0 > 1000000000ull)
			return false;
	}
	return true;
}

/* modes 1-3: a producer warp bulk-copies this CTA's tiles (blockIdx.x,
 * + gridDim.x, ...) into a ring of kRing stages (4, 6 or 2); a consumer warp touches one
 * word per 256 bytes of each landed tile and releases it */
template <uint32_t kRing>
__global__ void __launch_bounds__(64) read_bulk(const Tile *tiles, uint32_t ntiles, unsigned long long *sum,
	unsigned *err)
{
	extern __shared__ __align__(128) unsigned char sm[];
	uint64_t *full = reinterpret_cast<uint64_t *>(sm);
	uint64_t *empty = full + kRing;
	unsigned char *data = sm + 128;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (threadIdx.x == 0) {
		for (uint32_t s = 0; s < kRing; s++) {
			asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)));
			asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(empty + s)));
		}
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	const uint32_t mine = ntiles > blockIdx.x ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
	if (warp == 0) {
		for (uint32_t k = 0; k < mine; k++) {
			const uint32_t s = k % kRing;
			if (k >= kRing && !wait_phase(smem_u32(empty + s), ((k / kRing) - 1) & 1u)) {
				if (lane == 0)
					atomicCAS(err, 0u, 1u);
				break;
			}
			if (lane == 0) {
				const Tile tl = tiles[blockIdx.x + k * gridDim.x];
				asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
					::"r"(smem_u32(full + s)), "r"(tl.bytes) : "memory");
				asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
					::"r"(smem_u32(data + s * kTile)), "l"(tl.p), "r"(tl.bytes), "r"(smem_u32(full + s))
					: "memory");
			}
			__syncwarp();
		}
	} else {
		uint32_t acc = 0;
		for (uint32_t k = 0; k < mine; k++) {
			const uint32_t s = k % kRing;
			if (!wait_phase(smem_u32(full + s), (k / kRing) & 1u)) {
				if (lane == 0)
					atomicCAS(err, 0u, 2u);
				break;
			}
			const uint32_t *w = reinterpret_cast<const uint32_t *>(data + s * kTile);
#pragma unroll
			for (uint32_t i = 0; i < kTile / 256 / 32; i++)
				acc ^= w[64 * (32 * i + lane)];
			__syncwarp();
			if (lane == 0)
				asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(empty + s)) : "memory");
		}
		if (acc)
			atomicAdd(sum, (unsigned long long)acc);
	}
	/* every issued copy has landed before the CTA exits: the consumer waited
	 * for all of them, or the producer stopped issuing */
	__syncthreads();
}

}  // namespace

extern "C" int virg_gpu_table_read_ceiling(virg_gpu_table *t, const int *cols, unsigned ncols, unsigned mode,
	unsigned reps, double *ms_out, unsigned long long *bytes_out)
{
	VGPU_CHECK(t != nullptr && ms_out != nullptr && (cols != nullptr || ncols == 0), "null argument");
	VGPU_CHECK(mode <= 3, "mode 0 (loads) or 1-3 (bulk copies into 4, 6 or 2 stages)");
	virg_gpu_engine *e = t->e;
	std::lock_guard<std::mutex> lk(e->mu);
	VGPU_CHECK(cudaSetDevice(e->device) == cudaSuccess, "set device");
	std::vector<Tile> tiles;
	uint64_t total = 0;
	for (const SegDesc &sd : t->segs)
		for (unsigned c = 0; c < ncols; c++) {
			const int col = cols[c];
			VGPU_CHECK(col >= -1 && col < (int)t->schema.ncols, "column %d out of range", col);
			const void *p = sd.col[col < 0 ? kKeySlot : col];
			const int ty = col < 0 ? t->schema.key_type : t->schema.col_type[col];
			const uint64_t stride = (ty == 1 || ty == 3) ? 8 : ty == 4 ? 1 : 4;
			const uint64_t bytes = (uint64_t)sd.rows * stride / 16 * 16;
			if (!p)
				continue;
			for (uint64_t at = 0; at < bytes; at += kTile)
				tiles.push_back(Tile{static_cast<const unsigned char *>(p) + at,
					(uint32_t)std::min<uint64_t>(kTile, bytes - at), 0u});
			total += bytes;
		}
	*ms_out = 0;
	if (bytes_out)
		*bytes_out = total;
	if (tiles.empty())
		return 1;
	const uint32_t n = (uint32_t)tiles.size();
	Tile *d_tiles = nullptr;
	unsigned long long *d_sum = nullptr;
	unsigned *d_err = nullptr;
	cudaEvent_t a = nullptr, z = nullptr;
	int ok = cudaMalloc((void **)&d_tiles, n * sizeof(Tile)) == cudaSuccess &&
		cudaMalloc((void **)&d_sum, 8) == cudaSuccess && cudaMalloc((void **)&d_err, 4) == cudaSuccess &&
		cudaMemcpy(d_tiles, tiles.data(), n * sizeof(Tile), cudaMemcpyHostToDevice) == cudaSuccess &&
		cudaMemset(d_err, 0, 4) == cudaSuccess && cudaEventCreate(&a) == cudaSuccess &&
		cudaEventCreate(&z) == cudaSuccess;
	const uint32_t ring = mode == 1 ? 4 : mode == 2 ? 6 : 2;
	const size_t smem = 128 + (size_t)ring * kTile;
	auto bulk = mode == 1 ? read_bulk<4> : mode == 2 ? read_bulk<6> : read_bulk<2>;
	if (ok && mode >= 1)
		ok = cudaFuncSetAttribute(bulk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess;
	float best = 1e30f;
	for (unsigned r = 0; ok && r < std::max(reps, 1u) + 1; r++) {
		cudaEventRecord(a, e->stream);
		if (mode == 0) {
			read_ld<<<e->nsm * 4, 512, 0, e->stream>>>(d_tiles, n, d_sum);
		} else {
			/* as many CTAs as fit an SM's shared memory */
			const unsigned per_sm = (unsigned)std::max<size_t>(1, (size_t)e->smem_sm / (smem + 1024));
			bulk<<<e->nsm * per_sm, 64, smem, e->stream>>>(d_tiles, n, d_sum, d_err);
		}
		cudaEventRecord(z, e->stream);
		ok = cudaEventSynchronize(z) == cudaSuccess && cudaGetLastError() == cudaSuccess;
		float ms = 0;
		if (ok && r > 0 && cudaEventElapsedTime(&ms, a, z) == cudaSuccess)
			best = std::min(best, ms);  /* the first launch is a warm-up */
	}
	unsigned err = 0;
	if (ok)
		ok = cudaMemcpy(&err, d_err, 4, cudaMemcpyDeviceToHost) == cudaSuccess;
	if (a) cudaEventDestroy(a);
	if (z) cudaEventDestroy(z);
	cudaFree(d_tiles);
	cudaFree(d_sum);
	cudaFree(d_err);
	VGPU_CHECK(ok, "read ceiling: %s", cudaGetErrorString(cudaGetLastError()));
	VGPU_CHECK(err == 0, "read ceiling: a stage wait timed out");
	*ms_out = best;
	return 1;
}
