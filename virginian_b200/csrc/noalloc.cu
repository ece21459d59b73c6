/*
 * virg_gpu_query_prealloc: one program over one device-resident segment,
 * results into caller-owned device buffers, with no memory allocation.
 *
 * Who needs it: callers that must not allocate device memory around a
 * query.  A host framework whose caching allocator owns the device's free
 * memory (so a cudaMalloc from inside a library would fail or fragment its
 * pool), a latency-critical loop that must never reach the CUDA allocator
 * (whose calls can synchronise the device), and processes that already gave
 * all free memory to resident tables.  The engine path (virg_gpu_query)
 * allocates every result and grows its descriptor and status buffers on
 * demand; this path does neither, in device or in host memory.
 *
 * The kernel is the engine's VM kernel, unchanged.  What the engine keeps in
 * per-engine allocations (the launch descriptor, the work counter, the device
 * error word, the result row count and one look-back status word per tile)
 * lives here in one fixed file-scope device array, g_prealloc_scratch, of
 * kPreallocScratchBytes (about 520 KB).  That bounds a query to
 * kPreallocMaxTiles tiles: kPreallocMaxRows = 67,108,864 rows (2^26) at the
 * smallest tile of 1024 rows; larger segments are refused before anything
 * is launched.
 *
 * Set-up: the first call on each device (with that device current) looks up
 * the array's device address with cudaGetSymbolAddress, since the host-side
 * name of a __device__ array is not a device address, and reads the device's
 * SM count and shared-memory limit.  Make that first call before any stream
 * capture.
 *
 * The array is shared by every call on a device and keeps the last call's
 * contents: each call clears the counter, error word, row count and the
 * status words it will use before its launch.  Calls that overlap in time on
 * one device (two streams, or two host threads) race on the array; run them
 * one after another, or on one stream.
 */
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <mutex>

#include <cuda_runtime.h>

#include "virginian_b200.h"
#include "engine_internal.h"
#include "vgpu_util.h"

using namespace vgpu;

namespace {

constexpr uint32_t kPreallocMaxTiles = 65536;
constexpr uint32_t kPreallocMinTile = 1024;  /* 128 threads x 8 rows */
constexpr uint64_t kPreallocMaxRows = (uint64_t)kPreallocMaxTiles * kPreallocMinTile;

/* scratch layout: descriptor block | control words | status words */
constexpr size_t kDescBytes = 8192;
constexpr size_t kCtrlOff = kDescBytes;          /* u32 counter, u32 error, u64 row count */
constexpr size_t kCtrlBytes = 256;
constexpr size_t kStatusOff = kCtrlOff + kCtrlBytes;
constexpr size_t kPreallocScratchBytes = kStatusOff + (size_t)kPreallocMaxTiles * sizeof(uint64_t);

/* descriptor block: QDesc | q_work_prefix[2] | seg_tile_prefix[2] | SegDesc */
constexpr size_t align16(size_t x) { return (x + 15) / 16 * 16; }
constexpr size_t kOffPrefix = align16(sizeof(QDesc));
constexpr size_t kOffTiles = kOffPrefix + 2 * sizeof(uint64_t);
constexpr size_t kOffSeg = align16(kOffTiles + 2 * sizeof(uint32_t));
constexpr size_t kDescUsed = kOffSeg + sizeof(SegDesc);
static_assert(kDescUsed <= kDescBytes, "descriptor block too small");

__device__ __align__(256) unsigned char g_prealloc_scratch[kPreallocScratchBytes];

constexpr int kMaxDevices = 64;

struct DeviceSetup {
	bool ready;
	unsigned char *scratch;  /* device address of g_prealloc_scratch */
	int nsm;
	int smem_optin;
};

std::mutex g_setup_mu;
DeviceSetup g_setup[kMaxDevices];

int setup_device(int dev, DeviceSetup *out)
{
	VGPU_CHECK(dev >= 0 && dev < kMaxDevices, "device %d out of range", dev);
	std::lock_guard<std::mutex> lk(g_setup_mu);
	DeviceSetup &s = g_setup[dev];
	if (!s.ready) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_prealloc_scratch);
		VGPU_CHECK(e == cudaSuccess, "scratch address lookup: %s", cudaGetErrorString(e));
		e = cudaDeviceGetAttribute(&s.nsm, cudaDevAttrMultiProcessorCount, dev);
		VGPU_CHECK(e == cudaSuccess, "SM count: %s", cudaGetErrorString(e));
		e = cudaDeviceGetAttribute(&s.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
		VGPU_CHECK(e == cudaSuccess, "shared memory limit: %s", cudaGetErrorString(e));
		s.scratch = static_cast<unsigned char *>(p);
		s.ready = true;
	}
	*out = s;
	return 1;
}

/* the engine's default choice: two CTAs per SM if the program's stages fit,
 * else one */
int pick_shape(const Program &P, int smem_optin, Shape *shape, size_t *smem, uint32_t *stage_bytes,
	uint32_t *vec_bytes)
{
	static const unsigned cand[][2] = {{256, 4}, {128, 8}, {256, 8}, {512, 4}};
	const size_t limit = (size_t)smem_optin;
	for (int pass = 0; pass < 2; pass++)
		for (auto &c : cand)
			for (unsigned st : {3u, 2u}) {
				Shape s = {c[0], c[1], st, 0};
				uint32_t sb, rb, selb;
				program_layout(P, s.tile(), nullptr, &sb, &rb, &selb);
				const uint32_t vb = kSlots * rb + selb;
				sb = ((sb < 128 ? 128 : sb) + 127) / 128 * 128;
				const size_t need = smem_for(s, sb, vb);
				if (need <= (pass == 0 ? limit / 2 - 1024 : limit)) {
					*shape = s;
					*smem = need;
					*stage_bytes = sb;
					*vec_bytes = vb;
					return 1;
				}
			}
	VGPU_FAIL("program needs more shared memory than the device offers");
}

bool is_device_pointer(const void *p)
{
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int virg_gpu_query_prealloc(const virg_gpu_program *p, const virg_gpu_segment *seg,
	void *const *out_cols, uint64_t capacity, uint64_t *out_rows, void *stream)
{
	VGPU_CHECK(p != nullptr && seg != nullptr && out_rows != nullptr, "null argument");
	const Program &P = p->prog;
	VGPU_CHECK(seg->rows <= kPreallocMaxRows,
		"segment of %u rows: this entry point takes at most %llu rows (its fixed scratch holds %u tiles)",
		seg->rows, (unsigned long long)kPreallocMaxRows, kPreallocMaxTiles);
	VGPU_CHECK(out_cols != nullptr || P.nout == 0, "null result columns");
	for (unsigned i = 0; i < P.nload && seg->rows; i++) {
		const void *c = P.load_src[i] == kKeySlot ? seg->key : seg->col[P.load_src[i]];
		VGPU_CHECK(c != nullptr, "the program reads %s, which the segment does not give",
			P.load_src[i] == kKeySlot ? "the key column" : "a column");
		VGPU_CHECK(((uintptr_t)c & 15u) == 0, "input columns must be 16-byte aligned");
		VGPU_CHECK(is_device_pointer(c), "input columns must be in device memory");
	}
	for (unsigned j = 0; j < P.nout && seg->rows; j++) {
		VGPU_CHECK(out_cols[j] != nullptr, "result column %u is null", j);
		VGPU_CHECK(((uintptr_t)out_cols[j] % P.out_stride[j]) == 0, "result column %u is misaligned", j);
		VGPU_CHECK(is_device_pointer(out_cols[j]), "result columns must be in device memory");
	}

	int dev = 0;
	cudaError_t ce = cudaGetDevice(&dev);
	VGPU_CHECK(ce == cudaSuccess, "current device: %s", cudaGetErrorString(ce));
	DeviceSetup ds;
	if (!setup_device(dev, &ds))
		return 0;
	*out_rows = 0;
	if (seg->rows == 0)
		return 1;

	Shape shape;
	size_t smem;
	uint32_t stage_bytes, vec_bytes;
	if (!pick_shape(P, ds.smem_optin, &shape, &smem, &stage_bytes, &vec_bytes))
		return 0;
	const uint32_t tile = shape.tile();
	const uint32_t ntiles = (seg->rows + tile - 1) / tile;

	/* the descriptor block, built on the stack */
	alignas(16) unsigned char hb[kDescUsed];
	memset(hb, 0, sizeof(hb));
	unsigned char *const db = ds.scratch;
	QDesc &d = *reinterpret_cast<QDesc *>(hb);
	d.prog = P;
	uint32_t sb, rb, selb;
	program_layout(P, tile, d.load_off, &sb, &rb, &selb);
	vec_offsets(P, tile, rb, d.vec_off);
	d.vec_slot = rb;
	d.stage_bytes = sb;
	d.segs = reinterpret_cast<const SegDesc *>(db + kOffSeg);
	d.nsegs = 1;
	d.seg_tile_prefix = reinterpret_cast<const uint32_t *>(db + kOffTiles);
	d.work_first = 0;
	d.ntiles = ntiles;
	for (unsigned j = 0; j < P.nout; j++)
		d.out_ptr[j] = out_cols[j];
	d.capacity = capacity;
	d.total_out = reinterpret_cast<unsigned long long *>(db + kCtrlOff + 8);
	d.block_counts = nullptr;
	d.base_in = nullptr;
	const uint32_t vec_area = (uint32_t)(kSmemHeader + (size_t)shape.stages * stage_bytes);
	fill_operands(d, vec_area);
	uint64_t *prefix = reinterpret_cast<uint64_t *>(hb + kOffPrefix);
	prefix[0] = 0;
	prefix[1] = ntiles;
	uint32_t *tiles = reinterpret_cast<uint32_t *>(hb + kOffTiles);
	tiles[0] = 0;
	tiles[1] = ntiles;
	SegDesc &sd = *reinterpret_cast<SegDesc *>(hb + kOffSeg);
	for (int c = 0; c < kMaxCols; c++)
		sd.col[c] = seg->col[c];
	sd.col[kKeySlot] = seg->key;
	sd.rows = seg->rows;
	sd.block_base = 0;

	cudaStream_t st = static_cast<cudaStream_t>(stream);
	/* the block is copied from pageable memory: the call returns once the
	 * bytes are staged, so the stack buffer may go */
	ce = cudaMemcpyAsync(db, hb, sizeof(hb), cudaMemcpyHostToDevice, st);
	VGPU_CHECK(ce == cudaSuccess, "descriptor copy: %s", cudaGetErrorString(ce));
	/* counter, error word, row count and this launch's status words start at
	 * zero; the status words carry epoch 1, which no cleared word matches */
	ce = cudaMemsetAsync(db + kCtrlOff, 0, kCtrlBytes + (size_t)ntiles * sizeof(uint64_t), st);
	VGPU_CHECK(ce == cudaSuccess, "scratch clear: %s", cudaGetErrorString(ce));

	KParams kp;
	kp.queries = reinterpret_cast<const QDesc *>(db);
	kp.q_work_prefix = reinterpret_cast<const uint64_t *>(db + kOffPrefix);
	kp.nq = 1;
	kp.total_work = ntiles;
	kp.counter = reinterpret_cast<unsigned *>(db + kCtrlOff);
	kp.status = reinterpret_cast<uint64_t *>(db + kStatusOff);
	kp.error = reinterpret_cast<unsigned *>(db + kCtrlOff + 4);
	kp.epoch = 1;
	kp.nstages = shape.stages;
	kp.stage_bytes = stage_bytes;
	kp.stage_area = kSmemHeader;
	kp.vec_area = vec_area;
	kp.vec_bytes = vec_bytes;
	kp.sel_area = vec_area + vec_bytes;
	int per_sm = 0;
	if (!occupancy(shape, smem, &per_sm))
		VGPU_FAIL("occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
	if (per_sm < 1)
		per_sm = 1;
	const uint64_t slots = (uint64_t)per_sm * (uint64_t)ds.nsm;
	const unsigned grid = (unsigned)(ntiles < slots ? ntiles : slots);
	if (!launch_vm(shape, kp, grid, smem, st))
		VGPU_FAIL("kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));

	/* row count and device error word (8-byte aligned pair) */
	unsigned long long words[2] = {0, 0};
	ce = cudaMemcpyAsync(words, db + kCtrlOff, sizeof(words), cudaMemcpyDeviceToHost, st);
	VGPU_CHECK(ce == cudaSuccess, "result count read: %s", cudaGetErrorString(ce));
	ce = cudaStreamSynchronize(st);
	VGPU_CHECK(ce == cudaSuccess, "query: %s", cudaGetErrorString(ce));
	const unsigned err = (unsigned)(words[0] >> 32);
	*out_rows = words[1];
	VGPU_CHECK(err != DE_OUTPUT_OVERFLOW, "result has %llu rows, the buffers hold %llu",
		(unsigned long long)words[1], (unsigned long long)capacity);
	VGPU_CHECK(err == 0, "query failed on the device: %s", device_error_text(err));
	return 1;
}
