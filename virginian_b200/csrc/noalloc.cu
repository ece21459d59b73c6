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
 * error word, the result row count and one look-back status word per chunk)
 * lives here in one fixed file-scope device array, g_prealloc_scratch, of
 * kPreallocScratchBytes (about 520 KB).  That bounds a query to
 * kPreallocMaxChunks chunks; segments of more than kPreallocMaxRows =
 * 67,108,864 rows (2^26) are refused before anything is launched.
 *
 * Set-up: the first call on each device (with that device current) looks up
 * the array's device address with cudaGetSymbolAddress, since the host-side
 * name of a __device__ array is not a device address, and reads the device's
 * SM count and shared-memory limits.  Make that first call before any stream
 * capture.  The address is kept for the life of the process; a
 * cudaDeviceReset (or anything else that destroys the device's primary
 * context) makes it stale, so do not call this entry point after one.
 *
 * The array is shared by every call on a device and keeps the last call's
 * contents: each call clears the counter, error word, row count and the
 * status words it will use before its launch.  Calls that overlap in time on
 * one device (two streams, or two host threads) race on the array; run them
 * one after another, or on one stream.
 */
#include <algorithm>
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

constexpr uint32_t kPreallocMaxChunks = 65536;
constexpr uint64_t kPreallocMaxRows = 1ull << 26;
/* chunks of at most 4096 rows: at least 2048 rows each (a chunk is a whole
 * number of full-phase tiles, and a tile is at most a chunk) */
constexpr uint32_t kPreallocChunkRows = 4096;
static_assert(kPreallocMaxRows / (kPreallocChunkRows / 2) <= kPreallocMaxChunks, "status words per chunk");

/* scratch layout: descriptor block | control words | status words */
constexpr size_t kDescBytes = 8192;
constexpr size_t kCtrlOff = kDescBytes;          /* u32 counter, u32 error, u64 row count */
constexpr size_t kCtrlBytes = 256;
constexpr size_t kStatusOff = kCtrlOff + kCtrlBytes;
constexpr size_t kPreallocScratchBytes = kStatusOff + (size_t)kPreallocMaxChunks * sizeof(uint64_t);

/* descriptor block: QDesc | q_work_prefix[2] | seg_chunk_prefix[2] | SegDesc */
constexpr size_t align16(size_t x) { return (x + 15) / 16 * 16; }
constexpr size_t kOffPrefix = align16(sizeof(QDesc));
constexpr size_t kOffChunks = kOffPrefix + 2 * sizeof(uint64_t);
constexpr size_t kOffSeg = align16(kOffChunks + 2 * sizeof(uint32_t));
constexpr size_t kDescUsed = kOffSeg + sizeof(SegDesc);
static_assert(kDescUsed <= kDescBytes, "descriptor block too small");

__device__ __align__(256) unsigned char g_prealloc_scratch[kPreallocScratchBytes];

constexpr int kMaxDevices = 64;

struct DeviceSetup {
	bool ready;
	unsigned char *scratch;  /* device address of g_prealloc_scratch */
	int nsm;
	int smem_block;
	int smem_sm;
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
		e = cudaDeviceGetAttribute(&s.smem_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
		VGPU_CHECK(e == cudaSuccess, "shared memory limit: %s", cudaGetErrorString(e));
		e = cudaDeviceGetAttribute(&s.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
		VGPU_CHECK(e == cudaSuccess, "shared memory limit: %s", cudaGetErrorString(e));
		s.scratch = static_cast<unsigned char *>(p);
		s.ready = true;
	}
	*out = s;
	return 1;
}

/* the engine's default geometry: eight compute warps, 32 KB stages (more
 * for programs whose widest phase needs it), one CTA per SM */
int pick_geom(const ProgPlan &pp, const DeviceSetup &ds, Geom *g)
{
	const uint32_t bpr = std::max(pp.count_bpr, pp.mode == FM_GATHER ? 0u : pp.full_bpr);
	Shape s = {256, std::max<unsigned>(32, (kCountGroup * kBlockRows * bpr + 1023) / 1024), 0, 1, kPreallocChunkRows, 0};
	VGPU_CHECK(geom_make(s, pp.sel_bpr, pp.row_bpr, pp.gather_bpr, ds.smem_block, ds.smem_sm, g),
		"program needs more shared memory than the device offers");
	return 1;
}

/* device memory of the current device (the kernel reads and writes these
 * buffers directly; another GPU's memory would need peer access) */
bool on_device(const void *p, int dev)
{
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	if (a.type == cudaMemoryTypeManaged)
		return true;
	return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int virg_gpu_query_prealloc(const virg_gpu_program *p, const virg_gpu_segment *seg,
	void *const *out_cols, uint64_t capacity, uint64_t *out_rows, void *stream)
{
	VGPU_CHECK(p != nullptr && seg != nullptr && out_rows != nullptr, "null argument");
	const Program &P = p->prog;
	VGPU_CHECK(seg->rows <= kPreallocMaxRows,
		"segment of %u rows: this entry point takes at most %llu rows (its fixed scratch holds %u chunks)",
		seg->rows, (unsigned long long)kPreallocMaxRows, kPreallocMaxChunks);
	VGPU_CHECK(out_cols != nullptr || P.nout == 0, "null result columns");
	int dev = 0;
	cudaError_t ce = cudaGetDevice(&dev);
	VGPU_CHECK(ce == cudaSuccess, "current device: %s", cudaGetErrorString(ce));
	for (unsigned i = 0; i < P.nload && seg->rows; i++) {
		const void *c = P.load_src[i] == kKeySlot ? seg->key : seg->col[P.load_src[i]];
		VGPU_CHECK(c != nullptr, "the program reads %s, which the segment does not give",
			P.load_src[i] == kKeySlot ? "the key column" : "a column");
		VGPU_CHECK(((uintptr_t)c & 15u) == 0, "input columns must be 16-byte aligned");
		VGPU_CHECK(on_device(c, dev), "input columns must be in the current device's memory (device %d)", dev);
	}
	for (unsigned j = 0; j < P.nout && seg->rows; j++) {
		VGPU_CHECK(out_cols[j] != nullptr, "result column %u is null", j);
		VGPU_CHECK(((uintptr_t)out_cols[j] % P.out_stride[j]) == 0, "result column %u is misaligned", j);
		VGPU_CHECK(on_device(out_cols[j], dev), "result columns must be in the current device's memory (device %d)",
			dev);
	}

	DeviceSetup ds;
	if (!setup_device(dev, &ds))
		return 0;
	*out_rows = 0;
	if (seg->rows == 0)
		return 1;

	ProgPlan pp;
	plan_program(P, pp);
	Geom g;
	if (!pick_geom(pp, ds, &g))
		return 0;

	/* the descriptor block, built on the stack */
	alignas(16) unsigned char hb[kDescUsed];
	memset(hb, 0, sizeof(hb));
	unsigned char *const db = ds.scratch;
	QDesc &d = *reinterpret_cast<QDesc *>(hb);
	if (!desc_fill(d, P, pp, g, kPreallocChunkRows))
		return 0;
	const uint32_t nchunks = (seg->rows + d.chunk_rows - 1) / d.chunk_rows;
	VGPU_CHECK(nchunks <= kPreallocMaxChunks, "internal: %u chunks exceed the scratch", nchunks);
	d.segs = reinterpret_cast<const SegDesc *>(db + kOffSeg);
	d.nsegs = 1;
	d.seg_chunk_prefix = reinterpret_cast<const uint32_t *>(db + kOffChunks);
	d.work_first = 0;
	d.nchunks = nchunks;
	for (unsigned j = 0; j < P.nout; j++)
		d.out_ptr[j] = out_cols[j];
	d.capacity = capacity;
	d.total_out = reinterpret_cast<unsigned long long *>(db + kCtrlOff + 8);
	d.block_counts = nullptr;
	d.base_in = nullptr;
	uint64_t *prefix = reinterpret_cast<uint64_t *>(hb + kOffPrefix);
	prefix[0] = 0;
	prefix[1] = nchunks;
	uint32_t *chunks = reinterpret_cast<uint32_t *>(hb + kOffChunks);
	chunks[0] = 0;
	chunks[1] = nchunks;
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
	ce = cudaMemsetAsync(db + kCtrlOff, 0, kCtrlBytes + (size_t)nchunks * sizeof(uint64_t), st);
	VGPU_CHECK(ce == cudaSuccess, "scratch clear: %s", cudaGetErrorString(ce));

	KParams kp = geom_params(g);
	kp.queries = reinterpret_cast<const QDesc *>(db);
	kp.q_work_prefix = reinterpret_cast<const uint64_t *>(db + kOffPrefix);
	kp.nq = 1;
	kp.total_work = nchunks;
	kp.counter = reinterpret_cast<unsigned *>(db + kCtrlOff);
	kp.status = reinterpret_cast<uint64_t *>(db + kStatusOff);
	kp.error = reinterpret_cast<unsigned *>(db + kCtrlOff + 4);
	kp.epoch = 1;
	const unsigned grid = std::min<unsigned>(nchunks, (unsigned)ds.nsm);
	if (!launch_vm(g.shape, kp, grid, g.smem, st))
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
