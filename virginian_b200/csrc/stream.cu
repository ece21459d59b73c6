/*
 * Streamed execution over host-resident tablets.
 *
 * The reference moves tablets to the GPU one at a time: a blocking copy of a
 * whole 8 MB tablet, the kernel, then a blocking copy of a whole result
 * tablet back (serial mode, src/vm/vm_gpu.cu:147-236), or a single stream
 * that in practice serialises the same steps (:249-443).  Here only the
 * columns the program reads cross the host link, in chunks of several
 * tablets, through a ring of device staging buffers:
 *
 *   copy stream:    [H2D chunk 0][H2D chunk 1][H2D chunk 2] ...
 *   compute stream:              [VM chunk 0] [VM chunk 1 ] ...
 *
 * Buffer reuse is ordered by events (a buffer is refilled only after the
 * kernel that read it finished).  Each chunk is one launch of the VM kernel;
 * its first tile starts at the row count the previous chunk left in device
 * memory, so the chunks append one ordered result stream in HBM with no
 * host round trip between chunks.
 */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "vgpu_engine.h"
#include "vgpu_util.h"
#include "engine_internal.h"

using namespace vgpu;

#define CUDA_OK(call, what)                                                   \
	do {                                                                      \
		cudaError_t e_ = (call);                                              \
		if (e_ != cudaSuccess)                                                \
			VGPU_FAIL("%s: %s", what, cudaGetErrorString(e_));                 \
	} while (0)

namespace {

constexpr unsigned kRing = 3;

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct RingBuf {
	unsigned char *mem = nullptr;
	SegDesc *d_segs = nullptr;
	std::vector<SegDesc> h_segs;
	std::vector<uint32_t> rows;
	cudaEvent_t copied = nullptr, freed = nullptr, c0 = nullptr, c1 = nullptr;
	bool timed = false;
};

}  // namespace

extern "C" int virg_gpu_query_streamed(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_segment *segs, unsigned nsegs, unsigned segs_per_chunk, virg_gpu_result **out,
	virg_gpu_stream_stats *stats)
{
	VGPU_CHECK(e != nullptr && p != nullptr && out != nullptr && (segs != nullptr || nsegs == 0),
		"null argument");
	*out = nullptr;
	if (segs_per_chunk == 0)
		segs_per_chunk = 8;
	const Program &P = p->prog;
	CUDA_OK(cudaSetDevice(e->device), "set device");
	std::lock_guard<std::mutex> lk(e->mu);
	const auto t_start = std::chrono::steady_clock::now();

	uint64_t total_rows = 0;
	for (unsigned s = 0; s < nsegs; s++) {
		total_rows += segs[s].rows;
		if (!segs[s].rows)
			continue;
		for (unsigned i = 0; i < P.nload; i++) {
			const void *src = P.load_src[i] == kKeySlot ? segs[s].key : segs[s].col[P.load_src[i]];
			VGPU_CHECK(src != nullptr, "segment %u lacks a column the program reads", s);
		}
	}
	virg_gpu_result *r = nullptr;
	if (!result_alloc(e, P, total_rows, false, 0, &r))
		return 0;

	/* staging ring sized for the largest chunk */
	size_t chunk_bytes = 0;
	for (unsigned c0 = 0; c0 < nsegs; c0 += segs_per_chunk) {
		size_t b = 0;
		for (unsigned s = c0; s < std::min(nsegs, c0 + segs_per_chunk); s++)
			for (unsigned i = 0; i < P.nload; i++)
				b += align256((size_t)padded_rows(segs[s].rows) * P.load_stride[i]);
		chunk_bytes = std::max(chunk_bytes, b);
	}
	RingBuf ring[kRing];
	unsigned long long *d_totals = nullptr;
	int ok = 1;
	auto cleanup = [&]() {
		cudaStreamSynchronize(e->copy_stream);
		cudaStreamSynchronize(e->stream);
		for (RingBuf &b : ring) {
			if (b.mem) cudaFree(b.mem);
			if (b.d_segs) cudaFree(b.d_segs);
			for (cudaEvent_t ev : {b.copied, b.freed, b.c0, b.c1})
				if (ev) cudaEventDestroy(ev);
		}
		if (d_totals) cudaFree(d_totals);
	};
	for (RingBuf &b : ring) {
		if (cudaMalloc((void **)&b.mem, std::max<size_t>(chunk_bytes, 256)) != cudaSuccess ||
			cudaMalloc((void **)&b.d_segs, segs_per_chunk * sizeof(SegDesc)) != cudaSuccess ||
			cudaEventCreateWithFlags(&b.copied, cudaEventDisableTiming) != cudaSuccess ||
			cudaEventCreateWithFlags(&b.freed, cudaEventDisableTiming) != cudaSuccess ||
			cudaEventCreate(&b.c0) != cudaSuccess || cudaEventCreate(&b.c1) != cudaSuccess) {
			set_error("staging ring setup failed: %s", cudaGetErrorString(cudaGetLastError()));
			ok = 0;
			break;
		}
	}
	if (ok && cudaMalloc((void **)&d_totals, 2 * sizeof(unsigned long long)) != cudaSuccess) {
		set_error("totals alloc failed");
		ok = 0;
	}
	if (ok && cudaMemset(d_totals, 0, 2 * sizeof(unsigned long long)) != cudaSuccess)
		ok = 0;

	double copy_ms = 0;
	uint64_t h2d = 0;
	unsigned chunks = 0, cur = 0;  /* d_totals[cur] holds the running count */
	bool launched_any = false;
	for (unsigned c0 = 0; ok && c0 < nsegs; c0 += segs_per_chunk) {
		RingBuf &b = ring[chunks % kRing];
		if (b.timed) {
			/* the buffer's previous copy is done once its kernel freed it */
			float ms = 0;
			cudaEventSynchronize(b.c1);
			if (cudaEventElapsedTime(&ms, b.c0, b.c1) == cudaSuccess)
				copy_ms += ms;
			b.timed = false;
		}
		cudaStreamWaitEvent(e->copy_stream, b.freed, 0);
		b.h_segs.clear();
		b.rows.clear();
		cudaEventRecord(b.c0, e->copy_stream);
		unsigned char *dst = b.mem;
		uint64_t chunk_rows = 0;
		for (unsigned s = c0; s < std::min(nsegs, c0 + segs_per_chunk); s++) {
			SegDesc d;
			memset(&d, 0, sizeof(d));
			d.rows = segs[s].rows;
			for (unsigned i = 0; i < P.nload; i++) {
				const unsigned src_col = P.load_src[i];
				const void *src = src_col == kKeySlot ? segs[s].key : segs[s].col[src_col];
				const size_t bytes = (size_t)segs[s].rows * P.load_stride[i];
				if (bytes && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, e->copy_stream) !=
						cudaSuccess) {
					set_error("chunk copy failed: %s", cudaGetErrorString(cudaGetLastError()));
					ok = 0;
				}
				d.col[src_col] = dst;
				dst += align256((size_t)padded_rows(segs[s].rows) * P.load_stride[i]);
				h2d += bytes;
			}
			b.h_segs.push_back(d);
			b.rows.push_back(d.rows);
			chunk_rows += d.rows;
		}
		if (ok && cudaMemcpyAsync(b.d_segs, b.h_segs.data(), b.h_segs.size() * sizeof(SegDesc),
				cudaMemcpyHostToDevice, e->copy_stream) != cudaSuccess)
			ok = 0;
		cudaEventRecord(b.c1, e->copy_stream);
		b.timed = true;
		cudaEventRecord(b.copied, e->copy_stream);
		cudaStreamWaitEvent(e->stream, b.copied, 0);
		if (ok && chunk_rows) {
			QueryLaunch q;
			q.prog = &P;
			q.d_segs = b.d_segs;
			q.nsegs = (uint32_t)b.h_segs.size();
			q.seg_rows = b.rows.data();
			for (unsigned j = 0; j < P.nout; j++)
				q.out[j] = r->out[j];
			q.capacity = total_rows;
			q.base_in = launched_any ? d_totals + cur : nullptr;
			q.d_total = d_totals + (cur ^ 1);
			ok = run_queries(e, std::vector<QueryLaunch>(1, q), nullptr);
			cur ^= 1;
			launched_any = true;
		}
		cudaEventRecord(b.freed, e->stream);
		chunks++;
	}
	if (ok) {
		for (RingBuf &b : ring)
			if (b.timed) {
				float ms = 0;
				cudaEventSynchronize(b.c1);
				if (cudaEventElapsedTime(&ms, b.c0, b.c1) == cudaSuccess)
					copy_ms += ms;
				b.timed = false;
			}
		if (launched_any)
			ok = cudaMemcpyAsync(r->d_total, d_totals + cur, sizeof(unsigned long long),
				cudaMemcpyDeviceToDevice, e->stream) == cudaSuccess;
		else
			r->ntiles_zero = true;
	}
	cleanup();
	if (!ok) {
		virg_gpu_result_destroy(r);
		return 0;
	}
	if (stats) {
		stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
		stats->copy_seconds = copy_ms / 1000.0;
		stats->h2d_bytes = h2d;
		stats->chunks = chunks;
	}
	*out = r;
	return 1;
}
