/*
 * Execution over rows in host memory: the streamed executor
 * (virg_gpu_query_streamed) and the end-to-end call (virg_gpu_query_host).
 *
 * The reference moves tablets to the GPU one at a time: a blocking copy of a
 * whole 8 MB tablet, the kernel, then a blocking copy of a whole result
 * tablet back (serial mode, src/vm/vm_gpu.cu:147-236), or a single stream
 * that in practice serialises the same steps (:249-443).  Here only the
 * columns the program reads cross the host link, in chunks of tens of MB,
 * through the engine's ring of device staging buffers:
 *
 *   copy stream:    [H2D chunk 0][H2D chunk 1][H2D chunk 2] ...
 *   compute stream:              [VM chunk 0] [VM chunk 1 ] ...
 *
 * Segments whose columns lie back to back in host memory (tablets cut from
 * one buffer) are merged into one piece, so a chunk costs one copy per
 * column instead of one per tablet and column, and the kernel sees the
 * piece as one segment (results do not depend on tablet boundaries).
 * Buffer reuse is ordered by events (a buffer is refilled only after the
 * kernel that read it finished).  Each chunk is one launch of the VM kernel;
 * its first chunk of rows starts at the row count the previous launch left
 * in device memory, so the launches append one ordered result stream in HBM
 * with no host round trip between them.  The ring's buffers and events
 * belong to the engine and are reused by later calls.
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

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

/* rows [.., .. + rows) of the program's columns, contiguous in host memory */
struct Piece {
	uint64_t rows;
	const unsigned char *src[kMaxLoads];
};

struct Chunk {
	size_t first, n;   /* pieces */
	uint64_t rows;
	size_t bytes;      /* staging bytes */
};

/* the column the program's load i reads in segment s */
const unsigned char *load_ptr(const Program &P, const virg_gpu_segment &g, unsigned i)
{
	const unsigned src = P.load_src[i];
	return static_cast<const unsigned char *>(src == kKeySlot ? g.key : g.col[src]);
}

/* pieces and chunks of at most chunk_rows rows each (a chunk may hold
 * several pieces when the host rows are not contiguous) */
void plan_pieces(const Program &P, const virg_gpu_segment *segs, unsigned nsegs, uint64_t chunk_rows,
	std::vector<Piece> &pieces, std::vector<Chunk> &chunks)
{
	Chunk cur = {0, 0, 0, 0};
	auto close = [&]() {
		if (cur.n)
			chunks.push_back(cur);
		cur = {pieces.size(), 0, 0, 0};
	};
	for (unsigned s = 0; s < nsegs; s++) {
		uint64_t off = 0;
		while (off < segs[s].rows) {
			const uint64_t take = std::min<uint64_t>(segs[s].rows - off, chunk_rows - cur.rows);
			bool merge = cur.n > 0;
			if (merge) {
				const Piece &pc = pieces.back();
				for (unsigned i = 0; i < P.nload && merge; i++)
					merge = pc.src[i] + pc.rows * P.load_stride[i] == load_ptr(P, segs[s], i) + off * P.load_stride[i];
				/* a piece is one kernel segment: fewer than 2^31 rows */
				merge = merge && pc.rows + take < (1ull << 31);
			}
			if (merge) {
				pieces.back().rows += take;
			} else {
				Piece pc;
				pc.rows = take;
				for (unsigned i = 0; i < P.nload; i++)
					pc.src[i] = load_ptr(P, segs[s], i) + off * P.load_stride[i];
				pieces.push_back(pc);
				cur.n++;
			}
			cur.rows += take;
			off += take;
			if (cur.rows == chunk_rows)
				close();
		}
	}
	close();
	for (Chunk &c : chunks) {
		c.bytes = 0;
		for (size_t k = c.first; k < c.first + c.n; k++)
			for (unsigned i = 0; i < P.nload; i++)
				c.bytes += align256((size_t)padded_rows((uint32_t)pieces[k].rows) * P.load_stride[i]);
	}
}

/* buffers of at least `bytes` and `nseg` descriptors each */
int ring_reserve(virg_gpu_engine *e, size_t bytes, size_t nseg)
{
	HostRing &h = e->hring;
	if (!h.ready) {
		for (unsigned b = 0; b < HostRing::kBufs; b++) {
			CUDA_OK(cudaEventCreateWithFlags(&h.copied[b], cudaEventDisableTiming), "ring event");
			CUDA_OK(cudaEventCreateWithFlags(&h.freed[b], cudaEventDisableTiming), "ring event");
			CUDA_OK(cudaEventCreate(&h.c0[b]), "ring event");
			CUDA_OK(cudaEventCreate(&h.c1[b]), "ring event");
		}
		CUDA_OK(cudaMalloc((void **)&h.d_totals, 2 * sizeof(unsigned long long)), "ring totals");
		h.ready = true;
	}
	if (bytes > h.bytes || nseg > h.seg_cap) {
		/* earlier calls' kernels may still read the old buffers */
		CUDA_OK(cudaStreamSynchronize(e->copy_stream), "ring sync");
		CUDA_OK(cudaStreamSynchronize(e->stream), "ring sync");
		const size_t nb = std::max(bytes, h.bytes), ns = std::max(nseg, h.seg_cap);
		for (unsigned b = 0; b < HostRing::kBufs; b++) {
			if (nb > h.bytes) {
				cudaFree(h.mem[b]);
				h.mem[b] = nullptr;
				CUDA_OK(cudaMalloc((void **)&h.mem[b], nb), "staging buffer");
			}
			if (ns > h.seg_cap) {
				cudaFree(h.d_segs[b]);
				h.d_segs[b] = nullptr;
				CUDA_OK(cudaMalloc((void **)&h.d_segs[b], ns * sizeof(SegDesc)), "staging descriptors");
			}
		}
		h.bytes = nb;
		h.seg_cap = ns;
	}
	return 1;
}

}  // namespace

void vgpu::host_ring_free(virg_gpu_engine *e)
{
	HostRing &h = e->hring;
	cudaStreamSynchronize(e->copy_stream);
	for (unsigned b = 0; b < HostRing::kBufs; b++) {
		cudaFree(h.mem[b]);
		cudaFree(h.d_segs[b]);
		for (cudaEvent_t ev : {h.copied[b], h.freed[b], h.c0[b], h.c1[b]})
			if (ev)
				cudaEventDestroy(ev);
	}
	cudaFree(h.d_totals);
	h = HostRing();
}

int vgpu::host_pipeline(virg_gpu_engine *e, const Program &P, const virg_gpu_segment *segs, unsigned nsegs,
	uint64_t chunk_rows, virg_gpu_result *r, virg_gpu_stream_stats *stats)
{
	const auto t_start = std::chrono::steady_clock::now();
	std::vector<Piece> pieces;
	std::vector<Chunk> chunks;
	plan_pieces(P, segs, nsegs, std::max<uint64_t>(chunk_rows, kBlockRows), pieces, chunks);
	size_t need = 256, nseg = 1;
	for (const Chunk &c : chunks) {
		need = std::max(need, c.bytes);
		nseg = std::max(nseg, c.n);
	}
	if (!ring_reserve(e, need, nseg))
		return 0;
	HostRing &h = e->hring;
	CUDA_OK(cudaMemsetAsync(h.d_totals, 0, 2 * sizeof(unsigned long long), e->stream), "totals reset");
	uint64_t total_rows = 0;
	for (const Chunk &c : chunks)
		total_rows += c.rows;
	bool timed[HostRing::kBufs] = {false, false, false};
	double copy_ms = 0;
	uint64_t h2d = 0;
	auto collect = [&](unsigned b) {
		if (!timed[b])
			return;
		float ms = 0;
		cudaEventSynchronize(h.c1[b]);
		if (cudaEventElapsedTime(&ms, h.c0[b], h.c1[b]) == cudaSuccess)
			copy_ms += ms;
		timed[b] = false;
	};
	unsigned cur = 0;  /* h.d_totals[cur] holds the running count */
	for (size_t ci = 0; ci < chunks.size(); ci++) {
		const Chunk &c = chunks[ci];
		const unsigned b = (unsigned)(ci % HostRing::kBufs);
		collect(b);
		CUDA_OK(cudaStreamWaitEvent(e->copy_stream, h.freed[b], 0), "ring wait");
		CUDA_OK(cudaEventRecord(h.c0[b], e->copy_stream), "ring event");
		std::vector<SegDesc> ds(c.n);
		std::vector<uint32_t> rows(c.n);
		unsigned char *dst = h.mem[b];
		for (size_t k = 0; k < c.n; k++) {
			const Piece &pc = pieces[c.first + k];
			SegDesc &d = ds[k];
			memset(&d, 0, sizeof(d));
			d.rows = (uint32_t)pc.rows;
			rows[k] = d.rows;
			for (unsigned i = 0; i < P.nload; i++) {
				const size_t bytes = (size_t)pc.rows * P.load_stride[i];
				CUDA_OK(cudaMemcpyAsync(dst, pc.src[i], bytes, cudaMemcpyHostToDevice, e->copy_stream), "chunk copy");
				d.col[P.load_src[i]] = dst;
				dst += align256((size_t)padded_rows((uint32_t)pc.rows) * P.load_stride[i]);
				h2d += bytes;
			}
		}
		/* the descriptors are staged from host memory before the call returns */
		CUDA_OK(cudaMemcpyAsync(h.d_segs[b], ds.data(), ds.size() * sizeof(SegDesc), cudaMemcpyHostToDevice,
			e->copy_stream), "chunk descriptors");
		CUDA_OK(cudaEventRecord(h.c1[b], e->copy_stream), "ring event");
		timed[b] = true;
		CUDA_OK(cudaEventRecord(h.copied[b], e->copy_stream), "ring event");
		CUDA_OK(cudaStreamWaitEvent(e->stream, h.copied[b], 0), "ring wait");
		QueryLaunch q;
		q.prog = &P;
		q.d_segs = h.d_segs[b];
		q.nsegs = (uint32_t)c.n;
		q.seg_rows = rows.data();
		for (unsigned j = 0; j < P.nout; j++)
			q.out[j] = r->out[j];
		q.capacity = r->capacity;
		q.base_in = ci ? h.d_totals + cur : nullptr;
		q.d_total = h.d_totals + (cur ^ 1);
		q.block_counts = nullptr;
		if (!run_queries(e, std::vector<QueryLaunch>(1, q), nullptr))
			return 0;
		cur ^= 1;
		CUDA_OK(cudaEventRecord(h.freed[b], e->stream), "ring event");
	}
	for (unsigned b = 0; b < HostRing::kBufs; b++)
		collect(b);
	if (chunks.empty())
		r->ntiles_zero = true;
	else
		CUDA_OK(cudaMemcpyAsync(r->d_total, h.d_totals + cur, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
			e->stream), "result count");
	if (stats) {
		stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
		stats->copy_seconds = copy_ms / 1000.0;
		stats->h2d_bytes = h2d;
		stats->chunks = (unsigned)chunks.size();
	}
	(void)total_rows;
	return 1;
}

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
	uint64_t total_rows = 0, max_rows = 0;
	for (unsigned s = 0; s < nsegs; s++) {
		total_rows += segs[s].rows;
		max_rows = std::max<uint64_t>(max_rows, segs[s].rows);
		if (!segs[s].rows)
			continue;
		for (unsigned i = 0; i < P.nload; i++)
			VGPU_CHECK(load_ptr(P, segs[s], i) != nullptr, "segment %u lacks a column the program reads", s);
	}
	virg_gpu_result *r = nullptr;
	if (!result_alloc(e, P, total_rows, false, 0, &r))
		return 0;
	/* a chunk: segs_per_chunk of the largest segments' rows */
	if (!host_pipeline(e, P, segs, nsegs, std::max<uint64_t>(1, max_rows) * segs_per_chunk, r, stats)) {
		cudaStreamSynchronize(e->copy_stream);
		cudaStreamSynchronize(e->stream);
		virg_gpu_result_destroy(r);
		return 0;
	}
	*out = r;
	return 1;
}

/* ---- end to end from host buffers -------------------------------------- */

/* chunks of the end-to-end call: about this many bytes of the program's columns */
constexpr size_t kHostChunkBytes = 32u << 20;

extern "C" int virg_gpu_query_host(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_segment *segs, unsigned nsegs, void *const *out_cols, uint64_t capacity,
	uint64_t *out_rows)
{
	VGPU_CHECK(e != nullptr && p != nullptr && (segs != nullptr || nsegs == 0) && out_rows != nullptr,
		"null argument");
	CUDA_OK(cudaSetDevice(e->device), "set device");
	const Program &P = p->prog;
	uint64_t total_rows = 0;
	uint32_t bpr = 0;
	for (unsigned i = 0; i < P.nload; i++)
		bpr += P.load_stride[i];
	for (unsigned s = 0; s < nsegs; s++) {
		total_rows += segs[s].rows;
		if (!segs[s].rows)
			continue;
		for (unsigned i = 0; i < P.nload; i++)
			VGPU_CHECK(load_ptr(P, segs[s], i) != nullptr, "segment %u lacks a column the program reads", s);
	}
	std::lock_guard<std::mutex> lk(e->mu);
	virg_gpu_result *r = nullptr;
	if (!result_alloc(e, P, total_rows, false, 0, &r))
		return 0;
	int ok = host_pipeline(e, P, segs, nsegs, kHostChunkBytes / std::max<uint32_t>(bpr, 1), r, nullptr);
	uint64_t rows = 0;
	if (ok)
		ok = virg_gpu_result_rows(r, &rows);
	if (ok) {
		*out_rows = rows;
		const uint64_t n = std::min(rows, capacity);
		for (unsigned j = 0; j < P.nout && n && ok; j++) {
			const cudaError_t ce = cudaMemcpyAsync(out_cols[j], r->out[j], n * r->stride[j], cudaMemcpyDeviceToHost,
				e->stream);
			if (ce != cudaSuccess) {
				set_error("result copy: %s", cudaGetErrorString(ce));
				ok = 0;
			}
		}
		if (ok && cudaStreamSynchronize(e->stream) != cudaSuccess) {
			set_error("result copy sync failed");
			ok = 0;
		}
		if (ok && rows > capacity) {
			set_error("result has %llu rows, the buffers hold %llu", (unsigned long long)rows,
				(unsigned long long)capacity);
			ok = 0;
		}
	}
	cudaStreamSynchronize(e->copy_stream);
	cudaStreamSynchronize(e->stream);
	virg_gpu_result_destroy(r);
	return ok;
}
