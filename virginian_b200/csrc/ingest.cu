/*
 * Tablet ingest: a table of a Virginian database file read straight into a
 * resident table in the device layout.
 *
 * The reference brings tablets in one at a time through its host slot
 * cache: find a free 8 MB slot, pread the tablet's header and body into it
 * (src/db/load.c:22-98), lock it, and the GPU VM then copies columns out of
 * the slot for each query.  Here the tablets of one table are read from the
 * file (the tablet at disk slot i lives at block_size + i * VIRG_TABLET_SIZE,
 * found through the file's tablet-info array, src/db/load.c:45-66) into two
 * pinned staging buffers in turn, and each is copied into the table's device
 * segments on the engine's stream while the next one is read, so the file's
 * bytes go disk -> pinned -> HBM once, with no slot cache, locks or per-query
 * copies.  The chain follows each tablet's `next` until `last_tablet`, as the
 * reference's scans do.
 */
#include <fcntl.h>
#include <unistd.h>

#include <cstring>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "virginian_b200.h"
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

/* read exactly n bytes at off */
bool pread_all(int fd, void *dst, size_t n, off_t off)
{
	unsigned char *p = static_cast<unsigned char *>(dst);
	while (n) {
		const ssize_t r = pread(fd, p, n, off);
		if (r <= 0)
			return false;
		p += r;
		n -= (size_t)r;
		off += r;
	}
	return true;
}

struct Staging {
	void *buf[2] = {nullptr, nullptr};
	cudaEvent_t ev[2] = {nullptr, nullptr};
	int fd = -1;
	~Staging()
	{
		for (int b = 0; b < 2; b++) {
			if (ev[b]) {
				cudaEventSynchronize(ev[b]);
				cudaEventDestroy(ev[b]);
			}
			if (buf[b])
				cudaFreeHost(buf[b]);
		}
		if (fd >= 0)
			close(fd);
	}
};

}  // namespace

extern "C" int virg_gpu_table_load_db(virg_gpu_table *t, const char *path, const char *table, uint64_t *rows_out)
{
	VGPU_CHECK(t != nullptr && path != nullptr && table != nullptr, "null argument");
	virg_gpu_engine *e = t->e;
	CUDA_OK(cudaSetDevice(e->device), "set device");
	Staging st;
	st.fd = open(path, O_RDONLY);
	VGPU_CHECK(st.fd >= 0, "cannot open database file %s", path);
	virg_db db;
	VGPU_CHECK(pread_all(st.fd, &db, sizeof(db), 0), "%s: short database header", path);
	VGPU_CHECK(db.alloced_tablets > 0 && db.alloced_tablets < (1u << 24) &&
		db.block_size >= sizeof(virg_db) + (size_t)db.alloced_tablets * sizeof(virg_tablet_info),
		"%s: not a Virginian database file of this build's layout", path);
	std::vector<virg_tablet_info> info(db.alloced_tablets);
	VGPU_CHECK(pread_all(st.fd, info.data(), info.size() * sizeof(virg_tablet_info), sizeof(virg_db)),
		"%s: short tablet table", path);
	int ti = -1;
	for (int i = 0; i < VIRG_MAX_TABLES && ti < 0; i++)
		if (db.table_status[i] && strncmp(db.tables[i], table, VIRG_MAX_TABLE_NAME) == 0)
			ti = i;
	VGPU_CHECK(ti >= 0, "%s: no table named %s", path, table);
	std::map<unsigned, unsigned> disk_slot;  /* tablet id -> its place in the file */
	for (unsigned i = 0; i < db.alloced_tablets; i++)
		if (info[i].used == 1)
			disk_slot[info[i].id] = i;

	for (int b = 0; b < 2; b++) {
		CUDA_OK(cudaHostAlloc(&st.buf[b], VIRG_TABLET_SIZE, cudaHostAllocDefault), "pinned staging");
		CUDA_OK(cudaEventCreateWithFlags(&st.ev[b], cudaEventDisableTiming), "staging event");
	}
	/* a row sample from tablets spread over the table (estimates only) */
	const unsigned every = std::max(1u, db.table_tablets[ti] / 64u);
	uint64_t total = 0;
	unsigned id = db.first_tablet[ti];
	for (unsigned k = 0;; k++) {
		VGPU_CHECK(k < db.alloced_tablets, "%s: tablet chain of %s does not end", path, table);
		auto it = disk_slot.find(id);
		VGPU_CHECK(it != disk_slot.end(), "%s: tablet %u of %s is not in the file", path, id, table);
		const unsigned b = k & 1u;
		/* the buffer's previous tablet has been copied to the device */
		CUDA_OK(cudaEventSynchronize(st.ev[b]), "staging reuse");
		const off_t at = (off_t)db.block_size + (off_t)it->second * VIRG_TABLET_SIZE;
		virg_tablet_meta *m = static_cast<virg_tablet_meta *>(st.buf[b]);
		VGPU_CHECK(pread_all(st.fd, m, sizeof(virg_tablet_meta), at), "%s: short tablet header", path);
		VGPU_CHECK(m->size >= sizeof(virg_tablet_meta) && m->size <= VIRG_TABLET_SIZE && m->rows <= m->possible_rows,
			"%s: corrupt tablet %u", path, id);
		VGPU_CHECK(pread_all(st.fd, reinterpret_cast<unsigned char *>(m) + sizeof(virg_tablet_meta),
			m->size - sizeof(virg_tablet_meta), at + (off_t)sizeof(virg_tablet_meta)), "%s: short tablet %u", path, id);
		VGPU_CHECK(m->fixed_columns == t->schema.ncols && (int)m->key_type == t->schema.key_type,
			"tablet %u of %s has %u columns (key type %d), the table %u (key type %d)", id, table, m->fixed_columns,
			(int)m->key_type, t->schema.ncols, t->schema.key_type);
		virg_gpu_segment seg;
		memset(&seg, 0, sizeof(seg));
		seg.rows = m->rows;
		const unsigned char *base = reinterpret_cast<const unsigned char *>(m);
		seg.key = base + m->key_block;
		for (unsigned c = 0; c < m->fixed_columns; c++) {
			VGPU_CHECK((int)m->fixed_type[c] == t->schema.col_type[c], "tablet %u of %s: column %u has type %d, the table %d",
				id, table, c, (int)m->fixed_type[c], t->schema.col_type[c]);
			VGPU_CHECK(m->fixed_block + m->fixed_offset[c] + (size_t)m->rows * m->fixed_stride[c] <= m->size,
				"%s: corrupt tablet %u", path, id);
			seg.col[c] = base + m->fixed_block + m->fixed_offset[c];
		}
		if (seg.rows) {
			if (!table_add_segments(t, &seg, 1, nullptr, true, e->stream))
				return 0;
			CUDA_OK(cudaEventRecord(st.ev[b], e->stream), "staging event");
			if (k % every == 0)
				table_sample(t, &seg, 1);
		}
		total += m->rows;
		if (m->last_tablet)
			break;
		id = m->next;
	}
	CUDA_OK(cudaStreamSynchronize(e->stream), "table copy");
	if (rows_out)
		*rows_out = total;
	return table_sync_desc(t);
}
