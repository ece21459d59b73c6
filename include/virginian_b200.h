/*
 * virginian_b200.h - C ABI of the B200 (sm_100a) query VM for Virginian.
 *
 * Two groups of entry points:
 *
 * 1. The drop-in GPU VM.  virg_vm_gpu and virg_gpu_getsizes have exactly the
 *    reference's signatures (src/virginian.h:620-622) and replace
 *    src/vm/vm_gpu.cu in the reference's build.  virg_vm_execute
 *    (src/vm/execute.c:85-86) calls virg_vm_gpu at OP_Parallel when
 *    v->use_gpu is set; the reference's host library (tablet slot cache,
 *    result allocation, reader) stays as it is.
 *
 * 2. The engine API (virg_gpu_*): plain pointers and sizes, no reference
 *    structs except the opcode program itself (virg_op).  It exposes what the
 *    drop-in is built on: HBM-resident tables, one-launch queries with ordered
 *    output, host-buffer (end-to-end) queries, streamed execution of
 *    host-resident tables, batched persistent execution of many queries and a
 *    continuous-batching serving loop.  None of these has a reference
 *    counterpart; the reference runs one query per launch sequence.
 *
 * Every call returns VIRG_SUCCESS (1) or VIRG_FAIL (0), the reference's
 * convention (src/virginian.h:118-121); virg_gpu_last_error() gives the
 * reason for the calling thread's last failure.
 *
 * The reference's types below are declared with identical layouts
 * (src/virginian.h:166-503) so this header can stand alone; when the
 * reference's virginian.h is included first (it defines VIRGINIAN) the
 * declarations here are skipped and the reference's own are used.
 */
#ifndef VIRGINIAN_B200_H
#define VIRGINIAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifndef VIRGINIAN
#include <pthread.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#ifndef VIRGINIAN
/* ---- reference ABI (src/virginian.h), layouts must stay identical ---- */
#define VIRG_FAIL 0
#define VIRG_SUCCESS 1
#define VIRG_MAX_COLUMNS 16
#define VIRG_MAX_TABLES 16
#define VIRG_MAX_COLUMN_NAME 16
#define VIRG_MAX_TABLE_NAME 32
#define VIRG_MEM_TABLETS 64
#define VIRG_TABLET_SIZE (8 * 1024 * 1024)
#define VIRG_REGS 16
#define VIRG_GLOBAL_REGS 16
#define VIRG_OPS 32
#define VIRG_VM_TABLES 1
#define VIRG_ROW_BUFFER 256

/* opcodes, src/virginian.h:166-193 */
typedef enum {
	OP_Table = 0, OP_ResultColumn = 1, OP_Parallel = 2, OP_Finish = 3,
	OP_Column = 4, OP_Rowid = 5, OP_Result = 6, OP_Converge = 7,
	OP_Invalid = 8, OP_Cast = 9, OP_Integer = 10, OP_Float = 11,
	OP_Le = 12, OP_Lt = 13, OP_Ge = 14, OP_Gt = 15, OP_Eq = 16, OP_Neq = 17,
	OP_Add = 18, OP_Sub = 19, OP_Mul = 20, OP_Div = 21,
	OP_And = 22, OP_Or = 23, OP_Not = 24, OP_Nop = 25
} virg_ops;

/* value types, src/virginian.h:196-204 */
typedef enum {
	VIRG_INT = 0, VIRG_INT64 = 1, VIRG_FLOAT = 2, VIRG_DOUBLE = 3,
	VIRG_CHAR = 4, VIRG_STRING = 5, VIRG_NULL = 6
} virg_t;

/* src/virginian.h:227-234 */
typedef struct {
	unsigned id;
	int used;
	unsigned disk_slot;
} virg_tablet_info;

/* tablet header, src/virginian.h:251-302 */
typedef struct {
	unsigned rows;
	virg_t key_type;
	size_t key_stride;
	size_t key_pointer_stride;
	unsigned id;
	unsigned next;
	int last_tablet;
	int in_table;
	unsigned table_id;
	size_t key_block;
	size_t key_pointers_block;
	size_t fixed_block;
	size_t variable_block;
	size_t size;
	unsigned possible_rows;
	size_t row_stride;
	unsigned fixed_columns;
	char fixed_name[VIRG_MAX_COLUMNS][VIRG_MAX_COLUMN_NAME];
	virg_t fixed_type[VIRG_MAX_COLUMNS];
	size_t fixed_stride[VIRG_MAX_COLUMNS];
	size_t fixed_offset[VIRG_MAX_COLUMNS];
	virg_tablet_info *info;
} __attribute__((aligned(64))) virg_tablet_meta;

/* opcode argument, src/virginian.h:309-317 */
typedef union {
	int i;
	float f;
	long long int li;
	double d;
	char c;
	char *s;
} __attribute__((aligned(8))) virg_var;

/* one opcode, src/virginian.h:327-333 */
typedef struct {
	int op;
	int p1;
	int p2;
	int p3;
	virg_var p4;
} virg_op;

/* src/virginian.h:341-346 */
typedef struct virg_result_node_ {
	unsigned id;
	struct virg_result_node_ *next;
} virg_result_node;

/* opcode program + result list, src/virginian.h:356-377 */
typedef struct {
	unsigned pc;
	virg_op stmt[VIRG_OPS];
	unsigned num_ops;
	virg_var global_reg[VIRG_GLOBAL_REGS];
	virg_t type[VIRG_GLOBAL_REGS];
	unsigned table[VIRG_VM_TABLES];
	unsigned num_tables;
	virg_result_node *head_result;
	virg_result_node *tail_result;
	float timing1, timing2, timing3;
} virg_vm;

/* database file state, src/virginian.h:427-458 */
typedef struct {
	unsigned num_tablets;
	unsigned alloced_tablets;
	unsigned tablet_id_counter;
	size_t block_size;
	char tables[VIRG_MAX_TABLES][VIRG_MAX_TABLE_NAME];
	unsigned first_tablet[VIRG_MAX_TABLES];
	unsigned last_tablet[VIRG_MAX_TABLES];
	unsigned write_cursor[VIRG_MAX_TABLES];
	unsigned table_tablets[VIRG_MAX_TABLES];
	int table_status[VIRG_MAX_TABLES];
	virg_tablet_info *tablet_info;
} virg_db;

/* database state, src/virginian.h:468-503 */
typedef struct {
	virg_db db;
	unsigned tablet_slot_ids[VIRG_MEM_TABLETS];
	int tablet_slot_status[VIRG_MEM_TABLETS];
	unsigned tablet_slots_taken;
	unsigned tablet_slot_counter;
	virg_tablet_meta *tablet_slots[VIRG_MEM_TABLETS];
	void *gpu_slots;
	pthread_mutex_t slot_lock;
	int dbfd;
	unsigned threads_per_block;
	unsigned multi_threads;
	int use_multi;
	int use_gpu;
	int use_stream;
	int use_mmap;
} virginian;

/* src/virginian.h:512-523 */
typedef struct {
	virginian *v;
	virg_vm *vm;
	virg_tablet_meta *tab;
	virg_tablet_meta *res;
	unsigned row;
	unsigned num_rows;
	unsigned num_tablets;
	unsigned tablets_proced;
	pthread_mutex_t tab_lock;
	pthread_mutex_t res_lock;
} virg_vm_arg;

/* src/virginian.h:532-541 */
typedef struct {
	virg_vm *vm;
	virg_tablet_meta *res;
	unsigned row;
	char buffer[VIRG_ROW_BUFFER];
} virg_reader;
#endif /* VIRGINIAN */

/* ======================================================================
 * 1. Drop-in GPU VM
 * ====================================================================== */

/*
 * Replaces virg_vm_gpu (src/virginian.h:620-621, src/vm/vm_gpu.cu:107-578).
 * Runs the data-parallel section of vm (from vm->pc to its OP_Converge) over
 * the tablet chain starting at tab[0] and appends result rows to res[0],
 * allocating further result tablets with virg_vm_allocresult.  Result rows
 * are in original row order and split across result tablets exactly as the
 * single-core CPU VM splits them (src/vm/virginia.c:518-524).  On return,
 * tab[0] and res[0] are the final data and result tablets with one lock each,
 * as virg_vm_execute's OP_Finish expects (src/vm/execute.c:92-96).
 * num_tablets = 0 processes the whole chain.  vm->timing1..3 receive the
 * host-to-device, kernel and device-to-host times in seconds.
 */
int virg_vm_gpu(virginian *v, virg_vm *vm, virg_tablet_meta **tab,
	virg_tablet_meta **res, unsigned num_tablets);

/*
 * Replaces virg_gpu_getsizes (src/virginian.h:622, src/vm/vm_gpu.cu:27-30):
 * the 15 struct sizes of virg_testsizes (src/virginian.h:553-569) as this
 * library was compiled, for the host/GPU layout check of
 * src/test/virgstate.cc:64-80.
 */
const size_t *virg_gpu_getsizes(void);

/*
 * Residency cache of the drop-in (no reference counterpart; the reference
 * copies every tablet for every query, src/vm/vm_gpu.cu:147-160): with a
 * capacity in bytes, virg_vm_gpu keeps the data tablets it copies to HBM
 * (every column and the key, keyed by tablet id, checked against the
 * tablet's row count and host slot), evicting the least recently used.  0
 * (the default) turns it off and frees it; clear it after rebuilding a table
 * under the same tablet ids.  Stats: cache hits and misses of virg_vm_gpu
 * and bytes held.
 */
int virg_gpu_dropin_cache(uint64_t bytes);
int virg_gpu_dropin_cache_stats(uint64_t *hits, uint64_t *misses, uint64_t *bytes);

/* ======================================================================
 * 2. Engine API (no reference counterpart)
 * ====================================================================== */

typedef struct virg_gpu_engine virg_gpu_engine;
typedef struct virg_gpu_program virg_gpu_program;
typedef struct virg_gpu_table virg_gpu_table;
typedef struct virg_gpu_result virg_gpu_result;
typedef struct virg_gpu_batch virg_gpu_batch;
typedef struct virg_serve virg_serve;

/* column types of a table, in the reference's virg_t numbering */
typedef struct {
	int key_type;
	unsigned ncols;
	int col_type[VIRG_MAX_COLUMNS];
} virg_gpu_schema;

/* one tablet's columns as plain pointers: rows, the key column (read by
 * OP_Rowid) and each fixed column (read by OP_Column); host or device memory
 * depending on the call */
typedef struct {
	uint32_t rows;
	const void *key;
	const void *col[VIRG_MAX_COLUMNS];
} virg_gpu_segment;

/* what a compiled program reads and writes */
typedef struct {
	unsigned nload;                 /* distinct columns read */
	int load_column[VIRG_MAX_COLUMNS + 1]; /* column index, -1 = key */
	unsigned load_bytes_per_row;    /* sum of their strides */
	unsigned nout;                  /* result columns */
	int out_type[VIRG_MAX_COLUMNS];
	unsigned out_stride[VIRG_MAX_COLUMNS];
	unsigned out_bytes_per_row;
	unsigned nuops;                 /* interpreted device ops */
	unsigned row_vector_bytes;      /* per row: register vectors the filter writes */
	unsigned sel_vector_bytes;      /* per row: register vectors only the projection writes */
} virg_gpu_program_info;

/* thread-local description of the last failure on this thread */
const char *virg_gpu_last_error(void);

/* engine: one per device; owns its stream, scratch and caches */
int virg_gpu_engine_create(int device, virg_gpu_engine **out);
void virg_gpu_engine_destroy(virg_gpu_engine *e);
/* the engine's CUDA stream (a cudaStream_t), for event timing by callers */
void *virg_gpu_engine_stream(virg_gpu_engine *e);
/* device error word set by bounded waits inside kernels (0 = none); reading
 * it synchronises the engine stream and clears it */
int virg_gpu_engine_check(virg_gpu_engine *e, unsigned *device_error);
/* launch shape: compute threads per CTA (128, 256, 320, 448 or 512; the CTA adds a
 * producer and a look-back warp), bytes per staging buffer in KB, number of
 * staging buffers, CTAs per SM; 0 in a field keeps the automatic choice */
int virg_gpu_engine_set_shape(virg_gpu_engine *e, unsigned threads,
	unsigned stage_kb, unsigned stages, unsigned ctas_per_sm);
/* upper bound on the rows of a chunk (the unit a CTA claims and places in
 * the ordered result): a multiple of 256 in [256, 8192], 0 for automatic */
int virg_gpu_engine_set_chunk_rows(virg_gpu_engine *e, unsigned rows);
/* how the full phase reads the columns the results need: 0 (default)
 * stages tiles of them and reads the selected rows in place, 1 loads only
 * the selected rows' values straight from device memory (programs whose
 * results read at most 32 bytes per row), 2 runs the projection over every
 * row of a staged group and stores the rows that pass at their ranks
 * (programs whose computed values take at most 16 bytes per row; suits
 * filters that keep most rows).  Programs outside a mode's bounds, and
 * launches whose shape leaves no room for mode 2, keep mode 0. */
int virg_gpu_engine_set_full_mode(virg_gpu_engine *e, unsigned mode);
/* shared scans (off by default): in a launch of several queries, the
 * queries over the same table claim its chunks interleaved, so each chunk's
 * columns are read from device memory once and from L2 by the others.  Each
 * claim then usually changes query, which costs the producer a descriptor
 * load and the chunk slot a descriptor copy; on the bench's batch of 256
 * generated queries that outweighs the L2 reuse (11.3 ms against 9.5 ms) */
int virg_gpu_engine_set_shared_scan(virg_gpu_engine *e, int enable);
/* record CUDA events around each of the next kernel launches in a ring of
 * `slots` entries (0 turns it off) */
int virg_gpu_engine_timing(virg_gpu_engine *e, unsigned slots);
/* device durations (ms) of up to the last n timed launches, oldest first;
 * waits for the last one to finish */
int virg_gpu_engine_kernel_times(virg_gpu_engine *e, float *ms, unsigned n, unsigned *got);
/* how many kernels the engine has launched since creation */
unsigned long long virg_gpu_engine_launches(virg_gpu_engine *e);
/* launch shape chosen for the engine's last launch: shape4 = {compute
 * threads, stage KB, stages, CTAs per SM requested}, grid size, shared memory */
int virg_gpu_engine_last_launch(virg_gpu_engine *e, unsigned *shape4, unsigned *grid,
	unsigned *smem);

/* validate and decode the data-parallel section of a reference opcode
 * program (ops[pc] up to its OP_Converge) for a table schema; host only */
int virg_gpu_program_create(const virg_op *ops, unsigned num_ops, unsigned pc,
	const virg_gpu_schema *schema, virg_gpu_program **out);
int virg_gpu_program_info_get(const virg_gpu_program *p, virg_gpu_program_info *info);
/* 1 when some still-valid row can read a register its path never set (the
 * reference CPU VM then reads a stale lane), 0 otherwise */
int virg_gpu_program_flags(const virg_gpu_program *p);
void virg_gpu_program_destroy(virg_gpu_program *p);

/* Re-entrant SQL front end.  Emits the same opcode program as the
 * reference's parser and code generator (src/sql/sql.y:78-240,
 * src/sql/generate.c:820) for SELECT statements over catalog tables.
 * ops receives up to VIRG_OPS ops (ResultColumn p4 is left NULL; the names go
 * to names[k * VIRG_MAX_COLUMN_NAME] for op k), *pc the first op of the
 * data-parallel section, *table_id the table's catalog index. */
typedef struct virg_gpu_catalog virg_gpu_catalog;
int virg_gpu_catalog_create(virg_gpu_catalog **out);
int virg_gpu_catalog_add_table(virg_gpu_catalog *c, const char *name, int key_type,
	unsigned ncols, const char *const *col_names, const int *col_types, unsigned *table_id);
void virg_gpu_catalog_destroy(virg_gpu_catalog *c);
int virg_gpu_sql_compile(const virg_gpu_catalog *c, const char *sql, virg_op *ops,
	unsigned *num_ops, unsigned *pc, char *names, unsigned *table_id);

/* HBM-resident table: segments are copied from host (or device) memory into
 * 256-byte-aligned device columns and stay resident until destroyed */
int virg_gpu_table_create(virg_gpu_engine *e, const virg_gpu_schema *schema,
	virg_gpu_table **out);
int virg_gpu_table_append(virg_gpu_table *t, const virg_gpu_segment *segs,
	unsigned nsegs);
uint64_t virg_gpu_table_rows(const virg_gpu_table *t);
uint64_t virg_gpu_table_bytes(const virg_gpu_table *t);
void virg_gpu_table_destroy(virg_gpu_table *t);

/* run a program over a resident table; the ordered result stays in HBM.
 * Asynchronous on the engine stream; virg_gpu_result_rows waits for it. */
int virg_gpu_query(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_table *t, virg_gpu_result **out);
/* time the candidate launch shapes for this program over this table and
 * cache the fastest in the engine (keyed by program shape and table size
 * class); later queries with the same key use it.  shape4 (may be NULL)
 * receives {compute threads, stage KB, stages, CTAs per SM}. */
int virg_gpu_query_tune(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_table *t, unsigned *shape4);
int virg_gpu_result_rows(virg_gpu_result *r, uint64_t *rows);
/* device pointer of result column c (valid until the result is destroyed) */
const void *virg_gpu_result_column(const virg_gpu_result *r, unsigned c);
/* copy rows [first, first+count) of every result column to host buffers */
int virg_gpu_result_download(virg_gpu_result *r, void *const *host_cols,
	uint64_t first, uint64_t count);
void virg_gpu_result_destroy(virg_gpu_result *r);

/* read-bandwidth ceiling of a resident table (a measurement aid, no
 * reference counterpart): reads every listed column (-1 for the key) of
 * every segment, mode 0 with 16-byte loads, modes 1-3 with bulk copies into
 * a shared-memory ring of 4, 6 or 2 stages of 32 KB, and returns the best
 * device time of `reps` launches (ms) and the bytes one launch reads */
int virg_gpu_table_read_ceiling(virg_gpu_table *t, const int *cols, unsigned ncols, unsigned mode,
	unsigned reps, double *ms, unsigned long long *bytes);

/* Ingest, replacing the host-slot path src/db/load.c:22-98 for a resident
 * table: appends every tablet of table `table` of the Virginian database file
 * at `path` (this build's struct layout) to t, following the tablet chain;
 * tablets are read into pinned buffers and copied to the device while the
 * next is read.  *rows receives the rows appended. */
int virg_gpu_table_load_db(virg_gpu_table *t, const char *path, const char *table, uint64_t *rows);

/* No counterpart in the reference.  An estimate of the rows a program's
 * filter keeps in a table: the share of the table's host row sample (runs
 * of rows taken from segments spread over each append) the filter keeps,
 * times the table's rows.  Sizes reservations; never used for results. */
int virg_gpu_table_estimate(const virg_gpu_table *t, const virg_gpu_program *p, uint64_t *rows);

/* end to end: host segments in, host result columns out.  Copies the
 * referenced columns to the device, runs the program and copies the result
 * rows back; out_cols[c] must hold `capacity` rows of result column c. */
int virg_gpu_query_host(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_segment *segs, unsigned nsegs, void *const *out_cols,
	uint64_t capacity, uint64_t *out_rows);

/* No counterpart in the reference.  One program over one segment whose
 * columns are already in device memory (16-byte aligned, each readable up to
 * the next multiple of 16 bytes past its last row), writing the result rows,
 * in the reference's order, to caller-owned device buffers that hold
 * `capacity` rows each.  It allocates nothing, in device or host memory: for
 * callers whose allocator owns the device's free memory, or that must not
 * reach the CUDA allocator on a latency-critical path.  Its scratch is a
 * fixed device array of about 520 KB, so a segment has at most 67,108,864
 * rows (2^26); larger ones are refused before any launch.  The first call on
 * each device (with that device current) looks up the array's address; make
 * it before any stream capture.  Runs on `stream` (a cudaStream_t, NULL for
 * the default stream) and waits for it to return the row count in *out_rows.
 * All calls on a device share the array: calls that overlap in time (other
 * streams or host threads) race; run them one after another.
 * When the result has more rows than `capacity` the call returns 0 with an
 * error naming both counts, *out_rows still holds the full row count, and the
 * buffers hold the result's first `capacity` rows; nothing carries over to
 * the next call. */
int virg_gpu_query_prealloc(const virg_gpu_program *p, const virg_gpu_segment *seg,
	void *const *out_cols, uint64_t capacity, uint64_t *out_rows, void *stream);

/* Streamed execution over host-resident segments (tablets larger than HBM
 * residency allows): the columns the program reads are copied in chunks of
 * segs_per_chunk segments (0 = 8) through a ring of device staging buffers on
 * the engine's copy stream while the VM runs on earlier chunks; the ordered
 * result stays in HBM.  Segments should be in pinned host memory for the
 * copies to overlap.  stats (may be NULL) receives the wall time, the time
 * the copy stream spent copying and the bytes copied. */
typedef struct {
	double seconds;
	double copy_seconds;
	uint64_t h2d_bytes;
	unsigned chunks;
} virg_gpu_stream_stats;
int virg_gpu_query_streamed(virg_gpu_engine *e, const virg_gpu_program *p,
	const virg_gpu_segment *segs, unsigned nsegs, unsigned segs_per_chunk,
	virg_gpu_result **out, virg_gpu_stream_stats *stats);

/* Batched persistent execution: the queries added to a batch run in one
 * launch of the VM kernel (chunks of all queries in one ordered work list),
 * or up to three: a launch's compute warps hold vector areas for its widest
 * program, so programs too wide for three 48 KB data buffers beside eight
 * compute warps run in a launch of their own and leave the others their
 * larger buffers, and of the others those whose table's row sample says
 * they keep at least half of the rows run apart, so each launch is tuned
 * for its kind (the dense full phase suits mostly-kept rows).  A batch owns its descriptors and counters, so
 * virg_gpu_batch_run with use_graph captures its launches in a CUDA graph
 * once and replays it after.  With autotune on, the first run times the
 * candidate launch shapes for each launch on the batch and caches the
 * fastest in the engine per program-shape key.  Adding a query after a run
 * rebuilds the batch. */
int virg_gpu_batch_create(virg_gpu_engine *e, virg_gpu_batch **out);
int virg_gpu_batch_add(virg_gpu_batch *b, const virg_gpu_program *p, virg_gpu_table *t,
	unsigned *slot);
int virg_gpu_batch_set_autotune(virg_gpu_batch *b, int enable);
int virg_gpu_batch_run(virg_gpu_batch *b, int use_graph);
/* waits for the last run; fails if the device reported an error */
int virg_gpu_batch_wait(virg_gpu_batch *b);
int virg_gpu_batch_rows(virg_gpu_batch *b, unsigned slot, uint64_t *rows);
const void *virg_gpu_batch_column(const virg_gpu_batch *b, unsigned slot, unsigned c);
int virg_gpu_batch_download(virg_gpu_batch *b, unsigned slot, void *const *host_cols,
	uint64_t first, uint64_t count);
/* shape4 = {compute threads, stage KB, stages, grid} of the launch with the
 * most chunks; work = chunks of all launches */
int virg_gpu_batch_shape(const virg_gpu_batch *b, unsigned *shape4, uint64_t *work);
void virg_gpu_batch_destroy(virg_gpu_batch *b);

/* Serving loop (no reference counterpart; the reference runs one query per
 * launch sequence, src/vm/execute.c:85-86).  A scheduler thread keeps one
 * persistent VM kernel running over the engine's resident tables and folds
 * submitted queries into it while it runs (continuous batching): queries are
 * admitted in arrival order while the result budget has room for their
 * estimated result size, their descriptors are uploaded and published to
 * the running kernel through a doorbell in host-mapped memory, and the
 * kernel reports each finished query in a completion record.  A query whose
 * rows exceed its estimate is admitted again with its exact row count.
 * Results stay in the result budget's device memory until released.  Tables
 * must not be appended to while queries over them are in flight.  A
 * session's kernel holds vector areas for the programs it may take: the
 * bounds below size a wide layout; programs of at most 8 filter-vector and
 * 20 projection-vector bytes per row also fit a narrow layout with three
 * 48 KB data buffers, which a session uses while the queries at the head
 * of the queue fit it (a query that does not ends the session once its
 * queries are done, and the next session takes the other layout; arrival
 * order is kept). */
typedef struct {
	uint64_t result_budget_bytes;    /* device memory for results (0: 20 GB) */
	unsigned max_queries;            /* queries per kernel session (0: 4096) */
	unsigned idle_us;                /* end an idle session after this long (0: 50000) */
	unsigned max_load_bytes_per_row; /* staged column bytes a program may read (0: 32) */
	unsigned max_row_vector_bytes;   /* filter register-vector bytes per row (0: 12) */
	unsigned max_sel_vector_bytes;   /* projection register-vector bytes per row (0: 20) */
	unsigned wait_limit_ms;          /* bound of the kernel's waits (0: 60000) */
} virg_serve_config;

typedef struct {
	int done;                        /* rows are stored */
	uint64_t rows;
	unsigned readmits;               /* admissions after an estimate proved short */
	double queue_us;                 /* submission to (last) admission */
	double latency_us;               /* submission to completion seen by the host */
} virg_serve_status;

typedef struct {
	unsigned sessions;               /* kernel sessions launched */
	unsigned long long admitted, readmitted;
	unsigned long long pending, inflight;
	unsigned long long arena_used;   /* result bytes reserved */
	unsigned device_error;           /* first device error of any session */
	unsigned shape[4];               /* compute threads, stage KB, stages, grid */
	unsigned long long restarts;     /* sessions that ended by themselves (a
	                                  * bounded wait ran out); their unfinished
	                                  * queries ran again in the next session */
	unsigned long long work_items;   /* work items (query chunks) published to the
	                                  * running session */
	unsigned long long status_ring;  /* look-back words of a session's ring; work
	                                  * item i uses word i mod status_ring */
	unsigned long long sampled;      /* submissions whose reservation came from the
	                                  * table's row sample */
} virg_serve_counters;

int virg_serve_create(virg_gpu_engine *e, const virg_serve_config *cfg, virg_serve **out);
/* queue a query; estimated_rows 0 reserves the rows the same program last
 * returned on the same table, plus a quarter, else the fraction of the
 * table's host row sample the program's filter keeps, times its rows, plus
 * a quarter (else the bound, the table's rows); a short reservation is
 * admitted again with the exact rows */
int virg_serve_submit(virg_serve *s, const virg_gpu_program *p, virg_gpu_table *t,
	uint64_t estimated_rows, uint64_t *ticket);
/* a query's state; wait_ms < 0 waits for completion, > 0 up to that long.
 * Fails for a query whose exact result rows need more memory than the
 * whole result budget (found after it ran with a shorter estimate). */
int virg_serve_poll(virg_serve *s, uint64_t ticket, int wait_ms, virg_serve_status *st);
/* copy a completed query's rows to host buffers, one per result column;
 * submissions go on meanwhile (the copy runs outside the loop's lock), so a
 * ticket must not be released while it is being downloaded */
int virg_serve_download(virg_serve *s, uint64_t ticket, void *const *host_cols);
/* device pointer of result column c of a completed query */
const void *virg_serve_column(virg_serve *s, uint64_t ticket, unsigned c);
/* free a completed query's result memory */
int virg_serve_release(virg_serve *s, uint64_t ticket);
int virg_serve_stats(virg_serve *s, virg_serve_counters *c);
/* stops the scheduler and the running session */
void virg_serve_destroy(virg_serve *s);

#ifdef __cplusplus
}
#endif

#endif /* VIRGINIAN_B200_H */
