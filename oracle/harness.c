/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg, always as the checker or as the timed CPU
 * baseline, never as part of the product path.
 *
 * Thin helpers over the reference's own public API so Python (ctypes) can
 * build a database, load seeded columns, compile a query with the reference's
 * code generator and run the reference's CPU virtual machines:
 *   - tables are created with virg_table_create/virg_table_addcolumn and
 *     filled row by row with virg_table_insert (src/table/insert.c:38-88),
 *     exactly as the reference's own generator does (db/generate.c:41-48);
 *   - queries compile through virg_sql (oracle/sql_parse.c) and the
 *     reference's virg_sql_generate;
 *   - execution is virg_vm_execute (src/vm/execute.c:28) with the single-core
 *     (virginia_single) or multi-core (virginia_multi) VM selected through the
 *     virginian struct fields, timed like src/test/timing.cc:49-56;
 *   - results are read by walking the result-tablet chain directly, because
 *     virg_reader_row drops the final row (src/reader/row.c:42-47).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "virginian.h"

typedef struct {
	virginian v;
	char path[256];
} orc_db;

typedef struct {
	virg_vm *vm;
	unsigned ncols;
	int types[VIRG_MAX_COLUMNS];
	unsigned strides[VIRG_MAX_COLUMNS];
	unsigned long long rows;
	unsigned ntablets;
	double seconds;
} orc_result;

static double now_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + ts.tv_nsec * 1e-9;
}

orc_db *orc_open(const char *dir)
{
	static unsigned counter = 0;
	orc_db *d = calloc(1, sizeof(orc_db));
	if(!d)
		return NULL;
	snprintf(d->path, sizeof(d->path), "%s/oracle_db_%d_%u", dir, (int)getpid(), counter++);
	unlink(d->path);
	if(virg_init(&d->v) != VIRG_SUCCESS || virg_db_create(&d->v, d->path) != VIRG_SUCCESS) {
		free(d);
		return NULL;
	}
	return d;
}

void orc_close(orc_db *d)
{
	virg_close(&d->v);
	unlink(d->path);
	free(d);
}

/* closes the database, which writes every tablet to its file
 * (src/db/close.c:20-50), and keeps the file; its path goes to path_out */
int orc_close_keep(orc_db *d, char *path_out, unsigned n)
{
	snprintf(path_out, n, "%s", d->path);
	int ok = virg_close(&d->v) == VIRG_SUCCESS;
	free(d);
	return ok;
}

virginian *orc_virginian(orc_db *d) { return &d->v; }

int orc_create_table(orc_db *d, const char *name, int key_type, unsigned ncols,
	const char *const *names, const int *types, unsigned *table_id)
{
	unsigned i;
	if(virg_table_create(&d->v, name, (virg_t)key_type) != VIRG_SUCCESS)
		return VIRG_FAIL;
	if(virg_table_getid(&d->v, name, table_id) != VIRG_SUCCESS)
		return VIRG_FAIL;
	for(i = 0; i < ncols; i++)
		if(virg_table_addcolumn(&d->v, *table_id, names[i], (virg_t)types[i]) != VIRG_SUCCESS)
			return VIRG_FAIL;
	return VIRG_SUCCESS;
}

/* append rows given as one key array plus one array per fixed column */
int orc_insert(orc_db *d, unsigned table_id, unsigned long long nrows,
	const void *keys, unsigned key_stride, unsigned ncols,
	const void *const *cols, const unsigned *strides)
{
	unsigned long long r;
	unsigned c;
	size_t row_bytes = 0;
	for(c = 0; c < ncols; c++)
		row_bytes += strides[c];
	char *buf = malloc(row_bytes ? row_bytes : 1);
	char key[8];
	for(r = 0; r < nrows; r++) {
		char *p = buf;
		for(c = 0; c < ncols; c++) {
			memcpy(p, (const char*)cols[c] + r * strides[c], strides[c]);
			p += strides[c];
		}
		memcpy(key, (const char*)keys + r * key_stride, key_stride);
		virg_table_insert(&d->v, table_id, key, buf, NULL);
	}
	free(buf);
	return VIRG_SUCCESS;
}

int orc_loadmem(orc_db *d, unsigned table_id)
{
	return virg_table_loadmem(&d->v, table_id);
}

/* the compiled program of a query: the virg_vm struct (op array + count);
 * ResultColumn names are copied into `names` (VIRG_OPS x VIRG_MAX_COLUMN_NAME
 * bytes, indexed by op) and their pointers cleared in `out` */
int orc_compile(orc_db *d, const char *sql, virg_vm *out, char *names)
{
	unsigned i;
	virg_vm *vm = virg_vm_init();
	if(virg_sql(&d->v, sql, vm) != VIRG_SUCCESS) {
		free(vm);
		return VIRG_FAIL;
	}
	memcpy(out, vm, sizeof(virg_vm));
	for(i = 0; i < vm->num_ops; i++)
		if(vm->stmt[i].op == OP_ResultColumn) {
			if(names)
				strncpy(names + i * VIRG_MAX_COLUMN_NAME, vm->stmt[i].p4.s,
					VIRG_MAX_COLUMN_NAME - 1);
			out->stmt[i].p4.li = 0;
		}
	virg_vm_cleanup(&d->v, vm);
	return VIRG_SUCCESS;
}

/*
 * Run a query.  mode 0 = single-core VM, 1 = multi-core VM with `threads`
 * pthreads, 2 = the GPU VM through virg_vm_gpu (only meaningful when the
 * library was linked against a real GPU VM).  `repeat` executions are timed
 * and the best wall time is kept; the last run's results stay attached.
 */
static orc_result *run_query(orc_db *d, const char *sql, int mode, unsigned threads, unsigned repeat,
	const virg_op *ops, unsigned nops);

orc_result *orc_query(orc_db *d, const char *sql, int mode, unsigned threads, unsigned repeat)
{
	return run_query(d, sql, mode, threads, repeat, NULL, 0);
}

/*
 * Run a hand-assembled program: `sql` is compiled for its Table,
 * ResultColumn and Parallel ops (the result layout), then every op of
 * `ops` except the ResultColumn ops (whose names stay the compiled ones)
 * replaces the compiled op at the same index and num_ops becomes `nops`.
 * Used to run opcodes the code generator never emits (And, Or, Not).
 */
orc_result *orc_query_ops(orc_db *d, const char *sql, const virg_op *ops, unsigned nops)
{
	return run_query(d, sql, 0, 0, 1, ops, nops);
}

static orc_result *run_query(orc_db *d, const char *sql, int mode, unsigned threads, unsigned repeat,
	const virg_op *ops, unsigned nops)
{
	orc_result *res = calloc(1, sizeof(orc_result));
	virginian *v = &d->v;
	unsigned i;
	if(repeat == 0)
		repeat = 1;
	v->use_multi = (mode == 1);
	v->use_gpu = (mode == 2);
	v->use_mmap = 0;
	v->use_stream = 0;
	if(threads)
		v->multi_threads = threads;
	res->seconds = 1e30;
	for(i = 0; i < repeat; i++) {
		virg_vm *vm = virg_vm_init();
		if(virg_sql(v, sql, vm) != VIRG_SUCCESS) {
			free(vm);
			free(res);
			return NULL;
		}
		if(ops) {
			unsigned k;
			if(nops > VIRG_OPS) {
				virg_vm_cleanup(v, vm);
				free(res);
				return NULL;
			}
			for(k = 0; k < nops; k++)
				if(k >= vm->num_ops || vm->stmt[k].op != OP_ResultColumn)
					vm->stmt[k] = ops[k];
			vm->num_ops = nops;
		}
		virg_table_loadmem(v, vm->stmt[0].p1);
		double t0 = now_s();
		int rc = virg_vm_execute(v, vm);
		double t = now_s() - t0;
		if(rc != VIRG_SUCCESS) {
			virg_vm_cleanup(v, vm);
			free(res);
			return NULL;
		}
		if(t < res->seconds)
			res->seconds = t;
		if(res->vm)
			virg_vm_cleanup(v, res->vm);
		res->vm = vm;
	}

	/* describe the result layout from the head result tablet */
	virg_tablet_meta *t;
	virg_db_load(v, res->vm->head_result->id, &t);
	res->ncols = t->fixed_columns;
	for(i = 0; i < t->fixed_columns; i++) {
		res->types[i] = t->fixed_type[i];
		res->strides[i] = (unsigned)t->fixed_stride[i];
	}
	virg_tablet_unlock(v, t->id);

	virg_result_node *node;
	res->rows = 0;
	res->ntablets = 0;
	for(node = res->vm->head_result; node; node = node->next) {
		virg_db_load(v, node->id, &t);
		res->rows += t->rows;
		res->ntablets++;
		virg_tablet_unlock(v, t->id);
	}
	return res;
}

unsigned long long orc_result_rows(orc_result *r) { return r->rows; }
unsigned orc_result_ncols(orc_result *r) { return r->ncols; }
unsigned orc_result_ntablets(orc_result *r) { return r->ntablets; }
double orc_result_seconds(orc_result *r) { return r->seconds; }
/* the GPU VM's own timing of the last run, seconds (src/vm/vm_gpu.cu:207-240):
 * k = 1 host-to-device copies, 2 kernels, 3 device-to-host copies */
double orc_result_timing(orc_result *r, int k)
{
	if(!r->vm)
		return 0;
	return k == 1 ? r->vm->timing1 : k == 2 ? r->vm->timing2 : r->vm->timing3;
}
int orc_result_type(orc_result *r, unsigned c) { return r->types[c]; }
unsigned orc_result_stride(orc_result *r, unsigned c) { return r->strides[c]; }
const virg_vm *orc_result_vm(orc_result *r) { return r->vm; }

/* per result tablet row counts, in chain order */
int orc_result_tablet_rows(orc_db *d, orc_result *r, unsigned *out)
{
	virg_result_node *node;
	unsigned i = 0;
	for(node = r->vm->head_result; node; node = node->next) {
		virg_tablet_meta *t;
		virg_db_load(&d->v, node->id, &t);
		out[i++] = t->rows;
		virg_tablet_unlock(&d->v, t->id);
	}
	return VIRG_SUCCESS;
}

/* concatenate every result column over the chain into caller buffers */
int orc_result_copy(orc_db *d, orc_result *r, void *const *cols)
{
	virg_result_node *node;
	unsigned long long off = 0;
	unsigned c;
	for(node = r->vm->head_result; node; node = node->next) {
		virg_tablet_meta *t;
		virg_db_load(&d->v, node->id, &t);
		for(c = 0; c < t->fixed_columns; c++) {
			size_t s = t->fixed_stride[c];
			memcpy((char*)cols[c] + off * s,
				(char*)t + t->fixed_block + t->fixed_offset[c], s * t->rows);
		}
		off += t->rows;
		virg_tablet_unlock(&d->v, t->id);
	}
	return VIRG_SUCCESS;
}

/* reads rows through the reference's reader API, for API-level checks:
 * returns how many times virg_reader_row succeeded and copies the row
 * buffers (row_bytes each) of the first `max_rows` rows */
unsigned long long orc_reader_walk(orc_db *d, const char *sql, void *rows_out,
	unsigned row_bytes, unsigned long long max_rows, unsigned long long *getrows)
{
	virg_reader *r;
	unsigned long long n = 0;
	unsigned g = 0;
	virg_query(&d->v, &r, sql);
	virg_reader_getrows(&d->v, r, &g);
	*getrows = g;
	while(virg_reader_row(&d->v, r) != VIRG_FAIL) {
		if(n < max_rows)
			memcpy((char*)rows_out + n * row_bytes, r->buffer, row_bytes);
		n++;
	}
	virg_release(&d->v, r);
	return n;
}

void orc_result_free(orc_db *d, orc_result *r)
{
	if(r->vm)
		virg_vm_cleanup(&d->v, r->vm);
	free(r);
}

void orc_set_gpu_flags(orc_db *d, int use_gpu, int use_mmap, int use_stream)
{
	d->v.use_gpu = use_gpu;
	d->v.use_mmap = use_mmap;
	d->v.use_stream = use_stream;
}

const size_t *orc_testsizes(void) { return &virg_testsizes[0]; }
unsigned orc_sizeof_vm(void) { return sizeof(virg_vm); }
unsigned orc_sizeof_meta(void) { return sizeof(virg_tablet_meta); }
unsigned orc_mem_tablets(void) { return VIRG_MEM_TABLETS; }
unsigned orc_max_tables(void) { return VIRG_MAX_TABLES; }
