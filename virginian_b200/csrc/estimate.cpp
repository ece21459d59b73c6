/*
 * Result-size estimates for serving admission.
 *
 * A resident table keeps a small host sample of its rows: up to kSampleRuns
 * runs of kSampleRun consecutive rows, taken from segments spread evenly
 * over each append.  A program's filter uops are evaluated over the sample
 * on the host with the same row-state rules as the kernel (a row leaves the
 * active set when a compare jumps, parks in its target slot and is joined
 * again at the target; Invalid clears the validity of active rows), and the
 * fraction of sample rows left valid, times the table's rows, is the
 * estimate the serving loop reserves result memory for.  The estimate only
 * sizes a reservation: a query whose rows exceed it is admitted again with
 * its exact row count, so it never changes a result.
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "vgpu_engine.h"
#include "vgpu_util.h"
#include "engine_internal.h"

namespace vgpu {

namespace {

constexpr uint32_t kSampleRun = 64;
constexpr uint32_t kSampleRuns = 64;

uint32_t vt_bytes(uint8_t t) { return t == VT_INT64 || t == VT_DOUBLE ? 8u : t == VT_CHAR ? 1u : 4u; }

/* one value as a double (every type the filter compares converts exactly
 * enough for an estimate) */
double as_double(const unsigned char *p, uint8_t t)
{
	switch (t) {
	case VT_INT: { int32_t v; memcpy(&v, p, 4); return v; }
	case VT_INT64: { int64_t v; memcpy(&v, p, 8); return (double)v; }
	case VT_FLOAT: { float v; memcpy(&v, p, 4); return v; }
	case VT_DOUBLE: { double v; memcpy(&v, p, 8); return v; }
	default: return (double)(signed char)*p;
	}
}

bool cmp(uint8_t op, double a, double b)
{
	switch (op) {
	case CO_LE: return a <= b;
	case CO_LT: return a < b;
	case CO_GE: return a >= b;
	case CO_GT: return a > b;
	case CO_EQ: return a == b;
	case CO_NEQ: return a != b;
	case CO_AND: return a != 0 && b != 0;
	default: return a != 0 || b != 0;
	}
}

double math(uint8_t op, uint8_t t, double a, double b)
{
	const bool integer = t == VT_INT || t == VT_INT64 || t == VT_CHAR;
	switch (op) {
	case MO_ADD: return a + b;
	case MO_SUB: return a - b;
	case MO_MUL: return a * b;
	default:
		if (integer)
			return b == 0 ? 0 : std::trunc(a / b);
		return a / b;
	}
}

}  // namespace

void table_sample(virg_gpu_table *t, const virg_gpu_segment *segs, unsigned n)
{
	TableSample &s = t->sample;
	unsigned nonempty = 0;
	for (unsigned i = 0; i < n; i++)
		nonempty += segs[i].rows > 0;
	if (!nonempty || s.runs >= kSampleRuns)
		return;
	const unsigned want = std::min<unsigned>(kSampleRuns - s.runs, nonempty);
	const unsigned every = std::max(1u, nonempty / want);
	unsigned seen = 0;
	for (unsigned i = 0; i < n && s.runs < kSampleRuns; i++) {
		const virg_gpu_segment &g = segs[i];
		if (!g.rows)
			continue;
		if (seen++ % every)
			continue;
		const uint32_t take = std::min<uint32_t>(kSampleRun, g.rows);
		const uint64_t r0 = (g.rows - take) / 2;  /* from the segment's middle */
		bool ok = true;
		for (int c = 0; c <= (int)t->schema.ncols && ok; c++) {
			const bool key = c == (int)t->schema.ncols;
			const void *src = key ? g.key : g.col[c];
			const int slot = key ? kKeySlot : c;
			if (!src) {
				if (key)
					continue;  /* no key column: programs reading it are refused */
				ok = false;
				break;
			}
			const uint32_t sz = vt_bytes((uint8_t)(key ? t->schema.key_type : t->schema.col_type[c]));
			std::vector<unsigned char> &col = s.col[slot];
			const size_t at = col.size();
			col.resize(at + (size_t)take * sz);
			/* host or device memory alike (unified addressing) */
			ok = cudaMemcpy(col.data() + at, static_cast<const unsigned char *>(src) + r0 * sz, (size_t)take * sz,
				cudaMemcpyDefault) == cudaSuccess;
		}
		if (!ok) {
			cudaGetLastError();
			s = TableSample();  /* a sample with a hole is no sample */
			return;
		}
		s.rows += take;
		s.runs++;
	}
}

double sample_selectivity(const Program &P, const virg_gpu_table *t)
{
	const TableSample &s = t->sample;
	if (s.rows == 0)
		return -1.0;
	for (unsigned i = 0; i < P.nload; i++)
		if (s.col[P.load_src[i]].size() < (size_t)s.rows * P.load_stride[i])
			return -1.0;
	const uint32_t n = s.rows;
	std::vector<uint8_t> valid(n, 1), active(n, 1), parked(n, 0xff);
	std::vector<double> vec[kMaxRegs];
	auto operand = [&](uint8_t cls, uint8_t idx, uint8_t type, uint32_t r) -> double {
		if (cls == OC_COL)  /* idx: the program's load */
			return idx < P.nload ? as_double(s.col[P.load_src[idx]].data() + (size_t)r * P.load_stride[idx],
				P.load_type[idx]) : 0.0;
		if (cls == OC_VEC)
			return vec[idx].empty() ? 0 : vec[idx][r];
		uint64_t bits = P.consts[idx];
		unsigned char b[8];
		memcpy(b, &bits, 8);
		return as_double(b, type);
	};
	for (uint32_t k = 0; k < P.nfilter; k++) {
		const UOp &u = P.uops[k];
		if (u.join)
			for (uint32_t r = 0; r < n; r++)
				if (parked[r] != 0xff && ((u.join >> parked[r]) & 1u)) {
					active[r] = 1;
					parked[r] = 0xff;
				}
		switch (u.kind) {
		case UK_CMP:
		case UK_NOT:
			for (uint32_t r = 0; r < n; r++) {
				if (!active[r])
					continue;
				const double a = operand(u.a_cls, u.a_idx, u.type, r);
				const bool jump = u.kind == UK_NOT ? a == 0 : cmp(u.sub, a, operand(u.b_cls, u.b_idx, u.type, r));
				if (jump) {
					active[r] = 0;
					parked[r] = u.tslot;
					if (!u.vjump)
						valid[r] = 0;
				}
			}
			break;
		case UK_INVALID:
			for (uint32_t r = 0; r < n; r++)
				if (active[r])
					valid[r] = 0;
			break;
		case UK_MATH:
		case UK_SETCONST:
		case UK_COPYCOL:
			if (u.dst < kMaxRegs) {
				vec[u.dst].resize(n, 0.0);
				for (uint32_t r = 0; r < n; r++) {
					if (!active[r] && u.kind != UK_COPYCOL)
						continue;
					const double a = operand(u.a_cls, u.a_idx, u.type, r);
					vec[u.dst][r] = u.kind == UK_MATH ? math(u.sub, u.type, a, operand(u.b_cls, u.b_idx, u.type, r)) : a;
				}
			}
			break;
		default:
			break;
		}
	}
	uint32_t kept = 0;
	for (uint32_t r = 0; r < n; r++)
		kept += valid[r];
	return (double)kept / (double)n;
}

}  // namespace vgpu

extern "C" int virg_gpu_table_estimate(const virg_gpu_table *t, const virg_gpu_program *p, uint64_t *rows)
{
	VGPU_CHECK(t != nullptr && p != nullptr && rows != nullptr, "null argument");
	const double sel = vgpu::sample_selectivity(p->prog, t);
	VGPU_CHECK(sel >= 0.0, "the table has no row sample for the program's columns");
	*rows = (uint64_t)(sel * (double)t->rows + 0.5);
	return 1;
}
