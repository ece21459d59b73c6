/*
 * Host-side decoder: validates the data-parallel section of a Virginian
 * opcode program and lowers it to the uops the sm_100a kernel interprets.
 *
 * The section runs from vm->pc (the op after OP_Parallel, src/vm/execute.c:82)
 * to the first OP_Converge.  Every check below rejects a program the
 * reference's single-core CPU VM (src/vm/virginia.c:228-891) would not run to
 * a defined result:
 *  - compare and arithmetic operands must hold the same type, as the CPU VM
 *    asserts (src/vm/virginia.c:52, :143);
 *  - a register must have a type before it is read (the CPU's context.type[]
 *    starts uninitialised, src/vm/virginia.c:277);
 *  - jumps go forward (the CPU asserts row_pc >= pc, src/vm/virginia.c:375);
 *  - OP_Cast is refused: the CPU VM reads stale p1/p2 for it (no GETP1/GETP2
 *    at src/vm/virginia.c:682-683), and the code generator never emits it
 *    (src/sql/generate.c:431);
 *  - serial ops (Table, ResultColumn, Parallel, Finish) or Nop inside the
 *    section make the CPU VM print "Invalid OP" and abandon the tablet
 *    (src/vm/virginia.c:864-871) and are refused;
 *  - exactly one OP_Result, as the code generator emits
 *    (src/sql/generate.c:677-679); ops after it cannot change the output and
 *    are dropped.
 */
#include <cstring>
#include <string>
#include <vector>

#include "../../include/virginian_b200.h"
#include "vgpu_program.h"
#include "vgpu_util.h"
#include "vgpu_engine.h"

namespace vgpu {

static thread_local std::string g_error;

void set_error(const char *fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_error = buf;
}

const char *last_error() { return g_error.c_str(); }
void clear_error() { g_error.clear(); }

static int type_size(int t)
{
	switch (t) {
	case VT_INT: return 4;
	case VT_INT64: return 8;
	case VT_FLOAT: return 4;
	case VT_DOUBLE: return 8;
	case VT_CHAR: return 1;
	default: return 0;
	}
}

static const char *op_name(int op)
{
	static const char *names[] = {"Table", "ResultColumn", "Parallel", "Finish", "Column",
		"Rowid", "Result", "Converge", "Invalid", "Cast", "Integer", "Float", "Le", "Lt",
		"Ge", "Gt", "Eq", "Neq", "Add", "Sub", "Mul", "Div", "And", "Or", "Not", "Nop"};
	return (op >= 0 && op <= 25) ? names[op] : "unknown";
}

static bool is_cmp(int op)
{
	return (op >= OP_Le && op <= OP_Neq) || op == OP_And || op == OP_Or;
}

static bool is_math(int op) { return op >= OP_Add && op <= OP_Div; }

static uint8_t cmp_code(int op)
{
	switch (op) {
	case OP_Le: return CO_LE;
	case OP_Lt: return CO_LT;
	case OP_Ge: return CO_GE;
	case OP_Gt: return CO_GT;
	case OP_Eq: return CO_EQ;
	case OP_Neq: return CO_NEQ;
	case OP_And: return CO_AND;
	default: return CO_OR;
	}
}

/* how one op defines its p1 register */
enum DefKind { DK_NONE, DK_COL, DK_CONST, DK_ARITH };

struct Def {
	DefKind kind;
	int src;          /* column index or kKeySlot for DK_COL */
	uint64_t bits;    /* constant bits for DK_CONST */
	int type;
};

static Def def_of(const virg_op &o, const virg_gpu_schema &s)
{
	Def d{DK_NONE, 0, 0, -1};
	switch (o.op) {
	case OP_Column:
		d.kind = DK_COL; d.src = o.p2; d.type = s.col_type[o.p2];
		break;
	case OP_Rowid:
		d.kind = DK_COL; d.src = kKeySlot; d.type = s.key_type;
		break;
	case OP_Integer: {
		d.kind = DK_CONST; d.type = VT_INT;
		int32_t v = o.p2;
		uint32_t u;
		memcpy(&u, &v, 4);
		d.bits = u;
		break;
	}
	case OP_Float: {
		d.kind = DK_CONST; d.type = VT_FLOAT;
		uint32_t u;
		memcpy(&u, &o.p4.f, 4);
		d.bits = u;
		break;
	}
	default:
		if (is_math(o.op))
			d.kind = DK_ARITH;
		break;
	}
	return d;
}

int decode_program(const virg_op *ops, unsigned num_ops, unsigned pc,
	const virg_gpu_schema &schema, Program &P, ProgramExtra &X)
{
	memset(&P, 0, sizeof(P));
	memset(&X, 0, sizeof(X));
	VGPU_CHECK(ops != nullptr, "program has no ops");
	VGPU_CHECK(num_ops <= (unsigned)kMaxOps, "program has %u ops, more than VIRG_OPS (%d)",
		num_ops, kMaxOps);
	VGPU_CHECK(pc < num_ops, "parallel section start %u is past the program end (%u ops)", pc,
		num_ops);
	VGPU_CHECK(schema.ncols <= (unsigned)kMaxCols, "schema has %u columns", schema.ncols);
	for (unsigned c = 0; c < schema.ncols; c++)
		VGPU_CHECK(type_size(schema.col_type[c]) > 0,
			"column %u has type %d, which the VM cannot load", c, schema.col_type[c]);

	/* pass 1: find the section end and infer register types in program order
	 * (the CPU VM updates context.type[] whenever the block passes an op,
	 * independent of which rows are active) */
	int reg_type[kMaxRegs];
	for (int r = 0; r < kMaxRegs; r++)
		reg_type[r] = -1;
	int result_k = -1, converge_k = -1;
	int result_types[kMaxRegs];
	auto reg_ok = [](int r) { return r >= 0 && r < kMaxRegs; };
	for (unsigned k = pc; k < num_ops; k++) {
		const virg_op &o = ops[k];
		switch (o.op) {
		case OP_Column:
			VGPU_CHECK(reg_ok(o.p1), "op %u (Column): register %d out of range", k, o.p1);
			VGPU_CHECK(o.p2 >= 0 && (unsigned)o.p2 < schema.ncols,
				"op %u (Column): column %d not in table (%u columns)", k, o.p2, schema.ncols);
			reg_type[o.p1] = schema.col_type[o.p2];
			break;
		case OP_Rowid:
			VGPU_CHECK(reg_ok(o.p1), "op %u (Rowid): register %d out of range", k, o.p1);
			VGPU_CHECK(type_size(schema.key_type) > 0, "op %u (Rowid): key type %d unsupported",
				k, schema.key_type);
			reg_type[o.p1] = schema.key_type;
			break;
		case OP_Integer:
			VGPU_CHECK(reg_ok(o.p1), "op %u (Integer): register %d out of range", k, o.p1);
			reg_type[o.p1] = VT_INT;
			break;
		case OP_Float:
			VGPU_CHECK(reg_ok(o.p1), "op %u (Float): register %d out of range", k, o.p1);
			reg_type[o.p1] = VT_FLOAT;
			break;
		case OP_Invalid:
			break;
		case OP_Not:
			VGPU_CHECK(reg_ok(o.p1) && reg_type[o.p1] >= 0,
				"op %u (Not): register %d read before it is set", k, o.p1);
			VGPU_CHECK(o.p3 > (int)k && o.p3 <= 255, "op %u (Not): jump target %d is not forward",
				k, o.p3);
			break;
		case OP_Result:
			VGPU_CHECK(result_k < 0, "op %u: more than one Result in the parallel section", k);
			VGPU_CHECK(o.p2 >= 1 && reg_ok(o.p1) && o.p1 + o.p2 <= kMaxRegs,
				"op %u (Result): registers %d..%d out of range", k, o.p1, o.p1 + o.p2 - 1);
			for (int j = 0; j < o.p2; j++) {
				VGPU_CHECK(reg_type[o.p1 + j] >= 0,
					"op %u (Result): register %d read before it is set", k, o.p1 + j);
				result_types[j] = reg_type[o.p1 + j];
			}
			result_k = (int)k;
			break;
		case OP_Converge:
			converge_k = (int)k;
			break;
		default:
			if (is_cmp(o.op)) {
				VGPU_CHECK(reg_ok(o.p1) && reg_ok(o.p2), "op %u (%s): register out of range", k,
					op_name(o.op));
				VGPU_CHECK(reg_type[o.p1] >= 0 && reg_type[o.p2] >= 0,
					"op %u (%s): register read before it is set", k, op_name(o.op));
				VGPU_CHECK(reg_type[o.p1] == reg_type[o.p2],
					"op %u (%s): operand types differ (%d vs %d)", k, op_name(o.op),
					reg_type[o.p1], reg_type[o.p2]);
				VGPU_CHECK(o.p3 > (int)k && o.p3 <= 255,
					"op %u (%s): jump target %d is not forward", k, op_name(o.op), o.p3);
			} else if (is_math(o.op)) {
				VGPU_CHECK(reg_ok(o.p1) && reg_ok(o.p2) && reg_ok(o.p3),
					"op %u (%s): register out of range", k, op_name(o.op));
				VGPU_CHECK(reg_type[o.p2] >= 0 && reg_type[o.p3] >= 0,
					"op %u (%s): register read before it is set", k, op_name(o.op));
				VGPU_CHECK(reg_type[o.p2] == reg_type[o.p3],
					"op %u (%s): operand types differ (%d vs %d)", k, op_name(o.op),
					reg_type[o.p2], reg_type[o.p3]);
				reg_type[o.p1] = reg_type[o.p2];
			} else if (o.op == OP_Cast) {
				VGPU_FAIL("op %u: Cast is not supported (the reference CPU VM reads stale "
					"operands for it and the code generator never emits it)", k);
			} else {
				VGPU_FAIL("op %u: %s is not a data-parallel op", k, op_name(o.op));
			}
		}
		if (converge_k >= 0)
			break;
	}
	VGPU_CHECK(converge_k >= 0, "no Converge after the parallel section start %u", pc);
	VGPU_CHECK(result_k >= 0, "the parallel section has no Result op");

	/* pass 2: register definitions up to the Result op decide how each
	 * register is stored */
	std::vector<Def> defs[kMaxRegs];
	for (int k = (int)pc; k < result_k; k++) {
		Def d = def_of(ops[k], schema);
		if (d.kind == DK_NONE)
			continue;
		int r = ops[k].p1;
		if (d.kind == DK_ARITH)
			d.type = -2;  /* filled below from the operand type */
		defs[r].push_back(d);
	}
	/* arithmetic result types (same as pass 1 at that point) */
	{
		int t[kMaxRegs];
		for (int r = 0; r < kMaxRegs; r++)
			t[r] = -1;
		size_t idx[kMaxRegs] = {0};
		for (int k = (int)pc; k < result_k; k++) {
			Def d = def_of(ops[k], schema);
			if (d.kind == DK_NONE)
				continue;
			int r = ops[k].p1;
			int ty = d.kind == DK_ARITH ? t[ops[k].p2] : d.type;
			defs[r][idx[r]++].type = ty;
			t[r] = ty;
		}
	}

	enum { RC_NONE, RC_COL, RC_CONST, RC_VEC };
	int rclass[kMaxRegs], rsrc[kMaxRegs], rtype[kMaxRegs];
	uint64_t rbits[kMaxRegs];
	for (int r = 0; r < kMaxRegs; r++) {
		rclass[r] = RC_NONE;
		rtype[r] = -1;
		if (defs[r].empty())
			continue;
		bool same_type = true, all_col = true, all_const = true;
		for (const Def &d : defs[r]) {
			same_type &= d.type == defs[r][0].type;
			all_col &= d.kind == DK_COL && d.src == defs[r][0].src;
			all_const &= d.kind == DK_CONST && d.bits == defs[r][0].bits;
		}
		VGPU_CHECK(same_type, "register %d is set with different types", r);
		rtype[r] = defs[r][0].type;
		if (all_col) {
			rclass[r] = RC_COL;
			rsrc[r] = defs[r][0].src;
		} else if (all_const) {
			rclass[r] = RC_CONST;
			rbits[r] = defs[r][0].bits;
		} else {
			rclass[r] = RC_VEC;
		}
	}

	/* staged columns: every Column/Rowid source in the section, in order of
	 * first appearance (all of them are read by the CPU VM, so all of them
	 * count as algorithmic bytes) */
	int load_slot_of[kMaxLoads];
	for (int c = 0; c < kMaxLoads; c++)
		load_slot_of[c] = -1;
	for (int k = (int)pc; k < result_k; k++) {
		const virg_op &o = ops[k];
		if (o.op != OP_Column && o.op != OP_Rowid)
			continue;
		int src = o.op == OP_Rowid ? kKeySlot : o.p2;
		if (load_slot_of[src] >= 0)
			continue;
		int ty = o.op == OP_Rowid ? schema.key_type : schema.col_type[src];
		load_slot_of[src] = (int)P.nload;
		P.load_src[P.nload] = (uint8_t)src;
		P.load_type[P.nload] = (uint8_t)ty;
		P.load_stride[P.nload] = (uint8_t)type_size(ty);
		P.nload++;
	}

	/* vector and scalar slots */
	int slot[kMaxRegs];
	for (int r = 0; r < kMaxRegs; r++) {
		slot[r] = -1;
		if (rclass[r] == RC_VEC) {
			slot[r] = (int)P.nvec;
			P.vec_stride[P.nvec++] = (uint8_t)type_size(rtype[r]);
		} else if (rclass[r] == RC_CONST) {
			slot[r] = (int)P.nconst;
			P.consts[P.nconst++] = rbits[r];
		} else if (rclass[r] == RC_COL) {
			slot[r] = load_slot_of[rsrc[r]];
		}
	}
	auto operand = [&](int r, uint8_t &cls, uint8_t &idx) {
		cls = rclass[r] == RC_COL ? OC_COL : rclass[r] == RC_VEC ? OC_VEC : OC_CONST;
		idx = (uint8_t)slot[r];
	};

	/* pass 3: emit uops */
	int cur_type[kMaxRegs];
	for (int r = 0; r < kMaxRegs; r++)
		cur_type[r] = -1;
	for (int k = (int)pc; k <= result_k; k++) {
		const virg_op &o = ops[k];
		UOp u;
		memset(&u, 0, sizeof(u));
		u.pc = (uint8_t)k;
		bool emit = true;
		switch (o.op) {
		case OP_Column:
		case OP_Rowid: {
			int src = o.op == OP_Rowid ? kKeySlot : o.p2;
			cur_type[o.p1] = o.op == OP_Rowid ? schema.key_type : schema.col_type[o.p2];
			if (rclass[o.p1] != RC_VEC) {
				emit = false;
				break;
			}
			u.kind = UK_COPYCOL;
			u.flags = defs[o.p1].size() == 1 ? UF_SINGLE_DEF : 0;
			u.type = (uint8_t)cur_type[o.p1];
			u.dst = (uint8_t)slot[o.p1];
			u.a_cls = OC_COL;
			u.a_idx = (uint8_t)load_slot_of[src];
			break;
		}
		case OP_Integer:
		case OP_Float: {
			cur_type[o.p1] = o.op == OP_Integer ? VT_INT : VT_FLOAT;
			if (rclass[o.p1] != RC_VEC) {
				emit = false;
				break;
			}
			Def d = def_of(o, schema);
			u.kind = UK_SETCONST;
			u.flags = defs[o.p1].size() == 1 ? UF_SINGLE_DEF : 0;
			u.type = (uint8_t)d.type;
			u.dst = (uint8_t)slot[o.p1];
			u.a_cls = OC_CONST;
			VGPU_CHECK(P.nconst < (unsigned)kMaxRegs, "too many constants");
			u.a_idx = (uint8_t)P.nconst;
			P.consts[P.nconst++] = d.bits;
			break;
		}
		case OP_Invalid:
			u.kind = UK_INVALID;
			break;
		case OP_Not:
			u.kind = UK_NOT;
			u.type = (uint8_t)cur_type[o.p1];
			operand(o.p1, u.a_cls, u.a_idx);
			u.target = (uint8_t)o.p3;
			u.vjump = o.p4.i != 0;
			break;
		case OP_Result:
			u.kind = UK_RESULT;
			P.nout = (uint32_t)o.p2;
			for (int j = 0; j < o.p2; j++) {
				int r = o.p1 + j;
				operand(r, P.out_cls[j], P.out_idx[j]);
				P.out_type[j] = (uint8_t)result_types[j];
				P.out_stride[j] = (uint8_t)type_size(result_types[j]);
			}
			break;
		default:
			if (is_cmp(o.op)) {
				u.kind = UK_CMP;
				u.sub = cmp_code(o.op);
				u.type = (uint8_t)cur_type[o.p1];
				operand(o.p1, u.a_cls, u.a_idx);
				operand(o.p2, u.b_cls, u.b_idx);
				u.target = (uint8_t)o.p3;
				u.vjump = o.p4.i != 0;
			} else if (is_math(o.op)) {
				u.kind = UK_MATH;
				u.flags = defs[o.p1].size() == 1 ? UF_SINGLE_DEF : 0;
				u.sub = (uint8_t)(o.op - OP_Add);
				u.type = (uint8_t)cur_type[o.p2];
				u.dst = (uint8_t)slot[o.p1];
				operand(o.p2, u.a_cls, u.a_idx);
				operand(o.p3, u.b_cls, u.b_idx);
				cur_type[o.p1] = cur_type[o.p2];
			}
			break;
		}
		if (emit)
			P.uops[P.nuops++] = u;
	}

	/* definite-assignment analysis: can a row that is still valid read a
	 * register its path never set?  Only valid rows reach the output (a row
	 * never becomes valid again), so paths of rows that were invalidated by
	 * Invalid or by a jump with p4 = 0 are ignored.  Loads cover every row
	 * (the CPU copies the whole block), other definitions only the rows active
	 * at that op.  Such reads give unspecified values in the reference (stale
	 * lanes of an earlier block), so callers that need exact parity avoid
	 * these programs. */
	{
		uint32_t loaded = 0;                 /* registers set by a load so far */
		uint32_t in[kMaxOps + 2];
		bool reach[kMaxOps + 2];             /* reached by a still-valid row */
		for (int k = 0; k < kMaxOps + 2; k++) {
			in[k] = 0xFFFFFFFFu;
			reach[k] = false;
		}
		in[pc] = 0;
		reach[pc] = true;
		auto flow = [&](int to, uint32_t set) {
			if (to > kMaxOps + 1)
				return;
			in[to] = reach[to] ? (in[to] & set) : set;
			reach[to] = true;
		};
		for (int k = (int)pc; k <= result_k; k++) {
			const virg_op &o = ops[k];
			const bool r = reach[k];
			const uint32_t cur = in[k];
			auto use = [&](int reg) {
				if (r && !((loaded >> reg) & 1) && !((cur >> reg) & 1))
					X.maybe_undefined = 1;
			};
			if (is_cmp(o.op)) { use(o.p1); use(o.p2); }
			else if (o.op == OP_Not) use(o.p1);
			else if (is_math(o.op)) { use(o.p2); use(o.p3); }
			else if (o.op == OP_Result)
				for (int j = 0; j < o.p2; j++) use(o.p1 + j);
			uint32_t out = cur;
			if (o.op == OP_Column || o.op == OP_Rowid)
				loaded |= 1u << o.p1;
			else if (o.op == OP_Integer || o.op == OP_Float || is_math(o.op))
				out |= 1u << o.p1;
			if (!r)
				continue;
			if (o.op != OP_Invalid)
				flow(k + 1, out);
			if ((is_cmp(o.op) || o.op == OP_Not) && o.p4.i != 0)
				flow(o.p3, out);
		}
	}

	/* filter / projection split.  F is the first op from which the section up
	 * to Result only loads, sets constants and computes (the code
	 * generator's result-column block after its condition stub,
	 * src/sql/generate.c:643-648).  If every jump that keeps a row valid lands
	 * at or before F, every row valid at Result is active through [F, Result)
	 * and those ops only matter for valid rows: they run on each warp's
	 * selection list instead of on every row. */
	{
		int F = result_k;
		for (int k = result_k - 1; k >= (int)pc; k--) {
			const int op = ops[k].op;
			if (is_cmp(op) || op == OP_Not || op == OP_Invalid)
				break;
			F = k;
		}
		for (int k = (int)pc; k < F; k++) {
			const virg_op &o = ops[k];
			if ((is_cmp(o.op) || o.op == OP_Not) && o.p4.i != 0 && o.p3 > F)
				F = result_k;
		}
		P.nfilter = 0;
		while (P.nfilter < P.nuops && P.uops[P.nfilter].kind != UK_RESULT && P.uops[P.nfilter].pc < F)
			P.nfilter++;
		/* vectors defined only in the projection are indexed by selection */
		for (int r = 0; r < kMaxRegs; r++) {
			if (rclass[r] != RC_VEC)
				continue;
			bool only_proj = true;
			for (int k = (int)pc; k < result_k; k++) {
				const Def d = def_of(ops[k], schema);
				if (d.kind != DK_NONE && ops[k].p1 == r && k < F)
					only_proj = false;
			}
			P.vec_compact[slot[r]] = only_proj ? 1 : 0;
		}
		X.split_k = F;
	}

	/* pending-target slots for the filter: rows that jump to pc t wait in a
	 * slot until the first filter op at or after t; slots are reused */
	{
		int slot_target[kMaxSlots];
		for (int i = 0; i < kMaxSlots; i++)
			slot_target[i] = -1;
		for (uint32_t i = 0; i < P.nfilter; i++) {
			UOp &u = P.uops[i];
			for (int sl = 0; sl < kMaxSlots; sl++)
				if (slot_target[sl] >= 0 && slot_target[sl] <= u.pc) {
					u.join |= (uint8_t)(1u << sl);
					slot_target[sl] = -1;
				}
			if (u.kind != UK_CMP && u.kind != UK_NOT)
				continue;
			int use = -1;
			for (int sl = 0; sl < kMaxSlots; sl++)
				if (slot_target[sl] == u.target)
					use = sl;
			for (int sl = 0; sl < kMaxSlots && use < 0; sl++)
				if (slot_target[sl] < 0)
					use = sl;
			VGPU_CHECK(use >= 0, "more than %d jump targets pending at op %u", kMaxSlots, u.pc);
			slot_target[use] = u.target;
			u.tslot = (uint8_t)use;
		}
	}

	X.result_k = result_k;
	X.converge_k = converge_k;
	return 1;
}

}  // namespace vgpu

using namespace vgpu;

extern "C" {

const char *virg_gpu_last_error(void) { return vgpu::last_error(); }

int virg_gpu_program_create(const virg_op *ops, unsigned num_ops, unsigned pc,
	const virg_gpu_schema *schema, virg_gpu_program **out)
{
	VGPU_CHECK(out != nullptr && schema != nullptr, "null argument");
	virg_gpu_program *p = new virg_gpu_program();
	if (!decode_program(ops, num_ops, pc, *schema, p->prog, p->extra)) {
		delete p;
		*out = nullptr;
		return 0;
	}
	p->schema = *schema;
	*out = p;
	return 1;
}

int virg_gpu_program_info_get(const virg_gpu_program *p, virg_gpu_program_info *info)
{
	VGPU_CHECK(p != nullptr && info != nullptr, "null argument");
	memset(info, 0, sizeof(*info));
	const Program &P = p->prog;
	info->nload = P.nload;
	for (unsigned i = 0; i < P.nload; i++) {
		info->load_column[i] = P.load_src[i] == kKeySlot ? -1 : P.load_src[i];
		info->load_bytes_per_row += P.load_stride[i];
	}
	info->nout = P.nout;
	for (unsigned j = 0; j < P.nout; j++) {
		info->out_type[j] = P.out_type[j];
		info->out_stride[j] = P.out_stride[j];
		info->out_bytes_per_row += P.out_stride[j];
	}
	info->nuops = P.nuops;
	for (unsigned i = 0; i < P.nvec; i++)
		(P.vec_compact[i] ? info->sel_vector_bytes : info->row_vector_bytes) += P.vec_stride[i];
	return 1;
}

int virg_gpu_program_flags(const virg_gpu_program *p)
{
	return p ? (p->extra.maybe_undefined ? 1 : 0) : -1;
}

void virg_gpu_program_destroy(virg_gpu_program *p) { delete p; }

}  // extern "C"
