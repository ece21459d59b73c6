/*
 * Re-entrant SQL front end: SELECT text -> Virginian opcode program.
 *
 * The reference compiles queries with a flex/bison parser (src/sql/sql.l,
 * src/sql/sql.y) and a code generator that keeps its state in globals
 * (src/sql/generate.c:46-48, src/sql/node.h:40, src/sql/sql.y:24), so only one
 * query can compile at a time.  This restatement keeps all state in a
 * per-call context so the serving loop can compile while other queries run,
 * and it must emit exactly the reference's programs: the opcode program is
 * the interface between front end and VM.
 *
 * Grammar (sql.y:78-200), as bison resolves it:
 *  - arithmetic is right-associative with one precedence level: the rule
 *    `expr: expr operator expr` has no terminal and thus no precedence, so
 *    its four shift/reduce conflicts (`%expect 4`, sql.y:40) resolve to shift;
 *  - condition lists are right-recursive; `c AND rest` sets c.andcond,
 *    `c OR rest` sets c.orcond; a parenthesised `( c AND|OR rest )` is a whole
 *    list that can only end a list, and its OR form sets orfirst.
 * Lexer (sql.l:30-81): whitespace is space/tab/newline, keywords are
 * case-insensitive, identifiers [a-zA-Z][a-zA-Z0-9]*, `-?[0-9]+` ints and
 * `-?[0-9]+\.[0-9]+` floats by longest match, unknown characters skipped.
 *
 * Code generation follows generate.c's passes: 0 types (:147-249),
 * 1 constant folding (:296-389, including its truncation of float constants
 * to int before folding, :336-337), 2 structure (:394-690: register reuse of
 * structurally equal expressions, condition jumps, result registers moved to
 * the end), 3 op indices (:695-703), 4 register/jump resolution (:710-765),
 * 5 output (:770-776).  Differences: errors are returned instead of exiting
 * or asserting; result column names are truncated to 15 characters (the
 * reference overruns its 16-byte buffer, src/sql/node.c:55-99); integer
 * division by zero in a constant expression is an error (SIGFPE in the
 * reference).
 */
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/virginian_b200.h"
#include "vgpu_util.h"

namespace {

enum Tok {
	T_EOF, T_SELECT, T_FROM, T_WHERE, T_AS, T_AND, T_OR, T_COMMA, T_LP, T_RP,
	T_INT, T_FLOAT, T_STRING, T_PLUS, T_MINUS, T_MUL, T_DIV,
	T_CEQ, T_CNE, T_CLT, T_CLE, T_CGT, T_CGE
};

struct Token {
	Tok type;
	int i;
	float f;
	std::string s;
};

/* AST, mirroring src/sql/node.h:380-471 */
enum ExprKind { E_INT = 1, E_FLOAT = 2, E_OP = 3, E_COLUMN = 5 };
enum { OPN_PLUS = 1, OPN_MINUS = 2, OPN_MUL = 3, OPN_DIV = 4 };
enum { C_EQ = 1, C_NE, C_LT, C_LE, C_GT, C_GE };

struct Expr {
	int kind;
	int datatype = -1;
	Expr *lhs = nullptr, *rhs = nullptr;
	bool iskey = false;
	int ival = 0;        /* int value, op code, or column id */
	float fval = 0;
	std::string name;    /* column name */
};

struct Cond {
	int type;
	bool orfirst = false;
	Cond *andcond = nullptr, *orcond = nullptr;
	Expr *lhs, *rhs;
};

struct ResultCol {
	Expr *expr;
	std::string output_name;
	int output_reg = -1;
};

struct TableDesc {
	std::string name;
	int key_type;
	std::vector<std::string> cols;
	std::vector<int> types;
};

struct Fail {};

struct Parser {
	std::vector<Token> toks;
	size_t pos = 0;
	std::vector<std::unique_ptr<Expr>> exprs;
	std::vector<std::unique_ptr<Cond>> conds;
	std::string err;

	[[noreturn]] void fail(const char *m)
	{
		if (err.empty())
			err = m;
		throw Fail();
	}

	Tok peek() const { return toks[pos].type; }

	Expr *new_expr(int kind)
	{
		exprs.emplace_back(new Expr());
		exprs.back()->kind = kind;
		return exprs.back().get();
	}

	static bool kw(const char *p, size_t n, const char *w)
	{
		if (strlen(w) != n)
			return false;
		for (size_t i = 0; i < n; i++)
			if (tolower((unsigned char)p[i]) != w[i])
				return false;
		return true;
	}

	void lex(const char *q)
	{
		const char *p = q;
		while (*p) {
			Token t{T_EOF, 0, 0.0f, ""};
			if (*p == ' ' || *p == '\t' || *p == '\n') {
				p++;
				continue;
			}
			if (isalpha((unsigned char)*p)) {
				const char *s = p;
				while (isalnum((unsigned char)*p))
					p++;
				size_t n = (size_t)(p - s);
				if (kw(s, n, "select")) t.type = T_SELECT;
				else if (kw(s, n, "from")) t.type = T_FROM;
				else if (kw(s, n, "where")) t.type = T_WHERE;
				else if (kw(s, n, "as")) t.type = T_AS;
				else if (kw(s, n, "and")) t.type = T_AND;
				else if (kw(s, n, "or")) t.type = T_OR;
				else {
					t.type = T_STRING;
					t.s.assign(s, n);
				}
			} else if (isdigit((unsigned char)*p) || (*p == '-' && isdigit((unsigned char)p[1]))) {
				const char *s = p;
				if (*p == '-')
					p++;
				while (isdigit((unsigned char)*p))
					p++;
				bool is_float = false;
				if (*p == '.' && isdigit((unsigned char)p[1])) {
					is_float = true;
					p++;
					while (isdigit((unsigned char)*p))
						p++;
				}
				std::string txt(s, (size_t)(p - s));
				if (is_float) {
					t.type = T_FLOAT;
					t.f = (float)atof(txt.c_str());
				} else {
					t.type = T_INT;
					t.i = atoi(txt.c_str());
				}
			} else if (p[0] == '!' && p[1] == '=') { t.type = T_CNE; p += 2; }
			else if (p[0] == '<' && p[1] == '=') { t.type = T_CLE; p += 2; }
			else if (p[0] == '>' && p[1] == '=') { t.type = T_CGE; p += 2; }
			else if (*p == '=') { t.type = T_CEQ; p++; }
			else if (*p == '<') { t.type = T_CLT; p++; }
			else if (*p == '>') { t.type = T_CGT; p++; }
			else if (*p == '+') { t.type = T_PLUS; p++; }
			else if (*p == '-') { t.type = T_MINUS; p++; }
			else if (*p == '*') { t.type = T_MUL; p++; }
			else if (*p == '/') { t.type = T_DIV; p++; }
			else if (*p == ',') { t.type = T_COMMA; p++; }
			else if (*p == '(') { t.type = T_LP; p++; }
			else if (*p == ')') { t.type = T_RP; p++; }
			else { p++; continue; }
			toks.push_back(t);
		}
		toks.push_back(Token{T_EOF, 0, 0.0f, ""});
	}

	void expect(Tok t)
	{
		if (peek() != t)
			fail("syntax error");
		pos++;
	}

	static bool is_condop(Tok t) { return t >= T_CEQ && t <= T_CGE; }
	static int condop(Tok t) { return (int)(t - T_CEQ) + C_EQ; }
	static bool is_arith(Tok t) { return t >= T_PLUS && t <= T_DIV; }

	Expr *primary()
	{
		Expr *x;
		switch (peek()) {
		case T_LP:
			pos++;
			x = expr();
			expect(T_RP);
			return x;
		case T_INT:
			x = new_expr(E_INT);
			x->ival = toks[pos++].i;
			return x;
		case T_FLOAT:
			x = new_expr(E_FLOAT);
			x->fval = toks[pos++].f;
			return x;
		case T_STRING:
			x = new_expr(E_COLUMN);
			x->name = toks[pos++].s;
			return x;
		default:
			fail("syntax error");
		}
	}

	Expr *expr()
	{
		Expr *lhs = primary();
		if (is_arith(peek())) {
			int op = (int)(peek() - T_PLUS) + OPN_PLUS;
			pos++;
			Expr *x = new_expr(E_OP);
			x->ival = op;
			x->lhs = lhs;
			x->rhs = expr();
			return x;
		}
		return lhs;
	}

	Cond *new_cond(int type, Expr *l, Expr *r)
	{
		conds.emplace_back(new Cond());
		Cond *c = conds.back().get();
		c->type = type;
		c->lhs = l;
		c->rhs = r;
		return c;
	}

	/* speculative alternatives: try, and on failure rewind the position */
	template <typename F>
	bool attempt(F f)
	{
		size_t save = pos;
		std::string saved_err = err;
		try {
			f();
			return true;
		} catch (Fail &) {
			pos = save;
			err = saved_err;
			return false;
		}
	}

	Cond *condition()
	{
		Cond *c = nullptr;
		if (peek() == T_LP && attempt([&] {
				pos++;
				Expr *l = expr();
				if (!is_condop(peek()))
					fail("syntax error");
				int op = condop(peek());
				pos++;
				Expr *r = expr();
				expect(T_RP);
				c = new_cond(op, l, r);
			}))
			return c;
		Expr *l = expr();
		if (!is_condop(peek()))
			fail("syntax error");
		int op = condop(peek());
		pos++;
		Expr *r = expr();
		return new_cond(op, l, r);
	}

	Cond *conditions()
	{
		Cond *c = nullptr;
		if (peek() == T_LP && attempt([&] {
				pos++;
				Cond *head = condition();
				Tok link = peek();
				if (link != T_AND && link != T_OR)
					fail("syntax error");
				pos++;
				Cond *rest = conditions();
				expect(T_RP);
				if (link == T_AND)
					head->andcond = rest;
				else {
					head->orcond = rest;
					head->orfirst = true;
				}
				c = head;
			}))
			return c;
		c = condition();
		if (peek() == T_AND) {
			pos++;
			c->andcond = conditions();
		} else if (peek() == T_OR) {
			pos++;
			c->orcond = conditions();
		}
		return c;
	}
};

/* src/sql/node.c:55-110: the printed form of an expression, before folding */
void expr_string(const Expr *x, std::string &s)
{
	char buf[64];
	switch (x->kind) {
	case E_COLUMN: s += x->name; break;
	case E_INT: snprintf(buf, sizeof(buf), "%i", x->ival); s += buf; break;
	case E_FLOAT: snprintf(buf, sizeof(buf), "%f", (double)x->fval); s += buf; break;
	default: {
		static const char ops[] = "?+-*/";
		s += "(";
		expr_string(x->lhs, s);
		s += ops[x->ival];
		expr_string(x->rhs, s);
		s += ")";
	}
	}
}

/* src/util.c:14-26 */
int generalize(int t1, int t2)
{
	if (t1 == t2)
		return t1;
	if (t1 <= VIRG_DOUBLE && t2 <= VIRG_DOUBLE)
		return t1 > t2 ? t1 : t2;
	return -1;
}

struct AbsOp {
	int index = 0;
	virg_op op;
	AbsOp *opptr = nullptr;
};

struct Gen {
	const TableDesc &table;
	std::vector<std::unique_ptr<AbsOp>> pool;
	std::vector<AbsOp *> list;          /* the statement, in order */
	struct Reg { int index; Expr *expr; };
	std::vector<Reg> regs;
	std::string err;

	explicit Gen(const TableDesc &t) : table(t) {}

	[[noreturn]] void fail(const std::string &m)
	{
		err = m;
		throw Fail();
	}

	AbsOp *absop(int op, int p1, int p2, int p3, AbsOp *ptr)
	{
		pool.emplace_back(new AbsOp());
		AbsOp *a = pool.back().get();
		memset(&a->op, 0, sizeof(a->op));
		a->op.op = op;
		a->op.p1 = p1;
		a->op.p2 = p2;
		a->op.p3 = p3;
		a->opptr = ptr;
		return a;
	}

	/* pass 0 */
	void types(Expr *x)
	{
		switch (x->kind) {
		case E_COLUMN: {
			x->iskey = x->name == "id";
			if (x->iskey) {
				x->ival = 0;
				x->datatype = table.key_type;
			} else {
				int found = -1;
				for (size_t c = 0; c < table.cols.size(); c++)
					if (table.cols[c] == x->name) {
						found = (int)c;
						break;
					}
				if (found < 0)
					fail("no column named " + x->name);
				x->ival = found;
				x->datatype = table.types[found];
			}
			break;
		}
		case E_OP:
			types(x->lhs);
			types(x->rhs);
			x->datatype = generalize(x->lhs->datatype, x->rhs->datatype);
			if (x->datatype < 0)
				fail("operands of an operator have no common type");
			break;
		case E_INT: x->datatype = VIRG_INT; break;
		case E_FLOAT: x->datatype = VIRG_FLOAT; break;
		}
	}

	void cond_types(Cond *c)
	{
		types(c->lhs);
		types(c->rhs);
		if (c->andcond) cond_types(c->andcond);
		if (c->orcond) cond_types(c->orcond);
	}

	/* pass 1: the reference casts both constants with expr_valint, even in
	 * the float case (generate.c:336-337) */
	static int valint(const Expr *x) { return x->kind == E_INT ? x->ival : (int)x->fval; }

	void fold(Expr *x)
	{
		if (x->kind != E_OP)
			return;
		fold(x->lhs);
		fold(x->rhs);
		bool lc = x->lhs->kind == E_INT || x->lhs->kind == E_FLOAT;
		bool rc = x->rhs->kind == E_INT || x->rhs->kind == E_FLOAT;
		if (!lc || !rc)
			return;
		int target = generalize(x->lhs->kind == E_INT ? VIRG_INT : VIRG_FLOAT,
			x->rhs->kind == E_INT ? VIRG_INT : VIRG_FLOAT);
		if (target == VIRG_INT) {
			int a = valint(x->lhs), b = valint(x->rhs), r = 0;
			switch (x->ival) {
			case OPN_PLUS: r = (int)((unsigned)a + (unsigned)b); break;
			case OPN_MINUS: r = (int)((unsigned)a - (unsigned)b); break;
			case OPN_MUL: r = (int)((unsigned)a * (unsigned)b); break;
			default:
				if (b == 0 || (a == -2147483647 - 1 && b == -1))
					fail("integer division by zero in a constant expression");
				r = a / b;
			}
			x->kind = E_INT;
			x->ival = r;
		} else {
			volatile float a = (float)valint(x->lhs), b = (float)valint(x->rhs);
			volatile float r;
			switch (x->ival) {
			case OPN_PLUS: r = a + b; break;
			case OPN_MINUS: r = a - b; break;
			case OPN_MUL: r = a * b; break;
			default: r = a / b; break;
			}
			x->kind = E_FLOAT;
			x->fval = r;
		}
		x->datatype = target;
	}

	void cond_fold(Cond *c)
	{
		fold(c->lhs);
		fold(c->rhs);
		if (c->andcond) cond_fold(c->andcond);
		if (c->orcond) cond_fold(c->orcond);
	}

	/* generate.c:54-82 */
	static bool equal(const Expr *a, const Expr *b)
	{
		if (a->kind != b->kind)
			return false;
		switch (a->kind) {
		case E_INT: return a->ival == b->ival;
		case E_FLOAT: return a->fval == b->fval;
		case E_COLUMN: return a->iskey == b->iskey && a->ival == b->ival;
		default: return a->ival == b->ival && equal(a->lhs, b->lhs) && equal(a->rhs, b->rhs);
		}
	}

	int getreg()
	{
		if (regs.size() >= VIRG_REGS)
			fail("query needs more than 16 registers");
		regs.push_back(Reg{0, nullptr});
		return (int)regs.size() - 1;
	}

	/* generate.c:394-464 */
	int expr_reg(Expr *x)
	{
		for (size_t i = 0; i < regs.size(); i++)
			if (equal(x, regs[i].expr))
				return (int)i;
		int reg;
		switch (x->kind) {
		case E_INT:
			reg = getreg();
			list.push_back(absop(OP_Integer, reg, x->ival, 0, nullptr));
			break;
		case E_FLOAT: {
			reg = getreg();
			AbsOp *a = absop(OP_Float, reg, 0, 0, nullptr);
			a->op.p4.f = x->fval;
			list.push_back(a);
			break;
		}
		case E_OP: {
			int r1 = expr_reg(x->lhs);
			int r2 = expr_reg(x->rhs);
			reg = getreg();
			static const int ops[] = {0, OP_Add, OP_Sub, OP_Mul, OP_Div};
			list.push_back(absop(ops[x->ival], reg, r1, r2, nullptr));
			break;
		}
		default:
			reg = getreg();
			if (x->iskey)
				list.push_back(absop(OP_Rowid, reg, 0, 0, nullptr));
			else
				list.push_back(absop(OP_Column, reg, x->ival, 0, nullptr));
			break;
		}
		regs[reg].expr = x;
		return reg;
	}

	/* generate.c:477-578 */
	AbsOp *cond(Cond *x, AbsOp *onsuccess, AbsOp *onfailure, AbsOp *newop)
	{
		int r1 = expr_reg(x->lhs);
		int r2 = expr_reg(x->rhs);
		if (x->andcond == nullptr || (x->orcond != nullptr && x->orfirst)) {
			static const int jump_true[] = {0, OP_Eq, OP_Neq, OP_Lt, OP_Le, OP_Gt, OP_Ge};
			AbsOp *andop = nullptr;
			if (x->andcond) {
				andop = absop(OP_Nop, 0, 0, 0, nullptr);
				onsuccess = andop;
			}
			if (!newop)
				newop = absop(OP_Nop, 0, 0, 0, nullptr);
			newop->op.op = jump_true[x->type];
			newop->op.p1 = r1;
			newop->op.p2 = r2;
			newop->op.p4.i = 1;
			newop->opptr = onsuccess;
			list.push_back(newop);
			if (x->orcond)
				cond(x->orcond, onsuccess, onfailure, nullptr);
			if (x->andcond)
				cond(x->andcond, onfailure, onfailure, andop);
		} else {
			static const int jump_false[] = {0, OP_Neq, OP_Eq, OP_Ge, OP_Gt, OP_Le, OP_Lt};
			AbsOp *orop = nullptr;
			if (x->orcond) {
				orop = absop(OP_Nop, 0, 0, 0, nullptr);
				onfailure = orop;
			}
			if (!newop)
				newop = absop(OP_Nop, 0, 0, 0, nullptr);
			newop->op.op = jump_false[x->type];
			newop->op.p1 = r1;
			newop->op.p2 = r2;
			newop->op.p4.i = 0;
			newop->opptr = onfailure;
			list.push_back(newop);
			if (x->andcond)
				cond(x->andcond, onsuccess, onfailure, nullptr);
			if (x->orcond)
				cond(x->orcond, onsuccess, onfailure, orop);
		}
		return newop;
	}
};

}  // namespace

struct virg_gpu_catalog {
	std::vector<TableDesc> tables;
};

extern "C" int virg_gpu_catalog_create(virg_gpu_catalog **out)
{
	VGPU_CHECK(out != nullptr, "null argument");
	*out = new virg_gpu_catalog();
	return 1;
}

extern "C" void virg_gpu_catalog_destroy(virg_gpu_catalog *c) { delete c; }

extern "C" int virg_gpu_catalog_add_table(virg_gpu_catalog *c, const char *name, int key_type,
	unsigned ncols, const char *const *col_names, const int *col_types, unsigned *table_id)
{
	VGPU_CHECK(c != nullptr && name != nullptr, "null argument");
	VGPU_CHECK(ncols <= VIRG_MAX_COLUMNS, "at most %d columns", VIRG_MAX_COLUMNS);
	VGPU_CHECK(strlen(name) < VIRG_MAX_TABLE_NAME, "table name too long");
	TableDesc t;
	t.name = name;
	t.key_type = key_type;
	for (unsigned i = 0; i < ncols; i++) {
		VGPU_CHECK(col_names[i] && strlen(col_names[i]) < VIRG_MAX_COLUMN_NAME, "column name too long");
		t.cols.push_back(col_names[i]);
		t.types.push_back(col_types[i]);
	}
	c->tables.push_back(t);
	if (table_id)
		*table_id = (unsigned)c->tables.size() - 1;
	return 1;
}

extern "C" int virg_gpu_sql_compile(const virg_gpu_catalog *cat, const char *query, virg_op *ops,
	unsigned *num_ops, unsigned *pc, char *names, unsigned *table_id)
{
	VGPU_CHECK(cat != nullptr && query != nullptr && ops != nullptr && num_ops != nullptr,
		"null argument");
	Parser ps;
	ps.lex(query);
	std::vector<ResultCol> rcols;
	Cond *where = nullptr;
	std::string tname;
	try {
		ps.expect(T_SELECT);
		while (true) {
			ResultCol rc;
			rc.expr = ps.expr();
			if (ps.peek() == T_AS) {
				ps.pos++;
				if (ps.peek() != T_STRING)
					ps.fail("syntax error");
				rc.output_name = ps.toks[ps.pos++].s;
			} else if (ps.peek() == T_STRING) {
				rc.output_name = ps.toks[ps.pos++].s;
			} else {
				expr_string(rc.expr, rc.output_name);
			}
			rcols.push_back(rc);
			if (ps.peek() != T_COMMA)
				break;
			ps.pos++;
		}
		ps.expect(T_FROM);
		if (ps.peek() != T_STRING)
			ps.fail("syntax error");
		tname = ps.toks[ps.pos++].s;
		if (ps.peek() == T_WHERE) {
			ps.pos++;
			where = ps.conditions();
		}
		ps.expect(T_EOF);
	} catch (Fail &) {
		VGPU_FAIL("parse error: %s", ps.err.c_str());
	}
	int tid = -1;
	for (size_t i = 0; i < cat->tables.size(); i++)
		if (cat->tables[i].name == tname) {
			tid = (int)i;
			break;
		}
	VGPU_CHECK(tid >= 0, "could not find table %s", tname.c_str());

	Gen g(cat->tables[(size_t)tid]);
	AbsOp *result, *converge;
	try {
		/* pass 0 and 1 */
		for (ResultCol &rc : rcols)
			g.types(rc.expr);
		if (where)
			g.cond_types(where);
		for (ResultCol &rc : rcols)
			g.fold(rc.expr);
		if (where)
			g.cond_fold(where);
		/* pass 2 */
		g.list.push_back(g.absop(OP_Table, tid, 0, 0, nullptr));
		for (ResultCol &rc : rcols)
			g.list.push_back(g.absop(OP_ResultColumn, rc.expr->datatype, 0, 0, nullptr));
		result = g.absop(OP_Result, 0, 0, 0, nullptr);
		converge = g.absop(OP_Converge, 0, 0, 0, nullptr);
		g.list.push_back(g.absop(OP_Parallel, 0, 0, 0, converge));
		if (where) {
			AbsOp *stub = g.absop(OP_Nop, 0, 0, 0, nullptr);
			g.cond(where, stub, result, nullptr);
			g.list.push_back(g.absop(OP_Invalid, 0, 0, 0, nullptr));
			g.list.push_back(stub);
		}
		for (ResultCol &rc : rcols)
			rc.output_reg = g.expr_reg(rc.expr);
		/* move result registers to the end, in order (generate.c:653-674) */
		const int nregs = (int)g.regs.size();
		for (int i = 0; i < nregs; i++)
			g.regs[i].index = i;
		for (ResultCol &rc : rcols) {
			int i = rc.output_reg;
			if (g.regs[i].index == nregs - 1)
				continue;
			int oldindex = g.regs[i].index;
			g.regs[i].index = nregs - 1;
			for (int k = 0; k < nregs; k++)
				if (k != i && g.regs[k].index > oldindex)
					g.regs[k].index--;
		}
		result->op.p1 = rcols[0].output_reg;
		result->op.p2 = (int)rcols.size();
		g.list.push_back(result);
		g.list.push_back(converge);
		g.list.push_back(g.absop(OP_Finish, 0, 0, 0, nullptr));
	} catch (Fail &) {
		VGPU_FAIL("%s", g.err.c_str());
	}
	/* pass 3: Nop placeholders take the index of the next real op */
	int idx = 0;
	for (AbsOp *a : g.list) {
		if (a->op.op != OP_Nop)
			a->index = idx++;
		else
			a->index = idx;
	}
	VGPU_CHECK(idx <= VIRG_OPS, "query needs %d ops, more than %d", idx, VIRG_OPS);
	/* pass 4 */
	for (AbsOp *a : g.list) {
		virg_op &o = a->op;
		switch (o.op) {
		case OP_Parallel: o.p3 = a->opptr->index + 1; break;
		case OP_Integer: case OP_Column: case OP_Rowid: case OP_Result: case OP_Float:
			o.p1 = g.regs[o.p1].index;
			break;
		case OP_Add: case OP_Sub: case OP_Mul: case OP_Div:
			o.p1 = g.regs[o.p1].index;
			o.p2 = g.regs[o.p2].index;
			o.p3 = g.regs[o.p3].index;
			break;
		case OP_Eq: case OP_Neq: case OP_Le: case OP_Lt: case OP_Ge: case OP_Gt:
			o.p1 = g.regs[o.p1].index;
			o.p2 = g.regs[o.p2].index;
			o.p3 = a->opptr->index;
			break;
		default: break;
		}
	}
	/* pass 5 */
	unsigned n = 0, parallel = 0, rc = 0;
	if (names)
		memset(names, 0, VIRG_OPS * VIRG_MAX_COLUMN_NAME);
	for (AbsOp *a : g.list) {
		if (a->op.op == OP_Nop)
			continue;
		if (a->op.op == OP_Parallel)
			parallel = n + 1;
		if (a->op.op == OP_ResultColumn && names) {
			strncpy(names + n * VIRG_MAX_COLUMN_NAME, rcols[rc].output_name.c_str(),
				VIRG_MAX_COLUMN_NAME - 1);
			rc++;
		}
		ops[n++] = a->op;
	}
	*num_ops = n;
	if (pc)
		*pc = parallel;
	if (table_id)
		*table_id = (unsigned)tid;
	return 1;
}
