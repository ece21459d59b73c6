/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Hand-written replacement for the reference's flex/bison front end
 * (src/sql/sql.l:30-81 and src/sql/sql.y:78-240), because flex and bison are
 * not installed here.  It builds the reference's own AST through the
 * reference's own builders (src/sql/node.c) and then calls the reference's
 * unmodified code generator virg_sql_generate (src/sql/generate.c:820), so the
 * opcode programs the oracle executes are the reference's programs.
 *
 * Grammar decisions that must match bison's parse of sql.y:
 *  - `expr: expr operator expr` has no terminal symbol, so the rule has no
 *    precedence and bison resolves its four shift/reduce conflicts (the
 *    `%expect 4` at sql.y:40, one per operator token) by shifting.  Every
 *    arithmetic operator is therefore right-associative with equal precedence:
 *    `a - b - c` parses as `a - (b - c)` and `a * b + c` as `a * (b + c)`.
 *  - conditions are right-recursive: `c AND rest` sets c->andcond,
 *    `c OR rest` sets c->orcond, and a parenthesised `( c AND|OR rest )` is a
 *    whole `conditions` (sql.y:126-149) that can only end a condition list;
 *    the parenthesised OR form also sets orfirst = 1.
 * Lexer decisions that must match flex's longest-match scan of sql.l:
 *  - whitespace is space, tab and newline only;
 *  - keywords are case-insensitive and win ties against identifiers;
 *    identifiers are [a-zA-Z][a-zA-Z0-9]*;
 *  - `-?[0-9]+` is an int (atoi) and `-?[0-9]+\.[0-9]+` a float (atof), so a
 *    leading minus binds to a following digit (`a -1` is two operands);
 *  - a character no rule matches is skipped (flex's default rule echoes it).
 * On a syntax error the reference's yyerror exits the process (sql.y:206-209);
 * here yyerror long-jumps back to virg_sql, which returns VIRG_FAIL.
 */
#include <ctype.h>
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "virginian.h"
#include "node.h"

enum {
	T_EOF, T_SELECT, T_FROM, T_WHERE, T_AS, T_AND, T_OR, T_COMMA, T_LP, T_RP,
	T_INT, T_FLOAT, T_STRING,
	T_PLUS, T_MINUS, T_MUL, T_DIV,
	T_CEQ, T_CNE, T_CLT, T_CLE, T_CGT, T_CGE
};

typedef struct {
	int type;
	int i;
	float f;
	char *s;
} token;

#define MAX_TOKENS 1024

static token toks[MAX_TOKENS];
static int ntoks;
static int tpos;
static jmp_buf parse_fail;

void yyerror(char *s)
{
	fprintf(stderr, "Parse Error :: %s\n", s);
	longjmp(parse_fail, 1);
}

static int kw(const char *p, int n, const char *w)
{
	int i;
	if((int)strlen(w) != n)
		return 0;
	for(i = 0; i < n; i++)
		if(tolower((unsigned char)p[i]) != w[i])
			return 0;
	return 1;
}

static void lex(const char *q)
{
	const char *p = q;
	ntoks = 0;
	while(*p) {
		token t;
		memset(&t, 0, sizeof(t));
		if(*p == ' ' || *p == '\t' || *p == '\n') { p++; continue; }
		if(isalpha((unsigned char)*p)) {
			const char *s = p;
			while(isalnum((unsigned char)*p))
				p++;
			int n = (int)(p - s);
			if(kw(s, n, "select")) t.type = T_SELECT;
			else if(kw(s, n, "from")) t.type = T_FROM;
			else if(kw(s, n, "where")) t.type = T_WHERE;
			else if(kw(s, n, "as")) t.type = T_AS;
			else if(kw(s, n, "and")) t.type = T_AND;
			else if(kw(s, n, "or")) t.type = T_OR;
			else {
				t.type = T_STRING;
				t.s = malloc(n + 1);
				memcpy(t.s, s, n);
				t.s[n] = '\0';
			}
		}
		else if(isdigit((unsigned char)*p) ||
				(*p == '-' && isdigit((unsigned char)p[1]))) {
			const char *s = p;
			if(*p == '-')
				p++;
			while(isdigit((unsigned char)*p))
				p++;
			if(*p == '.' && isdigit((unsigned char)p[1])) {
				p++;
				while(isdigit((unsigned char)*p))
					p++;
				char buf[128];
				int n = (int)(p - s) < 127 ? (int)(p - s) : 127;
				memcpy(buf, s, n);
				buf[n] = '\0';
				t.type = T_FLOAT;
				t.f = (float)atof(buf);
			}
			else {
				char buf[128];
				int n = (int)(p - s) < 127 ? (int)(p - s) : 127;
				memcpy(buf, s, n);
				buf[n] = '\0';
				t.type = T_INT;
				t.i = atoi(buf);
			}
		}
		else if(p[0] == '!' && p[1] == '=') { t.type = T_CNE; p += 2; }
		else if(p[0] == '<' && p[1] == '=') { t.type = T_CLE; p += 2; }
		else if(p[0] == '>' && p[1] == '=') { t.type = T_CGE; p += 2; }
		else if(*p == '=') { t.type = T_CEQ; p++; }
		else if(*p == '<') { t.type = T_CLT; p++; }
		else if(*p == '>') { t.type = T_CGT; p++; }
		else if(*p == '+') { t.type = T_PLUS; p++; }
		else if(*p == '-') { t.type = T_MINUS; p++; }
		else if(*p == '*') { t.type = T_MUL; p++; }
		else if(*p == '/') { t.type = T_DIV; p++; }
		else if(*p == ',') { t.type = T_COMMA; p++; }
		else if(*p == '(') { t.type = T_LP; p++; }
		else if(*p == ')') { t.type = T_RP; p++; }
		else { p++; continue; }
		if(ntoks >= MAX_TOKENS - 1)
			yyerror("query too long");
		toks[ntoks++] = t;
	}
	toks[ntoks].type = T_EOF;
	toks[ntoks].s = NULL;
}

static int peek(void) { return toks[tpos].type; }

static void expect(int type)
{
	if(toks[tpos].type != type)
		yyerror("syntax error");
	tpos++;
}

/* string tokens are handed to the AST, which owns them afterwards; a token
 * that was consumed during a failed speculative parse gets a fresh copy */
static char *take_string(void)
{
	char *s = toks[tpos].s;
	char *c = malloc(strlen(s) + 1);
	strcpy(c, s);
	tpos++;
	return c;
}

static int is_condop(int t)
{
	return t == T_CEQ || t == T_CNE || t == T_CLT || t == T_CLE ||
		t == T_CGT || t == T_CGE;
}

static int condop_node(int t)
{
	switch(t) {
		case T_CEQ: return NODE_COND_EQ;
		case T_CNE: return NODE_COND_NE;
		case T_CLT: return NODE_COND_LT;
		case T_CLE: return NODE_COND_LE;
		case T_CGT: return NODE_COND_GT;
		default: return NODE_COND_GE;
	}
}

static int is_operator(int t)
{
	return t == T_PLUS || t == T_MINUS || t == T_MUL || t == T_DIV;
}

static int operator_node(int t)
{
	switch(t) {
		case T_PLUS: return NODE_OP_PLUS;
		case T_MINUS: return NODE_OP_MINUS;
		case T_MUL: return NODE_OP_MUL;
		default: return NODE_OP_DIV;
	}
}

/* speculative parsing: a failed alternative unwinds to the saved position */
static jmp_buf *spec_env;

static void spec_fail(void)
{
	if(spec_env)
		longjmp(*spec_env, 1);
	yyerror("syntax error");
}

static void sexpect(int type)
{
	if(toks[tpos].type != type)
		spec_fail();
	tpos++;
}

static node_expr *parse_expr(void);

static node_expr *parse_primary(void)
{
	node_expr *x;
	switch(peek()) {
		case T_LP:
			tpos++;
			x = parse_expr();
			sexpect(T_RP);
			return x;
		case T_INT:
			x = node_expr_buildint(toks[tpos].i);
			tpos++;
			return x;
		case T_FLOAT:
			x = node_expr_buildfloat(toks[tpos].f);
			tpos++;
			return x;
		case T_STRING:
			return node_expr_buildcolumn(take_string());
		default:
			spec_fail();
			return NULL;
	}
}

/* right-recursive, single precedence level: see the file comment */
static node_expr *parse_expr(void)
{
	node_expr *lhs = parse_primary();
	if(is_operator(peek())) {
		int op = operator_node(peek());
		tpos++;
		node_expr *rhs = parse_expr();
		return node_expr_buildop(op, lhs, rhs);
	}
	return lhs;
}

static node_condition *parse_condition(void)
{
	if(peek() == T_LP) {
		int save = tpos;
		jmp_buf env, *outer = spec_env;
		spec_env = &env;
		if(setjmp(env) == 0) {
			tpos++;
			node_expr *l = parse_expr();
			if(!is_condop(peek()))
				spec_fail();
			int op = condop_node(peek());
			tpos++;
			node_expr *r = parse_expr();
			sexpect(T_RP);
			spec_env = outer;
			return node_condition_build(op, l, r);
		}
		spec_env = outer;
		tpos = save;
	}
	node_expr *l = parse_expr();
	if(!is_condop(peek()))
		spec_fail();
	int op = condop_node(peek());
	tpos++;
	node_expr *r = parse_expr();
	return node_condition_build(op, l, r);
}

static node_condition *parse_conditions(void)
{
	if(peek() == T_LP) {
		int save = tpos;
		jmp_buf env, *outer = spec_env;
		spec_env = &env;
		if(setjmp(env) == 0) {
			tpos++;
			node_condition *c = parse_condition();
			int link = peek();
			if(link != T_AND && link != T_OR)
				spec_fail();
			tpos++;
			node_condition *rest = parse_conditions();
			sexpect(T_RP);
			spec_env = outer;
			if(link == T_AND)
				c->andcond = rest;
			else {
				c->orcond = rest;
				c->orfirst = 1;
			}
			return c;
		}
		spec_env = outer;
		tpos = save;
	}
	node_condition *c = parse_condition();
	if(peek() == T_AND) {
		tpos++;
		c->andcond = parse_conditions();
	}
	else if(peek() == T_OR) {
		tpos++;
		c->orcond = parse_conditions();
	}
	return c;
}

static node_resultcol *parse_resultcols(void)
{
	node_expr *x = parse_expr();
	node_resultcol *rc;
	if(peek() == T_AS) {
		tpos++;
		if(peek() != T_STRING)
			spec_fail();
		rc = node_resultcol_buildas(x, take_string());
	}
	else if(peek() == T_STRING)
		rc = node_resultcol_buildas(x, take_string());
	else
		rc = node_resultcol_build(x);
	rc->next = NULL;
	if(peek() == T_COMMA) {
		tpos++;
		rc->next = parse_resultcols();
	}
	return rc;
}

static virg_node_root *parse_query(void)
{
	expect(T_SELECT);
	node_resultcol *cols = parse_resultcols();
	expect(T_FROM);
	if(peek() != T_STRING)
		yyerror("syntax error");
	char *table = take_string();
	node_condition *conds = NULL;
	if(peek() == T_WHERE) {
		tpos++;
		conds = parse_conditions();
	}
	expect(T_EOF);
	node_select *sel = node_select_build(table, cols, conds);
	free(table);
	return node_root_build(QUERY_TYPE_SELECT, sel);
}

int virg_sql(virginian *v, const char *querystr, virg_vm *vm)
{
	int i;
	parse_virg = v;
	spec_env = NULL;
	if(setjmp(parse_fail)) {
		for(i = 0; i < ntoks; i++)
			free(toks[i].s);
		return VIRG_FAIL;
	}
	lex(querystr);
	tpos = 0;
	virg_node_root *root = parse_query();
	for(i = 0; i < ntoks; i++)
		free(toks[i].s);
	ntoks = 0;
	virg_sql_generate(root, vm);
	node_root_free(root);
	return VIRG_SUCCESS;
}
