// tg_expr.cu -- compiler of parameter-file expressions into tg_expr programs.
//
// Grammar and precedence are fparser's (the parser the reference uses for its
// initial and boundary conditions, src/fparser.h:20-36), lowest first:
//   |   &   = != < <= > >=   + -   * / %   unary - !   ^ (right-associative)
// with numbers, the variables x, y, t, the constant pi, the caller's named
// constants (the parameter file's constants section), the real functions of
// fparser and pert(type, x, y, p).  Sub-expressions without variables or pert
// are folded on the host; everything else is evaluated as written by
// tg_expr.cuh on the host or on the device.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/tensum_gpu.h"
#include "tg_expr.cuh"

using namespace tg::expr;

struct tg_expr {
  std::vector<int> code;
  std::vector<double> k;
  std::string text;
};

namespace {

thread_local std::string g_expr_error;

struct Node {
  int op;             // OP_*
  int arg;            // function id, constant index
  double val;         // OP_CONST value before the constant pool is built
  std::vector<int> kids;
};

struct Parser {
  const char* s;
  size_t pos = 0;
  std::map<std::string, double> consts;
  std::vector<Node> nodes;
  std::string err;

  int add(int op, int arg, double val, std::vector<int> kids) {
    nodes.push_back(Node{op, arg, val, std::move(kids)});
    return (int)nodes.size() - 1;
  }
  void ws() { while (s[pos] == ' ' || s[pos] == '\t' || s[pos] == '\n' || s[pos] == '\r') ++pos; }
  bool eat(const char* t) {
    ws();
    const size_t n = std::strlen(t);
    if (std::strncmp(s + pos, t, n) == 0) { pos += n; return true; }
    return false;
  }
  int fail(const std::string& m) {
    if (err.empty()) err = m + " at position " + std::to_string(pos) + " of \"" + s + "\"";
    return -1;
  }

  int parse_or() {
    int a = parse_and();
    while (a >= 0 && eat("|")) { int b = parse_and(); if (b < 0) return -1; a = add(OP_OR, 0, 0, {a, b}); }
    return a;
  }
  int parse_and() {
    int a = parse_cmp();
    while (a >= 0 && eat("&")) { int b = parse_cmp(); if (b < 0) return -1; a = add(OP_AND, 0, 0, {a, b}); }
    return a;
  }
  int parse_cmp() {
    int a = parse_add();
    while (a >= 0) {
      int op;
      if (eat("!=")) op = OP_NE;
      else if (eat("<=")) op = OP_LE;
      else if (eat(">=")) op = OP_GE;
      else if (eat("=")) op = OP_EQ;
      else if (eat("<")) op = OP_LT;
      else if (eat(">")) op = OP_GT;
      else break;
      int b = parse_add();
      if (b < 0) return -1;
      a = add(op, 0, 0, {a, b});
    }
    return a;
  }
  int parse_add() {
    int a = parse_mul();
    while (a >= 0) {
      int op;
      if (eat("+")) op = OP_ADD;
      else if (eat("-")) op = OP_SUB;
      else break;
      int b = parse_mul();
      if (b < 0) return -1;
      a = add(op, 0, 0, {a, b});
    }
    return a;
  }
  int parse_mul() {
    int a = parse_unary();
    while (a >= 0) {
      int op;
      if (eat("*")) op = OP_MUL;
      else if (eat("/")) op = OP_DIV;
      else if (eat("%")) op = OP_MOD;
      else break;
      int b = parse_unary();
      if (b < 0) return -1;
      a = add(op, 0, 0, {a, b});
    }
    return a;
  }
  int parse_unary() {
    if (eat("-")) { int a = parse_unary(); return a < 0 ? -1 : add(OP_NEG, 0, 0, {a}); }
    ws();
    if (s[pos] == '!' && s[pos + 1] != '=') { ++pos; int a = parse_unary(); return a < 0 ? -1 : add(OP_NOT, 0, 0, {a}); }
    return parse_pow();
  }
  int parse_pow() {
    int a = parse_primary();
    if (a >= 0 && eat("^")) {
      int b = parse_unary();   // right-associative, a signed exponent allowed
      if (b < 0) return -1;
      a = add(OP_POW, 0, 0, {a, b});
    }
    return a;
  }
  int parse_primary() {
    ws();
    const char c = s[pos];
    if (c == '(') {
      ++pos;
      int a = parse_or();
      if (a < 0) return -1;
      if (!eat(")")) return fail("missing ')'");
      return a;
    }
    if ((c >= '0' && c <= '9') || c == '.') {
      char* end = nullptr;
      const double v = std::strtod(s + pos, &end);
      if (end == s + pos) return fail("bad number");
      pos = end - s;
      return add(OP_CONST, 0, v, {});
    }
    if (std::isalpha((unsigned char)c) || c == '_') {
      size_t b = pos;
      while (std::isalnum((unsigned char)s[pos]) || s[pos] == '_') ++pos;
      const std::string id(s + b, pos - b);
      ws();
      if (s[pos] == '(') {
        ++pos;
        std::vector<int> args;
        if (!eat(")")) {
          for (;;) {
            int a = parse_or();
            if (a < 0) return -1;
            args.push_back(a);
            if (eat(")")) break;
            if (!eat(",")) return fail("expected ',' or ')'");
          }
        }
        return call(id, args);
      }
      if (id == "x") return add(OP_X, 0, 0, {});
      if (id == "y") return add(OP_Y, 0, 0, {});
      if (id == "t") return add(OP_T, 0, 0, {});
      auto it = consts.find(id);
      if (it != consts.end()) return add(OP_CONST, 0, it->second, {});
      return fail("unknown name '" + id + "'");
    }
    return fail("unexpected character");
  }
  int call(const std::string& f, const std::vector<int>& a) {
    static const std::map<std::string, int> one = {
        {"abs", F_ABS}, {"acos", F_ACOS}, {"acosh", F_ACOSH}, {"asin", F_ASIN}, {"asinh", F_ASINH},
        {"atan", F_ATAN}, {"atanh", F_ATANH}, {"cbrt", F_CBRT}, {"ceil", F_CEIL}, {"cos", F_COS},
        {"cosh", F_COSH}, {"cot", F_COT}, {"csc", F_CSC}, {"exp", F_EXP}, {"exp2", F_EXP2},
        {"floor", F_FLOOR}, {"int", F_INT}, {"log", F_LOG}, {"log10", F_LOG10}, {"log2", F_LOG2},
        {"sec", F_SEC}, {"sin", F_SIN}, {"sinh", F_SINH}, {"sqrt", F_SQRT}, {"tan", F_TAN},
        {"tanh", F_TANH}, {"trunc", F_TRUNC}};
    static const std::map<std::string, int> two = {
        {"atan2", F2_ATAN2}, {"hypot", F2_HYPOT}, {"max", F2_MAX}, {"min", F2_MIN}, {"pow", F2_POW}};
    auto i1 = one.find(f);
    if (i1 != one.end()) {
      if (a.size() != 1) return fail(f + " takes one argument");
      return add(OP_F1, i1->second, 0, a);
    }
    auto i2 = two.find(f);
    if (i2 != two.end()) {
      if (a.size() != 2) return fail(f + " takes two arguments");
      return add(OP_F2, i2->second, 0, a);
    }
    if (f == "if") {
      if (a.size() != 3) return fail("if takes three arguments");
      return add(OP_IF, 0, 0, a);
    }
    if (f == "pert") {
      if (a.size() != 4) return fail("pert takes four arguments (type, x, y, p)");
      return add(OP_PERT, 0, 0, a);
    }
    return fail("unknown function '" + f + "'");
  }

  // folds sub-expressions free of x, y, t and pert; returns whether node i is constant
  bool fold(int i) {
    Node& n = nodes[i];
    if (n.op == OP_CONST) return true;
    if (n.op == OP_X || n.op == OP_Y || n.op == OP_T) return false;
    bool all = true;
    for (int c : n.kids) all = fold(c) && all;
    if (!all || n.op == OP_PERT) return false;
    std::vector<int> code;
    std::vector<double> k;
    for (int c : nodes[i].kids) { code.push_back(OP_CONST | ((int)k.size() << 8)); k.push_back(nodes[c].val); }
    code.push_back(nodes[i].op | (nodes[i].arg << 8));
    int e = 0;
    const double v = eval(code.data(), (int)code.size(), k.data(), 0.0, 0.0, 0.0, nullptr, 0, &e);
    Node& m = nodes[i];
    m.op = OP_CONST; m.val = v; m.kids.clear();
    return true;
  }

  // postfix emission; returns the stack depth needed
  int emit(int i, std::vector<int>& code, std::vector<double>& k) {
    const Node& n = nodes[i];
    if (n.op == OP_CONST) {
      code.push_back(OP_CONST | ((int)k.size() << 8));
      k.push_back(n.val);
      return 1;
    }
    if (n.op == OP_X || n.op == OP_Y || n.op == OP_T) { code.push_back(n.op); return 1; }
    int depth = 0, j = 0;
    for (int c : n.kids) { depth = std::max(depth, j + emit(c, code, k)); ++j; }
    code.push_back(n.op | (n.arg << 8));
    return depth;
  }
};

}  // namespace

extern "C" {

tg_status tg_expr_create(const char* text, int n_const, const char* const* names, const double* values,
                         tg_expr** out) {
  if (!out || !text || n_const < 0 || (n_const > 0 && (!names || !values))) {
    g_expr_error = "NULL argument";
    return TG_INVALID_ARG;
  }
  *out = nullptr;
  Parser p;
  p.s = text;
  p.consts["pi"] = 3.14159265358979323846;   // src/fparser.h:25
  for (int i = 0; i < n_const; ++i) {
    if (!names[i]) { g_expr_error = "NULL constant name"; return TG_INVALID_ARG; }
    p.consts[names[i]] = values[i];
  }
  int root = p.parse_or();
  p.ws();
  if (root >= 0 && p.s[p.pos] != '\0') root = p.fail("unexpected trailing text");
  if (root < 0) { g_expr_error = p.err; return TG_INVALID_ARG; }
  p.fold(root);
  tg_expr* e = new (std::nothrow) tg_expr();
  if (!e) { g_expr_error = "out of host memory"; return TG_INVALID_ARG; }
  const int depth = p.emit(root, e->code, e->k);
  if (depth > kStack || e->k.size() >= (1u << 23) || e->code.size() > (1u << 20)) {
    delete e;
    g_expr_error = "expression too deep or too long";
    return TG_INVALID_ARG;
  }
  e->text = text;
  *out = e;
  return TG_OK;
}

tg_status tg_expr_destroy(tg_expr* e) {
  delete e;
  return TG_OK;
}

const char* tg_expr_last_error(void) { return g_expr_error.c_str(); }

tg_status tg_expr_eval(const tg_expr* e, double x, double y, double t, const double* rnd, int n_rnd, double* out) {
  if (!e || !out || n_rnd < 0 || (n_rnd > 0 && !rnd)) { g_expr_error = "bad argument"; return TG_INVALID_ARG; }
  int err = 0;
  *out = eval(e->code.data(), (int)e->code.size(), e->k.data(), x, y, t, rnd, n_rnd, &err);
  if (err) { g_expr_error = "pert: unknown type or random-number index out of range"; return TG_INVALID_ARG; }
  return TG_OK;
}

}  // extern "C"

namespace tg {
namespace expr {

// Packs five programs (entries may be NULL: the constant `fallback[c]`) into
// one code array with offsets and one constant pool, constant indices rebased.
void pack5(const tg_expr* const* f, const double* fallback, std::vector<int>& code, std::vector<int>& off,
           std::vector<double>& k) {
  code.clear(); off.assign(1, 0); k.clear();
  for (int c = 0; c < 5; ++c) {
    if (f && f[c]) {
      const int base = (int)k.size();
      for (int ins : f[c]->code) {
        const int op = ins & 0xff;
        code.push_back(op == OP_CONST ? (OP_CONST | (((ins >> 8) + base) << 8)) : ins);
      }
      k.insert(k.end(), f[c]->k.begin(), f[c]->k.end());
    } else {
      code.push_back(OP_CONST | ((int)k.size() << 8));
      k.push_back(fallback ? fallback[c] : 0.0);
    }
    off.push_back((int)code.size());
  }
}

}  // namespace expr
}  // namespace tg
