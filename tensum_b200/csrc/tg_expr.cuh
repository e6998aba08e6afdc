// tg_expr.cuh -- evaluation of compiled parameter-file expressions (host and device).
//
// The reference reads its initial and boundary conditions as fparser
// expressions of (x, y, t) with the constant pi, the user constants of the
// parameter file and the perturbation function pert(type, x, y, p)
// (src/fparser.h:20-36, src/perturb.cc:16-208).  tg_expr.cu compiles such an
// expression into the postfix program below (constant sub-expressions folded
// on the host); this header evaluates it for one point and one sample's random
// numbers, so a device kernel can fill a state or a boundary table without a
// host round trip.  The semantics follow fparser's for real values:
// comparisons carry the tolerance 1e-12 (x < y means x < y - 1e-12, x = y
// means |x - y| <= 1e-12), a value is true when |v| >= 0.5, and min / max pick
// d1 < d2 ? d1 : d2 / d1 > d2 ? d1 : d2.
#pragma once

#include <math.h>

#include <vector>

#include "../../include/tensum_gpu.h"

namespace tg {
namespace expr {

constexpr int kStack = 32;          // evaluation stack depth a program may use
constexpr double kEps = 1.0e-12;    // fparser's comparison tolerance for doubles

enum : int {
  OP_CONST = 0, OP_X, OP_Y, OP_T,
  OP_NEG, OP_NOT,
  OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MOD, OP_POW,
  OP_EQ, OP_NE, OP_LT, OP_LE, OP_GT, OP_GE, OP_AND, OP_OR,
  OP_F1, OP_F2, OP_IF, OP_PERT
};
// one-argument functions (OP_F1 operand)
enum : int {
  F_ABS = 0, F_ACOS, F_ACOSH, F_ASIN, F_ASINH, F_ATAN, F_ATANH, F_CBRT, F_CEIL, F_COS, F_COSH, F_COT, F_CSC,
  F_EXP, F_EXP2, F_FLOOR, F_INT, F_LOG, F_LOG10, F_LOG2, F_SEC, F_SIN, F_SINH, F_SQRT, F_TAN, F_TANH, F_TRUNC
};
// two-argument functions (OP_F2 operand)
enum : int { F2_ATAN2 = 0, F2_HYPOT, F2_MAX, F2_MIN, F2_POW };
// error bits of an evaluation
enum : int { ERR_PERT_INDEX = 1, ERR_PERT_TYPE = 2, ERR_STACK = 4 };

__host__ __device__ inline bool truth(double v) { return fabs(v) >= 0.5; }

__host__ __device__ inline double f1(int f, double a) {
  switch (f) {
    case F_ABS: return fabs(a);
    case F_ACOS: return acos(a);
    case F_ACOSH: return acosh(a);
    case F_ASIN: return asin(a);
    case F_ASINH: return asinh(a);
    case F_ATAN: return atan(a);
    case F_ATANH: return atanh(a);
    case F_CBRT: return cbrt(a);
    case F_CEIL: return ceil(a);
    case F_COS: return cos(a);
    case F_COSH: return cosh(a);
    case F_COT: return 1.0 / tan(a);
    case F_CSC: return 1.0 / sin(a);
    case F_EXP: return exp(a);
    case F_EXP2: return exp2(a);
    case F_FLOOR: return floor(a);
    case F_INT: return floor(a + 0.5);
    case F_LOG: return log(a);
    case F_LOG10: return log10(a);
    case F_LOG2: return log2(a);
    case F_SEC: return 1.0 / cos(a);
    case F_SIN: return sin(a);
    case F_SINH: return sinh(a);
    case F_SQRT: return sqrt(a);
    case F_TAN: return tan(a);
    case F_TANH: return tanh(a);
    default: return trunc(a);
  }
}

__host__ __device__ inline double f2(int f, double a, double b) {
  switch (f) {
    case F2_ATAN2: return atan2(a, b);
    case F2_HYPOT: return hypot(a, b);
    case F2_MAX: return a > b ? a : b;
    case F2_MIN: return a < b ? a : b;
    default: return pow(a, b);
  }
}

// pert(type, x, y, p) of src/perturb.cc:16-208 with the sample's random numbers
// rnd[0 .. n): 1 multi-modal sin(2 pi y + b_i) weighted a_i / sum(a) inside the
// centred band of width p, 2 piecewise-constant +-r_k over M sub-bands of that
// band, 3 as 1 with wavenumber i (sin(2 i pi y + b_i)), 4 the p-th random number.
__host__ __device__ inline double pert(double type, double x, double y, double p, const double* rnd, int n, int* err) {
  const double kPi = 3.14159265358979323846;
  (void)x;
  const int kind = (int)type;
  if (kind == 1 || kind == 3) {
    const int M = (int)floor(n / 2.0);
    const double frac = fmax(fmin(p, 1.0), 0.0);
    const double llim = (1.0 - frac) * 0.5, ulim = (frac + 1.0) * 0.5;
    double sum = 0.0;
    for (int i = 0; i < M; ++i) sum += rnd[i];
    double v = 0.0;
    if (y > llim && y < ulim)
      for (int i = 0; i < M; ++i)
        v += (rnd[i] / sum) * sin(kind == 1 ? 2 * kPi * y + rnd[M + i] : 2 * i * kPi * y + rnd[M + i]);
    return v;
  }
  if (kind == 2) {
    const int M = n;
    const double frac = fmax(fmin(p, 1.0), 0.0);
    const double llim = (1.0 - frac) * 0.5, ulim = (frac + 1.0) * 0.5;
    if (!(y > llim && y < ulim)) return 0.0;
    const double div_size = frac / (double)M;
    int div = (int)floor((y - llim) / div_size);
    if (div == M) div--;
    if (div < 0 || div >= M) { *err |= ERR_PERT_INDEX; return 0.0; }
    return rnd[div] * ((div & 1) ? -1.0 : 1.0);
  }
  if (kind == 4) {
    const int id = (int)p;
    if (n <= 0) return 0.0;
    if (id < 1 || id > n) { *err |= ERR_PERT_INDEX; return 0.0; }
    return rnd[id - 1];
  }
  *err |= ERR_PERT_TYPE;
  return 0.0;
}

// Evaluates program code[0 .. n) (instruction = op | operand << 8) with
// constants k at (x, y, t) for one sample's random numbers.
__host__ __device__ inline double eval(const int* code, int n, const double* k, double x, double y, double t,
                                       const double* rnd, int nrnd, int* err) {
  double st[kStack];
  int sp = 0;
  for (int i = 0; i < n; ++i) {
    const int op = code[i] & 0xff, arg = code[i] >> 8;
    if (op <= OP_T) {
      if (sp >= kStack) { *err |= ERR_STACK; return 0.0; }
      st[sp++] = op == OP_CONST ? k[arg] : op == OP_X ? x : op == OP_Y ? y : t;
      continue;
    }
    switch (op) {
      case OP_NEG: st[sp - 1] = -st[sp - 1]; break;
      case OP_NOT: st[sp - 1] = truth(st[sp - 1]) ? 0.0 : 1.0; break;
      case OP_F1: st[sp - 1] = f1(arg, st[sp - 1]); break;
      case OP_IF: sp -= 2; st[sp - 1] = truth(st[sp - 1]) ? st[sp] : st[sp + 1]; break;
      case OP_PERT: sp -= 3; st[sp - 1] = pert(st[sp - 1], st[sp], st[sp + 1], st[sp + 2], rnd, nrnd, err); break;
      default: {
        const double b = st[--sp], a = st[sp - 1];
        double r;
        switch (op) {
          case OP_ADD: r = a + b; break;
          case OP_SUB: r = a - b; break;
          case OP_MUL: r = a * b; break;
          case OP_DIV: r = a / b; break;
          case OP_MOD: r = fmod(a, b); break;
          case OP_POW: r = pow(a, b); break;
          case OP_EQ: r = fabs(a - b) <= kEps ? 1.0 : 0.0; break;
          case OP_NE: r = fabs(a - b) > kEps ? 1.0 : 0.0; break;
          case OP_LT: r = a < b - kEps ? 1.0 : 0.0; break;
          case OP_LE: r = a <= b + kEps ? 1.0 : 0.0; break;
          case OP_GT: r = b < a - kEps ? 1.0 : 0.0; break;
          case OP_GE: r = b <= a + kEps ? 1.0 : 0.0; break;
          case OP_AND: r = (truth(a) && truth(b)) ? 1.0 : 0.0; break;
          case OP_OR: r = (truth(a) || truth(b)) ? 1.0 : 0.0; break;
          default: r = f2(arg, a, b); break;
        }
        st[sp - 1] = r;
      }
    }
  }
  return st[0];
}

// Five programs (T, u, v, w, p) packed one after another: offsets off[0 .. 5]
// into code, constants in k (each program indexes the shared constant array).
struct Field5 {
  const int* code;
  const int* off;       // 6 entries
  const double* k;
};

__host__ __device__ inline double eval5(const Field5& f, int c, double x, double y, double t, const double* rnd,
                                        int nrnd, int* err) {
  return eval(f.code + f.off[c], f.off[c + 1] - f.off[c], f.k, x, y, t, rnd, nrnd, err);
}

// Packs five programs (NULL entries: the constant fallback[c], or 0) into one
// code array with offsets and one constant pool (tg_expr.cu).
void pack5(const tg_expr* const* f, const double* fallback, std::vector<int>& code, std::vector<int>& off,
           std::vector<double>& k);

}  // namespace expr
}  // namespace tg
