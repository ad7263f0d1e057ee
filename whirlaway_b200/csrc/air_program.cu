// Constraint programs: validation, register assignment for the interpreter kernels, and the
// host evaluation the verifier uses.
#include "air_program.h"

#include <algorithm>
#include <stdexcept>
#include <string>

namespace wl {

ProgramAir ProgramAir::build(int W, int n_constraints, int degree, int n_ops, const int32_t* ops, int n_consts,
                             const uint32_t* consts_canonical) {
  if (W < 1 || W > 32767) throw std::invalid_argument("AIR program: 1..32767 columns");
  if (n_constraints < 1) throw std::invalid_argument("AIR program: no constraints");
  if (degree < 1 || degree > 3) throw std::invalid_argument("AIR program: constraint degree must be 1, 2 or 3");
  if (n_ops < 1 || !ops) throw std::invalid_argument("AIR program: no instructions");
  if (n_consts < 0 || n_consts > 65535 || (n_consts > 0 && !consts_canonical))
    throw std::invalid_argument("AIR program: bad constants");
  ProgramAir p;
  p.W = W;
  p.NC = n_constraints;
  p.degree = degree;
  p.ops.assign(ops, ops + 3 * size_t(n_ops));
  for (int j = 0; j < n_consts; j++) {
    if (consts_canonical[j] >= kb::P) throw std::invalid_argument("AIR program: constant not below p");
    p.consts.push_back(kb::to_mont(consts_canonical[j]));
  }
  // validation; the register each value lives in is that of its root (EMIT aliases its operand)
  std::vector<int> root(n_ops), last(n_ops, -1);
  int emits = 0;
  for (int i = 0; i < n_ops; i++) {
    const int op = ops[3 * i], a = ops[3 * i + 1], b = ops[3 * i + 2];
    const bool two = op == PROG_ADD || op == PROG_SUB || op == PROG_MUL;
    root[i] = i;
    if (op == PROG_UP || op == PROG_DOWN) {
      if (a < 0 || a >= W) throw std::invalid_argument("AIR program: column out of range at " + std::to_string(i));
    } else if (op == PROG_CONST) {
      if (a < 0 || a >= n_consts) throw std::invalid_argument("AIR program: constant out of range at " + std::to_string(i));
    } else if (two || op == PROG_EMIT) {
      if (a < 0 || a >= i || (two && (b < 0 || b >= i)))
        throw std::invalid_argument("AIR program: operand is not an earlier value at " + std::to_string(i));
      if (op == PROG_EMIT) {
        root[i] = root[a];
        emits++;
      }
    } else {
      throw std::invalid_argument("AIR program: unknown instruction at " + std::to_string(i));
    }
  }
  if (emits != n_constraints) throw std::invalid_argument("AIR program: EMIT count differs from the constraint count");
  // Instructions with exactly one constant operand take the constant as an immediate:
  // MUL -> MULC, ADD -> ADDC, SUB(x, c) -> ADDC(x, -c). kind[i]: the device op, other[i]: the
  // non-constant operand, imm[i]: the constant (Montgomery form).
  auto const_of = [&](int v) { return ops[3 * root[v]] == PROG_CONST ? ops[3 * root[v] + 1] : -1; };
  std::vector<int> kind(n_ops), other(n_ops, -1);
  std::vector<uint32_t> imm(n_ops, 0);
  for (int i = 0; i < n_ops; i++) {
    const int op = ops[3 * i], a = ops[3 * i + 1], b = ops[3 * i + 2];
    kind[i] = op;
    if (op != PROG_ADD && op != PROG_SUB && op != PROG_MUL) continue;
    const int ca = const_of(a), cb = const_of(b);
    if ((ca >= 0) == (cb >= 0)) continue;  // no constant, or two
    if (op == PROG_SUB && ca >= 0) continue;  // c - x stays general
    const int x = ca >= 0 ? b : a;
    const uint32_t c = p.consts[ca >= 0 ? ca : cb];
    kind[i] = op == PROG_MUL ? PROG_MULC : PROG_ADDC;
    other[i] = x;
    imm[i] = op == PROG_SUB ? kb::neg(c) : c;
  }
  // operands read from registers (MULC / ADDC read one)
  auto reads = [&](int i, int& r0, int& r1) {
    const int op = ops[3 * i], a = ops[3 * i + 1], b = ops[3 * i + 2];
    r0 = r1 = -1;
    if (kind[i] == PROG_MULC || kind[i] == PROG_ADDC) {
      r0 = root[other[i]];
    } else if (op >= PROG_ADD) {
      r0 = root[a];
      if (op <= PROG_MUL) r1 = root[b];
    }
  };
  for (int i = 0; i < n_ops; i++) {
    int r0, r1;
    reads(i, r0, r1);
    if (r0 >= 0) last[r0] = std::max(last[r0], i);
    if (r1 >= 0) last[r1] = std::max(last[r1], i);
  }
  // linear scan: operands are read before the result is written, so a register whose last
  // use is this instruction can take the result
  std::vector<int> reg(n_ops, -1), free_regs;
  int next = 0;
  auto take = [&]() {
    if (!free_regs.empty()) {
      const int r = free_regs.back();
      free_regs.pop_back();
      return r;
    }
    if (next >= PROG_MAX_REGS)
      throw std::invalid_argument("AIR program: more than " + std::to_string(PROG_MAX_REGS) + " values live at once");
    return next++;
  };
  p.code.reserve(n_ops);
  for (int i = 0; i < n_ops; i++) {
    const int op = ops[3 * i], a = ops[3 * i + 1];
    if (op == PROG_CONST && last[i] < 0) continue;  // read only as an immediate (or never)
    int r0, r1;
    reads(i, r0, r1);
    const uint32_t ra = r0 >= 0 ? uint32_t(reg[r0]) : 0u, rb = r1 >= 0 ? uint32_t(reg[r1]) : 0u;
    // free the operands that die here (once each)
    if (r0 >= 0 && last[r0] == i) free_regs.push_back(reg[r0]);
    if (r1 >= 0 && last[r1] == i && r1 != r0) free_regs.push_back(reg[r1]);
    uint32_t dst = 0;
    if (op != PROG_EMIT) {
      reg[i] = take();
      dst = uint32_t(reg[i]);
      if (last[i] < 0) free_regs.push_back(reg[i]);  // never read
    }
    const uint32_t aa = op <= PROG_CONST ? uint32_t(a) : ra;
    const uint32_t y = (kind[i] == PROG_MULC || kind[i] == PROG_ADDC) ? imm[i] : rb;
    p.code.push_back(make_uint2(uint32_t(kind[i]) | dst << 8 | aa << 16, y));
  }
  p.nregs = next;
  return p;
}

void ProgramAir::set_preprocessed(int n_pre, const uint32_t* values, int log_n) {
  if (n_pre < 0 || n_pre >= W) throw std::invalid_argument("AIR program: 0 <= preprocessed columns < columns");
  if (n_pre > 0 && !values) throw std::invalid_argument("AIR program: preprocessed columns missing");
  const size_t n = size_t(n_pre) << log_n;
  P = n_pre;
  pre_log_n = log_n;
  pre.resize(n);
  for (size_t i = 0; i < n; i++) {
    if (values[i] >= kb::P) throw std::invalid_argument("AIR program: preprocessed value not below p");
    pre[i] = kb::to_mont(values[i]);
  }
}

kb::ef ProgramAir::eval_ef(const kb::ef* up, const kb::ef* down, const kb::ef* alphas) const {
  const size_t n = ops.size() / 3;
  std::vector<kb::ef> v(n);
  kb::ef acc = kb::ef_zero();
  int ci = 0;
  for (size_t i = 0; i < n; i++) {
    const int op = ops[3 * i], a = ops[3 * i + 1], b = ops[3 * i + 2];
    switch (op) {
      case PROG_UP: v[i] = up[a]; break;
      case PROG_DOWN: v[i] = down[a]; break;
      case PROG_CONST: v[i] = kb::ef_zero(), v[i].c[0] = consts[a]; break;
      case PROG_ADD: v[i] = kb::ef_add(v[a], v[b]); break;
      case PROG_SUB: v[i] = kb::ef_sub(v[a], v[b]); break;
      case PROG_MUL: v[i] = kb::ef_mul(v[a], v[b]); break;
      default:
        acc = kb::ef_add(acc, kb::ef_mul(alphas[ci++], v[a]));
        v[i] = v[a];
        break;
    }
  }
  return acc;
}

}  // namespace wl
