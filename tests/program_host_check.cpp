// Host check of the constraint-program compiler (whirlaway_b200/csrc/air_program.cu): the
// device code it emits (register assignment, constants as immediates in MULC / ADDC, constant
// instructions dropped when only read as immediates) is run by a host restatement of the
// interpreter kernels' dispatch, over the base field and over the extension, and compared with
// the program evaluated instruction by instruction (ProgramAir::eval_ef, which reads the
// instructions as given). Random programs with constants in every operand position, plus
// programs that exceed the register file. Built and run by tests/test_air_program.py.
#include <vector_types.h>
#include <vector_functions.h>

#include <cstdio>
#include <random>

#include "air_program.cu"

using namespace kb;
using wl::ProgramAir;

// The dispatch of k_prog_zc_ef for one row: values up[c], down[c] in place of the folded columns.
static ef run_ef(const ProgramAir& p, const ef* up, const ef* down, const ef* alphas) {
  ef reg[wl::PROG_MAX_REGS];
  ef acc = ef_zero();
  int ci = 0;
  for (const uint2 in : p.code) {
    const int op = int(in.x & 0xffu), dst = int((in.x >> 8) & 0xffu);
    const uint32_t a = in.x >> 16, b = in.y;
    switch (op) {
      case wl::PROG_UP: reg[dst] = up[a]; break;
      case wl::PROG_DOWN: reg[dst] = down[a]; break;
      case wl::PROG_CONST: reg[dst] = ef_zero(), reg[dst].c[0] = p.consts[a]; break;
      case wl::PROG_ADD: reg[dst] = ef_add(reg[a], reg[b]); break;
      case wl::PROG_SUB: reg[dst] = ef_sub(reg[a], reg[b]); break;
      case wl::PROG_MUL: reg[dst] = ef_mul(reg[a], reg[b]); break;
      case wl::PROG_MULC: reg[dst] = ef_mul_f(reg[a], b); break;
      case wl::PROG_ADDC: {
        ef v = reg[a];
        v.c[0] = add(v.c[0], b);
        reg[dst] = v;
        break;
      }
      default: acc = ef_add(acc, ef_mul(alphas[ci++], reg[a])); break;
    }
  }
  return acc;
}

// The dispatch of k_prog_zc0 for one row over the base field (the constraints' alpha-sum).
static ef run_base(const ProgramAir& p, const uint32_t* up, const uint32_t* down, const ef* alphas) {
  uint32_t reg[wl::PROG_MAX_REGS];
  ef acc = ef_zero();
  int ci = 0;
  for (const uint2 in : p.code) {
    const int op = int(in.x & 0xffu), dst = int((in.x >> 8) & 0xffu);
    const uint32_t a = in.x >> 16, b = in.y;
    switch (op) {
      case wl::PROG_UP: reg[dst] = up[a]; break;
      case wl::PROG_DOWN: reg[dst] = down[a]; break;
      case wl::PROG_CONST: reg[dst] = p.consts[a]; break;
      case wl::PROG_ADD: reg[dst] = add(reg[a], reg[b]); break;
      case wl::PROG_SUB: reg[dst] = sub(reg[a], reg[b]); break;
      case wl::PROG_MUL: reg[dst] = mul(reg[a], reg[b]); break;
      case wl::PROG_MULC: reg[dst] = mul(reg[a], b); break;
      case wl::PROG_ADDC: reg[dst] = add(reg[a], b); break;
      default: acc = ef_add(acc, ef_mul_f(alphas[ci++], reg[a])); break;
    }
  }
  return acc;
}

int main() {
  std::mt19937_64 g(5);
  auto rnd = [&](uint64_t n) { return int(g() % n); };
  long bad = 0, programs = 0, immediates = 0, dropped = 0, rejected = 0;
  for (int t = 0; t < 3000; t++) {
    const int W = 1 + rnd(6), NK = 1 + rnd(4), n_body = 4 + rnd(60), NC = 1 + rnd(4);
    std::vector<uint32_t> consts(NK);
    for (auto& c : consts) c = (t % 5 == 0) ? uint32_t(rnd(3)) : uint32_t(g() % P);  // 0, 1, 2 as well
    std::vector<int32_t> ops;
    int n = 0;
    auto push = [&](int op, int a, int b) { ops.push_back(op), ops.push_back(a), ops.push_back(b), n++; };
    for (int i = 0; i < n_body; i++) {
      const int r = rnd(10);
      if (n < 2 || r == 0) push(wl::PROG_UP, rnd(W), 0);
      else if (r == 1) push(wl::PROG_DOWN, rnd(W), 0);
      else if (r == 2) push(wl::PROG_CONST, rnd(NK), 0);
      else push(wl::PROG_ADD + rnd(3), rnd(n), rnd(n));
    }
    for (int e = 0; e < NC; e++) push(wl::PROG_EMIT, rnd(n), 0);
    ProgramAir p;
    try {
      p = ProgramAir::build(W, NC, 3, n, ops.data(), NK, consts.data());
    } catch (const std::invalid_argument&) {
      rejected++;  // register file exceeded (long random programs): the compiler says so
      continue;
    }
    programs++;
    for (const uint2 in : p.code) immediates += (in.x & 0xffu) >= wl::PROG_MULC;
    dropped += n - long(p.code.size());
    for (int rep = 0; rep < 4; rep++) {
      std::vector<ef> up(W), down(W), al(NC);
      std::vector<uint32_t> ub(W), db(W);
      for (int c = 0; c < W; c++) {
        ub[c] = to_mont(uint32_t(g() % P)), db[c] = to_mont(uint32_t(g() % P));
        up[c] = ef_zero(), down[c] = ef_zero();
        for (int j = 0; j < 8; j++) up[c].c[j] = to_mont(uint32_t(g() % P)), down[c].c[j] = to_mont(uint32_t(g() % P));
      }
      for (auto& a : al)
        for (int j = 0; j < 8; j++) a.c[j] = to_mont(uint32_t(g() % P));
      if (!ef_eq(run_ef(p, up.data(), down.data(), al.data()), p.eval_ef(up.data(), down.data(), al.data()))) bad++;
      std::vector<ef> ue(W), de(W);
      for (int c = 0; c < W; c++) ue[c] = ef_zero(), de[c] = ef_zero(), ue[c].c[0] = ub[c], de[c].c[0] = db[c];
      if (!ef_eq(run_base(p, ub.data(), db.data(), al.data()), p.eval_ef(ue.data(), de.data(), al.data()))) bad++;
    }
  }
  printf("programs %ld (rejected %ld), immediates %ld, dropped constants %ld, mismatches %ld\n", programs, rejected,
         immediates, dropped, bad);
  return (bad || programs < 1000 || immediates < 1000 || dropped < 100) ? 1 : 0;
}
