// AIRs beyond the built-in Poseidon2-KoalaBear one, given as constraint programs (the
// reference proves any p3-air Air through AirTable, crates/air/src/table.rs:15-60). A program
// is a list of SSA instructions over the up and down values of the W columns
// (crates/air/src/utils.rs:140-160); its EMITs, in order, are the constraints batched as
// sum_i alpha^i C_i. For the device the SSA values are assigned to a small register file
// (linear scan: a value's register is freed after its last use), so that the interpreter
// kernels keep PROG_MAX_REGS values per thread.
#pragma once
#include <vector_types.h>

#include <cstdint>
#include <vector>

#include "kb.cuh"

namespace wl {

enum ProgOp { PROG_UP = 0, PROG_DOWN = 1, PROG_CONST = 2, PROG_ADD = 3, PROG_SUB = 4, PROG_MUL = 5, PROG_EMIT = 6 };
// Device-only forms for an operand that is a constant (the constant's Montgomery value in y):
// value * c and value + c (x - c is value + (-c)). Over the extension they are a product and a
// sum by a base-field element, an eighth of the work of the general forms.
enum ProgDevOp { PROG_MULC = 7, PROG_ADDC = 8 };
constexpr int PROG_MAX_REGS = 64;

struct ProgramAir {
  int W = 0, NC = 0, degree = 0;
  int P = 0;                     // preprocessed columns: the first P of the W
  std::vector<int32_t> ops;      // (op, a, b) per instruction, as given
  std::vector<uint32_t> consts;  // Montgomery form
  std::vector<uint32_t> pre;     // the preprocessed columns, P x 2^log_n, Montgomery form
  int pre_log_n = -1;
  // Device form: x = op | dst << 8 | a << 16 (a: a column, a constant or a register), y = b (a
  // register, or for MULC / ADDC the constant's Montgomery value); EMIT's register is its
  // operand's. A constant read only as such an operand has no instruction and no register.
  std::vector<uint2> code;
  int nregs = 0;

  // Validates (columns and constants in range, operands earlier values, NC EMITs, degree
  // 1..3, at most PROG_MAX_REGS live values) and compiles; throws std::invalid_argument.
  // consts_canonical: the constants as canonical values.
  static ProgramAir build(int W, int n_constraints, int degree, int n_ops, const int32_t* ops, int n_consts,
                          const uint32_t* consts_canonical);
  // The first P columns are preprocessed (crates/air/src/table.rs:19,59-70): fixed by the AIR,
  // part of the zerocheck, not committed; values: P columns of 2^log_n canonical values.
  // Throws std::invalid_argument unless 0 <= P < W and every value is below p.
  void set_preprocessed(int n_pre, const uint32_t* values_canonical, int log_n);
  // Witness (committed) columns.
  int witness_columns() const { return W - P; }
  // sum_i alphas[i] C_i at a point of up values up[0..W) and down values down[0..W).
  kb::ef eval_ef(const kb::ef* up, const kb::ef* down, const kb::ef* alphas) const;
};

}  // namespace wl
