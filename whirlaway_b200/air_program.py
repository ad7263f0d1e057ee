"""AIRs as constraint programs, for the prover's generic-AIR path.

The reference proves any p3-air `Air` through `AirTable` (crates/air/src/table.rs:15-60): W
columns, constraints over the row's up and down values, a declared constraint degree. The
zerocheck sees every column twice (crates/air/src/utils.rs:140-160): its up version (row x, the
last row repeating the one before it) and its down version (row x + 1, the last row
repeating itself), so a transition constraint written over (local, next) must hold on every
up/down pair. The constraints are batched as sum_i alpha^i C_i in the order the AIR emits them.

Here an AIR is a constraint program: a list of SSA instructions, instruction i computing value
v_i from a column's up or down value, a constant, or the sum, difference or product of two
earlier values; EMIT marks a value as the next constraint. `AirBuilder` writes such programs
from Python expressions (shared subexpressions are emitted once).

    b = AirBuilder(2)
    x, y = b.up(0), b.up(1)
    b.assert_zero(b.down(0) - (x * x * x + y))
    b.assert_zero(b.down(1) - x)
    prog = b.build()                    # 2 columns, 2 constraints, degree 3

Constraint degrees 1 to 3 are supported. The first `preprocessed` columns of an AIR may be
preprocessed (AirTable::preprocessed_columns, crates/air/src/table.rs:19): fixed by the AIR,
given with the program when proving and verifying, part of the zerocheck but not committed.
"""
import numpy as np

P = 0x7F000001
OP_UP, OP_DOWN, OP_CONST, OP_ADD, OP_SUB, OP_MUL, OP_EMIT = range(7)


class Expr:
    """A value of a constraint program (an instruction index) with its degree in the columns."""

    __slots__ = ("b", "i", "deg")

    def __init__(self, builder, index, degree):
        self.b, self.i, self.deg = builder, index, degree

    def _other(self, o):
        if isinstance(o, Expr):
            if o.b is not self.b:
                raise ValueError("expressions of different builders")
            return o
        return self.b.const(int(o))

    def __add__(self, o):
        o = self._other(o)
        return self.b._op(OP_ADD, self, o, max(self.deg, o.deg))

    def __radd__(self, o):
        return self._other(o) + self

    def __sub__(self, o):
        o = self._other(o)
        return self.b._op(OP_SUB, self, o, max(self.deg, o.deg))

    def __rsub__(self, o):
        return self._other(o) - self

    def __mul__(self, o):
        o = self._other(o)
        return self.b._op(OP_MUL, self, o, self.deg + o.deg)

    def __rmul__(self, o):
        return self._other(o) * self

    def __neg__(self):
        return self.b.const(0) - self


class AirProgram:
    """W columns (the first n_preprocessed of them preprocessed), the constraint count, the
    degree, the instructions (int32 rows (op, a, b)) and the constants (canonical u32)."""

    def __init__(self, width, n_constraints, degree, ops, consts, n_preprocessed=0):
        self.width = int(width)
        self.n_constraints = int(n_constraints)
        self.degree = int(degree)
        self.n_preprocessed = int(n_preprocessed)
        if not 0 <= self.n_preprocessed < self.width:
            raise ValueError("0 <= preprocessed columns < columns")
        self.ops = np.ascontiguousarray(ops, dtype=np.int32).reshape(-1, 3)
        self.consts = np.ascontiguousarray(consts, dtype=np.uint32)
        if not 1 <= self.degree <= 3:
            raise ValueError("constraint degree must be 1, 2 or 3")

    def evaluate_rows(self, witness, log_n, preprocessed=None):
        """The constraint values of every up/down row pair of a column-major witness (after the
        preprocessed columns, if any; a host-side check for tests and examples; returns an
        (n_constraints, 2^log_n) array)."""
        n = 1 << log_n
        w = np.asarray(witness, dtype=np.uint64).reshape(-1, n)
        if self.n_preprocessed:
            w = np.concatenate([np.asarray(preprocessed, dtype=np.uint64).reshape(self.n_preprocessed, n), w])
        w = w.reshape(self.width, n)
        up = w.copy()
        up[:, n - 1] = w[:, n - 2]
        down = np.concatenate([w[:, 1:], w[:, n - 1:]], axis=1)
        vals, out = [], []
        for op, a, b in self.ops.tolist():
            if op == OP_UP:
                v = up[a]
            elif op == OP_DOWN:
                v = down[a]
            elif op == OP_CONST:
                v = np.full(n, int(self.consts[a]), dtype=np.uint64)
            elif op == OP_ADD:
                v = (vals[a] + vals[b]) % P
            elif op == OP_SUB:
                v = (vals[a] + P - vals[b]) % P
            elif op == OP_MUL:
                v = (vals[a] * vals[b]) % P
            else:
                v = vals[a]
                out.append(v)
            vals.append(v)
        return np.array(out, dtype=np.uint64)


class AirBuilder:
    """Writes a constraint program over `width` columns, the first `preprocessed` of them
    preprocessed."""

    def __init__(self, width, preprocessed=0):
        if width < 1:
            raise ValueError("an AIR needs at least one column")
        self.width = width
        self.preprocessed = preprocessed
        self.ops = []
        self.consts = []
        self._const_idx = {}
        self._memo = {}
        self.n_constraints = 0
        self.max_degree = 0

    def _emit(self, key, degree):
        if key[0] != OP_EMIT and key in self._memo:
            return self._memo[key]
        e = Expr(self, len(self.ops), degree)
        self.ops.append(key)
        if key[0] != OP_EMIT:
            self._memo[key] = e
        return e

    def _op(self, op, x, y, degree):
        return self._emit((op, x.i, y.i), degree)

    def up(self, c):
        """Column c at the current row."""
        if not 0 <= c < self.width:
            raise IndexError("column out of range")
        return self._emit((OP_UP, c, 0), 1)

    def down(self, c):
        """Column c at the next row."""
        if not 0 <= c < self.width:
            raise IndexError("column out of range")
        return self._emit((OP_DOWN, c, 0), 1)

    def const(self, v):
        """A field constant (any integer, reduced mod p)."""
        v = int(v) % P
        if v not in self._const_idx:
            self._const_idx[v] = len(self.consts)
            self.consts.append(v)
        return self._emit((OP_CONST, self._const_idx[v], 0), 0)

    def assert_zero(self, e):
        """The next constraint: e vanishes on every up/down row pair."""
        if not isinstance(e, Expr):
            e = self.const(e)
        self._emit((OP_EMIT, e.i, 0), e.deg)
        self.n_constraints += 1
        self.max_degree = max(self.max_degree, e.deg)

    def build(self, degree=None):
        """The program; degree defaults to the largest constraint degree (at least 1)."""
        if self.n_constraints == 0:
            raise ValueError("an AIR needs at least one constraint")
        d = max(1, self.max_degree) if degree is None else int(degree)
        if d < self.max_degree:
            raise ValueError("declared degree below a constraint's degree")
        return AirProgram(self.width, self.n_constraints, d, np.array(self.ops, dtype=np.int32).reshape(-1, 3),
                          np.array(self.consts, dtype=np.uint32), self.preprocessed)


def _poseidon2_diag16():
    inv = lambda k: pow(pow(2, k, P), P - 2, P)
    d = [-2, 1, 2, inv(1), 3, 4, -inv(1), -3, -4, inv(8), inv(3), inv(24), -inv(8), -inv(3), -inv(4), -inv(24)]
    return [x % P for x in d]


def poseidon2_air_program(air_constants):
    """The Poseidon2-KoalaBear width-16 AIR of the built-in path (165 columns, 148 degree-3
    constraints, same column layout and constraint order) as a constraint program, from its
    148 round constants (canonical; 4 x 16 beginning, 20 partial, 4 x 16 ending). Proofs of
    this program equal the built-in path's proofs bit for bit."""
    c = [int(x) for x in np.asarray(air_constants, dtype=np.uint32)[:148]]
    begin = [c[16 * r:16 * r + 16] for r in range(4)]
    partial = c[64:84]
    end = [c[84 + 16 * r:84 + 16 * r + 16] for r in range(4)]
    diag = _poseidon2_diag16()
    b = AirBuilder(165)
    m4 = [[2, 3, 1, 1], [1, 2, 3, 1], [1, 1, 2, 3], [3, 1, 1, 2]]

    def mds(s):
        y = []
        for ch in range(4):
            x = s[4 * ch:4 * ch + 4]
            for i in range(4):
                acc = None
                for j in range(4):
                    t = x[j] * m4[i][j] if m4[i][j] != 1 else x[j]
                    acc = t if acc is None else acc + t
                y.append(acc)
        sums = []
        for i in range(4):
            sums.append(y[i] + y[4 + i] + y[8 + i] + y[12 + i])
        return [y[i] + sums[i % 4] for i in range(16)]

    s = [b.up(1 + i) for i in range(16)]
    col = 17
    s = mds(s)
    for rcs in begin:
        s = [(s[i] + rcs[i]) * (s[i] + rcs[i]) * (s[i] + rcs[i]) for i in range(16)]
        s = mds(s)
        for i in range(16):
            b.assert_zero(s[i] - b.up(col))
            s[i] = b.up(col)
            col += 1
    for r in range(20):
        x = s[0] + partial[r]
        s[0] = x * x * x
        b.assert_zero(s[0] - b.up(col))
        s[0] = b.up(col)
        col += 1
        tot = s[0]
        for i in range(1, 16):
            tot = tot + s[i]
        s = [s[i] * diag[i] + tot for i in range(16)]
    for rcs in end:
        s = [(s[i] + rcs[i]) * (s[i] + rcs[i]) * (s[i] + rcs[i]) for i in range(16)]
        s = mds(s)
        for i in range(16):
            b.assert_zero(s[i] - b.up(col))
            s[i] = b.up(col)
            col += 1
    return b.build(3)
