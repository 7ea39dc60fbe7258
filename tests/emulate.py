"""Host-side emulators used to verify the bytecode compiler without a GPU.

Both evaluate with the same numpy float32 operator implementations, so they
must agree bit for bit whatever the platform's libm does: `run_prefix` is the
reference evaluation order (right-to-left token stack, reference
cl_cpu_eval.cpp:59-90), `run_bytecode` executes the compiled program
(accumulator + spill slots, operands folded in) as the device does.
"""
import numpy as np

F = np.float32
DELTA = F(1e-9)


def _loose(d):
    return np.where(np.abs(d) <= DELTA, np.where(d < 0, -DELTA, DELTA), d).astype(F)


def np_op(op, a, b):
    with np.errstate(all="ignore"):
        if op == 0:
            return a
        if op == 1:
            return (a + b).astype(F)
        if op == 2:
            return (a - b).astype(F)
        if op == 3:
            return (a * b).astype(F)
        if op == 4:
            return np.where(b == 0, F(np.nan), a / np.where(b == 0, F(1), b)).astype(F)
        if op == 5:
            return np.power(a, b).astype(F)
        if op == 6:
            return np.fmin(a, b).astype(F)
        if op == 7:
            return np.fmax(a, b).astype(F)
        if op == 8:
            return (a / _loose(b)).astype(F)
        if op == 9:
            return np.where((a == 0) & (b == 0), F(0), np.power(np.abs(a), b)).astype(F)
        table = {10: np.sin, 11: np.cos, 12: np.tan, 13: np.sinh, 14: np.cosh, 15: np.tanh,
                 16: np.exp, 17: np.log, 19: np.arcsin, 20: np.arccos, 21: np.arctan,
                 24: np.abs, 25: np.negative, 26: np.sqrt}
        if op in table:
            return table[op](a).astype(F)
        if op == 18:
            return (F(1) / a).astype(F)
        if op == 22:
            return np.where(a == 0, F(-1e9), np.log(np.abs(a))).astype(F)
        if op == 23:
            return (F(1) / _loose(a)).astype(F)
        if op == 27:
            return np.sqrt(np.abs(a)).astype(F)
        if op == 32:
            return np.exp(np.fmin(a, F(80))).astype(F)
    return np.zeros_like(a)


def run_prefix(tokens, values, X, V):
    N = X.shape[1]
    stack = []
    for tk, vl in zip(reversed(list(tokens)), reversed(list(values))):
        tk = int(tk)
        if tk == 0:
            stack.append(np.full(N, F(vl), F))
        elif tk == -1:
            vi = int(vl) if -2**31 < vl < 2**31 else -1
            stack.append(X[vi].astype(F) if 0 <= vi < V else np.zeros(N, F))
        else:
            a = stack.pop()
            b = stack.pop() if 1 <= tk <= 9 else np.zeros(N, F)
            stack.append(np_op(tk, a, b))
    return stack[0]


def _bin(op, a, b):
    """Device opcode semantics: 1..9 -> f(a, b); 40+k -> f_k(b, a)."""
    if op > 40:
        return np_op(op - 40, b, a)
    return np_op(op, a, b)


def run_bytecode(code, X, V, n_slots=16):
    """Execute compiled instructions [spill] [T = leaf] [b = operand] T = op(T, b)."""
    N = X.shape[1]
    T = np.zeros(N, F)
    S = [np.zeros(N, F) for _ in range(n_slots)]

    def const(bits):
        return np.full(N, np.array([bits], np.uint32).view(F)[0], F)

    def var(row):
        assert 0 <= int(row) < V
        return X[int(row)].astype(F)

    for w, a, b, _c in code:
        w = int(w)
        op = w & 63
        if w & (1 << 12):
            S[(w >> 13) & 31] = T.copy()
        if w & (1 << 6):
            lk = (w >> 7) & 3
            assert lk in (0, 1), "cached-subtree leaves need a cache"
            T = var(a) if lk == 0 else const(a)
        bk = (w >> 9) & 7
        if bk == 0:
            assert op == 0 or op >= 10, f"binary opcode {op} without operand"
            T = np_op(op, T, np.zeros(N, F))
        else:
            vb = {1: lambda: S[int(b)], 2: lambda: var(b), 3: lambda: const(b)}[bk]()
            assert 1 <= op <= 9 or 41 <= op <= 49, f"unary opcode {op} with operand"
            T = _bin(op, T, vb)
    return T
