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


# ---- FP64 reverse mode over the compiled bytecode ---------------------------

def _op64(op, a, b):
    """Operator semantics in float64 (the FP64 oracle's sro_op_f64)."""
    with np.errstate(all="ignore"):
        if op == 0:
            return a
        if op in (8, 23):
            d = b if op == 8 else a
            eps = np.full_like(d, 1e-9)  # the operand's dtype
            d = np.where(np.abs(d) <= eps, np.where(d < 0, -eps, eps), d)
            return a / d if op == 8 else 1.0 / d
        f = {1: lambda: a + b, 2: lambda: a - b, 3: lambda: a * b,
             4: lambda: np.where(b == 0, np.nan, a / np.where(b == 0, 1.0, b)),
             5: lambda: np.power(a, b), 6: lambda: np.fmin(a, b), 7: lambda: np.fmax(a, b),
             9: lambda: np.where((a == 0) & (b == 0), 0.0, np.power(np.abs(a), b)),
             10: lambda: np.sin(a), 11: lambda: np.cos(a), 12: lambda: np.tan(a),
             13: lambda: np.sinh(a), 14: lambda: np.cosh(a), 15: lambda: np.tanh(a),
             16: lambda: np.exp(a), 17: lambda: np.log(a), 18: lambda: 1.0 / a,
             19: lambda: np.arcsin(a), 20: lambda: np.arccos(a), 21: lambda: np.arctan(a),
             22: lambda: np.where(a == 0, -1e9, np.log(np.abs(a))), 24: lambda: np.abs(a),
             25: lambda: -a, 26: lambda: np.sqrt(a), 27: lambda: np.sqrt(np.abs(a)),
             32: lambda: np.exp(np.fmin(a, 80.0))}[op]
        return f()


def _partials64(op, a, b, out):
    """(d out / d a, d out / d b) with the conventions of the device adjoint."""
    one, zero = np.ones_like(a), np.zeros_like(a)
    sg = np.sign
    with np.errstate(all="ignore"):
        if op == 0:
            return one, zero
        if op == 1:
            return one, one
        if op == 2:
            return one, -one
        if op == 3:
            return b, a
        if op == 4:  # the device forms 1/b once and reuses it
            r = 1.0 / b
            return r, -out * r
        if op == 5:
            return b * np.power(a, b - 1.0), out * np.log(a)
        if op in (6, 7):
            first = np.isnan(b) | (~np.isnan(a) & ((a <= b) if op == 6 else (a >= b)))
            return first.astype(np.float64), (~first).astype(np.float64)
        if op == 8:
            tiny = np.abs(b) <= 1e-9
            eps = np.full_like(b, 1e-9)  # the operand's dtype
            r = 1.0 / np.where(tiny, np.where(b < 0, -eps, eps), b)
            return r, np.where(tiny, 0.0, -out * r)
        if op == 9:
            z = (a == 0) & (b == 0)
            return (np.where(z, 0.0, b * np.power(np.abs(a), b - 1.0) * sg(a)),
                    np.where(z, 0.0, out * np.log(np.abs(a))))
        d = {10: lambda: np.cos(a), 11: lambda: -np.sin(a), 12: lambda: 1.0 + out * out,
             13: lambda: np.cosh(a), 14: lambda: np.sinh(a), 15: lambda: 1.0 - out * out,
             16: lambda: out, 17: lambda: 1.0 / a, 18: lambda: -out * out,
             19: lambda: 1.0 / np.sqrt(1.0 - a * a), 20: lambda: -1.0 / np.sqrt(1.0 - a * a),
             21: lambda: 1.0 / (1.0 + a * a), 22: lambda: np.where(a == 0, 0.0, 1.0 / a),
             23: lambda: np.where(np.abs(a) <= 1e-9, 0.0, -out * out), 24: lambda: sg(a),
             25: lambda: -one, 26: lambda: 0.5 / out,
             27: lambda: np.where(a == 0, 0.0, sg(a) * 0.5 / out),
             32: lambda: np.where(a < 80.0, out, 0.0)}[op]()
        return d, zero


def _strong(g, d):
    with np.errstate(all="ignore"):
        return np.where(g == 0, 0.0, g * d)


def adjoint_bytecode(code, X, V, n_const, n_slots=16, dtype=np.float64, with_abs=False):
    """MSE and d MSE / d constants of one compiled program, run the way the
    adjoint kernel runs it: a forward pass recording every instruction's
    output (the tape), then a backward pass in reverse instruction order with
    an adjoint accumulator and adjoint spill slots.  A spilled operand's value
    is read back from the tape at the producer index held in bits 20-29 of the
    instruction's c word; the forward pass asserts that it equals the value
    the spill slot holds.  Constants enter as their float32 bits widened.
    dtype=np.float64: the FP64 restatement.  dtype=np.float32: every value,
    partial and adjoint product rounded to float32 (the device's arithmetic,
    numpy's libm), constant gradients accumulated in float64.  with_abs adds
    the mean over valid datapoints of |adjoint reaching each constant|."""
    N = X.shape[1]
    D = dtype
    y = X[V].astype(D)
    S = [np.zeros(N, D) for _ in range(n_slots)]
    tape = []
    T = np.zeros(N, D)

    def leaf(kind, payload):
        if kind == 0:
            return X[int(payload)].astype(D)
        return np.full(N, D(np.array([payload], np.uint32).view(F)[0]))

    def operand(bk, payload):
        return {2: lambda: X[int(payload)].astype(D),
                3: lambda: np.full(N, D(np.array([payload], np.uint32).view(F)[0]))}[bk]()

    for i, (w, a, b, c) in enumerate(code):
        w, c = int(w), int(c)
        op, bk = w & 63, (w >> 9) & 7
        if w & (1 << 12):
            S[(w >> 13) & 31] = T.copy()
        if w & (1 << 6):
            T = leaf((w >> 7) & 3, a)
        if bk == 0:
            T = _op64(op, T, None)
        else:
            if bk == 1:
                vb = S[int(b)]
                prod = (c >> 20) & 0x3FF
                assert prod < i and np.array_equal(vb, tape[prod], equal_nan=True), \
                    f"instruction {i}: spilled operand is not the output of instruction {prod}"
            else:
                vb = operand(bk, b)
            T = _op64(op - 40, vb, T) if op > 40 else _op64(op, T, vb)
        T = np.asarray(T, D)
        tape.append(T.copy())
    with np.errstate(all="ignore"):
        valid = ~np.isnan(T) & ~np.isinf(T.astype(np.float32))
    cnt = int(valid.sum())
    d = np.where(valid, T - y, 0.0).astype(D)
    mse = (d.astype(np.float64) ** 2).sum() / cnt if cnt else np.nan
    grad = np.zeros(n_const, np.float64)
    gabs = np.zeros(n_const, np.float64)
    gT = (2.0 * d).astype(D)
    G = [np.zeros(N, D) for _ in range(n_slots)]
    for i in range(len(code) - 1, -1, -1):
        w, a, b, c = (int(q) for q in code[i])
        op, bk = w & 63, (w >> 9) & 7
        to = tape[i]
        ti = leaf((w >> 7) & 3, a) if w & (1 << 6) else tape[i - 1]
        if bk == 1:
            bv = tape[(c >> 20) & 0x3FF]
        elif bk:
            bv = operand(bk, b)
        else:
            bv = np.zeros(N, D)
        if bk == 0:
            dT, db = _partials64(op, ti, None, to)
        elif op > 40:
            db, dT = _partials64(op - 40, bv, ti, to)
        else:
            dT, db = _partials64(op, ti, bv, to)
        gi = _strong(gT, np.asarray(dT, D)).astype(D)
        gb = _strong(gT, np.asarray(db, D)).astype(D)
        if bk == 3:
            grad[(c >> 10) & 0x3FF] += gb.sum(dtype=np.float64)
            gabs[(c >> 10) & 0x3FF] += np.abs(gb).sum(dtype=np.float64)
        elif bk == 1:
            G[b] = gb
        if w & (1 << 6):
            if (w >> 7) & 3 == 1:
                grad[c & 0x3FF] += gi.sum(dtype=np.float64)
                gabs[c & 0x3FF] += np.abs(gi).sum(dtype=np.float64)
            gT = G[(w >> 13) & 31] if w & (1 << 12) else np.zeros(N, D)
        else:
            gT = gi
    g = grad / cnt if cnt else np.full(n_const, np.nan)
    if with_abs:
        return mse, g, (gabs / cnt if cnt else np.full(n_const, np.nan))
    return mse, g


# ---- FP32 forward mode (tangents) over the compiled bytecode ----------------

MAX_TANGENT_CONSTS = 8  # expressions with at most this many constants
TANGENT_DPT = 8         # datapoints per thread of the forward-mode kernel


def _lane_sums(p, D):
    """Sum of the products p (length N, rounded to D) the way the forward-mode
    kernel adds them: tiles of 32 lanes x TANGENT_DPT datapoints (element k of
    lane l of a tile is datapoint (k // 4) * 128 + 4 l + k % 4), each lane's
    values added in order in D, then float64 over lanes and tiles."""
    tile = 32 * TANGENT_DPT
    n = -(-p.size // tile) * tile
    q = np.zeros(n, D)
    q[:p.size] = p
    q = q.reshape(-1, TANGENT_DPT // 4, 32, 4).transpose(0, 2, 1, 3).reshape(-1, 32, TANGENT_DPT)
    with np.errstate(all="ignore"):
        g = q[..., 0].copy()
        for k in range(1, TANGENT_DPT):
            g = (g + q[..., k]).astype(D)
    return g.astype(np.float64).sum()


def _kill(d, t, D):
    """d == 0 ? 0 : d * t, rounded to D."""
    with np.errstate(all="ignore"):
        return np.where(d == 0, D(0), (np.asarray(d, D) * np.asarray(t, D)).astype(D)).astype(D)


def tangent_bytecode(code, X, V, n_const, n_slots=16, dtype=np.float32, with_abs=False):
    """MSE and d MSE / d constants of one compiled program, run the way the
    forward-mode kernel runs it: tangents t_c = d T / d constant c carried
    beside T; per instruction t_c = dT * t_c for the constants under the
    accumulator and t_c = db * t_c(b) for the constants under the operand (a
    zero partial gives zero, whatever the tangent); a constant leaf starts
    t_c = 1.  Only the constants under a value are carried with it, so a
    partial never multiplies a constant that is not below it.  Gradients are
    sum over valid datapoints of (seed == 0 ? 0 : seed * t_c), seed =
    2 (pred - y), the products added as the kernel adds them (_lane_sums)."""
    N = X.shape[1]
    D = dtype
    y = X[V].astype(D)
    S = [np.zeros(N, D) for _ in range(n_slots)]
    ST = [dict() for _ in range(n_slots)]
    T = np.zeros(N, D)
    t = {}

    def leaf(kind, payload):
        if kind == 0:
            return X[int(payload)].astype(D)
        return np.full(N, D(np.array([payload], np.uint32).view(F)[0]))

    for i, (w, a, b, c) in enumerate(code):
        w, c = int(w), int(c)
        op, bk = w & 63, (w >> 9) & 7
        if w & (1 << 12):
            S[(w >> 13) & 31] = T.copy()
            ST[(w >> 13) & 31] = {k: v.copy() for k, v in t.items()}
        if w & (1 << 6):
            lk = (w >> 7) & 3
            T = leaf(lk, a)
            ca = c & 0x3FF
            t = {ca: np.ones(N, D)} if (lk == 1 and ca != 0x3FF) else {}
        tb = {}
        if bk == 0:
            vb = np.zeros(N, D)
        elif bk == 1:
            vb = S[int(b)]
            tb = ST[int(b)]
        else:
            vb = leaf(0 if bk == 2 else 1, b)
            cb = (c >> 10) & 0x3FF
            if bk == 3 and cb != 0x3FF:
                tb = {cb: np.ones(N, D)}
        Tin = T
        if bk == 0:
            T = _op64(op, Tin, None)
            dT, db = _partials64(op, Tin, None, np.asarray(T, D))
        elif op > 40:
            T = _op64(op - 40, vb, Tin)
            db, dT = _partials64(op - 40, vb, Tin, np.asarray(T, D))
        else:
            T = _op64(op, Tin, vb)
            dT, db = _partials64(op, Tin, vb, np.asarray(T, D))
        T = np.asarray(T, D)
        new = {k: _kill(dT, v, D) for k, v in t.items()}
        new.update({k: _kill(db, v, D) for k, v in tb.items()})
        t = new
    with np.errstate(all="ignore"):
        valid = ~np.isnan(T) & ~np.isinf(T.astype(np.float32))
    cnt = int(valid.sum())
    d = np.where(valid, T - y, 0.0).astype(D)
    mse = (d.astype(np.float64) ** 2).sum() / cnt if cnt else np.nan
    seed = (2.0 * d).astype(D)
    grad = np.zeros(n_const, np.float64)
    gabs = np.zeros(n_const, np.float64)
    for k in range(n_const):
        g = _kill(seed, t[k], D)
        grad[k] = _lane_sums(g, D)
        gabs[k] = np.abs(g.astype(np.float64)).sum()
    g = grad / cnt if cnt else np.full(n_const, np.nan)
    if with_abs:
        return mse, g, (gabs / cnt if cnt else np.full(n_const, np.nan))
    return mse, g
