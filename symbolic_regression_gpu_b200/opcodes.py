"""Token encoding of prefix expressions (reference src/utils/opcodes.h:10-40).

Token 0 is a constant (its value is the constant), -1 a variable (its value is
the variable index), 1..9 binary operators, 10..27 unary operators.  Token 32
(EXP_CLAMP) is an extension of this project with no reference counterpart:
exp with its argument clamped at 80.
"""

TOK_CONST = 0
TOK_VAR = -1

ADD, SUB, MUL, DIV, POW, MIN, MAX, LOOSE_DIV, LOOSE_POW = range(1, 10)
(SIN, COS, TAN, SINH, COSH, TANH, EXP, LOG, INV, ASIN, ACOS, ATAN, LOOSE_LOG,
 LOOSE_INV, ABS, NEG, SQRT, LOOSE_SQRT) = range(10, 28)
EXP_CLAMP = 32

BINARY_OPS = (ADD, SUB, MUL, DIV, POW, MIN, MAX, LOOSE_DIV, LOOSE_POW)
UNARY_OPS = (SIN, COS, TAN, SINH, COSH, TANH, EXP, LOG, INV, ASIN, ACOS, ATAN,
             LOOSE_LOG, LOOSE_INV, ABS, NEG, SQRT, LOOSE_SQRT, EXP_CLAMP)
REFERENCE_UNARY_OPS = UNARY_OPS[:-1]

# Operator set of the synthetic workloads: + - * protected-/ sin cos
# exp-clamped-at-80 protected-log|x| sqrt|x|.
WORKLOAD_BINARY = (ADD, SUB, MUL, LOOSE_DIV)
WORKLOAD_UNARY = (SIN, COS, EXP_CLAMP, LOOSE_LOG, LOOSE_SQRT)

NAMES = {
    ADD: "+", SUB: "-", MUL: "*", DIV: "/", POW: "**", MIN: "min", MAX: "max",
    LOOSE_DIV: "loose_div", LOOSE_POW: "loose_pow", SIN: "sin", COS: "cos",
    TAN: "tan", SINH: "sinh", COSH: "cosh", TANH: "tanh", EXP: "exp", LOG: "log",
    INV: "inv", ASIN: "asin", ACOS: "acos", ATAN: "atan", LOOSE_LOG: "loose_log",
    LOOSE_INV: "loose_inv", ABS: "abs", NEG: "-", SQRT: "sqrt",
    LOOSE_SQRT: "loose_sqrt", EXP_CLAMP: "exp_clamp80",
}


def arity(tok: int) -> int:
    """0 for leaves, 2 for 1..9, 1 otherwise (reference rule, detect.cpp:16-19)."""
    if tok <= 0:
        return 0
    return 2 if tok < 10 else 1


def format_formula(tokens, values) -> str:
    """Infix rendering of a prefix expression (reference format_formula,
    src/utils/utils.cpp:58-120): binary (a op b) with a the first popped."""
    stack = []
    for tok, val in zip(reversed(list(tokens)), reversed(list(values))):
        tok = int(tok)
        if tok == TOK_CONST:
            stack.append(f"{float(val):f}")
        elif tok == TOK_VAR:
            stack.append(f"x{int(val)}")
        elif 1 <= tok <= 9:
            if len(stack) < 2:
                return "INVALID"
            a = stack.pop()
            b = stack.pop()
            stack.append(f"({a} {NAMES[tok]} {b})")
        elif tok in NAMES:
            if not stack:
                return "INVALID"
            a = stack.pop()
            stack.append(f"(-{a})" if tok == NEG else f"{NAMES[tok]}({a})")
        else:
            return "UNKNOWN_TOKEN"
    return stack[0] if len(stack) == 1 else "INVALID"
