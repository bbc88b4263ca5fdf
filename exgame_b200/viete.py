"""viete: trace scalar-generic joint force laws and emit them as CUDA C device functions.

The reference traces each law, written once against a generic scalar, into a flattened SSA
program and emits shader text from it (crates/viete/src/api.rs:23-197 Tracer / Trace, ir.rs:28-180
Instr / Term, glsl.rs:24-85 the GLSL emitter; crates/newton/build.rs maps the boundary). This
module does the same for the B200 path: a law is a Python function over `pga_sym` multivectors
whose coefficients are traced scalars (`Var`); running it records every scalar operation once,
and `emit_cuda` writes the live part of that program as a C++ function template

    template <class S, class P = S>
    EXG_HD void user_law_<k>(const double* prm, const P* ma, const P* mb, const S* ta, const S* tb,
                             double dt, double warp, S* wa)

over the device algebra's carriers (motors: eight even slots; twists and the wrench on body a:
six bivector coefficients in blade order), the same signature as the hand-written laws of
csrc/laws.cuh. It is instantiated like them with S = double (plain FP64), float (mixed) and
Dual<N, R> (the Jacobian slices), so a traced law gets its derivative blocks from the existing dual
evaluation and runs inside the hand-written kernels (joint kernels, the island kernel, the wave).

Every SSA value carries a kind: 0 when it depends on parameters, dt and warp only (emitted as
double), 1 when it depends on the poses but not the twists (type P: the twist slices run these
chains without partials), 2 when it depends on a twist (type S). An operation takes the largest
kind of its operands and lifts the others (P(x), S(x), Lift<S>::from(x)).

Operations (the reference's op set, ir.rs:28-79): + - * / neg, sqrt sin cos exp ln abs atan2,
powi (repeated products), select on a comparison (the comparison reads value parts), fma.
"""
import math
import os

from . import pga_sym as G


class Trace:
    def __init__(self):
        self.instrs = []  # (id, kind, op, args); args hold Var ids, float literals or input names

    def new(self, kind, op, args):
        v = Var(self, len(self.instrs), kind)
        self.instrs.append((v.id, kind, op, args))
        return v


class Var:
    __slots__ = ("tr", "id", "kind")

    def __init__(self, tr, id_, kind):
        self.tr, self.id, self.kind = tr, id_, kind

    # ── arithmetic ──
    def _bin(self, op, o, swap=False):
        if isinstance(o, (int, float)):
            o = float(o)
            # exact identities: x*1 = x, x*(-1) = -x, x+0 = x, x-0 = x, x/1 = x
            if op == "mul" and o == 1.0:
                return self
            if op == "mul" and o == -1.0:
                return -self
            if op in ("add", "sub") and o == 0.0 and not (op == "sub" and swap):
                return self
            if op == "div" and o == 1.0 and not swap:
                return self
            k = self.kind
        else:
            k = max(self.kind, o.kind)
            # a + (-b) = a - b and (-a) + b = b - a, as written by sign-law products
            if op == "add" and self.tr.instrs[o.id][2] == "neg":
                return self._bin("sub", self.tr.instrs[o.id][3][0], swap)
        args = (o, self) if swap else (self, o)
        return self.tr.new(k, op, args)

    def __add__(self, o):
        return self._bin("add", o)

    def __radd__(self, o):
        return self._bin("add", o, True)

    def __sub__(self, o):
        return self._bin("sub", o)

    def __rsub__(self, o):
        return self._bin("sub", o, True)

    def __mul__(self, o):
        return self._bin("mul", o)

    def __rmul__(self, o):
        return self._bin("mul", o, True)

    def __truediv__(self, o):
        return self._bin("div", o)

    def __rtruediv__(self, o):
        return self._bin("div", o, True)

    def __neg__(self):
        return self.tr.new(self.kind, "neg", (self,))

    def __bool__(self):
        raise TypeError("a traced value has no truth value: branch with viete.select on a comparison")

    # ── comparisons (on value parts) give a condition for select ──
    def _cmp(self, op, o):
        k = self.kind if isinstance(o, (int, float)) else max(self.kind, o.kind)
        return self.tr.new(k, op, (self, float(o) if isinstance(o, (int, float)) else o))

    def __lt__(self, o):
        return self._cmp("lt", o)

    def __le__(self, o):
        return self._cmp("le", o)

    def __gt__(self, o):
        return self._cmp("gt", o)

    def __ge__(self, o):
        return self._cmp("ge", o)


def _unary(op, x, fallback):
    if isinstance(x, (int, float)):
        return fallback(float(x))
    return x.tr.new(x.kind, op, (x,))


def sqrt(x):
    return _unary("sqrt", x, math.sqrt)


def sin(x):
    return _unary("sin", x, math.sin)


def cos(x):
    return _unary("cos", x, math.cos)


def exp(x):
    return _unary("exp", x, math.exp)


def ln(x):
    return _unary("ln", x, math.log)


def abs_(x):
    return _unary("abs", x, abs)


def atan2(y, x):
    if isinstance(y, (int, float)) and isinstance(x, (int, float)):
        return math.atan2(y, x)
    t = y.tr if isinstance(y, Var) else x.tr
    k = max(v.kind for v in (y, x) if isinstance(v, Var))
    return t.new(k, "atan2", (y, x))


def fma(a, b, c):
    return a * b + c


def powi(x, n):
    """x^n for an integer n >= 0 by repeated products (the reference lowers Powi the same way)."""
    if n == 0:
        return 1.0
    r = x
    for _ in range(n - 1):
        r = r * x
    return r


def select(cond, a, b):
    """a where the condition holds, else b."""
    t = cond.tr
    k = max([cond.kind] + [v.kind for v in (a, b) if isinstance(v, Var)])
    return t.new(k, "select", (cond, a, b))


class LawContext:
    """What a traced law reads: its parameters, the two poses and world twists, dt and warp."""

    def __init__(self, tr, n_params):
        self.tr = tr
        self.params = [tr.new(0, "in", ("prm", k)) for k in range(n_params)]
        self.dt = tr.new(0, "in", ("dt", 0))
        self.warp = tr.new(0, "in", ("warp", 0))
        self.pose_a = G.motor([tr.new(1, "in", ("ma", k)) for k in range(8)])
        self.pose_b = G.motor([tr.new(1, "in", ("mb", k)) for k in range(8)])
        self.twist_a = G.bivector([tr.new(2, "in", ("ta", k)) for k in range(6)])
        self.twist_b = G.bivector([tr.new(2, "in", ("tb", k)) for k in range(6)])


class TracedLaw:
    def __init__(self, name, n_params, fn):
        self.name, self.n_params, self.fn = name, n_params, fn
        self.tr = Trace()
        ctx = LawContext(self.tr, n_params)
        w = fn(ctx)
        self.out = G.bivector_coeffs(w.grade2())

    def live(self):
        """Ids of the instructions the outputs depend on."""
        need = set()
        stack = [o.id for o in self.out if isinstance(o, Var)]
        while stack:
            i = stack.pop()
            if i in need:
                continue
            need.add(i)
            for a in self.tr.instrs[i][3]:
                if isinstance(a, Var):
                    stack.append(a.id)
        return need

    def counts(self):
        """Live instructions per operation (the analogue of the reference's per-law op counts)."""
        out = {}
        for i in sorted(self.live()):
            op = self.tr.instrs[i][2]
            if op != "in":
                out[op] = out.get(op, 0) + 1
        return out


_TYPES = {0: "double", 1: "P", 2: "S"}


def _lit(x, kind):
    r = repr(float(x))
    if r in ("inf", "-inf", "nan"):
        raise ValueError("non-finite literal in a traced law")
    return f"{_TYPES[kind]}({r})"


def _ref(a, kind):
    """Operand a in an expression of the given kind."""
    if not isinstance(a, Var):
        return _lit(a, kind)
    name = f"t{a.id}"
    if a.kind == kind:
        return name
    if kind == 2 and a.kind == 1:
        return f"Lift<S>::from({name})"
    return f"{_TYPES[kind]}({name})"


def _value(a):
    """The value part of an operand, for comparisons."""
    if not isinstance(a, Var):
        return repr(float(a))
    return f"t{a.id}" if a.kind == 0 else f"double(std_part(t{a.id}))"


_FUN = {"sqrt": "s_sqrt", "sin": "s_sin", "cos": "s_cos", "exp": "s_exp", "ln": "s_log", "abs": "s_abs",
        "atan2": "s_atan2"}
_DFUN = {"sqrt": "sqrt", "sin": "sin", "cos": "cos", "exp": "exp", "ln": "log", "abs": "fabs", "atan2": "atan2"}
_BIN = {"add": "+", "sub": "-", "mul": "*", "div": "/"}
_CMP = {"lt": "<", "le": "<=", "gt": ">", "ge": ">="}


def emit_cuda(law, index):
    """The law as a C++ function template over the device carriers (see the module docstring)."""
    live = law.live()
    lines = [f"// {law.name}: {law.n_params} parameters; traced ops {law.counts()}",
             "template <class S, class P = S>",
             f"EXG_HD void user_law_{index}(const double* prm, const P* ma, const P* mb, const S* ta, const S* tb, "
             "double dt, double warp, S* wa) {",
             "  (void)prm; (void)ma; (void)mb; (void)ta; (void)tb; (void)dt; (void)warp;"]
    for (i, kind, op, args) in law.tr.instrs:
        if i not in live:
            continue
        ty = "bool" if op in _CMP else _TYPES[kind]
        if op == "in":
            src, k = args
            expr = {"prm": f"prm[{k}]", "dt": "dt", "warp": "warp", "ma": f"ma[{k}]", "mb": f"mb[{k}]",
                    "ta": f"ta[{k}]", "tb": f"tb[{k}]"}[src]
        elif op in _BIN:
            expr = f"{_ref(args[0], kind)} {_BIN[op]} {_ref(args[1], kind)}"
        elif op == "neg":
            expr = f"-{_ref(args[0], kind)}"
        elif op in _CMP:
            expr = f"{_value(args[0])} {_CMP[op]} {_value(args[1])}"
        elif op == "select":
            expr = f"t{args[0].id} ? {_ref(args[1], kind)} : {_ref(args[2], kind)}"
        elif op in _FUN:
            fn = _DFUN[op] if kind == 0 else _FUN[op]
            expr = f"{fn}({', '.join(_ref(a, kind) for a in args)})"
        else:
            raise ValueError(f"op {op}")
        lines.append(f"  const {ty} t{i} = {expr};")
    for k, o in enumerate(law.out):
        lines.append(f"  wa[{k}] = {_ref(o, 2) if isinstance(o, Var) else _lit(o, 2)};")
    lines.append("}")
    return "\n".join(lines)


HEADER_NOTE = """// GENERATED by exgame_b200/viete.py from the laws registered in exgame_b200/user_laws.py;
// regenerated by every build (exgame_b200/build.py). Traced joint force laws as device functions
// over the device algebra's carriers, dispatched by law id >= kUserLawFirst from laws.cuh.
"""


def emit_header(laws):
    parts = [HEADER_NOTE, "#pragma once", '#include "geom.cuh"', "", "namespace exg {", "",
             "constexpr int kUserLawFirst = 4;", f"constexpr int kUserLaws = {len(laws)};", ""]
    for k, law in enumerate(laws):
        parts.append(emit_cuda(law, k))
        parts.append("")
    parts.append("template <class S, class P = S>")
    parts.append("EXG_HD void user_law_wrench(int idx, const double* prm, const P* ma, const P* mb, const S* ta, "
                 "const S* tb, double dt, double warp, S* wa) {")
    if laws:
        parts.append("  switch (idx) {")
        for k in range(len(laws)):
            parts.append(f"    case {k}: user_law_{k}<S, P>(prm, ma, mb, ta, tb, dt, warp, wa); return;")
        parts.append("    default: break;")
        parts.append("  }")
    parts.append("  for (int i = 0; i < 6; ++i) wa[i] = S(0.0);")
    parts.append("}")
    parts.append("")
    parts.append("struct UserLawInfo { const char* name; int n_params; };")
    table = ", ".join(f'{{"{law.name}", {law.n_params}}}' for law in laws) or '{"", 0}'
    parts.append(f"static const UserLawInfo kUserLawTable[] = {{{table}}};")
    parts.append("")
    parts.append("}  // namespace exg")
    return "\n".join(parts) + "\n"


def generate(path=None):
    """Trace every registered law and write the header (only when its text changes, so the
    build's timestamps stay put)."""
    from . import user_laws
    laws = [TracedLaw(name, n, fn) for name, n, fn in user_laws.LAWS]
    text = emit_header(laws)
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "user_laws.cuh")
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)
    return path, laws


if __name__ == "__main__":
    p, laws = generate()
    for law in laws:
        print(law.name, law.n_params, law.counts())
    print("wrote", p)
