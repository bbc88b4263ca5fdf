"""PGA3 = Cl(3,0,1) multivectors over any scalar type, for writing joint force laws once and
tracing them (viete.py) or evaluating them with floats.

The reference writes its laws against a scalar-generic algebra (crates/clifford/src/pga3/*,
JointImpl::wrench<S: Scalar>, crates/joints/src/lib.rs:217-253) and traces them into shader code.
This module is the Python counterpart of that algebra: a multivector is sixteen coefficients in
blade-bitmask order (e1, e2, e3 on bits 0..2, the degenerate e0 on bit 3), products follow the
sign law of motors_np (evaluated from the same rules as the device algebra), and a coefficient
that is the literal 0.0 is skipped, so a traced product contains only the terms the carriers can
produce. The named operations restate the reference's facade:

  Motor slots / Screw markup      crates/clifford/src/pga3/motor.rs:119-147, screw.rs:278-333
  compose, reverse, Ad / coAd     motor.rs:157-159, screw.rs:94-105
  anchor point  M p M~            crates/joints/src/lib.rs:258-263
  join of points                  crates/clifford/src/pga3/objects.rs:42-45
  soft weight norm                objects.rs:120-122 (mv.rs:436-438)
  wrench of a line                screw.rs:337-339
  power <w ^ dual(t)>_I           screw.rs:355-361
  velocity of a twist at a point  screw.rs:310-314
"""
from . import motors_np as T

EVEN = T.EVEN
BIV = [3, 5, 6, 9, 10, 12]
I3 = T.I3
TOP = T.TOP


def _is_zero(x):
    return isinstance(x, float) and x == 0.0


def _grade(b):
    return bin(b).count("1")


class Mv:
    """Sixteen coefficients of any scalar type supporting + - * and unary -."""

    __slots__ = ("c",)

    def __init__(self, c=None):
        self.c = list(c) if c is not None else [0.0] * 16

    def __add__(self, o):
        return Mv([_add(a, b) for a, b in zip(self.c, o.c)])

    def __sub__(self, o):
        return Mv([_sub(a, b) for a, b in zip(self.c, o.c)])

    def __neg__(self):
        return Mv([_neg(a) for a in self.c])

    def scale(self, k):
        return Mv([0.0 if _is_zero(a) else a * k for a in self.c])

    def gp(self, o):
        out = [0.0] * 16
        for i in range(16):
            a = self.c[i]
            if _is_zero(a):
                continue
            for j in range(16):
                b = o.c[j]
                s = T.SIGN[i, j]
                if s == 0.0 or _is_zero(b):
                    continue
                term = a * b
                m = int(T.MASK[i, j])
                out[m] = _add(out[m], term) if s > 0 else _sub(out[m], term)
        return Mv(out)

    def reverse(self):
        return Mv([a if (_grade(b) * (_grade(b) - 1) // 2) % 2 == 0 else _neg(a) for b, a in enumerate(self.c)])

    def dual(self):
        out = [0.0] * 16
        for b, a in enumerate(self.c):
            if _is_zero(a):
                continue
            comp = TOP ^ b
            out[comp] = _add(out[comp], a if T._complement_sign(b, comp) > 0 else _neg(a))
        return Mv(out)

    def undual(self):
        out = [0.0] * 16
        for b, a in enumerate(self.c):
            if _is_zero(a):
                continue
            comp = TOP ^ b
            out[comp] = _add(out[comp], a if T._complement_sign(comp, b) > 0 else _neg(a))
        return Mv(out)

    def wedge(self, o):
        """Outer product: the blade pairs with disjoint masks."""
        out = [0.0] * 16
        for i in range(16):
            a = self.c[i]
            if _is_zero(a):
                continue
            for j in range(16):
                b = o.c[j]
                if (i & j) or _is_zero(b):
                    continue
                s = T.SIGN[i, j]
                term = a * b
                out[i ^ j] = _add(out[i ^ j], term) if s > 0 else _sub(out[i ^ j], term)
        return Mv(out)

    def meet(self, o):
        return self.dual().wedge(o.dual()).undual()

    def conjugate(self, x):
        """self x self~ (the sandwich)."""
        return self.gp(x).gp(self.reverse())

    def grade2(self):
        return Mv([a if _grade(b) == 2 else 0.0 for b, a in enumerate(self.c)])

    def norm_squared(self):
        """The weight norm^2 of a line (mv.rs:428-434): the Euclidean bivector part squared."""
        acc = 0.0
        for b in (3, 5, 6):
            a = self.c[b]
            if not _is_zero(a):
                acc = _add(acc, a * a)
        return acc


def _add(a, b):
    if _is_zero(a):
        return b
    if _is_zero(b):
        return a
    return a + b


def _neg(a):
    return 0.0 if _is_zero(a) else -a


def _sub(a, b):
    if _is_zero(b):
        return a
    if _is_zero(a):
        return _neg(b)
    return a - b


# ── markups and named objects ───────────────────────────────────────────────
def write_dual(mv, v3, blades):
    for i in range(3):
        m, s = blades[i]
        mv.c[m] = _add(mv.c[m], v3[i] if s > 0 else _neg(v3[i]))
    return mv


def read_dual(mv, blades):
    out = []
    for i in range(3):
        m, s = blades[i]
        out.append(mv.c[m] if s > 0 else _neg(mv.c[m]))
    return out


def motor(slots):
    """A motor from its eight slots (even blades by increasing bitmask)."""
    mv = Mv()
    for k, b in enumerate(EVEN):
        mv.c[b] = slots[k]
    return mv


def motor_slots(mv):
    return [mv.c[b] for b in EVEN]


def screw(lin, ang):
    """A twist / wrench from its physical parts: linear on the radical blades, angular on the
    dual of the Euclidean axes times the angular embedding sign."""
    mv = Mv()
    write_dual(mv, lin, T.RADICAL)
    write_dual(mv, ang, T.ANGULAR)
    return mv


def screw_parts(mv):
    return read_dual(mv, T.RADICAL), read_dual(mv, T.ANGULAR)


def bivector(coeffs):
    """A screw from its six bivector coefficients in blade order (the device's BIV carrier)."""
    mv = Mv()
    for k, b in enumerate(BIV):
        mv.c[b] = coeffs[k]
    return mv


def bivector_coeffs(mv):
    return [mv.c[b] for b in BIV]


def point(v3):
    mv = Mv()
    mv.c[I3] = 1.0
    return write_dual(mv, v3, T.POINT)


def point_coords(p, inv_weight):
    return [x * inv_weight for x in read_dual(p, T.POINT)]


def anchor_point(m, local3):
    return m.conjugate(point(local3))


def join(pa, pb):
    return pa.meet(pb)


def line_direction(line):
    return read_dual(line, [(T._euclid(i)[0], T._euclid(i)[1]) for i in range(3)])


def soft_weight_norm(line, eps, sqrt):
    return sqrt(_add(line.norm_squared(), eps * eps))


def wrench_from_line(line):
    return line.dual().grade2()


def power(wrench, twist):
    return wrench.wedge(twist.dual()).c[TOP]


def velocity_at(twist, p):
    comm = twist.gp(p) - p.gp(twist)
    return [x * 0.5 for x in read_dual(comm, T.POINT)]
