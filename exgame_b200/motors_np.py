"""Host-side motor algebra in numpy, for building scenario poses without the CUDA library.

A restatement of the few PGA3 = Cl(3,0,1) operations the synthetic workloads need, vectorised
over arrays of motors and twists:

  twist_exp_n(t, dt)    Twist::exp(dt) = Motor::exp(t dt / 2) by the Study-number closed form
                        (crates/clifford/src/pga3/screw.rs:297-301, pga3/motor.rs:199-217);
  compose_n(a, b)       "first a, then b" = b * a (pga3/motor.rs:157-159);
  apply_point_n(m, p)   the world position of the local point p under m (joints/src/lib.rs:258-263).

Conventions are the reference's (crates/clifford/src/algebra/mod.rs:84-140, algebra/markup.rs:13-100):
e1, e2, e3 on bits 0..2 and the degenerate e0 on bit 3; a blade is a bitmask, and the product
sign is the parity of the merge permutation times the metric (e0 e0 = 0). A motor's eight slots are
the even blades by increasing bitmask; a twist (linear xyz, angular xyz) is written on the radical
blades e0 e_i and on the dual (complement) of e_i times the angular embedding sign. The tables below
are evaluated from those laws at import time.
"""
import numpy as np

ZERO_MASK = 0b1000
I3 = 0b0111
TOP = 15
EVEN = [b for b in range(16) if bin(b).count("1") % 2 == 0]  # 0,3,5,6,9,10,12,15


def _popc(x):
    return bin(x).count("1")


def blade_prod(a, b):
    """(sign, mask) of the product of blades a and b; sign 0 when e0 meets e0."""
    if (a & b) & ZERO_MASK:
        return 0, 0
    swaps = 0
    aa = a >> 1
    while aa:
        swaps += _popc(aa & b)
        aa >>= 1
    return (-1 if swaps & 1 else 1), a ^ b


def _complement_sign(a, b):
    inv = 0
    for bi in range(4):
        if (a >> bi) & 1:
            inv += _popc(b & ((1 << bi) - 1))
    return -1 if inv & 1 else 1


def _axis(i):
    return 1 << i  # e1, e2, e3 are the low bits of I3 in order


def _euclid(i):
    v = _axis(i)
    c = I3 ^ v
    return c, _complement_sign(v, c)


def _radical(i):
    s, m = blade_prod(ZERO_MASK, _axis(i))
    return m, s


def _point(i):
    m, s = _euclid(i)
    ps, pm = blade_prod(ZERO_MASK, m)
    return pm, s * ps


def _angular_sigma():
    ws, _ = blade_prod(_axis(2), _axis(0))
    _, e1s = _euclid(1)
    bm, bs = _euclid(2)
    pm, ps = _point(0)
    _, ds = _point(1)
    hs = (blade_prod(bm, pm)[0] - blade_prod(pm, bm)[0]) // 2
    return e1s * ws * ds * hs * bs * ps


SIGMA = _angular_sigma()
RADICAL = [_radical(i) for i in range(3)]
ANGULAR = [(_euclid(i)[0], _euclid(i)[1] * SIGMA) for i in range(3)]
POINT = [_point(i) for i in range(3)]
# full 16 x 16 product table
SIGN = np.zeros((16, 16))
MASK = np.zeros((16, 16), dtype=np.int64)
for _a in range(16):
    for _b in range(16):
        SIGN[_a, _b], MASK[_a, _b] = blade_prod(_a, _b)


def gp(a, b):
    """Geometric product of (n, 16) multivector arrays, term by term in blade order."""
    out = np.zeros(np.broadcast_shapes(a.shape, b.shape))
    for i in range(16):
        ai = a[..., i]
        if not np.any(ai):
            continue
        for j in range(16):
            s = SIGN[i, j]
            if s == 0.0:
                continue
            out[..., MASK[i, j]] += s * (ai * b[..., j])
    return out


def reverse(a):
    g = np.array([_popc(b) for b in range(16)])
    sign = np.where((g * (g - 1) // 2) % 2 == 1, -1.0, 1.0)
    return a * sign


def motor_to_mv(m):
    out = np.zeros(m.shape[:-1] + (16,))
    out[..., EVEN] = m
    return out


def mv_to_motor(x):
    return np.ascontiguousarray(x[..., EVEN])


def twist_to_mv(t):
    out = np.zeros(t.shape[:-1] + (16,))
    for i in range(3):
        m, s = RADICAL[i]
        out[..., m] += s * t[..., i]
        m, s = ANGULAR[i]
        out[..., m] += s * t[..., 3 + i]
    return out


def _study(u):
    """cos(sqrt u), sin(sqrt u)/sqrt u and its u-derivative, with the Taylor arms near u = 0
    (crates/peano/src/scalar.rs:67-131; thresholds 1e-9 and 1e-9 / 1e-5)."""
    u = np.asarray(u, dtype=np.float64)
    small = np.abs(u) < 1e-9
    small_d = np.abs(u * 1e-5) < 1e-9
    l = np.sqrt(np.where(small, 1.0, u))
    ld = np.sqrt(np.where(small_d, 1.0, u))
    cu = np.where(small, 1.0 - u * (0.5 - u * (1.0 / 24.0 - u * (1.0 / 720.0))), np.cos(l))
    su = np.where(small, 1.0 - u * (1.0 / 6.0 - u * (1.0 / 120.0 - u * (1.0 / 5040.0))), np.sin(l) / l)
    du = np.where(small_d, -1.0 / 6.0 + u * (1.0 / 60.0 - u * (1.0 / 1680.0 - u * (1.0 / 90720.0))),
                  (ld * np.cos(ld) - np.sin(ld)) / (2.0 * ld * ld * ld))
    return cu, su, du


def exp_biv(b):
    """Motor::exp of (n, 16) bivector multivectors (motor.rs:199-217)."""
    b2 = gp(b, b)
    u = -b2[..., 0]
    p = b2[..., TOP]
    cu, su, du = _study(u)
    i_mv = np.zeros(16)
    i_mv[TOP] = 1.0
    ib = gp(np.broadcast_to(i_mv, b.shape), b)
    out = b * su[..., None] - ib * (p * du)[..., None]
    out[..., 0] += cu
    out[..., TOP] += p * 0.5 * su
    return out


def twist_exp_n(twists, dt=1.0):
    """out[k] = Twist::exp(twists[k], dt): (n, 6) -> (n, 8)."""
    t = np.asarray(twists, dtype=np.float64).reshape(-1, 6)
    return mv_to_motor(exp_biv(twist_to_mv(t * (dt * 0.5))))


def compose_n(a, b):
    """out[k] = "first a[k], then b[k]" = b[k] * a[k]: (n, 8) x (n, 8) -> (n, 8)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 8)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 8)
    return mv_to_motor(gp(motor_to_mv(b), motor_to_mv(a)))


def apply_point_n(m, p):
    """World coordinates of local points p (n, 3) under motors m (n, 8): M p M~ read through the
    point markup (weight on e123)."""
    m = np.asarray(m, dtype=np.float64).reshape(-1, 8)
    p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    x = np.zeros((len(m), 16))
    x[:, I3] = 1.0  # the weight blade e123 (mv.rs:582-593)
    for i in range(3):
        mask, s = POINT[i]
        x[:, mask] += s * p[:, i]
    mv = motor_to_mv(m)
    y = gp(gp(mv, x), reverse(mv))
    w = y[:, I3]
    out = np.zeros((len(m), 3))
    for i in range(3):
        mask, s = POINT[i]
        out[:, i] = s * y[:, mask] / w
    return out
