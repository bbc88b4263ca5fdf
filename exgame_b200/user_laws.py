"""Joint force laws written once against the scalar-generic algebra (pga_sym) and compiled to the
device by viete: each is traced at build time into csrc/user_laws.cuh and gets the law id
4 + its index here (exg_law_lookup finds it by name, with its parameter count). A law receives a
LawContext (parameters, the two poses, the two world twists, dt, warp) and returns the wrench on
body a; the wrench on body b is its negation, as for every law (JointImpl::wrench,
crates/joints/src/lib.rs:217-253). Energy reports count no potential for these laws.

To add a law: write `def my_law(c): ...` with the operations of pga_sym and viete (select on a
comparison instead of `if`), append ("MyLaw", n_params, my_law) to LAWS and rebuild.
"""
from . import pga_sym as G
from . import viete as V


def traced_spring_damper(c):
    """The axial SimpleSpringDamper (crates/joints/src/axial_spring_damper/mod.rs:315-385, force
    k (d - L0) + c d' of :46-58), written against the generic algebra: parameters
    [a0..a2, b0..b2, rest, k, c, softening] in the reference's flatten order."""
    p = c.params
    pa = G.anchor_point(c.pose_a, p[0:3])
    pb = G.anchor_point(c.pose_b, p[3:6])
    line = G.join(pa, pb)
    d = G.soft_weight_norm(line, p[9], V.sqrt)
    inv_d = 1.0 / d
    unit = G.wrench_from_line(line).scale(inv_d)
    d_dot = G.power(unit, c.twist_a - c.twist_b)
    f = p[7] * (d - p[6]) + p[8] * d_dot
    return unit.scale(-f)


def point_bushing(c):
    """A point-to-point bushing (a ball joint's compliance): the anchors pa = M_a a and pb = M_b b
    are pulled together by a linear spring of zero rest length and damped by their relative
    velocity, F = -k (pa - pb) - (c / warp^2) (v_a(pa) - v_b(pb)), acting on body a at pa:
    the wrench (F, pa x F). Parameters [a0..a2, b0..b2, k, c]."""
    p = c.params
    ha = G.anchor_point(c.pose_a, p[0:3])
    hb = G.anchor_point(c.pose_b, p[3:6])
    wa, wb = 1.0 / ha.c[G.I3], 1.0 / hb.c[G.I3]
    xa, xb = G.point_coords(ha, wa), G.point_coords(hb, wb)
    va, vb = G.velocity_at(c.twist_a, ha), G.velocity_at(c.twist_b, hb)
    damping = p[7] / (c.warp * c.warp)
    F = [-(p[6] * (xa[i] - xb[i])) - damping * (va[i] - vb[i]) for i in range(3)]
    tq = [xa[1] * F[2] - xa[2] * F[1], xa[2] * F[0] - xa[0] * F[2], xa[0] * F[1] - xa[1] * F[0]]
    return G.screw(F, tq)


LAWS = [
    ("TracedSpringDamper", 10, traced_spring_damper),
    ("PointBushing", 8, point_bushing),
]
