// Test harness: compiles the device algebra and force-law headers of the CUDA path for the
// host so the CPU test suite can compare them with the oracle without a GPU.
#include "../../exgame_b200/csrc/joint_eval.cuh"
// body.cuh names CUDA's double4 (a device vector type); the host build gets a plain stand-in
struct double4 { double x, y, z, w; };
#include "../../exgame_b200/csrc/body.cuh"

extern "C" {
void dh_joint_plain(int law, const double* prm, const double* pa, const double* pb, const double* va, const double* vb,
                    double dt, double warp, double* out12) {
  exg::joint_plain<double>(law, prm, pa, pb, va, vb, dt, warp, out12);
}
void dh_joint_plain_f32(int law, const double* prm, const float* pa, const float* pb, const float* va, const float* vb,
                        double dt, double warp, float* out12) {
  exg::joint_plain<float>(law, prm, pa, pb, va, vb, dt, warp, out12);
}
// full 12 x 25 block from the four slices
void dh_joint_jacobian(int law, const double* prm, const double* pa, const double* pb, const double* va, const double* vb,
                       double dt, double warp, double* out300) {
  for (int s = 0; s < 4; ++s) {
    double v[6], d[36];
    exg::joint_jacobian_slice<double>(law, prm, pa, pb, va, vb, dt, warp, s, v, d);
    for (int r = 0; r < 6; ++r) {
      out300[r * 25] = v[r];
      out300[(6 + r) * 25] = -v[r];
      for (int c = 0; c < 6; ++c) {
        out300[r * 25 + 1 + 6 * s + c] = d[r * 6 + c];
        out300[(6 + r) * 25 + 1 + 6 * s + c] = -d[r * 6 + c];
      }
    }
  }
}
void dh_twist_exp(const double* t6, double dt, double* m8) { double b[6]; exg::screw_from6(t6, b); exg::twist_exp(b, dt, m8); }
void dh_motor_compose(const double* a, const double* b, double* o) { exg::motor_compose(a, b, o); }
void dh_apply_point(const double* m8, const double* p3, double* o3) { double p[4]; exg::anchor_point(m8, p3, p); exg::point_coords(p, o3); }
void dh_transport(const double* t6, const double* m8, int co, double* o6) {
  double b[6], r[6]; exg::screw_from6(t6, b);
  if (co) exg::wrench_transport(b, m8, r); else exg::twist_transport(b, m8, r);
  exg::screw_to6(r, o6);
}
double dh_power(const double* w6, const double* t6) { double w[6], t[6]; exg::screw_from6(w6, w); exg::screw_from6(t6, t); return exg::screw_power(w, t); }
void dh_coad(const double* w6, const double* t6, double* o6) {
  double w[6], t[6], r[6]; exg::screw_from6(w6, w); exg::screw_from6(t6, t); exg::coad_bracket(w, t, r); exg::screw_to6(r, o6);
}
void dh_rotation_part(const double* m8, double* o8) { exg::motor_rotation_part(m8, o8); }
// full 12 x 25 block from eight half slices (3 axes each), FP64 and FP32
void dh_joint_jacobian_halves(int law, const double* prm, const double* pa, const double* pb, const double* va,
                              const double* vb, double dt, double warp, double* out300) {
  for (int s = 0; s < 4; ++s) {
    double v[6], d[36];
    for (int h = 0; h < 2; ++h) exg::joint_jacobian_part<double, 3>(law, prm, pa, pb, va, vb, dt, warp, s, h, v, d);
    for (int r = 0; r < 6; ++r) {
      out300[r * 25] = v[r];
      out300[(6 + r) * 25] = -v[r];
      for (int c = 0; c < 6; ++c) {
        out300[r * 25 + 1 + 6 * s + c] = d[r * 6 + c];
        out300[(6 + r) * 25 + 1 + 6 * s + c] = -d[r * 6 + c];
      }
    }
  }
}
void dh_jacobian_slices_f32(int law, const double* prm, const float* pa, const float* pb, const float* va,
                            const float* vb, double dt, double warp, int halves, float* out168) {
  for (int s = 0; s < 4; ++s) {
    float* o = out168 + 42 * s;
    if (halves) {
      for (int h = 0; h < 2; ++h) exg::joint_jacobian_part<float, 3>(law, prm, pa, pb, va, vb, dt, warp, s, h, o, o + 6);
    } else {
      exg::joint_jacobian_part<float, 6>(law, prm, pa, pb, va, vb, dt, warp, s, 0, o, o + 6);
    }
  }
}
// One first-order dual-number operation of the device scalar carrier (exg::Dual<1, double>) on
// a = (av, ad) and b = (bv, bd): out = (value, derivative).
void dh_dual1(int op, double av, double ad, double bv, double bd, double* out2) {
  using D = exg::Dual<1, double>;
  D a, b, r;
  a.v = av; a.g[0] = ad;
  b.v = bv; b.g[0] = bd;
  switch (op) {
    case 0: r = a + b; break;
    case 1: r = a - b; break;
    case 2: r = a * b; break;
    case 3: r = a / b; break;
    case 4: r = a.recip(); break;
    case 5: r = exg::s_sqrt(a); break;
    case 6: r = exg::s_sin(a); break;
    case 7: r = exg::s_cos(a); break;
    case 8: r = exg::s_atan2(a, b); break;
    case 9: r = exg::s_exp(a); break;
    case 10: r = exg::s_log(a); break;
    case 11: r = exg::s_abs(a); break;
    case 12: r = a * b + a / b; break;
    case 13: r = exg::s_sin(a * a); break;
    case 14: r = exg::s_exp(exg::s_log(a)); break;
    default: out2[0] = out2[1] = 0.0; return;
  }
  out2[0] = r.v;
  out2[1] = r.g[0];
}
// The Study forms of the device's exp (sin(sqrt u)/sqrt u, cos(sqrt u), its u-derivative), each
// with its Taylor arm below the scalar's effective-zero threshold.
void dh_study_forms(double u, double* out3) {
  out3[0] = exg::sinc_sq(u); out3[1] = exg::cos_sq(u); out3[2] = exg::dsinc_sq(u);
}
void dh_study_forms_f32(float u, float* out3) {
  out3[0] = exg::sinc_sq(u); out3[1] = exg::cos_sq(u); out3[2] = exg::dsinc_sq(u);
}
// Body helpers: momentum <-> body twist through the inertia (diagonal, full tensor or kinematic),
// and the world twist of a body from its pose and momentum.
void dh_inertia(const double* I9, int diag, int kin, double mass, int inverse, const double* in6, double* out6) {
  if (inverse) exg::inertia_inverse<double>(I9, diag != 0, kin != 0, mass, in6, out6);
  else exg::inertia_apply<double>(I9, diag != 0, kin != 0, mass, in6, out6);
}
void dh_world_velocity(const double* pose8, const double* mom6, const double* I9, int diag, int kin, double mass,
                       double* out6) {
  exg::world_velocity(pose8, mom6, I9, diag != 0, kin != 0, mass, out6);
}
}
