// fw_adjoint.cuh -- reverse-mode (adjoint) substep for the differentiable form.
//
// Forward substep of a node (no damping, gravity / nodal-force BCs):
//   v' = v + dt * f(x) / m        f = contact(x) + sum_e f_e(x; E_e) + const
//   x' = x + dt * v'
// Reverse, given the adjoints (xb', vb') of (x', v'):
//   vt = vb' + dt * xb'           total adjoint of v'
//   fb = (dt / m) * vt            adjoint of the node force
//   xb = xb' + sum_e J_e^T fb_e + C^T fb      vb = vt
// Elastic and NeoHookean element forces are gradients of a strain energy
// (f_e = -A * B^T S = -d(A Psi)/dx with S = dPsi/dE, femspringmanager.py:240-280),
// so J_e is symmetric and J_e^T fb_e = J_e fb_e: a directional derivative,
// computed here in forward mode with dual numbers.  The force is linear in
// the element's Young's modulus (lambda, mu are), so df_e/dE_e = f_e / E_e.
// Plane contact (mixedcontact.py:660-684) contributes -k n n^T while the node
// penetrates; the broad-phase gate is piecewise constant and is replayed from
// the recorded forward pass.  Nodes with a fixed / enforced velocity pass no
// adjoint to their force or previous velocity.
#pragma once

namespace fw {

struct Dual {
  float v, d;
};
__device__ __forceinline__ Dual dmk(float v, float d = 0.f) { return Dual{v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual{-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(float a, Dual b) { return Dual{a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const float q = a.v / b.v;
  return Dual{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dlog(Dual a) { return Dual{fw_log(a.v), a.d / a.v}; }

// Corner forces of one triangle and their directional derivative along the
// node displacements (wa, wb, wc); Elastic and NeoHookean laws.
__device__ __forceinline__ void element_forces_jvp(float2 a, float2 b, float2 c, float2 wa, float2 wb,
                                                   float2 wc, float4 ji, int type, float lam, float mu,
                                                   float area, Dual out[6]) {
  const Dual j00 = dmk(a.x - c.x, wa.x - wc.x), j01 = dmk(b.x - c.x, wb.x - wc.x);
  const Dual j10 = dmk(a.y - c.y, wa.y - wc.y), j11 = dmk(b.y - c.y, wb.y - wc.y);
  const Dual F00 = j00 * dmk(ji.x) + j01 * dmk(ji.z);
  const Dual F01 = j00 * dmk(ji.y) + j01 * dmk(ji.w);
  const Dual F10 = j10 * dmk(ji.x) + j11 * dmk(ji.z);
  const Dual F11 = j10 * dmk(ji.y) + j11 * dmk(ji.w);
  const float d00 = ji.x, d01 = ji.y, d10 = ji.z, d11 = ji.w;
  const float d20 = -ji.x - ji.z, d21 = -ji.y - ji.w;
  const Dual C00 = F00 * F00 + F10 * F10;
  const Dual C01 = F00 * F01 + F10 * F11;
  const Dual C11 = F01 * F01 + F11 * F11;
  Dual s0, s1, s2;
  if (type == MAT_NEOHOOKEAN) {
    const Dual cdet = C00 * C11 - C01 * C01;
    const Dual i00 = C11 / cdet, i01 = -(C01 / cdet), i11 = C00 / cdet;
    const Dual J = F00 * F11 - F01 * F10;
    const Dual cc = lam * dlog(J) - dmk(mu);
    s0 = cc * i00 + dmk(mu);
    s1 = cc * i11 + dmk(mu);
    s2 = cc * i01;
  } else {  // Elastic (St-Venant-Kirchhoff on Green-Lagrange strain)
    const Dual e00 = 0.5f * (C00 - dmk(1.f)), e01 = 0.5f * C01, e11 = 0.5f * (C11 - dmk(1.f));
    const Dual lt = lam * (e00 + e11);
    s0 = lt + (2.f * mu) * e00;
    s1 = lt + (2.f * mu) * e11;
    s2 = (2.f * mu) * e01;
  }
  const Dual r0 = (d00 * F00) * s0 + (d01 * F01) * s1 + (d01 * F00 + d00 * F01) * s2;
  const Dual r1 = (d00 * F10) * s0 + (d01 * F11) * s1 + (d00 * F11 + d01 * F10) * s2;
  const Dual r2 = (d10 * F00) * s0 + (d11 * F01) * s1 + (d11 * F00 + d10 * F01) * s2;
  const Dual r3 = (d10 * F10) * s0 + (d11 * F11) * s1 + (d10 * F11 + d11 * F10) * s2;
  const Dual r4 = (d20 * F00) * s0 + (d21 * F01) * s1 + (d21 * F00 + d20 * F01) * s2;
  const Dual r5 = (d20 * F10) * s0 + (d21 * F11) * s1 + (d20 * F11 + d21 * F10) * s2;
  out[0] = -(area * r0);
  out[1] = -(area * r1);
  out[2] = -(area * r2);
  out[3] = -(area * r3);
  out[4] = -(area * r4);
  out[5] = -(area * r5);
}

}  // namespace fw
