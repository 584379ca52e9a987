// fw_adjoint.cuh -- reverse-mode (adjoint) substep for the differentiable form.
//
// Forward substep of a node (no damping, gravity / nodal-force BCs):
//   v' = v + dt * f(x) / m        f = contact(x) + sum_e f_e(x; E_e) + const
//   x' = x + dt * v'
// Reverse, given the adjoints (xb', vb') of (x', v'):
//   vt = vb' + dt * xb'           total adjoint of v'
//   fb = (dt / m) * vt            adjoint of the node force
//   xb = xb' + sum_e J_e^T fb_e + C^T fb      vb = vt
// J2 triangles (whose return map is not an energy gradient) carry the adjoint
// of their plastic state sb and take the transpose of their local Jacobian
// (corner forces and new state against corner positions, old state and
// Young's modulus) column by column in dual numbers.
// Elastic and NeoHookean element forces are gradients of a strain energy
// (f_e = -A * B^T S = -d(A Psi)/dx with S = dPsi/dE, femspringmanager.py:240-280),
// so J_e is symmetric and J_e^T fb_e = J_e fb_e: a directional derivative,
// computed here in forward mode with dual numbers.  The force is linear in
// the element's Young's modulus (lambda, mu are), so df_e/dE_e = f_e / E_e.
// Contact (mixedcontact.py:660-684, 1566-1643) contributes, while the node
// penetrates, dF/dx = -k n g^T (g = n for a plane or a voxel face, the
// gradient of the signed distance to the interpolated curve for a height
// field) and, for height fields and voxel grids while the normal velocity is
// negative, the damping term dF/dv = -(k dt / 2) n n^T, which also feeds the
// velocity adjoint.  The broad-phase gate, the contact branch, the curve's
// sample and normal indices and the voxel face are piecewise constant and are
// replayed from the recorded forward pass.  Nodes with a fixed / enforced
// velocity pass no adjoint to their force or previous velocity.
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
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const float r = sqrtf(a.v);
  return Dual{r, r > 0.f ? a.d / (2.f * r) : 0.f};
}

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

// Corner forces and new plastic state of a J2 triangle in dual numbers (the
// radial return of pk2_stress, misesReturnMap2D in materialfunctions.py:35-101,
// then the corner forces of element_forces): X = corner positions (a.x, a.y,
// b.x, b.y, c.x, c.y), S = plastic state (eps_p Voigt, eqps), lam / mu carry
// the Young's-modulus direction.  The yield branch follows the value part.
__device__ __forceinline__ void element_j2_dual(const Dual X[6], float4 ji, Dual lam, Dual mu, float sy, float H,
                                                const Dual S[4], float area, Dual F[6], Dual SN[4]) {
  const Dual j00 = X[0] - X[4], j01 = X[2] - X[4];
  const Dual j10 = X[1] - X[5], j11 = X[3] - X[5];
  const Dual F00 = j00 * dmk(ji.x) + j01 * dmk(ji.z);
  const Dual F01 = j00 * dmk(ji.y) + j01 * dmk(ji.w);
  const Dual F10 = j10 * dmk(ji.x) + j11 * dmk(ji.z);
  const Dual F11 = j10 * dmk(ji.y) + j11 * dmk(ji.w);
  const float d00 = ji.x, d01 = ji.y, d10 = ji.z, d11 = ji.w;
  const float d20 = -ji.x - ji.z, d21 = -ji.y - ji.w;
  const Dual C00 = F00 * F00 + F10 * F10;
  const Dual C01 = F00 * F01 + F10 * F11;
  const Dual C11 = F01 * F01 + F11 * F11;
  const Dual e00 = 0.5f * (C00 - dmk(1.f)), e01 = 0.5f * C01, e11 = 0.5f * (C11 - dmk(1.f));
  const Dual t0 = e00 - S[0], t1 = e11 - S[1], t2 = e01 - S[2];
  const Dual tr = t0 + t1;
  const Dual tm = 2.f * mu;
  Dual s0 = lam * tr + tm * t0;
  Dual s1 = lam * tr + tm * t1;
  Dual s2 = tm * t2;
  const Dual p = (s0 + s1) / dmk(3.f);
  const Dual q0 = s0 - p, q1 = s1 - p, q2 = s2;
  const Dual vm = dsqrt(q0 * q0 + q1 * q1 - q0 * q1 + 3.f * (q2 * q2));
  const Dual f = vm - (dmk(sy) + H * S[3]);
  for (int k = 0; k < 4; ++k) SN[k] = S[k];
  if (f.v > 0.0f) {
    const Dual dg = f / (3.f * mu + dmk(H));
    SN[3] = S[3] + dg;
    const Dual scale = dmk(1.f) - (3.f * mu) * dg / vm;
    s0 = q0 * scale + p;
    s1 = q1 * scale + p;
    s2 = q2 * scale;
    SN[0] = S[0] + dg * (q0 / vm);
    SN[1] = S[1] + dg * (q1 / vm);
    SN[2] = S[2] + dg * (q2 / vm);
  }
  const Dual r0 = (d00 * F00) * s0 + (d01 * F01) * s1 + (d01 * F00 + d00 * F01) * s2;
  const Dual r1 = (d00 * F10) * s0 + (d01 * F11) * s1 + (d00 * F11 + d01 * F10) * s2;
  const Dual r2 = (d10 * F00) * s0 + (d11 * F01) * s1 + (d11 * F00 + d10 * F01) * s2;
  const Dual r3 = (d10 * F10) * s0 + (d11 * F11) * s1 + (d10 * F11 + d11 * F10) * s2;
  const Dual r4 = (d20 * F00) * s0 + (d21 * F01) * s1 + (d21 * F00 + d20 * F01) * s2;
  const Dual r5 = (d20 * F10) * s0 + (d21 * F11) * s1 + (d20 * F11 + d21 * F10) * s2;
  F[0] = -(area * r0);
  F[1] = -(area * r1);
  F[2] = -(area * r2);
  F[3] = -(area * r3);
  F[4] = -(area * r4);
  F[5] = -(area * r5);
}

// Linearisation of one pair's contact force at (x, v), the same branches as
// contact_force: false when the node is outside (no force); else the normal
// n, the gradient g of the penetration term (dF/dx = -k n g^T) and whether
// the damping term is on (dF/dv = -(k dt / 2) n n^T).
__device__ __forceinline__ bool contact_lin(const Pair& p, const float* __restrict__ heights,
                                            const int8_t* __restrict__ occ, float2 x, float2 v, float2& n,
                                            float2& g, bool& damped) {
  damped = false;
  if (p.kind == PAIR_PLANE) {
    const float pen = (x.x - p.f[0]) * p.f[2] + (x.y - p.f[1]) * p.f[3];
    if (!(pen < 0.0f)) return false;
    n = make_float2(p.f[2], p.f[3]);
    g = n;
    return true;
  }
  if (p.kind == PAIR_HEIGHTFIELD) {
    const float* h = heights + p.table;
    const int nx = p.n0;
    const float lbx = p.f[0], ubx = p.f[1];
    const float span = ubx - lbx;
    float u = 0.0f;
    bool inside = false;
    if (span > 1e-12f) {
      u = (x.x - lbx) / span;
      inside = u > 0.0f && u < 1.0f;
    }
    u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
    const float s = u * (float)(nx - 1);
    int i0 = (int)floorf(s);
    int i1 = i0 + 1;
    if (i1 >= nx) i1 = nx - 1;
    if (i0 < 0) i0 = 0;
    const float t = s - (float)i0;
    const float hh = h[i0] + (h[i1] - h[i0]) * t;
    int ir = (int)roundf(s);
    ir = ir < 0 ? 0 : (ir >= nx ? nx - 1 : ir);
    int k0 = ir - 1, k1 = ir + 1;
    if (k0 < 0) k0 = 0;
    if (k1 >= nx) k1 = nx - 1;
    const float dxw = span / (float)(nx - 1);
    const float denom = dxw * (float)(k1 - k0);
    float dhdx = 0.0f;
    if (denom > 1e-6f) dhdx = (h[k1] - h[k0]) / denom;
    float n0 = -dhdx, n1 = 1.0f;
    if (p.n1 == 1) {
      n0 = -n0;
      n1 = -n1;
    }
    const float nl = sqrtf(n0 * n0 + n1 * n1);
    if (nl > 1e-12f) {
      n0 = n0 / nl;
      n1 = n1 / nl;
    }
    const float sd = (x.x - x.x) * n0 + (x.y - hh) * n1;
    if (!(sd < 0.0f)) return false;
    // d hh / dx along the interpolated segment (zero where u is clamped)
    const float slope = inside ? (h[i1] - h[i0]) * ((float)(nx - 1) / span) : 0.0f;
    n = make_float2(n0, n1);
    g = make_float2(-slope * n1, n1);
    damped = v.x * n0 + v.y * n1 < 0.0f;
    return true;
  }
  const int8_t* gr = occ + p.table;
  const int nx = p.n0, ny = p.n1;
  const float lbx = p.f[0], lby = p.f[1], dx = p.f[2], dz = p.f[3];
  const int i = (int)floorf((x.x - lbx) / dx);
  const int j = (int)floorf((x.y - lby) / dz);
  if (!(0 <= i && i < nx && 0 <= j && j < ny)) return false;
  if (gr[i * ny + j] != 1) return false;
  float dnx = 1e9f, dpx = 1e9f, dny = 1e9f, dpy = 1e9f;
  for (int st = 0; st < nx; ++st) {
    const int idx = i - 1 - st;
    if (idx < 0 || gr[idx * ny + j] == 0) {
      dnx = x.x - (lbx + (float)(idx + 1) * dx);
      break;
    }
  }
  for (int st = 0; st < nx; ++st) {
    const int idx = i + 1 + st;
    if (idx >= nx || gr[idx * ny + j] == 0) {
      dpx = (lbx + (float)idx * dx) - x.x;
      break;
    }
  }
  for (int st = 0; st < ny; ++st) {
    const int idx = j - 1 - st;
    if (idx < 0 || gr[i * ny + idx] == 0) {
      dny = x.y - (lby + (float)(idx + 1) * dz);
      break;
    }
  }
  for (int st = 0; st < ny; ++st) {
    const int idx = j + 1 + st;
    if (idx >= ny || gr[i * ny + idx] == 0) {
      dpy = (lby + (float)idx * dz) - x.y;
      break;
    }
  }
  float mv = dnx, sd;
  int face = 0;
  if (dpx < mv) { mv = dpx; face = 1; }
  if (dny < mv) { mv = dny; face = 2; }
  if (dpy < mv) { mv = dpy; face = 3; }
  if (face == 0) { sd = -dnx; n = make_float2(-1.0f, 0.0f); }
  else if (face == 1) { sd = -dpx; n = make_float2(1.0f, 0.0f); }
  else if (face == 2) { sd = -dny; n = make_float2(0.0f, -1.0f); }
  else { sd = -dpy; n = make_float2(0.0f, 1.0f); }
  if (!(sd < 0.0f)) return false;
  g = n;
  damped = v.x * n.x + v.y * n.y < 0.0f;
  return true;
}

// Adjoint of one pair's contact force: xb += (dF/dx)^T fb, vb += (dF/dv)^T fb.
__device__ __forceinline__ void contact_vjp(const Pair& p, const float* __restrict__ heights,
                                            const int8_t* __restrict__ occ, float2 x, float2 v, float dt,
                                            double2 fb, double2& xb, double2& vb) {
  float2 n, g;
  bool damped;
  if (!contact_lin(p, heights, occ, x, v, n, g, damped)) return;
  const double nf = (double)n.x * fb.x + (double)n.y * fb.y;
  const double t = -(double)p.penalty * nf;
  xb.x += t * g.x;
  xb.y += t * g.y;
  if (damped) {
    const double td = -0.5 * (double)p.penalty * (double)dt * nf;
    vb.x += td * n.x;
    vb.y += td * n.y;
  }
}

// Tangent of one pair's contact force along (dx, dv).
__device__ __forceinline__ void contact_jvp(const Pair& p, const float* __restrict__ heights,
                                            const int8_t* __restrict__ occ, float2 x, float2 v, float dt,
                                            double2 dx, double2 dv, double& fx, double& fy) {
  float2 n, g;
  bool damped;
  if (!contact_lin(p, heights, occ, x, v, n, g, damped)) return;
  double s = -(double)p.penalty * ((double)g.x * dx.x + (double)g.y * dx.y);
  if (damped) s += -0.5 * (double)p.penalty * (double)dt * ((double)n.x * dv.x + (double)n.y * dv.y);
  fx += s * n.x;
  fy += s * n.y;
}

}  // namespace fw
