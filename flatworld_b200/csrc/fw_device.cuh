// fw_device.cuh -- per-element and per-node arithmetic of the explicit 2D FEM
// substep, shared by every kernel variant.
//
// The operation order follows the reference's Warp kernels term by term (the
// file is compiled with -fmad=false and IEEE division / square root), so the
// FP32 results match a serial FP32 evaluation of the reference source (with
// log() evaluated by fw_log below instead of the math library):
//   element force  flatworld/femspringmanager.py:217-280 (+ 59-105 helpers)
//   stress laws    flatworld/materials/materialfunctions.py:10-29, 35-101
//   contact        flatworld/mixedcontact.py:166-302, 660-684, 1566-1643
//   integration    flatworld/femspringmanager.py:315-358
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fw {

constexpr int BC_U = 0x1;
constexpr int BC_V = 0x2;
constexpr int BC_A = 0x4;
constexpr int BC_FORCE = 0x8;
constexpr int BC_GRAVITY = 0x10;
constexpr uint32_t NODE_BC_MASK = 0x1FFu;
constexpr uint32_t NODE_BOUNDARY = 0x200u;
constexpr int NODE_BODY_SHIFT = 10;

constexpr int MAT_SPRING = 0;  // a 2-node spring of a spring-mass domain (elemType 0 in the reference)
constexpr int MAT_ELASTIC = 1;
constexpr int MAT_NEOHOOKEAN = 2;
constexpr int MAT_MISES = 3;

constexpr int PAIR_PLANE = 0;
constexpr int PAIR_HEIGHTFIELD = 1;
constexpr int PAIR_VOXEL = 2;

// Scene modes seen by the node kernel for one step.
constexpr int MODE_STEP = 0;    // ordinary advance()
constexpr int MODE_INIT = 1;    // zero-dt construction step (no contact)
constexpr int MODE_FROZEN = 2;  // inactive scene: state untouched

// One contact pair (FEM body vs one ground), 64 bytes.
struct __align__(16) Pair {
  int kind, body;
  float penalty;
  int table;             // offset into the height / occupancy table
  int n0, n1;            // heightfield: samples, reverse.  voxel: nx, ny.
  float glo[2], ghi[2];  // ground getBBox() box (broad-phase gate)
  // plane: p.x, p.y, n.x, n.y.  heightfield: lb.x, ub.x.
  // voxel: lb.x, lb.y, dx, dz.
  float f[4];
  int gate;  // 0: the static box above gates the pair; e + 1: the current box of rigid entry e
  int pad;   // rigid pairs: 1 when the pair is tied
};
static_assert(sizeof(Pair) == 64, "Pair record is 64 bytes");

// Material record of one element: rest area, Lame constants, and a packed
// word (material type in bits 0-1, body id in bits 2-31).
struct __align__(16) ElemMat {
  float area, lam, mu;
  int word;
};

__device__ __forceinline__ int elem_type(int word) { return word & 3; }
__device__ __forceinline__ int elem_body(int word) { return (int)((unsigned)word >> 2); }

// Order-preserving map float -> int for atomicMin/atomicMax (exact).
__device__ __forceinline__ int f2ord(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

// Natural logarithm in float32 from IEEE-rounded + - * / only, so that the
// same operations in the same order give the same bits on any IEEE machine
// (the CPU oracle evaluates the identical method).  Method: Cody-Waite range
// reduction x = 2^e m, m in [sqrt(1/2), sqrt(2)), ln 2 split into a 12-bit-short
// head and a tail; ln m = 2 atanh(s) with s = (m-1)/(m+1) and the atanh series
// (Abramowitz & Stegun 4.1.27) through s^13.  Measured error < 2 ulp over all
// floats in [0.5, 2) and on a 1-in-97 sample of all positive floats.
__device__ __forceinline__ float fw_log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -__int_as_float(0x7F800000) : __int_as_float(0x7FC00000);
  if (x == __int_as_float(0x7F800000)) return x;
  uint32_t u = __float_as_uint(x);
  int e = 0;
  if (u < 0x00800000u) {  // subnormal: scale by 2^23
    x = x * 8388608.0f;
    u = __float_as_uint(x);
    e = -23;
  }
  e += (int)((u >> 23) & 0xFFu) - 127;
  float m = __uint_as_float((u & 0x007FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float z = s * s;
  float p = 1.0f / 13.0f;
  p = p * z + 1.0f / 11.0f;
  p = p * z + 1.0f / 9.0f;
  p = p * z + 1.0f / 7.0f;
  p = p * z + 1.0f / 5.0f;
  p = p * z + 1.0f / 3.0f;
  const float r = z * p;
  const float s2 = 2.0f * s;
  const float lm = s2 + s2 * r;
  const float fe = (float)e;
  return fe * 0.693115234375f + (fe * 3.194618329871446e-05f + lm);
}

// PK2 stress (Voigt S11, S22, S12) of one element, J2 state in/out.
// getStress2D (materialfunctions.py:10-29), misesReturnMap2D (35-101).
__device__ __forceinline__ void pk2_stress(int type, float lam, float mu, float F00, float F01,
                                           float F10, float F11, float sy, float H, float4& j2,
                                           float& s0, float& s1, float& s2) {
  const float C00 = F00 * F00 + F10 * F10;
  const float C01 = F00 * F01 + F10 * F11;
  const float C11 = F01 * F01 + F11 * F11;
  const float e00 = 0.5f * (C00 - 1.0f);
  const float e01 = 0.5f * (C01 - 0.0f);
  const float e11 = 0.5f * (C11 - 1.0f);
  if (type == MAT_ELASTIC) {
    const float lt = lam * (e00 + e11);
    const float tm = 2.0f * mu;
    s0 = lt * 1.0f + tm * e00;
    s1 = lt * 1.0f + tm * e11;
    s2 = lt * 0.0f + tm * e01;
  } else if (type == MAT_NEOHOOKEAN) {
    const float cdet = C00 * C11 - C01 * C01;
    float i00 = 0.f, i01 = 0.f, i11 = 0.f;
    if (cdet != 0.0f) {
      const float r = 1.0f / cdet;
      i00 = C11 * r;
      i01 = -C01 * r;
      i11 = C00 * r;
    }
    const float J = F00 * F11 - F01 * F10;
    const float c = lam * fw_log(J) - mu;
    s0 = c * i00 + mu * 1.0f;
    s1 = c * i11 + mu * 1.0f;
    s2 = c * i01 + mu * 0.0f;
  } else {  // MAT_MISES: radial return on Green-Lagrange strain
    const float t0 = e00 - j2.x, t1 = e11 - j2.y, t2 = e01 - j2.z;
    const float tr = t0 + t1;
    s0 = lam * tr + 2.0f * mu * t0;
    s1 = lam * tr + 2.0f * mu * t1;
    s2 = 2.0f * mu * t2;
    const float p = (s0 + s1) / 3.0f;
    const float d0 = s0 - p, d1 = s1 - p, d2 = s2;
    const float vm = sqrtf(d0 * d0 + d1 * d1 - d0 * d1 + 3.0f * d2 * d2);
    const float f = vm - (sy + H * j2.w);
    if (f > 0.0f) {
      const float dg = f / (3.0f * mu + H);
      const float eq = j2.w + dg;
      const float scale = 1.0f - 3.0f * mu * dg / vm;
      s0 = d0 * scale + p;
      s1 = d1 * scale + p;
      s2 = d2 * scale;
      const float h0 = d0 / vm, h1 = d1 / vm, h2 = d2 / vm;
      j2 = make_float4(j2.x + dg * h0, j2.y + dg * h1, j2.z + dg * h2, eq);
    }
  }
}

// Corner forces -(B^T S) * area of one triangle (femspringmanager.py:240-280).
__device__ __forceinline__ void element_forces(float2 a, float2 b, float2 c, float4 ji,
                                               const ElemMat& m, float sy, float H, float4& j2,
                                               float2& f1, float2& f2, float2& f3) {
  const float j00 = a.x - c.x, j01 = b.x - c.x;
  const float j10 = a.y - c.y, j11 = b.y - c.y;
  const float F00 = j00 * ji.x + j01 * ji.z;
  const float F01 = j00 * ji.y + j01 * ji.w;
  const float F10 = j10 * ji.x + j11 * ji.z;
  const float F11 = j10 * ji.y + j11 * ji.w;
  const float d00 = ji.x, d01 = ji.y, d10 = ji.z, d11 = ji.w;
  const float d20 = -ji.x - ji.z, d21 = -ji.y - ji.w;
  float s0, s1, s2;
  pk2_stress(elem_type(m.word), m.lam, m.mu, F00, F01, F10, F11, sy, H, j2, s0, s1, s2);
  // column r of B (3x6) dotted with S, in row order 0,1,2
  const float r0 = (d00 * F00) * s0 + (d01 * F01) * s1 + (d01 * F00 + d00 * F01) * s2;
  const float r1 = (d00 * F10) * s0 + (d01 * F11) * s1 + (d00 * F11 + d01 * F10) * s2;
  const float r2 = (d10 * F00) * s0 + (d11 * F01) * s1 + (d11 * F00 + d10 * F01) * s2;
  const float r3 = (d10 * F10) * s0 + (d11 * F11) * s1 + (d10 * F11 + d11 * F10) * s2;
  const float r4 = (d20 * F00) * s0 + (d21 * F01) * s1 + (d21 * F00 + d20 * F01) * s2;
  const float r5 = (d20 * F10) * s0 + (d21 * F11) * s1 + (d20 * F11 + d21 * F10) * s2;
  f1 = make_float2(-(r0 * m.area), -(r1 * m.area));
  f2 = make_float2(-(r2 * m.area), -(r3 * m.area));
  f3 = make_float2(-(r4 * m.area), -(r5 * m.area));
}

// Broad-phase gate of one pair (bvh.py:40-46 test; 10% grown boxes on the
// rebuild steps counter % 100 == 0, bvh.py:321-342; raw boxes otherwise).
__device__ __forceinline__ bool box_gate(float alx, float aly, float ahx, float ahy, float blx, float bly,
                                         float bhx, float bhy, int counter) {
  if (counter % 100 == 0) {
    const float ax = 0.1f * (ahx - alx), ay = 0.1f * (ahy - aly);
    const float bx = 0.1f * (bhx - blx), by = 0.1f * (bhy - bly);
    alx = alx - ax; ahx = ahx + ax; aly = aly - ay; ahy = ahy + ay;
    blx = blx - bx; bhx = bhx + bx; bly = bly - by; bhy = bhy + by;
  }
  return alx <= bhx && ahx >= blx && aly <= bhy && ahy >= bly;
}

__device__ __forceinline__ bool pair_gate(const Pair& p, float alx, float aly, float ahx,
                                          float ahy, int counter) {
  return box_gate(alx, aly, ahx, ahy, p.glo[0], p.glo[1], p.ghi[0], p.ghi[1], counter);
}

// Penalty force of one pair on one boundary node; returns false when the node
// is outside (no force).  mixedcontact.py:660-684, 1566-1643.
__device__ __forceinline__ bool contact_force(const Pair& p, const float* __restrict__ heights,
                                              const int8_t* __restrict__ occ, float2 x, float2 v,
                                              float dt, float2& out) {
  if (p.kind == PAIR_PLANE) {
    const float pen = (x.x - p.f[0]) * p.f[2] + (x.y - p.f[1]) * p.f[3];
    if (pen < 0.0f) {
      out = make_float2(-(p.f[2] * p.penalty * pen), -(p.f[3] * p.penalty * pen));
      return true;
    }
    return false;
  }
  float n0, n1, sd;
  if (p.kind == PAIR_HEIGHTFIELD) {
    // _nearest_on_curve_2d (mixedcontact.py:166-217)
    const float* h = heights + p.table;
    const int nx = p.n0;
    const float lbx = p.f[0], ubx = p.f[1];
    const float span = ubx - lbx;
    float u = 0.0f;
    if (span > 1e-12f) u = (x.x - lbx) / span;
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
    n0 = -dhdx;
    n1 = 1.0f;
    if (p.n1 == 1) {  // reverse
      n0 = -n0;
      n1 = -n1;
    }
    const float nl = sqrtf(n0 * n0 + n1 * n1);
    if (nl > 1e-12f) {
      n0 = n0 / nl;
      n1 = n1 / nl;
    }
    sd = (x.x - x.x) * n0 + (x.y - hh) * n1;
    if (!(sd < 0.0f)) return false;
    float fx = -n0 * p.penalty * sd, fy = -n1 * p.penalty * sd;
    const float vn = v.x * n0 + v.y * n1;
    if (vn < 0.0f) {
      fx = fx + (-n0 * 0.5f * p.penalty * vn * dt);
      fy = fy + (-n1 * 0.5f * p.penalty * vn * dt);
    }
    out = make_float2(fx, fy);
    return true;
  }
  // voxel grid: _voxel_signed_distance_2d (mixedcontact.py:220-302), only the
  // interior branch (the device port has no edge-list fallback).
  const int8_t* g = occ + p.table;
  const int nx = p.n0, ny = p.n1;
  const float lbx = p.f[0], lby = p.f[1], dx = p.f[2], dz = p.f[3];
  const int i = (int)floorf((x.x - lbx) / dx);
  const int j = (int)floorf((x.y - lby) / dz);
  if (!(0 <= i && i < nx && 0 <= j && j < ny)) return false;
  if (g[i * ny + j] != 1) return false;
  float dnx = 1e9f, dpx = 1e9f, dny = 1e9f, dpy = 1e9f;
  for (int st = 0; st < nx; ++st) {
    const int idx = i - 1 - st;
    if (idx < 0 || g[idx * ny + j] == 0) {
      dnx = x.x - (lbx + (float)(idx + 1) * dx);
      break;
    }
  }
  for (int st = 0; st < nx; ++st) {
    const int idx = i + 1 + st;
    if (idx >= nx || g[idx * ny + j] == 0) {
      dpx = (lbx + (float)idx * dx) - x.x;
      break;
    }
  }
  for (int st = 0; st < ny; ++st) {
    const int idx = j - 1 - st;
    if (idx < 0 || g[i * ny + idx] == 0) {
      dny = x.y - (lby + (float)(idx + 1) * dz);
      break;
    }
  }
  for (int st = 0; st < ny; ++st) {
    const int idx = j + 1 + st;
    if (idx >= ny || g[i * ny + idx] == 0) {
      dpy = (lby + (float)idx * dz) - x.y;
      break;
    }
  }
  float mv = dnx;
  int face = 0;
  if (dpx < mv) { mv = dpx; face = 1; }
  if (dny < mv) { mv = dny; face = 2; }
  if (dpy < mv) { mv = dpy; face = 3; }
  if (face == 0) { sd = -dnx; n0 = -1.0f; n1 = 0.0f; }
  else if (face == 1) { sd = -dpx; n0 = 1.0f; n1 = 0.0f; }
  else if (face == 2) { sd = -dny; n0 = 0.0f; n1 = -1.0f; }
  else { sd = -dpy; n0 = 0.0f; n1 = 1.0f; }
  if (!(sd < 0.0f)) return false;
  const float pen = -sd;
  float fx = n0 * p.penalty * pen, fy = n1 * p.penalty * pen;
  const float vn = v.x * n0 + v.y * n1;
  if (vn < 0.0f) {
    fx = fx + (-n0 * 0.5f * p.penalty * vn * dt);
    fy = fy + (-n1 * 0.5f * p.penalty * vn * dt);
  }
  out = make_float2(fx, fy);
  return true;
}

// Boundary conditions and symplectic Euler (femspringmanager.py:334-358).
// im is 1.0f / m (the reference divides every step; dividing once gives the
// same bits).
__device__ __forceinline__ void integrate_im(int bc, float2 f, float m, float im, float2 bcv,
                                             float dt, float damping, float2& x, float2& v) {
  if (bc & BC_U) {
    f = make_float2(0.0f, 0.0f);
  } else if (bc & BC_A) {
    f = make_float2(m * bcv.x, m * bcv.y);
  } else if (bc & BC_GRAVITY) {
    f = make_float2(f.x + m * bcv.x, f.y + m * bcv.y);
  } else if (bc & BC_FORCE) {
    f = make_float2(f.x + bcv.x, f.y + bcv.y);
  }
  const float ax = 0.0f + (f.x - damping * v.x) * im;
  const float ay = 0.0f + (f.y - damping * v.y) * im;
  float2 nv = make_float2(v.x + ax * dt, v.y + ay * dt);
  if (bc & BC_V) {
    nv = bcv;
  } else if (bc & BC_U) {
    nv = make_float2(0.0f, 0.0f);
  }
  v = nv;
  x = make_float2(x.x + nv.x * dt, x.y + nv.y * dt);
}

__device__ __forceinline__ void integrate(int bc, float2 f, float m, float2 bcv, float dt,
                                          float damping, float2& x, float2& v) {
  if (bc & BC_U) {
    f = make_float2(0.0f, 0.0f);
  } else if (bc & BC_A) {
    f = make_float2(m * bcv.x, m * bcv.y);
  } else if (bc & BC_GRAVITY) {
    f = make_float2(f.x + m * bcv.x, f.y + m * bcv.y);
  } else if (bc & BC_FORCE) {
    f = make_float2(f.x + bcv.x, f.y + bcv.y);
  }
  const float im = 1.0f / m;
  const float ax = 0.0f + (f.x - damping * v.x) * im;
  const float ay = 0.0f + (f.y - damping * v.y) * im;
  float2 nv = make_float2(v.x + ax * dt, v.y + ay * dt);
  if (bc & BC_V) {
    nv = bcv;
  } else if (bc & BC_U) {
    nv = make_float2(0.0f, 0.0f);
  }
  v = nv;
  x = make_float2(x.x + nv.x * dt, x.y + nv.y * dt);
}

}  // namespace fw
