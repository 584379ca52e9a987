// fw_rigid.cuh -- rigid primitives (ball, box, capsule) touching FEM bodies.
//
// Restated reference code (paths relative to the FlatWorld project root):
//   flatworld/mixedcontact.py:1026-1115     _batched_rigid_prim_kernel (untied branch)
//   flatworld/contact_detection.py:148-190  detectPointToPrimitive
//   flatworld/utils.py:7-145, 235-300       cal2DRotationMat, sphere / capsule / OBB
//                                           SDF queries, primitive bounding boxes
//   flatworld/rigidmanager.py:766-794       _write_primitive_aabb
//   flatworld/rigidmanager.py:832-964       _rigid_step_wp, _update_u_and_bbox_wp
//   flatworld/explicitloop.py:533-552       the rigid update every N substeps
//
// Per substep, the node kernel evaluates each FEM-rigid work item of its node
// (pair order, after FEM-FEM contact and before the height fields) and writes
// the item's reaction (impulse, torque, rigid) to its slot; k_rigid then adds
// the reactions to the rigid accumulators in work-item order -- the order in
// which a serial run of the reference's atomic adds applies them -- and, on
// the substeps the schedule names, runs the rigid velocity and position update.
#pragma once
#include "fw_device.cuh"

namespace fw {

constexpr int PAIR_RIGID = 3;

// RigidType (flatworld/definitions.py:50-53)
constexpr int RIGID_BALL = 1;
constexpr int RIGID_BOX = 2;
constexpr int RIGID_CAPSULE = 8;
// An analytical entry of the rigid manager (a ground plane, height field or
// voxel grid of a loop where some ground plane has BCs): it moves with its BCs
// and its broad-phase box follows, rigidmanager.py:2486-2517, 832-964.
constexpr int RIGID_ANALYTICAL = 64;

// Rigid BC bits (flatworld/definitions.py:96-104)
constexpr int RBC_U = 0x1, RBC_V = 0x2, RBC_A = 0x4, RBC_FORCE = 0x8, RBC_GRAVITY = 0x10;
constexpr int RBC_R = 0x20, RBC_ROTV = 0x40, RBC_ROTA = 0x80, RBC_TORQUE = 0x100;

// One rigid body: the reference's rigidParams / quat / V / RotV / U / BC
// values / accumulators / cached rotation / box for that index.
struct __align__(16) Rigid {
  float c[2], prim[2];        // rigidParams[i, 0], rigidParams[i, 1]
  float radius, quat, mass, inertia;
  float V[2], W, bcR;          // velocity, angular velocity, BC rotation value
  float bcT[2], bcG[2];        // BC translation value, gravity
  float U[2], acc[2];          // displacement, accumulated impulse
  float accw;                  // accumulated rotational impulse
  int type, bc, in_contact;
  float rot[4];                // cached_rotation_matrix, row-major
  float lb[2], ub[2];          // the rigid's box (aabb[domain])
  int scene;                   // the scene (loop) the rigid belongs to
  int rs;                      // that scene's index in the list of scenes with rigids
  int pad[2];
};
static_assert(sizeof(Rigid) == 144, "Rigid record is 144 bytes");

// The rigids and grounds of one scene: rig[r0, r0 + rn), grounds [g0, g0 + gn).
struct RigidScene {
  int scene, r0, rn, g0, gn, pad[3];
};

// Schedule of the rigid update (host-computed from the float64 substep dt,
// explicitloop.py:535-538): every `every` substeps, with dt = every * dt.
struct RigidClock {
  int every;
  float dt;
  float damping;
  int pad;
};

// sin and cos from IEEE + - * only (the CPU oracle evaluates the identical
// operations): Cody-Waite reduction x = k pi/2 + r, pi/2 split into
// 1.5703125 + 0x1.fb4p-12 + 0x1.4442d2p-24 (k times the first two is exact
// for |k| < 2^13), Taylor series of sin through r^9 and of cos through r^10
// on |r| <= pi/4 (truncation below 2e-9), quadrant k mod 4.
__device__ __forceinline__ void fw_sincosf(float x, float& s_out, float& c_out) {
  const float k = floorf(x * 0.63661975f + 0.5f);
  const float r = ((x - k * 1.5703125f) - k * 4.837512969970703125e-4f) - k * 0x1.4442d2p-24f;
  const float z = r * r;
  const float sp = -1.0f / 6.0f + z * (1.0f / 120.0f + z * (-1.0f / 5040.0f + z * (1.0f / 362880.0f)));
  const float sr = r + r * z * sp;
  const float cp =
      -0.5f + z * (1.0f / 24.0f + z * (-1.0f / 720.0f + z * (1.0f / 40320.0f + z * (-1.0f / 3628800.0f))));
  const float cr = 1.0f + z * cp;
  const int q = ((int)k) & 3;
  s_out = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
  c_out = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
}

__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }

// cal2DRotationMat (utils.py:7-11)
__device__ __forceinline__ void rigid_rot(Rigid& g) {
  float s, c;
  fw_sincosf(g.quat, s, c);
  g.rot[0] = c;
  g.rot[1] = -s;
  g.rot[2] = s;
  g.rot[3] = c;
}

// _write_primitive_aabb with getBallBBox / getBoxBBox / getCapsuleBBox; for an
// analytical entry the moving-plane box of _update_u_and_bbox_wp
// (rigidmanager.py:950-964): +-100 along the tangent, +-0.1 along the rotated
// normal (a height field's or voxel grid's entry has zero point and normal).
__device__ __forceinline__ void rigid_aabb(Rigid& g) {
  const float* m = g.rot;
  if (g.type == RIGID_ANALYTICAL) {
    const float nx = m[0] * g.prim[0] + m[1] * g.prim[1], ny = m[2] * g.prim[0] + m[3] * g.prim[1];
    const float tx = -ny, ty = nx;
    const float lox = g.c[0] - tx * 100.0f - nx * 0.1f, loy = g.c[1] - ty * 100.0f - ny * 0.1f;
    const float hix = g.c[0] + tx * 100.0f + nx * 0.1f, hiy = g.c[1] + ty * 100.0f + ny * 0.1f;
    g.lb[0] = rmin(lox, hix);
    g.lb[1] = rmin(loy, hiy);
    g.ub[0] = rmax(lox, hix);
    g.ub[1] = rmax(loy, hiy);
  } else if (g.type == RIGID_BALL) {
    g.lb[0] = g.c[0] - g.radius;
    g.lb[1] = g.c[1] - g.radius;
    g.ub[0] = g.c[0] + g.radius;
    g.ub[1] = g.c[1] + g.radius;
  } else if (g.type == RIGID_BOX) {
    const float ex = g.prim[0], ey = g.prim[1];
    const float vx[4] = {ex, ex, ex, -ex}, vy[4] = {ey, -ey, ey, ey};
    const float sc[4] = {-0.5f, 0.5f, 0.5f, 0.5f};
    float px[4], py[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float rx = m[0] * vx[k] + m[1] * vy[k], ry = m[2] * vx[k] + m[3] * vy[k];
      px[k] = g.c[0] + sc[k] * rx;
      py[k] = g.c[1] + sc[k] * ry;
    }
    g.lb[0] = rmin(rmin(px[0], px[1]), rmin(px[2], px[3]));
    g.lb[1] = rmin(rmin(py[0], py[1]), rmin(py[2], py[3]));
    g.ub[0] = rmax(rmax(px[0], px[1]), rmax(px[2], px[3]));
    g.ub[1] = rmax(rmax(py[0], py[1]), rmax(py[2], py[3]));
  } else if (g.type == RIGID_CAPSULE) {
    const float ax = g.prim[0], ay = g.prim[1];
    const float alen = sqrtf(ax * ax + ay * ay);
    const float d0 = ax / alen, d1 = ay / alen;
    const float dx = m[0] * d0 + m[1] * d1, dy = m[2] * d0 + m[3] * d1;
    const float p0x = g.c[0] - dx * alen, p0y = g.c[1] - dy * alen;
    const float p1x = g.c[0] + dx * alen, p1y = g.c[1] + dy * alen;
    const float perp0 = g.radius * sqrtf(rmax(0.0f, 1.0f - dx * dx)), axial0 = g.radius * fabsf(dx);
    const float perp1 = g.radius * sqrtf(rmax(0.0f, 1.0f - dy * dy)), axial1 = g.radius * fabsf(dy);
    g.lb[0] = rmin(p0x, p1x) - perp0 - axial0;
    g.lb[1] = rmin(p0y, p1y) - perp1 - axial1;
    g.ub[0] = rmax(p0x, p1x) + perp0 + axial0;
    g.ub[1] = rmax(p0y, p1y) + perp1 + axial1;
  }
}

// detectPointToPrimitive: signed distance, outward normal, contact point.
__device__ __forceinline__ float rigid_detect(const Rigid& g, float px, float py, float& nx, float& ny,
                                              float& cx, float& cy) {
  float pen = 1e9f, n0 = 0.0f, n1 = 0.0f;
  const float* m = g.rot;
  if (g.type == RIGID_BALL) {
    const float qx = px - g.c[0], qy = py - g.c[1];
    const float len = sqrtf(qx * qx + qy * qy);
    pen = len - g.radius;
    const float dn = rmax(len, 1e-9f);
    n0 = qx / dn;
    n1 = qy / dn;
  } else if (g.type == RIGID_BOX) {
    const float hx = 0.5f * g.prim[0], hy = 0.5f * g.prim[1];
    const float wx = px - g.c[0], wy = py - g.c[1];
    const float lx = m[0] * wx + m[2] * wy, ly = m[1] * wx + m[3] * wy;  // transpose(rot) @ w
    const float sd0 = lx - hx, sd1 = -lx - hx, sd2 = ly - hy, sd3 = -ly - hy;
    float best = -1e9f, ln0 = 0.0f, ln1 = 0.0f;
    if (sd0 > best) { best = sd0; ln0 = 1.0f; ln1 = 0.0f; }
    if (sd1 > best) { best = sd1; ln0 = -1.0f; ln1 = 0.0f; }
    if (sd2 > best) { best = sd2; ln0 = 0.0f; ln1 = 1.0f; }
    if (sd3 > best) { best = sd3; ln0 = 0.0f; ln1 = -1.0f; }
    if (sd0 > 0.0f || sd1 > 0.0f || sd2 > 0.0f || sd3 > 0.0f) {
      float qx = lx, qy = ly;
      if (lx < -hx) qx = -hx; else if (lx > hx) qx = hx;
      if (ly < -hy) qy = -hy; else if (ly > hy) qy = hy;
      const float ddx = lx - qx, ddy = ly - qy;
      const float dist = sqrtf(ddx * ddx + ddy * ddy);
      if (dist > 1e-9f) {
        ln0 = ddx / dist;
        ln1 = ddy / dist;
      }
      best = dist;
    }
    pen = best;
    n0 = m[0] * ln0 + m[1] * ln1;
    n1 = m[2] * ln0 + m[3] * ln1;
  } else if (g.type == RIGID_CAPSULE) {
    const float lcx = g.c[0] + (m[0] * g.prim[0] + m[1] * g.prim[1]);
    const float lcy = g.c[1] + (m[2] * g.prim[0] + m[3] * g.prim[1]);
    const float qx = 2.0f * g.c[0] - lcx, qy = 2.0f * g.c[1] - lcy;
    const float apx = px - lcx, apy = py - lcy, abx = qx - lcx, aby = qy - lcy;
    const float ab2 = abx * abx + aby * aby;
    float t = (apx * abx + apy * aby) / ab2;
    t = rmax(0.0f, rmin(1.0f, t));
    const float clx = lcx + t * abx, cly = lcy + t * aby;
    const float ex = px - clx, ey = py - cly;
    const float dist = sqrtf(ex * ex + ey * ey);
    pen = dist - g.radius;
    const float dn = rmax(dist, 1e-9f);
    n0 = ex / dn;
    n1 = ey / dn;
  }
  nx = n0;
  ny = n1;
  cx = px;
  cy = py;
  if (pen < 0.0f) {
    cx = px - n0 * pen;
    cy = py - n1 * pen;
  }
  return pen;
}

// One FEM-rigid work item of one node: adds the contact force to f and
// returns the reaction record (impulse x, y, torque, rigid index bits; rigid
// -1 when the item does not touch).  mixedcontact.py:1054-1115; a tied pair
// (ExplicitLoop ties) pulls the node to the contact point with no offset and
// no friction (1073-1087).
__device__ __forceinline__ float4 rigid_item(const Rigid& g, int rigid, float penalty, float mu, bool tied,
                                             float2 x, float2 v, float dt, float2& f) {
  const float4 none = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
  if (rmin(x.x - g.lb[0], x.y - g.lb[1]) < 0.0f || rmin(g.ub[0] - x.x, g.ub[1] - x.y) < 0.0f) return none;
  float nx, ny, cx, cy;
  const float pen = rigid_detect(g, x.x, x.y, nx, ny, cx, cy);
  const float gx = g.ub[0] - g.lb[0], gy = g.ub[1] - g.lb[1];
  const float margin = sqrtf(gx * gx + gy * gy) * 0.5f;
  if (!(pen < margin)) return none;
  if (tied) {
    const float mx = cx - x.x, my = cy - x.y;
    const float px = penalty * mx, py = penalty * my;
    f.x += px;
    f.y += py;
    const float lx = cx - g.c[0], ly = cy - g.c[1];
    const float fx = -px, fy = -py;
    return make_float4(-px * dt, -py * dt, (lx * fy - ly * fx) * dt, __int_as_float(rigid));
  }
  const float depth = pen - 1e-4f;
  if (!(depth < 0.0f)) return none;
  const float fnx = -nx * penalty * depth, fny = -ny * penalty * depth;
  float tx = fnx, ty = fny;
  if (mu > 1e-9f) {
    const float rx = cx - g.c[0], ry = cy - g.c[1];
    const float svx = g.V[0] + -g.W * ry, svy = g.V[1] + g.W * rx;
    const float relx = v.x - svx, rely = v.y - svy;
    const float rn = relx * nx + rely * ny;
    const float tgx = relx - rn * nx, tgy = rely - rn * ny;
    const float tlen = sqrtf(tgx * tgx + tgy * tgy);
    if (tlen > 1e-9f) {
      const float dx = -tgx / tlen, dy = -tgy / tlen;
      const float fn = sqrtf(fnx * fnx + fny * fny);
      tx = tx + dx * mu * fn;
      ty = ty + dy * mu * fn;
    }
  }
  f.x += tx;
  f.y += ty;
  const float lx = cx - g.c[0], ly = cy - g.c[1];
  const float fx = -tx, fy = -ty;
  return make_float4(-tx * dt, -ty * dt, (lx * fy - ly * fx) * dt, __int_as_float(rigid));
}

// Clearance below which a rigid counts as meeting a ground or another rigid:
// 20x the reference's speculative rigid-ground contact margin (0.0005,
// rigidmanager.py:3257), so every state in which the reference's constraint
// solve could see a contact row is flagged.
constexpr float kRigidClearance = 0.01f;

// The rigid bodies' update (rigidmanager.py:2102-2197 without a constraint
// solve): _rigid_step_wp then _update_u_and_bbox_wp, serially.  A rigid within
// kRigidClearance of a ground plane (its box's support point, as
// _detect_analytical_prim_contacts_wp's early out measures it,
// rigidmanager.py:1127-1136), of a height-field / voxel box (gkind 1), or of
// another contact rigid's box sets bit 0 of *err: the reference would solve
// that contact, this library does not.  So does a rigid whose state is no
// longer finite.
__device__ __forceinline__ void rigid_update(Rigid* rig, int n, const float4* gbox, const int* gkind,
                                             int n_ground, float dt, float damping, int* err) {
  const float cl = kRigidClearance;
  for (int a = 0; a < n; ++a) {
    const Rigid& g = rig[a];
    if (g.type == RIGID_ANALYTICAL) continue;  // not a rigid body
    for (int q = 0; q < n_ground; ++q) {
      const float4 b = gbox[q];
      // written as "not clear", so that a non-finite box is flagged too
      if (gkind[q] == 0) {
        const float sx = b.z < 0.0f ? g.ub[0] : g.lb[0], sy = b.w < 0.0f ? g.ub[1] : g.lb[1];
        if (!((sx - b.x) * b.z + (sy - b.y) * b.w > cl)) *err |= 1;
      } else if (!(g.lb[0] - cl > b.z || g.ub[0] + cl < b.x || g.lb[1] - cl > b.w || g.ub[1] + cl < b.y)) {
        *err |= 1;
      }
    }
    for (int q = a + 1; q < n; ++q) {
      const Rigid& h = rig[q];
      if (h.type != RIGID_ANALYTICAL && g.in_contact && h.in_contact &&
          !(g.lb[0] - cl > h.ub[0] || g.ub[0] + cl < h.lb[0] || g.lb[1] - cl > h.ub[1] || g.ub[1] + cl < h.lb[1]))
        *err |= 1;
    }
    if (!(fabsf(g.c[0]) < 1e30f && fabsf(g.c[1]) < 1e30f && fabsf(g.quat) < 1e30f)) *err |= 1;
  }
  for (int a = 0; a < n; ++a) {  // _rigid_step_wp
    Rigid& g = rig[a];
    rigid_rot(g);
    if (g.type == RIGID_ANALYTICAL) continue;  // the impulse pass covers the rigid bodies only
    if (g.bc & RBC_A) {
      g.acc[0] = 0.0f;
      g.acc[1] = 0.0f;
    } else {
      if (g.bc & RBC_GRAVITY) {
        g.acc[0] = g.acc[0] + g.mass * g.bcG[0] * dt;
        g.acc[1] = g.acc[1] + g.mass * g.bcG[1] * dt;
      }
      if (g.bc & RBC_FORCE) {
        g.acc[0] = g.acc[0] + g.bcT[0] * dt;
        g.acc[1] = g.acc[1] + g.bcT[1] * dt;
      }
    }
    if (g.bc & RBC_ROTA) g.accw = 0.0f;
    else if (g.bc & RBC_TORQUE) g.accw = g.accw + g.bcR * dt;
    g.V[0] = g.V[0] + g.acc[0] / g.mass;
    g.V[1] = g.V[1] + g.acc[1] / g.mass;
    g.W = g.W + g.accw / (g.inertia + 1e-6f);
    const float damp = rmax(0.0f, 1.0f - damping * dt);
    g.V[0] = g.V[0] * damp;
    g.V[1] = g.V[1] * damp;
    g.W = g.W * damp;
  }
  for (int a = 0; a < n; ++a) {
    Rigid& g = rig[a];
    if (g.bc & RBC_A) {
      g.V[0] = g.V[0] + g.bcT[0] * dt;
      g.V[1] = g.V[1] + g.bcT[1] * dt;
    }
    if (g.bc & RBC_ROTA) g.W = g.W + g.bcR * dt;
  }
  for (int a = 0; a < n; ++a) {  // _update_u_and_bbox_wp
    Rigid& g = rig[a];
    if (g.bc & RBC_V) {
      g.V[0] = g.bcT[0];
      g.V[1] = g.bcT[1];
    } else if (g.bc & RBC_U) {
      g.V[0] = 0.0f;
      g.V[1] = 0.0f;
    } else if (g.bc & RBC_R) {
      g.V[0] = 0.0f;
      g.V[1] = 0.0f;
      g.W = 0.0f;
    }
    if (g.bc & RBC_ROTV) g.W = g.bcR;
    const float dux = g.V[0] * dt, duy = g.V[1] * dt;
    g.U[0] = g.U[0] + dux;
    g.U[1] = g.U[1] + duy;
    g.c[0] = g.c[0] + dux;
    g.c[1] = g.c[1] + duy;
    g.quat = g.quat + g.W * dt;
    if (g.quat > 3.141592653589793f) g.quat = g.quat - 2.0f * 3.141592653589793f;
    else if (g.quat < -3.141592653589793f) g.quat = g.quat + 2.0f * 3.141592653589793f;
  }
  for (int a = 0; a < n; ++a) {
    rig[a].acc[0] = 0.0f;
    rig[a].acc[1] = 0.0f;
    rig[a].accw = 0.0f;
  }
  for (int a = 0; a < n; ++a) rigid_aabb(rig[a]);
}

}  // namespace fw
