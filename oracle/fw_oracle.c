/*
 * fw_oracle.c -- CPU restatement of FlatWorld's explicit 2D FEM substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA path is
 * checked against; nothing in the product (flatworld_b200/) links, loads or
 * calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * and reference legs use it.
 *
 * Built twice from this one source (see oracle/Makefile):
 *   liboracle_f32.so : REAL=float  -- the reference's FP32 scheme, operation by
 *                      operation, compiled with -ffp-contract=off so that every
 *                      product and sum is rounded the way the source reads.
 *   liboracle_f64.so : REAL=double -- the same scheme in FP64 (error oracle).
 * A third build, liboracle_f32fma.so, contracts a*b+c into FMAs; the distance
 * between the two FP32 builds is the rounding noise floor of the scheme itself
 * (the reference's Warp GPU path is compiled by NVRTC with FMA contraction on).
 * A fourth, liboracle_f32libm.so, takes log from the C library, as the
 * reference's Warp CPU device does.
 *
 * Restated reference code (all paths relative to the FlatWorld project root):
 *   flatworld/femspringmanager.py:59-68    get_jacobian_2d, get_weights_2d
 *   flatworld/femspringmanager.py:71-105   get_b_matrix_2d
 *   flatworld/femspringmanager.py:113-138  _prepare_fem_data_kernel
 *   flatworld/femspringmanager.py:217-280  _fem_internal_force_kernel
 *   flatworld/femspringmanager.py:315-358  _integrate_nodes_kernel
 *   flatworld/femspringmanager.py:361-408  _update_bbox_kernel
 *   flatworld/femspringmanager.py:941-1012 femStep (launch order)
 *   flatworld/materials/materialfunctions.py:10-29  getStress2D
 *   flatworld/materials/materialfunctions.py:35-101 misesReturnMap2D
 *   flatworld/mixedcontact.py:166-217      _nearest_on_curve_2d
 *   flatworld/mixedcontact.py:220-302      _voxel_signed_distance_2d
 *   flatworld/mixedcontact.py:495-515      _activate_pairs_kernel (+ bvh.py:40-46,
 *                                          321-342, 393-478: box test semantics)
 *   flatworld/mixedcontact.py:660-684      _batched_analytical_contact_kernel
 *   flatworld/mixedcontact.py:1566-1643    heightfield / voxel contact kernels
 *   flatworld/mixedcontact.py:1654-1755    run_batched_contacts (launch order)
 *   flatworld/explicitloop.py:473-555      advance (contacts -> femStep)
 *   flatworld/mixedcontact.py:886-1018     _batched_flexflex_contact_kernel_sh (FEM-FEM)
 *   flatworld/mixedcontact.py:1654-1696    flex pair activation, hash refresh, launch
 *   flatworld/explicitloop.py:495-514      BVH domain stamps (+ :451-463 scan kernel)
 *   flatworld/contact_detection.py:15-92   pointToEdgeContact, detectPointToMeshBoundary
 *   flatworld/spatialmanager.py:30-198     add_element, query_point_with_buffer
 *   flatworld/spatialmanager.py:200-420, 613-712  hash build kernels, build()
 *   flatworld/femspringmanager.py:1035-1063 + its populate kernel  FEM hash refresh
 *   flatworld/mixedcontact.py:1026-1115     _batched_rigid_prim_kernel (FEM-rigid, untied)
 *   flatworld/contact_detection.py:148-190, utils.py:7-145, 235-300  primitive SDFs, boxes
 *   flatworld/rigidmanager.py:766-794, 832-964  rigid boxes, _rigid_step_wp, _update_u_and_bbox_wp
 *
 * Warp builtins (warp-lang, unpinned: requirements.txt `warp-lang>=1.7.0`) are
 * restated from their published definitions: mat22 @ mat22 and mat @ vec sum
 * products in index order; determinant(m) = m00*m11 - m01*m10; inverse(m22) =
 * adjugate * (1/det), the zero matrix when det == 0; round() rounds half away
 * from zero (C roundf); floor and sqrt are the C library functions; log is
 * or_logf below, sin and cos or_sincosf (or the C library's logf, sinf and
 * cosf in liboracle_f32libm.so); the serial
 * CPU device applies atomic_add in launch order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#ifndef REAL
#define REAL float
#endif

/* log of the FP32 builds: unless USE_LIBM_MATH is defined, the method below
 * (Cody-Waite reduction + atanh series, IEEE + - * / only), which the CUDA
 * kernels evaluate with the same operations in the same order.  Any accurate
 * log is a faithful reading of the reference's wp.log; this one makes CPU and
 * GPU agree bit for bit.  USE_LIBM_MATH builds use the C library's logf, as the
 * reference's Warp CPU device does. */
static float or_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  uint32_t u;
  memcpy(&u, &x, sizeof(u));
  int e = 0;
  if (u < 0x00800000u) {
    x = x * 8388608.0f;
    memcpy(&u, &x, sizeof(u));
    e = -23;
  }
  e += (int)((u >> 23) & 0xFFu) - 127;
  u = (u & 0x007FFFFFu) | 0x3F800000u;
  float m;
  memcpy(&m, &u, sizeof(m));
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

#if defined(REAL_IS_DOUBLE)
#define R_SQRT sqrt
#define R_LOG log
#define R_FLOOR floor
#define R_ROUND round
#define R_FABS fabs
#define R_CEIL ceil
#define R_POW pow
#else
#define R_SQRT sqrtf
#if defined(USE_LIBM_MATH)
#define R_LOG logf
#else
#define R_LOG or_logf
#endif
#define R_FLOOR floorf
#define R_ROUND roundf
#define R_FABS fabsf
#define R_CEIL ceilf
#define R_POW powf
#endif

/* Bit constants: flatworld/definitions.py:96-104 */
#define BC_U 0x1
#define BC_V 0x2
#define BC_A 0x4
#define BC_FORCE 0x8
#define BC_GRAVITY 0x10

/* MaterialType: flatworld/definitions.py:80-83 */
#define MAT_SPRING 0 /* a 2-node spring of a spring-mass domain (elemType 0) */
#define MAT_ELASTIC 1
#define MAT_NEOHOOKEAN 2
#define MAT_MISES 3

#define PAIR_PLANE 0
#define PAIR_HEIGHTFIELD 1
#define PAIR_VOXEL 2

typedef struct {
  int kind;
  int body;
  int entry; /* >= 0: gated by that rigid manager entry's current box (a loop with a moving plane) */
  REAL penalty;
  REAL glb[2], gub[2]; /* ground getBBox(), gate box */
  /* plane */
  REAL p[2], n[2];
  /* heightfield */
  int hnx, reverse;
  REAL hlbx, hubx;
  REAL* h;
  /* voxel */
  int vnx, vny;
  REAL vlb[2], vdx, vdz;
  int32_t* occ; /* occ[i*vny + j] */
} or_pair;

typedef struct {
  int n_nodes, n_elems, n_bodies, n_pairs, n_threads;
  REAL *x, *v, *u, *fext, *mass, *bcv;
  int32_t* bc;
  int32_t* conn; /* 3 per element */
  int32_t* type;
  REAL *E, *nu, *rho, *sy, *H;
  REAL *area, *jinv, *epsp, *eqps;
  int32_t *bn_off, *bn_cnt, *bnodes;
  REAL* aabb; /* per body: lbx, lby, ubx, uby */
  or_pair* pairs;
  /* CSR (node -> element corners, ascending element) for the threaded path */
  int32_t *csr_off, *csr_slot;
  REAL* corner; /* 6 per element */
  struct or_flex* flex; /* FEM-FEM contact, NULL when the loop has none */
  struct or_rigids* rig; /* rigid primitives, NULL when the loop has none */
} or_world;

static REAL* dupf(const float* src, size_t n) {
  REAL* d = (REAL*)malloc(sizeof(REAL) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) d[i] = (REAL)src[i];
  return d;
}
static int32_t* dupi(const int32_t* src, size_t n) {
  int32_t* d = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
  if (n) memcpy(d, src, sizeof(int32_t) * n);
  return d;
}

/* _prepare_fem_data_kernel (femspringmanager.py:113-138), serial element order. */
static void prepare(or_world* w) {
  for (int i = 0; i < w->n_nodes; ++i) w->mass[i] = 0;
  for (int e = 0; e < w->n_elems; ++e) {
    if (w->type[e] == MAT_SPRING) { /* addSpringDomain: elemVolume = rest length (rho slot) */
      w->area[e] = w->rho[e];
      for (int k = 0; k < 4; ++k) w->jinv[4 * e + k] = 0;
      continue;
    }
    int n1 = w->conn[3 * e], n2 = w->conn[3 * e + 1], n3 = w->conn[3 * e + 2];
    REAL j00 = w->x[2 * n1] - w->x[2 * n3], j01 = w->x[2 * n2] - w->x[2 * n3];
    REAL j10 = w->x[2 * n1 + 1] - w->x[2 * n3 + 1], j11 = w->x[2 * n2 + 1] - w->x[2 * n3 + 1];
    REAL det_w = j00 * j11 - j01 * j10;
    REAL vol = R_FABS(det_w) * (REAL)0.5;
    w->area[e] = vol;
    REAL det = j00 * j11 - j01 * j10;
    REAL* ji = w->jinv + 4 * e;
    if (det != (REAL)0) {
      REAL r = (REAL)1.0 / det;
      ji[0] = j11 * r;
      ji[1] = -j01 * r;
      ji[2] = -j10 * r;
      ji[3] = j00 * r;
    } else {
      ji[0] = ji[1] = ji[2] = ji[3] = 0;
    }
    REAL nd_mass = vol * w->rho[e] / (REAL)3.0;
    w->mass[n1] += nd_mass;
    w->mass[n2] += nd_mass;
    w->mass[n3] += nd_mass;
  }
}

/* getStress2D (materialfunctions.py:10-29) for ELASTIC / NEOHOOKEAN and
 * misesReturnMap2D (35-101) for MISES.  Returns Voigt PK2 (S11, S22, S12). */
static void stress(const or_world* w, int e, REAL F00, REAL F01, REAL F10, REAL F11,
                   REAL* s, REAL* epsp_out, REAL* eqps_out) {
  REAL E = w->E[e], nu = w->nu[e];
  REAL lam = E * nu / (((REAL)1.0 + nu) * ((REAL)1.0 - (REAL)2.0 * nu));
  REAL mu = E / ((REAL)2.0 * ((REAL)1.0 + nu));
  /* C = F^T F ; strain = 0.5 (C - I) */
  REAL C00 = F00 * F00 + F10 * F10;
  REAL C01 = F00 * F01 + F10 * F11;
  REAL C10 = F01 * F00 + F11 * F10;
  REAL C11 = F01 * F01 + F11 * F11;
  REAL e00 = (REAL)0.5 * (C00 - (REAL)1.0);
  REAL e01 = (REAL)0.5 * (C01 - (REAL)0.0);
  REAL e11 = (REAL)0.5 * (C11 - (REAL)1.0);
  int t = w->type[e];
  if (t == MAT_MISES) {
    REAL ep0 = w->epsp[3 * e], ep1 = w->epsp[3 * e + 1], ep2 = w->epsp[3 * e + 2];
    REAL eq = w->eqps[e];
    REAL t0 = e00 - ep0, t1 = e11 - ep1, t2 = e01 - ep2;
    REAL tr = t0 + t1;
    REAL s0 = lam * tr + (REAL)2.0 * mu * t0;
    REAL s1 = lam * tr + (REAL)2.0 * mu * t1;
    REAL s2 = (REAL)2.0 * mu * t2;
    REAL p = (s0 + s1) / (REAL)3.0;
    REAL d0 = s0 - p, d1 = s1 - p, d2 = s2;
    REAL vm = R_SQRT(d0 * d0 + d1 * d1 - d0 * d1 + (REAL)3.0 * d2 * d2);
    REAL f = vm - (w->sy[e] + w->H[e] * eq);
    s[0] = s0;
    s[1] = s1;
    s[2] = s2;
    epsp_out[0] = ep0;
    epsp_out[1] = ep1;
    epsp_out[2] = ep2;
    *eqps_out = eq;
    if (f > (REAL)0.0) {
      REAL denom = (REAL)3.0 * mu + w->H[e];
      REAL dg = f / denom;
      *eqps_out = eq + dg;
      REAL scale = (REAL)1.0 - (REAL)3.0 * mu * dg / vm;
      REAL n0 = d0 * scale, n1 = d1 * scale, n2 = d2 * scale;
      s[0] = n0 + p;
      s[1] = n1 + p;
      s[2] = n2;
      REAL h0 = d0 / vm, h1 = d1 / vm, h2 = d2 / vm;
      epsp_out[0] = ep0 + dg * h0;
      epsp_out[1] = ep1 + dg * h1;
      epsp_out[2] = ep2 + dg * h2;
    }
    return;
  }
  if (t == MAT_ELASTIC) {
    REAL tr = e00 + e11;
    REAL lt = lam * tr;
    REAL tm = (REAL)2.0 * mu;
    s[0] = lt * (REAL)1.0 + tm * e00;
    s[1] = lt * (REAL)1.0 + tm * e11;
    s[2] = lt * (REAL)0.0 + tm * e01;
  } else if (t == MAT_NEOHOOKEAN) {
    REAL cdet = C00 * C11 - C01 * C10;
    REAL i00 = 0, i01 = 0, i11 = 0;
    if (cdet != (REAL)0) {
      REAL r = (REAL)1.0 / cdet;
      i00 = C11 * r;
      i01 = -C01 * r;
      i11 = C00 * r;
    }
    REAL J = F00 * F11 - F01 * F10;
    REAL c = lam * R_LOG(J) - mu;
    s[0] = c * i00 + mu * (REAL)1.0;
    s[1] = c * i11 + mu * (REAL)1.0;
    s[2] = c * i01 + mu * (REAL)0.0;
  } else {
    s[0] = s[1] = s[2] = 0;
  }
}

/* _fem_internal_force_kernel (femspringmanager.py:217-280): writes the three
 * corner forces -(B^T S)*A of element e into out[6] and updates J2 state. */
static void element_force(or_world* w, int e, REAL* out) {
  if (w->type[e] == MAT_SPRING) { /* _spring_force_kernel (femspringmanager.py:283-312) */
    int a = w->conn[3 * e], b = w->conn[3 * e + 1];
    REAL xx = w->x[2 * a] - w->x[2 * b], xy = w->x[2 * a + 1] - w->x[2 * b + 1];
    REAL lnew = R_SQRT(xx * xx + xy * xy);
    REAL dx = xx / lnew, dy = xy / lnew;
    REAL sc = w->E[e] * (lnew / w->area[e] - (REAL)1.0);
    REAL fx = sc * dx, fy = sc * dy;
    REAL vx = w->v[2 * a] - w->v[2 * b], vy = w->v[2 * a + 1] - w->v[2 * b + 1];
    REAL dmp = w->nu[e] * (vx * dx + vy * dy); /* nu slot: damping */
    fx = fx + dmp * dx;
    fy = fy + dmp * dy;
    out[0] = -fx; out[1] = -fy; out[2] = fx; out[3] = fy; out[4] = 0; out[5] = 0;
    return;
  }
  int n1 = w->conn[3 * e], n2 = w->conn[3 * e + 1], n3 = w->conn[3 * e + 2];
  const REAL* x = w->x;
  REAL j00 = x[2 * n1] - x[2 * n3], j01 = x[2 * n2] - x[2 * n3];
  REAL j10 = x[2 * n1 + 1] - x[2 * n3 + 1], j11 = x[2 * n2 + 1] - x[2 * n3 + 1];
  const REAL* ji = w->jinv + 4 * e;
  REAL F00 = j00 * ji[0] + j01 * ji[2];
  REAL F01 = j00 * ji[1] + j01 * ji[3];
  REAL F10 = j10 * ji[0] + j11 * ji[2];
  REAL F11 = j10 * ji[1] + j11 * ji[3];
  /* get_b_matrix_2d (femspringmanager.py:71-105) */
  REAL d00 = ji[0], d01 = ji[1], d10 = ji[2], d11 = ji[3];
  REAL d20 = -ji[0] - ji[2], d21 = -ji[1] - ji[3];
  REAL B[3][6];
  B[0][0] = d00 * F00; B[0][1] = d00 * F10;
  B[1][0] = d01 * F01; B[1][1] = d01 * F11;
  B[2][0] = d01 * F00 + d00 * F01; B[2][1] = d00 * F11 + d01 * F10;
  B[0][2] = d10 * F00; B[0][3] = d10 * F10;
  B[1][2] = d11 * F01; B[1][3] = d11 * F11;
  B[2][2] = d11 * F00 + d10 * F01; B[2][3] = d10 * F11 + d11 * F10;
  B[0][4] = d20 * F00; B[0][5] = d20 * F10;
  B[1][4] = d21 * F01; B[1][5] = d21 * F11;
  B[2][4] = d21 * F00 + d20 * F01; B[2][5] = d20 * F11 + d21 * F10;
  REAL s[3], ep[3], eq;
  stress(w, e, F00, F01, F10, F11, s, ep, &eq);
  if (w->type[e] == MAT_MISES) {
    w->epsp[3 * e] = ep[0];
    w->epsp[3 * e + 1] = ep[1];
    w->epsp[3 * e + 2] = ep[2];
    w->eqps[e] = eq;
  }
  REAL a = w->area[e];
  for (int r = 0; r < 6; ++r) {
    REAL fi = B[0][r] * s[0] + B[1][r] * s[1] + B[2][r] * s[2];
    fi = fi * a;
    out[r] = -fi;
  }
}

/* _nearest_on_curve_2d (mixedcontact.py:166-217): returns n and signed. */
static REAL hf_signed(const or_pair* c, REAL px, REAL pz, REAL* nx_out, REAL* ny_out) {
  REAL span = c->hubx - c->hlbx;
  REAL u = 0;
  if (span > (REAL)1e-12) u = (px - c->hlbx) / span;
  if (u < (REAL)0.0) u = 0;
  if (u > (REAL)1.0) u = 1;
  int nx = c->hnx;
  REAL s = u * (REAL)(nx - 1);
  int i0 = (int)R_FLOOR(s);
  int i1 = i0 + 1;
  if (i1 >= nx) i1 = nx - 1;
  if (i0 < 0) i0 = 0;
  REAL t = s - (REAL)i0;
  REAL h = c->h[i0] + (c->h[i1] - c->h[i0]) * t;
  int ir = (int)R_ROUND(s);
  if (ir < 0) ir = 0;
  if (ir >= nx) ir = nx - 1;
  int j0 = ir - 1, j1 = ir + 1;
  if (j0 < 0) j0 = 0;
  if (j1 >= nx) j1 = nx - 1;
  REAL dxw = span / (REAL)(nx - 1);
  REAL denom = dxw * (REAL)(j1 - j0);
  REAL dhdx = 0;
  if (denom > (REAL)1e-6) dhdx = (c->h[j1] - c->h[j0]) / denom;
  REAL n0 = -dhdx, n1 = (REAL)1.0;
  if (c->reverse == 1) {
    n0 = -n0;
    n1 = -n1;
  }
  REAL nl = R_SQRT(n0 * n0 + n1 * n1);
  if (nl > (REAL)1e-12) {
    n0 = n0 / nl;
    n1 = n1 / nl;
  }
  *nx_out = n0;
  *ny_out = n1;
  return (px - px) * n0 + (pz - h) * n1;
}

/* _voxel_signed_distance_2d (mixedcontact.py:220-302). */
static REAL voxel_signed(const or_pair* c, REAL px, REAL py, REAL* nx_out, REAL* ny_out) {
  REAL best_d = (REAL)1e9;
  REAL b0 = 0, b1 = 1;
  int nx = c->vnx, ny = c->vny;
  int i = (int)R_FLOOR((px - c->vlb[0]) / c->vdx);
  int j = (int)R_FLOOR((py - c->vlb[1]) / c->vdz);
  if (0 <= i && i < nx && 0 <= j && j < ny && c->occ[i * ny + j] == 1) {
    REAL dnx = (REAL)1e9, dpx = (REAL)1e9, dny = (REAL)1e9, dpy = (REAL)1e9;
    for (int st = 0; st < nx; ++st) {
      int idx = i - 1 - st;
      if (idx < 0 || c->occ[idx * ny + j] == 0) {
        dnx = px - (c->vlb[0] + (REAL)(idx + 1) * c->vdx);
        break;
      }
    }
    for (int st = 0; st < nx; ++st) {
      int idx = i + 1 + st;
      if (idx >= nx || c->occ[idx * ny + j] == 0) {
        dpx = (c->vlb[0] + (REAL)idx * c->vdx) - px;
        break;
      }
    }
    for (int st = 0; st < ny; ++st) {
      int idx = j - 1 - st;
      if (idx < 0 || c->occ[i * ny + idx] == 0) {
        dny = py - (c->vlb[1] + (REAL)(idx + 1) * c->vdz);
        break;
      }
    }
    for (int st = 0; st < ny; ++st) {
      int idx = j + 1 + st;
      if (idx >= ny || c->occ[i * ny + idx] == 0) {
        dpy = (c->vlb[1] + (REAL)idx * c->vdz) - py;
        break;
      }
    }
    REAL mv = dnx;
    int face = 0;
    if (dpx < mv) { mv = dpx; face = 1; }
    if (dny < mv) { mv = dny; face = 2; }
    if (dpy < mv) { mv = dpy; face = 3; }
    if (face == 0) { best_d = -dnx; b0 = -1; b1 = 0; }
    else if (face == 1) { best_d = -dpx; b0 = 1; b1 = 0; }
    else if (face == 2) { best_d = -dny; b0 = 0; b1 = -1; }
    else { best_d = -dpy; b0 = 0; b1 = 1; }
  }
  *nx_out = b0;
  *ny_out = b1;
  return best_d;
}

/* Pair gate: the broad phase reports (fem, ground) when their leaf boxes
 * overlap (bvh.py:40-46 inclusive test).  On steps with counter % 100 == 0 the
 * tree is rebuilt from boxes grown by 10% of their extent (bvh.py:321-342); on
 * the other steps the leaves are refit to the raw boxes (bvh.py:393-416). */
static const REAL* rigid_domain_box(const or_world* w, int r); /* a rigid manager entry's current box */

static int pair_active(const or_world* w, const or_pair* c, long counter) {
  const REAL* bb = w->aabb + 4 * c->body;
  REAL alo[2] = {bb[0], bb[1]}, ahi[2] = {bb[2], bb[3]};
  REAL blo[2] = {c->glb[0], c->glb[1]}, bhi[2] = {c->gub[0], c->gub[1]};
  if (c->entry >= 0) {
    const REAL* e = rigid_domain_box(w, c->entry);
    blo[0] = e[0]; blo[1] = e[1]; bhi[0] = e[2]; bhi[1] = e[3];
  }
  if (counter % 100 == 0) {
    for (int k = 0; k < 2; ++k) {
      REAL ba = (REAL)0.1 * (ahi[k] - alo[k]);
      REAL bbuf = (REAL)0.1 * (bhi[k] - blo[k]);
      alo[k] = alo[k] - ba;
      ahi[k] = ahi[k] + ba;
      blo[k] = blo[k] - bbuf;
      bhi[k] = bhi[k] + bbuf;
    }
  }
  return alo[0] <= bhi[0] && ahi[0] >= blo[0] && alo[1] <= bhi[1] && ahi[1] >= blo[1];
}

/* planes: the pairs of kind PAIR_PLANE (launched before FEM-FEM contact);
 * otherwise the height-field and voxel pairs (launched after it). */
static void contacts(or_world* w, REAL dt, long counter, int planes) {
  for (int pi = 0; pi < w->n_pairs; ++pi) {
    const or_pair* c = &w->pairs[pi];
    if ((c->kind == PAIR_PLANE) != (planes != 0)) continue;
    if (!pair_active(w, c, counter)) continue;
    int off = w->bn_off[c->body], cnt = w->bn_cnt[c->body];
    for (int k = 0; k < cnt; ++k) {
      int nid = w->bnodes[off + k];
      REAL px = w->x[2 * nid], py = w->x[2 * nid + 1];
      REAL vx = w->v[2 * nid], vy = w->v[2 * nid + 1];
      REAL fx = 0, fy = 0;
      int hit = 0;
      if (c->kind == PAIR_PLANE) {
        REAL pen = (px - c->p[0]) * c->n[0] + (py - c->p[1]) * c->n[1];
        if (pen < (REAL)0.0) {
          fx = -(c->n[0] * c->penalty * pen);
          fy = -(c->n[1] * c->penalty * pen);
          hit = 1;
        }
      } else if (c->kind == PAIR_HEIGHTFIELD) {
        REAL n0, n1;
        REAL sg = hf_signed(c, px, py, &n0, &n1);
        if (sg < (REAL)0.0) {
          fx = -n0 * c->penalty * sg;
          fy = -n1 * c->penalty * sg;
          REAL vn = vx * n0 + vy * n1;
          if (vn < (REAL)0.0) {
            fx = fx + (-n0 * (REAL)0.5 * c->penalty * vn * dt);
            fy = fy + (-n1 * (REAL)0.5 * c->penalty * vn * dt);
          }
          hit = 1;
        }
      } else {
        REAL n0, n1;
        REAL sd = voxel_signed(c, px, py, &n0, &n1);
        if (sd < (REAL)0.0) {
          REAL pen = -sd;
          fx = n0 * c->penalty * pen;
          fy = n1 * c->penalty * pen;
          REAL vn = vx * n0 + vy * n1;
          if (vn < (REAL)0.0) {
            fx = fx + (-n0 * (REAL)0.5 * c->penalty * vn * dt);
            fy = fy + (-n1 * (REAL)0.5 * c->penalty * vn * dt);
          }
          hit = 1;
        }
      }
      if (hit) {
        w->fext[2 * nid] += fx;
        w->fext[2 * nid + 1] += fy;
      }
    }
  }
}

/* _integrate_nodes_kernel (femspringmanager.py:315-358) for node i. */
static void integrate_node(or_world* w, int i, REAL dt, REAL damping) {
  int bc = w->bc[i];
  REAL fx = w->fext[2 * i], fy = w->fext[2 * i + 1];
  REAL m = w->mass[i];
  REAL bx = w->bcv[2 * i], by = w->bcv[2 * i + 1];
  if (bc & BC_U) {
    fx = 0;
    fy = 0;
  } else if (bc & BC_A) {
    fx = m * bx;
    fy = m * by;
  } else if (bc & BC_GRAVITY) {
    fx = fx + m * bx;
    fy = fy + m * by;
  } else if (bc & BC_FORCE) {
    fx = fx + bx;
    fy = fy + by;
  }
  REAL vx = w->v[2 * i], vy = w->v[2 * i + 1];
  REAL im = (REAL)1.0 / m;
  REAL ax = (REAL)0.0 + (fx - damping * vx) * im;
  REAL ay = (REAL)0.0 + (fy - damping * vy) * im;
  REAL nvx = vx + ax * dt, nvy = vy + ay * dt;
  if (bc & BC_V) {
    nvx = bx;
    nvy = by;
  } else if (bc & BC_U) {
    nvx = 0;
    nvy = 0;
  }
  w->v[2 * i] = nvx;
  w->v[2 * i + 1] = nvy;
  REAL dux = nvx * dt, duy = nvy * dt;
  w->u[2 * i] = w->u[2 * i] + dux;
  w->u[2 * i + 1] = w->u[2 * i + 1] + duy;
  w->x[2 * i] = w->x[2 * i] + dux;
  w->x[2 * i + 1] = w->x[2 * i + 1] + duy;
}

/* _update_bbox_kernel (femspringmanager.py:361-408). */
static void update_bbox(or_world* w) {
  for (int b = 0; b < w->n_bodies; ++b) {
    REAL lbx = (REAL)1e30, lby = (REAL)1e30, ubx = (REAL)-1e30, uby = (REAL)-1e30;
    for (int k = 0; k < w->bn_cnt[b]; ++k) {
      int nid = w->bnodes[w->bn_off[b] + k];
      REAL px = w->x[2 * nid], py = w->x[2 * nid + 1];
      lbx = lbx < px ? lbx : px;
      lby = lby < py ? lby : py;
      ubx = ubx > px ? ubx : px;
      uby = uby > py ? uby : py;
    }
    w->aabb[4 * b] = lbx;
    w->aabb[4 * b + 1] = lby;
    w->aabb[4 * b + 2] = ubx;
    w->aabb[4 * b + 3] = uby;
  }
}

static void build_csr(or_world* w) {
  int N = w->n_nodes, E = w->n_elems;
  w->csr_off = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  w->csr_slot = (int32_t*)malloc(sizeof(int32_t) * (3 * (size_t)E + 1));
  w->corner = (REAL*)malloc(sizeof(REAL) * (6 * (size_t)E + 1));
  for (int e = 0; e < E; ++e)
    for (int c = 0; c < 3; ++c)
      if (w->conn[3 * e + c] >= 0) w->csr_off[w->conn[3 * e + c] + 1]++;
  for (int i = 0; i < N; ++i) w->csr_off[i + 1] += w->csr_off[i];
  int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * ((size_t)N + 1));
  for (int i = 0; i < N; ++i) fill[i] = w->csr_off[i];
  for (int e = 0; e < E; ++e)
    for (int c = 0; c < 3; ++c)
      if (w->conn[3 * e + c] >= 0) w->csr_slot[fill[w->conn[3 * e + c]]++] = 3 * e + c;
  free(fill);
}


/* ------------------------------------------------------------ threading */

typedef struct {
  or_world* w;
  int lo, hi;
  REAL dt, damping;
  void (*fn)(or_world*, int, int, REAL, REAL);
} par_job;

static void elem_range(or_world* w, int lo, int hi, REAL dt, REAL damping) {
  (void)dt;
  (void)damping;
  for (int e = lo; e < hi; ++e) element_force(w, e, w->corner + 6 * (size_t)e);
}

static void node_range(or_world* w, int lo, int hi, REAL dt, REAL damping) {
  for (int i = lo; i < hi; ++i) {
    REAL fx = w->fext[2 * i], fy = w->fext[2 * i + 1];
    for (int k = w->csr_off[i]; k < w->csr_off[i + 1]; ++k) {
      int s = w->csr_slot[k];
      int e = s / 3, c = s % 3;
      fx += w->corner[6 * (size_t)e + 2 * c];
      fy += w->corner[6 * (size_t)e + 2 * c + 1];
    }
    w->fext[2 * i] = fx;
    w->fext[2 * i + 1] = fy;
    integrate_node(w, i, dt, damping);
  }
}

static void* par_worker(void* arg) {
  par_job* j = (par_job*)arg;
  j->fn(j->w, j->lo, j->hi, j->dt, j->damping);
  return NULL;
}

static REAL g_step_dt, g_step_damping;

static void par_for(or_world* w, int n, void (*fn)(or_world*, int, int, REAL, REAL)) {
  int T = w->n_threads;
  if (T > 256) T = 256;
  pthread_t th[256];
  par_job jobs[256];
  int chunk = (n + T - 1) / T;
  for (int t = 0; t < T; ++t) {
    jobs[t].w = w;
    jobs[t].lo = t * chunk < n ? t * chunk : n;
    jobs[t].hi = (t + 1) * chunk < n ? (t + 1) * chunk : n;
    jobs[t].dt = g_step_dt;
    jobs[t].damping = g_step_damping;
    jobs[t].fn = fn;
    if (t > 0) pthread_create(&th[t], NULL, par_worker, &jobs[t]);
  }
  par_worker(&jobs[0]);
  for (int t = 1; t < T; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------- FEM-FEM contact
 *
 * One reference ExplicitLoop with ContactFlexFlex pairs.  Work items, in the
 * reference's order (mixedcontact.py:1876-1924): per pair (contact-creation
 * order) the boundary nodes of domain2 against domain1's boundary edges, then
 * those of domain1 against domain2's.  The spatial hash and the contact kernel
 * are restated with the serial semantics of Warp's CPU device: atomic counters
 * hand out indices in launch order, so every hash cell lists its elements in
 * registration order, and each work item's candidate list is its own (the
 * reference's GPU launch shares one 512-entry candidate array among all work
 * items, spatialmanager.py:564, mixedcontact.py:2545, which is a race; the
 * serial semantics are the race-free reading).  Contact forces go to fext in
 * work-item order: node, then the edge's two nodes (atomic_add in launch
 * order). */
#define FLEX_MAX_QUERY 512       /* SpatialHashManager max_query_results */
#define FLEX_MAX_CELLS 100000    /* SpatialHashManager max_cells */

typedef struct or_flex {
  int n_items, n_pairs, n_fem, n_dom, skip_bvh;
  int32_t *item_node, *item_target, *item_be_off, *item_be_cnt, *item_pair, *item_cache;
  REAL *item_pen, *item_fric;
  int32_t *pair_b1, *pair_b2; /* domain1, domain2 (fem-local = body index) */
  int n_be;
  int32_t *be;      /* 2 per boundary edge: global node ids */
  int32_t *be_off, *be_cnt; /* per fem domain */
  int32_t *dom_obj, *dom_body; /* per scene domain: BVH object?, body (or -1) */
  REAL* dom_box;    /* 4 per domain: static box of a ground domain */
  /* hash */
  int max_elements, max_pairs;
  int n_reg, tc, cnx, cny;
  REAL estimate, olx, oly, gsx, gsy;
  REAL* ebox;                 /* 4 per registered element */
  int32_t *edom, *eid;        /* domain id, element id per registered element */
  int32_t *pair_cell, *pair_elem, *sorted, *cell_count, *cell_offset, *cell_start, *cell_end;
  int32_t cand[FLEX_MAX_QUERY];
  /* tied pairs (ExplicitLoop(ties=...)): per work item */
  int32_t *item_tied, *tie_resolved, *tie_elem;
  REAL *tie_w0, *tie_w1, *tie_gap;
  int n_tied, tie_initialized;
} or_flex;

static REAL rmin(REAL a, REAL b) { return a < b ? a : b; }
static REAL rmax(REAL a, REAL b) { return a > b ? a : b; }

/* pointToEdgeContact (contact_detection.py:15-61) */
static void point_edge(REAL px, REAL py, REAL ax, REAL ay, REAL bx, REAL by, REAL* pen, REAL* nx,
                       REAL* ny, int* inside, REAL* w0, REAL* w1) {
  REAL ex = bx - ax, ey = by - ay;
  REAL len = R_SQRT(ex * ex + ey * ey);
  *pen = (REAL)1e9;
  *nx = 0;
  *ny = 0;
  *inside = 0;
  *w0 = 0;
  *w1 = 0;
  if (len > (REAL)1e-9) {
    REAL dx = ex / len, dy = ey / len;
    *nx = dy;
    *ny = -dx;
    REAL tx = px - ax, ty = py - ay;
    REAL t = tx * dx + ty * dy;
    t = t / len;
    if ((REAL)0.0 <= t && t <= (REAL)1.0) {
      *inside = 1;
      *pen = tx * *nx + ty * *ny;
      *w0 = (REAL)1.0 - t;
      *w1 = t;
    }
  }
}

/* detectPointToMeshBoundary (contact_detection.py:63-92): the penetration is
 * kept only when |pen| < limit and the point projects inside the edge;
 * the weights are pointToEdgeContact's either way. */
static REAL detect_edge(const or_world* w, REAL px, REAL py, int e, REAL limit, REAL* nx, REAL* ny,
                        REAL* w0, REAL* w1) {
  const or_flex* f = w->flex;
  int a = f->be[2 * e], b = f->be[2 * e + 1];
  REAL pen, mx, my;
  int inside;
  point_edge(px, py, w->x[2 * a], w->x[2 * a + 1], w->x[2 * b], w->x[2 * b + 1], &pen, &mx, &my, &inside, w0, w1);
  *nx = 0;
  *ny = 0;
  if (R_FABS(pen) < limit && inside) {
    *nx = mx;
    *ny = my;
    return pen;
  }
  return (REAL)1e9;
}

static int cell_coord(REAL d, REAL gs, int n) {
  int c = (int)R_FLOOR(d / gs);
  c = c > 0 ? c : 0;
  c = c < n - 1 ? c : n - 1;
  return c;
}

/* FemSpringManager.populate_fem_spatial_hash(0.0) (femspringmanager.py:1041-1063,
 * _populate_fem_spatial_hash_kernel) + SpatialHashManager.reset/build
 * (spatialmanager.py:200-420, 613-712), serial. */
void or_flex_rebuild(or_world* w) {
  or_flex* f = w->flex;
  if (!f) return;
  f->n_reg = 0;
  f->estimate = (REAL)1e30;
  f->tc = 0;
  REAL glx = (REAL)1e9, gly = (REAL)1e9, gux = (REAL)-1e9, guy = (REAL)-1e9;
  for (int d = 0; d < f->n_fem; ++d) {
    const REAL* bb = w->aabb + 4 * d;
    glx = rmin(glx, bb[0]);
    gly = rmin(gly, bb[1]);
    gux = rmax(gux, bb[2]);
    guy = rmax(guy, bb[3]);
  }
  REAL extent = rmax(gux - glx, guy - gly);
  REAL expand = extent * (REAL)0.01 + (REAL)0.0;
  glx = glx - expand;
  gly = gly - expand;
  gux = gux + expand;
  guy = guy + expand;
  for (int d = 0; d < f->n_fem; ++d)
    for (int k = 0; k < f->be_cnt[d]; ++k) {
      int e = f->be_off[d] + k;
      REAL lx = (REAL)1e30, ly = (REAL)1e30, ux = (REAL)-1e30, uy = (REAL)-1e30;
      for (int c = 0; c < 2; ++c) {
        int nid = f->be[2 * e + c];
        lx = rmin(lx, w->x[2 * nid]);
        ly = rmin(ly, w->x[2 * nid + 1]);
        ux = rmax(ux, w->x[2 * nid]);
        uy = rmax(uy, w->x[2 * nid + 1]);
      }
      int idx = f->n_reg++;
      if (idx < f->max_elements) {
        f->edom[idx] = d;
        f->eid[idx] = e;
        REAL blx = lx - (REAL)0.0, bly = ly - (REAL)0.0, bux = ux + (REAL)0.0, buy = uy + (REAL)0.0;
        f->ebox[4 * idx] = blx;
        f->ebox[4 * idx + 1] = bly;
        f->ebox[4 * idx + 2] = bux;
        f->ebox[4 * idx + 3] = buy;
        REAL ddx = bux - blx, ddy = buy - bly;
        REAL diag = R_SQRT(ddx * ddx + ddy * ddy);
        f->estimate = rmin(f->estimate, diag);
      }
    }
  f->olx = glx;
  f->oly = gly;
  /* _build_grid_kernel */
  REAL cell = f->estimate * (REAL)1.5;
  REAL exx = gux - glx, exy = guy - gly;
  REAL mpd = R_POW((REAL)FLEX_MAX_CELLS, (REAL)0.5);
  mpd = rmax(mpd, (REAL)1.0);
  cell = rmax(cell, exx / mpd);
  cell = rmax(cell, exy / mpd);
  REAL cs = cell + (REAL)1e-6;
  int nx = (int)rmax(R_CEIL(exx / cs), (REAL)1.0);
  int ny = (int)rmax(R_CEIL(exy / cs), (REAL)1.0);
  f->cnx = nx;
  f->cny = ny;
  f->gsx = exx / (REAL)nx;
  f->gsy = exy / (REAL)ny;
  int total = nx * ny;
  f->tc = total < FLEX_MAX_CELLS ? total : FLEX_MAX_CELLS;
  int ne = f->n_reg;
  if (ne == 0) return;
  if (ne > f->max_elements) ne = f->max_elements;
  /* _expand_pairs_kernel, serial */
  int npairs = 0;
  for (int i = 0; i < ne; ++i) {
    const REAL* eb = f->ebox + 4 * i;
    int lx = cell_coord(eb[0] - glx, f->gsx, nx), ly = cell_coord(eb[1] - gly, f->gsy, ny);
    int ux = cell_coord(eb[2] - glx, f->gsx, nx), uy = cell_coord(eb[3] - gly, f->gsy, ny);
    for (int ix = lx; ix <= ux; ++ix)
      for (int iy = ly; iy <= uy; ++iy) {
        int cid = ix + iy * nx;
        if (cid < f->tc) {
          int p = npairs++;
          if (p < f->max_pairs) {
            f->pair_cell[p] = cid;
            f->pair_elem[p] = i;
          }
        }
      }
  }
  int np_ = npairs < f->max_pairs ? npairs : f->max_pairs;
  for (int c = 0; c < f->tc; ++c) f->cell_count[c] = 0;
  for (int p = 0; p < np_; ++p) {
    int cid = f->pair_cell[p];
    if (0 <= cid && cid < f->tc) f->cell_count[cid] += 1;
  }
  if (f->tc > 0) {
    f->cell_offset[0] = 0;
    for (int c = 1; c < f->tc; ++c) f->cell_offset[c] = f->cell_offset[c - 1] + f->cell_count[c - 1];
  }
  for (int c = 0; c < f->tc; ++c) f->cell_count[c] = f->cell_offset[c];
  for (int p = 0; p < np_; ++p) {
    int cid = f->pair_cell[p];
    if (0 <= cid && cid < f->tc) {
      int dest = f->cell_count[cid]++;
      if (dest < f->max_pairs) f->sorted[dest] = f->pair_elem[p];
    }
  }
  for (int c = 0; c < f->tc; ++c) {
    f->cell_start[c] = f->cell_offset[c];
    f->cell_end[c] = f->cell_count[c];
  }
}

/* query_point_with_buffer (spatialmanager.py:126-197) with this item's own
 * candidate list. */
static int flex_query(or_flex* f, REAL px, REAL py, REAL buf, int domain) {
  int num = 0;
  if (f->tc <= 0) return 0;
  REAL qlx = px - buf, qly = py - buf, qux = px + buf, quy = py + buf;
  int lx = cell_coord(qlx - f->olx, f->gsx, f->cnx), ly = cell_coord(qly - f->oly, f->gsy, f->cny);
  int ux = cell_coord(qux - f->olx, f->gsx, f->cnx), uy = cell_coord(quy - f->oly, f->gsy, f->cny);
  for (int ix = lx; ix <= ux; ++ix)
    for (int iy = ly; iy <= uy; ++iy) {
      int cid = ix + iy * f->cnx;
      if (0 <= cid && cid < f->tc)
        for (int p = f->cell_start[cid]; p < f->cell_end[cid]; ++p) {
          int ei = f->sorted[p];
          if (ei >= 0 && f->edom[ei] == domain) {
            int id = f->eid[ei], dup = 0;
            for (int k = 0; k < num; ++k)
              if (f->cand[k] == id) dup = 1;
            if (!dup && num < FLEX_MAX_QUERY) f->cand[num++] = id;
          }
        }
    }
  return num;
}

static int boxes_overlap(const REAL* a, const REAL* b, long counter) {
  REAL alo[2] = {a[0], a[1]}, ahi[2] = {a[2], a[3]};
  REAL blo[2] = {b[0], b[1]}, bhi[2] = {b[2], b[3]};
  if (counter % 100 == 0) {
    for (int k = 0; k < 2; ++k) {
      REAL ba = (REAL)0.1 * (ahi[k] - alo[k]);
      REAL bbuf = (REAL)0.1 * (bhi[k] - blo[k]);
      alo[k] = alo[k] - ba;
      ahi[k] = ahi[k] + ba;
      blo[k] = blo[k] - bbuf;
      bhi[k] = bhi[k] + bbuf;
    }
  }
  return alo[0] <= bhi[0] && ahi[0] >= blo[0] && alo[1] <= bhi[1] && ahi[1] >= blo[1];
}

static const REAL* dom_box(const or_world* w, int g) {
  const or_flex* f = w->flex;
  if (f->dom_body[g] <= -2) return rigid_domain_box(w, -2 - f->dom_body[g]);
  return f->dom_body[g] >= 0 ? w->aabb + 4 * f->dom_body[g] : f->dom_box + 4 * g;
}

/* _batched_flexflex_contact_kernel_sh (mixedcontact.py:886-1018), serial.
 * Pair activation (mixedcontact.py:1662-1665, 2282-2291): every pair when the
 * loop skips the BVH (explicitloop.py:367-373), else the BVH overlap of the two
 * domain boxes.  Domain mask (explicitloop.py:501-511, mixedcontact.py:925): a
 * work item runs only if the domain whose GLOBAL index equals the item's target
 * FEM-local index appears in some BVH pair this step -- the reference indexes
 * the global stamp array with the FEM-local id; restated as written. */
/* _eval_fixed_tie_point and _fem_fem_tie_elem_normal (mixedcontact.py:136-163). */
static void tie_point(const or_world* w, int e, REAL w0, REAL w1, REAL* cx, REAL* cy) {
  const or_flex* f = w->flex;
  int a = f->be[2 * e], b = f->be[2 * e + 1];
  REAL x = 0, y = 0;
  x = x + w->x[2 * a] * w0;
  y = y + w->x[2 * a + 1] * w0;
  x = x + w->x[2 * b] * w1;
  y = y + w->x[2 * b + 1] * w1;
  *cx = x;
  *cy = y;
}
static void tie_normal(const or_world* w, int e, REAL* nx, REAL* ny) {
  const or_flex* f = w->flex;
  int a = f->be[2 * e], b = f->be[2 * e + 1];
  REAL ex = w->x[2 * b] - w->x[2 * a], ey = w->x[2 * b + 1] - w->x[2 * a + 1];
  REAL el = R_SQRT(ex * ex + ey * ey);
  REAL tx = 1, ty = 0;
  if (el > (REAL)1e-10) {
    tx = ex / el;
    ty = ey / el;
  }
  *nx = -ty;
  *ny = tx;
}

/* Tied pairs (mixedcontact.py:1680-1690): once, at the first substep, every
 * tied work item finds the boundary edge of its target domain nearest to its
 * node (_initialize_fem_fem_ties_once_kernel, mixedcontact.py:686-771) and
 * keeps its edge, weights and normal gap; then, every substep, a penalty
 * spring pulls the node to that point of the edge, with the reactions on the
 * edge's nodes (_apply_fem_fem_ties_fixed_kernel, mixedcontact.py:774-809).
 * Launched before the contact kernel, which skips tied items. */
static void flex_ties(or_world* w) {
  or_flex* f = w->flex;
  if (!f->tie_initialized) {
    REAL qbuf = rmax(rmax((REAL)1e-4, rmax(f->gsx, f->gsy)), (REAL)0.001);
    for (int it = 0; it < f->n_items; ++it) {
      if (!f->item_tied[it] || f->tie_resolved[it]) continue;
      int nid = f->item_node[it];
      REAL px = w->x[2 * nid], py = w->x[2 * nid + 1];
      REAL best = (REAL)1e9, bw0 = 0, bw1 = 0;
      int be = -1, found = 0;
      int n = flex_query(f, px, py, qbuf, f->item_target[it]);
      for (int j = 0; j < n; ++j) {
        int e = f->cand[j];
        REAL nx, ny, w0, w1;
        REAL pen = detect_edge(w, px, py, e, qbuf, &nx, &ny, &w0, &w1);
        if (R_FABS(pen) < R_FABS(best) && R_FABS(pen) < qbuf) {
          bw0 = w0;
          bw1 = w1;
          found = 1;
          be = e;
          best = pen;
        }
      }
      if (found) {
        REAL cx, cy, nx, ny;
        tie_point(w, be, bw0, bw1, &cx, &cy);
        REAL gx = px - cx, gy = py - cy;
        tie_normal(w, be, &nx, &ny);
        f->tie_resolved[it] = 1;
        f->tie_elem[it] = be;
        f->tie_w0[it] = bw0;
        f->tie_w1[it] = bw1;
        f->tie_gap[it] = gx * nx + gy * ny;
      }
    }
    f->tie_initialized = 1;
  }
  for (int it = 0; it < f->n_items; ++it) {
    if (!f->item_tied[it] || !f->tie_resolved[it]) continue;
    int nid = f->item_node[it], e = f->tie_elem[it];
    REAL w0 = f->tie_w0[it], w1 = f->tie_w1[it], gap = f->tie_gap[it], k = f->item_pen[it];
    REAL cx, cy, nx, ny;
    tie_point(w, e, w0, w1, &cx, &cy);
    tie_normal(w, e, &nx, &ny);
    REAL tx = cx + gap * nx, ty = cy + gap * ny;
    REAL mx = tx - w->x[2 * nid], my = ty - w->x[2 * nid + 1];
    REAL fx = k * mx, fy = k * my;
    int a = f->be[2 * e], b = f->be[2 * e + 1];
    w->fext[2 * nid] += fx;
    w->fext[2 * nid + 1] += fy;
    w->fext[2 * a] += -(fx * w0);
    w->fext[2 * a + 1] += -(fy * w0);
    w->fext[2 * b] += -(fx * w1);
    w->fext[2 * b + 1] += -(fy * w1);
  }
}

static void flex_contacts(or_world* w, long counter) {
  or_flex* f = w->flex;
  if (!f || f->n_items == 0) return;
  if (f->n_tied > 0) flex_ties(w);
  if (f->n_tied == f->n_items) return; /* the contact kernel runs only for untied items */
  int* active = (int*)malloc(sizeof(int) * (size_t)(f->n_pairs + 1));
  int* stamped = (int*)malloc(sizeof(int) * (size_t)(f->n_fem + 1));
  for (int p = 0; p < f->n_pairs; ++p)
    active[p] = f->skip_bvh ? 1 : boxes_overlap(w->aabb + 4 * f->pair_b1[p], w->aabb + 4 * f->pair_b2[p], counter);
  for (int g = 0; g < f->n_fem; ++g) {
    stamped[g] = 0;
    if (g < f->n_dom && f->dom_obj[g])
      for (int h = 0; h < f->n_dom; ++h)
        if (h != g && f->dom_obj[h] && boxes_overlap(dom_box(w, g), dom_box(w, h), counter)) stamped[g] = 1;
  }
  REAL qbuf = rmax(rmax((REAL)1e-4, rmax(f->gsx, f->gsy)), (REAL)0.016);
  for (int it = 0; it < f->n_items; ++it) {
    if (f->item_tied[it]) continue;
    if (!active[f->item_pair[it]]) continue;
    int target = f->item_target[it];
    if (!f->skip_bvh && !stamped[target]) continue;
    int nid = f->item_node[it];
    int be_off = f->item_be_off[it], be_cnt = f->item_be_cnt[it];
    REAL px = w->x[2 * nid], py = w->x[2 * nid + 1];
    REAL vx = w->v[2 * nid], vy = w->v[2 * nid + 1];
    REAL pen_k = f->item_pen[it], fric = f->item_fric[it];
    REAL best = (REAL)1e9, bnx = 0, bny = 0, bw0 = 0, bw1 = 0;
    int bn0 = 0, bn1 = 0, found = 0;
    int cached = f->item_cache[it];
    if (cached >= be_off && cached < be_off + be_cnt) {
      int a = f->be[2 * cached], b = f->be[2 * cached + 1];
      REAL lx = (REAL)1e30, ly = (REAL)1e30, ux = (REAL)-1e30, uy = (REAL)-1e30;
      lx = rmin(lx, w->x[2 * a]); ly = rmin(ly, w->x[2 * a + 1]);
      ux = rmax(ux, w->x[2 * a]); uy = rmax(uy, w->x[2 * a + 1]);
      lx = rmin(lx, w->x[2 * b]); ly = rmin(ly, w->x[2 * b + 1]);
      ux = rmax(ux, w->x[2 * b]); uy = rmax(uy, w->x[2 * b + 1]);
      REAL dx = ux - lx, dy = uy - ly;
      REAL margin = rmax((REAL)1e-4, (REAL)1e-2 * R_SQRT(dx * dx + dy * dy));
      lx = lx - margin; ly = ly - margin; ux = ux + margin; uy = uy + margin;
      int outside = rmin(px - lx, py - ly) < (REAL)0.0 || rmin(ux - px, uy - py) < (REAL)0.0;
      if (!outside) {
        REAL nx, ny, w0, w1;
        REAL pen = detect_edge(w, px, py, cached, margin, &nx, &ny, &w0, &w1);
        if (pen < (REAL)1e-4 && R_FABS(pen) < margin) {
          best = pen; bnx = nx; bny = ny; bw0 = w0; bw1 = w1; bn0 = a; bn1 = b; found = 1;
        }
      }
    }
    if (!found) {
      int n = flex_query(f, px, py, qbuf, target);
      for (int j = 0; j < n; ++j) {
        int e = f->cand[j];
        REAL nx, ny, w0, w1;
        REAL pen = detect_edge(w, px, py, e, qbuf, &nx, &ny, &w0, &w1);
        if (pen < best && pen < (REAL)1e-4 && R_FABS(pen) < qbuf) {
          best = pen; bnx = nx; bny = ny; bw0 = w0; bw1 = w1;
          bn0 = f->be[2 * e]; bn1 = f->be[2 * e + 1]; found = 1;
          f->item_cache[it] = e;
        }
      }
    }
    if (!found) f->item_cache[it] = -1;
    if (found && best < (REAL)0.0) {
      REAL fx = -bnx * pen_k * best, fy = -bny * pen_k * best;
      REAL tx = fx, ty = fy;
      if (fric > (REAL)1e-9) {
        REAL sx = w->v[2 * bn0] * bw0 + w->v[2 * bn1] * bw1;
        REAL sy = w->v[2 * bn0 + 1] * bw0 + w->v[2 * bn1 + 1] * bw1;
        REAL rx = vx - sx, ry = vy - sy;
        REAL dn = rx * bnx + ry * bny;
        REAL gx = rx - dn * bnx, gy = ry - dn * bny;
        REAL tl = R_SQRT(gx * gx + gy * gy);
        if (tl > (REAL)1e-9) {
          REAL dx = -gx / tl, dy = -gy / tl;
          REAL nl = R_SQRT(fx * fx + fy * fy);
          tx = tx + dx * fric * nl;
          ty = ty + dy * fric * nl;
        }
      }
      w->fext[2 * nid] += tx;
      w->fext[2 * nid + 1] += ty;
      w->fext[2 * bn0] += -(tx * bw0);
      w->fext[2 * bn0 + 1] += -(ty * bw0);
      w->fext[2 * bn1] += -(tx * bw1);
      w->fext[2 * bn1 + 1] += -(ty * bw1);
    }
  }
  free(active);
  free(stamped);
}

/* ------------------------------------------------ FEM-rigid (primitives) */

/* sin and cos of the FP32 builds, from IEEE + - * only, so that the CUDA
 * kernels evaluating the same operations in the same order give the same bits
 * (the reference's wp.sin / wp.cos are the platform's; any accurate pair is a
 * faithful reading).  Method: Cody-Waite reduction x = k pi/2 + r with pi/2
 * split into 1.5703125 + 0x1.fb4p-12 + 0x1.4442d2p-24 (the first two short
 * enough that k times them is exact for |k| < 2^13), then the Taylor series of
 * sin through r^9 and of cos through r^10 on |r| <= pi/4 (truncation error
 * below 2e-9), and the quadrant k mod 4.  USE_LIBM_MATH builds call the C
 * library's sinf and cosf instead, as the reference's Warp CPU device does. */
static void or_sincosf(float x, float* s_out, float* c_out) {
  const float k = floorf(x * 0.63661975f + 0.5f);
  const float r = ((x - k * 1.5703125f) - k * 4.837512969970703125e-4f) - k * 0x1.4442d2p-24f;
  const float z = r * r;
  const float sp = -1.0f / 6.0f + z * (1.0f / 120.0f + z * (-1.0f / 5040.0f + z * (1.0f / 362880.0f)));
  const float sr = r + r * z * sp;
  const float cp = -0.5f + z * (1.0f / 24.0f + z * (-1.0f / 720.0f + z * (1.0f / 40320.0f + z * (-1.0f / 3628800.0f))));
  const float cr = 1.0f + z * cp;
  const int q = ((int)k) & 3;
  *s_out = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
  *c_out = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
}

static void r_sincos(REAL x, REAL* s, REAL* c) {
#if defined(REAL_IS_DOUBLE)
  *s = sin(x);
  *c = cos(x);
#elif defined(USE_LIBM_MATH)
  *s = sinf(x);
  *c = cosf(x);
#else
  or_sincosf(x, s, c);
#endif
}

/* RigidType (flatworld/definitions.py:50-53); 64: an analytical entry of the
 * rigid manager (ground plane, height field, voxel grid) in a loop where some
 * ground plane has BCs (rigidmanager.py:2486-2517) */
#define RIGID_BALL 1
#define RIGID_BOX 2
#define RIGID_CAPSULE 8
#define RIGID_ANALYTICAL 64
/* rigid BC bits (definitions.py:96-104) */
#define RBC_U 0x1
#define RBC_V 0x2
#define RBC_A 0x4
#define RBC_FORCE 0x8
#define RBC_GRAVITY 0x10
#define RBC_R 0x20
#define RBC_ROTV 0x40
#define RBC_ROTA 0x80
#define RBC_TORQUE 0x100

typedef struct {
  int type, bc, in_contact;
  REAL c[2], prim[2], radius, quat, mass, inertia;
  REAL V[2], W, bcT[2], bcG[2], bcR, U[2];
  REAL rot[4]; /* cached_rotation_matrix (row-major), refreshed by the velocity pass */
  REAL acc[2], accw;
  REAL lb[2], ub[2];
  REAL box[4]; /* lb x, y, ub x, y: the rigid's box as a broad-phase domain box */
} or_rigid;

typedef struct or_rigids {
  int n, n_ground, err;
  or_rigid* r;
  REAL* gbox;  /* static grounds, 4 per ground: plane p x, y, n x, y or box lb x, y, ub x, y */
  int* gkind; /* 0: plane, 1: box (height field, voxel grid) */
  /* work items, reference order: per rigid pair its FEM body's boundary nodes */
  int n_rp;
  int *rp_body, *rp_rigid, *rp_skip, *rp_tied;
  REAL *rp_pen, *rp_fric;
} or_rigids;

static const REAL* rigid_domain_box(const or_world* w, int r) { return w->rig->r[r].box; }

/* cal2DRotationMat (flatworld/utils.py:7-11): [[c, -s], [s, c]]. */
static void rot_of(REAL theta, REAL* m) {
  REAL s, c;
  r_sincos(theta, &s, &c);
  m[0] = c; m[1] = -s; m[2] = s; m[3] = c;
}

/* _write_primitive_aabb (rigidmanager.py:766-794) with getBallBBox,
 * getBoxBBox, getCapsuleBBox (utils.py:235-300). */
static void rigid_aabb(or_rigid* g) {
  const REAL* m = g->rot;
  if (g->type == RIGID_ANALYTICAL) { /* _update_u_and_bbox_wp's moving-plane box (rigidmanager.py:950-964) */
    const REAL nx = m[0] * g->prim[0] + m[1] * g->prim[1], ny = m[2] * g->prim[0] + m[3] * g->prim[1];
    const REAL tx = -ny, ty = nx;
    const REAL lox = g->c[0] - tx * (REAL)100.0 - nx * (REAL)0.1, loy = g->c[1] - ty * (REAL)100.0 - ny * (REAL)0.1;
    const REAL hix = g->c[0] + tx * (REAL)100.0 + nx * (REAL)0.1, hiy = g->c[1] + ty * (REAL)100.0 + ny * (REAL)0.1;
    g->lb[0] = rmin(lox, hix); g->lb[1] = rmin(loy, hiy);
    g->ub[0] = rmax(lox, hix); g->ub[1] = rmax(loy, hiy);
  } else if (g->type == RIGID_BALL) {
    g->lb[0] = g->c[0] - g->radius; g->lb[1] = g->c[1] - g->radius;
    g->ub[0] = g->c[0] + g->radius; g->ub[1] = g->c[1] + g->radius;
  } else if (g->type == RIGID_BOX) {
    const REAL ex = g->prim[0], ey = g->prim[1];
    REAL px[4], py[4];
    const REAL vx[4] = {ex, ex, ex, -ex}, vy[4] = {ey, -ey, ey, ey};
    const REAL sc[4] = {(REAL)-0.5, (REAL)0.5, (REAL)0.5, (REAL)0.5};
    for (int k = 0; k < 4; ++k) {
      const REAL rx = m[0] * vx[k] + m[1] * vy[k], ry = m[2] * vx[k] + m[3] * vy[k];
      px[k] = g->c[0] + sc[k] * rx;
      py[k] = g->c[1] + sc[k] * ry;
    }
    g->lb[0] = rmin(rmin(px[0], px[1]), rmin(px[2], px[3]));
    g->lb[1] = rmin(rmin(py[0], py[1]), rmin(py[2], py[3]));
    g->ub[0] = rmax(rmax(px[0], px[1]), rmax(px[2], px[3]));
    g->ub[1] = rmax(rmax(py[0], py[1]), rmax(py[2], py[3]));
  } else if (g->type == RIGID_CAPSULE) {
    const REAL ax = g->prim[0], ay = g->prim[1];
    const REAL alen = R_SQRT(ax * ax + ay * ay);
    const REAL d0 = ax / alen, d1 = ay / alen;
    const REAL dx = m[0] * d0 + m[1] * d1, dy = m[2] * d0 + m[3] * d1;
    const REAL p0x = g->c[0] - dx * alen, p0y = g->c[1] - dy * alen;
    const REAL p1x = g->c[0] + dx * alen, p1y = g->c[1] + dy * alen;
    const REAL perp0 = g->radius * R_SQRT(rmax((REAL)0.0, (REAL)1.0 - dx * dx)), axial0 = g->radius * R_FABS(dx);
    const REAL perp1 = g->radius * R_SQRT(rmax((REAL)0.0, (REAL)1.0 - dy * dy)), axial1 = g->radius * R_FABS(dy);
    g->lb[0] = rmin(p0x, p1x) - perp0 - axial0;
    g->lb[1] = rmin(p0y, p1y) - perp1 - axial1;
    g->ub[0] = rmax(p0x, p1x) + perp0 + axial0;
    g->ub[1] = rmax(p0y, p1y) + perp1 + axial1;
  }
  g->box[0] = g->lb[0]; g->box[1] = g->lb[1]; g->box[2] = g->ub[0]; g->box[3] = g->ub[1];
}

/* detectPointToPrimitive (contact_detection.py:148-190) with sphereSDFQuery,
 * capsuleSDFQuery, obbSDFQuery and calMinDisNode2Segment (utils.py:34-145). */
static REAL detect_prim(const or_rigid* g, REAL px, REAL py, REAL* nx, REAL* ny, REAL* cx, REAL* cy) {
  REAL pen = (REAL)1e9, n0 = 0, n1 = 0;
  const REAL* m = g->rot;
  if (g->type == RIGID_BALL) {
    const REAL qx = px - g->c[0], qy = py - g->c[1];
    const REAL len = R_SQRT(qx * qx + qy * qy);
    pen = len - g->radius;
    const REAL dn = rmax(len, (REAL)1e-9);
    n0 = qx / dn;
    n1 = qy / dn;
  } else if (g->type == RIGID_BOX) {
    const REAL hx = (REAL)0.5 * g->prim[0], hy = (REAL)0.5 * g->prim[1];
    const REAL wx = px - g->c[0], wy = py - g->c[1];
    const REAL lx = m[0] * wx + m[2] * wy, ly = m[1] * wx + m[3] * wy; /* transpose(rot) @ w */
    const REAL sd0 = lx - hx, sd1 = -lx - hx, sd2 = ly - hy, sd3 = -ly - hy;
    REAL best = (REAL)-1e9, ln0 = 0, ln1 = 0;
    if (sd0 > best) { best = sd0; ln0 = 1; ln1 = 0; }
    if (sd1 > best) { best = sd1; ln0 = -1; ln1 = 0; }
    if (sd2 > best) { best = sd2; ln0 = 0; ln1 = 1; }
    if (sd3 > best) { best = sd3; ln0 = 0; ln1 = -1; }
    if (sd0 > 0 || sd1 > 0 || sd2 > 0 || sd3 > 0) {
      REAL qx = lx, qy = ly;
      if (lx < -hx) qx = -hx; else if (lx > hx) qx = hx;
      if (ly < -hy) qy = -hy; else if (ly > hy) qy = hy;
      const REAL ddx = lx - qx, ddy = ly - qy;
      const REAL dist = R_SQRT(ddx * ddx + ddy * ddy);
      if (dist > (REAL)1e-9) { ln0 = ddx / dist; ln1 = ddy / dist; }
      best = dist;
    }
    pen = best;
    n0 = m[0] * ln0 + m[1] * ln1;
    n1 = m[2] * ln0 + m[3] * ln1;
  } else if (g->type == RIGID_CAPSULE) {
    const REAL lcx = g->c[0] + (m[0] * g->prim[0] + m[1] * g->prim[1]);
    const REAL lcy = g->c[1] + (m[2] * g->prim[0] + m[3] * g->prim[1]);
    const REAL qx = (REAL)2.0 * g->c[0] - lcx, qy = (REAL)2.0 * g->c[1] - lcy;
    const REAL apx = px - lcx, apy = py - lcy, abx = qx - lcx, aby = qy - lcy;
    const REAL ab2 = abx * abx + aby * aby;
    REAL t = (apx * abx + apy * aby) / ab2;
    t = rmax((REAL)0.0, rmin((REAL)1.0, t));
    const REAL clx = lcx + t * abx, cly = lcy + t * aby;
    const REAL ex = px - clx, ey = py - cly;
    const REAL dist = R_SQRT(ex * ex + ey * ey);
    pen = dist - g->radius;
    const REAL dn = rmax(dist, (REAL)1e-9);
    n0 = ex / dn;
    n1 = ey / dn;
  }
  *nx = n0;
  *ny = n1;
  *cx = px;
  *cy = py;
  if (pen < (REAL)0.0) {
    *cx = px - n0 * pen;
    *cy = py - n1 * pen;
  }
  return pen;
}

/* Gate of a FEM-rigid pair: the broad phase on the FEM body's box and the
 * rigid's current box (bvh.py rules as pair_active), or the plain box overlap
 * of _activate_pairs_by_aabb_kernel (mixedcontact.py:474-492) when the loop
 * skips the BVH. */
static int rigid_pair_active(const or_world* w, int body, const or_rigid* g, int skip, long counter) {
  const REAL* bb = w->aabb + 4 * body;
  REAL alo[2] = {bb[0], bb[1]}, ahi[2] = {bb[2], bb[3]};
  REAL blo[2] = {g->lb[0], g->lb[1]}, bhi[2] = {g->ub[0], g->ub[1]};
  if (!skip && counter % 100 == 0) {
    for (int k = 0; k < 2; ++k) {
      REAL ba = (REAL)0.1 * (ahi[k] - alo[k]);
      REAL bbuf = (REAL)0.1 * (bhi[k] - blo[k]);
      alo[k] = alo[k] - ba; ahi[k] = ahi[k] + ba;
      blo[k] = blo[k] - bbuf; bhi[k] = bhi[k] + bbuf;
    }
  }
  return alo[0] <= bhi[0] && ahi[0] >= blo[0] && alo[1] <= bhi[1] && ahi[1] >= blo[1];
}

/* _batched_rigid_prim_kernel (mixedcontact.py:1026-1115), its work items
 * serially in order; the reaction impulse and torque of each hit are added to
 * the rigid's accumulators in that order.  A tied pair pulls the node to the
 * contact point with no offset and no friction (1073-1087). */
static void rigid_contacts(or_world* w, REAL dt, long counter) {
  or_rigids* R = w->rig;
  if (!R) return;
  for (int pi = 0; pi < R->n_rp; ++pi) {
    or_rigid* g = &R->r[R->rp_rigid[pi]];
    const int body = R->rp_body[pi];
    if (!rigid_pair_active(w, body, g, R->rp_skip[pi], counter)) continue;
    const REAL k = R->rp_pen[pi], mu = R->rp_fric[pi];
    const int off = w->bn_off[body], cnt = w->bn_cnt[body];
    for (int q = 0; q < cnt; ++q) {
      const int nid = w->bnodes[off + q];
      const REAL px = w->x[2 * nid], py = w->x[2 * nid + 1];
      if (rmin(px - g->lb[0], py - g->lb[1]) < (REAL)0.0 || rmin(g->ub[0] - px, g->ub[1] - py) < (REAL)0.0) continue;
      REAL nx, ny, cx, cy;
      const REAL pen = detect_prim(g, px, py, &nx, &ny, &cx, &cy);
      const REAL gx = g->ub[0] - g->lb[0], gy = g->ub[1] - g->lb[1];
      const REAL margin = R_SQRT(gx * gx + gy * gy) * (REAL)0.5;
      if (!(pen < margin)) continue;
      if (R->rp_tied[pi]) {
        const REAL tx = k * (cx - px), ty = k * (cy - py);
        w->fext[2 * nid] += tx;
        w->fext[2 * nid + 1] += ty;
        g->acc[0] += -tx * dt;
        g->acc[1] += -ty * dt;
        const REAL lx = cx - g->c[0], ly = cy - g->c[1];
        const REAL fx = -tx, fy = -ty;
        g->accw += (lx * fy - ly * fx) * dt;
        continue;
      }
      const REAL depth = pen - (REAL)1e-4;
      if (!(depth < (REAL)0.0)) continue;
      const REAL fnx = -nx * k * depth, fny = -ny * k * depth;
      REAL tx = fnx, ty = fny;
      if (mu > (REAL)1e-9) {
        const REAL rx = cx - g->c[0], ry = cy - g->c[1];
        const REAL svx = g->V[0] + -g->W * ry, svy = g->V[1] + g->W * rx;
        const REAL relx = w->v[2 * nid] - svx, rely = w->v[2 * nid + 1] - svy;
        const REAL rn = relx * nx + rely * ny;
        const REAL tgx = relx - rn * nx, tgy = rely - rn * ny;
        const REAL tlen = R_SQRT(tgx * tgx + tgy * tgy);
        if (tlen > (REAL)1e-9) {
          const REAL dx = -tgx / tlen, dy = -tgy / tlen;
          const REAL fn = R_SQRT(fnx * fnx + fny * fny);
          tx = tx + dx * mu * fn;
          ty = ty + dy * mu * fn;
        }
      }
      w->fext[2 * nid] += tx;
      w->fext[2 * nid + 1] += ty;
      g->acc[0] += -tx * dt;
      g->acc[1] += -ty * dt;
      const REAL lx = cx - g->c[0], ly = cy - g->c[1];
      const REAL fx = -tx, fy = -ty;
      g->accw += (lx * fy - ly * fx) * dt;
    }
  }
}

/* Clearance below which a rigid counts as meeting a ground or another rigid:
 * 20x the reference's speculative rigid-ground contact margin (0.0005,
 * rigidmanager.py:3257), so that every state where the reference's constraint
 * solve could see a contact row is flagged. */
#define RIGID_CLEARANCE 0.01

/* The rigid bodies' part of RigidManager.substep (rigidmanager.py:2102-2197)
 * for worlds without rigid-rigid / rigid-ground contact and joints (no
 * constraint solve): _rigid_step_wp (832-891) then _update_u_and_bbox_wp
 * (894-964).  A rigid within RIGID_CLEARANCE of a ground plane (its box's
 * support point, as _detect_analytical_prim_contacts_wp's early out measures
 * it, rigidmanager.py:1127-1136), of a height-field / voxel box, or of another
 * contact rigid's box sets the error flag: such a world needs the solver. */
void or_rigid_update(or_world* w, float dt_f, float damping_f) {
  or_rigids* R = w->rig;
  if (!R) return;
  const REAL dt = (REAL)dt_f, damping = (REAL)damping_f, cl = (REAL)RIGID_CLEARANCE;
  for (int a = 0; a < R->n; ++a) {
    const or_rigid* g = &R->r[a];
    if (g->type == RIGID_ANALYTICAL) continue; /* not a rigid body */
    for (int q = 0; q < R->n_ground; ++q) {
      const REAL* b = R->gbox + 4 * q;
      /* written as "not clear", so that a non-finite box is flagged too */
      if (R->gkind[q] == 0) {
        const REAL sx = b[2] < 0 ? g->ub[0] : g->lb[0], sy = b[3] < 0 ? g->ub[1] : g->lb[1];
        if (!((sx - b[0]) * b[2] + (sy - b[1]) * b[3] > cl)) R->err = 1;
      } else if (!(g->lb[0] - cl > b[2] || g->ub[0] + cl < b[0] || g->lb[1] - cl > b[3] || g->ub[1] + cl < b[1])) {
        R->err = 1;
      }
    }
    for (int q = a + 1; q < R->n; ++q) {
      const or_rigid* h = &R->r[q];
      if (h->type != RIGID_ANALYTICAL && g->in_contact && h->in_contact &&
          !(g->lb[0] - cl > h->ub[0] || g->ub[0] + cl < h->lb[0] || g->lb[1] - cl > h->ub[1] ||
            g->ub[1] + cl < h->lb[1]))
        R->err = 1;
    }
    if (!(R_FABS(g->c[0]) < (REAL)1e30 && R_FABS(g->c[1]) < (REAL)1e30 && R_FABS(g->quat) < (REAL)1e30)) R->err = 1;
  }
  for (int a = 0; a < R->n; ++a) { /* _rigid_step_wp */
    or_rigid* g = &R->r[a];
    rot_of(g->quat, g->rot);
    if (g->type == RIGID_ANALYTICAL) continue; /* the impulse pass covers the rigid bodies only */
    if (g->bc & RBC_A) {
      g->acc[0] = 0; g->acc[1] = 0;
    } else {
      if (g->bc & RBC_GRAVITY) {
        g->acc[0] = g->acc[0] + g->mass * g->bcG[0] * dt;
        g->acc[1] = g->acc[1] + g->mass * g->bcG[1] * dt;
      }
      if (g->bc & RBC_FORCE) {
        g->acc[0] = g->acc[0] + g->bcT[0] * dt;
        g->acc[1] = g->acc[1] + g->bcT[1] * dt;
      }
    }
    if (g->bc & RBC_ROTA) g->accw = 0;
    else if (g->bc & RBC_TORQUE) g->accw = g->accw + g->bcR * dt;
    g->V[0] = g->V[0] + g->acc[0] / g->mass;
    g->V[1] = g->V[1] + g->acc[1] / g->mass;
    g->W = g->W + g->accw / (g->inertia + (REAL)1e-6);
    const REAL damp = rmax((REAL)0.0, (REAL)1.0 - damping * dt);
    g->V[0] = g->V[0] * damp;
    g->V[1] = g->V[1] * damp;
    g->W = g->W * damp;
  }
  for (int a = 0; a < R->n; ++a) {
    or_rigid* g = &R->r[a];
    if (g->bc & RBC_A) {
      g->V[0] = g->V[0] + g->bcT[0] * dt;
      g->V[1] = g->V[1] + g->bcT[1] * dt;
    }
    if (g->bc & RBC_ROTA) g->W = g->W + g->bcR * dt;
  }
  for (int a = 0; a < R->n; ++a) { /* _update_u_and_bbox_wp */
    or_rigid* g = &R->r[a];
    if (g->bc & RBC_V) {
      g->V[0] = g->bcT[0]; g->V[1] = g->bcT[1];
    } else if (g->bc & RBC_U) {
      g->V[0] = 0; g->V[1] = 0;
    } else if (g->bc & RBC_R) {
      g->V[0] = 0; g->V[1] = 0;
      g->W = 0;
    }
    if (g->bc & RBC_ROTV) g->W = g->bcR;
    const REAL dux = g->V[0] * dt, duy = g->V[1] * dt;
    g->U[0] = g->U[0] + dux; g->U[1] = g->U[1] + duy;
    g->c[0] = g->c[0] + dux; g->c[1] = g->c[1] + duy;
    g->quat = g->quat + g->W * dt;
    if (g->quat > (REAL)3.141592653589793) g->quat = g->quat - (REAL)2.0 * (REAL)3.141592653589793;
    else if (g->quat < (REAL)-3.141592653589793) g->quat = g->quat + (REAL)2.0 * (REAL)3.141592653589793;
  }
  for (int a = 0; a < R->n; ++a) {
    R->r[a].acc[0] = 0; R->r[a].acc[1] = 0; R->r[a].accw = 0;
  }
  for (int a = 0; a < R->n; ++a) rigid_aabb(&R->r[a]);
}

/* ---------------------------------------------------------------- C API */

or_world* or_create(int n_nodes, const float* x, const float* v, const int32_t* bc, const float* bcv,
                    int n_elems, const int32_t* conn, const int32_t* type, const float* E,
                    const float* nu, const float* rho, const float* sy, const float* H,
                    int n_bodies, const int32_t* bn_off, const int32_t* bn_cnt,
                    int n_bnodes, const int32_t* bnodes) {
  or_world* w = (or_world*)calloc(1, sizeof(or_world));
  w->n_nodes = n_nodes;
  w->n_elems = n_elems;
  w->n_bodies = n_bodies;
  w->n_threads = 1;
  w->x = dupf(x, 2 * (size_t)n_nodes);
  w->v = dupf(v, 2 * (size_t)n_nodes);
  w->u = (REAL*)calloc(2 * (size_t)n_nodes + 1, sizeof(REAL));
  w->fext = (REAL*)calloc(2 * (size_t)n_nodes + 1, sizeof(REAL));
  w->mass = (REAL*)calloc((size_t)n_nodes + 1, sizeof(REAL));
  w->bc = dupi(bc, n_nodes);
  w->bcv = dupf(bcv, 2 * (size_t)n_nodes);
  w->conn = dupi(conn, 3 * (size_t)n_elems);
  w->type = dupi(type, n_elems);
  w->E = dupf(E, n_elems);
  w->nu = dupf(nu, n_elems);
  w->rho = dupf(rho, n_elems);
  w->sy = dupf(sy, n_elems);
  w->H = dupf(H, n_elems);
  w->area = (REAL*)calloc((size_t)n_elems + 1, sizeof(REAL));
  w->jinv = (REAL*)calloc(4 * (size_t)n_elems + 1, sizeof(REAL));
  w->epsp = (REAL*)calloc(3 * (size_t)n_elems + 1, sizeof(REAL));
  w->eqps = (REAL*)calloc((size_t)n_elems + 1, sizeof(REAL));
  w->bn_off = dupi(bn_off, n_bodies);
  w->bn_cnt = dupi(bn_cnt, n_bodies);
  w->bnodes = dupi(bnodes, n_bnodes);
  w->aabb = (REAL*)calloc(4 * (size_t)n_bodies + 1, sizeof(REAL));
  w->pairs = NULL;
  w->n_pairs = 0;
  prepare(w);
  build_csr(w);
  return w;
}

static or_pair* new_pair(or_world* w) {
  w->pairs = (or_pair*)realloc(w->pairs, sizeof(or_pair) * (size_t)(w->n_pairs + 1));
  or_pair* c = &w->pairs[w->n_pairs++];
  memset(c, 0, sizeof(*c));
  c->entry = -1;
  return c;
}

/* The last ground pair added is gated by rigid manager entry `entry`'s box. */
int or_gate_by_rigid(or_world* w, int entry) {
  if (w->n_pairs == 0) return -1;
  w->pairs[w->n_pairs - 1].entry = entry;
  return 0;
}

/* Pairs must be added in launch order: planes, then heightfields, then voxels
 * (mixedcontact.py:1657-1754), each group in contact-creation order. */
int or_add_plane(or_world* w, int body, float penalty, const float* glb, const float* gub,
                 float px, float py, float nx, float ny) {
  or_pair* c = new_pair(w);
  c->kind = PAIR_PLANE;
  c->body = body;
  c->penalty = penalty;
  c->glb[0] = glb[0]; c->glb[1] = glb[1]; c->gub[0] = gub[0]; c->gub[1] = gub[1];
  c->p[0] = px; c->p[1] = py; c->n[0] = nx; c->n[1] = ny;
  return w->n_pairs - 1;
}

int or_add_heightfield(or_world* w, int body, float penalty, const float* glb, const float* gub,
                       int nx, const float* h, float lbx, float ubx, int reverse) {
  or_pair* c = new_pair(w);
  c->kind = PAIR_HEIGHTFIELD;
  c->body = body;
  c->penalty = penalty;
  c->glb[0] = glb[0]; c->glb[1] = glb[1]; c->gub[0] = gub[0]; c->gub[1] = gub[1];
  c->hnx = nx;
  c->h = dupf(h, nx);
  c->hlbx = lbx;
  c->hubx = ubx;
  c->reverse = reverse;
  return w->n_pairs - 1;
}

int or_add_voxel(or_world* w, int body, float penalty, const float* glb, const float* gub,
                 int nx, int ny, const int32_t* occ, float lbx, float lby, float dx, float dz) {
  or_pair* c = new_pair(w);
  c->kind = PAIR_VOXEL;
  c->body = body;
  c->penalty = penalty;
  c->glb[0] = glb[0]; c->glb[1] = glb[1]; c->gub[0] = gub[0]; c->gub[1] = gub[1];
  c->vnx = nx;
  c->vny = ny;
  c->occ = dupi(occ, (size_t)nx * ny);
  c->vlb[0] = lbx; c->vlb[1] = lby; c->vdx = dx; c->vdz = dz;
  return w->n_pairs - 1;
}

void or_set_threads(or_world* w, int n) { w->n_threads = n < 1 ? 1 : n; }

/* FEM-FEM contact set-up of one loop.  be: 2 global node ids per boundary
 * edge, the edges of fem domain d at be[be_off[d] ..], in mesh order
 * (mesh.py:53-71); dom_obj / dom_body / dom_box: per domain of the loop (in
 * loop order) whether it is a BVH object (considerContact), its body (fem
 * index, or -1 for a ground) and a ground's static box; skip_bvh: the loop has
 * no plane, height-field, voxel or unbatched ground contact. */
int or_set_flex(or_world* w, int n_be, const int32_t* be, const int32_t* be_off, const int32_t* be_cnt,
                int n_dom, const int32_t* dom_obj, const int32_t* dom_body, const float* dom_box, int skip_bvh) {
  or_flex* f = (or_flex*)calloc(1, sizeof(or_flex));
  f->n_fem = w->n_bodies;
  f->n_dom = n_dom;
  f->skip_bvh = skip_bvh;
  f->n_be = n_be;
  f->be = dupi(be, 2 * (size_t)n_be);
  f->be_off = dupi(be_off, w->n_bodies);
  f->be_cnt = dupi(be_cnt, w->n_bodies);
  f->dom_obj = dupi(dom_obj, n_dom);
  f->dom_body = dupi(dom_body, n_dom);
  f->dom_box = dupf(dom_box, 4 * (size_t)n_dom);
  /* femspringmanager.py:545-548, spatialmanager.py:520-525 */
  int max_nodes = w->n_nodes + 1024 > 2048 ? w->n_nodes + 1024 : 2048;
  f->max_elements = n_be + 1024 > max_nodes ? n_be + 1024 : max_nodes;
  f->max_pairs = f->max_elements * 9;
  f->ebox = (REAL*)calloc(4 * (size_t)f->max_elements, sizeof(REAL));
  f->edom = (int32_t*)calloc((size_t)f->max_elements, sizeof(int32_t));
  f->eid = (int32_t*)calloc((size_t)f->max_elements, sizeof(int32_t));
  f->pair_cell = (int32_t*)calloc((size_t)f->max_pairs, sizeof(int32_t));
  f->pair_elem = (int32_t*)calloc((size_t)f->max_pairs, sizeof(int32_t));
  f->sorted = (int32_t*)calloc((size_t)f->max_pairs, sizeof(int32_t));
  f->cell_count = (int32_t*)calloc(FLEX_MAX_CELLS, sizeof(int32_t));
  f->cell_offset = (int32_t*)calloc(FLEX_MAX_CELLS, sizeof(int32_t));
  f->cell_start = (int32_t*)calloc(FLEX_MAX_CELLS, sizeof(int32_t));
  f->cell_end = (int32_t*)calloc(FLEX_MAX_CELLS, sizeof(int32_t));
  w->flex = f;
  return 0;
}

/* One ContactFlexFlex pair (mixedcontact.py:1876-1924): domain1 = b1, domain2 =
 * b2 (fem indices); work items for b2's boundary nodes against b1's edges,
 * then b1's nodes against b2's edges. */
int or_add_flex_pair(or_world* w, int b1, int b2, float penalty, float friction) {
  or_flex* f = w->flex;
  if (!f) return -1;
  int p = f->n_pairs++;
  f->pair_b1 = (int32_t*)realloc(f->pair_b1, sizeof(int32_t) * (size_t)f->n_pairs);
  f->pair_b2 = (int32_t*)realloc(f->pair_b2, sizeof(int32_t) * (size_t)f->n_pairs);
  f->pair_b1[p] = b1;
  f->pair_b2[p] = b2;
  int add = w->bn_cnt[b1] + w->bn_cnt[b2];
  int n0 = f->n_items, n = n0 + add;
  f->item_node = (int32_t*)realloc(f->item_node, sizeof(int32_t) * (size_t)n);
  f->item_target = (int32_t*)realloc(f->item_target, sizeof(int32_t) * (size_t)n);
  f->item_be_off = (int32_t*)realloc(f->item_be_off, sizeof(int32_t) * (size_t)n);
  f->item_be_cnt = (int32_t*)realloc(f->item_be_cnt, sizeof(int32_t) * (size_t)n);
  f->item_pair = (int32_t*)realloc(f->item_pair, sizeof(int32_t) * (size_t)n);
  f->item_cache = (int32_t*)realloc(f->item_cache, sizeof(int32_t) * (size_t)n);
  f->item_pen = (REAL*)realloc(f->item_pen, sizeof(REAL) * (size_t)n);
  f->item_fric = (REAL*)realloc(f->item_fric, sizeof(REAL) * (size_t)n);
  f->item_tied = (int32_t*)realloc(f->item_tied, sizeof(int32_t) * (size_t)n);
  f->tie_resolved = (int32_t*)realloc(f->tie_resolved, sizeof(int32_t) * (size_t)n);
  f->tie_elem = (int32_t*)realloc(f->tie_elem, sizeof(int32_t) * (size_t)n);
  f->tie_w0 = (REAL*)realloc(f->tie_w0, sizeof(REAL) * (size_t)n);
  f->tie_w1 = (REAL*)realloc(f->tie_w1, sizeof(REAL) * (size_t)n);
  f->tie_gap = (REAL*)realloc(f->tie_gap, sizeof(REAL) * (size_t)n);
  for (int i = n0; i < n; ++i) {
    f->item_tied[i] = 0;
    f->tie_resolved[i] = 0;
    f->tie_elem[i] = -1;
    f->tie_w0[i] = f->tie_w1[i] = f->tie_gap[i] = 0;
  }
  int k = n0;
  for (int side = 0; side < 2; ++side) {
    int src = side == 0 ? b2 : b1, dst = side == 0 ? b1 : b2;
    for (int i = 0; i < w->bn_cnt[src]; ++i, ++k) {
      f->item_node[k] = w->bnodes[w->bn_off[src] + i];
      f->item_target[k] = dst;
      f->item_be_off[k] = f->be_off[dst];
      f->item_be_cnt[k] = f->be_cnt[dst];
      f->item_pair[k] = p;
      f->item_cache[k] = -1;
      f->item_pen[k] = penalty;
      f->item_fric[k] = friction;
    }
  }
  f->n_items = n;
  return p;
}

/* Mark the work items of flex pair p tied (explicitloop.py:265-270: the pair
 * is named in ExplicitLoop(ties=...)). */
int or_set_flex_pair_tied(or_world* w, int p, int tied) {
  or_flex* f = w->flex;
  if (!f || p < 0 || p >= f->n_pairs) return -1;
  for (int i = 0; i < f->n_items; ++i)
    if (f->item_pair[i] == p && f->item_tied[i] != (tied != 0)) {
      f->item_tied[i] = tied != 0;
      f->n_tied += tied ? 1 : -1;
    }
  return 0;
}
int or_flex_counts(const or_world* w, int32_t* out) {
  const or_flex* f = w->flex;
  out[0] = f ? f->n_items : 0;
  out[1] = f ? f->n_tied : 0;
  out[2] = f ? f->tie_initialized : 0;
  return 0;
}

/* _mass_scaling_kernel (femspringmanager.py:139-196), FEM triangles, serial in
 * element order. */
void or_mass_scaling(or_world* w, float dt_target_f) {
  REAL dt_target = (REAL)dt_target_f;
  for (int e = 0; e < w->n_elems; ++e) {
    if (w->type[e] == MAT_SPRING) continue;
    int n1 = w->conn[3 * e], n2 = w->conn[3 * e + 1], n3 = w->conn[3 * e + 2];
    REAL ax = w->x[2 * n1], ay = w->x[2 * n1 + 1], bx = w->x[2 * n2], by = w->x[2 * n2 + 1];
    REAL cx = w->x[2 * n3], cy = w->x[2 * n3 + 1];
    REAL e01x = bx - ax, e01y = by - ay, e12x = cx - bx, e12y = cy - by, e20x = ax - cx, e20y = ay - cy;
    REAL e01 = R_SQRT(e01x * e01x + e01y * e01y), e12 = R_SQRT(e12x * e12x + e12y * e12y);
    REAL e20 = R_SQRT(e20x * e20x + e20y * e20y);
    REAL L = rmin(e01, rmin(e12, e20));
    REAL E = w->E[e], rho = w->rho[e];
    REAL ce = R_SQRT(E / rho);
    REAL dt_elem = (REAL)0.4 * L / ce;
    if (dt_elem < dt_target && L > (REAL)1e-15) {
      REAL q = dt_target / ((REAL)0.4 * L);
      REAL rho_new = E * q * q;
      REAL dm = (rho_new - rho) * w->area[e] / (REAL)3.0;
      w->mass[n1] = w->mass[n1] + dm;
      w->mass[n2] = w->mass[n2] + dm;
      w->mass[n3] = w->mass[n3] + dm;
    }
  }
  for (int e = 0; e < w->n_elems; ++e) { /* springs: at least 4 k dt^2 per node */
    if (w->type[e] != MAT_SPRING) continue;
    REAL m_min = (REAL)4.0 * w->E[e] * dt_target * dt_target;
    for (int k = 0; k < 2; ++k) {
      int nid = w->conn[3 * e + k];
      if (w->mass[nid] < m_min) w->mass[nid] = m_min;
    }
  }
}

/* A spring-mass body's nodes (its boundary-node list: all of them) carry its
 * node mass (femspringmanager.py:844-845). */
void or_set_spring_mass(or_world* w, int body, float mass) {
  for (int k = 0; k < w->bn_cnt[body]; ++k) w->mass[w->bnodes[w->bn_off[body] + k]] = (REAL)mass;
}

/* The hash grid: tc, nx, ny, origin x, origin y, cell x, cell y, estimate. */
void or_get_flex_grid(const or_world* w, double* out) {
  const or_flex* f = w->flex;
  if (!f) return;
  out[0] = f->tc; out[1] = f->cnx; out[2] = f->cny; out[3] = f->olx; out[4] = f->oly;
  out[5] = f->gsx; out[6] = f->gsy; out[7] = f->estimate;
}

/* The per-item element cache (for tests). */
void or_get_flex_cache(const or_world* w, int32_t* out) {
  if (w->flex)
    for (int i = 0; i < w->flex->n_items; ++i) out[i] = w->flex->item_cache[i];
}

/* One FemSpringManager.femStep plus, unless init_step, the contact launches of
 * ExplicitLoop.advance that precede it.  init_step reproduces the zero-dt step
 * setGlobalAABB runs at construction (femspringmanager.py:872-879). */
void or_step(or_world* w, float dt_f, float damping_f, long counter, int init_step) {
  REAL dt = (REAL)dt_f, damping = (REAL)damping_f;
  int N = w->n_nodes, E = w->n_elems;
  g_step_dt = dt;
  g_step_damping = damping;
  for (int i = 0; i < 2 * N; ++i) w->fext[i] = 0;
  if (!init_step) {
    contacts(w, dt, counter, 1);
    flex_contacts(w, counter);
    rigid_contacts(w, dt, counter); /* mixedcontact.py:1697-1715: after FEM-FEM, before height fields */
    contacts(w, dt, counter, 0);
  }
  if (w->n_threads <= 1) {
    REAL f[6];
    for (int e = 0; e < E; ++e) {
      element_force(w, e, f);
      int n1 = w->conn[3 * e], n2 = w->conn[3 * e + 1], n3 = w->conn[3 * e + 2];
      w->fext[2 * n1] += f[0];
      w->fext[2 * n1 + 1] += f[1];
      w->fext[2 * n2] += f[2];
      w->fext[2 * n2 + 1] += f[3];
      if (n3 >= 0) {  /* a spring has two nodes */
        w->fext[2 * n3] += f[4];
        w->fext[2 * n3 + 1] += f[5];
      }
    }
    for (int i = 0; i < N; ++i) integrate_node(w, i, dt, damping);
  } else {
    /* Threaded variant: element forces into a corner buffer, then each node
     * sums its corners in ascending element order -- the same additions in
     * the same order as the serial scatter above, so identical bits. */
    par_for(w, E, elem_range);
    par_for(w, N, node_range);
  }
  update_bbox(w);
}

void or_get_state(const or_world* w, double* x, double* v, double* u) {
  for (int i = 0; i < 2 * w->n_nodes; ++i) {
    if (x) x[i] = (double)w->x[i];
    if (v) v[i] = (double)w->v[i];
    if (u) u[i] = (double)w->u[i];
  }
}

void or_get_prepared(const or_world* w, double* mass, double* area, double* jinv) {
  for (int i = 0; i < w->n_nodes; ++i)
    if (mass) mass[i] = (double)w->mass[i];
  for (int e = 0; e < w->n_elems; ++e) {
    if (area) area[e] = (double)w->area[e];
    for (int k = 0; k < 4; ++k)
      if (jinv) jinv[4 * e + k] = (double)w->jinv[4 * e + k];
  }
}

void or_get_plastic(const or_world* w, double* epsp, double* eqps) {
  for (int e = 0; e < w->n_elems; ++e) {
    for (int k = 0; k < 3; ++k)
      if (epsp) epsp[3 * e + k] = (double)w->epsp[3 * e + k];
    if (eqps) eqps[e] = (double)w->eqps[e];
  }
}

void or_get_aabb(const or_world* w, double* aabb) {
  for (int i = 0; i < 4 * w->n_bodies; ++i) aabb[i] = (double)w->aabb[i];
}

/* Copy x (and v) from float arrays: lets a test restart the oracle from a
 * state that the GPU produced, to measure one-step error in isolation. */
void or_set_state(or_world* w, const float* x, const float* v) {
  for (int i = 0; i < 2 * w->n_nodes; ++i) {
    if (x) w->x[i] = (REAL)x[i];
    if (v) w->v[i] = (REAL)v[i];
  }
}

/* Stress of one material point, for unit tests of the material laws
 * (test2D/test_2Dmaterial_functions.py:85-105). */
void or_point_stress(int type, float E, float nu, float sy, float H, const float* F,
                     const float* epsp_in, float eqps_in, double* s_out, double* epsp_out,
                     double* eqps_out) {
  or_world w;
  memset(&w, 0, sizeof(w));
  REAL Ev = E, nuv = nu, syv = sy, Hv = H, eqv = eqps_in;
  REAL ep[3] = {epsp_in ? epsp_in[0] : 0, epsp_in ? epsp_in[1] : 0, epsp_in ? epsp_in[2] : 0};
  int32_t t = type;
  w.E = &Ev; w.nu = &nuv; w.sy = &syv; w.H = &Hv; w.type = &t; w.epsp = ep; w.eqps = &eqv;
  REAL s[3], epo[3], eqo;
  stress(&w, 0, F[0], F[1], F[2], F[3], s, epo, &eqo);
  for (int k = 0; k < 3; ++k) {
    s_out[k] = s[k];
    if (epsp_out) epsp_out[k] = (type == MAT_MISES) ? epo[k] : ep[k];
  }
  if (eqps_out) *eqps_out = (type == MAT_MISES) ? eqo : eqv;
}

/* The oracle's FP32 log, exported for its accuracy test. */
float or_log32(float x) { return R_LOG(x); }

/* Rigid primitives (RigidManager.packRigidParams / processConditions,
 * rigidmanager.py:2250-2400, 2527-2567): per entry 20 floats (center x, y,
 * primary x, y, radius, angle, mass, inertia, V x, y, angular velocity, BC
 * translation value x, y, gravity x, y, BC rotation value, an analytical
 * entry's first box) and 3 ints (type,
 * BC bits, considerContact); the static grounds, 5 floats each (kind 0 plane:
 * p x, y, n x, y; kind 1 box: lb x, y, ub x, y).  The
 * rotation cache and boxes are set as precompute_rigid_transforms + updateBBox
 * do at loop construction (explicitloop.py:198-201). */
int or_set_rigids(or_world* w, int n, const float* f, const int32_t* iv, int n_ground, const float* grounds) {
  or_rigids* R = (or_rigids*)calloc(1, sizeof(or_rigids));
  R->n = n;
  R->r = (or_rigid*)calloc((size_t)(n ? n : 1), sizeof(or_rigid));
  for (int a = 0; a < n; ++a) {
    or_rigid* g = &R->r[a];
    const float* q = f + 20 * a;
    g->type = iv[3 * a]; g->bc = iv[3 * a + 1]; g->in_contact = iv[3 * a + 2];
    g->c[0] = q[0]; g->c[1] = q[1]; g->prim[0] = q[2]; g->prim[1] = q[3];
    g->radius = q[4]; g->quat = q[5]; g->mass = q[6]; g->inertia = q[7];
    g->V[0] = q[8]; g->V[1] = q[9]; g->W = q[10];
    g->bcT[0] = q[11]; g->bcT[1] = q[12]; g->bcG[0] = q[13]; g->bcG[1] = q[14]; g->bcR = q[15];
    rot_of(g->quat, g->rot);
    if (g->type == RIGID_ANALYTICAL) { /* an analytical entry starts at getBBox() */
      g->lb[0] = q[16]; g->lb[1] = q[17]; g->ub[0] = q[18]; g->ub[1] = q[19];
      g->box[0] = q[16]; g->box[1] = q[17]; g->box[2] = q[18]; g->box[3] = q[19];
    } else {
      rigid_aabb(g);
    }
  }
  R->n_ground = n_ground;
  R->gbox = (REAL*)calloc(4 * (size_t)(n_ground ? n_ground : 1), sizeof(REAL));
  R->gkind = (int*)calloc((size_t)(n_ground ? n_ground : 1), sizeof(int));
  for (int q = 0; q < n_ground; ++q) {
    R->gkind[q] = (int)grounds[5 * q];
    for (int k = 0; k < 4; ++k) R->gbox[4 * q + k] = grounds[5 * q + 1 + k];
  }
  w->rig = R;
  return 0;
}

/* One FEM-rigid pair (its work items: the body's boundary nodes), added in
 * the reference's rigid-contact order (mixedcontact.py:1987-2030). */
int or_add_rigid_pair(or_world* w, int body, int rigid, float penalty, float friction, int skip_bvh, int tied) {
  or_rigids* R = w->rig;
  if (!R || rigid < 0 || rigid >= R->n || body < 0 || body >= w->n_bodies) return -1;
  const int k = R->n_rp++;
  R->rp_body = (int*)realloc(R->rp_body, sizeof(int) * R->n_rp);
  R->rp_rigid = (int*)realloc(R->rp_rigid, sizeof(int) * R->n_rp);
  R->rp_skip = (int*)realloc(R->rp_skip, sizeof(int) * R->n_rp);
  R->rp_tied = (int*)realloc(R->rp_tied, sizeof(int) * R->n_rp);
  R->rp_pen = (REAL*)realloc(R->rp_pen, sizeof(REAL) * R->n_rp);
  R->rp_fric = (REAL*)realloc(R->rp_fric, sizeof(REAL) * R->n_rp);
  R->rp_body[k] = body; R->rp_rigid[k] = rigid; R->rp_skip[k] = skip_bvh; R->rp_tied[k] = tied;
  R->rp_pen[k] = penalty; R->rp_fric[k] = friction;
  return 0;
}

/* Per rigid 12 doubles: center x, y, angle, V x, y, angular velocity, U x, y,
 * box lb x, y, ub x, y.  Returns the error flag of the update pass. */
int or_get_rigids(const or_world* w, double* out) {
  const or_rigids* R = w->rig;
  if (!R) return 0;
  for (int a = 0; a < R->n; ++a) {
    const or_rigid* g = &R->r[a];
    double* o = out + 12 * a;
    o[0] = g->c[0]; o[1] = g->c[1]; o[2] = g->quat; o[3] = g->V[0]; o[4] = g->V[1]; o[5] = g->W;
    o[6] = g->U[0]; o[7] = g->U[1]; o[8] = g->lb[0]; o[9] = g->lb[1]; o[10] = g->ub[0]; o[11] = g->ub[1];
  }
  return R->err;
}

void or_sincos32(float x, float* s, float* c) { or_sincosf(x, s, c); }


void or_destroy(or_world* w) {
  if (!w) return;
  free(w->x); free(w->v); free(w->u); free(w->fext); free(w->mass); free(w->bc); free(w->bcv);
  free(w->conn); free(w->type); free(w->E); free(w->nu); free(w->rho); free(w->sy); free(w->H);
  free(w->area); free(w->jinv); free(w->epsp); free(w->eqps);
  free(w->bn_off); free(w->bn_cnt); free(w->bnodes); free(w->aabb);
  for (int i = 0; i < w->n_pairs; ++i) {
    free(w->pairs[i].h);
    free(w->pairs[i].occ);
  }
  free(w->pairs);
  free(w->csr_off); free(w->csr_slot); free(w->corner);
  if (w->rig) {
    or_rigids* R = w->rig;
    free(R->r); free(R->gbox); free(R->gkind); free(R->rp_body); free(R->rp_rigid); free(R->rp_skip); free(R->rp_tied); free(R->rp_pen);
    free(R->rp_fric);
    free(R);
  }
  if (w->flex) {
    or_flex* f = w->flex;
    free(f->item_node); free(f->item_target); free(f->item_be_off); free(f->item_be_cnt);
    free(f->item_pair); free(f->item_cache); free(f->item_pen); free(f->item_fric);
    free(f->pair_b1); free(f->pair_b2); free(f->be); free(f->be_off); free(f->be_cnt);
    free(f->dom_obj); free(f->dom_body); free(f->dom_box); free(f->ebox); free(f->edom); free(f->eid);
    free(f->item_tied); free(f->tie_resolved); free(f->tie_elem); free(f->tie_w0); free(f->tie_w1); free(f->tie_gap);
    free(f->pair_cell); free(f->pair_elem); free(f->sorted); free(f->cell_count); free(f->cell_offset);
    free(f->cell_start); free(f->cell_end);
    free(f);
  }
  free(w);
}

/* ======================================================================
 * Adjoint of the substep (reverse mode), restated in REAL arithmetic.  Test
 * infrastructure for the differentiable form: the FP64 build gives the exact
 * derivative of the FP64 trajectory, which the tests compare with FP64
 * central differences (the formula check) and with the CUDA adjoint (whose
 * remaining distance is the FP32 trajectory's own rounding).
 *
 * Forward substep of node i (femspringmanager.py:315-358, mixedcontact.py):
 *   f  = contact(x, v) + sum_e f_e(x, state_e; E_e) [+ gravity / nodal force]
 *   v' = v + dt (f - c v) / m     (enforced / fixed velocity: v' = bc)
 *   x' = x + dt v'
 * J2 triangles also update their plastic state: state' = g_e(x, state_e; E_e).
 * Reverse, from the adjoints (xb', vb', sb') of (x', v', state'):
 *   vt = vb' + dt xb'
 *   fb = (dt / m) vt          (0 for fixed / enforced-velocity / prescribed-
 *                              acceleration nodes)
 *   vb = (1 - dt c / m) vt + (d contact / d v)^T fb      (0 when v' is fixed)
 *   xb = xb' + sum_e (d f_e / d x)^T fb + (d contact / d x)^T fb
 *        + sum_e (d g_e / d x)^T sb'
 *   sb = sum (d f_e / d state)^T fb + (d g_e / d state)^T sb'
 *   Eb += (d f_e / d E)^T fb + (d g_e / d E)^T sb'
 * Every local Jacobian is taken column by column in forward mode (dual
 * numbers) through the same formulas as element_force / stress / contacts
 * above, so the derivative is that of this very code.  The broad-phase gates,
 * the contact branches, the height-field sample / normal indices, the voxel
 * cell and face, and the J2 yield branch are piecewise constant and are taken
 * from the recorded forward pass.
 * ====================================================================== */
typedef struct {
  REAL v, d;
} dual;
static dual D(REAL v, REAL d) { dual r = {v, d}; return r; }
static dual dc(REAL v) { return D(v, 0); }
static dual dadd(dual a, dual b) { return D(a.v + b.v, a.d + b.d); }
static dual dsub(dual a, dual b) { return D(a.v - b.v, a.d - b.d); }
static dual dneg(dual a) { return D(-a.v, -a.d); }
static dual dmul(dual a, dual b) { return D(a.v * b.v, a.d * b.v + a.v * b.d); }
static dual ddiv(dual a, dual b) {
  REAL q = a.v / b.v;
  return D(q, (a.d - q * b.d) / b.v);
}
static dual dlog_(dual a) { return D(R_LOG(a.v), a.d / a.v); }
static dual dsqrt_(dual a) {
  REAL s = R_SQRT(a.v);
  return D(s, s > 0 ? a.d / ((REAL)2.0 * s) : (REAL)0.0);
}

/* element_force + stress in dual numbers: X[6] corner positions, S[4] J2 state
 * (eps_p Voigt, eqps), E Young's modulus -> F[6] corner forces, SN[4] new state. */
static void element_dual(const or_world* w, int e, const dual* X, const dual* S, dual E, dual* F, dual* SN) {
  dual nu = dc(w->nu[e]);
  dual one = dc(1), two = dc(2), half = dc((REAL)0.5);
  dual lam = ddiv(dmul(E, nu), dmul(dadd(one, nu), dsub(one, dmul(two, nu))));
  dual mu = ddiv(E, dmul(two, dadd(one, nu)));
  dual j00 = dsub(X[0], X[4]), j01 = dsub(X[2], X[4]);
  dual j10 = dsub(X[1], X[5]), j11 = dsub(X[3], X[5]);
  const REAL* ji = w->jinv + 4 * e;
  dual F00 = dadd(dmul(j00, dc(ji[0])), dmul(j01, dc(ji[2])));
  dual F01 = dadd(dmul(j00, dc(ji[1])), dmul(j01, dc(ji[3])));
  dual F10 = dadd(dmul(j10, dc(ji[0])), dmul(j11, dc(ji[2])));
  dual F11 = dadd(dmul(j10, dc(ji[1])), dmul(j11, dc(ji[3])));
  REAL d00 = ji[0], d01 = ji[1], d10 = ji[2], d11 = ji[3];
  REAL d20 = -ji[0] - ji[2], d21 = -ji[1] - ji[3];
  dual C00 = dadd(dmul(F00, F00), dmul(F10, F10));
  dual C01 = dadd(dmul(F00, F01), dmul(F10, F11));
  dual C11 = dadd(dmul(F01, F01), dmul(F11, F11));
  dual e00 = dmul(half, dsub(C00, one)), e01 = dmul(half, C01), e11 = dmul(half, dsub(C11, one));
  dual s0, s1, s2;
  for (int k = 0; k < 4; ++k) SN[k] = S[k];
  int t = w->type[e];
  if (t == MAT_MISES) {
    dual t0 = dsub(e00, S[0]), t1 = dsub(e11, S[1]), t2 = dsub(e01, S[2]);
    dual tr = dadd(t0, t1);
    dual tm = dmul(two, mu);
    s0 = dadd(dmul(lam, tr), dmul(tm, t0));
    s1 = dadd(dmul(lam, tr), dmul(tm, t1));
    s2 = dmul(tm, t2);
    dual p = ddiv(dadd(s0, s1), dc(3));
    dual q0 = dsub(s0, p), q1 = dsub(s1, p), q2 = s2;
    dual vm = dsqrt_(dadd(dsub(dadd(dmul(q0, q0), dmul(q1, q1)), dmul(q0, q1)), dmul(dc(3), dmul(q2, q2))));
    dual f = dsub(vm, dadd(dc(w->sy[e]), dmul(dc(w->H[e]), S[3])));
    if (f.v > (REAL)0.0) {
      dual dg = ddiv(f, dadd(dmul(dc(3), mu), dc(w->H[e])));
      SN[3] = dadd(S[3], dg);
      dual scale = dsub(one, ddiv(dmul(dmul(dc(3), mu), dg), vm));
      s0 = dadd(dmul(q0, scale), p);
      s1 = dadd(dmul(q1, scale), p);
      s2 = dmul(q2, scale);
      SN[0] = dadd(S[0], dmul(dg, ddiv(q0, vm)));
      SN[1] = dadd(S[1], dmul(dg, ddiv(q1, vm)));
      SN[2] = dadd(S[2], dmul(dg, ddiv(q2, vm)));
    }
  } else if (t == MAT_ELASTIC) {
    dual lt = dmul(lam, dadd(e00, e11));
    dual tm = dmul(two, mu);
    s0 = dadd(lt, dmul(tm, e00));
    s1 = dadd(lt, dmul(tm, e11));
    s2 = dmul(tm, e01);
  } else {  /* NeoHookean */
    dual cdet = dsub(dmul(C00, C11), dmul(C01, C01));
    dual r = ddiv(one, cdet);
    dual i00 = dmul(C11, r), i01 = dneg(dmul(C01, r)), i11 = dmul(C00, r);
    dual J = dsub(dmul(F00, F11), dmul(F01, F10));
    dual c = dsub(dmul(lam, dlog_(J)), mu);
    s0 = dadd(dmul(c, i00), mu);
    s1 = dadd(dmul(c, i11), mu);
    s2 = dmul(c, i01);
  }
  dual B[3][6];
  B[0][0] = dmul(dc(d00), F00); B[0][1] = dmul(dc(d00), F10);
  B[1][0] = dmul(dc(d01), F01); B[1][1] = dmul(dc(d01), F11);
  B[2][0] = dadd(dmul(dc(d01), F00), dmul(dc(d00), F01)); B[2][1] = dadd(dmul(dc(d00), F11), dmul(dc(d01), F10));
  B[0][2] = dmul(dc(d10), F00); B[0][3] = dmul(dc(d10), F10);
  B[1][2] = dmul(dc(d11), F01); B[1][3] = dmul(dc(d11), F11);
  B[2][2] = dadd(dmul(dc(d11), F00), dmul(dc(d10), F01)); B[2][3] = dadd(dmul(dc(d10), F11), dmul(dc(d11), F10));
  B[0][4] = dmul(dc(d20), F00); B[0][5] = dmul(dc(d20), F10);
  B[1][4] = dmul(dc(d21), F01); B[1][5] = dmul(dc(d21), F11);
  B[2][4] = dadd(dmul(dc(d21), F00), dmul(dc(d20), F01)); B[2][5] = dadd(dmul(dc(d20), F11), dmul(dc(d21), F10));
  dual a = dc(w->area[e]);
  for (int r = 0; r < 6; ++r) {
    dual fi = dadd(dadd(dmul(B[0][r], s0), dmul(B[1][r], s1)), dmul(B[2][r], s2));
    F[r] = dneg(dmul(fi, a));
  }
}

/* contact force of pair c on a node at (px, py) with velocity (vx, vy), dual. */
static int contact_dual(const or_pair* c, REAL dt, dual px, dual py, dual vx, dual vy, dual* fx, dual* fy) {
  dual k = dc(c->penalty);
  if (c->kind == PAIR_PLANE) {
    dual pen = dadd(dmul(dsub(px, dc(c->p[0])), dc(c->n[0])), dmul(dsub(py, dc(c->p[1])), dc(c->n[1])));
    if (!(pen.v < (REAL)0.0)) return 0;
    *fx = dneg(dmul(dmul(dc(c->n[0]), k), pen));
    *fy = dneg(dmul(dmul(dc(c->n[1]), k), pen));
    return 1;
  }
  REAL n0, n1;
  dual sd;
  if (c->kind == PAIR_HEIGHTFIELD) {
    REAL sg = hf_signed(c, px.v, py.v, &n0, &n1);
    if (!(sg < (REAL)0.0)) return 0;
    /* the interpolated height h(x) is the only x-dependent part of sd */
    REAL span = c->hubx - c->hlbx;
    dual u = dc(0);
    if (span > (REAL)1e-12) u = ddiv(dsub(px, dc(c->hlbx)), dc(span));
    if (u.v < (REAL)0.0) u = dc(0);
    if (u.v > (REAL)1.0) u = dc(1);
    int nx = c->hnx;
    dual s = dmul(u, dc((REAL)(nx - 1)));
    int i0 = (int)R_FLOOR(s.v);
    int i1 = i0 + 1;
    if (i1 >= nx) i1 = nx - 1;
    if (i0 < 0) i0 = 0;
    dual t = dsub(s, dc((REAL)i0));
    dual h = dadd(dc(c->h[i0]), dmul(dc(c->h[i1] - c->h[i0]), t));
    sd = dadd(dmul(dsub(px, px), dc(n0)), dmul(dsub(py, h), dc(n1)));
    *fx = dmul(dmul(dc(-n0), k), sd);
    *fy = dmul(dmul(dc(-n1), k), sd);
  } else {
    REAL s = voxel_signed(c, px.v, py.v, &n0, &n1);
    if (!(s < (REAL)0.0)) return 0;
    /* sd = -(distance to the chosen face): linear in the position */
    dual pd = (n0 != 0) ? px : py;
    REAL nn = (n0 != 0) ? n0 : n1;
    REAL face = (n0 != 0 ? px.v : py.v) + nn * (-s); /* face coordinate */
    sd = dmul(dc(nn), dsub(pd, dc(face)));
    dual pen = dneg(sd);
    *fx = dmul(dmul(dc(n0), k), pen);
    *fy = dmul(dmul(dc(n1), k), pen);
  }
  dual vn = dadd(dmul(vx, dc(n0)), dmul(vy, dc(n1)));
  if (vn.v < (REAL)0.0) {
    *fx = dadd(*fx, dmul(dmul(dmul(dmul(dc(-n0), dc((REAL)0.5)), k), vn), dc(dt)));
    *fy = dadd(*fy, dmul(dmul(dmul(dmul(dc(-n1), dc((REAL)0.5)), k), vn), dc(dt)));
  }
  return 1;
}

/* Reverse-mode derivative of n substeps of dt from the current state (which
 * the call advances, like n forward substeps).  xbar_T / vbar_T (2N, NULL =
 * 0) seed the adjoint of the final positions / velocities; the outputs are
 * dL/dx0, dL/dv0 (2N) and dL/dE (E).  Returns -1 for worlds this restatement
 * does not cover (FEM-FEM contact, rigids, springs). */
int or_adjoint(or_world* w, int n, float dt_f, float damping_f, long counter0, const double* xbar_T,
               const double* vbar_T, double* xbar0, double* vbar0, double* Ebar) {
  if (w->flex || w->rig) return -1;
  int N = w->n_nodes, E = w->n_elems, P = w->n_pairs;
  for (int e = 0; e < E; ++e)
    if (w->type[e] == MAT_SPRING) return -1;
  REAL dt = (REAL)dt_f, damping = (REAL)damping_f;
  size_t n2 = 2 * (size_t)N;
  REAL* xs = (REAL*)malloc(sizeof(REAL) * n2 * (size_t)(n > 0 ? n : 1));
  REAL* vs = (REAL*)malloc(sizeof(REAL) * n2 * (size_t)(n > 0 ? n : 1));
  int has_j2 = 0;
  for (int e = 0; e < E; ++e) has_j2 |= w->type[e] == MAT_MISES;
  REAL* ss = (REAL*)malloc(sizeof(REAL) * 4 * (size_t)(has_j2 ? E : 1) * (size_t)(n > 0 ? n : 1));
  char* gates = (char*)malloc((size_t)(P > 0 ? P : 1) * (size_t)(n > 0 ? n : 1));
  for (int j = 0; j < n; ++j) {
    memcpy(xs + n2 * j, w->x, sizeof(REAL) * n2);
    memcpy(vs + n2 * j, w->v, sizeof(REAL) * n2);
    for (int e = 0; has_j2 && e < E; ++e) {
      REAL* s = ss + 4 * ((size_t)E * j + e);
      s[0] = w->epsp[3 * e]; s[1] = w->epsp[3 * e + 1]; s[2] = w->epsp[3 * e + 2]; s[3] = w->eqps[e];
    }
    for (int p = 0; p < P; ++p) gates[(size_t)P * j + p] = (char)pair_active(w, &w->pairs[p], counter0 + j);
    or_step(w, dt_f, damping_f, counter0 + j, 0);
  }
  double* xb = (double*)calloc(n2, sizeof(double));
  double* vb = (double*)calloc(n2, sizeof(double));
  double* fb = (double*)calloc(n2, sizeof(double));
  double* sb = (double*)calloc(4 * (size_t)E + 1, sizeof(double));
  double* sbn = (double*)calloc(4 * (size_t)E + 1, sizeof(double));
  for (size_t i = 0; i < n2; ++i) {
    xb[i] = xbar_T ? xbar_T[i] : 0.0;
    vb[i] = vbar_T ? vbar_T[i] : 0.0;
  }
  for (int e = 0; e < E; ++e) Ebar[e] = 0.0;
  for (int j = n - 1; j >= 0; --j) {
    const REAL* x = xs + n2 * j;
    const REAL* v = vs + n2 * j;
    /* node adjoints through v' and x' */
    for (int i = 0; i < N; ++i) {
      int bc = w->bc[i];
      int vfixed = (bc & (BC_U | BC_V)) != 0;
      int fdead = vfixed || (bc & BC_A) != 0;
      double sc = (double)dt / (double)w->mass[i];
      double keep = 1.0 - sc * (double)damping;
      for (int k = 0; k < 2; ++k) {
        double vt = vb[2 * i + k] + (double)dt * xb[2 * i + k];
        fb[2 * i + k] = fdead ? 0.0 : sc * vt;
        vb[2 * i + k] = vfixed ? 0.0 : keep * vt;
      }
    }
    /* elements: column by column of the local Jacobian */
    for (int e = 0; e < E; ++e) {
      int nd[3] = {w->conn[3 * e], w->conn[3 * e + 1], w->conn[3 * e + 2]};
      int j2 = w->type[e] == MAT_MISES;
      static const REAL s_zero[4] = {0, 0, 0, 0};
      const REAL* s0 = j2 ? ss + 4 * ((size_t)E * j + e) : s_zero;
      double outb[10];
      for (int r = 0; r < 6; ++r) outb[r] = fb[2 * nd[r / 2] + (r & 1)];
      for (int k = 0; k < 4; ++k) outb[6 + k] = j2 ? sb[4 * e + k] : 0.0;
      int nin = j2 ? 11 : 7; /* 6 positions, [4 state], E */
      for (int col = 0; col < nin; ++col) {
        dual X[6], S[4], Fo[6], SN[4];
        for (int r = 0; r < 6; ++r) X[r] = D(x[2 * nd[r / 2] + (r & 1)], col == r ? 1 : 0);
        for (int k = 0; k < 4; ++k) S[k] = D(s0[k], (j2 && col == 6 + k) ? 1 : 0);
        dual Ed = D(w->E[e], col == nin - 1 ? 1 : 0);
        element_dual(w, e, X, S, Ed, Fo, SN);
        double dot = 0.0;
        for (int r = 0; r < 6; ++r) dot += outb[r] * (double)Fo[r].d;
        if (j2)
          for (int k = 0; k < 4; ++k) dot += outb[6 + k] * (double)SN[k].d;
        if (col < 6) xb[2 * nd[col / 2] + (col & 1)] += dot;
        else if (col < nin - 1) sbn[4 * e + (col - 6)] = dot;
        else Ebar[e] += dot;
      }
    }
    for (int e = 0; e < 4 * E; ++e) sb[e] = sbn[e];
    /* contacts (gated as in the forward pass) */
    for (int p = 0; p < P; ++p) {
      if (!gates[(size_t)P * j + p]) continue;
      const or_pair* c = &w->pairs[p];
      for (int k = 0; k < w->bn_cnt[c->body]; ++k) {
        int i = w->bnodes[w->bn_off[c->body] + k];
        for (int col = 0; col < 4; ++col) {
          dual px = D(x[2 * i], col == 0), py = D(x[2 * i + 1], col == 1);
          dual vx = D(v[2 * i], col == 2), vy = D(v[2 * i + 1], col == 3);
          dual fx, fy;
          if (!contact_dual(c, dt, px, py, vx, vy, &fx, &fy)) break;
          double dot = fb[2 * i] * (double)fx.d + fb[2 * i + 1] * (double)fy.d;
          if (col < 2) xb[2 * i + col] += dot;
          else vb[2 * i + col - 2] += dot;
        }
      }
    }
  }
  for (size_t i = 0; i < n2; ++i) {
    xbar0[i] = xb[i];
    vbar0[i] = vb[i];
  }
  free(xs); free(vs); free(ss); free(gates); free(xb); free(vb); free(fb); free(sb); free(sbn);
  return 0;
}

/* FP64 inputs for central differences: Young's modulus per element and the
 * node state, set without a float32 round trip (the FP64 build keeps them). */
void or_set_young64(or_world* w, const double* E) {
  for (int e = 0; e < w->n_elems; ++e) w->E[e] = (REAL)E[e];
}
void or_set_state64(or_world* w, const double* x, const double* v) {
  for (int i = 0; i < 2 * w->n_nodes; ++i) {
    if (x) w->x[i] = (REAL)x[i];
    if (v) w->v[i] = (REAL)v[i];
  }
}
