// fw_world.cu -- C ABI (include/fwb200.h) and the general ("gather") step of
// the explicit 2D FEM world: any number of scenes, bodies and contact pairs.
//
// Per substep two kernels run on the context stream:
//   k_elements  one thread per triangle: deformation gradient, PK2 stress
//               (elastic / NeoHookean / J2 radial return), the three corner
//               forces -(B^T S)A written to a corner buffer kept in node
//               order (each corner at its place in its node's ascending-
//               element list, so a node reads one contiguous run).  Block 0 first
//               runs the per-step control (scene modes, broad-phase gates,
//               step counters, AABB slot reset).
//   k_nodes     one thread per node: penalty contact (boundary nodes only),
//               the node's corner forces summed in ascending element order,
//               boundary conditions, symplectic Euler, and the per-body AABB of
//               boundary nodes (warp reduction + ordered-int atomics).
// Summing a node's corners in ascending element order after its contact terms
// is exactly the order in which the reference's serial CPU path applies its
// atomic adds (flatworld/mixedcontact.py:1654-1755 then
// flatworld/femspringmanager.py:217-280), so the sum is deterministic and
// identical run to run, with no float atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <map>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fwb200.h"
#include "fw_device.cuh"
#include "fw_rigid.cuh"
#include "fw_adjoint.cuh"

using fw::ElemMat;
using fw::Pair;
using fw::Rigid;

namespace {

constexpr int kBlock = 256;     // default block size of the gather kernels
constexpr int kMaxBlock = 512;  // launch bound (block sizes are a runtime option)
constexpr int kGraphSteps = 32;

struct Dev {
  float2* x;
  float2* x_alt;       // stream path: the other position buffer (swapped every substep)
  float2* v;
  float2* x0;
  float2* bcv;
  float2* corner;      // corner forces in node (CSR) order: node i's are corner[csr_off[i] .. csr_end[i])
  int32_t* corner_pos; // 3 per triangle: where corner (e, c) goes in corner[]
  uint32_t* node_word;
  float* mass;
  int32_t* csr_off;   // node i's corners are csr_slot[csr_off[i] .. csr_end[i]), ascending element
  int32_t* csr_end;
  int32_t* csr_slot;
  int32_t* conn;
  float4* jinv;
  ElemMat* emat;
  float2* body_lm;     // stream path: each body's Lame constants (its triangles share them)
  float2* j2par;
  float4* j2state;
  float4* j2_alt;      // stream path: the other J2 state buffer
  float* ndmass;
  int32_t* body_scene;
  int32_t* body_pair_off;
  int32_t* body_pair_cnt;
  Pair* pairs;
  int32_t* pair_active;
  float* heights;
  int8_t* occ;
  float* scene_dt;
  float* scene_damp;
  int32_t* scene_counter;
  int32_t* scene_active;
  int32_t* scene_mode_req;
  int32_t* scene_mode;
  int32_t* scene_bad;  // set to 1 when a node of the scene gets a non-finite position or velocity
  // stream arenas (fw_step_served_budget): substeps each active scene may
  // still run in this call; a scene whose budget is spent sits the rest out
  // (null: no budgets)
  int32_t* scene_budget;
  // optional second segment: once scene_budget[s] is spent the scene runs
  // scene_budget_next[s] more substeps at scene_dt_next[s] (null: none)
  int32_t* scene_budget_next;
  float* scene_dt_next;
  int32_t* aabb_ring;  // [2][B][4] ordered ints
  int N, E, B, S, P;
  int has_j2;
  // uniform_dt != 0: every scene steps dt_uniform (kernel argument, baked into
  // the captured graph); otherwise scene_dt[] holds one dt per scene.
  int uniform_dt;
  float dt_uniform;
  // chunked launch (arena worlds): only these element / node ranges are stepped
  int use_chunks;
  int n_e_chunks, n_n_chunks;
  const int2* e_chunks;  // (first element, count <= element block size)
  const int2* n_chunks;  // (first node, count <= node block size)
  // FEM-FEM contact (fw_flex.cuh); flex_slot == nullptr when the world has none.
  // Node i (if flex_slot[i] >= 0) receives this substep's contact forces as
  // (work item, force) entries flex_item/flex_force[slot * kFlexListCap ..
  // + flex_cnt[slot]), which node_step adds in work-item order.
  int32_t* flex_slot;
  int32_t* flex_cnt;
  int32_t* flex_item;
  float2* flex_force;
  // FEM-rigid contact (fw_rigid.cuh); rig == nullptr when the world has none.
  // A rigid pair's work item for node i is ritem[pair.n0 + bslot[i]]
  // (bslot: the node's index in its body's boundary node list).
  Rigid* rig;
  float4* ritem;
  int32_t* bslot;
  // The work items are evaluated by the element step's trailing blocks
  // (their inputs are the substep's start state): rwork[it] = (pair, node),
  // rforce[it] = the force the item adds to its node (when ritem[it] is a
  // hit); the node step adds the gated ones in pair order.
  int2* rwork;
  float2* rforce;
  int n_ritems;
  // CFL monitor (cfl_ord == nullptr: off): per scene, the smallest current-
  // shape stable time 0.4 L / c of its triangles since the last read, as the
  // int bits of a non-negative float (int order = float order); body_cfl =
  // 0.4 / sqrt(E / rho) per body (0 for spring domains: not monitored).
  int32_t* cfl_ord;
  float* body_cfl;
};

}  // namespace

#include "fw_flex.cuh"

namespace {

// ------------------------------------------------------------------ kernels

__device__ void step_control(const Dev& d) {
  const int t = threadIdx.x;
  for (int s = t; s < d.S; s += blockDim.x) {
    const int act = d.scene_active[s];
    const int req = d.scene_mode_req[s];
    d.scene_mode[s] = act ? (req ? fw::MODE_INIT : fw::MODE_STEP) : fw::MODE_FROZEN;
    if (act && req) d.scene_mode_req[s] = 0;
  }
  __syncthreads();
  for (int p = t; p < d.P; p += blockDim.x) {
    const Pair& pr = d.pairs[p];
    const int s = d.body_scene[pr.body];
    if (d.scene_mode[s] != fw::MODE_STEP) continue;
    const int k = d.scene_counter[s];
    const int* r = d.aabb_ring + ((size_t)(k & 1) * d.B + pr.body) * 4;
    if (pr.kind == fw::PAIR_RIGID) {  // the rigid's current box; plain overlap when the loop skips the BVH
      const Rigid& g = d.rig[pr.table];
      d.pair_active[p] = fw::box_gate(fw::ord2f(r[0]), fw::ord2f(r[1]), fw::ord2f(r[2]), fw::ord2f(r[3]),
                                      g.lb[0], g.lb[1], g.ub[0], g.ub[1], pr.n1 ? 1 : k) ? 1 : 0;
      continue;
    }
    if (pr.gate > 0) {  // a ground of a loop with a moving plane: its entry's current box
      const Rigid& g = d.rig[pr.gate - 1];
      d.pair_active[p] = fw::box_gate(fw::ord2f(r[0]), fw::ord2f(r[1]), fw::ord2f(r[2]), fw::ord2f(r[3]),
                                      g.lb[0], g.lb[1], g.ub[0], g.ub[1], k) ? 1 : 0;
      continue;
    }
    d.pair_active[p] = fw::pair_gate(pr, fw::ord2f(r[0]), fw::ord2f(r[1]), fw::ord2f(r[2]),
                                     fw::ord2f(r[3]), k) ? 1 : 0;
  }
  __syncthreads();
  for (int s = t; s < d.S; s += blockDim.x)
    if (d.scene_mode[s] == fw::MODE_STEP) d.scene_counter[s] += 1;
  __syncthreads();
  for (int b = t; b < d.B; b += blockDim.x) {
    const int s = d.body_scene[b];
    if (d.scene_mode[s] == fw::MODE_FROZEN) continue;
    int* r = d.aabb_ring + ((size_t)(d.scene_counter[s] & 1) * d.B + b) * 4;
    r[0] = fw::f2ord(1e30f);
    r[1] = fw::f2ord(1e30f);
    r[2] = fw::f2ord(-1e30f);
    r[3] = fw::f2ord(-1e30f);
  }
}

// step_control for a list of scenes (stream arenas: the active scenes of the
// call), one thread per scene: the same four steps for that scene -- mode
// (and budget), its pairs' gates from the box of the previous substep, its
// counter, the reset of its bodies' next box slot -- in the same order.
// Budgets (fw_step_served_budget): a scene runs scene_budget[s] substeps at
// its dt, then scene_budget_next[s] at scene_dt_next[s], then sits out.
// rng[s] = (first body, bodies, first pair, pairs) of scene s.
__global__ void k_control_scenes(Dev d, const int32_t* __restrict__ list, int n, const int4* __restrict__ rng) {
  // the patch step that follows may start now: it gathers positions, which
  // this kernel does not touch, and waits for this kernel before reading what
  // it writes (griddepcontrol.wait)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = list[i];
  int act = d.scene_active[s];
  if (act && d.scene_budget) {
    const int left = d.scene_budget[s];
    if (left > 0) {
      d.scene_budget[s] = left - 1;
    } else {
      const int left2 = d.scene_budget_next ? d.scene_budget_next[s] : 0;
      if (left2 > 0) {  // the second segment: switch to its step size once
        if (left == 0) {
          d.scene_dt[s] = d.scene_dt_next[s];
          d.scene_budget[s] = -1;
        }
        d.scene_budget_next[s] = left2 - 1;
      } else {
        act = 0;
      }
    }
  }
  const int req = d.scene_mode_req[s];
  const int mode = act ? (req ? fw::MODE_INIT : fw::MODE_STEP) : fw::MODE_FROZEN;
  d.scene_mode[s] = mode;
  if (act && req) d.scene_mode_req[s] = 0;
  if (mode != fw::MODE_STEP && mode != fw::MODE_INIT) return;
  const int4 r = rng[s];
  if (mode == fw::MODE_STEP) {
    const int k = d.scene_counter[s];
    for (int p = r.z; p < r.z + r.w; ++p) {
      const Pair& pr = d.pairs[p];
      const int* box = d.aabb_ring + ((size_t)(k & 1) * d.B + pr.body) * 4;
      d.pair_active[p] = fw::pair_gate(pr, fw::ord2f(box[0]), fw::ord2f(box[1]), fw::ord2f(box[2]),
                                       fw::ord2f(box[3]), k) ? 1 : 0;
    }
    d.scene_counter[s] = k + 1;
  }
  const int k2 = d.scene_counter[s];
  for (int b = r.x; b < r.x + r.y; ++b) {
    int* box = d.aabb_ring + ((size_t)(k2 & 1) * d.B + b) * 4;
    box[0] = fw::f2ord(1e30f);
    box[1] = fw::f2ord(1e30f);
    box[2] = fw::f2ord(-1e30f);
    box[3] = fw::f2ord(-1e30f);
  }
}

// CFL monitor: the current-shape stable time of one triangle, the reference's
// 0.4 * L_min / sqrt(E / rho) (femdomain.py:24) on the shortest edge of the
// deformed triangle (coef = 0.4 / sqrt(E / rho) of its body).  Every step
// implementation evaluates it with these operations.
__device__ __forceinline__ float cfl_bound(float2 a, float2 b, float2 c, float coef) {
  const float l0 = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y);
  const float l1 = (b.x - c.x) * (b.x - c.x) + (b.y - c.y) * (b.y - c.y);
  const float l2 = (c.x - a.x) * (c.x - a.x) + (c.y - a.y) * (c.y - a.y);
  return sqrtf(fminf(l0, fminf(l1, l2))) * coef;
}

// Minimum over a whole warp (every lane present) of a non-negative float;
// +inf where no lane had a value.
__device__ __forceinline__ int warp_min_bits(float v) {
  return (int)__reduce_min_sync(0xFFFFFFFFu, (unsigned)__float_as_int(v));
}

// Loads that depend only on the triangle index are issued before the scene
// check, so the gather of corner positions does not wait for it.
__device__ __forceinline__ float element_step(const Dev& d, int e) {
  {
    const ElemMat m = d.emat[e];
    const int c0 = d.conn[3 * e], c1 = d.conn[3 * e + 1], c2 = d.conn[3 * e + 2];
    const float4 ji = d.jinv[e];
    const int q0 = d.corner_pos[3 * e], q1 = d.corner_pos[3 * e + 1], q2 = d.corner_pos[3 * e + 2];
    const float2 a = d.x[c0], b = d.x[c1], c = d.x[c2];
    const int s = d.body_scene[fw::elem_body(m.word)];
    if (!d.scene_active[s]) return __int_as_float(0x7f800000);
    if (fw::elem_type(m.word) == fw::MAT_SPRING) {  // _spring_force_kernel, femspringmanager.py:283-312
      const float2 va = d.v[c0], vb = d.v[c1];
      const float xx = a.x - b.x, xy = a.y - b.y;
      const float lnew = sqrtf(xx * xx + xy * xy);
      const float dx = xx / lnew, dy = xy / lnew;
      const float sc = m.lam * (lnew / m.area - 1.0f);  // stiffness x strain; area holds the rest length
      float fx = sc * dx, fy = sc * dy;
      const float vx = va.x - vb.x, vy = va.y - vb.y;
      const float dmp = m.mu * (vx * dx + vy * dy);  // mu holds the damping
      fx = fx + dmp * dx;
      fy = fy + dmp * dy;
      d.corner[q0] = make_float2(-fx, -fy);
      d.corner[q1] = make_float2(fx, fy);
      return __int_as_float(0x7f800000);
    }
    float4 j2 = make_float4(0.f, 0.f, 0.f, 0.f);
    float sy = 0.f, H = 0.f;
    const bool mises = fw::elem_type(m.word) == fw::MAT_MISES;
    if (mises) {
      j2 = d.j2state[e];
      const float2 q = d.j2par[e];
      sy = q.x;
      H = q.y;
    }
    float2 f1, f2, f3;
    fw::element_forces(a, b, c, ji, m, sy, H, j2, f1, f2, f3);
    if (mises) d.j2state[e] = j2;
    d.corner[q0] = f1;
    d.corner[q1] = f2;
    d.corner[q2] = f3;
    if (!d.cfl_ord) return __int_as_float(0x7f800000);
    return cfl_bound(a, b, c, d.body_cfl[fw::elem_body(m.word)]);
  }
}

// Warp-shuffle minimum of the lanes' CFL bounds per scene (lanes of one warp
// can hold triangles of different scenes), one atomic per scene and warp.
__device__ __forceinline__ void cfl_reduce(const Dev& d, int e, float dtc) {
  const unsigned mask = __activemask();
  const int s = d.body_scene[fw::elem_body(d.emat[e].word)];
  const unsigned grp = __match_any_sync(mask, s);
  const int m = (int)__reduce_min_sync(grp, (unsigned)__float_as_int(dtc));
  if ((int)(threadIdx.x & 31) == __ffs(grp) - 1 && m < 0x7f800000) atomicMin(d.cfl_ord + s, m);
}

// The element step over blocks [0, nb) of the grid.
__device__ __forceinline__ void elements_pass(const Dev& d, int nb) {
  if (blockIdx.x == 0) step_control(d);
  if (d.use_chunks) {
    for (int c = blockIdx.x; c < d.n_e_chunks; c += nb) {
      const int2 ch = d.e_chunks[c];
      if ((int)threadIdx.x < ch.y) {
        const float dtc = element_step(d, ch.x + threadIdx.x);
        if (d.cfl_ord) cfl_reduce(d, ch.x + threadIdx.x, dtc);
      }
    }
    return;
  }
  const int stride = nb * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < d.E; e += stride) {
    const float dtc = element_step(d, e);
    if (d.cfl_ord) cfl_reduce(d, e, dtc);
  }
}

__global__ void __launch_bounds__(kMaxBlock) k_elements(Dev d) { elements_pass(d, gridDim.x); }

// Worlds with FEM-rigid contact: blocks [0, eb) run the element step, the
// others evaluate every FEM-rigid work item -- one thread per item instead of
// one thread per boundary node walking all its rigid pairs -- from the
// substep's start state, whatever the gate and the scene's mode (the node
// step uses an item only when its scene steps and its pair is gated on).
// rigid_item adds its force to a -0 start, which leaves it exactly as it
// would be added to the node's sum.
__global__ void __launch_bounds__(kMaxBlock) k_elements_rigid(Dev d, int eb) {
  if ((int)blockIdx.x < eb) {
    elements_pass(d, eb);
    return;
  }
  const int stride = (gridDim.x - eb) * blockDim.x;
  for (int it = (blockIdx.x - eb) * blockDim.x + threadIdx.x; it < d.n_ritems; it += stride) {
    const int2 w = d.rwork[it];
    const Pair& pr = d.pairs[w.x];
    const float dt = d.uniform_dt ? d.dt_uniform : d.scene_dt[d.body_scene[pr.body]];
    float2 f = make_float2(-0.0f, -0.0f);
    d.ritem[it] = fw::rigid_item(d.rig[pr.table], pr.table, pr.penalty, pr.f[0], pr.pad != 0, d.x[w.y], d.v[w.y],
                                 dt, f);
    d.rforce[it] = f;
  }
}

// This substep's FEM-FEM contact forces on one node, in work-item order (the
// reference adds them with atomic_add in launch order): the entries' item ids
// are distinct, so each pass adds the entry with the next larger id.  The list
// is emptied for the next substep.
__device__ __forceinline__ void flex_add(const Dev& d, int slot, float2& f) {
  const int n = min(d.flex_cnt[slot], kFlexListCap);
  const int* items = d.flex_item + slot * kFlexListCap;
  const float2* forces = d.flex_force + slot * kFlexListCap;
  int last = -1;
  for (int r = 0; r < n; ++r) {
    int pick = 0, best = 0x7FFFFFFF;
    for (int j = 0; j < n; ++j) {
      const int w = items[j];
      if (w > last && w < best) {
        best = w;
        pick = j;
      }
    }
    const float2 c = forces[pick];
    f.x += c.x;
    f.y += c.y;
    last = best;
  }
  d.flex_cnt[slot] = 0;
}

// The node's own state, its CSR range and its first kNodeCorners corner
// forces are loaded before the scene lookup, so one node waits on few
// dependent loads; the corners are then summed in the same ascending order.
constexpr int kNodeCorners = 6;  // an interior node of a structured triangulation has 6

template <bool FLEX, bool RIGID>
__device__ __forceinline__ void node_step(const Dev& d, int i, bool valid) {
  const uint32_t w = valid ? d.node_word[i] : 0u;
  float2 x = make_float2(0.f, 0.f), v = make_float2(0.f, 0.f), bv0 = make_float2(0.f, 0.f);
  int k0 = 0, k1 = 0;
  float mass = 1.0f;
  if (valid) {
    x = d.x[i];
    v = d.v[i];
    k0 = d.csr_off[i];
    k1 = d.csr_end[i];
    mass = d.mass[i];
    bv0 = d.bcv[i];
  }
  float2 cq[kNodeCorners];
#pragma unroll
  for (int u = 0; u < kNodeCorners; ++u) cq[u] = k0 + u < k1 ? d.corner[k0 + u] : make_float2(0.f, 0.f);
  const int b = (int)(w >> fw::NODE_BODY_SHIFT);
  const int s = valid ? d.body_scene[b] : 0;
  const int mode = valid ? d.scene_mode[s] : fw::MODE_FROZEN;
  const bool live = mode != fw::MODE_FROZEN;
  bool bnd = false;
  if (live) {
    const float dt = mode == fw::MODE_INIT ? 0.0f : (d.uniform_dt ? d.dt_uniform : d.scene_dt[s]);
    const float damp = mode == fw::MODE_INIT ? 0.0f : d.scene_damp[s];
    float2 f = make_float2(0.f, 0.f);
    bnd = (w & fw::NODE_BOUNDARY) != 0;
    if (bnd && mode == fw::MODE_STEP) {
      const int p0 = d.body_pair_off[b], pn = d.body_pair_cnt[b];
      const int fs = FLEX ? d.flex_slot[i] : -1;
      const int bs = RIGID ? d.bslot[i] : 0;  // this node's slot in its body's boundary list
      bool flex_done = !FLEX || fs < 0;
      for (int k = 0; k < pn; ++k) {
        if (FLEX && !flex_done && d.pairs[p0 + k].kind != fw::PAIR_PLANE) {
          flex_add(d, fs, f);  // FEM-FEM contact runs after the planes, before the height fields / voxels
          flex_done = true;
        }
        if (RIGID && d.pairs[p0 + k].kind == fw::PAIR_RIGID) {
          // the item was evaluated by k_elements_rigid from this same state
          const int slot = d.pairs[p0 + k].n0 + bs;
          if (d.pair_active[p0 + k]) {
            if (__float_as_int(d.ritem[slot].w) >= 0) {
              const float2 rf = d.rforce[slot];
              f.x += rf.x;
              f.y += rf.y;
            }
          } else {
            d.ritem[slot] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
          }
          continue;
        }
        if (!d.pair_active[p0 + k]) continue;
        float2 cf;
        if (fw::contact_force(d.pairs[p0 + k], d.heights, d.occ, x, v, dt, cf)) {
          f.x += cf.x;
          f.y += cf.y;
        }
      }
      if (FLEX && !flex_done) flex_add(d, fs, f);
    }
#pragma unroll
    for (int u = 0; u < kNodeCorners; ++u)  // contiguous, ascending element
      if (k0 + u < k1) {
        f.x += cq[u].x;
        f.y += cq[u].y;
      }
    for (int k = k0 + kNodeCorners; k < k1; ++k) {
      const float2 c = d.corner[k];
      f.x += c.x;
      f.y += c.y;
    }
    const int bc = (int)(w & fw::NODE_BC_MASK);
    const float2 bv = (bc & (fw::BC_A | fw::BC_GRAVITY | fw::BC_FORCE | fw::BC_V)) ? bv0 : make_float2(0.f, 0.f);
    fw::integrate(bc, f, mass, bv, dt, damp, x, v);
    d.x[i] = x;
    d.v[i] = v;
    if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) d.scene_bad[s] = 1;
  }
  // Per-body AABB of boundary nodes (femspringmanager.py:361-408).
  const unsigned full = 0xFFFFFFFFu;
  const unsigned mb = __ballot_sync(full, bnd);
  if (mb == 0u) return;
  const int leader = __ffs(mb) - 1;
  const int bl = __shfl_sync(full, b, leader);
  const bool uniform = __all_sync(full, !bnd || b == bl);
  float lx = bnd ? x.x : 1e30f, ly = bnd ? x.y : 1e30f;
  float hx = bnd ? x.x : -1e30f, hy = bnd ? x.y : -1e30f;
  if (uniform) {
    for (int o = 16; o > 0; o >>= 1) {
      lx = fminf(lx, __shfl_xor_sync(full, lx, o));
      ly = fminf(ly, __shfl_xor_sync(full, ly, o));
      hx = fmaxf(hx, __shfl_xor_sync(full, hx, o));
      hy = fmaxf(hy, __shfl_xor_sync(full, hy, o));
    }
    if ((int)(threadIdx.x & 31) == leader) {
      int* r = d.aabb_ring + ((size_t)(d.scene_counter[s] & 1) * d.B + b) * 4;
      atomicMin(r + 0, fw::f2ord(lx));
      atomicMin(r + 1, fw::f2ord(ly));
      atomicMax(r + 2, fw::f2ord(hx));
      atomicMax(r + 3, fw::f2ord(hy));
    }
  } else if (bnd) {
    int* r = d.aabb_ring + ((size_t)(d.scene_counter[s] & 1) * d.B + b) * 4;
    atomicMin(r + 0, fw::f2ord(lx));
    atomicMin(r + 1, fw::f2ord(ly));
    atomicMax(r + 2, fw::f2ord(hx));
    atomicMax(r + 3, fw::f2ord(hy));
  }
}

__global__ void __launch_bounds__(kMaxBlock) k_nodes(Dev d) {
  if (d.use_chunks) {
    for (int c = blockIdx.x; c < d.n_n_chunks; c += gridDim.x) {
      const int2 ch = d.n_chunks[c];
      node_step<false, false>(d, ch.x + (int)threadIdx.x, (int)threadIdx.x < ch.y);
    }
    return;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  node_step<false, false>(d, i, i < d.N);
}

// k_nodes of worlds with FEM-FEM contact: the node's contact forces from the
// work items join its plane and ground contact forces in launch order.
__global__ void __launch_bounds__(kMaxBlock) k_nodes_flex(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  node_step<true, false>(d, i, i < d.N);
}

// k_nodes of worlds with FEM-rigid contact (FLEX: FEM-FEM contact as well).
template <bool FLEX>
__global__ void __launch_bounds__(kMaxBlock) k_nodes_rigid(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  node_step<FLEX, true>(d, i, i < d.N);
}

// The rigid side of a substep: one warp per rigid of a stepping scene adds
// its work items' reactions to its accumulators in work-item order (its
// pairs in pair order, each pair's items in boundary-node order: lanes load
// 128 records at a time, and every lane adds the hits in ascending lane order
// through shuffles, so the sum is a serial run of the reference's atomic
// adds).  Then each stepping scene's substep is counted and, on the substeps
// of its schedule, its rigid update runs (fw_rigid.cuh): after a barrier, one
// thread per scene, when all rigids fit in one block; otherwise by the warp
// that finishes the scene's last rigid (a per-scene arrival count after a
// fence).  The update reads only finished accumulators either way.
struct RigidDev {
  Rigid* rig;
  int n;
  float4* gbox;
  int* gkind;
  int n_ground;
  float4* item;
  int n_items;
  int* rp_off;   // per rigid: its pairs' item ranges rp_rng[rp_off[g] .. rp_off[g + 1])
  int2* rp_rng;  // (first item, item count), pair order
  fw::RigidScene* rs;  // the scenes with rigids
  int n_rs;
  int* done;           // per scene with rigids: warps finished this substep
  const fw::RigidClock* clock;  // per scene
  int* count;                   // per scene: the reference's rigid_update_times
  int* err;
};

constexpr int kRigidThreads = 256;   // grid launch: 8 rigids per block
constexpr int kRigidOneBlock = 1024;  // up to 32 rigids: one block, scenes updated after a barrier

// The counter and, when due, the rigid update of scene-with-rigids k.
__device__ __forceinline__ void rigid_scene_update(const RigidDev& r, int k) {
  const fw::RigidScene rs = r.rs[k];
  const fw::RigidClock ck = r.clock[rs.scene];
  const int cnt = r.count[rs.scene] + 1;
  r.count[rs.scene] = cnt;
  if (ck.every < 1 || cnt % ck.every != 0) return;
  fw::rigid_update(r.rig + rs.r0, rs.rn, r.gbox + rs.g0, r.gkind + rs.g0, rs.gn, ck.dt, ck.damping, r.err);
}

__global__ void __launch_bounds__(kRigidOneBlock) k_rigid(Dev d, RigidDev r) {
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const float4 none = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
  const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const bool live = g < r.n && d.scene_mode[r.rig[min(g, r.n - 1)].scene] == fw::MODE_STEP;
  if (live) {
    Rigid& rg = r.rig[g];
    float ax = rg.acc[0], ay = rg.acc[1], aw = rg.accw;
    for (int q = r.rp_off[g]; q < r.rp_off[g + 1]; ++q) {
      const int2 rng = r.rp_rng[q];
      for (int base = 0; base < rng.y; base += 128) {
        float4 rec[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int it = base + 32 * u + lane;
          rec[u] = it < rng.y ? r.item[rng.x + it] : none;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          unsigned m = __ballot_sync(full, __float_as_int(rec[u].w) >= 0);
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            ax = ax + __shfl_sync(full, rec[u].x, l);
            ay = ay + __shfl_sync(full, rec[u].y, l);
            aw = aw + __shfl_sync(full, rec[u].z, l);
          }
        }
      }
    }
    if (lane == 0) {
      rg.acc[0] = ax;
      rg.acc[1] = ay;
      rg.accw = aw;
    }
  }
  if (gridDim.x == 1) {  // every rigid in this block: a barrier, then one thread per scene
    __syncthreads();
    for (int k = threadIdx.x; k < r.n_rs; k += blockDim.x)
      if (d.scene_mode[r.rs[k].scene] == fw::MODE_STEP) rigid_scene_update(r, k);
    return;
  }
  // grid: the warp that finishes a scene's last rigid runs that scene's update
  if (!live || lane != 0) return;
  __threadfence();
  const int k = r.rig[g].rs;
  if (atomicAdd(r.done + k, 1) + 1 != r.rs[k].rn) return;
  __threadfence();
  r.done[k] = 0;
  rigid_scene_update(r, k);
}

// Rotation cache and boxes of the rigids at construction
// (precompute_rigid_transforms + updateBBox, explicitloop.py:198-201).
__global__ void k_rigid_init(Rigid* rig, int n) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  fw::rigid_rot(rig[a]);
  if (rig[a].type != fw::RIGID_ANALYTICAL) fw::rigid_aabb(rig[a]);  // an analytical entry starts at getBBox()
}

// Reference-shape precompute, _prepare_fem_data_kernel
// (flatworld/femspringmanager.py:113-138), plus the Lame constants of
// getStress2D (materialfunctions.py:12-13), which depend only on E and nu.
__global__ void k_prepare_elements(Dev d, const float* __restrict__ young,
                                   const float* __restrict__ poisson,
                                   const float* __restrict__ rho, int e_lo, int e_hi) {
  const int e = e_lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e_hi) return;
  if (fw::elem_type(d.emat[e].word) == fw::MAT_SPRING) {  // addSpringDomain (femspringmanager.py:848-861)
    ElemMat m = d.emat[e];
    m.area = rho[e - e_lo];     // rest length
    m.lam = young[e - e_lo];    // spring stiffness
    m.mu = poisson[e - e_lo];   // damping
    d.emat[e] = m;
    d.jinv[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    d.ndmass[e] = 0.0f;         // the nodes carry the domain's mass
    return;
  }
  const int c0 = d.conn[3 * e], c1 = d.conn[3 * e + 1], c2 = d.conn[3 * e + 2];
  const float2 a = d.x0[c0], b = d.x0[c1], c = d.x0[c2];
  const float j00 = a.x - c.x, j01 = b.x - c.x, j10 = a.y - c.y, j11 = b.y - c.y;
  const float det = j00 * j11 - j01 * j10;
  const float area = fabsf(det) * 0.5f;
  float4 ji = make_float4(0.f, 0.f, 0.f, 0.f);
  if (det != 0.0f) {
    const float r = 1.0f / det;
    ji = make_float4(j11 * r, -j01 * r, -j10 * r, j00 * r);
  }
  d.jinv[e] = ji;
  const float E = young[e - e_lo], nu = poisson[e - e_lo];
  ElemMat m = d.emat[e];
  m.area = area;
  m.lam = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  m.mu = E / (2.0f * (1.0f + nu));
  d.emat[e] = m;
  d.ndmass[e] = area * rho[e - e_lo] / 3.0f;
}

// Lumped mass: each node adds its elements' shares in ascending element order,
// the order of the reference's serial atomic adds.
__global__ void k_prepare_mass(Dev d, int n_lo, int n_hi) {
  const int i = n_lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_hi) return;
  float m = 0.0f;
  for (int k = d.csr_off[i]; k < d.csr_end[i]; ++k) m += d.ndmass[d.csr_slot[k] / 3];
  d.mass[i] = m;
}

// Selective mass scaling, _mass_scaling_kernel (femspringmanager.py:139-196):
// a triangle whose critical step 0.4 L_min / sqrt(E / rho) is below dt_target
// gets the density that makes it dt_target, and its three nodes a third of
// the added mass each.  The reference runs it on one thread in element order;
// here k_mass_scale_elems finds each triangle's share and k_mass_scale_nodes
// adds a node's shares in ascending element order (its CSR list), the same
// additions in the same order.
__global__ void k_mass_scale_elems(Dev d, const float* __restrict__ young, const float* __restrict__ rho,
                                   float dt_target, float* __restrict__ dm, int32_t* __restrict__ hit) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  if (fw::elem_type(d.emat[e].word) == fw::MAT_SPRING) {  // springs: the node pass
    dm[e] = 0.0f;
    hit[e] = 0;
    return;
  }
  const float2 a = d.x[d.conn[3 * e]], b = d.x[d.conn[3 * e + 1]], c = d.x[d.conn[3 * e + 2]];
  const float e01x = b.x - a.x, e01y = b.y - a.y, e12x = c.x - b.x, e12y = c.y - b.y, e20x = a.x - c.x, e20y = a.y - c.y;
  const float e01 = sqrtf(e01x * e01x + e01y * e01y), e12 = sqrtf(e12x * e12x + e12y * e12y);
  const float e20 = sqrtf(e20x * e20x + e20y * e20y);
  const float m12 = e12 < e20 ? e12 : e20;
  const float L = e01 < m12 ? e01 : m12;
  const float E = young[e], r = rho[e];
  const float ce = sqrtf(E / r);
  const float dt_elem = 0.4f * L / ce;
  int h = 0;
  float add = 0.0f;
  if (dt_elem < dt_target && L > 1e-15f) {
    const float q = dt_target / (0.4f * L);
    const float rho_new = E * q * q;
    add = (rho_new - r) * d.emat[e].area / 3.0f;
    h = 1;
  }
  dm[e] = add;
  hit[e] = h;
}

__global__ void k_mass_scale_nodes(Dev d, const float* __restrict__ dm, const int32_t* __restrict__ hit,
                                   float dt_target) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  float m = d.mass[i];
  for (int k = d.csr_off[i]; k < d.csr_end[i]; ++k) {  // triangles first (the reference's first loop)
    const int e = d.csr_slot[k] / 3;
    if (hit[e]) m = m + dm[e];
  }
  for (int k = d.csr_off[i]; k < d.csr_end[i]; ++k) {  // then springs: at least 4 k dt^2 (its second loop)
    const int e = d.csr_slot[k] / 3;
    const ElemMat em = d.emat[e];
    if (fw::elem_type(em.word) != fw::MAT_SPRING) continue;
    const float m_min = 4.0f * em.lam * dt_target * dt_target;
    if (m < m_min) m = m_min;
  }
  d.mass[i] = m;
}

// Lame constants of elements [e_lo, e_hi) from new Young's moduli (same
// formula as k_prepare_elements).
__global__ void k_set_young(Dev d, const float* __restrict__ young, const float* __restrict__ poisson,
                            int e_lo, int e_hi) {
  const int e = e_lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e_hi) return;
  const float E = young[e - e_lo], nu = poisson[e];
  ElemMat m = d.emat[e];
  m.lam = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  m.mu = E / (2.0f * (1.0f + nu));
  d.emat[e] = m;
}

// The adjoint state is accumulated in FP64, so that summing thousands of
// substeps adds no error of its own; the element Jacobian products are FP32
// dual numbers on the recorded FP32 trajectory, i.e. this is the exact
// adjoint of the FP32 forward up to FP32 rounding of those products.
struct Adj {
  double2* xb;   // adjoint of positions
  double2* vb;   // adjoint of velocities
  double2* fb;   // adjoint of the node force of the current substep
  double* Eb;    // d loss / d Young's modulus, per element
  float* young;  // Young's modulus per element
  float2* traj;  // recorded positions of the segment, [K][N]
  float2* trajv;  // recorded velocities of the segment, [K][N] (contact damping terms)
  float4* trajs;  // recorded J2 state of the segment, [K][E] (worlds with J2 triangles)
  double* sb;     // adjoint of the J2 state (eps_p Voigt, eqps), 4 per element
  int32_t* gates;  // recorded broad-phase gates, [K][P]
  float2* io_x;  // FP32 staging of xb / vb / Eb for the C ABI
  float2* io_v;
  float* io_E;
};

// Adjoint of "v' = v + dt f / m; BC override" at every node: from (xb', vb')
// form the force adjoint fb and the velocity adjoint of the previous substep.
// With damping c, v' = v (1 - dt c / m) + dt f / m.
__device__ __forceinline__ void adj_node_prep(const Dev& d, const Adj& a, int i, float dt, float damp) {
  const int bc = (int)(d.node_word[i] & fw::NODE_BC_MASK);
  const double2 xb = a.xb[i], vb = a.vb[i];
  const double h = (double)dt;
  const double2 vt = make_double2(vb.x + h * xb.x, vb.y + h * xb.y);
  const bool vfixed = (bc & (fw::BC_U | fw::BC_V)) != 0;
  const bool fdead = vfixed || (bc & fw::BC_A) != 0;
  const double s = h / (double)d.mass[i];
  const double keep = 1.0 - s * (double)damp;
  a.fb[i] = fdead ? make_double2(0.0, 0.0) : make_double2(s * vt.x, s * vt.y);
  a.vb[i] = vfixed ? make_double2(0.0, 0.0) : make_double2(keep * vt.x, keep * vt.y);
}

__global__ void k_adj_seed(Adj a, int N, int has_x, int has_v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float2 x = has_x ? a.io_x[i] : make_float2(0.f, 0.f);
  const float2 v = has_v ? a.io_v[i] : make_float2(0.f, 0.f);
  a.xb[i] = make_double2(x.x, x.y);
  a.vb[i] = make_double2(v.x, v.y);
}

__global__ void k_adj_out(Adj a, int N, int E) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    a.io_x[i] = make_float2((float)a.xb[i].x, (float)a.xb[i].y);
    a.io_v[i] = make_float2((float)a.vb[i].x, (float)a.vb[i].y);
  }
  if (i < E) a.io_E[i] = (float)a.Eb[i];
}

__global__ void k_adj_prep(Dev d, Adj a, float dt, float damp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.N) adj_node_prep(d, a, i, dt, damp);
}

__global__ void k_adj_elements(Dev d, Adj a, const float2* __restrict__ x, const float4* __restrict__ st) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  const ElemMat m = d.emat[e];
  const int c0 = d.conn[3 * e], c1 = d.conn[3 * e + 1], c2 = d.conn[3 * e + 2];
  const double2 b0 = a.fb[c0], b1 = a.fb[c1], b2 = a.fb[c2];
  if (fw::elem_type(m.word) == fw::MAT_MISES) {
    // transpose of the local Jacobian, column by column: 6 positions, 4 state, E
    const float2 p0 = x[c0], p1 = x[c1], p2 = x[c2];
    const float xs[6] = {p0.x, p0.y, p1.x, p1.y, p2.x, p2.y};
    const float4 s4 = st[e];
    const float ss[4] = {s4.x, s4.y, s4.z, s4.w};
    double ob[10] = {b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, 0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 4; ++k) ob[6 + k] = a.sb[4 * (size_t)e + k];
    const float young = a.young[e];
    const float2 yp = d.j2par[e];
    float corner[6];
    double snew[4];
    double eb = 0.0;
    for (int col = 0; col < 11; ++col) {
      fw::Dual X[6], S[4], F[6], SN[4];
      for (int r = 0; r < 6; ++r) X[r] = fw::dmk(xs[r], col == r ? 1.f : 0.f);
      for (int k = 0; k < 4; ++k) S[k] = fw::dmk(ss[k], col == 6 + k ? 1.f : 0.f);
      const fw::Dual lam = fw::dmk(m.lam, col == 10 ? m.lam / young : 0.f);
      const fw::Dual mu = fw::dmk(m.mu, col == 10 ? m.mu / young : 0.f);
      fw::element_j2_dual(X, d.jinv[e], lam, mu, yp.x, yp.y, S, m.area, F, SN);
      double dot = 0.0;
      for (int r = 0; r < 6; ++r) dot += ob[r] * (double)F[r].d;
      for (int k = 0; k < 4; ++k) dot += ob[6 + k] * (double)SN[k].d;
      if (col < 6) corner[col] = (float)dot;
      else if (col < 10) snew[col - 6] = dot;
      else eb = dot;
    }
    d.corner[d.corner_pos[3 * e]] = make_float2(corner[0], corner[1]);
    d.corner[d.corner_pos[3 * e + 1]] = make_float2(corner[2], corner[3]);
    d.corner[d.corner_pos[3 * e + 2]] = make_float2(corner[4], corner[5]);
    for (int k = 0; k < 4; ++k) a.sb[4 * (size_t)e + k] = snew[k];
    a.Eb[e] += eb;
    return;
  }
  const float2 w0 = make_float2((float)b0.x, (float)b0.y), w1 = make_float2((float)b1.x, (float)b1.y),
               w2 = make_float2((float)b2.x, (float)b2.y);
  fw::Dual f[6];
  fw::element_forces_jvp(x[c0], x[c1], x[c2], w0, w1, w2, d.jinv[e], fw::elem_type(m.word), m.lam, m.mu,
                         m.area, f);
  d.corner[d.corner_pos[3 * e]] = make_float2(f[0].d, f[1].d);
  d.corner[d.corner_pos[3 * e + 1]] = make_float2(f[2].d, f[3].d);
  d.corner[d.corner_pos[3 * e + 2]] = make_float2(f[4].d, f[5].d);
  const double dot = b0.x * f[0].v + b0.y * f[1].v + b1.x * f[2].v + b1.y * f[3].v + b2.x * f[4].v + b2.y * f[5].v;
  a.Eb[e] += dot / (double)a.young[e];
}

// xb <- xb' + sum of element VJPs + plane-contact VJP; with prep, also the
// force / velocity adjoints of the previous substep (fused, saves a launch).
__global__ void k_adj_nodes(Dev d, Adj a, const float2* __restrict__ x, const float2* __restrict__ v,
                            const int32_t* __restrict__ gates, float dt, float damp, int prep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  double2 xb = a.xb[i];
  const double2 fb = a.fb[i];
  for (int k = d.csr_off[i]; k < d.csr_end[i]; ++k) {
    const float2 c = d.corner[k];
    xb.x += c.x;
    xb.y += c.y;
  }
  const uint32_t w = d.node_word[i];
  if (w & fw::NODE_BOUNDARY) {
    const int b = (int)(w >> fw::NODE_BODY_SHIFT);
    const float2 xi = x[i], vi = v[i];
    double2 vb = a.vb[i];
    for (int q = 0; q < d.body_pair_cnt[b]; ++q) {
      const int p = d.body_pair_off[b] + q;
      if (!gates[p]) continue;
      fw::contact_vjp(d.pairs[p], d.heights, d.occ, xi, vi, dt, fb, xb, vb);
    }
    a.vb[i] = vb;
  }
  a.xb[i] = xb;
  if (prep) adj_node_prep(d, a, i, dt, damp);
}

// ------------------------------------------------------------------ tangent
// Forward-mode derivative of the same substep along (dx, dv, dE), on the
// recorded FP32 trajectory and gates: df = J(x) dx + f_e dE_e / E_e
// (+ plane contact -k n (n . dx) while the node penetrates), then
// dv' = dv (1 - dt c / m) + dt df / m (zero for fixed / enforced-velocity
// nodes, no df for prescribed-acceleration nodes), dx' = dx + dt dv'.
// Used to check that the adjoint is the exact transpose (dot-product test) and
// for forward-mode gradients.
struct Tan {
  double2* dx;
  double2* dv;
  float* dE;     // perturbation of Young's modulus per element
  float* young;  // Young's modulus per element
  float2* xs;    // positions at the start of the substep
  float2* vs;    // velocities at the start of the substep
  float2* io_x;  // FP32 staging for the C ABI
  float2* io_v;
};

__global__ void k_tan_elements(Dev d, Tan t) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  const ElemMat m = d.emat[e];
  const int c0 = d.conn[3 * e], c1 = d.conn[3 * e + 1], c2 = d.conn[3 * e + 2];
  const double2 u0 = t.dx[c0], u1 = t.dx[c1], u2 = t.dx[c2];
  fw::Dual f[6];
  fw::element_forces_jvp(t.xs[c0], t.xs[c1], t.xs[c2], make_float2((float)u0.x, (float)u0.y),
                         make_float2((float)u1.x, (float)u1.y), make_float2((float)u2.x, (float)u2.y), d.jinv[e],
                         fw::elem_type(m.word), m.lam, m.mu, m.area, f);
  const float r = t.dE[e] / t.young[e];
  d.corner[d.corner_pos[3 * e]] = make_float2(f[0].d + f[0].v * r, f[1].d + f[1].v * r);
  d.corner[d.corner_pos[3 * e + 1]] = make_float2(f[2].d + f[2].v * r, f[3].d + f[3].v * r);
  d.corner[d.corner_pos[3 * e + 2]] = make_float2(f[4].d + f[4].v * r, f[5].d + f[5].v * r);
}

__global__ void k_tan_nodes(Dev d, Tan t, float dt, float damp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.N) return;
  const uint32_t w = d.node_word[i];
  const int bc = (int)(w & fw::NODE_BC_MASK);
  const double2 dx = t.dx[i], dv = t.dv[i];
  double fx = 0.0, fy = 0.0;
  if (w & fw::NODE_BOUNDARY) {
    const int b = (int)(w >> fw::NODE_BODY_SHIFT);
    const float2 xi = t.xs[i], vi = t.vs[i];
    for (int q = 0; q < d.body_pair_cnt[b]; ++q) {
      const int p = d.body_pair_off[b] + q;
      if (!d.pair_active[p]) continue;
      fw::contact_jvp(d.pairs[p], d.heights, d.occ, xi, vi, dt, dx, dv, fx, fy);
    }
  }
  for (int k = d.csr_off[i]; k < d.csr_end[i]; ++k) {
    const float2 c = d.corner[k];
    fx += c.x;
    fy += c.y;
  }
  const double h = (double)dt, s = h / (double)d.mass[i], keep = 1.0 - s * (double)damp;
  double2 nv;
  if (bc & (fw::BC_U | fw::BC_V)) nv = make_double2(0.0, 0.0);
  else if (bc & fw::BC_A) nv = make_double2(keep * dv.x, keep * dv.y);
  else nv = make_double2(keep * dv.x + s * fx, keep * dv.y + s * fy);
  t.dv[i] = nv;
  t.dx[i] = make_double2(dx.x + h * nv.x, dx.y + h * nv.y);
}

__global__ void k_tan_seed(Tan t, int N, int has_x, int has_v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float2 x = has_x ? t.io_x[i] : make_float2(0.f, 0.f);
  const float2 v = has_v ? t.io_v[i] : make_float2(0.f, 0.f);
  t.dx[i] = make_double2(x.x, x.y);
  t.dv[i] = make_double2(v.x, v.y);
}

__global__ void k_tan_out(Tan t, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  t.io_x[i] = make_float2((float)t.dx[i].x, (float)t.dx[i].y);
  t.io_v[i] = make_float2((float)t.dv[i].x, (float)t.dv[i].y);
}

// ------------------------------------------------------------------ energy
// Total energy, reduced in FP64 (the only FP64 step of the library).  Terms
// per node: kinetic 1/2 m |v|^2; external potential -m g.x (gravity BC) or
// -f.x (constant nodal force), following the BC precedence of the update
// (fixed / prescribed-acceleration nodes have none); penalty 1/2 k sd^2 for
// every penetrating boundary node and contact pair of its body (the elastic
// part of the contact force, evaluated at zero velocity; not gated by the
// broad phase).  Per triangle: area x strain energy density --
//   Elastic (St-Venant-Kirchhoff): lambda/2 tr(E)^2 + mu E:E
//   NeoHookean: mu/2 (tr C - 2) - mu ln J + lambda/2 (ln J)^2
//   J2: the St-Venant-Kirchhoff form of the elastic strain E - eps_p
// -- the energies whose E-derivatives are the stresses of the step
// (materialfunctions.py:10-101).  Positions and moduli are the FP32 state,
// every operation after loading them is FP64.
struct EnergyChunk {
  int group;   // output row
  int n0, nn;  // node range
  int e0, ne;  // triangle range
};

__device__ double elem_energy(const Dev& d, int e) {
  const ElemMat m = d.emat[e];
  const int c0 = d.conn[3 * e], c1 = d.conn[3 * e + 1], c2 = d.conn[3 * e + 2];
  const float2 a = d.x[c0], b = d.x[c1], c = d.x[c2];
  if (fw::elem_type(m.word) == fw::MAT_SPRING) {  // k L0 / 2 (l / L0 - 1)^2, whose l-derivative is the spring force
    const double dx = (double)a.x - b.x, dy = (double)a.y - b.y;
    const double st = sqrt(dx * dx + dy * dy) / (double)m.area - 1.0;
    return 0.5 * (double)m.lam * (double)m.area * st * st;
  }
  const float4 ji = d.jinv[e];
  const double j00 = (double)a.x - (double)c.x, j01 = (double)b.x - (double)c.x;
  const double j10 = (double)a.y - (double)c.y, j11 = (double)b.y - (double)c.y;
  const double F00 = j00 * ji.x + j01 * ji.z, F01 = j00 * ji.y + j01 * ji.w;
  const double F10 = j10 * ji.x + j11 * ji.z, F11 = j10 * ji.y + j11 * ji.w;
  const double C00 = F00 * F00 + F10 * F10, C01 = F00 * F01 + F10 * F11, C11 = F01 * F01 + F11 * F11;
  const double lam = m.lam, mu = m.mu;
  const int type = fw::elem_type(m.word);
  double W;
  if (type == fw::MAT_NEOHOOKEAN) {
    const double lj = log(F00 * F11 - F01 * F10);
    W = 0.5 * mu * (C00 + C11 - 2.0) - mu * lj + 0.5 * lam * lj * lj;
  } else {
    double e0 = 0.5 * (C00 - 1.0), e1 = 0.5 * (C11 - 1.0), e2 = 0.5 * C01;
    if (type == fw::MAT_MISES) {
      const float4 ep = d.j2state[e];
      e0 -= ep.x;
      e1 -= ep.y;
      e2 -= ep.z;
    }
    const double tr = e0 + e1;
    W = 0.5 * lam * tr * tr + mu * (e0 * e0 + e1 * e1 + 2.0 * e2 * e2);
  }
  return (double)m.area * W;
}

__device__ void node_energy(const Dev& d, int i, double& ke, double& ext, double& pen) {
  const float2 x = d.x[i], v = d.v[i], bcv = d.bcv[i];
  const double m = d.mass[i];
  ke += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y);
  const uint32_t w = d.node_word[i];
  const int bc = (int)(w & fw::NODE_BC_MASK);
  if (bc & (fw::BC_U | fw::BC_A)) {
  } else if (bc & fw::BC_GRAVITY) {
    ext -= m * ((double)bcv.x * x.x + (double)bcv.y * x.y);
  } else if (bc & fw::BC_FORCE) {
    ext -= (double)bcv.x * x.x + (double)bcv.y * x.y;
  }
  if (w & fw::NODE_BOUNDARY) {
    const int b = (int)(w >> fw::NODE_BODY_SHIFT);
    for (int q = 0; q < d.body_pair_cnt[b]; ++q) {
      const Pair& pr = d.pairs[d.body_pair_off[b] + q];
      float2 f;
      if (pr.kind == fw::PAIR_RIGID) {  // the normal penalty force of the primitive
        float nx, ny, cx, cy;
        const Rigid& g = d.rig[pr.table];
        const float depth = fw::rigid_detect(g, x.x, x.y, nx, ny, cx, cy) - 1e-4f;
        if (depth < 0.0f) pen += 0.5 * (double)pr.penalty * (double)depth * (double)depth;
        continue;
      }
      if (fw::contact_force(pr, d.heights, d.occ, x, make_float2(0.f, 0.f), 0.f, f))
        pen += 0.5 * ((double)f.x * f.x + (double)f.y * f.y) / (double)pr.penalty;
    }
  }
}

constexpr int kEnergyThreads = 256;
constexpr int kEnergyChunk = 8192;

// One block per chunk: fixed-order strided sums, then a fixed tree.
__global__ void __launch_bounds__(kEnergyThreads) k_energy_chunks(Dev d, const EnergyChunk* ch, double4* part) {
  __shared__ double sm[4][kEnergyThreads];
  const EnergyChunk c = ch[blockIdx.x];
  const int t = threadIdx.x;
  double ke = 0.0, st = 0.0, ext = 0.0, pen = 0.0;
  for (int i = t; i < c.nn; i += kEnergyThreads) node_energy(d, c.n0 + i, ke, ext, pen);
  for (int e = t; e < c.ne; e += kEnergyThreads) st += elem_energy(d, c.e0 + e);
  sm[0][t] = ke;
  sm[1][t] = st;
  sm[2][t] = ext;
  sm[3][t] = pen;
  __syncthreads();
  for (int h = kEnergyThreads / 2; h > 0; h >>= 1) {
    if (t < h)
      for (int k = 0; k < 4; ++k) sm[k][t] += sm[k][t + h];
    __syncthreads();
  }
  if (t == 0) part[blockIdx.x] = make_double4(sm[0][0], sm[1][0], sm[2][0], sm[3][0]);
}

// One thread per group: its chunks' partials in chunk order.
__global__ void k_energy_groups(const int* first, int n_groups, const double4* part, double4* out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  double4 s = make_double4(0.0, 0.0, 0.0, 0.0);
  for (int k = first[g]; k < first[g + 1]; ++k) {
    s.x += part[k].x;
    s.y += part[k].y;
    s.z += part[k].z;
    s.w += part[k].w;
  }
  out[g] = s;
}

}  // namespace

#include "fw_resident.cuh"
#include "fw_stream.cuh"

// ------------------------------------------------------------------ context

struct fw_ctx {
  int device = 0;
  std::string err;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool finalized = false;
  int64_t launches = 0;
  // host staging
  int N = 0, E = 0, B = 0, S = 0;
  std::vector<float> h_x, h_v, h_bcv;
  std::vector<int32_t> h_bc;
  std::vector<int32_t> h_conn, h_type;
  std::vector<float> h_E, h_nu, h_rho, h_sy, h_H;
  std::vector<int32_t> h_noff, h_ncnt, h_eoff, h_ecnt, h_scene, h_bnoff, h_bncnt, h_bnodes;
  std::vector<float> h_damp;
  std::vector<Pair> h_pairs;
  std::vector<float> h_heights;
  std::vector<int8_t> h_occ;
  std::vector<float> cur_dt;
  std::vector<int32_t> cur_active;
  Dev d{};
  std::vector<void*> allocs;
  // captured step graphs, keyed by (uniform flag, substeps, dt bits); the
  // adjoint's recompute / reverse graphs, keyed by (kind, substeps, dt bits)
  std::vector<std::pair<uint64_t, cudaGraphExec_t>> graphs;
  std::vector<std::pair<uint64_t, cudaGraphExec_t>> adj_graphs;
  cudaStream_t graph_stream = nullptr;
  int grid_e = 1, grid_n = 1;
  int block_e = kBlock, block_n = kBlock, grid_e_cap = 0, sms = 148;
  // snapshots: device copies of the full step state, one set per slot
  struct Snap {
    float2 *x = nullptr, *v = nullptr;
    float4* j2 = nullptr;
    int32_t *counter = nullptr, *ring = nullptr, *mode_req = nullptr;
    int64_t host_counter = 0;
    bool valid = false;
  };
  std::vector<Snap> snaps;
  // ---- arena (serving): fixed capacity, scenes inserted / removed at run time
  struct FreeList {
    std::map<int64_t, int64_t> free;  // start -> length, coalesced
    void init(int64_t cap) { free.clear(); if (cap > 0) free[0] = cap; }
    bool take(int64_t len, int64_t* off) {
      if (len == 0) { *off = 0; return true; }
      for (auto it = free.begin(); it != free.end(); ++it)
        if (it->second >= len) {
          *off = it->first;
          const int64_t rest = it->second - len, start = it->first + len;
          free.erase(it);
          if (rest) free[start] = rest;
          return true;
        }
      return false;
    }
    void give(int64_t off, int64_t len) {
      if (len == 0) return;
      auto it = free.emplace(off, len).first;
      auto nx = std::next(it);
      if (nx != free.end() && it->first + it->second == nx->first) { it->second += nx->second; free.erase(nx); }
      if (it != free.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) { pv->second += it->second; free.erase(it); }
      }
    }
    int64_t total() const { int64_t t = 0; for (auto& f : free) t += f.second; return t; }
  };
  struct ArenaScene {
    bool live = false;
    int64_t n0 = 0, nn = 0, e0 = 0, ne = 0, b0 = 0, nb = 0, p0 = 0, np = 0, h0 = 0, nh = 0, o0 = 0, no = 0;
    // stream arenas: patches, halo nodes, patch triangles, corner-list offsets
    int64_t pp0 = 0, npp = 0, hh0 = 0, nhh = 0, t0 = 0, nt = 0, cp0 = 0, ncp = 0;
  };
  bool arena = false;
  FreeList fl_nodes, fl_elems, fl_bodies, fl_pairs, fl_heights, fl_occ;
  // stream arenas (fw_set_path(FW_PATH_STREAM) before fw_arena_init): the
  // records of each committed scene's patches; owned-node records use the
  // scene's node range and corner lists its 3 x triangle range
  bool a_stream = false;
  FreeList fl_patch, fl_halo, fl_ptri, fl_csrp;
  int32_t* d_plist = nullptr;     // the active scenes' patches (CTA -> patch)
  int32_t* d_budget = nullptr;    // fw_step_served_budget: per-scene substep budgets
  int32_t* d_budget2 = nullptr;   // ... of the second segment
  float* d_dt2 = nullptr;         // ... and its step sizes
  std::vector<int32_t> h_budget, h_budget2;
  std::vector<float> h_dt2;
  unsigned char* d_stage = nullptr;  // device staging buffer of fw_arena_commit_pack
  size_t stage_cap = 0;
  int32_t* d_slist = nullptr;     // the active scenes (k_control_scenes)
  int4* d_srng = nullptr;         // per scene: first body, bodies, first pair, pairs
  std::vector<int32_t> h_slist;
  int st_slist_n = 0;
  std::vector<int32_t> h_plist;
  int st_list_n = 0;
  std::vector<ArenaScene> ascenes;
  std::vector<int> free_scene_ids;
  std::vector<int32_t> a_body_scene;
  bool chunks_dirty = true;
  std::vector<int2> h_echunks, h_nchunks;
  int2 *d_echunks = nullptr, *d_nchunks = nullptr;
  int64_t chunk_cap = 0;
  float *a_young = nullptr, *a_poisson = nullptr, *a_rho = nullptr;
  // differentiable form
  Adj adj{};
  int adj_cap = 0;  // steps per segment the trajectory buffer holds
  Tan tan{};
  // stream path (FW_PATH_STREAM)
  StreamDev sd{};
  int st_P = 0;
  size_t st_smem = 0;
  float2* x_buf0 = nullptr;  // the position buffer allocated first (parity of the swaps)
  int st_ne = 0, st_no = 0;  // patch triangles and owned nodes (record counts)
  int st_nodes = kStreamNodes;  // FW_OPT_STREAM_PATCH: owned nodes per patch = threads per CTA
  int st_minb = 32;             // FW_OPT_STREAM_MINB: CTAs per SM the kernel's registers are budgeted for
  int st_bulk = 0;              // FW_OPT_STREAM_BULK: stage triangle records with one bulk copy
  size_t st_smem_bulk = 0;
  bool res_adj = false;            // the reverse pass runs resident (k_res_adj)
  size_t res_adj_smem = 0;
  unsigned long long* fll = nullptr;  // [2][N][4] flag-in-data force adjoints of the reverse pass
  float* d_poisson = nullptr;
  // path selection and the resident (shared-memory) step
  int path_req = FW_PATH_AUTO, patches_req = 0;
  int front_warps = 6;
  int res_threads = 512;     // FW_OPT_RES_THREADS
  int res_sync = 0;          // FW_OPT_RES_SYNC
  int64_t wait_limit = 0;    // FW_OPT_WAIT_LIMIT (0: the built-in limits)
  int withhold_cta = -1;     // FW_OPT_TEST_WITHHOLD
  // fw_energy scratch (plain cudaMalloc, freed in fw_destroy)
  EnergyChunk* d_echunk = nullptr;
  double4* d_epart = nullptr;
  int* d_efirst = nullptr;
  double4* d_eout = nullptr;
  size_t energy_cap = 0, energy_gcap = 0;
  bool res_ll = false;       // resident path uses flag-in-data words
  uint32_t res_epoch = 1;    // epoch base of the next resident launch
  int path = FW_PATH_GATHER;
  Res res{};
  size_t res_smem = 0;
  std::string res_reason;
  int64_t host_counter = 0;  // step counter of scene 0 (single-scene worlds)
  // FEM-FEM contact (fw_flex.cuh): staging, then the device state
  std::vector<int2> h_be;                   // boundary edges, global node ids
  std::vector<int32_t> h_be_off, h_be_cnt;  // per body
  struct FlexPair {
    int b1, b2;
    float pen, fric;
    int tied;
  };
  std::vector<FlexPair> h_flex;
  struct FlexSceneHost {
    int skip_bvh = 0;
    std::vector<int32_t> dom_obj, dom_body;
    std::vector<float4> dom_box;
  };
  std::map<int, FlexSceneHost> h_flex_scene;  // scene -> its domains (fw_set_flex_scene)
  std::vector<int> flex_scene_of;              // per FEM-FEM scene (kernel order): the scene
  bool has_flex = false;
  FlexDev fx{};
  size_t flex_pre_smem = 0;  // k_flex_pre: (domains + FEM bodies) boxes
  std::vector<double> flex_clock;  // per FEM-FEM scene: the float64 substep dt (host copy)
  double flex_clock_all = 0.0;     // fw_set_flex_clock before fw_finalize
  double* d_flex_clock = nullptr;
  int* d_flex_err = nullptr;
  int32_t* cfl_ord_buf = nullptr;  // CFL monitor (fw_set_cfl_monitor)
  float* cfl_coef_buf = nullptr;
  // spring-mass domains: per body its node mass (0: an FEM body)
  std::vector<float> h_spring_mass;
  bool has_springs = false;
  // rigid primitives (fw_rigid.cuh): staging, then the device state
  std::vector<Rigid> h_rigid;
  std::vector<float4> h_gbox;
  std::vector<int> h_gkind, h_gscene;
  bool rigid_set = false, has_rigid = false;
  RigidDev rd{};
  fw::RigidClock* d_rclock = nullptr;
};

namespace {

int fail(fw_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

// On failure the runtime's last-error state is cleared too, so that a later
// launch check of this or another context does not report a stale error.
#define FW_CUDA(ctx, call)                                                                 \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      cudaGetLastError();                                                                  \
      return fail((ctx), _e == cudaErrorMemoryAllocation ? FW_ERR_OOM : FW_ERR_CUDA,       \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    }                                                                                      \
  } while (0)

template <typename T>
int dalloc(fw_ctx* c, T** p, size_t count) {
  size_t bytes = sizeof(T) * (count ? count : 1);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess)
    return fail(c, FW_ERR_OOM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  c->allocs.push_back((void*)*p);
  return FW_OK;
}

template <typename T>
int upload(fw_ctx* c, T** p, const std::vector<T>& h) {
  int rc = dalloc(c, p, h.size());
  if (rc) return rc;
  if (!h.empty())
    FW_CUDA(c, cudaMemcpyAsync(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, c->stream));
  return FW_OK;
}

int check_kernel(fw_ctx* c, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, FW_ERR_CUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
  return FW_OK;
}

void set_grids(fw_ctx* c) {
  const int E = c->E > 0 ? c->E : 1, N = c->N > 0 ? c->N : 1;
  const int cap = c->grid_e_cap > 0 ? c->grid_e_cap : c->sms * 8;
  c->grid_e = std::max(1, std::min((E + c->block_e - 1) / c->block_e, cap));
  c->grid_n = std::max(1, (N + c->block_n - 1) / c->block_n);
}

// The FEM-FEM contact of one substep (force: the construction-time hash
// build only): k_flex_pre (hash clock, the rebuild when it fires, activation,
// the active work items), then the contact work items.
void flex_launch(fw_ctx* c, int force) {
  const FlexDev& f = c->fx;
  k_flex_pre<<<f.n_fs, kFlexScanThreads, c->flex_pre_smem, c->stream>>>(c->d, f, force);
  c->launches += 1;
  if (!force) {
    const int64_t threads = (int64_t)f.n_items * kFlexLanes;
    const int64_t want = (threads + kFlexContactThreads - 1) / kFlexContactThreads;
    const int bx = (int)std::max<int64_t>(1, std::min<int64_t>(want, 8 * c->sms) / f.n_fs);
    k_flex_contact<<<dim3(bx, f.n_fs), kFlexContactThreads, 0, c->stream>>>(c->d, f);
    c->launches += 1;
  }
}

// Kernel launches of one gather-path substep.
int step_launches(const fw_ctx* c) { return 2 + (c->has_flex ? 2 : 0) + (c->has_rigid ? 1 : 0); }

int launch_step(fw_ctx* c) {
  if (c->has_flex) flex_launch(c, 0);
  if (c->has_rigid) {
    // the element step plus one thread per FEM-rigid work item
    const int rb = std::max(1, std::min((c->d.n_ritems + c->block_e - 1) / c->block_e, c->sms * 8));
    k_elements_rigid<<<c->grid_e + rb, c->block_e, 0, c->stream>>>(c->d, c->grid_e);
    if (c->has_flex)
      k_nodes_rigid<true><<<c->grid_n, c->block_n, 0, c->stream>>>(c->d);
    else
      k_nodes_rigid<false><<<c->grid_n, c->block_n, 0, c->stream>>>(c->d);
    if (c->rd.n <= kRigidOneBlock / 32)
      k_rigid<<<1, 32 * c->rd.n, 0, c->stream>>>(c->d, c->rd);
    else
      k_rigid<<<(c->rd.n + kRigidThreads / 32 - 1) / (kRigidThreads / 32), kRigidThreads, 0, c->stream>>>(c->d, c->rd);
    c->launches += 1;
  } else {
    k_elements<<<c->grid_e, c->block_e, 0, c->stream>>>(c->d);
    if (c->has_flex)
      k_nodes_flex<<<c->grid_n, c->block_n, 0, c->stream>>>(c->d);
    else
      k_nodes<<<c->grid_n, c->block_n, 0, c->stream>>>(c->d);
  }
  c->launches += 2;
  return check_kernel(c, "step");
}

void drop_graphs(fw_ctx* c) {
  for (auto& g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  for (auto& g : c->adj_graphs) cudaGraphExecDestroy(g.second);
  c->adj_graphs.clear();
}

// A graph of the work `body` queues on the context stream, cached under key
// in cache.  A graph holds the world descriptor and buffer addresses it was
// captured with, so caches are dropped when those change.
template <class Body>
int cached_graph(fw_ctx* c, std::vector<std::pair<uint64_t, cudaGraphExec_t>>& cache, uint64_t key, Body body,
                 cudaGraphExec_t* out) {
  if (c->graph_stream != c->stream) {
    drop_graphs(c);
    c->graph_stream = c->stream;
  }
  for (auto& g : cache)
    if (g.first == key) {
      *out = g.second;
      return FW_OK;
    }
  if (cache.size() >= 16) {
    for (auto& g : cache) cudaGraphExecDestroy(g.second);
    cache.clear();
  }
  cudaGraph_t g = nullptr;
  FW_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  body();
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (ce != cudaSuccess) return fail(c, FW_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
  cudaGraphExec_t exec = nullptr;
  ce = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(c, FW_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
  cache.push_back({key, exec});
  *out = exec;
  return FW_OK;
}

uint32_t float_bits(float v) {
  uint32_t bits;
  memcpy(&bits, &v, sizeof(bits));
  return bits;
}

// Graph of n substeps (n <= kGraphSteps) of the gather step.
int get_graph(fw_ctx* c, int n, cudaGraphExec_t* out) {
  const uint64_t key = ((uint64_t)(c->d.uniform_dt ? 1 : 0) << 63) | ((uint64_t)n << 32) |
                       (c->d.uniform_dt ? float_bits(c->d.dt_uniform) : 0u);
  const int64_t before = c->launches;
  const int rc = cached_graph(c, c->graphs, key, [&] {
    for (int k = 0; k < n; ++k) launch_step(c);  // every launch of a substep, FEM-FEM contact included
  }, out);
  c->launches = before;  // counted when the graph is launched
  return rc;
}

int launch_resident(fw_ctx* c, int n);

int rebuild_chunks(fw_ctx* c);

int stream_steps(fw_ctx* c, int n);

int arena_stream_steps(fw_ctx* c, int n);

int run_steps(fw_ctx* c, int n) {
  int rc = FW_OK;
  if (c->arena && c->a_stream) return arena_stream_steps(c, n);
  if (c->arena && (rc = rebuild_chunks(c))) return rc;
  if (c->path == FW_PATH_RESIDENT && c->d.uniform_dt) return launch_resident(c, n);
  if (c->path == FW_PATH_STREAM) return stream_steps(c, n);
  c->host_counter += n;
  if (n >= kGraphSteps) {
    cudaGraphExec_t g = nullptr;
    rc = get_graph(c, kGraphSteps, &g);
    if (rc) return rc;
    while (n >= kGraphSteps) {
      FW_CUDA(c, cudaGraphLaunch(g, c->stream));
      c->launches += step_launches(c) * kGraphSteps;
      n -= kGraphSteps;
    }
  }
  if (n >= 2) {  // the remainder as one graph too
    cudaGraphExec_t g = nullptr;
    if ((rc = get_graph(c, n, &g))) return rc;
    FW_CUDA(c, cudaGraphLaunch(g, c->stream));
    c->launches += step_launches(c) * n;
    n = 0;
  }
  for (int k = 0; k < n && rc == FW_OK; ++k) rc = launch_step(c);
  return rc;
}


using StreamKernel = void (*)(Dev, StreamDev, const float2*, float2*, const float4*, float4*);

// The stream kernel of a launch shape (patch size, register budget, staging);
// nullptr for a shape that is not built.
StreamKernel stream_kernel(int nodes, int minb, int bulk) {
  if (nodes == 64 && minb == 32) return bulk ? k_stream<64, 32, true> : k_stream<64, 32, false>;
  if (nodes == 64 && minb == 16) return bulk ? k_stream<64, 16, true> : k_stream<64, 16, false>;
  if (nodes == 128 && minb == 16) return bulk ? k_stream<128, 16, true> : k_stream<128, 16, false>;
  if (nodes == 128 && minb == 8) return bulk ? k_stream<128, 8, true> : k_stream<128, 8, false>;
  // intermediate register budgets (40 and 48 registers), per-thread record loads only
  if (!bulk && nodes == 64 && minb == 24) return k_stream<64, 24, false>;
  if (!bulk && nodes == 64 && minb == 20) return k_stream<64, 20, false>;
  if (!bulk && nodes == 128 && minb == 12) return k_stream<128, 12, false>;
  if (!bulk && nodes == 128 && minb == 10) return k_stream<128, 10, false>;
  return nullptr;
}

// n substeps of the stream path: k_control + k_stream each, alternating the
// position / J2 buffers; graphs of up to kGraphSteps substeps, cached per
// (starting buffer, dt mode, dt, count).
int stream_steps(fw_ctx* c, int n) {
  c->host_counter += n;
  while (n > 0) {
    const int m = std::min(n, kGraphSteps);
    const uint64_t parity = c->d.x == c->x_buf0 ? 0 : 1;
    const uint64_t key = (1ull << 62) | (parity << 61) | ((uint64_t)(c->d.uniform_dt ? 1 : 0) << 60) |
                         ((uint64_t)m << 32) | (c->d.uniform_dt ? float_bits(c->d.dt_uniform) : 0u);
    cudaGraphExec_t g = nullptr;
    int rc = cached_graph(c, c->graphs, key, [&] {
      float2 *xa = c->d.x, *xb = c->d.x_alt;
      float4 *ja = c->d.j2state, *jb = c->d.j2_alt;
      for (int k = 0; k < m; ++k) {
        k_control<<<1, kMaxBlock, 0, c->stream>>>(c->d);
        // the patch step as a programmatic dependent of the control (see k_stream)
        cudaLaunchAttribute pdl[1];
        pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        pdl[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c->st_P);
        cfg.blockDim = dim3(c->st_nodes);
        cfg.dynamicSmemBytes = c->st_bulk ? c->st_smem_bulk : c->st_smem;
        cfg.stream = c->stream;
        cfg.attrs = pdl;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, stream_kernel(c->st_nodes, c->st_minb, c->st_bulk), c->d, c->sd,
                           (const float2*)xa, xb, (const float4*)ja, jb);
        std::swap(xa, xb);
        std::swap(ja, jb);
      }
    }, &g);
    if (rc) return rc;
    FW_CUDA(c, cudaGraphLaunch(g, c->stream));
    c->launches += 2 * m;
    if (m & 1) {
      std::swap(c->d.x, c->d.x_alt);
      std::swap(c->d.j2state, c->d.j2_alt);
    }
    n -= m;
  }
  return check_kernel(c, "stream step");
}

void rcb(const std::vector<float2>& x, std::vector<int>& idx, int lo, int hi, int p0, int np,
         std::vector<int>& part);

// (Re)build the patch-ordered records of the stream path from the element and
// node arrays (after finalize, and after a Young's modulus changes).
int stream_records(fw_ctx* c) {
  if (c->st_ne > 0)
    k_stream_elems<<<(c->st_ne + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->d, c->sd.eid, c->sd.conn,
                                                                               c->sd.elem, c->sd.lm, c->st_ne);
  if (c->st_no > 0)
    k_stream_nodes<<<(c->st_no + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->d, c->sd.nodes, c->sd.node,
                                                                               c->st_no);
  c->launches += 2;
  return check_kernel(c, "stream records");
}

// Patches of the stream path (host side, no context state): each body
// [noff[b], +ncnt[b]) of a node set cut into patches of at most patch_nodes
// nodes; per patch the owned nodes, the triangles touching them, the halo
// nodes, local connectivity and the owned nodes' corner lists in ascending
// element order.  Ids in the result are those of the input (conn / off /
// slot); a patch's scene is its first owned node's body's scene.
struct PatchSet {
  std::vector<StreamPatch> patches;
  std::vector<int32_t> rn, rh, re;  // owned nodes, halo nodes, patch triangles
  std::vector<uint2> rc;            // local corners of each patch triangle
  std::vector<uint16_t> rcp, rcs;   // corner-list offsets, corner lists
  int no_max = 1, nh_max = 1, ne_max = 1;
};

int make_patches(int N, int E, const int32_t* conn, const std::vector<int32_t>& off,
                 const std::vector<int32_t>& slot, const std::vector<float2>& x0, const std::vector<int32_t>& noff,
                 const std::vector<int32_t>& ncnt, const std::vector<int32_t>& body_scene, int patch_nodes,
                 PatchSet& out, std::string& why) {
  std::vector<int> part(N, -1), idx;
  int P = 0;
  for (size_t b = 0; b < noff.size(); ++b) {
    const int n0 = noff[b], nn = ncnt[b];
    if (nn <= 0) continue;
    const int np = (nn + patch_nodes - 1) / patch_nodes;
    idx.resize(nn);
    for (int k = 0; k < nn; ++k) idx[k] = n0 + k;
    rcb(x0, idx, 0, nn, P, np, part);
    P += np;
  }
  std::vector<std::vector<int>> owned(P);
  for (int i = 0; i < N; ++i) {
    if (part[i] < 0) {
      why = "stream path: node " + std::to_string(i) + " belongs to no body";
      return FW_ERR_ARG;
    }
    owned[part[i]].push_back(i);
  }
  std::vector<int> node_scene(N, 0), node_body(N, 0);
  for (size_t b = 0; b < noff.size(); ++b)
    for (int k = 0; k < ncnt[b]; ++k) {
      node_scene[noff[b] + k] = body_scene[b];
      node_body[noff[b] + k] = (int)b;
    }
  std::vector<StreamPatch>& patches = out.patches;
  patches.assign(P, StreamPatch{});
  std::vector<int32_t>& rn = out.rn;
  std::vector<int32_t>& rh = out.rh;
  std::vector<int32_t>& re = out.re;
  std::vector<uint2>& rc = out.rc;
  std::vector<uint16_t>& rcs = out.rcs;
  std::vector<int32_t> rcp;
  std::vector<int> loc(N, -1), eloc(E, -1);
  int no_max = 1, nh_max = 1, ne_max = 1;
  for (int p = 0; p < P; ++p) {
    const std::vector<int>& ow = owned[p];
    if ((int)ow.size() > patch_nodes) {
      why = "stream path: patch larger than " + std::to_string(patch_nodes) + " nodes";
      return FW_ERR_ARG;
    }
    std::vector<int> tri;
    for (int n : ow)
      for (int k = off[n]; k < off[n + 1]; ++k) tri.push_back(slot[k] / 3);
    std::sort(tri.begin(), tri.end());
    tri.erase(std::unique(tri.begin(), tri.end()), tri.end());
    std::vector<int> hal;
    for (int e : tri)
      for (int k = 0; k < 3; ++k) {
        const int n = conn[3 * e + k];
        if (part[n] != p) hal.push_back(n);
      }
    std::sort(hal.begin(), hal.end());
    hal.erase(std::unique(hal.begin(), hal.end()), hal.end());
    if (ow.size() + hal.size() >= 65536 || 3 * tri.size() >= 65536) {
      why = "stream path: patch too large for 16-bit local indices";
      return FW_ERR_ARG;
    }
    StreamPatch& sp = patches[p];
    sp.node_off = (int)rn.size();
    sp.no = (int)ow.size();
    sp.halo_off = (int)rh.size();
    sp.nh = (int)hal.size();
    sp.elem_off = (int)re.size();
    sp.ne = (int)tri.size();
    sp.csrp_off = (int)rcp.size();
    sp.csr_off = (int)rcs.size();
    sp.scene = node_scene[ow[0]];
    sp.body = node_body[ow[0]];
    for (int i = 0; i < sp.no; ++i) {
      loc[ow[i]] = i;
      rn.push_back(ow[i]);
    }
    for (int h = 0; h < sp.nh; ++h) {
      loc[hal[h]] = sp.no + h;
      rh.push_back(hal[h]);
    }
    for (int q = 0; q < sp.ne; ++q) {
      const int e = tri[q];
      eloc[e] = q;
      re.push_back(e);
      const uint32_t a = loc[conn[3 * e]], b = loc[conn[3 * e + 1]], cc = loc[conn[3 * e + 2]];
      const uint32_t writer = part[conn[3 * e]] == p ? 1u : 0u;
      rc.push_back(make_uint2(a | (b << 16), cc | (writer << 16)));
    }
    int cnt = 0;
    for (int i = 0; i < sp.no; ++i) {
      rcp.push_back((int32_t)cnt);
      const int n = ow[i];
      for (int k = off[n]; k < off[n + 1]; ++k) {
        rcs.push_back((uint16_t)(3 * eloc[slot[k] / 3] + slot[k] % 3));
        ++cnt;
      }
    }
    rcp.push_back((int32_t)cnt);
    if (cnt >= 65536) {
      why = "stream path: patch corner list too long";
      return FW_ERR_ARG;
    }
    for (int n : ow) loc[n] = -1;
    for (int n : hal) loc[n] = -1;
    for (int e : tri) eloc[e] = -1;
    no_max = std::max(no_max, sp.no);
    nh_max = std::max(nh_max, sp.nh);
    ne_max = std::max(ne_max, sp.ne);
  }
  out.rcp.assign(rcp.begin(), rcp.end());
  out.no_max = no_max;
  out.nh_max = nh_max;
  out.ne_max = ne_max;
  return FW_OK;
}

// Stream path of a finalized world: its patches, device arrays and records.
int build_stream(fw_ctx* c, const std::vector<int32_t>& off, const std::vector<int32_t>& slot,
                 const std::vector<float2>& x0, bool has_j2) {
  const int N = c->N, E = c->E;
  PatchSet ps;
  std::string why;
  if (make_patches(N, E, c->h_conn.data(), off, slot, x0, c->h_noff, c->h_ncnt, c->h_scene, c->st_nodes, ps, why))
    return fail(c, FW_ERR_ARG, "%s", why.c_str());
  const int P = (int)ps.patches.size();
  const std::vector<StreamPatch>& patches = ps.patches;
  const std::vector<int32_t>&rn = ps.rn, &rh = ps.rh, &re = ps.re;
  const std::vector<uint2>& rc = ps.rc;
  const std::vector<uint16_t>& rcs = ps.rcs;
  const int no_max = ps.no_max, nh_max = ps.nh_max, ne_max = ps.ne_max;
  const std::vector<uint16_t>& rcp16 = ps.rcp;
  int r;
  StreamPatch* dp = nullptr;
  int32_t *dn = nullptr, *dh = nullptr, *de = nullptr;
  uint2* dc = nullptr;
  uint16_t *dcp = nullptr, *dcs = nullptr;
  if ((r = upload(c, &dp, patches)) || (r = upload(c, &dn, rn)) || (r = upload(c, &dh, rh)) ||
      (r = upload(c, &de, re)) || (r = upload(c, &dc, rc)) || (r = upload(c, &dcp, rcp16)) ||
      (r = upload(c, &dcs, rcs)) || (r = dalloc(c, &c->d.x_alt, N)) ||
      (r = dalloc(c, &c->d.j2_alt, has_j2 ? E : 1)))
    return r;
  FW_CUDA(c, cudaMemcpyAsync(c->d.x_alt, c->d.x, sizeof(float2) * N, cudaMemcpyDeviceToDevice, c->stream));
  if (has_j2)
    FW_CUDA(c, cudaMemcpyAsync(c->d.j2_alt, c->d.j2state, sizeof(float4) * E, cudaMemcpyDeviceToDevice, c->stream));
  StreamElem* dse = nullptr;
  StreamNode* dsn = nullptr;
  int* derr = nullptr;
  if ((r = dalloc(c, &dse, re.size())) || (r = dalloc(c, &dsn, rn.size())) || (r = dalloc(c, &derr, 1))) return r;
  FW_CUDA(c, cudaMemsetAsync(derr, 0, sizeof(int), c->stream));
  c->sd = StreamDev{dp, dn, dh, de, dc, dcp, dcs, no_max, nh_max, ne_max, dse, dsn, derr};
  c->st_ne = (int)re.size();
  c->st_no = (int)rn.size();
  if ((r = stream_records(c))) return r;
  c->st_P = P;
  c->st_smem = sizeof(float2) * (size_t)(no_max + nh_max) + sizeof(float2) * 3 * (size_t)ne_max;
  c->st_smem_bulk = stream_rec_offset(no_max, nh_max, ne_max) + sizeof(StreamElem) * (size_t)ne_max;
  c->x_buf0 = c->d.x;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if ((long)c->st_smem > optin) return fail(c, FW_ERR_ARG, "stream path: patch needs %zu B of shared memory", c->st_smem);
  if ((long)c->st_smem_bulk > optin) c->st_bulk = 0;  // staging does not fit: plain loads
  for (int minb : {8, 10, 12, 16, 20, 24, 32})
    for (int bulk = 0; bulk < 2; ++bulk)
      if (StreamKernel k = stream_kernel(c->st_nodes, minb, bulk))
        FW_CUDA(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 64));
  return FW_OK;
}

void rcb(const std::vector<float2>& x, std::vector<int>& idx, int lo, int hi, int p0, int np,
         std::vector<int>& part) {
  if (np <= 1 || hi - lo <= 1) {
    for (int k = lo; k < hi; ++k) part[idx[k]] = p0;
    return;
  }
  float mnx = 3e38f, mny = 3e38f, mxx = -3e38f, mxy = -3e38f;
  for (int k = lo; k < hi; ++k) {
    const float2 q = x[idx[k]];
    mnx = std::min(mnx, q.x); mxx = std::max(mxx, q.x);
    mny = std::min(mny, q.y); mxy = std::max(mxy, q.y);
  }
  const int axis = (mxx - mnx) >= (mxy - mny) ? 0 : 1;
  const int k1 = np / 2;
  const int mid = lo + (int)(((int64_t)(hi - lo) * k1) / np);
  std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int a, int b) {
    const float va = axis ? x[a].y : x[a].x, vb = axis ? x[b].y : x[b].x;
    return va < vb || (va == vb && a < b);
  });
  rcb(x, idx, lo, mid, p0, k1, part);
  rcb(x, idx, mid, hi, p0 + k1, np - k1, part);
}

// Build the patches of the resident path; returns FW_OK, or a positive value
// (with c->res_reason) when the world does not fit and the gather path is used.
int build_resident(fw_ctx* c, const std::vector<int32_t>& off, const std::vector<int32_t>& slot,
                   const std::vector<float2>& x0, bool has_j2) {
  const int N = c->N, E = c->E;
  if (c->S != 1) { c->res_reason = "more than one scene"; return 1; }
  if ((int)c->h_pairs.size() > kResMaxPairs) { c->res_reason = "more than 64 contact pairs"; return 1; }
  int sms = 148, optin = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  int P = c->patches_req > 0 ? c->patches_req : std::max(1, std::min(sms, (N + 127) / 128));
  if (P > N) P = N;
  std::vector<int> idx(N), part(N, 0);
  for (int i = 0; i < N; ++i) idx[i] = i;
  rcb(x0, idx, 0, N, 0, P, part);
  std::vector<std::vector<int>> owned(P), pel(P);
  for (int i = 0; i < N; ++i) owned[part[i]].push_back(i);
  for (int e = 0; e < E; ++e) {
    int ps[3] = {part[c->h_conn[3 * e]], part[c->h_conn[3 * e + 1]], part[c->h_conn[3 * e + 2]]};
    for (int k = 0; k < 3; ++k) {
      bool dup = false;
      for (int j = 0; j < k; ++j) dup |= ps[j] == ps[k];
      if (!dup) pel[ps[k]].push_back(e);
    }
  }
  std::vector<char> exported(N, 0);
  std::vector<std::vector<int>> halo(P);
  for (int p = 0; p < P; ++p) {
    std::vector<int>& h = halo[p];
    for (int e : pel[p])
      for (int k = 0; k < 3; ++k) {
        const int n = c->h_conn[3 * e + k];
        if (part[n] != p) h.push_back(n);
      }
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    for (int n : h) exported[n] = 1;
  }
  std::vector<char> body_bnd(N, 0);
  for (size_t k = 0; k < c->h_bnodes.size(); ++k) body_bnd[c->h_bnodes[k]] = 1;
  // group 1 first (read by other patches or on a body boundary), each group ascending
  for (int p = 0; p < P; ++p)
    std::stable_partition(owned[p].begin(), owned[p].end(),
                          [&](int n) { return exported[n] || body_bnd[n]; });
  std::vector<ResPatch> patches(P);
  std::vector<int32_t> rnodes, rhalo, reid, rcsrp;
  std::vector<uint2> rconn;
  std::vector<uint16_t> rcsrs;
  std::vector<int> loc(N, -1), eloc(E, -1);
  int no_max = 0, nh_max = 0, ne_max = 0, ncsr_max = 0;
  for (int p = 0; p < P; ++p) {
    ResPatch& rp = patches[p];
    const std::vector<int>& ow = owned[p];
    const std::vector<int>& h = halo[p];
    rp.node_off = (int)rnodes.size();
    rp.no = (int)ow.size();
    rp.n_g1 = 0;
    for (int n : ow) rp.n_g1 += (exported[n] || body_bnd[n]) ? 1 : 0;
    rp.halo_off = (int)rhalo.size();
    rp.nh = (int)h.size();
    if (rp.no + rp.nh >= 65536) { c->res_reason = "patch with >= 65536 nodes"; return 1; }
    for (int i = 0; i < rp.no; ++i) {
      loc[ow[i]] = i;
      rnodes.push_back(ow[i] | (exported[ow[i]] ? (int32_t)kExported : 0));
    }
    for (int j = 0; j < rp.nh; ++j) {
      loc[h[j]] = rp.no + j;
      rhalo.push_back(h[j]);
    }
    std::vector<int> inter, cut;
    for (int e : pel[p]) {
      const bool in = part[c->h_conn[3 * e]] == p && part[c->h_conn[3 * e + 1]] == p &&
                      part[c->h_conn[3 * e + 2]] == p;
      (in ? inter : cut).push_back(e);
    }
    rp.elem_off = (int)reid.size();
    rp.ne = (int)pel[p].size();
    rp.n_int = (int)inter.size();
    if (3 * rp.ne >= 65536) { c->res_reason = "patch with > 21845 triangles"; return 1; }
    int q = 0;
    for (const std::vector<int>* grp : {&inter, &cut})
      for (int e : *grp) {
        eloc[e] = q++;
        reid.push_back(e);
        const uint32_t a = loc[c->h_conn[3 * e]], b = loc[c->h_conn[3 * e + 1]], cc = loc[c->h_conn[3 * e + 2]];
        const uint32_t writer = part[c->h_conn[3 * e]] == p ? kJ2Writer : 0u;
        rconn.push_back(make_uint2(a | (b << 16), cc | (writer << 16)));
      }
    rp.csr_ptr_off = (int)rcsrp.size();
    rp.csr_off = (int)rcsrs.size();
    int cnt = 0;
    for (int i = 0; i < rp.no; ++i) {
      rcsrp.push_back(cnt);
      const int n = ow[i];
      for (int k = off[n]; k < off[n + 1]; ++k) {
        const int sl = slot[k];
        rcsrs.push_back((uint16_t)(3 * eloc[sl / 3] + sl % 3));
        ++cnt;
      }
    }
    rcsrp.push_back(cnt);
    rp.ncsr = cnt;
    for (int n : ow) loc[n] = -1;
    for (int n : h) loc[n] = -1;
    for (int e : pel[p]) eloc[e] = -1;
    no_max = std::max(no_max, rp.no);
    nh_max = std::max(nh_max, rp.nh);
    ne_max = std::max(ne_max, rp.ne);
    ncsr_max = std::max(ncsr_max, rp.ncsr);
  }
  Res& r = c->res;
  r.P = P;
  r.no_max = no_max;
  r.nh_max = nh_max;
  r.ne_max = ne_max;
  r.ncsr_max = ncsr_max;
  r.has_j2 = has_j2 ? 1 : 0;
  const size_t tab_bytes = c->h_heights.size() * sizeof(float) + c->h_occ.size();
  const bool stage = tab_bytes <= (size_t)kResTableBytes;
  r.tab_h = stage ? (int)c->h_heights.size() : 0;
  r.tab_o = stage ? (int)c->h_occ.size() : 0;
  r.n_bodies = c->B;
  if (c->B > 4096) { c->res_reason = "more than 4096 bodies"; return 1; }
  const size_t smem = res_layout(r, nullptr, nullptr);
  if ((long)smem + 64 > optin) {
    c->res_reason = "patch needs " + std::to_string(smem) + " B of shared memory";
    return 1;
  }
  const bool ll = c->res_sync == 0 && c->B <= kLLMaxBodies;
  ResKernel kern = res_kernel(c->front_warps, ll, c->res_threads);
  // The attribute is per function and process-wide: every context sets it to
  // the device maximum, so a context with small patches cannot lower the limit
  // below what another context launches with.
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, kern);
  cudaError_t e1 = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        optin - (int)fa.sharedSizeBytes);
  int per_sm = 0;
  cudaError_t e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, c->res_threads, smem);
  if (e1 != cudaSuccess || e2 != cudaSuccess || per_sm * sms < P) {
    cudaGetLastError();
    c->res_reason = "patches cannot all be resident";
    return 1;
  }
  int rc;
  ResPatch* dpatch = nullptr;
  int32_t *dn = nullptr, *dh = nullptr, *de = nullptr, *dcp = nullptr;
  uint2* dc = nullptr;
  uint16_t* dcs = nullptr;
  if ((rc = upload(c, &dpatch, patches)) || (rc = upload(c, &dn, rnodes)) || (rc = upload(c, &dh, rhalo)) ||
      (rc = upload(c, &de, reid)) || (rc = upload(c, &dc, rconn)) || (rc = upload(c, &dcp, rcsrp)) ||
      (rc = upload(c, &dcs, rcsrs)) || (rc = dalloc(c, &r.xpub, 2 * (size_t)N)) ||
      (rc = dalloc(c, &r.aabb3, 12 * (size_t)c->B)) || (rc = dalloc(c, &r.bar, 1)) ||
      (rc = dalloc(c, &r.err, 1)))
    return rc;
  if (ll) {
    const size_t nbll = 4 * (size_t)kBoxRing * c->B * P;
    if ((rc = dalloc(c, &r.xll, 4 * (size_t)N)) || (rc = dalloc(c, &r.bll, nbll))) return rc;
    FW_CUDA(c, cudaMemsetAsync(r.xll, 0, sizeof(unsigned long long) * 4 * (size_t)N, c->stream));
    FW_CUDA(c, cudaMemsetAsync(r.bll, 0, sizeof(unsigned long long) * nbll, c->stream));
  }
  c->res_ll = ll;
  c->res_epoch = 1;
  r.patch = dpatch;
  r.nodes = dn;
  r.halo = dh;
  r.eid = de;
  r.conn = dc;
  r.csr_ptr = dcp;
  r.csr_slot = dcs;
  FW_CUDA(c, cudaMemsetAsync(r.err, 0, sizeof(int), c->stream));
  c->res_smem = smem;
  return FW_OK;
}

int launch_resident(fw_ctx* c, int n) {
  // keep the arrivals counter (P * steps) far from int overflow
  constexpr int kMaxStepsPerLaunch = 1 << 20;
  while (n > kMaxStepsPerLaunch) {
    int rc = launch_resident(c, kMaxStepsPerLaunch);
    if (rc) return rc;
    n -= kMaxStepsPerLaunch;
  }
  if (n <= 0) return FW_OK;
  const int step0 = (int)c->host_counter;
  const bool ll = c->res_ll;
  if (ll && c->res_epoch > 0xF0000000u) {  // epochs about to wrap: clear the words, restart
    FW_CUDA(c, cudaMemsetAsync(c->res.xll, 0, sizeof(unsigned long long) * 4 * (size_t)c->N, c->stream));
    FW_CUDA(c, cudaMemsetAsync(c->res.bll, 0, sizeof(unsigned long long) * 4 * (size_t)kBoxRing * c->B * c->res.P,
                               c->stream));
    c->res_epoch = 1;
  }
  uint32_t ep0 = c->res_epoch;
  c->res_epoch += (uint32_t)n + 1u;
  c->res.wait_limit = c->wait_limit > 0 ? c->wait_limit : (ll ? kPollLimit : kSpinLimit);
  c->res.withhold_cta = c->withhold_cta;
  k_res_prologue<<<1, 256, 0, c->stream>>>(c->d, c->res, step0, ll ? 1 : 0);
  float dt = c->d.dt_uniform, damp = c->h_damp[0];
  void* args[] = {(void*)&c->d, (void*)&c->res, (void*)&step0, (void*)&n, (void*)&dt, (void*)&damp, (void*)&ep0};
  FW_CUDA(c, cudaLaunchCooperativeKernel((const void*)res_kernel(c->front_warps, ll, c->res_threads),
                                         dim3(c->res.P), dim3(c->res_threads), args, c->res_smem, c->stream));
  if (ll)
    k_res_epilogue_ll<<<1, 256, 0, c->stream>>>(c->d, c->res, step0, n);
  else
    k_res_epilogue<<<1, 256, 0, c->stream>>>(c->d, c->res, step0, n);
  c->launches += 3;
  c->host_counter += n;
  return check_kernel(c, "resident step");
}

int check_device_error(fw_ctx* c) {
  if (c->has_flex) {
    int ferr = 0;
    FW_CUDA(c, cudaMemcpyAsync(&ferr, c->d_flex_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
    if (ferr & 1)
      return fail(c, FW_ERR_ARG, "FEM-FEM contact: a node received more than %d contact forces in one substep",
                  kFlexListCap);
  }
  if (c->has_rigid) {
    int rerr = 0;
    FW_CUDA(c, cudaMemcpyAsync(&rerr, c->rd.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
    if (rerr & 1)
      return fail(c, FW_ERR_UNSUPPORTED,
                  "a rigid body came within 0.01 of a ground or of another contact rigid (rigid-rigid and "
                  "rigid-ground contact, the reference's constraint solve, are outside this library), or its "
                  "state is no longer finite");
  }
  if (c->path == FW_PATH_STREAM && c->sd.err) {
    int serr = 0;
    FW_CUDA(c, cudaMemcpyAsync(&serr, c->sd.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
    if (serr) return fail(c, FW_ERR_TIMEOUT, "stream step: a staged copy of triangle records did not complete");
  }
  if (c->path != FW_PATH_RESIDENT) return FW_OK;
  int err = 0;
  FW_CUDA(c, cudaMemcpyAsync(&err, c->res.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  if (err) return fail(c, FW_ERR_TIMEOUT, "resident step: a CTA gave up waiting for the others");
  return FW_OK;
}


int rebuild_chunks(fw_ctx* c) {
  if (!c->chunks_dirty) return FW_OK;
  c->h_echunks.clear();
  c->h_nchunks.clear();
  for (size_t s = 0; s < c->ascenes.size(); ++s) {
    const fw_ctx::ArenaScene& a = c->ascenes[s];
    if (!a.live || !c->cur_active[s]) continue;
    for (int64_t k = 0; k < a.ne; k += c->block_e)
      c->h_echunks.push_back(make_int2((int)(a.e0 + k), (int)std::min<int64_t>(c->block_e, a.ne - k)));
    for (int64_t k = 0; k < a.nn; k += c->block_n)
      c->h_nchunks.push_back(make_int2((int)(a.n0 + k), (int)std::min<int64_t>(c->block_n, a.nn - k)));
  }
  if ((int64_t)std::max(c->h_echunks.size(), c->h_nchunks.size()) > c->chunk_cap)
    return fail(c, FW_ERR_ARG, "arena: chunk list overflow");
  if (!c->h_echunks.empty())
    FW_CUDA(c, cudaMemcpyAsync(c->d_echunks, c->h_echunks.data(), sizeof(int2) * c->h_echunks.size(),
                               cudaMemcpyHostToDevice, c->stream));
  if (!c->h_nchunks.empty())
    FW_CUDA(c, cudaMemcpyAsync(c->d_nchunks, c->h_nchunks.data(), sizeof(int2) * c->h_nchunks.size(),
                               cudaMemcpyHostToDevice, c->stream));
  // pageable-source copies are staged before cudaMemcpyAsync returns, so the
  // host vectors may change again right away
  c->d.n_e_chunks = (int)c->h_echunks.size();
  c->d.n_n_chunks = (int)c->h_nchunks.size();
  c->grid_e = std::max(1, std::min(c->d.n_e_chunks, c->sms * 8));
  c->grid_n = std::max(1, std::min(c->d.n_n_chunks, c->sms * 8));
  drop_graphs(c);
  c->chunks_dirty = false;
  return FW_OK;
}

int set_scene_dt(fw_ctx* c, const float* dt) {
  bool same = c->cur_dt.size() == (size_t)c->S;
  for (int s = 0; same && s < c->S; ++s) same = memcmp(&c->cur_dt[s], &dt[s], sizeof(float)) == 0;
  if (same) return FW_OK;
  c->cur_dt.assign(dt, dt + c->S);
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_dt, c->cur_dt.data(), sizeof(float) * c->S,
                             cudaMemcpyHostToDevice, c->stream));
  // the copy reads c->cur_dt; keep it stable until the copy ran
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

// Relocation of one committed scene's arrays from scene-local to arena ids
// (fw_arena_commit_pack uploads them as packed), and the scene's control
// words (thread 0).
struct ArenaReloc {
  int n0, e0, b0, p0, h0, o0, s;
  int Ns, Es, Bs, Np;
  int32_t* rn;  // stream arenas: the scene's owned-node, halo and triangle id ranges (else null)
  int32_t* rh;
  int32_t* re;
  int Hs, Ts;
  StreamPatch* patch;  // stream arenas: the scene's patch records
  int Ps, hh0, t0, cp0;
  int4* srng;  // stream arenas: per-scene body / pair ranges
  float damp;
  int64_t count;  // max of the counts above and 3 Es
};

__global__ void k_arena_reloc(Dev d, ArenaReloc r) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    d.scene_damp[r.s] = r.damp;
    d.scene_counter[r.s] = 0;
    d.scene_mode_req[r.s] = 1;  // the zero-dt construction step at the next substep it runs
    d.scene_active[r.s] = 1;
    d.scene_bad[r.s] = 0;
    if (r.srng) r.srng[r.s] = make_int4(r.b0, r.Bs, r.p0, r.Np);
  }
  for (int64_t i = tid; i < r.count; i += stride) {
    if (i < r.Ns) {
      const int64_t g = r.n0 + i;
      d.node_word[g] += (uint32_t)r.b0 << fw::NODE_BODY_SHIFT;
      d.csr_off[g] += 3 * r.e0;
      d.csr_end[g] += 3 * r.e0;
      if (r.rn) r.rn[i] += r.n0;
    }
    if (i < 3 * (int64_t)r.Es) {
      const int64_t q = 3 * (int64_t)r.e0 + i;
      d.csr_slot[q] += 3 * r.e0;
      d.corner_pos[q] += 3 * r.e0;
      d.conn[q] += r.n0;
    }
    if (i < r.Es) d.emat[r.e0 + i].word += r.b0 << 2;
    if (i < r.Bs) {
      d.body_pair_off[r.b0 + i] += r.p0;
      d.body_scene[r.b0 + i] = r.s;
    }
    if (i < r.Np) {
      Pair& pr = d.pairs[r.p0 + i];
      pr.body += r.b0;
      if (pr.kind == fw::PAIR_HEIGHTFIELD) pr.table += r.h0;
      if (pr.kind == fw::PAIR_VOXEL) pr.table += r.o0;
    }
    if (r.rh && i < r.Hs) r.rh[i] += r.n0;
    if (r.re && i < r.Ts) r.re[i] += r.e0;
    if (r.patch && i < r.Ps) {
      StreamPatch& sp = r.patch[i];
      sp.node_off += r.n0;
      sp.halo_off += r.hh0;
      sp.elem_off += r.t0;
      sp.csrp_off += r.cp0;
      sp.csr_off += 3 * r.e0;
      sp.scene = r.s;
      sp.body += r.b0;
    }
  }
}

// Parts of a pack copied from the device staging buffer to their arena
// ranges: part k = stage[off[k] .. +len[k]) -> dst[k] (blockIdx.y = part).
constexpr int kScatterParts = 27;  // the pack's parts and the rest positions again (as the current ones)
struct ArenaScatter {
  unsigned char* dst[kScatterParts];
  uint32_t off[kScatterParts];
  uint32_t len[kScatterParts];
};

__global__ void k_arena_scatter(const unsigned char* __restrict__ stage, ArenaScatter sc) {
  const int k = blockIdx.y;
  const uint32_t len = sc.len[k];
  if (!len) return;
  const unsigned char* src = stage + sc.off[k];
  unsigned char* dst = sc.dst[k];
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (((uintptr_t)dst & 3) == 0 && (len & 3) == 0) {  // the source parts are 16-byte aligned
    const uint32_t* s4 = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d4 = reinterpret_cast<uint32_t*>(dst);
    for (uint32_t i = t; i < len / 4; i += stride) d4[i] = s4[i];
  } else {
    for (uint32_t i = t; i < len; i += stride) dst[i] = src[i];
  }
}

// Shared memory of a stream launch for the given patch maxima.
void stream_smem(int no_max, int nh_max, int ne_max, size_t* plain, size_t* bulk) {
  *plain = sizeof(float2) * (size_t)(no_max + nh_max) + sizeof(float2) * 3 * (size_t)ne_max;
  *bulk = stream_rec_offset(no_max, nh_max, ne_max) + sizeof(StreamElem) * (size_t)ne_max;
}

// Every built stream kernel of a patch size may use the device's opt-in shared memory.
int stream_attrs(fw_ctx* c, int optin) {
  for (int minb : {8, 10, 12, 16, 20, 24, 32})
    for (int bulk = 0; bulk < 2; ++bulk)
      if (StreamKernel k = stream_kernel(c->st_nodes, minb, bulk))
        FW_CUDA(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 64));
  return FW_OK;
}

// n substeps of a stream arena: k_control + k_stream over the active scenes'
// patches each, then (n odd) the carry back into the first buffers.
int arena_stream_steps(fw_ctx* c, int n) {
  if (c->chunks_dirty) {
    c->h_plist.clear();
    c->h_slist.clear();
    for (size_t s2 = 0; s2 < c->ascenes.size(); ++s2) {
      const fw_ctx::ArenaScene& a = c->ascenes[s2];
      if (!a.live || !c->cur_active[s2]) continue;
      c->h_slist.push_back((int32_t)s2);
      for (int64_t k = 0; k < a.npp; ++k) c->h_plist.push_back((int32_t)(a.pp0 + k));
    }
    // staged before the calls return
    if (!c->h_plist.empty())
      FW_CUDA(c, cudaMemcpyAsync(c->d_plist, c->h_plist.data(), sizeof(int32_t) * c->h_plist.size(),
                                 cudaMemcpyHostToDevice, c->stream));
    if (!c->h_slist.empty())
      FW_CUDA(c, cudaMemcpyAsync(c->d_slist, c->h_slist.data(), sizeof(int32_t) * c->h_slist.size(),
                                 cudaMemcpyHostToDevice, c->stream));
    c->st_list_n = (int)c->h_plist.size();
    c->st_slist_n = (int)c->h_slist.size();
    c->chunks_dirty = false;
  }
  c->host_counter += n;
  if (c->st_list_n == 0 || n <= 0) return FW_OK;
  float2 *xa = c->d.x, *xb = c->d.x_alt;
  float4 *ja = c->d.j2state, *jb = c->d.j2_alt;
  const StreamKernel k = stream_kernel(c->st_nodes, c->st_minb, c->st_bulk);
  const size_t smem = c->st_bulk ? c->st_smem_bulk : c->st_smem;
  const int gs = (c->st_slist_n + 127) / 128;
  // the patch step is a programmatic dependent of the control kernel (its
  // position gather overlaps the control; see k_stream)
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c->st_list_n);
  cfg.blockDim = dim3(c->st_nodes);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  for (int j = 0; j < n; ++j) {
    k_control_scenes<<<gs, 128, 0, c->stream>>>(c->d, c->d_slist, c->st_slist_n, c->d_srng);
    FW_CUDA(c, cudaLaunchKernelEx(&cfg, k, c->d, c->sd, (const float2*)xa, xb, (const float4*)ja, jb));
    std::swap(xa, xb);
    std::swap(ja, jb);
  }
  c->launches += 2 * (int64_t)n;
  if (n & 1) {
    k_stream_carry<<<c->st_list_n, c->st_nodes, 0, c->stream>>>(c->sd, xa, xb, ja, jb, c->d.has_j2);
    c->launches += 1;
  }
  return check_kernel(c, "arena stream step");
}

}  // namespace

// Host image of one staged scene with ids local to the scene (fw_arena_pack):
// every array an arena holds per scene, laid out in one host block (page-
// locked when asked for, so that a commit's copies run asynchronously).
struct fw_pack {
  enum Part {
    X0, V0, BCV, WORD, CBEG, CEND, SLOT, CPOS, CONN, EMAT, J2PAR, YOUNG, POISSON, RHO, POFF, PCNT, PAIRS,
    HEIGHTS, OCC, RN, RH, RE, RC, RCP, RCS, PATCH, NPARTS
  };
  int64_t Ns = 0, Es = 0, Bs = 0, Np = 0, Nh = 0, No = 0;
  int64_t Ps = 0, Hs = 0, Ts = 0, CPs = 0;  // stream records (patch_nodes > 0)
  int patch_nodes = 0;
  int no_max = 0, nh_max = 0, ne_max = 0;
  float damp = 0.f;
  unsigned char* block = nullptr;
  bool pinned = false;
  size_t bytes = 0;  // the block's size (parts 16-byte aligned)
  size_t off[NPARTS] = {}, len[NPARTS] = {};
  int64_t dev_bytes = 0;
  const void* at(Part p) const { return block + off[p]; }
  ~fw_pack() {
    if (pinned) cudaFreeHost(block);
    else free(block);
  }
};

namespace {

// The scene staged on context c (fw_set_nodes / fw_set_elements /
// fw_set_bodies / fw_set_scenes(1, ...) / fw_add_*_pair, ids local to the
// scene) as a pack; the stage is cleared.  Host work only.
int build_pack(fw_ctx* c, int patch_nodes, bool pinned, fw_pack** out) {
  const int64_t Ns = (int64_t)c->h_x.size() / 2, Es = (int64_t)c->h_conn.size() / 3;
  const int Bs = (int)c->h_noff.size();
  if (Ns <= 0 || Es <= 0 || Bs <= 0) return fail(c, FW_ERR_ARG, "fw_arena_pack: nothing staged");
  for (int b = 0; b < Bs; ++b)
    if (c->h_scene[b] != 0) return fail(c, FW_ERR_ARG, "fw_arena_pack: stage exactly one scene (scene 0)");
  if (patch_nodes != 0 && patch_nodes != 64 && patch_nodes != 128)
    return fail(c, FW_ERR_ARG, "fw_arena_pack: patch_nodes must be 0, 64 or 128");
  if (c->has_springs || !c->h_flex.empty() || !c->h_rigid.empty())
    return fail(c, FW_ERR_ARG, "fw_arena_pack: arena scenes hold FEM triangles and ground pairs only");
  std::vector<int32_t> node_body(Ns, -1), elem_body(Es, -1);
  for (int b = 0; b < Bs; ++b) {
    if (c->h_noff[b] < 0 || c->h_noff[b] + (int64_t)c->h_ncnt[b] > Ns || c->h_eoff[b] < 0 ||
        c->h_eoff[b] + (int64_t)c->h_ecnt[b] > Es)
      return fail(c, FW_ERR_ARG, "fw_arena_pack: body %d range out of bounds", b);
    for (int i = c->h_noff[b]; i < c->h_noff[b] + c->h_ncnt[b]; ++i) node_body[i] = b;
    for (int e = c->h_eoff[b]; e < c->h_eoff[b] + c->h_ecnt[b]; ++e) elem_body[e] = b;
  }
  for (int64_t e = 0; e < Es; ++e)
    for (int k = 0; k < 3; ++k) {
      const int n = c->h_conn[3 * e + k];
      if (elem_body[e] < 0 || n < 0 || n >= Ns || node_body[n] != elem_body[e])
        return fail(c, FW_ERR_ARG, "fw_arena_pack: element %lld has a bad node id", (long long)e);
    }
  for (int64_t i = 0; i < Ns; ++i)
    if (node_body[i] < 0) return fail(c, FW_ERR_ARG, "fw_arena_pack: node %lld belongs to no body", (long long)i);
  // node records (body ids local; the commit adds the scene's first body)
  std::vector<uint32_t> word(Ns);
  std::vector<float2> x0(Ns), v0(Ns), bcv(Ns);
  for (int64_t i = 0; i < Ns; ++i) {
    word[i] = (uint32_t)c->h_bc[i] | ((uint32_t)node_body[i] << fw::NODE_BODY_SHIFT);
    x0[i] = make_float2(c->h_x[2 * i], c->h_x[2 * i + 1]);
    v0[i] = make_float2(c->h_v[2 * i], c->h_v[2 * i + 1]);
    bcv[i] = make_float2(c->h_bcv[2 * i], c->h_bcv[2 * i + 1]);
  }
  for (int b = 0; b < Bs; ++b)
    for (int k = 0; k < c->h_bncnt[b]; ++k) word[c->h_bnodes[c->h_bnoff[b] + k]] |= fw::NODE_BOUNDARY;
  // triangles and the corner lists (ascending element per node)
  std::vector<int32_t> conn(c->h_conn.begin(), c->h_conn.end()), cbeg(Ns), cend(Ns), slot(3 * Es), cpos(3 * Es);
  std::vector<ElemMat> emat(Es);
  std::vector<float2> j2par(Es);
  for (int64_t e = 0; e < Es; ++e) {
    emat[e].area = emat[e].lam = emat[e].mu = 0.f;
    emat[e].word = (c->h_type[e] & 3) | (elem_body[e] << 2);
    j2par[e] = make_float2(c->h_sy[e], c->h_H[e]);
  }
  std::vector<int32_t> off(Ns + 1, 0);
  for (int64_t e = 0; e < Es; ++e)
    for (int k = 0; k < 3; ++k) off[conn[3 * e + k] + 1]++;
  for (int64_t i = 0; i < Ns; ++i) off[i + 1] += off[i];
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int64_t e = 0; e < Es; ++e)
      for (int k = 0; k < 3; ++k) {
        const int32_t at = fill[conn[3 * e + k]]++;
        slot[at] = (int32_t)(3 * e + k);
        cpos[3 * e + k] = at;
      }
    for (int64_t i = 0; i < Ns; ++i) {
      cbeg[i] = off[i];
      cend[i] = off[i + 1];
    }
  }
  // contact pairs grouped by body (stable: staging order within a body)
  std::vector<Pair> pairs = c->h_pairs;
  std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& x, const Pair& y) { return x.body < y.body; });
  std::vector<int32_t> poff(Bs, 0), pcnt(Bs, 0);
  for (const Pair& pr : pairs) {
    if (pr.body < 0 || pr.body >= Bs) return fail(c, FW_ERR_ARG, "fw_arena_pack: pair body out of range");
    pcnt[pr.body]++;
  }
  for (int b = 1; b < Bs; ++b) poff[b] = poff[b - 1] + pcnt[b - 1];
  // stream records
  PatchSet ps;
  if (patch_nodes) {
    std::string why;
    std::vector<int32_t> bscene(Bs, 0);
    if (make_patches((int)Ns, (int)Es, conn.data(), off, slot, x0, c->h_noff, c->h_ncnt, bscene, patch_nodes, ps, why))
      return fail(c, FW_ERR_ARG, "%s", why.c_str());
  }
  fw_pack* pk = new fw_pack();
  pk->Ns = Ns; pk->Es = Es; pk->Bs = Bs; pk->Np = (int64_t)pairs.size();
  pk->Nh = (int64_t)c->h_heights.size(); pk->No = (int64_t)c->h_occ.size();
  pk->damp = c->h_damp.empty() ? 0.f : c->h_damp[0];
  pk->patch_nodes = patch_nodes;
  pk->Ps = (int64_t)ps.patches.size(); pk->Hs = (int64_t)ps.rh.size(); pk->Ts = (int64_t)ps.re.size();
  pk->CPs = (int64_t)ps.rcp.size();
  pk->no_max = ps.no_max; pk->nh_max = ps.nh_max; pk->ne_max = ps.ne_max;
  struct Src { const void* p; size_t bytes; };
  const Src src[fw_pack::NPARTS] = {
      {x0.data(), sizeof(float2) * Ns}, {v0.data(), sizeof(float2) * Ns}, {bcv.data(), sizeof(float2) * Ns},
      {word.data(), sizeof(uint32_t) * Ns}, {cbeg.data(), sizeof(int32_t) * Ns}, {cend.data(), sizeof(int32_t) * Ns},
      {slot.data(), sizeof(int32_t) * 3 * Es}, {cpos.data(), sizeof(int32_t) * 3 * Es},
      {conn.data(), sizeof(int32_t) * 3 * Es}, {emat.data(), sizeof(ElemMat) * Es}, {j2par.data(), sizeof(float2) * Es},
      {c->h_E.data(), sizeof(float) * Es}, {c->h_nu.data(), sizeof(float) * Es}, {c->h_rho.data(), sizeof(float) * Es},
      {poff.data(), sizeof(int32_t) * Bs}, {pcnt.data(), sizeof(int32_t) * Bs}, {pairs.data(), sizeof(Pair) * pairs.size()},
      {c->h_heights.data(), sizeof(float) * c->h_heights.size()}, {c->h_occ.data(), c->h_occ.size()},
      {ps.rn.data(), sizeof(int32_t) * ps.rn.size()}, {ps.rh.data(), sizeof(int32_t) * ps.rh.size()},
      {ps.re.data(), sizeof(int32_t) * ps.re.size()}, {ps.rc.data(), sizeof(uint2) * ps.rc.size()},
      {ps.rcp.data(), sizeof(uint16_t) * ps.rcp.size()}, {ps.rcs.data(), sizeof(uint16_t) * ps.rcs.size()},
      {ps.patches.data(), sizeof(StreamPatch) * ps.patches.size()}};
  size_t total = 0;
  for (int k = 0; k < fw_pack::NPARTS; ++k) {
    pk->off[k] = total;
    pk->len[k] = src[k].bytes;
    total += (src[k].bytes + 15) & ~(size_t)15;
  }
  pk->bytes = total;
  if (pinned && cudaHostAlloc((void**)&pk->block, total ? total : 16, cudaHostAllocDefault) == cudaSuccess) {
    pk->pinned = true;
  } else {
    cudaGetLastError();
    pk->block = (unsigned char*)malloc(total ? total : 16);
    if (!pk->block) {
      delete pk;
      return fail(c, FW_ERR_OOM, "fw_arena_pack: host allocation of %zu bytes failed", total);
    }
  }
  for (int k = 0; k < fw_pack::NPARTS; ++k)
    if (src[k].bytes) memcpy(pk->block + pk->off[k], src[k].p, src[k].bytes);
  // device bytes of the scene's ranges
  int64_t dev = 48 * Ns + 136 * Es + 64 * pk->Np + 4 * pk->Nh + pk->No;
  if (patch_nodes)
    dev += (int64_t)sizeof(StreamPatch) * pk->Ps + 4 * pk->Hs + (4 + 8 + (int64_t)sizeof(StreamElem)) * pk->Ts +
           2 * pk->CPs + 6 * Es + (4 + (int64_t)sizeof(StreamNode)) * Ns;
  pk->dev_bytes = dev;
  // clear the stage for the next scene
  c->h_x.clear(); c->h_v.clear(); c->h_bc.clear(); c->h_bcv.clear();
  c->h_conn.clear(); c->h_type.clear(); c->h_E.clear(); c->h_nu.clear(); c->h_rho.clear(); c->h_sy.clear(); c->h_H.clear();
  c->h_noff.clear(); c->h_ncnt.clear(); c->h_eoff.clear(); c->h_ecnt.clear(); c->h_scene.clear();
  c->h_bnoff.clear(); c->h_bncnt.clear(); c->h_bnodes.clear(); c->h_pairs.clear(); c->h_heights.clear(); c->h_occ.clear();
  *out = pk;
  return FW_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" {

int fw_create(fw_ctx** out, int device) {
  if (!out) return FW_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return FW_ERR_CUDA;
  if (device < 0 || device >= ndev) return FW_ERR_ARG;
  fw_ctx* c = new fw_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return FW_ERR_CUDA;
  }
  c->stream = c->own_stream;
  *out = c;
  return FW_OK;
}

int fw_create_stage(fw_ctx** out) {
  if (!out) return FW_ERR_ARG;
  fw_ctx* c = new fw_ctx();
  c->device = -1;  // staging only: no device, no stream
  *out = c;
  return FW_OK;
}

void fw_destroy(fw_ctx* c) {
  if (!c) return;
  if (c->device < 0) {
    delete c;
    return;
  }
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  for (void* p : c->allocs) cudaFree(p);
  for (void* p : {(void*)c->d_echunk, (void*)c->d_epart, (void*)c->d_efirst, (void*)c->d_eout})
    if (p) cudaFree(p);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

const char* fw_last_error(const fw_ctx* c) { return c ? c->err.c_str() : "null context"; }

int fw_set_stream(fw_ctx* c, void* stream) {
  if (!c) return FW_ERR_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return FW_OK;
}

int fw_set_nodes(fw_ctx* c, int32_t n, const float* coords, const float* vel,
                 const int32_t* bc_bits, const float* bc_values) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized && !c->arena) return fail(c, FW_ERR_STATE, "fw_set_nodes after fw_finalize");
  if (n <= 0 || !coords) return fail(c, FW_ERR_ARG, "fw_set_nodes: need n_nodes > 0 and coords");
  if (!c->arena) c->N = n;
  c->h_x.assign(coords, coords + 2 * (size_t)n);
  c->h_v.assign(2 * (size_t)n, 0.f);
  if (vel) c->h_v.assign(vel, vel + 2 * (size_t)n);
  c->h_bc.assign(n, 0);
  if (bc_bits) c->h_bc.assign(bc_bits, bc_bits + n);
  c->h_bcv.assign(2 * (size_t)n, 0.f);
  if (bc_values) c->h_bcv.assign(bc_values, bc_values + 2 * (size_t)n);
  for (int i = 0; i < n; ++i)
    if (c->h_bc[i] & ~0x1FF) return fail(c, FW_ERR_ARG, "node %d: bc bits 0x%x outside 0x1FF", i, c->h_bc[i]);
  return FW_OK;
}

int fw_set_elements(fw_ctx* c, int32_t n, const int32_t* conn, const int32_t* mat_type,
                    const float* young, const float* poisson, const float* density,
                    const float* yield_stress, const float* hardening) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized && !c->arena) return fail(c, FW_ERR_STATE, "fw_set_elements after fw_finalize");
  if (n <= 0 || !conn || !mat_type || !young || !poisson || !density)
    return fail(c, FW_ERR_ARG, "fw_set_elements: need n_elems > 0 and conn/type/E/nu/rho");
  if (!c->arena) c->E = n;
  c->h_conn.assign(conn, conn + 3 * (size_t)n);
  c->h_type.assign(mat_type, mat_type + n);
  c->h_E.assign(young, young + n);
  c->h_nu.assign(poisson, poisson + n);
  c->h_rho.assign(density, density + n);
  c->h_sy.assign(n, 0.f);
  c->h_H.assign(n, 0.f);
  if (yield_stress) c->h_sy.assign(yield_stress, yield_stress + n);
  if (hardening) c->h_H.assign(hardening, hardening + n);
  for (int e = 0; e < n; ++e) {
    const int t = c->h_type[e];
    if (t != fw::MAT_SPRING && t != fw::MAT_ELASTIC && t != fw::MAT_NEOHOOKEAN && t != fw::MAT_MISES)
      return fail(c, FW_ERR_ARG, "element %d: unknown material type %d", e, t);
    if (t == fw::MAT_SPRING && c->arena)
      return fail(c, FW_ERR_ARG, "element %d: spring-mass domains are not served from an arena", e);
  }
  return FW_OK;
}

int fw_set_bodies(fw_ctx* c, int32_t nb, const int32_t* noff, const int32_t* ncnt,
                  const int32_t* eoff, const int32_t* ecnt, const int32_t* scene,
                  const int32_t* bnoff, const int32_t* bncnt, int32_t n_bnodes,
                  const int32_t* bnodes) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized && !c->arena) return fail(c, FW_ERR_STATE, "fw_set_bodies after fw_finalize");
  if (nb <= 0 || !noff || !ncnt || !eoff || !ecnt || !scene || !bnoff || !bncnt)
    return fail(c, FW_ERR_ARG, "fw_set_bodies: need n_bodies > 0 and all range arrays");
  if (nb >= (1 << 22)) return fail(c, FW_ERR_ARG, "fw_set_bodies: at most 4194303 bodies");
  if (!c->arena) c->B = nb;
  c->h_noff.assign(noff, noff + nb);
  c->h_ncnt.assign(ncnt, ncnt + nb);
  c->h_eoff.assign(eoff, eoff + nb);
  c->h_ecnt.assign(ecnt, ecnt + nb);
  c->h_scene.assign(scene, scene + nb);
  c->h_spring_mass.assign(nb, 0.0f);
  c->h_bnoff.assign(bnoff, bnoff + nb);
  c->h_bncnt.assign(bncnt, bncnt + nb);
  c->h_bnodes.assign(bnodes, bnodes + (n_bnodes > 0 ? n_bnodes : 0));
  return FW_OK;
}

int fw_set_scenes(fw_ctx* c, int32_t ns, const float* damping) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized && !c->arena) return fail(c, FW_ERR_STATE, "fw_set_scenes after fw_finalize");
  if (ns <= 0) return fail(c, FW_ERR_ARG, "fw_set_scenes: need n_scenes > 0");
  if (c->arena && ns != 1) return fail(c, FW_ERR_ARG, "arena: stage one scene at a time");
  if (!c->arena) c->S = ns;
  c->h_damp.assign(ns, 0.f);
  if (damping) c->h_damp.assign(damping, damping + ns);
  return FW_OK;
}

int fw_set_damping(fw_ctx* c, int32_t scene, float damping) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_set_damping needs a finalized world (not an arena)");
  if (scene < 0 || scene >= c->S) return fail(c, FW_ERR_ARG, "fw_set_damping: scene %d out of range", scene);
  c->h_damp[scene] = damping;
  // pageable source: the copy is staged before the call returns
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_damp + scene, &c->h_damp[scene], sizeof(float), cudaMemcpyHostToDevice,
                             c->stream));
  return FW_OK;
}

static int add_pair(fw_ctx* c, Pair p, const float* lo, const float* hi) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized && !c->arena) return fail(c, FW_ERR_STATE, "contact pair added after fw_finalize");
  if (!lo || !hi) return fail(c, FW_ERR_ARG, "contact pair: gate box required");
  if (p.body < 0) return fail(c, FW_ERR_ARG, "contact pair: bad body %d", p.body);
  p.glo[0] = lo[0];
  p.glo[1] = lo[1];
  p.ghi[0] = hi[0];
  p.ghi[1] = hi[1];
  c->h_pairs.push_back(p);
  return FW_OK;
}

int fw_add_plane_pair(fw_ctx* c, int32_t body, float penalty, const float* lo, const float* hi,
                      float px, float py, float nx, float ny) {
  Pair p{};
  p.kind = fw::PAIR_PLANE;
  p.body = body;
  p.penalty = penalty;
  p.f[0] = px;
  p.f[1] = py;
  p.f[2] = nx;
  p.f[3] = ny;
  return add_pair(c, p, lo, hi);
}

int fw_add_heightfield_pair(fw_ctx* c, int32_t body, float penalty, const float* lo,
                            const float* hi, int32_t n_samples, const float* heights, float lb_x,
                            float ub_x, int32_t reverse) {
  if (!c) return FW_ERR_ARG;
  if (n_samples < 2 || !heights)
    return fail(c, FW_ERR_ARG, "heightfield pair: need >= 2 samples");
  Pair p{};
  p.kind = fw::PAIR_HEIGHTFIELD;
  p.body = body;
  p.penalty = penalty;
  p.table = (int)c->h_heights.size();
  p.n0 = n_samples;
  p.n1 = reverse ? 1 : 0;
  p.f[0] = lb_x;
  p.f[1] = ub_x;
  c->h_heights.insert(c->h_heights.end(), heights, heights + n_samples);
  return add_pair(c, p, lo, hi);
}

int fw_add_voxel_pair(fw_ctx* c, int32_t body, float penalty, const float* lo, const float* hi,
                      int32_t nx, int32_t ny, const int32_t* occ, float lb_x, float lb_y, float dx,
                      float dz) {
  if (!c) return FW_ERR_ARG;
  if (nx <= 0 || ny <= 0 || !occ) return fail(c, FW_ERR_ARG, "voxel pair: need nx, ny > 0 and occupancy");
  Pair p{};
  p.kind = fw::PAIR_VOXEL;
  p.body = body;
  p.penalty = penalty;
  p.table = (int)c->h_occ.size();
  p.n0 = nx;
  p.n1 = ny;
  p.f[0] = lb_x;
  p.f[1] = lb_y;
  p.f[2] = dx;
  p.f[3] = dz;
  // 1 = occupied, 0 = free, 2 = any other value (neither test matches it)
  const size_t n = (size_t)nx * ny;
  const size_t base = c->h_occ.size();
  c->h_occ.resize(base + n);
  for (size_t k = 0; k < n; ++k) c->h_occ[base + k] = occ[k] == 1 ? 1 : (occ[k] == 0 ? 0 : 2);
  return add_pair(c, p, lo, hi);
}

int fw_set_boundary_edges(fw_ctx* c, int32_t n_edges, const int32_t* edges, const int32_t* body_off,
                          const int32_t* body_cnt) {
  if (!c || n_edges < 0 || (n_edges && !edges) || !body_off || !body_cnt) return FW_ERR_ARG;
  if (c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_set_boundary_edges after fw_finalize / on an arena");
  if (c->B <= 0) return fail(c, FW_ERR_STATE, "fw_set_boundary_edges before fw_set_bodies");
  for (int b = 0; b < c->B; ++b)
    if (body_off[b] < 0 || body_cnt[b] < 0 || (int64_t)body_off[b] + body_cnt[b] > n_edges)
      return fail(c, FW_ERR_ARG, "fw_set_boundary_edges: body %d range outside [0, %d)", b, n_edges);
  c->h_be.resize(n_edges);
  for (int k = 0; k < n_edges; ++k) c->h_be[k] = make_int2(edges[2 * k], edges[2 * k + 1]);
  c->h_be_off.assign(body_off, body_off + c->B);
  c->h_be_cnt.assign(body_cnt, body_cnt + c->B);
  return FW_OK;
}

int fw_set_flex_scene(fw_ctx* c, int32_t scene, int32_t skip_bvh, int32_t n_domains, const int32_t* dom_obj,
                      const int32_t* dom_body, const float* dom_box) {
  if (!c || n_domains < 0 || (n_domains && (!dom_obj || !dom_body || !dom_box))) return FW_ERR_ARG;
  if (c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_set_flex_scene after fw_finalize / on an arena");
  if (scene < 0) return fail(c, FW_ERR_ARG, "fw_set_flex_scene: scene %d", scene);
  fw_ctx::FlexSceneHost& h = c->h_flex_scene[scene];
  h.skip_bvh = skip_bvh ? 1 : 0;
  h.dom_obj.assign(dom_obj, dom_obj + n_domains);
  h.dom_body.assign(dom_body, dom_body + n_domains);
  h.dom_box.resize(n_domains);
  for (int g = 0; g < n_domains; ++g)
    h.dom_box[g] = make_float4(dom_box[4 * g], dom_box[4 * g + 1], dom_box[4 * g + 2], dom_box[4 * g + 3]);
  return FW_OK;
}

int fw_add_flex_pair(fw_ctx* c, int32_t body1, int32_t body2, float penalty, float friction) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_add_flex_pair after fw_finalize / on an arena");
  if (body1 < 0 || body2 < 0 || body1 >= c->B || body2 >= c->B || body1 == body2)
    return fail(c, FW_ERR_ARG, "fw_add_flex_pair: bodies %d, %d", body1, body2);
  c->h_flex.push_back(fw_ctx::FlexPair{body1, body2, penalty, friction, 0});
  return FW_OK;
}

int fw_tie_flex_pair(fw_ctx* c, int32_t pair) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_tie_flex_pair after fw_finalize / on an arena");
  if (pair < 0 || pair >= (int)c->h_flex.size()) return fail(c, FW_ERR_ARG, "fw_tie_flex_pair: pair %d", pair);
  c->h_flex[pair].tied = 1;
  return FW_OK;
}

int fw_mass_scaling(fw_ctx* c, float dt_target) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_mass_scaling needs a finalized world (not an arena)");
  if (!(dt_target > 0.0f)) return fail(c, FW_ERR_ARG, "fw_mass_scaling: dt_target must be > 0");
  if ((int)c->h_E.size() != c->E || (int)c->h_rho.size() != c->E)
    return fail(c, FW_ERR_STATE, "fw_mass_scaling: element materials are no longer staged");
  float *young = nullptr, *rho = nullptr, *dm = nullptr;
  int32_t* hit = nullptr;
  int rc;
  if ((rc = upload(c, &young, c->h_E)) || (rc = upload(c, &rho, c->h_rho)) || (rc = dalloc(c, &dm, c->E)) ||
      (rc = dalloc(c, &hit, c->E)))
    return rc;
  k_mass_scale_elems<<<(c->E + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->d, young, rho, dt_target, dm, hit);
  k_mass_scale_nodes<<<(c->N + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->d, dm, hit, dt_target);
  c->launches += 2;
  if ((rc = check_kernel(c, "mass scaling"))) return rc;
  if (c->path == FW_PATH_STREAM && (rc = stream_records(c))) return rc;  // its node records hold the masses
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_read_flex_state(fw_ctx* c, int32_t* item_cache, int32_t n_items, float* grid) {
  if (!c) return FW_ERR_ARG;
  if (!c->has_flex) return fail(c, FW_ERR_STATE, "fw_read_flex_state: the world has no FEM-FEM contact");
  if (n_items != c->fx.n_items) return fail(c, FW_ERR_ARG, "fw_read_flex_state: %d work items, not %d", c->fx.n_items, n_items);
  FlexGrid g{};
  if (item_cache)
    FW_CUDA(c, cudaMemcpyAsync(item_cache, c->fx.item_cache, sizeof(int32_t) * n_items, cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(&g, c->fx.g, sizeof(FlexGrid), cudaMemcpyDeviceToHost, c->stream));  // the first FEM-FEM scene
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  if (grid) {
    int est = g.estimate >= 0 ? g.estimate : g.estimate ^ 0x7FFFFFFF;  // ordered int -> float bits
    float estf;
    memcpy(&estf, &est, sizeof(float));
    const float v[8] = {(float)g.tc, (float)g.cnx, (float)g.cny, g.olx, g.oly, g.gsx, g.gsy, estf};
    memcpy(grid, v, sizeof(v));
  }
  return FW_OK;
}

int fw_set_spring_bodies(fw_ctx* c, int32_t n, const int32_t* bodies, const float* node_mass) {
  if (!c || n < 0 || (n && (!bodies || !node_mass))) return FW_ERR_ARG;
  if (c->finalized || c->arena) return fail(c, FW_ERR_STATE, "fw_set_spring_bodies after fw_finalize / on an arena");
  if ((int)c->h_spring_mass.size() != c->B) return fail(c, FW_ERR_STATE, "fw_set_spring_bodies before fw_set_bodies");
  for (int k = 0; k < n; ++k) {
    if (bodies[k] < 0 || bodies[k] >= c->B) return fail(c, FW_ERR_ARG, "fw_set_spring_bodies: body %d", bodies[k]);
    if (!(node_mass[k] > 0.0f)) return fail(c, FW_ERR_ARG, "fw_set_spring_bodies: node mass must be > 0");
    c->h_spring_mass[bodies[k]] = node_mass[k];
  }
  c->has_springs = n > 0;
  return FW_OK;
}

int fw_set_rigids(fw_ctx* c, int32_t n, const float* params, const int32_t* ints, int32_t n_ground,
                  const float* grounds) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized) return fail(c, FW_ERR_STATE, "fw_set_rigids after fw_finalize");
  if (c->arena) return fail(c, FW_ERR_STATE, "rigid bodies are not part of arena (served) worlds");
  if (n < 0 || n_ground < 0 || (n > 0 && (!params || !ints)) || (n_ground > 0 && !grounds))
    return fail(c, FW_ERR_ARG, "fw_set_rigids: bad sizes or pointers");
  c->h_rigid.assign(n, Rigid{});
  for (int a = 0; a < n; ++a) {
    const float* q = params + 20 * (size_t)a;
    Rigid& g = c->h_rigid[a];
    g.type = ints[4 * a];
    g.bc = ints[4 * a + 1];
    g.in_contact = ints[4 * a + 2];
    g.scene = ints[4 * a + 3];
    if (g.type != fw::RIGID_BALL && g.type != fw::RIGID_BOX && g.type != fw::RIGID_CAPSULE &&
        g.type != fw::RIGID_ANALYTICAL)
      return fail(c, FW_ERR_ARG, "rigid %d: type %d is not a ball, box, capsule or analytical entry", a, g.type);
    g.c[0] = q[0]; g.c[1] = q[1]; g.prim[0] = q[2]; g.prim[1] = q[3];
    g.radius = q[4]; g.quat = q[5]; g.mass = q[6]; g.inertia = q[7];
    g.V[0] = q[8]; g.V[1] = q[9]; g.W = q[10];
    g.bcT[0] = q[11]; g.bcT[1] = q[12]; g.bcG[0] = q[13]; g.bcG[1] = q[14]; g.bcR = q[15];
    g.lb[0] = q[16]; g.lb[1] = q[17]; g.ub[0] = q[18]; g.ub[1] = q[19];  // an analytical entry's first box
  }
  c->h_gbox.resize(n_ground);
  c->h_gkind.resize(n_ground);
  c->h_gscene.resize(n_ground);
  for (int k = 0; k < n_ground; ++k) {
    const float* q = grounds + 6 * (size_t)k;
    if (q[0] != 0.0f && q[0] != 1.0f) return fail(c, FW_ERR_ARG, "ground %d: kind must be 0 (plane) or 1 (box)", k);
    c->h_gkind[k] = (int)q[0];
    c->h_gbox[k] = make_float4(q[1], q[2], q[3], q[4]);
    c->h_gscene[k] = (int)q[5];
  }
  c->rigid_set = true;
  return FW_OK;
}

int fw_add_rigid_pair(fw_ctx* c, int32_t body, int32_t rigid, float penalty, float friction, int32_t skip_bvh,
                      int32_t tied) {
  if (!c) return FW_ERR_ARG;
  if (!c->rigid_set) return fail(c, FW_ERR_STATE, "fw_add_rigid_pair before fw_set_rigids");
  if (rigid < 0 || rigid >= (int)c->h_rigid.size())
    return fail(c, FW_ERR_ARG, "rigid pair: rigid %d outside [0, %d)", rigid, (int)c->h_rigid.size());
  Pair p{};
  p.kind = fw::PAIR_RIGID;
  p.body = body;
  p.penalty = penalty;
  p.table = rigid;
  p.n1 = skip_bvh ? 1 : 0;
  p.pad = tied ? 1 : 0;  // a tied pair (rigid pairs only)
  p.f[0] = friction;
  const float zero[2] = {0.0f, 0.0f};
  return add_pair(c, p, zero, zero);
}

int fw_gate_by_rigid(fw_ctx* c, int32_t entry) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized) return fail(c, FW_ERR_STATE, "fw_gate_by_rigid after fw_finalize");
  if (c->h_pairs.empty() || c->h_pairs.back().kind == fw::PAIR_RIGID)
    return fail(c, FW_ERR_STATE, "fw_gate_by_rigid: the last pair added is not a ground pair");
  if (entry < 0 || entry >= (int)c->h_rigid.size())
    return fail(c, FW_ERR_ARG, "fw_gate_by_rigid: entry %d outside [0, %d)", entry, (int)c->h_rigid.size());
  c->h_pairs.back().gate = entry + 1;
  return FW_OK;
}

int fw_set_rigid_clocks(fw_ctx* c, const int32_t* every, const float* dt, const float* damping) {
  if (!c || !every || !dt || !damping) return FW_ERR_ARG;
  if (!c->has_rigid) return fail(c, FW_ERR_STATE, "fw_set_rigid_clocks: no rigid bodies (or before fw_finalize)");
  std::vector<fw::RigidClock> ck(c->S);
  for (int s = 0; s < c->S; ++s) {
    if (every[s] < 1) return fail(c, FW_ERR_ARG, "fw_set_rigid_clocks: every[%d] must be >= 1", s);
    ck[s] = fw::RigidClock{every[s], dt[s], damping[s], 0};
  }
  FW_CUDA(c, cudaMemcpyAsync(c->d_rclock, ck.data(), sizeof(fw::RigidClock) * ck.size(), cudaMemcpyHostToDevice,
                             c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));  // ck lives on this stack frame
  return FW_OK;
}

int fw_set_rigid_clock(fw_ctx* c, int32_t every, float dt, float damping) {
  if (!c) return FW_ERR_ARG;
  if (!c->has_rigid) return fail(c, FW_ERR_STATE, "fw_set_rigid_clock: no rigid bodies (or before fw_finalize)");
  const std::vector<int32_t> e(c->S, every);
  const std::vector<float> t(c->S, dt), m(c->S, damping);
  return fw_set_rigid_clocks(c, e.data(), t.data(), m.data());
}

int fw_read_rigids(fw_ctx* c, float* out, int32_t* flags) {
  if (!c || !out) return FW_ERR_ARG;
  if (!c->has_rigid) return fail(c, FW_ERR_STATE, "fw_read_rigids: no rigid bodies (or before fw_finalize)");
  std::vector<Rigid> h(c->rd.n);
  int err = 0;
  FW_CUDA(c, cudaMemcpyAsync(h.data(), c->rd.rig, sizeof(Rigid) * h.size(), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(&err, c->rd.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  for (size_t a = 0; a < h.size(); ++a) {
    const Rigid& g = h[a];
    float* o = out + 12 * a;
    o[0] = g.c[0]; o[1] = g.c[1]; o[2] = g.quat; o[3] = g.V[0]; o[4] = g.V[1]; o[5] = g.W;
    o[6] = g.U[0]; o[7] = g.U[1]; o[8] = g.lb[0]; o[9] = g.lb[1]; o[10] = g.ub[0]; o[11] = g.ub[1];
  }
  if (flags) *flags = err;
  return FW_OK;
}

int fw_set_flex_clock(fw_ctx* c, double dt) {
  if (!c) return FW_ERR_ARG;
  for (double& v : c->flex_clock) v = dt;
  c->flex_clock_all = dt;
  if (c->has_flex)
    FW_CUDA(c, cudaMemcpyAsync(c->d_flex_clock, c->flex_clock.data(), sizeof(double) * c->flex_clock.size(),
                               cudaMemcpyHostToDevice, c->stream));
  return FW_OK;
}

int fw_set_flex_clocks(fw_ctx* c, const double* dt) {
  if (!c || !dt) return FW_ERR_ARG;
  if (!c->has_flex) return fail(c, FW_ERR_STATE, "fw_set_flex_clocks: no FEM-FEM contact (or before fw_finalize)");
  for (size_t k = 0; k < c->flex_clock.size(); ++k) c->flex_clock[k] = dt[c->flex_scene_of[k]];
  FW_CUDA(c, cudaMemcpyAsync(c->d_flex_clock, c->flex_clock.data(), sizeof(double) * c->flex_clock.size(),
                             cudaMemcpyHostToDevice, c->stream));
  return FW_OK;
}

// Device state of the FEM-FEM contact: per scene with ContactFlexFlex pairs,
// its work items in the reference's order (per pair: domain2's boundary nodes
// against domain1's edges, then domain1's against domain2's;
// mixedcontact.py:1876-1924), its spatial hash arrays sized as the reference
// sizes them for that loop (femspringmanager.py:545-548 MAX_BOUNDARY_ELEMENTS;
// spatialmanager.py:520-525: 3^2 pairs per element, 100000 cells), and the
// per-node contribution lists.
int build_flex(fw_ctx* c) {
  const int B = c->B, N = c->N;
  if ((int)c->h_be_off.size() != B) return fail(c, FW_ERR_ARG, "FEM-FEM contact: fw_set_boundary_edges missing");
  const int n_be = (int)c->h_be.size();
  std::vector<int32_t> be_dom(std::max(n_be, 1), 0), be_off(B), be_cnt(B);
  int run = 0;
  for (int b = 0; b < B; ++b) {
    if (c->h_be_off[b] != run) return fail(c, FW_ERR_ARG, "FEM-FEM contact: boundary edges must be stored body by body");
    be_off[b] = c->h_be_off[b];
    be_cnt[b] = c->h_be_cnt[b];
    for (int k = 0; k < be_cnt[b]; ++k) {
      const int2 e = c->h_be[run + k];
      if (e.x < c->h_noff[b] || e.x >= c->h_noff[b] + c->h_ncnt[b] || e.y < c->h_noff[b] ||
          e.y >= c->h_noff[b] + c->h_ncnt[b])
        return fail(c, FW_ERR_ARG, "FEM-FEM contact: boundary edge %d leaves body %d", run + k, b);
      be_dom[run + k] = b;
    }
    run += be_cnt[b];
  }
  if (run != n_be || n_be == 0) return fail(c, FW_ERR_ARG, "FEM-FEM contact: boundary edge counts do not add up");
  // bodies of each scene (contiguous, in body order)
  std::vector<int> s_b0(c->S, -1), s_nb(c->S, 0);
  for (int b = 0; b < B; ++b) {
    const int sc = c->h_scene[b];
    if (s_b0[sc] < 0) s_b0[sc] = b;
    if (s_b0[sc] + s_nb[sc] != b) return fail(c, FW_ERR_ARG, "FEM-FEM contact: a scene's bodies must be contiguous");
    ++s_nb[sc];
  }
  // pairs grouped by scene, creation order kept within a scene
  std::map<int, std::vector<int>> pairs_of;
  for (size_t p = 0; p < c->h_flex.size(); ++p) {
    const fw_ctx::FlexPair& fp = c->h_flex[p];
    if (c->h_scene[fp.b1] != c->h_scene[fp.b2]) return fail(c, FW_ERR_ARG, "FEM-FEM pair %zu joins two scenes", p);
    pairs_of[c->h_scene[fp.b1]].push_back((int)p);
  }
  std::vector<int32_t> item_node, item_target, item_pair;
  std::vector<float> item_pen, item_fric;
  std::vector<int2> pair_body;
  std::vector<int32_t> pair_tied;
  std::vector<int4> segs;  // (first item, count, pair in its scene, target)
  std::vector<FlexScene> scs;
  std::vector<int32_t> dom_obj, dom_body;
  std::vector<float4> dom_box;
  std::vector<int32_t> slot(N, -1);
  int n_slots = 0, pair_base = 0, max_dom_fem = 1;
  c->flex_scene_of.clear();
  for (auto& kv : pairs_of) {
    const int sc = kv.first;
    auto it = c->h_flex_scene.find(sc);
    if (it == c->h_flex_scene.end()) return fail(c, FW_ERR_ARG, "FEM-FEM contact: fw_set_flex_scene missing for scene %d", sc);
    const fw_ctx::FlexSceneHost& h = it->second;
    FlexScene fsd{};
    fsd.scene = sc;
    fsd.body0 = s_b0[sc];
    fsd.n_fem = s_nb[sc];
    fsd.dom_off = (int)dom_obj.size();
    fsd.n_dom = (int)h.dom_obj.size();
    fsd.skip_bvh = h.skip_bvh;
    for (int g = 0; g < fsd.n_dom; ++g) {
      const int db = h.dom_body[g];
      if (db >= 0 && (db < fsd.body0 || db >= fsd.body0 + fsd.n_fem))
        return fail(c, FW_ERR_ARG, "FEM-FEM contact: scene %d domain %d names body %d of another scene", sc, g, db);
      dom_obj.push_back(h.dom_obj[g]);
      dom_body.push_back(db);
      dom_box.push_back(h.dom_box[g]);
    }
    fsd.pair_off = (int)pair_body.size();
    fsd.n_pairs = (int)kv.second.size();
    fsd.seg_base = (int)segs.size();
    int scene_nodes = 0;
    for (int b = fsd.body0; b < fsd.body0 + fsd.n_fem; ++b) scene_nodes += c->h_ncnt[b];
    fsd.be0 = be_off[fsd.body0];
    fsd.n_be = 0;
    for (int b = fsd.body0; b < fsd.body0 + fsd.n_fem; ++b) fsd.n_be += be_cnt[b];
    const int max_nodes = std::max(scene_nodes + 1024, 2048);
    const int max_elements = std::max(fsd.n_be + 1024, max_nodes);
    fsd.max_pairs = 9 * max_elements;
    fsd.pair_base = pair_base;
    pair_base += fsd.max_pairs;
    fsd.cell_base = (int)scs.size() * kFlexMaxCells;
    for (int lp = 0; lp < fsd.n_pairs; ++lp) {
      const fw_ctx::FlexPair& fp = c->h_flex[kv.second[lp]];
      pair_body.push_back(make_int2(fp.b1, fp.b2));
      pair_tied.push_back(fp.tied);
      (fp.tied ? fsd.n_tied : fsd.n_untied) += c->h_bncnt[fp.b1] + c->h_bncnt[fp.b2];
      for (int side = 0; side < 2; ++side) {
        const int src = side == 0 ? fp.b2 : fp.b1, dst = side == 0 ? fp.b1 : fp.b2;
        segs.push_back(make_int4((int)item_node.size(), c->h_bncnt[src], lp, dst));
        for (int k = 0; k < c->h_bncnt[src]; ++k) {
          const int n = c->h_bnodes[c->h_bnoff[src] + k];
          item_node.push_back(n);
          item_target.push_back(dst);
          item_pair.push_back(fsd.pair_off + lp);
          item_pen.push_back(fp.pen);
          item_fric.push_back(fp.fric);
          if (slot[n] < 0) slot[n] = n_slots++;
        }
      }
    }
    fsd.n_seg = (int)segs.size() - fsd.seg_base;
    for (int k = fsd.be0; k < fsd.be0 + fsd.n_be; ++k)  // edge nodes receive the reactions
      for (int n : {c->h_be[k].x, c->h_be[k].y})
        if (slot[n] < 0) slot[n] = n_slots++;
    max_dom_fem = std::max(max_dom_fem, fsd.n_dom + fsd.n_fem);
    scs.push_back(fsd);
    c->flex_scene_of.push_back(sc);
  }
  const int n_fs = (int)scs.size();
  if (n_fs > 65535)  // the contact launch puts the scenes in gridDim.y
    return fail(c, FW_ERR_ARG, "FEM-FEM contact: %d scenes with FEM-FEM pairs in one world, at most 65535", n_fs);
  const int n_items = (int)item_node.size();
  FlexDev f{};
  f.n_items = n_items;
  f.n_fs = n_fs;
  f.mpd = std::max(powf(100000.0f, 0.5f), 1.0f);
  c->flex_clock.assign(n_fs, c->flex_clock_all);
  if (dom_obj.empty()) {
    dom_obj.push_back(0);
    dom_body.push_back(-1);
    dom_box.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
  }
  std::vector<int32_t> minus1(std::max(n_items, 1), -1);
  // each scene's seg_off has n_seg + 1 entries: seg_base + k
  const size_t n_segoff = segs.size() + (size_t)n_fs;
  int rc;
  int32_t *inode = nullptr, *itgt = nullptr, *ipair = nullptr, *icache = nullptr, *bdom = nullptr, *boff = nullptr,
          *bcnt = nullptr, *dobj = nullptr, *dbody = nullptr, *pact = nullptr, *stamp = nullptr, *ecount = nullptr,
          *ebase = nullptr, *ccount = nullptr, *cstart = nullptr, *cend = nullptr, *cursor = nullptr,
          *sorted = nullptr, *dslot = nullptr, *dcnt = nullptr, *ditem = nullptr, *dsegoff = nullptr;
  float *ipen = nullptr, *ifric = nullptr;
  int32_t *ptied = nullptr, *telem = nullptr;
  float *tw0 = nullptr, *tw1 = nullptr, *tgap = nullptr;
  int2 *pbody = nullptr, *dbe = nullptr, *crange = nullptr, *ecell = nullptr, *scell = nullptr;
  int4 *srec = nullptr, *dseg = nullptr;
  float4 *dbox = nullptr, *ebox = nullptr;
  float2* dforce = nullptr;
  FlexGrid* grid = nullptr;
  FlexScene* dsc = nullptr;
  const size_t cells = (size_t)n_fs * kFlexMaxCells;
  if ((rc = upload(c, &inode, item_node)) || (rc = upload(c, &itgt, item_target)) || (rc = upload(c, &ipair, item_pair)) ||
      (rc = upload(c, &ipen, item_pen)) || (rc = upload(c, &ifric, item_fric)) || (rc = upload(c, &icache, minus1)) ||
      (rc = upload(c, &pbody, pair_body)) || (rc = upload(c, &dbe, c->h_be)) || (rc = upload(c, &bdom, be_dom)) ||
      (rc = upload(c, &boff, be_off)) || (rc = upload(c, &bcnt, be_cnt)) || (rc = upload(c, &dobj, dom_obj)) ||
      (rc = upload(c, &dbody, dom_body)) || (rc = upload(c, &dbox, dom_box)) || (rc = upload(c, &dsc, scs)) ||
      (rc = dalloc(c, &pact, std::max<size_t>(1, pair_body.size()))) || (rc = dalloc(c, &stamp, B)) ||
      (rc = dalloc(c, &grid, n_fs)) || (rc = dalloc(c, &ebox, n_be)) || (rc = dalloc(c, &ecount, n_be)) ||
      (rc = dalloc(c, &ebase, n_be)) || (rc = dalloc(c, &ccount, cells)) || (rc = dalloc(c, &cstart, cells)) ||
      (rc = dalloc(c, &cend, cells)) || (rc = dalloc(c, &cursor, cells)) || (rc = dalloc(c, &crange, cells)) ||
      (rc = dalloc(c, &sorted, (size_t)pair_base)) || (rc = dalloc(c, &srec, (size_t)pair_base)) ||
      (rc = dalloc(c, &scell, (size_t)pair_base)) || (rc = dalloc(c, &ecell, n_be)) ||
      (rc = upload(c, &dseg, segs)) || (rc = dalloc(c, &dsegoff, n_segoff)) ||
      (rc = upload(c, &dslot, slot)) || (rc = dalloc(c, &dcnt, std::max(1, n_slots))) ||
      (rc = dalloc(c, &ditem, std::max(1, n_slots) * kFlexListCap)) ||
      (rc = dalloc(c, &dforce, std::max(1, n_slots) * kFlexListCap)) || (rc = dalloc(c, &c->d_flex_clock, n_fs)) ||
      (rc = dalloc(c, &c->d_flex_err, 1)) || (rc = upload(c, &ptied, pair_tied)) ||
      (rc = upload(c, &telem, minus1)) || (rc = dalloc(c, &tw0, std::max(n_items, 1))) ||
      (rc = dalloc(c, &tw1, std::max(n_items, 1))) || (rc = dalloc(c, &tgap, std::max(n_items, 1))))
    return rc;
  FW_CUDA(c, cudaMemsetAsync(grid, 0, sizeof(FlexGrid) * n_fs, c->stream));
  FW_CUDA(c, cudaMemsetAsync(c->d_flex_err, 0, sizeof(int), c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d_flex_clock, c->flex_clock.data(), sizeof(double) * n_fs, cudaMemcpyHostToDevice,
                             c->stream));
  FW_CUDA(c, cudaMemsetAsync(dcnt, 0, sizeof(int32_t) * std::max(1, n_slots), c->stream));
  FW_CUDA(c, cudaMemsetAsync(cstart, 0, sizeof(int32_t) * cells, c->stream));
  FW_CUDA(c, cudaMemsetAsync(cend, 0, sizeof(int32_t) * cells, c->stream));
  f.item_node = inode; f.item_target = itgt; f.item_pair = ipair; f.item_pen = ipen; f.item_fric = ifric;
  f.item_cache = icache; f.pair_body = pbody; f.be = dbe; f.be_dom = bdom; f.be_off = boff; f.be_cnt = bcnt;
  f.dom_obj = dobj; f.dom_body = dbody; f.dom_box = dbox; f.pair_active = pact; f.stamped = stamp; f.g = grid;
  f.ebox = ebox; f.ecount = ecount; f.ebase = ebase; f.cell_count = ccount; f.cell_start = cstart;
  f.cell_end = cend; f.cursor = cursor; f.sorted = sorted; f.crange = crange; f.ecell = ecell;
  f.srec = srec; f.scell = scell;
  f.seg = dseg; f.seg_off = dsegoff;
  f.sc = dsc; f.clock_dt = c->d_flex_clock; f.err = c->d_flex_err;
  f.pair_tied = ptied; f.tie_elem = telem; f.tie_w0 = tw0; f.tie_w1 = tw1; f.tie_gap = tgap;
  c->flex_pre_smem = sizeof(float4) * (size_t)max_dom_fem;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if ((long)c->flex_pre_smem > optin)
    return fail(c, FW_ERR_ARG, "FEM-FEM contact: a scene's domains need %zu B of shared memory", c->flex_pre_smem);
  if (c->flex_pre_smem > 48 * 1024)
    FW_CUDA(c, cudaFuncSetAttribute(k_flex_pre, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->flex_pre_smem));
  c->fx = f;
  c->d.flex_slot = dslot;
  c->d.flex_cnt = dcnt;
  c->d.flex_item = ditem;
  c->d.flex_force = dforce;
  c->has_flex = true;
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_finalize(fw_ctx* c) {
  if (!c) return FW_ERR_ARG;
  if (c->device < 0) return fail(c, FW_ERR_STATE, "fw_finalize on a staging context (fw_create_stage)");
  if (c->finalized) return fail(c, FW_ERR_STATE, "fw_finalize called twice");
  if (c->N <= 0 || c->E <= 0 || c->B <= 0 || c->S <= 0)
    return fail(c, FW_ERR_STATE, "fw_finalize: nodes, elements, bodies and scenes must be set");
  FW_CUDA(c, cudaSetDevice(c->device));
  const int N = c->N, E = c->E, B = c->B, S = c->S;
  // ---- validation and host-side packing
  std::vector<int32_t> node_body(N, -1), elem_body(E, -1);
  for (int b = 0; b < B; ++b) {
    if (c->h_scene[b] < 0 || c->h_scene[b] >= S) return fail(c, FW_ERR_ARG, "body %d: bad scene", b);
    if (c->h_noff[b] < 0 || c->h_ncnt[b] < 0 || (int64_t)c->h_noff[b] + c->h_ncnt[b] > N)
      return fail(c, FW_ERR_ARG, "body %d: node range outside [0, %d)", b, N);
    if (c->h_eoff[b] < 0 || c->h_ecnt[b] < 0 || (int64_t)c->h_eoff[b] + c->h_ecnt[b] > E)
      return fail(c, FW_ERR_ARG, "body %d: element range outside [0, %d)", b, E);
    for (int i = c->h_noff[b]; i < c->h_noff[b] + c->h_ncnt[b]; ++i) {
      if (node_body[i] >= 0) return fail(c, FW_ERR_ARG, "node %d in two bodies", i);
      node_body[i] = b;
    }
    for (int e = c->h_eoff[b]; e < c->h_eoff[b] + c->h_ecnt[b]; ++e) {
      if (elem_body[e] >= 0) return fail(c, FW_ERR_ARG, "element %d in two bodies", e);
      elem_body[e] = b;
    }
  }
  for (int i = 0; i < N; ++i)
    if (node_body[i] < 0) return fail(c, FW_ERR_ARG, "node %d belongs to no body", i);
  for (int e = 0; e < E; ++e) {
    if (elem_body[e] < 0) return fail(c, FW_ERR_ARG, "element %d belongs to no body", e);
    const bool spring = c->h_type[e] == fw::MAT_SPRING;
    if (spring != (c->h_spring_mass[elem_body[e]] > 0.0f))
      return fail(c, FW_ERR_ARG, "element %d: springs (type 0) belong to spring-mass bodies, triangles to FEM bodies", e);
    for (int k = 0; k < 3; ++k) {
      const int n = c->h_conn[3 * e + k];
      if (spring && k == 2) {
        if (n != -1) return fail(c, FW_ERR_ARG, "spring %d: third node id must be -1", e);
        continue;
      }
      if (n < 0 || n >= N) return fail(c, FW_ERR_ARG, "element %d: node id %d outside [0, %d)", e, n, N);
      if (node_body[n] != elem_body[e])
        return fail(c, FW_ERR_ARG, "element %d references node %d of another body", e, n);
    }
  }
  std::vector<uint32_t> word(N);
  for (int i = 0; i < N; ++i)
    word[i] = (uint32_t)c->h_bc[i] | ((uint32_t)node_body[i] << fw::NODE_BODY_SHIFT);
  for (int b = 0; b < B; ++b) {
    if (c->h_bnoff[b] < 0 || c->h_bncnt[b] < 0 ||
        (size_t)c->h_bnoff[b] + c->h_bncnt[b] > c->h_bnodes.size())
      return fail(c, FW_ERR_ARG, "body %d: boundary-node range out of bounds", b);
    for (int k = 0; k < c->h_bncnt[b]; ++k) {
      const int n = c->h_bnodes[c->h_bnoff[b] + k];
      if (n < 0 || n >= N || node_body[n] != b)
        return fail(c, FW_ERR_ARG, "body %d: boundary node %d not in the body", b, n);
      word[n] |= fw::NODE_BOUNDARY;
    }
  }
  // pairs grouped by body, launch order kept within a body
  std::vector<Pair> pairs = c->h_pairs;
  for (const Pair& p : pairs)
    if (p.body >= B) return fail(c, FW_ERR_ARG, "contact pair: body %d >= %d", p.body, B);
  int n_ritems = 0;  // FEM-rigid work items: per rigid pair (added order) its body's boundary nodes
  for (Pair& p : pairs)
    if (p.kind == fw::PAIR_RIGID) {
      if (p.table < 0 || p.table >= (int)c->h_rigid.size())
        return fail(c, FW_ERR_ARG, "rigid pair: rigid %d outside [0, %d)", p.table, (int)c->h_rigid.size());
      p.n0 = n_ritems;
      n_ritems += c->h_bncnt[p.body];
    }
  c->has_rigid = !c->h_rigid.empty();
  std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& a, const Pair& b) { return a.body < b.body; });
  std::vector<int32_t> poff(B, 0), pcnt(B, 0);
  for (size_t k = 0; k < pairs.size(); ++k) pcnt[pairs[k].body]++;
  for (int b = 1; b < B; ++b) poff[b] = poff[b - 1] + pcnt[b - 1];
  // CSR node -> (element, corner), ascending element
  std::vector<int32_t> off(N + 1, 0), slot(3 * (size_t)E);
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k)
      if (c->h_conn[3 * e + k] >= 0) off[c->h_conn[3 * e + k] + 1]++;
  for (int i = 0; i < N; ++i) off[i + 1] += off[i];
  std::vector<int32_t> cpos(3 * (size_t)E);
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int e = 0; e < E; ++e)
      for (int k = 0; k < 3; ++k) {
        if (c->h_conn[3 * e + k] < 0) {  // a spring's missing third corner: never written
          cpos[3 * (size_t)e + k] = cpos[3 * (size_t)e + k - 1];
          continue;
        }
        const int32_t at = fill[c->h_conn[3 * e + k]]++;
        slot[at] = 3 * e + k;
        cpos[3 * (size_t)e + k] = at;
      }
  }
  std::vector<ElemMat> emat(E);
  std::vector<float2> j2par(E);
  bool has_j2 = false;
  for (int e = 0; e < E; ++e) {
    emat[e].area = emat[e].lam = emat[e].mu = 0.f;
    emat[e].word = (c->h_type[e] & 3) | (elem_body[e] << 2);
    j2par[e] = make_float2(c->h_sy[e], c->h_H[e]);
    has_j2 |= c->h_type[e] == fw::MAT_MISES;
  }
  // device connectivity: a spring's missing third node repeats its second, so
  // loads that every element issues stay in bounds
  std::vector<int32_t> conn_dev(c->h_conn);
  for (int e = 0; e < E; ++e)
    if (conn_dev[3 * (size_t)e + 2] < 0) conn_dev[3 * (size_t)e + 2] = conn_dev[3 * (size_t)e + 1];
  std::vector<float2> x0(N), bcv(N), v0(N);
  for (int i = 0; i < N; ++i) {
    x0[i] = make_float2(c->h_x[2 * i], c->h_x[2 * i + 1]);
    v0[i] = make_float2(c->h_v[2 * i], c->h_v[2 * i + 1]);
    bcv[i] = make_float2(c->h_bcv[2 * i], c->h_bcv[2 * i + 1]);
  }
  // ---- device buffers
  Dev& d = c->d;
  d.N = N; d.E = E; d.B = B; d.S = S; d.P = (int)pairs.size(); d.has_j2 = has_j2;
  int rc = 0;
  if ((rc = upload(c, &d.x0, x0)) || (rc = upload(c, &d.x, x0)) || (rc = upload(c, &d.v, v0)) ||
      (rc = upload(c, &d.bcv, bcv)) || (rc = upload(c, &d.node_word, word)) ||
      (rc = dalloc(c, &d.mass, N)) || (rc = upload(c, &d.csr_off, off)) ||
      (rc = upload(c, &d.csr_slot, slot)) || (rc = upload(c, &d.corner_pos, cpos)) ||
      (rc = upload(c, &d.conn, conn_dev)) ||
      (rc = dalloc(c, &d.jinv, E)) || (rc = upload(c, &d.emat, emat)) ||
      (rc = upload(c, &d.j2par, j2par)) || (rc = dalloc(c, &d.j2state, has_j2 ? E : 1)) ||
      (rc = dalloc(c, &d.ndmass, E)) || (rc = dalloc(c, &d.corner, 3 * (size_t)E)) ||
      (rc = upload(c, &d.body_scene, c->h_scene)) || (rc = upload(c, &d.body_pair_off, poff)) ||
      (rc = dalloc(c, &d.body_lm, B)) ||
      (rc = upload(c, &d.body_pair_cnt, pcnt)) || (rc = upload(c, &d.pairs, pairs)) ||
      (rc = dalloc(c, &d.pair_active, pairs.size())) || (rc = upload(c, &d.heights, c->h_heights)) ||
      (rc = upload(c, &d.occ, c->h_occ)) || (rc = dalloc(c, &d.scene_dt, S)) ||
      (rc = upload(c, &d.scene_damp, c->h_damp)) || (rc = dalloc(c, &d.scene_counter, S)) ||
      (rc = dalloc(c, &d.scene_active, S)) || (rc = dalloc(c, &d.scene_mode_req, S)) ||
      (rc = dalloc(c, &d.scene_mode, S)) || (rc = dalloc(c, &d.aabb_ring, 8 * (size_t)B)) ||
      (rc = dalloc(c, &d.scene_bad, S)))
    return rc;
  FW_CUDA(c, cudaMemsetAsync(d.scene_bad, 0, sizeof(int32_t) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.j2state, 0, sizeof(float4) * (has_j2 ? E : 1), c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.pair_active, 0, sizeof(int32_t) * (pairs.empty() ? 1 : pairs.size()), c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_dt, 0, sizeof(float) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_counter, 0, sizeof(int32_t) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.aabb_ring, 0, sizeof(int32_t) * 8 * (size_t)B, c->stream));
  std::vector<int32_t> ones(S, 1);
  c->cur_active = ones;
  FW_CUDA(c, cudaMemcpyAsync(d.scene_active, ones.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(d.scene_mode_req, ones.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice, c->stream));
  float *dE = nullptr, *dnu = nullptr, *drho = nullptr;
  if ((rc = upload(c, &dE, c->h_E)) || (rc = upload(c, &dnu, c->h_nu)) || (rc = upload(c, &drho, c->h_rho)))
    return rc;
  d.csr_end = d.csr_off + 1;
  k_prepare_elements<<<(E + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(d, dE, dnu, drho, 0, E);
  k_prepare_mass<<<(N + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(d, 0, N);
  c->launches += 2;
  if ((rc = check_kernel(c, "prepare"))) return rc;
  if (c->has_springs) {  // a spring-mass domain's nodes carry its mass (femspringmanager.py:844-845)
    std::vector<float> sm(N);
    FW_CUDA(c, cudaMemcpyAsync(sm.data(), d.mass, sizeof(float) * N, cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int b = 0; b < B; ++b)
      if (c->h_spring_mass[b] > 0.0f)
        for (int k = 0; k < c->h_ncnt[b]; ++k) sm[c->h_noff[b] + k] = c->h_spring_mass[b];
    FW_CUDA(c, cudaMemcpyAsync(d.mass, sm.data(), sizeof(float) * N, cudaMemcpyHostToDevice, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  set_grids(c);
  if (c->has_springs && (c->path_req == FW_PATH_RESIDENT || c->path_req == FW_PATH_STREAM))
    return fail(c, FW_ERR_ARG, "spring-mass domains run on the gather path only");
  if (!c->h_flex.empty()) {
    if (c->path_req == FW_PATH_RESIDENT || c->path_req == FW_PATH_STREAM)
      return fail(c, FW_ERR_ARG, "FEM-FEM contact runs on the gather path only");
    if ((rc = build_flex(c))) return rc;
  }
  if (c->has_rigid) {
    if (c->path_req == FW_PATH_RESIDENT || c->path_req == FW_PATH_STREAM)
      return fail(c, FW_ERR_ARG, "FEM-rigid contact runs on the gather path only");
    std::vector<int32_t> bslot(N, 0);
    for (int b = 0; b < B; ++b)
      for (int k = 0; k < c->h_bncnt[b]; ++k) bslot[c->h_bnodes[c->h_bnoff[b] + k]] = k;
    // work item -> (pair, boundary node), for the element step's item blocks
    std::vector<int2> rwork(std::max(1, n_ritems), make_int2(0, 0));
    for (size_t q = 0; q < pairs.size(); ++q)
      if (pairs[q].kind == fw::PAIR_RIGID) {
        const Pair& p = pairs[q];
        for (int k = 0; k < c->h_bncnt[p.body]; ++k)
          rwork[p.n0 + k] = make_int2((int)q, c->h_bnodes[c->h_bnoff[p.body] + k]);
      }
    // per rigid, its pairs' item ranges in pair (= item) order; `pairs` is
    // grouped by body by now, so order the rigid pairs by first item again
    std::vector<Pair> rpairs;
    for (const Pair& p : pairs)
      if (p.kind == fw::PAIR_RIGID) rpairs.push_back(p);
    std::sort(rpairs.begin(), rpairs.end(), [](const Pair& a, const Pair& b) { return a.n0 < b.n0; });
    const int nr = (int)c->h_rigid.size();
    std::vector<int32_t> rp_off(nr + 1, 0);
    for (const Pair& p : rpairs) rp_off[p.table + 1]++;
    for (int g = 0; g < nr; ++g) rp_off[g + 1] += rp_off[g];
    std::vector<int2> rp_rng(std::max(1, rp_off[nr]));
    {
      std::vector<int32_t> fill(rp_off.begin(), rp_off.end() - 1);
      for (const Pair& p : rpairs) rp_rng[fill[p.table]++] = make_int2(p.n0, c->h_bncnt[p.body]);
    }
    // the scenes with rigids: their rigids and grounds, each a contiguous range
    std::vector<fw::RigidScene> rs;
    for (int a = 0, q = 0; a < nr;) {
      const int sc = c->h_rigid[a].scene;
      if (sc < 0 || sc >= S) return fail(c, FW_ERR_ARG, "rigid %d: scene %d outside [0, %d)", a, sc, S);
      if (!rs.empty() && sc <= rs.back().scene)
        return fail(c, FW_ERR_ARG, "rigids must be grouped by scene in ascending scene order");
      fw::RigidScene e{sc, a, 0, 0, 0, {0, 0, 0}};
      while (a < nr && c->h_rigid[a].scene == sc) c->h_rigid[a].rs = (int)rs.size(), ++a, ++e.rn;
      while (q < (int)c->h_gscene.size() && c->h_gscene[q] < sc) ++q;
      e.g0 = q;
      while (q < (int)c->h_gscene.size() && c->h_gscene[q] == sc) ++q, ++e.gn;
      rs.push_back(e);
    }
    for (size_t k = 1; k < c->h_gscene.size(); ++k)
      if (c->h_gscene[k] < c->h_gscene[k - 1]) return fail(c, FW_ERR_ARG, "grounds must be grouped by scene");
    RigidDev& r = c->rd;
    r.n = (int)c->h_rigid.size();
    r.n_ground = (int)c->h_gbox.size();
    r.n_items = n_ritems;
    r.n_rs = (int)rs.size();
    std::vector<fw::RigidClock> ck(S, fw::RigidClock{1, 0.0f, 0.0f, 0});
    if ((rc = upload(c, &r.rig, c->h_rigid)) || (rc = upload(c, &d.bslot, bslot)) ||
        (rc = upload(c, &d.rwork, rwork)) || (rc = dalloc(c, &d.rforce, (size_t)std::max(1, n_ritems))) ||
        (rc = dalloc(c, &r.item, (size_t)n_ritems)) || (rc = upload(c, &r.gbox, c->h_gbox)) ||
        (rc = upload(c, &r.gkind, c->h_gkind)) || (rc = upload(c, &r.rp_off, rp_off)) ||
        (rc = upload(c, &r.rp_rng, rp_rng)) || (rc = upload(c, &r.rs, rs)) ||
        (rc = upload(c, &c->d_rclock, ck)) || (rc = dalloc(c, &r.count, S)) || (rc = dalloc(c, &r.err, 1)) ||
        (rc = dalloc(c, &r.done, rs.size())))
      return rc;
    FW_CUDA(c, cudaMemsetAsync(r.count, 0, sizeof(int) * S, c->stream));
    FW_CUDA(c, cudaMemsetAsync(r.done, 0, sizeof(int) * rs.size(), c->stream));
    FW_CUDA(c, cudaMemsetAsync(r.err, 0, sizeof(int), c->stream));
    r.clock = c->d_rclock;
    d.rig = r.rig;
    d.ritem = r.item;
    d.n_ritems = n_ritems;
    k_rigid_init<<<(r.n + 127) / 128, 128, 0, c->stream>>>(r.rig, r.n);
    c->launches += 1;
    if ((rc = check_kernel(c, "rigid init"))) return rc;
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  // zero-dt construction step (setGlobalAABB -> substep(0, 0))
  if ((rc = launch_step(c))) return rc;
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  if (c->has_flex) {  // the initial FEM spatial hash (explicitloop.py:383-385)
    flex_launch(c, 1);
    if ((rc = check_kernel(c, "FEM-FEM hash"))) return rc;
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  c->path = FW_PATH_GATHER;
  if (c->has_flex || c->has_springs || c->has_rigid) {
    c->finalized = true;
    return FW_OK;
  }
  if (c->path_req == FW_PATH_STREAM) {
    if ((rc = build_stream(c, off, slot, x0, has_j2))) return rc;
    c->path = FW_PATH_STREAM;
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  } else if (c->path_req != FW_PATH_GATHER) {
    rc = build_resident(c, off, slot, x0, has_j2);
    if (rc < 0) return rc;
    if (rc == 0) {
      c->path = FW_PATH_RESIDENT;
    } else if (c->path_req == FW_PATH_RESIDENT) {
      return fail(c, FW_ERR_ARG, "resident path requested but unavailable: %s", c->res_reason.c_str());
    }
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  c->finalized = true;
  return FW_OK;
}

int fw_set_path(fw_ctx* c, int32_t path, int32_t patches) {
  if (!c) return FW_ERR_ARG;
  if (c->finalized) return fail(c, FW_ERR_STATE, "fw_set_path after fw_finalize");
  if (path != FW_PATH_AUTO && path != FW_PATH_GATHER && path != FW_PATH_RESIDENT && path != FW_PATH_STREAM)
    return fail(c, FW_ERR_ARG, "fw_set_path: unknown path %d", path);
  if (patches < 0) return fail(c, FW_ERR_ARG, "fw_set_path: patches < 0");
  c->path_req = path;
  c->patches_req = patches;
  return FW_OK;
}

static int shared_optin(fw_ctx* c) {
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  return optin;
}

int fw_set_option(fw_ctx* c, int32_t option, int32_t value) {
  if (!c) return FW_ERR_ARG;
  switch (option) {
    case FW_OPT_FRONT_WARPS: {
      if (c->finalized) return fail(c, FW_ERR_STATE, "FW_OPT_FRONT_WARPS after fw_finalize");
      bool ok = false;
      if (c->res_threads == 1024)
        for (int v : kFrontChoices1024) ok |= v == value;
      else
        for (int v : kFrontChoices) ok |= v == value;
      if (!ok)
        return fail(c, FW_ERR_ARG, "FW_OPT_FRONT_WARPS must be %s", c->res_threads == 1024 ? "8, 12 or 16 (1024 threads)"
                                                                                          : "2, 4, 6 or 8");
      c->front_warps = value;
      return FW_OK;
    }
    case FW_OPT_RES_THREADS: {
      if (c->finalized) return fail(c, FW_ERR_STATE, "FW_OPT_RES_THREADS after fw_finalize");
      if (value != 512 && value != 1024) return fail(c, FW_ERR_ARG, "FW_OPT_RES_THREADS must be 512 or 1024");
      c->res_threads = value;
      c->front_warps = value == 1024 ? 12 : 6;  // the default split for that size
      return FW_OK;
    }
    case FW_OPT_BLOCK_ELEMS:
    case FW_OPT_BLOCK_NODES: {
      if (value < 32 || value > kMaxBlock || value % 32)
        return fail(c, FW_ERR_ARG, "block size must be a multiple of 32 in [32, %d]", kMaxBlock);
      (option == FW_OPT_BLOCK_ELEMS ? c->block_e : c->block_n) = value;
      set_grids(c);
      drop_graphs(c);
      return FW_OK;
    }
    case FW_OPT_GRID_ELEMS: {
      if (value < 0) return fail(c, FW_ERR_ARG, "FW_OPT_GRID_ELEMS must be >= 0");
      c->grid_e_cap = value;
      set_grids(c);
      drop_graphs(c);
      return FW_OK;
    }
    case FW_OPT_WAIT_LIMIT:
      if (value < 0) return fail(c, FW_ERR_ARG, "FW_OPT_WAIT_LIMIT must be >= 0");
      c->wait_limit = value;
      return FW_OK;
    case FW_OPT_TEST_WITHHOLD:
      if (value < -1) return fail(c, FW_ERR_ARG, "FW_OPT_TEST_WITHHOLD must be >= -1");
      c->withhold_cta = value;
      return FW_OK;
    case FW_OPT_STREAM_PATCH: {
      if (c->finalized) return fail(c, FW_ERR_STATE, "FW_OPT_STREAM_PATCH after fw_finalize");
      if (value != 64 && value != 128) return fail(c, FW_ERR_ARG, "FW_OPT_STREAM_PATCH must be 64 or 128");
      c->st_nodes = value;
      c->st_minb = value == 64 ? 32 : 16;
      return FW_OK;
    }
    case FW_OPT_STREAM_MINB: {
      if (!stream_kernel(c->st_nodes, value, 0))
        return fail(c, FW_ERR_ARG, "FW_OPT_STREAM_MINB: %d-node patches are built for %s CTAs per SM", c->st_nodes,
                    c->st_nodes == 64 ? "16, 20, 24 or 32" : "8, 10, 12 or 16");
      c->st_minb = value;
      if (c->st_bulk && !stream_kernel(c->st_nodes, value, 1)) c->st_bulk = 0;  // loads-only budget
      drop_graphs(c);
      return FW_OK;
    }
    case FW_OPT_STREAM_BULK: {
      if (value != 0 && value != 1) return fail(c, FW_ERR_ARG, "FW_OPT_STREAM_BULK must be 0 or 1");
      if (value && c->finalized && c->path == FW_PATH_STREAM && c->st_smem_bulk + 64 > (size_t)shared_optin(c))
        return fail(c, FW_ERR_ARG, "FW_OPT_STREAM_BULK: the staged records do not fit in shared memory");
      if (value && !stream_kernel(c->st_nodes, c->st_minb, 1))
        return fail(c, FW_ERR_ARG, "FW_OPT_STREAM_BULK: no staged variant at %d CTAs per SM", c->st_minb);
      c->st_bulk = value;
      drop_graphs(c);
      return FW_OK;
    }
    case FW_OPT_RES_SYNC: {
      if (c->finalized) return fail(c, FW_ERR_STATE, "FW_OPT_RES_SYNC after fw_finalize");
      if (value != 0 && value != 1) return fail(c, FW_ERR_ARG, "FW_OPT_RES_SYNC must be 0 or 1");
      c->res_sync = value;
      return FW_OK;
    }
    default:
      return fail(c, FW_ERR_ARG, "fw_set_option: unknown option %d", option);
  }
}

int fw_get_option(const fw_ctx* c, int32_t option, int32_t* value) {
  if (!c || !value) return FW_ERR_ARG;
  switch (option) {
    case FW_OPT_FRONT_WARPS: *value = c->front_warps; return FW_OK;
    case FW_OPT_RES_THREADS: *value = c->res_threads; return FW_OK;
    case FW_OPT_BLOCK_ELEMS: *value = c->block_e; return FW_OK;
    case FW_OPT_BLOCK_NODES: *value = c->block_n; return FW_OK;
    case FW_OPT_STREAM_PATCH: *value = c->st_nodes; return FW_OK;
    case FW_OPT_STREAM_MINB: *value = c->st_minb; return FW_OK;
    case FW_OPT_STREAM_BULK: *value = c->st_bulk; return FW_OK;
    case FW_OPT_RES_SYNC: *value = c->res_sync; return FW_OK;
    default: return FW_ERR_ARG;
  }
}

int fw_snapshot(fw_ctx* c, int32_t slot) {
  if (c && c->has_rigid) return fail(c, FW_ERR_STATE, "snapshots do not hold the rigid bodies' state");
  if (c && c->has_flex)
    return fail(c, FW_ERR_STATE, "snapshots do not hold the FEM-FEM contact state (hash, element caches)");
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_snapshot before fw_finalize");
  if (slot < 0 || slot >= 1024) return fail(c, FW_ERR_ARG, "fw_snapshot: slot outside [0, 1024)");
  if ((int)c->snaps.size() <= slot) c->snaps.resize(slot + 1);
  fw_ctx::Snap& sn = c->snaps[slot];
  const size_t E = c->d.has_j2 ? c->E : 1;
  int rc;
  if (!sn.x) {
    if ((rc = dalloc(c, &sn.x, c->N)) || (rc = dalloc(c, &sn.v, c->N)) || (rc = dalloc(c, &sn.j2, E)) ||
        (rc = dalloc(c, &sn.counter, c->S)) || (rc = dalloc(c, &sn.ring, 8 * (size_t)c->B)) ||
        (rc = dalloc(c, &sn.mode_req, c->S)))
      return rc;
  }
  FW_CUDA(c, cudaMemcpyAsync(sn.x, c->d.x, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(sn.v, c->d.v, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(sn.j2, c->d.j2state, sizeof(float4) * E, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(sn.counter, c->d.scene_counter, sizeof(int32_t) * c->S, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(sn.ring, c->d.aabb_ring, sizeof(int32_t) * 8 * c->B, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(sn.mode_req, c->d.scene_mode_req, sizeof(int32_t) * c->S, cudaMemcpyDeviceToDevice, c->stream));
  sn.host_counter = c->host_counter;
  sn.valid = true;
  return FW_OK;
}

int fw_restore(fw_ctx* c, int32_t slot) {
  if (c && c->has_rigid) return fail(c, FW_ERR_STATE, "snapshots do not hold the rigid bodies' state");
  if (c && c->has_flex)
    return fail(c, FW_ERR_STATE, "snapshots do not hold the FEM-FEM contact state (hash, element caches)");
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_restore before fw_finalize");
  if (slot < 0 || slot >= (int)c->snaps.size() || !c->snaps[slot].valid)
    return fail(c, FW_ERR_ARG, "fw_restore: slot %d holds no snapshot", slot);
  fw_ctx::Snap& sn = c->snaps[slot];
  const size_t E = c->d.has_j2 ? c->E : 1;
  FW_CUDA(c, cudaMemcpyAsync(c->d.x, sn.x, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.v, sn.v, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.j2state, sn.j2, sizeof(float4) * E, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_counter, sn.counter, sizeof(int32_t) * c->S, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.aabb_ring, sn.ring, sizeof(int32_t) * 8 * c->B, cudaMemcpyDeviceToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_mode_req, sn.mode_req, sizeof(int32_t) * c->S, cudaMemcpyDeviceToDevice, c->stream));
  c->host_counter = sn.host_counter;
  return FW_OK;
}


int fw_arena_init(fw_ctx* c, int64_t max_nodes, int64_t max_elems, int32_t max_bodies, int32_t max_scenes,
                  int32_t max_pairs, int64_t max_heights, int64_t max_occ) {
  if (!c) return FW_ERR_ARG;
  if (c->device < 0) return fail(c, FW_ERR_STATE, "fw_arena_init on a staging context (fw_create_stage)");
  if (c->finalized) return fail(c, FW_ERR_STATE, "fw_arena_init on a finalized context");
  if (max_nodes <= 0 || max_elems <= 0 || max_bodies <= 0 || max_scenes <= 0 || max_pairs < 0 ||
      max_heights < 0 || max_occ < 0)
    return fail(c, FW_ERR_ARG, "fw_arena_init: capacities must be positive");
  if (max_nodes >= (1ll << 31) / 2 || 3 * max_elems >= (1ll << 31) || max_bodies >= (1 << 22))
    return fail(c, FW_ERR_ARG, "fw_arena_init: capacity beyond 32-bit indexing");
  FW_CUDA(c, cudaSetDevice(c->device));
  const int64_t N = max_nodes, E = max_elems;
  const int B = max_bodies, S = max_scenes + 1;  // scene S-1: the dead scene of free bodies
  Dev& d = c->d;
  d = Dev{};
  d.N = (int)N; d.E = (int)E; d.B = B; d.S = S; d.P = max_pairs; d.has_j2 = 1;
  int rc;
  if ((rc = dalloc(c, &d.x0, N)) || (rc = dalloc(c, &d.x, N)) || (rc = dalloc(c, &d.v, N)) ||
      (rc = dalloc(c, &d.bcv, N)) || (rc = dalloc(c, &d.node_word, N)) || (rc = dalloc(c, &d.mass, N)) ||
      (rc = dalloc(c, &d.csr_off, N)) || (rc = dalloc(c, &d.csr_end, N)) || (rc = dalloc(c, &d.csr_slot, 3 * E)) ||
      (rc = dalloc(c, &d.corner_pos, 3 * E)) ||
      (rc = dalloc(c, &d.conn, 3 * E)) || (rc = dalloc(c, &d.jinv, E)) || (rc = dalloc(c, &d.emat, E)) ||
      (rc = dalloc(c, &d.j2par, E)) || (rc = dalloc(c, &d.j2state, E)) || (rc = dalloc(c, &d.ndmass, E)) ||
      (rc = dalloc(c, &d.corner, 3 * E)) || (rc = dalloc(c, &d.body_scene, B)) ||
      (rc = dalloc(c, &d.body_pair_off, B)) || (rc = dalloc(c, &d.body_pair_cnt, B)) ||
      (rc = dalloc(c, &d.body_lm, B)) ||
      (rc = dalloc(c, &d.pairs, max_pairs)) || (rc = dalloc(c, &d.pair_active, max_pairs)) ||
      (rc = dalloc(c, &d.heights, max_heights)) || (rc = dalloc(c, &d.occ, max_occ)) ||
      (rc = dalloc(c, &d.scene_dt, S)) || (rc = dalloc(c, &d.scene_damp, S)) ||
      (rc = dalloc(c, &d.scene_counter, S)) || (rc = dalloc(c, &d.scene_active, S)) ||
      (rc = dalloc(c, &d.scene_mode_req, S)) || (rc = dalloc(c, &d.scene_mode, S)) ||
      (rc = dalloc(c, &d.aabb_ring, 8 * (size_t)B)) || (rc = dalloc(c, &c->a_young, E)) ||
      (rc = dalloc(c, &c->a_poisson, E)) || (rc = dalloc(c, &c->a_rho, E)) || (rc = dalloc(c, &d.scene_bad, S)))
    return rc;
  FW_CUDA(c, cudaMemsetAsync(d.scene_bad, 0, sizeof(int32_t) * S, c->stream));
  c->stage_cap = (size_t)64 << 20;  // packs up to 64 MB commit in one copy (larger ones part by part)
  if ((rc = dalloc(c, &c->d_stage, c->stage_cap))) return rc;
  c->chunk_cap = E / 32 + N / 32 + 2 * (int64_t)S + 16;
  if ((rc = dalloc(c, &c->d_echunks, c->chunk_cap)) || (rc = dalloc(c, &c->d_nchunks, c->chunk_cap))) return rc;
  std::vector<int32_t> dead(B, S - 1);
  FW_CUDA(c, cudaMemcpyAsync(d.body_scene, dead.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.body_pair_cnt, 0, sizeof(int32_t) * B, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.body_pair_off, 0, sizeof(int32_t) * B, c->stream));
  if (max_pairs) FW_CUDA(c, cudaMemsetAsync(d.pairs, 0, sizeof(Pair) * max_pairs, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_active, 0, sizeof(int32_t) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_mode_req, 0, sizeof(int32_t) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_counter, 0, sizeof(int32_t) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_dt, 0, sizeof(float) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.scene_damp, 0, sizeof(float) * S, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.aabb_ring, 0, sizeof(int32_t) * 8 * (size_t)B, c->stream));
  FW_CUDA(c, cudaMemsetAsync(d.j2state, 0, sizeof(float4) * E, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  d.use_chunks = 1;
  d.e_chunks = c->d_echunks;
  d.n_chunks = c->d_nchunks;
  c->fl_nodes.init(N);
  c->fl_elems.init(E);
  c->fl_bodies.init(B);
  c->fl_pairs.init(max_pairs);
  c->fl_heights.init(max_heights);
  c->fl_occ.init(max_occ);
  c->ascenes.assign(S, fw_ctx::ArenaScene{});
  c->a_body_scene.assign(B, S - 1);
  c->free_scene_ids.clear();
  for (int s2 = S - 2; s2 >= 0; --s2) c->free_scene_ids.push_back(s2);
  c->cur_active.assign(S, 0);
  c->N = (int)N; c->E = (int)E; c->B = B; c->S = S;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  c->arena = true;
  c->finalized = true;
  c->path = FW_PATH_GATHER;
  c->chunks_dirty = true;
  if (c->path_req == FW_PATH_STREAM) {
    // stream arena: record capacities (patches of a body: at most nodes / patch + 1;
    // patch triangles and halo nodes: at most twice the triangles / nodes, a
    // scene needing more waits like any scene that does not fit)
    const int64_t Pcap = N / c->st_nodes + B + 16, Hcap = 2 * N, Tcap = 2 * E, CPcap = N + Pcap;
    StreamPatch* dp = nullptr;
    int32_t *dn = nullptr, *dh = nullptr, *de = nullptr;
    uint2* dc = nullptr;
    uint16_t *dcp = nullptr, *dcs = nullptr;
    StreamElem* dse = nullptr;
    StreamNode* dsn = nullptr;
    int* derr = nullptr;
    if ((rc = dalloc(c, &dp, Pcap)) || (rc = dalloc(c, &dn, N)) || (rc = dalloc(c, &dh, Hcap)) ||
        (rc = dalloc(c, &de, Tcap)) || (rc = dalloc(c, &dc, Tcap)) || (rc = dalloc(c, &dcp, CPcap)) ||
        (rc = dalloc(c, &dcs, 3 * E)) || (rc = dalloc(c, &dse, Tcap)) || (rc = dalloc(c, &dsn, N)) ||
        (rc = dalloc(c, &derr, 1)) || (rc = dalloc(c, &c->d_plist, Pcap)) || (rc = dalloc(c, &c->d_budget, S)) ||
        (rc = dalloc(c, &c->d_budget2, S)) || (rc = dalloc(c, &c->d_dt2, S)) ||
        (rc = dalloc(c, &c->d_slist, S)) || (rc = dalloc(c, &c->d_srng, S)) ||
        (rc = dalloc(c, &d.x_alt, N)) ||
        (rc = dalloc(c, &d.j2_alt, E)))
      return rc;
    FW_CUDA(c, cudaMemsetAsync(derr, 0, sizeof(int), c->stream));
    c->sd = StreamDev{dp, dn, dh, de, dc, dcp, dcs, 1, 1, 1, dse, dsn, derr, c->d_plist};
    c->fl_patch.init(Pcap);
    c->fl_halo.init(Hcap);
    c->fl_ptri.init(Tcap);
    c->fl_csrp.init(CPcap);
    stream_smem(1, 1, 1, &c->st_smem, &c->st_smem_bulk);
    if ((rc = stream_attrs(c, shared_optin(c)))) return rc;
    c->st_list_n = 0;
    c->x_buf0 = d.x;
    c->a_stream = true;
    c->path = FW_PATH_STREAM;
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  c->h_x.clear(); c->h_conn.clear(); c->h_pairs.clear(); c->h_heights.clear(); c->h_occ.clear();
  return FW_OK;
}

int fw_arena_pack(fw_ctx* stage, int32_t patch_nodes, int32_t flags, fw_pack** out) {
  if (!stage || !out) return FW_ERR_ARG;
  *out = nullptr;
  if (stage->finalized && !stage->arena)
    return fail(stage, FW_ERR_STATE, "fw_arena_pack: stage on a context that is not finalized, or on an arena");
  return build_pack(stage, patch_nodes, (flags & FW_PACK_PINNED) != 0, out);
}

int fw_pack_info(const fw_pack* pk, int64_t* info) {
  if (!pk || !info) return FW_ERR_ARG;
  info[0] = pk->dev_bytes; info[1] = pk->Ns; info[2] = pk->Es; info[3] = pk->Bs;
  info[4] = pk->patch_nodes; info[5] = pk->Ps; info[6] = pk->Ts; info[7] = pk->pinned ? 1 : 0;
  return FW_OK;
}

void fw_pack_destroy(fw_pack* pk) { delete pk; }

int fw_arena_commit_pack(fw_ctx* c, const fw_pack* pk, int32_t* scene_out) {
  if (!c || !pk || !scene_out) return FW_ERR_ARG;
  if (!c->arena) return fail(c, FW_ERR_STATE, "fw_arena_commit_pack without fw_arena_init");
  if (c->a_stream && pk->patch_nodes != c->st_nodes)
    return fail(c, FW_ERR_ARG, "fw_arena_commit_pack: the pack is cut into %d-node patches, the arena steps %d-node "
                               "patches", pk->patch_nodes, c->st_nodes);
  if (c->free_scene_ids.empty()) return fail(c, FW_ERR_OOM, "arena: no free scene slot");
  fw_ctx::ArenaScene a;
  a.nn = pk->Ns; a.ne = pk->Es; a.nb = pk->Bs; a.np = pk->Np; a.nh = pk->Nh; a.no = pk->No;
  if (c->a_stream) { a.npp = pk->Ps; a.nhh = pk->Hs; a.nt = pk->Ts; a.ncp = pk->CPs; }
  fw_ctx::FreeList* lists[10] = {&c->fl_nodes, &c->fl_elems, &c->fl_bodies, &c->fl_pairs, &c->fl_heights,
                                 &c->fl_occ, &c->fl_patch, &c->fl_halo, &c->fl_ptri, &c->fl_csrp};
  int64_t* offs[10] = {&a.n0, &a.e0, &a.b0, &a.p0, &a.h0, &a.o0, &a.pp0, &a.hh0, &a.t0, &a.cp0};
  const int64_t lens[10] = {a.nn, a.ne, a.nb, a.np, a.nh, a.no, a.npp, a.nhh, a.nt, a.ncp};
  const int nl = c->a_stream ? 10 : 6;
  for (int k = 0; k < nl; ++k)
    if (!lists[k]->take(lens[k], offs[k])) {
      for (int j = 0; j < k; ++j) lists[j]->give(*offs[j], lens[j]);
      return fail(c, FW_ERR_OOM, "arena: not enough free capacity for this scene");
    }
  // stream arenas: the launch's shared memory covers the largest patch so far
  int no_max = c->sd.no_max, nh_max = c->sd.nh_max, ne_max = c->sd.ne_max;
  size_t smem = c->st_smem, smem_bulk = c->st_smem_bulk;
  if (c->a_stream) {
    no_max = std::max(no_max, pk->no_max);
    nh_max = std::max(nh_max, pk->nh_max);
    ne_max = std::max(ne_max, pk->ne_max);
    stream_smem(no_max, nh_max, ne_max, &smem, &smem_bulk);
    if ((long)smem > shared_optin(c) - 64) {
      for (int j = 0; j < nl; ++j) lists[j]->give(*offs[j], lens[j]);
      return fail(c, FW_ERR_ARG, "arena: a patch of this scene needs %zu B of shared memory", smem);
    }
  }
  const int s = c->free_scene_ids.back();
  c->free_scene_ids.pop_back();
  a.live = true;
  // upload (queued on the stream: the steps that follow see the scene, and a
  // pinned pack's copy runs asynchronously): the whole pack in one copy to
  // the device staging buffer, then one kernel puts each part in its range
  Dev& d = c->d;
  const int64_t n0 = a.n0, e0 = a.e0;
  static_assert(kScatterParts == fw_pack::NPARTS + 1, "one scatter slot per pack part, plus the current positions");
  unsigned char* dst[fw_pack::NPARTS] = {};
  auto B = [](const void* p) { return (unsigned char*)const_cast<void*>(p); };
  dst[fw_pack::X0] = B(d.x0 + n0); dst[fw_pack::V0] = B(d.v + n0); dst[fw_pack::BCV] = B(d.bcv + n0);
  dst[fw_pack::WORD] = B(d.node_word + n0); dst[fw_pack::CBEG] = B(d.csr_off + n0); dst[fw_pack::CEND] = B(d.csr_end + n0);
  dst[fw_pack::SLOT] = B(d.csr_slot + 3 * e0); dst[fw_pack::CPOS] = B(d.corner_pos + 3 * e0);
  dst[fw_pack::CONN] = B(d.conn + 3 * e0); dst[fw_pack::EMAT] = B(d.emat + e0); dst[fw_pack::J2PAR] = B(d.j2par + e0);
  dst[fw_pack::YOUNG] = B(c->a_young + e0); dst[fw_pack::POISSON] = B(c->a_poisson + e0);
  dst[fw_pack::RHO] = B(c->a_rho + e0); dst[fw_pack::POFF] = B(d.body_pair_off + a.b0);
  dst[fw_pack::PCNT] = B(d.body_pair_cnt + a.b0); dst[fw_pack::PAIRS] = B(d.pairs + a.p0);
  dst[fw_pack::HEIGHTS] = B(d.heights + a.h0); dst[fw_pack::OCC] = B(d.occ + a.o0);
  if (c->a_stream) {
    dst[fw_pack::RN] = B(c->sd.nodes + n0); dst[fw_pack::RH] = B(c->sd.halo + a.hh0); dst[fw_pack::RE] = B(c->sd.eid + a.t0);
    dst[fw_pack::RC] = B(c->sd.conn + a.t0); dst[fw_pack::RCP] = B(c->sd.csrp + a.cp0);
    dst[fw_pack::RCS] = B(c->sd.csrs + 3 * e0); dst[fw_pack::PATCH] = B(c->sd.patch + a.pp0);
  }
  if (pk->bytes <= c->stage_cap) {
    FW_CUDA(c, cudaMemcpyAsync(c->d_stage, pk->block, pk->bytes, cudaMemcpyHostToDevice, c->stream));
    ArenaScatter sc{};
    uint32_t most = 0;
    for (int k = 0; k < fw_pack::NPARTS; ++k) {
      sc.dst[k] = dst[k];
      sc.off[k] = (uint32_t)pk->off[k];
      sc.len[k] = dst[k] ? (uint32_t)pk->len[k] : 0u;
      most = std::max(most, sc.len[k]);
    }
    sc.dst[fw_pack::NPARTS] = B(d.x + n0);  // the current positions start at the rest positions
    sc.off[fw_pack::NPARTS] = (uint32_t)pk->off[fw_pack::X0];
    sc.len[fw_pack::NPARTS] = (uint32_t)pk->len[fw_pack::X0];
    const int gx = (int)std::max<uint32_t>(1u, std::min<uint32_t>((most / 4 + kBlock - 1) / kBlock, 256u));
    k_arena_scatter<<<dim3(gx, kScatterParts), kBlock, 0, c->stream>>>(c->d_stage, sc);
    c->launches += 1;
  } else {  // larger than the staging buffer: one copy per part
    for (int k = 0; k < fw_pack::NPARTS; ++k)
      if (dst[k] && pk->len[k])
        FW_CUDA(c, cudaMemcpyAsync(dst[k], pk->at((fw_pack::Part)k), pk->len[k], cudaMemcpyHostToDevice, c->stream));
    FW_CUDA(c, cudaMemcpyAsync(d.x + n0, pk->at(fw_pack::X0), pk->len[fw_pack::X0], cudaMemcpyHostToDevice, c->stream));
  }
  FW_CUDA(c, cudaMemsetAsync(d.j2state + e0, 0, sizeof(float4) * a.ne, c->stream));
  ArenaReloc r{};
  r.n0 = (int)n0; r.e0 = (int)e0; r.b0 = (int)a.b0; r.p0 = (int)a.p0; r.h0 = (int)a.h0; r.o0 = (int)a.o0; r.s = s;
  r.Ns = (int)a.nn; r.Es = (int)a.ne; r.Bs = (int)a.nb; r.Np = (int)a.np;
  r.damp = pk->damp;
  if (c->a_stream) {
    r.rn = const_cast<int32_t*>(c->sd.nodes) + n0;
    r.rh = const_cast<int32_t*>(c->sd.halo) + a.hh0;
    r.re = const_cast<int32_t*>(c->sd.eid) + a.t0;
    r.Hs = (int)a.nhh;
    r.Ts = (int)a.nt;
    r.patch = const_cast<StreamPatch*>(c->sd.patch) + a.pp0;
    r.Ps = (int)a.npp;
    r.hh0 = (int)a.hh0;
    r.t0 = (int)a.t0;
    r.cp0 = (int)a.cp0;
    r.srng = c->d_srng;
  }
  r.count = std::max<int64_t>({3 * a.ne, a.nn, a.nb, a.np, a.nhh, a.nt, a.npp});
  k_arena_reloc<<<(int)std::min<int64_t>((r.count + kBlock - 1) / kBlock, 8 * c->sms), kBlock, 0, c->stream>>>(d, r);
  const int e_lo = (int)e0, e_hi = (int)(e0 + a.ne), n_lo = (int)n0, n_hi = (int)(n0 + a.nn);
  k_prepare_elements<<<(int)((a.ne + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(d, c->a_young + e0, c->a_poisson + e0,
                                                                                  c->a_rho + e0, e_lo, e_hi);
  k_prepare_mass<<<(int)((a.nn + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(d, n_lo, n_hi);
  c->launches += 3;
  if (c->a_stream) {
    if (a.nt > 0)
      k_stream_elems<<<(int)((a.nt + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(
          d, c->sd.eid + a.t0, c->sd.conn + a.t0, c->sd.elem + a.t0, nullptr, (int)a.nt);
    k_stream_nodes<<<(int)((a.nn + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(d, c->sd.nodes + n0,
                                                                                  c->sd.node + n0, (int)a.nn);
    c->launches += 2;
    c->sd.no_max = no_max; c->sd.nh_max = nh_max; c->sd.ne_max = ne_max;
    c->st_smem = smem;
    c->st_smem_bulk = smem_bulk;
    if ((long)smem_bulk > shared_optin(c) - 64) c->st_bulk = 0;  // staging no longer fits: plain loads
  }
  int rc;
  if ((rc = check_kernel(c, "arena commit"))) return rc;
  c->ascenes[s] = a;
  for (int64_t b = 0; b < a.nb; ++b) c->a_body_scene[a.b0 + b] = s;
  c->cur_active[s] = 1;
  c->chunks_dirty = true;
  *scene_out = s;
  return FW_OK;
}

int fw_arena_commit(fw_ctx* c, int32_t* scene_out) {
  if (!c || !scene_out) return FW_ERR_ARG;
  if (!c->arena) return fail(c, FW_ERR_STATE, "fw_arena_commit without fw_arena_init");
  fw_pack* pk = nullptr;
  int rc = build_pack(c, c->a_stream ? c->st_nodes : 0, false, &pk);
  if (rc) return rc;
  rc = fw_arena_commit_pack(c, pk, scene_out);
  delete pk;  // pageable: its copies were staged before they returned
  return rc;
}

int fw_arena_remove(fw_ctx* c, int32_t s) {
  if (!c) return FW_ERR_ARG;
  if (!c->arena) return fail(c, FW_ERR_STATE, "fw_arena_remove without fw_arena_init");
  if (s < 0 || s >= c->S - 1 || !c->ascenes[s].live) return fail(c, FW_ERR_ARG, "fw_arena_remove: scene %d is not live", s);
  fw_ctx::ArenaScene& a = c->ascenes[s];
  std::vector<int32_t> dead(a.nb, c->S - 1);
  const int32_t zero = 0;
  FW_CUDA(c, cudaMemcpyAsync(c->d.body_scene + a.b0, dead.data(), sizeof(int32_t) * a.nb, cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_active + s, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_bad + s, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int64_t b = 0; b < a.nb; ++b) c->a_body_scene[a.b0 + b] = c->S - 1;
  c->fl_nodes.give(a.n0, a.nn);
  c->fl_elems.give(a.e0, a.ne);
  c->fl_bodies.give(a.b0, a.nb);
  c->fl_pairs.give(a.p0, a.np);
  c->fl_heights.give(a.h0, a.nh);
  c->fl_occ.give(a.o0, a.no);
  if (c->a_stream) {
    c->fl_patch.give(a.pp0, a.npp);
    c->fl_halo.give(a.hh0, a.nhh);
    c->fl_ptri.give(a.t0, a.nt);
    c->fl_csrp.give(a.cp0, a.ncp);
  }
  a = fw_ctx::ArenaScene{};
  c->cur_active[s] = 0;
  c->free_scene_ids.push_back(s);
  c->chunks_dirty = true;
  return FW_OK;
}

int fw_step_served(fw_ctx* c, const float* dt) { return fw_step_served_n(c, dt, 1); }

int fw_step_served_n(fw_ctx* c, const float* dt, int32_t n_steps) {
  if (!c || !dt || n_steps < 0) return FW_ERR_ARG;
  if (n_steps == 0) return FW_OK;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_step_served before fw_finalize / fw_arena_init");
  bool changed = false;
  for (int s = 0; s < c->S; ++s) {
    const int want = (dt[s] > 0.0f && (!c->arena || c->ascenes[s].live)) ? 1 : 0;
    if (want != c->cur_active[s]) {
      c->cur_active[s] = want;
      changed = true;
    }
  }
  if (changed) {
    FW_CUDA(c, cudaMemcpyAsync(c->d.scene_active, c->cur_active.data(), sizeof(int32_t) * c->S,
                               cudaMemcpyHostToDevice, c->stream));
    c->chunks_dirty = true;
  }
  c->cur_dt.assign(dt, dt + c->S);
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_dt, c->cur_dt.data(), sizeof(float) * c->S, cudaMemcpyHostToDevice,
                             c->stream));
  c->d.uniform_dt = 0;
  if (c->arena && c->a_stream) return arena_stream_steps(c, n_steps);
  int rc;
  if (c->arena && (rc = rebuild_chunks(c))) return rc;
  for (int k = 0; k < n_steps; ++k)
    if ((rc = launch_step(c))) return rc;
  return FW_OK;
}

int fw_step_served_budget(fw_ctx* c, const float* dt, const int32_t* budget, const float* dt_next,
                          const int32_t* budget_next, int32_t n_steps) {
  if (!c || !dt || !budget || n_steps < 0 || (!dt_next) != (!budget_next)) return FW_ERR_ARG;
  if (!c->arena || !c->a_stream)
    return fail(c, FW_ERR_STATE, "fw_step_served_budget needs a stream arena (fw_set_path FW_PATH_STREAM before "
                                 "fw_arena_init)");
  if (n_steps == 0) return FW_OK;
  // staged before the calls return
  c->h_budget.assign(budget, budget + c->S);
  FW_CUDA(c, cudaMemcpyAsync(c->d_budget, c->h_budget.data(), sizeof(int32_t) * c->S, cudaMemcpyHostToDevice,
                             c->stream));
  c->d.scene_budget = c->d_budget;
  if (budget_next) {
    c->h_budget2.assign(budget_next, budget_next + c->S);
    c->h_dt2.assign(dt_next, dt_next + c->S);
    FW_CUDA(c, cudaMemcpyAsync(c->d_budget2, c->h_budget2.data(), sizeof(int32_t) * c->S, cudaMemcpyHostToDevice,
                               c->stream));
    FW_CUDA(c, cudaMemcpyAsync(c->d_dt2, c->h_dt2.data(), sizeof(float) * c->S, cudaMemcpyHostToDevice, c->stream));
    c->d.scene_budget_next = c->d_budget2;
    c->d.scene_dt_next = c->d_dt2;
  }
  const int rc = fw_step_served_n(c, dt, n_steps);
  c->d.scene_budget = nullptr;
  c->d.scene_budget_next = nullptr;
  c->d.scene_dt_next = nullptr;
  return rc;
}

int fw_arena_scene_info(fw_ctx* c, int32_t s, int64_t* info) {
  if (!c || !info) return FW_ERR_ARG;
  if (!c->arena) return fail(c, FW_ERR_STATE, "fw_arena_scene_info without fw_arena_init");
  if (s < 0 || s >= c->S - 1 || !c->ascenes[s].live) return fail(c, FW_ERR_ARG, "scene %d is not live", s);
  const fw_ctx::ArenaScene& a = c->ascenes[s];
  info[0] = a.n0; info[1] = a.nn; info[2] = a.e0; info[3] = a.ne; info[4] = a.b0; info[5] = a.nb;
  info[6] = c->fl_nodes.total(); info[7] = c->fl_elems.total();
  return FW_OK;
}


int fw_set_element_young(fw_ctx* c, int32_t first, int32_t count, const float* young, int32_t on_device) {
  if (!c || !young) return FW_ERR_ARG;
  // (the resident step loads the Lame constants at every launch; the stream path's
  // patch records are rebuilt below)
  if (!c->finalized || c->arena)
    return fail(c, FW_ERR_STATE, "fw_set_element_young needs a finalized world (not an arena)");
  if (first < 0 || count < 0 || (int64_t)first + count > c->E) return fail(c, FW_ERR_ARG, "element range out of bounds");
  if (c->has_springs) return fail(c, FW_ERR_STATE, "fw_set_element_young: the world has spring-mass domains");
  if (count == 0) return FW_OK;
  int rc;
  if (!c->d_poisson && (rc = upload(c, &c->d_poisson, c->h_nu))) return rc;
  if (!c->adj.young && (rc = upload(c, &c->adj.young, c->h_E))) return rc;
  float* dst = c->adj.young + first;
  FW_CUDA(c, cudaMemcpyAsync(dst, young, sizeof(float) * count,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  k_set_young<<<(count + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->d, dst, c->d_poisson, first, first + count);
  c->launches += 1;
  if ((rc = check_kernel(c, "set young"))) return rc;
  if (c->path != FW_PATH_STREAM) return FW_OK;
  // a body's triangles may now differ: the stream records take their Lame
  // constants per triangle from here on
  if (!c->sd.lm) {
    if ((rc = dalloc(c, &c->sd.lm, (size_t)std::max(1, c->st_ne)))) return rc;
    drop_graphs(c);
  }
  return stream_records(c);
}

int fw_adj_begin(fw_ctx* c, int32_t max_segment_steps) {
  if (c && (c->has_flex || c->has_springs || c->has_rigid))
    return fail(c, FW_ERR_STATE, "the adjoint covers FEM triangles without FEM-FEM contact");
  if (!c) return FW_ERR_ARG;
  // The forward may run on either path (identical bits); the recompute and the
  // reverse use the gather kernels and data, which every non-arena world has.
  if (!c->finalized || c->arena || c->S != 1 || c->path == FW_PATH_STREAM)
    return fail(c, FW_ERR_STATE, "the adjoint needs a finalized single-scene world on the gather or resident path");
  if (max_segment_steps <= 0) return fail(c, FW_ERR_ARG, "max_segment_steps must be > 0");
  int rc;
  Adj& a = c->adj;
  if (!a.young) {
    if ((rc = upload(c, &a.young, c->h_E))) return rc;
  }
  if (!a.xb) {
    if ((rc = dalloc(c, &a.xb, c->N)) || (rc = dalloc(c, &a.vb, c->N)) || (rc = dalloc(c, &a.fb, c->N)) ||
        (rc = dalloc(c, &a.Eb, c->E)) || (rc = dalloc(c, &a.io_x, c->N)) || (rc = dalloc(c, &a.io_v, c->N)) ||
        (rc = dalloc(c, &a.io_E, c->E)))
      return rc;
  }
  if (c->adj_cap < max_segment_steps) {
    drop_graphs(c);  // graphs hold the old trajectory buffers
    if ((rc = dalloc(c, &a.traj, (size_t)max_segment_steps * c->N)) ||
        (rc = dalloc(c, &a.trajv, (size_t)max_segment_steps * c->N)) ||
        (rc = dalloc(c, &a.trajs, (size_t)max_segment_steps * (c->d.has_j2 ? c->E : 1))) ||
        (rc = dalloc(c, &a.gates, (size_t)max_segment_steps * std::max(1, c->d.P))))
      return rc;
    c->adj_cap = max_segment_steps;
  }
  if (c->d.has_j2 && !a.sb) {
    if ((rc = dalloc(c, &a.sb, 4 * (size_t)c->E))) return rc;
  }
  if (a.sb) FW_CUDA(c, cudaMemsetAsync(a.sb, 0, sizeof(double) * 4 * (size_t)c->E, c->stream));
  // Resident reverse pass when the world runs resident and the adjoint state
  // fits on chip too (J2 worlds reverse on the gather kernels).
  if (c->path == FW_PATH_RESIDENT && !c->res_adj && !c->d.has_j2) {
    int optin = 0, sms = 148;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const size_t need = res_layout(c->res, nullptr, nullptr) + res_adj_layout(c->res, nullptr, nullptr);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_res_adj);
    int per_sm = 0;
    if ((long)need + (long)fa.sharedSizeBytes + 64 <= optin &&
        cudaFuncSetAttribute(k_res_adj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_res_adj, kResThreads, need) == cudaSuccess &&
        per_sm * sms >= c->res.P) {
      if ((rc = dalloc(c, &c->fll, 8 * (size_t)c->N))) return rc;
      FW_CUDA(c, cudaMemsetAsync(c->fll, 0, sizeof(unsigned long long) * 8 * (size_t)c->N, c->stream));
      c->res_adj = true;
      c->res_adj_smem = need;
    }
    cudaGetLastError();
  }
  FW_CUDA(c, cudaMemsetAsync(a.Eb, 0, sizeof(double) * c->E, c->stream));
  FW_CUDA(c, cudaMemsetAsync(a.xb, 0, sizeof(double2) * c->N, c->stream));
  FW_CUDA(c, cudaMemsetAsync(a.vb, 0, sizeof(double2) * c->N, c->stream));
  return FW_OK;
}

int fw_adj_seed(fw_ctx* c, const float* xbar, const float* vbar, int32_t on_device) {
  if (!c) return FW_ERR_ARG;
  if (!c->adj.xb) return fail(c, FW_ERR_STATE, "fw_adj_seed before fw_adj_begin");
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (xbar) FW_CUDA(c, cudaMemcpyAsync(c->adj.io_x, xbar, sizeof(float2) * c->N, k, c->stream));
  if (vbar) FW_CUDA(c, cudaMemcpyAsync(c->adj.io_v, vbar, sizeof(float2) * c->N, k, c->stream));
  k_adj_seed<<<(c->N + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->adj, c->N, xbar != nullptr, vbar != nullptr);
  c->launches += 1;
  FW_CUDA(c, cudaMemsetAsync(c->adj.Eb, 0, sizeof(double) * c->E, c->stream));
  if (c->adj.sb) FW_CUDA(c, cudaMemsetAsync(c->adj.sb, 0, sizeof(double) * 4 * (size_t)c->E, c->stream));
  return check_kernel(c, "adjoint seed");
}

int fw_adj_segment(fw_ctx* c, int32_t n_steps, float dt) {
  if (!c) return FW_ERR_ARG;
  if (!c->adj.xb) return fail(c, FW_ERR_STATE, "fw_adj_segment before fw_adj_begin");
  if (n_steps <= 0 || n_steps > c->adj_cap) return fail(c, FW_ERR_ARG, "n_steps outside (0, max_segment_steps]");
  Adj& a = c->adj;
  const int N = c->N, E = c->E, P = std::max(1, c->d.P);
  c->d.uniform_dt = 1;
  c->d.dt_uniform = dt;
  int rc;
  if (c->res_adj) {
    // recompute on the resident step, recording positions and gates, then the resident reverse
    c->res.rec_x = a.traj;
    c->res.rec_v = a.trajv;
    c->res.rec_gates = a.gates;
    c->res.rec_stride = P;
    rc = launch_resident(c, n_steps);
    c->res.rec_x = nullptr;
    c->res.rec_v = nullptr;
    c->res.rec_gates = nullptr;
    if (rc) return rc;
    if (c->res_epoch > 0xF0000000u) {
      FW_CUDA(c, cudaMemsetAsync(c->fll, 0, sizeof(unsigned long long) * 8 * (size_t)N, c->stream));
      FW_CUDA(c, cudaMemsetAsync(c->res.xll, 0, sizeof(unsigned long long) * 4 * (size_t)N, c->stream));
      FW_CUDA(c, cudaMemsetAsync(c->res.bll, 0, sizeof(unsigned long long) * 4 * (size_t)kBoxRing * c->B * c->res.P,
                                 c->stream));
      c->res_epoch = 1;
    }
    uint32_t ep0 = c->res_epoch;
    c->res_epoch += (uint32_t)n_steps + 1u;
    float damp_f = c->h_damp.empty() ? 0.0f : c->h_damp[0];
    int nn = n_steps, gs = P;
    const float2* tx = a.traj;
    const float2* tv = a.trajv;
    const int* tg = a.gates;
    void* args[] = {(void*)&c->d, (void*)&c->res, (void*)&c->adj, (void*)&tx, (void*)&tv, (void*)&tg, (void*)&gs,
                    (void*)&c->fll, (void*)&nn, (void*)&dt, (void*)&damp_f, (void*)&ep0};
    FW_CUDA(c, cudaLaunchCooperativeKernel((const void*)k_res_adj, dim3(c->res.P), dim3(kResThreads), args,
                                           c->res_adj_smem, c->stream));
    c->launches += 1;
    return check_kernel(c, "resident adjoint segment");
  }
  const uint64_t key_lo = ((uint64_t)n_steps << 32) | float_bits(dt);
  // recompute the segment from the current state, recording positions and gates
  cudaGraphExec_t g_fwd = nullptr;
  rc = cached_graph(c, c->adj_graphs, (1ull << 62) | key_lo, [&] {
    for (int j = 0; j < n_steps; ++j) {
      cudaMemcpyAsync(a.traj + (size_t)j * N, c->d.x, sizeof(float2) * N, cudaMemcpyDeviceToDevice, c->stream);
      cudaMemcpyAsync(a.trajv + (size_t)j * N, c->d.v, sizeof(float2) * N, cudaMemcpyDeviceToDevice, c->stream);
      if (c->d.has_j2)
        cudaMemcpyAsync(a.trajs + (size_t)j * E, c->d.j2state, sizeof(float4) * E, cudaMemcpyDeviceToDevice,
                        c->stream);
      k_elements<<<c->grid_e, c->block_e, 0, c->stream>>>(c->d);
      k_nodes<<<c->grid_n, c->block_n, 0, c->stream>>>(c->d);
      if (c->d.P > 0)
        cudaMemcpyAsync(a.gates + (size_t)j * P, c->d.pair_active, sizeof(int32_t) * c->d.P,
                        cudaMemcpyDeviceToDevice, c->stream);
    }
  }, &g_fwd);
  if (rc) return rc;
  FW_CUDA(c, cudaGraphLaunch(g_fwd, c->stream));
  c->host_counter += n_steps;
  c->launches += 2 * n_steps;
  // (xb, vb) hold the adjoint of the segment's end state; the segment leaves
  // the adjoint of its start state there (the checkpoint it was restored from).
  const int gn = (N + kBlock - 1) / kBlock, ge = (E + kBlock - 1) / kBlock;
  const float damp = c->h_damp.empty() ? 0.0f : c->h_damp[0];
  cudaGraphExec_t g_rev = nullptr;
  rc = cached_graph(c, c->adj_graphs, (2ull << 62) | key_lo, [&] {
    k_adj_prep<<<gn, kBlock, 0, c->stream>>>(c->d, a, dt, damp);  // force / velocity adjoints of the last substep
    for (int j = n_steps - 1; j >= 0; --j) {
      const float2* x = a.traj + (size_t)j * N;
      const float2* v = a.trajv + (size_t)j * N;
      k_adj_elements<<<ge, kBlock, 0, c->stream>>>(c->d, a, x, a.trajs + (c->d.has_j2 ? (size_t)j * E : 0));
      k_adj_nodes<<<gn, kBlock, 0, c->stream>>>(c->d, a, x, v, a.gates + (size_t)j * P, dt, damp, j > 0);
    }
  }, &g_rev);
  if (rc) return rc;
  FW_CUDA(c, cudaGraphLaunch(g_rev, c->stream));
  c->launches += 1 + 2 * n_steps;
  return check_kernel(c, "adjoint segment");
}

int fw_adj_read(fw_ctx* c, float* xbar, float* vbar, float* Ebar, int32_t on_device) {
  if (!c) return FW_ERR_ARG;
  if (!c->adj.xb) return fail(c, FW_ERR_STATE, "fw_adj_read before fw_adj_begin");
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const int n = std::max(c->N, c->E);
  k_adj_out<<<(n + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->adj, c->N, c->E);
  c->launches += 1;
  if (xbar) FW_CUDA(c, cudaMemcpyAsync(xbar, c->adj.io_x, sizeof(float2) * c->N, k, c->stream));
  if (vbar) FW_CUDA(c, cudaMemcpyAsync(vbar, c->adj.io_v, sizeof(float2) * c->N, k, c->stream));
  if (Ebar) FW_CUDA(c, cudaMemcpyAsync(Ebar, c->adj.io_E, sizeof(float) * c->E, k, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_tan_begin(fw_ctx* c, const float* dx0, const float* dv0, const float* dE, int32_t on_device) {
  if (c && (c->has_flex || c->has_springs || c->has_rigid))
    return fail(c, FW_ERR_STATE, "the tangent covers FEM triangles without FEM-FEM contact");
  if (!c) return FW_ERR_ARG;
  if (!c->finalized || c->arena || c->S != 1 || c->path == FW_PATH_STREAM)
    return fail(c, FW_ERR_STATE, "the tangent needs a finalized single-scene world on the gather or resident path");
  if (c->d.has_j2) return fail(c, FW_ERR_ARG, "the tangent covers Elastic and NeoHookean triangles (no J2)");
  Tan& t = c->tan;
  int rc;
  if (!c->adj.young && (rc = upload(c, &c->adj.young, c->h_E))) return rc;
  t.young = c->adj.young;
  if (!t.dx) {
    if ((rc = dalloc(c, &t.dx, c->N)) || (rc = dalloc(c, &t.dv, c->N)) || (rc = dalloc(c, &t.dE, c->E)) ||
        (rc = dalloc(c, &t.xs, c->N)) || (rc = dalloc(c, &t.vs, c->N)) || (rc = dalloc(c, &t.io_x, c->N)) ||
        (rc = dalloc(c, &t.io_v, c->N)))
      return rc;
  }
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (dx0) FW_CUDA(c, cudaMemcpyAsync(t.io_x, dx0, sizeof(float2) * c->N, k, c->stream));
  if (dv0) FW_CUDA(c, cudaMemcpyAsync(t.io_v, dv0, sizeof(float2) * c->N, k, c->stream));
  if (dE) FW_CUDA(c, cudaMemcpyAsync(t.dE, dE, sizeof(float) * c->E, k, c->stream));
  else FW_CUDA(c, cudaMemsetAsync(t.dE, 0, sizeof(float) * c->E, c->stream));
  k_tan_seed<<<(c->N + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(t, c->N, dx0 != nullptr, dv0 != nullptr);
  c->launches += 1;
  return check_kernel(c, "tangent seed");
}

int fw_tan_step(fw_ctx* c, int32_t n_steps, float dt) {
  if (!c) return FW_ERR_ARG;
  if (!c->tan.dx) return fail(c, FW_ERR_STATE, "fw_tan_step before fw_tan_begin");
  if (n_steps < 0) return fail(c, FW_ERR_ARG, "n_steps must be >= 0");
  Tan& t = c->tan;
  c->d.uniform_dt = 1;
  c->d.dt_uniform = dt;
  const float damp = c->h_damp.empty() ? 0.0f : c->h_damp[0];
  const int gn = (c->N + kBlock - 1) / kBlock, ge = (c->E + kBlock - 1) / kBlock;
  int rc;
  for (int j = 0; j < n_steps; ++j) {
    FW_CUDA(c, cudaMemcpyAsync(t.xs, c->d.x, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    FW_CUDA(c, cudaMemcpyAsync(t.vs, c->d.v, sizeof(float2) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = launch_step(c))) return rc;  // the substep itself (sets this substep's gates)
    c->host_counter += 1;
    k_tan_elements<<<ge, kBlock, 0, c->stream>>>(c->d, t);
    k_tan_nodes<<<gn, kBlock, 0, c->stream>>>(c->d, t, dt, damp);
    c->launches += 2;
  }
  return check_kernel(c, "tangent step");
}

int fw_tan_read(fw_ctx* c, float* dx, float* dv, int32_t on_device) {
  if (!c) return FW_ERR_ARG;
  if (!c->tan.dx) return fail(c, FW_ERR_STATE, "fw_tan_read before fw_tan_begin");
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  k_tan_out<<<(c->N + kBlock - 1) / kBlock, kBlock, 0, c->stream>>>(c->tan, c->N);
  c->launches += 1;
  if (dx) FW_CUDA(c, cudaMemcpyAsync(dx, c->tan.io_x, sizeof(float2) * c->N, k, c->stream));
  if (dv) FW_CUDA(c, cudaMemcpyAsync(dv, c->tan.io_v, sizeof(float2) * c->N, k, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_get_path(const fw_ctx* c, int32_t* path, int32_t* patches) {
  if (!c || !path) return FW_ERR_ARG;
  *path = c->finalized ? c->path : FW_PATH_AUTO;
  if (patches) *patches = c->path == FW_PATH_RESIDENT ? c->res.P : (c->path == FW_PATH_STREAM ? c->st_P : 0);
  return FW_OK;
}

int fw_step(fw_ctx* c, int32_t n_steps, float dt) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_step before fw_finalize");
  if (n_steps < 0) return fail(c, FW_ERR_ARG, "fw_step: n_steps < 0");
  c->d.uniform_dt = 1;
  c->d.dt_uniform = dt;
  return run_steps(c, n_steps);
}

int fw_step_scenes(fw_ctx* c, int32_t n_steps, const float* dt) {
  if (!c || !dt) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_step_scenes before fw_finalize");
  if (n_steps < 0) return fail(c, FW_ERR_ARG, "fw_step_scenes: n_steps < 0");
  int rc = set_scene_dt(c, dt);
  if (rc) return rc;
  c->d.uniform_dt = 0;
  return run_steps(c, n_steps);
}

int fw_set_active(fw_ctx* c, const int32_t* active) {
  if (!c || !active) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_set_active before fw_finalize");
  c->cur_active.assign(active, active + c->S);
  if (c->arena)  // a scene that is not live stays inactive
    for (int s = 0; s < c->S; ++s)
      if (!c->ascenes[s].live) c->cur_active[s] = 0;
  FW_CUDA(c, cudaMemcpyAsync(c->d.scene_active, c->cur_active.data(), sizeof(int32_t) * c->S,
                             cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  c->chunks_dirty = true;
  return FW_OK;
}

int fw_synchronize(fw_ctx* c) {
  if (!c) return FW_ERR_ARG;
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return c->finalized ? check_device_error(c) : FW_OK;
}

int fw_read_nodes(fw_ctx* c, int32_t field, int32_t first, int32_t count, float* dst, int32_t on_device) {
  if (!c || !dst) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_read_nodes before fw_finalize");
  if (first < 0 || count < 0 || (int64_t)first + count > c->N)
    return fail(c, FW_ERR_ARG, "fw_read_nodes: range [%d, %d) outside [0, %d)", first, first + count, c->N);
  const void* src = nullptr;
  size_t per = 2 * sizeof(float);
  switch (field) {
    case FW_FIELD_X: src = c->d.x + first; break;
    case FW_FIELD_V: src = c->d.v + first; break;
    case FW_FIELD_X0: src = c->d.x0 + first; break;
    case FW_FIELD_MASS: src = c->d.mass + first; per = sizeof(float); break;
    default: return fail(c, FW_ERR_ARG, "fw_read_nodes: unknown field %d", field);
  }
  FW_CUDA(c, cudaMemcpyAsync(dst, src, per * count,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

int fw_write_nodes(fw_ctx* c, int32_t field, int32_t first, int32_t count, const float* src, int32_t on_device) {
  if (!c || !src) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_write_nodes before fw_finalize");
  if (first < 0 || count < 0 || (int64_t)first + count > c->N)
    return fail(c, FW_ERR_ARG, "fw_write_nodes: range [%d, %d) outside [0, %d)", first, first + count, c->N);
  void* dst = nullptr;
  switch (field) {
    case FW_FIELD_X: dst = c->d.x + first; break;
    case FW_FIELD_V: dst = c->d.v + first; break;
    default: return fail(c, FW_ERR_ARG, "fw_write_nodes: field %d is not writable", field);
  }
  FW_CUDA(c, cudaMemcpyAsync(dst, src, 2 * sizeof(float) * count,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_read_aabb(fw_ctx* c, float* dst) {
  if (!c || !dst) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_read_aabb before fw_finalize");
  std::vector<int32_t> ring(8 * (size_t)c->B), cnt(c->S);
  FW_CUDA(c, cudaMemcpyAsync(ring.data(), c->d.aabb_ring, sizeof(int32_t) * ring.size(), cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(cnt.data(), c->d.scene_counter, sizeof(int32_t) * c->S, cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int b = 0; b < c->B; ++b) {
    const int sc = c->arena ? c->a_body_scene[b] : c->h_scene[b];
    const int slot = cnt[sc] & 1;
    for (int k = 0; k < 4; ++k) {
      int v = ring[((size_t)slot * c->B + b) * 4 + k];
      v = v >= 0 ? v : v ^ 0x7FFFFFFF;
      memcpy(&dst[4 * b + k], &v, sizeof(float));
    }
  }
  return FW_OK;
}

int fw_read_plastic(fw_ctx* c, float* eps_p, float* eqps) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_read_plastic before fw_finalize");
  std::vector<float4> st(c->d.has_j2 ? c->E : 0);
  if (c->d.has_j2) {
    FW_CUDA(c, cudaMemcpyAsync(st.data(), c->d.j2state, sizeof(float4) * c->E, cudaMemcpyDeviceToHost, c->stream));
    FW_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  for (int e = 0; e < c->E; ++e) {
    const float4 s = c->d.has_j2 ? st[e] : make_float4(0.f, 0.f, 0.f, 0.f);
    if (eps_p) {
      eps_p[3 * e] = s.x;
      eps_p[3 * e + 1] = s.y;
      eps_p[3 * e + 2] = s.z;
    }
    if (eqps) eqps[e] = s.w;
  }
  return FW_OK;
}

int fw_read_reference_shape(fw_ctx* c, float* area, float* jinv) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_read_reference_shape before fw_finalize");
  std::vector<ElemMat> m(c->E);
  FW_CUDA(c, cudaMemcpyAsync(m.data(), c->d.emat, sizeof(ElemMat) * c->E, cudaMemcpyDeviceToHost, c->stream));
  if (jinv) FW_CUDA(c, cudaMemcpyAsync(jinv, c->d.jinv, sizeof(float4) * c->E, cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  if (area)
    for (int e = 0; e < c->E; ++e) area[e] = m[e].area;
  return FW_OK;
}

int fw_energy(fw_ctx* c, double* out) {
  if (!c || !out) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_energy before fw_finalize");
  // groups: bodies (summed per scene below) or, in an arena, scene slots
  struct Range { int n0, nn, e0, ne; };
  std::vector<Range> groups;
  if (c->arena) {
    for (const fw_ctx::ArenaScene& a : c->ascenes)
      groups.push_back(a.live ? Range{(int)a.n0, (int)a.nn, (int)a.e0, (int)a.ne} : Range{0, 0, 0, 0});
  } else {
    for (int b = 0; b < c->B; ++b) groups.push_back(Range{c->h_noff[b], c->h_ncnt[b], c->h_eoff[b], c->h_ecnt[b]});
  }
  const int G = (int)groups.size();
  std::vector<EnergyChunk> chunks;
  std::vector<int> first(G + 1, 0);
  for (int g = 0; g < G; ++g) {
    first[g] = (int)chunks.size();
    const Range& r = groups[g];
    const int n = std::max(1, (std::max(r.nn, r.ne) + kEnergyChunk - 1) / kEnergyChunk);
    for (int k = 0; k < n; ++k) {
      EnergyChunk ch;
      ch.group = g;
      ch.n0 = r.n0 + std::min(r.nn, k * kEnergyChunk);
      ch.nn = std::max(0, std::min(kEnergyChunk, r.nn - k * kEnergyChunk));
      ch.e0 = r.e0 + std::min(r.ne, k * kEnergyChunk);
      ch.ne = std::max(0, std::min(kEnergyChunk, r.ne - k * kEnergyChunk));
      chunks.push_back(ch);
    }
  }
  first[G] = (int)chunks.size();
  const size_t nc = chunks.size();
  if (nc > c->energy_cap || (size_t)G + 1 > c->energy_gcap) {
    for (void* p : {(void*)c->d_echunk, (void*)c->d_epart, (void*)c->d_efirst, (void*)c->d_eout})
      if (p) cudaFree(p);
    c->d_echunk = nullptr;
    c->d_epart = nullptr;
    c->d_efirst = nullptr;
    c->d_eout = nullptr;
    c->energy_cap = c->energy_gcap = 0;
    const size_t cap = std::max(nc, (size_t)64), gcap = std::max((size_t)G + 1, (size_t)64);
    FW_CUDA(c, cudaMalloc((void**)&c->d_echunk, sizeof(EnergyChunk) * cap));
    FW_CUDA(c, cudaMalloc((void**)&c->d_epart, sizeof(double4) * cap));
    FW_CUDA(c, cudaMalloc((void**)&c->d_efirst, sizeof(int) * gcap));
    FW_CUDA(c, cudaMalloc((void**)&c->d_eout, sizeof(double4) * gcap));
    c->energy_cap = cap;
    c->energy_gcap = gcap;
  }
  FW_CUDA(c, cudaMemcpyAsync(c->d_echunk, chunks.data(), sizeof(EnergyChunk) * nc, cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaMemcpyAsync(c->d_efirst, first.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, c->stream));
  k_energy_chunks<<<(unsigned)nc, kEnergyThreads, 0, c->stream>>>(c->d, c->d_echunk, c->d_epart);
  k_energy_groups<<<(G + 127) / 128, 128, 0, c->stream>>>(c->d_efirst, G, c->d_epart, c->d_eout);
  c->launches += 2;
  int rc = check_kernel(c, "energy");
  if (rc) return rc;
  std::vector<double4> res(G);
  FW_CUDA(c, cudaMemcpyAsync(res.data(), c->d_eout, sizeof(double4) * G, cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  const int S = c->arena ? (int)c->ascenes.size() : c->S;
  for (int s = 0; s < 4 * S; ++s) out[s] = 0.0;
  for (int g = 0; g < G; ++g) {  // bodies of a scene in ascending order
    const int sc = c->arena ? g : c->h_scene[g];
    out[4 * sc + 0] += res[g].x;
    out[4 * sc + 1] += res[g].y;
    out[4 * sc + 2] += res[g].z;
    out[4 * sc + 3] += res[g].w;
  }
  return FW_OK;
}

int fw_scene_status(fw_ctx* c, int32_t* bad, int32_t async) {
  if (!c || !bad) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_scene_status before fw_finalize");
  FW_CUDA(c, cudaMemcpyAsync(bad, c->d.scene_bad, sizeof(int32_t) * c->S, cudaMemcpyDeviceToHost, c->stream));
  if (!async) FW_CUDA(c, cudaStreamSynchronize(c->stream));
  return FW_OK;
}

int fw_clear_scene_status(fw_ctx* c, int32_t scene) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_clear_scene_status before fw_finalize");
  if (scene < -1 || scene >= c->S) return fail(c, FW_ERR_ARG, "scene %d out of range", scene);
  if (scene < 0) FW_CUDA(c, cudaMemsetAsync(c->d.scene_bad, 0, sizeof(int32_t) * c->S, c->stream));
  else FW_CUDA(c, cudaMemsetAsync(c->d.scene_bad + scene, 0, sizeof(int32_t), c->stream));
  return FW_OK;
}

int fw_set_cfl_monitor(fw_ctx* c, const float* coef_per_body) {
  if (!c) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_set_cfl_monitor before fw_finalize");

  int rc;
  drop_graphs(c);  // captured graphs hold the previous monitor pointers
  if (!coef_per_body) {
    c->d.cfl_ord = nullptr;
    return FW_OK;
  }
  if (!c->cfl_ord_buf) {
    if ((rc = dalloc(c, &c->cfl_ord_buf, (size_t)c->S)) || (rc = dalloc(c, &c->cfl_coef_buf, (size_t)c->B)))
      return rc;
  }
  FW_CUDA(c, cudaMemcpyAsync(c->cfl_coef_buf, coef_per_body, sizeof(float) * c->B, cudaMemcpyHostToDevice, c->stream));
  std::vector<int32_t> inf(c->S, 0x7f800000);
  FW_CUDA(c, cudaMemcpyAsync(c->cfl_ord_buf, inf.data(), sizeof(int32_t) * c->S, cudaMemcpyHostToDevice, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  c->d.cfl_ord = c->cfl_ord_buf;
  c->d.body_cfl = c->cfl_coef_buf;
  return FW_OK;
}

int fw_read_cfl(fw_ctx* c, float* out, int32_t reset) {
  if (!c || !out) return FW_ERR_ARG;
  if (!c->d.cfl_ord) return fail(c, FW_ERR_STATE, "fw_read_cfl: the CFL monitor is off");
  std::vector<int32_t> v(c->S);
  FW_CUDA(c, cudaMemcpyAsync(v.data(), c->d.cfl_ord, sizeof(int32_t) * c->S, cudaMemcpyDeviceToHost, c->stream));
  if (reset) {
    std::vector<int32_t> inf(c->S, 0x7f800000);
    FW_CUDA(c, cudaMemcpyAsync(c->d.cfl_ord, inf.data(), sizeof(int32_t) * c->S, cudaMemcpyHostToDevice, c->stream));
  }
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int s = 0; s < c->S; ++s) {
    float f;
    std::memcpy(&f, &v[s], sizeof(float));
    out[s] = f;
  }
  return FW_OK;
}

int fw_read_counters(fw_ctx* c, int64_t* counters) {
  if (!c || !counters) return FW_ERR_ARG;
  if (!c->finalized) return fail(c, FW_ERR_STATE, "fw_read_counters before fw_finalize");
  std::vector<int32_t> cnt(c->S);
  FW_CUDA(c, cudaMemcpyAsync(cnt.data(), c->d.scene_counter, sizeof(int32_t) * c->S, cudaMemcpyDeviceToHost, c->stream));
  FW_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int s = 0; s < c->S; ++s) counters[s] = cnt[s];
  return FW_OK;
}

int64_t fw_launch_count(const fw_ctx* c) { return c ? c->launches : 0; }

const char* fw_build_info(void) {
  return "libfwb200: sm_100a, -fmad=false, IEEE div/sqrt; gather step + shared-memory-resident step";
}

}  // extern "C"
