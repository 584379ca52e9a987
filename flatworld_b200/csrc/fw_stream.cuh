// fw_stream.cuh -- patch-streaming substep for worlds of many scenes.
//
// Every body is cut into patches of at most kStreamNodes nodes (recursive
// coordinate bisection).  One CTA per patch and substep: it gathers the
// positions of its owned and halo nodes into shared memory, evaluates every
// triangle touching an owned node (cut triangles are evaluated by each patch
// that holds them) into shared corner forces, and updates its owned nodes --
// contact, the corner forces in ascending element order, boundary conditions,
// symplectic Euler, body boxes -- so corner forces never go to DRAM and one
// kernel does the work of k_elements + k_nodes.  Other patches read halo
// positions while a patch writes its own, so positions are double-buffered
// (x_in -> x_out, the host swaps the buffers after each substep); so is the J2
// state, which the patch owning a triangle's first corner writes.  The scene
// control (modes, gates, counters, box slots) runs first in k_control, as in
// block 0 of k_elements.  Same arithmetic in the same order as the gather step:
// the results are the same bits.
//
// The kernel is bound by the latency of its dependent loads, not by DRAM
// bandwidth, so the static data of a patch is stored in patch order
// (StreamElem per patch triangle, StreamNode per owned node; built by
// k_stream_elems / k_stream_nodes and rebuilt when a Young's modulus changes):
// a record is one load at the CTA's own offset rather than an index load
// followed by a dependent gather.  Launch shapes (run-time options, chosen by
// the autotuner): patches of 64 or 128 owned nodes, one thread per owned node
// (larger patches carry fewer halo nodes and cut triangles per triangle, at
// the price of coarser load balance over ragged scenes); a register budget
// set by the CTAs the kernel is compiled to fit on an SM; and, optionally,
// the patch's triangle records staged into shared memory by one bulk copy
// (cp.async.bulk, completion on an mbarrier) that overlaps the position
// gather, instead of one load per triangle and thread.
//
// Arena worlds (the served form) launch one CTA per patch of the scenes that
// are active in the call only (StreamDev::list); their per-scene control runs
// in k_control_scenes over the active scenes' body and pair ranges, and after
// an odd number of substeps k_stream_carry copies their state back into the
// first buffers, so the scenes that sat the call out are never touched.
#pragma once

namespace {

constexpr int kStreamNodes = 64;  // default owned nodes per patch (and threads per CTA)
constexpr int kStreamThreads = 64;
constexpr long long kBulkWaitLimit = 1ll << 24;  // polls of the staged-copy barrier before giving up

struct StreamPatch {
  int node_off, no;  // owned nodes: nodes[node_off .. +no), ascending
  int halo_off, nh;  // halo nodes: halo[halo_off .. +nh), ascending
  int elem_off, ne;  // triangles touching an owned node: elem/eid/conn[elem_off .. +ne), ascending
  int csrp_off;      // csrp[csrp_off .. +no+1): local corner-list offsets of the owned nodes
  int csr_off;       // csrs[csr_off + csrp[..]]: 3 * local triangle + corner
  int scene;
  int body;          // the body its nodes and triangles belong to
  int pad[2];
};

// Static data of one patch triangle, in patch order (32 B: what the triangle
// step reads, in one record).  Its Lame constants come from its body's entry
// of Dev::body_lm -- a body's triangles share one material -- unless
// StreamDev::lm holds them per triangle (after a per-element Young's modulus
// change); its global index, needed by J2 triangles only, is StreamDev::eid
// at the same position.
struct __align__(16) StreamElem {
  float area;  // emat[e].area
  int word;    // emat[e].word (type, body)
  uint2 conn;  // StreamDev::conn: local corner ids
  float4 ji;   // jinv[e]
};

// Static data of one owned node, in patch order.
struct __align__(16) StreamNode {
  uint32_t word;  // node_word[g]
  float mass;     // mass[g]
  float2 bcv;     // bcv[g]
};

struct StreamDev {
  const StreamPatch* patch;
  const int32_t* nodes;
  const int32_t* halo;
  const int32_t* eid;
  const uint2* conn;        // x = a | b << 16, y = c | writer << 16 (local node ids)
  const uint16_t* csrp;
  const uint16_t* csrs;
  int no_max, nh_max, ne_max;
  StreamElem* elem;  // built from eid by k_stream_elems
  StreamNode* node;  // built from nodes by k_stream_nodes
  int* err;          // != 0: a staged copy did not complete in time
  const int32_t* list;  // arena worlds: CTA i runs patch list[i] (the active scenes' patches); else patch i
  float2* lm;           // per patch triangle (lam, mu) once a triangle's Young's modulus was set; else null
};

__global__ void k_stream_nodes(Dev d, const int32_t* nodes, StreamNode* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = nodes[i];
  StreamNode r;
  r.word = d.node_word[g];
  r.mass = d.mass[g];
  r.bcv = d.bcv[g];
  out[i] = r;
}

// Records of n patch triangles.  Without lm, each also writes its body's
// Lame constants to Dev::body_lm (the body's triangles all hold the same).
__global__ void k_stream_elems(Dev d, const int32_t* eid, const uint2* conn, StreamElem* out, float2* lm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = eid[i];
  const ElemMat m = d.emat[e];
  StreamElem r;
  r.area = m.area;
  r.word = m.word;
  r.conn = conn[i];
  r.ji = d.jinv[e];
  out[i] = r;
  if (lm)
    lm[i] = make_float2(m.lam, m.mu);
  else
    d.body_lm[fw::elem_body(m.word)] = make_float2(m.lam, m.mu);
}

__global__ void k_control(Dev d) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");  // the patch step may start its gather
  step_control(d);
}

// Arena worlds step only the active scenes' patches, so after an odd number
// of substeps their state sits in the other buffers: copy each listed
// patch's owned positions (and the J2 state of the triangles it writes) back,
// so that the first buffers hold every scene's state between calls.
__global__ void k_stream_carry(StreamDev sd, const float2* __restrict__ x_from, float2* __restrict__ x_to,
                               const float4* j2_from, float4* j2_to, int has_j2) {
  const StreamPatch P = sd.patch[sd.list[blockIdx.x]];
  for (int i = threadIdx.x; i < P.no; i += blockDim.x) {
    const int g = sd.nodes[P.node_off + i];
    x_to[g] = x_from[g];
  }
  if (has_j2)
    for (int q = threadIdx.x; q < P.ne; q += blockDim.x)
      if (sd.conn[P.elem_off + q].y >> 16) {
        const int e = sd.eid[P.elem_off + q];
        j2_to[e] = j2_from[e];
      }
}

// One triangle of the patch (element_step on shared positions).
__device__ __forceinline__ void stream_element(const Dev& d, const float2* sx, float2* sf, int q,
                                               const int32_t* eid, uint2 c, ElemMat m, float4 ji,
                                               const float4* j2_in, float4* j2_out) {
  float4 j2 = make_float4(0.f, 0.f, 0.f, 0.f);
  float sy = 0.f, H = 0.f;
  const bool mises = fw::elem_type(m.word) == fw::MAT_MISES;
  int e = 0;
  if (mises) {  // the global index only for J2 triangles (their state and parameters)
    e = eid[q];
    j2 = j2_in[e];
    const float2 jp = d.j2par[e];
    sy = jp.x;
    H = jp.y;
  }
  float2 f1, f2, f3;
  fw::element_forces(sx[c.x & 0xFFFFu], sx[c.x >> 16], sx[c.y & 0xFFFFu], ji, m, sy, H, j2, f1, f2, f3);
  if (mises && (c.y >> 16)) j2_out[e] = j2;
  sf[3 * q] = f1;
  sf[3 * q + 1] = f2;
  sf[3 * q + 2] = f3;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_done(uint32_t mb, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(mb), "r"(parity)
      : "memory");
  return ok != 0;
}

// Dynamic shared memory of a stream CTA: positions (owned, then halo), the
// corner forces of its triangles, then (staged launches) its triangle records.
__host__ __device__ inline size_t stream_rec_offset(int no_max, int nh_max, int ne_max) {
  const size_t b = sizeof(float2) * (size_t)(no_max + nh_max) + sizeof(float2) * 3 * (size_t)ne_max;
  return (b + 15) & ~(size_t)15;
}

template <int NT, int MINB, bool BULK>
__global__ void __launch_bounds__(NT, MINB) k_stream(Dev d, StreamDev sd, const float2* __restrict__ x_in,
                                                     float2* __restrict__ x_out, const float4* j2_in,
                                                     float4* j2_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long s_mbar;
  __shared__ int s_cfl;  // CFL monitor: this patch's minimum bound (float bits)
  float2* sx = reinterpret_cast<float2*>(smem_raw);  // owned, then halo
  float2* sf = sx + (sd.no_max + sd.nh_max);         // 3 per patch triangle
  StreamElem* srec = reinterpret_cast<StreamElem*>(smem_raw + stream_rec_offset(sd.no_max, sd.nh_max, sd.ne_max));
  const StreamPatch P = sd.patch[sd.list ? sd.list[blockIdx.x] : (int)blockIdx.x];
  const float2 blm = d.body_lm[P.body];  // the patch's Lame constants (sd.lm null)
  const int t = threadIdx.x, T = NT;
  if (t == 0) s_cfl = 0x7f800000;  // ordered before the triangles by the barrier below
  const bool staged = BULK && P.ne > 0;
  if (staged && t == 0) {
    // one bulk copy of the patch's contiguous triangle records (32 B each:
    // 16-byte aligned, a multiple of 16 bytes), completing on s_mbar
    const uint32_t mb = smem_addr(&s_mbar);
    const uint32_t bytes = (uint32_t)P.ne * (uint32_t)sizeof(StreamElem);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(srec)),
                 "l"(sd.elem + P.elem_off), "r"(bytes), "r"(mb)
                 : "memory");
  }
  // positions of the owned (one per thread) and halo nodes
  const bool valid = t < P.no;
  const int g = valid ? sd.nodes[P.node_off + t] : 0;
  if (valid) sx[t] = x_in[g];
  for (int h = t; h < P.nh; h += T) sx[P.no + h] = x_in[sd.halo[P.halo_off + h]];
  // Launched as a programmatic dependent of the scene control (k_control,
  // k_control_scenes): the loads above touch nothing the control writes, so
  // they overlap it; here the control's results become visible.  (Returns at
  // once for an ordinary launch.)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int mode = d.scene_mode[P.scene];
  if (mode == fw::MODE_FROZEN) {  // keep the state: carry it into the other buffers
    if (valid) x_out[g] = sx[t];
    if (d.has_j2)
      for (int q = t; q < P.ne; q += T)
        if (sd.conn[P.elem_off + q].y >> 16) {
          const int e = sd.eid[P.elem_off + q];
          j2_out[e] = j2_in[e];
        }
    if (staged && t == 0) {  // the staged copy writes this CTA's shared memory: let it land (bounded)
      const uint32_t mb = smem_addr(&s_mbar);
      bool ok = mbar_done(mb, 0);
      for (long long it = 0; !ok && it < kBulkWaitLimit; ++it) ok = mbar_done(mb, 0);
      if (!ok) atomicExch(sd.err, 1);
    }
    return;
  }
  __syncthreads();  // also orders the barrier's initialisation before the waits below
  if (staged) {
    // thread 0 waits (bounded) for the staged records; the barrier below
    // hands them, or the failure, to the whole CTA.  On a timeout the error
    // flag is set and thread 0 waits once more (the copy writes this CTA's
    // shared memory) before the CTA leaves.
    __shared__ int s_ok;
    if (t == 0) {
      const uint32_t mb = smem_addr(&s_mbar);
      long long it = 0;
      bool ok = mbar_done(mb, 0);
      while (!ok && ++it < kBulkWaitLimit) ok = mbar_done(mb, 0);
      s_ok = ok ? 1 : 0;
      if (!ok) {
        atomicExch(sd.err, 1);
        for (it = 0; !ok && it < kBulkWaitLimit; ++it) ok = mbar_done(mb, 0);
      }
    }
    __syncthreads();
    if (!s_ok) return;
  }
  // triangles (element_step)
  for (int q = t; q < P.ne; q += T) {
    const StreamElem r = staged ? srec[q] : sd.elem[P.elem_off + q];
    const float2 lm = sd.lm ? sd.lm[P.elem_off + q] : blm;
    ElemMat m;
    m.area = r.area;
    m.lam = lm.x;
    m.mu = lm.y;
    m.word = r.word;
    stream_element(d, sx, sf, q, sd.eid + P.elem_off, r.conn, m, r.ji, j2_in, j2_out);
  }
  if (d.cfl_ord)  // CFL monitor: each patch triangle's current-shape bound into the CTA's minimum
    for (int q = t; q < P.ne; q += T) {
      const uint2 c = sd.conn[P.elem_off + q];
      const int word = staged ? srec[q].word : sd.elem[P.elem_off + q].word;
      const float b = cfl_bound(sx[c.x & 0xFFFFu], sx[c.x >> 16], sx[c.y & 0xFFFFu], d.body_cfl[fw::elem_body(word)]);
      atomicMin(&s_cfl, __float_as_int(b));
    }
  __syncthreads();
  if (t == 0 && d.cfl_ord && s_cfl < 0x7f800000) atomicMin(d.cfl_ord + P.scene, s_cfl);  // one per patch
  // owned nodes (node_step)
  const StreamNode nr = valid ? sd.node[P.node_off + t] : StreamNode{0u, 1.0f, make_float2(0.f, 0.f)};
  const float2 v0 = valid ? d.v[g] : make_float2(0.f, 0.f);
  const int k0 = valid ? sd.csrp[P.csrp_off + t] : 0, k1 = valid ? sd.csrp[P.csrp_off + t + 1] : 0;
  float2 x = valid ? sx[t] : make_float2(0.f, 0.f);
  const uint32_t w = nr.word;
  const float mass = nr.mass;
  const float2 bv0 = nr.bcv;
  const int b = (int)(w >> fw::NODE_BODY_SHIFT);
  bool bnd = false;
  if (valid) {
    float2 v = v0;
    const int s = P.scene;
    const float dt = mode == fw::MODE_INIT ? 0.0f : (d.uniform_dt ? d.dt_uniform : d.scene_dt[s]);
    const float damp = mode == fw::MODE_INIT ? 0.0f : d.scene_damp[s];
    float2 f = make_float2(0.f, 0.f);
    bnd = (w & fw::NODE_BOUNDARY) != 0;
    if (bnd && mode == fw::MODE_STEP) {
      const int p0 = d.body_pair_off[b], pn = d.body_pair_cnt[b];
      for (int k = 0; k < pn; ++k) {
        if (!d.pair_active[p0 + k]) continue;
        float2 cf;
        if (fw::contact_force(d.pairs[p0 + k], d.heights, d.occ, x, v, dt, cf)) {
          f.x += cf.x;
          f.y += cf.y;
        }
      }
    }
    for (int k = k0; k < k1; ++k) {  // ascending element
      const float2 cq = sf[sd.csrs[P.csr_off + k]];
      f.x += cq.x;
      f.y += cq.y;
    }
    const int bc = (int)(w & fw::NODE_BC_MASK);
    const float2 bv = (bc & (fw::BC_A | fw::BC_GRAVITY | fw::BC_FORCE | fw::BC_V)) ? bv0 : make_float2(0.f, 0.f);
    fw::integrate(bc, f, mass, bv, dt, damp, x, v);
    x_out[g] = x;
    d.v[g] = v;
    if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) d.scene_bad[s] = 1;
  }
  // per-body box of boundary nodes (as node_step)
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
    if ((int)(t & 31) == leader) {
      int* r = d.aabb_ring + ((size_t)(d.scene_counter[P.scene] & 1) * d.B + b) * 4;
      atomicMin(r + 0, fw::f2ord(lx));
      atomicMin(r + 1, fw::f2ord(ly));
      atomicMax(r + 2, fw::f2ord(hx));
      atomicMax(r + 3, fw::f2ord(hy));
    }
  } else if (bnd) {
    int* r = d.aabb_ring + ((size_t)(d.scene_counter[P.scene] & 1) * d.B + b) * 4;
    atomicMin(r + 0, fw::f2ord(lx));
    atomicMin(r + 1, fw::f2ord(ly));
    atomicMax(r + 2, fw::f2ord(hx));
    atomicMax(r + 3, fw::f2ord(hy));
  }
}

}  // namespace
