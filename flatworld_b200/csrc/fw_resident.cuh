// fw_resident.cuh -- persistent, shared-memory-resident substep kernel.
//
// When the whole world fits in the SMs' shared memory (one scene, a few
// hundred thousand triangles), the mesh is cut into patches, one per CTA
// (recursive coordinate bisection of the nodes).  A patch owns a set of nodes
// and holds every triangle that touches one of them (triangles on a cut are
// held, and evaluated, by each patch that touches them), plus the positions of
// the one-ring "halo" nodes it does not own.  One cooperative launch advances
// all CTAs through n substeps; across substeps the patch's node state, element
// data, corner forces and the ground tables stay in shared memory.  Per
// substep only the positions other patches read (a double-buffered array in
// L2) and the body bounding boxes move between SMs.
//
// Owned nodes are ordered so that the ones other CTAs need -- positions read
// as halo, and body-boundary nodes that feed the body box -- come first
// ("group 1").  Per substep, per CTA:
//   1. wait until every CTA has arrived for the previous substep (bounded
//      spin), then fetch halo positions and the body boxes (one L2 round trip)
//   2. broad-phase gates; corner forces of the cut triangles (the interior
//      triangles were done by the other warps meanwhile)
//   3. all threads: every owned node -- contact, corner forces summed in
//      ascending element order, boundary conditions, symplectic Euler --
//      group 1 first, each group-1 position published as soon as it is
//      computed, the body-box reduction (ordered-int atomics)
//   4. box hand-off (fence and arrive), then the interior triangles of the
//      next substep -- this work overlaps the other CTAs' progress
// The node sums use the same ascending-element order as the gather path, so
// both paths produce identical bits.  Every wait is bounded: after
// kSpinLimit polls the CTA sets the error flag and leaves the loop, so a
// missing CTA cannot hang the device.
//
// Two ways to hand a substep's results to the other CTAs:
//  - counter (any number of bodies): positions go to a double-buffered array,
//    body boxes to ordered-int atomics; then a release fence and an arrival
//    count; consumers poll the count, then load halo positions and boxes.
//  - flag-in-data (up to kLLMaxBodies bodies, the default there): every
//    published value is a 64-bit word (epoch << 32 | value bits), stored and
//    loaded with single-copy-atomic 64-bit relaxed accesses, so a consumer that
//    sees the expected epoch in a word also sees its value -- no fence, no
//    counter, one L2 round trip.  Each CTA publishes its exported positions and
//    its partial box per body; every CTA polls its halo words and all partial
//    boxes and reduces the boxes itself.  Because every CTA waits for every
//    CTA's partial box, no CTA runs more than one substep ahead of another, so
//    two slots (parity of the substep) suffice: a slot is rewritten only after
//    all CTAs have consumed its previous contents.  Epochs count up per launch
//    from a host-side base, so words left by earlier launches never match.
#pragma once
#include <cuda/atomic>

namespace {

constexpr int kResThreads = 512;
constexpr int kResMaxPairs = 64;
constexpr long long kSpinLimit = 1ll << 26;
constexpr long long kPollLimit = 1ll << 22;  // flag-in-data polls (each one an L2 round trip)
constexpr int kLLMaxBodies = 8;
// Flag-in-data partial boxes: a ring of kBoxRing substep slots.  CTAs read
// everyone's partial boxes only when a gate cannot be decided locally, plus
// once every kBoxSync substeps; that periodic exchange bounds how far apart
// CTAs can run to kBoxSync substeps, so a ring of 2 * kBoxSync slots is never
// overwritten before every reader is done with it.
constexpr int kBoxSync = 64;
constexpr int kBoxRing = 2 * kBoxSync;
constexpr int kResTableBytes = 48 * 1024;

struct ResPatch {
  int node_off, no;      // owned nodes: res.nodes[node_off .. +no)
  int halo_off, nh;      // halo nodes: res.halo[halo_off .. +nh)
  int elem_off, ne;      // patch triangles: interior first, each group ascending
  int n_int;             // number of interior triangles
  int csr_ptr_off;       // res.csr_ptr[csr_ptr_off .. +no+1): local offsets
  int csr_off, ncsr;     // res.csr_slot[csr_off .. +ncsr)
  int n_g1;              // owned nodes [0, n_g1) are read by other CTAs / feed body boxes
  int pad;
};

struct Res {
  const ResPatch* patch;
  const int32_t* nodes;     // owned global node ids; bit 31 = read by another patch
  const int32_t* halo;      // halo global node ids
  const uint2* conn;        // local corner ids: x = c0 | c1 << 16, y = c2 | flags << 16
  const int32_t* eid;       // global triangle id of each patch triangle
  const int32_t* csr_ptr;
  const uint16_t* csr_slot; // 3 * local triangle + corner
  float2* xpub;             // [2][N] published positions (counter mode)
  int* aabb3;               // [3][B][4] ordered-int body boxes (flag-in-data mode: [B][4] start box)
  unsigned long long* xll;  // [2][N][2] flag-in-data positions (epoch << 32 | float bits)
  unsigned long long* bll;  // [kBoxRing][B][P][4] flag-in-data partial boxes (epoch << 32 | ordered int)
  int* bar;                 // arrivals counter (reset by the prologue)
  int* err;                 // != 0: a wait gave up
  long long wait_limit;     // polls before a wait gives up (kPollLimit / kSpinLimit unless set)
  int withhold_cta;         // test hook: this CTA skips its first publish (-1: none)
  float2* rec_x;            // if set: positions at the start of each substep, [nsteps][N] (adjoint recompute)
  float2* rec_v;            // if set: velocities at the start of each substep, [nsteps][N]
  int* rec_gates;           // if set: broad-phase gates of each substep, [nsteps][rec_stride]
  int rec_stride;
  int P, no_max, nh_max, ne_max, ncsr_max;
  int has_j2;
  int tab_h, tab_o;         // ground tables staged in shared memory (floats, bytes)
  int n_bodies;
};

constexpr uint32_t kExported = 0x80000000u;
constexpr uint32_t kJ2Writer = 1u;  // flag bit in conn.y >> 16

__device__ __forceinline__ int ld_acquire(const int* p) {
  cuda::atomic_ref<const int, cuda::thread_scope_device> a(*p);
  return a.load(cuda::memory_order_acquire);
}

// 64-bit relaxed device-scope accesses: naturally aligned, single-copy atomic.
__device__ __forceinline__ unsigned long long ll_load(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void ll_store(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ll_pack(uint32_t epoch, uint32_t bits) {
  return ((unsigned long long)epoch << 32) | bits;
}
__device__ __forceinline__ bool ll_has(unsigned long long w, uint32_t epoch) {
  return (uint32_t)(w >> 32) == epoch;
}

struct ResSmem {
  float4* jinv;
  ElemMat* mat;
  float4* j2;
  float2* j2p;
  float2* f;
  float2* x;
  float2* v;
  float2* bcv;
  uint2* conn;
  float* m;
  float* im;
  int32_t* hidx;
  float* heights;
  int8_t* occ;
  uint32_t* w;
  int32_t* gid;
  uint16_t* csrp;
  uint16_t* csrs;
  int* gate;
  Pair* pairs;
  int* bpo;  // body -> first pair
  int* bpc;  // body -> pair count
};

__host__ __device__ inline size_t res_align(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared-memory carve-up; returns the byte count (device: also the pointers).
__host__ __device__ inline size_t res_layout(const Res& r, unsigned char* base, ResSmem* s) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + o : nullptr;
    o += res_align(bytes);
    return p;
  };
  ResSmem t;
  t.jinv = (float4*)take(sizeof(float4) * r.ne_max);
  t.mat = (ElemMat*)take(sizeof(ElemMat) * r.ne_max);
  t.j2 = (float4*)take(r.has_j2 ? sizeof(float4) * r.ne_max : 0);
  t.j2p = (float2*)take(r.has_j2 ? sizeof(float2) * r.ne_max : 0);
  t.f = (float2*)take(sizeof(float2) * 3 * (size_t)r.ne_max);
  t.x = (float2*)take(sizeof(float2) * (size_t)(r.no_max + r.nh_max));
  t.v = (float2*)take(sizeof(float2) * r.no_max);
  t.bcv = (float2*)take(sizeof(float2) * r.no_max);
  t.conn = (uint2*)take(sizeof(uint2) * r.ne_max);
  t.m = (float*)take(sizeof(float) * r.no_max);
  t.im = (float*)take(sizeof(float) * r.no_max);
  t.hidx = (int32_t*)take(sizeof(int32_t) * r.nh_max);
  t.heights = (float*)take(sizeof(float) * r.tab_h);
  t.occ = (int8_t*)take(r.tab_o);
  t.w = (uint32_t*)take(sizeof(uint32_t) * r.no_max);
  t.gid = (int32_t*)take(sizeof(int32_t) * r.no_max);
  t.csrp = (uint16_t*)take(sizeof(uint16_t) * (r.no_max + 1));
  t.csrs = (uint16_t*)take(sizeof(uint16_t) * r.ncsr_max);
  t.gate = (int*)take(sizeof(int) * kResMaxPairs);
  t.pairs = (Pair*)take(sizeof(Pair) * kResMaxPairs);
  t.bpo = (int*)take(sizeof(int) * r.n_bodies);
  t.bpc = (int*)take(sizeof(int) * r.n_bodies);
  if (s) *s = t;
  return o;
}

// Corner forces of patch triangle q; returns its current-shape CFL bound when
// body_cfl is given (the monitor is on), else +inf.
__device__ __forceinline__ float res_element(const ResSmem& s, int q, const float* body_cfl) {
  const uint2 c = s.conn[q];
  const float2 a = s.x[c.x & 0xFFFFu], b = s.x[c.x >> 16], cc = s.x[c.y & 0xFFFFu];
  const ElemMat m = s.mat[q];
  float4 j2 = make_float4(0.f, 0.f, 0.f, 0.f);
  float sy = 0.f, H = 0.f;
  const bool mises = fw::elem_type(m.word) == fw::MAT_MISES;
  if (mises) {
    j2 = s.j2[q];
    sy = s.j2p[q].x;
    H = s.j2p[q].y;
  }
  float2 f1, f2, f3;
  fw::element_forces(a, b, cc, s.jinv[q], m, sy, H, j2, f1, f2, f3);
  if (mises) s.j2[q] = j2;
  s.f[3 * q] = f1;
  s.f[3 * q + 1] = f2;
  s.f[3 * q + 2] = f3;
  return body_cfl ? cfl_bound(a, b, cc, body_cfl[fw::elem_body(m.word)]) : __int_as_float(0x7f800000);
}

// CFL monitor: a warp's minimum over the triangles its lanes evaluated, folded
// into the CTA's minimum (shared memory) -- every lane of the warp present.
__device__ __forceinline__ void res_cfl_fold(int* s_cfl, float v) {
  const int mb = warp_min_bits(v);
  if ((threadIdx.x & 31) == 0 && mb < 0x7f800000) atomicMin(s_cfl, mb);
}

__device__ __forceinline__ void aabb_reset(int* r) {
  r[0] = fw::f2ord(1e30f);
  r[1] = fw::f2ord(1e30f);
  r[2] = fw::f2ord(-1e30f);
  r[3] = fw::f2ord(-1e30f);
}

// Can pair p add a force to any node inside box [lo, hi]?  False only when
// that is impossible whatever the gate (a margin covers the rounding of the
// contact arithmetic): the plane's penetration is positive at every corner;
// the box lies wholly above a height field's gate box (below it when the
// field is reversed), where the signed distance to the curve is positive; the
// box misses a voxel grid's cells.  An empty box (no boundary node of the
// pair's body in this patch) cannot be reached either.
__device__ __forceinline__ bool pair_reachable(const Pair& p, float lx, float ly, float hx, float hy) {
  if (!(lx <= hx && ly <= hy)) return !(lx > hx || ly > hy);  // empty box (identity) -> false; NaN -> true
  if (p.kind == fw::PAIR_PLANE) {
    const double px = p.f[0], py = p.f[1], nx = p.f[2], ny = p.f[3];
    const double cx = nx >= 0.0 ? lx : hx, cy = ny >= 0.0 ? ly : hy;  // corner of least penetration
    const double pen = (cx - px) * nx + (cy - py) * ny;
    const double mag = 1.0 + fabs((double)lx) + fabs((double)ly) + fabs((double)hx) + fabs((double)hy) +
                       fabs(px) + fabs(py);
    return !(pen > 1e-5 * mag);
  }
  if (p.kind == fw::PAIR_HEIGHTFIELD) return p.n1 == 1 ? !(hy < p.glo[1]) : !(ly > p.ghi[1]);
  const double lbx = p.f[0], lby = p.f[1], dx = p.f[2], dz = p.f[3];
  const double ex = (double)p.n0 * dx * (1.0 + 1e-4), ey = (double)p.n1 * dz * (1.0 + 1e-4);
  return !(hx < lbx || hy < lby || lx - lbx > ex || ly - lby > ey);
}

// Update one owned node (shared-memory state) for the current substep.
__device__ __forceinline__ float2 res_node(const Dev& d, const ResSmem& s, const float* heights,
                                           const int8_t* occ, int i, float dt, float damp) {
  const uint32_t w = s.w[i];
  const int body = (int)(w >> fw::NODE_BODY_SHIFT);
  float2 x = s.x[i];
  float2 v = s.v[i];
  float2 f = make_float2(0.f, 0.f);
  if (w & fw::NODE_BOUNDARY) {
    const int p0 = s.bpo[body], pn = s.bpc[body];
    for (int q = 0; q < pn; ++q) {
      if (!s.gate[p0 + q]) continue;
      float2 cf;
      if (fw::contact_force(s.pairs[p0 + q], heights, occ, x, v, dt, cf)) {
        f.x += cf.x;
        f.y += cf.y;
      }
    }
  }
  for (int q = s.csrp[i]; q < s.csrp[i + 1]; ++q) {
    const float2 c = s.f[s.csrs[q]];
    f.x += c.x;
    f.y += c.y;
  }
  fw::integrate_im((int)(w & fw::NODE_BC_MASK), f, s.m[i], s.im[i], s.bcv[i], dt, damp, x, v);
  if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) d.scene_bad[0] = 1;  // one scene
  s.x[i] = x;
  s.v[i] = v;
  return x;
}

__device__ __forceinline__ void named_bar(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Warp-specialised substep loop.  Warps [0, FRONT) run the critical chain
// (barrier wait, halo and box loads, gates, cut triangles, box hand-off);
// the other warps compute the interior triangles of the next substep, which
// need no data from other CTAs; all warps update the owned nodes together,
// group 1 first (published as they are computed).  Shared-memory hazards:
// interior and cut triangles write disjoint corner slots; the halo part of x
// is only read by the front warps; two CTA-wide barriers per substep order
// the rest.
template <int FRONT, bool LL, int NT>
__global__ void __launch_bounds__(NT, 1)
k_resident(Dev d, Res r, int step0, int nsteps, float dt, float damp, uint32_t ep0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_abort;
  __shared__ int s_box[LL ? 4 * kLLMaxBodies : 1];   // reduced body boxes (ordered ints)
  __shared__ int s_pbox[LL ? 4 * kLLMaxBodies : 1];  // this CTA's partial boxes
  __shared__ int s_lbox[LL ? 4 * kLLMaxBodies : 1];  // the same, as of the end of the previous substep
  __shared__ int s_need;                              // a gate needs everyone's boxes this substep
  __shared__ int s_cfl;                               // CFL monitor: this CTA's minimum (float bits)
  ResSmem s;
  res_layout(r, smem_raw, &s);
  const ResPatch P = r.patch[blockIdx.x];
  const int t = threadIdx.x, T = blockDim.x;
  const int N = d.N, B = d.B;
  // ---- load the patch once
  for (int q = t; q < P.ne; q += T) {
    const int e = r.eid[P.elem_off + q];
    s.jinv[q] = d.jinv[e];
    s.mat[q] = d.emat[e];
    s.conn[q] = r.conn[P.elem_off + q];
    if (r.has_j2) {
      s.j2[q] = d.j2state[e];
      s.j2p[q] = d.j2par[e];
    }
  }
  for (int i = t; i < P.no; i += T) {
    const int g = r.nodes[P.node_off + i];
    const int gi = g & 0x7FFFFFFF;
    s.gid[i] = g;
    s.x[i] = d.x[gi];
    s.v[i] = d.v[gi];
    s.m[i] = d.mass[gi];
    s.im[i] = 1.0f / d.mass[gi];
    s.w[i] = d.node_word[gi];
    s.bcv[i] = d.bcv[gi];
  }
  for (int i = t; i < P.nh; i += T) {
    const int h = r.halo[P.halo_off + i];
    s.hidx[i] = h;
    s.x[P.no + i] = d.x[h];
  }
  for (int i = t; i <= P.no; i += T) s.csrp[i] = (uint16_t)r.csr_ptr[P.csr_ptr_off + i];
  for (int i = t; i < P.ncsr; i += T) s.csrs[i] = r.csr_slot[P.csr_off + i];
  for (int i = t; i < r.tab_h; i += T) s.heights[i] = d.heights[i];
  for (int i = t; i < r.tab_o; i += T) s.occ[i] = d.occ[i];
  for (int i = t; i < d.P; i += T) s.pairs[i] = d.pairs[i];
  for (int b = t; b < B; b += T) {
    s.bpo[b] = d.body_pair_off[b];
    s.bpc[b] = d.body_pair_cnt[b];
  }
  if (t == 0) {
    s_abort = 0;
    s_cfl = 0x7f800000;
  }
  // CFL monitor (d.cfl_ord set): each thread keeps the minimum over the
  // triangles it evaluates in this launch; folded per CTA at the end
  const float* bcfl = d.cfl_ord ? d.body_cfl : nullptr;
  float cfl = __int_as_float(0x7f800000);
  if (LL && t < 4 * B) {
    const int ident = (t & 3) < 2 ? fw::f2ord(1e30f) : fw::f2ord(-1e30f);
    s_box[t] = ident;
    s_pbox[t] = ident;
    s_lbox[t] = ident;
  }
  const float* heights = r.tab_h ? s.heights : d.heights;
  const int8_t* occ = r.tab_o ? s.occ : d.occ;
  __syncthreads();

  constexpr int FT = FRONT * 32;
  const bool front = t < FT;
  const int BT = T - FT, bt = t - FT;
  if (r.rec_x)
    for (int i = t; i < P.no; i += T) {
      r.rec_x[s.gid[i] & 0x7FFFFFFF] = s.x[i];
      r.rec_v[s.gid[i] & 0x7FFFFFFF] = s.v[i];
    }
  if (!front)
    for (int q = bt; q < P.n_int; q += BT) cfl = fminf(cfl, res_element(s, q, bcfl));
  const int node_trips = (P.no + T - 1) / T;
  for (int k = 0; k < nsteps; ++k) {
    const int g = step0 + k;
    if (front) {
      // previous substep complete everywhere -> halo positions, body boxes
      if (k > 0 && LL) {
        const uint32_t want = ep0 + (uint32_t)k;
        // Gates decided from this patch's own boundary nodes where that is
        // exact (s_lbox: its partial boxes at the end of the previous
        // substep): the body box contains the partial box, so a partial box
        // that meets the ground box proves the gate on (on the 10%-growth
        // substeps too: growth only enlarges both boxes); and a pair that can
        // reach none of the patch's nodes changes no force here, on or off.
        // Otherwise (and every kBoxSync substeps, and while gates are being
        // recorded: s_need preset at the end of the previous substep) the
        // patch reads every CTA's partial box.  Decided before the halo poll,
        // which they do not depend on.
        if (t < d.P) {
          const Pair& pr = s.pairs[t];
          const int* lb = s_lbox + 4 * pr.body;
          const float lx = fw::ord2f(lb[0]), ly = fw::ord2f(lb[1]), hx = fw::ord2f(lb[2]), hy = fw::ord2f(lb[3]);
          if (lx <= pr.ghi[0] && hx >= pr.glo[0] && ly <= pr.ghi[1] && hy >= pr.glo[1]) {
            s.gate[t] = 1;
          } else if (!pair_reachable(pr, lx, ly, hx, hy)) {
            s.gate[t] = 0;
          } else {
            s_need = 1;
          }
        }
        const unsigned long long* src = r.xll + (size_t)(k & 1) * N * 2;
        for (int i = t; i < P.nh; i += FT) {
          const unsigned long long* w = src + 2 * (size_t)s.hidx[i];
          unsigned long long wx, wy;
          long long it = 0;
          while (true) {
            wx = ll_load(w);
            wy = ll_load(w + 1);
            if (ll_has(wx, want) && ll_has(wy, want)) break;
            if ((++it & 1023) == 0 && (it > r.wait_limit || *(volatile int*)r.err)) {
              atomicExch(r.err, 1);
              s_abort = 1;
              break;
            }
          }
          s.x[P.no + i] = make_float2(__uint_as_float((uint32_t)wx), __uint_as_float((uint32_t)wy));
        }
        named_bar(1, FT);  // halo positions, local gates and s_need are final
        if (s_need && !s_abort) {
          const unsigned long long* bsrc = r.bll + (size_t)(k % kBoxRing) * B * r.P * 4;
          for (int j = t; j < B * r.P; j += FT) {
            const unsigned long long* w = bsrc + (size_t)j * 4;
            unsigned long long b0, b1, b2, b3;
            long long it = 0;
            while (true) {
              b0 = ll_load(w);
              b1 = ll_load(w + 1);
              b2 = ll_load(w + 2);
              b3 = ll_load(w + 3);
              if (ll_has(b0, want) && ll_has(b1, want) && ll_has(b2, want) && ll_has(b3, want)) break;
              if ((++it & 1023) == 0 && (it > r.wait_limit || *(volatile int*)r.err)) {
                atomicExch(r.err, 1);
                s_abort = 1;
                break;
              }
            }
            int* bx = s_box + 4 * (j / r.P);
            atomicMin(bx + 0, (int)(uint32_t)b0);
            atomicMin(bx + 1, (int)(uint32_t)b1);
            atomicMax(bx + 2, (int)(uint32_t)b2);
            atomicMax(bx + 3, (int)(uint32_t)b3);
          }
          named_bar(1, FT);
        }
      } else if (k > 0) {
        if (t == 0) {
          long long it = 0;
          const int target = r.P * k;
          while (ld_acquire(r.bar) < target) {
            if (++it > r.wait_limit || *(volatile int*)r.err) {
              atomicExch(r.err, 1);
              s_abort = 1;
              break;
            }
            __nanosleep(20);
          }
        }
        named_bar(1, FT);
        if (!s_abort) {
          const float2* src = r.xpub + (size_t)(k & 1) * N;
          for (int i = t; i < P.nh; i += FT) s.x[P.no + i] = __ldcg(src + s.hidx[i]);
        }
      }
      const bool exact_gates = !LL || k == 0 || s_need;  // else decided locally above
      if (!s_abort) {
        if (t < d.P && exact_gates) {
          const Pair& pr = s.pairs[t];
          int4 bb;
          if (LL)
            bb = k > 0 ? make_int4(s_box[4 * pr.body], s_box[4 * pr.body + 1], s_box[4 * pr.body + 2],
                                   s_box[4 * pr.body + 3])
                       : __ldcg(reinterpret_cast<const int4*>(r.aabb3 + (size_t)pr.body * 4));
          else
            bb = __ldcg(reinterpret_cast<const int4*>(r.aabb3 + ((size_t)(g % 3) * B + pr.body) * 4));
          s.gate[t] = fw::pair_gate(pr, fw::ord2f(bb.x), fw::ord2f(bb.y), fw::ord2f(bb.z), fw::ord2f(bb.w), g) ? 1 : 0;
          if (r.rec_gates && blockIdx.x == 0) r.rec_gates[(size_t)k * r.rec_stride + t] = s.gate[t];
        }
        if (!LL && blockIdx.x == 0)
          for (int b = t; b < B; b += FT) aabb_reset(r.aabb3 + ((size_t)((g + 2) % 3) * B + b) * 4);
        if (exact_gates) {
          named_bar(1, FT);
          if (LL && t < 4 * B) s_box[t] = (t & 3) < 2 ? fw::f2ord(1e30f) : fw::f2ord(-1e30f);
        }
        for (int q = P.n_int + t; q < P.ne; q += FT) cfl = fminf(cfl, res_element(s, q, bcfl));
      }
    }
    __syncthreads();  // every triangle of substep k is done
    if (s_abort) break;
    {
      // Every owned node, all threads together (one pass when the patch has
      // at most T nodes); the nodes other CTAs read or that feed the body box
      // ([0, n_g1)) are the first ones, and each is published as soon as it
      // is computed.
      float2* dst = r.xpub + (size_t)((k + 1) & 1) * N;
      unsigned long long* dll = r.xll + (size_t)((k + 1) & 1) * N * 2;
      const uint32_t ep_out = ep0 + (uint32_t)k + 1u;
      int* box_w = r.aabb3 + (size_t)((g + 1) % 3) * B * 4;
      for (int trip = 0; trip < node_trips; ++trip) {
        const int i = trip * T + t;
        bool bnd = false;
        int body = 0;
        float2 x = make_float2(0.f, 0.f);
        if (i < P.no) {
          x = res_node(d, s, heights, occ, i, dt, damp);
          if (i < P.n_g1) {
            const uint32_t w = s.w[i];
            body = (int)(w >> fw::NODE_BODY_SHIFT);
            bnd = (w & fw::NODE_BOUNDARY) != 0;
            const int gid = s.gid[i];
            if (gid < 0 && !(k == 0 && (int)blockIdx.x == r.withhold_cta)) {
              const size_t gi = (size_t)(gid & 0x7FFFFFFF);
              if (LL) {
                ll_store(dll + 2 * gi, ll_pack(ep_out, __float_as_uint(x.x)));
                ll_store(dll + 2 * gi + 1, ll_pack(ep_out, __float_as_uint(x.y)));
              } else {
                __stcg(dst + gi, x);
              }
            }
          }
        }
        const unsigned full = 0xFFFFFFFFu;
        const unsigned mb = __ballot_sync(full, bnd);
        if (mb != 0u) {
          const int leader = __ffs(mb) - 1;
          const int bl = __shfl_sync(full, body, leader);
          const bool uniform = __all_sync(full, !bnd || body == bl);
          float lx = bnd ? x.x : 1e30f, ly = bnd ? x.y : 1e30f;
          float hx = bnd ? x.x : -1e30f, hy = bnd ? x.y : -1e30f;
          if (uniform) {
            for (int o = 16; o > 0; o >>= 1) {
              lx = fminf(lx, __shfl_xor_sync(full, lx, o));
              ly = fminf(ly, __shfl_xor_sync(full, ly, o));
              hx = fmaxf(hx, __shfl_xor_sync(full, hx, o));
              hy = fmaxf(hy, __shfl_xor_sync(full, hy, o));
            }
          }
          if ((uniform && (int)(t & 31) == leader) || (!uniform && bnd)) {
            int* rb = LL ? s_pbox + 4 * body : box_w + (size_t)body * 4;
            atomicMin(rb + 0, fw::f2ord(lx));
            atomicMin(rb + 1, fw::f2ord(ly));
            atomicMax(rb + 2, fw::f2ord(hx));
            atomicMax(rb + 3, fw::f2ord(hy));
          }
        }
      }
    }
    __syncthreads();  // every owned node of substep k is updated; this CTA's box partials are final
    if (front) {
      const bool withhold = k == 0 && (int)blockIdx.x == r.withhold_cta;
      if (LL) {
        if (t < 4 * B && !withhold) {  // this CTA's partial box of body t / 4, component t % 4
          unsigned long long* bdst =
              r.bll + ((size_t)((k + 1) % kBoxRing) * B * r.P + (size_t)(t >> 2) * r.P + blockIdx.x) * 4;
          ll_store(bdst + (t & 3), ll_pack(ep0 + (uint32_t)k + 1u, (uint32_t)s_pbox[t]));
        }
        if (t < 4 * B) {
          s_lbox[t] = s_pbox[t];
          s_pbox[t] = (t & 3) < 2 ? fw::f2ord(1e30f) : fw::f2ord(-1e30f);
        }
        if (t == 0) s_need = ((k + 1) % kBoxSync == 0 || r.rec_gates != nullptr) ? 1 : 0;
        named_bar(1, FT);  // s_lbox and s_need before the next substep's gate decisions
      } else if (t == 0 && !withhold) {
        cuda::atomic_ref<int, cuda::thread_scope_device> a(*r.bar);
        a.fetch_add(1, cuda::memory_order_release);
      }
    }
    if (r.rec_x && k + 1 < nsteps)  // owned positions stay as they are until the next CTA barrier
      for (int i = t; i < P.no; i += T) {
        r.rec_x[(size_t)(k + 1) * N + (s.gid[i] & 0x7FFFFFFF)] = s.x[i];
        r.rec_v[(size_t)(k + 1) * N + (s.gid[i] & 0x7FFFFFFF)] = s.v[i];
      }
    if (!front && k + 1 < nsteps)
      for (int q = bt; q < P.n_int; q += BT) cfl = fminf(cfl, res_element(s, q, bcfl));
  }
  // ---- write the patch state back
  __syncthreads();
  if (d.cfl_ord) {  // one atomic per CTA and launch (a single-scene world)
    res_cfl_fold(&s_cfl, cfl);
    __syncthreads();
    if (t == 0 && s_cfl < 0x7f800000) atomicMin(d.cfl_ord, s_cfl);
  }
  for (int i = t; i < P.no; i += T) {
    const int gi = s.gid[i] & 0x7FFFFFFF;
    d.x[gi] = s.x[i];
    d.v[gi] = s.v[i];
  }
  if (r.has_j2)
    for (int q = t; q < P.ne; q += T)
      if ((s.conn[q].y >> 16) & kJ2Writer) d.j2state[r.eid[P.elem_off + q]] = s.j2[q];
}

// ------------------------------------------------------------------ resident adjoint
// Reverse pass of one segment on the same patches (cooperative launch): the
// adjoint state of the owned nodes (xb, vb, fb in FP64) and dL/dE of the
// triangles whose first corner the patch owns stay in shared memory; the
// positions of each substep come from the recorded trajectory.  Per reverse
// substep the only cross-CTA traffic is the force adjoint of exported nodes,
// published as flag-in-data words (each FP64 value as two 32-bit halves, each
// with the epoch); halo membership is symmetric, so neighbours stay within one
// substep of each other and two parity slots suffice.  The arithmetic and its
// order are those of k_adj_prep / k_adj_elements / k_adj_nodes, so both
// reverse passes give the same bits.
struct ResAdjSmem {
  double2* xb;
  double2* vb;
  double2* fb;  // owned, then halo
  double* Eb;
  float* yng;
};

__host__ __device__ inline size_t res_adj_layout(const Res& r, unsigned char* base, ResAdjSmem* s) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + o : nullptr;
    o += res_align(bytes);
    return p;
  };
  ResAdjSmem t;
  t.xb = (double2*)take(sizeof(double2) * r.no_max);
  t.vb = (double2*)take(sizeof(double2) * r.no_max);
  t.fb = (double2*)take(sizeof(double2) * (size_t)(r.no_max + r.nh_max));
  t.Eb = (double*)take(sizeof(double) * r.ne_max);
  t.yng = (float*)take(sizeof(float) * r.ne_max);
  if (s) *s = t;
  return o;
}

__device__ __forceinline__ void res_adj_prep(const ResSmem& s, const ResAdjSmem& q, int i, double h, double damp) {
  const int bc = (int)(s.w[i] & fw::NODE_BC_MASK);
  const double2 xb = q.xb[i], vb = q.vb[i];
  const double2 vt = make_double2(vb.x + h * xb.x, vb.y + h * xb.y);
  const bool vfixed = (bc & (fw::BC_U | fw::BC_V)) != 0;
  const bool fdead = vfixed || (bc & fw::BC_A) != 0;
  const double sc = h / (double)s.m[i];
  const double keep = 1.0 - sc * damp;
  q.fb[i] = fdead ? make_double2(0.0, 0.0) : make_double2(sc * vt.x, sc * vt.y);
  q.vb[i] = vfixed ? make_double2(0.0, 0.0) : make_double2(keep * vt.x, keep * vt.y);
}

__device__ __forceinline__ uint32_t lo32(double v) { return (uint32_t)(__double_as_longlong(v) & 0xFFFFFFFFll); }
__device__ __forceinline__ uint32_t hi32(double v) { return (uint32_t)((unsigned long long)__double_as_longlong(v) >> 32); }
__device__ __forceinline__ double join64(uint32_t lo, uint32_t hi) {
  return __longlong_as_double((long long)(((unsigned long long)hi << 32) | lo));
}

__global__ void __launch_bounds__(kResThreads, 1)
k_res_adj(Dev d, Res r, Adj a, const float2* __restrict__ rec_x, const float2* __restrict__ rec_v,
          const int* __restrict__ rec_gates,
          int gate_stride, unsigned long long* fll, int nsteps, float dt, float damp, uint32_t ep0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_abort;
  ResSmem s;
  const size_t base = res_layout(r, smem_raw, &s);
  ResAdjSmem q;
  res_adj_layout(r, smem_raw + base, &q);
  const ResPatch P = r.patch[blockIdx.x];
  const int t = threadIdx.x, T = blockDim.x;
  const int N = d.N;
  // ---- load the patch and its adjoint state
  for (int k = t; k < P.ne; k += T) {
    const int e = r.eid[P.elem_off + k];
    s.jinv[k] = d.jinv[e];
    s.mat[k] = d.emat[e];
    s.conn[k] = r.conn[P.elem_off + k];
    q.yng[k] = a.young[e];
    q.Eb[k] = ((s.conn[k].y >> 16) & kJ2Writer) ? a.Eb[e] : 0.0;
  }
  for (int i = t; i < P.no; i += T) {
    const int g = r.nodes[P.node_off + i];
    const int gi = g & 0x7FFFFFFF;
    s.gid[i] = g;
    s.m[i] = d.mass[gi];
    s.w[i] = d.node_word[gi];
    q.xb[i] = a.xb[gi];
    q.vb[i] = a.vb[gi];
  }
  for (int i = t; i < P.nh; i += T) s.hidx[i] = r.halo[P.halo_off + i];
  for (int i = t; i <= P.no; i += T) s.csrp[i] = (uint16_t)r.csr_ptr[P.csr_ptr_off + i];
  for (int i = t; i < P.ncsr; i += T) s.csrs[i] = r.csr_slot[P.csr_off + i];
  for (int i = t; i < d.P; i += T) s.pairs[i] = d.pairs[i];
  for (int b = t; b < d.B; b += T) {
    s.bpo[b] = d.body_pair_off[b];
    s.bpc[b] = d.body_pair_cnt[b];
  }
  if (t == 0) s_abort = 0;
  __syncthreads();
  const double h = (double)dt, dmp = (double)damp;
  for (int i = t; i < P.no; i += T) res_adj_prep(s, q, i, h, dmp);  // the segment's last substep
  __syncthreads();
  for (int rr = 0; rr < nsteps; ++rr) {
    const int j = nsteps - 1 - rr;
    const uint32_t ep = ep0 + (uint32_t)rr + 1u;
    unsigned long long* slot = fll + (size_t)(rr & 1) * N * 4;
    // publish the force adjoints others read; positions of substep j
    for (int i = t; i < P.no; i += T) {
      const int g = s.gid[i];
      const int gi = g & 0x7FFFFFFF;
      s.x[i] = rec_x[(size_t)j * N + gi];
      if (g < 0) {
        const double2 f = q.fb[i];
        unsigned long long* w = slot + 4 * (size_t)gi;
        ll_store(w, ll_pack(ep, lo32(f.x)));
        ll_store(w + 1, ll_pack(ep, hi32(f.x)));
        ll_store(w + 2, ll_pack(ep, lo32(f.y)));
        ll_store(w + 3, ll_pack(ep, hi32(f.y)));
      }
    }
    for (int k = t; k < P.nh; k += T) {
      const int gi = s.hidx[k];
      s.x[P.no + k] = rec_x[(size_t)j * N + gi];
      const unsigned long long* w = slot + 4 * (size_t)gi;
      unsigned long long w0, w1, w2, w3;
      long long it = 0;
      while (true) {
        w0 = ll_load(w);
        w1 = ll_load(w + 1);
        w2 = ll_load(w + 2);
        w3 = ll_load(w + 3);
        if (ll_has(w0, ep) && ll_has(w1, ep) && ll_has(w2, ep) && ll_has(w3, ep)) break;
        if ((++it & 1023) == 0 && (it > r.wait_limit || *(volatile int*)r.err)) {
          atomicExch(r.err, 1);
          s_abort = 1;
          break;
        }
      }
      q.fb[P.no + k] = make_double2(join64((uint32_t)w0, (uint32_t)w1), join64((uint32_t)w2, (uint32_t)w3));
    }
    __syncthreads();
    if (s_abort) break;
    // element Jacobian products with the force adjoints (as k_adj_elements)
    for (int k = t; k < P.ne; k += T) {
      const uint2 c = s.conn[k];
      const int i0 = c.x & 0xFFFFu, i1 = c.x >> 16, i2 = c.y & 0xFFFFu;
      const double2 b0 = q.fb[i0], b1 = q.fb[i1], b2 = q.fb[i2];
      const float2 w0 = make_float2((float)b0.x, (float)b0.y), w1 = make_float2((float)b1.x, (float)b1.y),
                   w2 = make_float2((float)b2.x, (float)b2.y);
      const ElemMat m = s.mat[k];
      fw::Dual f[6];
      fw::element_forces_jvp(s.x[i0], s.x[i1], s.x[i2], w0, w1, w2, s.jinv[k], fw::elem_type(m.word), m.lam, m.mu,
                             m.area, f);
      s.f[3 * k] = make_float2(f[0].d, f[1].d);
      s.f[3 * k + 1] = make_float2(f[2].d, f[3].d);
      s.f[3 * k + 2] = make_float2(f[4].d, f[5].d);
      if ((c.y >> 16) & kJ2Writer) {
        const double dot = b0.x * f[0].v + b0.y * f[1].v + b1.x * f[2].v + b1.y * f[3].v + b2.x * f[4].v +
                           b2.y * f[5].v;
        q.Eb[k] += dot / (double)q.yng[k];
      }
    }
    __syncthreads();
    // xb += element VJPs + plane contact; then the previous substep's adjoints (as k_adj_nodes)
    for (int i = t; i < P.no; i += T) {
      double2 xb = q.xb[i];
      const double2 fb = q.fb[i];
      for (int k = s.csrp[i]; k < s.csrp[i + 1]; ++k) {
        const float2 c = s.f[s.csrs[k]];
        xb.x += c.x;
        xb.y += c.y;
      }
      const uint32_t w = s.w[i];
      if (w & fw::NODE_BOUNDARY) {
        const int b = (int)(w >> fw::NODE_BODY_SHIFT);
        const float2 xi = s.x[i], vi = rec_v[(size_t)j * N + (s.gid[i] & 0x7FFFFFFF)];
        double2 vb = q.vb[i];
        for (int k = 0; k < s.bpc[b]; ++k) {
          const int p = s.bpo[b] + k;
          if (!rec_gates[(size_t)j * gate_stride + p]) continue;
          fw::contact_vjp(s.pairs[p], d.heights, d.occ, xi, vi, dt, fb, xb, vb);
        }
        q.vb[i] = vb;
      }
      q.xb[i] = xb;
      if (j > 0) res_adj_prep(s, q, i, h, dmp);
    }
    __syncthreads();
  }
  // ---- write the adjoint state back
  __syncthreads();
  for (int i = t; i < P.no; i += T) {
    const int gi = s.gid[i] & 0x7FFFFFFF;
    a.xb[gi] = q.xb[i];
    a.vb[gi] = q.vb[i];
  }
  for (int k = t; k < P.ne; k += T)
    if ((s.conn[k].y >> 16) & kJ2Writer) a.Eb[r.eid[P.elem_off + k]] = q.Eb[k];
}

using ResKernel = void (*)(Dev, Res, int, int, float, float, uint32_t);
constexpr int kFrontChoices[] = {2, 4, 6, 8};          // of 16 warps (512 threads)
constexpr int kFrontChoices1024[] = {8, 12, 16};       // of 32 warps (1024 threads, 64 registers)
inline ResKernel res_kernel(int front, bool ll, int threads) {
  if (threads == 1024) {
    switch (front) {
      case 8: return ll ? k_resident<8, true, 1024> : k_resident<8, false, 1024>;
      case 16: return ll ? k_resident<16, true, 1024> : k_resident<16, false, 1024>;
      default: return ll ? k_resident<12, true, 1024> : k_resident<12, false, 1024>;
    }
  }
  switch (front) {
    case 2: return ll ? k_resident<2, true, 512> : k_resident<2, false, 512>;
    case 6: return ll ? k_resident<6, true, 512> : k_resident<6, false, 512>;
    case 8: return ll ? k_resident<8, true, 512> : k_resident<8, false, 512>;
    default: return ll ? k_resident<4, true, 512> : k_resident<4, false, 512>;
  }
}

// Before a resident launch: reset the barrier and error flag, copy the body
// boxes of the last substep into slot step0 % 3 and clear slot (step0+1) % 3.
// (Flag-in-data mode: the start boxes go to slot 0, nothing else.)
__global__ void k_res_prologue(Dev d, Res r, int step0, int ll) {
  if (threadIdx.x == 0) {
    *r.bar = 0;
    *r.err = 0;
  }
  const int cur = d.scene_counter[0] & 1;
  for (int b = threadIdx.x; b < d.B; b += blockDim.x) {
    const int* src = d.aabb_ring + ((size_t)cur * d.B + b) * 4;
    int* a = r.aabb3 + ((size_t)(ll ? 0 : step0 % 3) * d.B + b) * 4;
    for (int k = 0; k < 4; ++k) a[k] = src[k];
    if (!ll) aabb_reset(r.aabb3 + ((size_t)((step0 + 1) % 3) * d.B + b) * 4);
  }
}

// After a resident launch: publish the final body boxes to the gather path's
// slots and advance the step counter.
__global__ void k_res_epilogue(Dev d, Res r, int step0, int nsteps) {
  const int last = step0 + nsteps;
  const int dst_slot = last & 1;
  for (int b = threadIdx.x; b < d.B; b += blockDim.x) {
    const int* a = r.aabb3 + ((size_t)(last % 3) * d.B + b) * 4;
    int* dst = d.aabb_ring + ((size_t)dst_slot * d.B + b) * 4;
    for (int k = 0; k < 4; ++k) dst[k] = a[k];
  }
  if (threadIdx.x == 0) d.scene_counter[0] = last;
}

// Flag-in-data variant: the final boxes are the reduction of the partial
// boxes of the last substep (ring slot nsteps % kBoxRing); the launch has
// completed, so plain loads see them.
__global__ void k_res_epilogue_ll(Dev d, Res r, int step0, int nsteps) {
  __shared__ int box[4 * kLLMaxBodies];
  const int B = d.B, t = threadIdx.x;
  if (t < 4 * B) box[t] = (t & 3) < 2 ? fw::f2ord(1e30f) : fw::f2ord(-1e30f);
  __syncthreads();
  const unsigned long long* src = r.bll + (size_t)(nsteps % kBoxRing) * B * r.P * 4;
  for (int j = t; j < B * r.P; j += blockDim.x) {
    const unsigned long long* w = src + (size_t)j * 4;
    int* bx = box + 4 * (j / r.P);
    atomicMin(bx + 0, (int)(uint32_t)w[0]);
    atomicMin(bx + 1, (int)(uint32_t)w[1]);
    atomicMax(bx + 2, (int)(uint32_t)w[2]);
    atomicMax(bx + 3, (int)(uint32_t)w[3]);
  }
  __syncthreads();
  const int last = step0 + nsteps;
  if (t < 4 * B) d.aabb_ring[(size_t)(last & 1) * B * 4 + t] = box[t];
  if (t == 0) d.scene_counter[0] = last;
}

}  // namespace
