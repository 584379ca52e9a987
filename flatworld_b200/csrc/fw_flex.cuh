// fw_flex.cuh -- FEM-FEM penalty contact: the reference's ContactFlexFlex on
// its spatial-hash path (flatworld/mixedcontact.py:886-1018, launched from
// run_batched_contacts, mixedcontact.py:1662-1696).
//
// Work items (one per boundary node and contact pair side, built on the host
// in the reference's order, mixedcontact.py:1876-1924) look for the boundary
// edge of the other body that they penetrate: first the edge they hit last
// time (the per-item cache), then every candidate the spatial hash returns
// around the node.  The hash (flatworld/spatialmanager.py) is rebuilt on the
// device whenever 1/500 s of simulated time has accumulated
// (femspringmanager.py:1035-1039), from the boundary-edge boxes and the FEM
// domain boxes of the end of the previous substep.  Its cells list their
// elements in registration order -- what the reference's counting sort gives
// when its atomic counters hand out indices in launch order -- so here the
// cells are filled with atomics and then sorted.  Each work item keeps its own
// candidate list (the reference's GPU launch shares one 512-entry list among
// all items, spatialmanager.py:564 / mixedcontact.py:2545, a race; the serial
// reading is the race-free one).
//
// A contact adds a force to the node and the reactions to the edge's two
// nodes.  In the reference these are atomic_adds in work-item order; here each
// node keeps a short list of (work item, force) entries, which k_nodes sorts
// by work item and adds between the plane and the height-field / voxel
// contact forces -- the reference's launch order -- so no float atomics are
// needed and the sums repeat bit for bit.
#pragma once

namespace {

constexpr int kFlexMaxQuery = 512;                   // SpatialHashManager max_query_results
constexpr int kFlexMaxCells = 100000;                // SpatialHashManager max_cells
constexpr int kFlexListCap = 16;                     // contributions one node takes per substep
constexpr double kFlexRebuildInterval = 1.0 / 500.0; // FemSpringManager._sh_rebuild_interval
constexpr int kFlexScanThreads = 1024;

struct FlexGrid {
  int tc, cnx, cny, npairs;
  int simple;    // every element sits in every cell of its box (no cell cap, no pair truncation)
  int n_active;  // work items of active (pair, side) segments this substep
  int pad2[2];
  float olx, oly, gsx, gsy;
  int estimate;  // ordered-int minimum of the element box diagonals
  int rebuild;   // this substep rebuilds the hash
  int tie_init;  // the scene's tied work items have looked for their edges (first substep)
  int pad;
  double elapsed;   // simulated time since the last rebuild (float64, as the host's float)
};

// One scene with FEM-FEM contact: where its part of every array starts.
struct FlexScene {
  int scene, body0, n_fem;       // the scene and its bodies (FEM-local index = body - body0)
  int dom_off, n_dom, skip_bvh;  // its domains (dom_obj / dom_body / dom_box)
  int pair_off, n_pairs;         // its ContactFlexFlex pairs
  int seg_base, n_seg;           // its (pair, side) segments; seg_off holds n_seg + 1 entries at seg_base + k
  int be0, n_be;                 // its boundary edges (registration order)
  int max_pairs, pair_base;      // its (cell, element) pair capacity and slot base
  int cell_base, pad;            // its cells: k * kFlexMaxCells
  int n_tied, n_untied;          // its work items of tied / untied pairs
};

// The FEM-FEM state of a world; a kernel works on one scene's view of it
// (flex_view): the scalars are that scene's, the per-scene pointers start at
// its part.  Items, pairs' body ids, nodes, bodies and boundary edges keep
// global indices.
struct FlexDev {
  int n_items, n_fs;
  int n_pairs, n_fem, n_dom, skip_bvh, n_be, be0, body0, scene;  // the view's scene
  int max_pairs;
  float mpd;  // max(pow(100000.0f, 0.5f), 1.0f), evaluated on the host
  const FlexScene* sc;
  const double* clock_dt;  // per FEM-FEM scene: its substep dt as the host's float64 holds it
  int* err;                // bit 0: a node's contribution list overflowed
  const int32_t* item_node;
  const int32_t* item_target;  // the body whose edges the item searches
  const int32_t* item_pair;
  const float* item_pen;
  const float* item_fric;
  int32_t* item_cache;  // boundary edge hit last time, or -1
  const int2* pair_body;  // (domain1, domain2) global body ids
  const int2* be;         // per boundary edge: its two global node ids
  const int32_t* be_dom;  // per boundary edge: its body
  const int32_t* be_off;  // per body: its first boundary edge
  const int32_t* be_cnt;
  const int32_t* dom_obj;   // per domain of the scene: a broad-phase object (considerContact)
  const int32_t* dom_body;  // per domain: global body id, -1 for a ground, -2 - r for rigid r
  const float4* dom_box;    // per domain: a ground's static box
  int32_t* pair_active;
  int32_t* stamped;  // at body0 + g: the scene's domain g is in a broad-phase pair this substep
  FlexGrid* g;
  float4* ebox;
  int32_t* ecount;
  int32_t* ebase;
  int32_t* cell_count;
  int32_t* cell_start;
  int32_t* cell_end;
  int32_t* cursor;
  int32_t* sorted;
  int2* crange;  // (start, end) of cell (ix, iy) at ix * cny + iy: a column is contiguous
  int2* ecell;   // per element: its lowest cell (ix, iy), clamped to the grid
  int4* srec;    // per cell entry (cell order): element, its body, its two nodes
  int2* scell;   // per cell entry: the element's lowest cell
  int n_seg;            // (pair, side) segments of consecutive work items
  const int4* seg;      // per segment: first item, item count, pair (in the scene), target body
  int32_t* seg_off;     // [n_seg + 1]: exclusive scan of the active segments' item counts
  // tied pairs (ExplicitLoop(ties=...)): per pair, and per work item the edge
  // it found at the first substep (-1: none), its weights and normal gap
  const int32_t* pair_tied;
  int32_t* tie_elem;
  float* tie_w0;
  float* tie_w1;
  float* tie_gap;
  int n_tied, n_untied;  // the view's scene
};

__device__ __forceinline__ FlexDev flex_view(const FlexDev& f0, int k) {
  const FlexScene c = f0.sc[k];
  FlexDev f = f0;
  f.scene = c.scene; f.body0 = c.body0; f.n_fem = c.n_fem; f.n_dom = c.n_dom; f.skip_bvh = c.skip_bvh;
  f.n_pairs = c.n_pairs; f.n_seg = c.n_seg; f.be0 = c.be0; f.n_be = c.n_be; f.max_pairs = c.max_pairs;
  f.dom_obj += c.dom_off; f.dom_body += c.dom_off; f.dom_box += c.dom_off;
  f.pair_body += c.pair_off; f.pair_active += c.pair_off; f.pair_tied += c.pair_off;
  f.n_tied = c.n_tied; f.n_untied = c.n_untied;
  f.g += k;
  f.cell_count += c.cell_base; f.cell_start += c.cell_base; f.cell_end += c.cell_base;
  f.cursor += c.cell_base; f.crange += c.cell_base;
  f.sorted += c.pair_base; f.srec += c.pair_base; f.scell += c.pair_base;
  f.seg += c.seg_base; f.seg_off += c.seg_base + k;
  return f;
}

// wp.min / wp.max on floats: a < b ? a : b (first argument on ties)
__device__ __forceinline__ float wmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float wmax(float a, float b) { return a > b ? a : b; }

__device__ __forceinline__ bool flex_stepping(const Dev& d, int s) {
  return d.scene_active[s] && !d.scene_mode_req[s];
}

// A rigid domain's current box (lb x, y, ub x, y), as the broad phase sees it.
__device__ __forceinline__ float4 rigid_box(const Rigid& g) { return make_float4(g.lb[0], g.lb[1], g.ub[0], g.ub[1]); }

__device__ __forceinline__ float4 ring_box(const Dev& d, int slot, int body) {
  const int* r = d.aabb_ring + ((size_t)slot * d.B + body) * 4;
  return make_float4(fw::ord2f(r[0]), fw::ord2f(r[1]), fw::ord2f(r[2]), fw::ord2f(r[3]));
}

// Broad-phase overlap of two leaf boxes, grown by 10% of their extent on the
// steps the reference rebuilds its BVH (as fw::pair_gate).
__device__ __forceinline__ bool flex_boxes_overlap(float4 a, float4 b, int counter) {
  if (counter % 100 == 0) {
    const float ax = 0.1f * (a.z - a.x), ay = 0.1f * (a.w - a.y);
    const float bx = 0.1f * (b.z - b.x), by = 0.1f * (b.w - b.y);
    a.x = a.x - ax; a.z = a.z + ax; a.y = a.y - ay; a.w = a.w + ay;
    b.x = b.x - bx; b.z = b.z + bx; b.y = b.y - by; b.w = b.w + by;
  }
  return a.x <= b.z && a.z >= b.x && a.y <= b.w && a.w >= b.y;
}

__device__ __forceinline__ int flex_cell(float delta, float gs, int n) {
  int c = (int)floorf(delta / gs);
  c = c > 0 ? c : 0;
  c = c < n - 1 ? c : n - 1;
  return c;
}

// Exclusive scan of n ints (one CTA of kFlexScanThreads); returns the total.
// Each thread scans a contiguous chunk, the chunk sums are scanned in shared
// memory.
__device__ int flex_block_scan(const int32_t* in, int32_t* out, int n) {
  __shared__ int part[kFlexScanThreads];
  const int t = threadIdx.x;
  __syncthreads();  // a previous call's readers of part[] are done
  const int chunk = (n + kFlexScanThreads - 1) / kFlexScanThreads;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  int sum = 0;
  for (int i = lo; i < hi; ++i) sum += in[i];
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < kFlexScanThreads; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (int i = lo; i < hi; ++i) {
    const int v = in[i];
    out[i] = run;
    run += v;
  }
  return part[kFlexScanThreads - 1];
}

__device__ __forceinline__ void flex_elem_cells(const FlexGrid& g, float4 eb, int& lx, int& ly, int& ux, int& uy) {
  lx = flex_cell(eb.x - g.olx, g.gsx, g.cnx);
  ly = flex_cell(eb.y - g.oly, g.gsy, g.cny);
  ux = flex_cell(eb.z - g.olx, g.gsx, g.cnx);
  uy = flex_cell(eb.w - g.oly, g.gsy, g.cny);
}

// The spatial-hash rebuild, by the whole block, phase after phase:
// populate_fem_spatial_hash + SpatialHashManager.build (femspringmanager.py:
// 1041-1063; spatialmanager.py:200-420, 613-712).  Registration index =
// boundary-edge index.  The (cell, element) pairs get the pair indices of
// _expand_pairs_kernel's counter in launch order (a scan of the per-element
// counts), so the reference's MAX_PAIRS truncation is reproduced; cells are
// filled with atomics and then sorted, giving each cell its elements in
// registration order.
__device__ void flex_rebuild(const Dev& d, const FlexDev& f) {
  const int t = threadIdx.x, T = blockDim.x;
  const int e0 = f.be0, e1 = f.be0 + f.n_be;
  // add_element for every boundary edge
  for (int e = e0 + t; e < e1; e += T) {
    const int2 n = f.be[e];
    const float2 a = d.x[n.x], b = d.x[n.y];
    float lx = 1e30f, ly = 1e30f, ux = -1e30f, uy = -1e30f;
    lx = wmin(lx, a.x); ly = wmin(ly, a.y); ux = wmax(ux, a.x); uy = wmax(uy, a.y);
    lx = wmin(lx, b.x); ly = wmin(ly, b.y); ux = wmax(ux, b.x); uy = wmax(uy, b.y);
    const float4 bb = make_float4(lx - 0.0f, ly - 0.0f, ux + 0.0f, uy + 0.0f);
    f.ebox[e] = bb;
    const float dx = bb.z - bb.x, dy = bb.w - bb.y;
    atomicMin(&f.g->estimate, fw::f2ord(sqrtf(dx * dx + dy * dy)));
  }
  __syncthreads();
  // the global box of the FEM domains (populate kernel) and _build_grid_kernel
  if (t == 0) {
    const int slot = d.scene_counter[f.scene] & 1;
    float glx = 1e9f, gly = 1e9f, gux = -1e9f, guy = -1e9f;
    for (int k = 0; k < f.n_fem; ++k) {
      const float4 bb = ring_box(d, slot, f.body0 + k);
      glx = wmin(glx, bb.x);
      gly = wmin(gly, bb.y);
      gux = wmax(gux, bb.z);
      guy = wmax(guy, bb.w);
    }
    const float extent = wmax(gux - glx, guy - gly);
    const float expand = extent * 0.01f + 0.0f;
    glx = glx - expand;
    gly = gly - expand;
    gux = gux + expand;
    guy = guy + expand;
    float cell = fw::ord2f(f.g->estimate) * 1.5f;
    const float exx = gux - glx, exy = guy - gly;
    cell = wmax(cell, exx / f.mpd);
    cell = wmax(cell, exy / f.mpd);
    const float cs = cell + 1e-6f;
    const int nx = (int)wmax(ceilf(exx / cs), 1.0f);
    const int ny = (int)wmax(ceilf(exy / cs), 1.0f);
    FlexGrid* g = f.g;
    g->olx = glx;
    g->oly = gly;
    g->cnx = nx;
    g->cny = ny;
    g->gsx = exx / (float)nx;
    g->gsy = exy / (float)ny;
    const int total = nx * ny;
    g->tc = total < kFlexMaxCells ? total : kFlexMaxCells;
  }
  __syncthreads();
  FlexGrid g = *f.g;
  // zero the cell counts; per element its lowest cell and how many pairs it makes
  for (int c = t; c < g.tc; c += T) f.cell_count[c] = 0;
  for (int e = e0 + t; e < e1; e += T) {
    int lx, ly, ux, uy, n = 0;
    flex_elem_cells(g, f.ebox[e], lx, ly, ux, uy);
    f.ecell[e] = make_int2(lx, ly);
    for (int ix = lx; ix <= ux; ++ix)
      for (int iy = ly; iy <= uy; ++iy)
        if (ix + iy * g.cnx < g.tc) ++n;
    f.ecount[e] = n;
  }
  __syncthreads();
  const int npairs = flex_block_scan(f.ecount + e0, f.ebase + e0, f.n_be);
  if (t == 0) {
    f.g->npairs = npairs;
    f.g->simple = (g.tc == g.cnx * g.cny && npairs <= f.max_pairs) ? 1 : 0;
  }
  __syncthreads();  // every chunk of ebase is written
  // counts of the pairs kept (pair index < max_pairs)
  for (int e = e0 + t; e < e1; e += T) {
    int lx, ly, ux, uy, p = f.ebase[e];
    flex_elem_cells(g, f.ebox[e], lx, ly, ux, uy);
    for (int ix = lx; ix <= ux; ++ix)
      for (int iy = ly; iy <= uy; ++iy) {
        const int cid = ix + iy * g.cnx;
        if (cid < g.tc) {
          if (p < f.max_pairs) atomicAdd(&f.cell_count[cid], 1);
          ++p;
        }
      }
  }
  __syncthreads();
  flex_block_scan(f.cell_count, f.cell_start, g.tc);
  __syncthreads();
  for (int c = t; c < g.tc; c += T) {
    f.cursor[c] = f.cell_start[c];
    f.cell_end[c] = f.cell_start[c] + f.cell_count[c];
  }
  __syncthreads();
  for (int e = e0 + t; e < e1; e += T) {
    int lx, ly, ux, uy, p = f.ebase[e];
    flex_elem_cells(g, f.ebox[e], lx, ly, ux, uy);
    for (int ix = lx; ix <= ux; ++ix)
      for (int iy = ly; iy <= uy; ++iy) {
        const int cid = ix + iy * g.cnx;
        if (cid < g.tc) {
          if (p < f.max_pairs) f.sorted[atomicAdd(&f.cursor[cid], 1)] = e;
          ++p;
        }
      }
  }
  __syncthreads();
  const bool simple = f.g->simple != 0;
  // registration order inside every cell (insertion sort; cells hold few
  // elements), then what the contact walk reads of each entry
  for (int c = t; c < g.tc; c += T) {
    const int lo = f.cell_start[c], hi = f.cell_end[c];
    for (int i = lo + 1; i < hi; ++i) {
      const int v = f.sorted[i];
      int j = i - 1;
      while (j >= lo && f.sorted[j] > v) {
        f.sorted[j + 1] = f.sorted[j];
        --j;
      }
      f.sorted[j + 1] = v;
    }
    if (simple) {  // then tc = cnx * cny <= kFlexMaxCells: the column index is in range
      f.crange[(c % g.cnx) * g.cny + c / g.cnx] = make_int2(lo, hi);
      for (int i = lo; i < hi; ++i) {
        const int e = f.sorted[i];
        const int2 n = f.be[e];
        f.srec[i] = make_int4(e, f.be_dom[e], n.x, n.y);
        f.scell[i] = f.ecell[e];
      }
    }
  }
  __syncthreads();
}

__device__ void flex_ties(const Dev& d, const FlexDev& f);

// Per substep, before k_elements, one block: the hash clock and, when it
// fires, the rebuild (flex_rebuild); pair activation, the broad-phase domain
// stamps, and the compacted list of work items that run.  force != 0: the
// construction-time build (explicitloop.py:383-385) -- rebuild, no contact.
// Dynamic shared memory: (n_dom + n_fem) boxes -- every domain's, then every
// FEM body's.
__global__ void __launch_bounds__(kFlexScanThreads) k_flex_pre(Dev d, FlexDev f0, int force) {
  extern __shared__ float4 sbox[];
  __shared__ int s_rebuild;
  const FlexDev f = flex_view(f0, blockIdx.x);  // one block per scene with FEM-FEM contact
  const int s = f.scene;
  const bool step = !force && flex_stepping(d, s);
  if (threadIdx.x == 0) {
    int rb = force ? 1 : 0;
    // maybe_rebuild_fem_spatial_hash(self.dt), called while untied work items
    // remain or the tied ones have not looked for their edges yet
    // (mixedcontact.py:1667-1678)
    if (step && (f.n_untied > 0 || (f.n_tied > 0 && !f.g->tie_init))) {
      double e = f.g->elapsed + f.clock_dt[blockIdx.x];
      if (e >= kFlexRebuildInterval) {
        rb = 1;
        e = 0.0;
      }
      f.g->elapsed = e;
    }
    f.g->rebuild = rb;
    if (rb) f.g->estimate = fw::f2ord(1e30f);
    if (!step) f.g->n_active = 0;
    s_rebuild = rb;
  }
  __syncthreads();
  if (s_rebuild) flex_rebuild(d, f);
  if (!step) return;
  const int k = d.scene_counter[s];
  const int slot = k & 1;
  float4* body_box = sbox + f.n_dom;
  for (int g = threadIdx.x; g < f.n_dom; g += blockDim.x)
    sbox[g] = f.dom_body[g] >= 0    ? ring_box(d, slot, f.dom_body[g])
              : f.dom_body[g] <= -2 ? rigid_box(d.rig[-2 - f.dom_body[g]])
                                    : f.dom_box[g];
  for (int b = threadIdx.x; b < f.n_fem; b += blockDim.x) body_box[b] = ring_box(d, slot, f.body0 + b);
  __syncthreads();
  // _activate_or_fill_pairs: every pair when the loop has no BVH, else BVH overlap
  for (int p = threadIdx.x; p < f.n_pairs; p += blockDim.x) {
    const int2 pb = f.pair_body[p];
    f.pair_active[p] = f.skip_bvh ? 1 : (flex_boxes_overlap(body_box[pb.x - f.body0], body_box[pb.y - f.body0], k) ? 1 : 0);
  }
  // _scan_bvh_pairs_stamp_kernel: domain g (global index) is stamped when it
  // is in some broad-phase pair; the contact kernel reads the stamp at the
  // item's fem-local target index.  One warp per g.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int gi = warp; gi < f.n_fem; gi += nwarps) {
    bool st = false;
    if (gi < f.n_dom && f.dom_obj[gi]) {
      const float4 a = sbox[gi];
      for (int h0 = 0; h0 < f.n_dom && !st; h0 += 32) {
        const int h = h0 + lane;
        const bool hit = h < f.n_dom && h != gi && f.dom_obj[h] && flex_boxes_overlap(a, sbox[h], k);
        st = __any_sync(0xFFFFFFFFu, hit);
      }
    }
    if (lane == 0) f.stamped[f.body0 + gi] = st ? 1 : 0;
  }
  __syncthreads();
  // the work items that run: the (pair, side) segments whose pair is active
  // and whose target is stamped (or every one when the loop has no BVH),
  // compacted so the contact kernel visits nothing else
  for (int q = threadIdx.x; q < f.n_seg; q += blockDim.x) {
    const int4 sg = f.seg[q];
    const bool on = !f.pair_tied[sg.z] && f.pair_active[sg.z] && (f.skip_bvh || f.stamped[sg.w]);
    f.seg_off[q] = on ? sg.y : 0;
  }
  __syncthreads();
  const int total = flex_block_scan(f.seg_off, f.seg_off, f.n_seg);
  if (threadIdx.x == 0) {
    f.seg_off[f.n_seg] = total;
    f.g->n_active = total;
  }
  if (f.n_tied > 0) flex_ties(d, f);
}

// pointToEdgeContact + detectPointToMeshBoundary (contact_detection.py:15-92):
// the penetration if |pen| < limit and the point projects inside the edge,
// else 1e9; the weights either way.
__device__ __forceinline__ float flex_detect(float2 p, float2 a, float2 b, float limit, float& nx, float& ny,
                                             float& w0, float& w1) {
  const float ex = b.x - a.x, ey = b.y - a.y;
  const float len = sqrtf(ex * ex + ey * ey);
  float pen = 1e9f, mx = 0.f, my = 0.f;
  bool inside = false;
  w0 = 0.f;
  w1 = 0.f;
  if (len > 1e-9f) {
    const float dx = ex / len, dy = ey / len;
    mx = dy;
    my = -dx;
    const float tx = p.x - a.x, ty = p.y - a.y;
    float t = tx * dx + ty * dy;
    t = t / len;
    if (0.0f <= t && t <= 1.0f) {
      inside = true;
      pen = tx * mx + ty * my;
      w0 = 1.0f - t;
      w1 = t;
    }
  }
  nx = 0.f;
  ny = 0.f;
  if (fabsf(pen) < limit && inside) {
    nx = mx;
    ny = my;
    return pen;
  }
  return 1e9f;
}

__device__ __forceinline__ void flex_push(const Dev& d, int* err, int node, int item, float2 force) {
  const int slot = d.flex_slot[node];
  const int j = atomicAdd(&d.flex_cnt[slot], 1);
  if (j < kFlexListCap) {
    d.flex_item[slot * kFlexListCap + j] = item;
    d.flex_force[slot * kFlexListCap + j] = force;
  } else {
    atomicOr(err, 1);
  }
}

// Tied pairs (mixedcontact.py:1680-1690).  At the scene's first substep every
// tied work item looks for the boundary edge of its target nearest to its node
// (_initialize_fem_fem_ties_once_kernel, mixedcontact.py:686-771: the hash
// query with a buffer of max(1e-4, cell size, 0.001), the smallest |pen|
// inside it) and keeps the edge, the weights of the foot point and the gap
// along the edge normal; every substep a penalty spring then pulls the node to
// that point (_apply_fem_fem_ties_fixed_kernel, mixedcontact.py:774-809), with
// the reactions on the edge's nodes.  The reference launches the ties before
// the contact kernel, which skips tied items: tie entries carry the work item
// as their key, contact entries n_items + work item, so each node adds its tie
// forces first.
__device__ __forceinline__ float2 flex_tie_point(const Dev& d, int2 n, float w0, float w1) {
  const float2 a = d.x[n.x], b = d.x[n.y];
  float x = 0.0f, y = 0.0f;
  x = x + a.x * w0;
  y = y + a.y * w0;
  x = x + b.x * w1;
  y = y + b.y * w1;
  return make_float2(x, y);
}

__device__ __forceinline__ float2 flex_tie_normal(const Dev& d, int2 n) {
  const float2 a = d.x[n.x], b = d.x[n.y];
  const float ex = b.x - a.x, ey = b.y - a.y;
  const float el = sqrtf(ex * ex + ey * ey);
  float tx = 1.0f, ty = 0.0f;
  if (el > 1e-10f) {
    tx = ex / el;
    ty = ey / el;
  }
  return make_float2(-ty, tx);
}

__device__ void flex_tie_resolve(const Dev& d, const FlexDev& f, const FlexGrid& g, int it, int target) {
  if (g.tc <= 0) return;
  const int nid = f.item_node[it];
  const float2 p = d.x[nid];
  const float qbuf = wmax(wmax(1e-4f, wmax(g.gsx, g.gsy)), 0.001f);
  const int lx = flex_cell(p.x - qbuf - g.olx, g.gsx, g.cnx), ly = flex_cell(p.y - qbuf - g.oly, g.gsy, g.cny);
  const int ux = flex_cell(p.x + qbuf - g.olx, g.gsx, g.cnx), uy = flex_cell(p.y + qbuf - g.oly, g.gsy, g.cny);
  int cand[kFlexMaxQuery];
  int num = 0;
  for (int ix = lx; ix <= ux; ++ix)
    for (int iy = ly; iy <= uy; ++iy) {
      const int cid = ix + iy * g.cnx;
      if (cid < 0 || cid >= g.tc) continue;
      for (int q = f.cell_start[cid]; q < f.cell_end[cid]; ++q) {
        const int e = f.sorted[q];
        if (e < 0 || f.be_dom[e] != target) continue;
        bool dup = false;
        for (int k = 0; k < num; ++k) dup |= cand[k] == e;
        if (!dup && num < kFlexMaxQuery) cand[num++] = e;
      }
    }
  float best = 1e9f, bw0 = 0.f, bw1 = 0.f;
  int be = -1;
  for (int j = 0; j < num; ++j) {
    const int e = cand[j];
    const int2 n = f.be[e];
    float nx, ny, w0, w1;
    const float pen = flex_detect(p, d.x[n.x], d.x[n.y], qbuf, nx, ny, w0, w1);
    if (fabsf(pen) < fabsf(best) && fabsf(pen) < qbuf) {
      bw0 = w0;
      bw1 = w1;
      be = e;
      best = pen;
    }
  }
  if (be < 0) return;
  const int2 n = f.be[be];
  const float2 cp = flex_tie_point(d, n, bw0, bw1);
  const float gx = p.x - cp.x, gy = p.y - cp.y;
  const float2 nn = flex_tie_normal(d, n);
  f.tie_elem[it] = be;
  f.tie_w0[it] = bw0;
  f.tie_w1[it] = bw1;
  f.tie_gap[it] = gx * nn.x + gy * nn.y;
}

__device__ void flex_ties(const Dev& d, const FlexDev& f) {
  __syncthreads();  // the hash (if rebuilt) and the grid are final
  const bool init = f.g->tie_init == 0;
  const FlexGrid g = *f.g;
  __syncthreads();  // every thread has read tie_init
  for (int q = 0; q < f.n_seg; ++q) {
    const int4 sg = f.seg[q];
    if (!f.pair_tied[sg.z]) continue;
    for (int it = sg.x + threadIdx.x; it < sg.x + sg.y; it += blockDim.x) {
      if (init && f.tie_elem[it] < 0) flex_tie_resolve(d, f, g, it, sg.w);
      const int e = f.tie_elem[it];
      if (e < 0) continue;
      const int nid = f.item_node[it];
      const int2 n = f.be[e];
      const float w0 = f.tie_w0[it], w1 = f.tie_w1[it], gap = f.tie_gap[it], k = f.item_pen[it];
      const float2 cp = flex_tie_point(d, n, w0, w1);
      const float2 nn = flex_tie_normal(d, n);
      const float2 x = d.x[nid];
      const float tx = cp.x + gap * nn.x, ty = cp.y + gap * nn.y;
      const float mx = tx - x.x, my = ty - x.y;
      const float fx = k * mx, fy = k * my;
      flex_push(d, f.err, nid, it, make_float2(fx, fy));
      flex_push(d, f.err, n.x, it, make_float2(-(fx * w0), -(fy * w0)));
      flex_push(d, f.err, n.y, it, make_float2(-(fx * w1), -(fy * w1)));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && init) f.g->tie_init = 1;
}

// _batched_flexflex_contact_kernel_sh.  A work item's pair is active only
// where two bodies meet, so few items run; to keep the SMs busy each item
// gets kFlexLanes lanes.  The query walks cells ix-major then iy, each cell's
// elements in order, strict < keeping the first minimum.  When every element
// sits in every cell of its box (no cell cap, no pair truncation: g.simple),
// an element is new at cell (ix, iy) exactly when that is the first cell of
// its box inside the query window, so no candidate list is needed: the
// window's cells are cut into kFlexLanes contiguous runs of the walk, each
// lane keeps the first minimum of its run, and the group takes the smallest
// penetration, ties to the lower lane (earlier in the walk) -- the serial
// result.  Otherwise, or past the reference's 512 unique candidates, the walk
// keeps the candidate list as written.
constexpr int kFlexLanes = 8;
constexpr int kFlexContactThreads = 128;

struct FlexBest {
  float pen, nx, ny, w0, w1;
  int e, n0, n1;
};

__device__ __forceinline__ void flex_item(const Dev& d, const FlexDev& f, const FlexGrid& g, int it, int target,
                                          int sub, unsigned gmask) {
  const int nid = f.item_node[it];
  const int be_off = f.be_off[target], be_cnt = f.be_cnt[target];
  const float2 p = d.x[nid], vp = d.v[nid];
  const float pen_k = f.item_pen[it], fric = f.item_fric[it];
  const float qbuf = wmax(wmax(1e-4f, wmax(g.gsx, g.gsy)), 0.016f);
  float best = 1e9f, bnx = 0.f, bny = 0.f, bw0 = 0.f, bw1 = 0.f;
  int bn0 = 0, bn1 = 0;
  bool found = false;
  const int cached = f.item_cache[it];
  int cache_out = cached;
  if (cached >= be_off && cached < be_off + be_cnt) {
    const int2 n = f.be[cached];
    const float2 a = d.x[n.x], b = d.x[n.y];
    float lx = 1e30f, ly = 1e30f, ux = -1e30f, uy = -1e30f;
    lx = wmin(lx, a.x); ly = wmin(ly, a.y); ux = wmax(ux, a.x); uy = wmax(uy, a.y);
    lx = wmin(lx, b.x); ly = wmin(ly, b.y); ux = wmax(ux, b.x); uy = wmax(uy, b.y);
    const float dx = ux - lx, dy = uy - ly;
    const float margin = wmax(1e-4f, 1e-2f * sqrtf(dx * dx + dy * dy));
    lx = lx - margin; ly = ly - margin; ux = ux + margin; uy = uy + margin;
    const bool outside = wmin(p.x - lx, p.y - ly) < 0.0f || wmin(ux - p.x, uy - p.y) < 0.0f;
    if (!outside) {
      float nx, ny, w0, w1;
      const float pen = flex_detect(p, a, b, margin, nx, ny, w0, w1);
      if (pen < 1e-4f && fabsf(pen) < margin) {
        best = pen; bnx = nx; bny = ny; bw0 = w0; bw1 = w1; bn0 = n.x; bn1 = n.y; found = true;
      }
    }
  }
  if (!found && g.tc > 0) {  // query_point_with_buffer, then every candidate in order
    const int lx = flex_cell(p.x - qbuf - g.olx, g.gsx, g.cnx), ly = flex_cell(p.y - qbuf - g.oly, g.gsy, g.cny);
    const int ux = flex_cell(p.x + qbuf - g.olx, g.gsx, g.cnx), uy = flex_cell(p.y + qbuf - g.oly, g.gsy, g.cny);
    bool serial = !g.simple;
    if (g.simple) {
      const int h = uy - ly + 1, ncell = (ux - lx + 1) * h;
      const int chunk = (ncell + kFlexLanes - 1) / kFlexLanes;
      const int t1 = min(ncell, (sub + 1) * chunk);
      FlexBest b{1e9f, 0.f, 0.f, 0.f, 0.f, -1, 0, 0};
      int num = 0;
      for (int t = min(ncell, sub * chunk); t < t1; ++t) {
        const int ix = lx + t / h, iy = ly + t % h;
        const int2 r = f.crange[ix * g.cny + iy];
        for (int q = r.x; q < r.y; ++q) {
          const int4 rec = f.srec[q];  // element, domain, nodes
          if (rec.y != target) continue;
          const int2 ec = f.scell[q];
          if (ix != (lx > ec.x ? lx : ec.x) || iy != (ly > ec.y ? ly : ec.y)) continue;  // seen earlier
          ++num;
          float nx, ny, w0, w1;
          const float pen = flex_detect(p, d.x[rec.z], d.x[rec.w], qbuf, nx, ny, w0, w1);
          if (pen < b.pen && pen < 1e-4f && fabsf(pen) < qbuf) b = FlexBest{pen, nx, ny, w0, w1, rec.x, rec.z, rec.w};
        }
      }
      for (int o = kFlexLanes / 2; o > 0; o >>= 1) num += __shfl_xor_sync(gmask, num, o);
      if (num > kFlexMaxQuery) {
        serial = true;  // the reference stops adding candidates at 512: walk as written
      } else {
        float wp = b.pen;
        int wl = sub;
        for (int o = kFlexLanes / 2; o > 0; o >>= 1) {  // min penetration, ties to the lower lane
          const float op = __shfl_xor_sync(gmask, wp, o);
          const int ol = __shfl_xor_sync(gmask, wl, o);
          if (op < wp || (op == wp && ol < wl)) {
            wp = op;
            wl = ol;
          }
        }
        const int src = (threadIdx.x & 31 & ~(kFlexLanes - 1)) + wl;
        const int we = __shfl_sync(gmask, b.e, src);
        const float pbest = __shfl_sync(gmask, b.pen, src), pnx = __shfl_sync(gmask, b.nx, src);
        const float pny = __shfl_sync(gmask, b.ny, src), pw0 = __shfl_sync(gmask, b.w0, src);
        const float pw1 = __shfl_sync(gmask, b.w1, src);
        const int pn0 = __shfl_sync(gmask, b.n0, src), pn1 = __shfl_sync(gmask, b.n1, src);
        if (we >= 0) {
          best = pbest; bnx = pnx; bny = pny; bw0 = pw0; bw1 = pw1; bn0 = pn0; bn1 = pn1;
          found = true;
          cache_out = we;
        }
      }
    }
    if (serial) {  // every lane of the group walks the window (same result in each)
      int cand[kFlexMaxQuery];
      int num = 0;
      for (int ix = lx; ix <= ux; ++ix)
        for (int iy = ly; iy <= uy; ++iy) {
          const int cid = ix + iy * g.cnx;
          if (cid < 0 || cid >= g.tc) continue;
          for (int q = f.cell_start[cid]; q < f.cell_end[cid]; ++q) {
            const int e = f.sorted[q];
            if (e < 0 || f.be_dom[e] != target) continue;
            bool dup = false;
            for (int k = 0; k < num; ++k) dup |= cand[k] == e;
            if (!dup && num < kFlexMaxQuery) cand[num++] = e;
          }
        }
      for (int j = 0; j < num; ++j) {
        const int e = cand[j];
        const int2 n = f.be[e];
        float nx, ny, w0, w1;
        const float pen = flex_detect(p, d.x[n.x], d.x[n.y], qbuf, nx, ny, w0, w1);
        if (pen < best && pen < 1e-4f && fabsf(pen) < qbuf) {
          best = pen; bnx = nx; bny = ny; bw0 = w0; bw1 = w1; bn0 = n.x; bn1 = n.y; found = true;
          cache_out = e;
        }
      }
    }
  }
  if (sub != 0) return;
  if (!found) cache_out = -1;
  if (cache_out != cached) f.item_cache[it] = cache_out;
  if (found && best < 0.0f) {
    const float fx = -bnx * pen_k * best, fy = -bny * pen_k * best;
    float tx = fx, ty = fy;
    if (fric > 1e-9f) {
      const float2 va = d.v[bn0], vb = d.v[bn1];
      const float sx = va.x * bw0 + vb.x * bw1, sy = va.y * bw0 + vb.y * bw1;
      const float rx = vp.x - sx, ry = vp.y - sy;
      const float dn = rx * bnx + ry * bny;
      const float gx = rx - dn * bnx, gy = ry - dn * bny;
      const float tl = sqrtf(gx * gx + gy * gy);
      if (tl > 1e-9f) {
        const float ddx = -gx / tl, ddy = -gy / tl;
        const float nl = sqrtf(fx * fx + fy * fy);
        tx = tx + ddx * fric * nl;
        ty = ty + ddy * fric * nl;
      }
    }
    const int key = f.n_items + it;  // after every tie entry of the node
    flex_push(d, f.err, nid, key, make_float2(tx, ty));
    flex_push(d, f.err, bn0, key, make_float2(-(tx * bw0), -(ty * bw0)));
    flex_push(d, f.err, bn1, key, make_float2(-(tx * bw1), -(ty * bw1)));
  }
}

// Each group of kFlexLanes lanes takes active work items in turn (grid
// stride over the compacted list): the item's segment by binary search over
// the segment offsets, then flex_item.
__global__ void __launch_bounds__(kFlexContactThreads) k_flex_contact(Dev d, FlexDev f0) {
  const FlexDev f = flex_view(f0, blockIdx.y);  // blockIdx.y: the scene
  const int sub = threadIdx.x % kFlexLanes;
  const unsigned gmask = ((1u << kFlexLanes) - 1u) << ((threadIdx.x & 31) & ~(kFlexLanes - 1));
  const FlexGrid g = *f.g;
  const int groups = gridDim.x * (blockDim.x / kFlexLanes);
  for (int a = blockIdx.x * (blockDim.x / kFlexLanes) + threadIdx.x / kFlexLanes; a < g.n_active; a += groups) {
    int lo = 0, hi = f.n_seg - 1;  // the last segment whose offset is <= a (the active one of a run)
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (f.seg_off[mid] <= a) lo = mid;
      else hi = mid - 1;
    }
    const int4 sg = f.seg[lo];
    flex_item(d, f, g, sg.x + (a - f.seg_off[lo]), sg.w, sub, gmask);
  }
}

}  // namespace
