/*
 * fwb200.h -- C ABI of the B200 explicit 2D FEM step (libfwb200.so).
 *
 * The reference (FlatWorld) has no foreign-function interface: its "plugin
 * API" is the Python object model, and the device work happens in Warp kernels
 * launched by two Python classes.  Each entry point below replaces one of those
 * launch sites; the Python package flatworld_b200 binds them with ctypes and
 * keeps the reference's class names on top.  References are file:line in the
 * FlatWorld project.
 *
 * Conventions
 *   - Plain C types only: pointers, sizes, float/double/int.  No torch types.
 *   - Every function returns 0 (FW_OK) or a negative FW_ERR_* code; the text of
 *     the last error of a context is fw_last_error(ctx).  No C++ exception
 *     crosses this boundary.
 *   - Host arrays passed in are copied during the call; the library owns all
 *     device memory of a context.  Arrays are little-endian, C order.
 *   - A world holds S independent scenes (S = 1 for one ExplicitLoop).  Each
 *     scene has its own time step, damping, step counter and active flag;
 *     scenes never exchange forces.  Bodies (FEM domains) belong to a scene,
 *     contact pairs to a body.
 *   - Calls on one context are not re-entrant; different contexts are
 *     independent.  Device work is queued on the context's stream
 *     (fw_set_stream, default: a non-blocking stream the context creates).
 */
#ifndef FWB200_H
#define FWB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FW_OK 0
#define FW_ERR_ARG -1       /* bad argument (size, index, pointer) */
#define FW_ERR_OOM -2       /* device allocation failed */
#define FW_ERR_CUDA -3      /* a CUDA runtime call failed */
#define FW_ERR_TIMEOUT -4   /* a bounded device wait gave up */
#define FW_ERR_NONFINITE -5 /* a NaN/inf was found in the state */
#define FW_ERR_STATE -6     /* call out of order (e.g. step before finalize) */
#define FW_ERR_UNSUPPORTED -7 /* the world reached a state outside the library (rigid-rigid / rigid-ground contact) */

/* Node boundary-condition bits: same values as the reference's
 * flatworld/definitions.py:96-104. */
#define FW_BC_U 0x1
#define FW_BC_V 0x2
#define FW_BC_A 0x4
#define FW_BC_FORCE 0x8
#define FW_BC_GRAVITY 0x10

/* Material types: flatworld/definitions.py:80-83. */
#define FW_MAT_ELASTIC 1
#define FW_MAT_NEOHOOKEAN 2
#define FW_MAT_MISES 3

/* Node array selectors for fw_read_nodes / fw_write_nodes. */
#define FW_FIELD_X 0    /* current coordinates (FemSpringManager.coords) */
#define FW_FIELD_V 1    /* velocities (FemSpringManager.V) */
#define FW_FIELD_MASS 2 /* lumped mass, one float per node (FemSpringManager.mass) */
#define FW_FIELD_X0 3   /* rest coordinates */

/* Step implementations (fw_set_path). */
#define FW_PATH_AUTO 0     /* resident when the world fits, else gather */
#define FW_PATH_GATHER 1   /* two kernels per substep, any world */
#define FW_PATH_RESIDENT 2 /* one persistent kernel per fw_step call */
#define FW_PATH_STREAM 3   /* one patch-streaming kernel per substep (worlds of many scenes) */

typedef struct fw_ctx fw_ctx;
typedef struct fw_pack fw_pack; /* a scene prepared for an arena (fw_arena_pack) */

/* Create / destroy a context on CUDA device `device`.
 * Replaces: FemSpringManager.__init__ buffer allocation,
 * flatworld/femspringmanager.py:509-637. */
int fw_create(fw_ctx** out, int device);
void fw_destroy(fw_ctx* ctx);
const char* fw_last_error(const fw_ctx* ctx);
/* Queue work on a caller stream (a cudaStream_t passed as void*; NULL = the
 * context's own stream). */
int fw_set_stream(fw_ctx* ctx, void* stream);

/* Packed nodes of all bodies of all scenes: coords[2n], vel[2n] (initial
 * velocities), bc_bits[n] (OR of FW_BC_*), bc_values[2n] (value of the last BC
 * that touched the node).
 * Replaces: addFemDomain coords packing and processConditions,
 * flatworld/femspringmanager.py:660-705, 741. */
int fw_set_nodes(fw_ctx* ctx, int32_t n_nodes, const float* coords, const float* vel,
                 const int32_t* bc_bits, const float* bc_values);

/* Packed triangles: conn[3e] (global node ids), per-element material.
 * Replaces: addFemDomain element packing, flatworld/femspringmanager.py:743-766. */
int fw_set_elements(fw_ctx* ctx, int32_t n_elems, const int32_t* conn, const int32_t* mat_type,
                    const float* young, const float* poisson, const float* density,
                    const float* yield_stress, const float* hardening);

/* Bodies (FEM domains): node range, element range, owning scene and the
 * sorted boundary-node ids (global) of each body.
 * Replaces: addFemDomain offsets and boundary-node packing,
 * flatworld/femspringmanager.py:735-799. */
int fw_set_bodies(fw_ctx* ctx, int32_t n_bodies, const int32_t* node_offset,
                  const int32_t* node_count, const int32_t* elem_offset, const int32_t* elem_count,
                  const int32_t* scene_of_body, const int32_t* bnode_offset,
                  const int32_t* bnode_count, int32_t n_bnodes, const int32_t* bnodes);

/* Scenes: per-scene damping (ExplicitLoop damping kwarg).
 * Replaces: ExplicitLoop.__init__ state, flatworld/explicitloop.py:72-85, 172-175. */
int fw_set_scenes(fw_ctx* ctx, int32_t n_scenes, const float* damping);

/* Change scene `scene`'s velocity damping after fw_finalize; it applies from
 * the next substep on.  The reference reads ExplicitLoop.damping at every
 * substep (explicitloop.py:528, 537), so assigning it mid-run takes effect. */
int fw_set_damping(fw_ctx* ctx, int32_t scene, float damping);

/* Contact pairs (one FEM body against one ground), in the reference's launch
 * order within a body: planes, then height fields, then voxel grids, each in
 * contact-creation order.  gate_lo/gate_hi is the ground's getBBox() box used
 * by the broad-phase gate.  penalty is the float32 value of 2*K.
 * Replaces: _build_batched_contacts work lists and the per-substep launches of
 * _batched_analytical_contact_kernel / _batched_heightfield_contact_kernel /
 * _batched_voxelmap_contact_kernel, flatworld/mixedcontact.py:1794-1856,
 * 2131-2261, 660-684, 1566-1643. */
int fw_add_plane_pair(fw_ctx* ctx, int32_t body, float penalty, const float* gate_lo,
                      const float* gate_hi, float px, float py, float nx, float ny);
int fw_add_heightfield_pair(fw_ctx* ctx, int32_t body, float penalty, const float* gate_lo,
                            const float* gate_hi, int32_t n_samples, const float* heights,
                            float lb_x, float ub_x, int32_t reverse);
/* occupancy is nx*ny int32 in C order occ[i*ny + j] (VoxelGridDomain.occ). */
int fw_add_voxel_pair(fw_ctx* ctx, int32_t body, float penalty, const float* gate_lo,
                      const float* gate_hi, int32_t nx, int32_t ny, const int32_t* occupancy,
                      float lb_x, float lb_y, float dx, float dz);

/* FEM-FEM penalty contact (gather path; any number of scenes, each with its
 * own spatial hash).
 * fw_set_boundary_edges: every body's boundary edges (2 global node ids each,
 * in mesh order and orientation, mesh.py:53-71), stored body by body:
 * body b's at edges[2*body_off[b] ..], body_cnt[b] of them.  Replaces the
 * boundaryElements / domainBoundaryElemOffset packing, femspringmanager.py:783-799.
 * fw_set_flex_scene (once per scene that has FEM-FEM pairs): the loop's domains in loop order -- dom_obj[g] != 0 if
 * domain g takes part in the broad phase (considerContact), dom_body[g] its
 * body id (-1 for a ground), dom_box the ground's getBBox() (lo x, lo y, hi x,
 * hi y); skip_bvh != 0 when the loop has no plane, height-field, voxel or
 * unbatched ground contact (every FEM-FEM pair then stays active).  Replaces
 * the BVH set-up and domain stamps, explicitloop.py:203-227, 362-373, 495-514.
 * fw_add_flex_pair: one ContactFlexFlex (femcontact.py:199-206): body1 =
 * domain1, body2 = domain2, penalty = float32 of min(2 K1, 2 K2), friction =
 * max of the two domains'.  Work lists and the per-substep launch replace
 * mixedcontact.py:1869-1935 and _batched_flexflex_contact_kernel_sh,
 * mixedcontact.py:886-1018, with the spatial hash of spatialmanager.py.
 * fw_set_flex_clock: the substep dt as the host's float64 holds it, which the
 * hash-refresh clock accumulates (femspringmanager.py:1035-1039: rebuilt once
 * 1/500 s has accumulated); call it before fw_step whenever dt changes. */
int fw_set_boundary_edges(fw_ctx* ctx, int32_t n_edges, const int32_t* edges, const int32_t* body_off,
                          const int32_t* body_cnt);
int fw_set_flex_scene(fw_ctx* ctx, int32_t scene, int32_t skip_bvh, int32_t n_domains, const int32_t* dom_obj,
                      const int32_t* dom_body, const float* dom_box);
int fw_add_flex_pair(fw_ctx* ctx, int32_t body1, int32_t body2, float penalty, float friction);
/* Mark FEM-FEM pair `pair` (creation order of fw_add_flex_pair) tied, as
 * ExplicitLoop(ties=[(i, j)]) marks the contact of domains i and j
 * (flatworld/explicitloop.py:265-270, 400-439).  A tied pair's work items do
 * not run the contact search; at the scene's first substep each finds the
 * nearest boundary edge of the other body and from then on a penalty spring
 * holds its node at that point of the edge, with the reactions on the edge's
 * nodes (flatworld/mixedcontact.py:686-809, launched before the contact
 * kernel, mixedcontact.py:1680-1690).  Before fw_finalize. */
int fw_tie_flex_pair(fw_ctx* ctx, int32_t pair);
int fw_set_flex_clock(fw_ctx* ctx, double dt);
/* The same per scene (dt[scene], one entry per scene of the world; scenes
 * without FEM-FEM contact are ignored), for worlds whose scenes step with their
 * own dt (batched advanceWithTime).  After fw_finalize. */
int fw_set_flex_clocks(fw_ctx* ctx, const double* dt);
/* Spring-mass domains (SpringMassDomain, femspringmanager.py:815-870): the
 * listed bodies are spring-mass bodies whose nodes each carry node_mass (the
 * domain's prop[2]).  Their elements are 2-node springs given to
 * fw_set_elements as type 0 with the third node id -1, young = stiffness
 * (prop[0]), poisson = damping (prop[1]) and density = rest length; the
 * force is _spring_force_kernel's (femspringmanager.py:283-312), added after
 * the triangles' as the reference launches it.  Pass every node of a spring
 * body as its boundary nodes (its contact work items and box cover all of
 * them, mixedcontact.py:1822-1829).  Call after fw_set_bodies.  Gather path
 * only. */
int fw_set_spring_bodies(fw_ctx* ctx, int32_t n, const int32_t* bodies, const float* node_mass);

/* Selective mass scaling (ExplicitLoop(mass_scaling_dt=...)): every triangle
 * whose critical step 0.4 L_min / sqrt(E / rho) is below dt_target adds
 * (rho_new - rho) * area / 3 to each of its nodes, rho_new = E (dt_target /
 * (0.4 L_min))^2, node by node in ascending element order.  Call once, right
 * after fw_finalize, as the reference calls it right after setGlobalAABB.
 * Spring nodes are then raised to at least 4 k dt_target^2 (the kernel's second
 * loop).
 * Replaces applyMassScaling / _mass_scaling_kernel, femspringmanager.py:139-196,
 * explicitloop.py:168-170. */
int fw_mass_scaling(fw_ctx* ctx, float dt_target);

/* The work items' edge caches (boundary edge index hit last substep, or -1;
 * n_items must equal the world's count) and the spatial hash grid: tc, nx, ny,
 * origin x, origin y, cell x, cell y, element-box diagonal minimum.  The
 * reference keeps these in bc_flex_cache_elem and SpatialHashManager
 * (mixedcontact.py:1915, spatialmanager.py:538-551); here for tests. */
int fw_read_flex_state(fw_ctx* ctx, int32_t* item_cache, int32_t n_items, float* grid);

/* Rigid primitives touching FEM bodies (RigidBodyDomain with BallRigid /
 * BoxRigid / CapsuleRigid) and the rigid manager's analytical entries of
 * loops with a moving ground plane, before fw_finalize, gather path.  Per
 * entry 20 floats -- center x, y; primary x, y (box: full extents; capsule:
 * lower end minus center; analytical: the plane normal); radius; angle; mass;
 * inertia; velocity x, y; angular velocity; BC translation value x, y;
 * gravity x, y; BC rotation value; an analytical entry's first box lb x, y,
 * ub x, y -- and 4 ints: type (1 ball, 2 box, 8 capsule, 64 analytical), BC
 * bits (definitions.py:96-104), considerContact, scene; grouped by scene in
 * ascending order.
 * grounds: 6 floats per ground domain -- kind 0 (plane): point x, y, normal
 * x, y; kind 1 (height field, voxel grid): box lb x, y, ub x, y; then its
 * scene (grouped by scene too).  A rigid that comes within 0.01 of a
 * ground (20x the reference's rigid-ground contact margin) or of another
 * contact rigid's box at an update makes the next synchronising call return
 * FW_ERR_UNSUPPORTED.
 * Replaces RigidManager.processDomains_ / packRigidParams / processConditions
 * and precompute_rigid_transforms + updateBBox, rigidmanager.py:2448-2598,
 * 4001-4015, 4643-4662, explicitloop.py:198-201. */
int fw_set_rigids(fw_ctx* ctx, int32_t n, const float* params, const int32_t* ints, int32_t n_ground,
                  const float* grounds);
/* One FEM-rigid pair (ContactFlexRigid, femcontact.py:173-179): the body's
 * boundary nodes against the rigid, penalty 2K of the body, the rigid's
 * friction; skip_bvh: the loop activates the pair by plain box overlap
 * (mixedcontact.py:1697-1713, 474-492) instead of the broad phase; tied: a
 * pair named in ExplicitLoop(ties=...), which pulls each node to its contact
 * point without the 1e-4 offset or friction.  Add in the
 * reference's launch order: plane pairs, rigid pairs (contact order), height
 * field, voxel.  Replaces _build_batched_contacts' rigid work lists and
 * _batched_rigid_prim_kernel, mixedcontact.py:1963-2130, 1026-1115. */
int fw_add_rigid_pair(fw_ctx* ctx, int32_t body, int32_t rigid, float penalty, float friction, int32_t skip_bvh,
                      int32_t tied);
/* The last ground pair added (plane, height field, voxel) is gated by the
 * current box of analytical entry `entry` (fw_set_rigids) instead of its
 * static box: in a loop where some ground plane has BCs, every ground's
 * broad-phase box follows the rigid manager (rigidmanager.py:950-964), while
 * the contact itself keeps the plane of construction time
 * (mixedcontact.py:1815-1818). */
int fw_gate_by_rigid(fw_ctx* ctx, int32_t entry);
/* The rigid update schedule of the coming substeps: the rigids move every
 * `every` substeps by dt (the reference's N = max(1, 1e-3 // dt) and N * dt,
 * explicitloop.py:533-538, computed by the caller from its float64 dt), with
 * the loop's damping; every scene alike, or per scene (arrays of one entry per
 * scene of the world).  After fw_finalize. */
int fw_set_rigid_clock(fw_ctx* ctx, int32_t every, float dt, float damping);
int fw_set_rigid_clocks(fw_ctx* ctx, const int32_t* every, const float* dt, const float* damping);
/* Per rigid 12 floats: center x, y, angle, velocity x, y, angular velocity,
 * displacement x, y, box lb x, y, ub x, y; *flags (may be NULL): bit 0 set
 * once a rigid met a ground or another rigid.  The reference's
 * getCurrentRefPoint / getCurrentRefAngles / getCurrentVelocity / getBBox,
 * rigiddomain.py:128-155. */
int fw_read_rigids(fw_ctx* ctx, float* out, int32_t* flags);

/* Upload, precompute reference-shape data (area, Dm^-1, lumped mass, Lame
 * constants, node->element gather lists) and run the zero-dt step that the
 * reference runs at construction.
 * Replaces: prepareFEMData_ / _prepare_fem_data_kernel and setGlobalAABB ->
 * substep(0, 0), flatworld/femspringmanager.py:113-138, 872-897. */
int fw_finalize(fw_ctx* ctx);

/* Choose the step implementation before fw_finalize.  GATHER: per substep an
 * element kernel writes corner forces and a node kernel gathers them (any
 * number of scenes).  RESIDENT: the mesh is cut into `patches` patches (0 =
 * automatic, at most one per SM) that stay in shared memory while one
 * cooperative launch runs all substeps of an fw_step call (single-scene worlds
 * that fit on chip).  AUTO picks RESIDENT when possible.  Both paths give
 * identical results.  No reference counterpart: the reference has one Warp
 * path (flatworld/femspringmanager.py:941-1012). */
int fw_set_path(fw_ctx* ctx, int32_t path, int32_t patches);
/* Tuning options (fw_set_option), set before fw_finalize.
 * FW_OPT_FRONT_WARPS: warps of a resident CTA that run the cross-CTA critical
 * chain (2, 4, 6 or 8 of 16; default 6). */
#define FW_OPT_FRONT_WARPS 1
/* FW_OPT_BLOCK_ELEMS / FW_OPT_BLOCK_NODES: block size of the gather path's
 * element / node kernel (multiple of 32, <= 512; default 256).
 * FW_OPT_GRID_ELEMS: cap on the element kernel's grid (0 = 8 x SMs).
 * These three may also be changed after fw_finalize (used by the autotuner). */
#define FW_OPT_BLOCK_ELEMS 2
#define FW_OPT_BLOCK_NODES 3
#define FW_OPT_GRID_ELEMS 4
/* FW_OPT_RES_SYNC: how resident CTAs hand each substep's halo positions and
 * body boxes to each other: 0 = flag-in-data words (epoch-tagged 64-bit
 * values polled directly; used when the scene has at most 8 bodies, default),
 * 1 = arrival counter + release fence (any number of bodies).  Set before
 * fw_finalize.  Both give identical results. */
#define FW_OPT_RES_SYNC 5
/* FW_OPT_WAIT_LIMIT: polls a resident CTA makes before a cross-CTA wait gives
 * up (0 = built-in: 2^22 flag-in-data, 2^26 counter); then the launch ends
 * early and the next synchronising call returns FW_ERR_TIMEOUT.
 * FW_OPT_TEST_WITHHOLD: test hook -- resident CTA n withholds its first
 * publish, so the others' waits run out (-1 = off).  Both may be set at any
 * time; they apply from the next launch. */
#define FW_OPT_WAIT_LIMIT 6
#define FW_OPT_TEST_WITHHOLD 7
/* Stream path (FW_PATH_STREAM) launch shape:
 * FW_OPT_STREAM_PATCH: owned nodes per patch = threads per CTA, 64 (default)
 *   or 128; before fw_finalize (the patches are cut there).
 * FW_OPT_STREAM_MINB: CTAs per SM the kernel's registers are budgeted for
 *   (64-node patches: 32 (default), 24, 20 or 16; 128-node patches: 16
 *   (default), 12, 10 or 8; the intermediate budgets stage no records, so
 *   selecting one turns FW_OPT_STREAM_BULK off).
 * FW_OPT_STREAM_BULK: 1 stages each patch's triangle records into shared
 *   memory with one bulk copy instead of a load per triangle (default 0).
 * All give the same bits; the autotuner picks them. */
#define FW_OPT_STREAM_PATCH 8
#define FW_OPT_STREAM_MINB 9
#define FW_OPT_STREAM_BULK 10
/* FW_OPT_RES_THREADS: threads of a resident CTA, 512 (default; up to 128
 * registers per thread) or 1024 (32 warps, 64 registers); before
 * fw_finalize, and before FW_OPT_FRONT_WARPS, whose choices it sets: 2, 4,
 * 6 or 8 of 16 warps (default 6), or 8, 12 or 16 of 32 (default 12).  Same
 * bits. */
#define FW_OPT_RES_THREADS 11
int fw_set_option(fw_ctx* ctx, int32_t option, int32_t value);
/* The value an option has now.  Readable: FRONT_WARPS, RES_THREADS,
 * BLOCK_ELEMS, BLOCK_NODES, STREAM_PATCH, STREAM_MINB, STREAM_BULK, RES_SYNC;
 * FW_ERR_ARG for the others.  No reference counterpart (a tuning readout). */
int fw_get_option(const fw_ctx* ctx, int32_t option, int32_t* value);

/* Checkpoint / resume: copy the whole step state (positions, velocities, J2
 * state, step counters, body boxes) into snapshot `slot` (device memory owned
 * by the context, allocated on first use), or back.  Queued on the stream.
 * No reference counterpart: the reference's reset() leaves FEM state alone
 * (flatworld/explicitloop.py:635-679). */
int fw_snapshot(fw_ctx* ctx, int32_t slot);
int fw_restore(fw_ctx* ctx, int32_t slot);

/* Active path (FW_PATH_GATHER, FW_PATH_RESIDENT or FW_PATH_STREAM) and patch count. */
int fw_get_path(const fw_ctx* ctx, int32_t* path, int32_t* patches);

/* Advance every active scene by n_steps substeps of dt (float32), i.e. n_steps
 * calls of ExplicitLoop.advance(): gated contact, element force, integration,
 * body AABB.  Queued on the stream; returns without waiting.
 * Replaces: ExplicitLoop.advance / FemSpringManager.femStep,
 * flatworld/explicitloop.py:473-555, flatworld/femspringmanager.py:941-1012. */
int fw_step(fw_ctx* ctx, int32_t n_steps, float dt);

/* Like fw_step with a per-scene dt[] (float32, n_scenes entries) for the
 * batched and served forms, where each scene has its own step. */
int fw_step_scenes(fw_ctx* ctx, int32_t n_steps, const float* dt_per_scene);

/* One substep for a served world: scene s advances by dt[s] if dt[s] > 0 and
 * is frozen otherwise (dt has one entry per scene; for an arena world
 * max_scenes + 1).  Never waits for the device: the active set and the step
 * sizes are copied from staged host memory.  Replaces the per-body
 * ExplicitLoop.advance calls of a request loop (explicitloop.py:473-555). */
int fw_step_served(fw_ctx* ctx, const float* dt);

/* n_steps substeps of fw_step_served with the same dt[] (one copy of dt and
 * of the active set, then n_steps launches): a request loop calls it with
 * n_steps no larger than the substeps any in-flight request has left at its
 * current dt, so requests still leave the batch at the substep they finish. */
int fw_step_served_n(fw_ctx* ctx, const float* dt, int32_t n_steps);

/* Stream arenas: n_steps substeps of fw_step_served in which scene s (dt[s]
 * > 0) runs only its first budget[s] substeps at dt[s], then (when given)
 * budget_next[s] substeps at dt_next[s], and sits out the rest (its state
 * carried unchanged); every array has one entry per scene, dt_next and
 * budget_next both or neither.  A request loop passes each in-flight
 * request's remaining substeps, and the next run (the request's own
 * remainder, or the body's next queued request), so one call spans many
 * request ends and a body does not wait for the call to end to go on.  Same
 * bits as calls of fw_step_served_n that stop at each end. */
int fw_step_served_budget(fw_ctx* ctx, const float* dt, const int32_t* budget, const float* dt_next,
                          const int32_t* budget_next, int32_t n_steps);

/* Mark scenes active (1) / frozen (0).  Frozen scenes keep their state and do
 * not advance. */
int fw_set_active(fw_ctx* ctx, const int32_t* active);

/* Wait for all queued work of the context. */
int fw_synchronize(fw_ctx* ctx);

/* Read / write a node field for nodes [first, first+count).  X, V, X0: 2 floats
 * per node; MASS: 1 float.  on_device != 0 means dst/src is a device pointer.
 * Replaces: coords.numpy(), V.numpy(), mass.numpy(); FemDomain.getCurrentCoords,
 * flatworld/femdomain.py:47-50. */
int fw_read_nodes(fw_ctx* ctx, int32_t field, int32_t first, int32_t count, float* dst,
                  int32_t on_device);
int fw_write_nodes(fw_ctx* ctx, int32_t field, int32_t first, int32_t count, const float* src,
                   int32_t on_device);

/* Per-body boundary AABB after the last step: 4 floats per body
 * (lb.x, lb.y, ub.x, ub.y).  Replaces: _update_bbox_kernel output aabb[],
 * flatworld/femspringmanager.py:361-408; FemDomain.getBBox femdomain.py:23-29. */
int fw_read_aabb(fw_ctx* ctx, float* dst);

/* Per-element J2 state: eps_p (3 floats per element) and equivalent plastic
 * strain (1 float); zeros for non-J2 elements.  Replaces: plasticStrain /
 * eqPlasticStrain .numpy(), flatworld/femspringmanager.py:592-593. */
int fw_read_plastic(fw_ctx* ctx, float* eps_p, float* eqps);

/* Precomputed reference-shape data: area[e], jinv[4e] (row-major Dm^-1).
 * Replaces: elemVolume / J_inv .numpy(), femspringmanager.py:581-582. */
int fw_read_reference_shape(fw_ctx* ctx, float* area, float* jinv);

/* Per-scene step counters (number of advance() calls since finalize). */
int fw_read_counters(fw_ctx* ctx, int64_t* counters);

/* Non-finite detection: bad[s] = 1 once a node of scene s got a NaN/inf
 * position or velocity in a step (n_scenes entries; arena: max_scenes + 1).
 * The step sets the flag and carries on -- scenes never exchange forces, so a
 * broken scene cannot spoil the others; a request loop evicts it.  async = 1
 * only queues the copy (bad must then be pinned host memory, valid once the
 * stream reaches this point); async = 0 waits for it.  fw_clear_scene_status
 * clears scene s (s = -1: all).  The reference has no such check (it raises
 * only on buffer overflow, femspringmanager.py:708-730). */
int fw_scene_status(fw_ctx* ctx, int32_t* bad, int32_t async);
int fw_clear_scene_status(fw_ctx* ctx, int32_t scene);

/* CFL monitor: the stable time of the current (deformed) shape, reported
 * without changing dt.  The reference fixes dt once from the rest shape
 * (explicitloop.py:160-166, femdomain.py:24: 0.4 * L_min / sqrt(E / rho));
 * with the monitor on, the step that evaluates the triangles also evaluates
 * that bound on every triangle's current shortest edge and reduces it per
 * scene (warp shuffles; gather and stream steps: one atomic per warp and
 * scene; resident step: one per CTA and launch), so a caller can see a body's
 * bound shrink as it compresses.  fw_set_cfl_monitor(ctx, coef): coef[b] =
 * 0.4 / sqrt(E / rho) for body b (0 for spring domains); NULL turns it off.
 * Every step implementation.  fw_read_cfl(ctx, out, reset): out[s] = the
 * smallest bound of scene s over the substeps since the last reset (+inf if
 * none); reset = 1 starts a new window.  No reference counterpart. */
int fw_set_cfl_monitor(fw_ctx* ctx, const float* coef_per_body);
int fw_read_cfl(fw_ctx* ctx, float* out, int32_t reset);

/* Total energy per scene, reduced in FP64 on the device (deterministic order):
 * out[4 s + 0..3] = kinetic, strain, external potential (gravity -m g.x or
 * constant nodal force -f.x), contact penalty (1/2 k sd^2 of every
 * penetrating boundary node, ungated) of scene s (arena: scene slot).  Strain
 * energy densities: St-Venant-Kirchhoff lambda/2 tr(E)^2 + mu E:E (Elastic,
 * and J2 on E - eps_p); mu/2 (tr C - 2) - mu ln J + lambda/2 (ln J)^2
 * (NeoHookean).  Synchronises the stream.  No reference counterpart: the
 * reference computes no energies. */
int fw_energy(fw_ctx* ctx, double* out);

/* Number of kernel launches this context queued since creation (evidence
 * that the CUDA path ran; used by the benchmark's gpu_launches field). */
int64_t fw_launch_count(const fw_ctx* ctx);

/* Allocation-free substep for callers that must not allocate device memory
 * (a real-time loop where cudaMalloc may block and synchronise the device, or
 * a process whose device memory is handed out by its own pool allocator under
 * a fixed budget).  No counterpart in the reference: it has no C interface.
 * Advances n_steps substeps of the gather step without ground contact
 * (elastic / NeoHookean / J2 triangles, nodal boundary conditions, symplectic
 * Euler); identical arithmetic to fw_step on a world without contact pairs.
 * Every pointer is caller-owned DEVICE memory on the current device:
 *   x, v        [2*n_nodes]  positions / velocities, updated in place
 *   node_bc     [n_nodes]    OR of FW_BC_*;  bc_values [2*n_nodes];  mass [n_nodes]
 *   conn        [3*n_elems]  node ids;  jinv [4*n_elems] row-major Dm^-1
 *   elem_mat    [4*n_elems]  rest area, lambda, mu, material type (1, 2, 3 as float);
 *               a record of any other type (e.g. a spring, type 0) or with a
 *               node id outside [0, n_nodes) adds no force and is never read
 *               beyond its own fields
 *   j2_state    [4*n_elems]  eps_p (3) + eqps, updated; j2_param [2*n_elems]
 *               (yield stress, hardening).  Give both or neither (one NULL
 *               and the other not is FW_ERR_ARG).  With both NULL, J2
 *               triangles never yield: they respond with the elastic trial
 *               stress on zero plastic strain, and no state is stored.
 *   csr_off     [n_nodes+1], csr_slot [3*n_elems]  node -> (3*e + corner),
 *               ascending e within a node
 * The scratch (one float2 per corner) is a fixed array inside the library:
 * at most FW_NOALLOC_MAX_ELEMS triangles (3 MiB, held by every GPU that loads
 * the library); larger meshes are rejected with FW_ERR_ARG.  The first call on
 * a device looks the array's address up (cudaGetSymbolAddress) and caches it;
 * make that first call before any stream capture.  Calls after a
 * cudaDeviceReset of that device in the same process are not supported (the
 * cached address is not looked up again).  All calls share the array, so calls
 * that overlap on the GPU race.  A CUDA error pending before the call is
 * reported (FW_ERR_CUDA, left in place) and nothing is launched.  Work is
 * queued on `stream` (NULL: legacy default).
 * err/err_len: optional buffer for the error text. */
#define FW_NOALLOC_MAX_ELEMS 131072
int fw_step_noalloc(int32_t n_nodes, int32_t n_elems, int32_t n_steps, float dt, float damping,
                    float* x, float* v, const int32_t* node_bc, const float* bc_values,
                    const float* mass, const int32_t* conn, const float* jinv,
                    const float* elem_mat, float* j2_state, const float* j2_param,
                    const int32_t* csr_off, const int32_t* csr_slot, void* stream, char* err,
                    int32_t err_len);

/* Arena (served form).  fw_arena_init replaces the fw_set_* / fw_finalize
 * flow: it reserves device capacity once (nodes, triangles, bodies, scenes,
 * contact pairs, height samples, voxel cells).  With fw_set_path(ctx,
 * FW_PATH_STREAM, 0) (and FW_OPT_STREAM_PATCH) before fw_arena_init the arena
 * steps on the patch-streaming kernel: each committed scene also holds its
 * patch records, and a substep runs one CTA per patch of the active scenes
 * only; otherwise it steps on the gather kernels.  Both give the same bits.
 * Then, any number of times: stage ONE scene with fw_set_nodes /
 * fw_set_elements / fw_set_bodies (scene 0) / fw_set_scenes(1, ...) /
 * fw_add_*_pair using ids local to that scene, and fw_arena_commit copies it
 * into free ranges, precomputes its reference shape and schedules its zero-dt
 * construction step for the next substep (queued on the stream; the call does
 * not wait for the device); fw_arena_remove frees a scene's ranges (it waits
 * for the stream).  Steps touch only the active scenes' ranges.
 * fw_step_scenes then takes max_scenes + 1 dt values.  fw_arena_scene_info
 * fills info[8] = {first node, nodes, first triangle, triangles, first body,
 * bodies, free node capacity, free triangle capacity}.
 * No reference counterpart: each reference ExplicitLoop is built once
 * (flatworld/explicitloop.py:72-398). */
int fw_arena_init(fw_ctx* ctx, int64_t max_nodes, int64_t max_elems, int32_t max_bodies,
                  int32_t max_scenes, int32_t max_pairs, int64_t max_heights, int64_t max_occ);
int fw_arena_commit(fw_ctx* ctx, int32_t* scene_out);
int fw_arena_remove(fw_ctx* ctx, int32_t scene);

/* Split commit, so that a scene is prepared away from the thread that steps
 * the arena.  fw_arena_pack: the scene staged on `stage` (a context of its
 * own, never finalized, used by one thread at a time; the staging calls as
 * above) becomes a pack -- validation, corner lists, contact-pair order and,
 * for patch_nodes 64 or 128 (that of the arena it goes to; 0 for a gather
 * arena), its stream patches -- host work only; the stage is cleared.  With
 * flags & FW_PACK_PINNED the pack lives in page-locked memory, so the
 * commit's copies do not wait for the stream.  fw_arena_commit_pack uploads a
 * pack into an arena (queued on the arena's stream, ids relocated on the
 * device) and may be called again with the same pack to commit the scene
 * afresh.  fw_pack_info fills info[8] = {device bytes the scene occupies,
 * nodes, triangles, bodies, patch nodes, patches, patch triangles, pinned}.
 * fw_pack_destroy frees a pack; no commit from it may still be in flight
 * (synchronize the arena's stream first). */
#define FW_PACK_PINNED 1
int fw_arena_pack(fw_ctx* stage, int32_t patch_nodes, int32_t flags, fw_pack** out);
/* A staging context: holds staged scene data for fw_arena_pack and nothing
 * else (no device, no stream; fw_finalize and fw_arena_init refuse it).  Works
 * without a GPU.  Free it with fw_destroy. */
int fw_create_stage(fw_ctx** out);
int fw_arena_commit_pack(fw_ctx* ctx, const fw_pack* pack, int32_t* scene_out);
int fw_pack_info(const fw_pack* pack, int64_t* info);
void fw_pack_destroy(fw_pack* pack);
int fw_arena_scene_info(fw_ctx* ctx, int32_t scene, int64_t* info);

/* Differentiable form.  fw_set_element_young: new per-element Young's moduli
 * for elements [first, first+count) (Lame constants recomputed; either step path).
 * The reference stores E per element (femspringmanager.py:584, 753) but has no
 * setter or adjoint.  Reverse pass of a rollout of dt-substeps:
 *   fw_adj_begin(ctx, K)      adjoint buffers for segments of up to K substeps
 *   fw_adj_seed(ctx, xb, vb)  adjoint of the final positions / velocities
 *                             (NULL = zero); clears dL/dE
 *   fw_adj_segment(ctx, n, dt) from the current state (restore the segment's
 *                             checkpoint first with fw_restore) recompute n
 *                             substeps, then run them backward
 *   fw_adj_read(ctx, xb, vb, Eb) dL/dx, dL/dv at the segment start; dL/dE
 * Covers Elastic, NeoHookean and J2 triangles (the plastic state carried
 * backward), plane, height-field and voxel contact (penalty and velocity
 * damping), gravity / nodal force / fixed / enforced-velocity / enforced-
 * acceleration BCs; refuses FEM-FEM contact, spring-mass domains, rigid bodies,
 * worlds of several scenes, arenas and the stream path. */
int fw_set_element_young(fw_ctx* ctx, int32_t first, int32_t count, const float* young,
                         int32_t on_device);
int fw_adj_begin(fw_ctx* ctx, int32_t max_segment_steps);
int fw_adj_seed(fw_ctx* ctx, const float* xbar, const float* vbar, int32_t on_device);
int fw_adj_segment(fw_ctx* ctx, int32_t n_steps, float dt);
int fw_adj_read(fw_ctx* ctx, float* xbar, float* vbar, float* Ebar, int32_t on_device);

/* Forward-mode derivative (tangent) of a rollout along (dx0, dv0, dE), carried
 * with the substeps themselves on the same trajectory and gates as the
 * adjoint; no reference counterpart.
 *   fw_tan_begin(ctx, dx0, dv0, dE)  tangent of the current state (NULL = 0)
 *   fw_tan_step(ctx, n, dt)          n substeps of dt, state and tangent
 *   fw_tan_read(ctx, dx, dv)         tangent of positions and velocities
 * <w, dx_T> equals the adjoint's <dL/dE, dE> + <dL/dv0, dv0> + <dL/dx0, dx0>
 * for L = <w, x_T> up to rounding (the dot-product test of the adjoint).
 * Same scope as the adjoint. */
int fw_tan_begin(fw_ctx* ctx, const float* dx0, const float* dv0, const float* dE, int32_t on_device);
int fw_tan_step(fw_ctx* ctx, int32_t n_steps, float dt);
int fw_tan_read(fw_ctx* ctx, float* dx, float* dv, int32_t on_device);

/* Library build identification string (arch, flags). */
const char* fw_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* FWB200_H */
