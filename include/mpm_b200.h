/*
 * mpm_b200.h -- C ABI of the B200-native MLS-MPM substep library
 * (libmpm_b200.so).  Plain pointers and sizes only; no CUDA or framework
 * types cross this boundary.
 *
 * Each entry point backs one device-touching member of the reference's GPU
 * solver interface `MpmMlsGpuSolver` (7korobi/powder-play,
 * src/lib/mpm/kernels/solver.ts:106-144).  Host-side policy that the
 * reference keeps in TypeScript (input validation and packing,
 * src/lib/mpm/kernels/layout.ts; CFL planning, cfl.ts / cfl-bounds.ts /
 * step-scheduler.ts; the adaptive retry loop, solver.ts:1724-2021) stays in
 * the host language above this ABI.
 *
 * Wire format: a particle is the reference's packed 20-word record
 * (src/lib/mpm/kernels/layout.ts:385-437): words 0-1 position, 2-3 velocity,
 * 4-7 C (m00,m01,m10,m11), 8-11 F, 12 plastic volume, 13 model code (u32),
 * 14 lambda, 15 mu, 16 density, 17 volume, 18 material parameter (Tait
 * exponent / powder friction / Neo-Hookean damage), 19 bonded-vertex marker
 * (u32, 0 = none, 1..3 = vertex 0..2).
 *
 * Status: the 8-word numerical status of the reference
 * (src/lib/mpm/kernels/shaders.ts:157-172, decoded by solver.ts:232-284):
 * [0] flag bits, [1] particle index (0xffffffff = none), [2..5] f32
 * diagnostics, [6] diagnostic claim (1 deformation, 2 projected F, 3 CFL),
 * [7] surface flags.
 *
 * Threading: a handle is not thread-safe.  Calls are ordered on the handle's
 * CUDA stream; only the read* and queue-completion calls block.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_OK 0
#define MPM_ERR_INVALID_ARGUMENT (-1) /* reference RangeError / TypeError class */
#define MPM_ERR_CUDA (-2)             /* device allocation, launch or copy failed */
#define MPM_ERR_STATE (-3)            /* call not valid in the handle's state */

#define MPM_P2G_GATHER 0u      /* createMpmMlsGpuSolver (solver.ts:390-397) */
#define MPM_P2G_FIXED_POINT 1u /* createExperimentalMpmMlsAtomicGpuSolver (solver.ts:399-406) */

#define MPM_PARTICLE_WORDS 20u
#define MPM_STATUS_WORDS 8u
#define MPM_FRACTURE_BOND_WORDS 6u

typedef struct mpm_solver mpm_solver;

/* The validated configuration (MpmMlsGpuConfig, layout.ts:17-19) as the
 * float32 values that the reference packs into SimulationParams
 * (layout.ts:950-996). */
typedef struct mpm_config {
    uint32_t cells_x;
    uint32_t cells_y;
    float cell_size;
    float particle_mass;
    float particle_volume;
    float bond_rest_length;   /* 0 when absent */
    float bond_stiffness;     /* default 0.35 */
    float bond_reference_dt;  /* 0 when absent: each batch supplies it */
    float wall_friction;
    float lambda;             /* config material, as packed in SimulationParams */
    float mu;
    uint32_t capacity;        /* >= initial particle count */
    uint32_t p2g_mode;        /* MPM_P2G_GATHER or MPM_P2G_FIXED_POINT */
    uint32_t fixed_point_shift; /* fixed-point scale 2^shift; 24 = reference */
    int32_t device;           /* CUDA device ordinal */
} mpm_config;

/* CFL guard of one batch: cflBounds.x/y of SimulationParams. */
typedef struct mpm_cfl_guard {
    float wave_speed_bound;
    float velocity_limit;
} mpm_cfl_guard;

/* Interaction drag of finishGridVelocity (shaders.ts:1748-1777). */
typedef struct mpm_drag {
    float target_x, target_y, radius, stiffness, damping;
} mpm_drag;

/* Replaces createMpmMlsGpuSolver / createExperimentalMpmMlsAtomicGpuSolver
 * (solver.ts:390-406 -> createGpuSolver :408-469, createRuntime :605-1230)
 * minus the canvas: uploads validated, packed input.  `body_starts` are the
 * bonded-triangle body starts (layout.ts:457-493); `fracture_bonds` are
 * packed 6-word bonds (layout.ts:508-545) and `fracture_topology` the CSR
 * incidence (layout.ts:546-564). */
int mpm_create(const mpm_config *config, const float *packed_particles, const uint32_t *object_ids,
               uint32_t particle_count, const uint32_t *body_starts, uint32_t body_count,
               const uint32_t *fracture_bonds, uint32_t fracture_bond_count,
               const uint32_t *fracture_topology, uint32_t fracture_topology_words, mpm_solver **out);

/* Encodes `step_count` full substeps of `dt` in one graph launch:
 * stepBatch (solver.ts:1407-1599).  `guard` non-NULL = CFL batch
 * (stepCflBatch, solver.ts:1601-1722, after host-side plan certification):
 * the committed-microstep counter is reset, per-particle CFL validation
 * runs, and the batch ends with the maximum-speed reduction.
 * `bond_reference_dt` <= 0 uses the configured value, else dt. */
int mpm_step_batch(mpm_solver *solver, uint32_t step_count, float dt, float gravity_x, float gravity_y,
                   const mpm_cfl_guard *guard, float bond_reference_dt);

/* measureMaximumParticleSpeed (solver.ts:2388-2512): the 40-byte compact
 * readback of maximum speed, committed microsteps and status.  Blocks. */
int mpm_read_compact(mpm_solver *solver, float *maximum_speed, uint32_t *completed_microsteps,
                     uint32_t status[8]);

/* checkNumericalStatus (solver.ts:2514-2570).  Blocks. */
int mpm_read_status(mpm_solver *solver, uint32_t status[8]);

/* Clears the persistent status before an adaptive retry
 * (solver.ts:1878-1882, :1933-1937). */
int mpm_clear_status(mpm_solver *solver);

/* readParticles (solver.ts:2594-): packed 20-word records and object ids of
 * the requested particles (all when indices == NULL).  Blocks. */
int mpm_read_particles(mpm_solver *solver, const uint32_t *indices, uint32_t count, float *packed_out,
                       uint32_t *object_ids_out);

/* Overwrites the particle state from packed records (the upload of
 * createRuntime, solver.ts:724-): count must equal the particle count. */
int mpm_write_particles(mpm_solver *solver, const float *packed_particles, uint32_t count);

/* Interaction drag (beginDrag/updateDrag/endDrag, solver.ts:2700-2790);
 * drag == NULL ends the drag. */
int mpm_set_drag(mpm_solver *solver, const mpm_drag *drag);

/* measureQueueCompletionMs (solver.ts:106-144): milliseconds until the
 * handle's queued work completes.  Blocks. */
int mpm_queue_completion_ms(mpm_solver *solver, double *milliseconds);

/* particleCount / particleCapacity (solver.ts:108-110); allocatedParticleCount
 * (:109): original indices handed out, particles removed by an outlet
 * included. */
uint32_t mpm_particle_count(const mpm_solver *solver);
uint32_t mpm_particle_capacity(const mpm_solver *solver);
uint32_t mpm_allocated_particle_count(const mpm_solver *solver);

/* ---- interaction (single-scene solvers) ---- */

/* appendParticles (solver.ts:2108-2278): `count` validated packed particles
 * (no bonded-triangle markers) become original indices
 * allocated .. allocated + count - 1 (*first_index = the first) under their
 * object ids.  The caller applies the reference's refusal rules (pending
 * readbacks, capacity split into accepted / dropped) before calling. */
int mpm_append_particles(mpm_solver *solver, const float *packed_particles, const uint32_t *object_ids,
                         uint32_t count, uint32_t *first_index);

/* removeParticlesInOutlet (solver.ts:2280-2386, shaders.ts:3041-3065): water
 * and oil particles inside the bounds leave the simulation; their original
 * indices stay allocated and read back with material model 0xffffffff and
 * their last state.  Blocks. */
int mpm_remove_particles_in_outlet(mpm_solver *solver, float min_x, float min_y, float max_x, float max_y,
                                   uint32_t *removed_count);

/* pick (solver.ts:2733-2815, shaders.ts:3082-3116): the active particle
 * nearest to (x, y) within `radius` (lowest index among equally near ones):
 * its original index (0xffffffff: none), position and object id.  Blocks. */
int mpm_pick(mpm_solver *solver, float x, float y, float radius, uint32_t *particle_index, float *anchor_xy,
             uint32_t *object_id);

/* clone (solver.ts:2852-2940, shaders.ts:3118-3147): the particles with
 * original indices start .. start + count - 1 (an object's range) are copied
 * as new original indices (*first_index = the first), moved by the offset
 * and clamped to the domain, under `object_id`.  Refused (MPM_ERR_STATE)
 * after an outlet removal and in scenes with bonded bodies or fracture
 * bonds. */
int mpm_clone_range(mpm_solver *solver, uint32_t start, uint32_t count, float offset_x, float offset_y,
                    uint32_t object_id, uint32_t *first_index);

/* The water/oil free-surface field of render('surface') without the
 * renderer (solver.ts:2043-2066: clearSurfaceOccupancy, buildBuckets,
 * gatherSurfaceOccupancy; shaders.ts:700-806): per halo node, row-major
 * (node_w x node_h, node (x, y) at (y + 1) * node_w + x + 1), the water and
 * oil display area 2 V det(F) w / cellSize^2 of the liquid particles of the
 * current state.  The sums are 64-bit fixed point (2^40 per unit), so the
 * field is bit-identical from run to run.  field_out (2 floats per node)
 * and surface_flags_out (status word 7: 1 bucket / stencil, 2 particle
 * area, 4 accumulation; decodeSurfaceError, solver.ts:208-224, 286-294) may
 * be NULL.  Nothing is gathered (the field is zero) while a numerical status
 * or surface flag is pending.  Single-scene solvers.  Blocks. */
int mpm_gather_surface_occupancy(mpm_solver *solver, float *field_out, uint32_t *surface_flags_out);

/* The device buffer of the last gathered surface field (2 floats per halo
 * node, owned by the solver, valid until the next gather or mpm_destroy),
 * for consumers that read it on the GPU; node_w / node_h may be NULL. */
int mpm_surface_field_device(mpm_solver *solver, const float **device_field, uint32_t *node_w, uint32_t *node_h);

/* dispose (solver.ts:143). */
void mpm_destroy(mpm_solver *solver);

/* Message of the last failing call on this thread ("" if none). */
const char *mpm_last_error(void);

/* ---- parity probes (no reference counterpart; used by the parity tests) ---- */

/* Runs the cell sort of the next substep on the current state and returns,
 * per particle, its base-cell key, the sorted permutation (slot -> particle)
 * and cell starts (node_count + 1 words).  Does not advance the state. */
int mpm_probe_sort(mpm_solver *solver, float dt, uint32_t *keys_out, uint32_t *perm_out,
                   uint32_t *cell_start_out);

/* Runs the fixed-point scatter of the next substep on the current state and
 * returns the 11 integer words per halo node and each particle's prepared
 * affine momentum (4 floats).  Does not advance the state. */
int mpm_probe_fixed_point(mpm_solver *solver, float dt, int32_t *words_out, float *affine_out);

/* Builds the bonded-triangle field of the current particles
 * (buildTriangleField, src/lib/mpm/kernels/shaders.ts:1299-1436) and copies
 * it out: 8 words per halo node, row-major (cellsX+3) x (cellsY+3): signed
 * distance f32, first-vertex index + 1 u32 (0: none), normal 2 x f32,
 * barycentric weights of the second and third vertex 2 x f32, impulse 2 x f32
 * (zero).  MPM_ERR_STATE when the scene has no bodies.  No reference
 * counterpart: the reference keeps this buffer internal. */
int mpm_probe_triangle_field(mpm_solver *solver, float dt, float *field_out);

/* Evaluates G2P's deformation-gradient trial on `device` for `count` (F, C)
 * pairs (4 floats each, row-major m00 m01 m10 m11) at step `dt`: the
 * increment dt * max row sum |C|, the substep count n = ceil(increment /
 * 0.25) doubled while det <= 0 (at most 64), the trial F of n fused products
 * and its compensated determinant; `flags_out` holds 0, or 32 (more than 64
 * substeps) / 16 (a non-finite product).  The same device function G2P runs
 * (integrateDeformation and its retries, src/lib/mpm/kernels/shaders.ts:1459-1483,
 * :2249-2298); the reference pins it with the float32 known answer of
 * src/lib/mpm/kernels/solver.spec.ts:197-278. */
int mpm_probe_deformation(int device, const float *F, const float *C, uint32_t count, float dt, float *trial_out,
                          float *increment_out, float *determinant_out, uint32_t *substeps_out, uint32_t *flags_out);

/* Halo node count ((cells_x + 3) * (cells_y + 3)). */
uint32_t mpm_node_count(const mpm_solver *solver);

/* ---- measurement (no reference counterpart; the reference times batches
 * with WebGPU timestamp queries, src/lib/mpm/experiments/si-performance.ts:131-196) ---- */

/* Device time of the last mpm_step_batch, from CUDA events recorded on the
 * handle's stream around it.  Blocks until that batch completes. */
int mpm_last_batch_device_ms(mpm_solver *solver, double *milliseconds);

/* Runs `step_count` real substeps without a graph, with an event after every
 * kernel, and returns per kernel slot the summed milliseconds and launch
 * counts (arrays of mpm_profile_kernel_slots() entries). */
int mpm_profile_substeps(mpm_solver *solver, uint32_t step_count, float dt, float gravity_x, float gravity_y,
                         const mpm_cfl_guard *guard, double *kernel_ms, uint32_t *kernel_launches);
const char *mpm_profile_kernel_name(uint32_t slot);
uint32_t mpm_profile_kernel_slots(void);

/* Launch shape of the default path: the persistent grids (CTAs) of its P2G
 * and G2P kernels; 0 keeps a value.  Results do not depend on it (every sum
 * has a fixed order). */
int mpm_set_launch_shape(mpm_solver *solver, uint32_t p2g_ctas, uint32_t g2p_ctas);
int mpm_get_launch_shape(mpm_solver *solver, uint32_t *p2g_ctas, uint32_t *g2p_ctas, uint32_t *sm_count);

/* The autotuner: times `substeps` real substeps of the last submit's
 * parameters (the whole graph, device time) for each candidate variant and
 * keeps the fastest: for each P2G stage capacity (640, 384), the one-launch
 * substep over persistent grids of 1 .. co-resident CTAs per SM, and the
 * four-launch substep over its P2G grids, then its G2P grids with the best
 * P2G, then both ways of handing prepareParticle's results to P2G.  Restores the particle state and counters it started from.  Returns
 * the chosen four-launch grids (mpm_get_substep_variant gives the rest) and
 * the best milliseconds per substep.  Needs one submitted batch.  Blocks. */
int mpm_autotune(mpm_solver *solver, uint32_t substeps, uint32_t *p2g_ctas, uint32_t *g2p_ctas, double *best_ms);

/* The default path's substep variant (no counterpart in the reference,
 * whose substep is a sequence of WebGPU compute passes).  `fused` 1 runs each
 * substep as ONE cooperative launch of persistent CTAs (tile allocation,
 * bucketing, P2G, grid update + G2P, with grid barriers between them), 0 as
 * four launches; `stage_capacity` is the P2G stage (640 or 384 particles;
 * 0 keeps it); `substep_ctas` the one-launch form's persistent grid (0 keeps
 * it; at most the CTAs that fit on the GPU at once); `liquid_kernels` 1 lets
 * G2P run its instantiation compiled for water and oil only whenever every
 * material of the solver is one of them (the default), 0 keeps the general
 * one; `p2g_records` 1 has G2P write each particle's prepared P2G record
 * (prepareParticle, evaluated where G2P has F and C in registers) for the
 * next P2G, 0 has P2G prepare each particle from its state, 2 picks by the
 * materials (records unless every material is a liquid with the linear EOS;
 * the one-launch form always prepares in P2G).  Solvers with bonded bodies or
 * fracture bonds always take four launches and the general G2P.  Results do
 * not depend on `fused`, the grids, `liquid_kernels` or `p2g_records` (the
 * same arithmetic); the stage capacity changes only the rounding of tiles
 * holding more particles than it.  mpm_get_substep_variant reports whether
 * substeps run as one launch, the capacity, the grid, its co-resident limit,
 * whether the water-and-oil G2P runs and whether records are used. */
int mpm_set_substep_variant(mpm_solver *solver, uint32_t fused, uint32_t stage_capacity, uint32_t substep_ctas,
                            uint32_t liquid_kernels, uint32_t p2g_records);
int mpm_get_substep_variant(mpm_solver *solver, uint32_t *fused, uint32_t *stage_capacity, uint32_t *substep_ctas,
                            uint32_t *max_substep_ctas, uint32_t *liquid_kernels, uint32_t *p2g_records);

/* The one-launch substep's grid-barrier waits give up after `limit_ns`
 * nanoseconds (default 1 s; 1 us .. 60 s): the CTA that gave up raises status
 * flag 1 << 20 in every scene, the others leave at their next barrier, and the
 * batch's particle state is undefined (write the particles again).
 * `skip_cta` below the grid makes that CTA leave before the first barrier
 * without arriving, so that the others' waits run out: a test of the limit
 * (0xffffffff: none).  No counterpart in the reference. */
int mpm_set_barrier_limit(mpm_solver *solver, uint64_t limit_ns, uint32_t skip_cta);

/* Nodes of the last substep with positive solid / water / oil mass. */
int mpm_count_active_nodes(mpm_solver *solver, uint32_t counts[3]);

/* The handle's CUDA stream (cudaStream_t), for callers that order their own
 * work after the solver's. */
void *mpm_stream(mpm_solver *solver);

/* ---- batched scenes ---- */

/* No counterpart in the reference, which runs one scene per solver
 * (createMpmMlsGpuSolver, src/lib/mpm/kernels/solver.ts:390-406): one handle
 * over `scene_count` independent scenes of uneven particle counts and grids,
 * stepped together (one launch per kernel and substep, every scene's tiles in
 * one tile list).  Scene k holds particle_counts[k] particles, packed one
 * scene after another in packed_particles / object_ids (20 words each, as
 * mpm_create); configs[k] gives its grid and material constants (its
 * capacity is ignored: a scene holds exactly its particles).  Every scene
 * runs the default gather P2G; the device comes from configs[0].  No bonded
 * bodies or fracture bonds.  mpm_read_particles reads all scenes' particles
 * in this packed order; mpm_clear_status clears every scene. */
int mpmb_create(const mpm_config *configs, uint32_t scene_count, const uint32_t *particle_counts,
                const float *packed_particles, const uint32_t *object_ids, mpm_solver **out);

/* One submit of per-scene step batches (stepBatch, src/lib/mpm/kernels/
 * solver.ts:1407-1498, for every scene at once): scene k runs step_counts[k]
 * substeps of dts[k] (0: the scene sits the submit out) under gravity
 * (gravity_xy[2k], gravity_xy[2k+1]) and, when `guards` is not NULL, the CFL
 * guard guards[k].  A scene whose status is raised stops there, its state
 * rolled back to the start of the failed substep; the others go on. */
int mpmb_step_batch(mpm_solver *solver, const uint32_t *step_counts, const float *dts, const float *gravity_xy,
                    const mpm_cfl_guard *guards);

/* mpm_read_compact for every scene: maximum_speeds[k], completed[k] and the
 * 8 status words status[8k .. 8k+7], whose particle index (word 1) counts
 * within the scene (any output may be NULL).  Blocks. */
int mpmb_read_compact(mpm_solver *solver, float *maximum_speeds, uint32_t *completed_microsteps, uint32_t *status);

/* Scenes of the handle (1 for a handle from mpm_create). */
uint32_t mpmb_scene_count(const mpm_solver *solver);

/* ---- differentiable form (adjoint) ---- */

/* No counterpart in the reference, which has no gradients.  An engine over a
 * batch of scenes of Tait water (model 2 with a Tait exponent) and
 * fixed-corotated solid (model 5) particles, stepped with the default path's
 * arithmetic for those models on dense per-scene grids at a fixed dt per
 * scene, with the loss sum over particles of |x(T) - target|^2 per scene and
 * its adjoint by checkpoint and recompute.  Particles come as the 20-word
 * records of mpm_create, scene after scene; a scene's water particles share
 * one material, as do its solid particles.  The differentiated parameters,
 * 3 per scene: the water's Tait pressure coefficient (word 14 of a water
 * record), the solid's lambda and mu (words 14 and 15 of a solid record).
 * gravity_xy: 2 per scene. */
typedef struct mpm_adjoint mpm_adjoint;
int mpma_create(const mpm_config *configs, uint32_t scene_count, const uint32_t *particle_counts,
                const float *packed_particles, const float *gravity_xy, mpm_adjoint **out);

/* Replaces / reads the parameters (3 per scene, in the order above). */
int mpma_set_parameters(mpm_adjoint *engine, const float *parameters);
int mpma_get_parameters(mpm_adjoint *engine, float *parameters);

/* Replaces the initial velocities (2 per particle). */
int mpma_set_velocities(mpm_adjoint *engine, const float *velocities);

/* Runs `substeps` substeps of dts[k] in scene k from the initial state,
 * keeping the state at every `checkpoint_every`-th substep, and returns the
 * loss per scene against `targets` (2 per particle).  With
 * checkpoint_every >= substeps the pass keeps every substep's state and node
 * sums (48 B per particle and 32 B per node, per substep) and
 * mpma_backward recomputes nothing.  Blocks. */
int mpma_forward(mpm_adjoint *engine, uint32_t substeps, const float *dts, uint32_t checkpoint_every,
                 const float *targets, double *loss);

/* The gradients of the last forward pass's total loss with respect to the
 * initial velocities (2 per particle) and the parameters (3 per scene): each
 * segment of checkpoint_every substeps is recomputed from its checkpoint and
 * then reversed substep by substep.  Either output may be NULL.  Blocks. */
int mpma_backward(mpm_adjoint *engine, float *grad_velocities, double *grad_parameters);

/* Final positions of the last forward pass (2 per particle). */
int mpma_read_positions(mpm_adjoint *engine, float *positions);

/* Device milliseconds of the last forward and backward passes. */
int mpma_last_ms(mpm_adjoint *engine, double *forward_ms, double *backward_ms);

void mpma_destroy(mpm_adjoint *engine);

/* ---- allocation-free cell sort ---- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host whose GPU memory belongs to an embedding application with a fixed
 * budget, a frame loop that must not take an allocation's implicit device
 * synchronisation, a foreign-function host with no allocator of its own):
 * the stable counting sort of particles by base cell that the gather path
 * runs (same keys, permutation and cell starts as mpm_probe_sort), with all
 * device scratch in one static array built into the library (about 3.5 MiB
 * held by every GPU that loads it, until exit).  `positions` are `count`
 * (x, y) float pairs in host memory; outputs are host arrays of `count`,
 * `count` and (cells_x+3)*(cells_y+3)+1 words.  Limits: count <= 65536 and
 * (cells_x+3)*(cells_y+3) <= 262144, else MPM_ERR_INVALID_ARGUMENT with the
 * reason written to `error_out` (may be NULL).  The first call on a device
 * resolves the array's address and keeps it (make that call before any stream
 * capture; after a cudaDeviceReset of that device the kept address is stale,
 * so do not call it there again); calls share the array, so calls that
 * overlap on one GPU race.  The caller's current device is restored on
 * return.  Blocks until done. */
int mpm_cell_sort_static(int32_t device, uint32_t cells_x, uint32_t cells_y, float cell_size,
                         const float *positions, uint32_t count, uint32_t *keys_out, uint32_t *perm_out,
                         uint32_t *cell_start_out, char *error_out, uint32_t error_capacity);

#ifdef __cplusplus
}
#endif
#endif
