// mpm_kernels.cuh -- kernel entry points of one MLS-MPM substep on B200.
//
// Data layout in HBM (all per-particle arrays are SoA, 16-byte aligned):
//   particle state, ping-pong A/B, indexed by slot: pos float2, vel float2,
//     C float4, F float4, plastic volume float, damage float, volume float,
//     material index u32, original index u32.  In the gather path the slots
//     are kept sorted by base cell: G2P of substep k reads slot perm[d] and
//     writes slot d, so every particle kernel reads and writes coalesced.
//   per original particle (constant): object id u32, bonded-vertex marker u32
//   with the records variant, P2G records per slot: float4 (fx, fy, mass,
//     liquid volume), float4 affine momentum, float2 m v, u32 local cell |
//     channel
//   tile buckets: key u32 (tile | local cell << 24) and rank u32 per slot, permutation u32
//     (bucketed position -> slot), per-tile count/start u32; the cell sort of
//     the probes adds per-cell count/start u32 and a bucket scratch u32
//   halo grid, (cellsX+3) x (cellsY+3) nodes, row-major by (y+1)*W + (x+1),
//     cut into 16x8-node tiles: per tile the f32 P2G sums of its particles
//     over its 18x10-node ring (11 words, word-major) with a (stamp, channel
//     mask) pair, and the list of tiles holding particles; updated velocities solid
//     float2, water float4 (vx,vy,mass_l,vol_l), oil float4 -- exactly what
//     G2P reads per channel.  The reference-exact fixed-point path adds 11
//     i32 words per node, its decoded sums 3 x float4, and one stamp u32 per
//     tile (tiles touched this substep).
#pragma once

#include "mpm_device.cuh"

namespace mpm {

struct ParticleBuffers {
    float2 *pos;
    float2 *vel;
    float4 *C;
    float4 *F;
    float *pvol;
    float *damage;
    float *vol;
    uint32_t *mat;
    uint32_t *orig;
};

// Nearest bonded-triangle (pebble) sample of one halo node
// (TriangleFieldNode, src/lib/mpm/kernels/shaders.ts; 32 B).
struct TriField {
    float sd;        // signed distance, the band when no body is near
    uint32_t body1;  // original index of the body's first vertex + 1 (0: none)
    float nx, ny;    // outward normal
    float b1, b2;    // barycentric weights of the second and third vertex
    float ix, iy;    // impulse the fluid put on the body at this node
};

struct Ctx {
    const StepParams *P;  // the scene's parameters (scene 0 outside the scene-aware kernels)
    // a batch of scenes: per scene its parameters and SCENE_WORDS words of
    // status [0, 32) and counters [32, 64); shared work counters; the scene of
    // each tile; the first slot of each scene (n_scenes + 1 entries)
    const StepParams *scenes;
    uint32_t *dyn;
    uint32_t *work;
    const uint32_t *tile_scene;
    const uint32_t *scene_p_base;
    uint32_t n_scenes;
    uint32_t parity;   // the buffer `in` reads (0 / 1): picks the substep's tile list
    uint32_t n;        // particle count of all scenes
    uint32_t n_tiles;  // 16x8-node tiles of all scenes' halo grids (with one sentinel each)
    ParticleBuffers in;
    ParticleBuffers out;
    const Material *mats;
    const uint32_t *bonded;  // by original index
    const uint32_t *obj;     // by original index
    uint32_t *status;    // the scene's status words
    uint32_t *counters;  // the scene's counters
    // cell sort
    uint32_t *keys;
    uint32_t *ranks;
    uint32_t *tmp;
    uint32_t *perm;  // sorted position -> slot (NULL: identity, fixed-point path)
    uint32_t *cell_count;
    uint32_t *cell_start;
    uint32_t *block_sums;
    uint32_t cell_pad;  // padded length of cell_count (multiple of SCAN_CHUNK)
    uint32_t count_next;  // G2P also counts the next substep's tiles
    // tile buckets and the per-tile partial node sums of the default P2G
    uint32_t *tile_count;
    uint2 *tile_range;       // per tile listed this substep: first bucket entry, particles
    uint32_t *active_tiles;  // tiles holding particles this substep
    const uint32_t *scene_chunk;  // per scene: its first CTA of k_tile_alloc, then the CTA total
    float *part;             // per tile: ACC_WORDS x RING_NODES sums, word-major
    uint2 *tile_info;        // per tile: (substep stamp of the sums, channel mask)
    // the records variant: P2G records of the particles in the input slots,
    // written by the batch prologue and by each G2P for the next substep
    // (NULL: P2G prepares each particle from its state)
    float4 *rec_state;   // fx, fy, mass, liquid volume (failed: flags, indexed)
    float4 *rec_affine;  // A = m C + (-dt V 4/dx^2) P F^T
    float2 *rec_mom;     // m v
    uint32_t *rec_cell;  // local cell in its tile | channel << 8 | REC_FAILED
    // grid
    float4 *p2g_solid;
    float4 *p2g_water;
    float4 *p2g_oil;
    float2 *g_solid;
    float4 *g_water;
    float4 *g_oil;
    int32_t *fixed;
    uint32_t *tile_stamp;
    float4 *affine_out;  // optional: prepared affine per slot (parity checks)
    // bonded-triangle bodies and fracture bonds (NULL / 0 when the scene has none)
    TriField *field;              // per halo node
    const uint32_t *body_starts;  // per body: original index of its first vertex
    uint32_t *slot_in, *slot_out; // current slot of each tracked original index (input / output buffer)
    const uint32_t *track_flag;   // per original index: 1 when its slot is tracked
    const uint32_t *tracked;      // tracked original indices
    uint32_t n_tracked;
    float4 *pair_cache;           // per ordered body pair (a < b): contact normal, penetration
    uint32_t *contact_count;      // per body
    float2 *body_vel;             // per body: mean vertex velocity
    uint32_t *bonds;              // 6 words per fracture bond
    const uint32_t *topology;     // fracture CSR: offsets[n + 1], then bond indices
    const uint32_t *endpoints;    // original indices with at least one fracture bond
    uint32_t n_endpoints;
    // k_substep's grid barriers: how long a CTA waits for the others, and a
    // CTA that leaves before the first barrier without arriving (0xffffffff:
    // none; set only to exercise the wait limit)
    unsigned long long barrier_limit_ns;
    uint32_t barrier_skip;
    uint32_t alloc_chunks;  // allocation chunks of 1024 tiles over all scenes
};

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;
constexpr int SCAN_TOP_THREADS = 1024;
constexpr int ALLOC_THREADS = 256;  // k_tile_alloc: 4 tiles per thread, 1024 per CTA
constexpr int ALLOC_ITEMS = 4;
constexpr uint32_t ALLOC_TILES = ALLOC_THREADS * ALLOC_ITEMS;

// default P2G: the particles whose base node lies in one 16x8-node tile reach
// the 18x10 nodes of its ring (the tile plus two columns and two rows)
constexpr int RING_X = TILE_X + 2;
constexpr int RING_Y = TILE_Y + 2;
constexpr int RING_NODES = RING_X * RING_Y;
constexpr int TILE_CELLS = TILE_X * TILE_Y;
constexpr int STAGE_CAP = 640;         // particles of a tile staged in shared memory at once (default variant)
constexpr int STAGE_CAP_NARROW = 384;  // the narrow-stage variant (smaller stages, more tiles in flight)
constexpr int ACC_WORDS = 11;   // solid m,px,py | water m,px,py,V | oil m,px,py,V
constexpr uint32_t REC_FAILED = 1u << 16;  // a P2G entry whose prepareParticle failed
constexpr uint32_t KEY_CELL_SHIFT = 24;    // bucket key: tile in the low 24 bits, local cell above
constexpr uint32_t KEY_TILE_MASK = (1u << KEY_CELL_SHIFT) - 1u;
constexpr int VOL_X = RING_X + 2;          // ring nodes and their neighbours
constexpr int VOL_Y = RING_Y + 2;
constexpr int G2P_THREADS = 256;
constexpr int FIELD_BODY_CHUNK = TILE_NODES;  // bodies staged per pass of k_triangle_field
constexpr int BODY_THREADS = 64;              // k_body_impulses: one CTA per body
constexpr uint32_t PAIR_CACHE_BODIES = 2048;  // bodies up to which pair contacts are cached
constexpr int BONDED_TRIANGLE_SOLVER_ITERATIONS = 2;
constexpr int G2P_STAGE = 2 * G2P_THREADS;  // particles of a tile staged at once
constexpr int END_BATCH_THREADS = 256;      // k_end_batch: threads per CTA and
constexpr int END_BATCH_ITEMS = 4;          // particles per thread and pass
static_assert(VOL_X * VOL_Y <= G2P_THREADS && RING_NODES <= G2P_THREADS, "one node per thread");

// device counters beyond the three of mpm_device.cuh
constexpr int COUNTER_SUBSTEP = 8;       // the substep of this batch under way (failed and skipped included)
constexpr int COUNTER_FRESH = 9;         // 1 from the start of a batch until its first substep starts
constexpr int COUNTER_STOP = 10;         // substeps completed in this batch (STOP_NONE while running)
constexpr int COUNTER_CURSOR = 11;       // the next free bucket entry of the scene (k_tile_alloc)
constexpr int COUNTER_RUNS = 12;         // the scene takes part in the substep under way (k_tile_alloc)
constexpr uint32_t STOP_NONE = 0xffffffffu;
constexpr int SCENE_WORDS = 64;  // per scene: status [0, 32), counters [32, 64)
constexpr int WORK_ACTIVE = 0;   // work[0], work[1]: tiles listed for the substeps from buffer 0 / 1
constexpr int WORK_BARRIER = 2;  // work[2]: arrivals at the substep kernel's grid barrier, work[3]: its generation
constexpr int WORK_ABORT = 4;    // work[4]: non-zero once a barrier wait of the substep kernel ran out
constexpr int WORK_HEAVY = 5;    // work[5], work[6]: heavy tiles listed for the substeps from buffer 0 / 1
constexpr int WORK_CLAIM = 7;    // work[7], work[8]: tiles claimed so far by this substep's P2G / G2P (several scenes)
constexpr int WORK_WORDS = 16;
constexpr uint32_t HEAVY_TILE = 640;  // a tile holding more particles is listed first (it takes longest)
constexpr int SUBSTEP_THREADS = 256;  // k_substep: one CTA shape for all four phases

__global__ void k_count(Ctx c);
__global__ void k_scan_reduce(Ctx c, uint32_t n_chunks);
__global__ void k_scan_top(Ctx c, uint32_t n_chunks);
__global__ void k_scan_apply(Ctx c, uint32_t n_chunks);
__global__ void k_scatter(Ctx c);
__global__ void k_stable_rank(Ctx c);
__global__ void k_tile_count(Ctx c);
__global__ void k_tile_alloc(Ctx c);
__global__ void k_tile_scatter(Ctx c);
// SCENES: the solver holds several scenes; CAP: particles staged at once;
// LIQ: every material is water or oil; REC: the records variant (P2G reads
// the records G2P wrote instead of preparing each particle from its state)
template <bool SCENES, int CAP, bool LIQ, bool REC>
__global__ void k_p2g_gather(Ctx c);
// The whole substep of the default path in one cooperative launch: tile
// allocation, bucketing, P2G and G2P, separated by grid barriers whose waits
// give up after Ctx::barrier_limit_ns (then ERROR_BARRIER is raised in every
// scene and the launch returns).
template <bool SCENES, int CAP, bool LIQ>
__global__ void k_substep(Ctx c);
// dynamic shared memory of k_p2g_gather and k_substep for stage capacity cap
size_t p2g_shared_bytes(int cap);
size_t substep_shared_bytes(int cap);
// BODIES: the solver holds bonded-triangle bodies or fracture bonds; LIQ:
// every material is water or oil (the other models' code compiled out);
// REC: the records variant (G2P also writes the next P2G's records)
template <bool SCENES, bool BODIES, bool LIQ, bool REC>
__global__ void k_g2p_tile(Ctx c);
__global__ void k_prepare_scatter(Ctx c);
__global__ void k_fixed_decode(Ctx c);
__global__ void k_grid_update(Ctx c);
__global__ void k_g2p(Ctx c);
__global__ void k_substep_begin(Ctx c);
__global__ void k_end_batch(Ctx c, uint32_t total_steps, uint32_t measure_speed);
__global__ void k_begin_batch(Ctx c, uint32_t reset_progress);
// bodies and fracture
__global__ void k_triangle_field(Ctx c);
__global__ void k_body_impulses(Ctx c);
__global__ void k_body_bonded(Ctx c);
__global__ void k_body_states(Ctx c);
__global__ void k_body_pairs(Ctx c);
__global__ void k_body_apply(Ctx c);
__global__ void k_validate_cfl(Ctx c);
__global__ void k_fracture_bonds(Ctx c);
__global__ void k_fracture_damage(Ctx c);
__global__ void k_body_finish(Ctx c);
__global__ void k_count_active_nodes(Ctx c, uint32_t *counts);
__global__ void k_count_ring_nodes(Ctx c0, uint32_t *counts);
__global__ void k_probe_deformation(const float4 *F, const float4 *C, float dt, uint32_t n, float4 *trial,
                                    float2 *increment_det, uint32_t *substeps, uint32_t *flags);
// surface occupancy (status word 7 flags: shaders.ts:187-189)
constexpr uint32_t SURFACE_ERROR_BUCKET = 1u;
constexpr uint32_t SURFACE_ERROR_PARTICLE_AREA = 2u;
constexpr uint32_t SURFACE_ERROR_ACCUMULATION = 4u;
constexpr double SURFACE_SCALE = 1099511627776.0;  // 2^40 fixed-point units per unit of area
constexpr double SURFACE_LIMIT = 4611686018427387904.0;  // 2^62: the largest single contribution
struct SurfaceGeometry {
    float dx;
    uint32_t cells_x, cells_y, node_w;
};
__global__ void k_surface_gather(Ctx c, SurfaceGeometry g, unsigned long long *acc);
__global__ void k_surface_decode(const unsigned long long *acc, float2 *field, uint32_t nodes);
// interaction
__global__ void k_outlet_compact(Ctx c, float4 bounds, ParticleBuffers removed, uint32_t *counters);
__global__ void k_pick(Ctx c, float px, float py, float r2, unsigned long long *best);
__global__ void k_clone(Ctx c, uint32_t start, uint32_t count, float2 offset, float2 domain, uint32_t orig_base,
                        uint32_t object_id);

}  // namespace mpm
