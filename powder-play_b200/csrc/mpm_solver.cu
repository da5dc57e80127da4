// mpm_solver.cu -- host side of the C ABI (include/mpm_b200.h): device
// allocation, packing between the reference's 20-word particle record and the
// SoA device layout, CUDA-graph capture of substep batches, and the compact
// status/speed readback.
//
// In the gather path the particle slots are re-sorted by cell every substep;
// each slot carries its original index, and every transfer at this boundary
// (upload, readback, probes, status particle indices) speaks original indices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_kernels.cuh"

using namespace mpm;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t err__ = (expr);                                                                      \
        if (err__ != cudaSuccess)                                                                        \
            return set_error(MPM_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(err__));          \
    } while (0)

template <typename T>
cudaError_t dalloc(T **ptr, size_t count)
{
    *ptr = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void **>(ptr), count * sizeof(T));
}

uint32_t f2u(float v)
{
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return u;
}

float u2f(uint32_t u)
{
    float v;
    std::memcpy(&v, &u, 4);
    return v;
}

// One scene of a solver: its configuration, particle count and place in the
// shared slot and tile ranges.
struct SceneHost {
    mpm_config cfg{};
    uint32_t n = 0, p_base = 0;
    uint32_t node_w = 0, node_h = 0, node_count = 0, tiles_x = 0, tiles_y = 0, tiles = 0, tile_base = 0;
};

}  // namespace

struct mpm_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    mpm_config cfg{};
    uint32_t n = 0, capacity = 0;  // particles in device slots, slots allocated
    // original indices handed out (appends and clones add some); particles
    // removed by an outlet keep theirs, with their last state kept here
    uint32_t allocated = 0;
    std::vector<float> removed_words;   // 20 per original index (valid where removed)
    std::vector<uint8_t> removed;       // per original index
    uint32_t node_w = 0, node_h = 0, node_count = 0, tiles_x = 0, tiles_y = 0;
    uint32_t cell_pad = 0, n_chunks = 0;
    uint32_t n_bodies = 0, n_bonds = 0;
    int cur = 0;  // buffer holding the current particle state
    // scenes: one for mpm_create, several for mpmb_create
    std::vector<SceneHost> scenes;
    uint32_t n_scenes = 1, n_tiles_total = 0;
    uint32_t *dyn = nullptr;           // per scene: 32 status words, 32 counters
    uint32_t *work = nullptr;          // tile list sizes of the two buffer parities
    uint32_t *tile_scene = nullptr;    // per tile
    uint32_t *scene_p_base = nullptr;  // per scene, then the particle count

    StepParams *d_params = nullptr;  // per scene
    StepParams *h_params = nullptr;  // pinned staging, per scene
    std::vector<StepParams> full_params;  // the last submit every scene took part in (several scenes)
    cudaEvent_t params_copied = nullptr;
    uint32_t *d_status = nullptr;    // scene 0's status words (in dyn)
    uint32_t *d_counters = nullptr;  // scene 0's counters (in dyn)
    uint32_t *h_readback = nullptr;  // pinned: 2 counters + 8 status words (+ spare)

    ParticleBuffers buf[2]{};
    uint32_t *bonded = nullptr, *obj = nullptr;  // by original index
    Material *d_mats = nullptr;
    std::vector<Material> mats;

    uint32_t *keys = nullptr, *ranks = nullptr, *tmp = nullptr, *perm = nullptr;
    uint32_t *cell_count = nullptr, *cell_start = nullptr, *block_sums = nullptr;
    float4 *p2g_solid = nullptr, *p2g_water = nullptr, *p2g_oil = nullptr;
    float2 *g_solid = nullptr;
    float4 *g_water = nullptr, *g_oil = nullptr;
    int32_t *fixed = nullptr;
    uint32_t *tile_stamp = nullptr;
    uint32_t *tile_count = nullptr, *active_tiles = nullptr;
    uint2 *tile_range = nullptr;
    uint32_t *scene_chunk = nullptr;  // per scene: first CTA of k_tile_alloc, then the total
    uint32_t alloc_ctas = 1;
    float *part = nullptr;
    uint2 *tile_info = nullptr;
    float4 *rec_state = nullptr, *rec_affine = nullptr;  // the records variant's P2G records
    float2 *rec_mom = nullptr;
    uint32_t *rec_cell = nullptr;
    // bonded-triangle bodies and fracture bonds
    TriField *field = nullptr;
    uint32_t *body_starts = nullptr, *slot_of[2] = {nullptr, nullptr}, *track_flag = nullptr, *tracked = nullptr;
    uint32_t n_tracked = 0;
    float4 *pair_cache = nullptr;
    uint32_t *contact_count = nullptr;
    float2 *body_vel = nullptr;
    uint32_t *bonds = nullptr, *topology = nullptr, *endpoints = nullptr;
    uint32_t n_endpoints = 0, fracture_particles = 0, fracture_incidence = 0;
    unsigned p2g_ctas = 1, g2p_ctas = 1;  // persistent grids of the default path's P2G and G2P kernels
    // the default path's substep variant: one cooperative launch (k_substep)
    // or four launches, the P2G stage capacity, k_substep's persistent grid
    // and the most CTAs of it that fit on the GPU at once
    bool fused = false;
    int stage_cap = STAGE_CAP;
    // G2P compiled for water and oil only, used when every material is one
    bool liquid_kernels = true;
    // the records variant (G2P writes the next P2G's prepared records): 1 on,
    // 0 off (P2G prepares each particle from its state), -1 by the materials
    int records = -1;
    unsigned substep_ctas = 1, substep_max_ctas = 1;
    // k_substep's barrier waits: the limit, and a CTA that leaves without
    // arriving (tests of the limit only)
    unsigned long long barrier_limit_ns = 1000000000ull;
    uint32_t barrier_skip = 0xffffffffu;

    mpm_drag drag{};
    bool drag_active = false;

    // surface occupancy (allocated at the first gather)
    unsigned long long *surface_acc = nullptr;  // per halo node: water, oil fixed-point sums
    float2 *surface_field = nullptr;            // per halo node: water, oil area

    cudaEvent_t batch_start = nullptr, batch_stop = nullptr;
    bool batch_timed = false;
    // the last batch's device milliseconds, once a readback waited for it
    float batch_ms = 0.0f;
    bool batch_ms_known = false;
    uint32_t *d_active = nullptr;

    // graphs of 2^k substeps starting from buffer parity p
    std::map<std::tuple<int, int>, cudaGraphExec_t> graphs;
    // graphs of whole short batches: (substeps, start parity, guarded)
    std::map<std::tuple<uint32_t, int, int>, cudaGraphExec_t> batch_graphs;
    // the last batch's graph copied the compact readback (counters and
    // status) to h_readback, and no call since could have changed them
    bool readback_ready = false;

    bool gather() const { return cfg.p2g_mode == MPM_P2G_GATHER; }
};

namespace {

// A call that may change the counters or status words: the next
// mpm_read_compact copies them again instead of using the batch graph's copy.
void forget_readback(mpm_solver *s)
{
    if (s) s->readback_ready = false;
}

// Drops every captured graph (they hold launch sizes and buffer pointers).
void drop_graphs(mpm_solver *s)
{
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    for (auto &kv : s->batch_graphs) cudaGraphExecDestroy(kv.second);
    s->batch_graphs.clear();
}

// Whether the records variant runs: as chosen, or by default when a material
// is not a liquid with the linear EOS (preparing a Tait liquid or a solid
// costs P2G more than reading a record; a linear-EOS liquid costs it less
// than G2P writing one).
bool uses_records(const mpm_solver *s)
{
    if (s->fused && s->n_tracked == 0 && s->n_bodies == 0) return false;  // the one-launch form prepares in P2G
    if (s->records >= 0) return s->records != 0;
    if (s->n_scenes > 1) return true;
    for (const Material &m : s->mats)
        if ((m.model != MODEL_WATER && m.model != MODEL_OIL) || m.param > 0.0f) return true;
    return false;
}

Ctx make_ctx(mpm_solver *s, int parity)
{
    Ctx c{};
    c.P = s->d_params;
    c.scenes = s->d_params;
    c.dyn = s->dyn;
    c.work = s->work;
    c.tile_scene = s->tile_scene;
    c.scene_p_base = s->scene_p_base;
    c.n_scenes = s->n_scenes;
    c.parity = (uint32_t)parity;
    c.n = s->n;
    c.n_tiles = s->n_tiles_total;
    c.in = s->buf[parity];
    c.out = s->buf[1 - parity];
    c.mats = s->d_mats;
    c.bonded = s->bonded;
    c.obj = s->obj;
    c.status = s->d_status;
    c.counters = s->d_counters;
    c.keys = s->keys;
    c.ranks = s->ranks;
    c.tmp = s->tmp;
    c.perm = s->gather() ? s->perm : nullptr;
    c.cell_count = s->cell_count;
    c.cell_start = s->cell_start;
    c.block_sums = s->block_sums;
    c.cell_pad = s->cell_pad;
    c.count_next = s->gather() ? 1u : 0u;
    c.p2g_solid = s->p2g_solid;
    c.p2g_water = s->p2g_water;
    c.p2g_oil = s->p2g_oil;
    c.g_solid = s->g_solid;
    c.g_water = s->g_water;
    c.g_oil = s->g_oil;
    c.fixed = s->fixed;
    c.tile_stamp = s->tile_stamp;
    c.tile_count = s->tile_count;
    c.tile_range = s->tile_range;
    c.scene_chunk = s->scene_chunk;
    c.active_tiles = s->active_tiles;
    c.part = s->part;
    c.tile_info = s->tile_info;
    const bool rec = s->gather() && uses_records(s);
    c.rec_state = rec ? s->rec_state : nullptr;
    c.rec_affine = rec ? s->rec_affine : nullptr;
    c.rec_mom = rec ? s->rec_mom : nullptr;
    c.rec_cell = rec ? s->rec_cell : nullptr;
    c.affine_out = nullptr;
    c.field = s->field;
    c.body_starts = s->body_starts;
    c.slot_in = s->slot_of[parity];
    c.slot_out = s->slot_of[1 - parity];
    c.track_flag = s->track_flag;
    c.tracked = s->tracked;
    c.n_tracked = s->n_tracked;
    c.pair_cache = s->pair_cache;
    c.contact_count = s->contact_count;
    c.body_vel = s->body_vel;
    c.bonds = s->bonds;
    c.topology = s->topology;
    c.endpoints = s->endpoints;
    c.n_endpoints = s->n_endpoints;
    c.barrier_limit_ns = s->barrier_limit_ns;
    c.barrier_skip = s->barrier_skip;
    c.alloc_chunks = s->alloc_ctas;
    return c;
}

inline unsigned blocks_for(uint32_t n, unsigned threads) { return std::max(1u, (n + threads - 1) / threads); }

constexpr unsigned PARTICLE_THREADS = 256;

// Kernel slots of the profiled substep (mpm_profile_substeps).
enum KernelSlot {
    K_TILE_COUNT, K_TILE_ALLOC, K_TILE_SCATTER, K_P2G_GATHER, K_G2P_TILE, K_PREPARE_SCATTER,
    K_FIXED_DECODE, K_GRID_UPDATE, K_G2P, K_SUBSTEP_BEGIN, K_END_BATCH, K_SUBSTEP, K_SLOTS
};
const char *const KERNEL_NAMES[K_SLOTS] = {
    "k_tile_count", "k_tile_alloc", "k_tile_scatter", "k_p2g_gather", "k_g2p_tile", "k_prepare_scatter",
    "k_fixed_decode", "k_grid_update", "k_g2p", "k_substep_begin", "k_end_batch", "k_substep"};

// When set, an event is recorded after every kernel launch so that the
// kernels of a substep can be timed one by one.  The profiled substeps are
// captured into a graph with external event-record nodes between the
// kernels, so host launch gaps do not enter the timings.
struct Recorder {
    cudaStream_t stream;
    std::vector<cudaEvent_t> events;
    std::vector<int> slots;
    cudaError_t error = cudaSuccess;
    void mark(int slot)
    {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err == cudaSuccess) err = cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal);
        if (err != cudaSuccess) {
            if (error == cudaSuccess) error = err;
            return;
        }
        events.push_back(e);
        slots.push_back(slot);
    }
};
thread_local Recorder *g_recorder = nullptr;

inline void mark(int slot)
{
    if (g_recorder) g_recorder->mark(slot);
}

// The first tile count of a batch (later substeps are counted by G2P).
void enqueue_tile_count(mpm_solver *s, const Ctx &c)
{
    cudaMemsetAsync(s->tile_count, 0, (size_t)s->n_tiles_total * sizeof(uint32_t), s->stream);
    k_tile_count<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c);
    mark(K_TILE_COUNT);
}

// The cell sort of the probes: count -> scan -> scatter -> stable rank.
void enqueue_cell_sort(mpm_solver *s, const Ctx &c)
{
    const unsigned pb = blocks_for(s->n, PARTICLE_THREADS);
    cudaMemsetAsync(s->cell_count, 0, (size_t)s->cell_pad * sizeof(uint32_t), s->stream);
    k_count<<<pb, PARTICLE_THREADS, 0, s->stream>>>(c);
    k_scan_reduce<<<s->n_chunks, SCAN_THREADS, 0, s->stream>>>(c, s->n_chunks);
    k_scan_top<<<1, SCAN_TOP_THREADS, 0, s->stream>>>(c, s->n_chunks);
    k_scan_apply<<<s->n_chunks, SCAN_THREADS, 0, s->stream>>>(c, s->n_chunks);
    k_scatter<<<pb, PARTICLE_THREADS, 0, s->stream>>>(c);
    k_stable_rank<<<pb, PARTICLE_THREADS, 0, s->stream>>>(c);
}

// The passes after G2P for bonded-triangle bodies and fracture bonds, in the
// reference's order (solver.ts:1505-1562): contact impulses, bonded edges,
// contact states, pair contacts, the CFL check, fracture; then the tile
// counts and P2G records of the particles those passes moved.
void enqueue_bodies(mpm_solver *s, const Ctx &c)
{
    const uint32_t nb = s->n_bodies;
    if (nb) {
        const unsigned bb = blocks_for(nb, 64);
        k_body_impulses<<<std::min(nb, 1024u), BODY_THREADS, 0, s->stream>>>(c);
        k_body_bonded<<<bb, 64, 0, s->stream>>>(c);
        k_body_states<<<bb, 64, 0, s->stream>>>(c);
        if (s->pair_cache) k_body_pairs<<<blocks_for(nb * nb, 256), 256, 0, s->stream>>>(c);
        k_body_apply<<<bb, 64, 0, s->stream>>>(c);
        // captured graphs serve batches with and without a CFL guard: the
        // kernel reads the batch's flag from the device parameters
        k_validate_cfl<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c);
    }
    if (s->n_bonds) {
        k_fracture_bonds<<<blocks_for(s->n_bonds, 64), 64, 0, s->stream>>>(c);
        if (s->n_endpoints) k_fracture_damage<<<blocks_for(s->n_endpoints, 64), 64, 0, s->stream>>>(c);
    }
    if (s->gather() && s->n_tracked) k_body_finish<<<blocks_for(s->n_tracked, 64), 64, 0, s->stream>>>(c);
}

// The k_substep instantiation for the scene count, stage capacity and
// material set.
const void *substep_kernel(bool scenes, int cap, bool liq)
{
    if (liq) {
        if (cap == STAGE_CAP_NARROW)
            return scenes ? (const void *)k_substep<true, STAGE_CAP_NARROW, true>
                          : (const void *)k_substep<false, STAGE_CAP_NARROW, true>;
        return scenes ? (const void *)k_substep<true, STAGE_CAP, true> : (const void *)k_substep<false, STAGE_CAP, true>;
    }
    if (cap == STAGE_CAP_NARROW)
        return scenes ? (const void *)k_substep<true, STAGE_CAP_NARROW, false>
                      : (const void *)k_substep<false, STAGE_CAP_NARROW, false>;
    return scenes ? (const void *)k_substep<true, STAGE_CAP, false> : (const void *)k_substep<false, STAGE_CAP, false>;
}

template <bool REC>
const void *p2g_kernel_rec(bool scenes, int cap, bool liq)
{
    if (liq) {
        if (cap == STAGE_CAP_NARROW)
            return scenes ? (const void *)k_p2g_gather<true, STAGE_CAP_NARROW, true, REC>
                          : (const void *)k_p2g_gather<false, STAGE_CAP_NARROW, true, REC>;
        return scenes ? (const void *)k_p2g_gather<true, STAGE_CAP, true, REC>
                      : (const void *)k_p2g_gather<false, STAGE_CAP, true, REC>;
    }
    if (cap == STAGE_CAP_NARROW)
        return scenes ? (const void *)k_p2g_gather<true, STAGE_CAP_NARROW, false, REC>
                      : (const void *)k_p2g_gather<false, STAGE_CAP_NARROW, false, REC>;
    return scenes ? (const void *)k_p2g_gather<true, STAGE_CAP, false, REC>
                  : (const void *)k_p2g_gather<false, STAGE_CAP, false, REC>;
}

// The k_p2g_gather instantiation for the scene count, stage capacity,
// material set and records variant.
const void *p2g_kernel(bool scenes, int cap, bool liq, bool rec)
{
    return rec ? p2g_kernel_rec<true>(scenes, cap, liq) : p2g_kernel_rec<false>(scenes, cap, liq);
}

// Whether the substeps of this solver run as one k_substep launch each:
// the default path without bonded bodies or fracture bonds (their passes
// run between and after P2G and G2P), when that variant is chosen.
bool runs_fused(const mpm_solver *s) { return s->gather() && s->fused && s->n_tracked == 0 && s->n_bodies == 0; }

// Whether G2P runs its water-and-oil instantiation: every material of the
// solver is water or oil and it holds no bodies or fracture bonds.
bool runs_liquid(const mpm_solver *s)
{
    if (!s->liquid_kernels || s->n_tracked != 0 || s->n_bodies != 0 || s->mats.empty()) return false;
    for (const Material &m : s->mats)
        if (m.model != MODEL_WATER && m.model != MODEL_OIL) return false;
    return true;
}

// Enqueues k_substep as a cooperative launch (every CTA resident at once).
cudaError_t launch_substep(mpm_solver *s, const Ctx &c)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(s->substep_ctas);
    cfg.blockDim = dim3(SUBSTEP_THREADS);
    cfg.dynamicSmemBytes = substep_shared_bytes(s->stage_cap);
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {const_cast<Ctx *>(&c)};
    return cudaLaunchKernelExC(&cfg, substep_kernel(s->n_scenes > 1, s->stage_cap, runs_liquid(s)), args);
}

// Shared-memory limits of the stage variants (set once per process and
// device; the attributes are per function).
cudaError_t configure_variant_kernels()
{
    const int caps[2] = {STAGE_CAP, STAGE_CAP_NARROW};
    for (int cap : caps) {
        for (int scenes = 0; scenes < 2; ++scenes) {
            const void *fns[6] = {p2g_kernel(scenes != 0, cap, false, false), p2g_kernel(scenes != 0, cap, true, false),
                                  p2g_kernel(scenes != 0, cap, false, true),  p2g_kernel(scenes != 0, cap, true, true),
                                  substep_kernel(scenes != 0, cap, false), substep_kernel(scenes != 0, cap, true)};
            const size_t bytes[6] = {p2g_shared_bytes(cap), p2g_shared_bytes(cap), p2g_shared_bytes(cap),
                                     p2g_shared_bytes(cap), substep_shared_bytes(cap), substep_shared_bytes(cap)};
            for (int k = 0; k < 6; ++k) {
                cudaError_t e = cudaFuncSetAttribute(fns[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes[k]);
                if (e == cudaSuccess) e = cudaFuncSetAttribute(fns[k], cudaFuncAttributePreferredSharedMemoryCarveout, 100);
                if (e != cudaSuccess) return e;
            }
        }
    }
    return cudaSuccess;
}

// CTAs per SM of the P2G kernel and of k_substep for stage capacity `cap`.
cudaError_t variant_occupancy(int cap, int *per_sm_p2g, int *per_sm_substep)
{
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm_p2g, p2g_kernel(false, cap, false, false), TILE_CELLS,
                                                                  p2g_shared_bytes(cap));
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm_substep, substep_kernel(false, cap, false), SUBSTEP_THREADS,
                                                          substep_shared_bytes(cap));
    return e;
}

// The k_g2p_tile instantiation for the solver's scenes, bodies, materials
// and records variant.
template <bool REC>
void launch_g2p(mpm_solver *s, const Ctx &c, bool liq)
{
    if (s->n_scenes > 1 && liq)
        k_g2p_tile<true, false, true, REC><<<s->g2p_ctas, G2P_THREADS, 0, s->stream>>>(c);
    else if (s->n_scenes > 1)
        k_g2p_tile<true, false, false, REC><<<s->g2p_ctas, G2P_THREADS, 0, s->stream>>>(c);
    else if (s->n_tracked > 0)
        k_g2p_tile<false, true, false, REC><<<s->g2p_ctas, G2P_THREADS, 0, s->stream>>>(c);
    else if (liq)
        k_g2p_tile<false, false, true, REC><<<s->g2p_ctas, G2P_THREADS, 0, s->stream>>>(c);
    else
        k_g2p_tile<false, false, false, REC><<<s->g2p_ctas, G2P_THREADS, 0, s->stream>>>(c);
}

// One full substep from buffer `parity` into 1 - parity.
void enqueue_substep(mpm_solver *s, int parity)
{
    const Ctx c = make_ctx(s, parity);
    const unsigned pb = blocks_for(s->n, PARTICLE_THREADS);
    const dim3 tiles(s->tiles_x, s->tiles_y);
    if (runs_fused(s)) {
        const cudaError_t e = launch_substep(s, c);
        if (e != cudaSuccess && g_recorder && g_recorder->error == cudaSuccess) g_recorder->error = e;
        mark(K_SUBSTEP);
    } else if (s->gather()) {
        k_tile_alloc<<<s->alloc_ctas, ALLOC_THREADS, 0, s->stream>>>(c);
        mark(K_TILE_ALLOC);
        k_tile_scatter<<<blocks_for((s->n + 3) / 4, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c);
        mark(K_TILE_SCATTER);
        {
            void *args[] = {const_cast<Ctx *>(&c)};
            cudaLaunchKernel(p2g_kernel(s->n_scenes > 1, s->stage_cap, runs_liquid(s), uses_records(s)), dim3(s->p2g_ctas),
                             dim3(TILE_CELLS), args,
                             p2g_shared_bytes(s->stage_cap), s->stream);
        }
        mark(K_P2G_GATHER);
        if (s->n_bodies) k_triangle_field<<<tiles, TILE_NODES, 0, s->stream>>>(c);
        const bool liq = runs_liquid(s);
        if (uses_records(s))
            launch_g2p<true>(s, c, liq);
        else
            launch_g2p<false>(s, c, liq);
        mark(K_G2P_TILE);
    } else {
        k_substep_begin<<<blocks_for(s->n_scenes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c);
        mark(K_SUBSTEP_BEGIN);
        k_prepare_scatter<<<pb, PARTICLE_THREADS, 0, s->stream>>>(c);
        mark(K_PREPARE_SCATTER);
        k_fixed_decode<<<tiles, TILE_NODES, 0, s->stream>>>(c);
        mark(K_FIXED_DECODE);
        if (s->n_bodies) k_triangle_field<<<tiles, TILE_NODES, 0, s->stream>>>(c);
        k_grid_update<<<tiles, TILE_NODES, 0, s->stream>>>(c);
        mark(K_GRID_UPDATE);
        k_g2p<<<pb, PARTICLE_THREADS, 0, s->stream>>>(c);
        mark(K_G2P);
    }
    enqueue_bodies(s, c);
}

// The end of a batch of `total` substeps that ended in buffer `parity`.
void enqueue_end_batch(mpm_solver *s, int parity, uint32_t total, bool measure_speed)
{
    const Ctx c = make_ctx(s, 1 - parity);  // out: the buffer the batch ends in
    const unsigned ctas = s->n_scenes == 1 ? blocks_for(s->n, END_BATCH_THREADS * END_BATCH_ITEMS)
                                           : std::min(blocks_for(s->n, END_BATCH_THREADS), 1184u);
    k_end_batch<<<ctas, END_BATCH_THREADS, 0, s->stream>>>(c, total, measure_speed ? 1u : 0u);
    mark(K_END_BATCH);
}

// Substeps per captured graph: at most 2^MAX_GRAPH_LOG2.
constexpr int MAX_GRAPH_LOG2 = 9;

int get_graph(mpm_solver *s, int log2_steps, int parity, cudaGraphExec_t *out)
{
    auto key = std::make_tuple(log2_steps, parity);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return MPM_OK;
    }
    cudaGraph_t graph = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int p = parity;
    for (int k = 0; k < (1 << log2_steps); ++k) {
        enqueue_substep(s, p);
        p = 1 - p;
    }
    cudaError_t err = cudaStreamEndCapture(s->stream, &graph);
    if (err != cudaSuccess) return set_error(MPM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(err));
    cudaGraphExec_t exec = nullptr;
    err = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) return set_error(MPM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(err));
    s->graphs[key] = exec;
    *out = exec;
    return MPM_OK;
}

// The largest float t >= 0 with sqrt(t) <= bound (square roots correctly
// rounded, as the device's are): a square root of s > bound exactly when
// s > t, for every finite s >= 0.  sqrt is monotone, so t is found from
// bound^2 by stepping one ulp at a time (a step or two).
static float square_bound(float bound)
{
    if (std::isnan(bound)) return bound;
    if (bound < 0.0f) return -1.0f;
    if (std::isinf(bound)) return bound;
    float t = (float)((double)bound * (double)bound);
    while (t > 0.0f && std::sqrt(t) > bound) t = std::nextafter(t, 0.0f);
    for (;;) {
        const float up = std::nextafter(t, INFINITY);
        if (!std::isfinite(up) || std::sqrt(up) > bound) break;
        t = up;
    }
    return t;
}

void fill_params(mpm_solver *s, uint32_t scene, StepParams &p, float dt, float gx, float gy,
                 const mpm_cfl_guard *guard, float bond_reference_dt, uint32_t steps)
{
    std::memset(&p, 0, sizeof p);
    const SceneHost &sc = s->scenes[scene];
    const mpm_config &c = sc.cfg;
    p.cells_x = c.cells_x;
    p.cells_y = c.cells_y;
    p.node_w = sc.node_w;
    p.node_h = sc.node_h;
    p.n_particles = sc.n;
    p.n_nodes = sc.node_count;
    p.tiles_x = sc.tiles_x;
    p.tiles_y = sc.tiles_y;
    p.p_base = sc.p_base;
    p.tile_base = sc.tile_base;
    p.scene_tiles = sc.tiles;
    p.n_bodies = s->n_bodies;
    p.cfl_enabled = guard ? 1u : 0u;
    p.n_bonds = s->n_bonds;
    p.fracture_particles = s->fracture_particles;
    p.fracture_incidence = s->fracture_incidence;
    p.pair_cache_enabled = s->pair_cache ? 1u : 0u;
    p.batch_steps = steps;
    p.fixed_shift = c.fixed_point_shift;
    p.dx = c.cell_size;
    p.inv_dx = 1.0f / c.cell_size;
    p.particle_mass = c.particle_mass;
    p.particle_volume = c.particle_volume;
    p.dt = dt;
    p.lambda = c.lambda;
    p.mu = c.mu;
    // stress scale and gradient scale as float32 (layout.ts:944-948, :235)
    const double cs = (double)c.cell_size;
    p.gradient_scale = (float)(4.0 / (cs * cs));
    p.stress_scale = (float)(-(double)dt * (double)c.particle_volume * (4.0 / (cs * cs)));
    p.gx = gx;
    p.gy = gy;
    p.domain_w = (float)((double)c.cells_x * (double)c.cell_size);
    p.domain_h = (float)((double)c.cells_y * (double)c.cell_size);
    p.bond_rest_length = c.bond_rest_length;
    p.bond_stiffness = c.bond_stiffness;
    p.band = c.cell_size * 2.0f;
    p.contact_reach = (float)(std::sqrt((double)c.particle_volume / M_PI) + (double)c.cell_size * 0.75);
    p.cfl_wave_bound = guard ? guard->wave_speed_bound : 0.0f;
    p.cfl_velocity_limit = guard ? guard->velocity_limit : 0.0f;
    p.cfl_wave2_bound = square_bound(p.cfl_wave_bound);
    p.cfl_speed2_bound = square_bound(p.cfl_velocity_limit);
    p.bond_reference_dt = bond_reference_dt > 0.0f ? bond_reference_dt
                                                   : (c.bond_reference_dt > 0.0f ? c.bond_reference_dt : dt);
    p.wall_friction = c.wall_friction;
    p.fixed_scale = std::ldexp(1.0f, (int)c.fixed_point_shift);
    if (s->drag_active) {
        p.drag_x = s->drag.target_x;
        p.drag_y = s->drag.target_y;
        p.drag_radius = s->drag.radius;
        p.drag_stiffness = s->drag.stiffness;
        p.drag_damping = s->drag.damping;
    }
}

// Copies the pinned parameters to the device (a batch graph holds this copy
// itself) and marks when the host may write them again.
int copy_params(mpm_solver *s)
{
    CUDA_TRY(cudaMemcpyAsync(s->d_params, s->h_params, s->n_scenes * sizeof(StepParams), cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaEventRecord(s->params_copied, s->stream));
    return MPM_OK;
}

// The same step for every scene; `copy` false leaves the copy to run_batch.
int upload_params(mpm_solver *s, float dt, float gx, float gy, const mpm_cfl_guard *guard, float bond_reference_dt,
                  uint32_t steps, bool copy = true)
{
    CUDA_TRY(cudaEventSynchronize(s->params_copied));
    for (uint32_t k = 0; k < s->n_scenes; ++k)
        fill_params(s, k, s->h_params[k], dt, gx, gy, guard, bond_reference_dt, steps);
    return copy ? copy_params(s) : MPM_OK;
}

// A step of its own for each scene (steps[k] 0: the scene sits the batch
// out); the copy is left to run_batch.
int upload_scene_params(mpm_solver *s, const uint32_t *steps, const float *dt, const float *gx, const float *gy,
                        const mpm_cfl_guard *guards)
{
    CUDA_TRY(cudaEventSynchronize(s->params_copied));
    bool every = true;
    for (uint32_t k = 0; k < s->n_scenes; ++k) {
        fill_params(s, k, s->h_params[k], dt[k], gx[k], gy[k], guards ? guards + k : nullptr, 0.0f, steps[k]);
        every = every && steps[k] > 0;
    }
    // the autotuner times the substeps of the last submit every scene took
    // part in (a retry submit holds only the scenes that failed)
    if (every) s->full_params.assign(s->h_params, s->h_params + s->n_scenes);
    return MPM_OK;
}

// material table key: model + lambda + mu + density + parameter (the
// parameter of a Neo-Hookean particle is its damage, kept per particle)
uint32_t intern_material(std::vector<Material> &table, const float *w)
{
    Material m{};
    m.model = f2u(w[13]);
    m.lambda = w[14];
    m.mu = w[15];
    m.density = w[16];
    m.param = m.model == MODEL_NEO_HOOKEAN ? 0.0f : w[18];
    // the quotient the CFL wave-speed bound would divide out per particle
    // (both IEEE float32 divisions: the same bits)
    const bool liquid = m.model == MODEL_WATER || m.model == MODEL_OIL;
    m.c2 = liquid && std::isfinite(m.lambda) && std::isfinite(m.density) && m.lambda > 0.0f && m.density > 0.0f
               ? m.lambda / m.density
               : 0.0f;
    for (size_t k = 0; k < table.size(); ++k) {
        const Material &t = table[k];
        if (t.model == m.model && f2u(t.lambda) == f2u(m.lambda) && f2u(t.mu) == f2u(m.mu) &&
            f2u(t.density) == f2u(m.density) && f2u(t.param) == f2u(m.param))
            return (uint32_t)k;
    }
    table.push_back(m);
    return (uint32_t)(table.size() - 1);
}

// Uploads packed records in original order: slot i holds particle i.
// Uploads `count` packed particles into slots slot_base.. of buffer `target`
// as original indices orig_base..
int unpack_and_upload(mpm_solver *s, const float *packed, uint32_t count, int target, uint32_t slot_base = 0,
                      uint32_t orig_base = 0)
{
    std::vector<float2> pos(count), vel(count);
    std::vector<float4> C(count), F(count);
    std::vector<float> pvol(count), damage(count), vol(count);
    std::vector<uint32_t> mat(count), bonded(count), orig(count);
    const size_t before = s->mats.size();
    for (uint32_t i = 0; i < count; ++i) {
        const float *w = packed + (size_t)i * MPM_PARTICLE_WORDS;
        const uint32_t model = f2u(w[13]);
        if (model > MODEL_FIXED_COROTATED)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "particle %u has an unsupported MPM material model %u", i, model);
        pos[i] = make_float2(w[0], w[1]);
        vel[i] = make_float2(w[2], w[3]);
        C[i] = make_float4(w[4], w[5], w[6], w[7]);
        F[i] = make_float4(w[8], w[9], w[10], w[11]);
        pvol[i] = w[12];
        damage[i] = model == MODEL_NEO_HOOKEAN ? w[18] : 0.0f;
        vol[i] = w[17];
        mat[i] = intern_material(s->mats, w);
        bonded[i] = f2u(w[19]);
        orig[i] = orig_base + i;
        if (bonded[i] > 3u) return set_error(MPM_ERR_INVALID_ARGUMENT, "particle %u has an invalid bonded triangle marker", i);
    }
    if (s->mats.size() > 65536) return set_error(MPM_ERR_INVALID_ARGUMENT, "more than 65536 distinct materials");
    if (s->mats.size() != before || s->d_mats == nullptr) {
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        if (s->d_mats) cudaFree(s->d_mats);
        s->d_mats = nullptr;
        CUDA_TRY(dalloc(&s->d_mats, s->mats.size()));
        CUDA_TRY(cudaMemcpyAsync(s->d_mats, s->mats.data(), s->mats.size() * sizeof(Material), cudaMemcpyHostToDevice,
                                 s->stream));
        // captured graphs hold the old table pointer
        drop_graphs(s);
    }
    ParticleBuffers &b = s->buf[target];
    const size_t d = slot_base;
    CUDA_TRY(cudaMemcpyAsync(b.pos + d, pos.data(), count * sizeof(float2), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.vel + d, vel.data(), count * sizeof(float2), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.C + d, C.data(), count * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.F + d, F.data(), count * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.pvol + d, pvol.data(), count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.damage + d, damage.data(), count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.vol + d, vol.data(), count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.mat + d, mat.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(b.orig + d, orig.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->bonded + orig_base, bonded.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             s->stream));
    if (s->slot_of[target]) {
        // the uploaded slots are in original order
        std::vector<uint32_t> slots(count);
        for (uint32_t i = 0; i < count; ++i) slots[i] = slot_base + i;
        CUDA_TRY(cudaMemcpyAsync(s->slot_of[target] + orig_base, slots.data(), count * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    // the copies above read pageable host vectors; wait before they go away
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

// Copies the slot arrays of the current buffer to the host.
struct HostState {
    std::vector<float2> pos, vel;
    std::vector<float4> C, F;
    std::vector<float> pvol, damage, vol;
    std::vector<uint32_t> mat, orig;
};

int download_state(mpm_solver *s, HostState &h)
{
    const uint32_t n = s->n;
    h.pos.resize(n);
    h.vel.resize(n);
    h.C.resize(n);
    h.F.resize(n);
    h.pvol.resize(n);
    h.damage.resize(n);
    h.vol.resize(n);
    h.mat.resize(n);
    h.orig.resize(n);
    const ParticleBuffers &b = s->buf[s->cur];
    if (n > 0) {
        CUDA_TRY(cudaMemcpyAsync(h.pos.data(), b.pos, n * sizeof(float2), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.vel.data(), b.vel, n * sizeof(float2), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.C.data(), b.C, n * sizeof(float4), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.F.data(), b.F, n * sizeof(float4), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.pvol.data(), b.pvol, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.damage.data(), b.damage, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.vol.data(), b.vol, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.mat.data(), b.mat, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(h.orig.data(), b.orig, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

void free_solver(mpm_solver *s)
{
    if (!s) return;
    if (s->device >= 0) cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graphs(s);
    void *ptrs[] = {s->d_params, s->dyn, s->work, s->tile_scene, s->scene_p_base, s->bonded, s->obj, s->d_mats, s->keys, s->ranks,
                    s->tmp, s->perm, s->cell_count, s->cell_start, s->block_sums, s->p2g_solid, s->p2g_water,
                    s->p2g_oil, s->g_solid, s->g_water, s->g_oil, s->fixed, s->tile_stamp, s->d_active,
                    s->tile_count, s->tile_range, s->scene_chunk, s->active_tiles, s->part, s->tile_info,
                    s->rec_state, s->rec_affine, s->rec_mom, s->rec_cell, s->field, s->body_starts,
                    s->slot_of[0], s->slot_of[1], s->track_flag, s->tracked, s->pair_cache, s->contact_count,
                    s->body_vel, s->bonds, s->topology, s->endpoints, s->surface_acc, s->surface_field};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int b = 0; b < 2; ++b) {
        void *bp[] = {s->buf[b].pos, s->buf[b].vel, s->buf[b].C, s->buf[b].F, s->buf[b].pvol,
                      s->buf[b].damage, s->buf[b].vol, s->buf[b].mat, s->buf[b].orig};
        for (void *p : bp)
            if (p) cudaFree(p);
    }
    if (s->h_params) cudaFreeHost(s->h_params);
    if (s->h_readback) cudaFreeHost(s->h_readback);
    if (s->params_copied) cudaEventDestroy(s->params_copied);
    if (s->batch_start) cudaEventDestroy(s->batch_start);
    if (s->batch_stop) cudaEventDestroy(s->batch_stop);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// Validates one scene's configuration for `count` particles.
int check_config(const mpm_config &c, uint32_t count)
{
    if (c.cells_x < 1 || c.cells_y < 1 || (uint64_t)c.cells_x + 3 > 0xffffffffull || (uint64_t)c.cells_y + 3 > 0xffffffffull)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "grid.cellsX must be a positive safe integer that fits the GPU layout");
    if (!(c.cell_size > 0.0f) || !std::isfinite(c.cell_size))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "grid.cellSize must be greater than zero");
    if (!(c.particle_mass > 0.0f) || !(c.particle_volume > 0.0f))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "particleMass and particleVolume must be greater than zero");
    if (c.capacity < count) return set_error(MPM_ERR_INVALID_ARGUMENT, "capacity must be at least the initial particle count and fit the GPU layout");
    if (c.p2g_mode > MPM_P2G_FIXED_POINT) return set_error(MPM_ERR_INVALID_ARGUMENT, "unknown p2g_mode %u", c.p2g_mode);
    if (c.fixed_point_shift > 30) return set_error(MPM_ERR_INVALID_ARGUMENT, "fixed_point_shift must be at most 30");
    const uint64_t nodes = ((uint64_t)c.cells_x + 3) * ((uint64_t)c.cells_y + 3);
    if (nodes > 0x7fffffffull / FIXED_WORDS)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "halo grid dimensions exceed the GPU index range");
    const uint64_t tile_records = (((uint64_t)c.cells_x + 3 + TILE_X - 1) / TILE_X) *
                                  (((uint64_t)c.cells_y + 3 + TILE_Y - 1) / TILE_Y) * (ACC_WORDS * RING_NODES);
    if (tile_records > 0xffffffffull)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "halo grid dimensions exceed the GPU index range");
    if ((uint64_t)c.capacity * 9ull > 0x7fffffffull)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "particle stencil entries exceed the index range");
    return MPM_OK;
}

// Creates a solver over `n_scenes` scenes: configs[k] with counts[k]
// particles, packed one scene after another.  Bonded bodies, fracture bonds
// and the fixed-point P2G take a single scene; the scenes of a batch hold
// exactly their particles.
int create_impl(const mpm_config *configs, uint32_t n_scenes, const uint32_t *counts, const float *packed,
                const uint32_t *object_ids, const uint32_t *body_starts, uint32_t body_count, const uint32_t *bonds,
                uint32_t bond_count, const uint32_t *topology, uint32_t topology_words, mpm_solver **out)
{
    if (!configs || !counts || !out) return set_error(MPM_ERR_INVALID_ARGUMENT, "configs, counts and out must not be NULL");
    *out = nullptr;
    if (n_scenes < 1) return set_error(MPM_ERR_INVALID_ARGUMENT, "a solver needs at least one scene");
    uint64_t total = 0;
    for (uint32_t k = 0; k < n_scenes; ++k) {
        mpm_config ck = configs[k];
        if (n_scenes > 1) ck.capacity = counts[k];
        const int rc = check_config(ck, counts[k]);
        if (rc != MPM_OK) return n_scenes > 1 ? set_error(rc, "scene %u: %s", k, g_last_error.c_str()) : rc;
        total += counts[k];
    }
    if (total * 9ull > 0x7fffffffull)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "particle stencil entries exceed the index range");
    const uint32_t count = (uint32_t)total;
    if (count > 0 && (!packed || !object_ids))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "packed_particles and object_ids must not be NULL");
    const mpm_config &c = configs[0];
    if (n_scenes > 1) {
        if (c.p2g_mode != MPM_P2G_GATHER)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "a batch of scenes runs the default P2G only");
        if (body_count > 0 || bond_count > 0)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "bonded triangle bodies and fracture bonds take a single scene");
    }
    if (body_count > 0 && !body_starts) return set_error(MPM_ERR_INVALID_ARGUMENT, "body_starts must not be NULL");
    for (uint32_t b = 0; b < body_count; ++b)
        if ((uint64_t)body_starts[b] + 2u >= count)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "bonded triangle body %u starts outside the particles", b);
    if (bond_count > 0) {
        // packed 6-word bonds and CSR incidence (layout.ts:498-564)
        if (!bonds || !topology) return set_error(MPM_ERR_INVALID_ARGUMENT, "fracture bonds and topology must not be NULL");
        if ((uint64_t)topology_words != (uint64_t)count + 1u + 2ull * bond_count)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "fracture topology must hold %u offsets and %u incidences",
                             count + 1u, 2u * bond_count);
        for (uint32_t i = 0; i < count; ++i)
            if (topology[i + 1] < topology[i]) return set_error(MPM_ERR_INVALID_ARGUMENT, "fracture topology offsets must not decrease");
        if (topology[0] != 0u || topology[count] != 2u * bond_count)
            return set_error(MPM_ERR_INVALID_ARGUMENT, "fracture topology offsets must span every incidence");
        for (uint32_t b = 0; b < bond_count; ++b)
            if (bonds[6 * b] >= count || bonds[6 * b + 1] >= count)
                return set_error(MPM_ERR_INVALID_ARGUMENT, "fracture bond %u connects a missing particle", b);
    }

    int device_count = 0;
    CUDA_TRY(cudaGetDeviceCount(&device_count));
    if (c.device < 0 || c.device >= device_count)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "device %d is not available (%d devices)", c.device, device_count);
    CUDA_TRY(cudaSetDevice(c.device));

    mpm_solver *s = new mpm_solver();
    s->device = c.device;
    s->cfg = c;
    s->n = count;
    s->allocated = count;
    s->capacity = std::max<uint32_t>(n_scenes > 1 ? count : c.capacity, 1u);
    s->n_scenes = n_scenes;
    s->scenes.resize(n_scenes);
    {
        uint32_t p_base = 0, tile_base = 0;
        for (uint32_t k = 0; k < n_scenes; ++k) {
            SceneHost &sc = s->scenes[k];
            sc.cfg = configs[k];
            sc.n = counts[k];
            sc.p_base = p_base;
            sc.node_w = sc.cfg.cells_x + 3;
            sc.node_h = sc.cfg.cells_y + 3;
            sc.node_count = sc.node_w * sc.node_h;
            sc.tiles_x = (sc.node_w + TILE_X - 1) / TILE_X;
            sc.tiles_y = (sc.node_h + TILE_Y - 1) / TILE_Y;
            sc.tiles = sc.tiles_x * sc.tiles_y;
            sc.tile_base = tile_base;
            p_base += sc.n;
            // the scene's tiles, its sentinel, then an 8-tile boundary (the
            // tile scan reads counts in aligned groups of 8)
            tile_base = (uint32_t)std::min<uint64_t>(((uint64_t)tile_base + sc.tiles + 1u + 7u) & ~7ull, 0xffffffffull);
        }
        s->n_tiles_total = tile_base;
    }
    s->n_bodies = body_count;
    s->n_bonds = bond_count;
    if (bond_count > 0) {
        s->fracture_particles = count;
        s->fracture_incidence = 2u * bond_count;
    }
    s->node_w = c.cells_x + 3;
    s->node_h = c.cells_y + 3;
    s->node_count = s->node_w * s->node_h;
    s->tiles_x = (s->node_w + TILE_X - 1) / TILE_X;
    s->tiles_y = (s->node_h + TILE_Y - 1) / TILE_Y;
    s->cell_pad = ((s->node_count + SCAN_CHUNK - 1) / SCAN_CHUNK) * SCAN_CHUNK;
    s->n_chunks = s->cell_pad / SCAN_CHUNK;

    auto fail = [&](int code) {
        free_solver(s);
        return code;
    };
    // (this also keeps every tile index below 2^24, the tile field of a bucket key)
    static_assert(0xffffffffull / (ACC_WORDS * RING_NODES) <= KEY_TILE_MASK, "tile indices must fit a bucket key");
    if ((uint64_t)s->n_tiles_total * (ACC_WORDS * RING_NODES) >= 0xffffffffull)
        return fail(set_error(MPM_ERR_INVALID_ARGUMENT, "the scenes' halo grids exceed the GPU index range"));
#define ALLOC(ptr, n)                                                                                          \
    do {                                                                                                       \
        cudaError_t e__ = dalloc(&(ptr), (n));                                                                 \
        if (e__ != cudaSuccess) return fail(set_error(MPM_ERR_CUDA, "cudaMalloc(%s) failed: %s", #ptr, cudaGetErrorString(e__))); \
    } while (0)

    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_error(MPM_ERR_CUDA, "cudaStreamCreate failed"));
    if (cudaEventCreateWithFlags(&s->params_copied, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&s->batch_start) != cudaSuccess || cudaEventCreate(&s->batch_stop) != cudaSuccess)
        return fail(set_error(MPM_ERR_CUDA, "cudaEventCreate failed"));
    if (cudaMallocHost(reinterpret_cast<void **>(&s->h_params), n_scenes * sizeof(StepParams)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void **>(&s->h_readback), 16 * sizeof(uint32_t)) != cudaSuccess)
        return fail(set_error(MPM_ERR_CUDA, "cudaMallocHost failed"));
    cudaEventRecord(s->params_copied, s->stream);

    const size_t cap = s->capacity;
    ALLOC(s->d_params, n_scenes);
    ALLOC(s->dyn, (size_t)n_scenes * SCENE_WORDS);
    ALLOC(s->work, WORK_WORDS);
    ALLOC(s->scene_p_base, (size_t)n_scenes + 1);
    s->d_status = s->dyn;  // scene 0
    s->d_counters = s->dyn + 32;
    for (int b = 0; b < 2; ++b) {
        ALLOC(s->buf[b].pos, cap);
        ALLOC(s->buf[b].vel, cap);
        ALLOC(s->buf[b].C, cap);
        ALLOC(s->buf[b].F, cap);
        ALLOC(s->buf[b].pvol, cap);
        ALLOC(s->buf[b].damage, cap);
        ALLOC(s->buf[b].vol, cap);
        ALLOC(s->buf[b].mat, cap);
        ALLOC(s->buf[b].orig, cap);
    }
    ALLOC(s->bonded, cap);
    ALLOC(s->obj, cap);
    ALLOC(s->keys, cap);
    ALLOC(s->ranks, cap);
    ALLOC(s->tmp, cap);
    ALLOC(s->perm, cap);
    ALLOC(s->cell_count, s->cell_pad);
    ALLOC(s->cell_start, (size_t)s->cell_pad + 1);
    ALLOC(s->block_sums, (size_t)s->n_chunks + 1);
    ALLOC(s->g_solid, s->node_count);
    ALLOC(s->g_water, s->node_count);
    ALLOC(s->g_oil, s->node_count);
    cudaMemsetAsync(s->g_solid, 0, (size_t)s->node_count * sizeof(float2), s->stream);
    cudaMemsetAsync(s->g_water, 0, (size_t)s->node_count * sizeof(float4), s->stream);
    cudaMemsetAsync(s->g_oil, 0, (size_t)s->node_count * sizeof(float4), s->stream);
    ALLOC(s->tile_stamp, (size_t)s->tiles_x * s->tiles_y);
    ALLOC(s->d_active, 4);
    const size_t n_tiles = s->n_tiles_total;
    ALLOC(s->tile_count, n_tiles);
    ALLOC(s->tile_range, n_tiles);
    ALLOC(s->tile_scene, n_tiles);
    ALLOC(s->scene_chunk, (size_t)n_scenes + 1);
    {
        std::vector<uint32_t> tile_scene(n_tiles, 0u), p_bases(n_scenes + 1), chunks(n_scenes + 1);
        uint32_t chunk = 0;
        for (uint32_t k = 0; k < n_scenes; ++k) {
            const SceneHost &sc = s->scenes[k];
            const uint32_t end = k + 1 < n_scenes ? s->scenes[k + 1].tile_base : (uint32_t)n_tiles;
            for (uint32_t t = sc.tile_base; t < end; ++t) tile_scene[t] = k;
            p_bases[k] = sc.p_base;
            chunks[k] = chunk;
            chunk += (sc.tiles + ALLOC_TILES - 1) / ALLOC_TILES;
        }
        p_bases[n_scenes] = count;
        chunks[n_scenes] = chunk;
        s->alloc_ctas = chunk;
        if (cudaMemcpy(s->tile_scene, tile_scene.data(), n_tiles * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(s->scene_p_base, p_bases.data(), (n_scenes + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(s->scene_chunk, chunks.data(), (n_scenes + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "scene table upload failed"));
    }
    if (c.p2g_mode == MPM_P2G_GATHER) {
        ALLOC(s->active_tiles, n_tiles);
        ALLOC(s->part, n_tiles * ACC_WORDS * RING_NODES);
        ALLOC(s->tile_info, n_tiles);
        ALLOC(s->rec_state, cap);
        ALLOC(s->rec_affine, cap);
        ALLOC(s->rec_mom, cap);
        ALLOC(s->rec_cell, cap);
        if (cudaMemsetAsync(s->tile_info, 0xff, n_tiles * sizeof(uint2), s->stream) != cudaSuccess ||
            cudaMemsetAsync(s->tile_count, 0, n_tiles * sizeof(uint32_t), s->stream) != cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "cudaMemset failed"));
        int sms = 0, per_sm_p2g = 0, per_sm_g2p = 0, per_sm_substep = 0;
        if (configure_variant_kernels() != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess ||
            variant_occupancy(s->stage_cap, &per_sm_p2g, &per_sm_substep) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_g2p, k_g2p_tile<false, false, false, false>, G2P_THREADS, 0) !=
                cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "occupancy query failed"));
        s->p2g_ctas = (unsigned)std::max<size_t>(1, std::min<size_t>(n_tiles, (size_t)sms * std::max(1, per_sm_p2g)));
        s->g2p_ctas = (unsigned)std::max<size_t>(1, std::min<size_t>(n_tiles, (size_t)sms * std::max(1, per_sm_g2p)));
        s->substep_max_ctas = (unsigned)std::max(1, sms * per_sm_substep);
        s->substep_ctas = s->substep_max_ctas;
    }
    if (c.p2g_mode == MPM_P2G_FIXED_POINT) {
        ALLOC(s->p2g_solid, s->node_count);
        ALLOC(s->p2g_water, s->node_count);
        ALLOC(s->p2g_oil, s->node_count);
        ALLOC(s->fixed, (size_t)s->node_count * FIXED_WORDS);
        if (cudaMemsetAsync(s->fixed, 0, (size_t)s->node_count * FIXED_WORDS * sizeof(int32_t), s->stream) != cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "cudaMemset failed"));
    }
    if (body_count > 0 || bond_count > 0) {
        // tracked particles: bonded-triangle vertices and fracture endpoints
        std::vector<uint32_t> flag(count, 0u), tracked, endpoints, identity(count);
        for (uint32_t i = 0; i < count; ++i) {
            identity[i] = i;
            const uint32_t marker = f2u(packed[(size_t)i * MPM_PARTICLE_WORDS + 19]);
            const bool endpoint = bond_count > 0 && topology[i + 1] > topology[i];
            if (endpoint) endpoints.push_back(i);
            if (marker != 0u || endpoint) {
                flag[i] = 1u;
                tracked.push_back(i);
            }
        }
        s->n_tracked = (uint32_t)tracked.size();
        s->n_endpoints = (uint32_t)endpoints.size();
        ALLOC(s->track_flag, cap);
        if (cudaMemset(s->track_flag, 0, cap * sizeof(uint32_t)) != cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "cudaMemset failed"));
        ALLOC(s->tracked, tracked.size());
        ALLOC(s->endpoints, endpoints.size());
        for (int b = 0; b < 2; ++b) ALLOC(s->slot_of[b], cap);
        if (body_count > 0) {
            ALLOC(s->field, s->node_count);
            ALLOC(s->body_starts, body_count);
            ALLOC(s->contact_count, body_count);
            ALLOC(s->body_vel, body_count);
            if (body_count <= PAIR_CACHE_BODIES) {
                ALLOC(s->pair_cache, (size_t)body_count * body_count);
                cudaMemsetAsync(s->pair_cache, 0, (size_t)body_count * body_count * sizeof(float4), s->stream);
            }
            cudaMemsetAsync(s->field, 0, (size_t)s->node_count * sizeof(TriField), s->stream);
        }
        if (bond_count > 0) {
            ALLOC(s->bonds, 6u * (size_t)bond_count);
            ALLOC(s->topology, topology_words);
        }
        bool ok = cudaMemcpy(s->track_flag, flag.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        if (!tracked.empty())
            ok = ok && cudaMemcpy(s->tracked, tracked.data(), tracked.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        if (!endpoints.empty())
            ok = ok && cudaMemcpy(s->endpoints, endpoints.data(), endpoints.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        for (int b = 0; b < 2; ++b)
            ok = ok && cudaMemcpy(s->slot_of[b], identity.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        if (body_count > 0)
            ok = ok && cudaMemcpy(s->body_starts, body_starts, body_count * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        if (bond_count > 0) {
            ok = ok && cudaMemcpy(s->bonds, bonds, 6u * (size_t)bond_count * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
            ok = ok && cudaMemcpy(s->topology, topology, (size_t)topology_words * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
        }
        if (!ok) return fail(set_error(MPM_ERR_CUDA, "body and fracture upload failed"));
    }
#undef ALLOC
    cudaMemsetAsync(s->cell_count, 0, (size_t)s->cell_pad * sizeof(uint32_t), s->stream);
    cudaMemsetAsync(s->tile_stamp, 0, (size_t)s->tiles_x * s->tiles_y * sizeof(uint32_t), s->stream);
    {
        // per scene: status word 1 (the particle index) empty; tile stamps
        // start at 0 and the counter above them
        std::vector<uint32_t> dyn((size_t)n_scenes * SCENE_WORDS, 0u);
        for (uint32_t k = 0; k < n_scenes; ++k) {
            dyn[(size_t)k * SCENE_WORDS + 1] = 0xffffffffu;
            dyn[(size_t)k * SCENE_WORDS + 32 + COUNTER_STAMP] = 1u;
        }
        const uint32_t zeros[WORK_WORDS] = {};
        if (cudaMemcpy(s->dyn, dyn.data(), dyn.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->work, zeros, sizeof zeros, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "status upload failed"));
    }
    if (count > 0) {
        int rc = unpack_and_upload(s, packed, count, 0);
        if (rc != MPM_OK) return fail(rc);
        if (cudaMemcpyAsync(s->obj, object_ids, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream) !=
            cudaSuccess)
            return fail(set_error(MPM_ERR_CUDA, "object id upload failed"));
    } else {
        Material dummy{};
        s->mats.push_back(dummy);
        if (dalloc(&s->d_mats, 1) != cudaSuccess) return fail(set_error(MPM_ERR_CUDA, "cudaMalloc failed"));
        cudaMemcpyAsync(s->d_mats, &dummy, sizeof dummy, cudaMemcpyHostToDevice, s->stream);
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return fail(set_error(MPM_ERR_CUDA, "initial upload failed: %s", cudaGetErrorString(e)));
    *out = s;
    return MPM_OK;
}

// Runs `step_count` real substeps with the uploaded parameters, captured in
// one graph with an event after every kernel, and sums each kernel slot's
// milliseconds and launches.
int profile_run(mpm_solver *s, uint32_t step_count, bool guarded, double *kernel_ms, uint32_t *kernel_launches)
{
    for (int k = 0; k < K_SLOTS; ++k) {
        kernel_ms[k] = 0.0;
        kernel_launches[k] = 0;
    }
    Recorder rec;
    rec.stream = s->stream;
    const Ctx c0 = make_ctx(s, s->cur);
    const int start_parity = s->cur;
    CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    k_begin_batch<<<blocks_for(s->n_scenes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c0, guarded ? 1u : 0u);
    rec.mark(-1);
    g_recorder = &rec;
    if (s->gather() && s->n > 0) enqueue_tile_count(s, c0);
    int parity = start_parity;
    for (uint32_t k = 0; k < step_count; ++k) {
        enqueue_substep(s, parity);
        parity = 1 - parity;
    }
    if (s->n > 0) enqueue_end_batch(s, parity, step_count, guarded);
    g_recorder = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (e == cudaSuccess) e = rec.error;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) s->cur = parity;
    for (size_t k = 1; e == cudaSuccess && k < rec.events.size(); ++k) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, rec.events[k - 1], rec.events[k]);
        if (rec.slots[k] >= 0) {
            kernel_ms[rec.slots[k]] += ms;
            kernel_launches[rec.slots[k]] += 1;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t ev : rec.events) cudaEventDestroy(ev);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "profiled substeps failed: %s", cudaGetErrorString(e));
    return MPM_OK;
}

// Runs `step_count` real substeps with the uploaded parameters as one graph
// (prologue, substeps, epilogue; no events between kernels) and returns its
// device milliseconds (events around the graph launch).
int timed_run(mpm_solver *s, uint32_t step_count, bool guarded, double *ms)
{
    const Ctx c0 = make_ctx(s, s->cur);
    CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    k_begin_batch<<<blocks_for(s->n_scenes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c0, guarded ? 1u : 0u);
    if (s->gather() && s->n > 0) enqueue_tile_count(s, c0);
    int parity = s->cur;
    for (uint32_t k = 0; k < step_count; ++k) {
        enqueue_substep(s, parity);
        parity = 1 - parity;
    }
    if (s->n > 0) enqueue_end_batch(s, parity, step_count, guarded);
    cudaError_t e = cudaGetLastError();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s->stream, &graph);
    if (e == cudaSuccess) e = end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaEventRecord(s->batch_start, s->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(s->batch_stop, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, s->batch_start, s->batch_stop);
    if (e == cudaSuccess) {
        s->cur = parity;
        *ms = t;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "timed substeps failed: %s", cudaGetErrorString(e));
    return MPM_OK;
}

int run_batch(mpm_solver *s, uint32_t step_count, bool guarded);

// After the particle count of a single-scene solver changed: its parameters
// and scene table follow, and the captured graphs (launch sizes) are dropped.
int refresh_count(mpm_solver *s)
{
    s->scenes[0].n = s->n;
    const uint32_t bounds[2] = {0u, s->n};
    CUDA_TRY(cudaMemcpy(s->scene_p_base, bounds, sizeof bounds, cudaMemcpyHostToDevice));
    drop_graphs(s);
    return MPM_OK;
}

}  // namespace

namespace mpm {

// The last-error channel of the library for its other host sources.
int host_error(int code, const char *message)
{
    g_last_error = message;
    return code;
}

void host_clear_error() { g_last_error.clear(); }

}  // namespace mpm

extern "C" {

int mpm_create(const mpm_config *config, const float *packed_particles, const uint32_t *object_ids,
               uint32_t particle_count, const uint32_t *body_starts, uint32_t body_count,
               const uint32_t *fracture_bonds, uint32_t fracture_bond_count, const uint32_t *fracture_topology,
               uint32_t fracture_topology_words, mpm_solver **out)
{
    g_last_error.clear();
    return create_impl(config, 1u, &particle_count, packed_particles, object_ids, body_starts, body_count,
                       fracture_bonds, fracture_bond_count, fracture_topology, fracture_topology_words, out);
}

int mpm_step_batch(mpm_solver *s, uint32_t step_count, float dt, float gx, float gy, const mpm_cfl_guard *guard,
                   float bond_reference_dt)
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (step_count < 1) return set_error(MPM_ERR_INVALID_ARGUMENT, "stepCount must be a positive safe integer.");
    if (!(dt > 0.0f) || !std::isfinite(dt)) return set_error(MPM_ERR_INVALID_ARGUMENT, "dt must be greater than zero");
    if (!std::isfinite(gx) || !std::isfinite(gy)) return set_error(MPM_ERR_INVALID_ARGUMENT, "gravity must be finite");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_params(s, dt, gx, gy, guard, bond_reference_dt, step_count, false);
    if (rc != MPM_OK) return rc;
    return run_batch(s, step_count, guard != nullptr);
}

int mpmb_create(const mpm_config *configs, uint32_t scene_count, const uint32_t *particle_counts,
                const float *packed_particles, const uint32_t *object_ids, mpm_solver **out)
{
    g_last_error.clear();
    return create_impl(configs, scene_count, particle_counts, packed_particles, object_ids, nullptr, 0u, nullptr,
                       0u, nullptr, 0u, out);
}

int mpmb_step_batch(mpm_solver *s, const uint32_t *step_counts, const float *dts, const float *gravity_xy,
                    const mpm_cfl_guard *guards)
{
    g_last_error.clear();
    if (!s || !step_counts || !dts || !gravity_xy)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "solver, step_counts, dts and gravity_xy must not be NULL");
    uint32_t most = 0;
    std::vector<float> dt(s->n_scenes), gx(s->n_scenes), gy(s->n_scenes);
    for (uint32_t k = 0; k < s->n_scenes; ++k) {
        if (step_counts[k] > 0 && (!(dts[k] > 0.0f) || !std::isfinite(dts[k])))
            return set_error(MPM_ERR_INVALID_ARGUMENT, "scene %u: dt must be greater than zero", k);
        if (!std::isfinite(gravity_xy[2 * k]) || !std::isfinite(gravity_xy[2 * k + 1]))
            return set_error(MPM_ERR_INVALID_ARGUMENT, "scene %u: gravity must be finite", k);
        dt[k] = step_counts[k] > 0 ? dts[k] : 1.0f;  // a scene sitting the batch out keeps finite parameters
        gx[k] = gravity_xy[2 * k];
        gy[k] = gravity_xy[2 * k + 1];
        most = std::max(most, step_counts[k]);
    }
    if (most < 1) return set_error(MPM_ERR_INVALID_ARGUMENT, "stepCount must be a positive safe integer.");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_scene_params(s, step_counts, dt.data(), gx.data(), gy.data(), guards);
    if (rc != MPM_OK) return rc;
    return run_batch(s, most, guards != nullptr);
}

int mpmb_read_compact(mpm_solver *s, float *maximum_speeds, uint32_t *completed_microsteps, uint32_t *status)
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    CUDA_TRY(cudaSetDevice(s->device));
    std::vector<uint32_t> dyn((size_t)s->n_scenes * SCENE_WORDS);
    CUDA_TRY(cudaMemcpyAsync(dyn.data(), s->dyn, dyn.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (uint32_t k = 0; k < s->n_scenes; ++k) {
        const uint32_t *w = dyn.data() + (size_t)k * SCENE_WORDS;
        if (maximum_speeds) maximum_speeds[k] = u2f(w[32 + COUNTER_MAX_SPEED]);
        if (completed_microsteps) completed_microsteps[k] = w[32 + COUNTER_PROGRESS];
        if (status) {
            std::memcpy(status + (size_t)k * 8, w, 8 * sizeof(uint32_t));
            // the particle index within the scene
            const uint32_t base = s->scenes[k].p_base;
            if (w[1] != 0xffffffffu && w[1] >= base) status[(size_t)k * 8 + 1] = w[1] - base;
        }
    }
    return MPM_OK;
}

uint32_t mpmb_scene_count(const mpm_solver *s) { return s ? s->n_scenes : 0u; }

}  // extern "C"

namespace {

// Batches of at most this many substeps of a single scene run as one graph
// (see capture_batch); longer ones launch graphs of 2^k substeps.
constexpr uint32_t MAX_BATCH_GRAPH_STEPS = 16;

// The whole batch on the stream being captured: the parameter copy from
// pinned memory, the batch events, the prologue, the substeps, the epilogue
// and the compact readback (counters and status words) to pinned memory.
// Returns the first error; the caller ends the capture either way.
cudaError_t capture_batch(mpm_solver *s, uint32_t step_count, int parity, bool guarded)
{
    cudaError_t e = cudaMemcpyAsync(s->d_params, s->h_params, s->n_scenes * sizeof(StepParams),
                                    cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(s->batch_start, s->stream, cudaEventRecordExternal);
    if (e != cudaSuccess) return e;
    const Ctx c0 = make_ctx(s, parity);
    k_begin_batch<<<blocks_for(s->n_scenes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c0, guarded ? 1u : 0u);
    if (s->gather()) enqueue_tile_count(s, c0);
    int p = parity;
    for (uint32_t k = 0; k < step_count; ++k) {
        enqueue_substep(s, p);
        p = 1 - p;
    }
    enqueue_end_batch(s, p, step_count, guarded);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(s->batch_stop, s->stream, cudaEventRecordExternal);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_readback, s->d_counters + COUNTER_PROGRESS, 2 * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_readback + 2, s->d_status, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    return e;
}

int get_batch_graph(mpm_solver *s, uint32_t step_count, int parity, bool guarded, cudaGraphExec_t *out)
{
    const auto key = std::make_tuple(step_count, parity, guarded ? 1 : 0);
    auto it = s->batch_graphs.find(key);
    if (it != s->batch_graphs.end()) {
        *out = it->second;
        return MPM_OK;
    }
    CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t body = capture_batch(s, step_count, parity, guarded);
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s->stream, &graph);
    cudaError_t err = body != cudaSuccess ? body : end;
    cudaGraphExec_t exec = nullptr;
    if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (err != cudaSuccess) return set_error(MPM_ERR_CUDA, "batch graph capture failed: %s", cudaGetErrorString(err));
    s->batch_graphs[key] = exec;
    *out = exec;
    return MPM_OK;
}

// Submits one batch of `step_count` substeps (the most any scene takes) with
// the parameters filled in h_params; `guarded`: a CFL guard is on.  A short
// batch of one scene is a single graph launch (the host call is then one
// launch and one event record); otherwise the parameters are copied, then
// the prologue, graphs of 2^k substeps and the epilogue are launched.
int run_batch(mpm_solver *s, uint32_t step_count, bool guarded)
{
    int rc = MPM_OK;
    s->readback_ready = false;
    s->batch_ms_known = false;
    if (s->n_scenes == 1 && s->n > 0 && step_count <= MAX_BATCH_GRAPH_STEPS) {
        cudaGraphExec_t exec;
        rc = get_batch_graph(s, step_count, s->cur, guarded, &exec);
        if (rc != MPM_OK) return rc;
        CUDA_TRY(cudaGraphLaunch(exec, s->stream));
        CUDA_TRY(cudaEventRecord(s->params_copied, s->stream));
        if (step_count & 1u) s->cur = 1 - s->cur;
        s->batch_timed = true;
        s->readback_ready = true;
        return MPM_OK;
    }
    rc = copy_params(s);
    if (rc != MPM_OK) return rc;
    const Ctx c0 = make_ctx(s, s->cur);
    CUDA_TRY(cudaEventRecord(s->batch_start, s->stream));
    k_begin_batch<<<blocks_for(s->n_scenes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c0, guarded ? 1u : 0u);
    if (s->gather() && s->n > 0) enqueue_tile_count(s, c0);
    CUDA_TRY(cudaGetLastError());
    if (s->n > 0) {
        // graphs of 2^k substeps, k <= MAX_GRAPH_LOG2; the largest repeats
        uint32_t remaining = step_count;
        for (int k = MAX_GRAPH_LOG2; k >= 0; --k) {
            while (remaining >= (1u << k)) {
                cudaGraphExec_t exec;
                rc = get_graph(s, k, s->cur, &exec);
                if (rc != MPM_OK) return rc;
                CUDA_TRY(cudaGraphLaunch(exec, s->stream));
                if (k == 0) s->cur = 1 - s->cur;  // only an odd substep count flips the buffer
                remaining -= 1u << k;
                if (k < MAX_GRAPH_LOG2) break;
            }
        }
        enqueue_end_batch(s, s->cur, step_count, guarded);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaEventRecord(s->batch_stop, s->stream));
    s->batch_timed = true;
    return MPM_OK;
}

}  // namespace

extern "C" {

int mpm_last_batch_device_ms(mpm_solver *s, double *milliseconds)
{
    g_last_error.clear();
    if (!s || !milliseconds) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and milliseconds must not be NULL");
    if (!s->batch_timed) return set_error(MPM_ERR_STATE, "no batch has been submitted");
    if (!s->batch_ms_known) {
        CUDA_TRY(cudaSetDevice(s->device));
        CUDA_TRY(cudaEventSynchronize(s->batch_stop));
        CUDA_TRY(cudaEventElapsedTime(&s->batch_ms, s->batch_start, s->batch_stop));
        s->batch_ms_known = true;
    }
    *milliseconds = s->batch_ms;
    return MPM_OK;
}

int mpm_profile_substeps(mpm_solver *s, uint32_t step_count, float dt, float gx, float gy,
                         const mpm_cfl_guard *guard, double *kernel_ms, uint32_t *kernel_launches)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !kernel_ms || !kernel_launches)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and outputs must not be NULL");
    if (step_count < 1) return set_error(MPM_ERR_INVALID_ARGUMENT, "stepCount must be a positive safe integer.");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_params(s, dt, gx, gy, guard, 0.0f, step_count);
    if (rc != MPM_OK) return rc;
    return profile_run(s, step_count, guard != nullptr, kernel_ms, kernel_launches);
}

int mpm_set_launch_shape(mpm_solver *s, uint32_t p2g_ctas, uint32_t g2p_ctas)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (!s->gather()) return set_error(MPM_ERR_STATE, "launch shapes apply to the default P2G path");
    if (p2g_ctas) s->p2g_ctas = p2g_ctas;
    if (g2p_ctas) s->g2p_ctas = g2p_ctas;
    drop_graphs(s);
    return MPM_OK;
}

int mpm_get_launch_shape(mpm_solver *s, uint32_t *p2g_ctas, uint32_t *g2p_ctas, uint32_t *sm_count)
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    if (p2g_ctas) *p2g_ctas = s->p2g_ctas;
    if (g2p_ctas) *g2p_ctas = s->g2p_ctas;
    if (sm_count) *sm_count = (uint32_t)sms;
    return MPM_OK;
}

int mpm_set_substep_variant(mpm_solver *s, uint32_t fused, uint32_t stage_capacity, uint32_t substep_ctas,
                            uint32_t liquid_kernels, uint32_t p2g_records)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (!s->gather()) return set_error(MPM_ERR_STATE, "substep variants apply to the default P2G path");
    if (fused > 1u || liquid_kernels > 1u) return set_error(MPM_ERR_INVALID_ARGUMENT, "fused and liquid_kernels must be 0 or 1");
    if (p2g_records > 2u) return set_error(MPM_ERR_INVALID_ARGUMENT, "p2g_records must be 0, 1 or 2");
    if (stage_capacity != 0u && stage_capacity != (uint32_t)STAGE_CAP && stage_capacity != (uint32_t)STAGE_CAP_NARROW)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "stage capacity must be %d or %d", STAGE_CAP, STAGE_CAP_NARROW);
    CUDA_TRY(cudaSetDevice(s->device));
    const int cap = stage_capacity ? (int)stage_capacity : s->stage_cap;
    int sms = 0, per_sm_p2g = 1, per_sm_substep = 1;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    CUDA_TRY(variant_occupancy(cap, &per_sm_p2g, &per_sm_substep));
    const unsigned most = (unsigned)std::max(1, sms * per_sm_substep);
    if (substep_ctas > most)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "substep_ctas %u exceeds the %u CTAs that fit on the GPU at once",
                         substep_ctas, most);
    s->fused = fused != 0u;
    s->liquid_kernels = liquid_kernels != 0u;
    s->records = p2g_records == 2u ? -1 : (int)p2g_records;
    s->stage_cap = cap;
    s->substep_max_ctas = most;
    if (substep_ctas) s->substep_ctas = substep_ctas;
    s->substep_ctas = std::min(s->substep_ctas, most);
    drop_graphs(s);
    return MPM_OK;
}

int mpm_get_substep_variant(mpm_solver *s, uint32_t *fused, uint32_t *stage_capacity, uint32_t *substep_ctas,
                            uint32_t *max_substep_ctas, uint32_t *liquid_kernels, uint32_t *p2g_records)
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (fused) *fused = runs_fused(s) ? 1u : 0u;
    if (stage_capacity) *stage_capacity = (uint32_t)s->stage_cap;
    if (substep_ctas) *substep_ctas = s->substep_ctas;
    if (max_substep_ctas) *max_substep_ctas = s->substep_max_ctas;
    if (liquid_kernels) *liquid_kernels = s->gather() && runs_liquid(s) ? 1u : 0u;
    if (p2g_records) *p2g_records = s->gather() && uses_records(s) ? 1u : 0u;
    return MPM_OK;
}

int mpm_set_barrier_limit(mpm_solver *s, uint64_t limit_ns, uint32_t skip_cta)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (limit_ns < 1000u || limit_ns > 60000000000ull)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "the barrier limit must lie in [1 us, 60 s]");
    s->barrier_limit_ns = limit_ns;
    s->barrier_skip = skip_cta;
    drop_graphs(s);
    return MPM_OK;
}

int mpm_autotune(mpm_solver *s, uint32_t substeps, uint32_t *p2g_ctas, uint32_t *g2p_ctas, double *best_ms)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (!s->gather()) return set_error(MPM_ERR_STATE, "launch shapes apply to the default P2G path");
    if (!s->batch_timed) return set_error(MPM_ERR_STATE, "tune after a first batch (its parameters are reused)");
    if (substeps < 1 || substeps > 64) return set_error(MPM_ERR_INVALID_ARGUMENT, "substeps must lie in [1, 64]");
    if (s->n == 0) return set_error(MPM_ERR_STATE, "there are no particles to time");
    CUDA_TRY(cudaSetDevice(s->device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    // the state the trials start from, restored before each and at the end
    const uint32_t n = s->n;
    const int start = s->cur;
    ParticleBuffers save{};
    std::vector<uint32_t> dyn((size_t)s->n_scenes * SCENE_WORDS);
    uint32_t *slots = nullptr;
    cudaError_t e = dalloc(&save.pos, n);
    if (e == cudaSuccess) e = dalloc(&save.vel, n);
    if (e == cudaSuccess) e = dalloc(&save.C, n);
    if (e == cudaSuccess) e = dalloc(&save.F, n);
    if (e == cudaSuccess) e = dalloc(&save.pvol, n);
    if (e == cudaSuccess) e = dalloc(&save.damage, n);
    if (e == cudaSuccess) e = dalloc(&save.vol, n);
    if (e == cudaSuccess) e = dalloc(&save.mat, n);
    if (e == cudaSuccess) e = dalloc(&save.orig, n);
    if (e == cudaSuccess && s->slot_of[0]) e = dalloc(&slots, s->allocated);
    auto copy_buffers = [&](const ParticleBuffers &dst, const ParticleBuffers &src) {
        const std::pair<void *, const void *> pairs[] = {{dst.pos, src.pos}, {dst.vel, src.vel}, {dst.C, src.C},
                                                         {dst.F, src.F}, {dst.pvol, src.pvol},
                                                         {dst.damage, src.damage}, {dst.vol, src.vol},
                                                         {dst.mat, src.mat}, {dst.orig, src.orig}};
        const size_t bytes[] = {sizeof(float2), sizeof(float2), sizeof(float4), sizeof(float4), sizeof(float),
                                sizeof(float), sizeof(float), sizeof(uint32_t), sizeof(uint32_t)};
        cudaError_t r = cudaSuccess;
        for (int k = 0; k < 9 && r == cudaSuccess; ++k)
            r = cudaMemcpyAsync(pairs[k].first, pairs[k].second, n * bytes[k], cudaMemcpyDeviceToDevice, s->stream);
        return r;
    };
    auto restore = [&]() {
        cudaError_t r = copy_buffers(s->buf[start], save);
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(s->dyn, dyn.data(), dyn.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream);
        if (r == cudaSuccess && slots)
            r = cudaMemcpyAsync(s->slot_of[start], slots, s->allocated * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                s->stream);
        if (r == cudaSuccess) r = cudaStreamSynchronize(s->stream);
        s->cur = start;
        return r;
    };
    if (e == cudaSuccess) e = copy_buffers(save, s->buf[start]);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dyn.data(), s->dyn, dyn.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && slots)
        e = cudaMemcpyAsync(slots, s->slot_of[start], s->allocated * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    // the parameters of the last submit every scene took part in (else the
    // last submit's), `substeps` for every scene that takes part
    if (s->full_params.size() == s->n_scenes)
        std::copy(s->full_params.begin(), s->full_params.end(), s->h_params);
    for (uint32_t k = 0; k < s->n_scenes; ++k)
        if (s->h_params[k].batch_steps > 0) s->h_params[k].batch_steps = substeps;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d_params, s->h_params, s->n_scenes * sizeof(StepParams), cudaMemcpyHostToDevice,
                            s->stream);
    int sms = 0, per_sm_g2p = 1;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_g2p, k_g2p_tile<false, false, false, false>, G2P_THREADS, 0);
    int rc = e == cudaSuccess ? MPM_OK : set_error(MPM_ERR_CUDA, "autotune set-up failed: %s", cudaGetErrorString(e));
    const bool guarded = s->h_params[0].cfl_enabled != 0u;
    // one candidate: every setting of the variant, timed over `substeps`
    // real substeps from the saved state (the whole graph, no events between
    // kernels, so the four-launch and one-launch forms compare fairly)
    struct Candidate {
        bool fused;
        int cap;
        unsigned p2g, g2p, substep;
        int records;
    };
    auto trial = [&](const Candidate &v, double &ms) {
        s->fused = v.fused;
        s->stage_cap = v.cap;
        s->p2g_ctas = v.p2g;
        s->g2p_ctas = v.g2p;
        s->substep_ctas = v.substep;
        s->records = v.records;
        const cudaError_t r = restore();
        if (r != cudaSuccess) return set_error(MPM_ERR_CUDA, "autotune restore failed: %s", cudaGetErrorString(r));
        return timed_run(s, substeps, guarded, &ms);
    };
    const Candidate v0{s->fused, s->stage_cap, s->p2g_ctas, s->g2p_ctas, s->substep_ctas, s->records};
    Candidate best = v0;
    double best_ms_total = 1e300;
    auto consider = [&](const Candidate &v) {
        double ms = 0.0;
        if (rc == MPM_OK) rc = trial(v, ms);
        if (rc == MPM_OK && ms < best_ms_total) best_ms_total = ms, best = v;
    };
    // the stage variants; for each, the one-launch form over persistent grids
    // of 1 .. (co-resident limit) CTAs per SM, and the four-launch form over
    // its P2G grids, then its G2P grids with the best P2G (a grid of one CTA
    // per tile is not a candidate: it pays for every tile of every scene in
    // substeps that list few)
    const unsigned tiles = std::max(1u, s->n_tiles_total);
    const bool can_fuse = s->n_tracked == 0 && s->n_bodies == 0;
    const int caps[2] = {STAGE_CAP, STAGE_CAP_NARROW};
    for (int cap : caps) {
        int per_sm_p2g = 1, per_sm_substep = 1;
        if (rc == MPM_OK) {
            const cudaError_t q = variant_occupancy(cap, &per_sm_p2g, &per_sm_substep);
            if (q != cudaSuccess) rc = set_error(MPM_ERR_CUDA, "autotune occupancy failed: %s", cudaGetErrorString(q));
        }
        for (int k = 1; can_fuse && rc == MPM_OK && k <= per_sm_substep; ++k)
            consider(Candidate{true, cap, v0.p2g, v0.g2p, (unsigned)(sms * k), v0.records});
        Candidate four{false, cap, v0.p2g, v0.g2p, v0.substep, v0.records};
        double four_ms = 1e300;
        for (int k = 1; rc == MPM_OK && k <= std::max(1, per_sm_p2g); ++k) {
            const Candidate v{false, cap, std::min(tiles, (unsigned)(sms * k)), v0.g2p, v0.substep, v0.records};
            double ms = 0.0;
            rc = trial(v, ms);
            if (rc == MPM_OK && ms < four_ms) four_ms = ms, four = v;
        }
        for (int k = 1; rc == MPM_OK && k <= std::max(1, per_sm_g2p); ++k) {
            const Candidate v{false, cap, four.p2g, std::min(tiles, (unsigned)(sms * k)), v0.substep, v0.records};
            double ms = 0.0;
            rc = trial(v, ms);
            if (rc == MPM_OK && ms < four_ms) four_ms = ms, four = v;
        }
        // both ways of handing prepareParticle's results to P2G, with the best grids
        for (int r = 0; can_fuse && rc == MPM_OK && r < 2; ++r) {
            const Candidate v{false, cap, four.p2g, four.g2p, v0.substep, r};
            double ms = 0.0;
            rc = trial(v, ms);
            if (rc == MPM_OK && ms < four_ms) four_ms = ms, four = v;
        }
        if (rc == MPM_OK && four_ms < best_ms_total) best_ms_total = four_ms, best = four;
    }
    s->substep_max_ctas = 1;
    {
        int per_sm_p2g = 1, per_sm_substep = 1;
        if (variant_occupancy(rc == MPM_OK ? best.cap : v0.cap, &per_sm_p2g, &per_sm_substep) == cudaSuccess)
            s->substep_max_ctas = (unsigned)std::max(1, sms * per_sm_substep);
    }
    const cudaError_t r = restore();
    if (rc == MPM_OK && r != cudaSuccess) rc = set_error(MPM_ERR_CUDA, "autotune restore failed: %s", cudaGetErrorString(r));
    void *ptrs[] = {save.pos, save.vel, save.C, save.F, save.pvol, save.damage, save.vol, save.mat, save.orig, slots};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    const Candidate &chosen = rc == MPM_OK ? best : v0;
    s->fused = chosen.fused;
    s->stage_cap = chosen.cap;
    s->p2g_ctas = chosen.p2g;
    s->g2p_ctas = chosen.g2p;
    s->substep_ctas = chosen.substep;
    s->records = chosen.records;
    drop_graphs(s);
    s->batch_timed = false;  // the batch events now time the trials
    if (rc != MPM_OK) return rc;
    if (p2g_ctas) *p2g_ctas = best.p2g;
    if (g2p_ctas) *g2p_ctas = best.g2p;
    if (best_ms) *best_ms = best_ms_total / substeps;
    return MPM_OK;
}

const char *mpm_profile_kernel_name(uint32_t slot) { return slot < K_SLOTS ? KERNEL_NAMES[slot] : ""; }

uint32_t mpm_profile_kernel_slots(void) { return K_SLOTS; }

int mpm_count_active_nodes(mpm_solver *s, uint32_t counts[3])
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !counts) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and counts must not be NULL");
    CUDA_TRY(cudaSetDevice(s->device));
    CUDA_TRY(cudaMemsetAsync(s->d_active, 0, 4 * sizeof(uint32_t), s->stream));
    const Ctx c = make_ctx(s, s->cur);
    if (s->gather())  // the ring records of the last substep, every scene
        k_count_ring_nodes<<<s->n_tiles_total, TILE_NODES, 0, s->stream>>>(c, s->d_active);
    else
        k_count_active_nodes<<<dim3(s->tiles_x, s->tiles_y), TILE_NODES, 0, s->stream>>>(c, s->d_active);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(s->h_readback, s->d_active, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    std::memcpy(counts, s->h_readback, 3 * sizeof(uint32_t));
    return MPM_OK;
}

void *mpm_stream(mpm_solver *s) { return s ? (void *)s->stream : nullptr; }

int mpm_read_compact(mpm_solver *s, float *maximum_speed, uint32_t *completed, uint32_t status[8])
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    CUDA_TRY(cudaSetDevice(s->device));
    if (!s->readback_ready) {
        CUDA_TRY(cudaMemcpyAsync(s->h_readback, s->d_counters + COUNTER_PROGRESS, 2 * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(s->h_readback + 2, s->d_status, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 s->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (s->batch_timed && !s->batch_ms_known) {
        // the batch has ended: its time is read now, for mpm_last_batch_device_ms
        CUDA_TRY(cudaEventElapsedTime(&s->batch_ms, s->batch_start, s->batch_stop));
        s->batch_ms_known = true;
    }
    if (completed) *completed = s->h_readback[0];
    if (maximum_speed) *maximum_speed = u2f(s->h_readback[1]);
    if (status) std::memcpy(status, s->h_readback + 2, 8 * sizeof(uint32_t));
    return MPM_OK;
}

int mpm_read_status(mpm_solver *s, uint32_t status[8])
{
    return mpm_read_compact(s, nullptr, nullptr, status);
}

int mpm_clear_status(mpm_solver *s)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    CUDA_TRY(cudaSetDevice(s->device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    // every scene's status words
    std::vector<uint32_t> init_status((size_t)s->n_scenes * 8, 0u);
    for (uint32_t k = 0; k < s->n_scenes; ++k) init_status[(size_t)k * 8 + 1] = 0xffffffffu;
    CUDA_TRY(cudaMemcpy2D(s->dyn, SCENE_WORDS * sizeof(uint32_t), init_status.data(), 8 * sizeof(uint32_t),
                          8 * sizeof(uint32_t), s->n_scenes, cudaMemcpyHostToDevice));
    return MPM_OK;
}

int mpm_read_particles(mpm_solver *s, const uint32_t *indices, uint32_t count, float *packed_out,
                       uint32_t *object_ids_out)
{
    g_last_error.clear();
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (!packed_out) return set_error(MPM_ERR_INVALID_ARGUMENT, "packed_out must not be NULL");
    const uint32_t total = s->allocated;  // original indices, removed ones included
    if (!indices && count != total) return set_error(MPM_ERR_INVALID_ARGUMENT, "count must equal the particle count");
    for (uint32_t k = 0; indices && k < count; ++k)
        if (indices[k] >= total) return set_error(MPM_ERR_INVALID_ARGUMENT, "particleIndices must identify active GPU particles.");
    CUDA_TRY(cudaSetDevice(s->device));
    const uint32_t n = s->n;
    HostState h;
    int rc = download_state(s, h);
    if (rc != MPM_OK) return rc;
    std::vector<uint32_t> bonded(total), obj(total), slot_of(total, 0xffffffffu);
    if (total > 0) {
        CUDA_TRY(cudaMemcpyAsync(bonded.data(), s->bonded, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(obj.data(), s->obj, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    for (uint32_t d = 0; d < n; ++d) {
        if (h.orig[d] >= total) return set_error(MPM_ERR_CUDA, "corrupt particle slot map");
        slot_of[h.orig[d]] = d;
    }
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t i = indices ? indices[k] : k;
        const uint32_t d = slot_of[i];
        float *w = packed_out + (size_t)k * MPM_PARTICLE_WORDS;
        if (object_ids_out) object_ids_out[k] = obj[i];
        if (d == 0xffffffffu) {
            // removed by an outlet: its last state, material model 0xffffffff
            // (MODEL_REMOVED, shaders.ts:195)
            if (i >= s->removed.size() || !s->removed[i]) return set_error(MPM_ERR_CUDA, "corrupt particle slot map");
            std::memcpy(w, s->removed_words.data() + (size_t)i * MPM_PARTICLE_WORDS, MPM_PARTICLE_WORDS * sizeof(float));
            continue;
        }
        const Material &m = s->mats[h.mat[d]];
        w[0] = h.pos[d].x;
        w[1] = h.pos[d].y;
        w[2] = h.vel[d].x;
        w[3] = h.vel[d].y;
        w[4] = h.C[d].x;
        w[5] = h.C[d].y;
        w[6] = h.C[d].z;
        w[7] = h.C[d].w;
        w[8] = h.F[d].x;
        w[9] = h.F[d].y;
        w[10] = h.F[d].z;
        w[11] = h.F[d].w;
        w[12] = h.pvol[d];
        w[13] = u2f(m.model);
        w[14] = m.lambda;
        w[15] = m.mu;
        w[16] = m.density;
        w[17] = h.vol[d];
        w[18] = m.model == MODEL_NEO_HOOKEAN ? h.damage[d] : m.param;
        w[19] = u2f(bonded[i]);
    }
    return MPM_OK;
}

int mpm_write_particles(mpm_solver *s, const float *packed, uint32_t count)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !packed) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and packed_particles must not be NULL");
    if (count != s->n) return set_error(MPM_ERR_INVALID_ARGUMENT, "count must equal the particle count");
    if (s->allocated != s->n) return set_error(MPM_ERR_STATE, "particles were removed; the state cannot be overwritten");
    CUDA_TRY(cudaSetDevice(s->device));
    return unpack_and_upload(s, packed, count, s->cur);
}

int mpm_set_drag(mpm_solver *s, const mpm_drag *drag)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (drag) {
        if (!(drag->radius > 0.0f) || !std::isfinite(drag->radius))
            return set_error(MPM_ERR_INVALID_ARGUMENT, "drag radius must be greater than zero.");
        s->drag = *drag;
        s->drag_active = true;
    } else {
        s->drag_active = false;
    }
    return MPM_OK;
}

int mpm_queue_completion_ms(mpm_solver *s, double *ms)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    CUDA_TRY(cudaSetDevice(s->device));
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    cudaEventRecord(a, s->stream);
    cudaEventRecord(b, s->stream);
    cudaEventSynchronize(b);
    float elapsed = 0.0f;
    cudaEventElapsedTime(&elapsed, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = elapsed;
    return MPM_OK;
}

int mpm_append_particles(mpm_solver *s, const float *packed, const uint32_t *object_ids, uint32_t count,
                         uint32_t *first_index)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || (count > 0 && (!packed || !object_ids)))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "solver, packed_particles and object_ids must not be NULL");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "particles are appended to a single-scene solver");
    if ((uint64_t)s->allocated + count > s->capacity)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "particle slot capacity %u is full", s->capacity);
    for (uint32_t k = 0; k < count; ++k)
        if (f2u(packed[(size_t)k * MPM_PARTICLE_WORDS + 19]) != 0u)
            return set_error(MPM_ERR_INVALID_ARGUMENT,
                             "triangle-bonded particles cannot be appended without a complete object topology");
    if (first_index) *first_index = s->allocated;
    if (count == 0) return MPM_OK;
    CUDA_TRY(cudaSetDevice(s->device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    int rc = unpack_and_upload(s, packed, count, s->cur, s->n, s->allocated);
    if (rc != MPM_OK) return rc;
    CUDA_TRY(cudaMemcpy(s->obj + s->allocated, object_ids, count * sizeof(uint32_t), cudaMemcpyHostToDevice));
    s->allocated += count;
    s->n += count;
    return refresh_count(s);
}

int mpm_remove_particles_in_outlet(mpm_solver *s, float min_x, float min_y, float max_x, float max_y,
                                   uint32_t *removed_count)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "outlets act on a single-scene solver");
    if (!(min_x <= max_x) || !(min_y <= max_y))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "outlet minimum coordinates must not exceed the maximum.");
    if (removed_count) *removed_count = 0;
    if (s->n == 0) return MPM_OK;
    CUDA_TRY(cudaSetDevice(s->device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    const uint32_t n = s->n;
    ParticleBuffers r{};
    uint32_t *counters = nullptr;
    cudaError_t e = dalloc(&r.pos, n);
    if (e == cudaSuccess) e = dalloc(&r.vel, n);
    if (e == cudaSuccess) e = dalloc(&r.C, n);
    if (e == cudaSuccess) e = dalloc(&r.F, n);
    if (e == cudaSuccess) e = dalloc(&r.pvol, n);
    if (e == cudaSuccess) e = dalloc(&r.damage, n);
    if (e == cudaSuccess) e = dalloc(&r.vol, n);
    if (e == cudaSuccess) e = dalloc(&r.mat, n);
    if (e == cudaSuccess) e = dalloc(&r.orig, n);
    if (e == cudaSuccess) e = dalloc(&counters, 2);
    uint32_t h_counts[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), s->stream);
    if (e == cudaSuccess) {
        const Ctx c = make_ctx(s, s->cur);
        k_outlet_compact<<<blocks_for(n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(
            c, make_float4(min_x, min_y, max_x, max_y), r, counters);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_counts, counters, sizeof h_counts, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    const uint32_t removed = h_counts[1];
    std::vector<float2> pos(removed), vel(removed);
    std::vector<float4> C(removed), F(removed);
    std::vector<float> pvol(removed), vol(removed);
    std::vector<uint32_t> mat(removed), orig(removed);
    if (e == cudaSuccess && removed > 0) {
        e = cudaMemcpy(pos.data(), r.pos, removed * sizeof(float2), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(vel.data(), r.vel, removed * sizeof(float2), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(C.data(), r.C, removed * sizeof(float4), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(F.data(), r.F, removed * sizeof(float4), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(pvol.data(), r.pvol, removed * sizeof(float), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(vol.data(), r.vol, removed * sizeof(float), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(mat.data(), r.mat, removed * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(orig.data(), r.orig, removed * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    }
    void *ptrs[] = {r.pos, r.vel, r.C, r.F, r.pvol, r.damage, r.vol, r.mat, r.orig, counters};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "outlet removal failed: %s", cudaGetErrorString(e));
    if (h_counts[0] + removed != n) return set_error(MPM_ERR_CUDA, "outlet removal lost particles");
    // the kept particles are in the other buffer now
    s->cur = 1 - s->cur;
    s->n = h_counts[0];
    if (removed > 0) {
        if (s->removed.size() < s->allocated) {
            s->removed.resize(s->allocated, 0u);
            s->removed_words.resize((size_t)s->allocated * MPM_PARTICLE_WORDS, 0.0f);
        }
        for (uint32_t k = 0; k < removed; ++k) {
            const uint32_t i = orig[k];
            const Material &m = s->mats[mat[k]];
            float *w = s->removed_words.data() + (size_t)i * MPM_PARTICLE_WORDS;
            const float words[MPM_PARTICLE_WORDS] = {pos[k].x, pos[k].y, vel[k].x, vel[k].y, C[k].x, C[k].y,
                                                     C[k].z, C[k].w, F[k].x, F[k].y, F[k].z, F[k].w, pvol[k],
                                                     u2f(0xffffffffu), m.lambda, m.mu, m.density, vol[k], m.param,
                                                     0.0f};
            std::memcpy(w, words, sizeof words);
            s->removed[i] = 1u;
        }
    }
    if (removed_count) *removed_count = removed;
    return refresh_count(s);
}

int mpm_pick(mpm_solver *s, float x, float y, float radius, uint32_t *particle_index, float *anchor_xy,
             uint32_t *object_id)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !particle_index) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and particle_index must not be NULL");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "picking acts on a single-scene solver");
    if (!(radius >= 0.0f) || !std::isfinite(radius))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "pick radius must be non-negative");
    *particle_index = 0xffffffffu;
    if (s->n == 0) return MPM_OK;
    CUDA_TRY(cudaSetDevice(s->device));
    unsigned long long *best = nullptr, h_best = ~0ull;
    CUDA_TRY(dalloc(&best, 1));
    cudaError_t e = cudaMemcpyAsync(best, &h_best, sizeof h_best, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
        const Ctx c = make_ctx(s, s->cur);
        k_pick<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c, x, y, radius * radius, best);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_best, best, sizeof h_best, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(best);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "particle pick failed: %s", cudaGetErrorString(e));
    if (h_best == ~0ull) return MPM_OK;
    const uint32_t index = (uint32_t)(h_best & 0xffffffffull);
    float packed[MPM_PARTICLE_WORDS];
    uint32_t id = 0;
    const int rc = mpm_read_particles(s, &index, 1, packed, &id);
    if (rc != MPM_OK) return rc;
    *particle_index = index;
    if (anchor_xy) {
        anchor_xy[0] = packed[0];
        anchor_xy[1] = packed[1];
    }
    if (object_id) *object_id = id;
    return MPM_OK;
}

int mpm_gather_surface_occupancy(mpm_solver *s, float *field_out, uint32_t *surface_flags_out)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "the surface field belongs to a single-scene solver");
    CUDA_TRY(cudaSetDevice(s->device));
    const uint32_t nodes = s->node_count;
    if (!s->surface_acc) {
        CUDA_TRY(dalloc(&s->surface_acc, 2 * (size_t)nodes));
        CUDA_TRY(dalloc(&s->surface_field, nodes));
    }
    CUDA_TRY(cudaMemsetAsync(s->surface_acc, 0, 2 * (size_t)nodes * sizeof(unsigned long long), s->stream));
    const SurfaceGeometry g{s->cfg.cell_size, s->cfg.cells_x, s->cfg.cells_y, s->node_w};
    if (s->n > 0) {
        const Ctx c = make_ctx(s, s->cur);
        k_surface_gather<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c, g, s->surface_acc);
        CUDA_TRY(cudaGetLastError());
    }
    k_surface_decode<<<blocks_for(nodes, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(s->surface_acc,
                                                                                           s->surface_field, nodes);
    CUDA_TRY(cudaGetLastError());
    if (field_out)
        CUDA_TRY(cudaMemcpyAsync(field_out, s->surface_field, (size_t)nodes * sizeof(float2), cudaMemcpyDeviceToHost,
                                 s->stream));
    if (surface_flags_out)
        CUDA_TRY(cudaMemcpyAsync(surface_flags_out, s->d_status + 7, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

int mpm_surface_field_device(mpm_solver *s, const float **device_field, uint32_t *node_w, uint32_t *node_h)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !device_field) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and device_field must not be NULL");
    if (!s->surface_field) return set_error(MPM_ERR_STATE, "no surface field has been gathered");
    *device_field = reinterpret_cast<const float *>(s->surface_field);
    if (node_w) *node_w = s->node_w;
    if (node_h) *node_h = s->node_h;
    return MPM_OK;
}

int mpm_clone_range(mpm_solver *s, uint32_t start, uint32_t count, float offset_x, float offset_y,
                    uint32_t object_id, uint32_t *first_index)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "cloning acts on a single-scene solver");
    if (!std::isfinite(offset_x) || !std::isfinite(offset_y))
        return set_error(MPM_ERR_INVALID_ARGUMENT, "clone offset must be finite");
    if ((uint64_t)start + count > s->allocated)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "the cloned range must hold allocated particles");
    if (s->allocated != s->n) return set_error(MPM_ERR_STATE, "objects are not cloned after an outlet removed particles");
    if ((uint64_t)s->allocated + count > s->capacity)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "particle slot capacity %u is full", s->capacity);
    if (s->n_bodies > 0 || s->n_bonds > 0)
        return set_error(MPM_ERR_STATE, "scenes with bonded triangle bodies or fracture bonds are not cloned");
    if (first_index) *first_index = s->allocated;
    if (count == 0) return MPM_OK;
    CUDA_TRY(cudaSetDevice(s->device));
    const Ctx c = make_ctx(s, s->cur);
    const float2 domain = make_float2((float)((double)s->cfg.cells_x * (double)s->cfg.cell_size),
                                      (float)((double)s->cfg.cells_y * (double)s->cfg.cell_size));
    k_clone<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(
        c, start, count, make_float2(offset_x, offset_y), domain, s->allocated, object_id);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->allocated += count;
    s->n += count;
    return refresh_count(s);
}

uint32_t mpm_allocated_particle_count(const mpm_solver *s) { return s ? s->allocated : 0u; }

uint32_t mpm_particle_count(const mpm_solver *s) { return s ? s->n : 0u; }
uint32_t mpm_particle_capacity(const mpm_solver *s) { return s ? s->capacity : 0u; }
uint32_t mpm_node_count(const mpm_solver *s) { return s ? s->node_count : 0u; }

void mpm_destroy(mpm_solver *s) { free_solver(s); }

const char *mpm_last_error(void) { return g_last_error.c_str(); }

int mpm_probe_sort(mpm_solver *s, float dt, uint32_t *keys_out, uint32_t *perm_out, uint32_t *cell_start_out)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (!s->gather()) return set_error(MPM_ERR_STATE, "the cell sort runs in gather mode only");
    if (s->n_scenes > 1) return set_error(MPM_ERR_STATE, "the sort probe takes a single-scene solver");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_params(s, dt, 0.0f, 0.0f, nullptr, 0.0f, 1u);
    if (rc != MPM_OK) return rc;
    const Ctx c = make_ctx(s, s->cur);
    enqueue_cell_sort(s, c);
    CUDA_TRY(cudaGetLastError());
    const uint32_t n = s->n;
    std::vector<uint32_t> keys(n), perm(n), orig(n);
    if (n > 0) {
        CUDA_TRY(cudaMemcpyAsync(keys.data(), s->keys, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(perm.data(), s->perm, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(orig.data(), s->buf[s->cur].orig, n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 s->stream));
    }
    if (cell_start_out)
        CUDA_TRY(cudaMemcpyAsync(cell_start_out, s->cell_start, ((size_t)s->node_count + 1) * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    // report by original particle index
    for (uint32_t slot = 0; slot < n; ++slot)
        if (keys_out) keys_out[orig[slot]] = keys[slot];
    for (uint32_t d = 0; d < n; ++d)
        if (perm_out) perm_out[d] = orig[perm[d]];
    return MPM_OK;
}

int mpm_probe_triangle_field(mpm_solver *s, float dt, float *field_out)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s || !field_out) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver and field_out must not be NULL");
    if (!s->field) return set_error(MPM_ERR_STATE, "the scene has no bonded triangle bodies");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_params(s, dt, 0.0f, 0.0f, nullptr, 0.0f, 1u);
    if (rc != MPM_OK) return rc;
    const Ctx c = make_ctx(s, s->cur);
    // the tracked slots of the current buffer, counted as at the start of a
    // batch of one substep
    CUDA_TRY(cudaMemsetAsync(s->d_counters + COUNTER_SUBSTEP, 0, sizeof(uint32_t), s->stream));
    if (s->gather()) enqueue_tile_count(s, c);
    k_triangle_field<<<dim3(s->tiles_x, s->tiles_y), TILE_NODES, 0, s->stream>>>(c);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(field_out, s->field, (size_t)s->node_count * sizeof(TriField), cudaMemcpyDeviceToHost,
                             s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return MPM_OK;
}

int mpm_probe_deformation(int device, const float *F, const float *C, uint32_t count, float dt, float *trial_out,
                          float *increment_out, float *determinant_out, uint32_t *substeps_out, uint32_t *flags_out)
{
    g_last_error.clear();
    if (count == 0) return MPM_OK;
    if (!F || !C || !trial_out || !increment_out || !determinant_out || !substeps_out || !flags_out)
        return set_error(MPM_ERR_INVALID_ARGUMENT, "every array must be given");
    if (!std::isfinite(dt) || dt <= 0.0f) return set_error(MPM_ERR_INVALID_ARGUMENT, "dt must be positive and finite");
    CUDA_TRY(cudaSetDevice(device));
    float4 *dF = nullptr, *dC = nullptr, *dT = nullptr;
    float2 *dI = nullptr;
    uint32_t *dS = nullptr, *dFl = nullptr;
    cudaError_t e = dalloc(&dF, count);
    if (e == cudaSuccess) e = dalloc(&dC, count);
    if (e == cudaSuccess) e = dalloc(&dT, count);
    if (e == cudaSuccess) e = dalloc(&dI, count);
    if (e == cudaSuccess) e = dalloc(&dS, count);
    if (e == cudaSuccess) e = dalloc(&dFl, count);
    if (e == cudaSuccess) e = cudaMemcpy(dF, F, count * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dC, C, count * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_probe_deformation<<<(count + 127u) / 128u, 128>>>(dF, dC, dt, count, dT, dI, dS, dFl);
        e = cudaGetLastError();
    }
    std::vector<float2> inc(count);
    if (e == cudaSuccess) e = cudaMemcpy(trial_out, dT, count * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(inc.data(), dI, count * sizeof(float2), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(substeps_out, dS, count * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(flags_out, dFl, count * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(dF);
    cudaFree(dC);
    cudaFree(dT);
    cudaFree(dI);
    cudaFree(dS);
    cudaFree(dFl);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "deformation probe failed: %s", cudaGetErrorString(e));
    for (uint32_t i = 0; i < count; ++i) {
        increment_out[i] = inc[i].x;
        determinant_out[i] = inc[i].y;
    }
    return MPM_OK;
}

int mpm_probe_fixed_point(mpm_solver *s, float dt, int32_t *words_out, float *affine_out)
{
    g_last_error.clear();
    forget_readback(s);
    if (!s) return set_error(MPM_ERR_INVALID_ARGUMENT, "solver must not be NULL");
    if (s->cfg.p2g_mode != MPM_P2G_FIXED_POINT) return set_error(MPM_ERR_STATE, "the solver was not created in fixed-point mode");
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = upload_params(s, dt, 0.0f, 0.0f, nullptr, 0.0f, 1u);
    if (rc != MPM_OK) return rc;
    float4 *aff = nullptr;
    CUDA_TRY(dalloc(&aff, s->n));
    Ctx c = make_ctx(s, s->cur);
    c.affine_out = aff;
    k_prepare_scatter<<<blocks_for(s->n, PARTICLE_THREADS), PARTICLE_THREADS, 0, s->stream>>>(c);
    cudaError_t e = cudaGetLastError();
    const size_t words = (size_t)s->node_count * FIXED_WORDS;
    if (e == cudaSuccess && words_out)
        e = cudaMemcpyAsync(words_out, s->fixed, words * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && affine_out)
        e = cudaMemcpyAsync(affine_out, aff, (size_t)s->n * sizeof(float4), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->fixed, 0, words * sizeof(int32_t), s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(aff);
    if (e != cudaSuccess) return set_error(MPM_ERR_CUDA, "fixed-point probe failed: %s", cudaGetErrorString(e));
    return MPM_OK;
}

}  // extern "C"
