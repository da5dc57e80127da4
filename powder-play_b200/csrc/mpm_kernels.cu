// mpm_kernels.cu -- sm_100a kernels of one MLS-MPM substep.
//
// Substep, default P2G (the role of the reference's gather path,
// src/lib/mpm/kernels/solver.ts:1465-1570):
//   k_tile_alloc (starts the substep) -> k_tile_scatter -> k_p2g_gather
//   -> k_g2p_tile (grid update + G2P + next substep's tile counts)
//   (k_begin_batch and k_tile_count run once at the start of a batch);
//   or the same four phases in one cooperative launch, k_substep, with grid
//   barriers between them
// The cell sort (k_count, k_scan_*, k_scatter, k_stable_rank) backs the sort
// probe and the allocation-free cell sort.
// Substep, fixed-point atomic P2G (createExperimentalMpmMlsAtomicGpuSolver):
//   k_substep_begin -> k_prepare_scatter -> k_fixed_decode -> k_grid_update
//   -> k_g2p
// After a batch: k_end_batch (rollback, maximum particle speed).
//
// Every kernel returns early once the persistent status word is non-zero, as
// every WGSL entry point does (shaders.ts: `atomicLoad(&stateError[0]) != 0u`).
// A substep that raises it is rolled back (commitParticles,
// shaders.ts:3067-3080): the batch ends on that substep's input, which no
// later substep of the batch writes.
#include <math_constants.h>

#include "mpm_kernels.cuh"

namespace mpm {

namespace {

__device__ __forceinline__ void fail(uint32_t *status, uint32_t flags) { atomicOr(status, flags); }

__device__ __forceinline__ void fail_at(uint32_t *status, uint32_t index, uint32_t flags)
{
    atomicMin(status + 1, index);
    atomicOr(status, flags);
}

__device__ __forceinline__ bool stencil_fits(const StepParams &P, int bx, int by)
{
    // stencilFitsHalo: shaders.ts:511-516
    return bx >= -1 && by >= -1 && bx + 2 <= (int)P.cells_x + 1 && by + 2 <= (int)P.cells_y + 1;
}

__device__ __forceinline__ uint32_t node_index(const StepParams &P, int x, int y)
{
    // gridIndex: shaders.ts:518-520 (x, y are node coordinates, -1 based)
    return (uint32_t)(y + 1) * P.node_w + (uint32_t)(x + 1);
}

__device__ __forceinline__ uint32_t tile_of_node(const StepParams &P, uint32_t hx, uint32_t hy)
{
    return (hy / TILE_Y) * P.tiles_x + hx / TILE_X;
}

// Base cell and fraction of a particle (shaders.ts:1003-1008).
struct Stencil {
    int bx, by;
    float fx, fy;
};

__device__ __forceinline__ bool stencil_from_grid(float gx, float gy, Stencil &s)
{
    if (!finite_f(gx) || !finite_f(gy)) return false;
    float fbx = floorf(__fsub_rn(gx, 0.5f)), fby = floorf(__fsub_rn(gy, 0.5f));
    s.bx = (int)fbx;
    s.by = (int)fby;
    s.fx = __fsub_rn(gx, (float)s.bx);
    s.fy = __fsub_rn(gy, (float)s.by);
    return true;
}

// Grid coordinates by a correctly rounded division (the cell sort probes and
// the fixed-point path, whose CPU emulation divides the same way).
__device__ __forceinline__ bool make_stencil(const StepParams &P, float2 pos, Stencil &s)
{
    return stencil_from_grid(__fdiv_rn(pos.x, P.dx), __fdiv_rn(pos.y, P.dx), s);
}

// Grid coordinates as position * (1 / cellSize), within an ulp of the
// quotient (WGSL's f32 division itself is only specified to 2.5 ulp).  Every
// stencil of the default path -- bucketing, P2G records, G2P -- comes from
// this one formula, so they agree for every particle.
__device__ __forceinline__ bool make_stencil_fast(const StepParams &P, float2 pos, Stencil &s)
{
    return stencil_from_grid(__fmul_rn(pos.x, P.inv_dx), __fmul_rn(pos.y, P.inv_dx), s);
}


// The liquid branch of prepareParticle's stress (shaders.ts:808-963): the
// Tait pressure, or the legacy linear EOS when the exponent is 0.  Returns
// false for invalid material parameters.
__device__ __forceinline__ bool liquid_stress(const Material &m, float det, float tait_pow, float4 &s)
{
    if (!finite_f(m.density) || m.density <= 0.0f || !finite_f(m.lambda) || m.lambda <= 0.0f || !finite_f(m.param) ||
        m.param < 0.0f)
        return false;
    if (m.param > 0.0f) {
        const float pw = tait_pow >= 0.0f ? tait_pow : pow_wgsl(__frcp_rn(det), m.param);
        const float pressure = m.lambda * (pw - 1.0f);
        const float stress = -det * pressure;
        s = make_float4(stress, 0.f, 0.f, stress);
    } else {
        const float pressure = m.lambda * fminf(det - 1.0f, 0.0f);
        s = make_float4(pressure, 0.f, 0.f, pressure);
    }
    return true;
}

// prepareParticle: shaders.ts:808-963.  Computes the per-particle stress
// cache (affine momentum A = m C + (-dt V 4/dx^2) P F^T), mass and current
// liquid area from the particle's state.  Returns 0, or the reference's
// status flags for the failure with `indexed` telling whether the reference
// also reports the particle index.  LIQ: every material of the solver is
// water or oil, so the other models' branches are compiled out.
template <bool LIQ = false>
__device__ __forceinline__ uint32_t prepare_core(const StepParams &P, const Material &m, float4 F, float volume,
                                                 float damage, float pvol, float4 C, float4 &affine, float &mass,
                                                 float &vliq, bool &indexed, float tait_pow = -1.0f)
{
    indexed = true;
    const float det = det2(F);
    if (!finite_f(det) || det <= 0.0f || !finite_f(volume) || volume <= 0.0f) {
        indexed = false;
        return ERROR_DEFORMATION;
    }
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t bad = ERROR_P2G | ERROR_P2G_INVALID_MATERIAL;
    if constexpr (LIQ) {
        if (!liquid_stress(m, det, tait_pow, s)) return bad;
    } else {
        if (m.model == MODEL_NEO_HOOKEAN) {
            if (!finite_f(damage) || damage < 0.0f || damage > 1.0f) return bad;
            const float4 it = make_float4(F.w / det, -F.z / det, -F.y / det, F.x / det);
            const float pressure = m.lambda * logf(det);
            const float4 pk = make_float4(m.mu * (F.x - it.x) + pressure * it.x, m.mu * (F.y - it.y) + pressure * it.y,
                                          m.mu * (F.z - it.z) + pressure * it.z, m.mu * (F.w - it.w) + pressure * it.w);
            const float keep = 1.0f - fminf(fmaxf(damage, 0.0f), 1.0f);
            s = make_float4((pk.x * F.x + pk.y * F.y) * keep, (pk.x * F.z + pk.y * F.w) * keep,
                            (pk.z * F.x + pk.w * F.y) * keep, (pk.z * F.z + pk.w * F.w) * keep);
        } else if (m.model == MODEL_SNOW || m.model == MODEL_FIXED_COROTATED) {
            float hardening = 1.0f;
            if (m.model == MODEL_SNOW) {
                if (!finite_f(pvol) || pvol < SNOW_MIN_PLASTIC_VOLUME || pvol > SNOW_MAX_PLASTIC_VOLUME) return bad;
                const float e = fminf(fmaxf(SNOW_HARDENING * (1.0f - pvol), -SNOW_MAX_HARDENING_EXPONENT),
                                      SNOW_MAX_HARDENING_EXPONENT);
                hardening = expf(e);
            }
            const Decomp d = decompose(F);
            if (!finite_f(d.s0) || !finite_f(d.s1) || d.s0 <= 0.0f || d.s1 <= 0.0f) return bad;
            const float4 R = polar_rotation(d);
            const float mu = m.mu * hardening, lambda = m.lambda * hardening;
            const float4 diff = make_float4(F.x - R.x, F.y - R.y, F.z - R.z, F.w - R.w);
            const float shear = 2.0f * mu;
            const float volumetric = lambda * det * (det - 1.0f);
            s = make_float4(shear * (diff.x * F.x + diff.y * F.y) + volumetric, shear * (diff.x * F.z + diff.y * F.w),
                            shear * (diff.z * F.x + diff.w * F.y), shear * (diff.z * F.z + diff.w * F.w) + volumetric);
        } else if (m.model == MODEL_WATER || m.model == MODEL_OIL) {
            if (!liquid_stress(m, det, tait_pow, s)) return bad;
        } else if (m.model == MODEL_POWDER) {
            if (!finite_f(m.lambda) || !finite_f(m.mu) || m.mu <= 0.0f || !finite_f(m.param) || m.param < 0.0f)
                return bad;
            // granularStressTimesFt: shaders.ts:408-441
            const Decomp d = decompose(F);
            const float l0 = logf(d.s0), l1 = logf(d.s1);
            const float lv = l0 + l1;
            const float blv = fmaxf(logf(MIN_POWDER_DETERMINANT), lv);
            const float pressure = fmaxf(0.0f, -(m.lambda + m.mu) * blv);
            const float dev = 0.5f * (l0 - l1);
            const float maxdev = m.param * pressure / (2.0f * m.mu);
            const float pdev = fminf(dev, maxdev);
            const float mean = 0.5f * lv;
            const float p0 = 2.0f * m.mu * (mean + pdev) + m.lambda * lv;
            const float p1 = 2.0f * m.mu * (mean - pdev) + m.lambda * lv;
            s = make_float4(p0 * d.u0.x * d.u0.x + p1 * d.u1.x * d.u1.x, p0 * d.u0.x * d.u0.y + p1 * d.u1.x * d.u1.y,
                            p0 * d.u0.y * d.u0.x + p1 * d.u1.y * d.u1.x, p0 * d.u0.y * d.u0.y + p1 * d.u1.y * d.u1.y);
        } else {
            return bad;
        }
    }
    const bool liquid = LIQ || m.model == MODEL_WATER || m.model == MODEL_OIL;
    mass = liquid ? __fmul_rn(m.density, volume) : P.particle_mass;
    vliq = liquid ? __fmul_rn(volume, det) : 0.0f;
    const float scale = -P.dt * volume * P.gradient_scale;
    affine = make_float4(mass * C.x + scale * s.x, mass * C.y + scale * s.y, mass * C.z + scale * s.z,
                         mass * C.w + scale * s.w);
    if (!finite4(s) || !finite4(affine)) return ERROR_P2G | ERROR_P2G_NONFINITE_PARTICLE;
    return 0u;
}

// prepareParticle for the particle in slot i, raising its status on failure.
__device__ bool prepare_particle(const Ctx &c, uint32_t i, float4 &affine, float &mass, float &vliq,
                                 uint32_t &model)
{
    const Material m = c.mats[c.in.mat[i]];
    model = m.model;
    const float damage = m.model == MODEL_NEO_HOOKEAN ? c.in.damage[i] : 0.0f;
    const float pvol = m.model == MODEL_SNOW ? c.in.pvol[i] : 1.0f;
    bool indexed;
    const uint32_t flags =
        prepare_core(*c.P, m, c.in.F[i], c.in.vol[i], damage, pvol, c.in.C[i], affine, mass, vliq, indexed);
    if (flags == 0u) return true;
    if (indexed)
        fail_at(c.status, c.in.orig[i], flags);
    else
        fail(c.status, flags);
    return false;
}

// The context of scene s: its parameters, status and counters.
__device__ __forceinline__ Ctx scene_ctx(const Ctx &c, uint32_t s)
{
    Ctx cs = c;
    cs.P = c.scenes + s;
    cs.status = c.dyn + (size_t)s * SCENE_WORDS;
    cs.counters = c.dyn + (size_t)s * SCENE_WORDS + 32;
    return cs;
}

// The scene owning slot d (scenes hold contiguous slot ranges).
__device__ __forceinline__ uint32_t scene_of_slot(const Ctx &c, uint32_t d)
{
    uint32_t lo = 0, hi = c.n_scenes;  // scene_p_base[lo] <= d < scene_p_base[hi]
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if (c.scene_p_base[mid] <= d)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// The context of a tile's scene (SCENES: the solver holds several).
template <bool SCENES>
__device__ __forceinline__ Ctx tile_ctx(const Ctx &c0, uint32_t tile)
{
    if constexpr (SCENES)
        return scene_ctx(c0, c0.tile_scene[tile]);
    else
        return c0;
}

// The substep's listed tiles: the heavy ones (more particles than a stage)
// first, from the end of the list array, then the light ones from its start.
__device__ __forceinline__ uint32_t listed_count(const Ctx &c)
{
    return __ldcg(c.work + WORK_ACTIVE + c.parity) + __ldcg(c.work + WORK_HEAVY + c.parity);
}

__device__ __forceinline__ uint32_t heavy_count(const Ctx &c) { return __ldcg(c.work + WORK_HEAVY + c.parity); }

__device__ __forceinline__ const uint32_t *listed_tile(const Ctx &c, uint32_t item, uint32_t heavy)
{
    return item < heavy ? c.active_tiles + (c.n_tiles - 1u - item) : c.active_tiles + (item - heavy);
}

// Whether the scene takes part in the current substep: no status raised and
// substeps of this batch left.
__device__ __forceinline__ bool takes_part(const Ctx &c)
{
    return *(volatile uint32_t *)c.status == 0u && c.counters[COUNTER_SUBSTEP] < c.P->batch_steps;
}

// The start of a substep (one thread): a new tile stamp, the substep index,
// and, once the state stops taking part, the substeps completed (a status
// raised in the previous substep leaves that substep's input, the state after
// the substeps before it, as the result).  Returns whether the substep runs.
__device__ __forceinline__ bool begin_substep(const Ctx &c)
{
    uint32_t *k = c.counters;
    k[COUNTER_STAMP] += 1u;
    if (k[COUNTER_FRESH] != 0u)
        k[COUNTER_FRESH] = 0u;
    else
        k[COUNTER_SUBSTEP] += 1u;
    const uint32_t sub = k[COUNTER_SUBSTEP];
    const bool failed = *(volatile uint32_t *)c.status != 0u;
    const bool runs = !failed && sub < c.P->batch_steps;
    if (!runs && k[COUNTER_STOP] == STOP_NONE) k[COUNTER_STOP] = failed ? (sub == 0u ? 0u : sub - 1u) : c.P->batch_steps;
    return runs;
}

// begin_substep's answer without its effects: whether the scene runs the
// substep about to start, from the counters and status as they are before it.
__device__ __forceinline__ bool substep_runs(const Ctx &c)
{
    const uint32_t *k = c.counters;
    const uint32_t sub = k[COUNTER_FRESH] != 0u ? k[COUNTER_SUBSTEP] : k[COUNTER_SUBSTEP] + 1u;
    return *(volatile uint32_t *)c.status == 0u && sub < c.P->batch_steps;
}

// Substeps completed in a batch of `total` substeps, at its end (the same
// answer however often it is asked).
__device__ __forceinline__ uint32_t batch_stop(const Ctx &c, uint32_t total)
{
    const uint32_t *k = c.counters;
    const uint32_t stop = k[COUNTER_STOP];
    if (stop != STOP_NONE) return stop;
    if (k[COUNTER_FRESH] != 0u) return 0u;  // no substep started
    // it ran the last substep, total - 1
    return *(volatile uint32_t *)c.status != 0u ? total - 1u : total;
}

// Whether the slot of original particle `orig` is tracked (a bonded-triangle
// vertex or a fracture-bond endpoint).
__device__ __forceinline__ bool is_tracked(const Ctx &c, uint32_t orig)
{
    return c.track_flag != nullptr && c.track_flag[orig] != 0u;
}

// Writes the P2G record of slot d for a particle with the given state and
// base stencil (the next substep's prepareParticle, evaluated early; the
// records variant).  A failure is kept in the record and raised by the P2G
// that reads it, so the status appears in the same substep as in the
// reference.
template <bool LIQ = false>
__device__ __forceinline__ void write_record(const Ctx &c, uint32_t d, const Material &m, const Stencil &st,
                                             float2 vel, float4 F, float volume, float damage, float pvol, float4 C,
                                             float tait_pow = -1.0f)
{
    float4 A;
    float mass, vliq;
    bool indexed;
    const uint32_t flags = prepare_core<LIQ>(*c.P, m, F, volume, damage, pvol, C, A, mass, vliq, indexed, tait_pow);
    const uint32_t lx = (uint32_t)(st.bx + 1) % TILE_X, ly = (uint32_t)(st.by + 1) % TILE_Y;
    const uint32_t ch = m.model == MODEL_WATER ? 1u : (LIQ || m.model == MODEL_OIL ? 2u : 0u);
    uint32_t cell = (ly * TILE_X + lx) | (ch << 8);
    if (flags != 0u) {
        c.rec_state[d] = make_float4(__uint_as_float(flags), __uint_as_float(indexed ? 1u : 0u), 0.f, 0.f);
        cell |= REC_FAILED;
    } else {
        c.rec_state[d] = make_float4(st.fx, st.fy, mass, vliq);
        c.rec_affine[d] = A;
        c.rec_mom[d] = make_float2(mass * vel.x, mass * vel.y);
    }
    c.rec_cell[d] = cell;
}

template <int N>
__device__ __forceinline__ void cp_async(void *dst, const void *src)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if (N == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim multiple of 32).
template <int THREADS, class T = uint32_t>
__device__ __forceinline__ T block_exclusive_scan(T v, T &total)
{
    __shared__ T warp_totals[THREADS / 32];
    __shared__ T s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += n;
    }
    if (lane == 31) warp_totals[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < THREADS / 32 ? warp_totals[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T n = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += n;
        }
        if (lane < THREADS / 32) warp_totals[lane] = wi - w;
    }
    __syncthreads();
    const T warp_offset = warp_totals[warp];
    if (threadIdx.x == THREADS - 1) s_total = warp_offset + inc;
    __syncthreads();
    total = s_total;
    return warp_offset + inc - v;
}

// Adds one to the cell count of `key` for every active lane, one atomic per
// distinct key in the warp; returns this lane's rank among the cell's
// particles counted so far (ranks are made stable later).
__device__ __forceinline__ uint32_t warp_count(uint32_t *cell_count, uint32_t key, unsigned active)
{
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(&cell_count[key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

}  // namespace

// ---------------------------------------------------------------- batch --

// Resets every scene's per-batch counters (reference: cflStepProgress write
// before the batch, solver.ts:1444-1450; the speed scalar is recomputed
// after it) and the tile lists.
__global__ void k_begin_batch(Ctx c, uint32_t reset_progress)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < c.n_scenes; s += gridDim.x * blockDim.x) {
        uint32_t *counters = c.dyn + (size_t)s * SCENE_WORDS + 32;
        if (reset_progress) counters[COUNTER_PROGRESS] = 0u;
        counters[COUNTER_MAX_SPEED] = 0u;
        counters[COUNTER_SUBSTEP] = 0u;
        counters[COUNTER_FRESH] = 1u;
        counters[COUNTER_STOP] = STOP_NONE;
        counters[COUNTER_CURSOR] = c.scenes[s].p_base;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.work[WORK_ACTIVE] = 0u;
        c.work[WORK_ACTIVE + 1] = 0u;
        c.work[WORK_HEAVY] = 0u;
        c.work[WORK_HEAVY + 1] = 0u;
        c.work[WORK_BARRIER] = 0u;  // an abandoned launch may have left arrivals
        c.work[WORK_ABORT] = 0u;
    }
}

// ----------------------------------------------------------- cell sort --

// Base-cell key and rank within the cell of the particle in each slot;
// replaces the per-node linked lists of insertParticleBucket
// (shaders.ts:657-693).  Runs at the start of a batch; later substeps get
// their counts from the previous G2P.
__global__ void k_count(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < P.n_particles && *(volatile uint32_t *)c.status == 0u;
    uint32_t key = 0;
    if (valid) {
        Stencil s;
        if (!make_stencil(P, c.in.pos[i], s) || !stencil_fits(P, s.bx, s.by)) {
            fail(c.status, ERROR_STENCIL);
            valid = false;
        } else {
            key = node_index(P, s.bx, s.by);
        }
    }
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    c.ranks[i] = warp_count(c.cell_count, key, active);
    c.keys[i] = key;
}

// Exclusive scan of the dense cell counts in three launches; the counts are
// zeroed on the way for the next substep.  These kernels ignore the status
// word so that counts never survive into a later batch.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(Ctx c, uint32_t n_chunks)
{
    const uint32_t chunk = blockIdx.x;
    const uint4 *src = reinterpret_cast<const uint4 *>(c.cell_count + (size_t)chunk * SCAN_CHUNK);
    const uint4 a = src[threadIdx.x * 2], b = src[threadIdx.x * 2 + 1];
    uint32_t v = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
    v = warp_sum(v);
    __shared__ uint32_t partial[SCAN_THREADS / 32];
    if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t w = threadIdx.x < SCAN_THREADS / 32 ? partial[threadIdx.x] : 0u;
        w = warp_sum(w);
        if (threadIdx.x == 0) c.block_sums[chunk] = w;
    }
}

__global__ void __launch_bounds__(SCAN_TOP_THREADS) k_scan_top(Ctx c, uint32_t n_chunks)
{
    // one CTA; each thread owns a contiguous run of chunk sums
    const uint32_t per = (n_chunks + SCAN_TOP_THREADS - 1) / SCAN_TOP_THREADS;
    const uint32_t begin = threadIdx.x * per;
    uint32_t local = 0;
    for (uint32_t k = 0; k < per; ++k) {
        const uint32_t idx = begin + k;
        if (idx < n_chunks) local += c.block_sums[idx];
    }
    uint32_t total;
    uint32_t offset = block_exclusive_scan<SCAN_TOP_THREADS>(local, total);
    for (uint32_t k = 0; k < per; ++k) {
        const uint32_t idx = begin + k;
        if (idx < n_chunks) {
            const uint32_t v = c.block_sums[idx];
            c.block_sums[idx] = offset;
            offset += v;
        }
    }
    if (threadIdx.x == 0) c.block_sums[n_chunks] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(Ctx c, uint32_t n_chunks)
{
    const uint32_t chunk = blockIdx.x;
    uint4 *src = reinterpret_cast<uint4 *>(c.cell_count + (size_t)chunk * SCAN_CHUNK);
    uint4 a = src[threadIdx.x * 2], b = src[threadIdx.x * 2 + 1];
    const uint32_t local = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
    uint32_t total;
    uint32_t run = block_exclusive_scan<SCAN_THREADS>(local, total) + c.block_sums[chunk];
    uint32_t out[8];
    const uint32_t in[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        out[k] = run;
        run += in[k];
    }
    uint4 *dst = reinterpret_cast<uint4 *>(c.cell_start + (size_t)chunk * SCAN_CHUNK);
    dst[threadIdx.x * 2] = make_uint4(out[0], out[1], out[2], out[3]);
    dst[threadIdx.x * 2 + 1] = make_uint4(out[4], out[5], out[6], out[7]);
    src[threadIdx.x * 2] = make_uint4(0, 0, 0, 0);
    src[threadIdx.x * 2 + 1] = make_uint4(0, 0, 0, 0);
    if (chunk == n_chunks - 1 && threadIdx.x == 0) c.cell_start[(size_t)n_chunks * SCAN_CHUNK] = c.block_sums[n_chunks];
}

__global__ void k_scatter(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    c.tmp[c.cell_start[c.keys[i]] + c.ranks[i]] = i;
}

// Stable order within each cell: ascending original particle index, so the
// sorted order is a pure function of (cell key, original index) -- a stable
// counting sort of the particles in their original order.
__global__ void k_stable_rank(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    const uint32_t s = c.tmp[j];
    const uint32_t key = c.keys[s];
    const uint32_t id = c.in.orig[s];
    const uint32_t lo = c.cell_start[key], hi = c.cell_start[key + 1];
    uint32_t rank = 0;
    for (uint32_t t = lo; t < hi; ++t) rank += c.in.orig[c.tmp[t]] < id ? 1u : 0u;
    c.perm[lo + rank] = s;
}

// ----------------------------------------------- fused gather P2G + grid --

namespace {

__device__ __forceinline__ float2 finish_velocity(const StepParams &P, float mass, float px, float py, int x, int y)
{
    // finishGridVelocity: shaders.ts:1748-1777
    if (mass <= 0.0f) return make_float2(0.f, 0.f);
    const float inv = __frcp_rn(mass);
    float2 vel = make_float2(px * inv + P.dt * P.gx, py * inv + P.dt * P.gy);
    if (P.drag_radius > 0.0f && x >= 0 && y >= 0 && x <= (int)P.cells_x && y <= (int)P.cells_y) {
        const float nx = (float)x * P.dx, ny = (float)y * P.dx;
        const float ddx = P.drag_x - nx, ddy = P.drag_y - ny;
        const float dist = sqrtf(ddx * ddx + ddy * ddy);
        if (dist < P.drag_radius) {
            const float falloff = 1.0f - dist / P.drag_radius;
            const float ax = ddx * P.drag_stiffness - vel.x * P.drag_damping;
            const float ay = ddy * P.drag_stiffness - vel.y * P.drag_damping;
            vel.x += P.dt * falloff * ax;
            vel.y += P.dt * falloff * ay;
        }
    }
    return vel;
}

// Per-channel node velocities G2P reads: solid (vx, vy); water and oil
// (vx, vy, liquid mass, liquid volume).
struct NodeVel {
    float2 vs;
    float4 vw, vo;
    float2 impulse;  // the fluid's impulse on a nearby body (zero without one)
};

// The node update of updateGrid (shaders.ts:1485-1746) for one node given its
// P2G sums and the water/oil volumes of its four neighbours (xp, xm, yp, ym;
// zero outside the halo or where no particle deposited).  Returns false
// after raising a status.  LIQ: the solver holds no solid particle, so the
// solid channel (its sums are zero) is not evaluated and its velocity is 0.
// near_wall false: the caller knows the node lies at least one wall cushion
// from every wall, where the cushion and the friction leave velocities as
// they are, so they are not evaluated.
template <bool BODIES, bool LIQ = false>
__device__ __forceinline__ bool node_velocity(const Ctx &c, uint32_t n, int x, int y, float4 S, float4 W, float4 O,
                                              float2 xp, float2 xm, float2 yp, float2 ym, NodeVel &out,
                                              bool near_wall = true)
{
    const StepParams &P = *c.P;
    if ((!LIQ && (!finite_f(S.x) || S.x < 0.f || !finite_f(S.y) || !finite_f(S.z))) || !finite_f(W.x) || W.x < 0.f ||
        !finite_f(W.y) || !finite_f(W.z) || !finite_f(W.w) || W.w < 0.f || !finite_f(O.x) || O.x < 0.f ||
        !finite_f(O.y) || !finite_f(O.z) || !finite_f(O.w) || O.w < 0.f) {
        fail(c.status, ERROR_GRID);
        return false;
    }
    float2 vs = LIQ ? make_float2(0.f, 0.f) : finish_velocity(P, S.x, S.y, S.z, x, y);
    float2 vw = finish_velocity(P, W.x, W.y, W.z, x, y);
    float2 vo = finish_velocity(P, O.x, O.y, O.z, x, y);
    if (x >= 0 && y >= 0 && x <= (int)P.cells_x && y <= (int)P.cells_y && W.x > 0.f && O.x > 0.f && W.w > 0.f &&
        O.w > 0.f) {
        // phaseVolumeGradient (shaders.ts:1779-1799): unscaled central differences
        const float2 wgrad = make_float2(xp.x - xm.x, yp.x - ym.x);
        const float2 ograd = make_float2(xp.y - xm.y, yp.y - ym.y);
        const float2 sep = make_float2(ograd.x - wgrad.x, ograd.y - wgrad.y);
        const float sl = sqrtf(sep.x * sep.x + sep.y * sep.y);
        if (finite_f(sl) && sl > 1e-8f) {
            const float isl = __frcp_rn(sl);
            float2 nrm = make_float2(sep.x * isl, sep.y * isl);
            const float wd = __fdividef(W.x, W.w), od = __fdividef(O.x, O.w);
            const float ds = fmaxf(wd, od);
            const float contrast = __fdividef(od - wd, ds);
            const float gm = sqrtf(P.gx * P.gx + P.gy * P.gy);
            float align = 0.f;
            if (!finite_f(wd) || wd <= 0.f || !finite_f(od) || od <= 0.f || !finite_f(contrast) || !finite_f(gm)) {
                fail(c.status, ERROR_GRID);
                return false;
            }
            if (gm > 0.f) align = __fdividef(nrm.x * P.gx + nrm.y * P.gy, gm);
            if (!finite_f(align)) {
                fail(c.status, ERROR_GRID);
                return false;
            }
            if (contrast * align < -LIQUID_STABLE_ORDER_EPSILON) nrm = make_float2(-nrm.x, -nrm.y);
            const float rel = (vo.x - vw.x) * nrm.x + (vo.y - vw.y) * nrm.y;
            const float overlap = fminf(fmaxf(__fdividef(2.0f * fminf(W.w, O.w), W.w + O.w), 0.f), 1.f);
            const float minsep = fmaxf(LIQUID_CONTACT_SEPARATION_FRACTION * overlap * P.dx / LIQUID_CONTACT_RELAXATION_SECONDS,
                                       fmaxf(-rel, 0.f) * LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER);
            if (rel < minsep) {
                const float iwm = __frcp_rn(W.x), iom = __frcp_rn(O.x);
                const float mag = __fdividef(minsep - rel, iwm + iom);
                const float ix = mag * nrm.x, iy = mag * nrm.y;
                vw = make_float2(vw.x - ix * iwm, vw.y - iy * iwm);
                vo = make_float2(vo.x + ix * iom, vo.y + iy * iom);
            }
        }
    }
    float2 impulse = make_float2(0.f, 0.f);
    if (BODIES && c.field) {
        // fluid-pebble contact: updateGrid, shaders.ts:1596-1665
        const TriField f = c.field[n];
        if (f.body1 != 0u && f.sd <= P.contact_reach) {
            const uint32_t start = f.body1 - 1u;
            if (start + 2u >= P.n_particles) {
                fail(c.status, ERROR_TRIANGLE_CONTACT);
                return false;
            }
            const float3 bary = make_float3(1.0f - f.b1 - f.b2, f.b1, f.b2);
            const float2 v0 = c.in.vel[c.slot_in[start]], v1 = c.in.vel[c.slot_in[start + 1u]],
                         v2 = c.in.vel[c.slot_in[start + 2u]];
            const float2 sv = make_float2(bary.x * v0.x + bary.y * v1.x + bary.z * v2.x,
                                          bary.x * v0.y + bary.y * v1.y + bary.z * v2.y);
            const float inv_body = (bary.x * bary.x + bary.y * bary.y + bary.z * bary.z) / P.particle_mass;
            const float nl = sqrtf(f.nx * f.nx + f.ny * f.ny);
            if (!finite2(sv) || !finite_f(inv_body) || inv_body <= 0.f || !finite_f(nl) || nl <= 1e-8f) {
                fail(c.status, ERROR_TRIANGLE_CONTACT);
                return false;
            }
            const float2 nrm = make_float2(f.nx / nl, f.ny / nl);
            const float damping = 1.0f - expf(-TRIANGLE_FLUID_TANGENTIAL_DRAG_RATE * P.dt);
            if (W.x > 0.f && W.w > 0.f) {
                const float2 rel = make_float2(vw.x - sv.x, vw.y - sv.y);
                const float rn = rel.x * nrm.x + rel.y * nrm.y;
                const float iem = 1.0f / W.x + inv_body;
                float2 imp = make_float2(0.f, 0.f);
                if (rn < 0.f) imp = make_float2((-rn / iem) * nrm.x, (-rn / iem) * nrm.y);
                const float2 tv = make_float2(rel.x - rn * nrm.x, rel.y - rn * nrm.y);
                imp = make_float2(imp.x - (damping / iem) * tv.x, imp.y - (damping / iem) * tv.y);
                vw = make_float2(vw.x + imp.x / W.x, vw.y + imp.y / W.x);
                impulse = make_float2(impulse.x - imp.x, impulse.y - imp.y);
            }
            if (O.x > 0.f && O.w > 0.f) {
                const float2 rel = make_float2(vo.x - sv.x, vo.y - sv.y);
                const float rn = rel.x * nrm.x + rel.y * nrm.y;
                const float iem = 1.0f / O.x + inv_body;
                float2 imp = make_float2(0.f, 0.f);
                if (rn < 0.f) imp = make_float2((-rn / iem) * nrm.x, (-rn / iem) * nrm.y);
                const float2 tv = make_float2(rel.x - rn * nrm.x, rel.y - rn * nrm.y);
                imp = make_float2(imp.x - (damping / iem) * tv.x, imp.y - (damping / iem) * tv.y);
                vo = make_float2(vo.x + imp.x / O.x, vo.y + imp.y / O.x);
                impulse = make_float2(impulse.x - imp.x, impulse.y - imp.y);
            }
        }
    }
    if ((!LIQ && !finite2(vs)) || !finite2(vw) || !finite2(vo) || !finite2(impulse)) {
        fail(c.status, ERROR_GRID | ERROR_TRIANGLE_CONTACT);
        return false;
    }
    if (near_wall) {
        const int cx = (int)P.cells_x, cy = (int)P.cells_y;
        const float fr = P.wall_friction;
        if (!LIQ) {
            vs.x = wall_cushion(vs.x, x, cx);
            vs.y = wall_cushion(vs.y, y, cy);
        }
        vw.x = wall_cushion(vw.x, x, cx);
        vw.y = wall_cushion(vw.y, y, cy);
        vo.x = wall_cushion(vo.x, x, cx);
        vo.y = wall_cushion(vo.y, y, cy);
        if (!LIQ) {
            vs.x = wall_friction(vs.x, y, cy, fr);
            vs.y = wall_friction(vs.y, x, cx, fr);
        }
        vw.x = wall_friction(vw.x, y, cy, fr);
        vw.y = wall_friction(vw.y, x, cx, fr);
        vo.x = wall_friction(vo.x, y, cy, fr);
        vo.y = wall_friction(vo.y, x, cx, fr);
    }
    const float lm = W.x + O.x, lv = W.w + O.w;
    out.vs = vs;
    out.vw = make_float4(vw.x, vw.y, lm, lv);
    out.vo = make_float4(vo.x, vo.y, lm, lv);
    out.impulse = impulse;
    return true;
}

// node_velocity stored to the global velocity grid (fixed-point path).
__device__ bool update_node(const Ctx &c, uint32_t n, int x, int y, float4 S, float4 W, float4 O, float2 xp,
                            float2 xm, float2 yp, float2 ym)
{
    NodeVel v;
    if (!node_velocity<true>(c, n, x, y, S, W, O, xp, xm, yp, ym, v)) return false;
    c.g_solid[n] = v.vs;
    c.g_water[n] = v.vw;
    c.g_oil[n] = v.vo;
    if (c.field) {
        c.field[n].ix = v.impulse.x;
        c.field[n].iy = v.impulse.y;
    }
    return true;
}

}  // namespace

// ---------------------------------------------------- tile buckets + P2G --

// The tile (16x8 nodes) that holds a particle's base node; its 3x3 stencil
// then lies in the tile's 18x10-node ring (tile plus two columns and rows).
__device__ __forceinline__ uint32_t particle_tile(const StepParams &P, int bx, int by)
{
    return P.tile_base + tile_of_node(P, (uint32_t)(bx + 1), (uint32_t)(by + 1));
}

// The bucket key stored per slot: the particle's tile in the low 24 bits and
// its base node's cell within the tile in the top 8 (P2G's crowded path
// orders a tile's entries by that cell without recomputing the stencil).
__device__ __forceinline__ uint32_t bucket_key(uint32_t tile, int bx, int by)
{
    const uint32_t cell = ((uint32_t)(by + 1) % TILE_Y) * TILE_X + (uint32_t)(bx + 1) % TILE_X;
    return tile | (cell << KEY_CELL_SHIFT);
}

// Batch prologue of the default path: tile key and rank within the tile of
// the particle in each slot, and with the records variant its P2G record
// (later substeps get them from G2P).
__global__ void k_tile_count(Ctx c0)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const Ctx c = scene_ctx(c0, c0.n_scenes == 1u || i >= c0.n ? 0u : scene_of_slot(c0, i));
    const StepParams &P = *c.P;
    bool valid;
    if (c0.n_scenes == 1u) {
        // one scene: whether it takes part, read once per CTA
        __shared__ int s_part;
        if (threadIdx.x == 0) s_part = takes_part(c) ? 1 : 0;
        __syncthreads();
        valid = i < c0.n && s_part != 0;
    } else {
        valid = i < c0.n && takes_part(c);
    }
    uint32_t tile = 0, key = 0;
    if (valid) {
        const float2 pos = c.in.pos[i];
        const uint32_t orig = c.in.orig[i];
        Stencil s;
        if (!make_stencil_fast(P, pos, s) || !stencil_fits(P, s.bx, s.by)) {
            fail(c.status, ERROR_STENCIL);
            valid = false;
        } else {
            tile = particle_tile(P, s.bx, s.by);
            key = bucket_key(tile, s.bx, s.by);
            if (is_tracked(c, orig)) c.slot_in[orig] = i;
            if (c.rec_state) {
                // the records variant: the first substep's P2G records
                const float2 vel = c.in.vel[i];
                const float4 F = c.in.F[i], C = c.in.C[i];
                const float vol = c.in.vol[i], damage_in = c.in.damage[i], pvol_in = c.in.pvol[i];
                const Material m = c.mats[c.in.mat[i]];
                const float damage = m.model == MODEL_NEO_HOOKEAN ? damage_in : 0.0f;
                const float pvol = m.model == MODEL_SNOW ? pvol_in : 1.0f;
                write_record(c, i, m, s, vel, F, vol, damage, pvol, C);
            }
        }
    }
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    c.ranks[i] = warp_count(c.tile_count, tile, active);
    c.keys[i] = key;
}

// The scene of allocation CTA b: scene_chunk[scene] <= b < scene_chunk[scene + 1].
__device__ __forceinline__ uint32_t scene_of_chunk(const Ctx &c, uint32_t b)
{
    uint32_t lo = 0, hi = c.n_scenes;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if (c.scene_chunk[mid] <= b)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Whether scene `scene` takes part in the substep under way, as k_tile_alloc
// found it (read while k_tile_scatter starts the substep).
__device__ __forceinline__ bool runs_flag(const Ctx &c, uint32_t scene)
{
    return __ldcg(c.dyn + (size_t)scene * SCENE_WORDS + 32 + COUNTER_RUNS) != 0u;
}

// The first kernel of a substep of the default path: each CTA takes 1024
// consecutive tiles of one scene (4 per thread, vector loads and stores),
// and, when the scene runs the substep, gives each of its tiles holding
// particles a range of the scene's bucket entries -- one atomic per CTA on
// the scene's cursor, so the ranges of different CTAs lie in the order the
// CTAs got there -- and a place in the substep's tile list (one atomic per
// CTA on the list size), and zeroes the counts for the next substep.  Every
// CTA reads whether the scene runs (substep_runs) and stores the answer in
// the scene's counters; k_tile_scatter then starts the substep
// (begin_substep) and resets the cursor.  A scene that does not take part
// lists no tile (the counts are cleared at the start of every batch).  CTA
// 0 empties the tile list of the next substep (the other buffer parity).
// Neither the order of the bucket ranges nor that of the list changes any
// sum: P2G orders each tile's particles by cell, channel and original index.
// Allocation chunk b (1024 tiles of one scene) with ALLOC_THREADS threads.
__device__ __forceinline__ void alloc_chunk(const Ctx &c0, uint32_t b)
{
    __shared__ uint32_t s_base[3];
    __shared__ bool s_runs;
    const bool one_scene = c0.n_scenes == 1u;
    const uint32_t scene = one_scene ? 0u : scene_of_chunk(c0, b);
    const uint32_t chunk = one_scene ? b : b - c0.scene_chunk[scene];
    const Ctx c = scene_ctx(c0, scene);
    const StepParams &P = *c.P;
    __syncthreads();  // the previous chunk's readers of s_base and s_runs are done
    if (threadIdx.x == 0) {
        const bool runs = substep_runs(c);
        s_runs = runs;
        c.counters[COUNTER_RUNS] = runs ? 1u : 0u;  // the same value from every CTA of the scene
        if (b == 0) {
            // the next substep's lists start empty; this substep's tile claims start at 0
            c0.work[WORK_ACTIVE + (c0.parity ^ 1u)] = 0u;
            c0.work[WORK_HEAVY + (c0.parity ^ 1u)] = 0u;
            c0.work[WORK_CLAIM] = 0u;
            c0.work[WORK_CLAIM + 1] = 0u;
        }
    }
    // the counts are read before the answer is known (they exist either way)
    uint32_t *count = c.tile_count + P.tile_base;  // 32-byte aligned: scenes start on 8-tile boundaries
    const uint32_t n_tiles = P.scene_tiles;
    const uint32_t first = chunk * ALLOC_TILES + threadIdx.x * ALLOC_ITEMS;
    const bool whole = first + ALLOC_ITEMS <= n_tiles;
    uint32_t v[ALLOC_ITEMS];
    if (whole) {
        const uint4 a = *reinterpret_cast<const uint4 *>(count + first);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
    } else {
#pragma unroll
        for (int k = 0; k < ALLOC_ITEMS; ++k) v[k] = first + k < n_tiles ? count[first + k] : 0u;
    }
    __syncthreads();
    if (s_runs) {
        uint2 *range = c.tile_range + P.tile_base;
        uint32_t sum = 0, light = 0, heavy = 0;
#pragma unroll
        for (int k = 0; k < ALLOC_ITEMS; ++k) {
            sum += v[k];
            light += v[k] != 0u && v[k] <= HEAVY_TILE;
            heavy += v[k] > HEAVY_TILE;
        }
        // particles in the high word; listed light and heavy tiles (at most
        // 1024 each) in the low and high halves of the low word
        unsigned long long total;
        const unsigned long long offset = block_exclusive_scan<ALLOC_THREADS, unsigned long long>(
            ((unsigned long long)sum << 32) | (heavy << 16) | light, total);
        if (threadIdx.x == 0) {
            const uint32_t particles = (uint32_t)(total >> 32), n_light = (uint32_t)total & 0xffffu,
                           n_heavy = ((uint32_t)total >> 16) & 0xffffu;
            s_base[0] = particles ? atomicAdd(c.counters + COUNTER_CURSOR, particles) : 0u;
            s_base[1] = n_light ? atomicAdd(c0.work + WORK_ACTIVE + c0.parity, n_light) : 0u;
            s_base[2] = n_heavy ? atomicAdd(c0.work + WORK_HEAVY + c0.parity, n_heavy) : 0u;
        }
        __syncthreads();
        uint32_t at = s_base[0] + (uint32_t)(offset >> 32);
        uint32_t slot = s_base[1] + ((uint32_t)offset & 0xffffu);
        uint32_t heavy_slot = s_base[2] + (((uint32_t)offset >> 16) & 0xffffu);
        uint2 r[ALLOC_ITEMS];
#pragma unroll
        for (int k = 0; k < ALLOC_ITEMS; ++k) {
            r[k] = make_uint2(at, v[k]);
            at += v[k];
        }
        if (whole) {
            *reinterpret_cast<uint4 *>(range + first) = make_uint4(r[0].x, r[0].y, r[1].x, r[1].y);
            *reinterpret_cast<uint4 *>(range + first + 2) = make_uint4(r[2].x, r[2].y, r[3].x, r[3].y);
            *reinterpret_cast<uint4 *>(count + first) = make_uint4(0u, 0u, 0u, 0u);
        } else {
#pragma unroll
            for (int k = 0; k < ALLOC_ITEMS; ++k) {
                if (first + k < n_tiles) {
                    range[first + k] = r[k];
                    count[first + k] = 0u;
                }
            }
        }
        if (light | heavy) {
            // light tiles from the front of the list, heavy ones from its end
#pragma unroll
            for (int k = 0; k < ALLOC_ITEMS; ++k) {
                if (v[k] > HEAVY_TILE)
                    c.active_tiles[c0.n_tiles - 1u - heavy_slot++] = P.tile_base + first + k;
                else if (v[k] != 0u)
                    c.active_tiles[slot++] = P.tile_base + first + k;
            }
        }
    }
}

__global__ void __launch_bounds__(ALLOC_THREADS) k_tile_alloc(Ctx c0) { alloc_chunk(c0, blockIdx.x); }

// Starts the substep of every scene (the first threads of CTA 0) and buckets
// the slots 4q .. 4q + 3 of every quad q = q0 + lane for q0 from `first`
// (a warp's first quad) in steps of `stride` quads (a multiple of 32).
__device__ __forceinline__ void scatter_quads(const Ctx &c, uint32_t first, uint32_t stride)
{
    if (blockIdx.x == 0) {
        for (uint32_t s = threadIdx.x; s < c.n_scenes; s += blockDim.x) {
            const Ctx cs = scene_ctx(c, s);
            begin_substep(cs);
            cs.counters[COUNTER_CURSOR] = cs.P->p_base;
        }
    }
    const uint32_t lane = threadIdx.x & 31u;
    if (c.n_scenes > 1u) {
        for (uint32_t q0 = first; q0 * 4u < c.n; q0 += stride) {
            const uint32_t i = (q0 + lane) * 4u;
            const uint32_t first_slot = min(i, c.n - 1u);
            const uint32_t scene = scene_of_slot(c, first_slot);
            const uint32_t lead = __shfl_sync(0xffffffffu, scene, 0);
            const uint32_t end = c.scene_p_base[lead + 1u];
            const uint32_t warp_last = min((q0 + 31u) * 4u + 3u, c.n - 1u);
            const bool one = warp_last < end;
            if (one && !runs_flag(c, lead)) continue;
            if (i >= c.n) continue;
            for (uint32_t j = i; j < min(i + 4u, c.n); ++j) {
                if (!one && !runs_flag(c, scene_of_slot(c, j))) continue;
                c.perm[__ldcg(c.tile_range + (__ldcg(c.keys + j) & KEY_TILE_MASK)).x + __ldcg(c.ranks + j)] = j;
            }
        }
        return;
    }
    const bool runs = runs_flag(c, 0u);
    if (!runs) return;
    for (uint32_t q0 = first; q0 * 4u < c.n; q0 += stride) {
        const uint32_t i = (q0 + lane) * 4u;
        if (i >= c.n) break;
        if (i + 4u <= c.n) {
            const uint4 key = __ldcs(reinterpret_cast<const uint4 *>(c.keys + i));
            const uint4 rank = __ldcs(reinterpret_cast<const uint4 *>(c.ranks + i));
            const uint32_t s0 = __ldcg(c.tile_range + (key.x & KEY_TILE_MASK)).x,
                           s1 = __ldcg(c.tile_range + (key.y & KEY_TILE_MASK)).x,
                           s2 = __ldcg(c.tile_range + (key.z & KEY_TILE_MASK)).x,
                           s3 = __ldcg(c.tile_range + (key.w & KEY_TILE_MASK)).x;
            c.perm[s0 + rank.x] = i;
            c.perm[s1 + rank.y] = i + 1u;
            c.perm[s2 + rank.z] = i + 2u;
            c.perm[s3 + rank.w] = i + 3u;
        } else {
            for (uint32_t j = i; j < c.n; ++j) c.perm[__ldcg(c.tile_range + (c.keys[j] & KEY_TILE_MASK)).x + c.ranks[j]] = j;
        }
    }
}

// Bucket the slots by tile: perm[first entry of the tile + rank] = slot,
// four slots per thread, for the scenes taking part in the substep (the
// answer k_tile_alloc stored).  The first threads of CTA 0 start the substep
// of every scene (begin_substep) and reset the scenes' bucket cursors.  With
// several scenes, a warp whose slots lie in one scene asks once whether that
// scene takes part.
__global__ void k_tile_scatter(Ctx c)
{
    scatter_quads(c, blockIdx.x * blockDim.x + (threadIdx.x & ~31u), gridDim.x * blockDim.x);
}

namespace {

// Shared-memory staging of the particles of one tile (or of one chunk of a
// crowded tile): their P2G records (prepared in place from the staged
// state), their grouping by base cell (in the order channel, original index
// within a cell) and the ring accumulator.
template <int CAP>
struct Stage {
    float4 state[CAP];     // fx, fy, mass, liquid volume
    float4 affine[CAP];    // A = m C + (-dt V 4/dx^2) P F^T
    float2 momentum[CAP];  // m v
    uint32_t orig[CAP];    // original index; after the count pass channel << 30 | original index
    uint32_t cell[CAP];    // local cell | channel << 8 | REC_FAILED
    uint16_t order[CAP];   // arrival rank within the cell, then rank by (channel, original index)
    uint16_t sorted[CAP];  // staged indices grouped by cell
    uint32_t count[TILE_CELLS];
    uint32_t start[TILE_CELLS + 1];
    float acc[ACC_WORDS][RING_NODES];
    uint32_t cells[TILE_CELLS + 1];  // a crowded tile: its cells' first entries in the cell-ordered list
    uint8_t active[TILE_CELLS];      // the chunk's cells holding entries, ascending
    uint32_t warp_active[TILE_CELLS / 32];
    uint32_t mask;
    int failed;
    uint32_t item;  // the tile this group claimed (several scenes)
};

// A P2G tile is taken by a group of TILE_CELLS threads (one per cell of the
// tile in the count and scan passes): the whole CTA of k_p2g_gather, or one
// of the GROUPS halves of a k_substep CTA, which then synchronise on named
// barriers 1 and 2 (barrier 0 stays the CTA's).
template <int GROUPS>
__device__ __forceinline__ uint32_t p2g_group() { return GROUPS == 1 ? 0u : threadIdx.x / TILE_CELLS; }

template <int GROUPS>
__device__ __forceinline__ void group_sync()
{
    if constexpr (GROUPS == 1) {
        __syncthreads();
    } else {
        // barrier ids as immediates (the group is uniform per warp)
        if (p2g_group<GROUPS>() == 0u)
            asm volatile("bar.sync 1, %0;" ::"n"(TILE_CELLS) : "memory");
        else
            asm volatile("bar.sync 2, %0;" ::"n"(TILE_CELLS) : "memory");
    }
}

template <int GROUPS>
__device__ __forceinline__ uint32_t group_sync_count(bool pred)
{
    if constexpr (GROUPS == 1) {
        return (uint32_t)__syncthreads_count(pred);
    } else {
        uint32_t r;
        if (p2g_group<GROUPS>() == 0u)
            asm volatile("{\n .reg .pred p;\n setp.ne.u32 p, %1, 0;\n bar.red.popc.u32 %0, 1, %2, p;\n}\n"
                         : "=r"(r)
                         : "r"(pred ? 1u : 0u), "n"(TILE_CELLS)
                         : "memory");
        else
            asm volatile("{\n .reg .pred p;\n setp.ne.u32 p, %1, 0;\n bar.red.popc.u32 %0, 2, %2, p;\n}\n"
                         : "=r"(r)
                         : "r"(pred ? 1u : 0u), "n"(TILE_CELLS)
                         : "memory");
        return r;
    }
}

// First sorted entry of channel >= ch in the cell's entries [lo, hi) (they
// are ordered by channel, then original index).
template <int CAP>
__device__ __forceinline__ uint32_t channel_start(const Stage<CAP> &sm, uint32_t lo, uint32_t hi, uint32_t ch)
{
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2u;
        if (((sm.cell[sm.sorted[mid]] >> 8) & 3u) < ch)
            lo = mid + 1u;
        else
            hi = mid;
    }
    return lo;
}

template <int CAP>
__device__ __forceinline__ uint32_t sort_key(const Stage<CAP> &sm, uint32_t k)
{
    return sm.orig[k];  // channel << 30 | original index, set by p2g_chunk's count pass
}

// Exclusive scan of the 128 cell counts by the group's first warp (4 cells
// per lane, `lane` its lane) into out[0 .. TILE_CELLS] (and into out2 when
// given).
__device__ __forceinline__ void scan_cell_counts(uint32_t lane, const uint32_t *count, uint32_t *out, uint32_t *out2)
{
    const uint32_t a = count[4 * lane], b = count[4 * lane + 1], d = count[4 * lane + 2], e = count[4 * lane + 3];
    const uint32_t t = a + b + d + e;
    uint32_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += up;
    }
    const uint32_t ex = inc - t;
    out[4 * lane] = ex;
    out[4 * lane + 1] = ex + a;
    out[4 * lane + 2] = ex + a + b;
    out[4 * lane + 3] = ex + a + b + d;
    if (lane == 31) out[TILE_CELLS] = inc;
    if (out2) {
        out2[4 * lane] = ex;
        out2[4 * lane + 1] = ex + a;
        out2[4 * lane + 2] = ex + a + b;
        out2[4 * lane + 3] = ex + a + b + d;
    }
}

// Stages the particles of the slots src[i0 .. i1) with asynchronous copies
// and prepares each of them in shared memory (REC: stages the records G2P
// wrote), raises the status of failed preparations and groups the entries by
// cell.  Then the thread of each cell sums the P2G contributions of its
// particles of one channel, in original-index order, over the 3x3 stencil
// nodes in registers, and the cells add those sums into the ring accumulator
// in nine phases, one stencil offset per phase (no two cells of a phase share
// a node), so every sum has a fixed order.  Returns false once a particle
// failed.
template <int CAP, int GROUPS, bool LIQ, bool REC>
__device__ __forceinline__ bool p2g_chunk(const Ctx &c, Stage<CAP> &sm, const uint32_t *src, uint32_t i0, uint32_t i1)
{
    const StepParams &P = *c.P;
    const uint32_t me = threadIdx.x % TILE_CELLS;  // this thread's cell
    sm.count[me] = 0u;
    group_sync<GROUPS>();
    const uint32_t n = i1 - i0;
    // Up to the cell counts every thread works on the entries it copies in
    // itself (k = me, me + TILE_CELLS, ...), which its own cp.async wait makes
    // visible to it, so no group barrier is needed before the counts are read.
    uint32_t mask = 0;
    // the entry's arrival rank within its cell; from here on its word holds
    // its sort key: channel in the top two bits over the original index
    // (below 2^30: far more particles than the device memory holds)
    auto count_entry = [&](uint32_t k, uint32_t cell) {
        sm.order[k] = (uint16_t)atomicAdd(&sm.count[cell & 0xffu], 1u);
        mask |= 1u << ((cell >> 8) & 3u);
        sm.orig[k] |= ((cell >> 8) & 3u) << 30;
    };
    if constexpr (REC) {
        // the records variant: the P2G records the previous G2P (or the
        // batch prologue) wrote
        for (uint32_t i = i0 + me; i < i1; i += TILE_CELLS) {
            const uint32_t s = src[i];
            const uint32_t k = i - i0;
            cp_async<16>(&sm.state[k], &c.rec_state[s]);
            cp_async<16>(&sm.affine[k], &c.rec_affine[s]);
            cp_async<8>(&sm.momentum[k], &c.rec_mom[s]);
            cp_async<4>(&sm.orig[k], &c.in.orig[s]);
            cp_async<4>(&sm.cell[k], &c.rec_cell[s]);
        }
        cp_async_wait_all();
        for (uint32_t k = me; k < n; k += TILE_CELLS) {
            const uint32_t cell = sm.cell[k];
            if (cell & REC_FAILED) {  // the record carries prepareParticle's flags
                const float4 f = sm.state[k];
                if (__float_as_uint(f.y) != 0u)
                    fail_at(c.status, sm.orig[k], __float_as_uint(f.x));
                else
                    fail(c.status, __float_as_uint(f.x));
                sm.failed = 1;
                continue;
            }
            count_entry(k, cell);
        }
    } else {
        // the state prepareParticle reads: F, C, v and the material index copied
        // into the slots their results replace (state, affine, momentum, cell);
        // position, volume (and damage and plastic volume for the general
        // models) loaded into this thread's registers while the copies fly
        constexpr int PER = (CAP + TILE_CELLS - 1) / TILE_CELLS;  // entries per thread
        float2 pos[PER];
        float vol[PER], dmg[PER], pvl[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const uint32_t i = i0 + me + (uint32_t)u * TILE_CELLS;
            if (i < i1) {
                const uint32_t s = src[i];
                const uint32_t k = i - i0;
                cp_async<16>(&sm.state[k], &c.in.F[s]);
                cp_async<16>(&sm.affine[k], &c.in.C[s]);
                cp_async<8>(&sm.momentum[k], &c.in.vel[s]);
                cp_async<4>(&sm.orig[k], &c.in.orig[s]);
                cp_async<4>(&sm.cell[k], &c.in.mat[s]);
                pos[u] = c.in.pos[s];
                vol[u] = c.in.vol[s];
                if constexpr (!LIQ) {
                    dmg[u] = c.in.damage[s];
                    pvl[u] = c.in.pvol[s];
                }
            }
        }
        cp_async_wait_all();
        // prepareParticle (shaders.ts:808-963) of this thread's entries, in place:
        // (fx, fy, mass, liquid volume), the affine momentum, m v and the entry's
        // local cell | channel << 8 (| REC_FAILED after raising its status)
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const uint32_t k = me + (uint32_t)u * TILE_CELLS;
            if (k < n) {
                const Material m = c.mats[sm.cell[k]];
                const float4 F = sm.state[k], C = sm.affine[k];
                const float2 v = sm.momentum[k];
                const float damage = (!LIQ && m.model == MODEL_NEO_HOOKEAN) ? dmg[u] : 0.0f;
                const float pvol = (!LIQ && m.model == MODEL_SNOW) ? pvl[u] : 1.0f;
                Stencil st;
                uint32_t cell = REC_FAILED;
                if (!make_stencil_fast(P, pos[u], st) || !stencil_fits(P, st.bx, st.by)) {
                    fail(c.status, ERROR_STENCIL);
                } else {
                    float4 A;
                    float mass, vliq;
                    bool indexed;
                    const uint32_t flags = prepare_core<LIQ>(P, m, F, vol[u], damage, pvol, C, A, mass, vliq, indexed);
                    const uint32_t lx = (uint32_t)(st.bx + 1) % TILE_X, ly = (uint32_t)(st.by + 1) % TILE_Y;
                    const uint32_t ch = m.model == MODEL_WATER ? 1u : (LIQ || m.model == MODEL_OIL ? 2u : 0u);
                    cell = (ly * TILE_X + lx) | (ch << 8);
                    if (flags != 0u) {
                        if (indexed)
                            fail_at(c.status, sm.orig[k], flags);
                        else
                            fail(c.status, flags);
                        cell |= REC_FAILED;
                    } else {
                        sm.state[k] = make_float4(st.fx, st.fy, mass, vliq);
                        sm.affine[k] = A;
                        sm.momentum[k] = make_float2(mass * v.x, mass * v.y);
                    }
                }
                sm.cell[k] = cell;
                if (cell & REC_FAILED)  // its status is raised
                    sm.failed = 1;
                else
                    count_entry(k, cell);
            }
        }
    }
    if (mask) atomicOr(&sm.mask, mask);
    group_sync<GROUPS>();
    if (sm.failed) return false;
    if (me < 32) scan_cell_counts(me, sm.count, sm.start, nullptr);
    group_sync<GROUPS>();
    for (uint32_t k = me; k < n; k += TILE_CELLS) sm.sorted[sm.start[sm.cell[k] & 0xffu] + sm.order[k]] = (uint16_t)k;
    group_sync<GROUPS>();
    // order each cell's entries by (channel, original index): every entry
    // counts the entries of its cell with a smaller key (keys are distinct),
    // so crowded cells spread over all threads
    for (uint32_t k = me; k < n; k += TILE_CELLS) {
        const uint32_t cell = sm.cell[k] & 0xffu, key = sort_key(sm, k);
        uint32_t rank = 0;
        for (uint32_t j = sm.start[cell]; j < sm.start[cell + 1]; ++j) rank += sort_key(sm, sm.sorted[j]) < key;
        sm.order[k] = (uint16_t)rank;
    }
    group_sync<GROUPS>();
    for (uint32_t k = me; k < n; k += TILE_CELLS) sm.sorted[sm.start[sm.cell[k] & 0xffu] + sm.order[k]] = (uint16_t)k;
    group_sync<GROUPS>();
    // the cells holding entries, compacted; each gets a group of `share`
    // consecutive threads of one warp (a power of two up to 32, so that the
    // groups fill the 128 threads): a crowded chunk of few cells spreads each
    // cell's particles over its group, which adds their sums in a fixed tree
    // order (with more than 64 such cells every thread takes its own cell)
    const bool has = sm.start[me + 1] > sm.start[me];
    const uint32_t n_cells = group_sync_count<GROUPS>(has);
    uint32_t share = 1;
    while (share < 32u && n_cells * share * 2u <= (uint32_t)TILE_CELLS) share *= 2u;
    if (share > 1u) {
        const unsigned ballot = __ballot_sync(0xffffffffu, has);
        const uint32_t lane = me & 31u, warp = me >> 5;
        if (lane == 0u) sm.warp_active[warp] = __popc(ballot);
        group_sync<GROUPS>();
        uint32_t before = 0;
        for (uint32_t w = 0; w < warp; ++w) before += sm.warp_active[w];
        if (has) sm.active[before + __popc(ballot & ((1u << lane) - 1u))] = (uint8_t)me;
        group_sync<GROUPS>();
    }
    const uint32_t group = me / share, part = me % share;
    const bool mine = share == 1u || group < n_cells;
    const uint32_t cell = share == 1u ? me : (mine ? sm.active[group] : 0u);
    const uint32_t lo = mine ? sm.start[cell] : 0u, hi = mine ? sm.start[cell + 1] : 0u;
    const int cx = (int)(cell % TILE_X), cy = (int)(cell / TILE_X);
    const float dx = P.dx;
    const uint32_t tile_mask = sm.mask;
    uint32_t lo_ch = lo;
#pragma unroll 1
    for (uint32_t ch = 0; ch < 3u; ++ch) {
        if (!(tile_mask & (1u << ch))) continue;
        float m[9], px[9], py[9], vl[9];
#pragma unroll
        for (int o = 0; o < 9; ++o) m[o] = px[o] = py[o] = vl[o] = 0.f;
        // this channel's entries of the cell: [a, b)
        const uint32_t a = lo_ch;
        const uint32_t b = ch == 2u ? hi : channel_start(sm, a, hi, ch + 1u);
        lo_ch = b;
        for (uint32_t j = a + part; j < b; j += share) {
            const uint32_t k = sm.sorted[j];
            const float4 q = sm.state[k];
            const float4 A = sm.affine[k];
            const float2 mv = sm.momentum[k];
            float wx[3], wy[3], dpx[3], dpy[3];
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                wx[t] = quad_weight(q.x, t);
                wy[t] = quad_weight(q.y, t);
                dpx[t] = ((float)t - q.x) * dx;
                dpy[t] = ((float)t - q.y) * dx;
            }
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
#pragma unroll
                for (int ox = 0; ox < 3; ++ox) {
                    const int o = oy * 3 + ox;
                    const float w = wx[ox] * wy[oy];
                    const float mx = mv.x + A.x * dpx[ox] + A.y * dpy[oy];
                    const float my = mv.y + A.z * dpx[ox] + A.w * dpy[oy];
                    m[o] += w * q.z;
                    px[o] += w * mx;
                    py[o] += w * my;
                    vl[o] += w * q.w;
                }
            }
        }
        if (share > 1u) {
            // the group's partial sums, added pairwise (lane + off into lane)
            for (uint32_t off = share / 2u; off > 0u; off /= 2u) {
#pragma unroll
                for (int o = 0; o < 9; ++o) {
                    m[o] += __shfl_down_sync(0xffffffffu, m[o], off, (int)share);
                    px[o] += __shfl_down_sync(0xffffffffu, px[o], off, (int)share);
                    py[o] += __shfl_down_sync(0xffffffffu, py[o], off, (int)share);
                    vl[o] += __shfl_down_sync(0xffffffffu, vl[o], off, (int)share);
                }
            }
        }
        const bool adds = mine && part == 0u;
        const int word = ch == 0u ? 0 : (ch == 1u ? 3 : 7);
#pragma unroll
        for (int oy = 0; oy < 3; ++oy) {
#pragma unroll
            for (int ox = 0; ox < 3; ++ox) {
                const int o = oy * 3 + ox;
                group_sync<GROUPS>();  // the previous phase's adds are done
                if (adds) {
                    const int r = (cy + oy) * RING_X + cx + ox;
                    sm.acc[word][r] += m[o];
                    sm.acc[word + 1][r] += px[o];
                    sm.acc[word + 2][r] += py[o];
                    if (ch != 0u) sm.acc[word + 3][r] += vl[o];
                }
            }
        }
    }
    group_sync<GROUPS>();
    return true;
}

// P2G (prepareParticle + the p2g of shaders.ts:808-963, :1072-1211; each
// staged particle is prepared in shared memory from its state) for the tiles
// holding particles, one tile per group iteration, one thread per cell.
// The sums of a tile's particles over its 18x10-node ring have a fixed
// order (cell-major phases, original particle index within a cell), so they
// do not depend on the order of the tile buckets and every run is
// bit-identical.  A tile with more than CAP particles is taken in chunks of
// consecutive whole cells (a cell holding more than CAP particles in chunks
// of the bucket, whose order then decides the rounding of its sums).  The
// sums go to the tile's own ring record; the G2P adds the up to four
// records that cover a node.  The GROUPS groups of a CTA take interleaved
// tiles of the list, each with its own stage.
template <bool SCENES, int CAP, int GROUPS, bool LIQ, bool REC>
__device__ __forceinline__ void p2g_tiles(const Ctx &c0, Stage<CAP> *stages)
{
    const uint32_t g = p2g_group<GROUPS>();
    const uint32_t me = threadIdx.x % TILE_CELLS;
    Stage<CAP> &sm = stages[g];
    const uint32_t n_active = listed_count(c0), n_heavy = heavy_count(c0);
    // several scenes: each group claims its next tile (the heavy ones are
    // listed first), which evens out tiles of very different sizes; one scene
    // (tiles of similar size): a fixed stride
    auto next = [&](uint32_t prev) -> uint32_t {
        if constexpr (SCENES) {
            group_sync<GROUPS>();  // the readers of the previous claim are done
            if (me == 0) sm.item = atomicAdd(c0.work + WORK_CLAIM, 1u);
            group_sync<GROUPS>();
            return sm.item;
        } else {
            return prev + gridDim.x * GROUPS;
        }
    };
    for (uint32_t item = SCENES ? next(0u) : blockIdx.x * GROUPS + g; item < n_active; item = next(item)) {
        const uint32_t tile = __ldcg(listed_tile(c0, item, n_heavy));
        const Ctx c = tile_ctx<SCENES>(c0, tile);
        const uint32_t stamp = __ldcg(c.counters + COUNTER_STAMP);
        const uint2 range = __ldcg(c.tile_range + tile);
        const uint32_t begin = range.x, n_tile = range.y;
        group_sync<GROUPS>();  // the previous tile's readers of sm are done
        for (int k = me; k < ACC_WORDS * RING_NODES; k += TILE_CELLS) (&sm.acc[0][0])[k] = 0.f;
        if (me == 0) {
            sm.failed = *(volatile uint32_t *)c.status != 0u ? 1 : 0;  // one read for the whole group
            sm.mask = 0u;
        }
        group_sync<GROUPS>();
        if (sm.failed) continue;  // the scene's substep is rolled back
        // a tile above one stage: its entries are first ordered by cell into
        // the scratch list tmp[begin .. begin + n_tile) (arrival order within
        // a cell), then taken in chunks of consecutive whole cells holding at
        // most CAP particles in all; a cell holding more is taken in chunks of
        // its list, whose arrival order then decides the rounding
        const uint32_t *src = c.perm + begin;
        if (n_tile > (uint32_t)CAP) {
            sm.count[me] = 0u;  // one thread per cell
            group_sync<GROUPS>();
            for (uint32_t i = me; i < n_tile; i += 4 * TILE_CELLS) {
                uint32_t s[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) s[u] = i + u * TILE_CELLS < n_tile ? src[i + u * TILE_CELLS] : 0xffffffffu;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (s[u] != 0xffffffffu) atomicAdd(&sm.count[c.keys[s[u]] >> KEY_CELL_SHIFT], 1u);
            }
            group_sync<GROUPS>();
            // the cells' first entries, and cursors for the placement below
            if (me < 32) scan_cell_counts(me, sm.count, sm.cells, sm.start);
            group_sync<GROUPS>();
            uint32_t *list = c.tmp + begin;
            for (uint32_t i = me; i < n_tile; i += 4 * TILE_CELLS) {
                uint32_t s[4], cell[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) s[u] = i + u * TILE_CELLS < n_tile ? src[i + u * TILE_CELLS] : 0xffffffffu;
#pragma unroll
                for (int u = 0; u < 4; ++u) cell[u] = s[u] != 0xffffffffu ? c.keys[s[u]] >> KEY_CELL_SHIFT : 0u;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (s[u] != 0xffffffffu) list[atomicAdd(&sm.start[cell[u]], 1u)] = s[u];
            }
            // the list is written (global, read back by this group)
            if constexpr (GROUPS > 1) __threadfence_block();
            group_sync<GROUPS>();
            src = list;
        }
        bool ok = true;
        uint32_t q = 0, i0 = 0;
        while (ok && q < (uint32_t)TILE_CELLS) {
            uint32_t q1 = TILE_CELLS, lo = 0, hi = n_tile;
            if (n_tile > (uint32_t)CAP) {
                if (sm.cells[q + 1] - sm.cells[q] > (uint32_t)CAP) {
                    q1 = q + 1;
                    lo = sm.cells[q] + i0;
                    hi = min(lo + (uint32_t)CAP, sm.cells[q + 1]);
                } else {
                    q1 = q;
                    while (q1 < (uint32_t)TILE_CELLS && sm.cells[q1 + 1] - sm.cells[q] <= (uint32_t)CAP) ++q1;
                    lo = sm.cells[q];
                    hi = sm.cells[q1];
                }
            }
            ok = p2g_chunk<CAP, GROUPS, LIQ, REC>(c, sm, src, lo, hi);
            if (n_tile > (uint32_t)CAP && q1 == q + 1 && hi < sm.cells[q + 1]) {
                i0 += (uint32_t)CAP;  // next chunk of the same crowded cell
            } else {
                q = q1;
                i0 = 0;
            }
        }
        if (!ok) continue;
        const uint32_t mask = sm.mask;
        if (me == 0) c.tile_info[tile] = make_uint2(stamp, mask);
        float *out = c.part + (size_t)tile * (ACC_WORDS * RING_NODES);
        for (int k = me; k < ACC_WORDS * RING_NODES; k += TILE_CELLS) {
            const int word = k / RING_NODES;
            const uint32_t bit = word < 3 ? 1u : (word < 7 ? 2u : 4u);
            if (mask & bit) out[k] = (&sm.acc[0][0])[k];
        }
    }
}

}  // namespace

template <bool SCENES, int CAP, bool LIQ, bool REC>
__global__ void __launch_bounds__(TILE_CELLS, 5) k_p2g_gather(Ctx c0)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    p2g_tiles<SCENES, CAP, 1, LIQ, REC>(c0, reinterpret_cast<Stage<CAP> *>(dsm));
}

namespace {

// The (up to four) tile ring records that hold sums for one halo node, in
// the fixed order own tile, left, below, below-left: `base` is the record
// offset of the node's first word, `mask` the record's channels (0: none).
struct NodeSources {
    uint32_t base[4];
    uint32_t mask[4];
};

// Sources of halo node (hx, hy) (both >= 0), which lies in the 3x3 tiles
// around tile (tx, ty); info[] holds those tiles' (stamp, mask), row-major
// from (-1, -1).
__device__ __forceinline__ NodeSources node_sources(const StepParams &P, const uint2 *info, int tx, int ty, int hx,
                                                    int hy, uint32_t stamp)
{
    NodeSources ns;
    const int ntx = (int)((uint32_t)hx / TILE_X), nty = (int)((uint32_t)hy / TILE_Y);
    const int lx = (int)((uint32_t)hx % TILE_X), ly = (int)((uint32_t)hy % TILE_Y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int sx = (k & 1) ? ntx - 1 : ntx, sy = (k & 2) ? nty - 1 : nty;
        const int rx = (k & 1) ? lx + TILE_X : lx, ry = (k & 2) ? ly + TILE_Y : ly;
        const int ox = sx - tx, oy = sy - ty;
        ns.base[k] = 0u;
        ns.mask[k] = 0u;
        if (rx >= RING_X || ry >= RING_Y || ox < -1 || ox > 1 || oy < -1 || oy > 1) continue;
        const uint2 in = info[(oy + 1) * 3 + (ox + 1)];
        if (in.x != stamp) continue;
        ns.base[k] = (P.tile_base + (uint32_t)sy * P.tiles_x + (uint32_t)sx) * (uint32_t)(ACC_WORDS * RING_NODES) +
                     (uint32_t)(ry * RING_X + rx);
        ns.mask[k] = in.y;
    }
    return ns;
}

// Adds words W0 .. W0 + NW - 1 of a node's (up to four) ring records into
// sum[] in source order.  All the loads are issued before the first add (one
// L2 round trip, not one per source); a source without the channel adds +0,
// which leaves the sum's bits unchanged (a sum that starts at +0 is never -0).
template <int W0, int NW>
__device__ __forceinline__ void add_channel(const float *part, const NodeSources &ns, uint32_t bit,
                                            float (&sum)[ACC_WORDS])
{
    float v[4][NW];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool has = (ns.mask[k] & bit) != 0u;
        const float *src = part + ns.base[k];
#pragma unroll
        for (int w = 0; w < NW; ++w) v[k][w] = has ? __ldcg(src + (W0 + w) * RING_NODES) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int w = 0; w < NW; ++w) sum[W0 + w] += v[k][w];
}

// add_channel for two channels at once: every load of both is issued before
// the first add (one L2 round trip for the water and oil sums together); each
// word's sum keeps its source order, so the result is add_channel's.
template <int W0, int NW, int W1, int NW1>
__device__ __forceinline__ void add_two_channels(const float *part, const NodeSources &ns, uint32_t bit0,
                                                 uint32_t bit1, float (&sum)[ACC_WORDS])
{
    float v[4][NW], u[4][NW1];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool has0 = (ns.mask[k] & bit0) != 0u, has1 = (ns.mask[k] & bit1) != 0u;
        const float *src = part + ns.base[k];
#pragma unroll
        for (int w = 0; w < NW; ++w) v[k][w] = has0 ? __ldcg(src + (W0 + w) * RING_NODES) : 0.0f;
#pragma unroll
        for (int w = 0; w < NW1; ++w) u[k][w] = has1 ? __ldcg(src + (W1 + w) * RING_NODES) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int w = 0; w < NW; ++w) sum[W0 + w] += v[k][w];
#pragma unroll
        for (int w = 0; w < NW1; ++w) sum[W1 + w] += u[k][w];
    }
}

// Adds the ring records of a node into sum[] in source order: every word of
// the channels in `channels` when `all`, else only the water and oil volumes
// (words 6 and 10).  `channels` (the union of the neighbour records' masks)
// is the same for the whole CTA, so its branches do not diverge.  With LIQ
// (no solid channel) the water and oil words are loaded together.
template <bool LIQ = false>
__device__ __forceinline__ void add_sources(const Ctx &c, const NodeSources &ns, bool all, uint32_t channels,
                                            float (&sum)[ACC_WORDS])
{
    if (LIQ && channels == 6u) {
        if (all)
            add_two_channels<3, 4, 7, 4>(c.part, ns, 2u, 4u, sum);
        else
            add_two_channels<6, 1, 10, 1>(c.part, ns, 2u, 4u, sum);
        return;
    }
    if (all) {
        if (channels & 1u) add_channel<0, 3>(c.part, ns, 1u, sum);
        if (channels & 2u) add_channel<3, 4>(c.part, ns, 2u, sum);
        if (channels & 4u) add_channel<7, 4>(c.part, ns, 4u, sum);
    } else {
        if (channels & 2u) add_channel<6, 1>(c.part, ns, 2u, sum);
        if (channels & 4u) add_channel<10, 1>(c.part, ns, 4u, sum);
    }
}

}  // namespace


// ----------------------------------------------------- fixed-point P2G --

namespace {

// addFixedPoint: shaders.ts:971-985.  The rounding is ties-to-even.
__device__ __forceinline__ bool add_fixed(const Ctx &c, uint32_t index, float value)
{
    const float scaled = rintf(__fmul_rn(value, c.P->fixed_scale));
    if (!finite_f(scaled) || fabsf(scaled) > 2147483520.0f) {
        fail(c.status, ERROR_FIXED_POINT_RANGE);
        return false;
    }
    const int32_t inc = (int32_t)scaled;
    const int32_t prev = atomicAdd(&c.fixed[index], inc);
    if ((inc > 0 && prev > 2147483647 - inc) || (inc < 0 && prev < (-2147483647 - 1) - inc)) {
        fail(c.status, ERROR_FIXED_POINT_RANGE);
    }
    return true;
}

}  // namespace

// prepareAndScatterParticles: shaders.ts:987-1043.  Integer sums are
// order-independent, so this path is bit-reproducible and is checked
// bit-exactly against a CPU emulation of the same integers.
__global__ void k_prepare_scatter(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    float4 A;
    float mass, vliq;
    uint32_t model;
    if (!prepare_particle(c, i, A, mass, vliq, model)) return;
    if (c.affine_out) c.affine_out[i] = A;
    if (*(volatile uint32_t *)c.status != 0u) return;
    Stencil s;
    if (!make_stencil(P, c.in.pos[i], s) || !stencil_fits(P, s.bx, s.by)) {
        fail(c.status, ERROR_STENCIL);
        return;
    }
    const uint32_t stamp = c.counters[COUNTER_STAMP];
    const uint32_t hx0 = (uint32_t)(s.bx + 1), hy0 = (uint32_t)(s.by + 1);
    c.tile_stamp[tile_of_node(P, hx0, hy0)] = stamp;
    c.tile_stamp[tile_of_node(P, hx0 + 2, hy0)] = stamp;
    c.tile_stamp[tile_of_node(P, hx0, hy0 + 2)] = stamp;
    c.tile_stamp[tile_of_node(P, hx0 + 2, hy0 + 2)] = stamp;
    const float2 v = c.in.vel[i];
    const bool liquid = model == MODEL_WATER || model == MODEL_OIL;
    const uint32_t channel = model == MODEL_WATER ? 3u : (model == MODEL_OIL ? 7u : 0u);
    const float pm = P.particle_mass, pv = P.particle_volume;
    for (int oy = 0; oy < 3; ++oy) {
        for (int ox = 0; ox < 3; ++ox) {
            const float w = __fmul_rn(quad_weight(s.fx, ox), quad_weight(s.fy, oy));
            const float dpx = __fmul_rn(__fsub_rn((float)ox, s.fx), P.dx);
            const float dpy = __fmul_rn(__fsub_rn((float)oy, s.fy), P.dx);
            const float mx = __fadd_rn(__fadd_rn(__fmul_rn(mass, v.x), __fmul_rn(A.x, dpx)), __fmul_rn(A.y, dpy));
            const float my = __fadd_rn(__fadd_rn(__fmul_rn(mass, v.y), __fmul_rn(A.z, dpx)), __fmul_rn(A.w, dpy));
            if (!finite_f(w) || w < 0.0f || !finite_f(mx) || !finite_f(my)) {
                fail_at(c.status, c.in.orig[i], ERROR_P2G | ERROR_P2G_NONFINITE_PARTICLE);
                return;
            }
            const uint32_t field = node_index(P, s.bx + ox, s.by + oy) * FIXED_WORDS + channel;
            if (!add_fixed(c, field, __fdiv_rn(__fmul_rn(w, mass), pm))) return;
            if (!add_fixed(c, field + 1, __fdiv_rn(__fmul_rn(w, mx), pm))) return;
            if (!add_fixed(c, field + 2, __fdiv_rn(__fmul_rn(w, my), pm))) return;
            if (liquid && !add_fixed(c, field + 3, __fdiv_rn(__fmul_rn(w, vliq), pv))) return;
        }
    }
}

// gatherAtomicGrid: shaders.ts:1045-1070.  Decodes and clears the integer
// words of every node of a touched tile.  Decoding ignores the status word so
// the accumulators are always clean for the next substep.
__global__ void __launch_bounds__(TILE_NODES) k_fixed_decode(Ctx c)
{
    const StepParams &P = *c.P;
    const int tx = blockIdx.x, ty = blockIdx.y;
    if (c.tile_stamp[ty * P.tiles_x + tx] != c.counters[COUNTER_STAMP]) return;
    const int hx = tx * TILE_X + (threadIdx.x % TILE_X), hy = ty * TILE_Y + (threadIdx.x / TILE_X);
    if (hx >= (int)P.node_w || hy >= (int)P.node_h) return;
    const uint32_t n = (uint32_t)hy * P.node_w + (uint32_t)hx;
    int32_t *w = c.fixed + (size_t)n * FIXED_WORDS;
    float v[FIXED_WORDS];
    const float inv = 1.0f / P.fixed_scale;
#pragma unroll
    for (int k = 0; k < FIXED_WORDS; ++k) {
        v[k] = (float)w[k] * inv;
        w[k] = 0;
    }
    if (*(volatile uint32_t *)c.status != 0u) return;
    const float pm = P.particle_mass, pv = P.particle_volume;
    c.p2g_solid[n] = make_float4(v[0] * pm, v[1] * pm, v[2] * pm, 0.f);
    c.p2g_water[n] = make_float4(v[3] * pm, v[4] * pm, v[5] * pm, v[6] * pv);
    c.p2g_oil[n] = make_float4(v[7] * pm, v[8] * pm, v[9] * pm, v[10] * pv);
}

namespace {

// volumeAtNode: shaders.ts:1779-1790, reading zero for tiles that no particle
// touched this substep (their storage is stale, not cleared).
__device__ __forceinline__ float2 phase_volume(const Ctx &c, int hx, int hy, uint32_t stamp)
{
    const StepParams &P = *c.P;
    if (hx < 0 || hy < 0 || hx >= (int)P.node_w || hy >= (int)P.node_h) return make_float2(0.f, 0.f);
    if (c.tile_stamp[tile_of_node(P, (uint32_t)hx, (uint32_t)hy)] != stamp) return make_float2(0.f, 0.f);
    const uint32_t n = (uint32_t)hy * P.node_w + (uint32_t)hx;
    return make_float2(c.p2g_water[n].w, c.p2g_oil[n].w);
}

}  // namespace

// updateGrid of the fixed-point path: the same node update over the decoded
// sums of touched tiles.
__global__ void __launch_bounds__(TILE_NODES) k_grid_update(Ctx c)
{
    const StepParams &P = *c.P;
    const int tx = blockIdx.x, ty = blockIdx.y;
    const uint32_t stamp = c.counters[COUNTER_STAMP];
    if (c.tile_stamp[ty * P.tiles_x + tx] != stamp) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    const int hx = tx * TILE_X + (threadIdx.x % TILE_X), hy = ty * TILE_Y + (threadIdx.x / TILE_X);
    if (hx >= (int)P.node_w || hy >= (int)P.node_h) return;
    const uint32_t n = (uint32_t)hy * P.node_w + (uint32_t)hx;
    update_node(c, n, hx - 1, hy - 1, c.p2g_solid[n], c.p2g_water[n], c.p2g_oil[n],
                phase_volume(c, hx + 1, hy, stamp), phase_volume(c, hx - 1, hy, stamp),
                phase_volume(c, hx, hy + 1, stamp), phase_volume(c, hx, hy - 1, stamp));
}

// ------------------------------------------------------------------ G2P --

namespace {

// particleWaveSpeedBound: shaders.ts:268-353, squared: returns the square
// whose square root the reference returns, or -1 where it returns FLOAT_MAX.
// `tait_pow` is (1 / det F)^gamma of a Tait liquid when the caller has it
// (negative: not computed); (1 / det)^(gamma - 1) is then tait_pow * det.
template <bool LIQ = false>
__device__ float wave_speed_sq(const Ctx &c, const Material &m, float4 F, float damage, float volume, float tait_pow)
{
    if (LIQ || m.model == MODEL_WATER || m.model == MODEL_OIL) {
        if (!finite_f(m.lambda) || !finite_f(m.density) || m.lambda <= 0.f || m.density <= 0.f) return -1.0f;
        float c2 = m.c2;  // lambda / density, divided once on the host
        if (m.param > 0.0f) {
            const float det = det2(F);
            if (!finite_f(m.param) || m.param <= 0.f || !finite_f(det) || det <= 0.f) return -1.0f;
            const float scale = tait_pow >= 0.0f ? tait_pow * det : pow_wgsl(1.0f / det, m.param - 1.0f);
            c2 = m.param * c2 * scale;
        }
        if (!finite_f(c2) || c2 < 0.f) return -1.0f;
        return c2;
    }
    if (m.model != MODEL_NEO_HOOKEAN) return -1.0f;
    if (!finite_f(damage)) return -1.0f;
    const float remaining = 1.0f - fminf(fmaxf(damage, 0.f), 1.f);
    if (remaining <= 0.f) return 0.f;
    const float lambda = m.lambda * remaining, mu = m.mu * remaining;
    const float det = det2(F);
    const float tr = F.x * F.x + F.y * F.y + F.z * F.z + F.w * F.w;
    if (!finite_f(det) || det <= 0.f || !finite_f(tr) || !finite_f(lambda) || !finite_f(mu) || mu < 0.f)
        return -1.0f;
    const float disc = sqrtf(fmaxf(0.f, tr * tr - 4.0f * det * det));
    const float maxs2 = 0.5f * (tr + disc);
    const float vt = fabsf(lambda + mu - lambda * logf(det));
    const float rho = c.P->particle_mass / volume;
    const float c2 = (mu * maxs2 + vt) / rho;
    if (!finite_f(rho) || rho <= 0.f || !finite_f(c2) || c2 < 0.f) return -1.0f;
    return c2;
}

__device__ __forceinline__ void copy_particle(const Ctx &c, uint32_t from, uint32_t to)
{
    c.out.pos[to] = c.in.pos[from];
    c.out.vel[to] = c.in.vel[from];
    c.out.C[to] = c.in.C[from];
    c.out.F[to] = c.in.F[from];
    c.out.pvol[to] = c.in.pvol[from];
    c.out.damage[to] = c.in.damage[from];
    c.out.vol[to] = c.in.vol[from];
    c.out.mat[to] = c.in.mat[from];
    c.out.orig[to] = c.in.orig[from];
}

// validateCflParticle: shaders.ts:2423-2454
template <bool LIQ = false>
__device__ void validate_cfl(const Ctx &c, uint32_t id, const Material &m, float2 vel, float4 F, float damage,
                             float volume, float tait_pow)
{
    const StepParams &P = *c.P;
    if (!P.cfl_enabled) return;
    // The speed and the wave speed are compared through their squares: a
    // correctly rounded square root exceeds a bound exactly when its argument
    // exceeds the bound's square_bound (a non-finite square is a non-finite
    // speed), and the wave speed is finite (FLOAT_MAX where the reference
    // gives up), so the decisions are the reference's.
    const float s2 = __fadd_rn(__fmul_rn(vel.x, vel.x), __fmul_rn(vel.y, vel.y));
    const float c2 = wave_speed_sq<LIQ>(c, m, F, damage, volume, tait_pow);
    const bool wave_out = c2 < 0.0f ? FLOAT_MAX > P.cfl_wave_bound : c2 > P.cfl_wave2_bound;
    if (!finite2(vel) || !finite_f(s2) || s2 > P.cfl_speed2_bound || wave_out) {
        // the reference reads the status word before the bounds; a particle
        // within them records nothing either way, so only a violation reads it
        if (*(volatile uint32_t *)c.status != 0u) return;
        const float speed = length2(vel);
        const float wave = c2 < 0.0f ? FLOAT_MAX : sqrtf(c2);
        const uint32_t prev = atomicOr(c.status + 6, 3u);
        if (prev == 0u) {
            atomicExch(c.status + 1, id);
            atomicExch(c.status + 2, __float_as_uint(speed));
            atomicExch(c.status + 3, __float_as_uint(wave));
            atomicExch(c.status + 4, __float_as_uint(P.cfl_velocity_limit));
            atomicExch(c.status + 5, __float_as_uint(P.cfl_wave_bound));
        }
        fail(c.status, ERROR_CFL_BOUND);
    }
}

// Node velocities of the global grid, around base node n00.
struct GlobalGrid {
    const float2 *solid;
    const float4 *water, *oil;
    uint32_t n00, row;
    __device__ __forceinline__ uint32_t at(int ox, int oy) const { return n00 + (uint32_t)oy * row + (uint32_t)ox; }
};

// Node velocities of a tile's ring in shared memory, around ring node r00.
struct RingGrid {
    const float2 *solid;
    const float4 *water, *oil;
    uint32_t n00, row;
    __device__ __forceinline__ uint32_t at(int ox, int oy) const { return n00 + (uint32_t)oy * row + (uint32_t)ox; }
};

// projectLiquidFromTriangles (shaders.ts:1801-1854): pushes a liquid
// particle of the given radius out of the nearest pebble of its stencil.
__device__ float2 project_from_triangles(const Ctx &c, float2 pos, float radius)
{
    const StepParams &P = *c.P;
    Stencil st;
    if (!make_stencil(P, pos, st)) return pos;
    float wx[3], wy[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        wx[k] = quad_weight(st.fx, k);
        wy[k] = quad_weight(st.fy, k);
    }
    float sd = 0.f, closest = FLOAT_MAX;
    uint32_t body1 = 0u;
    float2 selected = make_float2(0.f, 0.f);
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const TriField f = c.field[node_index(P, st.bx + ox, st.by + oy)];
            sd += wx[ox] * wy[oy] * f.sd;
            if (f.body1 != 0u && f.sd < closest) {
                closest = f.sd;
                body1 = f.body1;
                selected = make_float2(f.nx, f.ny);
            }
        }
    if (body1 == 0u) return pos;
    float2 nrm = make_float2(0.f, 0.f);
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const TriField f = c.field[node_index(P, st.bx + ox, st.by + oy)];
            if (f.body1 == body1) {
                nrm.x += wx[ox] * wy[oy] * f.nx;
                nrm.y += wx[ox] * wy[oy] * f.ny;
            }
        }
    const float nl = sqrtf(nrm.x * nrm.x + nrm.y * nrm.y);
    if (!finite_f(nl) || nl <= 1e-8f)
        nrm = selected;
    else
        nrm = make_float2(nrm.x / nl, nrm.y / nl);
    if (!finite_f(sd) || sd >= radius || !finite2(nrm)) return pos;
    return make_float2(pos.x + (radius - sd) * nrm.x, pos.y + (radius - sd) * nrm.y);
}

// projectLiquidDeformation (shaders.ts:474-488): the rotation of the trial F
// scaled by the square root of its clamped determinant.
__device__ __forceinline__ float4 project_liquid(float4 trial)
{
    const float2 rn = make_float2(trial.x + trial.w, trial.z - trial.y);
    const float rs = fmaxf(fabsf(rn.x), fabsf(rn.y));
    const float irs = __frcp_rn(rs);
    const float2 nr = make_float2(rn.x * irs, rn.y * irs);
    const float irl = rsqrtf(nr.x * nr.x + nr.y * nr.y);
    const float2 rot = make_float2(nr.x * irl, nr.y * irl);
    const float vol = det2(trial);
    const float bv = fminf(fmaxf(vol, MIN_LIQUID_DETERMINANT), MAX_LIQUID_DETERMINANT);
    const float sc = sqrtf(bv);
    return make_float4(sc * rot.x, sc * -rot.y, sc * rot.y, sc * rot.x);
}

// The input state G2P reads for one particle.
struct ParticleIn {
    float2 pos;
    float4 F;
    float vol, pvol, damage;
    uint32_t mat, orig;
};

__device__ __forceinline__ ParticleIn load_particle(const Ctx &c, uint32_t s)
{
    ParticleIn in;
    in.pos = c.in.pos[s];
    in.F = c.in.F[s];
    in.vol = c.in.vol[s];
    in.pvol = c.in.pvol[s];
    in.damage = c.in.damage[s];
    in.mat = c.in.mat[s];
    in.orig = c.in.orig[s];
    return in;
}

// The G2P of one particle with base stencil st: reads `in`, writes slot d.
// Returns false when the particle raised a status (the substep is then
// rolled back).  When the next substep's tiles are counted, `next` receives
// the stencil of the new position.
// BODIES: the solver may hold bonded-triangle bodies or fracture bonds; LIQ:
// every material is water or oil (the other models' code is compiled out);
// REC: the records variant, which also writes the slot's P2G record.
template <bool BODIES, bool LIQ, bool REC, class Grid>
__device__ __forceinline__ bool g2p_particle(const Ctx &c, const ParticleIn &in, uint32_t d, const Stencil &st,
                                             const Grid &grid, Stencil &next, bool &count_next)
{
    count_next = false;
    const StepParams &P = *c.P;
    const float2 pos = in.pos;
    const uint32_t id = in.orig;
    const Material m = c.mats[in.mat];
    const bool water = m.model == MODEL_WATER, oil = !water && (LIQ || m.model == MODEL_OIL), liquid = water || oil;
    float wx[3], wy[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        wx[k] = quad_weight(st.fx, k);
        wy[k] = quad_weight(st.fy, k);
    }
    float2 vel = make_float2(0.f, 0.f);
    float4 aff = make_float4(0.f, 0.f, 0.f, 0.f);
    float pmass = 0.f, pvolume = 0.f;
    const float4 *gliq = water ? grid.water : grid.oil;
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
        const float dpy = ((float)oy - st.fy) * P.dx;
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const uint32_t n = grid.at(ox, oy);
            const float w = wx[ox] * wy[oy];
            const float dpx = ((float)ox - st.fx) * P.dx;
            // The reference also checks w, dp, the node velocity and the
            // node's liquid mass and volume for finiteness and sign here.
            // None of those checks can fire on this path: w and dp are
            // finite and w >= 0 for a finite fraction in [0.5, 1.5), and every
            // node G2P reads was written by this substep's grid update,
            // which raises a status (and so stops this kernel) instead of
            // writing a non-finite velocity or a negative or non-finite sum.
            float2 gv;
            float nm = 0.f, nv = 0.f;
            if (liquid) {
                const float4 g = gliq[n];
                gv = make_float2(g.x, g.y);
                nm = g.z;
                nv = g.w;
            } else {
                gv = grid.solid[n];
            }
            vel.x += w * gv.x;
            vel.y += w * gv.y;
            if (liquid) {
                pmass += w * nm;
                pvolume += w * nv;
            }
            aff.x += w * gv.x * dpx;
            aff.y += w * gv.x * dpy;
            aff.z += w * gv.y * dpx;
            aff.w += w * gv.y * dpy;
        }
    }
    const float4 F0 = in.F;
    if (liquid) {
        const float pdet = det2(F0);
        if (!finite_f(pmass) || pmass <= 0.f || !finite_f(pvolume) || pvolume <= 0.f || !finite_f(pdet) ||
            pdet <= 0.f) {
            fail_at(c.status, id, ERROR_G2P);
            return false;
        }
        const float pd = __fdividef(m.density, pdet);
        const float ld = __fdividef(pmass, pvolume);
        const float rd = __fdividef(pd - ld, pd);
        vel.x += P.dt * (rd * P.gx);
        vel.y += P.dt * (rd * P.gy);
        if (!finite_f(pd) || pd <= 0.f || !finite_f(ld) || ld <= 0.f || !finite_f(rd) || !finite2(vel)) {
            fail_at(c.status, id, ERROR_G2P);
            return false;
        }
    }
    const float gs = P.gradient_scale, dt = P.dt;
    const float4 Cn = make_float4(aff.x * gs, aff.y * gs, aff.z * gs, aff.w * gs);
    const float2 npos = make_float2(pos.x + dt * vel.x, pos.y + dt * vel.y);
    if (!finite2(vel) || !finite4(Cn) || !finite2(npos)) {
        fail(c.status, ERROR_G2P);
        return false;
    }
    DeformationTrial dtr;
    const uint32_t dflags = deformation_trial(F0, Cn, dt, dtr);
    if (dflags == ERROR_DEFORMATION_SUBSTEP_LIMIT) {
        fail_at(c.status, id, ERROR_DEFORMATION_SUBSTEP_LIMIT);
        return false;
    }
    if (dflags != 0u) {
        fail(c.status, dflags);
        return false;
    }
    const float4 trial = dtr.F;
    const float tdet = dtr.det, inc = dtr.increment;
    float4 Fn = trial;
    float pv = in.pvol;
    if (!finite_f(tdet) || tdet <= 0.f) {
        // recordDeformationFailure: shaders.ts:224-237
        const uint32_t prev = atomicOr(c.status + 6, 1u);
        if (prev == 0u) {
            atomicExch(c.status + 1, id);
            atomicExch(c.status + 2, __float_as_uint(tdet));
            atomicExch(c.status + 3, __float_as_uint(inc));
            atomicExch(c.status + 4, __float_as_uint(det2(F0)));
        }
        fail(c.status, ERROR_DEFORMATION);
        return false;
    }
    if constexpr (LIQ) {
        Fn = project_liquid(trial);
    } else {
        if (m.model == MODEL_SNOW) {
            const Decomp dd = decompose(trial);
            if (!finite_f(dd.s0) || !finite_f(dd.s1) || dd.s0 <= 0.f || dd.s1 <= 0.f) {
                fail(c.status, ERROR_G2P);
                return false;
            }
            const float lo = 1.0f - SNOW_COMPRESSION_YIELD, hi = 1.0f + SNOW_STRETCH_YIELD;
            const float a = fminf(fmaxf(dd.s0, lo), hi), b = fminf(fmaxf(dd.s1, lo), hi);
            pv = fminf(fmaxf(pv * tdet / (a * b), SNOW_MIN_PLASTIC_VOLUME), SNOW_MAX_PLASTIC_VOLUME);
            Fn = reconstruct(dd, a, b);
        } else if (m.model == MODEL_POWDER) {
            if (!finite_f(m.lambda) || !finite_f(m.mu) || m.mu <= 0.f || !finite_f(m.param) || m.param < 0.f) {
                fail(c.status, ERROR_G2P);
                return false;
            }
            // projectGranularDeformation: shaders.ts:443-472
            const Decomp dd = decompose(trial);
            const float l0 = logf(dd.s0), l1 = logf(dd.s1);
            const float lv = l0 + l1;
            const float minlv = logf(MIN_POWDER_DETERMINANT);
            const float blv = fmaxf(minlv, lv);
            const float pressure = fmaxf(0.f, -(m.lambda + m.mu) * blv);
            const float dev = 0.5f * (l0 - l1);
            const float maxdev = m.param * pressure / (2.0f * m.mu);
            if (!(dev <= maxdev && lv >= minlv)) {
                const float pdev = fminf(dev, maxdev);
                const float mean = 0.5f * blv;
                Fn = reconstruct(dd, expf(mean + pdev), expf(mean - pdev));
            }
        } else if (liquid) {
            Fn = project_liquid(trial);
        } else if (m.model == MODEL_NEO_HOOKEAN) {
            const float tr = trial.x * trial.x + trial.y * trial.y + trial.z * trial.z + trial.w * trial.w;
            if (!finite_f(tr)) {
                fail(c.status, ERROR_G2P);
                return false;
            }
            if (tdet < MIN_NEO_HOOKEAN_STRETCH * sqrtf(tr) || tr > MAX_NEO_HOOKEAN_STRETCH * MAX_NEO_HOOKEAN_STRETCH) {
                const Decomp dd = decompose(trial);
                Fn = reconstruct(dd, fminf(fmaxf(dd.s0, MIN_NEO_HOOKEAN_STRETCH), MAX_NEO_HOOKEAN_STRETCH),
                                 fminf(fmaxf(dd.s1, MIN_NEO_HOOKEAN_STRETCH), MAX_NEO_HOOKEAN_STRETCH));
            }
        } else if (m.model != MODEL_FIXED_COROTATED) {
            fail(c.status, ERROR_G2P);
            return false;
        }
    }
    const float udet = det2(Fn);
    if (!finite4(Fn) || !finite_f(pv) || pv < SNOW_MIN_PLASTIC_VOLUME || pv > SNOW_MAX_PLASTIC_VOLUME) {
        fail(c.status, ERROR_G2P);
        return false;
    }
    if (!finite_f(udet) || udet <= 0.f) {
        // recordProjectedDeformationFailure: shaders.ts:239-248
        const uint32_t prev = atomicOr(c.status + 6, 2u);
        if (prev == 0u) {
            atomicExch(c.status + 1, id);
            atomicExch(c.status + 2, __float_as_uint(Fn.x));
            atomicExch(c.status + 3, __float_as_uint(Fn.y));
            atomicExch(c.status + 4, __float_as_uint(Fn.z));
            atomicExch(c.status + 5, __float_as_uint(Fn.w));
        }
        fail(c.status, ERROR_PROJECTED_DEFORMATION);
        return false;
    }
    const float2 bx = confine_axis(npos.x, vel.x, P.domain_w);
    const float2 by = confine_axis(npos.y, vel.y, P.domain_h);
    float2 projected = make_float2(bx.x, by.x);
    if (BODIES && liquid && c.field) {
        const float radius = sqrtf(in.vol * udet / 3.14159265359f);
        if (!finite_f(radius)) {
            fail_at(c.status, id, ERROR_G2P);
            return false;
        }
        projected = project_from_triangles(c, projected, radius);
    }
    const float2 fx = confine_axis(projected.x, bx.y, P.domain_w);
    const float2 fy = confine_axis(projected.y, by.y, P.domain_h);
    const float2 outv = make_float2(fx.y, fy.y);
    const float damage = in.damage;
    const float volume = in.vol;
    const float2 out_pos = make_float2(fx.x, fy.x);
    c.out.pos[d] = out_pos;
    c.out.vel[d] = outv;
    c.out.C[d] = Cn;
    c.out.F[d] = Fn;
    c.out.pvol[d] = pv;
    c.out.damage[d] = damage;
    c.out.vol[d] = volume;
    c.out.mat[d] = in.mat;
    c.out.orig[d] = id;
    // (1 / det F)^gamma of a Tait liquid at the new F, for the CFL wave speed
    // and the next substep's pressure (the record here, or the next P2G, which
    // evaluates the same expression)
    float tait_pow = -1.0f;
    if ((REC || P.cfl_enabled) && liquid && m.param > 0.0f && finite_f(m.param))
        tait_pow = pow_wgsl(__frcp_rn(udet), m.param);
    if (!BODIES || P.n_bodies == 0u) validate_cfl<LIQ>(c, id, m, outv, Fn, damage, volume, tait_pow);
    if (BODIES && is_tracked(c, id)) {
        // a body vertex or fracture particle: its final state comes after the
        // body kernels, which then count its tile and write its record
        c.slot_out[id] = d;
    } else if (c.count_next) {
        if (!make_stencil_fast(P, out_pos, next) || !stencil_fits(P, next.bx, next.by)) {
            fail(c.status, ERROR_STENCIL);
            return false;
        }
        if constexpr (REC) write_record<LIQ>(c, d, m, next, outv, Fn, volume, damage, pv, Cn, tait_pow);
        count_next = true;
    }
    return true;
}

}  // namespace

// g2p: shaders.ts:2114-2421 (APIC velocity and affine C, liquid
// density-contrast acceleration, adaptive fused F update with retries,
// per-model projection, wall confinement, fused CFL validation).  Thread d
// takes the particle at sorted position d (slot perm[d]) and writes slot d,
// so the output is sorted by cell; in the gather path it also counts the
// particle's new base cell for the next substep's sort.
__global__ void k_g2p(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in_range = d < P.n_particles;
    const uint32_t s = in_range ? (c.perm ? c.perm[d] : d) : 0u;
    bool counted = false;
    uint32_t key = 0;
    if (in_range) {
        if (*(volatile uint32_t *)c.status != 0u) {
            // the substep is rolled back: the batch ends on its input
        } else {
            const ParticleIn in = load_particle(c, s);
            Stencil st, next;
            if (!make_stencil(P, in.pos, st) || !stencil_fits(P, st.bx, st.by)) {
                fail(c.status, ERROR_STENCIL);
            } else {
                const GlobalGrid grid{c.g_solid, c.g_water, c.g_oil, node_index(P, st.bx, st.by), P.node_w};
                bool count_it;
                if (g2p_particle<true, false, false>(c, in, d, st, grid, next, count_it) && count_it) {
                    key = particle_tile(P, next.bx, next.by);
                    counted = true;
                }
            }
        }
    }
    if (!c.count_next) return;
    const unsigned active = __ballot_sync(0xffffffffu, counted);
    if (!counted) return;
    c.ranks[d] = warp_count(c.tile_count, key, active);
    c.keys[d] = key;
}

namespace {

// Copies the G2P input of slot s to shared-memory index i (asynchronously).
__device__ __forceinline__ void stage_particle(const Ctx &c, uint32_t s, uint32_t i, float2 *pos, float4 *F,
                                               float *vol, float *pvol, float *damage, uint32_t *mat, uint32_t *orig)
{
    cp_async<8>(&pos[i], &c.in.pos[s]);
    cp_async<16>(&F[i], &c.in.F[s]);
    cp_async<4>(&vol[i], &c.in.vol[s]);
    cp_async<4>(&pvol[i], &c.in.pvol[s]);
    cp_async<4>(&damage[i], &c.in.damage[s]);
    cp_async<4>(&mat[i], &c.in.mat[s]);
    cp_async<4>(&orig[i], &c.in.orig[s]);
}

// Copies the G2P inputs of the slots entries[0 .. count) (bucket entries, in
// global or shared memory) to shared indices 0..count-1; count <= G2P_STAGE =
// 2 * G2P_THREADS, and both entries of a thread are read before either copy
// is issued.
__device__ __forceinline__ void stage_chunk(const Ctx &c, const uint32_t *entries, uint32_t count, float2 *pos,
                                            float4 *F, float *vol, float *pvol, float *damage, uint32_t *mat,
                                            uint32_t *orig)
{
    const uint32_t i0 = threadIdx.x, i1 = threadIdx.x + G2P_THREADS;
    const uint32_t s0 = i0 < count ? entries[i0] : 0u;
    const uint32_t s1 = i1 < count ? entries[i1] : 0u;
    if (i0 < count) stage_particle(c, s0, i0, pos, F, vol, pvol, damage, mat, orig);
    if (i1 < count) stage_particle(c, s1, i1, pos, F, vol, pvol, damage, mat, orig);
}

}  // namespace


// The grid update and G2P of one tile holding particles (updateGrid,
// shaders.ts:1485-1746, then g2p as in k_g2p), one tile per CTA iteration.
// The CTA first evaluates the node update of the tile's 18x10-node ring --
// every node its particles' stencils reach -- from the P2G ring records
// (sums added in the fixed order of node_sources, neighbour volumes from the
// 20x12 nodes around the ring) into shared memory, then moves its particles with
// those velocities.  Ring nodes shared by neighbouring tiles are evaluated
// by each of them from the same sums, so they agree bit for bit.  A tile
// whose ring holds a failing node raises the grid status and moves none of
// its particles (the substep is rolled back); tiles elsewhere still move
// theirs, so their G2P flags can join the status of that substep.
// Shared memory of the G2P phase.
struct G2PShared {
    // per buffer parity: the tile, its bucket range and its 3x3 neighbours'
    // (stamp, mask); with one scene the next tile's are copied in while this
    // one's particles move, and the index of the one after it
    uint32_t tile[2];
    uint2 range[2];
    uint2 infos[2][9];
    // with one scene: the next tile's first G2P_STAGE bucket entries and the
    // scene's status words, copied in while this tile's particles move
    uint32_t perm[2][G2P_STAGE];
    __align__(16) uint32_t status[2][4];
    float2 vol[VOL_X * VOL_Y];
    float2 vs[RING_NODES];
    float4 vw[RING_NODES];
    float4 vo[RING_NODES];
    int fail;
    uint32_t claim;  // the tile this CTA claimed (several scenes)
    // the particles of the tile (or of one chunk of a crowded tile), copied
    // in while the node phase runs
    float4 F[G2P_STAGE];
    float2 pos[G2P_STAGE];
    float pvol_in[G2P_STAGE], vol_in[G2P_STAGE], damage[G2P_STAGE];
    uint32_t mat[G2P_STAGE], orig[G2P_STAGE];
};

template <bool SCENES, bool BODIES, bool LIQ, bool REC>
__device__ __forceinline__ void g2p_tiles(const Ctx &c0, G2PShared &sh)
{
    uint32_t *const s_tile = sh.tile;
    uint2 *const s_range = sh.range;
    uint2(*const s_infos)[9] = sh.infos;
    uint32_t(*const s_perm)[G2P_STAGE] = sh.perm;
    uint32_t(*const s_status)[4] = sh.status;
    float2 *const s_vol = sh.vol;
    float2 *const s_vs = sh.vs;
    float4 *const s_vw = sh.vw;
    float4 *const s_vo = sh.vo;
    int &s_fail = sh.fail;
    float4 *const p_F = sh.F;
    float2 *const p_pos = sh.pos;
    float *const p_vol = sh.vol_in, *const p_pvol = sh.pvol_in, *const p_damage = sh.damage;
    uint32_t *const p_mat = sh.mat, *const p_orig = sh.orig;
    const uint32_t n_active = listed_count(c0), n_heavy = heavy_count(c0);
    if constexpr (!SCENES) {
        // visible after the first iteration's barrier
        if (threadIdx.x == 0 && blockIdx.x + gridDim.x < n_active)
            s_tile[1] = *listed_tile(c0, blockIdx.x + gridDim.x, n_heavy);
    }
    // several scenes: each CTA claims its next tile (the heavy ones are listed
    // first); one scene: a fixed stride, with the next tile's data copied in
    auto next = [&](uint32_t prev) -> uint32_t {
        if constexpr (SCENES) {
            __syncthreads();  // the readers of the previous claim are done
            if (threadIdx.x == 0) sh.claim = atomicAdd(c0.work + WORK_CLAIM + 1, 1u);
            __syncthreads();
            return sh.claim;
        } else {
            return prev + gridDim.x;
        }
    };
    uint32_t it = 0;
    for (uint32_t item = SCENES ? next(0u) : blockIdx.x; item < n_active; item = next(item), ++it) {
        const uint32_t buf = it & 1u;
        const bool fetched = !SCENES && it > 0u;  // copied in during the previous tile
        uint2 *const info = s_infos[buf];
        // (the copies read here landed, and were made visible by a barrier,
        // during the previous tile)
        const uint32_t tile = fetched ? s_tile[buf] : *listed_tile(c0, item, n_heavy);
        const uint32_t nb = buf ^ 1u;
        const Ctx c = tile_ctx<SCENES>(c0, tile);
        const StepParams &P = *c.P;
        const uint32_t stamp = c.counters[COUNTER_STAMP];
        // the next tile's first bucket entries and the status words, copied in
        // during this tile (it has no particle phase when its scene failed)
        auto prefetch_next = [&]() {
            if constexpr (!SCENES) {
                if (item + gridDim.x < n_active) {
                    const uint2 nr = s_range[nb];
                    const uint32_t count = min(nr.y, (uint32_t)G2P_STAGE);
                    for (uint32_t i = threadIdx.x; i < count; i += G2P_THREADS)
                        cp_async<4>(&s_perm[nb][i], &c.perm[nr.x + i]);
                    if (threadIdx.x == G2P_THREADS - 1) cp_async<16>(&s_status[nb][0], c.status);
                }
            }
        };
        const int tiles_x = (int)P.tiles_x, tiles_y = (int)P.tiles_y;
        const int node_w = (int)P.node_w, node_h = (int)P.node_h;
        const uint32_t local = tile - P.tile_base;
        const int tx = (int)(local % P.tiles_x), ty = (int)(local / P.tiles_x);
        const int x0 = tx * TILE_X, y0 = ty * TILE_Y;
        const uint2 range = fetched ? s_range[buf] : c.tile_range[tile];
        const uint32_t begin = range.x, end = range.x + range.y;
        if (fetched) cp_async_wait_all();  // this tile's entries and status words (visible after the barrier)
        __syncthreads();  // readers of the previous tile's shared data are done
        if (!fetched && threadIdx.x < 9) {
            const int sx = tx + (int)(threadIdx.x % 3) - 1, sy = ty + (int)(threadIdx.x / 3) - 1;
            info[threadIdx.x] = (sx >= 0 && sy >= 0 && sx < tiles_x && sy < tiles_y)
                                    ? c.tile_info[P.tile_base + (uint32_t)(sy * tiles_x + sx)]
                                    : make_uint2(0xffffffffu, 0u);
        }
        // the status as the previous tile copied it in (a scene that failed
        // since then has this tile computed for nothing: its substep is
        // rolled back either way)
        if (threadIdx.x == 0) s_fail = (fetched ? s_status[buf][0] : *(volatile uint32_t *)c.status) != 0u ? 2 : 0;
        // the first chunk of particles, copied in while the node phase runs
        stage_chunk(c, fetched ? s_perm[buf] : c.perm + begin, min(end - begin, (uint32_t)G2P_STAGE), p_pos, p_F,
                    p_vol, p_pvol, p_damage, p_mat, p_orig);
        __syncthreads();
        if constexpr (!SCENES) {
            // the next tile's range and neighbour records (its index came in
            // during the previous tile) and the index of the tile after it;
            // every copy has landed by this tile's cp.async waits
            if (item + gridDim.x < n_active && threadIdx.x < 10) {
                const uint32_t tn = s_tile[nb];
                if (threadIdx.x == 9) {
                    cp_async<8>(&s_range[nb], &c.tile_range[tn]);
                } else {
                    const uint32_t ln = tn - P.tile_base;
                    const int sx = (int)(ln % P.tiles_x) + (int)(threadIdx.x % 3) - 1;
                    const int sy = (int)(ln / P.tiles_x) + (int)(threadIdx.x / 3) - 1;
                    if (sx >= 0 && sy >= 0 && sx < tiles_x && sy < tiles_y)
                        cp_async<8>(&s_infos[nb][threadIdx.x], &c.tile_info[P.tile_base + (uint32_t)(sy * tiles_x + sx)]);
                    else
                        s_infos[nb][threadIdx.x] = make_uint2(0xffffffffu, 0u);
                }
            }
            if (threadIdx.x == 10 && item + 2u * gridDim.x < n_active)
                cp_async<4>(&s_tile[buf], listed_tile(c0, item + 2u * gridDim.x, n_heavy));
        }
        if (s_fail) {
            cp_async_wait_all();  // no copy may land after this tile's shared data is reused
            __syncthreads();      // and the copies are visible to the next tile
            prefetch_next();
            continue;             // the scene's substep is rolled back
        }
        // node phase: thread t takes node (x0 - 1 + t % VOL_X, y0 - 1 + t / VOL_X)
        // of the region around the ring; ring nodes load their full sums,
        // the border only its water / oil volumes
        const int t = (int)threadIdx.x;
        const int vx = t % VOL_X, vy = t / VOL_X;
        const int hx = x0 - 1 + vx, hy = y0 - 1 + vy;
        const bool in_region = t < VOL_X * VOL_Y;
        const bool ring_node = in_region && vx >= 1 && vx <= RING_X && vy >= 1 && vy <= RING_Y;
        const bool in_grid = in_region && hx >= 0 && hy >= 0 && hx < node_w && hy < node_h;
        float sum[ACC_WORDS];
#pragma unroll
        for (int k = 0; k < ACC_WORDS; ++k) sum[k] = 0.f;
        uint32_t channels = 0u;  // the channels any neighbour record of this substep holds
#pragma unroll
        for (int k = 0; k < 9; ++k) channels |= info[k].x == stamp ? info[k].y : 0u;
        if (in_grid) {
            const NodeSources ns = node_sources(P, info, tx, ty, hx, hy, stamp);
            add_sources<LIQ>(c, ns, ring_node, channels, sum);
        }
        if (in_region) s_vol[t] = make_float2(sum[6], sum[10]);
        // ring nodes have coordinates x0 - 1 .. x0 + TILE_X, y0 - 1 .. y0 + TILE_Y
        const bool near_wall = !(beyond_wall_cushion(x0 - 1, x0 + TILE_X, (int)P.cells_x) &&
                                 beyond_wall_cushion(y0 - 1, y0 + TILE_Y, (int)P.cells_y));
        __syncthreads();
        if (ring_node) {
            const int rx = vx - 1, ry = vy - 1, r = ry * RING_X + rx;
            NodeVel v;
            v.vs = make_float2(0.f, 0.f);
            v.vw = v.vo = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in_grid) {
                const float4 S = make_float4(sum[0], sum[1], sum[2], 0.f);
                const float4 W = make_float4(sum[3], sum[4], sum[5], sum[6]);
                const float4 O = make_float4(sum[7], sum[8], sum[9], sum[10]);
                const uint32_t n = (uint32_t)hy * (uint32_t)node_w + (uint32_t)hx;
                if (!node_velocity<BODIES, LIQ>(c, n, hx - 1, hy - 1, S, W, O, s_vol[t + 1], s_vol[t - 1], s_vol[t + VOL_X],
                                   s_vol[t - VOL_X], v, near_wall)) {
                    s_fail = 1;
                } else if (BODIES && c.field) {
                    // the body impulse of a node is stored once: by the first
                    // active tile of (its tile, left, below, below-left)
                    const int dx = rx >= TILE_X ? 1 : 0, dy = ry >= TILE_Y ? 1 : 0;
                    int ox = dx, oy = dy;
                    if (info[(dy + 1) * 3 + dx + 1].x != stamp) {
                        if (info[(dy + 1) * 3 + dx].x == stamp)
                            ox = dx - 1;
                        else if (info[dy * 3 + dx + 1].x == stamp)
                            oy = dy - 1;
                        else
                            ox = dx - 1, oy = dy - 1;
                    }
                    if (ox == 0 && oy == 0) {
                        c.field[n].ix = v.impulse.x;
                        c.field[n].iy = v.impulse.y;
                    }
                }
            }
            s_vs[r] = v.vs;
            s_vw[r] = v.vw;
            s_vo[r] = v.vo;
        }
        cp_async_wait_all();
        __syncthreads();
        prefetch_next();
        if (s_fail) continue;
        for (uint32_t base = begin; base < end; base += G2P_THREADS) {
            const uint32_t p = base + threadIdx.x;
            const uint32_t chunk = (base - begin) % G2P_STAGE;
            if (base != begin && chunk == 0u) {
                // next chunk of a crowded tile
                __syncthreads();
                stage_chunk(c, c.perm + base, min(end - base, (uint32_t)G2P_STAGE), p_pos, p_F, p_vol, p_pvol,
                            p_damage, p_mat, p_orig);
                cp_async_wait_all();
                __syncthreads();
            }
            bool counted = false;
            uint32_t key = 0, packed_key = 0;
            if (p < end) {
                const uint32_t k = chunk + threadIdx.x;
                ParticleIn in;
                in.pos = p_pos[k];
                in.F = p_F[k];
                in.vol = p_vol[k];
                in.pvol = p_pvol[k];
                in.damage = p_damage[k];
                in.mat = p_mat[k];
                in.orig = p_orig[k];
                Stencil st, next;
                const bool ok = make_stencil_fast(P, in.pos, st) && stencil_fits(P, st.bx, st.by);
                const int lx = st.bx + 1 - x0, ly = st.by + 1 - y0;  // base node in the tile
                if (!ok || lx < 0 || lx >= TILE_X || ly < 0 || ly >= TILE_Y) {
                    fail(c.status, ERROR_STENCIL);
                } else {
                    const RingGrid grid{s_vs, s_vw, s_vo, (uint32_t)(ly * RING_X + lx), RING_X};
                    bool count_it;
                    if (g2p_particle<BODIES, LIQ, REC>(c, in, p, st, grid, next, count_it) && count_it) {
                        key = particle_tile(P, next.bx, next.by);
                        packed_key = bucket_key(key, next.bx, next.by);
                        counted = true;
                    }
                }
            }
            const unsigned active = __ballot_sync(0xffffffffu, counted);
            if (counted) {
                c.ranks[p] = warp_count(c.tile_count, key, active);
                c.keys[p] = packed_key;
            }
        }
    }
}

template <bool SCENES, bool BODIES, bool LIQ, bool REC>
__global__ void __launch_bounds__(G2P_THREADS, 4) k_g2p_tile(Ctx c0)
{
    __shared__ G2PShared sh;
    g2p_tiles<SCENES, BODIES, LIQ, REC>(c0, sh);
}

// ------------------------------------------------- one launch per substep --

namespace {

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Marks the launch abandoned and raises ERROR_BARRIER in every scene.
__device__ void abandon_launch(const Ctx &c)
{
    atomicExch(c.work + WORK_ABORT, 1u);
    for (uint32_t s = 0; s < c.n_scenes; ++s) fail(c.dyn + (size_t)s * SCENE_WORDS, ERROR_BARRIER);
}

// Grid-wide barrier of k_substep: every CTA of the cooperative launch calls
// it the same number of times.  Thread 0 of each CTA arrives on
// work[WORK_BARRIER]; the last arrival resets the count and advances the
// generation work[WORK_BARRIER + 1], which the others wait for (the
// release / acquire pair makes every CTA's writes before the barrier visible
// to every CTA after it).  A wait gives up after c.barrier_limit_ns: that CTA
// marks the launch abandoned, raises ERROR_BARRIER in every scene and
// returns false; a CTA that finds the launch abandoned, before arriving or
// while waiting, returns false too, so no CTA outlasts the limit by more than
// one phase.  With `index` 0, CTA c.barrier_skip leaves without arriving (the
// others' waits then run out: the test of the limit).
__device__ bool grid_barrier(const Ctx &c, uint32_t index)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t *count = c.work + WORK_BARRIER, *gen = c.work + WORK_BARRIER + 1;
        const uint32_t *abandoned = c.work + WORK_ABORT;
        int ok = ld_acquire_gpu(abandoned) == 0u;
        if (ok && index == 0u && blockIdx.x == c.barrier_skip) ok = 0;
        if (ok) {
            // the generation cannot move before this CTA arrives
            const uint32_t g = ld_acquire_gpu(gen);
            __threadfence();
            if (atomicAdd(count, 1u) == gridDim.x - 1u) {
                atomicExch(count, 0u);
                __threadfence();
                st_release_gpu(gen, g + 1u);
            } else {
                const unsigned long long t0 = global_ns();
                while (ld_acquire_gpu(gen) == g) {
                    if (ld_acquire_gpu(abandoned) != 0u) {
                        ok = 0;
                        break;
                    }
                    if (global_ns() - t0 > c.barrier_limit_ns) {
                        abandon_launch(c);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace

static_assert(SUBSTEP_THREADS == ALLOC_THREADS && SUBSTEP_THREADS == 2 * TILE_CELLS && SUBSTEP_THREADS == G2P_THREADS,
              "the substep kernel runs every phase with one CTA shape");

// One substep of the default path in one cooperative launch of persistent
// CTAs (at most as many as fit on the GPU at once, so every CTA runs to each
// barrier): the tile allocation chunks over the CTAs (k_tile_alloc), then the
// bucketing of every slot with the start of the substep (k_tile_scatter),
// then P2G over the listed tiles with two tiles at a time per CTA, one per
// 128-thread group (k_p2g_gather), then the grid update and G2P over the
// same list (k_g2p_tile), with a grid barrier between phases.  The phases
// run the four kernels' device functions, so the two forms are
// bit-identical.  Shared memory is one dynamic buffer: the two P2G stages in
// that phase, the G2P arrays in the next.
template <bool SCENES, int CAP, bool LIQ>
__global__ void __launch_bounds__(SUBSTEP_THREADS, CAP == STAGE_CAP ? 2 : 3) k_substep(Ctx c0)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    for (uint32_t b = blockIdx.x; b < c0.alloc_chunks; b += gridDim.x) alloc_chunk(c0, b);
    if (!grid_barrier(c0, 0u)) return;
    scatter_quads(c0, blockIdx.x * SUBSTEP_THREADS + (threadIdx.x & ~31u), gridDim.x * SUBSTEP_THREADS);
    if (!grid_barrier(c0, 1u)) return;
    p2g_tiles<SCENES, CAP, 2, LIQ, false>(c0, reinterpret_cast<Stage<CAP> *>(dsm));
    if (!grid_barrier(c0, 2u)) return;
    g2p_tiles<SCENES, false, LIQ, false>(c0, *reinterpret_cast<G2PShared *>(dsm));
}

size_t p2g_shared_bytes(int cap)
{
    return cap == STAGE_CAP_NARROW ? sizeof(Stage<STAGE_CAP_NARROW>) : sizeof(Stage<STAGE_CAP>);
}

size_t substep_shared_bytes(int cap) { return std::max(2 * p2g_shared_bytes(cap), sizeof(G2PShared)); }

// The start of a substep of the fixed-point path (k_tile_alloc starts those
// of the default path): begin_substep for every scene.
__global__ void k_substep_begin(Ctx c)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < c.n_scenes; s += gridDim.x * blockDim.x)
        begin_substep(scene_ctx(c, s));
}

// The end of a batch of `total` substeps (commitParticles,
// shaders.ts:3067-3080, once per batch), with `out` the buffer the batch
// ends in and `in` the other one.  A scene whose completed substeps and
// `total` differ in parity (a raised status, or fewer substeps than the
// batch) has its state in `in`: its slots (and tracked slots) are copied
// over, the whole-substep rollback.  Then, when `measure_speed` is set,
// measureParticleSpeedPartials + reduceParticleSpeedPartials
// (shaders.ts:2463-2533) of each scene's final state as one warp-shuffle
// reduction with an atomic max on the order-preserving bits of the
// non-negative speed.  Thread s of CTA 0 records scene s's completed
// substeps and, under a CFL guard, its committed microsteps; every thread
// may ask batch_stop first, which answers the same before and after.
__global__ void k_end_batch(Ctx c0, uint32_t total, uint32_t measure_speed)
{
    if (blockIdx.x == 0) {
        for (uint32_t s = threadIdx.x; s < c0.n_scenes; s += blockDim.x) {
            const Ctx cs = scene_ctx(c0, s);
            const uint32_t stop = batch_stop(cs, total);
            cs.counters[COUNTER_STOP] = stop;
            if (cs.P->cfl_enabled) cs.counters[COUNTER_PROGRESS] = stop;
        }
    }
    // tracked slots: bodies and fracture bonds take a single scene
    if (c0.n_tracked > 0u && ((batch_stop(c0, total) ^ total) & 1u) != 0u) {
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < c0.n_tracked; k += gridDim.x * blockDim.x)
            c0.slot_out[c0.tracked[k]] = c0.slot_in[c0.tracked[k]];
    }
    const bool one_scene = c0.n_scenes == 1u;
    if (one_scene) {
        // the batch's outcome, read once per CTA
        __shared__ int s_restore;
        if (threadIdx.x == 0) s_restore = ((batch_stop(c0, total) ^ total) & 1u) != 0u ? 1 : 0;
        __syncthreads();
        const bool restore_one = s_restore != 0;
        float best = 0.0f;
        // END_BATCH_ITEMS particles per thread and pass, their loads in flight together
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < c0.n; i0 += END_BATCH_ITEMS * stride) {
            float2 v[END_BATCH_ITEMS];
#pragma unroll
            for (int u = 0; u < END_BATCH_ITEMS; ++u) {
                const uint32_t i = i0 + (uint32_t)u * stride;
                v[u] = make_float2(0.f, 0.f);
                if (i < c0.n) {
                    if (restore_one) copy_particle(c0, i, i);
                    if (measure_speed) v[u] = restore_one ? c0.in.vel[i] : c0.out.vel[i];
                }
            }
            if (measure_speed) {
#pragma unroll
                for (int u = 0; u < END_BATCH_ITEMS; ++u) {
                    const float sp = length2(v[u]);
                    best = fmaxf(best, finite_f(sp) ? sp : FLOAT_MAX);
                }
            }
        }
        if (!measure_speed) return;
        // one atomic per CTA: every warp of the grid on one word serialises in L2
        __shared__ float s_best[32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = best;
        __syncthreads();
        if (threadIdx.x < 32) {
            best = threadIdx.x < (blockDim.x >> 5) ? s_best[threadIdx.x] : 0.0f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (threadIdx.x == 0) atomicMax(c0.counters + COUNTER_MAX_SPEED, __float_as_uint(best));
        }
        return;
    }
    for (uint32_t base = blockIdx.x * blockDim.x; base < c0.n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        float best = 0.0f;
        uint32_t scene = 0u;
        if (i < c0.n) {
            scene = scene_of_slot(c0, i);
            const bool restore = ((batch_stop(scene_ctx(c0, scene), total) ^ total) & 1u) != 0u;
            if (restore) copy_particle(c0, i, i);
            if (measure_speed) {
                const float sp = length2(restore ? c0.in.vel[i] : c0.out.vel[i]);
                best = finite_f(sp) ? sp : FLOAT_MAX;
            }
        }
        if (!measure_speed) continue;
        if (__all_sync(0xffffffffu, scene == __shfl_sync(0xffffffffu, scene, 0))) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(c0.dyn + (size_t)scene * SCENE_WORDS + 32 + COUNTER_MAX_SPEED, __float_as_uint(best));
        } else if (i < c0.n) {
            atomicMax(c0.dyn + (size_t)scene * SCENE_WORDS + 32 + COUNTER_MAX_SPEED, __float_as_uint(best));
        }
    }
}

// Counts the nodes of the last fixed-point substep whose solid / water / oil
// mass is positive (the N_ch of the algorithmic-byte model), over stamped
// tiles.  The default path counts them inside k_grid_from_acc instead.
__global__ void __launch_bounds__(TILE_NODES) k_count_active_nodes(Ctx c, uint32_t *counts)
{
    const StepParams &P = *c.P;
    const int tx = blockIdx.x, ty = blockIdx.y;
    // the stamp of the last substep is still current
    if (c.tile_stamp[ty * P.tiles_x + tx] != c.counters[COUNTER_STAMP]) return;
    const int hx = tx * TILE_X + (threadIdx.x % TILE_X), hy = ty * TILE_Y + (threadIdx.x / TILE_X);
    uint32_t s = 0, w = 0, o = 0;
    if (hx < (int)P.node_w && hy < (int)P.node_h) {
        const uint32_t n = (uint32_t)hy * P.node_w + (uint32_t)hx;
        s = c.p2g_solid[n].x > 0.f;
        w = c.p2g_water[n].x > 0.f;
        o = c.p2g_oil[n].x > 0.f;
    }
    s = __reduce_add_sync(0xffffffffu, s);
    w = __reduce_add_sync(0xffffffffu, w);
    o = __reduce_add_sync(0xffffffffu, o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counts, s);
        atomicAdd(counts + 1, w);
        atomicAdd(counts + 2, o);
    }
}

// Nodes of the last substep with positive solid / water / oil mass on the
// default path: CTA b takes tile b (of all scenes) and sums its own 16x8
// nodes' ring records in node_sources' order, as G2P does.
__global__ void __launch_bounds__(TILE_NODES) k_count_ring_nodes(Ctx c0, uint32_t *counts)
{
    const uint32_t tile = blockIdx.x;
    const Ctx c = scene_ctx(c0, c0.tile_scene[tile]);
    const StepParams &P = *c.P;
    const uint32_t local = tile - P.tile_base;
    if (local >= P.tiles_x * P.tiles_y) return;  // the scene's sentinel entry
    const uint32_t stamp = c.counters[COUNTER_STAMP];
    const int tx = (int)(local % P.tiles_x), ty = (int)(local / P.tiles_x);
    __shared__ uint2 info[9];
    if (threadIdx.x < 9) {
        const int sx = tx + (int)(threadIdx.x % 3) - 1, sy = ty + (int)(threadIdx.x / 3) - 1;
        info[threadIdx.x] = (sx >= 0 && sy >= 0 && sx < (int)P.tiles_x && sy < (int)P.tiles_y)
                                ? c.tile_info[P.tile_base + (uint32_t)(sy * (int)P.tiles_x + sx)]
                                : make_uint2(0xffffffffu, 0u);
    }
    __syncthreads();
    const int hx = tx * TILE_X + (int)(threadIdx.x % TILE_X), hy = ty * TILE_Y + (int)(threadIdx.x / TILE_X);
    uint32_t s = 0, w = 0, o = 0;
    if (hx < (int)P.node_w && hy < (int)P.node_h) {
        uint32_t channels = 0u;
#pragma unroll
        for (int k = 0; k < 9; ++k) channels |= info[k].x == stamp ? info[k].y : 0u;
        float sum[ACC_WORDS];
#pragma unroll
        for (int k = 0; k < ACC_WORDS; ++k) sum[k] = 0.f;
        add_sources(c, node_sources(P, info, tx, ty, hx, hy, stamp), true, channels, sum);
        s = sum[0] > 0.f;
        w = sum[3] > 0.f;
        o = sum[7] > 0.f;
    }
    s = __reduce_add_sync(0xffffffffu, s);
    w = __reduce_add_sync(0xffffffffu, w);
    o = __reduce_add_sync(0xffffffffu, o);
    if ((threadIdx.x & 31) == 0) {
        if (s) atomicAdd(counts, s);
        if (w) atomicAdd(counts + 1, w);
        if (o) atomicAdd(counts + 2, o);
    }
}

// ------------------------------------------------------ bodies, fracture --
// Bonded-triangle bodies ("pebbles") and fracture bonds of the multi-material
// scenes.  Body vertices and fracture endpoints are particles whose slots
// move every substep; their current slots are tracked per original index
// (slot_in for the substep's input buffer, slot_out for its output).

namespace {

// triangleDistanceSample of the CPU reference (src/lib/mpm/reference/solver.ts:
// 1190-1291) in float64 with its operations in order and no contraction.  The
// field uses this form: next to an edge the float32 offset to the closest
// point is rounding noise, and its direction is the node's normal, which the
// liquid projection and the contact impulses follow.  Returns false for a
// degenerate triangle.
__device__ bool triangle_sample_f64(double px, double py, double ax, double ay, double bx, double by, double cx,
                                    double cy, double &sd, double &nx, double &ny, double (&bary)[3])
{
    const double abx = __dsub_rn(bx, ax), aby = __dsub_rn(by, ay), acx = __dsub_rn(cx, ax), acy = __dsub_rn(cy, ay);
    const double area = __dsub_rn(__dmul_rn(abx, acy), __dmul_rn(aby, acx));
    if (!isfinite(area) || fabs(area) <= 1e-10) return false;
    const double bcx = __dsub_rn(cx, bx), bcy = __dsub_rn(cy, by), cax = __dsub_rn(ax, cx), cay = __dsub_rn(ay, cy);
    const double apx = __dsub_rn(px, ax), apy = __dsub_rn(py, ay), bpx = __dsub_rn(px, bx), bpy = __dsub_rn(py, by),
                 cpx = __dsub_rn(px, cx), cpy = __dsub_rn(py, cy);
    const double cab = __dsub_rn(__dmul_rn(abx, apy), __dmul_rn(aby, apx));
    const double cbc = __dsub_rn(__dmul_rn(bcx, bpy), __dmul_rn(bcy, bpx));
    const double cca = __dsub_rn(__dmul_rn(cax, cpy), __dmul_rn(cay, cpx));
    const bool inside = area > 0 ? (cab >= -1e-10 && cbc >= -1e-10 && cca >= -1e-10)
                                 : (cab <= 1e-10 && cbc <= 1e-10 && cca <= 1e-10);
    double best = CUDART_INF, bnx = 0, bny = 0;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const double sx = e == 0 ? ax : (e == 1 ? bx : cx), sy = e == 0 ? ay : (e == 1 ? by : cy);
        const double ex = e == 0 ? bx : (e == 1 ? cx : ax), ey = e == 0 ? by : (e == 1 ? cy : ay);
        const double dx = __dsub_rn(ex, sx), dy = __dsub_rn(ey, sy);
        const double l2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        const double ox = __dsub_rn(px, sx), oy = __dsub_rn(py, sy);
        const double t = fmax(0.0, fmin(1.0, __ddiv_rn(__dadd_rn(__dmul_rn(ox, dx), __dmul_rn(oy, dy)), l2)));
        const double qx = __dadd_rn(sx, __dmul_rn(dx, t)), qy = __dadd_rn(sy, __dmul_rn(dy, t));
        const double ddx = __dsub_rn(px, qx), ddy = __dsub_rn(py, qy);
        const double d2 = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
        if (d2 >= best) continue;
        best = d2;
        if (e == 0) {
            bary[0] = __dsub_rn(1.0, t), bary[1] = t, bary[2] = 0;
        } else if (e == 1) {
            bary[0] = 0, bary[1] = __dsub_rn(1.0, t), bary[2] = t;
        } else {
            bary[0] = t, bary[1] = 0, bary[2] = __dsub_rn(1.0, t);
        }
        if (d2 > 1e-20 && !inside) {
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(d2));
            bnx = __dmul_rn(ddx, inv);
            bny = __dmul_rn(ddy, inv);
        } else {
            const double orient = area > 0 ? 1.0 : -1.0;
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(l2));
            bnx = __dmul_rn(__dmul_rn(orient, dy), inv);
            bny = __dmul_rn(-__dmul_rn(orient, dx), inv);
        }
    }
    const double d = __dsqrt_rn(best);
    if (!isfinite(d) || !isfinite(bnx) || !isfinite(bny)) return false;
    sd = inside ? -d : d;
    nx = bnx;
    ny = bny;
    return true;
}

__device__ __forceinline__ bool body_markers_valid(const Ctx &c, uint32_t start)
{
    return start + 2u < c.n && c.bonded[start] == 1u && c.bonded[start + 1u] == 2u && c.bonded[start + 2u] == 3u;
}

__device__ __forceinline__ float2 in_position(const Ctx &c, uint32_t orig) { return c.in.pos[c.slot_in[orig]]; }

// trianglePairContact: shaders.ts:1873-1953 (SAT over the six edge normals);
// (normal, penetration), zero when apart beyond the skin or degenerate.
__device__ float3 triangle_pair_contact(const float2 (&A)[3], const float2 (&B)[3], float skin)
{
    float2 axes[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float2 *T = k < 3 ? A : B;
        const int e = k % 3;
        const float2 edge = make_float2(T[(e + 1) % 3].x - T[e].x, T[(e + 1) % 3].y - T[e].y);
        const float el = sqrtf(edge.x * edge.x + edge.y * edge.y);
        if (!finite_f(el) || el <= 1e-10f) return make_float3(0.f, 0.f, 0.f);
        axes[k] = make_float2(edge.y / el, -edge.x / el);
    }
    bool separated = false;
    float largest = -FLOAT_MAX, smallest = FLOAT_MAX;
    float2 axis = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float2 u = axes[k];
        const float a0 = A[0].x * u.x + A[0].y * u.y, a1 = A[1].x * u.x + A[1].y * u.y, a2 = A[2].x * u.x + A[2].y * u.y;
        const float b0 = B[0].x * u.x + B[0].y * u.y, b1 = B[1].x * u.x + B[1].y * u.y, b2 = B[2].x * u.x + B[2].y * u.y;
        const float min_a = fminf(a0, fminf(a1, a2)), max_a = fmaxf(a0, fmaxf(a1, a2));
        const float min_b = fminf(b0, fminf(b1, b2)), max_b = fmaxf(b0, fmaxf(b1, b2));
        const float gap = fmaxf(min_b - max_a, min_a - max_b);
        if (gap > 0.f) {
            separated = true;
            if (gap > largest) {
                largest = gap;
                axis = u;
            }
        } else if (!separated && -gap < smallest) {
            smallest = -gap;
            axis = u;
        }
    }
    if (separated && largest > skin) return make_float3(0.f, 0.f, 0.f);
    const float2 delta = make_float2((A[0].x + A[1].x + A[2].x - B[0].x - B[1].x - B[2].x) / 3.0f,
                                     (A[0].y + A[1].y + A[2].y - B[0].y - B[1].y - B[2].y) / 3.0f);
    if (delta.x * axis.x + delta.y * axis.y < 0.f) axis = make_float2(-axis.x, -axis.y);
    const float pen = separated ? skin - largest : skin + smallest;
    if (!finite_f(pen) || pen <= 0.f) return make_float3(0.f, 0.f, 0.f);
    return make_float3(axis.x, axis.y, pen);
}

// triangleBodyContact: shaders.ts:1955-1992, on the substep's input
// positions; the normal points from `other` towards `body`.
__device__ float3 body_contact(const Ctx &c, uint32_t body, uint32_t other)
{
    const bool first_is_body = body < other;
    const uint32_t fs = c.body_starts[first_is_body ? body : other];
    const uint32_t ss = c.body_starts[first_is_body ? other : body];
    float2 A[3], B[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        A[k] = in_position(c, fs + (uint32_t)k);
        B[k] = in_position(c, ss + (uint32_t)k);
    }
    const float2 amin = make_float2(fminf(A[0].x, fminf(A[1].x, A[2].x)), fminf(A[0].y, fminf(A[1].y, A[2].y)));
    const float2 amax = make_float2(fmaxf(A[0].x, fmaxf(A[1].x, A[2].x)), fmaxf(A[0].y, fmaxf(A[1].y, A[2].y)));
    const float2 bmin = make_float2(fminf(B[0].x, fminf(B[1].x, B[2].x)), fminf(B[0].y, fminf(B[1].y, B[2].y)));
    const float2 bmax = make_float2(fmaxf(B[0].x, fmaxf(B[1].x, B[2].x)), fmaxf(B[0].y, fmaxf(B[1].y, B[2].y)));
    const float2 gap = make_float2(fmaxf(bmin.x - amax.x, amin.x - bmax.x), fmaxf(bmin.y - amax.y, amin.y - bmax.y));
    const float skin = c.P->dx * TRIANGLE_CONTACT_SKIN_CELLS;
    if (fmaxf(gap.x, gap.y) > skin) return make_float3(0.f, 0.f, 0.f);
    const float3 contact = triangle_pair_contact(A, B, skin);
    return first_is_body ? contact : make_float3(-contact.x, -contact.y, contact.z);
}

// bondEdgeCorrection: shaders.ts:1856-1871
__device__ __forceinline__ bool edge_correction(float2 first, float2 second, float rest, float stiffness,
                                                float2 &corr)
{
    const float2 d = make_float2(second.x - first.x, second.y - first.y);
    const float dist = sqrtf(d.x * d.x + d.y * d.y);
    if (!finite_f(dist) || dist <= 1e-10f) return false;
    const float k = (dist - rest) * stiffness * 0.5f / dist;
    corr = make_float2(d.x * k, d.y * k);
    return true;
}

__device__ __forceinline__ bool move_vertex(const Ctx &c, uint32_t slot, float2 pos, float2 vel)
{
    const StepParams &P = *c.P;
    const float2 bx = confine_axis(pos.x, vel.x, P.domain_w);
    const float2 by = confine_axis(pos.y, vel.y, P.domain_h);
    const float2 p = make_float2(bx.x, by.x), v = make_float2(bx.y, by.y);
    if (!finite2(p) || !finite2(v)) return false;
    c.out.pos[slot] = p;
    c.out.vel[slot] = v;
    return true;
}

}  // namespace

// buildTriangleField (shaders.ts:1299-1436): for every halo node, the nearest
// body within the band (ties keep the lower body), its normal and barycentric
// weights, with bodies staged in shared memory in ascending order; samples in
// float64 (triangle_sample_f64).
__global__ void __launch_bounds__(TILE_NODES) k_triangle_field(Ctx c)
{
    const StepParams &P = *c.P;
    __shared__ float2 s_v0[FIELD_BODY_CHUNK], s_v1[FIELD_BODY_CHUNK], s_v2[FIELD_BODY_CHUNK];
    __shared__ float2 s_min[FIELD_BODY_CHUNK], s_max[FIELD_BODY_CHUNK];
    __shared__ uint32_t s_start[FIELD_BODY_CHUNK], s_valid[FIELD_BODY_CHUNK];
    const int hx = blockIdx.x * TILE_X + (int)(threadIdx.x % TILE_X);
    const int hy = blockIdx.y * TILE_Y + (int)(threadIdx.x / TILE_X);
    const bool active = hx < (int)P.node_w && hy < (int)P.node_h && *(volatile uint32_t *)c.status == 0u;
    const double px = (double)(hx - 1) * (double)P.dx, py = (double)(hy - 1) * (double)P.dx;
    const double band = (double)P.band;
    double best = band, best_nx = 0, best_ny = 0, best_bary[3] = {0, 0, 0};
    uint32_t body1 = 0u;
    bool failed = false;
    for (uint32_t chunk = 0; chunk < P.n_bodies; chunk += FIELD_BODY_CHUNK) {
        __syncthreads();
        const uint32_t b = chunk + threadIdx.x;
        if (b < P.n_bodies) {
            const uint32_t start = c.body_starts[b];
            s_start[threadIdx.x] = start;
            if (start + 2u >= c.n) {
                s_valid[threadIdx.x] = 0u;
            } else {
                const float2 p0 = in_position(c, start), p1 = in_position(c, start + 1u),
                             p2 = in_position(c, start + 2u);
                s_v0[threadIdx.x] = p0;
                s_v1[threadIdx.x] = p1;
                s_v2[threadIdx.x] = p2;
                s_min[threadIdx.x] = make_float2(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)));
                s_max[threadIdx.x] = make_float2(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)));
                s_valid[threadIdx.x] = 1u;
            }
        }
        __syncthreads();
        if (!active || failed) continue;
        const uint32_t count = min((uint32_t)FIELD_BODY_CHUNK, P.n_bodies - chunk);
        for (uint32_t k = 0; k < count; ++k) {
            if (!s_valid[k]) {
                fail(c.status, ERROR_TRIANGLE_BOND);
                failed = true;
                break;
            }
            const double ox = fmax(fmax((double)s_min[k].x - px, 0.0), px - (double)s_max[k].x);
            const double oy = fmax(fmax((double)s_min[k].y - py, 0.0), py - (double)s_max[k].y);
            if (ox * ox + oy * oy > band * band) continue;
            double sd, nx, ny, bary[3];
            if (!triangle_sample_f64(px, py, s_v0[k].x, s_v0[k].y, s_v1[k].x, s_v1[k].y, s_v2[k].x, s_v2[k].y, sd, nx,
                                     ny, bary)) {
                fail_at(c.status, s_start[k], ERROR_TRIANGLE_CONTACT);
                failed = true;
                break;
            }
            // a node joins the field within the band; a later body takes it
            // only when strictly nearer (buildTriangleField, solver.ts:1064-1165)
            if (body1 == 0u ? sd <= band : sd < best) {
                best = sd;
                body1 = s_start[k] + 1u;
                best_nx = nx;
                best_ny = ny;
                best_bary[0] = bary[0];
                best_bary[1] = bary[1];
                best_bary[2] = bary[2];
            }
        }
    }
    if (active && !failed) {
        TriField f;
        f.sd = (float)best;
        f.body1 = body1;
        f.nx = (float)best_nx;
        f.ny = (float)best_ny;
        f.b1 = (float)best_bary[1];
        f.b2 = (float)best_bary[2];
        f.ix = 0.f;
        f.iy = 0.f;
        c.field[(uint32_t)hy * P.node_w + (uint32_t)hx] = f;
    }
}

// applyTriangleContactImpulses (shaders.ts:2535-2670): one CTA per body sums
// the barycentric shares of the fluid impulses stored at the field nodes it
// owns (strided partial sums, then a halving reduction) and adds them to the
// vertex velocities.
__global__ void __launch_bounds__(BODY_THREADS) k_body_impulses(Ctx c)
{
    const StepParams &P = *c.P;
    __shared__ int s_valid;
    __shared__ int s_box[4];
    __shared__ uint32_t s_start;
    __shared__ float2 s_i[3][BODY_THREADS];
    for (uint32_t b = blockIdx.x; b < P.n_bodies; b += gridDim.x) {
        if (threadIdx.x == 0) {
            s_valid = 0;
            if (*(volatile uint32_t *)c.status == 0u) {
                const uint32_t start = c.body_starts[b];
                if (!body_markers_valid(c, start)) {
                    fail_at(c.status, start, ERROR_TRIANGLE_BOND);
                } else {
                    const float2 p0 = in_position(c, start), p1 = in_position(c, start + 1u),
                                 p2 = in_position(c, start + 2u);
                    const float r = P.contact_reach;
                    const float mnx = fminf(p0.x, fminf(p1.x, p2.x)) - r, mny = fminf(p0.y, fminf(p1.y, p2.y)) - r;
                    const float mxx = fmaxf(p0.x, fmaxf(p1.x, p2.x)) + r, mxy = fmaxf(p0.y, fmaxf(p1.y, p2.y)) + r;
                    const int hi_x = (int)P.cells_x + 1, hi_y = (int)P.cells_y + 1;
                    s_box[0] = min(max((int)floorf(mnx / P.dx), -1), hi_x);
                    s_box[1] = min(max((int)floorf(mny / P.dx), -1), hi_y);
                    s_box[2] = min(max((int)ceilf(mxx / P.dx), -1), hi_x);
                    s_box[3] = min(max((int)ceilf(mxy / P.dx), -1), hi_y);
                    s_start = start;
                    s_valid = 1;
                }
            }
        }
        __syncthreads();
        float2 i0 = make_float2(0.f, 0.f), i1 = i0, i2 = i0;
        if (s_valid) {
            const int w = s_box[2] - s_box[0] + 1, h = s_box[3] - s_box[1] + 1;
            const uint32_t body1 = s_start + 1u;
            for (int k = threadIdx.x; k < w * h; k += BODY_THREADS) {
                const TriField f = c.field[node_index(P, s_box[0] + k % w, s_box[1] + k / w)];
                if (f.body1 != body1) continue;
                const float w0 = 1.0f - f.b1 - f.b2;
                i0 = make_float2(i0.x + w0 * f.ix, i0.y + w0 * f.iy);
                i1 = make_float2(i1.x + f.b1 * f.ix, i1.y + f.b1 * f.iy);
                i2 = make_float2(i2.x + f.b2 * f.ix, i2.y + f.b2 * f.iy);
            }
        }
        s_i[0][threadIdx.x] = i0;
        s_i[1][threadIdx.x] = i1;
        s_i[2][threadIdx.x] = i2;
        __syncthreads();
        for (int stride = BODY_THREADS / 2; stride > 0; stride /= 2) {
            if ((int)threadIdx.x < stride) {
#pragma unroll
                for (int v = 0; v < 3; ++v)
                    s_i[v][threadIdx.x] = make_float2(s_i[v][threadIdx.x].x + s_i[v][threadIdx.x + stride].x,
                                                      s_i[v][threadIdx.x].y + s_i[v][threadIdx.x + stride].y);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0 && s_valid && *(volatile uint32_t *)c.status == 0u) {
            const float inv_m = 1.0f / P.particle_mass;
            float2 v[3];
            bool ok = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float2 old = c.out.vel[c.slot_out[s_start + (uint32_t)k]];
                v[k] = make_float2(old.x + inv_m * s_i[k][0].x, old.y + inv_m * s_i[k][0].y);
                ok = ok && finite2(v[k]);
            }
            if (!ok) {
                fail_at(c.status, s_start, ERROR_TRIANGLE_CONTACT);
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k) c.out.vel[c.slot_out[s_start + (uint32_t)k]] = v[k];
            }
        }
        __syncthreads();
    }
}

// solveBondedTriangles (shaders.ts:2672-2797): two Gauss-Seidel passes over
// the three edges in offsets from the first vertex, stiffness
// min(k (dt / dtRef)^2, 1); the displacement also enters the velocity.
__global__ void k_body_bonded(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.n_bodies || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t start = c.body_starts[b];
    if (!body_markers_valid(c, start)) {
        fail_at(c.status, start, ERROR_TRIANGLE_BOND);
        return;
    }
    uint32_t slot[3];
    float2 pos[3], vel[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        slot[k] = c.slot_out[start + (uint32_t)k];
        pos[k] = c.out.pos[slot[k]];
        vel[k] = c.out.vel[slot[k]];
    }
    const float2 orig[3] = {make_float2(0.f, 0.f), make_float2(pos[1].x - pos[0].x, pos[1].y - pos[0].y),
                            make_float2(pos[2].x - pos[0].x, pos[2].y - pos[0].y)};
    float2 off[3] = {orig[0], orig[1], orig[2]};
    const float dt = P.dt, inv_dt = 1.0f / dt;
    const float ratio = dt / P.bond_reference_dt;
    const float stiffness = fminf(P.bond_stiffness * ratio * ratio, 1.0f);
    for (int it = 0; it < BONDED_TRIANGLE_SOLVER_ITERATIONS; ++it) {
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const int a0 = e, a1 = (e + 1) % 3;
            float2 corr;
            if (!edge_correction(off[a0], off[a1], P.bond_rest_length, stiffness, corr)) {
                fail_at(c.status, start, ERROR_TRIANGLE_BOND);
                return;
            }
            off[a0] = make_float2(off[a0].x + corr.x, off[a0].y + corr.y);
            off[a1] = make_float2(off[a1].x - corr.x, off[a1].y - corr.y);
        }
    }
    float2 np[3], nv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 disp = make_float2(off[k].x - orig[k].x, off[k].y - orig[k].y);
        np[k] = make_float2(pos[k].x + disp.x, pos[k].y + disp.y);
        nv[k] = make_float2(vel[k].x + disp.x * inv_dt, vel[k].y + disp.y * inv_dt);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 bx = confine_axis(np[k].x, nv[k].x, P.domain_w);
        const float2 by = confine_axis(np[k].y, nv[k].y, P.domain_h);
        np[k] = make_float2(bx.x, by.x);
        nv[k] = make_float2(bx.y, by.y);
        if (!finite2(np[k]) || !finite2(nv[k])) {
            fail_at(c.status, start, ERROR_TRIANGLE_CONTACT);
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        c.out.pos[slot[k]] = np[k];
        c.out.vel[slot[k]] = nv[k];
    }
}

// gatherTriangleContactStates (shaders.ts:2044-2112): mean vertex velocity;
// the contact degree comes from k_body_pairs when pair contacts are cached,
// else from a scan of the other bodies here.
__global__ void k_body_states(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.n_bodies || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t start = c.body_starts[b];
    if (!body_markers_valid(c, start)) {
        fail_at(c.status, start, ERROR_TRIANGLE_BOND);
        return;
    }
    uint32_t count = 0;
    if (!c.pair_cache) {
        const uint32_t obj = c.obj[start];
        for (uint32_t o = 0; o < P.n_bodies; ++o) {
            if (o == b) continue;
            const uint32_t os = c.body_starts[o];
            if (!body_markers_valid(c, os)) {
                fail_at(c.status, os, ERROR_TRIANGLE_BOND);
                return;
            }
            if (c.obj[os] == obj) continue;
            if (body_contact(c, b, o).z > 0.f) ++count;
        }
    }
    float2 v = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 vk = c.out.vel[c.slot_out[start + (uint32_t)k]];
        v = make_float2(v.x + vk.x, v.y + vk.y);
    }
    c.body_vel[b] = make_float2(v.x / 3.0f, v.y / 3.0f);
    c.contact_count[b] = count;
}

// gatherTrianglePairContacts (shaders.ts:1994-2042): the contact of every
// unordered body pair of different objects, and the contact degrees.
__global__ void k_body_pairs(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t nb = P.n_bodies;
    const uint32_t pair = blockIdx.x * blockDim.x + threadIdx.x;
    if (pair >= nb * nb) return;
    const uint32_t b = pair / nb, o = pair % nb;
    if (b >= o || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t bs = c.body_starts[b], os = c.body_starts[o];
    if (c.obj[os] == c.obj[bs]) return;
    const float3 contact = body_contact(c, b, o);
    c.pair_cache[pair] = make_float4(contact.x, contact.y, contact.z, 0.f);
    if (contact.z > 0.f) {
        atomicAdd(&c.contact_count[b], 1u);
        atomicAdd(&c.contact_count[o], 1u);
    }
}

// applyTrianglePairContacts (shaders.ts:2799-2955): Jacobi normal impulses
// against every contacting body in ascending order, relaxed by 0.25 over the
// larger contact degree, added to the three vertex velocities.
__global__ void k_body_apply(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t nb = P.n_bodies;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t start = c.body_starts[b];
    if (!body_markers_valid(c, start)) {
        fail_at(c.status, start, ERROR_TRIANGLE_BOND);
        return;
    }
    const float2 vb = c.body_vel[b];
    const uint32_t count = c.contact_count[b];
    const uint32_t obj = c.obj[start];
    const float body_mass = 3.0f * P.particle_mass;
    float2 delta = make_float2(0.f, 0.f);
    for (uint32_t o = 0; count != 0u && o < nb; ++o) {
        if (o == b) continue;
        float3 contact = make_float3(0.f, 0.f, 0.f);
        if (c.pair_cache) {
            const float4 cached = c.pair_cache[min(b, o) * nb + max(b, o)];
            if (c.obj[c.body_starts[o]] == obj || cached.z <= 0.f) continue;
            contact = b < o ? make_float3(cached.x, cached.y, cached.z) : make_float3(-cached.x, -cached.y, cached.z);
        }
        const uint32_t os = c.body_starts[o];
        if (!body_markers_valid(c, os)) {
            fail_at(c.status, os, ERROR_TRIANGLE_BOND);
            return;
        }
        if (c.obj[os] == obj) continue;
        if (!c.pair_cache) {
            contact = body_contact(c, b, o);
            if (contact.z <= 0.f) continue;
        }
        const float2 vo = c.body_vel[o];
        const uint32_t degree = max(count, c.contact_count[o]);
        if (degree == 0u) {
            fail_at(c.status, start, ERROR_TRIANGLE_CONTACT);
            return;
        }
        const float weight = 1.0f / (float)degree;
        const float rn = (vb.x - vo.x) * contact.x + (vb.y - vo.y) * contact.y;
        if (rn < 0.f) {
            const float magnitude = -rn / (2.0f / body_mass);
            const float iw = TRIANGLE_CONTACT_IMPULSE_RELAXATION * weight;
            delta = make_float2(delta.x + iw * magnitude * contact.x / body_mass,
                                delta.y + iw * magnitude * contact.y / body_mass);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t slot = c.slot_out[start + (uint32_t)k];
        const float2 v = c.out.vel[slot];
        if (!move_vertex(c, slot, c.out.pos[slot], make_float2(v.x + delta.x, v.y + delta.y))) {
            fail_at(c.status, start, ERROR_TRIANGLE_CONTACT);
            return;
        }
    }
}

// validateCflParticles (shaders.ts:2456-2461): the CFL check of every particle
// after the body passes (G2P checks them itself when there are no bodies).
__global__ void k_validate_cfl(Ctx c)
{
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= c.n) return;
    const Material m = c.mats[c.out.mat[d]];
    validate_cfl(c, c.out.orig[d], m, c.out.vel[d], c.out.F[d], c.out.damage[d], c.out.vol[d], -1.0f);
}

// updateFractureBonds (shaders.ts:2957-3003): tensile strain of each bond
// from the committed positions -> damage, broken latch.
__global__ void k_fracture_bonds(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t bi = blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= P.n_bonds || *(volatile uint32_t *)c.status != 0u) return;
    uint32_t *w = c.bonds + 6u * bi;
    const uint32_t first = w[0], second = w[1];
    const float rest = __uint_as_float(w[2]), failure = __uint_as_float(w[3]);
    float damage = __uint_as_float(w[4]);
    if (first >= P.fracture_particles || second >= P.fracture_particles || first >= c.n || second >= c.n ||
        !finite_f(rest) || rest <= 0.f || !finite_f(failure) || failure <= 0.f) {
        fail_at(c.status, min(first, second), ERROR_FRACTURE_BOND);
        return;
    }
    if (w[5] != 0u) {
        w[4] = __float_as_uint(1.0f);
        return;
    }
    const float2 a = c.out.pos[c.slot_out[first]], b = c.out.pos[c.slot_out[second]];
    const float sx = b.x - a.x, sy = b.y - a.y;
    const float dist = sqrtf(sx * sx + sy * sy);
    if (!finite_f(dist)) {
        fail_at(c.status, first, ERROR_FRACTURE_BOND);
        return;
    }
    const float strain = fmaxf(0.f, (dist - rest) / rest);
    damage = fmaxf(damage, fminf(1.0f, strain / failure));
    if (strain >= failure) {
        damage = 1.0f;
        w[5] = 1u;
    }
    w[4] = __float_as_uint(damage);
}

// applyFractureParticleDamage (shaders.ts:3005-3039): a Neo-Hookean endpoint
// takes the largest damage of its bonds (CSR incidence).
__global__ void k_fracture_damage(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.n_endpoints || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t i = c.endpoints[k];
    const uint32_t first = c.topology[i], next = c.topology[i + 1u];
    if (next < first || next > P.fracture_incidence) {
        fail_at(c.status, i, ERROR_FRACTURE_BOND);
        return;
    }
    const uint32_t slot = c.slot_out[i];
    if (c.mats[c.out.mat[slot]].model != MODEL_NEO_HOOKEAN) return;
    float damage = fminf(fmaxf(c.out.damage[slot], 0.f), 1.0f);
    const uint32_t base = P.fracture_particles + 1u;
    for (uint32_t inc = first; inc < next; ++inc) {
        const uint32_t bond = c.topology[base + inc];
        if (bond >= P.n_bonds) {
            fail_at(c.status, i, ERROR_FRACTURE_BOND);
            return;
        }
        damage = fmaxf(damage, __uint_as_float(c.bonds[6u * bond + 4u]));
    }
    c.out.damage[slot] = damage;
}

// The tile count (and with the records variant the P2G record) of each
// tracked particle, from its state after the body and fracture passes (G2P
// left them out).
__global__ void k_body_finish(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.n_tracked || *(volatile uint32_t *)c.status != 0u) return;
    const uint32_t orig = c.tracked[k];
    const uint32_t d = c.slot_out[orig];
    Stencil st;
    if (!make_stencil_fast(P, c.out.pos[d], st) || !stencil_fits(P, st.bx, st.by)) {
        fail(c.status, ERROR_STENCIL);
        return;
    }
    const uint32_t key = particle_tile(P, st.bx, st.by);
    c.ranks[d] = atomicAdd(&c.tile_count[key], 1u);
    c.keys[d] = bucket_key(key, st.bx, st.by);
    if (c.rec_state) {
        const Material m = c.mats[c.out.mat[d]];
        write_record(c, d, m, st, c.out.vel[d], c.out.F[d], c.out.vol[d], c.out.damage[d], c.out.pvol[d], c.out.C[d]);
    }
}

// --------------------------------------------------------- interaction --

// removeParticlesInOutlet (shaders.ts:3041-3065): water and oil particles of
// the current state inside `bounds` (min x, min y, max x, max y) leave the
// slot range.  Kept particles are packed into `out` (slot order free: every
// sum of the default path has a fixed order regardless), removed ones into
// `removed` with their original index; counters[0] / [1] count them.
__global__ void k_outlet_compact(Ctx c, float4 bounds, ParticleBuffers removed, uint32_t *counters)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const Material m = c.mats[c.in.mat[i]];
    const float2 p = c.in.pos[i];
    const bool liquid = m.model == MODEL_WATER || m.model == MODEL_OIL;
    if (liquid && p.x >= bounds.x && p.y >= bounds.y && p.x <= bounds.z && p.y <= bounds.w) {
        const uint32_t j = atomicAdd(counters + 1, 1u);
        removed.pos[j] = p;
        removed.vel[j] = c.in.vel[i];
        removed.C[j] = c.in.C[i];
        removed.F[j] = c.in.F[i];
        removed.pvol[j] = c.in.pvol[i];
        removed.damage[j] = c.in.damage[i];
        removed.vol[j] = c.in.vol[i];
        removed.mat[j] = c.in.mat[i];
        removed.orig[j] = c.in.orig[i];
        return;
    }
    const uint32_t j = atomicAdd(counters, 1u);
    copy_particle(c, i, j);
    const uint32_t orig = c.in.orig[i];
    if (is_tracked(c, orig)) c.slot_out[orig] = j;
}

// pickParticle (shaders.ts:3082-3116): the particle nearest to (px, py)
// within sqrt(r2), the lowest original index among equally near ones, as the
// minimum of (squared distance bits << 32 | original index).
__global__ void k_pick(Ctx c, float px, float py, float r2, unsigned long long *best)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = ~0ull;
    if (i < c.n) {
        const float2 p = c.in.pos[i];
        const float ox = __fsub_rn(p.x, px), oy = __fsub_rn(p.y, py);
        const float d2 = __fadd_rn(__fmul_rn(ox, ox), __fmul_rn(oy, oy));
        if (d2 <= r2) key = ((unsigned long long)__float_as_uint(d2) << 32) | c.in.orig[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
    }
    if ((threadIdx.x & 31u) == 0u && key != ~0ull) atomicMin(best, key);
}

// cloneObject (shaders.ts:3118-3147): the particles with original indices
// [start, start + count) of the current state are copied to the new slots
// n .. n + count - 1 as original indices orig_base .. orig_base + count - 1,
// moved by `offset` and clamped to the domain [0, domain.x] x [0, domain.y],
// under `object_id`.
__global__ void k_clone(Ctx c, uint32_t start, uint32_t count, float2 offset, float2 domain, uint32_t orig_base,
                        uint32_t object_id)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const uint32_t orig = c.in.orig[i];
    if (orig < start || orig - start >= count) return;
    const uint32_t k = orig - start, j = c.n + k;
    const float2 p = c.in.pos[i];
    c.in.pos[j] = make_float2(fminf(fmaxf(__fadd_rn(p.x, offset.x), 0.0f), domain.x),
                              fminf(fmaxf(__fadd_rn(p.y, offset.y), 0.0f), domain.y));
    c.in.vel[j] = c.in.vel[i];
    c.in.C[j] = c.in.C[i];
    c.in.F[j] = c.in.F[i];
    c.in.pvol[j] = c.in.pvol[i];
    c.in.damage[j] = c.in.damage[i];
    c.in.vol[j] = c.in.vol[i];
    c.in.mat[j] = c.in.mat[i];
    c.in.orig[j] = orig_base + k;
    const_cast<uint32_t *>(c.obj)[orig_base + k] = object_id;
    const_cast<uint32_t *>(c.bonded)[orig_base + k] = 0u;
}

// ------------------------------------------------ surface occupancy --

// gatherSurfaceOccupancy (shaders.ts:710-806): the water and oil display
// area of the liquid particles in the current slots spread over their 3x3
// stencils, 2 V det(F) w / dx^2 per node, one thread per slot.  Each
// contribution is added as a 64-bit fixed-point integer (SURFACE_SCALE
// units per unit of area), so the sums do not depend on the order of the
// atomics and every run is bit-identical (the reference adds floats in the
// order of its node buckets).  Nothing is gathered while a numerical status
// or surface flag is pending (status words 0 and 7).  Flags go to status
// word 7 as in the reference: SURFACE_ERROR_BUCKET when the stencil leaves
// the halo, SURFACE_ERROR_PARTICLE_AREA for a non-finite position or an
// invalid area, determinant or weight, SURFACE_ERROR_ACCUMULATION when a
// sum leaves the fixed-point range.  The geometry comes as arguments: the
// solver's step parameters need not be uploaded yet.
__global__ void k_surface_gather(Ctx c, SurfaceGeometry g, unsigned long long *acc)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    if (*(volatile uint32_t *)c.status != 0u || *(volatile uint32_t *)(c.status + 7) != 0u) return;
    const Material m = c.mats[c.in.mat[i]];
    const uint32_t phase = m.model == MODEL_WATER ? 0u : (m.model == MODEL_OIL ? 1u : 2u);
    if (phase == 2u) return;
    Stencil s;
    const float2 pos = c.in.pos[i];
    if (!stencil_from_grid(__fdiv_rn(pos.x, g.dx), __fdiv_rn(pos.y, g.dx), s)) {
        fail(c.status + 7, SURFACE_ERROR_PARTICLE_AREA);
        return;
    }
    if (s.bx < -1 || s.by < -1 || s.bx + 2 > (int)g.cells_x + 1 || s.by + 2 > (int)g.cells_y + 1) {
        fail(c.status + 7, SURFACE_ERROR_BUCKET);
        return;
    }
    const float det = det2(c.in.F[i]);
    const float volume = c.in.vol[i];
    const float area = __fmul_rn(volume, det);
    const float display = __fmul_rn(area, 2.0f);
    const float cell = __fmul_rn(g.dx, g.dx);
    if (!finite_f(det) || det <= 0.0f || !finite_f(volume) || volume <= 0.0f || !finite_f(area) || area <= 0.0f) {
        fail(c.status + 7, SURFACE_ERROR_PARTICLE_AREA);
        return;
    }
    unsigned long long units[9];
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const float w = __fmul_rn(quad_weight(s.fx, ox), quad_weight(s.fy, oy));
            const float a = __fdiv_rn(__fmul_rn(display, w), cell);
            if (!finite_f(w) || w < 0.0f || !finite_f(a) || a < 0.0f) {
                fail(c.status + 7, SURFACE_ERROR_PARTICLE_AREA);
                return;
            }
            const double scaled = rint((double)a * SURFACE_SCALE);
            if (scaled >= SURFACE_LIMIT) {
                fail(c.status + 7, SURFACE_ERROR_ACCUMULATION);
                return;
            }
            units[oy * 3 + ox] = (unsigned long long)scaled;
        }
    }
    const uint32_t n00 = (uint32_t)(s.by + 1) * g.node_w + (uint32_t)(s.bx + 1);
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const unsigned long long u = units[oy * 3 + ox];
            if (u == 0ull) continue;
            const uint32_t n = n00 + (uint32_t)oy * g.node_w + (uint32_t)ox;
            const unsigned long long prev = atomicAdd(acc + 2u * n + phase, u);
            if (prev + u < prev) fail(c.status + 7, SURFACE_ERROR_ACCUMULATION);
        }
    }
}

// The fixed-point sums of k_surface_gather as (water, oil) areas per node.
__global__ void k_surface_decode(const unsigned long long *acc, float2 *field, uint32_t nodes)
{
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    const ulonglong2 v = reinterpret_cast<const ulonglong2 *>(acc)[n];
    field[n] = make_float2((float)((double)v.x / SURFACE_SCALE), (float)((double)v.y / SURFACE_SCALE));
}

// the instances the host launches
// The trial deformation G2P computes (deformation_trial) for `n` given
// (F, C) pairs: trial F, increment, determinant and substep count, or the
// flags of a failed integration in `flags`.
__global__ void k_probe_deformation(const float4 *F, const float4 *C, float dt, uint32_t n, float4 *trial,
                                    float2 *increment_det, uint32_t *substeps, uint32_t *flags)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DeformationTrial t;
    t.F = make_float4(0.f, 0.f, 0.f, 0.f);
    t.increment = t.det = 0.f;
    t.substeps = 0u;
    flags[i] = deformation_trial(F[i], C[i], dt, t);
    trial[i] = t.F;
    increment_det[i] = make_float2(t.increment, t.det);
    substeps[i] = t.substeps;
}

template __global__ void k_p2g_gather<false, STAGE_CAP, false, false>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP, false, false>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP_NARROW, false, false>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP_NARROW, false, false>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP, true, false>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP, true, false>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP_NARROW, true, false>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP_NARROW, true, false>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP, false, true>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP, false, true>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP_NARROW, false, true>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP_NARROW, false, true>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP, true, true>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP, true, true>(Ctx);
template __global__ void k_p2g_gather<false, STAGE_CAP_NARROW, true, true>(Ctx);
template __global__ void k_p2g_gather<true, STAGE_CAP_NARROW, true, true>(Ctx);
template __global__ void k_substep<false, STAGE_CAP, false>(Ctx);
template __global__ void k_substep<true, STAGE_CAP, false>(Ctx);
template __global__ void k_substep<false, STAGE_CAP_NARROW, false>(Ctx);
template __global__ void k_substep<true, STAGE_CAP_NARROW, false>(Ctx);
template __global__ void k_substep<false, STAGE_CAP, true>(Ctx);
template __global__ void k_substep<true, STAGE_CAP, true>(Ctx);
template __global__ void k_substep<false, STAGE_CAP_NARROW, true>(Ctx);
template __global__ void k_substep<true, STAGE_CAP_NARROW, true>(Ctx);
template __global__ void k_g2p_tile<false, false, false, false>(Ctx);
template __global__ void k_g2p_tile<false, true, false, false>(Ctx);
template __global__ void k_g2p_tile<true, false, false, false>(Ctx);
template __global__ void k_g2p_tile<false, false, true, false>(Ctx);
template __global__ void k_g2p_tile<true, false, true, false>(Ctx);
template __global__ void k_g2p_tile<false, false, false, true>(Ctx);
template __global__ void k_g2p_tile<false, true, false, true>(Ctx);
template __global__ void k_g2p_tile<true, false, false, true>(Ctx);
template __global__ void k_g2p_tile<false, false, true, true>(Ctx);
template __global__ void k_g2p_tile<true, false, true, true>(Ctx);

}  // namespace mpm
