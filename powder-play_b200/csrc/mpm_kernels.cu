// mpm_kernels.cu -- sm_100a kernels of one MLS-MPM substep.
//
// Substep, gather P2G (the reference default path, src/lib/mpm/kernels/solver.ts:1465-1570):
//   k_count -> k_scan_reduce -> k_scan_top -> k_scan_apply -> k_scatter
//   -> k_rank_prepare -> k_p2g_gather -> k_grid_update -> k_g2p -> k_commit
// Substep, fixed-point atomic P2G (createExperimentalMpmMlsAtomicGpuSolver):
//   k_prepare_scatter -> k_fixed_decode -> k_grid_update -> k_g2p -> k_commit
// After a CFL-guarded batch: k_speed_max.
//
// Every kernel returns early once the persistent status word is non-zero, as
// every WGSL entry point does (shaders.ts: `atomicLoad(&stateError[0]) != 0u`).
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

__device__ __forceinline__ bool make_stencil(const StepParams &P, float2 pos, Stencil &s)
{
    float gx = __fdiv_rn(pos.x, P.dx), gy = __fdiv_rn(pos.y, P.dx);
    if (!finite_f(gx) || !finite_f(gy)) return false;
    float fbx = floorf(__fsub_rn(gx, 0.5f)), fby = floorf(__fsub_rn(gy, 0.5f));
    s.bx = (int)fbx;
    s.by = (int)fby;
    s.fx = __fsub_rn(gx, (float)s.bx);
    s.fy = __fsub_rn(gy, (float)s.by);
    return true;
}

// prepareParticle: shaders.ts:808-963.  Computes the per-particle stress
// cache (affine momentum A = m C + (-dt V 4/dx^2) P F^T), mass and current
// liquid area.  Returns false after raising the reference's status flags.
__device__ bool prepare_particle(const Ctx &c, uint32_t i, float4 &affine, float &mass, float &vliq,
                                 uint32_t &model)
{
    const StepParams &P = *c.P;
    const float4 F = c.in.F[i];
    const float volume = c.vol[i];
    const Material m = c.mats[c.mat[i]];
    model = m.model;
    const float det = det2(F);
    if (!finite_f(det) || det <= 0.0f || !finite_f(volume) || volume <= 0.0f) {
        fail(c.status, ERROR_DEFORMATION);
        return false;
    }
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t bad = ERROR_P2G | ERROR_P2G_INVALID_MATERIAL;
    if (m.model == MODEL_NEO_HOOKEAN) {
        const float damage = c.in.damage[i];
        if (!finite_f(damage) || damage < 0.0f || damage > 1.0f) {
            fail_at(c.status, i, bad);
            return false;
        }
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
            const float pv = c.in.pvol[i];
            if (!finite_f(pv) || pv < SNOW_MIN_PLASTIC_VOLUME || pv > SNOW_MAX_PLASTIC_VOLUME) {
                fail_at(c.status, i, bad);
                return false;
            }
            const float e = fminf(fmaxf(SNOW_HARDENING * (1.0f - pv), -SNOW_MAX_HARDENING_EXPONENT),
                                  SNOW_MAX_HARDENING_EXPONENT);
            hardening = expf(e);
        }
        const Decomp d = decompose(F);
        if (!finite_f(d.s0) || !finite_f(d.s1) || d.s0 <= 0.0f || d.s1 <= 0.0f) {
            fail_at(c.status, i, bad);
            return false;
        }
        const float4 R = polar_rotation(d);
        const float mu = m.mu * hardening, lambda = m.lambda * hardening;
        const float4 diff = make_float4(F.x - R.x, F.y - R.y, F.z - R.z, F.w - R.w);
        const float shear = 2.0f * mu;
        const float volumetric = lambda * det * (det - 1.0f);
        s = make_float4(shear * (diff.x * F.x + diff.y * F.y) + volumetric, shear * (diff.x * F.z + diff.y * F.w),
                        shear * (diff.z * F.x + diff.w * F.y), shear * (diff.z * F.z + diff.w * F.w) + volumetric);
    } else if (m.model == MODEL_WATER || m.model == MODEL_OIL) {
        if (!finite_f(m.density) || m.density <= 0.0f || !finite_f(m.lambda) || m.lambda <= 0.0f ||
            !finite_f(m.param) || m.param < 0.0f) {
            fail_at(c.status, i, bad);
            return false;
        }
        if (m.param > 0.0f) {
            const float pressure = m.lambda * (powf(__fdiv_rn(1.0f, det), m.param) - 1.0f);
            const float stress = -det * pressure;
            s = make_float4(stress, 0.f, 0.f, stress);
        } else {
            const float pressure = m.lambda * fminf(det - 1.0f, 0.0f);
            s = make_float4(pressure, 0.f, 0.f, pressure);
        }
    } else if (m.model == MODEL_POWDER) {
        if (!finite_f(m.lambda) || !finite_f(m.mu) || m.mu <= 0.0f || !finite_f(m.param) || m.param < 0.0f) {
            fail_at(c.status, i, bad);
            return false;
        }
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
        fail_at(c.status, i, bad);
        return false;
    }
    const bool liquid = m.model == MODEL_WATER || m.model == MODEL_OIL;
    mass = liquid ? __fmul_rn(m.density, volume) : P.particle_mass;
    vliq = liquid ? __fmul_rn(volume, det) : 0.0f;
    const float scale = -P.dt * volume * P.gradient_scale;
    const float4 C = c.in.C[i];
    affine = make_float4(mass * C.x + scale * s.x, mass * C.y + scale * s.y, mass * C.z + scale * s.z,
                         mass * C.w + scale * s.w);
    if (!finite4(s) || !finite4(affine)) {
        fail_at(c.status, i, ERROR_P2G | ERROR_P2G_NONFINITE_PARTICLE);
        return false;
    }
    return true;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim multiple of 32).
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t &total)
{
    __shared__ uint32_t warp_totals[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += n;
    }
    if (lane == 31) warp_totals[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? warp_totals[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t n = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += n;
        }
        if (lane < THREADS / 32) warp_totals[lane] = wi - w;
        if (lane == THREADS / 32 - 1) warp_totals[THREADS / 32 - 1] += 0u;
    }
    __syncthreads();
    const uint32_t warp_offset = warp_totals[warp];
    // total = last warp offset + last warp inclusive total
    __shared__ uint32_t s_total;
    if (threadIdx.x == THREADS - 1) s_total = warp_offset + inc;
    __syncthreads();
    total = s_total;
    return warp_offset + inc - v;
}

}  // namespace

// ---------------------------------------------------------------- batch --

// Resets the per-batch counters (reference: cflStepProgress write before the
// batch, solver.ts:1444-1450; the speed scalar is recomputed after it).
__global__ void k_begin_batch(Ctx c, uint32_t reset_progress)
{
    if (threadIdx.x == 0) {
        if (reset_progress) c.counters[COUNTER_PROGRESS] = 0u;
        c.counters[COUNTER_MAX_SPEED] = 0u;
    }
}

// ----------------------------------------------------------- cell sort --

// Base-cell key and rank within the cell for each particle; replaces the
// per-node linked lists of insertParticleBucket (shaders.ts:657-693).
__global__ void k_count(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    Stencil s;
    if (!make_stencil(P, c.in.pos[i], s) || !stencil_fits(P, s.bx, s.by)) {
        fail(c.status, ERROR_STENCIL);
        return;
    }
    const uint32_t key = node_index(P, s.bx, s.by);
    c.keys[i] = key;
    c.ranks[i] = atomicAdd(&c.cell_count[key], 1u);
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

// Stable in-cell order (ascending particle index, i.e. a stable counting sort)
// fused with the stress-cache preparation; writes the P2G record of each
// particle at its sorted slot.
__global__ void k_rank_prepare(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    const uint32_t i = c.tmp[s];
    const uint32_t key = c.keys[i];
    const uint32_t lo = c.cell_start[key], hi = c.cell_start[key + 1];
    uint32_t rank = 0;
    for (uint32_t j = lo; j < hi; ++j) rank += c.tmp[j] < i ? 1u : 0u;
    const uint32_t d = lo + rank;
    c.perm[d] = i;
    float4 A;
    float mass, vliq;
    uint32_t model;
    if (!prepare_particle(c, i, A, mass, vliq, model)) return;
    Stencil st;
    make_stencil(P, c.in.pos[i], st);
    const float2 v = c.in.vel[i];
    const float sv = model == MODEL_WATER ? vliq : (model == MODEL_OIL ? -vliq : 0.0f);
    c.rec0[d] = make_float4(st.fx, st.fy, mass, sv);
    c.rec1[d] = make_float4(mass * v.x, mass * v.y, A.x, A.y);
    c.rec2[d] = make_float2(A.z, A.w);
    if (c.affine_out) c.affine_out[i] = A;
}

// ---------------------------------------------------------- gather P2G --

// One CTA per 16x8 node tile.  Each node sums, in a fixed order (base-cell
// rows, then cells, then ascending particle index), the contributions of the
// particles whose 3x3 stencil covers it: the gather of shaders.ts:1072-1211
// without linked lists and therefore deterministic.
__global__ void __launch_bounds__(TILE_NODES) k_p2g_gather(Ctx c)
{
    const StepParams &P = *c.P;
    const int tx = blockIdx.x, ty = blockIdx.y;
    __shared__ uint32_t s_count;
    if (threadIdx.x < 32) {
        uint32_t cnt = 0;
        const int kx0 = max(tx * TILE_X - 2, 0), kx1 = min(tx * TILE_X + TILE_X - 1, (int)P.cells_x);
        for (int r = threadIdx.x; r < TILE_Y + 2; r += 32) {
            const int ky = ty * TILE_Y - 2 + r;
            if (ky >= 0 && ky <= (int)P.cells_y && kx0 <= kx1) {
                const uint32_t row = (uint32_t)ky * P.node_w;
                cnt += c.cell_start[row + kx1 + 1] - c.cell_start[row + kx0];
            }
        }
        cnt = warp_sum(cnt);
        if (threadIdx.x == 0) s_count = cnt;
    }
    __syncthreads();
    if (s_count == 0u) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    if (threadIdx.x == 0) c.tile_stamp[ty * P.tiles_x + tx] = c.counters[COUNTER_STAMP];
    const int hx = tx * TILE_X + (threadIdx.x % TILE_X), hy = ty * TILE_Y + (threadIdx.x / TILE_X);
    if (hx >= (int)P.node_w || hy >= (int)P.node_h) return;

    float sm = 0.f, spx = 0.f, spy = 0.f;
    float wm = 0.f, wpx = 0.f, wpy = 0.f, wv = 0.f;
    float om = 0.f, opx = 0.f, opy = 0.f, ov = 0.f;
    const float dx = P.dx;
    for (int oy = 0; oy < 3; ++oy) {
        const int ky = hy - oy;
        if (ky < 0 || ky > (int)P.cells_y) continue;
        for (int ox = 0; ox < 3; ++ox) {
            const int kx = hx - ox;
            if (kx < 0 || kx > (int)P.cells_x) continue;
            const uint32_t key = (uint32_t)ky * P.node_w + (uint32_t)kx;
            const uint32_t lo = c.cell_start[key], hi = c.cell_start[key + 1];
            for (uint32_t j = lo; j < hi; ++j) {
                const float4 r0 = c.rec0[j];
                const float4 r1 = c.rec1[j];
                const float2 r2 = c.rec2[j];
                const float w = quad_weight(r0.x, ox) * quad_weight(r0.y, oy);
                const float dpx = ((float)ox - r0.x) * dx, dpy = ((float)oy - r0.y) * dx;
                const float mx = r1.x + r1.z * dpx + r1.w * dpy;
                const float my = r1.y + r2.x * dpx + r2.y * dpy;
                if (!finite_f(w) || w < 0.0f || !finite_f(mx) || !finite_f(my)) {
                    fail_at(c.status, c.perm[j], ERROR_P2G | ERROR_P2G_NONFINITE_PARTICLE);
                    return;
                }
                const float wmass = w * r0.z;
                if (r0.w > 0.0f) {
                    wm += wmass;
                    wpx += w * mx;
                    wpy += w * my;
                    wv += w * r0.w;
                } else if (r0.w < 0.0f) {
                    om += wmass;
                    opx += w * mx;
                    opy += w * my;
                    ov += w * -r0.w;
                } else {
                    sm += wmass;
                    spx += w * mx;
                    spy += w * my;
                }
            }
        }
    }
    if (!finite_f(sm) || !finite_f(spx) || !finite_f(spy) || !finite_f(wm) || !finite_f(wpx) || !finite_f(wpy) ||
        !finite_f(wv) || !finite_f(om) || !finite_f(opx) || !finite_f(opy) || !finite_f(ov)) {
        fail(c.status, ERROR_P2G | ERROR_P2G_NONFINITE_ACCUMULATION);
        return;
    }
    const uint32_t n = (uint32_t)hy * P.node_w + (uint32_t)hx;
    c.p2g_solid[n] = make_float4(sm, spx, spy, 0.f);
    c.p2g_water[n] = make_float4(wm, wpx, wpy, wv);
    c.p2g_oil[n] = make_float4(om, opx, opy, ov);
}

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
                fail_at(c.status, i, ERROR_P2G | ERROR_P2G_NONFINITE_PARTICLE);
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

// ---------------------------------------------------------- grid update --

namespace {

__device__ __forceinline__ float2 finish_velocity(const StepParams &P, float mass, float px, float py, int x, int y)
{
    // finishGridVelocity: shaders.ts:1748-1777
    if (mass <= 0.0f) return make_float2(0.f, 0.f);
    float2 vel = make_float2(px / mass + P.dt * P.gx, py / mass + P.dt * P.gy);
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

// updateGrid: shaders.ts:1485-1746 (mass normalise, gravity, drag, water/oil
// normal contact from phase-volume gradients, walls).  Writes the per-channel
// velocities G2P reads, with the liquid mass/area sums packed beside the
// water and oil velocities.
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
    const int x = hx - 1, y = hy - 1;
    const float4 S = c.p2g_solid[n], W = c.p2g_water[n], O = c.p2g_oil[n];
    if (!finite_f(S.x) || S.x < 0.f || !finite_f(S.y) || !finite_f(S.z) || !finite_f(W.x) || W.x < 0.f ||
        !finite_f(W.y) || !finite_f(W.z) || !finite_f(W.w) || W.w < 0.f || !finite_f(O.x) || O.x < 0.f ||
        !finite_f(O.y) || !finite_f(O.z) || !finite_f(O.w) || O.w < 0.f) {
        fail(c.status, ERROR_GRID);
        return;
    }
    float2 vs = finish_velocity(P, S.x, S.y, S.z, x, y);
    float2 vw = finish_velocity(P, W.x, W.y, W.z, x, y);
    float2 vo = finish_velocity(P, O.x, O.y, O.z, x, y);
    if (x >= 0 && y >= 0 && x <= (int)P.cells_x && y <= (int)P.cells_y && W.x > 0.f && O.x > 0.f && W.w > 0.f &&
        O.w > 0.f) {
        const float2 xp = phase_volume(c, hx + 1, hy, stamp), xm = phase_volume(c, hx - 1, hy, stamp);
        const float2 yp = phase_volume(c, hx, hy + 1, stamp), ym = phase_volume(c, hx, hy - 1, stamp);
        const float2 wgrad = make_float2(xp.x - xm.x, yp.x - ym.x);
        const float2 ograd = make_float2(xp.y - xm.y, yp.y - ym.y);
        const float2 sep = make_float2(ograd.x - wgrad.x, ograd.y - wgrad.y);
        const float sl = sqrtf(sep.x * sep.x + sep.y * sep.y);
        if (finite_f(sl) && sl > 1e-8f) {
            float2 nrm = make_float2(sep.x / sl, sep.y / sl);
            const float wd = W.x / W.w, od = O.x / O.w;
            const float ds = fmaxf(wd, od);
            const float contrast = (od - wd) / ds;
            const float gm = sqrtf(P.gx * P.gx + P.gy * P.gy);
            float align = 0.f;
            if (!finite_f(wd) || wd <= 0.f || !finite_f(od) || od <= 0.f || !finite_f(contrast) || !finite_f(gm)) {
                fail(c.status, ERROR_GRID);
                return;
            }
            if (gm > 0.f) align = (nrm.x * P.gx + nrm.y * P.gy) / gm;
            if (!finite_f(align)) {
                fail(c.status, ERROR_GRID);
                return;
            }
            if (contrast * align < -LIQUID_STABLE_ORDER_EPSILON) nrm = make_float2(-nrm.x, -nrm.y);
            const float rel = (vo.x - vw.x) * nrm.x + (vo.y - vw.y) * nrm.y;
            const float overlap = fminf(fmaxf(2.0f * fminf(W.w, O.w) / (W.w + O.w), 0.f), 1.f);
            const float minsep = fmaxf(LIQUID_CONTACT_SEPARATION_FRACTION * overlap * P.dx / LIQUID_CONTACT_RELAXATION_SECONDS,
                                       fmaxf(-rel, 0.f) * LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER);
            if (rel < minsep) {
                const float mag = (minsep - rel) / (1.0f / W.x + 1.0f / O.x);
                const float ix = mag * nrm.x, iy = mag * nrm.y;
                vw = make_float2(vw.x - ix / W.x, vw.y - iy / W.x);
                vo = make_float2(vo.x + ix / O.x, vo.y + iy / O.x);
            }
        }
    }
    if (!finite2(vs) || !finite2(vw) || !finite2(vo)) {
        fail(c.status, ERROR_GRID | ERROR_TRIANGLE_CONTACT);
        return;
    }
    const int cx = (int)P.cells_x, cy = (int)P.cells_y;
    const float fr = P.wall_friction;
    vs.x = wall_cushion(vs.x, x, cx);
    vs.y = wall_cushion(vs.y, y, cy);
    vw.x = wall_cushion(vw.x, x, cx);
    vw.y = wall_cushion(vw.y, y, cy);
    vo.x = wall_cushion(vo.x, x, cx);
    vo.y = wall_cushion(vo.y, y, cy);
    vs.x = wall_friction(vs.x, y, cy, fr);
    vs.y = wall_friction(vs.y, x, cx, fr);
    vw.x = wall_friction(vw.x, y, cy, fr);
    vw.y = wall_friction(vw.y, x, cx, fr);
    vo.x = wall_friction(vo.x, y, cy, fr);
    vo.y = wall_friction(vo.y, x, cx, fr);
    const float lm = W.x + O.x, lv = W.w + O.w;
    c.g_solid[n] = vs;
    c.g_water[n] = make_float4(vw.x, vw.y, lm, lv);
    c.g_oil[n] = make_float4(vo.x, vo.y, lm, lv);
}

// ------------------------------------------------------------------ G2P --

namespace {

// particleWaveSpeedBound: shaders.ts:268-353
__device__ float wave_speed_bound(const Ctx &c, const Material &m, float4 F, float damage, float volume)
{
    if (m.model == MODEL_WATER || m.model == MODEL_OIL) {
        if (!finite_f(m.lambda) || !finite_f(m.density) || m.lambda <= 0.f || m.density <= 0.f) return FLOAT_MAX;
        float c2 = m.lambda / m.density;
        if (m.param > 0.0f) {
            const float det = det2(F);
            if (!finite_f(m.param) || m.param <= 0.f || !finite_f(det) || det <= 0.f) return FLOAT_MAX;
            c2 = m.param * c2 * powf(1.0f / det, m.param - 1.0f);
        }
        if (!finite_f(c2) || c2 < 0.f) return FLOAT_MAX;
        return sqrtf(c2);
    }
    if (m.model != MODEL_NEO_HOOKEAN) return FLOAT_MAX;
    if (!finite_f(damage)) return FLOAT_MAX;
    const float remaining = 1.0f - fminf(fmaxf(damage, 0.f), 1.f);
    if (remaining <= 0.f) return 0.f;
    const float lambda = m.lambda * remaining, mu = m.mu * remaining;
    const float det = det2(F);
    const float tr = F.x * F.x + F.y * F.y + F.z * F.z + F.w * F.w;
    if (!finite_f(det) || det <= 0.f || !finite_f(tr) || !finite_f(lambda) || !finite_f(mu) || mu < 0.f)
        return FLOAT_MAX;
    const float disc = sqrtf(fmaxf(0.f, tr * tr - 4.0f * det * det));
    const float maxs2 = 0.5f * (tr + disc);
    const float vt = fabsf(lambda + mu - lambda * logf(det));
    const float rho = c.P->particle_mass / volume;
    const float c2 = (mu * maxs2 + vt) / rho;
    if (!finite_f(rho) || rho <= 0.f || !finite_f(c2) || c2 < 0.f) return FLOAT_MAX;
    return sqrtf(c2);
}

__device__ __forceinline__ void copy_particle(const Ctx &c, uint32_t i)
{
    c.out.pos[i] = c.in.pos[i];
    c.out.vel[i] = c.in.vel[i];
    c.out.C[i] = c.in.C[i];
    c.out.F[i] = c.in.F[i];
    c.out.pvol[i] = c.in.pvol[i];
    c.out.damage[i] = c.in.damage[i];
}

// validateCflParticle: shaders.ts:2423-2454
__device__ void validate_cfl(const Ctx &c, uint32_t i, const Material &m, float2 vel, float4 F, float damage,
                             float volume)
{
    const StepParams &P = *c.P;
    if (!P.cfl_enabled) return;
    if (*(volatile uint32_t *)c.status != 0u) return;
    const float speed = length2(vel);
    const float wave = wave_speed_bound(c, m, F, damage, volume);
    if (!finite2(vel) || !finite_f(speed) || !finite_f(wave) || speed > P.cfl_velocity_limit ||
        wave > P.cfl_wave_bound) {
        const uint32_t prev = atomicOr(c.status + 6, 3u);
        if (prev == 0u) {
            atomicExch(c.status + 1, i);
            atomicExch(c.status + 2, __float_as_uint(speed));
            atomicExch(c.status + 3, __float_as_uint(wave));
            atomicExch(c.status + 4, __float_as_uint(P.cfl_velocity_limit));
            atomicExch(c.status + 5, __float_as_uint(P.cfl_wave_bound));
        }
        fail(c.status, ERROR_CFL_BOUND);
    }
}

}  // namespace

// g2p: shaders.ts:2114-2421 (APIC velocity and affine C, liquid
// density-contrast acceleration, adaptive fused F update with retries,
// per-model projection, wall confinement, fused CFL validation).
__global__ void k_g2p(Ctx c)
{
    const StepParams &P = *c.P;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_particles) return;
    if (*(volatile uint32_t *)c.status != 0u) {
        copy_particle(c, i);
        return;
    }
    const float2 pos = c.in.pos[i];
    Stencil s;
    if (!make_stencil(P, pos, s) || !stencil_fits(P, s.bx, s.by)) {
        fail(c.status, ERROR_STENCIL);
        return;
    }
    const Material m = c.mats[c.mat[i]];
    const bool water = m.model == MODEL_WATER, oil = m.model == MODEL_OIL, liquid = water || oil;
    float2 vel = make_float2(0.f, 0.f);
    float4 aff = make_float4(0.f, 0.f, 0.f, 0.f);
    float pmass = 0.f, pvolume = 0.f;
    for (int oy = 0; oy < 3; ++oy) {
        const float wy = quad_weight(s.fy, oy);
        const float dpy = ((float)oy - s.fy) * P.dx;
        for (int ox = 0; ox < 3; ++ox) {
            const uint32_t n = node_index(P, s.bx + ox, s.by + oy);
            const float w = quad_weight(s.fx, ox) * wy;
            const float dpx = ((float)ox - s.fx) * P.dx;
            float2 gv;
            float nm = 0.f, nv = 0.f;
            if (liquid) {
                const float4 g = water ? c.g_water[n] : c.g_oil[n];
                gv = make_float2(g.x, g.y);
                nm = g.z;
                nv = g.w;
            } else {
                gv = c.g_solid[n];
            }
            if (!finite_f(w) || w < 0.f || !finite_f(dpx) || !finite_f(dpy) || !finite2(gv)) {
                fail(c.status, ERROR_G2P);
                return;
            }
            vel.x += w * gv.x;
            vel.y += w * gv.y;
            if (liquid) {
                if (!finite_f(nm) || nm < 0.f || !finite_f(nv) || nv < 0.f) {
                    fail_at(c.status, i, ERROR_G2P);
                    return;
                }
                pmass += w * nm;
                pvolume += w * nv;
            }
            aff.x += w * gv.x * dpx;
            aff.y += w * gv.x * dpy;
            aff.z += w * gv.y * dpx;
            aff.w += w * gv.y * dpy;
        }
    }
    const float4 F0 = c.in.F[i];
    if (liquid) {
        const float pdet = det2(F0);
        if (!finite_f(pmass) || pmass <= 0.f || !finite_f(pvolume) || pvolume <= 0.f || !finite_f(pdet) ||
            pdet <= 0.f) {
            fail_at(c.status, i, ERROR_G2P);
            return;
        }
        const float pd = m.density / pdet;
        const float ld = pmass / pvolume;
        const float rd = (pd - ld) / pd;
        vel.x += P.dt * (rd * P.gx);
        vel.y += P.dt * (rd * P.gy);
        if (!finite_f(pd) || pd <= 0.f || !finite_f(ld) || ld <= 0.f || !finite_f(rd) || !finite2(vel)) {
            fail_at(c.status, i, ERROR_G2P);
            return;
        }
    }
    const float gs = P.gradient_scale, dt = P.dt;
    const float4 Cn = make_float4(aff.x * gs, aff.y * gs, aff.z * gs, aff.w * gs);
    const float2 npos = make_float2(pos.x + dt * vel.x, pos.y + dt * vel.y);
    if (!finite2(vel) || !finite4(Cn) || !finite2(npos)) {
        fail(c.status, ERROR_G2P);
        return;
    }
    const float row = fmaxf(fabsf(Cn.x) + fabsf(Cn.y), fabsf(Cn.z) + fabsf(Cn.w));
    const float inc = dt * row;
    const float req = ceilf(inc / MAX_DEFORMATION_INCREMENT);
    if (!finite_f(req) || req > MAX_DEFORMATION_SUBSTEPS) {
        fail_at(c.status, i, ERROR_DEFORMATION_SUBSTEP_LIMIT);
        return;
    }
    uint32_t sub = max(1u, (uint32_t)req);
    float4 trial = integrate_deformation(F0, Cn, dt, sub);
    if (!finite4(trial)) {
        fail(c.status, ERROR_G2P);
        return;
    }
    float tdet = det2(trial);
    while (finite_f(tdet) && tdet <= 0.f && sub < 64u) {
        sub = min(sub * 2u, 64u);
        trial = integrate_deformation(F0, Cn, dt, sub);
        if (!finite4(trial)) {
            fail(c.status, ERROR_G2P);
            return;
        }
        tdet = det2(trial);
    }
    float4 Fn = trial;
    float pv = c.in.pvol[i];
    if (!finite_f(tdet) || tdet <= 0.f) {
        // recordDeformationFailure: shaders.ts:224-237
        const uint32_t prev = atomicOr(c.status + 6, 1u);
        if (prev == 0u) {
            atomicExch(c.status + 1, i);
            atomicExch(c.status + 2, __float_as_uint(tdet));
            atomicExch(c.status + 3, __float_as_uint(inc));
            atomicExch(c.status + 4, __float_as_uint(det2(F0)));
        }
        fail(c.status, ERROR_DEFORMATION);
        return;
    }
    if (m.model == MODEL_SNOW) {
        const Decomp d = decompose(trial);
        if (!finite_f(d.s0) || !finite_f(d.s1) || d.s0 <= 0.f || d.s1 <= 0.f) {
            fail(c.status, ERROR_G2P);
            return;
        }
        const float lo = 1.0f - SNOW_COMPRESSION_YIELD, hi = 1.0f + SNOW_STRETCH_YIELD;
        const float a = fminf(fmaxf(d.s0, lo), hi), b = fminf(fmaxf(d.s1, lo), hi);
        pv = fminf(fmaxf(pv * tdet / (a * b), SNOW_MIN_PLASTIC_VOLUME), SNOW_MAX_PLASTIC_VOLUME);
        Fn = reconstruct(d, a, b);
    } else if (m.model == MODEL_POWDER) {
        if (!finite_f(m.lambda) || !finite_f(m.mu) || m.mu <= 0.f || !finite_f(m.param) || m.param < 0.f) {
            fail(c.status, ERROR_G2P);
            return;
        }
        // projectGranularDeformation: shaders.ts:443-472
        const Decomp d = decompose(trial);
        const float l0 = logf(d.s0), l1 = logf(d.s1);
        const float lv = l0 + l1;
        const float minlv = logf(MIN_POWDER_DETERMINANT);
        const float blv = fmaxf(minlv, lv);
        const float pressure = fmaxf(0.f, -(m.lambda + m.mu) * blv);
        const float dev = 0.5f * (l0 - l1);
        const float maxdev = m.param * pressure / (2.0f * m.mu);
        if (!(dev <= maxdev && lv >= minlv)) {
            const float pdev = fminf(dev, maxdev);
            const float mean = 0.5f * blv;
            Fn = reconstruct(d, expf(mean + pdev), expf(mean - pdev));
        }
    } else if (liquid) {
        // projectLiquidDeformation: shaders.ts:474-488
        const float2 rn = make_float2(trial.x + trial.w, trial.z - trial.y);
        const float rs = fmaxf(fabsf(rn.x), fabsf(rn.y));
        const float2 nr = make_float2(rn.x / rs, rn.y / rs);
        const float rl = sqrtf(nr.x * nr.x + nr.y * nr.y);
        const float2 rot = make_float2(nr.x / rl, nr.y / rl);
        const float vol = det2(trial);
        const float bv = fminf(fmaxf(vol, MIN_LIQUID_DETERMINANT), MAX_LIQUID_DETERMINANT);
        const float sc = sqrtf(bv);
        Fn = make_float4(sc * rot.x, sc * -rot.y, sc * rot.y, sc * rot.x);
    } else if (m.model == MODEL_NEO_HOOKEAN) {
        const float tr = trial.x * trial.x + trial.y * trial.y + trial.z * trial.z + trial.w * trial.w;
        if (!finite_f(tr)) {
            fail(c.status, ERROR_G2P);
            return;
        }
        if (tdet < MIN_NEO_HOOKEAN_STRETCH * sqrtf(tr) || tr > MAX_NEO_HOOKEAN_STRETCH * MAX_NEO_HOOKEAN_STRETCH) {
            const Decomp d = decompose(trial);
            Fn = reconstruct(d, fminf(fmaxf(d.s0, MIN_NEO_HOOKEAN_STRETCH), MAX_NEO_HOOKEAN_STRETCH),
                             fminf(fmaxf(d.s1, MIN_NEO_HOOKEAN_STRETCH), MAX_NEO_HOOKEAN_STRETCH));
        }
    } else if (m.model != MODEL_FIXED_COROTATED) {
        fail(c.status, ERROR_G2P);
        return;
    }
    const float udet = det2(Fn);
    if (!finite4(Fn) || !finite_f(pv) || pv < SNOW_MIN_PLASTIC_VOLUME || pv > SNOW_MAX_PLASTIC_VOLUME) {
        fail(c.status, ERROR_G2P);
        return;
    }
    if (!finite_f(udet) || udet <= 0.f) {
        // recordProjectedDeformationFailure: shaders.ts:239-248
        const uint32_t prev = atomicOr(c.status + 6, 2u);
        if (prev == 0u) {
            atomicExch(c.status + 1, i);
            atomicExch(c.status + 2, __float_as_uint(Fn.x));
            atomicExch(c.status + 3, __float_as_uint(Fn.y));
            atomicExch(c.status + 4, __float_as_uint(Fn.z));
            atomicExch(c.status + 5, __float_as_uint(Fn.w));
        }
        fail(c.status, ERROR_PROJECTED_DEFORMATION);
        return;
    }
    const float2 bx = confine_axis(npos.x, vel.x, P.domain_w);
    const float2 by = confine_axis(npos.y, vel.y, P.domain_h);
    const float2 fx = confine_axis(bx.x, bx.y, P.domain_w);
    const float2 fy = confine_axis(by.x, by.y, P.domain_h);
    const float2 outv = make_float2(fx.y, fy.y);
    const float damage = c.in.damage[i];
    c.out.pos[i] = make_float2(fx.x, fy.x);
    c.out.vel[i] = outv;
    c.out.C[i] = Cn;
    c.out.F[i] = Fn;
    c.out.pvol[i] = pv;
    c.out.damage[i] = damage;
    if (P.n_bodies == 0u) validate_cfl(c, i, m, outv, Fn, damage, c.vol[i]);
}

// commitParticles: shaders.ts:3067-3080.  On a failed substep every particle
// is restored from the substep's input (whole-substep rollback); otherwise the
// committed CFL microstep counter advances.  The substep stamp advances
// unconditionally.
__global__ void k_commit(Ctx c)
{
    const StepParams &P = *c.P;
    if (*(volatile uint32_t *)c.status != 0u) {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_particles; i += gridDim.x * blockDim.x)
            copy_particle(c, i);
    } else if (blockIdx.x == 0 && threadIdx.x == 0 && P.cfl_enabled) {
        c.counters[COUNTER_PROGRESS] += 1u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) c.counters[COUNTER_STAMP] += 1u;
}

// measureParticleSpeedPartials + reduceParticleSpeedPartials
// (shaders.ts:2463-2533) as one warp-shuffle reduction with an atomic max on
// the order-preserving bits of the non-negative speed.
__global__ void k_speed_max(Ctx c)
{
    const StepParams &P = *c.P;
    float best = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_particles; i += gridDim.x * blockDim.x) {
        const float sp = length2(c.in.vel[i]);
        best = fmaxf(best, finite_f(sp) ? sp : FLOAT_MAX);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(c.counters + COUNTER_MAX_SPEED, __float_as_uint(best));
}

// Counts the nodes of the last substep whose solid / water / oil mass is
// positive (the N_act of the algorithmic-byte model), over stamped tiles.
__global__ void __launch_bounds__(TILE_NODES) k_count_active_nodes(Ctx c, uint32_t *counts)
{
    const StepParams &P = *c.P;
    const int tx = blockIdx.x, ty = blockIdx.y;
    // the commit of the last substep advanced the stamp by one
    if (c.tile_stamp[ty * P.tiles_x + tx] + 1u != c.counters[COUNTER_STAMP]) return;
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

}  // namespace mpm
