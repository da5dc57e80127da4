// mpm_device.cuh -- device-side types and FP32 helpers of the B200 MLS-MPM
// substep.  The helpers follow the WGSL arithmetic of the reference GPU
// pipeline (src/lib/mpm/kernels/shaders.ts) where that arithmetic is part of
// its contract: the compensated determinant (:261-266), the fused 2x2
// deformation products (:1459-1483), ties-to-even fixed-point rounding
// (:971-985).  Everything else may be contracted freely by the compiler.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

// Status flag bits: src/lib/mpm/kernels/shaders.ts:157-172.
constexpr uint32_t ERROR_STENCIL = 1u;
constexpr uint32_t ERROR_DEFORMATION = 2u;
constexpr uint32_t ERROR_P2G = 4u;
constexpr uint32_t ERROR_GRID = 8u;
constexpr uint32_t ERROR_G2P = 16u;
constexpr uint32_t ERROR_DEFORMATION_SUBSTEP_LIMIT = 32u;
constexpr uint32_t ERROR_PROJECTED_DEFORMATION = 64u;
constexpr uint32_t ERROR_P2G_INVALID_MATERIAL = 128u;
constexpr uint32_t ERROR_P2G_NONFINITE_PARTICLE = 256u;
constexpr uint32_t ERROR_P2G_NONFINITE_ACCUMULATION = 1024u;
constexpr uint32_t ERROR_P2G_NONFINITE_NODE = 2048u;
constexpr uint32_t ERROR_TRIANGLE_CONTACT = 4096u;
constexpr uint32_t ERROR_TRIANGLE_BOND = 8192u;
constexpr uint32_t ERROR_CFL_BOUND = 16384u;
constexpr uint32_t ERROR_FRACTURE_BOND = 32768u;
constexpr uint32_t ERROR_FIXED_POINT_RANGE = 65536u;
// no counterpart in the reference: a grid barrier wait of the fused substep
// kernel ran out (every scene of the launch gets it; the state is undefined)
constexpr uint32_t ERROR_BARRIER = 1u << 20;

// Constitutive model codes: src/lib/mpm/materials.ts:8-16, plus 5 =
// fixed-corotated (no reference counterpart).
constexpr uint32_t MODEL_NEO_HOOKEAN = 0u;
constexpr uint32_t MODEL_SNOW = 1u;
constexpr uint32_t MODEL_WATER = 2u;
constexpr uint32_t MODEL_OIL = 3u;
constexpr uint32_t MODEL_POWDER = 4u;
constexpr uint32_t MODEL_FIXED_COROTATED = 5u;

// Material constants: src/lib/mpm/kernels/shaders.ts:196-210, materials.ts:40-53.
constexpr float SNOW_COMPRESSION_YIELD = 0.025f;
constexpr float SNOW_STRETCH_YIELD = 0.0075f;
constexpr float SNOW_HARDENING = 10.0f;
constexpr float SNOW_MIN_PLASTIC_VOLUME = 0.6f;
constexpr float SNOW_MAX_PLASTIC_VOLUME = 20.0f;
constexpr float SNOW_MAX_HARDENING_EXPONENT = 20.0f;
constexpr float MIN_LIQUID_DETERMINANT = 0.5f;
constexpr float MAX_LIQUID_DETERMINANT = 2.0f;
constexpr float MIN_POWDER_DETERMINANT = 0.5f;
constexpr float MIN_NEO_HOOKEAN_STRETCH = 0.05f;
constexpr float MAX_NEO_HOOKEAN_STRETCH = 20.0f;
constexpr float MAX_DEFORMATION_INCREMENT = 0.25f;
constexpr float MAX_DEFORMATION_SUBSTEPS = 64.0f;
constexpr float WALL_CUSHION_CELLS = 8.0f;
constexpr float LIQUID_CONTACT_SEPARATION_FRACTION = 0.25f;
constexpr float LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER = 1.0f;
constexpr float LIQUID_CONTACT_RELAXATION_SECONDS = 0.05f;
constexpr float LIQUID_STABLE_ORDER_EPSILON = 1e-3f;
constexpr float TRIANGLE_FLUID_TANGENTIAL_DRAG_RATE = 4.0f;
constexpr float TRIANGLE_CONTACT_SKIN_CELLS = 0.1f;
constexpr float TRIANGLE_CONTACT_IMPULSE_RELAXATION = 0.25f;
constexpr float FLOAT_MAX = 3.402823466e38f;

// Node tile handled by one CTA in the grid kernels (16 x 8 = 128 nodes).
constexpr int TILE_X = 16;
constexpr int TILE_Y = 8;
constexpr int TILE_NODES = TILE_X * TILE_Y;

// Fixed-point accumulator words per node (solid m,px,py | water m,px,py,V |
// oil m,px,py,V): src/lib/mpm/kernels/shaders.ts:174, :1029-1040.
constexpr int FIXED_WORDS = 11;

struct Material {
    uint32_t model;
    float lambda;
    float mu;
    float density;
    float param;  // Tait exponent (liquids, 0 = linear EOS) or powder friction
    float c2;     // liquids: lambda / density (the rest wave speed squared), rounded once
    float pad1, pad2;
};

// Per-batch parameters, written by the host before each batch launch.  The
// field set is the 144-byte SimulationParams of the reference
// (src/lib/mpm/kernels/layout.ts:950-996) re-grouped, plus B200 extras.
struct alignas(16) StepParams {
    uint32_t cells_x, cells_y, node_w, node_h;
    uint32_t n_particles, n_nodes, tiles_x, tiles_y;
    uint32_t n_bodies, cfl_enabled, n_bonds, fracture_particles;
    uint32_t pair_cache_enabled, fixed_shift, fracture_incidence, batch_steps;  // substeps of this batch
    float dx, particle_mass, particle_volume, dt;
    float lambda, mu, stress_scale, gradient_scale;
    float gx, gy, domain_w, domain_h;
    float bond_rest_length, bond_stiffness, band, contact_reach;
    float cfl_wave_bound, cfl_velocity_limit, bond_reference_dt, wall_friction;
    float fixed_scale, drag_x, drag_y, drag_radius;
    // cfl_speed2_bound / cfl_wave2_bound: the largest float whose correctly
    // rounded square root is at most cfl_velocity_limit / cfl_wave_bound, so
    // a speed or wave speed exceeds its bound exactly when its square exceeds
    // this (NaN for a NaN bound, -1 for a negative one)
    float drag_stiffness, drag_damping, inv_dx, cfl_speed2_bound;
    // the scene's place in a batch of scenes: its first slot and first tile
    // (its tiles are followed by one sentinel entry) and its tile count
    uint32_t p_base, tile_base, scene_tiles;
    float cfl_wave2_bound;
};

// Device counters (one 32-word line): stamp of the current substep, committed
// CFL microsteps, bits of the maximum particle speed.
constexpr int COUNTER_STAMP = 0;
constexpr int COUNTER_PROGRESS = 1;
constexpr int COUNTER_MAX_SPEED = 2;

// |v| < infinity: false for both infinities and every NaN (one compare with
// an absolute-value operand, where a test of the exponent bits takes two
// instructions)
__device__ __forceinline__ bool finite_f(float v) { return fabsf(v) < __int_as_float(0x7f800000); }
__device__ __forceinline__ bool finite2(float2 v) { return finite_f(v.x) && finite_f(v.y); }
__device__ __forceinline__ bool finite4(float4 v)
{
    return finite_f(v.x) && finite_f(v.y) && finite_f(v.z) && finite_f(v.w);
}

// determinant2x2 with the product residual: shaders.ts:261-266.
__device__ __forceinline__ float det2(float4 m)
{
    float second = __fmul_rn(m.y, m.z);
    float err = __fmaf_rn(m.y, m.z, -second);
    return __fsub_rn(__fmaf_rn(m.x, m.w, -second), err);
}

// quadraticWeights: shaders.ts:500-509, evaluated without contraction so the
// fixed-point contributions are reproducible by the CPU emulation.
__device__ __forceinline__ float quad_weight(float f, int o)
{
    if (o == 0) {
        float l = __fsub_rn(1.5f, f);
        return __fmul_rn(__fmul_rn(0.5f, l), l);
    }
    if (o == 1) {
        float c = __fsub_rn(f, 1.0f);
        return __fsub_rn(0.75f, __fmul_rn(c, c));
    }
    float r = __fsub_rn(f, 0.5f);
    return __fmul_rn(__fmul_rn(0.5f, r), r);
}

struct Decomp {
    float s0, s1;
    float2 u0, u1, v0, v1;
};

// decompose2x2: shaders.ts:355-377.
__device__ __forceinline__ Decomp decompose(float4 m)
{
    float c00 = m.x * m.x + m.z * m.z;
    float c01 = m.x * m.y + m.z * m.w;
    float c11 = m.y * m.y + m.w * m.w;
    float radius = sqrtf((c00 - c11) * (c00 - c11) + 4.0f * c01 * c01);
    Decomp d;
    d.s0 = sqrtf(fmaxf(0.0f, 0.5f * (c00 + c11 + radius)));
    float det = det2(m);
    float guard = fmaxf(d.s0, 1.0e-30f);
    d.s1 = det / guard;
    float angle = 0.5f * atan2f(2.0f * c01, c00 - c11);
    float c = cosf(angle), s = sinf(angle);
    d.v0 = make_float2(c, s);
    d.v1 = make_float2(-s, c);
    d.u0 = make_float2((m.x * d.v0.x + m.y * d.v0.y) / guard, (m.z * d.v0.x + m.w * d.v0.y) / guard);
    d.u1 = make_float2(-d.u0.y, d.u0.x);
    return d;
}

__device__ __forceinline__ float4 polar_rotation(const Decomp &d)
{
    return make_float4(d.u0.x * d.v0.x + d.u1.x * d.v1.x, d.u0.x * d.v0.y + d.u1.x * d.v1.y,
                       d.u0.y * d.v0.x + d.u1.y * d.v1.x, d.u0.y * d.v0.y + d.u1.y * d.v1.y);
}

__device__ __forceinline__ float4 reconstruct(const Decomp &d, float a, float b)
{
    return make_float4(a * d.u0.x * d.v0.x + b * d.u1.x * d.v1.x, a * d.u0.x * d.v0.y + b * d.u1.x * d.v1.y,
                       a * d.u0.y * d.v0.x + b * d.u1.y * d.v1.x, a * d.u0.y * d.v0.y + b * d.u1.y * d.v1.y);
}

// integrateDeformation: shaders.ts:1459-1483.  The update matrix terms are
// rounded separately and every row-column product keeps one fused term.
__device__ __forceinline__ float4 integrate_deformation(float4 f, float4 c, float dt, uint32_t substeps)
{
    float h = substeps == 1u ? dt : __fdiv_rn(dt, (float)substeps);
    float4 u = make_float4(__fadd_rn(1.0f, __fmul_rn(h, c.x)), __fmul_rn(h, c.y), __fmul_rn(h, c.z),
                           __fadd_rn(1.0f, __fmul_rn(h, c.w)));
    float4 r = f;
    for (uint32_t s = 0; s < substeps; ++s) {
        r = make_float4(__fmaf_rn(u.x, r.x, __fmul_rn(u.y, r.z)), __fmaf_rn(u.x, r.y, __fmul_rn(u.y, r.w)),
                        __fmaf_rn(u.z, r.x, __fmul_rn(u.w, r.z)), __fmaf_rn(u.z, r.y, __fmul_rn(u.w, r.w)));
    }
    return r;
}

// The trial deformation of G2P (shaders.ts:2249-2298): the increment
// dt * max row sum |C|, n = max(1, ceil(increment / 0.25)) fused products of
// integrateDeformation, n doubled (at most 64) while det F <= 0.
struct DeformationTrial {
    float4 F;
    float increment, det;
    uint32_t substeps;
};

// Returns 0, ERROR_DEFORMATION_SUBSTEP_LIMIT when n would exceed 64, or
// ERROR_G2P when a product is not finite.  A finite det <= 0 after the
// retries is left to the caller (recordDeformationFailure).
__device__ __forceinline__ uint32_t deformation_trial(float4 F0, float4 Cn, float dt, DeformationTrial &t)
{
    const float row = fmaxf(fabsf(Cn.x) + fabsf(Cn.y), fabsf(Cn.z) + fabsf(Cn.w));
    t.increment = dt * row;
    const float req = ceilf(t.increment * (1.0f / MAX_DEFORMATION_INCREMENT));  // exact: the increment is 2^-2
    if (!finite_f(req) || req > MAX_DEFORMATION_SUBSTEPS) return ERROR_DEFORMATION_SUBSTEP_LIMIT;
    uint32_t sub = max(1u, (uint32_t)req);
    float4 trial = integrate_deformation(F0, Cn, dt, sub);
    if (!finite4(trial)) return ERROR_G2P;
    float tdet = det2(trial);
    while (finite_f(tdet) && tdet <= 0.f && sub < 64u) {
        sub = min(sub * 2u, 64u);
        trial = integrate_deformation(F0, Cn, dt, sub);
        if (!finite4(trial)) return ERROR_G2P;
        tdet = det2(trial);
    }
    t.F = trial;
    t.det = tdet;
    t.substeps = sub;
    return 0u;
}

// confineAxis: shaders.ts:522-534 -> (position, velocity)
__device__ __forceinline__ float2 confine_axis(float next, float vel, float maximum)
{
    if (next < 0.0f || (next == 0.0f && vel < 0.0f)) return make_float2(0.0f, 0.0f);
    if (next > maximum || (next == maximum && vel > 0.0f)) return make_float2(maximum, 0.0f);
    return make_float2(next, vel);
}

// applyWallCushion / applyWallTangentialFriction: shaders.ts:1438-1457
// (dist / cushion clamped to [0, 1] is exactly 1 once dist >= cushion, so
// nodes away from the walls skip the division.)
__device__ __forceinline__ float wall_cushion(float vel, int coord, int extent)
{
    float cushion = fminf(WALL_CUSHION_CELLS, (float)extent / 4.0f);
    float dist = vel < 0.0f ? (float)coord : (float)(extent - coord);
    if (dist >= cushion) return vel;
    return vel * fminf(fmaxf(dist / cushion, 0.0f), 1.0f);
}

// Whether every coordinate in [lo, hi] lies at least the cushion from both
// walls of an axis of `extent` cells: wall_cushion and wall_friction then
// return the velocity they are given, for either sign.
__device__ __forceinline__ bool beyond_wall_cushion(int lo, int hi, int extent)
{
    const float cushion = fminf(WALL_CUSHION_CELLS, (float)extent / 4.0f);
    return (float)lo >= cushion && (float)(extent - hi) >= cushion;
}

__device__ __forceinline__ float wall_friction(float vel, int coord, int extent, float friction)
{
    if (friction <= 0.0f) return vel;
    float dist = fmaxf(0.0f, fminf((float)coord, (float)(extent - coord)));
    float cushion = fminf(WALL_CUSHION_CELLS, (float)extent / 4.0f);
    if (dist >= cushion) return vel;
    float influence = 1.0f - fminf(fmaxf(dist / cushion, 0.0f), 1.0f);
    return vel * (1.0f - friction * influence);
}

// pow as WGSL specifies it: its accuracy is inherited from
// exp2(y * log2(x)), so the reference's Tait terms are that expression.
__device__ __forceinline__ float pow_wgsl(float x, float y) { return exp2f(y * log2f(x)); }

__device__ __forceinline__ float length2(float2 v)
{
    return __fsqrt_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)));
}

}  // namespace mpm
