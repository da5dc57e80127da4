/*
 * fixed_point_emu.c -- CPU emulation of the fixed-point atomic P2G integers.
 *
 * TEST INFRASTRUCTURE ONLY (the bit-exact checker of k_prepare_scatter).
 *
 * Restates prepareAndScatterParticles + addFixedPoint of the reference's WGSL
 * (src/lib/mpm/kernels/shaders.ts:971-1043, 7korobi/powder-play) in IEEE
 * float32 with the same operation order as the CUDA kernel: every product,
 * quotient and sum separately rounded (built with -ffp-contract=off), the
 * compensated determinant with fmaf (shaders.ts:261-266), ties-to-even
 * rounding of value * 2^shift, and wrap-around int32 accumulation (integer
 * addition is associative, so the order of the GPU's atomics cannot matter).
 * The prepared affine momentum (the per-particle stress cache) is an input:
 * it involves transcendental functions whose last bits are not specified.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define FIXED_WORDS 11

static float quad_weight(float f, int o)
{
    if (o == 0) {
        float l = 1.5f - f;
        return (0.5f * l) * l;
    }
    if (o == 1) {
        float c = f - 1.0f;
        return 0.75f - c * c;
    }
    float r = f - 0.5f;
    return (0.5f * r) * r;
}

static float det2(const float *m)
{
    float second = m[1] * m[2];
    float err = fmaf(m[1], m[2], -second);
    return fmaf(m[0], m[3], -second) - err;
}

/* Returns the range-error flag (65536) or 0.  words has node_count * 11
 * int32 entries, zero on entry. */
uint32_t emu_fixed_point_scatter(int32_t n, const float *pos, const float *vel, const float *F,
                                 const float *volume, const uint32_t *model, const float *density,
                                 const float *affine, float dx, float particle_mass, float particle_volume,
                                 int32_t cells_x, int32_t cells_y, int32_t shift, int32_t *words)
{
    uint32_t flags = 0;
    const uint32_t node_w = (uint32_t)cells_x + 3u;
    const float scale = ldexpf(1.0f, shift);
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t m = model[i];
        const int liquid = m == 2u || m == 3u;
        const float mass = liquid ? density[i] * volume[i] : particle_mass;
        const float vliq = liquid ? volume[i] * det2(F + 4 * i) : 0.0f;
        const float gx = pos[2 * i] / dx, gy = pos[2 * i + 1] / dx;
        const int bx = (int)floorf(gx - 0.5f), by = (int)floorf(gy - 0.5f);
        if (bx < -1 || by < -1 || bx + 2 > cells_x + 1 || by + 2 > cells_y + 1) return 1u; /* stencil */
        const float fx = gx - (float)bx, fy = gy - (float)by;
        const float *A = affine + 4 * i;
        const uint32_t channel = m == 2u ? 3u : (m == 3u ? 7u : 0u);
        for (int oy = 0; oy < 3; ++oy)
            for (int ox = 0; ox < 3; ++ox) {
                const float w = quad_weight(fx, ox) * quad_weight(fy, oy);
                const float dpx = ((float)ox - fx) * dx, dpy = ((float)oy - fy) * dx;
                const float mx = (mass * vel[2 * i] + A[0] * dpx) + A[1] * dpy;
                const float my = (mass * vel[2 * i + 1] + A[2] * dpx) + A[3] * dpy;
                const uint32_t node = (uint32_t)(by + oy + 1) * node_w + (uint32_t)(bx + ox + 1);
                const float values[4] = {(w * mass) / particle_mass, (w * mx) / particle_mass,
                                         (w * my) / particle_mass, (w * vliq) / particle_volume};
                const int count = liquid ? 4 : 3;
                for (int k = 0; k < count; ++k) {
                    const float scaled = rintf(values[k] * scale);
                    if (!isfinite(scaled) || fabsf(scaled) > 2147483520.0f) {
                        flags |= 65536u;
                        continue;
                    }
                    const int32_t inc = (int32_t)scaled;
                    int32_t *slot = &words[(size_t)node * FIXED_WORDS + channel + (uint32_t)k];
                    const int32_t prev = *slot;
                    if ((inc > 0 && prev > 2147483647 - inc) || (inc < 0 && prev < (-2147483647 - 1) - inc))
                        flags |= 65536u;
                    *slot = (int32_t)((uint32_t)prev + (uint32_t)inc);
                }
            }
    }
    return flags;
}
