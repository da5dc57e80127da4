// mpm_adjoint.cu -- the differentiable form of the substep: a batch of scenes
// of Tait water and fixed-corotated solid particles stepped on dense per-scene
// halo grids with a fixed dt per scene, the loss sum |x(T) - target|^2, and
// its adjoint by checkpoint and recompute (include/mpm_b200.h, mpma_*).
//
// The forward is the default path's arithmetic for these two models
// (prepareParticle, p2g, updateGrid + finishGridVelocity, g2p of
// src/lib/mpm/kernels/shaders.ts:808-963, :1072-1211, :1485-1777,
// :2114-2421): Tait stress -det * lambda * (det^-gamma - 1), fixed-corotated
// stress 2 mu (F - R) F^T + lambda J (J - 1), APIC transfer with the
// quadratic B-spline, liquid density-contrast acceleration, the deformation
// update in (I + h C)^k increments, liquid projection to sqrt(clamp(J)) R,
// wall cushion and friction, confinement.  Sums are scattered with vector
// atomics (their order is not fixed; the gradient does not need it to be).
//
// The adjoint differentiates that arithmetic exactly where it is smooth and
// keeps the forward's branch where it is not (subgradients): confinement and
// the wall factors act as masks, the liquid determinant clamp stops the
// gradient outside [0.5, 2], the increment count k and the stencil's base
// node are held.  The polar rotation of a 2x2 F with det F > 0 is the
// rotation by atan2(F10 - F01, F00 + F11), which is what both the forward and
// the adjoint use.
//
// Per backward segment of K substeps: the segment's start state is restored
// from its checkpoint, the K substeps are recomputed keeping each substep's
// input state and grid sums, then each substep is reversed by two kernels: the
// G2P adjoint (scatters the node-velocity adjoints) and the fused grid + P2G
// adjoint (gathers them back to the particle and adds the parameter
// gradients).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_device.cuh"

namespace mpm {
int host_error(int code, const char *message);
void host_clear_error();
}  // namespace mpm

using namespace mpm;

namespace {

constexpr unsigned ADJ_THREADS = 256;

// Per-scene constants; tait, lambda_s and mu_s are the differentiated
// material parameters.
struct AdjScene {
    uint32_t n, p_base, node_base, node_w;
    uint32_t cells_x, cells_y, tile_base, tiles_x;  // 16x16-node tiles of the halo grid, row-major
    float dx, inv_dx, gs, dt;
    float gx, gy, domain_w, domain_h;
    float solid_mass, wall_friction, rho, gamma;
    float tait, lambda_s, mu_s, pad2;
};

struct AdjState {
    float2 *x, *v;
    float4 *C, *F;
};

struct AdjCtx {
    const AdjScene *scenes;
    const uint32_t *scene_of;  // per particle
    const uint32_t *liquid;    // per particle: 1 Tait water, 0 fixed-corotated solid
    const float *vol;          // per particle
    uint32_t n;
    uint32_t *status;
    AdjState in, out;
    float4 *sum_s, *sum_w;  // per node: solid (m, qx, qy, 0), water (m, qx, qy, V)
    float2 *gv_s;           // per node: solid velocity (k_adj_grid_fwd)
    float4 *gv_w;           // per node: water velocity (x, y), liquid mass, liquid volume
    // adjoints: of the substep's outputs (next) and inputs (cur)
    float2 *xb_next, *vb_next, *xb, *vb;
    float4 *Cb_next, *Fb_next, *Cb, *Fb;
    float2 *xg;            // the G2P part of the input position adjoint
    float4 *Fg;            // the G2P part of the input F adjoint
    float4 *ub_s;          // per node: solid velocity adjoint (x, y), then (Qx, Qy, M) adjoints, 0
    float4 *ub_w;          // per node: water velocity, liquid mass, liquid volume adjoints
    double *param_grad;    // per scene: tait, lambda_s, mu_s
    const float2 *target;  // per particle
    double *loss;          // per scene
    uint8_t *mark_out;     // per tile: marked when a new position's stencil reaches it (k_adj_g2p), or NULL
};

constexpr int ADJ_TILE = 16;  // nodes per side of a clearing tile

constexpr uint32_t ADJ_ERR_STENCIL = 1u, ADJ_ERR_NONFINITE = 2u, ADJ_ERR_DETERMINANT = 4u;

__device__ __forceinline__ void adj_fail(const AdjCtx &c, uint32_t flag) { atomicOr(c.status, flag); }

// ------------------------------------------------------------ 2x2 helpers --

__device__ __forceinline__ float4 cofactor(float4 F) { return make_float4(F.w, -F.z, -F.y, F.x); }

// d(det)/dF for a row-major (F00, F01, F10, F11).
__device__ __forceinline__ float4 axpy4(float a, float4 x, float4 y)
{
    return make_float4(y.x + a * x.x, y.y + a * x.y, y.z + a * x.z, y.w + a * x.w);
}

// Rotation by phi = atan2(F10 - F01, F00 + F11), as (cos, sin); the polar
// rotation of F when det F > 0.
__device__ __forceinline__ float2 polar_angle(float4 F)
{
    const float a = F.x + F.w, b = F.z - F.y;
    const float r = sqrtf(a * a + b * b);
    return r > 0.0f ? make_float2(a / r, b / r) : make_float2(1.0f, 0.0f);
}

__device__ __forceinline__ float4 rotation(float2 cs) { return make_float4(cs.x, -cs.y, cs.y, cs.x); }

// Adds phi_bar * d(phi)/dF to Fb (phi = atan2(F10 - F01, F00 + F11)).
__device__ __forceinline__ float4 angle_adjoint(float4 F, float phi_bar, float4 Fb)
{
    const float a = F.x + F.w, b = F.z - F.y, r2 = a * a + b * b;
    if (!(r2 > 0.0f)) return Fb;
    const float da = -b / r2 * phi_bar, db = a / r2 * phi_bar;
    return make_float4(Fb.x + da, Fb.y - db, Fb.z + db, Fb.w + da);
}

// ------------------------------------------------------------- stencil ----

struct AdjStencil {
    int bx, by;
    float fx, fy;
    float wx[3], wy[3], dwx[3], dwy[3];  // weights and their derivatives in the fraction
};

__device__ __forceinline__ bool adj_stencil(const AdjScene &S, float2 x, AdjStencil &st)
{
    const float gx = __fmul_rn(x.x, S.inv_dx), gy = __fmul_rn(x.y, S.inv_dx);
    if (!finite_f(gx) || !finite_f(gy)) return false;
    st.bx = (int)floorf(__fsub_rn(gx, 0.5f));
    st.by = (int)floorf(__fsub_rn(gy, 0.5f));
    st.fx = __fsub_rn(gx, (float)st.bx);
    st.fy = __fsub_rn(gy, (float)st.by);
    if (st.bx < -1 || st.by < -1 || st.bx + 2 > (int)S.cells_x + 1 || st.by + 2 > (int)S.cells_y + 1) return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        st.wx[k] = quad_weight(st.fx, k);
        st.wy[k] = quad_weight(st.fy, k);
    }
    // d/df of 0.5 (1.5 - f)^2, 0.75 - (f - 1)^2, 0.5 (f - 0.5)^2
    st.dwx[0] = st.fx - 1.5f, st.dwx[1] = -2.0f * (st.fx - 1.0f), st.dwx[2] = st.fx - 0.5f;
    st.dwy[0] = st.fy - 1.5f, st.dwy[1] = -2.0f * (st.fy - 1.0f), st.dwy[2] = st.fy - 0.5f;
    return true;
}

__device__ __forceinline__ uint32_t adj_node(const AdjScene &S, int ix, int iy)
{
    return S.node_base + (uint32_t)(iy + 1) * S.node_w + (uint32_t)(ix + 1);
}

// ------------------------------------------------------------ materials ---

struct Prepared {
    float m, vliq, scale, det;
    float4 s, A;
};

// prepareParticle for the two differentiable models.
__device__ __forceinline__ bool adj_prepare(const AdjScene &S, bool liquid, float vol, float4 C, float4 F, Prepared &p)
{
    p.det = det2(F);
    if (!finite_f(p.det) || p.det <= 0.0f) return false;
    if (liquid) {
        const float pw = pow_wgsl(__fdiv_rn(1.0f, p.det), S.gamma);
        const float sigma = -p.det * (S.tait * (pw - 1.0f));
        p.s = make_float4(sigma, 0.f, 0.f, sigma);
        p.m = __fmul_rn(S.rho, vol);
        p.vliq = __fmul_rn(vol, p.det);
    } else {
        const float4 R = rotation(polar_angle(F));
        const float4 d = make_float4(F.x - R.x, F.y - R.y, F.z - R.z, F.w - R.w);
        const float shear = 2.0f * S.mu_s, volumetric = S.lambda_s * p.det * (p.det - 1.0f);
        p.s = make_float4(shear * (d.x * F.x + d.y * F.y) + volumetric, shear * (d.x * F.z + d.y * F.w),
                          shear * (d.z * F.x + d.w * F.y), shear * (d.z * F.z + d.w * F.w) + volumetric);
        p.m = S.solid_mass;
        p.vliq = 0.0f;
    }
    p.scale = -S.dt * vol * S.gs;
    p.A = make_float4(p.m * C.x + p.scale * p.s.x, p.m * C.y + p.scale * p.s.y, p.m * C.z + p.scale * p.s.z,
                      p.m * C.w + p.scale * p.s.w);
    return finite4(p.A);
}

// Stress adjoint: adds dL/dF to Fb and returns the parameter adjoints
// (tait, lambda_s, mu_s) for the stress adjoint sb.
__device__ __forceinline__ float3 stress_adjoint(const AdjScene &S, bool liquid, float4 F, float det, float4 sb,
                                                 float4 &Fb)
{
    if (liquid) {
        const float pw = pow_wgsl(__fdiv_rn(1.0f, det), S.gamma);
        const float sigma_b = sb.x + sb.w;
        // sigma = -tait (det^(1-gamma) - det)
        const float dsigma = -S.tait * ((1.0f - S.gamma) * pw - 1.0f);
        Fb = axpy4(sigma_b * dsigma, cofactor(F), Fb);
        return make_float3(sigma_b * -(det * pw - det), 0.f, 0.f);
    }
    const float2 cs = polar_angle(F);
    const float4 R = rotation(cs);
    const float4 D = make_float4(F.x - R.x, F.y - R.y, F.z - R.z, F.w - R.w);
    // mu: s : 2 (F - R) F^T
    const float4 DFt = make_float4(D.x * F.x + D.y * F.y, D.x * F.z + D.y * F.w, D.z * F.x + D.w * F.y,
                                   D.z * F.z + D.w * F.w);
    const float mu_b = 2.0f * (sb.x * DFt.x + sb.y * DFt.y + sb.z * DFt.z + sb.w * DFt.w);
    const float trace_b = sb.x + sb.w;
    const float lambda_b = trace_b * det * (det - 1.0f);
    Fb = axpy4(trace_b * S.lambda_s * (2.0f * det - 1.0f), cofactor(F), Fb);
    // 2 mu (F F^T - R F^T): (sb + sb^T) F - sb^T R for F, sb F for R
    const float m2 = 2.0f * S.mu_s;
    const float4 sym = make_float4(2.0f * sb.x, sb.y + sb.z, sb.z + sb.y, 2.0f * sb.w);
    const float4 symF = make_float4(sym.x * F.x + sym.y * F.z, sym.x * F.y + sym.y * F.w, sym.z * F.x + sym.w * F.z,
                                    sym.z * F.y + sym.w * F.w);
    const float4 sTR = make_float4(sb.x * R.x + sb.z * R.z, sb.x * R.y + sb.z * R.w, sb.y * R.x + sb.w * R.z,
                                   sb.y * R.y + sb.w * R.w);
    Fb = make_float4(Fb.x + m2 * (symF.x - sTR.x), Fb.y + m2 * (symF.y - sTR.y), Fb.z + m2 * (symF.z - sTR.z),
                     Fb.w + m2 * (symF.w - sTR.w));
    // R adjoint -m2 sb F, then through the angle: dR/dphi = (-sin, -cos, cos, -sin)
    const float4 sF = make_float4(sb.x * F.x + sb.y * F.y, sb.x * F.z + sb.y * F.w, sb.z * F.x + sb.w * F.y,
                                  sb.z * F.z + sb.w * F.w);
    const float4 Rb = make_float4(-m2 * sF.x, -m2 * sF.y, -m2 * sF.z, -m2 * sF.w);
    const float phi_b = Rb.x * -cs.y + Rb.y * -cs.x + Rb.z * cs.x + Rb.w * -cs.y;
    Fb = angle_adjoint(F, phi_b, Fb);
    return make_float3(0.f, lambda_b, mu_b);
}

// ------------------------------------------------------------ grid node ---

// The wall factors of updateGrid's applyWallCushion / applyWallTangentialFriction
// (shaders.ts:1438-1457) for a pre-wall velocity u at node (x, y).
__device__ __forceinline__ float cushion_factor(float u, int coord, int extent)
{
    const float cushion = fminf(WALL_CUSHION_CELLS, (float)extent / 4.0f);
    const float dist = u < 0.0f ? (float)coord : (float)(extent - coord);
    if (dist >= cushion) return 1.0f;
    return fminf(fmaxf(dist / cushion, 0.0f), 1.0f);
}

__device__ __forceinline__ float friction_factor(int coord, int extent, float friction)
{
    if (friction <= 0.0f) return 1.0f;
    const float dist = fmaxf(0.0f, fminf((float)coord, (float)(extent - coord)));
    const float cushion = fminf(WALL_CUSHION_CELLS, (float)extent / 4.0f);
    if (dist >= cushion) return 1.0f;
    return 1.0f - friction * (1.0f - fminf(fmaxf(dist / cushion, 0.0f), 1.0f));
}

// Node velocity from its sums (finishGridVelocity + walls); D receives the
// wall factors per axis.
__device__ __forceinline__ float2 node_velocity_adj(const AdjScene &S, float4 sum, int ix, int iy, float2 &D)
{
    D = make_float2(0.f, 0.f);
    if (!(sum.x > 0.0f)) return make_float2(0.f, 0.f);
    const float inv = __frcp_rn(sum.x);
    const float2 u0 = make_float2(sum.y * inv + S.dt * S.gx, sum.z * inv + S.dt * S.gy);
    const int cx = (int)S.cells_x, cy = (int)S.cells_y;
    D.x = cushion_factor(u0.x, ix, cx) * friction_factor(iy, cy, S.wall_friction);
    D.y = cushion_factor(u0.y, iy, cy) * friction_factor(ix, cx, S.wall_friction);
    return make_float2(u0.x * D.x, u0.y * D.y);
}

// --------------------------------------------------------------- G2P ------

// The forward G2P quantities of one particle that its adjoint reuses.
struct G2pFwd {
    float2 vp;       // interpolated velocity (after the liquid acceleration)
    float4 B;        // sum w u dp^T
    float pm, pv;    // interpolated liquid mass and volume
    float pdet;      // det of the input F
    float4 Cn;       // new C
    float4 trial;    // F before the projection
    uint32_t sub;    // deformation increments
    float2 xn;       // new position before confinement
};

// With `keep_u` / `keep_mv` (shared memory, [stencil node][ADJ_THREADS]) it
// also keeps each stencil node's velocity and, for a liquid, its liquid mass
// and volume, for this thread's adjoint.
template <bool KEEP = false>
__device__ __forceinline__ bool g2p_forward(const AdjCtx &c, const AdjScene &S, bool liquid, const AdjStencil &st,
                                            float2 x, float4 F0, G2pFwd &g, float2 (*keep_u)[ADJ_THREADS] = nullptr,
                                            float2 (*keep_mv)[ADJ_THREADS] = nullptr)
{
    g.vp = make_float2(0.f, 0.f);
    g.B = make_float4(0.f, 0.f, 0.f, 0.f);
    g.pm = g.pv = 0.f;
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
        const float dpy = ((float)oy - st.fy) * S.dx;
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const float w = st.wx[ox] * st.wy[oy];
            const float dpx = ((float)ox - st.fx) * S.dx;
            const uint32_t n = adj_node(S, st.bx + ox, st.by + oy);
            float2 u;
            float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);  // liquid mass in x, liquid volume in w
            if (liquid) {
                const float4 gw = c.gv_w[n];
                u = make_float2(gw.x, gw.y);
                sum.x = gw.z;
                sum.w = gw.w;
            } else {
                u = c.gv_s[n];
            }
            if constexpr (KEEP) {
                keep_u[oy * 3 + ox][threadIdx.x] = u;
                keep_mv[oy * 3 + ox][threadIdx.x] = make_float2(sum.x, sum.w);
            }
            g.vp.x += w * u.x;
            g.vp.y += w * u.y;
            g.B.x += w * u.x * dpx;
            g.B.y += w * u.x * dpy;
            g.B.z += w * u.y * dpx;
            g.B.w += w * u.y * dpy;
            if (liquid) {
                g.pm += w * sum.x;
                g.pv += w * sum.w;
            }
        }
    }
    g.pdet = det2(F0);
    if (liquid) {
        if (!(g.pm > 0.f) || !(g.pv > 0.f) || !(g.pdet > 0.f)) return false;
        const float pd = S.rho / g.pdet, ld = g.pm / g.pv;
        const float rd = (pd - ld) / pd;
        g.vp.x += S.dt * (rd * S.gx);
        g.vp.y += S.dt * (rd * S.gy);
    }
    g.Cn = make_float4(g.B.x * S.gs, g.B.y * S.gs, g.B.z * S.gs, g.B.w * S.gs);
    g.xn = make_float2(x.x + S.dt * g.vp.x, x.y + S.dt * g.vp.y);
    const float row = fmaxf(fabsf(g.Cn.x) + fabsf(g.Cn.y), fabsf(g.Cn.z) + fabsf(g.Cn.w));
    const float req = ceilf(S.dt * row * (1.0f / MAX_DEFORMATION_INCREMENT));
    if (!finite_f(req) || req > MAX_DEFORMATION_SUBSTEPS) return false;
    g.sub = max(1u, (uint32_t)req);
    g.trial = integrate_deformation(F0, g.Cn, S.dt, g.sub);
    float tdet = det2(g.trial);
    while (finite_f(tdet) && tdet <= 0.f && g.sub < 64u) {
        g.sub = min(g.sub * 2u, 64u);
        g.trial = integrate_deformation(F0, g.Cn, S.dt, g.sub);
        tdet = det2(g.trial);
    }
    return finite_f(tdet) && tdet > 0.f && finite2(g.vp) && finite4(g.Cn);
}

// projectLiquidDeformation (shaders.ts:474-488) as sqrt(clamp(det T)) R(T).
__device__ __forceinline__ float4 project_liquid(float4 T)
{
    const float2 cs = polar_angle(T);
    const float sc = sqrtf(fminf(fmaxf(det2(T), MIN_LIQUID_DETERMINANT), MAX_LIQUID_DETERMINANT));
    return make_float4(sc * cs.x, -sc * cs.y, sc * cs.y, sc * cs.x);
}

}  // namespace

// Marks the clearing tiles that the stencil with base (bx, by) reaches (its
// corner nodes lie in at most four).  Lanes of a warp storing to the same
// mark byte in one instruction make one memory transaction.
__device__ __forceinline__ void mark_tiles(uint8_t *mark, const AdjScene &S, int bx, int by)
{
    const uint32_t x0 = (uint32_t)(bx + 1) / ADJ_TILE, x1 = (uint32_t)(bx + 3) / ADJ_TILE;
    const uint32_t y0 = (uint32_t)(by + 1) / ADJ_TILE, y1 = (uint32_t)(by + 3) / ADJ_TILE;
    uint8_t *row0 = mark + S.tile_base + y0 * S.tiles_x, *row1 = mark + S.tile_base + y1 * S.tiles_x;
    row0[x0] = 1u;
    if (x1 != x0) row0[x1] = 1u;
    if (y1 != y0) {
        row1[x0] = 1u;
        if (x1 != x0) row1[x1] = 1u;
    }
}

// ------------------------------------------------------------- kernels ----

__global__ void __launch_bounds__(ADJ_THREADS) k_adj_p2g(AdjCtx c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const AdjScene &S = c.scenes[c.scene_of[i]];
    const bool liquid = c.liquid[i] != 0u;
    const float2 x = c.in.x[i], v = c.in.v[i];
    Prepared p;
    if (!adj_prepare(S, liquid, c.vol[i], c.in.C[i], c.in.F[i], p)) {
        adj_fail(c, ADJ_ERR_DETERMINANT);
        return;
    }
    AdjStencil st;
    if (!adj_stencil(S, x, st)) {
        adj_fail(c, ADJ_ERR_STENCIL);
        return;
    }
    float4 *sums = liquid ? c.sum_w : c.sum_s;
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
        const float dpy = ((float)oy - st.fy) * S.dx;
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const float w = st.wx[ox] * st.wy[oy];
            const float dpx = ((float)ox - st.fx) * S.dx;
            const float qx = p.m * v.x + p.A.x * dpx + p.A.y * dpy;
            const float qy = p.m * v.y + p.A.z * dpx + p.A.w * dpy;
            atomicAdd(&sums[adj_node(S, st.bx + ox, st.by + oy)],
                      make_float4(w * p.m, w * qx, w * qy, liquid ? w * p.vliq : 0.f));
        }
    }
}

__global__ void __launch_bounds__(ADJ_THREADS) k_adj_g2p(AdjCtx c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const AdjScene &S = c.scenes[c.scene_of[i]];
    const bool liquid = c.liquid[i] != 0u;
    const float2 x = c.in.x[i];
    const float4 F0 = c.in.F[i];
    AdjStencil st;
    G2pFwd g;
    if (!adj_stencil(S, x, st) || !g2p_forward(c, S, liquid, st, x, F0, g)) {
        adj_fail(c, ADJ_ERR_NONFINITE);
        return;
    }
    const float4 Fn = liquid ? project_liquid(g.trial) : g.trial;
    const float2 bx = confine_axis(g.xn.x, g.vp.x, S.domain_w);
    const float2 by = confine_axis(g.xn.y, g.vp.y, S.domain_h);
    if (c.mark_out) {
        AdjStencil next;
        if (adj_stencil(S, make_float2(bx.x, by.x), next)) mark_tiles(c.mark_out, S, next.bx, next.by);
    }
    c.out.x[i] = make_float2(bx.x, by.x);
    c.out.v[i] = make_float2(bx.y, by.y);
    c.out.C[i] = g.Cn;
    c.out.F[i] = Fn;
}

// Loss sum |x - target|^2 per scene (one atomic per warp whose particles
// share a scene) and its adjoint seeds.
// Marks the clearing tiles the stencils of the particles in c.in reach (the
// first substep's; later substeps' marks come from k_adj_g2p).
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_mark(AdjCtx c, uint8_t *mark)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const AdjScene &S = c.scenes[c.scene_of[i]];
    AdjStencil st;
    if (adj_stencil(S, c.in.x[i], st)) mark_tiles(mark, S, st.bx, st.by);
}

constexpr int COMPACT_THREADS = 256;

// Appends the marked tiles of one substep to its list (list[0], zeroed before,
// counts them; list[1 ..] holds them in no particular order: each tile is
// cleared and updated on its own).  One tile per thread, one atomic per warp.
__global__ void __launch_bounds__(COMPACT_THREADS) k_adj_compact(const uint8_t *mark, uint32_t n_tiles, uint32_t *list)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool marked = t < n_tiles && mark[t] != 0u;
    const unsigned ballot = __ballot_sync(0xffffffffu, marked);
    if (!ballot) return;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (lane == 0u) base = atomicAdd(list, (uint32_t)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (marked) list[1 + base + __popc(ballot & ((1u << lane) - 1u))] = t;
}

// Zeroes the nodes of the listed (marked) tiles in up to three node arrays
// (NULL: skipped), one tile per CTA iteration and one node per thread: every
// node a substep adds to or reads lies in a tile its particles mark.  The rest
// of the grid keeps stale values that no stencil reads.  tile_scene gives each
// tile's scene; list[0] counts the tiles in list[1 ..].
__global__ void __launch_bounds__(ADJ_TILE * ADJ_TILE) k_adj_clear(const AdjScene *scenes, const uint32_t *tile_scene,
                                                                   const uint32_t *list, float4 *a, float4 *b, float2 *c2)
{
    const uint32_t count = list[0];
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t t = list[1 + i];
        const AdjScene &S = scenes[tile_scene[t]];
        const uint32_t local = t - S.tile_base;
        const uint32_t hx = (local % S.tiles_x) * ADJ_TILE + threadIdx.x % ADJ_TILE;
        const uint32_t hy = (local / S.tiles_x) * ADJ_TILE + threadIdx.x / ADJ_TILE;
        if (hx >= S.node_w || hy >= S.cells_y + 3u) continue;
        const uint32_t n = S.node_base + hy * S.node_w + hx;
        if (a) a[n] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (b) b[n] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c2) c2[n] = make_float2(0.f, 0.f);
    }
}

// The grid update of the marked tiles' nodes (finishGridVelocity with the
// wall factors, node_velocity_adj): each node's velocity from its sums, once
// per node, for the G2P kernels; the water record also carries the node's
// liquid mass and volume.  One tile per CTA iteration, one node per thread.
__global__ void __launch_bounds__(ADJ_TILE * ADJ_TILE) k_adj_grid_fwd(AdjCtx c, const uint32_t *tile_scene,
                                                                      const uint32_t *list)
{
    const uint32_t count = list[0];
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t t = list[1 + i];
        const AdjScene &S = c.scenes[tile_scene[t]];
        const uint32_t local = t - S.tile_base;
        const uint32_t hx = (local % S.tiles_x) * ADJ_TILE + threadIdx.x % ADJ_TILE;
        const uint32_t hy = (local / S.tiles_x) * ADJ_TILE + threadIdx.x / ADJ_TILE;
        if (hx >= S.node_w || hy >= S.cells_y + 3u) continue;
        const uint32_t n = S.node_base + hy * S.node_w + hx;
        const int ix = (int)hx - 1, iy = (int)hy - 1;
        float2 D;
        c.gv_s[n] = node_velocity_adj(S, c.sum_s[n], ix, iy, D);
        const float4 w = c.sum_w[n];
        const float2 u = node_velocity_adj(S, w, ix, iy, D);
        c.gv_w[n] = make_float4(u.x, u.y, w.x, w.w);
    }
}

// The grid-update adjoint of the marked tiles' nodes, in place: the node
// velocity adjoints that k_adj_g2p_bwd scattered become the adjoints of the
// node sums (u = D (q / m + dt g): momentum q, mass m; the liquid volume's
// passes through), once per node instead of once per particle reaching it.
// One tile per CTA iteration, one node per thread.
__global__ void __launch_bounds__(ADJ_TILE * ADJ_TILE) k_adj_grid_bwd(AdjCtx c, const uint32_t *tile_scene,
                                                                      const uint32_t *list)
{
    const uint32_t count = list[0];
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t t = list[1 + i];
        const AdjScene &S = c.scenes[tile_scene[t]];
        const uint32_t local = t - S.tile_base;
        const uint32_t hx = (local % S.tiles_x) * ADJ_TILE + threadIdx.x % ADJ_TILE;
        const uint32_t hy = (local / S.tiles_x) * ADJ_TILE + threadIdx.x / ADJ_TILE;
        if (hx >= S.node_w || hy >= S.cells_y + 3u) continue;
        const uint32_t n = S.node_base + hy * S.node_w + hx;
        const int ix = (int)hx - 1, iy = (int)hy - 1;
#pragma unroll
        for (int channel = 0; channel < 2; ++channel) {
            float4 *ub = channel ? c.ub_w : c.ub_s;
            const float4 sum = channel ? c.sum_w[n] : c.sum_s[n];
            const float4 b = ub[n];  // velocity (x, y), liquid mass, liquid volume adjoints
            float M_b = channel ? b.z : 0.f, Qx_b = 0.f, Qy_b = 0.f;
            if (sum.x > 0.0f) {
                float2 D;
                node_velocity_adj(S, sum, ix, iy, D);
                const float inv = 1.0f / sum.x;
                const float udx = D.x * b.x, udy = D.y * b.y;
                Qx_b = udx * inv;
                Qy_b = udy * inv;
                M_b -= (udx * sum.y + udy * sum.z) * inv * inv;
            }
            ub[n] = make_float4(Qx_b, Qy_b, M_b, channel ? b.w : 0.f);
        }
    }
}

__global__ void __launch_bounds__(ADJ_THREADS) k_adj_loss(AdjCtx c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < c.n;
    const uint32_t scene = valid ? c.scene_of[i] : 0u;
    double term = 0.0;
    if (valid) {
        const float2 x = c.in.x[i], t = c.target[i];
        const float dx = x.x - t.x, dy = x.y - t.y;
        term = (double)dx * dx + (double)dy * dy;
        c.xb_next[i] = make_float2(2.0f * dx, 2.0f * dy);
        c.vb_next[i] = make_float2(0.f, 0.f);
        c.Cb_next[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        c.Fb_next[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const unsigned full = 0xffffffffu;
    const uint32_t lead = __shfl_sync(full, scene, 0);
    if (__all_sync(full, !valid || scene == lead)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(full, term, o);
        if ((threadIdx.x & 31u) == 0u) atomicAdd(&c.loss[lead], term);
    } else if (valid) {
        atomicAdd(&c.loss[scene], term);
    }
}

// The G2P adjoint of one substep: from the adjoints of the substep's outputs
// (x, v, C, F) to the node-velocity adjoints (scattered) and the G2P parts of
// the input position and F adjoints.
__global__ void __launch_bounds__(ADJ_THREADS, 3) k_adj_g2p_bwd(AdjCtx c)
{
    // this thread's stencil node velocities and liquid sums from the forward
    // recompute, read again by the adjoint's scatter
    __shared__ float2 s_u[9][ADJ_THREADS];
    __shared__ float2 s_mv[9][ADJ_THREADS];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const AdjScene &S = c.scenes[c.scene_of[i]];
    const bool liquid = c.liquid[i] != 0u;
    const float2 x = c.in.x[i];
    const float4 F0 = c.in.F[i];
    AdjStencil st;
    G2pFwd g;
    if (!adj_stencil(S, x, st) || !g2p_forward<true>(c, S, liquid, st, x, F0, g, s_u, s_mv)) {
        adj_fail(c, ADJ_ERR_NONFINITE);
        return;
    }
    const float2 xbo = c.xb_next[i], vbo = c.vb_next[i];
    const float4 Cbo = c.Cb_next[i], Fbo = c.Fb_next[i];
    // confinement: a clamped axis passes no gradient
    const float2 cxa = confine_axis(g.xn.x, g.vp.x, S.domain_w);
    const float2 cya = confine_axis(g.xn.y, g.vp.y, S.domain_h);
    const bool free_x = cxa.x == g.xn.x, free_y = cya.x == g.xn.y;
    float2 xb = make_float2(free_x ? xbo.x : 0.f, free_y ? xbo.y : 0.f);
    float2 vpb = make_float2(free_x ? vbo.x + S.dt * xbo.x : 0.f, free_y ? vbo.y + S.dt * xbo.y : 0.f);
    // projection
    float4 Tb = Fbo;
    if (liquid) {
        const float4 T = g.trial;
        const float2 cs = polar_angle(T);
        const float J = det2(T);
        const float Jc = fminf(fmaxf(J, MIN_LIQUID_DETERMINANT), MAX_LIQUID_DETERMINANT);
        const float sc = sqrtf(Jc);
        // F = sc (cos, -sin, sin, cos)
        const float sc_b = Fbo.x * cs.x - Fbo.y * cs.y + Fbo.z * cs.y + Fbo.w * cs.x;
        const float phi_b = sc * (Fbo.x * -cs.y + Fbo.y * -cs.x + Fbo.z * cs.x + Fbo.w * -cs.y);
        const float J_b = (J == Jc) ? sc_b * 0.5f / sc : 0.f;
        Tb = make_float4(0.f, 0.f, 0.f, 0.f);
        Tb = axpy4(J_b, cofactor(T), Tb);
        Tb = angle_adjoint(T, phi_b, Tb);
    }
    // deformation increments: T = U^k F0, U = I + h C'
    const float h = g.sub == 1u ? S.dt : __fdiv_rn(S.dt, (float)g.sub);
    const float4 U = make_float4(1.0f + h * g.Cn.x, h * g.Cn.y, h * g.Cn.z, 1.0f + h * g.Cn.w);
    float4 G = Tb, Ub = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = (int)g.sub - 1; j >= 0; --j) {
        float4 Fj = F0;  // U^j F0
        for (int q = 0; q < j; ++q)
            Fj = make_float4(U.x * Fj.x + U.y * Fj.z, U.x * Fj.y + U.y * Fj.w, U.z * Fj.x + U.w * Fj.z,
                             U.z * Fj.y + U.w * Fj.w);
        // Ub += G Fj^T; G = U^T G
        Ub = make_float4(Ub.x + G.x * Fj.x + G.y * Fj.y, Ub.y + G.x * Fj.z + G.y * Fj.w,
                         Ub.z + G.z * Fj.x + G.w * Fj.y, Ub.w + G.z * Fj.z + G.w * Fj.w);
        G = make_float4(U.x * G.x + U.z * G.z, U.x * G.y + U.z * G.w, U.y * G.x + U.w * G.z, U.y * G.y + U.w * G.w);
    }
    float4 Fg = G;
    const float4 Cnb = make_float4(Cbo.x + h * Ub.x, Cbo.y + h * Ub.y, Cbo.z + h * Ub.z, Cbo.w + h * Ub.w);
    const float4 Bb = make_float4(Cnb.x * S.gs, Cnb.y * S.gs, Cnb.z * S.gs, Cnb.w * S.gs);
    // liquid acceleration v += dt g (1 - ld pdet / rho), ld = pm / pv
    float pm_b = 0.f, pv_b = 0.f;
    if (liquid) {
        const float rd_b = S.dt * (S.gx * vpb.x + S.gy * vpb.y);
        const float ld = g.pm / g.pv;
        const float ld_b = -rd_b * g.pdet / S.rho;
        const float pdet_b = -rd_b * ld / S.rho;
        Fg = axpy4(pdet_b, cofactor(F0), Fg);
        pm_b = ld_b / g.pv;
        pv_b = -ld_b * g.pm / (g.pv * g.pv);
    }
    // interpolation: scatter the node adjoints; the position adjoint through
    // the weights and offsets
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) {
        const float dpy = ((float)oy - st.fy) * S.dx;
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            const float w = st.wx[ox] * st.wy[oy];
            const float dpx = ((float)ox - st.fx) * S.dx;
            const uint32_t n = adj_node(S, st.bx + ox, st.by + oy);
            const float2 u = s_u[oy * 3 + ox][threadIdx.x];
            const float2 mv = s_mv[oy * 3 + ox][threadIdx.x];  // liquid mass and volume
            // node velocity adjoint: w vpb + w Bb dp
            const float ubx = w * (vpb.x + Bb.x * dpx + Bb.y * dpy);
            const float uby = w * (vpb.y + Bb.z * dpx + Bb.w * dpy);
            if (liquid)
                atomicAdd(&c.ub_w[n], make_float4(ubx, uby, w * pm_b, w * pv_b));
            else
                atomicAdd(reinterpret_cast<float2 *>(&c.ub_s[n]), make_float2(ubx, uby));
            // d/dx of w: (dwx wy, wx dwy) / dx
            const float gwx = st.dwx[ox] * st.wy[oy] * S.inv_dx, gwy = st.wx[ox] * st.dwy[oy] * S.inv_dx;
            float sval = u.x * (vpb.x + Bb.x * dpx + Bb.y * dpy) + u.y * (vpb.y + Bb.z * dpx + Bb.w * dpy);
            if (liquid) sval += pm_b * mv.x + pv_b * mv.y;
            // dp = (k - f) dx: d/dx = -1 per axis
            xb.x += gwx * sval - w * (u.x * Bb.x + u.y * Bb.z);
            xb.y += gwy * sval - w * (u.x * Bb.y + u.y * Bb.w);
        }
    }
    c.xg[i] = xb;
    c.Fg[i] = Fg;
}

// Sum of a value over the lanes of a warp whose particles all belong to one
// scene, else over the lanes of each scene separately through atomics.
__device__ __forceinline__ void add_param_grads(double *grad, uint32_t scene, float3 g, bool valid)
{
    const unsigned full = 0xffffffffu;
    const uint32_t lead = __shfl_sync(full, scene, 0);
    if (__all_sync(full, !valid || scene == lead)) {
        double a = valid ? g.x : 0.0, b = valid ? g.y : 0.0, d = valid ? g.z : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(full, a, o);
            b += __shfl_xor_sync(full, b, o);
            d += __shfl_xor_sync(full, d, o);
        }
        if ((threadIdx.x & 31u) == 0u) {
            if (a != 0.0) atomicAdd(grad + 3 * lead, a);
            if (b != 0.0) atomicAdd(grad + 3 * lead + 1, b);
            if (d != 0.0) atomicAdd(grad + 3 * lead + 2, d);
        }
    } else if (valid) {
        if (g.x != 0.f) atomicAdd(grad + 3 * scene, (double)g.x);
        if (g.y != 0.f) atomicAdd(grad + 3 * scene + 1, (double)g.y);
        if (g.z != 0.f) atomicAdd(grad + 3 * scene + 2, (double)g.z);
    }
}

// The grid-update and P2G adjoint of one substep, fused: each particle
// gathers, for its nine nodes, the adjoints of the node sums (from the node
// velocity adjoints and the sums, finishGridVelocity and the wall factors
// reversed), then reverses its own P2G contribution and stress; adds the G2P
// parts; writes the adjoints of the substep's inputs and the parameter
// gradients.
__global__ void __launch_bounds__(ADJ_THREADS, 3) k_adj_p2g_bwd(AdjCtx c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < c.n;
    const uint32_t scene = valid ? c.scene_of[i] : 0u;
    float3 pg = make_float3(0.f, 0.f, 0.f);
    bool ok = valid;
    if (valid) {
        const AdjScene &S = c.scenes[scene];
        const bool liquid = c.liquid[i] != 0u;
        const float2 x = c.in.x[i], v = c.in.v[i];
        const float4 C = c.in.C[i], F = c.in.F[i];
        const float vol = c.vol[i];
        Prepared p;
        AdjStencil st;
        ok = adj_prepare(S, liquid, vol, C, F, p) && adj_stencil(S, x, st);
        if (ok) {
            float2 xb = c.xg[i], vb = make_float2(0.f, 0.f);
            float4 Ab = make_float4(0.f, 0.f, 0.f, 0.f);
            float vliq_b = 0.f;
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float dpy = ((float)oy - st.fy) * S.dx;
#pragma unroll
                for (int ox = 0; ox < 3; ++ox) {
                    const float w = st.wx[ox] * st.wy[oy];
                    const float dpx = ((float)ox - st.fx) * S.dx;
                    const int ix = st.bx + ox, iy = st.by + oy;
                    const uint32_t n = adj_node(S, ix, iy);
                    // the node's sum adjoints (k_adj_grid_bwd): momentum, mass, liquid volume
                    const float4 g = liquid ? c.ub_w[n] : c.ub_s[n];
                    const float Qx_b = g.x, Qy_b = g.y, M_b = g.z, V_b = g.w;
                    // P2G adjoint of M += w m, Q += w (m v + A dp), V += w vliq
                    vb.x += w * p.m * Qx_b;
                    vb.y += w * p.m * Qy_b;
                    Ab.x += w * Qx_b * dpx;
                    Ab.y += w * Qx_b * dpy;
                    Ab.z += w * Qy_b * dpx;
                    Ab.w += w * Qy_b * dpy;
                    if (liquid) vliq_b += w * V_b;
                    const float qx = p.m * v.x + p.A.x * dpx + p.A.y * dpy;
                    const float qy = p.m * v.y + p.A.z * dpx + p.A.w * dpy;
                    const float sval = M_b * p.m + Qx_b * qx + Qy_b * qy + (liquid ? V_b * p.vliq : 0.f);
                    const float gwx = st.dwx[ox] * st.wy[oy] * S.inv_dx, gwy = st.wx[ox] * st.dwy[oy] * S.inv_dx;
                    xb.x += gwx * sval - w * (p.A.x * Qx_b + p.A.z * Qy_b);
                    xb.y += gwy * sval - w * (p.A.y * Qx_b + p.A.w * Qy_b);
                }
            }
            // A = m C + scale s
            const float4 Cb = make_float4(p.m * Ab.x, p.m * Ab.y, p.m * Ab.z, p.m * Ab.w);
            const float4 sb = make_float4(p.scale * Ab.x, p.scale * Ab.y, p.scale * Ab.z, p.scale * Ab.w);
            float4 Fb = c.Fg[i];
            if (liquid) Fb = axpy4(vliq_b * vol, cofactor(F), Fb);
            pg = stress_adjoint(S, liquid, F, p.det, sb, Fb);
            c.xb[i] = xb;
            c.vb[i] = vb;
            c.Cb[i] = Cb;
            c.Fb[i] = Fb;
            if (!finite2(xb) || !finite2(vb) || !finite4(Cb) || !finite4(Fb)) adj_fail(c, ADJ_ERR_NONFINITE);
        } else {
            adj_fail(c, ADJ_ERR_NONFINITE);
        }
    }
    add_param_grads(c.param_grad, scene, pg, ok);
}

// ----------------------------------------------------------------- host ---

struct mpm_adjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, n_scenes = 0, n_nodes = 0;
    std::vector<AdjScene> scenes;
    AdjScene *d_scenes = nullptr;
    uint32_t *scene_of = nullptr, *liquid = nullptr, *status = nullptr;
    float *vol = nullptr;
    AdjState init{}, ping[2]{};
    std::vector<AdjState> checkpoints, tape;
    float4 *sum_s = nullptr, *sum_w = nullptr;   // forward scratch
    uint8_t *mark = nullptr;                     // per substep (0 .. steps) and clearing tile
    size_t mark_count = 0;
    uint32_t *lists = nullptr;                   // per substep: marked-tile count, then the tiles
    uint32_t *tile_scene = nullptr;              // per clearing tile
    uint32_t n_tiles = 0;
    unsigned clear_ctas = 1;
    std::vector<float4 *> tape_s, tape_w;       // per recomputed substep
    float2 *xb[2]{}, *vb[2]{}, *xg = nullptr;
    float4 *Cb[2]{}, *Fb[2]{}, *Fg = nullptr, *ub_w = nullptr, *ub_s = nullptr;
    float2 *gv_s = nullptr;  // node velocities of the substep at hand
    float4 *gv_w = nullptr;
    double *param_grad = nullptr, *loss = nullptr;
    float2 *target = nullptr, *final_x = nullptr;
    uint32_t steps = 0, every = 0;
    int final_buffer = 0;
    bool forward_done = false;
    bool taped = false;  // the forward kept every substep's state and sums (one segment)
    cudaEvent_t ev[4]{};
    float forward_ms = 0.f, backward_ms = 0.f;
};

namespace {

template <typename T>
cudaError_t adj_alloc(T **ptr, size_t count)
{
    *ptr = nullptr;
    return cudaMalloc(reinterpret_cast<void **>(ptr), std::max<size_t>(count, 1) * sizeof(T));
}

cudaError_t alloc_state(AdjState &s, size_t n)
{
    cudaError_t e = adj_alloc(&s.x, n);
    if (e == cudaSuccess) e = adj_alloc(&s.v, n);
    if (e == cudaSuccess) e = adj_alloc(&s.C, n);
    if (e == cudaSuccess) e = adj_alloc(&s.F, n);
    return e;
}

void free_state(AdjState &s)
{
    for (void *p : {(void *)s.x, (void *)s.v, (void *)s.C, (void *)s.F})
        if (p) cudaFree(p);
    s = AdjState{};
}

cudaError_t copy_state(const AdjState &dst, const AdjState &src, size_t n, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(dst.x, src.x, n * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.v, src.v, n * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.C, src.C, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.F, src.F, n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    return e;
}

void free_engine(mpm_adjoint *a)
{
    if (!a) return;
    cudaSetDevice(a->device);
    if (a->stream) cudaStreamSynchronize(a->stream);
    free_state(a->init);
    free_state(a->ping[0]);
    free_state(a->ping[1]);
    for (auto &s : a->checkpoints) free_state(s);
    for (auto &s : a->tape) free_state(s);
    for (float4 *p : a->tape_s) cudaFree(p);
    for (float4 *p : a->tape_w) cudaFree(p);
    void *ptrs[] = {a->mark, a->lists, a->tile_scene, a->d_scenes, a->scene_of, a->liquid, a->status, a->vol, a->sum_s, a->sum_w, a->xb[0], a->xb[1],
                    a->vb[0], a->vb[1], a->xg, a->ub_s, a->Cb[0], a->Cb[1], a->Fb[0], a->Fb[1], a->Fg, a->ub_w, a->gv_s, a->gv_w,
                    a->param_grad, a->loss, a->target, a->final_x};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : a->ev)
        if (e) cudaEventDestroy(e);
    if (a->stream) cudaStreamDestroy(a->stream);
    delete a;
}

int err(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return host_error(code, buf);
}

#define ADJ_TRY(expr)                                                                                    \
    do {                                                                                                 \
        cudaError_t e__ = (expr);                                                                        \
        if (e__ != cudaSuccess) return err(MPM_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e__)); \
    } while (0)

AdjCtx make_adj_ctx(mpm_adjoint *a, const AdjState &in, const AdjState &out, float4 *sum_s, float4 *sum_w, int adj)
{
    AdjCtx c{};
    c.scenes = a->d_scenes;
    c.scene_of = a->scene_of;
    c.liquid = a->liquid;
    c.vol = a->vol;
    c.n = a->n;
    c.status = a->status;
    c.in = in;
    c.out = out;
    c.sum_s = sum_s;
    c.sum_w = sum_w;
    c.xb_next = a->xb[adj];
    c.vb_next = a->vb[adj];
    c.Cb_next = a->Cb[adj];
    c.Fb_next = a->Fb[adj];
    c.xb = a->xb[1 - adj];
    c.vb = a->vb[1 - adj];
    c.Cb = a->Cb[1 - adj];
    c.Fb = a->Fb[1 - adj];
    c.xg = a->xg;
    c.Fg = a->Fg;
    c.ub_s = a->ub_s;
    c.gv_s = a->gv_s;
    c.gv_w = a->gv_w;
    c.ub_w = a->ub_w;
    c.param_grad = a->param_grad;
    c.target = a->target;
    c.loss = a->loss;
    return c;
}

unsigned blocks(uint32_t n) { return std::max(1u, (n + ADJ_THREADS - 1) / ADJ_THREADS); }

// One forward substep from `in` to `out` with the sums in (ss, sw).
// The clearing-tile marks of substep k (its input positions).
uint8_t *marks_of(mpm_adjoint *a, uint32_t k) { return a->mark + (size_t)k * a->n_tiles; }

// The marked-tile list of substep k.
uint32_t *list_of(mpm_adjoint *a, uint32_t k) { return a->lists + (size_t)k * (a->n_tiles + 1u); }

// Lists the marked tiles of substep k.
void compact_marks(mpm_adjoint *a, uint32_t k)
{
    cudaMemsetAsync(list_of(a, k), 0, sizeof(uint32_t), a->stream);
    k_adj_compact<<<blocks(a->n_tiles), COMPACT_THREADS, 0, a->stream>>>(marks_of(a, k), a->n_tiles, list_of(a, k));
}

// Zeroes the node arrays over the marked tiles of substep k (NULL arrays are skipped).
void clear_marked(mpm_adjoint *a, uint32_t k, float4 *x, float4 *y, float2 *z)
{
    k_adj_clear<<<a->clear_ctas, ADJ_TILE * ADJ_TILE, 0, a->stream>>>(a->d_scenes, a->tile_scene, list_of(a, k), x, y,
                                                                        z);
}

// One forward substep k from `in` into `out`, its node sums in ss / sw: they
// are zeroed over the substep's marked tiles first, and the new positions
// mark substep k + 1's tiles (adding to the marks when a segment is
// recomputed: float atomics may move a position by its last bits).
cudaError_t forward_substep(mpm_adjoint *a, uint32_t k, const AdjState &in, const AdjState &out, float4 *ss, float4 *sw,
                            bool run_g2p = true)
{
    clear_marked(a, k, ss, sw, nullptr);
    AdjCtx c = make_adj_ctx(a, in, out, ss, sw, 0);
    c.mark_out = marks_of(a, k + 1);
    k_adj_p2g<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(c);
    if (run_g2p) {
        k_adj_grid_fwd<<<a->clear_ctas, ADJ_TILE * ADJ_TILE, 0, a->stream>>>(c, a->tile_scene, list_of(a, k));
        k_adj_g2p<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(c);
        compact_marks(a, k + 1);
    }
    return cudaGetLastError();
}

int check_status(mpm_adjoint *a, const char *what)
{
    uint32_t st = 0;
    ADJ_TRY(cudaMemcpyAsync(&st, a->status, sizeof st, cudaMemcpyDeviceToHost, a->stream));
    ADJ_TRY(cudaStreamSynchronize(a->stream));
    if (st != 0u)
        return err(MPM_ERR_STATE, "%s stopped: %s%s%s", what, (st & ADJ_ERR_STENCIL) ? "a particle left the grid; " : "",
                   (st & ADJ_ERR_DETERMINANT) ? "a deformation gradient lost its positive determinant; " : "",
                   (st & ADJ_ERR_NONFINITE) ? "a non-finite value appeared" : "");
    return MPM_OK;
}

}  // namespace

extern "C" {

int mpma_create(const mpm_config *configs, uint32_t scene_count, const uint32_t *particle_counts,
                const float *packed_particles, const float *gravity_xy, mpm_adjoint **out)
{
    host_clear_error();
    if (!configs || !particle_counts || !packed_particles || !gravity_xy || !out)
        return err(MPM_ERR_INVALID_ARGUMENT, "configs, particle_counts, packed_particles, gravity_xy and out must not be NULL");
    *out = nullptr;
    if (scene_count < 1) return err(MPM_ERR_INVALID_ARGUMENT, "a batch needs at least one scene");
    std::vector<AdjScene> scenes(scene_count);
    std::vector<uint32_t> scene_of, liquid;
    std::vector<float> vol;
    std::vector<float2> x, v;
    std::vector<float4> C, F;
    uint64_t total = 0, nodes = 0;
    std::vector<uint32_t> tile_scene;  // per clearing tile
    for (uint32_t k = 0; k < scene_count; ++k) {
        const mpm_config &cfg = configs[k];
        if (cfg.cells_x < 1 || cfg.cells_y < 1 || cfg.cells_x > 65536 || cfg.cells_y > 65536 || !(cfg.cell_size > 0.f))
            return err(MPM_ERR_INVALID_ARGUMENT, "scene %u: invalid grid", k);
        AdjScene &S = scenes[k];
        S.n = particle_counts[k];
        S.p_base = (uint32_t)total;
        S.node_base = (uint32_t)nodes;
        S.node_w = cfg.cells_x + 3;
        S.cells_x = cfg.cells_x;
        S.cells_y = cfg.cells_y;
        S.dx = cfg.cell_size;
        S.inv_dx = 1.0f / cfg.cell_size;
        S.gs = (float)(4.0 / ((double)cfg.cell_size * cfg.cell_size));
        S.gx = gravity_xy[2 * k];
        S.gy = gravity_xy[2 * k + 1];
        S.domain_w = (float)((double)cfg.cells_x * cfg.cell_size);
        S.domain_h = (float)((double)cfg.cells_y * cfg.cell_size);
        S.solid_mass = cfg.particle_mass;
        S.wall_friction = cfg.wall_friction;
        bool have_liquid = false, have_solid = false;
        for (uint32_t j = 0; j < S.n; ++j) {
            const float *w = packed_particles + (size_t)(total + j) * MPM_PARTICLE_WORDS;
            uint32_t model;
            std::memcpy(&model, &w[13], 4);
            const bool liq = model == MODEL_WATER;
            if (!liq && model != MODEL_FIXED_COROTATED)
                return err(MPM_ERR_INVALID_ARGUMENT,
                           "scene %u particle %u: the adjoint takes Tait water and fixed-corotated solids only", k, j);
            if (liq) {
                if (!(w[18] > 0.f) || !(w[14] > 0.f) || !(w[16] > 0.f))
                    return err(MPM_ERR_INVALID_ARGUMENT, "scene %u particle %u: water needs a Tait exponent", k, j);
                if (!have_liquid) {
                    S.tait = w[14], S.rho = w[16], S.gamma = w[18];
                    have_liquid = true;
                } else if (w[14] != S.tait || w[16] != S.rho || w[18] != S.gamma) {
                    return err(MPM_ERR_INVALID_ARGUMENT, "scene %u: every water particle must share its material", k);
                }
            } else {
                if (!have_solid) {
                    S.lambda_s = w[14], S.mu_s = w[15];
                    have_solid = true;
                } else if (w[14] != S.lambda_s || w[15] != S.mu_s) {
                    return err(MPM_ERR_INVALID_ARGUMENT, "scene %u: every solid particle must share its material", k);
                }
            }
            x.push_back(make_float2(w[0], w[1]));
            v.push_back(make_float2(w[2], w[3]));
            C.push_back(make_float4(w[4], w[5], w[6], w[7]));
            F.push_back(make_float4(w[8], w[9], w[10], w[11]));
            vol.push_back(w[17]);
            scene_of.push_back(k);
            liquid.push_back(liq ? 1u : 0u);
        }
        total += S.n;
        nodes += (uint64_t)(cfg.cells_x + 3) * (cfg.cells_y + 3);
        S.tile_base = (uint32_t)tile_scene.size();
        S.tiles_x = (cfg.cells_x + 3 + ADJ_TILE - 1) / ADJ_TILE;
        tile_scene.insert(tile_scene.end(), (size_t)S.tiles_x * ((cfg.cells_y + 3 + ADJ_TILE - 1) / ADJ_TILE), k);
        if (total > 0x7fffffffull || nodes > 0x7fffffffull)
            return err(MPM_ERR_INVALID_ARGUMENT, "the batch exceeds the GPU index range");
    }
    int device = configs[0].device, count = 0;
    ADJ_TRY(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return err(MPM_ERR_INVALID_ARGUMENT, "device %d is not available", device);
    ADJ_TRY(cudaSetDevice(device));
    mpm_adjoint *a = new mpm_adjoint();
    a->device = device;
    a->n = (uint32_t)total;
    a->n_scenes = scene_count;
    a->n_nodes = (uint32_t)nodes;
    a->scenes = scenes;
    auto fail = [&](int code) {
        free_engine(a);
        return code;
    };
#define ADJ_ALLOC(ptr, cnt)                                                                             \
    do {                                                                                                \
        cudaError_t e__ = adj_alloc(&(ptr), (cnt));                                                     \
        if (e__ != cudaSuccess) return fail(err(MPM_ERR_CUDA, "cudaMalloc(%s) failed: %s", #ptr, cudaGetErrorString(e__))); \
    } while (0)
    if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(err(MPM_ERR_CUDA, "cudaStreamCreate failed"));
    for (cudaEvent_t &e : a->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(err(MPM_ERR_CUDA, "cudaEventCreate failed"));
    const size_t n = a->n;
    ADJ_ALLOC(a->d_scenes, scene_count);
    ADJ_ALLOC(a->scene_of, n);
    ADJ_ALLOC(a->liquid, n);
    ADJ_ALLOC(a->status, 1);
    ADJ_ALLOC(a->vol, n);
    if (alloc_state(a->init, n) != cudaSuccess || alloc_state(a->ping[0], n) != cudaSuccess ||
        alloc_state(a->ping[1], n) != cudaSuccess)
        return fail(err(MPM_ERR_CUDA, "state allocation failed"));
    ADJ_ALLOC(a->sum_s, nodes);
    ADJ_ALLOC(a->sum_w, nodes);
    for (int b = 0; b < 2; ++b) {
        ADJ_ALLOC(a->xb[b], n);
        ADJ_ALLOC(a->vb[b], n);
        ADJ_ALLOC(a->Cb[b], n);
        ADJ_ALLOC(a->Fb[b], n);
    }
    ADJ_ALLOC(a->xg, n);
    ADJ_ALLOC(a->Fg, n);
    ADJ_ALLOC(a->ub_s, nodes);
    ADJ_ALLOC(a->ub_w, nodes);
    ADJ_ALLOC(a->gv_s, nodes);
    ADJ_ALLOC(a->gv_w, nodes);
    ADJ_ALLOC(a->param_grad, 3 * (size_t)scene_count);
    ADJ_ALLOC(a->loss, scene_count);
    ADJ_ALLOC(a->target, n);
    ADJ_ALLOC(a->final_x, n);
    a->n_tiles = (uint32_t)tile_scene.size();
    ADJ_ALLOC(a->tile_scene, tile_scene.size());
#undef ADJ_ALLOC
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            return fail(err(MPM_ERR_CUDA, "device query failed"));
        a->clear_ctas = (unsigned)std::max<size_t>(1, std::min<size_t>(tile_scene.size(), (size_t)sms * 8));
    }
    bool ok = cudaMemcpy(a->d_scenes, scenes.data(), scene_count * sizeof(AdjScene), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->scene_of, scene_of.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->liquid, liquid.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->vol, vol.data(), n * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->init.x, x.data(), n * sizeof(float2), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->init.v, v.data(), n * sizeof(float2), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->init.C, C.data(), n * sizeof(float4), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(a->init.F, F.data(), n * sizeof(float4), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemset(a->status, 0, sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMemcpy(a->tile_scene, tile_scene.data(), tile_scene.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) return fail(err(MPM_ERR_CUDA, "upload failed"));
    *out = a;
    return MPM_OK;
}

int mpma_set_parameters(mpm_adjoint *a, const float *parameters)
{
    host_clear_error();
    if (!a || !parameters) return err(MPM_ERR_INVALID_ARGUMENT, "engine and parameters must not be NULL");
    for (uint32_t k = 0; k < a->n_scenes; ++k) {
        const float *p = parameters + 3 * k;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || p[0] < 0.f)
            return err(MPM_ERR_INVALID_ARGUMENT, "scene %u: parameters must be finite", k);
        a->scenes[k].tait = p[0];
        a->scenes[k].lambda_s = p[1];
        a->scenes[k].mu_s = p[2];
    }
    ADJ_TRY(cudaSetDevice(a->device));
    ADJ_TRY(cudaMemcpy(a->d_scenes, a->scenes.data(), a->n_scenes * sizeof(AdjScene), cudaMemcpyHostToDevice));
    a->forward_done = false;
    return MPM_OK;
}

int mpma_get_parameters(mpm_adjoint *a, float *parameters)
{
    host_clear_error();
    if (!a || !parameters) return err(MPM_ERR_INVALID_ARGUMENT, "engine and parameters must not be NULL");
    for (uint32_t k = 0; k < a->n_scenes; ++k) {
        parameters[3 * k] = a->scenes[k].tait;
        parameters[3 * k + 1] = a->scenes[k].lambda_s;
        parameters[3 * k + 2] = a->scenes[k].mu_s;
    }
    return MPM_OK;
}

int mpma_set_velocities(mpm_adjoint *a, const float *velocities)
{
    host_clear_error();
    if (!a || !velocities) return err(MPM_ERR_INVALID_ARGUMENT, "engine and velocities must not be NULL");
    ADJ_TRY(cudaSetDevice(a->device));
    ADJ_TRY(cudaMemcpy(a->init.v, velocities, (size_t)a->n * sizeof(float2), cudaMemcpyHostToDevice));
    a->forward_done = false;
    return MPM_OK;
}

int mpma_forward(mpm_adjoint *a, uint32_t substeps, const float *dts, uint32_t checkpoint_every,
                 const float *targets, double *loss)
{
    host_clear_error();
    if (!a || !dts || !targets) return err(MPM_ERR_INVALID_ARGUMENT, "engine, dts and targets must not be NULL");
    if (substeps < 1) return err(MPM_ERR_INVALID_ARGUMENT, "substeps must be positive");
    if (checkpoint_every < 1 || checkpoint_every > 1024)
        return err(MPM_ERR_INVALID_ARGUMENT, "checkpoint_every must lie in [1, 1024]");
    for (uint32_t k = 0; k < a->n_scenes; ++k) {
        if (!(dts[k] > 0.f) || !std::isfinite(dts[k])) return err(MPM_ERR_INVALID_ARGUMENT, "scene %u: dt must be positive", k);
        a->scenes[k].dt = dts[k];
    }
    ADJ_TRY(cudaSetDevice(a->device));
    ADJ_TRY(cudaMemcpy(a->d_scenes, a->scenes.data(), a->n_scenes * sizeof(AdjScene), cudaMemcpyHostToDevice));
    ADJ_TRY(cudaMemcpy(a->target, targets, (size_t)a->n * sizeof(float2), cudaMemcpyHostToDevice));
    const uint32_t n_check = (substeps + checkpoint_every - 1) / checkpoint_every;
    if (a->checkpoints.size() != n_check || a->every != checkpoint_every) {
        for (auto &s : a->checkpoints) free_state(s);
        for (auto &s : a->tape) free_state(s);
        for (float4 *p : a->tape_s) cudaFree(p);
        for (float4 *p : a->tape_w) cudaFree(p);
        a->checkpoints.assign(n_check, AdjState{});
        a->tape.assign(checkpoint_every, AdjState{});
        a->tape_s.assign(checkpoint_every, nullptr);
        a->tape_w.assign(checkpoint_every, nullptr);
        for (auto &s : a->checkpoints)
            if (alloc_state(s, a->n) != cudaSuccess) return err(MPM_ERR_CUDA, "checkpoint allocation failed");
        for (uint32_t j = 0; j < checkpoint_every; ++j) {
            if (alloc_state(a->tape[j], a->n) != cudaSuccess || adj_alloc(&a->tape_s[j], a->n_nodes) != cudaSuccess ||
                adj_alloc(&a->tape_w[j], a->n_nodes) != cudaSuccess)
                return err(MPM_ERR_CUDA, "recompute tape allocation failed");
        }
    }
    a->steps = substeps;
    a->every = checkpoint_every;
    const size_t marks = ((size_t)substeps + 1) * a->n_tiles;
    if (a->mark_count < marks) {
        cudaFree(a->mark);
        a->mark = nullptr;
        a->mark_count = 0;
        cudaFree(a->lists);
        a->lists = nullptr;
        if (adj_alloc(&a->mark, marks) != cudaSuccess ||
            adj_alloc(&a->lists, ((size_t)substeps + 1) * (a->n_tiles + 1u)) != cudaSuccess)
            return err(MPM_ERR_CUDA, "tile mark allocation failed");
        a->mark_count = marks;
    }
    ADJ_TRY(cudaMemsetAsync(a->mark, 0, marks, a->stream));
    ADJ_TRY(cudaMemsetAsync(a->status, 0, sizeof(uint32_t), a->stream));
    ADJ_TRY(cudaMemsetAsync(a->loss, 0, a->n_scenes * sizeof(double), a->stream));
    ADJ_TRY(cudaEventRecord(a->ev[0], a->stream));
    int cur = 0;
    a->taped = n_check == 1;
    if (a->taped) {
        // one segment: the forward runs on the recompute tape itself (every
        // substep's input state and node sums stay in HBM), so the backward
        // pass recomputes nothing; the final state lands in ping[0]
        ADJ_TRY(copy_state(a->tape[0], a->init, a->n, a->stream));
        k_adj_mark<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(
            make_adj_ctx(a, a->tape[0], a->tape[0], nullptr, nullptr, 0), marks_of(a, 0));
        compact_marks(a, 0);
        for (uint32_t k = 0; k < substeps; ++k)
            ADJ_TRY(forward_substep(a, k, a->tape[k], k + 1 < substeps ? a->tape[k + 1] : a->ping[0], a->tape_s[k],
                                    a->tape_w[k]));
    } else {
        ADJ_TRY(copy_state(a->ping[0], a->init, a->n, a->stream));
        k_adj_mark<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(
            make_adj_ctx(a, a->ping[0], a->ping[0], nullptr, nullptr, 0), marks_of(a, 0));
        compact_marks(a, 0);
        for (uint32_t k = 0; k < substeps; ++k) {
            if (k % checkpoint_every == 0)
                ADJ_TRY(copy_state(a->checkpoints[k / checkpoint_every], a->ping[cur], a->n, a->stream));
            ADJ_TRY(forward_substep(a, k, a->ping[cur], a->ping[1 - cur], a->sum_s, a->sum_w));
            cur = 1 - cur;
        }
    }
    ADJ_TRY(cudaEventRecord(a->ev[1], a->stream));
    a->final_buffer = cur;
    const AdjCtx c = make_adj_ctx(a, a->ping[cur], a->ping[cur], a->sum_s, a->sum_w, 0);
    k_adj_loss<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(c);
    ADJ_TRY(cudaGetLastError());
    ADJ_TRY(cudaMemcpyAsync(a->final_x, a->ping[cur].x, (size_t)a->n * sizeof(float2), cudaMemcpyDeviceToDevice,
                            a->stream));
    int rc = check_status(a, "the forward pass");
    if (rc != MPM_OK) return rc;
    ADJ_TRY(cudaEventElapsedTime(&a->forward_ms, a->ev[0], a->ev[1]));
    if (loss) ADJ_TRY(cudaMemcpy(loss, a->loss, a->n_scenes * sizeof(double), cudaMemcpyDeviceToHost));
    a->forward_done = true;
    return MPM_OK;
}

int mpma_backward(mpm_adjoint *a, float *grad_velocities, double *grad_parameters)
{
    host_clear_error();
    if (!a) return err(MPM_ERR_INVALID_ARGUMENT, "engine must not be NULL");
    if (!a->forward_done) return err(MPM_ERR_STATE, "backward needs a completed forward pass of the same inputs");
    ADJ_TRY(cudaSetDevice(a->device));
    ADJ_TRY(cudaMemsetAsync(a->param_grad, 0, 3 * a->n_scenes * sizeof(double), a->stream));
    ADJ_TRY(cudaEventRecord(a->ev[2], a->stream));
    int adj = 0;  // the adjoint of the current substep's outputs sits in buffer `adj` (seeded by the loss)
    const uint32_t K = a->every;
    for (int seg = (int)a->checkpoints.size() - 1; seg >= 0; --seg) {
        const uint32_t start = (uint32_t)seg * K, len = std::min(K, a->steps - start);
        if (!a->taped) ADJ_TRY(copy_state(a->tape[0], a->checkpoints[seg], a->n, a->stream));
        for (uint32_t j = 0; j < len && !a->taped; ++j)
            ADJ_TRY(forward_substep(a, start + j, a->tape[j], j + 1 < len ? a->tape[j + 1] : a->ping[0], a->tape_s[j],
                                    a->tape_w[j], j + 1 < len));
        for (int j = (int)len - 1; j >= 0; --j) {
            const uint32_t k = start + (uint32_t)j;
            clear_marked(a, k, a->ub_w, a->ub_s, nullptr);
            const AdjCtx c = make_adj_ctx(a, a->tape[j], a->tape[j], a->tape_s[j], a->tape_w[j], adj);
            k_adj_grid_fwd<<<a->clear_ctas, ADJ_TILE * ADJ_TILE, 0, a->stream>>>(c, a->tile_scene, list_of(a, k));
            k_adj_g2p_bwd<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(c);
            k_adj_grid_bwd<<<a->clear_ctas, ADJ_TILE * ADJ_TILE, 0, a->stream>>>(c, a->tile_scene, list_of(a, k));
            k_adj_p2g_bwd<<<blocks(a->n), ADJ_THREADS, 0, a->stream>>>(c);
            adj = 1 - adj;
        }
        ADJ_TRY(cudaGetLastError());
    }
    ADJ_TRY(cudaEventRecord(a->ev[3], a->stream));
    int rc = check_status(a, "the adjoint pass");
    if (rc != MPM_OK) return rc;
    ADJ_TRY(cudaEventElapsedTime(&a->backward_ms, a->ev[2], a->ev[3]));
    if (grad_velocities)
        ADJ_TRY(cudaMemcpy(grad_velocities, a->vb[adj], (size_t)a->n * sizeof(float2), cudaMemcpyDeviceToHost));
    if (grad_parameters)
        ADJ_TRY(cudaMemcpy(grad_parameters, a->param_grad, 3 * a->n_scenes * sizeof(double), cudaMemcpyDeviceToHost));
    return MPM_OK;
}

int mpma_read_positions(mpm_adjoint *a, float *positions)
{
    host_clear_error();
    if (!a || !positions) return err(MPM_ERR_INVALID_ARGUMENT, "engine and positions must not be NULL");
    if (!a->forward_done) return err(MPM_ERR_STATE, "no forward pass has completed");
    ADJ_TRY(cudaSetDevice(a->device));
    ADJ_TRY(cudaMemcpy(positions, a->final_x, (size_t)a->n * sizeof(float2), cudaMemcpyDeviceToHost));
    return MPM_OK;
}

int mpma_last_ms(mpm_adjoint *a, double *forward_ms, double *backward_ms)
{
    host_clear_error();
    if (!a) return err(MPM_ERR_INVALID_ARGUMENT, "engine must not be NULL");
    if (forward_ms) *forward_ms = a->forward_ms;
    if (backward_ms) *backward_ms = a->backward_ms;
    return MPM_OK;
}

void mpma_destroy(mpm_adjoint *a) { free_engine(a); }

}  // extern "C"
