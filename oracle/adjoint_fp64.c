/*
 * adjoint_fp64.c -- TEST INFRASTRUCTURE ONLY: the FP64 CPU adjoint that the
 * GPU adjoint (powder-play_b200/csrc/mpm_adjoint.cu) is checked against.
 *
 * The reference has no gradients, so this is the build's own statement of the
 * differentiable form in double precision: one scene of Tait water and
 * fixed-corotated solid particles, the MLS-MPM substep with the reference's
 * formulas for those models (stress of prepareParticle, the APIC P2G and G2P,
 * finishGridVelocity with the wall factors of applyWallCushion /
 * applyWallTangentialFriction, the liquid density-contrast acceleration, the
 * deformation update in (I + h C)^k increments, the liquid projection,
 * confinement; src/lib/mpm/kernels/shaders.ts:474-534, :808-963,
 * :1072-1211, :1438-1777, :2114-2421), the loss sum |x(T) - target|^2, and
 * its reverse-mode gradient with respect to the initial velocities and the
 * parameters (Tait pressure coefficient, solid lambda, solid mu) from a full
 * tape.  Non-smooth steps keep the forward's branch (confinement, wall
 * factors, the liquid determinant clamp, the increment count, the stencil
 * base), as the GPU adjoint does.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mpm_oracle.h"

#define WALL_CUSHION_CELLS 8.0
#define MAX_DEFORMATION_INCREMENT 0.25
#define MAX_DEFORMATION_SUBSTEPS 64.0

typedef struct { double a, b, c, d; } M2; /* row-major (00, 01, 10, 11) */

static double det2(M2 m) { return m.a * m.d - m.b * m.c; }
static M2 cof2(M2 m) { M2 r = {m.d, -m.c, -m.b, m.a}; return r; }
static M2 mul2(M2 x, M2 y) { M2 r = {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d}; return r; }
static M2 mulT2(M2 x, M2 y) /* x y^T */ { M2 r = {x.a * y.a + x.b * y.b, x.a * y.c + x.b * y.d, x.c * y.a + x.d * y.b, x.c * y.c + x.d * y.d}; return r; }
static M2 Tmul2(M2 x, M2 y) /* x^T y */ { M2 r = {x.a * y.a + x.c * y.c, x.a * y.b + x.c * y.d, x.b * y.a + x.d * y.c, x.b * y.b + x.d * y.d}; return r; }
static M2 add2(M2 x, M2 y) { M2 r = {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; return r; }
static M2 scale2(double s, M2 x) { M2 r = {s * x.a, s * x.b, s * x.c, s * x.d}; return r; }
static double dot2(M2 x, M2 y) { return x.a * y.a + x.b * y.b + x.c * y.c + x.d * y.d; }

/* polar rotation angle of F (det F > 0): (cos, sin) of atan2(F10 - F01, F00 + F11) */
static void polar_cs(M2 F, double *c, double *s)
{
    double a = F.a + F.d, b = F.c - F.b, r = sqrt(a * a + b * b);
    if (r > 0) { *c = a / r; *s = b / r; } else { *c = 1; *s = 0; }
}
static M2 rot2(double c, double s) { M2 r = {c, -s, s, c}; return r; }
static M2 angle_adjoint(M2 F, double phib, M2 Fb)
{
    double a = F.a + F.d, b = F.c - F.b, r2 = a * a + b * b;
    if (!(r2 > 0)) return Fb;
    double da = -b / r2 * phib, db = a / r2 * phib;
    Fb.a += da; Fb.b -= db; Fb.c += db; Fb.d += da;
    return Fb;
}

static double quad_w(double f, int k)
{
    if (k == 0) return 0.5 * (1.5 - f) * (1.5 - f);
    if (k == 1) return 0.75 - (f - 1.0) * (f - 1.0);
    return 0.5 * (f - 0.5) * (f - 0.5);
}
static double quad_dw(double f, int k)
{
    if (k == 0) return f - 1.5;
    if (k == 1) return -2.0 * (f - 1.0);
    return f - 0.5;
}

static double cushion_factor(double u, int coord, int extent)
{
    double cushion = fmin(WALL_CUSHION_CELLS, extent / 4.0);
    double dist = u < 0 ? coord : extent - coord;
    if (dist >= cushion) return 1.0;
    return fmin(fmax(dist / cushion, 0.0), 1.0);
}
static double friction_factor(int coord, int extent, double fr)
{
    if (fr <= 0) return 1.0;
    double dist = fmax(0.0, fmin((double)coord, (double)(extent - coord)));
    double cushion = fmin(WALL_CUSHION_CELLS, extent / 4.0);
    if (dist >= cushion) return 1.0;
    return 1.0 - fr * (1.0 - fmin(fmax(dist / cushion, 0.0), 1.0));
}

typedef struct {
    const orc_adj_scene *S;
    int32_t n, W, H, nodes;
} Ctx;

typedef struct {
    int bx, by;
    double fx, fy, wx[3], wy[3], dwx[3], dwy[3];
} Sten;

static int stencil(const Ctx *c, double x, double y, Sten *st)
{
    double gx = x / c->S->dx, gy = y / c->S->dx;
    if (!isfinite(gx) || !isfinite(gy)) return 0;
    st->bx = (int)floor(gx - 0.5);
    st->by = (int)floor(gy - 0.5);
    st->fx = gx - st->bx;
    st->fy = gy - st->by;
    if (st->bx < -1 || st->by < -1 || st->bx + 2 > c->S->cells_x + 1 || st->by + 2 > c->S->cells_y + 1) return 0;
    for (int k = 0; k < 3; ++k) {
        st->wx[k] = quad_w(st->fx, k);
        st->wy[k] = quad_w(st->fy, k);
        st->dwx[k] = quad_dw(st->fx, k);
        st->dwy[k] = quad_dw(st->fy, k);
    }
    return 1;
}
static int node_of(const Ctx *c, int ix, int iy) { return (iy + 1) * c->W + (ix + 1); }

/* stress of prepareParticle */
static M2 stress(const orc_adj_scene *S, int liquid, M2 F, double det)
{
    if (liquid) {
        double sigma = -S->tait * (pow(det, 1.0 - S->gamma) - det);
        M2 r = {sigma, 0, 0, sigma};
        return r;
    }
    double cs, sn;
    polar_cs(F, &cs, &sn);
    M2 D = add2(F, scale2(-1.0, rot2(cs, sn)));
    M2 s = scale2(2.0 * S->mu_s, mulT2(D, F));
    double vol = S->lambda_s * det * (det - 1.0);
    s.a += vol;
    s.d += vol;
    return s;
}

/* grid node velocity with wall factors D */
static void node_vel(const Ctx *c, const double *sum, int ix, int iy, double *u, double *D)
{
    const orc_adj_scene *S = c->S;
    D[0] = D[1] = 0;
    u[0] = u[1] = 0;
    if (!(sum[0] > 0)) return;
    double u0x = sum[1] / sum[0] + S->dt * S->gx, u0y = sum[2] / sum[0] + S->dt * S->gy;
    D[0] = cushion_factor(u0x, ix, S->cells_x) * friction_factor(iy, S->cells_y, S->wall_friction);
    D[1] = cushion_factor(u0y, iy, S->cells_y) * friction_factor(ix, S->cells_x, S->wall_friction);
    u[0] = u0x * D[0];
    u[1] = u0y * D[1];
}

/* one forward substep; sums: 4 doubles per node per channel (solid, water) */
static int p2g(const Ctx *c, const double *x, const double *v, const M2 *C, const M2 *F, const double *vol,
               const int32_t *liquid, double *ss, double *sw)
{
    const orc_adj_scene *S = c->S;
    memset(ss, 0, sizeof(double) * 4 * c->nodes);
    memset(sw, 0, sizeof(double) * 4 * c->nodes);
    for (int i = 0; i < c->n; ++i) {
        double det = det2(F[i]);
        if (!(det > 0)) return -1;
        M2 s = stress(S, liquid[i], F[i], det);
        double m = liquid[i] ? S->rho * vol[i] : S->solid_mass, vliq = liquid[i] ? vol[i] * det : 0;
        double scale = -S->dt * vol[i] * 4.0 / (S->dx * S->dx);
        M2 A = add2(scale2(m, C[i]), scale2(scale, s));
        Sten st;
        if (!stencil(c, x[2 * i], x[2 * i + 1], &st)) return -1;
        double *sum = liquid[i] ? sw : ss;
        for (int oy = 0; oy < 3; ++oy)
            for (int ox = 0; ox < 3; ++ox) {
                double w = st.wx[ox] * st.wy[oy], dpx = (ox - st.fx) * S->dx, dpy = (oy - st.fy) * S->dx;
                double *q = sum + 4 * node_of(c, st.bx + ox, st.by + oy);
                q[0] += w * m;
                q[1] += w * (m * v[2 * i] + A.a * dpx + A.b * dpy);
                q[2] += w * (m * v[2 * i + 1] + A.c * dpx + A.d * dpy);
                q[3] += w * vliq;
            }
    }
    return 0;
}

typedef struct {
    double vp[2];
    M2 B, Cn, T;
    double pm, pv, pdet, xn[2];
    int sub;
} G2p;

static int g2p_fwd(const Ctx *c, const double *ss, const double *sw, int liquid, const Sten *st, const double *x, M2 F0,
                   G2p *g)
{
    const orc_adj_scene *S = c->S;
    memset(g, 0, sizeof *g);
    for (int oy = 0; oy < 3; ++oy)
        for (int ox = 0; ox < 3; ++ox) {
            double w = st->wx[ox] * st->wy[oy], dpx = (ox - st->fx) * S->dx, dpy = (oy - st->fy) * S->dx;
            const double *sum = (liquid ? sw : ss) + 4 * node_of(c, st->bx + ox, st->by + oy);
            double u[2], D[2];
            node_vel(c, sum, st->bx + ox, st->by + oy, u, D);
            g->vp[0] += w * u[0];
            g->vp[1] += w * u[1];
            g->B.a += w * u[0] * dpx;
            g->B.b += w * u[0] * dpy;
            g->B.c += w * u[1] * dpx;
            g->B.d += w * u[1] * dpy;
            if (liquid) {
                g->pm += w * sum[0];
                g->pv += w * sum[3];
            }
        }
    g->pdet = det2(F0);
    if (liquid) {
        if (!(g->pm > 0) || !(g->pv > 0) || !(g->pdet > 0)) return -1;
        double rd = 1.0 - (g->pm / g->pv) * g->pdet / S->rho;
        g->vp[0] += S->dt * rd * S->gx;
        g->vp[1] += S->dt * rd * S->gy;
    }
    double gs = 4.0 / (S->dx * S->dx);
    g->Cn = scale2(gs, g->B);
    g->xn[0] = x[0] + S->dt * g->vp[0];
    g->xn[1] = x[1] + S->dt * g->vp[1];
    double row = fmax(fabs(g->Cn.a) + fabs(g->Cn.b), fabs(g->Cn.c) + fabs(g->Cn.d));
    double req = ceil(S->dt * row / MAX_DEFORMATION_INCREMENT);
    if (!isfinite(req) || req > MAX_DEFORMATION_SUBSTEPS) return -1;
    g->sub = req < 1 ? 1 : (int)req;
    for (;;) {
        double h = S->dt / g->sub;
        M2 U = {1 + h * g->Cn.a, h * g->Cn.b, h * g->Cn.c, 1 + h * g->Cn.d};
        M2 T = F0;
        for (int k = 0; k < g->sub; ++k) T = mul2(U, T);
        g->T = T;
        if (det2(T) > 0 || g->sub >= 64) break;
        g->sub = g->sub * 2 > 64 ? 64 : g->sub * 2;
    }
    return det2(g->T) > 0 ? 0 : -1;
}

static M2 project_liquid(M2 T)
{
    double cs, sn;
    polar_cs(T, &cs, &sn);
    double J = det2(T), sc = sqrt(fmin(fmax(J, 0.5), 2.0));
    return scale2(sc, rot2(cs, sn));
}

static void confine(double next, double vel, double maximum, double *pos, double *v)
{
    if (next < 0 || (next == 0 && vel < 0)) { *pos = 0; *v = 0; return; }
    if (next > maximum || (next == maximum && vel > 0)) { *pos = maximum; *v = 0; return; }
    *pos = next;
    *v = vel;
}

int orc_adjoint_run(const orc_adj_scene *S, int32_t n, const double *x0, const double *v0, const double *C0,
                    const double *F0, const double *vol, const int32_t *liquid, const double *target, int32_t steps,
                    double *loss, double *grad_v0, double *grad_params, double *x_out)
{
    Ctx c = {S, n, S->cells_x + 3, S->cells_y + 3, (S->cells_x + 3) * (S->cells_y + 3)};
    const size_t N = (size_t)n, T1 = (size_t)steps + 1;
    double *xs = malloc(sizeof(double) * 2 * N * T1), *vs = malloc(sizeof(double) * 2 * N * T1);
    M2 *Cs = malloc(sizeof(M2) * N * T1), *Fs = malloc(sizeof(M2) * N * T1);
    double *ss = malloc(sizeof(double) * 4 * c.nodes * steps), *sw = malloc(sizeof(double) * 4 * c.nodes * steps);
    double *xb = calloc(2 * N, sizeof(double)), *vb = calloc(2 * N, sizeof(double));
    M2 *Cb = calloc(N, sizeof(M2)), *Fb = calloc(N, sizeof(M2));
    double *xb2 = calloc(2 * N, sizeof(double)), *vb2 = calloc(2 * N, sizeof(double));
    M2 *Cb2 = calloc(N, sizeof(M2)), *Fb2 = calloc(N, sizeof(M2));
    double *ubs = calloc(2 * (size_t)c.nodes, sizeof(double)), *ubw = calloc(4 * (size_t)c.nodes, sizeof(double));
    double *xg = calloc(2 * N, sizeof(double));
    M2 *Fg = calloc(N, sizeof(M2));
    int rc = 0;
    if (!xs || !vs || !Cs || !Fs || !ss || !sw || !xb || !vb || !Cb || !Fb || !xb2 || !vb2 || !Cb2 || !Fb2 || !ubs ||
        !ubw || !xg || !Fg) {
        rc = -2;
        goto done;
    }
    memcpy(xs, x0, sizeof(double) * 2 * N);
    memcpy(vs, v0, sizeof(double) * 2 * N);
    for (size_t i = 0; i < N; ++i) {
        M2 cc = {C0[4 * i], C0[4 * i + 1], C0[4 * i + 2], C0[4 * i + 3]};
        M2 ff = {F0[4 * i], F0[4 * i + 1], F0[4 * i + 2], F0[4 * i + 3]};
        Cs[i] = cc;
        Fs[i] = ff;
    }
    const double gs = 4.0 / (S->dx * S->dx);
    const double dw = S->cells_x * S->dx, dh = S->cells_y * S->dx;
    /* forward with a full tape */
    for (int k = 0; k < steps; ++k) {
        const double *x = xs + 2 * N * k, *v = vs + 2 * N * k;
        const M2 *C = Cs + N * k, *F = Fs + N * k;
        double *sk = ss + 4 * (size_t)c.nodes * k, *wk = sw + 4 * (size_t)c.nodes * k;
        if (p2g(&c, x, v, C, F, vol, liquid, sk, wk) != 0) { rc = -1; goto done; }
        for (size_t i = 0; i < N; ++i) {
            Sten st;
            G2p g;
            if (!stencil(&c, x[2 * i], x[2 * i + 1], &st) ||
                g2p_fwd(&c, sk, wk, liquid[i], &st, x + 2 * i, F[i], &g) != 0) { rc = -1; goto done; }
            double *xo = xs + 2 * N * (k + 1) + 2 * i, *vo = vs + 2 * N * (k + 1) + 2 * i;
            confine(g.xn[0], g.vp[0], dw, &xo[0], &vo[0]);
            confine(g.xn[1], g.vp[1], dh, &xo[1], &vo[1]);
            Cs[N * (k + 1) + i] = g.Cn;
            Fs[N * (k + 1) + i] = liquid[i] ? project_liquid(g.T) : g.T;
        }
    }
    /* loss and its seed */
    double L = 0;
    const double *xT = xs + 2 * N * steps;
    for (size_t i = 0; i < 2 * N; ++i) {
        double d = xT[i] - target[i];
        L += d * d;
        xb[i] = 2 * d;
    }
    if (x_out) memcpy(x_out, xT, sizeof(double) * 2 * N);
    grad_params[0] = grad_params[1] = grad_params[2] = 0;
    /* reverse */
    for (int k = steps - 1; k >= 0; --k) {
        const double *x = xs + 2 * N * k, *v = vs + 2 * N * k;
        const M2 *C = Cs + N * k, *F = Fs + N * k;
        const double *sk = ss + 4 * (size_t)c.nodes * k, *wk = sw + 4 * (size_t)c.nodes * k;
        memset(ubs, 0, sizeof(double) * 2 * c.nodes);
        memset(ubw, 0, sizeof(double) * 4 * c.nodes);
        /* G2P adjoint */
        for (size_t i = 0; i < N; ++i) {
            Sten st;
            G2p g;
            stencil(&c, x[2 * i], x[2 * i + 1], &st);
            g2p_fwd(&c, sk, wk, liquid[i], &st, x + 2 * i, F[i], &g);
            double cx, vx_, cy, vy_;
            confine(g.xn[0], g.vp[0], dw, &cx, &vx_);
            confine(g.xn[1], g.vp[1], dh, &cy, &vy_);
            int fx = cx == g.xn[0], fy = cy == g.xn[1];
            double xbi[2] = {fx ? xb[2 * i] : 0, fy ? xb[2 * i + 1] : 0};
            double vpb[2] = {fx ? vb[2 * i] + S->dt * xb[2 * i] : 0, fy ? vb[2 * i + 1] + S->dt * xb[2 * i + 1] : 0};
            M2 Tb = Fb[i];
            if (liquid[i]) {
                double cs, sn;
                polar_cs(g.T, &cs, &sn);
                double J = det2(g.T), Jc = fmin(fmax(J, 0.5), 2.0), sc = sqrt(Jc);
                M2 Fo = Fb[i];
                double scb = Fo.a * cs - Fo.b * sn + Fo.c * sn + Fo.d * cs;
                double phib = sc * (Fo.a * -sn + Fo.b * -cs + Fo.c * cs + Fo.d * -sn);
                double Jb = J == Jc ? scb * 0.5 / sc : 0;
                M2 zero = {0, 0, 0, 0};
                Tb = add2(zero, scale2(Jb, cof2(g.T)));
                Tb = angle_adjoint(g.T, phib, Tb);
            }
            double h = S->dt / g.sub;
            M2 U = {1 + h * g.Cn.a, h * g.Cn.b, h * g.Cn.c, 1 + h * g.Cn.d};
            M2 G = Tb, Ub = {0, 0, 0, 0};
            for (int j = g.sub - 1; j >= 0; --j) {
                M2 Fj = F[i];
                for (int q = 0; q < j; ++q) Fj = mul2(U, Fj);
                Ub = add2(Ub, mulT2(G, Fj));
                G = Tmul2(U, G);
            }
            M2 Fgi = G;
            M2 Cnb = add2(Cb[i], scale2(h, Ub));
            M2 Bb = scale2(gs, Cnb);
            double pmb = 0, pvb = 0;
            if (liquid[i]) {
                double rdb = S->dt * (S->gx * vpb[0] + S->gy * vpb[1]);
                double ld = g.pm / g.pv, ldb = -rdb * g.pdet / S->rho, pdetb = -rdb * ld / S->rho;
                Fgi = add2(Fgi, scale2(pdetb, cof2(F[i])));
                pmb = ldb / g.pv;
                pvb = -ldb * g.pm / (g.pv * g.pv);
            }
            for (int oy = 0; oy < 3; ++oy)
                for (int ox = 0; ox < 3; ++ox) {
                    double w = st.wx[ox] * st.wy[oy], dpx = (ox - st.fx) * S->dx, dpy = (oy - st.fy) * S->dx;
                    int nd = node_of(&c, st.bx + ox, st.by + oy);
                    const double *sum = (liquid[i] ? wk : sk) + 4 * nd;
                    double u[2], D[2];
                    node_vel(&c, sum, st.bx + ox, st.by + oy, u, D);
                    double ubx = w * (vpb[0] + Bb.a * dpx + Bb.b * dpy), uby = w * (vpb[1] + Bb.c * dpx + Bb.d * dpy);
                    if (liquid[i]) {
                        ubw[4 * nd] += ubx;
                        ubw[4 * nd + 1] += uby;
                        ubw[4 * nd + 2] += w * pmb;
                        ubw[4 * nd + 3] += w * pvb;
                    } else {
                        ubs[2 * nd] += ubx;
                        ubs[2 * nd + 1] += uby;
                    }
                    double gwx = st.dwx[ox] * st.wy[oy] / S->dx, gwy = st.wx[ox] * st.dwy[oy] / S->dx;
                    double sval = u[0] * (vpb[0] + Bb.a * dpx + Bb.b * dpy) + u[1] * (vpb[1] + Bb.c * dpx + Bb.d * dpy);
                    if (liquid[i]) sval += pmb * sum[0] + pvb * sum[3];
                    xbi[0] += gwx * sval - w * (u[0] * Bb.a + u[1] * Bb.c);
                    xbi[1] += gwy * sval - w * (u[0] * Bb.b + u[1] * Bb.d);
                }
            xg[2 * i] = xbi[0];
            xg[2 * i + 1] = xbi[1];
            Fg[i] = Fgi;
        }
        /* grid + P2G adjoint */
        for (size_t i = 0; i < N; ++i) {
            double det = det2(F[i]);
            M2 s = stress(S, liquid[i], F[i], det);
            double m = liquid[i] ? S->rho * vol[i] : S->solid_mass, vliq = liquid[i] ? vol[i] * det : 0;
            double scale = -S->dt * vol[i] * gs;
            M2 A = add2(scale2(m, C[i]), scale2(scale, s));
            Sten st;
            stencil(&c, x[2 * i], x[2 * i + 1], &st);
            double xbi[2] = {xg[2 * i], xg[2 * i + 1]}, vbi[2] = {0, 0}, vliqb = 0;
            M2 Ab = {0, 0, 0, 0};
            for (int oy = 0; oy < 3; ++oy)
                for (int ox = 0; ox < 3; ++ox) {
                    double w = st.wx[ox] * st.wy[oy], dpx = (ox - st.fx) * S->dx, dpy = (oy - st.fy) * S->dx;
                    int ix = st.bx + ox, iy = st.by + oy, nd = node_of(&c, ix, iy);
                    const double *sum = (liquid[i] ? wk : sk) + 4 * nd;
                    double ub[2], lmb = 0, lvb = 0;
                    if (liquid[i]) {
                        ub[0] = ubw[4 * nd];
                        ub[1] = ubw[4 * nd + 1];
                        lmb = ubw[4 * nd + 2];
                        lvb = ubw[4 * nd + 3];
                    } else {
                        ub[0] = ubs[2 * nd];
                        ub[1] = ubs[2 * nd + 1];
                    }
                    double Mb = lmb, Qxb = 0, Qyb = 0;
                    if (sum[0] > 0) {
                        double u[2], D[2];
                        node_vel(&c, sum, ix, iy, u, D);
                        double udx = D[0] * ub[0], udy = D[1] * ub[1];
                        Qxb = udx / sum[0];
                        Qyb = udy / sum[0];
                        Mb -= (udx * sum[1] + udy * sum[2]) / (sum[0] * sum[0]);
                    }
                    vbi[0] += w * m * Qxb;
                    vbi[1] += w * m * Qyb;
                    Ab.a += w * Qxb * dpx;
                    Ab.b += w * Qxb * dpy;
                    Ab.c += w * Qyb * dpx;
                    Ab.d += w * Qyb * dpy;
                    if (liquid[i]) vliqb += w * lvb;
                    double qx = m * v[2 * i] + A.a * dpx + A.b * dpy, qy = m * v[2 * i + 1] + A.c * dpx + A.d * dpy;
                    double sval = Mb * m + Qxb * qx + Qyb * qy + (liquid[i] ? lvb * vliq : 0);
                    double gwx = st.dwx[ox] * st.wy[oy] / S->dx, gwy = st.wx[ox] * st.dwy[oy] / S->dx;
                    xbi[0] += gwx * sval - w * (A.a * Qxb + A.c * Qyb);
                    xbi[1] += gwy * sval - w * (A.b * Qxb + A.d * Qyb);
                }
            M2 Cbi = scale2(m, Ab), sb = scale2(scale, Ab);
            M2 Fbi = Fg[i];
            if (liquid[i]) Fbi = add2(Fbi, scale2(vliqb * vol[i], cof2(F[i])));
            if (liquid[i]) {
                double sigb = sb.a + sb.d;
                double pw = pow(det, -S->gamma);
                double dsig = -S->tait * ((1.0 - S->gamma) * pw - 1.0);
                Fbi = add2(Fbi, scale2(sigb * dsig, cof2(F[i])));
                grad_params[0] += sigb * -(det * pw - det);
            } else {
                double cs, sn;
                polar_cs(F[i], &cs, &sn);
                M2 R = rot2(cs, sn), D = add2(F[i], scale2(-1.0, R));
                grad_params[2] += 2.0 * dot2(sb, mulT2(D, F[i]));
                double trb = sb.a + sb.d;
                grad_params[1] += trb * det * (det - 1.0);
                Fbi = add2(Fbi, scale2(trb * S->lambda_s * (2.0 * det - 1.0), cof2(F[i])));
                double m2 = 2.0 * S->mu_s;
                M2 sym = {2 * sb.a, sb.b + sb.c, sb.c + sb.b, 2 * sb.d};
                Fbi = add2(Fbi, scale2(m2, add2(mul2(sym, F[i]), scale2(-1.0, Tmul2(sb, R)))));
                M2 Rb = scale2(-m2, mul2(sb, F[i]));
                double phib = Rb.a * -sn + Rb.b * -cs + Rb.c * cs + Rb.d * -sn;
                Fbi = angle_adjoint(F[i], phib, Fbi);
            }
            xb2[2 * i] = xbi[0];
            xb2[2 * i + 1] = xbi[1];
            vb2[2 * i] = vbi[0];
            vb2[2 * i + 1] = vbi[1];
            Cb2[i] = Cbi;
            Fb2[i] = Fbi;
        }
        memcpy(xb, xb2, sizeof(double) * 2 * N);
        memcpy(vb, vb2, sizeof(double) * 2 * N);
        memcpy(Cb, Cb2, sizeof(M2) * N);
        memcpy(Fb, Fb2, sizeof(M2) * N);
    }
    *loss = L;
    memcpy(grad_v0, vb, sizeof(double) * 2 * N);
done:
    free(xs); free(vs); free(Cs); free(Fs); free(ss); free(sw);
    free(xb); free(vb); free(Cb); free(Fb); free(xb2); free(vb2); free(Cb2); free(Fb2);
    free(ubs); free(ubw); free(xg); free(Fg);
    return rc;
}
