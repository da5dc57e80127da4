/*
 * mpm_oracle.c -- CPU FP64 restatement of the reference CPU MLS-MPM step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; never shipped).
 * Every function cites the reference function it restates, by path:line in
 * 7korobi/powder-play.  Compile with -ffp-contract=off so that, like the
 * JavaScript original, no multiply-add is fused.
 */
#include "mpm_oracle.h"

#include <math.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* constants: src/lib/mpm/reference/solver.ts:266-283, materials.ts:40-53 */
#define WALL_CUSHION_CELLS 8.0
#define MIN_LIQUID_DETERMINANT 0.5
#define MAX_LIQUID_DETERMINANT 2.0
#define MIN_POWDER_DETERMINANT 0.5
#define MIN_NEO_HOOKEAN_STRETCH 0.05
#define MAX_NEO_HOOKEAN_STRETCH 20.0
#define MAX_DEFORMATION_INCREMENT 0.25
#define MAX_DEFORMATION_SUBSTEPS 64
#define DEFAULT_BONDED_TRIANGLE_STIFFNESS 0.35
#define BONDED_TRIANGLE_SOLVER_ITERATIONS 2
#define TRIANGLE_CONTACT_SKIN_CELLS 0.1
#define TRIANGLE_CONTACT_IMPULSE_RELAXATION 0.25
#define TRIANGLE_FIELD_BAND_CELLS 2.0
#define GRID_CONTACT_REACH_CELLS 0.75
#define LIQUID_CONTACT_SEPARATION_FRACTION 0.25
#define LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER 1.0
#define LIQUID_CONTACT_RELAXATION_SECONDS 0.05
#define LIQUID_STABLE_ORDER_EPSILON 1e-3
#define TRIANGLE_FLUID_TANGENTIAL_DRAG_RATE 4.0
#define SNOW_COMPRESSION_YIELD 0.025
#define SNOW_STRETCH_YIELD 0.0075
#define SNOW_HARDENING 10.0
#define SNOW_MIN_PLASTIC_VOLUME 0.6
#define SNOW_MAX_PLASTIC_VOLUME 20.0
#define SNOW_MAX_HARDENING_EXPONENT 20.0

typedef struct { double m00, m01, m10, m11; } mat2;
typedef struct { double x, y; } vec2;

typedef struct {
    jmp_buf jump;
    char *err;
    int err_len;
} ctx_t;

static void fail(ctx_t *ctx, const char *fmt, ...)
{
    if (ctx->err && ctx->err_len > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->err, (size_t)ctx->err_len, fmt, ap);
        va_end(ap);
    }
    longjmp(ctx->jump, 1);
}

static int is_fin(double v) { return isfinite(v) != 0; }

static void assert_finite(ctx_t *ctx, double v, const char *name)
{
    if (!is_fin(v)) fail(ctx, "%s became non-finite", name);
}

static void assert_matrix_finite(ctx_t *ctx, mat2 m, const char *name)
{
    if (!is_fin(m.m00) || !is_fin(m.m01) || !is_fin(m.m10) || !is_fin(m.m11))
        fail(ctx, "%s became non-finite", name);
}

static double det2(mat2 m) { return m.m00 * m.m11 - m.m01 * m.m10; }

static mat2 mul2(mat2 l, mat2 r)
{
    mat2 o = {l.m00 * r.m00 + l.m01 * r.m10, l.m00 * r.m01 + l.m01 * r.m11,
              l.m10 * r.m00 + l.m11 * r.m10, l.m10 * r.m01 + l.m11 * r.m11};
    return o;
}

static mat2 scale2(mat2 m, double s)
{
    mat2 o = {m.m00 * s, m.m01 * s, m.m10 * s, m.m11 * s};
    return o;
}

static mat2 add2(mat2 a, mat2 b)
{
    mat2 o = {a.m00 + b.m00, a.m01 + b.m01, a.m10 + b.m10, a.m11 + b.m11};
    return o;
}

static mat2 transpose2(mat2 m)
{
    mat2 o = {m.m00, m.m10, m.m01, m.m11};
    return o;
}

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

/* ---------------------------------------------------------------- grid -- */

/* GridNode, src/lib/mpm/reference/solver.ts:131-151 */
typedef struct {
    int32_t x, y;
    double mass, mx, my, vx, vy;
    double w_mass, w_mx, w_my, w_vx, w_vy, w_vol;
    double o_mass, o_mx, o_my, o_vx, o_vy, o_vol;
} node_t;

/* TriangleContactField, src/lib/mpm/reference/solver.ts:164-172 */
typedef struct {
    int32_t body_start;
    int32_t key;
    double signed_distance;
    double nx, ny;
    double bary[3];
    double ix, iy;
} field_t;

/* Dense node store with generation stamps and an insertion-ordered active
 * list: DenseGridNodeStore, src/lib/mpm/reference/solver.ts:285-333. */
typedef struct {
    int64_t count;
    node_t *nodes;
    uint32_t *gen;
    uint32_t generation;
    int64_t *active;
    int64_t n_active;
    field_t *fields;
    uint32_t *field_gen;
    uint32_t field_generation;
} grid_t;

static void grid_begin(grid_t *g)
{
    g->n_active = 0;
    g->generation += 1;
    if (g->generation == 0) {
        memset(g->gen, 0, (size_t)g->count * sizeof(uint32_t));
        g->generation = 1;
    }
    g->field_generation += 1;
    if (g->field_generation == 0) {
        memset(g->field_gen, 0, (size_t)g->count * sizeof(uint32_t));
        g->field_generation = 1;
    }
}

static int grid_alloc(grid_t *g, int64_t count)
{
    memset(g, 0, sizeof(*g));
    g->count = count;
    g->nodes = (node_t *)malloc((size_t)count * sizeof(node_t));
    g->gen = (uint32_t *)calloc((size_t)count, sizeof(uint32_t));
    g->active = (int64_t *)malloc((size_t)count * sizeof(int64_t));
    g->fields = (field_t *)malloc((size_t)count * sizeof(field_t));
    g->field_gen = (uint32_t *)calloc((size_t)count, sizeof(uint32_t));
    return g->nodes && g->gen && g->active && g->fields && g->field_gen;
}

static void grid_free(grid_t *g)
{
    free(g->nodes);
    free(g->gen);
    free(g->active);
    free(g->fields);
    free(g->field_gen);
    memset(g, 0, sizeof(*g));
}

static node_t *grid_get(grid_t *g, int64_t key)
{
    if (key < 0 || key >= g->count) return NULL;
    return g->gen[key] == g->generation ? &g->nodes[key] : NULL;
}

static node_t *grid_get_or_create(grid_t *g, int64_t key, int32_t x, int32_t y)
{
    if (g->gen[key] != g->generation) {
        node_t *n = &g->nodes[key];
        memset(n, 0, sizeof(*n));
        n->x = x;
        n->y = y;
        g->gen[key] = g->generation;
        g->active[g->n_active++] = key;
        return n;
    }
    return &g->nodes[key];
}

static field_t *field_get(grid_t *g, int64_t key)
{
    if (key < 0 || key >= g->count) return NULL;
    return g->field_gen[key] == g->field_generation ? &g->fields[key] : NULL;
}

/* --------------------------------------------------------- validation -- */

typedef struct {
    double dt;
    int32_t cells_x, cells_y;
    double cell_size;
    double particle_mass, particle_volume;
    int32_t has_bond_rest_length;
    double bond_rest_length, bond_stiffness, bond_reference_dt;
    const orc_material *material;
    double gx, gy, wall_friction;
    double domain_w, domain_h, gradient_scale;
    int64_t node_width, node_count;
} vcfg_t;

/* validateMaterial, src/lib/mpm/reference/solver.ts:2063-2119 */
static void validate_material(ctx_t *ctx, const orc_material *m, const char *name)
{
    if (!is_fin(m->lambda)) fail(ctx, "%s.lambda must be a finite number", name);
    if (!is_fin(m->mu)) fail(ctx, "%s.mu must be a finite number", name);
    if (m->model < 0 || m->model > ORC_FIXED_COROTATED)
        fail(ctx, "%s.model must be 'neo-hookean', 'snow', 'water', 'oil', or 'powder'", name);
    if (!is_fin(m->lambda + 2 * m->mu))
        fail(ctx, "%s parameters are outside the supported numeric range", name);
    if (m->model == ORC_WATER || m->model == ORC_OIL) {
        if (m->tait && (!is_fin(m->exponent) || m->exponent <= 0))
            fail(ctx, "%s.equationOfState.exponent must be positive and finite.", name);
        if (!is_fin(m->density)) fail(ctx, "%s.density must be a finite number", name);
        if (m->lambda <= 0) fail(ctx, "%s.lambda must be greater than zero", name);
        if (m->mu != 0) fail(ctx, "%s.mu must be zero for a liquid material", name);
        if (m->density <= 0) fail(ctx, "%s.density must be greater than zero", name);
        return;
    }
    if (m->model == ORC_POWDER) {
        if (!is_fin(m->friction)) fail(ctx, "%s.frictionCoefficient must be a finite number", name);
        if (m->lambda < 0) fail(ctx, "%s.lambda must be non-negative", name);
        if (m->mu <= 0) fail(ctx, "%s.mu must be greater than zero", name);
        if (m->friction < 0) fail(ctx, "%s.frictionCoefficient must be non-negative", name);
        return;
    }
    if (m->lambda < 0) fail(ctx, "%s.lambda must be non-negative", name);
    if (m->mu <= 0) fail(ctx, "%s.mu must be greater than zero", name);
}

/* validateConfig, src/lib/mpm/reference/solver.ts:826-948 */
static void validate_config(ctx_t *ctx, const orc_material *mats, int32_t n_mats,
                            const orc_config *c, vcfg_t *v)
{
    if (c->material < 0 || c->material >= n_mats) fail(ctx, "material must be an object");
    v->material = &mats[c->material];
    validate_material(ctx, v->material, "material");
    v->dt = c->dt;
    v->cells_x = c->cells_x;
    v->cells_y = c->cells_y;
    v->cell_size = c->cell_size;
    v->particle_mass = c->particle_mass;
    v->particle_volume = c->particle_volume;
    v->has_bond_rest_length = c->has_bond_rest_length;
    v->bond_rest_length = c->bond_rest_length;
    v->bond_stiffness = c->bond_stiffness;
    v->bond_reference_dt = c->bond_reference_dt > 0 ? c->bond_reference_dt : c->dt;
    v->gx = c->gx;
    v->gy = c->gy;
    v->wall_friction = c->wall_friction;
    if (!is_fin(v->dt)) fail(ctx, "dt must be a finite number");
    if (!is_fin(v->cell_size)) fail(ctx, "grid.cellSize must be a finite number");
    if (!is_fin(v->particle_mass)) fail(ctx, "particleMass must be a finite number");
    if (!is_fin(v->particle_volume)) fail(ctx, "particleVolume must be a finite number");
    if (!is_fin(v->bond_stiffness)) fail(ctx, "bondStiffness must be a finite number");
    if (!is_fin(v->wall_friction)) fail(ctx, "wallFriction must be a finite number");
    if (!is_fin(v->gx) || !is_fin(v->gy)) fail(ctx, "gravity.x must be a finite number");
    if (v->dt <= 0) fail(ctx, "dt must be greater than zero");
    if (v->bond_reference_dt <= 0) fail(ctx, "bondReferenceDt must be greater than zero");
    if (v->cells_x < 1) fail(ctx, "grid.cellsX must be a positive safe integer");
    if (v->cells_y < 1) fail(ctx, "grid.cellsY must be a positive safe integer");
    v->node_width = (int64_t)v->cells_x + 3;
    v->node_count = v->node_width * ((int64_t)v->cells_y + 3);
    if (v->cell_size <= 0) fail(ctx, "grid.cellSize must be greater than zero");
    if (v->particle_mass <= 0) fail(ctx, "particleMass must be greater than zero");
    if (v->particle_volume <= 0) fail(ctx, "particleVolume must be greater than zero");
    if (v->has_bond_rest_length && (!is_fin(v->bond_rest_length) || v->bond_rest_length <= 0))
        fail(ctx, "bondRestLength must be greater than zero");
    if (v->bond_stiffness <= 0 || v->bond_stiffness > 1)
        fail(ctx, "bondStiffness must be greater than zero and at most one");
    if (v->wall_friction < 0 || v->wall_friction > 1)
        fail(ctx, "wallFriction must be between zero and one");
    v->domain_w = v->cells_x * v->cell_size;
    v->domain_h = v->cells_y * v->cell_size;
    double cs2 = v->cell_size * v->cell_size;
    v->gradient_scale = 4 / cs2;
    if (!is_fin(v->domain_w) || !is_fin(v->domain_h))
        fail(ctx, "grid dimensions produce a non-finite domain");
    if (!is_fin(cs2) || cs2 <= 0 || !is_fin(v->gradient_scale))
        fail(ctx, "grid.cellSize is outside the supported numeric range");
    if (!is_fin(v->particle_mass / v->particle_volume) || v->particle_mass / v->particle_volume <= 0 ||
        !is_fin(v->material->lambda + 2 * v->material->mu))
        fail(ctx, "mass and material parameters are outside the supported numeric range");
    if (!is_fin(-v->dt * v->particle_volume * v->gradient_scale))
        fail(ctx, "dt, particleVolume, and grid.cellSize produce a non-finite stress scale");
}

static const orc_material *particle_material(const orc_material *mats, int32_t n_mats,
                                             const orc_particle *p, const vcfg_t *v, ctx_t *ctx,
                                             int32_t index)
{
    if (p->material < 0) return v->material;
    if (p->material >= n_mats) fail(ctx, "particles[%d].material must be an object", index);
    return &mats[p->material];
}

/* validateParticles, src/lib/mpm/reference/solver.ts:950-1021 */
static void validate_particles(ctx_t *ctx, const orc_material *mats, int32_t n_mats,
                               const orc_particle *ps, int32_t n, const vcfg_t *v)
{
    for (int32_t i = 0; i < n; ++i) {
        const orc_particle *p = &ps[i];
        char name[64];
        if (!is_fin(p->px) || !is_fin(p->py)) fail(ctx, "particles[%d].position.x must be a finite number", i);
        if (!is_fin(p->vx) || !is_fin(p->vy)) fail(ctx, "particles[%d].velocity.x must be a finite number", i);
        if (!is_fin(p->c00) || !is_fin(p->c01) || !is_fin(p->c10) || !is_fin(p->c11))
            fail(ctx, "particles[%d].C.m00 must be a finite number", i);
        if (!is_fin(p->f00) || !is_fin(p->f01) || !is_fin(p->f10) || !is_fin(p->f11))
            fail(ctx, "particles[%d].F.m00 must be a finite number", i);
        const orc_material *m = particle_material(mats, n_mats, p, v, ctx, i);
        if (p->material >= 0) {
            snprintf(name, sizeof name, "particles[%d].material", i);
            validate_material(ctx, m, name);
        }
        if (p->volume > 0 || p->volume < 0 || !is_fin(p->volume)) {
            if (!is_fin(p->volume)) fail(ctx, "particles[%d].volume must be a finite number", i);
            if (p->volume < 0) fail(ctx, "particles[%d].volume must be greater than zero", i);
        }
        if (p->has_damage) {
            if (!is_fin(p->damage)) fail(ctx, "particles[%d].damage must be a finite number", i);
            if (p->damage < 0 || p->damage > 1) fail(ctx, "particles[%d].damage must be between zero and one", i);
            if (m->model != ORC_NEO_HOOKEAN)
                fail(ctx, "particles[%d].damage is only valid for neo-hookean solids", i);
        }
        if (!is_fin(p->plastic_volume)) fail(ctx, "particles[%d].plasticVolume must be a finite number", i);
        if (p->plastic_volume < SNOW_MIN_PLASTIC_VOLUME || p->plastic_volume > SNOW_MAX_PLASTIC_VOLUME)
            fail(ctx, "particles[%d].plasticVolume must be between 0.6 and 20", i);
        if (p->bonded_vertex < -1 || p->bonded_vertex > 2)
            fail(ctx, "particles[%d].bondedTriangleVertex must be 0, 1, or 2", i);
        if (p->px < 0 || p->px > v->domain_w || p->py < 0 || p->py > v->domain_h)
            fail(ctx, "particles[%d].position must be inside the grid domain", i);
        mat2 F = {p->f00, p->f01, p->f10, p->f11};
        double J = det2(F);
        if (!is_fin(J) || J <= 0) fail(ctx, "particles[%d].F must have a finite positive determinant", i);
    }
}

/* validateMpmSolidBondGraph, src/lib/mpm/reference/solid-bonds.ts:12-70 */
static void validate_bonds(ctx_t *ctx, const orc_material *mats, int32_t n_mats,
                           const orc_particle *ps, int32_t n, const orc_bond *bonds, int32_t nb,
                           const vcfg_t *v)
{
    for (int32_t b = 0; b < nb; ++b) {
        const orc_bond *bond = &bonds[b];
        if (bond->first < 0 || bond->first >= n)
            fail(ctx, "fractureBonds[%d].firstParticle must identify an existing particle", b);
        if (bond->second < 0 || bond->second >= n)
            fail(ctx, "fractureBonds[%d].secondParticle must identify an existing particle", b);
        if (bond->first == bond->second)
            fail(ctx, "fractureBonds[%d] must connect two distinct particles", b);
        if (!is_fin(bond->rest_length) || bond->rest_length <= 0)
            fail(ctx, "fractureBonds[%d].restLength must be positive and finite", b);
        if (!is_fin(bond->failure_strain) || bond->failure_strain <= 0)
            fail(ctx, "fractureBonds[%d].failureStrain must be positive and finite", b);
        if (!is_fin(bond->damage) || bond->damage < 0 || bond->damage > 1)
            fail(ctx, "fractureBonds[%d].damage must be between zero and one", b);
        const orc_particle *f = &ps[bond->first], *s = &ps[bond->second];
        if (f->object_id != s->object_id)
            fail(ctx, "fractureBonds[%d] must connect particles of one object", b);
        if (f->bonded_vertex >= 0 || s->bonded_vertex >= 0)
            fail(ctx, "fractureBonds[%d] cannot reuse bonded triangle vertices", b);
        if (particle_material(mats, n_mats, f, v, ctx, bond->first)->model != ORC_NEO_HOOKEAN ||
            particle_material(mats, n_mats, s, v, ctx, bond->second)->model != ORC_NEO_HOOKEAN)
            fail(ctx, "fractureBonds[%d] endpoints must be neo-hookean solids", b);
        int32_t lo = bond->first < bond->second ? bond->first : bond->second;
        int32_t hi = bond->first < bond->second ? bond->second : bond->first;
        for (int32_t o = 0; o < b; ++o) {
            int32_t l2 = bonds[o].first < bonds[o].second ? bonds[o].first : bonds[o].second;
            int32_t h2 = bonds[o].first < bonds[o].second ? bonds[o].second : bonds[o].first;
            if (l2 == lo && h2 == hi) fail(ctx, "fractureBonds[%d] duplicates an existing particle pair", b);
        }
    }
}

/* collectBondedBodyStarts, src/lib/mpm/reference/solver.ts:1023-1062 */
static int32_t collect_body_starts(ctx_t *ctx, const orc_material *mats, int32_t n_mats,
                                   const orc_particle *ps, int32_t n, const vcfg_t *v,
                                   int32_t *starts)
{
    int32_t count = 0;
    for (int32_t i = 0; i < n; ++i) {
        const orc_particle *p = &ps[i];
        if (p->bonded_vertex < 0) continue;
        if (p->bonded_vertex != 0)
            fail(ctx, "particles[%d].bondedTriangleVertex must start each triangle at zero", i);
        if (!v->has_bond_rest_length) fail(ctx, "bondRestLength is required for bonded triangle particles");
        if (i + 2 >= n) fail(ctx, "bonded triangle at particle %d is incomplete", i);
        for (int32_t vtx = 0; vtx < 3; ++vtx) {
            const orc_particle *m = &ps[i + vtx];
            if (m->bonded_vertex != vtx || m->object_id != p->object_id)
                fail(ctx, "bonded triangle at particle %d must contain contiguous vertices 0, 1, and 2 of one object", i);
            int32_t model = particle_material(mats, n_mats, m, v, ctx, i + vtx)->model;
            if (model == ORC_WATER || model == ORC_OIL)
                fail(ctx, "bonded triangle vertices must use a solid material");
        }
        starts[count++] = i;
        i += 2;
    }
    return count;
}

/* ----------------------------------------------------------- stencil -- */

typedef struct {
    int32_t bx, by;
    double fx, fy;
    double wx[3], wy[3];
} stencil_t;

/* updateParticleStencil, src/lib/mpm/reference/solver.ts:2017-2034 */
static void make_stencil(double px, double py, double dx, stencil_t *s)
{
    double gx = px / dx, gy = py / dx;
    s->bx = (int32_t)floor(gx - 0.5);
    s->by = (int32_t)floor(gy - 0.5);
    s->fx = gx - s->bx;
    s->fy = gy - s->by;
    double a;
    a = 1.5 - s->fx; s->wx[0] = 0.5 * (a * a);
    a = s->fx - 1;   s->wx[1] = 0.75 - a * a;
    a = s->fx - 0.5; s->wx[2] = 0.5 * (a * a);
    a = 1.5 - s->fy; s->wy[0] = 0.5 * (a * a);
    a = s->fy - 1;   s->wy[1] = 0.75 - a * a;
    a = s->fy - 0.5; s->wy[2] = 0.5 * (a * a);
}

static int64_t node_key(int32_t x, int32_t y, int64_t width)
{
    return ((int64_t)y + 1) * width + ((int64_t)x + 1); /* solver.ts:2594-2600 */
}

static void assert_weight(ctx_t *ctx, double w)
{
    if (!is_fin(w) || w < 0) fail(ctx, "quadratic B-spline weights must be finite and non-negative");
}

/* ------------------------------------------------------ constitutive -- */

typedef struct {
    double s1, s2;
    vec2 u1, u2, v1, v2;
    mat2 R;
} decomp_t;

/* decompose2x2, src/lib/mpm/reference/solver.ts:2425-2463 */
static decomp_t decompose(ctx_t *ctx, mat2 F)
{
    decomp_t d;
    double c00 = F.m00 * F.m00 + F.m10 * F.m10;
    double c01 = F.m00 * F.m01 + F.m10 * F.m11;
    double c11 = F.m01 * F.m01 + F.m11 * F.m11;
    double radius = hypot(c00 - c11, 2 * c01);
    d.s1 = sqrt(dmax(0, (c00 + c11 + radius) * 0.5));
    d.s2 = det2(F) / d.s1;
    if (!is_fin(d.s1) || !is_fin(d.s2) || d.s1 <= 0 || d.s2 <= 0)
        fail(ctx, "snow deformation cannot be decomposed into finite positive stretches");
    double angle = 0.5 * atan2(2 * c01, c00 - c11);
    double c = cos(angle), s = sin(angle);
    d.v1.x = c; d.v1.y = s;
    d.v2.x = -s; d.v2.y = c;
    d.u1.x = (F.m00 * d.v1.x + F.m01 * d.v1.y) / d.s1;
    d.u1.y = (F.m10 * d.v1.x + F.m11 * d.v1.y) / d.s1;
    d.u2.x = -d.u1.y;
    d.u2.y = d.u1.x;
    d.R.m00 = d.u1.x * d.v1.x + d.u2.x * d.v2.x;
    d.R.m01 = d.u1.x * d.v1.y + d.u2.x * d.v2.y;
    d.R.m10 = d.u1.y * d.v1.x + d.u2.y * d.v2.x;
    d.R.m11 = d.u1.y * d.v1.y + d.u2.y * d.v2.y;
    assert_matrix_finite(ctx, d.R, "snow polar rotation");
    return d;
}

static mat2 reconstruct(const decomp_t *d, double s1, double s2)
{
    mat2 o;
    o.m00 = s1 * d->u1.x * d->v1.x + s2 * d->u2.x * d->v2.x;
    o.m01 = s1 * d->u1.x * d->v1.y + s2 * d->u2.x * d->v2.y;
    o.m10 = s1 * d->u1.y * d->v1.x + s2 * d->u2.y * d->v2.x;
    o.m11 = s1 * d->u1.y * d->v1.y + s2 * d->u2.y * d->v2.y;
    return o;
}

/* granularStressTimesFt, src/lib/mpm/reference/solver.ts:2222-2265 */
static mat2 granular_stress(ctx_t *ctx, mat2 F, const orc_material *m)
{
    decomp_t d = decompose(ctx, F);
    double l1 = log(d.s1), l2 = log(d.s2);
    double lv = l1 + l2;
    double blv = dmax(log(MIN_POWDER_DETERMINANT), lv);
    double pressure = dmax(0, -(m->lambda + m->mu) * blv);
    double dev = 0.5 * (l1 - l2);
    double maxdev = (m->friction * pressure) / (2 * m->mu);
    double pdev = dmin(dev, maxdev);
    double mean = 0.5 * lv;
    double p1 = 2 * m->mu * (mean + pdev) + m->lambda * lv;
    double p2 = 2 * m->mu * (mean - pdev) + m->lambda * lv;
    mat2 o;
    o.m00 = p1 * d.u1.x * d.u1.x + p2 * d.u2.x * d.u2.x;
    o.m01 = p1 * d.u1.x * d.u1.y + p2 * d.u2.x * d.u2.y;
    o.m10 = p1 * d.u1.y * d.u1.x + p2 * d.u2.y * d.u2.x;
    o.m11 = p1 * d.u1.y * d.u1.y + p2 * d.u2.y * d.u2.y;
    assert_matrix_finite(ctx, o, "powder stress");
    return o;
}

/* neoHookeanFirstPiola, src/lib/mpm/reference/solver.ts:2036-2061 */
static mat2 neo_hookean_piola(ctx_t *ctx, mat2 F, const orc_material *m)
{
    double J = det2(F);
    mat2 it = {F.m11 / J, -F.m10 / J, -F.m01 / J, F.m00 / J};
    double pressure = m->lambda * log(J);
    mat2 P;
    P.m00 = m->mu * (F.m00 - it.m00) + pressure * it.m00;
    P.m01 = m->mu * (F.m01 - it.m01) + pressure * it.m01;
    P.m10 = m->mu * (F.m10 - it.m10) + pressure * it.m10;
    P.m11 = m->mu * (F.m11 - it.m11) + pressure * it.m11;
    assert_matrix_finite(ctx, P, "first Piola stress");
    return P;
}

/* corotated stress shared by snow and the fixed-corotated model:
 * src/lib/mpm/reference/solver.ts:2171-2203 */
static mat2 corotated_stress(ctx_t *ctx, mat2 F, double lambda, double mu, const char *name)
{
    decomp_t d = decompose(ctx, F);
    double J = det2(F);
    double shear = 2 * mu;
    double volumetric = lambda * J * (J - 1);
    mat2 diff = {F.m00 - d.R.m00, F.m01 - d.R.m01, F.m10 - d.R.m10, F.m11 - d.R.m11};
    mat2 o;
    o.m00 = shear * (diff.m00 * F.m00 + diff.m01 * F.m01) + volumetric;
    o.m01 = shear * (diff.m00 * F.m10 + diff.m01 * F.m11);
    o.m10 = shear * (diff.m10 * F.m00 + diff.m11 * F.m01);
    o.m11 = shear * (diff.m10 * F.m10 + diff.m11 * F.m11) + volumetric;
    assert_matrix_finite(ctx, o, name);
    return o;
}

/* constitutiveStressTimesFt, src/lib/mpm/reference/solver.ts:2148-2213 */
static mat2 stress_times_ft(ctx_t *ctx, mat2 F, double plastic_volume, const orc_material *m,
                            double damage)
{
    if (m->model == ORC_WATER || m->model == ORC_OIL) {
        double J = det2(F);
        double p = m->tait ? -J * m->lambda * (pow(1 / J, m->exponent) - 1)
                           : m->lambda * dmin(J - 1, 0);
        mat2 o = {p, 0, 0, p};
        assert_matrix_finite(ctx, o, m->model == ORC_WATER ? "water stress" : "oil stress");
        return o;
    }
    if (m->model == ORC_SNOW) {
        double he = dmax(-SNOW_MAX_HARDENING_EXPONENT,
                         dmin(SNOW_MAX_HARDENING_EXPONENT, SNOW_HARDENING * (1 - plastic_volume)));
        double h = exp(he);
        return corotated_stress(ctx, F, m->lambda * h, m->mu * h, "snow stress");
    }
    if (m->model == ORC_FIXED_COROTATED) return corotated_stress(ctx, F, m->lambda, m->mu, "fixed-corotated stress");
    if (m->model == ORC_POWDER) return granular_stress(ctx, F, m);
    mat2 P = neo_hookean_piola(ctx, F, m);
    return scale2(mul2(P, transpose2(F)), dmax(0, 1 - damage));
}

/* projectSnowDeformation, src/lib/mpm/reference/solver.ts:2267-2303 */
static mat2 project_snow(ctx_t *ctx, mat2 F, double pv, double *pv_out)
{
    decomp_t d = decompose(ctx, F);
    double lo = 1 - SNOW_COMPRESSION_YIELD, hi = 1 + SNOW_STRETCH_YIELD;
    double s1 = dmax(lo, dmin(hi, d.s1));
    double s2 = dmax(lo, dmin(hi, d.s2));
    double upv = dmax(SNOW_MIN_PLASTIC_VOLUME, dmin(SNOW_MAX_PLASTIC_VOLUME, (pv * det2(F)) / (s1 * s2)));
    mat2 o = reconstruct(&d, s1, s2);
    assert_matrix_finite(ctx, o, "projected snow deformation");
    assert_finite(ctx, upv, "snow plastic volume");
    if (det2(o) <= 0) fail(ctx, "snow projection produced a non-positive deformation determinant");
    *pv_out = upv;
    return o;
}

/* projectGranularDeformation, src/lib/mpm/reference/solver.ts:2305-2357 */
static mat2 project_granular(ctx_t *ctx, mat2 F, const orc_material *m)
{
    decomp_t d = decompose(ctx, F);
    double l1 = log(d.s1), l2 = log(d.s2);
    double lv = l1 + l2;
    double minlv = log(MIN_POWDER_DETERMINANT);
    double blv = dmax(minlv, lv);
    double pressure = dmax(0, -(m->lambda + m->mu) * blv);
    double dev = 0.5 * (l1 - l2);
    double maxdev = (m->friction * pressure) / (2 * m->mu);
    if (dev <= maxdev && lv >= minlv) return F;
    double pdev = dmin(dev, maxdev);
    double mean = 0.5 * blv;
    mat2 o = reconstruct(&d, exp(mean + pdev), exp(mean - pdev));
    assert_matrix_finite(ctx, o, "projected powder deformation");
    if (det2(o) <= 0) fail(ctx, "powder projection produced a non-positive deformation determinant");
    return o;
}

/* projectLiquidDeformation, src/lib/mpm/reference/solver.ts:2359-2392 */
static mat2 project_liquid(ctx_t *ctx, mat2 F)
{
    double J = det2(F);
    double cn = F.m00 + F.m11, sn = F.m10 - F.m01;
    double mag = hypot(cn, sn);
    if (!is_fin(mag) || mag <= 0 || !is_fin(J) || J <= 0)
        fail(ctx, "liquid deformation cannot be projected to a finite rotation");
    double bj = dmin(MAX_LIQUID_DETERMINANT, dmax(MIN_LIQUID_DETERMINANT, J));
    double s = sqrt(bj);
    double c = cn / mag, si = sn / mag;
    mat2 o = {s * c, -s * si, s * si, s * c};
    assert_matrix_finite(ctx, o, "projected liquid deformation");
    return o;
}

/* projectNeoHookeanDeformation, src/lib/mpm/reference/solver.ts:2394-2423 */
static mat2 project_neo_hookean(ctx_t *ctx, mat2 F)
{
    decomp_t d = decompose(ctx, F);
    double s1 = dmax(MIN_NEO_HOOKEAN_STRETCH, dmin(MAX_NEO_HOOKEAN_STRETCH, d.s1));
    double s2 = dmax(MIN_NEO_HOOKEAN_STRETCH, dmin(MAX_NEO_HOOKEAN_STRETCH, d.s2));
    mat2 o = reconstruct(&d, s1, s2);
    assert_matrix_finite(ctx, o, "projected Neo-Hookean deformation");
    if (det2(o) <= 0) fail(ctx, "Neo-Hookean projection produced a non-positive deformation determinant");
    return o;
}

/* updateDeformationGradient, src/lib/mpm/reference/solver.ts:2561-2592 */
static mat2 update_deformation(ctx_t *ctx, mat2 F, mat2 C, double dt)
{
    double row = dmax(fabs(C.m00) + fabs(C.m01), fabs(C.m10) + fabs(C.m11));
    double inc = dt * row;
    assert_finite(ctx, inc, "deformation increment");
    double sub = ceil(inc / MAX_DEFORMATION_INCREMENT);
    if (sub < 1) sub = 1;
    if (sub > MAX_DEFORMATION_SUBSTEPS) fail(ctx, "deformation update exceeds the adaptive substep limit");
    int32_t n = (int32_t)sub;
    double h = dt / n;
    mat2 out = F;
    for (int32_t s = 0; s < n; ++s) {
        mat2 u = {1 + h * C.m00, h * C.m01, h * C.m10, 1 + h * C.m11};
        out = mul2(u, out);
    }
    assert_matrix_finite(ctx, out, "deformation gradient");
    return out;
}

/* confineAxis, src/lib/mpm/reference/solver.ts:2528-2540 */
static void confine(double next, double vel, double maximum, double *p, double *v)
{
    if (next < 0 || (next == 0 && vel < 0)) { *p = 0; *v = 0; return; }
    if (next > maximum || (next == maximum && vel > 0)) { *p = maximum; *v = 0; return; }
    *p = next;
    *v = vel;
}

/* applyWallCushion, src/lib/mpm/reference/solver.ts:2542-2546 */
static double wall_cushion(double vel, double coord, double extent)
{
    double distance = vel < 0 ? coord : extent - coord;
    double cushion = dmin(WALL_CUSHION_CELLS, extent / 4);
    return vel * dmax(0, dmin(1, distance / cushion));
}

/* applyWallTangentialFriction, src/lib/mpm/reference/solver.ts:2548-2559 */
static double wall_friction(double vel, double coord, double extent, double friction)
{
    if (friction == 0) return vel;
    double distance = dmax(0, dmin(coord, extent - coord));
    double cushion = dmin(WALL_CUSHION_CELLS, extent / 4);
    double influence = 1 - dmax(0, dmin(1, distance / cushion));
    return vel * (1 - friction * influence);
}

/* updateGridVelocity, src/lib/mpm/reference/solver.ts:1507-1524 */
static void grid_velocity(ctx_t *ctx, double mass, double mx, double my, const vcfg_t *v,
                          double *vx, double *vy)
{
    if (mass <= 0) { *vx = 0; *vy = 0; return; }
    *vx = mx / mass + v->dt * v->gx;
    *vy = my / mass + v->dt * v->gy;
    assert_finite(ctx, *vx, "grid velocity");
    assert_finite(ctx, *vy, "grid velocity");
}

/* volumeGradient, src/lib/mpm/reference/solver.ts:1381-1409 */
static vec2 volume_gradient(grid_t *g, int32_t x, int32_t y, int water, const vcfg_t *v)
{
    double vol[4];
    int32_t xs[4] = {x + 1, x - 1, x, x};
    int32_t ys[4] = {y, y, y + 1, y - 1};
    for (int k = 0; k < 4; ++k) {
        if (xs[k] < -1 || xs[k] > v->cells_x + 1 || ys[k] < -1 || ys[k] > v->cells_y + 1) {
            vol[k] = 0;
            continue;
        }
        node_t *n = grid_get(g, node_key(xs[k], ys[k], v->node_width));
        vol[k] = n == NULL ? 0 : (water ? n->w_vol : n->o_vol);
    }
    double scale = 1 / (2 * v->cell_size * v->cell_size);
    vec2 o = {(vol[0] - vol[1]) * scale, (vol[2] - vol[3]) * scale};
    return o;
}

/* solveLiquidGridContact, src/lib/mpm/reference/solver.ts:1293-1379 */
static void liquid_contact(ctx_t *ctx, node_t *n, grid_t *g, const vcfg_t *v)
{
    if (n->w_mass <= 0 || n->o_mass <= 0 || n->w_vol <= 0 || n->o_vol <= 0 || n->x < 0 ||
        n->x > v->cells_x || n->y < 0 || n->y > v->cells_y)
        return;
    vec2 wg = volume_gradient(g, n->x, n->y, 1, v);
    vec2 og = volume_gradient(g, n->x, n->y, 0, v);
    vec2 grad = {og.x - wg.x, og.y - wg.y};
    double len = hypot(grad.x, grad.y);
    if (!is_fin(len) || len <= 1e-12) return;
    vec2 normal = {grad.x * (1 / len), grad.y * (1 / len)};
    double wd = n->w_mass / n->w_vol;
    double od = n->o_mass / n->o_vol;
    double ds = dmax(wd, od);
    double contrast = (od - wd) / ds;
    double gm = hypot(v->gx, v->gy);
    double align = gm > 0 ? (normal.x * v->gx + normal.y * v->gy) / gm : 0;
    assert_finite(ctx, wd, "water contact density");
    assert_finite(ctx, od, "oil contact density");
    assert_finite(ctx, contrast, "liquid contact density contrast");
    assert_finite(ctx, gm, "gravity magnitude");
    assert_finite(ctx, align, "liquid contact gravity alignment");
    if (ds <= 0 || wd <= 0 || od <= 0) fail(ctx, "liquid contact densities must be positive");
    if (contrast * align < -LIQUID_STABLE_ORDER_EPSILON) {
        normal.x = normal.x * -1;
        normal.y = normal.y * -1;
    }
    double rel = (n->o_vx - n->w_vx) * normal.x + (n->o_vy - n->w_vy) * normal.y;
    double overlap = dmin(1, (2 * dmin(n->w_vol, n->o_vol)) / (n->w_vol + n->o_vol));
    double minsep = dmax((LIQUID_CONTACT_SEPARATION_FRACTION * overlap * v->cell_size) /
                             LIQUID_CONTACT_RELAXATION_SECONDS,
                         dmax(-rel, 0) * LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER);
    if (rel >= minsep) return;
    double impulse = (minsep - rel) / (1 / n->w_mass + 1 / n->o_mass);
    n->w_vx -= (impulse / n->w_mass) * normal.x;
    n->w_vy -= (impulse / n->w_mass) * normal.y;
    n->o_vx += (impulse / n->o_mass) * normal.x;
    n->o_vy += (impulse / n->o_mass) * normal.y;
}

/* ----------------------------------------------------------- triangles -- */

typedef struct {
    double sd, nx, ny;
    double bary[3];
} sample_t;

/* triangleDistanceSample, src/lib/mpm/reference/solver.ts:1190-1291 */
static void triangle_sample(ctx_t *ctx, double px, double py, const vec2 tri[3], sample_t *s)
{
    vec2 a = tri[0], b = tri[1], c = tri[2];
    double abx = b.x - a.x, aby = b.y - a.y, acx = c.x - a.x, acy = c.y - a.y;
    double area = abx * acy - aby * acx;
    if (!is_fin(area) || fabs(area) <= 1e-10) fail(ctx, "bonded triangle became degenerate");
    double bcx = c.x - b.x, bcy = c.y - b.y, cax = a.x - c.x, cay = a.y - c.y;
    double apx = px - a.x, apy = py - a.y, bpx = px - b.x, bpy = py - b.y, cpx = px - c.x, cpy = py - c.y;
    double cab = abx * apy - aby * apx;
    double cbc = bcx * bpy - bcy * bpx;
    double cca = cax * cpy - cay * cpx;
    int inside = area > 0 ? (cab >= -1e-10 && cbc >= -1e-10 && cca >= -1e-10)
                          : (cab <= 1e-10 && cbc <= 1e-10 && cca <= 1e-10);
    double best = INFINITY, bnx = 0, bny = 0;
    for (int e = 0; e < 3; ++e) {
        vec2 st = e == 0 ? a : e == 1 ? b : c;
        vec2 en = e == 0 ? b : e == 1 ? c : a;
        double dx = en.x - st.x, dy = en.y - st.y;
        double l2 = dx * dx + dy * dy;
        double ox = px - st.x, oy = py - st.y;
        double t = dmax(0, dmin(1, (ox * dx + oy * dy) / l2));
        double qx = st.x + dx * t, qy = st.y + dy * t;
        double ddx = px - qx, ddy = py - qy;
        double d2 = ddx * ddx + ddy * ddy;
        if (d2 >= best) continue;
        best = d2;
        if (e == 0) { s->bary[0] = 1 - t; s->bary[1] = t; s->bary[2] = 0; }
        else if (e == 1) { s->bary[0] = 0; s->bary[1] = 1 - t; s->bary[2] = t; }
        else { s->bary[0] = t; s->bary[1] = 0; s->bary[2] = 1 - t; }
        if (d2 > 1e-20 && !inside) {
            double d = sqrt(d2);
            double inv = 1 / d;
            bnx = ddx * inv;
            bny = ddy * inv;
        } else {
            double orient = area > 0 ? 1 : -1;
            double outx = orient * dy, outy = -orient * dx;
            double el = sqrt(l2);
            double inv = 1 / el;
            bnx = outx * inv;
            bny = outy * inv;
        }
    }
    double d = sqrt(best);
    if (!is_fin(d) || !is_fin(bnx) || !is_fin(bny)) fail(ctx, "bonded triangle contact field became non-finite");
    s->sd = inside ? -d : d;
    s->nx = bnx;
    s->ny = bny;
}

static void triangle_vertices(const orc_particle *ps, int32_t start, vec2 tri[3])
{
    for (int k = 0; k < 3; ++k) {
        tri[k].x = ps[start + k].px;
        tri[k].y = ps[start + k].py;
    }
}

typedef struct {
    int32_t min_x, max_x, min_y, max_y;
    double fmin_x, fmax_x, fmin_y, fmax_y;
} scan_t;

static void body_scan_range(const vec2 tri[3], const vcfg_t *v, scan_t *s)
{
    double md = v->cell_size * TRIANGLE_FIELD_BAND_CELLS;
    double mnx = dmin(dmin(tri[0].x, tri[1].x), tri[2].x), mxx = dmax(dmax(tri[0].x, tri[1].x), tri[2].x);
    double mny = dmin(dmin(tri[0].y, tri[1].y), tri[2].y), mxy = dmax(dmax(tri[0].y, tri[1].y), tri[2].y);
    s->min_x = (int32_t)dmax(-1, floor((mnx - md) / v->cell_size) - 1);
    s->max_x = (int32_t)dmin(v->cells_x + 1, ceil((mxx + md) / v->cell_size) + 1);
    s->min_y = (int32_t)dmax(-1, floor((mny - md) / v->cell_size) - 1);
    s->max_y = (int32_t)dmin(v->cells_y + 1, ceil((mxy + md) / v->cell_size) + 1);
    s->fmin_x = mnx - md;
    s->fmax_x = mxx + md;
    s->fmin_y = mny - md;
    s->fmax_y = mxy + md;
}

/* buildTriangleField, src/lib/mpm/reference/solver.ts:1064-1165.  Returns the
 * number of bodies that own at least one field node (nodesByBody.size). */
static int32_t build_triangle_field(ctx_t *ctx, grid_t *g, const int32_t *starts, int32_t nb,
                                    const orc_particle *ps, const vcfg_t *v)
{
    if (nb == 0) return 0;
    double md = v->cell_size * TRIANGLE_FIELD_BAND_CELLS;
    sample_t s = {0, 0, 0, {0, 0, 0}};
    for (int32_t b = 0; b < nb; ++b) {
        vec2 tri[3];
        triangle_vertices(ps, starts[b], tri);
        scan_t r;
        body_scan_range(tri, v, &r);
        for (int32_t y = r.min_y; y <= r.max_y; ++y) {
            double pyv = y * v->cell_size;
            if (pyv < r.fmin_y || pyv > r.fmax_y) continue;
            for (int32_t x = r.min_x; x <= r.max_x; ++x) {
                double pxv = x * v->cell_size;
                if (pxv < r.fmin_x || pxv > r.fmax_x) continue;
                triangle_sample(ctx, pxv, pyv, tri, &s);
                if (s.sd > md) continue;
                int64_t key = node_key(x, y, v->node_width);
                field_t *nearest = field_get(g, key);
                if (nearest && s.sd >= nearest->signed_distance) continue;
                field_t *f = &g->fields[key];
                f->body_start = starts[b];
                f->key = (int32_t)key;
                f->signed_distance = s.sd;
                f->nx = s.nx;
                f->ny = s.ny;
                f->bary[0] = s.bary[0];
                f->bary[1] = s.bary[1];
                f->bary[2] = s.bary[2];
                f->ix = 0;
                f->iy = 0;
                g->field_gen[key] = g->field_generation;
            }
        }
    }
    /* count bodies that finally own at least one node */
    int32_t owners = 0;
    for (int32_t b = 0; b < nb; ++b) {
        vec2 tri[3];
        triangle_vertices(ps, starts[b], tri);
        scan_t r;
        body_scan_range(tri, v, &r);
        int found = 0;
        for (int32_t y = r.min_y; y <= r.max_y && !found; ++y)
            for (int32_t x = r.min_x; x <= r.max_x && !found; ++x) {
                field_t *f = field_get(g, node_key(x, y, v->node_width));
                if (f && f->body_start == starts[b]) found = 1;
            }
        owners += found;
    }
    return owners;
}

/* resolveFluidTriangleContact, src/lib/mpm/reference/solver.ts:1462-1505 */
static void resolve_fluid_triangle(ctx_t *ctx, double fm, double *fvx, double *fvy, vec2 sv,
                                   double nx, double ny, double inv_body, double dt,
                                   double *bix, double *biy)
{
    double iem = 1 / fm + inv_body;
    assert_finite(ctx, iem, "triangle contact inverse effective mass");
    if (iem <= 0) fail(ctx, "triangle contact inverse effective mass must be positive");
    double rvx = *fvx - sv.x, rvy = *fvy - sv.y;
    double rn = rvx * nx + rvy * ny;
    double nmag = rn < 0 ? -rn / iem : 0;
    double nix = nx * nmag, niy = ny * nmag;
    double tvx = rvx - nx * rn, tvy = rvy - ny * rn;
    double damping = 1 - exp(-TRIANGLE_FLUID_TANGENTIAL_DRAG_RATE * dt);
    double tix = tvx * (-damping / iem), tiy = tvy * (-damping / iem);
    double ifx = nix + tix, ify = niy + tiy;
    double nvx = *fvx + ifx * (1 / fm), nvy = *fvy + ify * (1 / fm);
    double bx = ifx * -1, by = ify * -1;
    assert_finite(ctx, nvx, "triangle contact fluid velocity x");
    assert_finite(ctx, nvy, "triangle contact fluid velocity y");
    assert_finite(ctx, bx, "triangle contact body impulse x");
    assert_finite(ctx, by, "triangle contact body impulse y");
    *fvx = nvx;
    *fvy = nvy;
    *bix = bx;
    *biy = by;
}

/* solveFluidTriangleGridContact, src/lib/mpm/reference/solver.ts:1411-1460 */
static void fluid_triangle_contact(ctx_t *ctx, node_t *n, field_t *f, const orc_particle *ps,
                                   const vcfg_t *v)
{
    double radius = sqrt(v->particle_volume / M_PI);
    double reach = radius + GRID_CONTACT_REACH_CELLS * v->cell_size;
    if (f->signed_distance > reach) return;
    vec2 sv = {0, 0};
    double inv_body = 0;
    for (int k = 0; k < 3; ++k) {
        double w = f->bary[k];
        sv.x += w * ps[f->body_start + k].vx;
        sv.y += w * ps[f->body_start + k].vy;
        inv_body += (w * w) / v->particle_mass;
    }
    if (inv_body <= 0) return;
    double bix, biy;
    if (n->w_mass > 0) {
        resolve_fluid_triangle(ctx, n->w_mass, &n->w_vx, &n->w_vy, sv, f->nx, f->ny, inv_body, v->dt, &bix, &biy);
        f->ix += bix;
        f->iy += biy;
    }
    if (n->o_mass > 0) {
        resolve_fluid_triangle(ctx, n->o_mass, &n->o_vx, &n->o_vy, sv, f->nx, f->ny, inv_body, v->dt, &bix, &biy);
        f->ix += bix;
        f->iy += biy;
    }
}

/* projectParticleOutsideTriangles, src/lib/mpm/reference/solver.ts:1526-1590 */
static void project_outside_triangles(ctx_t *ctx, double *px, double *py, double radius, grid_t *g,
                                      int32_t owners, const vcfg_t *v)
{
    if (owners == 0) return;
    stencil_t s;
    make_stencil(*px, *py, v->cell_size, &s);
    double band = v->cell_size * TRIANGLE_FIELD_BAND_CELLS;
    double sd = 0;
    int32_t closest = -1;
    double closest_d = INFINITY;
    double selx = 0, sely = 0;
    int has_sel = 0;
    for (int oy = 0; oy < 3; ++oy)
        for (int ox = 0; ox < 3; ++ox) {
            double w = s.wx[ox] * s.wy[oy];
            field_t *f = field_get(g, node_key(s.bx + ox, s.by + oy, v->node_width));
            sd += w * (f ? f->signed_distance : band);
            if (f && f->signed_distance < closest_d) {
                closest_d = f->signed_distance;
                closest = f->body_start;
                selx = f->nx;
                sely = f->ny;
                has_sel = 1;
            }
        }
    if (closest < 0 || sd >= radius) return;
    double nx = 0, ny = 0;
    for (int oy = 0; oy < 3; ++oy)
        for (int ox = 0; ox < 3; ++ox) {
            double w = s.wx[ox] * s.wy[oy];
            field_t *f = field_get(g, node_key(s.bx + ox, s.by + oy, v->node_width));
            if (!f || f->body_start != closest) continue;
            nx += w * f->nx;
            ny += w * f->ny;
        }
    double len = hypot(nx, ny);
    double ux, uy;
    if (len > 1e-12 && is_fin(len)) { ux = nx / len; uy = ny / len; }
    else if (has_sel) { ux = selx; uy = sely; }
    else return;
    double corr = radius - sd;
    double qx = *px + corr * ux, qy = *py + corr * uy;
    assert_finite(ctx, qx, "triangle contact projection x");
    assert_finite(ctx, qy, "triangle contact projection y");
    *px = qx;
    *py = qy;
}

/* ------------------------------------------------------------- stepMpm -- */

typedef struct {
    double mass, volume;
    const orc_material *m;
} state_t;

static int32_t step_impl(ctx_t *ctx, grid_t *g, const orc_material *mats, int32_t n_mats,
                         const orc_config *cfg, const orc_particle *in, orc_particle *out,
                         int32_t n, const orc_bond *bonds, orc_bond *bonds_out, orc_diag *diag,
                         int32_t *starts, state_t *st)
{
    vcfg_t v;
    validate_config(ctx, mats, n_mats, cfg, &v);
    validate_particles(ctx, mats, n_mats, in, n, &v);
    int32_t nbonds = cfg->has_fracture_bonds ? cfg->n_bonds : 0;
    if (nbonds > 0) validate_bonds(ctx, mats, n_mats, in, n, bonds, nbonds, &v);
    int32_t nb = collect_body_starts(ctx, mats, n_mats, in, n, &v, starts);

    /* resolveParticleState, src/lib/mpm/reference/solver.ts:2130-2146 */
    for (int32_t i = 0; i < n; ++i) {
        st[i].m = particle_material(mats, n_mats, &in[i], &v, ctx, i);
        st[i].volume = in[i].volume > 0 ? in[i].volume : v.particle_volume;
        st[i].mass = (st[i].m->model == ORC_WATER || st[i].m->model == ORC_OIL)
                         ? st[i].m->density * st[i].volume
                         : v.particle_mass;
        assert_finite(ctx, st[i].volume, "particle volume");
        assert_finite(ctx, st[i].mass, "particle mass");
        if (st[i].volume <= 0 || st[i].mass <= 0) fail(ctx, "particle mass and volume must be greater than zero");
    }
    double in_mass = 0, in_mx = 0, in_my = 0;
    for (int32_t i = 0; i < n; ++i) in_mass += st[i].mass;
    for (int32_t i = 0; i < n; ++i) {
        in_mx += st[i].mass * in[i].vx;
        in_my += st[i].mass * in[i].vy;
    }
    assert_finite(ctx, in_mass, "input mass");
    grid_begin(g);
    double dx = v.cell_size;

    /* P2G, src/lib/mpm/reference/solver.ts:418-479 */
    for (int32_t i = 0; i < n; ++i) {
        const orc_particle *p = &in[i];
        stencil_t s;
        make_stencil(p->px, p->py, dx, &s);
        mat2 F = {p->f00, p->f01, p->f10, p->f11};
        mat2 C = {p->c00, p->c01, p->c10, p->c11};
        mat2 stress = stress_times_ft(ctx, F, p->plastic_volume, st[i].m, p->has_damage ? p->damage : 0);
        double sscale = -v.dt * st[i].volume * v.gradient_scale;
        assert_finite(ctx, sscale, "particle stress scale");
        int liquid = st[i].m->model == ORC_WATER || st[i].m->model == ORC_OIL;
        double lvol = liquid ? st[i].volume * det2(F) : 0;
        if (liquid) assert_finite(ctx, lvol, "liquid particle volume");
        mat2 A = add2(scale2(C, st[i].mass), scale2(stress, sscale));
        assert_matrix_finite(ctx, A, "particle affine momentum");
        for (int oy = 0; oy < 3; ++oy)
            for (int ox = 0; ox < 3; ++ox) {
                double w = s.wx[ox] * s.wy[oy];
                assert_weight(ctx, w);
                if (w == 0) continue;
                int32_t xi = s.bx + ox, yi = s.by + oy;
                int64_t key = node_key(xi, yi, v.node_width);
                if (key < 0 || key >= g->count) fail(ctx, "particle stencil is outside the halo grid");
                node_t *nd = grid_get_or_create(g, key, xi, yi);
                double dpx = (ox - s.fx) * dx, dpy = (oy - s.fy) * dx;
                double pmx = st[i].mass * p->vx + A.m00 * dpx + A.m01 * dpy;
                double pmy = st[i].mass * p->vy + A.m10 * dpx + A.m11 * dpy;
                if (st[i].m->model == ORC_WATER) {
                    nd->w_mass += w * st[i].mass;
                    nd->w_mx += w * pmx;
                    nd->w_my += w * pmy;
                    nd->w_vol += w * lvol;
                } else if (st[i].m->model == ORC_OIL) {
                    nd->o_mass += w * st[i].mass;
                    nd->o_mx += w * pmx;
                    nd->o_my += w * pmy;
                    nd->o_vol += w * lvol;
                } else {
                    nd->mass += w * st[i].mass;
                    nd->mx += w * pmx;
                    nd->my += w * pmy;
                }
            }
    }

    double gmass = 0, gmx = 0, gmy = 0;
    for (int64_t a = 0; a < g->n_active; ++a) {
        node_t *nd = &g->nodes[g->active[a]];
        if (nd->mass < 0 || nd->w_mass < 0 || nd->w_vol < 0 || nd->o_mass < 0 || nd->o_vol < 0)
            fail(ctx, "grid node mass and phase volume must be non-negative");
        gmass += nd->mass + nd->w_mass + nd->o_mass;
        gmx += nd->mx + nd->w_mx + nd->o_mx;
        gmy += nd->my + nd->w_my + nd->o_my;
    }
    assert_finite(ctx, gmass, "grid mass");
    assert_finite(ctx, gmx, "grid momentum");
    assert_finite(ctx, gmy, "grid momentum");

    int32_t owners = build_triangle_field(ctx, g, starts, nb, in, &v);

    /* grid update, src/lib/mpm/reference/solver.ts:500-608 */
    for (int64_t a = 0; a < g->n_active; ++a) {
        node_t *nd = &g->nodes[g->active[a]];
        grid_velocity(ctx, nd->mass, nd->mx, nd->my, &v, &nd->vx, &nd->vy);
        grid_velocity(ctx, nd->w_mass, nd->w_mx, nd->w_my, &v, &nd->w_vx, &nd->w_vy);
        grid_velocity(ctx, nd->o_mass, nd->o_mx, nd->o_my, &v, &nd->o_vx, &nd->o_vy);
        liquid_contact(ctx, nd, g, &v);
        field_t *f = nb > 0 ? field_get(g, node_key(nd->x, nd->y, v.node_width)) : NULL;
        if (f) fluid_triangle_contact(ctx, nd, f, in, &v);
        double cx = v.cells_x, cy = v.cells_y, fr = v.wall_friction;
        nd->vx = wall_cushion(nd->vx, nd->x, cx);
        nd->vy = wall_cushion(nd->vy, nd->y, cy);
        nd->vx = wall_friction(nd->vx, nd->y, cy, fr);
        nd->vy = wall_friction(nd->vy, nd->x, cx, fr);
        nd->w_vx = wall_cushion(nd->w_vx, nd->x, cx);
        nd->w_vy = wall_cushion(nd->w_vy, nd->y, cy);
        nd->w_vx = wall_friction(nd->w_vx, nd->y, cy, fr);
        nd->w_vy = wall_friction(nd->w_vy, nd->x, cx, fr);
        nd->o_vx = wall_cushion(nd->o_vx, nd->x, cx);
        nd->o_vy = wall_cushion(nd->o_vy, nd->y, cy);
        nd->o_vx = wall_friction(nd->o_vx, nd->y, cy, fr);
        nd->o_vy = wall_friction(nd->o_vy, nd->x, cx, fr);
        if (!is_fin(nd->vx) || !is_fin(nd->vy) || !is_fin(nd->w_vx) || !is_fin(nd->w_vy) ||
            !is_fin(nd->o_vx) || !is_fin(nd->o_vy))
            fail(ctx, "grid node velocityX became non-finite");
    }

    /* G2P, src/lib/mpm/reference/solver.ts:612-773 */
    for (int32_t i = 0; i < n; ++i) {
        const orc_particle *p = &in[i];
        stencil_t s;
        make_stencil(p->px, p->py, dx, &s);
        double vx = 0, vy = 0, c00 = 0, c01 = 0, c10 = 0, c11 = 0, lmass = 0, lvol = 0;
        int water = st[i].m->model == ORC_WATER, oil = st[i].m->model == ORC_OIL;
        int liquid = water || oil;
        for (int oy = 0; oy < 3; ++oy)
            for (int ox = 0; ox < 3; ++ox) {
                double w = s.wx[ox] * s.wy[oy];
                assert_weight(ctx, w);
                if (w == 0) continue;
                node_t *nd = grid_get(g, node_key(s.bx + ox, s.by + oy, v.node_width));
                if (!nd) fail(ctx, "particle stencil is missing a deposited grid node");
                double dpx = (ox - s.fx) * dx, dpy = (oy - s.fy) * dx;
                double nvx = water ? nd->w_vx : oil ? nd->o_vx : nd->vx;
                double nvy = water ? nd->w_vy : oil ? nd->o_vy : nd->vy;
                vx += w * nvx;
                vy += w * nvy;
                if (liquid) {
                    lmass += w * (nd->w_mass + nd->o_mass);
                    lvol += w * (nd->w_vol + nd->o_vol);
                }
                c00 += w * nvx * dpx;
                c01 += w * nvx * dpy;
                c10 += w * nvy * dpx;
                c11 += w * nvy * dpy;
            }
        mat2 F = {p->f00, p->f01, p->f10, p->f11};
        if (liquid) {
            assert_finite(ctx, lmass, "local liquid mass");
            assert_finite(ctx, lvol, "local liquid volume");
            if (lmass <= 0 || lvol <= 0) fail(ctx, "liquid particle stencil has no local liquid density");
            double pd = st[i].mass / (st[i].volume * det2(F));
            double ld = lmass / lvol;
            assert_finite(ctx, pd, "particle density");
            assert_finite(ctx, ld, "local liquid density");
            if (pd <= 0 || ld <= 0) fail(ctx, "liquid densities must be positive");
            double rd = (pd - ld) / pd;
            vx += v.dt * v.gx * rd;
            vy += v.dt * v.gy * rd;
        }
        mat2 C = {c00 * v.gradient_scale, c01 * v.gradient_scale, c10 * v.gradient_scale, c11 * v.gradient_scale};
        assert_finite(ctx, vx, "particle velocity");
        assert_finite(ctx, vy, "particle velocity");
        assert_matrix_finite(ctx, C, "particle affine velocity");
        mat2 trial = update_deformation(ctx, F, C, v.dt);
        double J = det2(trial);
        if (!is_fin(J) || J <= 0) fail(ctx, "step would produce a non-positive deformation determinant");
        mat2 Fn = trial;
        double npv = p->plastic_volume;
        int model = st[i].m->model;
        if (model == ORC_SNOW) Fn = project_snow(ctx, trial, p->plastic_volume, &npv);
        else if (model == ORC_POWDER) Fn = project_granular(ctx, trial, st[i].m);
        else if (liquid) Fn = project_liquid(ctx, trial);
        else if (model == ORC_NEO_HOOKEAN) {
            double tr = trial.m00 * trial.m00 + trial.m01 * trial.m01 + trial.m10 * trial.m10 + trial.m11 * trial.m11;
            if (!is_fin(tr)) fail(ctx, "Neo-Hookean deformation stretch is outside the supported range");
            if (J < MIN_NEO_HOOKEAN_STRETCH * sqrt(tr) || tr > MAX_NEO_HOOKEAN_STRETCH * MAX_NEO_HOOKEAN_STRETCH)
                Fn = project_neo_hookean(ctx, trial);
        }
        double nx = p->px + v.dt * vx, ny = p->py + v.dt * vy;
        assert_finite(ctx, nx, "particle position");
        assert_finite(ctx, ny, "particle position");
        double bpx, bvx, bpy, bvy;
        confine(nx, vx, v.domain_w, &bpx, &bvx);
        confine(ny, vy, v.domain_h, &bpy, &bvy);
        double qx = bpx, qy = bpy;
        if (liquid) project_outside_triangles(ctx, &qx, &qy, sqrt((st[i].volume * det2(Fn)) / M_PI), g, owners, &v);
        orc_particle *o = &out[i];
        *o = *p;
        confine(qx, bvx, v.domain_w, &o->px, &o->vx);
        confine(qy, bvy, v.domain_h, &o->py, &o->vy);
        o->c00 = C.m00; o->c01 = C.m01; o->c10 = C.m10; o->c11 = C.m11;
        o->f00 = Fn.m00; o->f01 = Fn.m01; o->f10 = Fn.m10; o->f11 = Fn.m11;
        o->plastic_volume = npv;
        o->volume = st[i].volume;
        o->material = (int32_t)(st[i].m - mats);
    }

    /* applyTriangleContactImpulses, src/lib/mpm/reference/solver.ts:1592-1622 */
    for (int32_t b = 0; b < nb; ++b) {
        double ix[3] = {0, 0, 0}, iy[3] = {0, 0, 0};
        vec2 tri[3];
        triangle_vertices(in, starts[b], tri);
        scan_t r;
        body_scan_range(tri, &v, &r);
        for (int32_t y = r.min_y; y <= r.max_y; ++y)
            for (int32_t x = r.min_x; x <= r.max_x; ++x) {
                field_t *f = field_get(g, node_key(x, y, v.node_width));
                if (!f || f->body_start != starts[b]) continue;
                for (int k = 0; k < 3; ++k) {
                    ix[k] += f->bary[k] * f->ix;
                    iy[k] += f->bary[k] * f->iy;
                }
            }
        for (int k = 0; k < 3; ++k) {
            orc_particle *o = &out[starts[b] + k];
            double m = st[starts[b] + k].mass;
            o->vx = o->vx + ix[k] / m;
            o->vy = o->vy + iy[k] / m;
            assert_finite(ctx, o->vx, "triangle reaction velocity x");
            assert_finite(ctx, o->vy, "triangle reaction velocity y");
        }
    }

    /* enforceBondedTriangleConstraints, src/lib/mpm/reference/solver.ts:1624-1700 */
    if (nb > 0) {
        double ratio = v.dt / v.bond_reference_dt;
        double stiff = dmin(v.bond_stiffness * ratio * ratio, 1);
        if (!is_fin(stiff)) fail(ctx, "bonded triangle substep stiffness is outside the supported range");
        stiff = dmax(0, dmin(1, stiff));
        static const int edges[3][2] = {{0, 1}, {1, 2}, {2, 0}};
        for (int32_t b = 0; b < nb; ++b) {
            vec2 orig[3], pos[3];
            triangle_vertices(out, starts[b], orig);
            for (int k = 0; k < 3; ++k) pos[k] = orig[k];
            for (int it = 0; it < BONDED_TRIANGLE_SOLVER_ITERATIONS; ++it)
                for (int e = 0; e < 3; ++e) {
                    int a0 = edges[e][0], a1 = edges[e][1];
                    double ddx = pos[a1].x - pos[a0].x, ddy = pos[a1].y - pos[a0].y;
                    double dist = hypot(ddx, ddy);
                    if (!is_fin(dist) || dist <= 1e-10) fail(ctx, "bonded triangle at particle %d collapsed", starts[b]);
                    double k = ((dist - v.bond_rest_length) * stiff * 0.5) / dist;
                    double cx = ddx * k, cy = ddy * k;
                    pos[a0].x = pos[a0].x + cx; pos[a0].y = pos[a0].y + cy;
                    pos[a1].x = pos[a1].x - cx; pos[a1].y = pos[a1].y - cy;
                }
            for (int k = 0; k < 3; ++k) {
                orc_particle *o = &out[starts[b] + k];
                double disx = pos[k].x - orig[k].x, disy = pos[k].y - orig[k].y;
                double nvx = o->vx + disx / v.dt, nvy = o->vy + disy / v.dt;
                confine(pos[k].x, nvx, v.domain_w, &o->px, &o->vx);
                confine(pos[k].y, nvy, v.domain_h, &o->py, &o->vy);
            }
        }
    }

    /* resolveBondedTriangleContacts, src/lib/mpm/reference/solver.ts:1702-1802 */
    if (nb >= 2) {
        double skin = v.cell_size * TRIANGLE_CONTACT_SKIN_CELLS;
        int32_t *deg = (int32_t *)calloc((size_t)nb, sizeof(int32_t));
        double *cn = (double *)malloc((size_t)nb * (size_t)nb * 2 * sizeof(double));
        char *has = (char *)calloc((size_t)nb * (size_t)nb, 1);
        double *mvx = (double *)malloc((size_t)nb * sizeof(double));
        double *mvy = (double *)malloc((size_t)nb * sizeof(double));
        if (!deg || !cn || !has || !mvx || !mvy) {
            free(deg); free(cn); free(has); free(mvx); free(mvy);
            fail(ctx, "out of memory");
        }
        for (int32_t b = 0; b < nb; ++b) {
            const orc_particle *q = &out[starts[b]];
            mvx[b] = (q[0].vx + q[1].vx + q[2].vx) / 3;
            mvy[b] = (q[0].vy + q[1].vy + q[2].vy) / 3;
        }
        for (int32_t a = 0; a < nb; ++a)
            for (int32_t b = a + 1; b < nb; ++b) {
                if (in[starts[a]].object_id == in[starts[b]].object_id) continue;
                vec2 A[3], B[3];
                triangle_vertices(in, starts[a], A);
                triangle_vertices(in, starts[b], B);
                /* trianglePairContact, src/lib/mpm/reference/solver.ts:1804-1874 */
                int separated = 0, has_axis = 0, degenerate = 0;
                double largest = -INFINITY, smallest = INFINITY, axx = 0, axy = 0;
                for (int t = 0; t < 2 && !degenerate; ++t) {
                    const vec2 *T = t == 0 ? A : B;
                    for (int e = 0; e < 3; ++e) {
                        vec2 st0 = T[e], en = T[(e + 1) % 3];
                        double ex = en.x - st0.x, ey = en.y - st0.y;
                        double el = hypot(ex, ey);
                        if (el <= 1e-10) { degenerate = 1; break; }
                        double ux = ey / el, uy = -ex / el;
                        double a0 = A[0].x * ux + A[0].y * uy, a1 = A[1].x * ux + A[1].y * uy, a2 = A[2].x * ux + A[2].y * uy;
                        double b0 = B[0].x * ux + B[0].y * uy, b1 = B[1].x * ux + B[1].y * uy, b2 = B[2].x * ux + B[2].y * uy;
                        double mina = dmin(dmin(a0, a1), a2), maxa = dmax(dmax(a0, a1), a2);
                        double minb = dmin(dmin(b0, b1), b2), maxb = dmax(dmax(b0, b1), b2);
                        double gap = dmax(minb - maxa, mina - maxb);
                        if (gap > 0) {
                            separated = 1;
                            if (gap > largest) { largest = gap; axx = ux; axy = uy; has_axis = 1; }
                        } else if (!separated && -gap < smallest) {
                            smallest = -gap; axx = ux; axy = uy; has_axis = 1;
                        }
                    }
                }
                if (degenerate) continue;
                if (separated && largest > skin) continue;
                if (!has_axis) continue;
                double dirx = (A[0].x + A[1].x + A[2].x) / 3 - (B[0].x + B[1].x + B[2].x) / 3;
                double diry = (A[0].y + A[1].y + A[2].y) / 3 - (B[0].y + B[1].y + B[2].y) / 3;
                double sign = dirx * axx + diry * axy >= 0 ? 1 : -1;
                double pen = separated ? skin - largest : skin + smallest;
                if (!(pen > 0)) continue;
                size_t ab = (size_t)a * (size_t)nb + (size_t)b, ba = (size_t)b * (size_t)nb + (size_t)a;
                has[ab] = has[ba] = 1;
                cn[2 * ab] = sign * axx; cn[2 * ab + 1] = sign * axy;
                cn[2 * ba] = (sign * axx) * -1; cn[2 * ba + 1] = (sign * axy) * -1;
                deg[a] += 1;
                deg[b] += 1;
            }
        double body_mass = 3 * v.particle_mass;
        /* contacts per body are visited in push order: others with a < b were
         * pushed while iterating the outer loop first (ascending), then b > a */
        for (int32_t b = 0; b < nb; ++b) {
            double ix = 0, iy = 0;
            for (int32_t o = 0; o < nb; ++o) {
                size_t bo = (size_t)b * (size_t)nb + (size_t)o;
                if (o == b || !has[bo]) continue;
                double cw = 1 / (double)(deg[b] > deg[o] ? deg[b] : deg[o]);
                double rn = (mvx[b] - mvx[o]) * cn[2 * bo] + (mvy[b] - mvy[o]) * cn[2 * bo + 1];
                if (rn < 0) {
                    double imp = -rn / (2 / body_mass);
                    double iw = cw * TRIANGLE_CONTACT_IMPULSE_RELAXATION;
                    ix += (iw * imp * cn[2 * bo]) / body_mass;
                    iy += (iw * imp * cn[2 * bo + 1]) / body_mass;
                }
            }
            for (int k = 0; k < 3; ++k) {
                orc_particle *q = &out[starts[b] + k];
                double px = q->px, py = q->py;
                confine(px, q->vx + ix, v.domain_w, &q->px, &q->vx);
                confine(py, q->vy + iy, v.domain_h, &q->py, &q->vy);
            }
        }
        free(deg); free(cn); free(has); free(mvx); free(mvy);
    }

    /* updateMpmSolidBondDamage, src/lib/mpm/reference/solid-bonds.ts:72-109 */
    if (cfg->has_fracture_bonds) {
        if (nbonds > 0) validate_bonds(ctx, mats, n_mats, out, n, bonds, nbonds, &v);
        double *pd = nbonds > 0 ? (double *)malloc((size_t)n * sizeof(double)) : NULL;
        char *hp = nbonds > 0 ? (char *)calloc((size_t)n, 1) : NULL;
        for (int32_t b = 0; b < nbonds; ++b) {
            const orc_bond *bd = &bonds[b];
            const orc_particle *f = &out[bd->first], *s = &out[bd->second];
            double dist = hypot(s->px - f->px, s->py - f->py);
            if (!is_fin(dist)) { free(pd); free(hp); fail(ctx, "fracture bond length became non-finite"); }
            double strain = dmax(0, (dist - bd->rest_length) / bd->rest_length);
            int broken = bd->broken || strain >= bd->failure_strain;
            double dmg = broken ? 1 : dmax(bd->damage, dmin(1, strain / bd->failure_strain));
            orc_bond nbd = *bd;
            nbd.damage = dmg;
            nbd.broken = broken;
            int32_t ends[2] = {bd->first, bd->second};
            for (int k = 0; k < 2; ++k) {
                int32_t pi = ends[k];
                if (!hp[pi] || dmg > pd[pi]) pd[pi] = hp[pi] ? dmax(pd[pi], dmg) : dmg;
                hp[pi] = 1;
            }
            bonds_out[b] = nbd;
        }
        for (int32_t i = 0; i < n && nbonds > 0; ++i) {
            if (!hp[i]) continue;
            double cur = out[i].has_damage ? out[i].damage : 0;
            if (pd[i] <= cur) continue;
            out[i].damage = pd[i];
            out[i].has_damage = 1;
        }
        free(pd);
        free(hp);
    }

    double out_mx = 0, out_my = 0;
    for (int32_t i = 0; i < n; ++i) {
        out_mx += st[i].mass * out[i].vx;
        out_my += st[i].mass * out[i].vy;
    }
    assert_finite(ctx, out_mx, "output momentum");
    assert_finite(ctx, out_my, "output momentum");
    if (diag) {
        diag->input_mass = in_mass;
        diag->grid_mass = gmass;
        diag->output_mass = in_mass;
        diag->input_mx = in_mx;
        diag->input_my = in_my;
        diag->grid_mx = gmx;
        diag->grid_my = gmy;
        diag->output_mx = out_mx;
        diag->output_my = out_my;
    }
    return 0;
}

typedef struct {
    grid_t grid;
    int32_t *starts;
    state_t *st;
    orc_particle *scratch;
    int32_t n;
} work_t;

static int work_prepare(work_t *w, const orc_config *cfg, int32_t n)
{
    int64_t count = ((int64_t)cfg->cells_x + 3) * ((int64_t)cfg->cells_y + 3);
    if (cfg->cells_x < 1 || cfg->cells_y < 1 || count > ((int64_t)1 << 31)) return 0;
    memset(w, 0, sizeof(*w));
    if (!grid_alloc(&w->grid, count)) return 0;
    w->starts = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    w->st = (state_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(state_t));
    w->scratch = (orc_particle *)malloc((size_t)(n > 0 ? n : 1) * sizeof(orc_particle));
    w->n = n;
    return w->starts && w->st && w->scratch;
}

static void work_free(work_t *w)
{
    grid_free(&w->grid);
    free(w->starts);
    free(w->st);
    free(w->scratch);
}

int orc_step(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
             const orc_particle *in, orc_particle *out, int32_t n, const orc_bond *bonds,
             orc_bond *bonds_out, orc_diag *diag, char *err, int32_t err_len)
{
    work_t w;
    ctx_t ctx;
    ctx.err = err;
    ctx.err_len = err_len;
    if (err && err_len > 0) err[0] = 0;
    if (!work_prepare(&w, cfg, n)) {
        work_free(&w);
        if (err && err_len > 0) snprintf(err, (size_t)err_len, "grid dimensions exceed the oracle's dense grid");
        return 1;
    }
    orc_bond *tmp_bonds = NULL;
    int32_t nbonds = cfg->has_fracture_bonds ? cfg->n_bonds : 0;
    if (nbonds > 0) {
        tmp_bonds = (orc_bond *)malloc((size_t)nbonds * sizeof(orc_bond));
        memcpy(tmp_bonds, bonds, (size_t)nbonds * sizeof(orc_bond));
    }
    if (setjmp(ctx.jump)) {
        free(tmp_bonds);
        work_free(&w);
        return 1;
    }
    step_impl(&ctx, &w.grid, mats, n_mats, cfg, in, w.scratch, n, tmp_bonds ? tmp_bonds : bonds,
              tmp_bonds, diag, w.starts, w.st);
    memcpy(out, w.scratch, (size_t)n * sizeof(orc_particle));
    if (nbonds > 0 && bonds_out) memcpy(bonds_out, tmp_bonds, (size_t)nbonds * sizeof(orc_bond));
    free(tmp_bonds);
    work_free(&w);
    return 0;
}

int32_t orc_run(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
                orc_particle *particles, int32_t n, orc_bond *bonds, int32_t steps, char *err,
                int32_t err_len)
{
    work_t w;
    ctx_t ctx;
    ctx.err = err;
    ctx.err_len = err_len;
    if (err && err_len > 0) err[0] = 0;
    if (!work_prepare(&w, cfg, n)) {
        work_free(&w);
        if (err && err_len > 0) snprintf(err, (size_t)err_len, "grid dimensions exceed the oracle's dense grid");
        return 0;
    }
    volatile int32_t done = 0;
    if (setjmp(ctx.jump)) {
        work_free(&w);
        return done;
    }
    for (int32_t s = 0; s < steps; ++s) {
        step_impl(&ctx, &w.grid, mats, n_mats, cfg, particles, w.scratch, n, bonds, bonds, NULL,
                  w.starts, w.st);
        memcpy(particles, w.scratch, (size_t)n * sizeof(orc_particle));
        done = s + 1;
    }
    work_free(&w);
    return done;
}

/* The bonded-triangle field of the given particles (buildTriangleField,
 * src/lib/mpm/reference/solver.ts:1064-1165), dense over the halo nodes:
 * per node the signed distance (the band where no body is near), the body's
 * first-vertex index (-1: none), the normal and the three barycentric
 * weights.  Returns 0, or 1 with the reference's message in err. */
int orc_triangle_field(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
                       const orc_particle *particles, int32_t n, double *sd, int32_t *body, double *normal,
                       double *bary, char *err, int32_t err_len)
{
    work_t w;
    ctx_t ctx;
    ctx.err = err;
    ctx.err_len = err_len;
    if (err && err_len > 0) err[0] = 0;
    if (!work_prepare(&w, cfg, n)) {
        work_free(&w);
        if (err && err_len > 0) snprintf(err, (size_t)err_len, "grid dimensions exceed the oracle's dense grid");
        return 1;
    }
    if (setjmp(ctx.jump)) {
        work_free(&w);
        return 1;
    }
    vcfg_t v;
    validate_config(&ctx, mats, n_mats, cfg, &v);
    validate_particles(&ctx, mats, n_mats, particles, n, &v);
    int32_t nb = collect_body_starts(&ctx, mats, n_mats, particles, n, &v, w.starts);
    grid_begin(&w.grid);
    build_triangle_field(&ctx, &w.grid, w.starts, nb, particles, &v);
    double band = v.cell_size * TRIANGLE_FIELD_BAND_CELLS;
    for (int64_t k = 0; k < v.node_count; ++k) {
        field_t *f = field_get(&w.grid, k);
        sd[k] = f ? f->signed_distance : band;
        body[k] = f ? f->body_start : -1;
        normal[2 * k] = f ? f->nx : 0;
        normal[2 * k + 1] = f ? f->ny : 0;
        for (int j = 0; j < 3; ++j) bary[3 * k + j] = f ? f->bary[j] : 0;
    }
    work_free(&w);
    return 0;
}

int32_t orc_sizeof_particle(void) { return (int32_t)sizeof(orc_particle); }
int32_t orc_sizeof_material(void) { return (int32_t)sizeof(orc_material); }
int32_t orc_sizeof_bond(void) { return (int32_t)sizeof(orc_bond); }
int32_t orc_sizeof_config(void) { return (int32_t)sizeof(orc_config); }
