/*
 * mpm_oracle.h -- CPU FP64 restatement of the reference CPU MLS-MPM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * The product (powder-play_b200) never links, loads or calls it.
 *
 * It restates `stepMpm` from src/lib/mpm/reference/solver.ts:396-824 of
 * 7korobi/powder-play (P2G :418-479, grid update :500-608, G2P :612-773,
 * triangle contact / bonds :775-791, fracture :792-800 with
 * src/lib/mpm/reference/solid-bonds.ts:72-109).  Numbers are IEEE double as in
 * the JavaScript original.
 *
 * Parity pinning: the reference ships no stored trajectories.  The oracle is
 * pinned by the reference's own property tests and known answers (conservation
 * 1e-12 / 1e-10, wall confinement, Tait-vs-linear ordering, fracture
 * localisation, triangle-contact bounds) which tests/test_oracle_*.py re-run
 * against this code.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Constitutive model codes; 0..4 follow src/lib/mpm/materials.ts:8-16.
 * 5 = fixed-corotated (snow stress with Jp = 1, no plastic projection), a
 * model the reference does not have (used by the adjoint form). */
enum {
    ORC_NEO_HOOKEAN = 0,
    ORC_SNOW = 1,
    ORC_WATER = 2,
    ORC_OIL = 3,
    ORC_POWDER = 4,
    ORC_FIXED_COROTATED = 5
};

typedef struct {
    int32_t model;
    int32_t tait;        /* 1: Tait EOS with `exponent`; 0: legacy linear EOS */
    double lambda;
    double mu;
    double density;      /* liquids only */
    double friction;     /* powder only */
    double exponent;     /* Tait exponent when tait == 1 */
} orc_material;

typedef struct {
    double px, py, vx, vy;
    double c00, c01, c10, c11;
    double f00, f01, f10, f11;
    double damage;          /* valid when has_damage */
    double plastic_volume;  /* 1 when absent */
    double volume;          /* <= 0: use config particle_volume */
    int32_t material;       /* index into the material table; -1: config material */
    int32_t object_id;
    int32_t bonded_vertex;  /* -1: none; 0, 1, 2 */
    int32_t has_damage;
} orc_particle;

typedef struct {
    int32_t first;
    int32_t second;
    double rest_length;
    double failure_strain;
    double damage;
    int32_t broken;
    int32_t pad;
} orc_bond;

typedef struct {
    double dt;
    int32_t cells_x;
    int32_t cells_y;
    double cell_size;
    double particle_mass;
    double particle_volume;
    int32_t has_bond_rest_length;
    int32_t material;           /* default material index */
    double bond_rest_length;
    double bond_stiffness;      /* default 0.35 */
    double bond_reference_dt;   /* <= 0: use dt */
    double gx, gy;
    double wall_friction;
    int32_t n_bonds;            /* fracture bonds; 0 = none */
    int32_t has_fracture_bonds; /* config.fractureBonds !== undefined */
} orc_config;

typedef struct {
    double input_mass, grid_mass, output_mass;
    double input_mx, input_my, grid_mx, grid_my, output_mx, output_my;
} orc_diag;

/* One explicit MLS-MPM step.  `in` and `out` hold n particles; `bonds` holds
 * cfg->n_bonds fracture bonds (read) and `bonds_out` receives their updated
 * state (may alias `bonds`).  Returns 0 on success; on a reference
 * RangeError/TypeError it returns 1 and writes the message into err. */
int orc_step(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
             const orc_particle *in, orc_particle *out, int32_t n,
             const orc_bond *bonds, orc_bond *bonds_out, orc_diag *diag,
             char *err, int32_t err_len);

/* Runs `steps` steps in place with a fixed config (the worker loop of
 * src/lib/mpm/reference/cpu-simulation.worker.ts:71-104 with constant dt and
 * gravity).  Returns the number of steps completed before an error. */
int32_t orc_run(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
                orc_particle *particles, int32_t n, orc_bond *bonds,
                int32_t steps, char *err, int32_t err_len);

/* The bonded-triangle field of `particles`, dense over the halo nodes
 * ((cellsX+3) x (cellsY+3), row-major): signed distance, first-vertex index of
 * the nearest body (-1: none), normal (2 per node), barycentric weights (3 per
 * node).  Returns 0, or 1 with the reference's message in err. */
int orc_triangle_field(const orc_material *mats, int32_t n_mats, const orc_config *cfg,
                       const orc_particle *particles, int32_t n, double *sd, int32_t *body, double *normal,
                       double *bary, char *err, int32_t err_len);

/* The differentiable form in FP64 (adjoint_fp64.c): one scene of Tait water
 * (liquid[i] = 1) and fixed-corotated solid particles. */
typedef struct orc_adj_scene {
    int32_t cells_x, cells_y;
    double dx, dt, gx, gy, solid_mass, wall_friction;
    double rho, gamma, tait, lambda_s, mu_s;
} orc_adj_scene;

/* `steps` substeps from (x0, v0, C0, F0) (2, 2, 4, 4 per particle), the loss
 * sum |x(T) - target|^2, and its gradients with respect to the initial
 * velocities (2 per particle) and (tait, lambda_s, mu_s).  x_out (may be NULL)
 * receives x(T).  Returns 0, -1 when a particle leaves the grid or a value
 * turns non-finite, -2 when memory runs out. */
int orc_adjoint_run(const orc_adj_scene *scene, int32_t n, const double *x0, const double *v0, const double *C0,
                    const double *F0, const double *vol, const int32_t *liquid, const double *target, int32_t steps,
                    double *loss, double *grad_v0, double *grad_params, double *x_out);

/* Sizes of the structs, so a binding can check its layout. */
int32_t orc_sizeof_particle(void);
int32_t orc_sizeof_material(void);
int32_t orc_sizeof_bond(void);
int32_t orc_sizeof_config(void);

#ifdef __cplusplus
}
#endif
#endif
