// mpm_kernels.cuh -- kernel entry points of one MLS-MPM substep on B200.
//
// Data layout in HBM (all per-particle arrays are SoA, 16-byte aligned):
//   particle state (ping-pong A/B): pos float2, vel float2, C float4, F float4,
//     plastic volume float, damage float           -> 56 B read + 56 B write
//   particle constants: volume float, material index u32, object id u32,
//     bonded-vertex marker u32 (1-based like the reference record word 19)
//   cell sort (gather P2G): key u32, rank u32, scratch index u32, permutation
//     u32, P2G record 40 B (float4 fx,fy,m,V | float4 m*vx,m*vy,A00,A01 |
//     float2 A10,A11) stored in sorted order
//   halo grid, (cellsX+3) x (cellsY+3) nodes, row-major by (y+1)*W + (x+1):
//     per-cell count/start u32; P2G sums 3 x float4 (solid m,px,py,- |
//     water m,px,py,V | oil m,px,py,V); updated velocities solid float2,
//     water float4 (vx,vy,mass_l,vol_l), oil float4; fixed-point words
//     11 x i32; one stamp u32 per 16x8 node tile marks tiles touched this
//     substep so that untouched tiles are never cleared nor read.
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
};

struct Ctx {
    const StepParams *P;
    ParticleBuffers in;
    ParticleBuffers out;
    const float *vol;
    const uint32_t *mat;
    const Material *mats;
    const uint32_t *bonded;
    const uint32_t *obj;
    uint32_t *status;
    uint32_t *counters;
    // cell sort
    uint32_t *keys;
    uint32_t *ranks;
    uint32_t *tmp;
    uint32_t *perm;
    uint32_t *cell_count;
    uint32_t *cell_start;
    uint32_t *block_sums;
    uint32_t cell_pad;  // padded length of cell_count (multiple of SCAN_CHUNK)
    float4 *rec0;
    float4 *rec1;
    float2 *rec2;
    // grid
    float4 *p2g_solid;
    float4 *p2g_water;
    float4 *p2g_oil;
    float2 *g_solid;
    float4 *g_water;
    float4 *g_oil;
    int32_t *fixed;
    uint32_t *tile_stamp;
    float4 *affine_out;  // optional: prepared affine per particle (parity checks)
};

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;
constexpr int SCAN_TOP_THREADS = 1024;

__global__ void k_count(Ctx c);
__global__ void k_scan_reduce(Ctx c, uint32_t n_chunks);
__global__ void k_scan_top(Ctx c, uint32_t n_chunks);
__global__ void k_scan_apply(Ctx c, uint32_t n_chunks);
__global__ void k_scatter(Ctx c);
__global__ void k_rank_prepare(Ctx c);
__global__ void k_p2g_gather(Ctx c);
__global__ void k_prepare_scatter(Ctx c);
__global__ void k_fixed_decode(Ctx c);
__global__ void k_grid_update(Ctx c);
__global__ void k_g2p(Ctx c);
__global__ void k_commit(Ctx c);
__global__ void k_speed_max(Ctx c);
__global__ void k_begin_batch(Ctx c, uint32_t reset_progress);
__global__ void k_count_active_nodes(Ctx c, uint32_t *counts);

}  // namespace mpm
