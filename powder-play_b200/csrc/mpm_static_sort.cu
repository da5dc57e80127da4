// mpm_static_sort.cu -- a cell sort that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host whose GPU memory is handed out
// by an embedding application with a fixed budget, a real-time frame loop
// that must not take the implicit device synchronisation of an allocation,
// or a thin foreign-function binding (a JavaScript or WebAssembly host) that
// has no allocator of its own.  mpm_cell_sort_static serves them: it runs the
// same stable counting sort of particles by base cell as the solver's gather
// path (k_count, the three-pass scan, k_scatter, then a stable in-cell
// ranking), but its scratch lives in one file-scope __device__ array whose
// size is fixed at build time.
//
// Limits: at most STATIC_SORT_MAX_PARTICLES particles and
// STATIC_SORT_MAX_NODES halo nodes ((cellsX + 3) * (cellsY + 3)); larger
// requests are rejected with MPM_ERR_INVALID_ARGUMENT.  Every GPU that loads
// the library keeps the array (about 3.5 MiB) until the process exits.
//
// The array is shared by every call on a device and keeps what the last call
// left in it; each call clears the parts that must start at zero.  Calls that
// overlap on the same GPU (from two host threads) race on it: serialise them.
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress and keeps it; make that first call before any stream
// capture.  A cudaDeviceReset (or any teardown of the device's primary
// context) invalidates the kept address: do not call this entry point on that
// device afterwards.  The caller's current device is restored on return.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/mpm_b200.h"
#include "mpm_kernels.cuh"

using namespace mpm;

namespace {

constexpr uint32_t STATIC_SORT_MAX_PARTICLES = 65536u;
constexpr uint32_t STATIC_SORT_MAX_NODES = 262144u;  // a multiple of SCAN_CHUNK
constexpr int STATIC_SORT_MAX_DEVICES = 64;

constexpr size_t align256(size_t v) { return (v + 255u) & ~size_t(255u); }

// byte offsets of the regions inside the scratch array
constexpr size_t OFF_PARAMS = 0;
constexpr size_t OFF_STATUS = align256(OFF_PARAMS + sizeof(StepParams));
constexpr size_t OFF_COUNTERS = align256(OFF_STATUS + 32 * sizeof(uint32_t));
constexpr size_t OFF_POS = align256(OFF_COUNTERS + 32 * sizeof(uint32_t));
constexpr size_t OFF_KEYS = align256(OFF_POS + STATIC_SORT_MAX_PARTICLES * sizeof(float2));
constexpr size_t OFF_RANKS = align256(OFF_KEYS + STATIC_SORT_MAX_PARTICLES * sizeof(uint32_t));
constexpr size_t OFF_TMP = align256(OFF_RANKS + STATIC_SORT_MAX_PARTICLES * sizeof(uint32_t));
constexpr size_t OFF_PERM = align256(OFF_TMP + STATIC_SORT_MAX_PARTICLES * sizeof(uint32_t));
constexpr size_t OFF_COUNT = align256(OFF_PERM + STATIC_SORT_MAX_PARTICLES * sizeof(uint32_t));
constexpr size_t OFF_START = align256(OFF_COUNT + STATIC_SORT_MAX_NODES * sizeof(uint32_t));
constexpr size_t OFF_BLOCKS = align256(OFF_START + (STATIC_SORT_MAX_NODES + 1) * sizeof(uint32_t));
constexpr size_t STATIC_SORT_BYTES =
    align256(OFF_BLOCKS + (STATIC_SORT_MAX_NODES / SCAN_CHUNK + 1) * sizeof(uint32_t));
// k_scan_apply writes cell starts over the whole padded scan range (a
// multiple of SCAN_CHUNK) plus one word: with the maximum a multiple of the
// chunk, that range ends inside the start region
static_assert(STATIC_SORT_MAX_NODES % SCAN_CHUNK == 0, "the node maximum must be a multiple of the scan chunk");
static_assert(OFF_BLOCKS >= OFF_START + (STATIC_SORT_MAX_NODES + 1) * sizeof(uint32_t),
              "the start region must hold the padded scan range and its end word");
static_assert(OFF_START >= OFF_COUNT + STATIC_SORT_MAX_NODES * sizeof(uint32_t), "the count region is too small");

// The scratch.  In host code this name is only a stand-in for the symbol:
// kernels get the address that cudaGetSymbolAddress returns for the current
// device, never the name itself.
static __device__ __align__(256) unsigned char g_static_sort_scratch[STATIC_SORT_BYTES];

unsigned char *g_scratch_address[STATIC_SORT_MAX_DEVICES] = {};

// Copies the message into the caller's buffer (if any) and returns code.
int fail(char *error_out, uint32_t error_capacity, int code, const char *message)
{
    if (error_out && error_capacity > 0) {
        std::strncpy(error_out, message, error_capacity - 1);
        error_out[error_capacity - 1] = 0;
    }
    return code;
}

// The permutation step of the stable counting sort: the particle bucketed
// at slot s moves to its cell's start plus the number of cell members with a
// smaller index.
__global__ void k_static_stable_rank(Ctx c)
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
    c.perm[lo + rank] = i;
}

int sort_on_current_device(int32_t device, uint32_t cells_x, uint32_t cells_y, float cell_size,
                           const float *positions, uint32_t count, uint64_t nodes, uint32_t *keys_out,
                           uint32_t *perm_out, uint32_t *cell_start_out, char *error_out, uint32_t error_capacity);

}  // namespace

extern "C" int mpm_cell_sort_static(int32_t device, uint32_t cells_x, uint32_t cells_y, float cell_size,
                                    const float *positions, uint32_t count, uint32_t *keys_out,
                                    uint32_t *perm_out, uint32_t *cell_start_out, char *error_out,
                                    uint32_t error_capacity)
{
    if (error_out && error_capacity > 0) error_out[0] = 0;
    if (!positions || !keys_out || !perm_out || !cell_start_out)
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT, "positions and outputs must not be NULL");
    if (cells_x < 1 || cells_y < 1 || !(cell_size > 0.0f) || !std::isfinite(cell_size))
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT, "the grid must have positive cell counts and cell size");
    const uint64_t nodes = ((uint64_t)cells_x + 3) * ((uint64_t)cells_y + 3);
    if (nodes > STATIC_SORT_MAX_NODES)
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT,
                    "the grid exceeds the static sort maximum of 262144 halo nodes ((cellsX+3)*(cellsY+3))");
    if (count > STATIC_SORT_MAX_PARTICLES)
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT, "the particle count exceeds the static sort maximum of 65536");
    if (device < 0 || device >= STATIC_SORT_MAX_DEVICES)
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    int previous = -1;
    if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    if (cudaSetDevice(device) != cudaSuccess) return fail(error_out, error_capacity, MPM_ERR_CUDA, "cudaSetDevice failed");
    const int rc = sort_on_current_device(device, cells_x, cells_y, cell_size, positions, count, nodes, keys_out,
                                          perm_out, cell_start_out, error_out, error_capacity);
    if (previous >= 0 && previous != device) cudaSetDevice(previous);
    return rc;
}

namespace {

int sort_on_current_device(int32_t device, uint32_t cells_x, uint32_t cells_y, float cell_size,
                           const float *positions, uint32_t count, uint64_t nodes, uint32_t *keys_out,
                           uint32_t *perm_out, uint32_t *cell_start_out, char *error_out, uint32_t error_capacity)
{

    // one-time set-up on this device (must precede any stream capture)
    if (!g_scratch_address[device]) {
        void *address = nullptr;
        if (cudaGetSymbolAddress(&address, g_static_sort_scratch) != cudaSuccess || !address)
            return fail(error_out, error_capacity, MPM_ERR_CUDA, "cudaGetSymbolAddress of the static sort scratch failed");
        g_scratch_address[device] = static_cast<unsigned char *>(address);
    }
    unsigned char *base = g_scratch_address[device];

    const uint32_t node_count = (uint32_t)nodes;
    const uint32_t cell_pad = ((node_count + SCAN_CHUNK - 1) / SCAN_CHUNK) * SCAN_CHUNK;
    const uint32_t n_chunks = cell_pad / SCAN_CHUNK;
    StepParams params;
    std::memset(&params, 0, sizeof params);
    params.cells_x = cells_x;
    params.cells_y = cells_y;
    params.node_w = cells_x + 3;
    params.node_h = cells_y + 3;
    params.n_particles = count;
    params.n_nodes = node_count;
    params.dx = cell_size;

    Ctx c{};
    c.P = reinterpret_cast<const StepParams *>(base + OFF_PARAMS);
    c.status = reinterpret_cast<uint32_t *>(base + OFF_STATUS);
    c.counters = reinterpret_cast<uint32_t *>(base + OFF_COUNTERS);
    c.in.pos = reinterpret_cast<float2 *>(base + OFF_POS);
    c.keys = reinterpret_cast<uint32_t *>(base + OFF_KEYS);
    c.ranks = reinterpret_cast<uint32_t *>(base + OFF_RANKS);
    c.tmp = reinterpret_cast<uint32_t *>(base + OFF_TMP);
    c.perm = reinterpret_cast<uint32_t *>(base + OFF_PERM);
    c.cell_count = reinterpret_cast<uint32_t *>(base + OFF_COUNT);
    c.cell_start = reinterpret_cast<uint32_t *>(base + OFF_START);
    c.block_sums = reinterpret_cast<uint32_t *>(base + OFF_BLOCKS);
    c.cell_pad = cell_pad;

    const cudaStream_t stream = 0;
    const uint32_t init_status[8] = {0, 0xffffffffu, 0, 0, 0, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(base + OFF_PARAMS, &params, sizeof params, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c.status, init_status, sizeof init_status, cudaMemcpyHostToDevice, stream);
    // the counts must start at zero: clear the whole padded range this call scans
    if (e == cudaSuccess) e = cudaMemsetAsync(c.cell_count, 0, (size_t)cell_pad * sizeof(uint32_t), stream);
    if (e == cudaSuccess && count > 0)
        e = cudaMemcpyAsync(c.in.pos, positions, (size_t)count * sizeof(float2), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return fail(error_out, error_capacity, MPM_ERR_CUDA, cudaGetErrorString(e));

    const unsigned threads = 256;
    const unsigned blocks = count > 0 ? (count + threads - 1) / threads : 1;
    k_count<<<blocks, threads, 0, stream>>>(c);
    k_scan_reduce<<<n_chunks, SCAN_THREADS, 0, stream>>>(c, n_chunks);
    k_scan_top<<<1, SCAN_TOP_THREADS, 0, stream>>>(c, n_chunks);
    k_scan_apply<<<n_chunks, SCAN_THREADS, 0, stream>>>(c, n_chunks);
    k_scatter<<<blocks, threads, 0, stream>>>(c);
    k_static_stable_rank<<<blocks, threads, 0, stream>>>(c);
    e = cudaGetLastError();

    uint32_t status[8] = {};
    if (e == cudaSuccess && count > 0)
        e = cudaMemcpyAsync(keys_out, c.keys, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && count > 0)
        e = cudaMemcpyAsync(perm_out, c.perm, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cell_start_out, c.cell_start, ((size_t)node_count + 1) * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, c.status, sizeof status, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(error_out, error_capacity, MPM_ERR_CUDA, cudaGetErrorString(e));
    if (status[0] != 0u)
        return fail(error_out, error_capacity, MPM_ERR_INVALID_ARGUMENT,
                    "a position is non-finite or its stencil leaves the grid halo (status 1)");
    return MPM_OK;
}

}  // namespace
