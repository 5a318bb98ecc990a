// noalloc.cu -- beat_b200_resolve_noalloc: re-apply the current LU factors
// to new right-hand sides without allocating any device memory.
//
// Who needs it: a caller whose device memory is owned by its own pool (the
// Julia worker's CUDA.jl allocator keeps its own accounting of free memory,
// which a library-side cudaMalloc bypasses and can push into out-of-memory),
// and a caller that cannot afford cudaMalloc/cudaFree on its thread
// (cudaFree synchronises the whole device).  Such a caller passes every input
// and output buffer itself; the only other memory this entry point touches is
// the context's factors, made by an earlier beat_b200_solve.
//
// The block substitution needs a claim counter and one flag per 64-row
// block.  Here they live in g_resolve_scratch, a file-scope __device__ array:
// every GPU that loads this library holds its 16 KB until the process exits.
// Host code must not use the symbol's host-side name as a device pointer; the
// device address is looked up once per device with cudaGetSymbolAddress (on
// the first call on that device, with that device current) and passed to the
// kernels.  The looked-up address is kept for the life of the process; a
// cudaDeviceReset of the device would invalidate it, and callers are told not
// to call this entry point on a device after resetting it.
// All calls on a device share the one array: the entry point clears
// it at the start of every call, and calls whose work overlaps on the GPU
// (other threads, other streams or other contexts on the same device) race on
// it, so they must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <new>

#include "internal.cuh"

namespace bb {
void lu_resolve_into(beat_b200_ctx *c, int R, const double *b, double *x, int *scratch);
}

using namespace bb;

namespace {

// claim counter (32 ints, first used) + one flag per 64-row block
constexpr int RESOLVE_MAX_BLOCKS = 4096;                      // N <= 4096 * 64 = 262,144 unknowns
constexpr int RESOLVE_SCRATCH_INTS = RESOLVE_MAX_BLOCKS + 32;  // 16,512 bytes

__device__ __align__(256) int g_resolve_scratch[RESOLVE_SCRATCH_INTS];

constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mu;
int *g_addr[MAX_DEVICES] = {};

// device address of g_resolve_scratch on `device` (which must be current)
int *scratch_address(int device) {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    BB_REQUIRE(device >= 0 && device < MAX_DEVICES, BEAT_B200_INVALID_ARG, "device ordinal out of range");
    if (!g_addr[device]) {
        void *p = nullptr;
        BB_CUDA(cudaGetSymbolAddress(&p, g_resolve_scratch));
        BB_REQUIRE(p != nullptr, BEAT_B200_CUDA_ERROR, "cudaGetSymbolAddress returned a null address");
        g_addr[device] = static_cast<int *>(p);
    }
    return g_addr[device];
}

}  // namespace

extern "C" int32_t beat_b200_resolve_noalloc(beat_b200_ctx *c, int32_t R, const void *d_b, void *d_x) {
    if (!c) return BEAT_B200_INVALID_ARG;
    try {
        BB_CUDA(cudaSetDevice(c->device));
        BB_REQUIRE(c->F > 0, BEAT_B200_STATE, "no mesh: call beat_b200_set_mesh first");
        BB_REQUIRE(c->ws.lu_valid, BEAT_B200_STATE,
                   "no current factorisation: call beat_b200_solve (or beat_b200_solve_device) first");
        BB_REQUIRE(R >= 1, BEAT_B200_INVALID_ARG, "R must be >= 1");
        BB_REQUIRE(d_b && d_x, BEAT_B200_INVALID_ARG,
                   "d_b and d_x must be non-null device buffers of N x R complex doubles");
        // the row permutation reads b while it writes x: the ranges must not overlap
        const uintptr_t span = (uintptr_t)c->V * (uintptr_t)R * 16u;
        const uintptr_t ub = (uintptr_t)d_b, ux = (uintptr_t)d_x;
        BB_REQUIRE(ub + span <= ux || ux + span <= ub, BEAT_B200_INVALID_ARG,
                   "d_b and d_x overlap: they must be separate N x R complex-double buffers");
        const int nblk = (c->V + 63) / 64;
        BB_REQUIRE(nblk <= RESOLVE_MAX_BLOCKS, BEAT_B200_INVALID_ARG,
                   "beat_b200_resolve_noalloc supports at most 262144 unknowns (its static scratch holds "
                   "4096 block flags); this system has " + std::to_string(c->V));
        int *scratch = scratch_address(c->device);
        BB_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
        lu_resolve_into(c, R, static_cast<const double *>(d_b), static_cast<double *>(d_x), scratch);
        const int st = read_status(c);  // synchronises the context's stream
        BB_REQUIRE(!(st & DEV_BARRIER_TIMEOUT), BEAT_B200_TIMEOUT,
                   "triangular solve: a block wait ran out of its budget");
        c->last_error.clear();
        return BEAT_B200_OK;
    } catch (const Error &e) {
        c->last_error = e.msg;
        cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc &) {
        c->last_error = "host allocation failed";
        return BEAT_B200_OOM;
    } catch (...) {
        c->last_error = "unexpected exception";
        return BEAT_B200_CUDA_ERROR;
    }
}
