// Allocation-free form of sx_bool_eval.
//
// Some callers cannot allocate device memory themselves.  A host
// application may own the whole device heap under a fixed budget and give
// plugins no allocator.  Or a latency-critical loop may not accept the
// implicit device-wide synchronisation that cudaMalloc and cudaFree can
// cause.  Such callers also cannot provide the caller-owned workspace that
// sx_bool_eval needs for its look-back state.
//
// sx_bool_eval_static keeps that state in a fixed array in this library's
// own device memory: a file-scope __device__ array that every GPU loading
// the library holds until the process exits.  The caller still passes its
// inputs and outputs; nothing here allocates.
//
// Host code must not use the array's name as a device address.  In host
// code the name refers to a host-side stand-in: a kernel given it would
// fault or, where the GPU can reach host memory, use the wrong memory.  The
// real device address is fetched once per device with
// cudaGetSymbolAddress, with that device current, on the first call made
// on it (so that first call should come before any stream capture).  The
// address is kept together with the CUDA context it was fetched in; after a
// device reset, or when the primary context was destroyed and created
// again, the next call sees a different context and fetches it anew instead
// of writing through a stale address.

#include <cstdio>
#include <mutex>

#include "../../include/subsetix_b200.h"
#include "sx_internal.cuh"

// 1 MiB: look-back state for up to 123,264 tiles of 32 rows, i.e. inputs of
// at most 3,944,448 aligned rows.
#define SX_STATIC_SCRATCH_BYTES (1u << 20)
#define SX_STATIC_MAX_ROWS 3944448
#define SX_STATIC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char sx_static_scratch[SX_STATIC_SCRATCH_BYTES];

namespace {

std::mutex g_static_mutex;
void* g_static_ptr[SX_STATIC_MAX_DEVICES] = {nullptr};
void* g_static_ctx[SX_STATIC_MAX_DEVICES] = {nullptr};

// The current driver context, reached through the runtime's entry-point
// query so that the library needs no link against the driver library.
typedef int (*CtxGetCurrentFn)(void**);

void* current_context()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (CtxGetCurrentFn)p;
        looked = true;
    }
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

}  // namespace

extern "C" int sx_bool_eval_static(const sx_leaf* leaves, int k, int32_t rows, const uint32_t* table, int mode,
                                   int32_t* out_begin, int32_t* out_end, int32_t* out_offsets, int64_t capacity,
                                   int32_t* result, void* stream)
{
    if (rows < 0 || rows > SX_STATIC_MAX_ROWS) {
        char msg[160];
        snprintf(msg, sizeof(msg), "sx_bool_eval_static: %d rows outside [0, %d], the limit of the built-in scratch",
                 rows, SX_STATIC_MAX_ROWS);
        return sx_set_error(SX_ERR_CAPACITY, msg);
    }
    if (sx_sweep_state_bytes(sx_sweep_tiles(rows < 1 ? 1 : rows)) > SX_STATIC_SCRATCH_BYTES) {
        return sx_set_error(SX_ERR_CAPACITY, "sx_bool_eval_static: built-in scratch too small");
    }
    int dev = -1;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= SX_STATIC_MAX_DEVICES) {
        char msg[160];
        snprintf(msg, sizeof(msg), "sx_bool_eval_static: no usable current device (%s)", cudaGetErrorString(err));
        return sx_set_error(SX_ERR_CUDA, msg);
    }
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mutex);
        if (g_static_ptr[dev]) {
            // a cached address is valid only in the context it was fetched in
            void* ctx = current_context();
            if (ctx != g_static_ctx[dev]) g_static_ptr[dev] = nullptr;
        }
        if (!g_static_ptr[dev]) {
            // once per device (and context), with that device current
            err = cudaGetSymbolAddress(&g_static_ptr[dev], sx_static_scratch);
            if (err != cudaSuccess) {
                g_static_ptr[dev] = nullptr;
                char msg[160];
                snprintf(msg, sizeof(msg), "sx_bool_eval_static: cudaGetSymbolAddress: %s", cudaGetErrorString(err));
                return sx_set_error(SX_ERR_CUDA, msg);
            }
            g_static_ctx[dev] = current_context();
        }
        scratch = g_static_ptr[dev];
    }
    // The look-back state is cleared on `stream` inside the launch
    // (cudaMemsetAsync), so each call starts from zero.  Calls that overlap
    // on the GPU share this one array and race.
    return sx_bool_eval(leaves, k, rows, table, mode, out_begin, out_end, out_offsets, capacity, result, scratch,
                        SX_STATIC_SCRATCH_BYTES, nullptr, stream);
}
