// Shared device utilities for the subsetix B200 kernels.
//
// * Device flag codes raised by kernels and reported through the C ABI.
// * Single-pass chained scan with decoupled look-back for block tiles.  Tile
//   ids are handed out dynamically.  Every launch clears its own state first
//   (a memset on its stream), so the workspace may hold any earlier scratch.
// * A block-wide exclusive scan.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define SX_MAX_LEAVES 9
#define SX_TABLE_MAX_LEAVES 8
#define SX_BLOCK 256

// Bits of the device flag word that kernels raise.
#define SXF_CONTRACT 1u   // input outside the fast path's contract: rerun the exact path
#define SXF_LONG_TILE 2u  // reserved: a tile exceeded a capacity limit
#define SXF_CAPACITY 4u   // an output would have exceeded the caller's capacity
#define SXF_TIMEOUT 8u    // a bounded wait gave up (look-back predecessor never published)

// Scan state kept in caller workspace.  status[t] holds the published value
// of tile t: bits 0-31 the value, bits 32-33 the kind (1 = tile aggregate,
// 2 = inclusive prefix), bits 34-63 the launch epoch.  counters[0] hands out
// tile tickets, counters[1] counts finished tiles, counters[2] is the epoch
// and counters[3] accumulates the SXF_* flags.
struct SxScanState {
    unsigned long long* status;
    unsigned int* counters;
    int max_tiles;
};

#define SX_EPOCH_MASK 0x3FFFFFFFu
#define SX_KIND_AGG 1ull
#define SX_KIND_PREFIX 2ull
#define SX_LOOKBACK_SPIN_LIMIT (1u << 22)

__device__ __forceinline__ unsigned long long sx_pack(unsigned epoch, unsigned long long kind, int value)
{
    return ((unsigned long long)(epoch & SX_EPOCH_MASK) << 34) | (kind << 32) | (unsigned long long)(unsigned)value;
}

__device__ __forceinline__ void sx_publish(unsigned long long* slot, unsigned long long word)
{
    atomicExch(slot, word);
}

// Thread 0 takes a tile ticket and reads the epoch.  Every thread of the
// block gets both back through shared memory.
__device__ __forceinline__ void sx_ticket(const SxScanState& st, int* s_tile, unsigned* s_epoch)
{
    if (threadIdx.x == 0) {
        *s_tile = (int)atomicAdd(&st.counters[0], 1u);
        *s_epoch = *((volatile unsigned*)&st.counters[2]) & SX_EPOCH_MASK;
    }
    __syncthreads();
}

// Decoupled look-back, run by one full warp.  Returns the exclusive prefix
// of tile `tile` and publishes its inclusive prefix.  Every wait is bounded.
// If a predecessor never publishes, SXF_TIMEOUT is raised in `flags` and its
// value counts as zero, so the kernel always finishes.
__device__ __forceinline__ int sx_lookback_warp(const SxScanState& st, int tile, unsigned epoch, int aggregate,
                                                unsigned& flags)
{
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) sx_publish(&st.status[0], sx_pack(epoch, SX_KIND_PREFIX, aggregate));
        return 0;
    }
    if (lane == 0) sx_publish(&st.status[tile], sx_pack(epoch, SX_KIND_AGG, aggregate));
    int exclusive = 0;
    int pos = tile - 1;
    bool timed_out = false;
    while (true) {
        int t = pos - lane;
        unsigned long long word = 0ull;
        unsigned kind = SX_KIND_PREFIX;  // lanes past tile 0 act as a zero prefix
        int value = 0;
        if (t >= 0) {
            unsigned spins = 0;
            while (true) {
                word = *((volatile unsigned long long*)&st.status[t]);
                unsigned e = (unsigned)(word >> 34) & SX_EPOCH_MASK;
                kind = (unsigned)((word >> 32) & 3ull);
                if (e == epoch && kind != 0) break;
                if (++spins > SX_LOOKBACK_SPIN_LIMIT) {
                    timed_out = true;
                    kind = SX_KIND_PREFIX;
                    word = 0ull;
                    break;
                }
                if (spins > 8) __nanosleep(64);
            }
            value = (int)(unsigned)(word & 0xFFFFFFFFull);
        }
        unsigned prefix_mask = __ballot_sync(0xFFFFFFFFu, kind == SX_KIND_PREFIX);
        int stop_lane = prefix_mask ? (__ffs(prefix_mask) - 1) : 32;
        int contrib = (lane <= stop_lane) ? value : 0;
        for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xFFFFFFFFu, contrib, o);
        exclusive += contrib;
        if (prefix_mask) break;
        pos -= 32;
    }
    if (__any_sync(0xFFFFFFFFu, timed_out)) flags |= SXF_TIMEOUT;
    if (lane == 0) sx_publish(&st.status[tile], sx_pack(epoch, SX_KIND_PREFIX, exclusive + aggregate));
    return exclusive;
}

// End of kernel.  Every block ORs its flags into counters[3].  The last
// block to finish then writes result[0] (the inclusive prefix of the last
// tile, i.e. the grand total) and result[1] (the flags).
__device__ __forceinline__ void sx_retire(const SxScanState& st, unsigned epoch, unsigned block_flags, int* result)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        if (block_flags) atomicOr(&st.counters[3], block_flags);
        __threadfence();
        unsigned prev = atomicAdd(&st.counters[1], 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            unsigned long long last = *((volatile unsigned long long*)&st.status[gridDim.x - 1]);
            unsigned flags = atomicExch(&st.counters[3], 0u);
            if (result) {
                result[0] = (int)(unsigned)(last & 0xFFFFFFFFull);
                result[1] = (int)flags;
            }
            atomicExch(&st.counters[2], (epoch + 1u) & SX_EPOCH_MASK);
        }
    }
}

// Block-wide exclusive scan of one int per thread (blockDim.x == SX_BLOCK).
// Returns the exclusive prefix; *total receives the block total.
__device__ __forceinline__ int sx_block_exclusive_scan(int v, int* s_warp, int* total)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < (SX_BLOCK / 32)) ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (SX_BLOCK / 32)) s_warp[lane] = w;
    }
    __syncthreads();
    int warp_prefix = warp > 0 ? s_warp[warp - 1] : 0;
    int result = warp_prefix + x - v;
    if (total) *total = s_warp[SX_BLOCK / 32 - 1];
    __syncthreads();
    return result;
}

// ---------------------------------------------------------------------------
// The reference's float32 formulas with the contraction its NVRTC build
// applies.  The reference compiles its kernels with NVRTC's default
// --fmad=true, which fuses each multiply into the add that consumes it:
//   upwind  c - dt * (a * du_dx + b * du_dy)  ->  fma(-dt, fma(a, du_dx, b * du_dy), c)
//   |grad|  sqrtf(gx * gx + gy * gy)           ->  sqrt(fma(gx, gx, gy * gy))
// (interval_stencil.py:105-111, regrid.py:196-217; established on a B200 by
// running the reference's own kernels, compiled with its NVRTC options,
// against every candidate grouping: only this one agrees on every cell).
// Float64 has no reference counterpart and rounds every operation once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sx_upwind_update(float c, float du_dx, float du_dy, float a, float b, float dt)
{
    return __fmaf_rn(-dt, __fmaf_rn(a, du_dx, __fmul_rn(b, du_dy)), c);
}

__device__ __forceinline__ double sx_upwind_update(double c, double du_dx, double du_dy, double a, double b, double dt)
{
    return __dsub_rn(c, __dmul_rn(dt, __dadd_rn(__dmul_rn(a, du_dx), __dmul_rn(b, du_dy))));
}

__device__ __forceinline__ float sx_grad_norm(float gx, float gy)
{
    return __fsqrt_rn(__fmaf_rn(gx, gx, __fmul_rn(gy, gy)));
}

