// Internal argument structures and launch entry points shared by the
// kernel files and the C ABI layer (sx_api.cu).
#pragma once

#include "sx_common.cuh"

struct SxLeafDev {
    const int* begin;
    const int* end;
    const int* off;  // aligned row offsets, length rows + 1
    int widen;       // begin - widen, end + widen on load (0 for set operations)
};

struct SxBoolArgs {
    SxLeafDev leaf[SX_MAX_LEAVES];
    int k;
    int rows;
    int tile_weight;
    int row_weight;
    int elem_cap;
    int row_cap;
    unsigned table[8];  // truth table over the k-bit membership state (bit l = leaf l)
    int func_or;        // 1: f = any leaf (ignores table)
    int* out_begin;
    int* out_end;
    int* out_off;
    long long capacity;
    int* result;  // written by the last block: [0] total intervals, [1] SXF_* flags
    SxScanState scan;
    // launch tuning (0 = automatic): kernel 1 = global-memory sweep, 2 = staged
    // sweep; blocks_per_sm caps residency (via shared-memory padding);
    // staging_cap is the staged kernel's per-warp element capacity
    int tune_kernel;
    int tune_blocks_per_sm;
    int tune_staging_cap;
};

struct SxRowList {
    const int* rows;
    const int* off;  // row offsets of the list's set (length count + 1); needed when skip_empty
    int count;
    int shift;
    int skip_empty;
};

struct SxAlignArgs {
    SxRowList list[SX_MAX_LEAVES * 2];
    int k;
    int row_min;
    long long nbits;
    unsigned* bitmap;  // [nwords]
    int* wcount;       // [nwords]
    int* wprefix;      // [nwords + 1]
    int* rows_out;     // capacity = sum of counts
    int* aligned[SX_MAX_LEAVES * 2];  // per list, [rows_out + 1]; null to skip
    int* result;       // [0] rows_out count, [1] flags
};

cudaError_t sx_sweep_launch(const SxBoolArgs& A, bool union_mode, void* workspace, cudaStream_t stream);
size_t sx_sweep_state_bytes(long long tiles);
long long sx_sweep_tiles(int rows);
cudaError_t sx_scan_i32_launch(const int* in, long long n, int* out, int* result, const SxScanState& st,
                               cudaStream_t stream);
int sx_scan_tiles(long long n);
cudaError_t sx_exact_setop_launch(int op, int rows, const int* lb, const int* le, const int* loff, const int* rb,
                                  const int* re, const int* roff, int* counts, const int* offsets, int* ob, int* oe,
                                  cudaStream_t stream);
cudaError_t sx_merge_rows_launch(int rows, const int* b, const int* e, const int* off, int* counts, const int* out_off,
                                 int* ob, int* oe, cudaStream_t stream);
cudaError_t sx_align_launch(SxAlignArgs& A, int out_capacity, const SxScanState& st, cudaStream_t stream);

// Records `msg` as the calling thread's sx_last_error() text and returns `code`.
int sx_set_error(int code, const char* msg);
