// extern "C" layer: argument checks, workspace layout, error strings.
// Declarations and their reference counterparts: include/subsetix_b200.h.

#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/subsetix_b200.h"
#include "sx_internal.cuh"

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t err, const char* where)
{
    return fail(SX_ERR_CUDA, "%s: %s", where, cudaGetErrorString(err));
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Scan state occupies the front of every workspace: 4 counters, then one
// status word per tile.
size_t scan_state_bytes(long long tiles) { return align256(16 + (size_t)tiles * 8); }

SxScanState scan_state(void* ws, long long tiles)
{
    SxScanState st;
    st.counters = (unsigned int*)ws;
    st.status = (unsigned long long*)((char*)ws + 16);
    st.max_tiles = (int)tiles;
    return st;
}

}  // namespace

extern "C" {

int sx_abi_version(void) { return SX_ABI_VERSION; }

const char* sx_last_error(void) { return g_err; }

size_t sx_bool_workspace_bytes(int32_t rows) { return sx_sweep_state_bytes(sx_sweep_tiles(rows < 1 ? 1 : rows)); }

int sx_bool_eval(const sx_leaf* leaves, int k, int32_t rows, const uint32_t* table, int mode, int32_t* out_begin,
                 int32_t* out_end, int32_t* out_offsets, int64_t capacity, int32_t* result, void* workspace,
                 size_t workspace_bytes, const sx_tuning* tuning, void* stream)
{
    if (mode != SX_MODE_TABLE && mode != SX_MODE_UNION)
        return fail(SX_ERR_INVALID, "sx_bool_eval: unknown mode %d", mode);
    const int kmax = mode == SX_MODE_TABLE ? SX_TABLE_MAX_LEAVES : SX_MAX_LEAVES;
    if (k < 1 || k > kmax) return fail(SX_ERR_INVALID, "sx_bool_eval: k=%d outside [1, %d]", k, kmax);
    if (rows < 0) return fail(SX_ERR_INVALID, "sx_bool_eval: negative row count");
    if (!leaves || !out_offsets || !result) return fail(SX_ERR_INVALID, "sx_bool_eval: null argument");
    if (mode == SX_MODE_TABLE) {
        if (!table) return fail(SX_ERR_INVALID, "sx_bool_eval: missing truth table");
        if (table[0] & 1u) return fail(SX_ERR_INVALID, "sx_bool_eval: f(empty) must be false (unbounded output)");
    }
    if (capacity < 0) return fail(SX_ERR_INVALID, "sx_bool_eval: negative capacity");
    if (rows == 0) return SX_OK;
    if (!workspace || workspace_bytes < sx_bool_workspace_bytes(rows))
        return fail(SX_ERR_WORKSPACE, "sx_bool_eval: workspace needs %zu bytes, got %zu",
                    sx_bool_workspace_bytes(rows), workspace_bytes);
    SxBoolArgs A;
    memset(&A, 0, sizeof(A));
    for (int l = 0; l < k; ++l) {
        if (!leaves[l].row_offsets) return fail(SX_ERR_INVALID, "sx_bool_eval: leaf %d has no offsets", l);
        A.leaf[l].begin = leaves[l].begin;
        A.leaf[l].end = leaves[l].end;
        A.leaf[l].off = leaves[l].row_offsets;
        A.leaf[l].widen = mode == SX_MODE_UNION ? leaves[l].widen : 0;
    }
    A.k = k;
    A.rows = rows;
    for (int i = 0; i < 8; ++i) A.table[i] = table ? table[i] : 0u;
    A.out_begin = out_begin;
    A.out_end = out_end;
    A.out_off = out_offsets;
    A.capacity = capacity;
    A.result = result;
    if (tuning) {
        if (tuning->kernel < 0 || tuning->kernel > 2 || tuning->blocks_per_sm < 0 || tuning->staging_cap < 0)
            return fail(SX_ERR_INVALID, "sx_bool_eval: bad tuning");
        A.tune_kernel = tuning->kernel;
        A.tune_blocks_per_sm = tuning->blocks_per_sm;
        A.tune_staging_cap = tuning->staging_cap;
    }
    cudaError_t err = sx_sweep_launch(A, mode == SX_MODE_UNION, workspace, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_bool_eval");
    return SX_OK;
}

int sx_exact_setop(int op, int32_t rows, const int32_t* lhs_begin, const int32_t* lhs_end, const int32_t* lhs_offsets,
                   const int32_t* rhs_begin, const int32_t* rhs_end, const int32_t* rhs_offsets, int32_t* counts,
                   const int32_t* offsets, int32_t* out_begin, int32_t* out_end, void* stream)
{
    if (op < 0 || op > 2) return fail(SX_ERR_INVALID, "sx_exact_setop: op %d not in {0,1,2}", op);
    if (rows < 0) return fail(SX_ERR_INVALID, "sx_exact_setop: negative row count");
    if (rows == 0) return SX_OK;
    if (!lhs_offsets || !rhs_offsets) return fail(SX_ERR_INVALID, "sx_exact_setop: null offsets");
    if (!out_begin && !counts) return fail(SX_ERR_INVALID, "sx_exact_setop: need counts (count mode) or outputs");
    if (out_begin && (!out_end || !offsets)) return fail(SX_ERR_INVALID, "sx_exact_setop: write mode needs offsets");
    cudaError_t err = sx_exact_setop_launch(op, rows, lhs_begin, lhs_end, lhs_offsets, rhs_begin, rhs_end, rhs_offsets,
                                            counts, offsets, out_begin, out_end, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_exact_setop");
    return SX_OK;
}

int sx_merge_rows(int32_t rows, const int32_t* begin, const int32_t* end, const int32_t* row_offsets, int32_t* counts,
                  const int32_t* out_offsets, int32_t* out_begin, int32_t* out_end, void* stream)
{
    if (rows < 0) return fail(SX_ERR_INVALID, "sx_merge_rows: negative row count");
    if (rows == 0) return SX_OK;
    if (!row_offsets) return fail(SX_ERR_INVALID, "sx_merge_rows: null offsets");
    if (!out_begin && !counts) return fail(SX_ERR_INVALID, "sx_merge_rows: need counts or outputs");
    if (out_begin && (!out_end || !out_offsets)) return fail(SX_ERR_INVALID, "sx_merge_rows: write mode needs offsets");
    cudaError_t err = sx_merge_rows_launch(rows, begin, end, row_offsets, counts, out_offsets, out_begin, out_end,
                                           (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_merge_rows");
    return SX_OK;
}

size_t sx_scan_workspace_bytes(int64_t n) { return scan_state_bytes(sx_scan_tiles(n)); }

int sx_scan_i32(const int32_t* in, int64_t n, int32_t* out, int32_t* result, void* workspace, size_t workspace_bytes,
                void* stream)
{
    if (n < 0) return fail(SX_ERR_INVALID, "sx_scan_i32: negative length");
    if (!out || !result || (n > 0 && !in)) return fail(SX_ERR_INVALID, "sx_scan_i32: null argument");
    const long long tiles = sx_scan_tiles(n);
    if (!workspace || workspace_bytes < scan_state_bytes(tiles))
        return fail(SX_ERR_WORKSPACE, "sx_scan_i32: workspace needs %zu bytes", scan_state_bytes(tiles));
    cudaError_t err = sx_scan_i32_launch(in, n, out, result, scan_state(workspace, tiles), (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_scan_i32");
    return SX_OK;
}

size_t sx_align_workspace_bytes(int32_t row_min, int32_t row_max)
{
    long long nbits = (long long)row_max - row_min + 1;
    if (nbits < 1) nbits = 1;
    long long nwords = (nbits + 31) / 32;
    size_t bytes = scan_state_bytes(sx_scan_tiles(nwords));
    bytes += align256((size_t)nwords * 4);        // bitmap
    bytes += align256((size_t)nwords * 4);        // per-word counts
    bytes += align256((size_t)(nwords + 1) * 4);  // word prefix
    return bytes;
}

int sx_align_rows(const sx_rowlist* lists, int k, int32_t row_min, int32_t row_max, int32_t* rows_out,
                  int32_t out_capacity, int32_t* const* aligned, int32_t* result, void* workspace,
                  size_t workspace_bytes, void* stream)
{
    if (k < 1 || k > 2 * SX_MAX_LEAVES) return fail(SX_ERR_INVALID, "sx_align_rows: k=%d outside [1, %d]", k,
                                                    2 * SX_MAX_LEAVES);
    if (!lists || !rows_out || !result) return fail(SX_ERR_INVALID, "sx_align_rows: null argument");
    if (row_max < row_min) row_max = row_min;
    const size_t need = sx_align_workspace_bytes(row_min, row_max);
    if (!workspace || workspace_bytes < need)
        return fail(SX_ERR_WORKSPACE, "sx_align_rows: workspace needs %zu bytes, got %zu", need, workspace_bytes);
    long long cap_needed = 0;
    SxAlignArgs A;
    memset(&A, 0, sizeof(A));
    for (int l = 0; l < k; ++l) {
        A.list[l].rows = lists[l].rows;
        A.list[l].off = lists[l].row_offsets;
        A.list[l].count = lists[l].count;
        A.list[l].shift = lists[l].shift;
        A.list[l].skip_empty = lists[l].skip_empty;
        if (lists[l].count < 0) return fail(SX_ERR_INVALID, "sx_align_rows: negative count");
        if (lists[l].count > 0 && !lists[l].rows) return fail(SX_ERR_INVALID, "sx_align_rows: null rows");
        if ((lists[l].skip_empty || (aligned && aligned[l])) && !lists[l].row_offsets)
            return fail(SX_ERR_INVALID, "sx_align_rows: list %d needs row offsets", l);
        cap_needed += lists[l].count;
        A.aligned[l] = aligned ? aligned[l] : nullptr;
    }
    long long span = (long long)row_max - row_min + 1;
    if (out_capacity < cap_needed && out_capacity < span)
        return fail(SX_ERR_CAPACITY, "sx_align_rows: capacity %d below %lld", out_capacity,
                    cap_needed < span ? cap_needed : span);
    A.k = k;
    A.row_min = row_min;
    A.nbits = span;
    A.rows_out = rows_out;
    A.result = result;
    const long long nwords = (span + 31) / 32;
    const long long tiles = sx_scan_tiles(nwords);
    char* p = (char*)workspace;
    SxScanState st = scan_state(p, tiles);
    p += scan_state_bytes(tiles);
    A.bitmap = (unsigned*)p;
    p += align256((size_t)nwords * 4);
    A.wcount = (int*)p;
    p += align256((size_t)nwords * 4);
    A.wprefix = (int*)p;
    cudaError_t err = sx_align_launch(A, out_capacity, st, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_align_rows");
    return SX_OK;
}

}  // extern "C"

int sx_set_error(int code, const char* msg) { return fail(code, "%s", msg); }
