// extern "C" layer: argument checks, workspace layout, error strings.
// Declarations and their reference counterparts: include/subsetix_b200.h.

#include <cstdarg>
#include <cstdio>
#include <climits>
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

size_t sx_bool_workspace_bytes(int32_t rows)
{
    const long long r = rows < 1 ? 1 : rows;
    return sx_sweep_state_bytes(r);  // the look-back state of 1-row tiles: every tuning fits
}

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
    const size_t ws_min = sx_sweep_state_bytes(sx_sweep_tiles(rows));
    if (!workspace || workspace_bytes < ws_min)
        return fail(SX_ERR_WORKSPACE, "sx_bool_eval: workspace needs %zu bytes, got %zu", ws_min, workspace_bytes);
    SxBoolArgs A;
    memset(&A, 0, sizeof(A));
    for (int l = 0; l < k; ++l) {
        if (!leaves[l].row_offsets) return fail(SX_ERR_INVALID, "sx_bool_eval: leaf %d has no offsets", l);
        A.leaf[l].begin = leaves[l].begin;
        A.leaf[l].end = leaves[l].end;
        A.leaf[l].off = leaves[l].row_offsets;
        A.leaf[l].widen = mode == SX_MODE_UNION ? leaves[l].widen : 0;
        A.leaf[l].scale = mode == SX_MODE_UNION ? leaves[l].scale : 0;
        A.leaf[l].off_end = leaves[l].row_ends;
        if (leaves[l].row_ends && mode != SX_MODE_UNION)
            return fail(SX_ERR_INVALID, "sx_bool_eval: row_ends is only supported in SX_MODE_UNION");
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
        if (tuning->kernel < 0 || tuning->kernel > 7 || tuning->blocks_per_sm < 0 || tuning->staging_cap < 0 ||
            tuning->warps < 0 || tuning->warps > 8 ||
            tuning->tile_rows < 0 || tuning->tile_rows > 32 || tuning->wait_limit < 0 || tuning->withhold_tile < 0)
            return fail(SX_ERR_INVALID, "sx_bool_eval: bad tuning");
        A.wait_limit = (unsigned)tuning->wait_limit;
        A.withhold_tile = tuning->withhold_tile;
        A.tune_kernel = tuning->kernel;
        A.tune_blocks_per_sm = tuning->blocks_per_sm;
        A.tune_staging_cap = tuning->staging_cap;
        A.tune_warps = tuning->warps;
        A.tune_tile_rows = tuning->tile_rows;
        if (tuning->kernel == 7 && tuning->tile_rows != 0 && tuning->tile_rows != 8 && tuning->tile_rows != 16 &&
            tuning->tile_rows != 32)
            return fail(SX_ERR_INVALID, "sx_bool_eval: bad tuning: kernel 7 sweeps tiles of 8, 16 or 32 rows, got tile_rows=%d",
                        tuning->tile_rows);
    }
    if (mode == SX_MODE_TABLE && A.tune_tile_rows > 0 && (A.tune_kernel == 0 || A.tune_kernel >= 4)) {
        // an explicit tile height is honoured exactly or refused, never changed behind the caller's back
        const int tr = A.tune_kernel == 6 && A.tune_tile_rows > 8 ? 8 : A.tune_tile_rows;
        const size_t need = sx_sweep_state_bytes(((long long)rows + tr - 1) / tr);
        if (need > workspace_bytes)
            return fail(SX_ERR_WORKSPACE, "sx_bool_eval: %d-row tiles need %zu bytes of workspace, got %zu", tr, need,
                        workspace_bytes);
    }
    cudaError_t err = sx_sweep_launch(A, mode == SX_MODE_UNION, workspace, workspace_bytes, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_bool_eval");
    return SX_OK;
}

int sx_tile_boundaries_max(const sx_leaf* leaves, int k, int32_t rows, int32_t tile_rows_a, int32_t tile_rows_b,
                           int32_t* out, void* stream)
{
    if (k < 1 || k > SX_MAX_LEAVES) return fail(SX_ERR_INVALID, "sx_tile_boundaries_max: k=%d outside [1, %d]", k,
                                                SX_MAX_LEAVES);
    if (!leaves || !out) return fail(SX_ERR_INVALID, "sx_tile_boundaries_max: null argument");
    if (rows < 0 || tile_rows_a < 1 || tile_rows_b < 1)
        return fail(SX_ERR_INVALID, "sx_tile_boundaries_max: bad rows or tile heights");
    const int *offs[SX_MAX_LEAVES], *begs[SX_MAX_LEAVES], *ends[SX_MAX_LEAVES];
    for (int l = 0; l < k; ++l) {
        if (!leaves[l].row_offsets) return fail(SX_ERR_INVALID, "sx_tile_boundaries_max: leaf %d has no offsets", l);
        offs[l] = leaves[l].row_offsets;
        begs[l] = leaves[l].begin;
        ends[l] = leaves[l].end;
    }
    if (rows == 0) {
        cudaError_t err = cudaMemsetAsync(out, 0, 3 * sizeof(int32_t), (cudaStream_t)stream);
        return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_tile_boundaries_max");
    }
    cudaError_t err =
        sx_tile_max_launch(offs, begs, ends, k, rows, tile_rows_a, tile_rows_b, out, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_tile_boundaries_max");
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
                  int32_t out_capacity, int32_t* const* aligned, int32_t* const* aligned_ends, int32_t* result,
                  void* workspace,
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
        A.list[l].div = lists[l].div > 1 ? lists[l].div : 1;
        A.list[l].phase = lists[l].phase;
        A.aligned_end[l] = aligned_ends ? aligned_ends[l] : nullptr;
        if (A.aligned_end[l] && !lists[l].row_offsets)
            return fail(SX_ERR_INVALID, "sx_align_rows: list %d needs row offsets for ranges", l);
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

// ---------------------------------------------------------------------------
// Interval fields
// ---------------------------------------------------------------------------

int sx_check_rows(const int32_t* begin, const int32_t* end, const int32_t* row_offsets, int32_t rows, int64_t n,
                  int32_t* flags, void* stream)
{
    if (rows < 0 || n < 0) return fail(SX_ERR_INVALID, "sx_check_rows: negative size");
    if (!flags || (n > 0 && (!begin || !end || !row_offsets))) return fail(SX_ERR_INVALID, "sx_check_rows: null argument");
    if (n > INT32_MAX) return fail(SX_ERR_INVALID, "sx_check_rows: more than 2^31-1 intervals");
    cudaError_t err = sx_check_rows_launch(begin, end, row_offsets, rows, n, flags, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_check_rows");
    return SX_OK;
}

int sx_cell_offsets(const int32_t* begin, const int32_t* end, int64_t n, int32_t* cell_offsets, int32_t* result,
                    void* workspace, size_t workspace_bytes, void* stream)
{
    if (n < 0 || n > INT32_MAX) return fail(SX_ERR_INVALID, "sx_cell_offsets: interval count out of range");
    if (!cell_offsets || !result || (n > 0 && (!begin || !end))) return fail(SX_ERR_INVALID, "sx_cell_offsets: null argument");
    const long long tiles = sx_scan_tiles(n);
    if (!workspace || workspace_bytes < scan_state_bytes(tiles))
        return fail(SX_ERR_WORKSPACE, "sx_cell_offsets: workspace needs %zu bytes", scan_state_bytes(tiles));
    cudaError_t err = sx_cell_offsets_launch(begin, end, n, cell_offsets, result, scan_state(workspace, tiles),
                                             (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_cell_offsets");
    return SX_OK;
}

size_t sx_prolong_set_workspace_bytes(int32_t rows)
{
    const long long r = rows < 1 ? 1 : rows;
    return scan_state_bytes(sx_scan_tiles(r)) + align256((size_t)r * 4) + align256((size_t)(r + 1) * 4);
}

int sx_prolong_set(const int32_t* rows, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                   int32_t row_count, int64_t n, int32_t ratio, int32_t* rows_out, int32_t* offsets_out,
                   int32_t* out_begin, int32_t* out_end, int32_t* result, void* workspace, size_t workspace_bytes,
                   void* stream)
{
    if (ratio < 2) return fail(SX_ERR_INVALID, "sx_prolong_set: ratio must be >= 2 (ratio 1 is the identity)");
    if (row_count < 0 || n < 0) return fail(SX_ERR_INVALID, "sx_prolong_set: negative size");
    if ((long long)row_count * ratio + 1 > INT32_MAX || n * ratio > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_prolong_set: output exceeds int32 indexing");
    if (!result || !offsets_out) return fail(SX_ERR_INVALID, "sx_prolong_set: null argument");
    if (row_count == 0) return SX_OK;
    if (!rows || !row_offsets || !rows_out || (n > 0 && (!begin || !end || !out_begin || !out_end)))
        return fail(SX_ERR_INVALID, "sx_prolong_set: null argument");
    if (!workspace || workspace_bytes < sx_prolong_set_workspace_bytes(row_count))
        return fail(SX_ERR_WORKSPACE, "sx_prolong_set: workspace needs %zu bytes",
                    sx_prolong_set_workspace_bytes(row_count));
    const long long tiles = sx_scan_tiles(row_count);
    char* p = (char*)workspace;
    SxScanState st = scan_state(p, tiles);
    p += scan_state_bytes(tiles);
    int* occupied = (int*)p;
    p += align256((size_t)row_count * 4);
    int* ord = (int*)p;
    cudaError_t err = sx_prolong_set_launch(rows, row_offsets, begin, end, row_count, (int)n, ratio, occupied, ord,
                                            result, st, rows_out, offsets_out, out_begin, out_end,
                                            (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_prolong_set");
    return SX_OK;
}

int sx_prolong_field(int dtype, const int32_t* coarse_row_offsets, int32_t coarse_rows,
                     const int32_t* coarse_cell_offsets, int64_t n, const int32_t* fine_row_offsets,
                     const int32_t* fine_cell_offsets, int32_t ratio, const void* coarse_values, void* fine_values,
                     void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_prolong_field: dtype %d", dtype);
    if (ratio < 1) return fail(SX_ERR_INVALID, "sx_prolong_field: ratio must be >= 1");
    if (coarse_rows < 0 || n < 0 || n > INT32_MAX || (long long)coarse_rows * ratio > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_prolong_field: bad size");
    if (n == 0 || coarse_rows == 0) return SX_OK;
    if (!coarse_row_offsets || !coarse_cell_offsets || !fine_row_offsets || !fine_cell_offsets || !coarse_values ||
        !fine_values)
        return fail(SX_ERR_INVALID, "sx_prolong_field: null argument");
    cudaError_t err = sx_prolong_field_launch(coarse_row_offsets, coarse_rows, coarse_cell_offsets, (int)n,
                                              fine_row_offsets, fine_cell_offsets, ratio, coarse_values, fine_values,
                                              dtype == SX_F64, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_prolong_field");
    return SX_OK;
}

int sx_prolong_field_f32(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                         int64_t n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets, int32_t ratio,
                         const float* coarse_values, float* fine_values, void* stream)
{
    return sx_prolong_field(SX_F32, coarse_row_offsets, coarse_rows, coarse_cell_offsets, n, fine_row_offsets,
                            fine_cell_offsets, ratio, coarse_values, fine_values, stream);
}

int sx_prolong_field_f64(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                         int64_t n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets, int32_t ratio,
                         const double* coarse_values, double* fine_values, void* stream)
{
    return sx_prolong_field(SX_F64, coarse_row_offsets, coarse_rows, coarse_cell_offsets, n, fine_row_offsets,
                            fine_cell_offsets, ratio, coarse_values, fine_values, stream);
}

int sx_coarse_fine_check(const int32_t* coarse_rows, int32_t coarse_row_count, const int32_t* coarse_row_offsets,
                         const int32_t* coarse_begin, const int32_t* coarse_end, int64_t coarse_n,
                         const int32_t* fine_rows, int32_t fine_row_count, const int32_t* fine_row_offsets,
                         const int32_t* fine_begin, const int32_t* fine_end, int64_t fine_n, int32_t ratio,
                         int32_t* flags, void* stream)
{
    if (ratio < 1) return fail(SX_ERR_INVALID, "sx_coarse_fine_check: ratio must be >= 1");
    if (coarse_row_count < 0 || fine_row_count < 0 || coarse_n < 0 || fine_n < 0 || coarse_n > INT32_MAX ||
        fine_n > INT32_MAX || (long long)coarse_row_count * ratio > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_coarse_fine_check: bad size");
    if (!flags) return fail(SX_ERR_INVALID, "sx_coarse_fine_check: null flags");
    cudaError_t err = cudaMemsetAsync(flags, 0, sizeof(int32_t), (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_coarse_fine_check");
    if (coarse_row_count == 0 && fine_row_count == 0) return SX_OK;
    err = sx_restrict_check_launch(coarse_rows, coarse_row_count, coarse_row_offsets, coarse_begin, coarse_end,
                                   (int)coarse_n, fine_rows, fine_row_count, fine_row_offsets, fine_begin, fine_end,
                                   (int)fine_n, ratio, flags, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_coarse_fine_check");
    return SX_OK;
}

int sx_restrict_field(int dtype, const int32_t* coarse_row_offsets, int32_t coarse_rows,
                      const int32_t* coarse_cell_offsets, int64_t coarse_n, const int32_t* fine_row_offsets,
                      const int32_t* fine_cell_offsets, int32_t ratio, int reducer, const void* fine_values,
                      void* coarse_values, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_restrict_field: dtype %d", dtype);
    if (ratio < 1) return fail(SX_ERR_INVALID, "sx_restrict_field: ratio must be >= 1");
    if (reducer < 0 || reducer > 3) return fail(SX_ERR_INVALID, "sx_restrict_field: reducer %d", reducer);
    if (coarse_rows < 0 || coarse_n < 0 || coarse_n > INT32_MAX) return fail(SX_ERR_INVALID, "sx_restrict_field: bad size");
    if (coarse_n == 0 || coarse_rows == 0) return SX_OK;
    if (!coarse_row_offsets || !coarse_cell_offsets || !fine_row_offsets || !fine_cell_offsets || !fine_values ||
        !coarse_values)
        return fail(SX_ERR_INVALID, "sx_restrict_field: null argument");
    // norm = 1 / r^2 rounded once to the value type, as the reference computes it
    const double norm = reducer == 0 ? 1.0 / ((double)ratio * ratio) : 1.0;
    cudaError_t err = sx_restrict_field_launch(coarse_row_offsets, coarse_rows, coarse_cell_offsets, (int)coarse_n,
                                               fine_row_offsets, fine_cell_offsets, ratio, reducer, norm, fine_values,
                                               coarse_values, dtype == SX_F64, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_restrict_field");
    return SX_OK;
}

int sx_restrict_field_f32(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                          int64_t coarse_n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets,
                          int32_t ratio, int reducer, const float* fine_values, float* coarse_values, void* stream)
{
    return sx_restrict_field(SX_F32, coarse_row_offsets, coarse_rows, coarse_cell_offsets, coarse_n, fine_row_offsets,
                             fine_cell_offsets, ratio, reducer, fine_values, coarse_values, stream);
}

int sx_restrict_field_f64(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                          int64_t coarse_n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets,
                          int32_t ratio, int reducer, const double* fine_values, double* coarse_values, void* stream)
{
    return sx_restrict_field(SX_F64, coarse_row_offsets, coarse_rows, coarse_cell_offsets, coarse_n, fine_row_offsets,
                             fine_cell_offsets, ratio, reducer, fine_values, coarse_values, stream);
}

int sx_subset_rows(const int32_t* sub_row_offsets, const int32_t* sub_rows, int32_t sub_row_count, int64_t sub_n,
                   const int32_t* sup_rows, int32_t sup_row_count, int32_t* pos, int32_t* flags, void* stream)
{
    if (sub_row_count < 0 || sup_row_count < 0 || sub_n < 0 || sub_n > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_subset_rows: bad size");
    if (!flags) return fail(SX_ERR_INVALID, "sx_subset_rows: null flags");
    cudaError_t err = cudaMemsetAsync(flags, 0, sizeof(int32_t), (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_subset_rows");
    if (sub_n == 0) return SX_OK;
    if (!sub_row_offsets || !sub_rows || !pos || (sup_row_count > 0 && !sup_rows))
        return fail(SX_ERR_INVALID, "sx_subset_rows: null argument");
    err = sx_subset_rows_launch(sub_row_offsets, sub_rows, sub_row_count, (int)sub_n, sup_rows, sup_row_count, pos,
                                flags, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_subset_rows");
    return SX_OK;
}

int sx_subset_copy(int scatter, int64_t sub_n, const int32_t* pos, const int32_t* sub_begin, const int32_t* sub_end,
                   const int32_t* sub_cell_offsets, const int32_t* sup_row_offsets, const int32_t* sup_begin,
                   const int32_t* sup_end, const int32_t* sup_cell_offsets, int32_t sup_row_count, void* sub_values,
                   void* sup_values, int elem_size, void* stream)
{
    if (scatter != 0 && scatter != 1) return fail(SX_ERR_INVALID, "sx_subset_copy: scatter must be 0 or 1");
    if (elem_size != 1 && elem_size != 4 && elem_size != 8)
        return fail(SX_ERR_INVALID, "sx_subset_copy: element size %d not in {1, 4, 8}", elem_size);
    if (sub_n < 0 || sub_n > INT32_MAX || sup_row_count < 0) return fail(SX_ERR_INVALID, "sx_subset_copy: bad size");
    if (sub_n == 0 || sup_row_count == 0) return SX_OK;
    if (!pos || !sub_begin || !sub_end || !sub_cell_offsets || !sup_row_offsets || !sup_begin || !sup_end ||
        !sup_cell_offsets || !sub_values || !sup_values)
        return fail(SX_ERR_INVALID, "sx_subset_copy: null argument");
    cudaError_t err = sx_subset_copy_launch(scatter, (int)sub_n, pos, sub_begin, sub_end, sub_cell_offsets,
                                            sup_row_offsets, sup_begin, sup_end, sup_cell_offsets, sup_row_count,
                                            sub_values, sup_values, elem_size, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_subset_copy");
    return SX_OK;
}

int sx_row_lookup(const int32_t* rows, int32_t row_count, int32_t height, int32_t* lookup, int32_t* flags,
                  void* stream)
{
    if (row_count < 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_row_lookup: bad size");
    if (!lookup || !flags || (row_count > 0 && !rows)) return fail(SX_ERR_INVALID, "sx_row_lookup: null argument");
    cudaError_t err = cudaMemsetAsync(flags, 0, sizeof(int32_t), (cudaStream_t)stream);
    if (err == cudaSuccess) err = sx_row_lookup_launch(rows, row_count, height, lookup, flags, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_row_lookup");
    return SX_OK;
}

int sx_upwind(int dtype, const int32_t* rows, const int32_t* row_ids, const int32_t* row_offsets, int32_t row_count,
              const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
              const void* values, void* out, int32_t width, int32_t height, double a, double b, double dt, double dx,
              double dy, int direct, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind: dtype %d", dtype);
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_upwind: width and height must be positive");
    if (row_count < 0 || n < 0 || n > INT32_MAX || cells < 0 || cells > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_upwind: bad size");
    if (n == 0 || cells == 0) return SX_OK;
    if (!rows || !row_offsets || !begin || !end || !cell_offsets || !lookup || !values || !out)
        return fail(SX_ERR_INVALID, "sx_upwind: null argument");
    cudaError_t err = sx_upwind_launch(rows, row_ids, row_offsets, row_count, begin, end, cell_offsets, (int)n, cells, lookup,
                                       values, out, width, height, a, b, dt, dx, dy, direct ? 1 : 0, dtype == SX_F64,
                                       (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind");
    return SX_OK;
}

int sx_upwind_plan(const int32_t* begin, const int32_t* end, int64_t n, int32_t* chunk_offsets, int32_t* result,
                   void* workspace, size_t workspace_bytes, void* stream)
{
    if (n < 0 || n > INT32_MAX) return fail(SX_ERR_INVALID, "sx_upwind_plan: bad size");
    if (!chunk_offsets || !result || (n > 0 && (!begin || !end))) return fail(SX_ERR_INVALID, "sx_upwind_plan: null argument");
    const long long tiles = sx_scan_tiles(n);
    if (!workspace || workspace_bytes < scan_state_bytes(tiles))
        return fail(SX_ERR_WORKSPACE, "sx_upwind_plan: workspace needs %zu bytes", scan_state_bytes(tiles));
    cudaError_t err = sx_upwind_plan_launch(begin, end, (int)n, chunk_offsets, result, scan_state(workspace, tiles),
                                            (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_plan");
    return SX_OK;
}

int sx_upwind_plan_fill(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                        const int32_t* end, const int32_t* cell_offsets, int64_t n, const int32_t* chunk_offsets,
                        int64_t chunks, const int32_t* lookup, int32_t height, int32_t* chunk_info, void* stream)
{
    if (row_count < 0 || n < 0 || n > INT32_MAX || chunks < 0 || height <= 0)
        return fail(SX_ERR_INVALID, "sx_upwind_plan_fill: bad size");
    if (n == 0 || chunks == 0) return SX_OK;
    if (!rows || !row_offsets || !begin || !end || !cell_offsets || !chunk_offsets || !lookup || !chunk_info)
        return fail(SX_ERR_INVALID, "sx_upwind_plan_fill: null argument");
    if (((uintptr_t)chunk_info & 15u) != 0) return fail(SX_ERR_INVALID, "sx_upwind_plan_fill: chunk_info must be 16-byte aligned");
    cudaError_t err = sx_upwind_plan_fill_launch(rows, row_offsets, row_count, begin, end, cell_offsets, (int)n,
                                                 chunk_offsets, chunks, lookup, height, chunk_info,
                                                 (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_plan_fill");
    return SX_OK;
}

int sx_upwind_plan_table(const int32_t* begin, const int32_t* end, const int32_t* cell_offsets,
                         const int32_t* chunk_info, int64_t chunks, uint16_t* neighbours, int32_t* status,
                         void* stream)
{
    if (chunks < 0) return fail(SX_ERR_INVALID, "sx_upwind_plan_table: bad size");
    if (!status) return fail(SX_ERR_INVALID, "sx_upwind_plan_table: null status");
    if (chunks > 0 && (!begin || !end || !cell_offsets || !chunk_info || !neighbours))
        return fail(SX_ERR_INVALID, "sx_upwind_plan_table: null argument");
    if (((uintptr_t)chunk_info & 15u) != 0 || ((uintptr_t)neighbours & 1u) != 0)
        return fail(SX_ERR_INVALID, "sx_upwind_plan_table: chunk_info must be 16-byte and neighbours 2-byte aligned");
    cudaError_t err = sx_upwind_table_launch(begin, end, cell_offsets, chunk_info, chunks, neighbours, status,
                                             (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_plan_table");
    return SX_OK;
}

int sx_upwind_chunked(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                      const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks, const int32_t* lookup,
                      const uint16_t* neighbours, const void* values, void* out, int32_t width, int32_t height,
                      double a, double b, double dt, double dx, double dy, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_chunked: dtype %d", dtype);
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_upwind_chunked: width and height must be positive");
    if (chunks < 0) return fail(SX_ERR_INVALID, "sx_upwind_chunked: bad size");
    if (chunks == 0) return SX_OK;
    if (!row_offsets || !begin || !end || !cell_offsets || !chunk_info || !lookup || !values || !out)
        return fail(SX_ERR_INVALID, "sx_upwind_chunked: null argument");
    if (((uintptr_t)chunk_info & 15u) != 0) return fail(SX_ERR_INVALID, "sx_upwind_chunked: chunk_info must be 16-byte aligned");
    if (values == out) return fail(SX_ERR_INVALID, "sx_upwind_chunked: out must not alias values");
    if (((uintptr_t)neighbours & 1u) != 0) return fail(SX_ERR_INVALID, "sx_upwind_chunked: neighbours must be 2-byte aligned");
    cudaError_t err = sx_upwind_chunk_launch(row_offsets, begin, end, cell_offsets, chunk_info, chunks, lookup,
                                             neighbours, values, out, width, height, a, b, dt, dx, dy,
                                             dtype == SX_F64, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_chunked");
    return SX_OK;
}

int sx_upwind_band_table(int dtype, const double* spacing, int32_t nbands, void* table)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_band_table: dtype %d", dtype);
    if (nbands < 0) return fail(SX_ERR_INVALID, "sx_upwind_band_table: negative band count");
    if (nbands == 0) return SX_OK;
    if (!spacing || !table) return fail(SX_ERR_INVALID, "sx_upwind_band_table: null argument");
    for (int q = 0; q < nbands; ++q)
        if (!(spacing[3 * q] > 0.0) || !(spacing[3 * q + 1] > 0.0))
            return fail(SX_ERR_INVALID, "sx_upwind_band_table: band %d has a spacing that is not positive", q);
    sx_upwind_band_table_fill(dtype == SX_F64, spacing, nbands, table);
    return SX_OK;
}

int sx_upwind_chunked_bands(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                            const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks,
                            const int32_t* lookup, const uint16_t* neighbours, const void* values, void* out,
                            int32_t width, int32_t height, double a, double b, const int32_t* row_band,
                            const void* band_table, int32_t nbands, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: dtype %d", dtype);
    if (width <= 0 || height <= 0)
        return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: width and height must be positive");
    if (chunks < 0 || nbands < 0) return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: bad size");
    if (chunks == 0) return SX_OK;
    if (!row_offsets || !begin || !end || !cell_offsets || !chunk_info || !lookup || !values || !out || !row_band ||
        !band_table)
        return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: null argument");
    if (((uintptr_t)chunk_info & 15u) != 0)
        return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: chunk_info must be 16-byte aligned");
    if (values == out) return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: out must not alias values");
    if (((uintptr_t)neighbours & 1u) != 0)
        return fail(SX_ERR_INVALID, "sx_upwind_chunked_bands: neighbours must be 2-byte aligned");
    cudaError_t err = sx_upwind_chunk_bands_launch(row_offsets, begin, end, cell_offsets, chunk_info, chunks, lookup,
                                                   neighbours, values, out, width, height, a, b, row_band, band_table,
                                                   nbands, dtype == SX_F64, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_chunked_bands");
    return SX_OK;
}

int sx_upwind_f32(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                  const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
                  const float* values, float* out, int32_t width, int32_t height, float a, float b, float dt, float dx,
                  float dy, int direct, void* stream)
{
    return sx_upwind(SX_F32, rows, nullptr, row_offsets, row_count, begin, end, cell_offsets, n, cells, lookup, values, out,
                     width, height, a, b, dt, dx, dy, direct, stream);
}

int sx_upwind_f64(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                  const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
                  const double* values, double* out, int32_t width, int32_t height, double a, double b, double dt,
                  double dx, double dy, int direct, void* stream)
{
    return sx_upwind(SX_F64, rows, nullptr, row_offsets, row_count, begin, end, cell_offsets, n, cells, lookup, values, out,
                     width, height, a, b, dt, dx, dy, direct, stream);
}

size_t sx_upwind_adjoint_scratch_bytes(int64_t cells)
{
    return (size_t)sx_upwind_adjoint_parts(cells) * 2 * sizeof(double);
}

int sx_upwind_adjoint(int dtype, const int32_t* rows, const int32_t* row_offsets, int32_t row_count,
                      const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells,
                      const int32_t* lookup, const void* grad_out, const void* values, void* grad_in, int32_t width,
                      int32_t height, double a, double b, double dt, double dx, double dy, int direct,
                      double* grad_velocity, void* scratch, size_t scratch_bytes, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_adjoint: dtype %d", dtype);
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_upwind_adjoint: width and height must be positive");
    if (row_count < 0 || n < 0 || n > INT32_MAX || cells < 0 || cells > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_upwind_adjoint: bad size");
    if (!grad_velocity) return fail(SX_ERR_INVALID, "sx_upwind_adjoint: null grad_velocity");
    if (n == 0 || cells == 0) {
        cudaError_t err = cudaMemsetAsync(grad_velocity, 0, 2 * sizeof(double), (cudaStream_t)stream);
        return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_upwind_adjoint");
    }
    if (!rows || !row_offsets || !begin || !end || !cell_offsets || !lookup || !grad_out || !values || !grad_in)
        return fail(SX_ERR_INVALID, "sx_upwind_adjoint: null argument");
    if (!scratch || scratch_bytes < sx_upwind_adjoint_scratch_bytes(cells))
        return fail(SX_ERR_WORKSPACE, "sx_upwind_adjoint: scratch needs %zu bytes", sx_upwind_adjoint_scratch_bytes(cells));
    cudaError_t err = sx_upwind_adjoint_launch(rows, row_offsets, row_count, begin, end, cell_offsets, (int)n, cells,
                                               lookup, grad_out, values, grad_in, width, height, a, b, dt, dx, dy,
                                               direct ? 1 : 0, dtype == SX_F64, (double*)scratch, grad_velocity,
                                               (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_adjoint");
    return SX_OK;
}

size_t sx_upwind_adjoint_chunked_scratch_bytes(int64_t chunks)
{
    return (size_t)sx_upwind_adjoint_chunk_parts(chunks) * 2 * sizeof(double);
}

int sx_upwind_adjoint_chunked(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                              const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks,
                              const int32_t* lookup, const uint16_t* neighbours, const void* grad_out,
                              const void* values, void* grad_in, int32_t width, int32_t height, double a, double b,
                              double dt, double dx, double dy, double* grad_velocity, void* scratch,
                              size_t scratch_bytes, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: dtype %d", dtype);
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: width and height must be positive");
    if (chunks < 0) return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: bad size");
    if (!grad_velocity) return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: null grad_velocity");
    if (chunks == 0) {
        cudaError_t err = cudaMemsetAsync(grad_velocity, 0, 2 * sizeof(double), (cudaStream_t)stream);
        return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_upwind_adjoint_chunked");
    }
    if (!row_offsets || !begin || !end || !cell_offsets || !chunk_info || !lookup || !grad_out || !values || !grad_in)
        return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: null argument");
    if (((uintptr_t)chunk_info & 15u) != 0)
        return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: chunk_info must be 16-byte aligned");
    if (!scratch || scratch_bytes < sx_upwind_adjoint_chunked_scratch_bytes(chunks))
        return fail(SX_ERR_WORKSPACE, "sx_upwind_adjoint_chunked: scratch needs %zu bytes",
                    sx_upwind_adjoint_chunked_scratch_bytes(chunks));
    if (((uintptr_t)neighbours & 1u) != 0)
        return fail(SX_ERR_INVALID, "sx_upwind_adjoint_chunked: neighbours must be 2-byte aligned");
    cudaError_t err = sx_upwind_adjoint_chunk_launch(row_offsets, begin, end, cell_offsets, chunk_info, chunks, lookup,
                                                     neighbours, grad_out, values, grad_in, width, height, a, b, dt,
                                                     dx, dy,
                                                     dtype == SX_F64, (double*)scratch, grad_velocity,
                                                     (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_adjoint_chunked");
    return SX_OK;
}

int sx_threshold_rle(const float* values, int32_t width, int32_t height, float threshold, int gradient, int32_t* counts,
                     const int32_t* offsets, int32_t* out_begin, int32_t* out_end, void* stream)
{
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_threshold_rle: width and height must be positive");
    if ((long long)width * height > INT32_MAX) return fail(SX_ERR_INVALID, "sx_threshold_rle: grid too large");
    if (!values) return fail(SX_ERR_INVALID, "sx_threshold_rle: null values");
    if (!out_begin && !counts) return fail(SX_ERR_INVALID, "sx_threshold_rle: need counts or outputs");
    if (out_begin && (!out_end || !offsets)) return fail(SX_ERR_INVALID, "sx_threshold_rle: write mode needs offsets");
    cudaError_t err = sx_threshold_launch(values, width, height, threshold, gradient ? 1 : 0, out_begin ? nullptr : counts,
                                          offsets, out_begin, out_end, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_threshold_rle");
    return SX_OK;
}

int sx_gradient_magnitude(const float* values, int32_t width, int32_t height, float* out, void* stream)
{
    if (width <= 0 || height <= 0) return fail(SX_ERR_INVALID, "sx_gradient_magnitude: width and height must be positive");
    if ((long long)width * height > INT32_MAX) return fail(SX_ERR_INVALID, "sx_gradient_magnitude: grid too large");
    if (!values || !out) return fail(SX_ERR_INVALID, "sx_gradient_magnitude: null argument");
    cudaError_t err = sx_gradient_launch(values, width, height, out, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_gradient_magnitude");
    return SX_OK;
}

int sx_gradient_threshold_rle(const float* values, int32_t width, int32_t height, float threshold, int32_t* counts,
                              const int32_t* offsets, int32_t* out_begin, int32_t* out_end, void* stream)
{
    return sx_threshold_rle(values, width, height, threshold, 1, counts, offsets, out_begin, out_end, stream);
}

int sx_locate_cells(const int32_t* rows, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                    int32_t row_count, const int32_t* query_rows, const int32_t* query_cols, int64_t count,
                    int32_t* out, void* stream)
{
    if (row_count < 0 || count < 0) return fail(SX_ERR_INVALID, "sx_locate_cells: negative size");
    if (count == 0) return SX_OK;
    if (!query_rows || !query_cols || !out || (row_count > 0 && (!rows || !row_offsets)))
        return fail(SX_ERR_INVALID, "sx_locate_cells: null argument");
    cudaError_t err = sx_locate_cells_launch(rows, row_offsets, begin, end, row_count, query_rows, query_cols, count,
                                             out, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_locate_cells");
    return SX_OK;
}

int sx_value_runs(int type, const void* values, const int32_t* cell_offsets, int64_t n, const void* target,
                  int32_t* counts, const int32_t* run_offsets, const int32_t* begin, int32_t* out_begin,
                  int32_t* out_end, void* stream)
{
    if (type < SX_VALUE_F32 || type > SX_VALUE_I64) return fail(SX_ERR_INVALID, "sx_value_runs: type %d", type);
    if (n < 0 || n > INT32_MAX) return fail(SX_ERR_INVALID, "sx_value_runs: bad size");
    if (!target) return fail(SX_ERR_INVALID, "sx_value_runs: null target");
    if (n == 0) return SX_OK;
    if (!cell_offsets || (!out_begin && !counts)) return fail(SX_ERR_INVALID, "sx_value_runs: null argument");
    if (out_begin && (!out_end || !run_offsets || !begin))
        return fail(SX_ERR_INVALID, "sx_value_runs: write mode needs run offsets and begins");
    cudaError_t err = sx_value_runs_launch(type, values, cell_offsets, (int)n, target, out_begin ? nullptr : counts,
                                           run_offsets, begin, out_begin, out_end, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_value_runs");
    return SX_OK;
}

int sx_gather_i32(const int32_t* index, int32_t count, const int32_t* src, int32_t* dst, void* stream)
{
    if (count < 0) return fail(SX_ERR_INVALID, "sx_gather_i32: negative count");
    if (count == 0) return SX_OK;
    if (!index || !src || !dst) return fail(SX_ERR_INVALID, "sx_gather_i32: null argument");
    cudaError_t err = sx_gather_i32_launch(index, count, src, dst, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_gather_i32");
    return SX_OK;
}

int sx_cell_quads(int dtype, const int32_t* row_offsets, const int32_t* rows, int32_t row_count,
                  const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int32_t n,
                  const void* values, float dx, float dy, float ox, float oy, float* points, float* out_values,
                  void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_cell_quads: dtype %d", dtype);
    if (n < 0 || row_count < 0) return fail(SX_ERR_INVALID, "sx_cell_quads: negative size");
    if (n == 0) return SX_OK;
    if (row_count == 0 || !row_offsets || !rows || !begin || !end || !cell_offsets || !values || !points ||
        !out_values)
        return fail(SX_ERR_INVALID, "sx_cell_quads: null argument");
    cudaError_t err = sx_cell_quads_launch(dtype, row_offsets, rows, row_count, begin, end, cell_offsets, n, values,
                                           dx, dy, ox, oy, points, out_values, (cudaStream_t)stream);
    return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_cell_quads");
}

static int coupling_check(const char* what, int dtype, long long n)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "%s: dtype must be SX_F32 or SX_F64", what);
    if (n < 0) return fail(SX_ERR_INVALID, "%s: negative count", what);
    return SX_OK;
}

int sx_index_copy(int dtype, int64_t n, const int32_t* dst_idx, const int32_t* src_idx, const void* src, void* dst,
                  void* stream)
{
    if (int rc = coupling_check("sx_index_copy", dtype, n)) return rc;
    if (n == 0) return SX_OK;
    if (!src || !dst) return fail(SX_ERR_INVALID, "sx_index_copy: null value array");
    cudaError_t err = sx_index_copy_launch(dtype, n, dst_idx, src_idx, src, dst, (cudaStream_t)stream);
    return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_index_copy");
}

int sx_index_block_mean(int dtype, int64_t n, int32_t group, double norm, const int32_t* out_idx,
                        const int32_t* in_idx, const void* in, void* out, void* stream)
{
    if (int rc = coupling_check("sx_index_block_mean", dtype, n)) return rc;
    if (n == 0) return SX_OK;
    if (group < 1) return fail(SX_ERR_INVALID, "sx_index_block_mean: group must be positive");
    if (!out_idx || !in_idx || !in || !out) return fail(SX_ERR_INVALID, "sx_index_block_mean: null argument");
    cudaError_t err = sx_index_block_mean_launch(dtype, n, group, norm, out_idx, in_idx, in, out, (cudaStream_t)stream);
    return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_index_block_mean");
}

int sx_index_block_mean_adj(int dtype, int64_t n, int32_t group, double norm, const int32_t* out_idx,
                            const int32_t* in_idx, void* out_bar, void* in_bar, void* stream)
{
    if (int rc = coupling_check("sx_index_block_mean_adj", dtype, n)) return rc;
    if (n == 0) return SX_OK;
    if (group < 1) return fail(SX_ERR_INVALID, "sx_index_block_mean_adj: group must be positive");
    if (!out_idx || !in_idx || !out_bar || !in_bar)
        return fail(SX_ERR_INVALID, "sx_index_block_mean_adj: null argument");
    cudaError_t err =
        sx_index_block_mean_adj_launch(dtype, n, group, norm, out_idx, in_idx, out_bar, in_bar, (cudaStream_t)stream);
    return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_index_block_mean_adj");
}

int sx_index_segment_add(int dtype, int64_t nseg, const int32_t* seg_off, const int32_t* src_idx,
                         const int32_t* dst_idx, void* src, void* dst, int zero_src, void* stream)
{
    if (int rc = coupling_check("sx_index_segment_add", dtype, nseg)) return rc;
    if (nseg == 0) return SX_OK;
    if (!seg_off || !src_idx || !dst_idx || !src || !dst)
        return fail(SX_ERR_INVALID, "sx_index_segment_add: null argument");
    cudaError_t err = sx_index_segment_add_launch(dtype, nseg, seg_off, src_idx, dst_idx, src, dst, zero_src,
                                                  (cudaStream_t)stream);
    return err == cudaSuccess ? SX_OK : cuda_fail(err, "sx_index_segment_add");
}

static int full_grid_check(const char* what, int W, int H, int batch)
{
    if (W <= 0 || H <= 0 || batch <= 0) return fail(SX_ERR_INVALID, "%s: width, height and batch must be positive", what);
    if (H > 65535 || batch > 65535) return fail(SX_ERR_INVALID, "%s: height and batch must not exceed 65535", what);
    if ((long long)W * H * batch > (1ll << 40)) return fail(SX_ERR_INVALID, "%s: grid too large", what);
    return SX_OK;
}

int sx_upwind_full(int dtype, const void* values, void* out, int32_t width, int32_t height, int32_t batch, double a,
                   double b, double dt, double dx, double dy, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_upwind_full: dtype %d", dtype);
    int rc = full_grid_check("sx_upwind_full", width, height, batch);
    if (rc != SX_OK) return rc;
    if (!values || !out || values == out) return fail(SX_ERR_INVALID, "sx_upwind_full: need distinct input and output");
    cudaError_t err = sx_upwind_full_launch(dtype == SX_F64, values, out, width, height, batch, a, b, dt, dx, dy,
                                            (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_upwind_full");
    return SX_OK;
}

int sx_amr_sync_full(int dtype, void* coarse, void* fine, const int8_t* actions, int32_t width, int32_t height,
                     int32_t batch, int32_t ratio, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_amr_sync_full: dtype %d", dtype);
    int rc = full_grid_check("sx_amr_sync_full", width, height, batch);
    if (rc != SX_OK) return rc;
    if (ratio < 1 || (long long)width * ratio > INT32_MAX || (long long)height * ratio > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_amr_sync_full: bad ratio");
    if (!coarse || !fine || !actions) return fail(SX_ERR_INVALID, "sx_amr_sync_full: null argument");
    cudaError_t err = sx_amr_sync_full_launch(dtype == SX_F64, coarse, fine, (const signed char*)actions, width, height,
                                              batch, ratio, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_amr_sync_full");
    return SX_OK;
}

int sx_amr_step_full(int dtype, const void* coarse_in, const void* fine_in, void* coarse_out, void* fine_out,
                     const int8_t* actions, int32_t width, int32_t height, int32_t batch, double a, double b,
                     double dt, double dx_coarse, double dy_coarse, double dx_fine, double dy_fine, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_amr_step_full: dtype %d", dtype);
    int rc = full_grid_check("sx_amr_step_full", width, height, batch);
    if (rc != SX_OK) return rc;
    if ((long long)width * 2 > INT32_MAX || (long long)height * 2 > INT32_MAX)
        return fail(SX_ERR_INVALID, "sx_amr_step_full: grid too large");
    if (!coarse_in || !fine_in || !coarse_out || !fine_out || !actions)
        return fail(SX_ERR_INVALID, "sx_amr_step_full: null argument");
    if (coarse_in == coarse_out || fine_in == fine_out)
        return fail(SX_ERR_INVALID, "sx_amr_step_full: outputs must not alias inputs");
    cudaError_t err = sx_amr_step_full_launch(dtype == SX_F64, coarse_in, fine_in, coarse_out, fine_out,
                                              (const signed char*)actions, width, height, batch, a, b, dt, dx_coarse,
                                              dy_coarse, dx_fine, dy_fine, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_amr_step_full");
    return SX_OK;
}

int sx_amr_regrid_full(int dtype, const void* coarse, uint8_t* tags, int8_t* actions, int32_t width, int32_t height,
                       int32_t batch, float threshold, int32_t padding, int mode, void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_amr_regrid_full: dtype %d", dtype);
    int rc = full_grid_check("sx_amr_regrid_full", width, height, batch);
    if (rc != SX_OK) return rc;
    if (mode != 0 && mode != 1) return fail(SX_ERR_INVALID, "sx_amr_regrid_full: mode must be 0 (von Neumann) or 1 (Moore)");
    if (!coarse || !tags || !actions) return fail(SX_ERR_INVALID, "sx_amr_regrid_full: null argument");
    cudaError_t err = sx_amr_regrid_full_launch(dtype == SX_F64, coarse, tags, (signed char*)actions, width, height,
                                                batch, threshold, padding, mode, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_amr_regrid_full");
    return SX_OK;
}

int sx_mass_integral(int dtype, const void* values, int64_t n, double scale, double* partials, int parts, double* out,
                     void* stream)
{
    if (dtype != SX_F32 && dtype != SX_F64) return fail(SX_ERR_INVALID, "sx_mass_integral: dtype %d", dtype);
    if (n < 0 || parts < 1 || parts > 4096) return fail(SX_ERR_INVALID, "sx_mass_integral: bad size");
    if (!partials || !out || (n > 0 && !values)) return fail(SX_ERR_INVALID, "sx_mass_integral: null argument");
    cudaError_t err = sx_mass_launch(values, n, dtype == SX_F64, scale, partials, parts, out, (cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_fail(err, "sx_mass_integral");
    return SX_OK;
}

int sx_mass_integral_f64(const double* values, int64_t n, double scale, double* partials, int parts, double* out,
                         void* stream)
{
    return sx_mass_integral(SX_F64, values, n, scale, partials, parts, out, stream);
}

}  // extern "C"

int sx_set_error(int code, const char* msg) { return fail(code, "%s", msg); }
