/*
 * subsetix_b200 — C ABI of the B200 (sm_100a) interval-set AMR kernels.
 *
 * Data model (same as the reference's IntervalSet,
 * subsetix_cupy/expressions.py:144-227): a set is CSR-like over rows,
 * with int32 `row_offsets[R + 1]`, half-open int32 `begin[n]` / `end[n]`
 * and a strictly increasing int32 `rows[R]`.  Intervals are sorted and
 * disjoint inside each row.
 *
 * Conventions for every entry point:
 *   - every pointer is a DEVICE pointer unless its comment says otherwise;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *   - nothing synchronises the host; results that size later work (totals,
 *     flags) are written to a device `result` pair: result[0] = count,
 *     result[1] = SX_FLAG_* bits;
 *   - the return value is an sx_status; on failure sx_last_error() gives a
 *     message for the calling thread;
 *   - `workspace` is caller-owned device scratch of at least the size the
 *     matching *_workspace_bytes() reports.  It needs no initialisation:
 *     every call clears the state it uses on its own stream.  A workspace
 *     must not be shared by calls that may run at the same time on
 *     different streams.
 */
#ifndef SUBSETIX_B200_H
#define SUBSETIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SX_ABI_VERSION 1

typedef enum sx_status {
    SX_OK = 0,
    SX_ERR_INVALID = 1,   /* bad argument (maps to ValueError/TypeError in Python) */
    SX_ERR_CUDA = 2,      /* a CUDA call failed */
    SX_ERR_CAPACITY = 3,  /* caller buffer too small */
    SX_ERR_WORKSPACE = 4  /* workspace too small */
} sx_status;

/* Device flag bits reported in result[1]. */
#define SX_FLAG_CONTRACT 1u  /* input outside the fused path's contract: rerun the exact path */
#define SX_FLAG_LONG_TILE 2u /* a row tile exceeded the shared-memory cap: rerun the exact path */
#define SX_FLAG_CAPACITY 4u  /* output capacity exceeded (outputs truncated) */
#define SX_FLAG_TIMEOUT 8u   /* a bounded device wait gave up (results invalid) */

int sx_abi_version(void);
const char* sx_last_error(void);

/* ---------------------------------------------------------------------------
 * Row-wise boolean evaluation: set algebra, fused expressions and dilation.
 *
 * Replaces: subsetix_cupy/expressions.py:446-528 (_apply_binary with the
 * count_segments / write_segments kernels, subsetix_cupy/kernels.py:11-235),
 * the recursive evaluation of expression trees,
 * subsetix_cupy/expressions.py:351-410 (evaluate, make_union,
 * make_intersection, make_difference, make_symmetric_difference,
 * make_complement), and the sort-and-merge rebuild of dilation,
 * subsetix_cupy/morphology.py:21-107,211-248 with
 * subsetix_cupy/kernels.py:292-381.
 *
 * The k leaves share `rows` aligned rows: their row_offsets are expressed on
 * one common row list (see sx_align_rows).  Each row is swept as a k-way
 * merge of the leaves' boundaries.
 *   mode SX_MODE_TABLE (k <= 8): leaves must be canonical (per row:
 *     non-empty, strictly increasing, non-touching).  `table` is the truth
 *     table of the expression over the k-bit membership state (bit l = leaf
 *     l; bit s of table[s >> 5] is f(s); f(0) must be 0).  Output: the
 *     maximal runs of f.
 *   mode SX_MODE_UNION (k <= 9): leaves are widened by `widen` ([b - w, e + w))
 *     and must have non-empty intervals with strictly increasing begins and
 *     ends per row.  Output: the merged union (runs whose next begin is <=
 *     the running end join).
 * Inputs outside the contract set SX_FLAG_CONTRACT in result[1]; the caller
 * then uses the exact kernels.  Outputs: `out_offsets[rows + 1]`,
 * result = {total, flags}.  A capacity of sum(leaf sizes) always suffices.
 * ------------------------------------------------------------------------- */
#define SX_MODE_TABLE 0
#define SX_MODE_UNION 1

typedef struct sx_leaf {
    const int32_t* begin;
    const int32_t* end;
    const int32_t* row_offsets; /* aligned, rows + 1 entries */
    int32_t widen;
} sx_leaf;

/* Launch tuning for sx_bool_eval; NULL or zero fields select automatic values.
 * kernel: 1 = global-memory sweep, 2 = shared-memory staged sweep (table mode);
 * blocks_per_sm: residency cap of the global sweep; staging_cap: elements per
 * warp of the staged sweep.  Results never depend on the tuning. */
typedef struct sx_tuning {
    int32_t kernel;
    int32_t blocks_per_sm;
    int32_t staging_cap;
} sx_tuning;

size_t sx_bool_workspace_bytes(int32_t rows);
int sx_bool_eval(const sx_leaf* leaves /* host array of k */, int k, int32_t rows, const uint32_t* table /* host, 8 */,
                 int mode, int32_t* out_begin, int32_t* out_end, int32_t* out_offsets, int64_t capacity,
                 int32_t* result, void* workspace, size_t workspace_bytes, const sx_tuning* tuning /* host */,
                 void* stream);

/* ---------------------------------------------------------------------------
 * sx_bool_eval without a caller workspace.  This entry point has no
 * counterpart in the reference; it exists for callers that cannot allocate
 * device memory: a host application that owns the device heap under a fixed
 * budget and gives plugins no allocator, or a latency-critical loop that
 * cannot accept the device-wide synchronisation cudaMalloc/cudaFree may
 * cause.  Inputs and outputs are still the caller's.  The look-back scratch
 * is a fixed 1 MiB array in this library's device memory, which every GPU
 * that loads the library holds until the process exits, so rows must not
 * exceed 3,944,448 (larger inputs fail with SX_ERR_CAPACITY).  Nothing is
 * allocated and the tuning is automatic.
 * The first call on each device looks up the array's device address with
 * that device current; make that first call before any stream capture.
 * Every call shares the one array and clears the part it uses on its own
 * stream, so calls that overlap on the GPU race: serialise them.
 * ------------------------------------------------------------------------- */
int sx_bool_eval_static(const sx_leaf* leaves /* host array of k */, int k, int32_t rows,
                        const uint32_t* table /* host, 8 */, int mode, int32_t* out_begin, int32_t* out_end,
                        int32_t* out_offsets, int64_t capacity, int32_t* result, void* stream);

/* ---------------------------------------------------------------------------
 * Exact reference-order binary operation, one thread per row.
 * Replaces: subsetix_cupy/kernels.py:11-117 (count_segments) when out_begin
 * is NULL, and subsetix_cupy/kernels.py:120-235 (write_segments) otherwise.
 * op: 0 union, 1 intersection, 2 difference.  Operands must be aligned.
 * ------------------------------------------------------------------------- */
int sx_exact_setop(int op, int32_t rows, const int32_t* lhs_begin, const int32_t* lhs_end,
                   const int32_t* lhs_offsets, const int32_t* rhs_begin, const int32_t* rhs_end,
                   const int32_t* rhs_offsets, int32_t* counts, const int32_t* offsets, int32_t* out_begin,
                   int32_t* out_end, void* stream);

/* ---------------------------------------------------------------------------
 * Run merge of rows whose intervals are sorted by begin.
 * Replaces: subsetix_cupy/kernels.py:292-333 (count_merged_segments) when
 * out_begin is NULL, and :336-381 (write_merged_segments) otherwise.
 * ------------------------------------------------------------------------- */
int sx_merge_rows(int32_t rows, const int32_t* begin, const int32_t* end, const int32_t* row_offsets, int32_t* counts,
                  const int32_t* out_offsets, int32_t* out_begin, int32_t* out_end, void* stream);

/* ---------------------------------------------------------------------------
 * Exclusive int32 prefix sum: out[0..n] with out[n] = total, result = {total,
 * flags}.  Replaces the cumsum step of every count/write pair in the
 * reference (e.g. subsetix_cupy/expressions.py:500-503).
 * ------------------------------------------------------------------------- */
size_t sx_scan_workspace_bytes(int64_t n);
int sx_scan_i32(const int32_t* in, int64_t n, int32_t* out, int32_t* result, void* workspace, size_t workspace_bytes,
                void* stream);

/* ---------------------------------------------------------------------------
 * Row alignment: rows_out = sorted union over lists of (rows + shift),
 * optionally skipping empty rows, and aligned[l][y] = list l's offsets
 * re-expressed on rows_out (aligned[l] may be NULL).
 * Replaces: subsetix_cupy/expressions.py:58-141 (_reindex_interval_set,
 * _align_interval_sets) and the row-id construction of dilation,
 * subsetix_cupy/morphology.py:236-247.
 * row_min / row_max bound every (row + shift) that should be kept.
 * result = {number of output rows, flags}.
 * ------------------------------------------------------------------------- */
typedef struct sx_rowlist {
    const int32_t* rows;
    const int32_t* row_offsets; /* count + 1 entries */
    int32_t count;
    int32_t shift;
    int32_t skip_empty;
} sx_rowlist;

size_t sx_align_workspace_bytes(int32_t row_min, int32_t row_max);
int sx_align_rows(const sx_rowlist* lists /* host array of k */, int k, int32_t row_min, int32_t row_max,
                  int32_t* rows_out, int32_t out_capacity, int32_t* const* aligned /* host array of k */,
                  int32_t* result, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SUBSETIX_B200_H */
