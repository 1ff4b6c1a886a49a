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
 *     or coarsened by `scale`, and after that must have non-empty intervals
 *     whose begins and whose ends are each non-decreasing per row.  Output:
 *     the merged union (runs whose next begin is <= the running end join).
 * Inputs outside the contract set SX_FLAG_CONTRACT in result[1]; the caller
 * then uses the exact kernels.  Outputs: `out_offsets[rows + 1]`,
 * result = {total, flags}.  A capacity of sum(leaf sizes) always suffices.
 * ------------------------------------------------------------------------- */
#define SX_MODE_TABLE 0
#define SX_MODE_UNION 1

typedef struct sx_leaf {
    const int32_t* begin;
    const int32_t* end;
    const int32_t* row_offsets; /* aligned, rows + 1 entries: row y = [row_offsets[y], row_offsets[y+1]) */
    const int32_t* row_ends;    /* optional: row y = [row_offsets[y], row_ends[y]) (rows entries) */
    int32_t widen;              /* SX_MODE_UNION: intervals read as [b - widen, e + widen) */
    int32_t scale;              /* SX_MODE_UNION, > 1: intervals read as [floor(b/scale), ceil(e/scale)) */
} sx_leaf;

/* Launch tuning for sx_bool_eval; NULL or zero fields select automatic values.
 * kernel: 1 = global-memory sweep, 2 = shared-memory staged sweep, 3 =
 * merge-path tile kernel, 4 = segmented sweep in block tiles, 5 = segmented
 * sweep in warp tiles (table mode; the default), 6 = kernel 5 with 16-bit
 * keys (tiles of at most 8 rows; wider-spanning tiles take the row sweep),
 * 7 = row-lane sweep (a warp per 32-row tile, a lane per row, 16-bit
 * coordinates in shared memory; tiles spanning more than 65534 columns take
 * the row sweep over global memory);
 * blocks_per_sm: residency cap of the global sweep; staging_cap: elements per
 * warp of the staged sweep, or boundaries per tile of kernels 3 to 7; warps:
 * warps per block of kernels 4 to 7 (in 5 to 7 each warp owns a tile);
 * tile_rows: rows per tile of kernels 4 to 6 (at most 32, at most 8 for 6;
 * kernel 7 takes 0 or 32).  Results never depend on the tuning.
 * Two fields exist for tests of the failure path and are zero otherwise:
 * wait_limit caps the polls of every look-back wait of kernels 4 to 7 (0 =
 * the built-in limit of 2^22 polls); withhold_tile = t + 1 makes tile t of
 * those kernels never publish its look-back status, so the tiles after it
 * wait until the limit, give up and report SX_FLAG_TIMEOUT (their outputs
 * are then invalid; every write stays inside the caller's buffers). */
typedef struct sx_tuning {
    int32_t kernel;
    int32_t blocks_per_sm;
    int32_t staging_cap;
    int32_t warps;
    int32_t tile_rows;
    int32_t wait_limit;
    int32_t withhold_tile;
} sx_tuning;

/* Workspace for sx_bool_eval: the size returned here (the look-back state of
 * 1-row tiles) fits every tuning.  Without an explicit tile_rows,
 * sx_bool_eval accepts down to 8 bytes per 32 rows plus a few KiB (the
 * look-back state of 32-row tiles) and then uses 32-row tiles; with an
 * explicit tile_rows a workspace too small for those tiles is refused
 * (SX_ERR_WORKSPACE). */
size_t sx_bool_workspace_bytes(int32_t rows);
int sx_bool_eval(const sx_leaf* leaves /* host array of k */, int k, int32_t rows, const uint32_t* table /* host, 8 */,
                 int mode, int32_t* out_begin, int32_t* out_end, int32_t* out_offsets, int64_t capacity,
                 int32_t* result, void* workspace, size_t workspace_bytes, const sx_tuning* tuning /* host */,
                 void* stream);

/* Largest number of leaf boundaries (2 x intervals, summed over the leaves)
 * in one tile of tile_rows_a aligned rows (out[0]) and of tile_rows_b aligned
 * rows (out[1]), and the largest coordinate span of a tile_rows_a-row tile
 * (out[2]: last end minus first begin over its rows), asynchronously on
 * `stream`.  The leaves' row_offsets are aligned (rows + 1 entries each);
 * begin and end may be NULL for a leaf without intervals; widen, scale and
 * row_ends are ignored.  Callers size sx_tuning.staging_cap
 * with it, and take the 16-bit-key kernel (6) where the span is at most 8190.
 * No reference counterpart. */
int sx_tile_boundaries_max(const sx_leaf* leaves /* host array of k */, int k, int32_t rows, int32_t tile_rows_a,
                           int32_t tile_rows_b, int32_t* out /* device, 3 */, void* stream);

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
 * row_min / row_max bound every (row + shift) that should be kept; the
 * closing offset aligned[l][R] stops after the last output row, so source
 * rows past row_max are excluded too.  result = {number of output rows,
 * flags}.
 * ------------------------------------------------------------------------- */
typedef struct sx_rowlist {
    const int32_t* rows;
    const int32_t* row_offsets; /* count + 1 entries */
    int32_t count;
    int32_t shift;      /* row v maps to output row floor((v + shift) / div) */
    int32_t skip_empty; /* rows without intervals produce no output row */
    int32_t div;        /* >= 1; 0 is read as 1 */
    int32_t phase;      /* ranges: output row y reads source row y * div + phase - shift */
} sx_rowlist;

size_t sx_align_workspace_bytes(int32_t row_min, int32_t row_max);
int sx_align_rows(const sx_rowlist* lists /* host array of k */, int k, int32_t row_min, int32_t row_max,
                  int32_t* rows_out, int32_t out_capacity, int32_t* const* aligned /* host array of k */,
                  int32_t* const* aligned_ends /* host array of k, may be NULL */, int32_t* result, void* workspace,
                  size_t workspace_bytes, void* stream);
/* With aligned_ends[l] set, list l gets explicit ranges instead of
 * consecutive offsets: aligned[l][y] = start and aligned_ends[l][y] = stop of
 * source row y * div + phase - shift (empty when that row is absent). */

/* ---------------------------------------------------------------------------
 * Row shape check.  flags (device int, overwritten) receives the OR of
 *   SX_ROWS_UNSORTED_BEGIN  a begin is smaller than the previous begin of its row
 *   SX_ROWS_OVERLAP         an interval starts before the previous one ends
 *   SX_ROWS_EMPTY           an interval has end <= begin
 *   SX_ROWS_TOUCH           an interval starts where the previous one ends
 *   SX_ROWS_UNSORTED_END    an end is smaller than the previous end of its row
 * No reference counterpart: the reference never checks, and its kernels
 * follow their own visiting order on such rows.  Callers use the check to
 * pick between the fast paths and the exact reference-order paths.
 * ------------------------------------------------------------------------- */
#define SX_ROWS_UNSORTED_BEGIN 1
#define SX_ROWS_OVERLAP 2
#define SX_ROWS_EMPTY 4
#define SX_ROWS_TOUCH 8
#define SX_ROWS_UNSORTED_END 16
int sx_check_rows(const int32_t* begin, const int32_t* end, const int32_t* row_offsets, int32_t rows, int64_t n,
                  int32_t* flags, void* stream);

/* ---------------------------------------------------------------------------
 * Interval fields: one value per active cell, stored row by row, with int32
 * cell offsets per interval (subsetix_cupy/interval_field.py:19-89).
 * Value types: SX_F32 or SX_F64 (the reference computes in float32 only;
 * float64 is this library's addition with the same formulas).
 * ------------------------------------------------------------------------- */
#define SX_F32 0
#define SX_F64 1

/* cell_offsets[n + 1] = exclusive prefix sum of end - begin; result = {total
 * cells, flags}.  Replaces interval_field.py:67-73 (cumsum + .item()).
 * Workspace: sx_scan_workspace_bytes(n). */
int sx_cell_offsets(const int32_t* begin, const int32_t* end, int64_t n, int32_t* cell_offsets, int32_t* result,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Prolongation of a set by `ratio` (>= 2): [b*r, e*r) on rows row*r + 0..r-1
 * for every occupied row, intervals in input order.
 * Replaces subsetix_cupy/multilevel.py:213-264 (_prolong_set_impl).
 * Outputs (capacities rows*ratio, rows*ratio + 1, n*ratio, n*ratio):
 * rows_out, offsets_out, out_begin, out_end.  result = {occupied input rows,
 * flags}; the output has result[0] * ratio rows.  result[1] gets
 * SX_ROWS_UNSORTED_BEGIN when a row's begins decrease; the reference sorts
 * each output row by begin, so the caller must then sort.
 * Workspace: sx_prolong_set_workspace_bytes(rows). */
size_t sx_prolong_set_workspace_bytes(int32_t rows);
int sx_prolong_set(const int32_t* rows, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                   int32_t row_count, int64_t n, int32_t ratio, int32_t* rows_out, int32_t* offsets_out,
                   int32_t* out_begin, int32_t* out_end, int32_t* result, void* workspace, size_t workspace_bytes,
                   void* stream);

/* Piecewise-constant injection of a coarse field onto the fine field of
 * prolong_set(coarse).  Every coarse row must hold an interval (the
 * reference raises otherwise).  Coarse interval i, ordinal o in row ordinal
 * p, maps in sub-row d to fine interval f = fine_row_offsets[p*ratio + d] +
 * o, and fine cell k of f takes coarse cell k / ratio.
 * Replaces subsetix_cupy/multilevel.py:365-407 with the kernel of
 * subsetix_cupy/kernels.py:384-418. */
int sx_prolong_field(int dtype, const int32_t* coarse_row_offsets, int32_t coarse_rows,
                     const int32_t* coarse_cell_offsets, int64_t n, const int32_t* fine_row_offsets,
                     const int32_t* fine_cell_offsets, int32_t ratio, const void* coarse_values, void* fine_values,
                     void* stream);
int sx_prolong_field_f32(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                         int64_t n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets, int32_t ratio,
                         const float* coarse_values, float* fine_values, void* stream);
int sx_prolong_field_f64(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                         int64_t n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets, int32_t ratio,
                         const double* coarse_values, double* fine_values, void* stream);

/* Alignment checks of a fine set against a coarse set for restriction
 * (subsetix_cupy/multilevel.py:169-210,433-451), in the reference's order.
 * flags (device int, overwritten): 1 = fine row count != coarse rows *
 * ratio, 2 = fine rows differ from coarse_row*ratio + dy, 8 = a mapped fine
 * interval is not [r*b, r*e) of its coarse interval. */
int sx_coarse_fine_check(const int32_t* coarse_rows, int32_t coarse_row_count, const int32_t* coarse_row_offsets,
                         const int32_t* coarse_begin, const int32_t* coarse_end, int64_t coarse_n,
                         const int32_t* fine_rows, int32_t fine_row_count, const int32_t* fine_row_offsets,
                         const int32_t* fine_begin, const int32_t* fine_end, int64_t fine_n, int32_t ratio,
                         int32_t* flags, void* stream);

/* ratio x ratio block reduction of a fine field onto a coarse field whose
 * set is restrict_set(fine set) and which passed sx_coarse_fine_check.
 * reducer: 0 mean (sum * 1/r^2), 1 sum, 2 min, 3 max; sums run sub-row
 * outer, column inner, stopping at the fine interval's end.
 * Replaces subsetix_cupy/multilevel.py:410-479 with the kernel of
 * subsetix_cupy/kernels.py:458-527. */
int sx_restrict_field(int dtype, const int32_t* coarse_row_offsets, int32_t coarse_rows,
                      const int32_t* coarse_cell_offsets, int64_t coarse_n, const int32_t* fine_row_offsets,
                      const int32_t* fine_cell_offsets, int32_t ratio, int reducer, const void* fine_values,
                      void* coarse_values, void* stream);
int sx_restrict_field_f32(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                          int64_t coarse_n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets,
                          int32_t ratio, int reducer, const float* fine_values, float* coarse_values, void* stream);
int sx_restrict_field_f64(const int32_t* coarse_row_offsets, int32_t coarse_rows, const int32_t* coarse_cell_offsets,
                          int64_t coarse_n, const int32_t* fine_row_offsets, const int32_t* fine_cell_offsets,
                          int32_t ratio, int reducer, const double* fine_values, double* coarse_values, void* stream);

/* Subset copies between fields on a subset geometry and a superset geometry
 * with the same coordinates (subsetix_amr2/fields.py:127-294, K15/K16).
 * sx_subset_rows: pos[i] = superset row ordinal of subset interval i; flags
 * (device int, overwritten) = 1 when a subset row is missing from the
 * superset (fields.py:310-316).  sx_subset_copy: scatter 0 copies superset
 * -> subset (gather), 1 copies subset -> superset; elem_size 1, 4 or 8
 * bytes covers bool, int8, int32, float32, int64 and float64. */
int sx_subset_rows(const int32_t* sub_row_offsets, const int32_t* sub_rows, int32_t sub_row_count, int64_t sub_n,
                   const int32_t* sup_rows, int32_t sup_row_count, int32_t* pos, int32_t* flags, void* stream);
int sx_subset_copy(int scatter, int64_t sub_n, const int32_t* pos, const int32_t* sub_begin, const int32_t* sub_end,
                   const int32_t* sub_cell_offsets, const int32_t* sup_row_offsets, const int32_t* sup_begin,
                   const int32_t* sup_end, const int32_t* sup_cell_offsets, int32_t sup_row_count, void* sub_values,
                   void* sup_values, int elem_size, void* stream);

/* First-order upwind step with zero exterior
 * (subsetix_cupy/interval_stencil.py:16-251, K9):
 *   out = c - dt * (a * du_dx + b * du_dy)
 * with the upwind side chosen by the sign of a and b, and cells outside
 * [0, width) x [0, height) or outside the set reading as 0.
 * sx_row_lookup fills lookup[height] with the row ordinal of each row id
 * (-1 when absent) and sets flags (device int, overwritten) to 1 when a
 * row lies outside [0, height); the reference wraps such rows instead.
 * direct = 1 is allowed when sx_check_rows reported no UNSORTED_BEGIN,
 * OVERLAP or EMPTY flag: neighbours inside the cell's own interval are then
 * read without a search (same results).  row_ids (optional, one per
 * interval) overrides the row each interval's stencil is taken in, like the
 * reference's row_ids argument; NULL uses the set's own rows. */
int sx_row_lookup(const int32_t* rows, int32_t row_count, int32_t height, int32_t* lookup, int32_t* flags,
                  void* stream);
int sx_upwind(int dtype, const int32_t* rows, const int32_t* row_ids, const int32_t* row_offsets, int32_t row_count,
              const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
              const void* values, void* out, int32_t width, int32_t height, double a, double b, double dt, double dx,
              double dy, int direct, void* stream);
/* Chunked form of sx_upwind for fixed geometry whose rows are sorted and
 * disjoint (sx_check_rows reports no UNSORTED_BEGIN, OVERLAP or EMPTY); same
 * results.  A plan is built once per geometry:
 *   sx_upwind_plan       chunk_offsets[n + 1] = exclusive scan of
 *                        ceil(len / 128) per interval; result = {chunks,
 *                        flags}; workspace: sx_scan_workspace_bytes(n);
 *   sx_upwind_plan_fill  chunk_info[16 * chunks] (16-byte aligned): per
 *                        128-cell chunk its first column, value index and
 *                        interval bounds, its row, whether its interval
 *                        touches its neighbours in the row, and where the
 *                        rows above and below start to overlap it (lookup
 *                        as for sx_upwind);
 *   sx_upwind_plan_table optional: neighbours[cells] (2-byte aligned), one
 *                        16-bit word per cell giving where its neighbours
 *                        in the rows below (low byte) and above (high byte)
 *                        sit in `values` (offsets from the chunk's first
 *                        neighbour cell), 0xFF for none; `cells` is
 *                        cell_offsets[n].  With cell_offsets the prefix sum
 *                        of the interval lengths every offset is below 128;
 *                        with gaps between intervals one may not fit a byte,
 *                        and then *status (device) becomes nonzero and the
 *                        table must not be used.
 * Each step is then sx_upwind_chunked (values != out), with the neighbour
 * table or NULL (then the rows above and below are searched every step).
 * The table is the same for every width; it depends on `height` through the
 * plan. */
int sx_upwind_plan(const int32_t* begin, const int32_t* end, int64_t n, int32_t* chunk_offsets, int32_t* result,
                   void* workspace, size_t workspace_bytes, void* stream);
int sx_upwind_plan_fill(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                        const int32_t* end, const int32_t* cell_offsets, int64_t n, const int32_t* chunk_offsets,
                        int64_t chunks, const int32_t* lookup, int32_t height, int32_t* chunk_info, void* stream);
int sx_upwind_plan_table(const int32_t* begin, const int32_t* end, const int32_t* cell_offsets,
                         const int32_t* chunk_info, int64_t chunks, uint16_t* neighbours, int32_t* status,
                         void* stream);
int sx_upwind_chunked(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                      const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks, const int32_t* lookup,
                      const uint16_t* neighbours, const void* values, void* out, int32_t width, int32_t height,
                      double a, double b, double dt, double dx, double dy, void* stream);
/* Banded form for batches of independent sets laid on row bands (subsetix_b200/batch.py): every row
 * belongs to band row_band[row] (device, `height` entries) with its own spacing and time step, so
 * each set keeps the dx = 1/side and CFL time step of its own step_upwind_interval call
 * (subsetix_cupy/interval_stencil.py:126-219).  sx_upwind_band_table turns host triples
 * (dx, dy, dt) into the kernel's table (host, 4 * nbands values of dtype), which the caller
 * uploads once; chunks in rows whose band index is outside [0, nbands) are left unwritten.
 * No reference counterpart for the batching. */
int sx_upwind_band_table(int dtype, const double* spacing, int32_t nbands, void* table);
int sx_upwind_chunked_bands(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                            const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks,
                            const int32_t* lookup, const uint16_t* neighbours, const void* values, void* out,
                            int32_t width, int32_t height, double a, double b, const int32_t* row_band,
                            const void* band_table, int32_t nbands, void* stream);
int sx_upwind_f32(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                  const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
                  const float* values, float* out, int32_t width, int32_t height, float a, float b, float dt, float dx,
                  float dy, int direct, void* stream);
int sx_upwind_f64(const int32_t* rows, const int32_t* row_offsets, int32_t row_count, const int32_t* begin,
                  const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells, const int32_t* lookup,
                  const double* values, double* out, int32_t width, int32_t height, double a, double b, double dt,
                  double dx, double dy, int direct, void* stream);

/* Adjoint of sx_upwind for fixed velocity and dt (no reference
 * counterpart).  grad_out = dL/du' in, grad_in = dL/du out (may not alias),
 * values = the step's input u; grad_velocity[2] (device doubles) receives
 * (dL/da, dL/db) with dt held fixed, summed in a fixed order.  The
 * transpose follows the forward's neighbour rules exactly (zero exterior,
 * cells outside the set read 0).  scratch: sx_upwind_adjoint_scratch_bytes
 * bytes of device memory. */
size_t sx_upwind_adjoint_scratch_bytes(int64_t cells);
int sx_upwind_adjoint(int dtype, const int32_t* rows, const int32_t* row_offsets, int32_t row_count,
                      const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int64_t n, int64_t cells,
                      const int32_t* lookup, const void* grad_out, const void* values, void* grad_in, int32_t width,
                      int32_t height, double a, double b, double dt, double dx, double dy, int direct,
                      double* grad_velocity, void* scratch, size_t scratch_bytes, void* stream);

/* sx_upwind_adjoint on a chunk plan (sx_upwind_plan / sx_upwind_plan_fill;
 * rows sorted and disjoint); same values.  neighbours: the plan's neighbour
 * table (sx_upwind_plan_table) or NULL.  scratch:
 * sx_upwind_adjoint_chunked_scratch_bytes(chunks) bytes. */
size_t sx_upwind_adjoint_chunked_scratch_bytes(int64_t chunks);
int sx_upwind_adjoint_chunked(int dtype, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                              const int32_t* cell_offsets, const int32_t* chunk_info, int64_t chunks,
                              const int32_t* lookup, const uint16_t* neighbours, const void* grad_out,
                              const void* values, void* grad_in, int32_t width, int32_t height, double a, double b,
                              double dt, double dx, double dy, double* grad_velocity, void* scratch,
                              size_t scratch_bytes, void* stream);

/* Threshold run-length encoding of a full width x height float32 grid
 * (subsetix_amr2/regrid.py:20-124 K11/K12, and regrid.py:172-223 K14 when
 * gradient = 1): a run is a stretch of value >= threshold, where value is
 * the grid itself or its gradient magnitude sqrt(gx^2 + gy^2) with central
 * differences inside and one-sided ones at the borders.  Count pass:
 * out_begin == NULL, counts[height] written.  Write pass: offsets[height]
 * (exclusive scan of counts), out_begin/out_end written. */
int sx_threshold_rle(const float* values, int32_t width, int32_t height, float threshold, int gradient, int32_t* counts,
                     const int32_t* offsets, int32_t* out_begin, int32_t* out_end, void* stream);
/* Gradient magnitude of a full grid, same formula (regrid.py:172-274, K14). */
int sx_gradient_magnitude(const float* values, int32_t width, int32_t height, float* out, void* stream);
int sx_gradient_threshold_rle(const float* values, int32_t width, int32_t height, float threshold, int32_t* counts,
                              const int32_t* offsets, int32_t* out_begin, int32_t* out_end, void* stream);

/* Global interval index holding each (row, col) query, or -1
 * (subsetix_cupy/interval_field.py:162-297, locate_interval_cells). */
int sx_locate_cells(const int32_t* rows, const int32_t* row_offsets, const int32_t* begin, const int32_t* end,
                    int32_t row_count, const int32_t* query_rows, const int32_t* query_cols, int64_t count,
                    int32_t* out, void* stream);

/* Runs of cells whose value equals *target (host pointer to one value of
 * the field's type), per interval; runs never cross intervals
 * (subsetix_amr2/fields.py:39-100).  Count pass (out_begin NULL): counts[n]
 * runs per interval.  Write pass: run_offsets[n] (exclusive scan of the
 * counts) and the intervals' begins give [begin + first, begin + last + 1).
 * Types: SX_VALUE_F32, F64, I8 (also uint8 and bool), I32, I64. */
#define SX_VALUE_F32 0
#define SX_VALUE_F64 1
#define SX_VALUE_I8 2
#define SX_VALUE_I32 3
#define SX_VALUE_I64 4
int sx_value_runs(int type, const void* values, const int32_t* cell_offsets, int64_t n, const void* target,
                  int32_t* counts, const int32_t* run_offsets, const int32_t* begin, int32_t* out_begin,
                  int32_t* out_end, void* stream);

/* dst[p] = src[index[p]] for p < count (row offsets of derived sets). */
int sx_gather_i32(const int32_t* index, int32_t count, const int32_t* src, int32_t* dst, void* stream);

/* VTK export of an interval field (subsetix_cupy/export_vtk.py:205-316, the
 * quads of _interval_field_chunk): for every cell c (value order) four corner
 * points (x, y, 0) into points[12 c .. 12 c + 11] and its value as float32
 * into out_values[c].  Corners in float32, each operation rounded once:
 * x_left = ox + col * dx, x_right = x_left + dx, y_bottom = oy + row * dy,
 * y_top = y_bottom + dy.  dtype SX_F32 or SX_F64 for `values`. */
int sx_cell_quads(int dtype, const int32_t* row_offsets, const int32_t* rows, int32_t row_count,
                  const int32_t* begin, const int32_t* end, const int32_t* cell_offsets, int32_t n,
                  const void* values, float dx, float dy, float ox, float oy, float* points, float* out_values,
                  void* stream);

/* ---------------------------------------------------------------------------
 * Coupling of nested levels by index tables, for the composite multi-level
 * advection and its adjoint (subsetix_b200/adjoint.py).  dtype SX_F32 or
 * SX_F64; index tables are int32 positions into value arrays.
 *   sx_index_copy            dst[dst_idx[i]] = src[src_idx[i]], i < n (a null
 *                            table means the identity): ghost cells take their
 *                            coarse parent's value, the injection of
 *                            prolong_field (subsetix_cupy/multilevel.py:365-407);
 *   sx_index_block_mean      out[out_idx[j]] = (sum over m < group, in order, of
 *                            in[in_idx[j*group+m]]) * norm: restrict_field's
 *                            mean (multilevel.py:410-479, kernels.py:458-527);
 *   sx_index_block_mean_adj  the transpose: in_bar[in_idx[j*group+m]] +=
 *                            out_bar[out_idx[j]] * norm, then out_bar[out_idx[j]]
 *                            = 0; in_idx entries must be distinct;
 *   sx_index_segment_add     dst[dst_idx[s]] += sum over t in [seg_off[s],
 *                            seg_off[s+1]) of src[src_idx[t]], in order, and
 *                            src[src_idx[t]] = 0 when zero_src: the transpose
 *                            of sx_index_copy when parents repeat.
 * The reference has no multi-level coupling of this form (its AMR driver has
 * two whole-grid levels) and no derivatives.
 * ------------------------------------------------------------------------- */
int sx_index_copy(int dtype, int64_t n, const int32_t* dst_idx, const int32_t* src_idx, const void* src, void* dst,
                  void* stream);
int sx_index_block_mean(int dtype, int64_t n, int32_t group, double norm, const int32_t* out_idx,
                        const int32_t* in_idx, const void* in, void* out, void* stream);
int sx_index_block_mean_adj(int dtype, int64_t n, int32_t group, double norm, const int32_t* out_idx,
                            const int32_t* in_idx, void* out_bar, void* in_bar, void* stream);
int sx_index_segment_add(int dtype, int64_t nseg, const int32_t* seg_off, const int32_t* src_idx,
                         const int32_t* dst_idx, void* src, void* dst, int zero_src, void* stream);

/* ---------------------------------------------------------------------------
 * Two-level AMR on full grids, batched: arrays are [batch][height][width]
 * (coarse) and [batch][height*ratio][width*ratio] (fine).  In the
 * reference's AMR2Simulation both levels are full rectangles, and these are
 * its interval kernels specialised to that case, with the same results:
 *   sx_upwind_full      step_upwind_interval on a full grid
 *                       (subsetix_cupy/interval_stencil.py:59-219); in != out;
 *   sx_amr_sync_full    synchronize_interval_fields(..., reducer="mean",
 *                       fill_fine_outside=True, copy=False)
 *                       (subsetix_amr2/fields.py:570-612): coarse cells with
 *                       action 1 (REFINE) take the mean of their fine block,
 *                       the others are copied into it;
 *   sx_amr_regrid_full  the regrid of simulation.py:289-304: gradient tag
 *                       (regrid.py:336-350) then two-level grading with
 *                       `padding` (regrid.py:404-442; mode 0 von Neumann,
 *                       1 Moore), written as action bytes (1 REFINE, 0 KEEP)
 *                       like ActionField.set_from_interval_set.  `tags` is
 *                       scratch of batch*width*height bytes; threshold is
 *                       max(refine_threshold, epsilon) rounded to float32.
 * No counterpart in the reference for the batching.
 * ------------------------------------------------------------------------- */
int sx_upwind_full(int dtype, const void* values, void* out, int32_t width, int32_t height, int32_t batch, double a,
                   double b, double dt, double dx, double dy, void* stream);
int sx_amr_sync_full(int dtype, void* coarse, void* fine, const int8_t* actions, int32_t width, int32_t height,
                     int32_t batch, int32_t ratio, void* stream);
/* One fixed-geometry step for ratio 2 in one pass: sx_upwind_full on both
 * levels followed by sx_amr_sync_full, value for value (a coarse cell's
 * synchronisation reads only its own new value and its fine block's). */
int sx_amr_step_full(int dtype, const void* coarse_in, const void* fine_in, void* coarse_out, void* fine_out,
                     const int8_t* actions, int32_t width, int32_t height, int32_t batch, double a, double b,
                     double dt, double dx_coarse, double dy_coarse, double dx_fine, double dy_fine, void* stream);
int sx_amr_regrid_full(int dtype, const void* coarse, uint8_t* tags, int8_t* actions, int32_t width, int32_t height,
                       int32_t batch, float threshold, int32_t padding, int mode, void* stream);

/* Compensated (Neumaier) FP64 sum of n values times `scale`, in a fixed
 * order (deterministic).  partials: 2 * parts doubles of scratch, parts in
 * [1, 4096].  No reference counterpart (the reference has no mass
 * integral); used for conservation checks. */
int sx_mass_integral(int dtype, const void* values, int64_t n, double scale, double* partials, int parts, double* out,
                     void* stream);
int sx_mass_integral_f64(const double* values, int64_t n, double scale, double* partials, int parts, double* out,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SUBSETIX_B200_H */
