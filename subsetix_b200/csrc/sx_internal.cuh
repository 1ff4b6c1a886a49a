// Internal argument structures and launch entry points shared by the
// kernel files and the C ABI layer (sx_api.cu).
#pragma once

#include "sx_common.cuh"

struct SxLeafDev {
    const int* begin;
    const int* end;
    const int* off;      // aligned row offsets, length rows + 1 (row y = [off[y], off[y+1]))
    const int* off_end;  // when set, row y = [off[y], off_end[y]) instead
    int widen;           // begin - widen, end + widen on load (0 for set operations)
    int scale;           // > 1: [floor(b/scale), ceil(e/scale)) on load (restriction)
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
    // sweep, 3 = merge-path tiles, 4 = segmented sweep in block tiles, 5 =
    // segmented sweep in warp tiles (the default for tables), 6 = kernel 5
    // with 16-bit keys; blocks_per_sm caps residency (via shared-memory
    // padding); staging_cap is the staged kernel's per-warp element capacity,
    // or boundaries per tile for kernels 3 to 6
    int tune_kernel;
    int tune_blocks_per_sm;
    int tune_staging_cap;
    int tune_warps;      // segmented sweeps: warps per block
    int tune_tile_rows;  // segmented sweeps: rows per tile (at most 32; 8 for kernel 6)
    unsigned wait_limit; // look-back polls before giving up (0: SX_LOOKBACK_SPIN_LIMIT); tests of the failure path
    int withhold_tile;   // t + 1: tile t never publishes its look-back status (tests of the failure path)
};

struct SxRowList {
    const int* rows;
    const int* off;  // row offsets of the list's set (length count + 1); needed when skip_empty
    int count;
    int shift;
    int skip_empty;
    int div;    // >= 1: row v maps to output row floor((v + shift) / div)
    int phase;  // ranges: output row y reads source row y * div + phase - shift
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
    int* aligned[SX_MAX_LEAVES * 2];      // per list, [rows_out + 1]; null to skip
    int* aligned_end[SX_MAX_LEAVES * 2];  // per list, [rows_out]; when set, explicit [start, stop) ranges
    int* result;       // [0] rows_out count, [1] flags
};

cudaError_t sx_sweep_launch(const SxBoolArgs& A, bool union_mode, void* workspace, size_t workspace_bytes,
                            cudaStream_t stream);
cudaError_t sx_tile_max_launch(const int* const* offsets, const int* const* begins, const int* const* ends, int k,
                               int rows, int tra, int trb, int* out, cudaStream_t stream);
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

// Interval fields (sx_fields.cu)
cudaError_t sx_check_rows_launch(const int* b, const int* e, const int* off, int rows, long long n, int* flags,
                                 cudaStream_t stream);
cudaError_t sx_cell_offsets_launch(const int* b, const int* e, long long n, int* out, int* result, const SxScanState& st,
                                   cudaStream_t stream);
cudaError_t sx_prolong_set_launch(const int* rows_in, const int* off, const int* b, const int* e, int rows, int n, int r,
                                  int* occupied, int* ord, int* result, const SxScanState& st, int* rows_out,
                                  int* off_out, int* ob, int* oe, cudaStream_t stream);
cudaError_t sx_prolong_field_launch(const int* off, int rows, const int* coff, int n, const int* foff_rows,
                                    const int* fcoff, int r, const void* cv, void* fv, int dbl, cudaStream_t stream);
cudaError_t sx_restrict_check_launch(const int* crows, int crow_count, const int* coff_rows, const int* cb,
                                     const int* ce, int cn, const int* frows, int frow_count, const int* foff_rows,
                                     const int* fb, const int* fe, int fn, int r, int* flags, cudaStream_t stream);
cudaError_t sx_restrict_field_launch(const int* coff_rows, int crow_count, const int* ccoff, int cn,
                                     const int* foff_rows, const int* fcoff, int r, int reducer, double norm,
                                     const void* fv, void* cv, int dbl, cudaStream_t stream);
cudaError_t sx_subset_rows_launch(const int* soff, const int* srows, int srow_count, int sn, const int* urows,
                                  int urow_count, int* pos, int* flags, cudaStream_t stream);
cudaError_t sx_subset_copy_launch(int scatter, int n, const int* pos, const int* sb, const int* se, const int* scoff,
                                  const int* uoff, const int* ub, const int* ue, const int* ucoff, int urows,
                                  void* sub, void* sup, int elem_size, cudaStream_t stream);
cudaError_t sx_row_lookup_launch(const int* rows, int row_count, int height, int* lookup, int* flags,
                                 cudaStream_t stream);
cudaError_t sx_upwind_launch(const int* rows, const int* rid, const int* off, int row_count, const int* b, const int* e, const int* coff,
                             int n, long long cells, const int* lookup, const void* v, void* out, int width, int height,
                             double a, double bb, double dt, double dx, double dy, int direct, int dbl,
                             cudaStream_t stream);
cudaError_t sx_threshold_launch(const float* d, int width, int height, float thr, int grad, int* counts,
                                const int* offsets, int* ob, int* oe, cudaStream_t stream);
cudaError_t sx_mass_launch(const void* v, long long n, int dbl, double scale, double* part, int parts, double* out,
                           cudaStream_t stream);
cudaError_t sx_locate_cells_launch(const int* rows, const int* off, const int* b, const int* e, int row_count,
                                   const int* qr, const int* qc, long long q, int* out, cudaStream_t stream);
cudaError_t sx_value_runs_launch(int type, const void* v, const int* coff, int n, const void* target, int* counts,
                                 const int* run_off, const int* b, int* ob, int* oe, cudaStream_t stream);
cudaError_t sx_gather_i32_launch(const int* idx, int count, const int* src, int* dst, cudaStream_t stream);
cudaError_t sx_gradient_launch(const float* d, int width, int height, float* out, cudaStream_t stream);

// Full-grid two-level AMR (sx_amr.cu)
cudaError_t sx_upwind_full_launch(int dbl, const void* in, void* out, int W, int H, int batch, double a, double b,
                                  double dt, double dx, double dy, cudaStream_t stream);
cudaError_t sx_amr_sync_full_launch(int dbl, void* coarse, void* fine, const signed char* actions, int W, int H,
                                    int batch, int ratio, cudaStream_t stream);
cudaError_t sx_amr_regrid_full_launch(int dbl, const void* coarse, unsigned char* tags, signed char* actions, int W,
                                      int H, int batch, float threshold, int padding, int mode, cudaStream_t stream);
cudaError_t sx_amr_step_full_launch(int dbl, const void* cin, const void* fin, void* cout, void* fout,
                                    const signed char* actions, int W, int H, int batch, double a, double b, double dt,
                                    double dxc, double dyc, double dxf, double dyf, cudaStream_t stream);
int sx_upwind_adjoint_parts(long long cells);
cudaError_t sx_upwind_adjoint_launch(const int* rows, const int* off, int row_count, const int* b, const int* e,
                                     const int* coff, int n, long long cells, const int* lookup, const void* w,
                                     const void* u, void* ubar, int width, int height, double a, double bb, double dt,
                                     double dx, double dy, int direct, int dbl, double* partial, double* grads,
                                     cudaStream_t stream);
cudaError_t sx_upwind_plan_launch(const int* b, const int* e, int n, int* chunk_off, int* result, const SxScanState& st,
                                  cudaStream_t stream);
cudaError_t sx_upwind_plan_fill_launch(const int* rows, const int* off, int row_count, const int* b, const int* e,
                                       const int* coff, int n, const int* chunk_off, long long chunks,
                                       const int* lookup, int height, int* info, cudaStream_t stream);
// nbr: the plan's neighbour table (sx_upwind_table_launch), or null to search the neighbour rows.
cudaError_t sx_upwind_table_launch(const int* b, const int* e, const int* coff, const int* info, long long chunks,
                                   unsigned short* nbr, int* status, cudaStream_t stream);
cudaError_t sx_upwind_chunk_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                   long long chunks, const int* lookup, const unsigned short* nbr, const void* v,
                                   void* out, int width, int height, double a, double bb, double dt, double dx,
                                   double dy, int dbl, cudaStream_t stream);
cudaError_t sx_upwind_chunk_bands_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                         long long chunks, const int* lookup, const unsigned short* nbr, const void* v,
                                         void* out, int width, int height, double a, double bb, const int* row_band,
                                         const void* band_table, int nbands, int dbl, cudaStream_t stream);
void sx_upwind_band_table_fill(int dbl, const double* spacing, int nbands, void* table);
int sx_upwind_adjoint_chunk_parts(long long chunks);
cudaError_t sx_upwind_adjoint_chunk_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                           long long chunks, const int* lookup, const unsigned short* nbr,
                                           const void* w, const void* u, void* ubar, int width, int height, double a,
                                           double bb, double dt, double dx, double dy, int dbl, double* partial,
                                           double* grads, cudaStream_t stream);
// Level coupling by index tables (sx_coupling.cu)
cudaError_t sx_index_copy_launch(int dtype, long long n, const int* dst_idx, const int* src_idx, const void* src,
                                 void* dst, cudaStream_t stream);
cudaError_t sx_index_block_mean_launch(int dtype, long long n, int group, double norm, const int* out_idx,
                                       const int* in_idx, const void* in, void* out, cudaStream_t stream);
cudaError_t sx_index_block_mean_adj_launch(int dtype, long long n, int group, double norm, const int* out_idx,
                                           const int* in_idx, void* out_bar, void* in_bar, cudaStream_t stream);
cudaError_t sx_index_segment_add_launch(int dtype, long long nseg, const int* seg_off, const int* src_idx,
                                        const int* dst_idx, void* src, void* dst, int zero_src, cudaStream_t stream);
// VTK quad assembly (sx_export.cu)
cudaError_t sx_cell_quads_launch(int dtype, const int* off, const int* rows, int row_count, const int* b, const int* e,
                                 const int* coff, int n, const void* v, float dx, float dy, float ox, float oy,
                                 float* pts, float* vals, cudaStream_t stream);
