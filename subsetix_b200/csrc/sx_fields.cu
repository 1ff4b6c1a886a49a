// Interval fields: cell offsets, prolongation/restriction, subset copies,
// first-order upwind, gradient-threshold run-length encoding, and the
// compensated mass integral.
//
// A field stores one value per active cell, row by row, with int32 cell
// offsets per interval (subsetix_cupy/interval_field.py:19-89).  Every
// float formula below follows the reference's source order and is written
// with explicit rounding intrinsics, so the compiler makes no choice of its
// own.  Where the reference's NVRTC build fuses a multiply into an add (the
// upwind update and the gradient norm in float32), the fusion is written
// out as the same FMA (sx_upwind_update, sx_grad_norm in sx_common.cuh), so
// float32 results equal the reference's on the GPU bit for bit; float64
// rounds every operation once.

#include <climits>
#include <cmath>

#include "sx_internal.cuh"

// ---------------------------------------------------------------------------
// Arithmetic helpers without contraction (float and double)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sx_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sx_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float sx_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float sx_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sx_sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sx_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sx_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double sx_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sx_div(double a, double b) { return __ddiv_rn(a, b); }

// x / d, or x * d when the launcher passed the reciprocal of a power-of-two
// spacing instead (pow2 != 0): dividing by 2^k and multiplying by 2^-k have
// the same exact real result, so the rounded results are identical.
template <typename T>
__device__ __forceinline__ T sx_over(T x, T d, int pow2)
{
    return pow2 ? sx_mul(x, d) : sx_div(x, d);
}

// Spacings that are powers of two (in the kernel's precision) become their
// exact reciprocals.
template <typename T>
static int sx_pow2_pair(T& dx, T& dy)
{
    int ex, ey;
    if (!(frexp((double)dx, &ex) == 0.5 && frexp((double)dy, &ey) == 0.5)) return 0;
    const T ix = (T)1 / dx, iy = (T)1 / dy;
    if (!std::isfinite((double)ix) || !std::isfinite((double)iy)) return 0;  // reciprocal out of range
    dx = ix;
    dy = iy;
    return 1;
}

// Row ordinal of interval i: the last p with off[p] <= i and off[p+1] > i.
__device__ __forceinline__ int sx_row_of(const int* __restrict__ off, int rows, int i)
{
    int lo = 0, hi = rows - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Exclusive scan of interval lengths: int32 cell offsets
// (interval_field.py:67-73).  Single pass with look-back, like sx_scan_i32.
// ---------------------------------------------------------------------------
#define SX_LEN_ITEMS 8
__global__ void __launch_bounds__(SX_BLOCK) sx_cell_offsets_kernel(const int* __restrict__ b, const int* __restrict__ e,
                                                                   long long n, int* __restrict__ out, int* result,
                                                                   SxScanState st)
{
    __shared__ int s_tile;
    __shared__ unsigned s_epoch;
    __shared__ int s_warp[SX_BLOCK / 32];
    __shared__ int s_base;
    __shared__ unsigned s_flags;
    sx_ticket(st, &s_tile, &s_epoch);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    const long long base_idx = (long long)tile * SX_BLOCK * SX_LEN_ITEMS + (long long)threadIdx.x * SX_LEN_ITEMS;
    int v[SX_LEN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SX_LEN_ITEMS; ++i) {
        const long long idx = base_idx + i;
        v[i] = idx < n ? (e[idx] - b[idx]) : 0;
        sum += v[i];
    }
    int total;
    const int ex = sx_block_exclusive_scan(sum, s_warp, &total);
    if (threadIdx.x < 32) {
        unsigned f = 0u;
        const int base = sx_lookback_warp(st, tile, epoch, total, f);
        if (threadIdx.x == 0) {
            s_base = base;
            s_flags = f;
        }
    }
    __syncthreads();
    int run = s_base + ex;
#pragma unroll
    for (int i = 0; i < SX_LEN_ITEMS; ++i) {
        const long long idx = base_idx + i;
        if (idx < n) out[idx] = run;
        run += v[i];
        if (idx == n - 1) out[n] = run;
    }
    if (n == 0 && tile == 0 && threadIdx.x == 0) out[0] = 0;
    sx_retire(st, epoch, s_flags, result);
}

cudaError_t sx_cell_offsets_launch(const int* b, const int* e, long long n, int* out, int* result, const SxScanState& st,
                                   cudaStream_t stream)
{
    const long long per = (long long)SX_BLOCK * SX_LEN_ITEMS;
    const int tiles = (int)((n + per - 1) / per > 0 ? (n + per - 1) / per : 1);
    cudaError_t err = cudaMemsetAsync(st.counters, 0, 16 + (size_t)tiles * 8, stream);
    if (err != cudaSuccess) return err;
    sx_cell_offsets_kernel<<<tiles, SX_BLOCK, 0, stream>>>(b, e, n, out, result, st);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Prolongation of a set (multilevel.py:213-264): [b*r, e*r) on rows
// row*r + 0..r-1, for occupied rows only, in the same order.  `ord` holds
// the exclusive scan of the occupied-row flags.
// ---------------------------------------------------------------------------
__global__ void sx_occupied_kernel(const int* __restrict__ off, int rows, int* __restrict__ flags)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rows; q += gridDim.x * blockDim.x)
        flags[q] = off[q + 1] > off[q] ? 1 : 0;
}

__global__ void sx_prolong_set_rows_kernel(const int* __restrict__ rows_in, const int* __restrict__ off, int rows,
                                           const int* __restrict__ ord, int r, int* __restrict__ rows_out,
                                           int* __restrict__ off_out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rows; q += gridDim.x * blockDim.x) {
        const int n_q = off[q + 1] - off[q];
        if (n_q > 0) {
            const int p = ord[q];
            for (int k = 0; k < r; ++k) {
                rows_out[p * r + k] = rows_in[q] * r + k;
                off_out[p * r + k] = r * off[q] + k * n_q;
            }
        }
        if (q == rows - 1) off_out[ord[rows] * r] = r * off[rows];
    }
}

__global__ void sx_prolong_set_intervals_kernel(const int* __restrict__ b, const int* __restrict__ e,
                                                const int* __restrict__ off, int rows, int n, int r,
                                                int* __restrict__ ob, int* __restrict__ oe, int* result)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int q = sx_row_of(off, rows, i);
        const int n_q = off[q + 1] - off[q];
        if (i + 1 < off[q + 1] && b[i + 1] < b[i]) atomicOr(&result[1], 1);
        const int bi = b[i] * r, ei = e[i] * r;
        const int base = r * off[q] + (i - off[q]);
        for (int k = 0; k < r; ++k) {
            ob[base + k * n_q] = bi;
            oe[base + k * n_q] = ei;
        }
    }
}

// ---------------------------------------------------------------------------
// Field prolongation (kernels.py:384-455): piecewise-constant injection onto
// the prolonged set.  Every coarse row must be occupied (the caller checks,
// as the reference's alignment check does).  Coarse interval i (ordinal o
// in row ordinal p) maps in sub-row d to the fine interval
// f = fine_off[p*r + d] + o, and fine cell k of f takes coarse cell k / r.
// One warp handles one coarse interval.  RT > 0 fixes the ratio at compile
// time (2, the common one: k / r becomes a shift), RT = 0 takes r.
// ---------------------------------------------------------------------------
template <typename T, int RT>
__global__ void sx_prolong_field_kernel(const int* __restrict__ off, int rows, const int* __restrict__ coff, int n,
                                        const int* __restrict__ foff_rows, const int* __restrict__ fcoff, int rr,
                                        const T* __restrict__ cv, T* __restrict__ fv)
{
    const int r = RT > 0 ? RT : rr;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const long long ncells = coff[n];
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int cb = coff[i];
        if (coff[i + 1] - cb <= 0) continue;
        const int p = sx_row_of(off, rows, i);
        const int o = i - off[p];
        for (int d = 0; d < r; ++d) {
            const int f = foff_rows[p * r + d] + o;
            const int fs = fcoff[f];
            const int fw = fcoff[f + 1] - fs;
            // Rows whose begins decrease are re-sorted on the fine level, so
            // fine interval f may be wider than coarse interval i; the
            // reference then reads past i, and past the array at its end.
            // Here reads stay inside the array (0 beyond it).
            for (int t = lane; t < fw; t += 32) {
                const long long src = (long long)cb + t / r;
                fv[fs + t] = src < ncells ? cv[src] : (T)0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Field restriction (kernels.py:458-599 and multilevel.py:410-479).  The
// coarse set is restrict_set(fine).  For coarse interval i (row ordinal p)
// and sub-row dy, the fine interval is fine_off[p*r + dy] + (i -
// coarse_off[p]).
// Checks, with the reference's error order (flag bits):
//   1  the fine row count differs from coarse rows x r
//   2  fine rows are not coarse_row*r + dy
//   8  a fine interval is not [r*cb, r*ce)
// The reduction keeps the reference's order: sub-row outer, column inner,
// stop early at the fine interval's end; mean = sum * norm.
// ---------------------------------------------------------------------------
__global__ void sx_restrict_check_kernel(const int* __restrict__ crows, int crow_count, const int* __restrict__ coff_rows,
                                         const int* __restrict__ cb, const int* __restrict__ ce, int cn,
                                         const int* __restrict__ frows, int frow_count, const int* __restrict__ foff_rows,
                                         const int* __restrict__ fb, const int* __restrict__ fe, int fn, int r,
                                         int* __restrict__ flags)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (tid == 0 && frow_count != crow_count * r) atomicOr(flags, 1);
    if (frow_count != crow_count * r) return;
    for (long long j = tid; j < (long long)crow_count * r; j += stride) {
        const int p = (int)(j / r), dy = (int)(j % r);
        if (frows[j] != crows[p] * r + dy) atomicOr(flags, 2);
    }
    for (long long j = tid; j < (long long)cn * r; j += stride) {
        const int i = (int)(j / r), dy = (int)(j % r);
        const int p = sx_row_of(coff_rows, crow_count, i);
        const long long f = (long long)foff_rows[p * r + dy] + (i - coff_rows[p]);
        if (f < 0 || f >= fn) {
            atomicOr(flags, 8);
            continue;
        }
        if (fb[f] != cb[i] * r || fe[f] != ce[i] * r) atomicOr(flags, 8);
    }
}

// RT as in sx_prolong_field_kernel.
template <typename T, int RT>
__global__ void sx_restrict_field_kernel(const int* __restrict__ coff_rows, int crow_count, const int* __restrict__ ccoff,
                                         int cn, const int* __restrict__ foff_rows, const int* __restrict__ fcoff,
                                         int rr, int reducer, T norm, const T* __restrict__ fv, T* __restrict__ cv)
{
    const int r = RT > 0 ? RT : rr;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < cn; i += warps) {
        const int p = sx_row_of(coff_rows, crow_count, i);
        const int cb = ccoff[i];
        const int w = ccoff[i + 1] - cb;
        if (w <= 0) continue;
        const int ordinal = i - coff_rows[p];
        for (int k = lane; k < w; k += 32) {
            T acc = (T)0, lo = (T)0, hi = (T)0;
            bool have = false;
            for (int dy = 0; dy < r; ++dy) {
                const int f = foff_rows[p * r + dy] + ordinal;
                const int fend = fcoff[f + 1];
                const int start = fcoff[f] + k * r;
                for (int dx = 0; dx < r; ++dx) {
                    const int idx = start + dx;
                    if (idx >= fend) break;
                    const T v = fv[idx];
                    if (reducer == 2) {
                        if (!have || v < lo) lo = v;
                    } else if (reducer == 3) {
                        if (!have || v > hi) hi = v;
                    } else {
                        acc = sx_add(acc, v);
                    }
                    have = true;
                }
            }
            cv[cb + k] = reducer == 0 ? sx_mul(acc, norm) : reducer == 1 ? acc : reducer == 2 ? lo : hi;
        }
    }
}

// ---------------------------------------------------------------------------
// Subset gather / scatter (fields.py:127-294): copy the cells of each subset
// interval between a subset field and a superset field with the same
// coordinates.  A binary search finds the superset interval, then the walk
// goes across superset intervals in the reference's way (cells of the
// subset that the superset lacks are skipped).  `pos` maps each subset
// interval to its superset row ordinal.  One warp per subset interval: lane
// 0 walks, and the warp copies each piece.
// ---------------------------------------------------------------------------
template <typename E>
__global__ void sx_subset_copy_kernel(int scatter, int n, const int* __restrict__ pos, const int* __restrict__ sb,
                                      const int* __restrict__ se, const int* __restrict__ scoff,
                                      const int* __restrict__ uoff, const int* __restrict__ ub,
                                      const int* __restrict__ ue, const int* __restrict__ ucoff, int urows,
                                      E* __restrict__ sub, E* __restrict__ sup)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int row = pos[i];
        if (row < 0 || row >= urows) continue;
        const int start = sb[i], stop = se[i];
        if (stop <= start) continue;
        const int rs = uoff[row], rt = uoff[row + 1];
        if (rs >= rt) continue;
        int idx = rs;
        if (lane == 0) {
            int lo = rs, hi = rt - 1;
            bool found = false;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                if (start < ub[mid]) hi = mid - 1;
                else if (start >= ue[mid]) lo = mid + 1;
                else {
                    idx = mid;
                    found = true;
                    break;
                }
            }
            if (!found) idx = lo;
            if (idx < rs) idx = rs;
        }
        idx = __shfl_sync(0xFFFFFFFFu, idx, 0);
        int cur = start, done = 0;
        const int sub_base = scoff[i];
        while (cur < stop && idx < rt) {
            const int b = ub[idx], e = ue[idx];
            if (cur < b) {
                cur = b;
                continue;
            }
            const int stop2 = stop < e ? stop : e;
            const int len = stop2 - cur;
            if (len > 0) {
                const long long sp = (long long)ucoff[idx] + (cur - b);
                const long long dp = (long long)sub_base + done;
                for (int t = lane; t < len; t += 32) {
                    if (scatter) sup[sp + t] = sub[dp + t];
                    else sub[dp + t] = sup[sp + t];
                }
                done += len;
                cur = stop2;
            }
            if (cur >= e) ++idx;
            if (len == 0 && cur < stop) ++cur;
        }
    }
}

// Superset row ordinal of each subset interval (searchsorted), or a flag
// when the row is missing (fields.py:310-316).
__global__ void sx_subset_rows_kernel(const int* __restrict__ soff, const int* __restrict__ srows, int srow_count,
                                      int sn, const int* __restrict__ urows, int urow_count, int* __restrict__ pos,
                                      int* __restrict__ flags)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sn; i += gridDim.x * blockDim.x) {
        const int p = sx_row_of(soff, srow_count, i);
        const int row = srows[p];
        int lo = 0, hi = urow_count;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (urows[mid] < row) lo = mid + 1; else hi = mid;
        }
        if (lo >= urow_count || urows[lo] != row) atomicOr(flags, 1);
        pos[i] = lo;
    }
}

// ---------------------------------------------------------------------------
// First-order upwind with zero exterior (interval_stencil.py:16-113).
// A cell outside [0, width) x [0, height), or outside the set, reads as 0.
// `lookup[row id]` gives the row ordinal or -1.  Blocks take runs of 256
// consecutive cells.  Thread 0 locates the block's first interval and row,
// and each thread walks forward to its own cell.  Neighbours inside the
// cell's own interval are read directly; the others are found by binary
// search in their row.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T sx_sample(int row, int x, int height, int width, const int* __restrict__ lookup,
                                       const int* __restrict__ off, const int* __restrict__ b,
                                       const int* __restrict__ e, const int* __restrict__ coff,
                                       const T* __restrict__ v)
{
    if (row < 0 || row >= height || x < 0 || x >= width) return (T)0;
    const int ord = lookup[row];
    if (ord < 0) return (T)0;
    int lo = off[ord], hi = off[ord + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (x < b[mid]) hi = mid - 1;
        else if (x >= e[mid]) lo = mid + 1;
        else return v[coff[mid] + (x - b[mid])];
    }
    return (T)0;
}

template <typename T>
__global__ void __launch_bounds__(256) sx_upwind_kernel(const int* __restrict__ rows, const int* __restrict__ rid,
                                                        const int* __restrict__ off,
                                                        int row_count, const int* __restrict__ b,
                                                        const int* __restrict__ e, const int* __restrict__ coff, int n,
                                                        const int* __restrict__ lookup, const T* __restrict__ v,
                                                        T* __restrict__ out, int width, int height, T a, T bb, T dt,
                                                        T dx, T dy, int direct, long long value_count)
{
    __shared__ int s_i, s_p;
    const long long cells = coff[n] < value_count ? (long long)coff[n] : value_count;
    for (long long c0 = (long long)blockIdx.x * blockDim.x; c0 < cells; c0 += (long long)gridDim.x * blockDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) {
            int lo = 0, hi = n - 1;  // last interval with coff <= c0
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (coff[mid] <= c0) lo = mid; else hi = mid - 1;
            }
            s_i = lo;
            s_p = sx_row_of(off, row_count, lo);
        }
        __syncthreads();
        const long long c = c0 + threadIdx.x;
        if (c >= cells) continue;
        int i = s_i, p = s_p;
        while (coff[i + 1] <= c) ++i;  // skips empty intervals too
        while (off[p + 1] <= i) ++p;
        const int row = rid ? rid[i] : rows[p];
        const int ib = b[i], ie = e[i];
        const int x = ib + (int)(c - coff[i]);
        const T center = v[c];
        // Inside the cell's own interval of a row whose intervals are sorted
        // and disjoint, the search below would return this interval, so the
        // neighbour is read directly.
        T left, right;
        if (direct && x - 1 >= ib) left = (x - 1 >= 0 && x - 1 < width) ? v[c - 1] : (T)0;
        else left = sx_sample<T>(row, x - 1, height, width, lookup, off, b, e, coff, v);
        if (direct && x + 1 < ie) right = (x + 1 >= 0 && x + 1 < width) ? v[c + 1] : (T)0;
        else right = sx_sample<T>(row, x + 1, height, width, lookup, off, b, e, coff, v);
        const T down = sx_sample<T>(row - 1, x, height, width, lookup, off, b, e, coff, v);
        const T up = sx_sample<T>(row + 1, x, height, width, lookup, off, b, e, coff, v);
        const T du_dx = a >= (T)0 ? sx_div(sx_sub(center, left), dx) : sx_div(sx_sub(right, center), dx);
        const T du_dy = bb >= (T)0 ? sx_div(sx_sub(center, down), dy) : sx_div(sx_sub(up, center), dy);
        out[c] = sx_upwind_update(center, du_dx, du_dy, a, bb, dt);
    }
}

// ---------------------------------------------------------------------------
// Adjoint of the upwind step (no reference counterpart).  For fixed
// velocity the step is linear, u' = u - dt (a Dx u + b Dy u), where Dx, Dy
// are the one-sided differences chosen by the signs of a and b, with zero
// exterior.  Given w = dL/du', this kernel writes dL/du = w - dt (a Dx^T w
// + b Dy^T w) and per-block float64 partial sums of dL/da = sum w (-dt Dx u)
// and dL/db = sum w (-dt Dy u), dt held fixed.
//
// The transpose mirrors the forward validity rules exactly: cell i reads
// its left neighbour j only when j is in the set and inside the domain, so
// j receives w_i from the cell to its right whenever that cell is in the set
// (whatever its own position) and j is inside the domain.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T sx_in_set(int row, int x, int height, const int* __restrict__ lookup,
                                       const int* __restrict__ off, const int* __restrict__ b,
                                       const int* __restrict__ e, const int* __restrict__ coff,
                                       const T* __restrict__ v)
{
    if (row < 0 || row >= height) return (T)0;
    const int ord = lookup[row];
    if (ord < 0) return (T)0;
    int lo = off[ord], hi = off[ord + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (x < b[mid]) hi = mid - 1;
        else if (x >= e[mid]) lo = mid + 1;
        else return v[coff[mid] + (x - b[mid])];
    }
    return (T)0;
}

template <typename T>
__global__ void __launch_bounds__(256) sx_upwind_adjoint_kernel(const int* __restrict__ rows,
                                                                const int* __restrict__ off, int row_count,
                                                                const int* __restrict__ b, const int* __restrict__ e,
                                                                const int* __restrict__ coff, int n,
                                                                const int* __restrict__ lookup,
                                                                const T* __restrict__ w, const T* __restrict__ u,
                                                                T* __restrict__ ubar, int width, int height, T a, T bb,
                                                                T dt, T dx, T dy, int direct, long long value_count,
                                                                double* __restrict__ partial)
{
    __shared__ int s_i, s_p;
    __shared__ double s_ga[256 / 32], s_gb[256 / 32];
    const long long cells = coff[n] < value_count ? (long long)coff[n] : value_count;
    double ga = 0.0, gb = 0.0;
    for (long long c0 = (long long)blockIdx.x * blockDim.x; c0 < cells; c0 += (long long)gridDim.x * blockDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) {
            int lo = 0, hi = n - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (coff[mid] <= c0) lo = mid; else hi = mid - 1;
            }
            s_i = lo;
            s_p = sx_row_of(off, row_count, lo);
        }
        __syncthreads();
        const long long c = c0 + threadIdx.x;
        if (c >= cells) continue;
        int i = s_i, p = s_p;
        while (coff[i + 1] <= c) ++i;
        while (off[p + 1] <= i) ++p;
        const int row = rows[p];
        const int ib = b[i], ie = e[i];
        const int x = ib + (int)(c - coff[i]);
        const bool jdom = x >= 0 && x < width && row >= 0 && row < height;
        const T wc = w[c];
        // transpose of the x difference
        T tx;
        if (a >= (T)0) {
            T wr = (T)0;
            if (jdom) wr = (direct && x + 1 < ie) ? w[c + 1] : sx_in_set<T>(row, x + 1, height, lookup, off, b, e, coff, w);
            tx = sx_div(sx_sub(wc, wr), dx);
        } else {
            T wl = (T)0;
            if (jdom) wl = (direct && x - 1 >= ib) ? w[c - 1] : sx_in_set<T>(row, x - 1, height, lookup, off, b, e, coff, w);
            tx = sx_div(sx_sub(wl, wc), dx);
        }
        // transpose of the y difference
        T ty;
        if (bb >= (T)0) {
            const T wu = jdom ? sx_in_set<T>(row + 1, x, height, lookup, off, b, e, coff, w) : (T)0;
            ty = sx_div(sx_sub(wc, wu), dy);
        } else {
            const T wd = jdom ? sx_in_set<T>(row - 1, x, height, lookup, off, b, e, coff, w) : (T)0;
            ty = sx_div(sx_sub(wd, wc), dy);
        }
        ubar[c] = sx_sub(wc, sx_mul(dt, sx_add(sx_mul(a, tx), sx_mul(bb, ty))));
        // forward differences of u for the velocity gradient (forward validity rules)
        const T uc = u[c];
        T ul, ur;
        if (direct && x - 1 >= ib) ul = (x - 1 >= 0 && x - 1 < width) ? u[c - 1] : (T)0;
        else ul = sx_sample<T>(row, x - 1, height, width, lookup, off, b, e, coff, u);
        if (direct && x + 1 < ie) ur = (x + 1 >= 0 && x + 1 < width) ? u[c + 1] : (T)0;
        else ur = sx_sample<T>(row, x + 1, height, width, lookup, off, b, e, coff, u);
        const T ud = sx_sample<T>(row - 1, x, height, width, lookup, off, b, e, coff, u);
        const T uu = sx_sample<T>(row + 1, x, height, width, lookup, off, b, e, coff, u);
        const T dux = a >= (T)0 ? sx_div(sx_sub(uc, ul), dx) : sx_div(sx_sub(ur, uc), dx);
        const T duy = bb >= (T)0 ? sx_div(sx_sub(uc, ud), dy) : sx_div(sx_sub(uu, uc), dy);
        ga -= (double)dt * (double)wc * (double)dux;
        gb -= (double)dt * (double)wc * (double)duy;
    }
    // block reduction of the velocity gradients, fixed order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ga += __shfl_down_sync(0xFFFFFFFFu, ga, o);
        gb += __shfl_down_sync(0xFFFFFFFFu, gb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_ga[threadIdx.x >> 5] = ga;
        s_gb[threadIdx.x >> 5] = gb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int q = 0; q < 256 / 32; ++q) {
            ta += s_ga[q];
            tb += s_gb[q];
        }
        partial[2 * blockIdx.x] = ta;
        partial[2 * blockIdx.x + 1] = tb;
    }
}

// Sum of (a, b) pairs, one block of 256 threads: thread t adds pairs t,
// t + 256, ... in order, then a fixed tree combines the threads, so the
// result does not depend on timing.
__global__ void __launch_bounds__(256) sx_sum_pairs_kernel(const double* __restrict__ partial, int parts,
                                                           double* __restrict__ out)
{
    __shared__ double sa[256], sb[256];
    double a = 0.0, b = 0.0;
    for (int q = threadIdx.x; q < parts; q += 256) {
        a += partial[2 * q];
        b += partial[2 * q + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sa[threadIdx.x] += sa[threadIdx.x + h];
            sb[threadIdx.x] += sb[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

// ---------------------------------------------------------------------------
// Upwind, chunked form, for rows whose intervals are sorted and disjoint
// (touching allowed).  Same results as sx_upwind_kernel.  Work is split
// into chunks of SX_CHUNK = 128 consecutive cells of one interval
// (`chunk_off[i]` is the first chunk of interval i); a warp takes a
// contiguous range of chunks and covers a chunk in four sub-rounds of 32
// cells, so every load is coalesced and the four sub-rounds' loads are
// independent.  Left and right neighbours come from the neighbouring lanes
// (or the neighbouring sub-round); for the rows above and below, the warp
// finds the first interval ending after the chunk's first cell once per
// chunk, then each lane steps forward through intervals ending inside the
// chunk (fewer than 128: they are disjoint and non-empty).
// ---------------------------------------------------------------------------
#define SX_CHUNK 128
// Blocks of 256 threads the chunked stencil asks to keep resident per SM
// (a register cap for the compiler); a build-time tuning knob.
#ifndef SX_UPWIND_MIN_BLOCKS
#define SX_UPWIND_MIN_BLOCKS 1
#endif
// The same for the table-driven form, which holds fewer values per lane: six
// blocks (48 warps per SM, 40 registers) hide the two dependent loads of a
// chunk best (config-4 batch on a B200: 1.79 ms at 1 block, 1.42 ms at 6,
// 1.45 ms at 8).
// The same for the adjoint chunk kernel: four blocks (64 registers, no
// spills) took the three-level backward pass from 16.7 to 15.5 ms on a B200;
// five and six spill and are slower.  Both knobs apply to float32; the
// float64 forms keep two (adjoint) and three (table) blocks, where their
// registers fit without spilling.
#ifndef SX_UPWIND_ADJOINT_MIN_BLOCKS
#define SX_UPWIND_ADJOINT_MIN_BLOCKS 4
#endif
#ifndef SX_UPWIND_TABLE_MIN_BLOCKS
#define SX_UPWIND_TABLE_MIN_BLOCKS 6
#endif
#define SX_CHUNK_SUB (SX_CHUNK / 32)

__global__ void sx_chunk_count_kernel(const int* __restrict__ b, const int* __restrict__ e, int n,
                                      int* __restrict__ counts)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const long long len = (long long)e[i] - b[i];
        counts[i] = len > 0 ? (int)((len + SX_CHUNK - 1) / SX_CHUNK) : 0;
    }
}

// Neighbour-row reader: first interval of row `row` ending after x0 (warp-uniform search).
struct SxRowCursor {
    int j, je;
};

__device__ __forceinline__ SxRowCursor sx_row_cursor(int row, int x0, int height, const int* __restrict__ lookup,
                                                     const int* __restrict__ off, const int* __restrict__ e)
{
    SxRowCursor cur{0, 0};
    if (row < 0 || row >= height) return cur;
    const int ord = lookup[row];
    if (ord < 0) return cur;
    int lo = off[ord], hi = off[ord + 1];
    const int je = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] <= x0) lo = mid + 1; else hi = mid;
    }
    cur.j = lo;
    cur.je = je;
    return cur;
}

// Value at column x of a neighbour row.  The cursor keeps the current
// interval's bounds and cell offset in registers and reloads them only when
// it steps (x non-decreasing between calls of one lane).
struct SxRowReader {
    int j, je, cb, ce, cc;
};

__device__ __forceinline__ SxRowReader sx_row_reader(int j, int je, const int* __restrict__ b,
                                                     const int* __restrict__ e, const int* __restrict__ coff)
{
    SxRowReader r{j, je, 0, 0, 0};
    if (j < je) {
        r.cb = b[j];
        r.ce = e[j];
        r.cc = coff[j];
    }
    return r;
}

// Value index of column x in the reader's row (advancing the reader), or
// -1 when x is outside the row's intervals, the domain or the active cells.
__device__ __forceinline__ int sx_row_index(SxRowReader& r, int x, int width, const int* __restrict__ b,
                                            const int* __restrict__ e, const int* __restrict__ coff, bool act)
{
    while (r.j < r.je && r.ce <= x) {
        ++r.j;
        if (r.j < r.je) {
            r.cb = b[r.j];
            r.ce = e[r.j];
            r.cc = coff[r.j];
        }
    }
    if (!act || r.j >= r.je || r.cb > x || x < 0 || x >= width) return -1;
    return r.cc + (x - r.cb);
}

// Value indices of the neighbour-row cells under a chunk's active cells, for
// all its sub-rounds at once (the whole warp calls it with the same plan
// entry).  When the plan's first interval reaches past the chunk, no load is
// needed.  Otherwise the warp loads the row's next 32 intervals with one
// coalesced load per array and every lane finds the interval under each of
// its columns by a binary search over the lanes' interval ends (shuffles):
// one memory round trip per 32 intervals instead of one per interval
// stepped over.  idx[q] = -1 where the cell has no neighbour in the set or
// lies outside [0, width) (the column test only with XDOM).
template <int SUB, bool XDOM = true>
__device__ __forceinline__ void sx_row_indices(const SxRowReader& r0, int x0, int nq, int ie, int width,
                                               const int* __restrict__ b, const int* __restrict__ e,
                                               const int* __restrict__ coff, int lane, int (&idx)[SUB])
{
    bool done[SUB];
#pragma unroll
    for (int q = 0; q < SUB; ++q) {
        idx[q] = -1;
        done[q] = !(q < nq && x0 + 32 * q + lane < ie);
    }
    if (r0.j >= r0.je) return;
    const int xlast = min(ie, x0 + 32 * nq) - 1;
    if (r0.ce > xlast) {  // one interval reaches past the chunk
#pragma unroll
        for (int q = 0; q < SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            if (!done[q] && x >= r0.cb && (!XDOM || (x >= 0 && x < width))) idx[q] = r0.cc + (x - r0.cb);
        }
        return;
    }
    for (int k0 = r0.j; k0 < r0.je; k0 += 32) {
        const int k = k0 + lane;
        int bk = INT_MAX, ek = INT_MAX, ck = 0;
        if (k < r0.je) {
            bk = b[k];
            ek = e[k];
            ck = coff[k];
        }
#pragma unroll
        for (int q = 0; q < SUB; ++q) {
            if (q >= nq) break;
            const int x = x0 + 32 * q + lane;
            // first lane m whose interval ends after x (ends rise across the lanes)
            int m = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int em = __shfl_sync(0xFFFFFFFFu, ek, m + step - 1);
                if (em <= x) m += step;
            }
            const int em = __shfl_sync(0xFFFFFFFFu, ek, m);
            const int bm = __shfl_sync(0xFFFFFFFFu, bk, m);
            const int cm = __shfl_sync(0xFFFFFFFFu, ck, m);
            if (!done[q] && em > x) {
                done[q] = true;
                if (bm <= x && (!XDOM || (x >= 0 && x < width))) idx[q] = cm + (x - bm);
            }
        }
        const int elast = __shfl_sync(0xFFFFFFFFu, ek, 31);
        if (elast > xlast) break;  // every column is resolved (or the row has ended)
    }
}

template <typename T>
__device__ __forceinline__ T sx_row_take(SxRowReader& r, int x, int width, const int* __restrict__ b,
                                         const int* __restrict__ e, const int* __restrict__ coff,
                                         const T* __restrict__ v, bool act)
{
    while (r.j < r.je && r.ce <= x) {
        ++r.j;
        if (r.j < r.je) {
            r.cb = b[r.j];
            r.ce = e[r.j];
            r.cc = coff[r.j];
        }
    }
    if (!act || r.j >= r.je || r.cb > x || x < 0 || x >= width) return (T)0;
    return v[r.cc + (x - r.cb)];
}

// Per-chunk plan, SX_PLAN_INTS ints per 128-cell chunk, everything a warp
// needs before its data loads:
//   [0..3]   first column x0, interval end, value index of x0, touching bits
//   [4..7]   row below: first interval ending after x0, end of the row's
//            intervals, that interval's begin and end
//   [8..11]  row below: its value offset; row above: first interval, end,
//            begin
//   [12..15] row above: end and value offset; row id; interval begin
// Touching bits: on sorted disjoint rows the cell just left of an interval
// is in the set exactly when the previous interval ends there (bit 0; value
// index c - 1), likewise on the right (bit 1; c + 1).  The plan depends only
// on the geometry and is built once per set.
#define SX_PLAN_INTS 16

__global__ void sx_chunk_info_kernel(const int* __restrict__ rows, const int* __restrict__ off, int row_count,
                                     const int* __restrict__ b, const int* __restrict__ e,
                                     const int* __restrict__ coff, int n, const int* __restrict__ chunk_off,
                                     long long chunks, const int* __restrict__ lookup, int height,
                                     int* __restrict__ info)
{
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < chunks;
         u += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunk_off[mid] <= u) lo = mid; else hi = mid - 1;
        }
        const int i = lo;
        const int k = (int)(u - chunk_off[i]);
        const int p = sx_row_of(off, row_count, i);
        const int row = rows[p];
        const int x0 = b[i] + SX_CHUNK * k;
        const int c0 = coff[i] + SX_CHUNK * k;
        const SxRowCursor dn = sx_row_cursor(row - 1, x0, height, lookup, off, e);
        const SxRowCursor up = sx_row_cursor(row + 1, x0, height, lookup, off, e);
        const int touch = ((i > off[p] && e[i - 1] == b[i]) ? 1 : 0) | ((i + 1 < off[p + 1] && b[i + 1] == e[i]) ? 2 : 0);
        const bool hd = dn.j < dn.je, hu = up.j < up.je;
        int4* o = (int4*)(info + (long long)SX_PLAN_INTS * u);
        o[0] = make_int4(x0, e[i], c0, touch);
        o[1] = make_int4(dn.j, dn.je, hd ? b[dn.j] : 0, hd ? e[dn.j] : 0);
        o[2] = make_int4(hd ? coff[dn.j] : 0, up.j, up.je, hu ? b[up.j] : 0);
        o[3] = make_int4(hu ? e[up.j] : 0, hu ? coff[up.j] : 0, row, b[i]);
    }
}

// Neighbour table of a chunk plan, one 16-bit word per cell: the low byte
// is the offset of the cell below from the chunk's base in that row, the
// high byte the same for the row above, 0xFF where the neighbour is not in
// the set (the column test against the domain stays with the step).  The
// base of a neighbour row is the value index of its first cell at or right
// of the chunk's first column; with values packed in interval order the
// row's cells under the chunk are consecutive from there, so an offset is
// below 128.  An offset that does not fit (values not packed) sets *status.
__device__ __forceinline__ int sx_chunk_base(const SxRowReader& r, int x0)
{
    return r.j < r.je ? r.cc + max(0, x0 - r.cb) : 0;
}

__global__ void __launch_bounds__(256) sx_chunk_table_kernel(const int* __restrict__ b, const int* __restrict__ e,
                                                             const int* __restrict__ coff,
                                                             const int* __restrict__ info, long long chunks,
                                                             unsigned short* __restrict__ nbr, int* __restrict__ status)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    bool bad = false;
    for (long long u = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < chunks; u += warps) {
        const int4* pl = (const int4*)(info + (long long)SX_PLAN_INTS * u);
        const int4 p0 = __ldg(pl), p1 = __ldg(pl + 1), p2 = __ldg(pl + 2), p3 = __ldg(pl + 3);
        const int x0 = p0.x, ie = p0.y;
        const long long c0 = p0.z;
        const int nq = min(SX_CHUNK_SUB, (ie - x0 + 31) >> 5);
        const SxRowReader dn{p1.x, p1.y, p1.z, p1.w, p2.x};
        const SxRowReader upc{p2.y, p2.z, p2.w, p3.x, p3.y};
        int idn[SX_CHUNK_SUB], iup[SX_CHUNK_SUB];
        sx_row_indices<SX_CHUNK_SUB, false>(dn, x0, nq, ie, 0, b, e, coff, lane, idn);
        sx_row_indices<SX_CHUNK_SUB, false>(upc, x0, nq, ie, 0, b, e, coff, lane, iup);
        const int bdn = sx_chunk_base(dn, x0), bup = sx_chunk_base(upc, x0);
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            if (q >= nq) break;
            if (x0 + 32 * q + lane >= ie) continue;
            unsigned lo = 0xFFu, hi = 0xFFu;
            if (idn[q] >= 0) {
                const int d = idn[q] - bdn;
                if (d >= 0 && d < 0xFF) lo = (unsigned)d; else bad = true;
            }
            if (iup[q] >= 0) {
                const int d = iup[q] - bup;
                if (d >= 0 && d < 0xFF) hi = (unsigned)d; else bad = true;
            }
            nbr[c0 + 32 * q + lane] = (unsigned short)(lo | (hi << 8));
        }
    }
    if (bad) atomicOr(status, 1);
}

// With BANDS, every row belongs to a band (row_band[row]) with its own
// spacing and time step: band_table[4 q .. 4 q + 3] = dx, dy (or their
// exact reciprocals), dt, and 1 when the reciprocals are given.  Chunks of a
// row whose band index is outside [0, nbands) are left unwritten.  With
// TABLE the neighbour-row indices come from the plan's neighbour table
// (sx_chunk_table_kernel) instead of a search: one coalesced 16-bit load per
// cell, issued together with the cell's own value.
// One chunk's update (the body of sx_upwind_chunk_kernel).  With EDGE false
// the chunk's cells and their left and right neighbours all lie in
// [0, width), so the domain tests are known to pass and are left out.  SGN
// holds the upwind sides the velocity selects (bit 0: a >= 0, the left
// neighbour; bit 1: b >= 0, the row below): the other side's neighbours are
// never read, as in the reference's update, which uses one side per axis.
template <typename T, bool TABLE, bool EDGE, int SGN>
__device__ __forceinline__ void sx_chunk_upwind(const int4 p0, const int4 p1, const int4 p2, const int4 p3, int lane,
                                                const int* __restrict__ b, const int* __restrict__ e,
                                                const int* __restrict__ coff, const unsigned short* __restrict__ nbr,
                                                const T* __restrict__ v, T* __restrict__ out, int width, T a, T bb,
                                                T dt, T dx, T dy, int pow2)
{
    constexpr bool LEFT = (SGN & 1) != 0, DOWN = (SGN & 2) != 0;
    const int x0 = p0.x, ie = p0.y, touch = p0.w, ib = p3.w;
    const long long c0 = p0.z;
    // sub-rounds that hold cells (the same for the whole warp): chunks of
    // short intervals skip the empty ones instead of issuing them masked
    const int nq = min(SX_CHUNK_SUB, (ie - x0 + 31) >> 5);
    T cen[SX_CHUNK_SUB];
    int inb[SX_CHUNK_SUB];  // value index of the neighbour in the row the velocity selects, -1 for none
    const SxRowReader rd = DOWN ? SxRowReader{p1.x, p1.y, p1.z, p1.w, p2.x} : SxRowReader{p2.y, p2.z, p2.w, p3.x, p3.y};
    if (TABLE) {
        const int base = sx_chunk_base(rd, x0);
        unsigned nb[SX_CHUNK_SUB];
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            const bool act = q < nq && x < ie;
            cen[q] = act ? v[c0 + 32 * q + lane] : (T)0;
            nb[q] = act ? (unsigned)__ldg(nbr + c0 + 32 * q + lane) : 0xFFFFu;
        }
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            const bool xin = !EDGE || (x >= 0 && x < width);
            const unsigned o = DOWN ? nb[q] & 0xFFu : nb[q] >> 8;
            inb[q] = (xin && o != 0xFFu) ? base + (int)o : -1;
        }
    } else {
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            cen[q] = (q < nq && x < ie) ? v[c0 + 32 * q + lane] : (T)0;
        }
        // neighbour-row value indices of all four sub-rounds first, then all
        // their loads at once, so the chunk waits for one round trip
        sx_row_indices<SX_CHUNK_SUB, EDGE>(rd, x0, nq, ie, width, b, e, coff, lane, inb);
    }
    T vnb[SX_CHUNK_SUB];
#pragma unroll
    for (int q = 0; q < SX_CHUNK_SUB; ++q) vnb[q] = inb[q] >= 0 ? v[inb[q]] : (T)0;
    T prev_last = (T)0;  // lane 31's centre of the previous sub-round
#pragma unroll
    for (int q = 0; q < SX_CHUNK_SUB; ++q) {
        if (q >= nq) break;
        const int x = x0 + 32 * q + lane;
        const bool act = x < ie;
        const long long c = c0 + 32 * q + lane;
        const T center = cen[q];
        T side;  // the horizontal neighbour the velocity selects
        if (LEFT) {
            T from_left = __shfl_up_sync(0xFFFFFFFFu, center, 1);
            if (lane == 0) from_left = prev_last;
            prev_last = __shfl_sync(0xFFFFFFFFu, center, 31);
            const bool lin = !EDGE || (x - 1 >= 0 && x - 1 < width);
            if (x - 1 >= ib) side = lin ? ((lane > 0 || q > 0) ? from_left : v[c - 1]) : (T)0;
            else side = (act && (touch & 1) && lin) ? v[c - 1] : (T)0;
        } else {
            T from_right = __shfl_down_sync(0xFFFFFFFFu, center, 1);
            const T next_first =
                q + 1 < SX_CHUNK_SUB ? __shfl_sync(0xFFFFFFFFu, cen[q + 1 < SX_CHUNK_SUB ? q + 1 : q], 0) : (T)0;
            if (lane == 31) from_right = next_first;
            const bool rin = !EDGE || (x + 1 >= 0 && x + 1 < width);
            if (x + 1 < ie) side = rin ? ((lane < 31 || q + 1 < SX_CHUNK_SUB) ? from_right : v[c + 1]) : (T)0;
            else side = (act && (touch & 2) && rin) ? v[c + 1] : (T)0;
        }
        if (act) {
            const T du_dx = sx_over(LEFT ? sx_sub(center, side) : sx_sub(side, center), dx, pow2);
            const T du_dy = sx_over(DOWN ? sx_sub(center, vnb[q]) : sx_sub(vnb[q], center), dy, pow2);
            out[c] = sx_upwind_update(center, du_dx, du_dy, a, bb, dt);
        }
    }
}

template <typename T, bool BANDS, bool TABLE, int SGN>
__global__ void __launch_bounds__(256, TABLE ? (sizeof(T) == 4 ? SX_UPWIND_TABLE_MIN_BLOCKS : 3) : SX_UPWIND_MIN_BLOCKS)
    sx_upwind_chunk_kernel(const int* __restrict__ off, const int* __restrict__ b, const int* __restrict__ e,
                           const int* __restrict__ coff, const int* __restrict__ info, long long chunks,
                           const int* __restrict__ lookup, const T* __restrict__ v, T* __restrict__ out, int width,
                           int height, T a, T bb, T dt_all, T dx_all, T dy_all, int pow2_all,
                           const int* __restrict__ row_band, const T* __restrict__ band_table, int nbands,
                           const unsigned short* __restrict__ nbr)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long u = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < chunks; u += warps) {
        const int4* pl = (const int4*)(info + (long long)SX_PLAN_INTS * u);
        const int4 p0 = __ldg(pl), p1 = __ldg(pl + 1), p2 = __ldg(pl + 2), p3 = __ldg(pl + 3);
        const int x0 = p0.x, ie = p0.y;
        T dt = dt_all, dx = dx_all, dy = dy_all;
        int pow2 = pow2_all;
        if (BANDS) {
            const int q = __ldg(row_band + p3.z);
            if (q < 0 || q >= nbands) continue;
            dx = __ldg(band_table + 4 * q);
            dy = __ldg(band_table + 4 * q + 1);
            dt = __ldg(band_table + 4 * q + 2);
            pow2 = __ldg(band_table + 4 * q + 3) != (T)0;
        }
        // interior chunk: every cell and its left and right neighbours inside [0, width)
        const bool edge = !(x0 >= 1 && x0 + min(ie - x0, SX_CHUNK) < width);  // x0 + ... <= ie: no overflow
        if (edge)
            sx_chunk_upwind<T, TABLE, true, SGN>(p0, p1, p2, p3, lane, b, e, coff, nbr, v, out, width, a, bb, dt, dx,
                                                 dy, pow2);
        else
            sx_chunk_upwind<T, TABLE, false, SGN>(p0, p1, p2, p3, lane, b, e, coff, nbr, v, out, width, a, bb, dt, dx,
                                                  dy, pow2);
    }
}

// Adjoint of the upwind step on a chunk plan (rows sorted and disjoint);
// same values as sx_upwind_adjoint_kernel.  One row reader per direction
// serves both arrays (w and u share the geometry).  Per-block float64
// partial sums of dL/da, dL/db go to partial[2 * block].
// One chunk of sx_upwind_adjoint_chunk_kernel; dL/da and dL/db are added
// into ga and gb.  With EDGE false the chunk's row lies in [0, height) and its
// cells and their left and right neighbours in [0, width), so the domain tests
// are known to pass and are left out.
template <typename T, bool TABLE, bool EDGE, int SGN>
__device__ __forceinline__ void sx_chunk_adjoint(const int4 p0, const int4 p1, const int4 p2, const int4 p3, int lane,
                                                 const int* __restrict__ b, const int* __restrict__ e,
                                                 const int* __restrict__ coff,
                                                 const unsigned short* __restrict__ nbr, const T* __restrict__ w,
                                                 const T* __restrict__ u, T* __restrict__ ubar, int width, int height,
                                                 T a, T bb, T dt, T dx, T dy, int pow2, double& ga, double& gb)
{
    const int x0 = p0.x, ie = p0.y, touch = p0.w, row = p3.z, ib = p3.w;
    const long long c0 = p0.z;
    T wc[SX_CHUNK_SUB], uc[SX_CHUNK_SUB];
#pragma unroll
    for (int q = 0; q < SX_CHUNK_SUB; ++q) {
        const bool act = x0 + 32 * q + lane < ie;
        wc[q] = act ? w[c0 + 32 * q + lane] : (T)0;
        uc[q] = act ? u[c0 + 32 * q + lane] : (T)0;
    }
    SxRowReader dn{p1.x, p1.y, p1.z, p1.w, p2.x};
    SxRowReader upr{p2.y, p2.z, p2.w, p3.x, p3.y};
    // neighbour-row value indices of all four sub-rounds first, then all
    // their loads at once.  u reads need the forward's domain test (made by
    // the index), w reads need this cell's domain as well (jdom).
    const bool rdom = !EDGE || (row >= 0 && row < height);
    int idn[SX_CHUNK_SUB], iup[SX_CHUNK_SUB];
    if (TABLE) {  // the plan's neighbour table, as in the forward step
        const int bdn = sx_chunk_base(dn, x0), bup = sx_chunk_base(upr, x0);
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            const unsigned nb = x < ie ? (unsigned)__ldg(nbr + c0 + 32 * q + lane) : 0xFFFFu;
            const bool xin = !EDGE || (x >= 0 && x < width);
            idn[q] = (xin && (nb & 0xFFu) != 0xFFu) ? bdn + (int)(nb & 0xFFu) : -1;
            iup[q] = (xin && (nb >> 8) != 0xFFu) ? bup + (int)(nb >> 8) : -1;
        }
    } else {
#pragma unroll
        for (int q = 0; q < SX_CHUNK_SUB; ++q) {
            const int x = x0 + 32 * q + lane;
            idn[q] = sx_row_index(dn, x, width, b, e, coff, x < ie);
            iup[q] = sx_row_index(upr, x, width, b, e, coff, x < ie);
        }
    }
    // u is read on the forward's upwind side, w on the other one (SGN as in sx_chunk_upwind)
    constexpr bool LEFT = (SGN & 1) != 0, DOWN = (SGN & 2) != 0;
    T urow[SX_CHUNK_SUB], wrow[SX_CHUNK_SUB];
#pragma unroll
    for (int q = 0; q < SX_CHUNK_SUB; ++q) {
        const int iu = DOWN ? idn[q] : iup[q], iw = DOWN ? iup[q] : idn[q];
        urow[q] = iu >= 0 ? u[iu] : (T)0;
        wrow[q] = iw >= 0 && rdom ? w[iw] : (T)0;
    }
    T wprev = (T)0, uprev = (T)0;
#pragma unroll
    for (int q = 0; q < SX_CHUNK_SUB; ++q) {
        const int x = x0 + 32 * q + lane;
        const bool act = x < ie;
        const long long c = c0 + 32 * q + lane;
        const bool jdom = !EDGE || (x >= 0 && x < width && row >= 0 && row < height);
        const bool first = lane == 0 && q == 0, last = lane == 31 && q + 1 == SX_CHUNK_SUB;
        // in-set values of w on one side and u on the other (the transpose checks only this cell's domain)
        T w_side, u_side;
        if (LEFT) {  // u from the left, w from the right
            T ul = __shfl_up_sync(0xFFFFFFFFu, uc[q], 1);
            if (lane == 0) ul = uprev;
            uprev = __shfl_sync(0xFFFFFFFFu, uc[q], 31);
            T wr = __shfl_down_sync(0xFFFFFFFFu, wc[q], 1);
            const int qn = q + 1 < SX_CHUNK_SUB ? q + 1 : q;
            const T wn = __shfl_sync(0xFFFFFFFFu, wc[qn], 0);
            if (lane == 31) wr = wn;
            if (x - 1 >= ib) {
                const T uv = first ? u[c - 1] : ul;
                u_side = (!EDGE || (x - 1 >= 0 && x - 1 < width)) ? uv : (T)0;
            } else {
                const bool t = act && (touch & 1);
                u_side = (t && (!EDGE || (x - 1 >= 0 && x - 1 < width))) ? u[c - 1] : (T)0;
            }
            if (x + 1 < ie) w_side = last ? w[c + 1] : wr;
            else w_side = (act && (touch & 2)) ? w[c + 1] : (T)0;
        } else {  // u from the right, w from the left
            T wl = __shfl_up_sync(0xFFFFFFFFu, wc[q], 1);
            if (lane == 0) wl = wprev;
            wprev = __shfl_sync(0xFFFFFFFFu, wc[q], 31);
            T ur = __shfl_down_sync(0xFFFFFFFFu, uc[q], 1);
            const int qn = q + 1 < SX_CHUNK_SUB ? q + 1 : q;
            const T un = __shfl_sync(0xFFFFFFFFu, uc[qn], 0);
            if (lane == 31) ur = un;
            if (x - 1 >= ib) w_side = first ? w[c - 1] : wl;
            else w_side = (act && (touch & 1)) ? w[c - 1] : (T)0;
            if (x + 1 < ie) {
                const T uv = last ? u[c + 1] : ur;
                u_side = (!EDGE || (x + 1 >= 0 && x + 1 < width)) ? uv : (T)0;
            } else {
                const bool t = act && (touch & 2);
                u_side = (t && (!EDGE || (x + 1 >= 0 && x + 1 < width))) ? u[c + 1] : (T)0;
            }
        }
        // rows above and below: w in-set needs jdom only (x is then inside the domain, so the
        // reader's domain test is the same), u needs the forward's domain test
        const T w_r = wrow[q], u_r = urow[q];
        if (act) {
            const T c_w = wc[q];
            const T tx = LEFT ? sx_over(sx_sub(c_w, jdom ? w_side : (T)0), dx, pow2)
                              : sx_over(sx_sub(jdom ? w_side : (T)0, c_w), dx, pow2);
            const T ty = DOWN ? sx_over(sx_sub(c_w, w_r), dy, pow2) : sx_over(sx_sub(w_r, c_w), dy, pow2);
            ubar[c] = sx_sub(c_w, sx_mul(dt, sx_add(sx_mul(a, tx), sx_mul(bb, ty))));
            const T c_u = uc[q];
            const T dux = LEFT ? sx_over(sx_sub(c_u, u_side), dx, pow2) : sx_over(sx_sub(u_side, c_u), dx, pow2);
            const T duy = DOWN ? sx_over(sx_sub(c_u, u_r), dy, pow2) : sx_over(sx_sub(u_r, c_u), dy, pow2);
            ga -= (double)dt * (double)c_w * (double)dux;
            gb -= (double)dt * (double)c_w * (double)duy;
        }
    }
}

template <typename T, bool TABLE, int SGN>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? SX_UPWIND_ADJOINT_MIN_BLOCKS : 2) sx_upwind_adjoint_chunk_kernel(const int* __restrict__ off,
                                                                      const int* __restrict__ b,
                                                                      const int* __restrict__ e,
                                                                      const int* __restrict__ coff,
                                                                      const int* __restrict__ info, long long chunks,
                                                                      const int* __restrict__ lookup,
                                                                      const unsigned short* __restrict__ nbr,
                                                                      const T* __restrict__ w, const T* __restrict__ u,
                                                                      T* __restrict__ ubar, int width, int height, T a,
                                                                      T bb, T dt, T dx, T dy, int pow2,
                                                                      double* __restrict__ partial)
{
    __shared__ double s_ga[8], s_gb[8];
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    double ga = 0.0, gb = 0.0;
    for (long long q0 = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); q0 < chunks; q0 += warps) {
        const int4* pl = (const int4*)(info + (long long)SX_PLAN_INTS * q0);
        const int4 p0 = __ldg(pl), p1 = __ldg(pl + 1), p2 = __ldg(pl + 2), p3 = __ldg(pl + 3);
        const int x0 = p0.x, ie = p0.y, row = p3.z;
        const bool edge = !(row >= 0 && row < height && x0 >= 1 && x0 + min(ie - x0, SX_CHUNK) < width);
        if (edge)
            sx_chunk_adjoint<T, TABLE, true, SGN>(p0, p1, p2, p3, lane, b, e, coff, nbr, w, u, ubar, width, height, a,
                                                  bb, dt, dx, dy, pow2, ga, gb);
        else
            sx_chunk_adjoint<T, TABLE, false, SGN>(p0, p1, p2, p3, lane, b, e, coff, nbr, w, u, ubar, width, height, a,
                                                   bb, dt, dx, dy, pow2, ga, gb);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ga += __shfl_down_sync(0xFFFFFFFFu, ga, o);
        gb += __shfl_down_sync(0xFFFFFFFFu, gb, o);
    }
    if (lane == 0) {
        s_ga[threadIdx.x >> 5] = ga;
        s_gb[threadIdx.x >> 5] = gb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int q = 0; q < 8; ++q) {
            ta += s_ga[q];
            tb += s_gb[q];
        }
        partial[2 * blockIdx.x] = ta;
        partial[2 * blockIdx.x + 1] = tb;
    }
}

__global__ void sx_row_lookup_kernel(const int* __restrict__ rows, int row_count, int height, int* __restrict__ lookup,
                                     int* __restrict__ flags)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < row_count; p += gridDim.x * blockDim.x) {
        const int r = rows[p];
        if (r < 0 || r >= height) {
            atomicOr(flags, 1);
            continue;
        }
        lookup[r] = p;
    }
}

// ---------------------------------------------------------------------------
// Gradient magnitude and threshold run-length encoding on a full
// width x height grid (regrid.py:20-124,172-223).  The gradient uses
// central differences inside and one-sided ones at the borders, with no
// /dx, and is sqrt(fma(gx, gx, gy*gy)) as the reference's GPU build
// computes it.  A run is a stretch of value >= threshold.  One warp per
// row, 32 columns per step: a ballot gives the mask, and the run starts and
// stops come from the mask and the carry bit.  Each run end is written once;
// when the width is not a multiple of 32 and a row's last cell is set, the
// reference writes that row's final end a second time into the next row's
// first slot (a race between its row blocks, regrid.py:66-124), which
// equals this result when its blocks retire in order.
// ---------------------------------------------------------------------------
template <bool GRAD>
__device__ __forceinline__ bool sx_pred(const float* __restrict__ d, int x, int y, int width, int height, float thr)
{
    const long long idx = (long long)y * width + x;
    if (!GRAD) return d[idx] >= thr;
    const float c = d[idx];
    float gx = 0.0f, gy = 0.0f;
    if (width > 1) {
        if (x == 0) gx = __fsub_rn(d[idx + 1], c);
        else if (x == width - 1) gx = __fsub_rn(c, d[idx - 1]);
        else gx = __fmul_rn(__fsub_rn(d[idx + 1], d[idx - 1]), 0.5f);
    }
    if (height > 1) {
        if (y == 0) gy = __fsub_rn(d[idx + width], c);
        else if (y == height - 1) gy = __fsub_rn(c, d[idx - width]);
        else gy = __fmul_rn(__fsub_rn(d[idx + width], d[idx - width]), 0.5f);
    }
    return sx_grad_norm(gx, gy) >= thr;
}

template <bool GRAD>
__global__ void sx_threshold_rle_kernel(const float* __restrict__ d, int width, int height, float thr,
                                        int* __restrict__ counts, const int* __restrict__ offsets,
                                        int* __restrict__ ob, int* __restrict__ oe)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; y < height; y += warps) {
        unsigned prev = 0u;
        int n = 0;
        const int base_out = ob ? offsets[y] : 0;
        for (int base = 0; base < width; base += 32) {
            const int x = base + lane;
            const bool on = x < width && sx_pred<GRAD>(d, x, y, width, height, thr);
            const unsigned m = __ballot_sync(0xFFFFFFFFu, on);
            const unsigned starts = m & ~((m << 1) | prev);
            const unsigned stops = ((m << 1) | prev) & ~m & ((width - base >= 32) ? 0xFFFFFFFFu : ((1u << (width - base)) - 1u));
            if (ob) {
                const unsigned below = (1u << lane) - 1u;
                if ((starts >> lane) & 1u) ob[base_out + n + __popc(starts & below)] = x;
                // a stop at bit j closes the run that started before it
                if ((stops >> lane) & 1u) oe[base_out + n + __popc(starts & below) - 1] = x;
            }
            n += __popc(starts);
            prev = (width - base >= 32) ? (m >> 31) & 1u : (m >> (width - base - 1)) & 1u;
        }
        if (ob && prev && lane == 0) oe[base_out + n - 1] = width;
        if (counts && lane == 0) counts[y] = n;
    }
}

// ---------------------------------------------------------------------------
// Compensated (Neumaier) sum in FP64 of a float or double array, in two
// stages: per-block partial (sum, compensation) pairs, then one block that
// combines them in a fixed order.  The result is deterministic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sx_neumaier(double& s, double& c, double v)
{
    const double t = __dadd_rn(s, v);
    if (fabs(s) >= fabs(v)) c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, t), v));
    else c = __dadd_rn(c, __dadd_rn(__dsub_rn(v, t), s));
    s = t;
}

template <typename T>
__global__ void sx_mass_partial_kernel(const T* __restrict__ v, long long n, double* __restrict__ part)
{
    __shared__ double ss[SX_BLOCK], sc[SX_BLOCK];
    double s = 0.0, c = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        sx_neumaier(s, c, (double)v[i]);
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, C = 0.0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            sx_neumaier(S, C, ss[t]);
            C = __dadd_rn(C, sc[t]);
        }
        part[2 * blockIdx.x] = S;
        part[2 * blockIdx.x + 1] = C;
    }
}

// Final combination of the per-block (sum, compensation) pairs, one block of
// 256 threads: each thread folds parts t, t + 256, ... with Neumaier steps,
// then a fixed tree merges the threads' pairs (Neumaier on the sums, the
// compensations added).  Deterministic.
__global__ void __launch_bounds__(256) sx_mass_final_kernel(const double* __restrict__ part, int parts, double scale,
                                                            double* __restrict__ out)
{
    __shared__ double ss[256], sc[256];
    double S = 0.0, C = 0.0;
    for (int t = threadIdx.x; t < parts; t += 256) {
        sx_neumaier(S, C, part[2 * t]);
        C = __dadd_rn(C, part[2 * t + 1]);
    }
    ss[threadIdx.x] = S;
    sc[threadIdx.x] = C;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            double s1 = ss[threadIdx.x], c1 = sc[threadIdx.x];
            sx_neumaier(s1, c1, ss[threadIdx.x + h]);
            ss[threadIdx.x] = s1;
            sc[threadIdx.x] = __dadd_rn(c1, sc[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = __dmul_rn(__dadd_rn(ss[0], sc[0]), scale);
}

// ---------------------------------------------------------------------------
// Row shape check: OR of SX_ROWS_* bits over all adjacent interval pairs.
// ---------------------------------------------------------------------------
__global__ void sx_check_rows_kernel(const int* __restrict__ b, const int* __restrict__ e, const int* __restrict__ off,
                                     int rows, long long n, int* flags)
{
    unsigned f = 0u;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int bi = b[i], ei = e[i];
        if (ei <= bi) f |= 4u;
        const int q = sx_row_of(off, rows, (int)i);
        if (i + 1 < off[q + 1]) {
            const int nb = b[i + 1], ne = e[i + 1];
            if (nb < bi) f |= 1u;
            if (nb < ei) f |= 2u;
            else if (nb == ei) f |= 8u;
            if (ne < ei) f |= 16u;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xFFFFFFFFu, f, o);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, (int)f);
}

cudaError_t sx_check_rows_launch(const int* b, const int* e, const int* off, int rows, long long n, int* flags,
                                 cudaStream_t stream)
{
    cudaError_t err = cudaMemsetAsync(flags, 0, sizeof(int), stream);
    if (err != cudaSuccess || n <= 0 || rows <= 0) return err;
    long long g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    sx_check_rows_kernel<<<(int)g, 256, 0, stream>>>(b, e, off, rows, n, flags);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Cell lookup (interval_field.py:162-297): global interval index holding
// (row, col), or -1.  Binary search over the row ids, then over the row's
// intervals (same search order as the reference).
// ---------------------------------------------------------------------------
__global__ void sx_locate_cells_kernel(const int* __restrict__ rows, const int* __restrict__ off, const int* __restrict__ b,
                                       const int* __restrict__ e, int row_count, const int* __restrict__ qr,
                                       const int* __restrict__ qc, long long q, int* __restrict__ out)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q; t += (long long)gridDim.x * blockDim.x) {
        int found = -1;
        if (row_count > 0) {
            const int row = qr[t], col = qc[t];
            int lo = 0, hi = row_count - 1, pos = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                const int v = rows[mid];
                if (v == row) {
                    pos = mid;
                    break;
                }
                if (v < row) lo = mid + 1; else hi = mid - 1;
            }
            if (pos >= 0) {
                lo = off[pos];
                hi = off[pos + 1] - 1;
                while (lo <= hi) {
                    const int mid = (lo + hi) >> 1;
                    if (col < b[mid]) hi = mid - 1;
                    else if (col >= e[mid]) lo = mid + 1;
                    else {
                        found = mid;
                        break;
                    }
                }
            }
        }
        out[t] = found;
    }
}

cudaError_t sx_locate_cells_launch(const int* rows, const int* off, const int* b, const int* e, int row_count,
                                   const int* qr, const int* qc, long long q, int* out, cudaStream_t stream)
{
    if (q <= 0) return cudaSuccess;
    long long g = (q + 255) / 256;
    if (g > 148 * 64) g = 148 * 64;
    sx_locate_cells_kernel<<<(int)g, 256, 0, stream>>>(rows, off, b, e, row_count, qr, qc, q, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Runs of cells equal to a target value, per interval
// (subsetix_amr2/fields.py:39-100).  Runs never cross an interval boundary.
// One warp per interval, 32 cells per step with a ballot, as in the
// threshold RLE.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void sx_value_runs_kernel(const T* __restrict__ v, const int* __restrict__ coff, int n, T target,
                                     int* __restrict__ counts, const int* __restrict__ run_off,
                                     const int* __restrict__ b, int* __restrict__ ob, int* __restrict__ oe)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int c0 = coff[i];
        const int w = coff[i + 1] - c0;
        const int base_out = ob ? run_off[i] : 0;
        const int x0 = ob ? b[i] : 0;
        unsigned prev = 0u;
        int k = 0;
        for (int base = 0; base < w; base += 32) {
            const int t = base + lane;
            const bool on = t < w && v[c0 + t] == target;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, on);
            const unsigned valid = (w - base >= 32) ? 0xFFFFFFFFu : ((1u << (w - base)) - 1u);
            const unsigned starts = m & ~((m << 1) | prev);
            const unsigned stops = ((m << 1) | prev) & ~m & valid;
            if (ob) {
                const unsigned below = (1u << lane) - 1u;
                if ((starts >> lane) & 1u) ob[base_out + k + __popc(starts & below)] = x0 + t;
                if ((stops >> lane) & 1u) oe[base_out + k + __popc(starts & below) - 1] = x0 + t;
            }
            k += __popc(starts);
            prev = (w - base >= 32) ? (m >> 31) & 1u : (m >> (w - base - 1)) & 1u;
        }
        if (ob && prev && lane == 0) oe[base_out + k - 1] = x0 + w;
        if (counts && lane == 0) counts[i] = w > 0 ? k : 0;
    }
}

__global__ void sx_gather_i32_kernel(const int* __restrict__ idx, int count, const int* __restrict__ src,
                                     int* __restrict__ dst)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) dst[p] = src[idx[p]];
}

cudaError_t sx_value_runs_launch(int type, const void* v, const int* coff, int n, const void* target, int* counts,
                                 const int* run_off, const int* b, int* ob, int* oe, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    long long g = ((long long)n * 32 + 255) / 256;
    if (g > 148 * 64) g = 148 * 64;
    const int grid = (int)g;
    switch (type) {
        case 0:
            sx_value_runs_kernel<float><<<grid, 256, 0, stream>>>((const float*)v, coff, n, *(const float*)target,
                                                                  counts, run_off, b, ob, oe);
            break;
        case 1:
            sx_value_runs_kernel<double><<<grid, 256, 0, stream>>>((const double*)v, coff, n, *(const double*)target,
                                                                   counts, run_off, b, ob, oe);
            break;
        case 2:
            sx_value_runs_kernel<signed char><<<grid, 256, 0, stream>>>((const signed char*)v, coff, n,
                                                                        *(const signed char*)target, counts, run_off,
                                                                        b, ob, oe);
            break;
        case 3:
            sx_value_runs_kernel<int><<<grid, 256, 0, stream>>>((const int*)v, coff, n, *(const int*)target, counts,
                                                                run_off, b, ob, oe);
            break;
        case 4:
            sx_value_runs_kernel<long long><<<grid, 256, 0, stream>>>((const long long*)v, coff, n,
                                                                      *(const long long*)target, counts, run_off, b,
                                                                      ob, oe);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t sx_gather_i32_launch(const int* idx, int count, const int* src, int* dst, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    long long g = (count + 255) / 256;
    if (g > 148 * 64) g = 148 * 64;
    sx_gather_i32_kernel<<<(int)g, 256, 0, stream>>>(idx, count, src, dst);
    return cudaGetLastError();
}

// Gradient magnitude of a full width x height grid into a float32 array
// (regrid.py:172-274); the same per-cell formula as the fused RLE.
__global__ void sx_gradient_kernel(const float* __restrict__ d, int width, int height, float* __restrict__ out)
{
    const long long cells = (long long)width * height;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < cells;
         idx += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(idx / width), x = (int)(idx - (long long)y * width);
        const float c = d[idx];
        float gx = 0.0f, gy = 0.0f;
        if (width > 1) {
            if (x == 0) gx = __fsub_rn(d[idx + 1], c);
            else if (x == width - 1) gx = __fsub_rn(c, d[idx - 1]);
            else gx = __fmul_rn(__fsub_rn(d[idx + 1], d[idx - 1]), 0.5f);
        }
        if (height > 1) {
            if (y == 0) gy = __fsub_rn(d[idx + width], c);
            else if (y == height - 1) gy = __fsub_rn(c, d[idx - width]);
            else gy = __fmul_rn(__fsub_rn(d[idx + width], d[idx - width]), 0.5f);
        }
        out[idx] = sx_grad_norm(gx, gy);
    }
}

cudaError_t sx_gradient_launch(const float* d, int width, int height, float* out, cudaStream_t stream)
{
    const long long cells = (long long)width * height;
    if (cells <= 0) return cudaSuccess;
    long long g = (cells + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    sx_gradient_kernel<<<(int)g, 256, 0, stream>>>(d, width, height, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static int sx_grid(long long work, int block, int cap = 65535 * 8)
{
    long long g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

cudaError_t sx_prolong_set_launch(const int* rows_in, const int* off, const int* b, const int* e, int rows, int n, int r,
                                  int* occupied, int* ord, int* result, const SxScanState& st, int* rows_out,
                                  int* off_out, int* ob, int* oe, cudaStream_t stream)
{
    sx_occupied_kernel<<<sx_grid(rows, 256), 256, 0, stream>>>(off, rows, occupied);
    cudaError_t err = sx_scan_i32_launch(occupied, rows, ord, result, st, stream);
    if (err != cudaSuccess) return err;
    sx_prolong_set_rows_kernel<<<sx_grid(rows, 256), 256, 0, stream>>>(rows_in, off, rows, ord, r, rows_out, off_out);
    if (n > 0)
        sx_prolong_set_intervals_kernel<<<sx_grid(n, 256), 256, 0, stream>>>(b, e, off, rows, n, r, ob, oe, result);
    return cudaGetLastError();
}

cudaError_t sx_prolong_field_launch(const int* off, int rows, const int* coff, int n, const int* foff_rows,
                                    const int* fcoff, int r, const void* cv, void* fv, int dbl, cudaStream_t stream)
{
    const int grid = sx_grid((long long)n * 32, 256);
    if (dbl) {
        if (r == 2)
            sx_prolong_field_kernel<double, 2><<<grid, 256, 0, stream>>>(off, rows, coff, n, foff_rows, fcoff, r,
                                                                         (const double*)cv, (double*)fv);
        else
            sx_prolong_field_kernel<double, 0><<<grid, 256, 0, stream>>>(off, rows, coff, n, foff_rows, fcoff, r,
                                                                         (const double*)cv, (double*)fv);
    } else {
        if (r == 2)
            sx_prolong_field_kernel<float, 2><<<grid, 256, 0, stream>>>(off, rows, coff, n, foff_rows, fcoff, r,
                                                                        (const float*)cv, (float*)fv);
        else
            sx_prolong_field_kernel<float, 0><<<grid, 256, 0, stream>>>(off, rows, coff, n, foff_rows, fcoff, r,
                                                                        (const float*)cv, (float*)fv);
    }
    return cudaGetLastError();
}

cudaError_t sx_restrict_check_launch(const int* crows, int crow_count, const int* coff_rows, const int* cb,
                                     const int* ce, int cn, const int* frows, int frow_count, const int* foff_rows,
                                     const int* fb, const int* fe, int fn, int r, int* flags, cudaStream_t stream)
{
    long long work = (long long)(crow_count > cn ? crow_count : cn) * r;
    sx_restrict_check_kernel<<<sx_grid(work, 256), 256, 0, stream>>>(crows, crow_count, coff_rows, cb, ce, cn, frows,
                                                                     frow_count, foff_rows, fb, fe, fn, r, flags);
    return cudaGetLastError();
}

cudaError_t sx_restrict_field_launch(const int* coff_rows, int crow_count, const int* ccoff, int cn,
                                     const int* foff_rows, const int* fcoff, int r, int reducer, double norm,
                                     const void* fv, void* cv, int dbl, cudaStream_t stream)
{
    const int grid = sx_grid((long long)cn * 32, 256);
    if (dbl) {
        if (r == 2)
            sx_restrict_field_kernel<double, 2><<<grid, 256, 0, stream>>>(coff_rows, crow_count, ccoff, cn, foff_rows,
                                                                          fcoff, r, reducer, norm, (const double*)fv,
                                                                          (double*)cv);
        else
            sx_restrict_field_kernel<double, 0><<<grid, 256, 0, stream>>>(coff_rows, crow_count, ccoff, cn, foff_rows,
                                                                          fcoff, r, reducer, norm, (const double*)fv,
                                                                          (double*)cv);
    } else {
        if (r == 2)
            sx_restrict_field_kernel<float, 2><<<grid, 256, 0, stream>>>(coff_rows, crow_count, ccoff, cn, foff_rows,
                                                                         fcoff, r, reducer, (float)norm,
                                                                         (const float*)fv, (float*)cv);
        else
            sx_restrict_field_kernel<float, 0><<<grid, 256, 0, stream>>>(coff_rows, crow_count, ccoff, cn, foff_rows,
                                                                         fcoff, r, reducer, (float)norm,
                                                                         (const float*)fv, (float*)cv);
    }
    return cudaGetLastError();
}

cudaError_t sx_subset_rows_launch(const int* soff, const int* srows, int srow_count, int sn, const int* urows,
                                  int urow_count, int* pos, int* flags, cudaStream_t stream)
{
    if (sn <= 0) return cudaSuccess;
    sx_subset_rows_kernel<<<sx_grid(sn, 256), 256, 0, stream>>>(soff, srows, srow_count, sn, urows, urow_count, pos,
                                                                 flags);
    return cudaGetLastError();
}

cudaError_t sx_subset_copy_launch(int scatter, int n, const int* pos, const int* sb, const int* se, const int* scoff,
                                  const int* uoff, const int* ub, const int* ue, const int* ucoff, int urows,
                                  void* sub, void* sup, int elem_size, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int grid = sx_grid((long long)n * 32, 256);
    switch (elem_size) {
        case 1:
            sx_subset_copy_kernel<unsigned char><<<grid, 256, 0, stream>>>(scatter, n, pos, sb, se, scoff, uoff, ub, ue,
                                                                           ucoff, urows, (unsigned char*)sub,
                                                                           (unsigned char*)sup);
            break;
        case 4:
            sx_subset_copy_kernel<unsigned int><<<grid, 256, 0, stream>>>(scatter, n, pos, sb, se, scoff, uoff, ub, ue,
                                                                          ucoff, urows, (unsigned int*)sub,
                                                                          (unsigned int*)sup);
            break;
        case 8:
            sx_subset_copy_kernel<unsigned long long><<<grid, 256, 0, stream>>>(scatter, n, pos, sb, se, scoff, uoff, ub,
                                                                                ue, ucoff, urows,
                                                                                (unsigned long long*)sub,
                                                                                (unsigned long long*)sup);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t sx_row_lookup_launch(const int* rows, int row_count, int height, int* lookup, int* flags,
                                 cudaStream_t stream)
{
    cudaError_t err = cudaMemsetAsync(lookup, 0xFF, (size_t)height * sizeof(int), stream);
    if (err != cudaSuccess) return err;
    if (row_count > 0)
        sx_row_lookup_kernel<<<sx_grid(row_count, 256), 256, 0, stream>>>(rows, row_count, height, lookup, flags);
    return cudaGetLastError();
}

cudaError_t sx_upwind_launch(const int* rows, const int* rid, const int* off, int row_count, const int* b, const int* e, const int* coff,
                             int n, long long cells, const int* lookup, const void* v, void* out, int width, int height,
                             double a, double bb, double dt, double dx, double dy, int direct, int dbl,
                             cudaStream_t stream)
{
    if (n <= 0 || cells <= 0) return cudaSuccess;
    const int grid = sx_grid(cells, 256, 148 * 16);
    if (dbl)
        sx_upwind_kernel<double><<<grid, 256, 0, stream>>>(rows, rid, off, row_count, b, e, coff, n, lookup, (const double*)v,
                                                           (double*)out, width, height, a, bb, dt, dx, dy, direct, cells);
    else
        sx_upwind_kernel<float><<<grid, 256, 0, stream>>>(rows, rid, off, row_count, b, e, coff, n, lookup, (const float*)v,
                                                          (float*)out, width, height, (float)a, (float)bb, (float)dt,
                                                          (float)dx, (float)dy, direct, cells);
    return cudaGetLastError();
}

cudaError_t sx_threshold_launch(const float* d, int width, int height, float thr, int grad, int* counts,
                                const int* offsets, int* ob, int* oe, cudaStream_t stream)
{
    const int grid = sx_grid((long long)height * 32, 256);
    if (grad) sx_threshold_rle_kernel<true><<<grid, 256, 0, stream>>>(d, width, height, thr, counts, offsets, ob, oe);
    else sx_threshold_rle_kernel<false><<<grid, 256, 0, stream>>>(d, width, height, thr, counts, offsets, ob, oe);
    return cudaGetLastError();
}

cudaError_t sx_mass_launch(const void* v, long long n, int dbl, double scale, double* part, int parts, double* out,
                           cudaStream_t stream)
{
    if (dbl) sx_mass_partial_kernel<double><<<parts, SX_BLOCK, 0, stream>>>((const double*)v, n, part);
    else sx_mass_partial_kernel<float><<<parts, SX_BLOCK, 0, stream>>>((const float*)v, n, part);
    sx_mass_final_kernel<<<1, 256, 0, stream>>>(part, parts, scale, out);
    return cudaGetLastError();
}

int sx_upwind_adjoint_parts(long long cells)
{
    long long g = (cells + 255) / 256;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

cudaError_t sx_upwind_adjoint_launch(const int* rows, const int* off, int row_count, const int* b, const int* e,
                                     const int* coff, int n, long long cells, const int* lookup, const void* w,
                                     const void* u, void* ubar, int width, int height, double a, double bb, double dt,
                                     double dx, double dy, int direct, int dbl, double* partial, double* grads,
                                     cudaStream_t stream)
{
    const int grid = sx_upwind_adjoint_parts(cells);
    if (dbl)
        sx_upwind_adjoint_kernel<double><<<grid, 256, 0, stream>>>(rows, off, row_count, b, e, coff, n, lookup,
                                                                   (const double*)w, (const double*)u, (double*)ubar,
                                                                   width, height, a, bb, dt, dx, dy, direct, cells,
                                                                   partial);
    else
        sx_upwind_adjoint_kernel<float><<<grid, 256, 0, stream>>>(rows, off, row_count, b, e, coff, n, lookup,
                                                                  (const float*)w, (const float*)u, (float*)ubar, width,
                                                                  height, (float)a, (float)bb, (float)dt, (float)dx,
                                                                  (float)dy, direct, cells, partial);
    sx_sum_pairs_kernel<<<1, 256, 0, stream>>>(partial, grid, grads);
    return cudaGetLastError();
}

cudaError_t sx_upwind_plan_launch(const int* b, const int* e, int n, int* chunk_off, int* result, const SxScanState& st,
                                  cudaStream_t stream)
{
    if (n > 0) sx_chunk_count_kernel<<<sx_grid(n, 256), 256, 0, stream>>>(b, e, n, chunk_off);
    // in place: each scan thread reads its own items before writing them
    return sx_scan_i32_launch(chunk_off, n, chunk_off, result, st, stream);
}

cudaError_t sx_upwind_plan_fill_launch(const int* rows, const int* off, int row_count, const int* b, const int* e,
                                       const int* coff, int n, const int* chunk_off, long long chunks,
                                       const int* lookup, int height, int* info, cudaStream_t stream)
{
    if (n <= 0 || chunks <= 0) return cudaSuccess;
    sx_chunk_info_kernel<<<sx_grid(chunks, 256, 148 * 32), 256, 0, stream>>>(rows, off, row_count, b, e, coff, n,
                                                                             chunk_off, chunks, lookup, height, info);
    return cudaGetLastError();
}

cudaError_t sx_upwind_table_launch(const int* b, const int* e, const int* coff, const int* info, long long chunks,
                                   unsigned short* nbr, int* status, cudaStream_t stream)
{
    cudaError_t err = cudaMemsetAsync(status, 0, sizeof(int), stream);
    if (err != cudaSuccess || chunks <= 0) return err;
    long long blocks = (chunks + 7) / 8;
    if (blocks > 148 * 64) blocks = 148 * 64;
    sx_chunk_table_kernel<<<(int)blocks, 256, 0, stream>>>(b, e, coff, info, chunks, nbr, status);
    return cudaGetLastError();
}

// The upwind sides of the velocity (SGN) select the kernel instance.
template <typename T, bool BANDS, int SGN>
static void sx_upwind_chunk_go_s(int blocks, const int* off, const int* b, const int* e, const int* coff,
                                 const int* info, long long chunks, const int* lookup, const T* v, T* out, int width,
                                 int height, T a, T bb, T dt, T dx, T dy, int p, const int* row_band,
                                 const T* band_table, int nbands, const unsigned short* nbr, cudaStream_t stream)
{
    if (nbr)
        sx_upwind_chunk_kernel<T, BANDS, true, SGN><<<blocks, 256, 0, stream>>>(off, b, e, coff, info, chunks, lookup,
                                                                               v, out, width, height, a, bb, dt, dx,
                                                                               dy, p, row_band, band_table, nbands,
                                                                               nbr);
    else
        sx_upwind_chunk_kernel<T, BANDS, false, SGN><<<blocks, 256, 0, stream>>>(off, b, e, coff, info, chunks,
                                                                                lookup, v, out, width, height, a, bb,
                                                                                dt, dx, dy, p, row_band, band_table,
                                                                                nbands, nullptr);
}

template <typename T, bool BANDS>
static void sx_upwind_chunk_go(int blocks, const int* off, const int* b, const int* e, const int* coff,
                               const int* info, long long chunks, const int* lookup, const T* v, T* out, int width,
                               int height, T a, T bb, T dt, T dx, T dy, int p, const int* row_band, const T* band_table,
                               int nbands, const unsigned short* nbr, cudaStream_t stream)
{
    const int sgn = (a >= (T)0 ? 1 : 0) | (bb >= (T)0 ? 2 : 0);
    switch (sgn) {
        case 0: return sx_upwind_chunk_go_s<T, BANDS, 0>(blocks, off, b, e, coff, info, chunks, lookup, v, out, width,
                                                         height, a, bb, dt, dx, dy, p, row_band, band_table, nbands,
                                                         nbr, stream);
        case 1: return sx_upwind_chunk_go_s<T, BANDS, 1>(blocks, off, b, e, coff, info, chunks, lookup, v, out, width,
                                                         height, a, bb, dt, dx, dy, p, row_band, band_table, nbands,
                                                         nbr, stream);
        case 2: return sx_upwind_chunk_go_s<T, BANDS, 2>(blocks, off, b, e, coff, info, chunks, lookup, v, out, width,
                                                         height, a, bb, dt, dx, dy, p, row_band, band_table, nbands,
                                                         nbr, stream);
        default: return sx_upwind_chunk_go_s<T, BANDS, 3>(blocks, off, b, e, coff, info, chunks, lookup, v, out,
                                                          width, height, a, bb, dt, dx, dy, p, row_band, band_table,
                                                          nbands, nbr, stream);
    }
}

static int sx_chunk_blocks(long long chunks)
{
    long long blocks = (chunks + 7) / 8;
    return (int)(blocks > 148 * 64 ? 148 * 64 : blocks);
}

cudaError_t sx_upwind_chunk_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                   long long chunks, const int* lookup, const unsigned short* nbr, const void* v,
                                   void* out, int width, int height, double a, double bb, double dt, double dx,
                                   double dy, int dbl, cudaStream_t stream)
{
    if (chunks <= 0) return cudaSuccess;
    const int blocks = sx_chunk_blocks(chunks);
    if (dbl) {
        double ddx = dx, ddy = dy;
        const int p = sx_pow2_pair(ddx, ddy);
        sx_upwind_chunk_go<double, false>(blocks, off, b, e, coff, info, chunks, lookup, (const double*)v,
                                          (double*)out, width, height, a, bb, dt, ddx, ddy, p, nullptr, nullptr, 0, nbr,
                                          stream);
    } else {
        float fdx = (float)dx, fdy = (float)dy;
        const int p = sx_pow2_pair(fdx, fdy);
        sx_upwind_chunk_go<float, false>(blocks, off, b, e, coff, info, chunks, lookup, (const float*)v, (float*)out,
                                         width, height, (float)a, (float)bb, (float)dt, fdx, fdy, p, nullptr, nullptr,
                                         0, nbr, stream);
    }
    return cudaGetLastError();
}

cudaError_t sx_upwind_chunk_bands_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                         long long chunks, const int* lookup, const unsigned short* nbr, const void* v,
                                         void* out, int width, int height, double a, double bb, const int* row_band,
                                         const void* band_table, int nbands, int dbl, cudaStream_t stream)
{
    if (chunks <= 0) return cudaSuccess;
    const int blocks = sx_chunk_blocks(chunks);
    if (dbl)
        sx_upwind_chunk_go<double, true>(blocks, off, b, e, coff, info, chunks, lookup, (const double*)v, (double*)out,
                                         width, height, a, bb, 0.0, 1.0, 1.0, 0, row_band, (const double*)band_table,
                                         nbands, nbr, stream);
    else
        sx_upwind_chunk_go<float, true>(blocks, off, b, e, coff, info, chunks, lookup, (const float*)v, (float*)out,
                                        width, height, (float)a, (float)bb, 0.0f, 1.0f, 1.0f, 0, row_band,
                                        (const float*)band_table, nbands, nbr, stream);
    return cudaGetLastError();
}

// Host: per-band table of the banded launch in the kernel's precision.
template <typename T>
static void sx_band_table_fill(const double* spacing, int nbands, T* table)
{
    for (int q = 0; q < nbands; ++q) {
        T dx = (T)spacing[3 * q], dy = (T)spacing[3 * q + 1];
        const int p = sx_pow2_pair(dx, dy);
        table[4 * q] = dx;
        table[4 * q + 1] = dy;
        table[4 * q + 2] = (T)spacing[3 * q + 2];
        table[4 * q + 3] = (T)p;
    }
}

void sx_upwind_band_table_fill(int dbl, const double* spacing, int nbands, void* table)
{
    if (dbl) sx_band_table_fill<double>(spacing, nbands, (double*)table);
    else sx_band_table_fill<float>(spacing, nbands, (float*)table);
}

int sx_upwind_adjoint_chunk_parts(long long chunks)
{
    long long blocks = (chunks + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 16) blocks = 148 * 16;
    return (int)blocks;
}

template <typename T, int SGN>
static void sx_upwind_adjoint_chunk_go_s(int blocks, const int* off, const int* b, const int* e, const int* coff,
                                         const int* info, long long chunks, const int* lookup,
                                         const unsigned short* nbr, const T* w, const T* u, T* ubar, int width,
                                         int height, T a, T bb, T dt, T dx, T dy, int p, double* partial,
                                         cudaStream_t stream)
{
    if (nbr)
        sx_upwind_adjoint_chunk_kernel<T, true, SGN><<<blocks, 256, 0, stream>>>(off, b, e, coff, info, chunks, lookup,
                                                                                 nbr, w, u, ubar, width, height, a, bb,
                                                                                 dt, dx, dy, p, partial);
    else
        sx_upwind_adjoint_chunk_kernel<T, false, SGN><<<blocks, 256, 0, stream>>>(off, b, e, coff, info, chunks,
                                                                                  lookup, nullptr, w, u, ubar, width,
                                                                                  height, a, bb, dt, dx, dy, p,
                                                                                  partial);
}

// The upwind sides of the velocity select the kernel instance (as in the forward step).
template <typename T>
static void sx_upwind_adjoint_chunk_go(int blocks, const int* off, const int* b, const int* e, const int* coff,
                                       const int* info, long long chunks, const int* lookup, const unsigned short* nbr,
                                       const T* w, const T* u, T* ubar, int width, int height, T a, T bb, T dt, T dx,
                                       T dy, int p, double* partial, cudaStream_t stream)
{
    switch ((a >= (T)0 ? 1 : 0) | (bb >= (T)0 ? 2 : 0)) {
        case 0: return sx_upwind_adjoint_chunk_go_s<T, 0>(blocks, off, b, e, coff, info, chunks, lookup, nbr, w, u,
                                                          ubar, width, height, a, bb, dt, dx, dy, p, partial, stream);
        case 1: return sx_upwind_adjoint_chunk_go_s<T, 1>(blocks, off, b, e, coff, info, chunks, lookup, nbr, w, u,
                                                          ubar, width, height, a, bb, dt, dx, dy, p, partial, stream);
        case 2: return sx_upwind_adjoint_chunk_go_s<T, 2>(blocks, off, b, e, coff, info, chunks, lookup, nbr, w, u,
                                                          ubar, width, height, a, bb, dt, dx, dy, p, partial, stream);
        default: return sx_upwind_adjoint_chunk_go_s<T, 3>(blocks, off, b, e, coff, info, chunks, lookup, nbr, w, u,
                                                           ubar, width, height, a, bb, dt, dx, dy, p, partial, stream);
    }
}

cudaError_t sx_upwind_adjoint_chunk_launch(const int* off, const int* b, const int* e, const int* coff, const int* info,
                                           long long chunks, const int* lookup, const unsigned short* nbr,
                                           const void* w, const void* u, void* ubar, int width, int height, double a,
                                           double bb, double dt, double dx, double dy, int dbl, double* partial,
                                           double* grads, cudaStream_t stream)
{
    const int blocks = sx_upwind_adjoint_chunk_parts(chunks);
    if (dbl) {
        double ddx = dx, ddy = dy;
        const int p = sx_pow2_pair(ddx, ddy);
        sx_upwind_adjoint_chunk_go<double>(blocks, off, b, e, coff, info, chunks, lookup, nbr, (const double*)w,
                                           (const double*)u, (double*)ubar, width, height, a, bb, dt, ddx, ddy, p,
                                           partial, stream);
    } else {
        float fdx = (float)dx, fdy = (float)dy;
        const int p = sx_pow2_pair(fdx, fdy);
        sx_upwind_adjoint_chunk_go<float>(blocks, off, b, e, coff, info, chunks, lookup, nbr, (const float*)w,
                                          (const float*)u, (float*)ubar, width, height, (float)a, (float)bb, (float)dt,
                                          fdx, fdy, p, partial, stream);
    }
    sx_sum_pairs_kernel<<<1, 256, 0, stream>>>(partial, blocks, grads);
    return cudaGetLastError();
}
