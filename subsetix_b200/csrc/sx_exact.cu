// Exact reference-order kernels: the fallback of the fused fast path.
//
// These kernels give the reference's results for any input, including
// touching, overlapping, empty or unsorted intervals.  They follow its
// sequential per-row sweeps exactly.
//   * binary set operations (subsetix_cupy/kernels.py:11-235): the union
//     merges by begin with ties to the left operand and extends a run while
//     begin <= running end; the intersection emits [max b, min e) and
//     advances the left operand when a_end <= b_end; the difference runs a
//     cursor over the right operand and carries its index across left
//     intervals;
//   * run merge of begin-sorted rows (kernels.py:292-381).
// One thread handles one row, and every kernel has a count mode and a write
// mode.  Offsets come from sx_scan_i32.  The fused kernel (sx_bool.cu)
// covers canonical inputs and is much faster.  These kernels run only when
// it raises SXF_CONTRACT or SXF_LONG_TILE.

#include "sx_internal.cuh"

template <bool WRITE>
__device__ __forceinline__ int sx_row_op(int op, const int* __restrict__ lb, const int* __restrict__ le, int li, int ln,
                                         const int* __restrict__ rb, const int* __restrict__ re, int rj, int rn,
                                         int* __restrict__ ob, int* __restrict__ oe)
{
    int n = 0;
    if (op == 0) {
        bool have = false;
        int cb = 0, ce = 0;
        while (li < ln || rj < rn) {
            const bool left = (rj >= rn) || (li < ln && lb[li] <= rb[rj]);
            const int sb = left ? lb[li] : rb[rj];
            const int se = left ? le[li] : re[rj];
            if (left) ++li; else ++rj;
            if (!have) {
                have = true;
                cb = sb;
                ce = se;
            } else if (sb <= ce) {
                if (se > ce) ce = se;
            } else {
                if (WRITE) { ob[n] = cb; oe[n] = ce; }
                ++n;
                cb = sb;
                ce = se;
            }
        }
        if (have) {
            if (WRITE) { ob[n] = cb; oe[n] = ce; }
            ++n;
        }
    } else if (op == 1) {
        while (li < ln && rj < rn) {
            const int a0 = lb[li], a1 = le[li], b0 = rb[rj], b1 = re[rj];
            const int s0 = a0 > b0 ? a0 : b0;
            const int s1 = a1 < b1 ? a1 : b1;
            if (s0 < s1) {
                if (WRITE) { ob[n] = s0; oe[n] = s1; }
                ++n;
            }
            if (a1 <= b1) ++li; else ++rj;
        }
    } else {
        for (; li < ln; ++li) {
            const int a1 = le[li];
            int cur = lb[li];
            while (cur < a1) {
                while (rj < rn && re[rj] <= cur) ++rj;
                if (rj >= rn || rb[rj] >= a1) {
                    if (WRITE) { ob[n] = cur; oe[n] = a1; }
                    ++n;
                    break;
                }
                const int b0 = rb[rj];
                if (b0 > cur) {
                    const int stop = b0 < a1 ? b0 : a1;
                    if (stop > cur) {
                        if (WRITE) { ob[n] = cur; oe[n] = stop; }
                        ++n;
                    }
                }
                cur = re[rj];  // re[rj] > cur after the skip loop
            }
        }
    }
    return n;
}

__global__ void sx_exact_setop_kernel(int op, int rows, const int* __restrict__ lb, const int* __restrict__ le,
                                      const int* __restrict__ loff, const int* __restrict__ rb,
                                      const int* __restrict__ re, const int* __restrict__ roff,
                                      int* __restrict__ counts, const int* __restrict__ offsets,
                                      int* __restrict__ ob, int* __restrict__ oe)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    if (ob == nullptr) {
        counts[r] = sx_row_op<false>(op, lb, le, loff[r], loff[r + 1], rb, re, roff[r], roff[r + 1], nullptr, nullptr);
    } else {
        const int o = offsets[r];
        sx_row_op<true>(op, lb, le, loff[r], loff[r + 1], rb, re, roff[r], roff[r + 1], ob + o, oe + o);
    }
}

__global__ void sx_merge_rows_kernel(int rows, const int* __restrict__ b, const int* __restrict__ e,
                                     const int* __restrict__ off, int* __restrict__ counts,
                                     const int* __restrict__ out_off, int* __restrict__ ob, int* __restrict__ oe)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int s = off[r], t = off[r + 1];
    int n = 0;
    if (s < t) {
        int cb = b[s], ce = e[s];
        int w = ob ? out_off[r] : 0;
        for (int i = s + 1; i < t; ++i) {
            const int bi = b[i], ei = e[i];
            if (bi <= ce) {
                if (ei > ce) ce = ei;
            } else {
                if (ob) { ob[w] = cb; oe[w] = ce; ++w; }
                ++n;
                cb = bi;
                ce = ei;
            }
        }
        if (ob) { ob[w] = cb; oe[w] = ce; }
        ++n;
    }
    if (counts) counts[r] = n;
}

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total), with a
// single-pass decoupled look-back.  result[0] receives the total and
// result[1] the flags.
#define SX_SCAN_ITEMS 8
__global__ void __launch_bounds__(SX_BLOCK) sx_scan_i32_kernel(const int* __restrict__ in, long long n,
                                                               int* __restrict__ out, int* result, SxScanState st)
{
    __shared__ int s_tile;
    __shared__ unsigned s_epoch;
    __shared__ int s_warp[SX_BLOCK / 32];
    __shared__ int s_base;
    __shared__ unsigned s_flags;
    sx_ticket(st, &s_tile, &s_epoch);
    const int tile = s_tile;
    const unsigned epoch = s_epoch;
    if (threadIdx.x == 0) s_flags = 0u;
    const long long base_idx = (long long)tile * SX_BLOCK * SX_SCAN_ITEMS + (long long)threadIdx.x * SX_SCAN_ITEMS;
    int v[SX_SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SX_SCAN_ITEMS; ++i) {
        const long long idx = base_idx + i;
        v[i] = idx < n ? in[idx] : 0;
        sum += v[i];
    }
    int total;
    const int ex = sx_block_exclusive_scan(sum, s_warp, &total);
    if (threadIdx.x < 32) {
        unsigned f = 0u;
        const int b = sx_lookback_warp(st, tile, epoch, total, f);
        if (threadIdx.x == 0) {
            s_base = b;
            s_flags = f;
        }
    }
    __syncthreads();
    int run = s_base + ex;
#pragma unroll
    for (int i = 0; i < SX_SCAN_ITEMS; ++i) {
        const long long idx = base_idx + i;
        if (idx < n) out[idx] = run;
        run += v[i];
        if (idx == n - 1) out[n] = run;
    }
    if (n == 0 && tile == 0 && threadIdx.x == 0) out[0] = 0;
    sx_retire(st, epoch, s_flags, result);
}

int sx_scan_tiles(long long n)
{
    long long per = (long long)SX_BLOCK * SX_SCAN_ITEMS;
    long long t = (n + per - 1) / per;
    return t < 1 ? 1 : (int)t;
}

cudaError_t sx_scan_i32_launch(const int* in, long long n, int* out, int* result, const SxScanState& st,
                               cudaStream_t stream)
{
    const int tiles = sx_scan_tiles(n);
    // Clear the look-back state: the workspace may hold scratch from earlier
    // calls.  The counters (16 bytes) are immediately followed by the status words.
    cudaError_t err = cudaMemsetAsync(st.counters, 0, 16 + (size_t)tiles * 8, stream);
    if (err != cudaSuccess) return err;
    sx_scan_i32_kernel<<<tiles, SX_BLOCK, 0, stream>>>(in, n, out, result, st);
    return cudaGetLastError();
}

cudaError_t sx_exact_setop_launch(int op, int rows, const int* lb, const int* le, const int* loff, const int* rb,
                                  const int* re, const int* roff, int* counts, const int* offsets, int* ob, int* oe,
                                  cudaStream_t stream)
{
    if (rows <= 0) return cudaSuccess;
    const int block = 128;
    sx_exact_setop_kernel<<<(rows + block - 1) / block, block, 0, stream>>>(op, rows, lb, le, loff, rb, re, roff, counts,
                                                                          offsets, ob, oe);
    return cudaGetLastError();
}

cudaError_t sx_merge_rows_launch(int rows, const int* b, const int* e, const int* off, int* counts, const int* out_off,
                                 int* ob, int* oe, cudaStream_t stream)
{
    if (rows <= 0) return cudaSuccess;
    const int block = 128;
    sx_merge_rows_kernel<<<(rows + block - 1) / block, block, 0, stream>>>(rows, b, e, off, counts, out_off, ob, oe);
    return cudaGetLastError();
}
