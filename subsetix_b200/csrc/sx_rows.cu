// Row alignment: the sorted union of several row-id lists, and each list's
// row offsets re-expressed on that union.
//
// This is the device form of the reference's _align_interval_sets /
// _reindex_interval_set (subsetix_cupy/expressions.py:58-141).  The output
// row list is union1d of the operands' rows.  Each operand keeps its
// intervals in order, and rows it lacks become empty rows.  Because the
// intervals keep their order, only the offsets change:
//     aligned_off[y] = off[lower_bound(rows + shift, rows_out[y])].
// Dilation uses the same kernels.  There each list is a set's occupied rows
// shifted by dy (skip_empty = 1), matching morphology.py:236-247.
//
// The union is built from a bitmap over [row_min, row_max], a scan of the
// per-word popcounts, and a compaction.  row_min and row_max come from the
// host.

#include <climits>

#include "sx_internal.cuh"

__global__ void sx_align_clear_kernel(unsigned* bitmap, long long nwords)
{
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x)
        bitmap[w] = 0u;
}

__global__ void sx_align_mark_kernel(SxAlignArgs A)
{
    const int l = blockIdx.y;
    const SxRowList L = A.list[l];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        if (L.skip_empty && L.off[i + 1] <= L.off[i]) continue;
        long long u = (long long)L.rows[i] + L.shift;
        if (L.div > 1) u = u >= 0 ? u / L.div : -((-u + L.div - 1) / L.div);  // floor division
        const long long v = u - A.row_min;
        if (v < 0 || v >= A.nbits) continue;  // excluded by the caller's bounds
        atomicOr(&A.bitmap[v >> 5], 1u << (v & 31));
    }
}

__global__ void sx_align_popc_kernel(const unsigned* bitmap, long long nwords, int* wcount)
{
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x)
        wcount[w] = __popc(bitmap[w]);
}

__global__ void sx_align_compact_kernel(SxAlignArgs A, long long nwords)
{
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        unsigned m = A.bitmap[w];
        int o = A.wprefix[w];
        while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1u;
            A.rows_out[o++] = A.row_min + (int)(w * 32 + bit);
        }
    }
}

// aligned[l][y] for y in [0, R_out]; R_out is read from the device.
__global__ void sx_align_offsets_kernel(SxAlignArgs A)
{
    const int l = blockIdx.y;
    int* dst = A.aligned[l];
    if (dst == nullptr) return;
    const SxRowList L = A.list[l];
    int* dst_end = A.aligned_end[l];
    const int rout = A.result[0];
    const long long div = L.div > 1 ? L.div : 1;
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y <= rout; y += gridDim.x * blockDim.x) {
        // The closing offset stops after the last output row, so source rows
        // beyond row_max do not leak into it.
        int pos;
        long long key = 0;
        if (y == rout && rout == 0) {
            pos = L.count;
        } else {
            key = y == rout ? ((long long)A.rows_out[rout - 1] + 1) * div + L.phase - L.shift
                            : (long long)A.rows_out[y] * div + L.phase - L.shift;
            int lo = 0, hi = L.count;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if ((long long)L.rows[mid] < key) lo = mid + 1; else hi = mid;
            }
            pos = lo;
        }
        const int start = L.count > 0 ? L.off[pos] : 0;
        dst[y] = start;
        if (dst_end && y < rout)
            dst_end[y] = (pos < L.count && (long long)L.rows[pos] == key) ? L.off[pos + 1] : start;
    }
}

cudaError_t sx_align_launch(SxAlignArgs& A, int out_capacity, const SxScanState& st, cudaStream_t stream)
{
    const long long nwords = (A.nbits + 31) / 32;
    const int block = 256;
    int grid = (int)((nwords + block - 1) / block);
    if (grid < 1) grid = 1;
    if (grid > 4096) grid = 4096;
    sx_align_clear_kernel<<<grid, block, 0, stream>>>(A.bitmap, nwords);
    int maxc = 1;
    for (int l = 0; l < A.k; ++l) maxc = A.list[l].count > maxc ? A.list[l].count : maxc;
    int gx = (maxc + block - 1) / block;
    if (gx > 4096) gx = 4096;
    sx_align_mark_kernel<<<dim3(gx, A.k), block, 0, stream>>>(A);
    sx_align_popc_kernel<<<grid, block, 0, stream>>>(A.bitmap, nwords, A.wcount);
    cudaError_t err = sx_scan_i32_launch(A.wcount, nwords, A.wprefix, A.result, st, stream);
    if (err != cudaSuccess) return err;
    sx_align_compact_kernel<<<grid, block, 0, stream>>>(A, nwords);
    int gy = (out_capacity + 1 + block - 1) / block;
    if (gy > 4096) gy = 4096;
    if (gy < 1) gy = 1;
    sx_align_offsets_kernel<<<dim3(gy, A.k), block, 0, stream>>>(A);
    return cudaGetLastError();
}

// Largest number of leaf boundaries (2 x intervals, all leaves together) in
// a tile of `tra` aligned rows (out[0]) and of `trb` aligned rows (out[1]),
// and the largest coordinate span of a `tra`-row tile (out[2]: the last end
// of its rows minus their first begin; rows are assumed canonical, anything
// else only overstates it).  out must start at zero.
struct SxOffList {
    const int* off[SX_MAX_LEAVES];
    const int* begin[SX_MAX_LEAVES];
    const int* end[SX_MAX_LEAVES];
};

__global__ void sx_tile_max_kernel(SxOffList L, int k, int rows, int tra, int trb, int* out)
{
    const int tiles_a = (rows + tra - 1) / tra, tiles_b = (rows + trb - 1) / trb;
    int ma = 0, mb = 0, span = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles_a || t < tiles_b; t += gridDim.x * blockDim.x) {
        if (t < tiles_a) {
            const int r0 = t * tra, r1 = min(rows, r0 + tra);
            int c = 0;
            long long lo = LLONG_MAX, hi = LLONG_MIN;
            for (int l = 0; l < k; ++l) {
                c += L.off[l][r1] - L.off[l][r0];
                if (!L.begin[l] || !L.end[l]) continue;  // a leaf without intervals has no arrays
                for (int r = r0; r < r1; ++r) {
                    const int a = L.off[l][r], b = L.off[l][r + 1];
                    if (b > a) {
                        lo = min(lo, (long long)min(L.begin[l][a], L.end[l][a]));
                        hi = max(hi, (long long)max(L.end[l][b - 1], L.begin[l][b - 1]));
                    }
                }
            }
            ma = max(ma, c);
            if (hi >= lo) span = (int)min((long long)INT_MAX, max((long long)span, hi - lo));
        }
        if (t < tiles_b) {
            const int r0 = t * trb, r1 = min(rows, r0 + trb);
            int c = 0;
            for (int l = 0; l < k; ++l) c += L.off[l][r1] - L.off[l][r0];
            mb = max(mb, c);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ma = max(ma, __shfl_xor_sync(0xFFFFFFFFu, ma, o));
        mb = max(mb, __shfl_xor_sync(0xFFFFFFFFu, mb, o));
        span = max(span, __shfl_xor_sync(0xFFFFFFFFu, span, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (ma > 0) atomicMax(&out[0], 2 * ma);
        if (mb > 0) atomicMax(&out[1], 2 * mb);
        if (span > 0) atomicMax(&out[2], span);
    }
}

// The same for tile heights that are powers of two up to 32: one thread per
// row, tiles reduced over groups of lanes, one atomic per block.
__global__ void sx_tile_max_rows_kernel(SxOffList L, int k, int rows, int tra, int trb, int* out)
{
    __shared__ int s_max[3];
    if (threadIdx.x < 3) s_max[threadIdx.x] = 0;
    __syncthreads();
    int ma = 0, mb = 0, span = 0;
    const int stride = gridDim.x * blockDim.x;
    const int rows_up = (rows + 31) & ~31;  // whole warps, so the shuffles see full groups
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows_up; r += stride) {
        int c = 0;
        long long lo = LLONG_MAX, hi = LLONG_MIN;
        if (r < rows) {
            for (int l = 0; l < k; ++l) {
                const int a = L.off[l][r], b = L.off[l][r + 1];
                c += b - a;
                if (b > a && L.begin[l] && L.end[l]) {
                    lo = min(lo, (long long)min(L.begin[l][a], L.end[l][a]));
                    hi = max(hi, (long long)max(L.end[l][b - 1], L.begin[l][b - 1]));
                }
            }
        }
        int ca = c, cb = c;
        for (int o = 1; o < tra; o <<= 1) {
            ca += __shfl_xor_sync(0xFFFFFFFFu, ca, o);
            lo = min(lo, (long long)__shfl_xor_sync(0xFFFFFFFFu, lo, o));
            hi = max(hi, (long long)__shfl_xor_sync(0xFFFFFFFFu, hi, o));
        }
        for (int o = 1; o < trb; o <<= 1) cb += __shfl_xor_sync(0xFFFFFFFFu, cb, o);
        ma = max(ma, ca);
        mb = max(mb, cb);
        if (hi >= lo) span = (int)min((long long)INT_MAX, max((long long)span, hi - lo));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ma = max(ma, __shfl_xor_sync(0xFFFFFFFFu, ma, o));
        mb = max(mb, __shfl_xor_sync(0xFFFFFFFFu, mb, o));
        span = max(span, __shfl_xor_sync(0xFFFFFFFFu, span, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&s_max[0], ma);
        atomicMax(&s_max[1], mb);
        atomicMax(&s_max[2], span);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_max[0] > 0) atomicMax(&out[0], 2 * s_max[0]);
        if (s_max[1] > 0) atomicMax(&out[1], 2 * s_max[1]);
        if (s_max[2] > 0) atomicMax(&out[2], s_max[2]);
    }
}

cudaError_t sx_tile_max_launch(const int* const* offsets, const int* const* begins, const int* const* ends, int k,
                               int rows, int tra, int trb, int* out, cudaStream_t stream)
{
    SxOffList L;
    for (int l = 0; l < SX_MAX_LEAVES; ++l) {
        L.off[l] = l < k ? offsets[l] : nullptr;
        L.begin[l] = l < k ? begins[l] : nullptr;
        L.end[l] = l < k ? ends[l] : nullptr;
    }
    cudaError_t err = cudaMemsetAsync(out, 0, 3 * sizeof(int), stream);
    if (err != cudaSuccess) return err;
    const bool pow2 = tra <= 32 && trb <= 32 && (tra & (tra - 1)) == 0 && (trb & (trb - 1)) == 0;
    if (pow2) {
        int grid = (rows + 255) / 256;
        if (grid > 2368) grid = 2368;
        if (grid < 1) grid = 1;
        sx_tile_max_rows_kernel<<<grid, 256, 0, stream>>>(L, k, rows, tra, trb, out);
        return cudaGetLastError();
    }
    const int tiles = (rows + min(tra, trb) - 1) / min(tra, trb);
    int grid = (tiles + 255) / 256;
    if (grid > 1184) grid = 1184;
    if (grid < 1) grid = 1;
    sx_tile_max_kernel<<<grid, 256, 0, stream>>>(L, k, rows, tra, trb, out);
    return cudaGetLastError();
}
