// Level coupling of a nested multi-level field by index tables: ghost
// filling from the coarser level, restriction onto it, and the transposes of
// both.  The tables are built once per fixed geometry on the host side
// (subsetix_b200/adjoint.py), so every kernel here is a gather or a
// scatter over precomputed indices, bound by HBM bandwidth:
//
//   sx_index_copy            dst[dst_idx[i]] = src[src_idx[i]]
//                            (ghost fill: a fine ghost cell takes its coarse
//                            parent's value, as injection does in
//                            subsetix_cupy/multilevel.py:365-407);
//   sx_index_block_mean      out[out_idx[j]] = (sum_m in[in_idx[j*g+m]]) * norm
//                            summed in table order (sub-row outer, column
//                            inner), then scaled: the order of
//                            restrict_field's mean (multilevel.py:410-479);
//   sx_index_block_mean_adj  its transpose: in_bar[in_idx[j*g+m]] +=
//                            out_bar[out_idx[j]] * norm, out_bar[out_idx[j]] = 0
//                            (the in_idx entries are distinct, so no two
//                            threads write one cell);
//   sx_index_segment_add     transpose of a gather with repeats: dst[dst_idx[s]]
//                            += sum of src[src_idx[t]] over segment s, in
//                            segment order, then src[src_idx[t]] = 0 when asked
//                            (deterministic: one thread per segment).
//
// Float arithmetic uses explicit round-to-nearest operations, so float32
// and float64 results do not depend on the compiler's contraction choices.

#include "sx_internal.cuh"

namespace {

__device__ __forceinline__ float cp_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double cp_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float cp_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double cp_mul(double a, double b) { return __dmul_rn(a, b); }

template <typename T>
__global__ void index_copy_kernel(long long n, const int* __restrict__ dst_idx, const int* __restrict__ src_idx,
                                  const T* __restrict__ src, T* __restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long s = src_idx ? src_idx[i] : i;
        const long long d = dst_idx ? dst_idx[i] : i;
        dst[d] = src[s];
    }
}

template <typename T>
__global__ void block_mean_kernel(long long n, int group, T norm, const int* __restrict__ out_idx,
                                  const int* __restrict__ in_idx, const T* __restrict__ in, T* __restrict__ out)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const int* idx = in_idx + j * group;
        T acc = T(0);
        for (int m = 0; m < group; ++m) acc = cp_add(acc, in[idx[m]]);
        out[out_idx[j]] = cp_mul(acc, norm);
    }
}

template <typename T>
__global__ void block_mean_adj_kernel(long long n, int group, T norm, const int* __restrict__ out_idx,
                                      const int* __restrict__ in_idx, T* __restrict__ out_bar, T* __restrict__ in_bar)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const int* idx = in_idx + j * group;
        const T w = cp_mul(out_bar[out_idx[j]], norm);
        for (int m = 0; m < group; ++m) in_bar[idx[m]] = cp_add(in_bar[idx[m]], w);
        out_bar[out_idx[j]] = T(0);
    }
}

template <typename T>
__global__ void segment_add_kernel(long long nseg, const int* __restrict__ seg_off, const int* __restrict__ src_idx,
                                   const int* __restrict__ dst_idx, T* __restrict__ src, T* __restrict__ dst,
                                   int zero_src)
{
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nseg;
         s += (long long)gridDim.x * blockDim.x) {
        T acc = dst[dst_idx[s]];
        for (int t = seg_off[s]; t < seg_off[s + 1]; ++t) {
            acc = cp_add(acc, src[src_idx[t]]);
            if (zero_src) src[src_idx[t]] = T(0);
        }
        dst[dst_idx[s]] = acc;
    }
}

int grid_for(long long n)
{
    long long g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t sx_index_copy_launch(int dtype, long long n, const int* dst_idx, const int* src_idx, const void* src,
                                 void* dst, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    if (dtype == 1)
        index_copy_kernel<double><<<grid_for(n), 256, 0, stream>>>(n, dst_idx, src_idx, (const double*)src,
                                                                    (double*)dst);
    else
        index_copy_kernel<float><<<grid_for(n), 256, 0, stream>>>(n, dst_idx, src_idx, (const float*)src, (float*)dst);
    return cudaGetLastError();
}

cudaError_t sx_index_block_mean_launch(int dtype, long long n, int group, double norm, const int* out_idx,
                                       const int* in_idx, const void* in, void* out, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    if (dtype == 1)
        block_mean_kernel<double><<<grid_for(n), 256, 0, stream>>>(n, group, norm, out_idx, in_idx, (const double*)in,
                                                                    (double*)out);
    else
        block_mean_kernel<float><<<grid_for(n), 256, 0, stream>>>(n, group, (float)norm, out_idx, in_idx,
                                                                   (const float*)in, (float*)out);
    return cudaGetLastError();
}

cudaError_t sx_index_block_mean_adj_launch(int dtype, long long n, int group, double norm, const int* out_idx,
                                           const int* in_idx, void* out_bar, void* in_bar, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    if (dtype == 1)
        block_mean_adj_kernel<double><<<grid_for(n), 256, 0, stream>>>(n, group, norm, out_idx, in_idx,
                                                                        (double*)out_bar, (double*)in_bar);
    else
        block_mean_adj_kernel<float><<<grid_for(n), 256, 0, stream>>>(n, group, (float)norm, out_idx, in_idx,
                                                                       (float*)out_bar, (float*)in_bar);
    return cudaGetLastError();
}

cudaError_t sx_index_segment_add_launch(int dtype, long long nseg, const int* seg_off, const int* src_idx,
                                        const int* dst_idx, void* src, void* dst, int zero_src, cudaStream_t stream)
{
    if (nseg <= 0) return cudaSuccess;
    if (dtype == 1)
        segment_add_kernel<double><<<grid_for(nseg), 256, 0, stream>>>(nseg, seg_off, src_idx, dst_idx, (double*)src,
                                                                        (double*)dst, zero_src);
    else
        segment_add_kernel<float><<<grid_for(nseg), 256, 0, stream>>>(nseg, seg_off, src_idx, dst_idx, (float*)src,
                                                                       (float*)dst, zero_src);
    return cudaGetLastError();
}
