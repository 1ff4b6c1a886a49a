// Quad assembly for VTK export of interval fields: every active cell
// becomes four corner points (x, y, 0) in float32 and one float32 value,
// written in cell order, so one device-to-host copy brings a whole chunk
// back (the host side only adds the trivial connectivity arrays).  The
// corners follow the reference's float32 arithmetic
// (subsetix_cupy/export_vtk.py:205-268): x_left = x0 + col * dx,
// x_right = x_left + dx, y_bottom = y0 + row * dy, y_top = y_bottom + dy,
// each operation rounded once.

#include "sx_internal.cuh"

namespace {

__device__ __forceinline__ int quad_row_of(const int* __restrict__ off, int rows, int i)
{
    int lo = 0, hi = rows - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename T>
__global__ void cell_quads_kernel(const int* __restrict__ off, const int* __restrict__ rows, int row_count,
                                  const int* __restrict__ b, const int* __restrict__ e, const int* __restrict__ coff,
                                  int n, const T* __restrict__ v, float dx, float dy, float ox, float oy,
                                  float* __restrict__ pts, float* __restrict__ vals)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const int row = rows[quad_row_of(off, row_count, (int)i)];
        const int x0 = b[i], len = e[i] - x0;
        const long long c0 = coff[i];
        const float yb = __fadd_rn(oy, __fmul_rn((float)row, dy));
        const float yt = __fadd_rn(yb, dy);
        for (int k = lane; k < len; k += 32) {
            const long long c = c0 + k;
            const float xl = __fadd_rn(ox, __fmul_rn((float)(x0 + k), dx));
            const float xr = __fadd_rn(xl, dx);
            float* p = pts + 12 * c;
            p[0] = xl; p[1] = yb; p[2] = 0.0f;
            p[3] = xr; p[4] = yb; p[5] = 0.0f;
            p[6] = xr; p[7] = yt; p[8] = 0.0f;
            p[9] = xl; p[10] = yt; p[11] = 0.0f;
            vals[c] = (float)v[c];
        }
    }
}

}  // namespace

cudaError_t sx_cell_quads_launch(int dtype, const int* off, const int* rows, int row_count, const int* b, const int* e,
                                 const int* coff, int n, const void* v, float dx, float dy, float ox, float oy,
                                 float* pts, float* vals, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    long long blocks = ((long long)n + 7) / 8;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (dtype == 1)
        cell_quads_kernel<double><<<(int)blocks, 256, 0, stream>>>(off, rows, row_count, b, e, coff, n,
                                                                   (const double*)v, dx, dy, ox, oy, pts, vals);
    else
        cell_quads_kernel<float><<<(int)blocks, 256, 0, stream>>>(off, rows, row_count, b, e, coff, n,
                                                                  (const float*)v, dx, dy, ox, oy, pts, vals);
    return cudaGetLastError();
}
