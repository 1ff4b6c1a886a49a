// Two-level AMR step on full grids, batched over independent simulations.
//
// In the reference's AMR2Simulation both levels are full rectangles: the
// coarse field covers [0, W) x [0, H) and the fine field [0, rW) x [0, rH),
// one interval per row (subsetix_amr2/simulation.py:159-213).  On such sets
// the interval kernels reduce to dense ones, and this file runs them
// directly on [batch][rows][cols] arrays:
//
//   sx_upwind_full     the upwind update of interval_stencil.py:59-113 with
//                      zero exterior (cells outside the grid read 0);
//   sx_amr_sync_full   synchronize_interval_fields with the mean reducer and
//                      copy=False (fields.py:570-612): a coarse cell marked
//                      REFINE takes the mean of its r x r fine block, summed
//                      sub-row outer, column inner, times 1/r^2
//                      (kernels.py:458-527); any other coarse cell is copied
//                      into its fine block (kernels.py:384-418).  Refine and
//                      coarse-only cells partition the grid, so one pass per
//                      coarse cell does both halves;
//   sx_amr_tag_full    the gradient tag of regrid.py:172-223,336-350: the
//                      field is read as float32, the gradient has central
//                      differences inside and one-sided ones at the edges,
//                      and a cell is tagged when sqrt(gx^2 + gy^2) >=
//                      threshold;
//   sx_amr_grade_full  enforce_two_level_grading_set (regrid.py:404-442) as
//                      a cell set: a coarse cell is refined when a tagged
//                      cell lies within `padding` along a row or a column
//                      (von Neumann) or within the (2p+1)^2 box (Moore),
//                      clipped to the grid.  The action byte is REFINE (1)
//                      or KEEP (0), as ActionField.set_from_interval_set
//                      writes it (fields.py:520-546).
//
// Float formulas use explicit rounding intrinsics, including the float32
// fusions the reference's NVRTC build makes (sx_upwind_update and
// sx_grad_norm), so results are bit-identical to the interval kernels (and
// to the reference) on the same inputs, in float32 and in float64.

#include <cmath>

#include "sx_internal.cuh"

__device__ __forceinline__ float sxa_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sxa_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float sxa_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float sxa_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double sxa_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sxa_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double sxa_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sxa_div(double a, double b) { return __ddiv_rn(a, b); }

// x / d, or x * d when the launcher passed the reciprocal of a power-of-two
// spacing instead (pow2 != 0).  Dividing by 2^k and multiplying by 2^-k
// have the same exact real result, so the rounded results are identical.
template <typename T>
__device__ __forceinline__ T sxa_over(T x, T d, int pow2)
{
    return pow2 ? sxa_mul(x, d) : sxa_div(x, d);
}

// One thread per cell; x fastest.  blockIdx.z is the batch entry.
// The upwind update of one cell from the neighbours the velocity selects:
// SGN bit 0 (a >= 0) the left one in h, else the right one; bit 1 (b >= 0)
// the one below in v, else the one above.  The reference's formula uses one
// side per axis, so the other side is never read.
template <typename T, int SGN>
__device__ __forceinline__ T sxa_upwind_side(T c, T h, T v, T a, T b, T dt, T dx, T dy, int pow2)
{
    const T du_dx = (SGN & 1) ? sxa_over(sxa_sub(c, h), dx, pow2) : sxa_over(sxa_sub(h, c), dx, pow2);
    const T du_dy = (SGN & 2) ? sxa_over(sxa_sub(c, v), dy, pow2) : sxa_over(sxa_sub(v, c), dy, pow2);
    return sx_upwind_update(c, du_dx, du_dy, a, b, dt);
}

template <typename T, int SGN>
__global__ void __launch_bounds__(256) sx_upwind_full_kernel(const T* __restrict__ in, T* __restrict__ out, int W,
                                                             int H, T a, T b, T dt, T dx, T dy, int pow2)
{
    const long long plane = (long long)W * H;
    const T* v = in + plane * blockIdx.z;
    T* o = out + plane * blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const long long idx = (long long)y * W + x;
    const T c = v[idx];
    const T h = (SGN & 1) ? (x > 0 ? v[idx - 1] : (T)0) : (x + 1 < W ? v[idx + 1] : (T)0);
    const T w = (SGN & 2) ? (y > 0 ? v[idx - W] : (T)0) : (y + 1 < H ? v[idx + W] : (T)0);
    o[idx] = sxa_upwind_side<T, SGN>(c, h, w, a, b, dt, dx, dy, pow2);
}

// One thread per coarse cell.  R is the refinement ratio (template for the
// common 2, runtime otherwise).
template <typename T, int RT>
__global__ void __launch_bounds__(256) sx_amr_sync_full_kernel(T* __restrict__ coarse, T* __restrict__ fine,
                                                               const signed char* __restrict__ actions, int W, int H,
                                                               int rr, T norm)
{
    const int R = RT > 0 ? RT : rr;
    const int b = blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const long long plane = (long long)W * H;
    const long long ci = plane * b + (long long)y * W + x;
    const int FW = W * R;
    T* f = fine + plane * R * R * b + ((long long)y * R) * FW + (long long)x * R;
    if (actions[ci] == 1) {
        T acc = (T)0;
        for (int dy = 0; dy < R; ++dy)
            for (int dx = 0; dx < R; ++dx) acc = sxa_add(acc, f[(long long)dy * FW + dx]);
        coarse[ci] = sxa_mul(acc, norm);
    } else {
        const T c = coarse[ci];
        for (int dy = 0; dy < R; ++dy)
            for (int dx = 0; dx < R; ++dx) f[(long long)dy * FW + dx] = c;
    }
}

// Whole fixed-geometry step for ratio 2: upwind of the coarse cell and of
// its 2 x 2 fine block (from the previous values, zero exterior), then the
// synchronisation of that coarse cell with its block.  A step's
// synchronisation of a coarse cell reads only that cell's and that block's
// new values, so this equals upwind(coarse); upwind(fine); sync, value for
// value.  in/out are distinct buffers.  SGN: the velocity's upwind sides, as
// in sxa_upwind_side.
template <typename T, int SGN>
__global__ void __launch_bounds__(256) sx_amr_step_full_kernel(const T* __restrict__ cin, const T* __restrict__ fin,
                                                               T* __restrict__ cout, T* __restrict__ fout,
                                                               const signed char* __restrict__ actions, int W, int H,
                                                               T a, T b, T dt, T dxc, T dyc, T dxf, T dyf, T norm,
                                                               int pow2c, int pow2f)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const long long plane = (long long)W * H;
    const int FW = 2 * W, FH = 2 * H;
    const T* C = cin + plane * blockIdx.z;
    const T* F = fin + 4 * plane * blockIdx.z;
    const long long ci = (long long)y * W + x;
    // coarse cell, with the neighbours the velocity selects
    const T c = C[ci];
    const T ch = (SGN & 1) ? (x > 0 ? C[ci - 1] : (T)0) : (x + 1 < W ? C[ci + 1] : (T)0);
    const T cv = (SGN & 2) ? (y > 0 ? C[ci - W] : (T)0) : (y + 1 < H ? C[ci + W] : (T)0);
    const T cn = sxa_upwind_side<T, SGN>(c, ch, cv, a, b, dt, dxc, dyc, pow2c);
    const int fx = 2 * x, fy = 2 * y;
    T* CO = cout + plane * blockIdx.z;
    T* FO = fout + 4 * plane * blockIdx.z;
    if (actions[plane * blockIdx.z + ci] != 1) {
        // not refined: the synchronisation overwrites the fine block with the
        // new coarse value, so its own upwind update is never needed
        CO[ci] = cn;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            T* row = FO + (long long)(fy + j) * FW + fx;
            row[0] = cn;
            row[1] = cn;
        }
        return;
    }
    // refined: fine block, rows 2y-1 .. 2y+2, columns 2x-1 .. 2x+2; only the
    // 2 x 2 block and the column and row on its upwind sides are read
    T v[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int yy = fy - 1 + j;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int xx = fx - 1 + i;
            const bool inner_row = j == 1 || j == 2, inner_col = i == 1 || i == 2;
            const bool needed = (inner_row && inner_col) ||
                                (inner_row && (((SGN & 1) && i == 0) || (!(SGN & 1) && i == 3))) ||
                                (inner_col && (((SGN & 2) && j == 0) || (!(SGN & 2) && j == 3)));
            v[j][i] = (needed && yy >= 0 && yy < FH && xx >= 0 && xx < FW) ? F[(long long)yy * FW + xx] : (T)0;
        }
    }
    T fn[2][2];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i)
            fn[j][i] = sxa_upwind_side<T, SGN>(v[j + 1][i + 1], (SGN & 1) ? v[j + 1][i] : v[j + 1][i + 2],
                                               (SGN & 2) ? v[j][i + 1] : v[j + 2][i + 1], a, b, dt, dxf, dyf, pow2f);
    T acc = sxa_add(sxa_add(sxa_add(sxa_add((T)0, fn[0][0]), fn[0][1]), fn[1][0]), fn[1][1]);
    CO[ci] = sxa_mul(acc, norm);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        T* row = FO + (long long)(fy + j) * FW + fx;
        row[0] = fn[j][0];
        row[1] = fn[j][1];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) sx_amr_tag_full_kernel(const T* __restrict__ in, unsigned char* __restrict__ tags,
                                                              int W, int H, float thr)
{
    const long long plane = (long long)W * H;
    const T* v = in + plane * blockIdx.z;
    unsigned char* t = tags + plane * blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const long long idx = (long long)y * W + x;
    const float c = (float)v[idx];
    float gx = 0.0f, gy = 0.0f;
    if (W > 1) {
        if (x == 0) gx = __fsub_rn((float)v[idx + 1], c);
        else if (x == W - 1) gx = __fsub_rn(c, (float)v[idx - 1]);
        else gx = __fmul_rn(__fsub_rn((float)v[idx + 1], (float)v[idx - 1]), 0.5f);
    }
    if (H > 1) {
        if (y == 0) gy = __fsub_rn((float)v[idx + W], c);
        else if (y == H - 1) gy = __fsub_rn(c, (float)v[idx - W]);
        else gy = __fmul_rn(__fsub_rn((float)v[idx + W], (float)v[idx - W]), 0.5f);
    }
    t[idx] = sx_grad_norm(gx, gy) >= thr ? 1 : 0;
}

// mode 0: von Neumann (row or column within p), 1: Moore (box), 2: no grading
__global__ void __launch_bounds__(256) sx_amr_grade_full_kernel(const unsigned char* __restrict__ tags,
                                                               signed char* __restrict__ actions, int W, int H, int p,
                                                               int mode)
{
    const long long plane = (long long)W * H;
    const unsigned char* t = tags + plane * blockIdx.z;
    signed char* a = actions + plane * blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    bool on = t[(long long)y * W + x] != 0;
    if (!on && mode != 2) {
        const int x0 = max(0, x - p), x1 = min(W - 1, x + p);
        const int y0 = max(0, y - p), y1 = min(H - 1, y + p);
        if (mode == 1) {
            for (int yy = y0; yy <= y1 && !on; ++yy)
                for (int xx = x0; xx <= x1; ++xx)
                    if (t[(long long)yy * W + xx]) {
                        on = true;
                        break;
                    }
        } else {
            for (int xx = x0; xx <= x1 && !on; ++xx) on = t[(long long)y * W + xx] != 0;
            for (int yy = y0; yy <= y1 && !on; ++yy) on = t[(long long)yy * W + x] != 0;
        }
    }
    a[(long long)y * W + x] = on ? 1 : 0;
}

static dim3 sxa_grid(int W, int H, int batch) { return dim3((unsigned)((W + 255) / 256), (unsigned)H, (unsigned)batch); }

// Spacings that are powers of two (in the kernel's precision) are passed
// as their exact reciprocals, turning divisions into multiplications.
template <typename T>
static int sxa_pow2_pair(T& dx, T& dy)
{
    int ex, ey;
    const bool p = frexp((double)dx, &ex) == 0.5 && frexp((double)dy, &ey) == 0.5;
    if (!p) return 0;
    const T ix = (T)1 / dx, iy = (T)1 / dy;
    if (!std::isfinite((double)ix) || !std::isfinite((double)iy)) return 0;  // reciprocal out of range
    dx = ix;
    dy = iy;
    return 1;
}

// Kernel instances by the velocity's upwind sides, tested in the kernel's precision.
template <typename T>
static void sxa_upwind_full_go(dim3 g, const T* in, T* out, int W, int H, T a, T b, T dt, T dx, T dy, int p,
                               cudaStream_t stream)
{
    switch ((a >= (T)0 ? 1 : 0) | (b >= (T)0 ? 2 : 0)) {
        case 0: sx_upwind_full_kernel<T, 0><<<g, 256, 0, stream>>>(in, out, W, H, a, b, dt, dx, dy, p); break;
        case 1: sx_upwind_full_kernel<T, 1><<<g, 256, 0, stream>>>(in, out, W, H, a, b, dt, dx, dy, p); break;
        case 2: sx_upwind_full_kernel<T, 2><<<g, 256, 0, stream>>>(in, out, W, H, a, b, dt, dx, dy, p); break;
        default: sx_upwind_full_kernel<T, 3><<<g, 256, 0, stream>>>(in, out, W, H, a, b, dt, dx, dy, p); break;
    }
}

template <typename T>
static void sxa_step_full_go(dim3 g, const T* cin, const T* fin, T* cout, T* fout, const signed char* actions, int W,
                             int H, T a, T b, T dt, T cx, T cy, T fx, T fy, T norm, int pc, int pf,
                             cudaStream_t stream)
{
    switch ((a >= (T)0 ? 1 : 0) | (b >= (T)0 ? 2 : 0)) {
        case 0:
            sx_amr_step_full_kernel<T, 0><<<g, 256, 0, stream>>>(cin, fin, cout, fout, actions, W, H, a, b, dt, cx, cy,
                                                                 fx, fy, norm, pc, pf);
            break;
        case 1:
            sx_amr_step_full_kernel<T, 1><<<g, 256, 0, stream>>>(cin, fin, cout, fout, actions, W, H, a, b, dt, cx, cy,
                                                                 fx, fy, norm, pc, pf);
            break;
        case 2:
            sx_amr_step_full_kernel<T, 2><<<g, 256, 0, stream>>>(cin, fin, cout, fout, actions, W, H, a, b, dt, cx, cy,
                                                                 fx, fy, norm, pc, pf);
            break;
        default:
            sx_amr_step_full_kernel<T, 3><<<g, 256, 0, stream>>>(cin, fin, cout, fout, actions, W, H, a, b, dt, cx, cy,
                                                                 fx, fy, norm, pc, pf);
            break;
    }
}

cudaError_t sx_upwind_full_launch(int dbl, const void* in, void* out, int W, int H, int batch, double a, double b,
                                  double dt, double dx, double dy, cudaStream_t stream)
{
    const dim3 g = sxa_grid(W, H, batch);
    if (dbl) {
        double ddx = dx, ddy = dy;
        const int p = sxa_pow2_pair(ddx, ddy);
        sxa_upwind_full_go<double>(g, (const double*)in, (double*)out, W, H, a, b, dt, ddx, ddy, p, stream);
    } else {
        float fdx = (float)dx, fdy = (float)dy;
        const int p = sxa_pow2_pair(fdx, fdy);
        sxa_upwind_full_go<float>(g, (const float*)in, (float*)out, W, H, (float)a, (float)b, (float)dt, fdx, fdy, p,
                                  stream);
    }
    return cudaGetLastError();
}

cudaError_t sx_amr_sync_full_launch(int dbl, void* coarse, void* fine, const signed char* actions, int W, int H,
                                    int batch, int ratio, cudaStream_t stream)
{
    const dim3 g = sxa_grid(W, H, batch);
    const double norm = 1.0 / ((double)ratio * ratio);
    if (dbl) {
        if (ratio == 2)
            sx_amr_sync_full_kernel<double, 2><<<g, 256, 0, stream>>>((double*)coarse, (double*)fine, actions, W, H, 2,
                                                                      norm);
        else
            sx_amr_sync_full_kernel<double, 0><<<g, 256, 0, stream>>>((double*)coarse, (double*)fine, actions, W, H,
                                                                      ratio, norm);
    } else {
        if (ratio == 2)
            sx_amr_sync_full_kernel<float, 2><<<g, 256, 0, stream>>>((float*)coarse, (float*)fine, actions, W, H, 2,
                                                                     (float)norm);
        else
            sx_amr_sync_full_kernel<float, 0><<<g, 256, 0, stream>>>((float*)coarse, (float*)fine, actions, W, H, ratio,
                                                                     (float)norm);
    }
    return cudaGetLastError();
}

cudaError_t sx_amr_regrid_full_launch(int dbl, const void* coarse, unsigned char* tags, signed char* actions, int W,
                                      int H, int batch, float threshold, int padding, int mode, cudaStream_t stream)
{
    const dim3 g = sxa_grid(W, H, batch);
    if (dbl)
        sx_amr_tag_full_kernel<double><<<g, 256, 0, stream>>>((const double*)coarse, tags, W, H, threshold);
    else
        sx_amr_tag_full_kernel<float><<<g, 256, 0, stream>>>((const float*)coarse, tags, W, H, threshold);
    sx_amr_grade_full_kernel<<<g, 256, 0, stream>>>(tags, actions, W, H, padding, padding <= 0 ? 2 : mode);
    return cudaGetLastError();
}

cudaError_t sx_amr_step_full_launch(int dbl, const void* cin, const void* fin, void* cout, void* fout,
                                    const signed char* actions, int W, int H, int batch, double a, double b, double dt,
                                    double dxc, double dyc, double dxf, double dyf, cudaStream_t stream)
{
    const dim3 g = sxa_grid(W, H, batch);
    if (dbl) {
        double cx = dxc, cy = dyc, fx = dxf, fy = dyf;
        const int pc = sxa_pow2_pair(cx, cy), pf = sxa_pow2_pair(fx, fy);
        sxa_step_full_go<double>(g, (const double*)cin, (const double*)fin, (double*)cout, (double*)fout, actions, W,
                                 H, a, b, dt, cx, cy, fx, fy, 0.25, pc, pf, stream);
    } else {
        float cx = (float)dxc, cy = (float)dyc, fx = (float)dxf, fy = (float)dyf;
        const int pc = sxa_pow2_pair(cx, cy), pf = sxa_pow2_pair(fx, fy);
        sxa_step_full_go<float>(g, (const float*)cin, (const float*)fin, (float*)cout, (float*)fout, actions, W, H,
                                (float)a, (float)b, (float)dt, cx, cy, fx, fy, 0.25f, pc, pf, stream);
    }
    return cudaGetLastError();
}
