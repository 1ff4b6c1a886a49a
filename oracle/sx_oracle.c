/*
 * CPU restatement of the reference's per-row interval algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle.  Only tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py load it,
 * and they use it as the checker.  The product path in subsetix_b200/ never
 * calls it.
 *
 * Each function restates the sequential algorithm of one reference kernel,
 * row by row (or interval by interval), with OpenMP across rows.  The file
 * and line of the restated reference code are given with each function.
 * Float code is built with -ffp-contract=off.  The reference's formulas are
 * therefore evaluated in source order with no fused multiply-add.
 */

#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_UNION 0
#define ORC_INTERSECTION 1
#define ORC_DIFFERENCE 2

/* One row pair of a binary set operation.  When out_b is NULL, only the
 * output count is returned.  Restates the three sweeps of
 * subsetix_cupy/kernels.py:36-113 (count) and :147-233 (write):
 *   union: merge by begin, ties to lhs; extend while begin <= active end;
 *   intersection: emit [max b, min e) when non-empty; advance lhs when
 *                 a_end <= b_end;
 *   difference: per lhs interval, a cursor sweep over rhs that carries the
 *               rhs index across lhs intervals. */
static int64_t orc_row_op(int op,
                          const int32_t* lb, const int32_t* le, int64_t li, int64_t ln,
                          const int32_t* rb, const int32_t* re, int64_t rj, int64_t rn,
                          int32_t* out_b, int32_t* out_e)
{
    int64_t n = 0;
    if (op == ORC_UNION) {
        int have = 0;
        int32_t cur_b = 0, cur_e = 0;
        while (li < ln || rj < rn) {
            int from_left = (rj >= rn) || (li < ln && lb[li] <= rb[rj]);
            int32_t sb = from_left ? lb[li] : rb[rj];
            int32_t se = from_left ? le[li] : re[rj];
            if (from_left) ++li; else ++rj;
            if (!have) {
                have = 1; cur_b = sb; cur_e = se;
            } else if (sb <= cur_e) {
                if (se > cur_e) cur_e = se;
            } else {
                if (out_b) { out_b[n] = cur_b; out_e[n] = cur_e; }
                ++n;
                cur_b = sb; cur_e = se;
            }
        }
        if (have) {
            if (out_b) { out_b[n] = cur_b; out_e[n] = cur_e; }
            ++n;
        }
    } else if (op == ORC_INTERSECTION) {
        while (li < ln && rj < rn) {
            int32_t lo = lb[li] > rb[rj] ? lb[li] : rb[rj];
            int32_t hi = le[li] < re[rj] ? le[li] : re[rj];
            if (lo < hi) {
                if (out_b) { out_b[n] = lo; out_e[n] = hi; }
                ++n;
            }
            if (le[li] <= re[rj]) ++li; else ++rj;
        }
    } else {
        for (; li < ln; ++li) {
            int32_t a_end = le[li];
            int32_t cur = lb[li];
            while (cur < a_end) {
                while (rj < rn && re[rj] <= cur) ++rj;
                if (rj >= rn || rb[rj] >= a_end) {
                    if (out_b) { out_b[n] = cur; out_e[n] = a_end; }
                    ++n;
                    break;
                }
                if (rb[rj] > cur) {
                    int32_t stop = rb[rj] < a_end ? rb[rj] : a_end;
                    if (stop > cur) {
                        if (out_b) { out_b[n] = cur; out_e[n] = stop; }
                        ++n;
                    }
                }
                /* after the skip loop re[rj] > cur, so the cursor jumps */
                cur = re[rj];
            }
        }
    }
    return n;
}

/* Per-row counts of a binary op over aligned rows (kernels.py:11-117). */
void orc_setop_count(int op, int64_t rows,
                     const int32_t* lb, const int32_t* le, const int32_t* loff,
                     const int32_t* rb, const int32_t* re, const int32_t* roff,
                     int32_t* counts)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < rows; ++r) {
        counts[r] = (int32_t)orc_row_op(op, lb, le, loff[r], loff[r + 1], rb, re, roff[r], roff[r + 1], NULL, NULL);
    }
}

/* Writes a binary op's intervals at the given offsets (kernels.py:120-235). */
void orc_setop_write(int op, int64_t rows,
                     const int32_t* lb, const int32_t* le, const int32_t* loff,
                     const int32_t* rb, const int32_t* re, const int32_t* roff,
                     const int32_t* offsets, int32_t* ob, int32_t* oe)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < rows; ++r) {
        orc_row_op(op, lb, le, loff[r], loff[r + 1], rb, re, roff[r], roff[r + 1], ob + offsets[r], oe + offsets[r]);
    }
}

/* Merge of intervals sorted by begin inside each row, where an interval
 * whose begin is <= the running end extends the run
 * (subsetix_cupy/kernels.py:292-381).  When ob is NULL only counts are
 * produced. */
void orc_merge_rows(int64_t rows, const int32_t* b, const int32_t* e, const int32_t* off,
                    const int32_t* out_off, int32_t* counts, int32_t* ob, int32_t* oe)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < rows; ++r) {
        int64_t s = off[r], t = off[r + 1];
        int32_t n = 0;
        if (s < t) {
            int32_t cb = b[s], ce = e[s];
            int64_t w = ob ? out_off[r] : 0;
            for (int64_t i = s + 1; i < t; ++i) {
                if (b[i] <= ce) {
                    if (e[i] > ce) ce = e[i];
                } else {
                    if (ob) { ob[w] = cb; oe[w] = ce; ++w; }
                    ++n;
                    cb = b[i]; ce = e[i];
                }
            }
            if (ob) { ob[w] = cb; oe[w] = ce; }
            ++n;
        }
        if (counts) counts[r] = n;
    }
}

/* Piecewise-constant injection, one coarse interval at a time
 * (subsetix_cupy/kernels.py:384-455). */
#define ORC_PROLONG(NAME, T)                                                              \
void NAME(int64_t intervals, int ratio, const int32_t* coff, const int32_t* foff,        \
          const int32_t* fidx, const T* cv, T* fv)                                        \
{                                                                                         \
    _Pragma("omp parallel for schedule(dynamic, 64)")                                     \
    for (int64_t i = 0; i < intervals; ++i) {                                             \
        int32_t cb = coff[i];                                                             \
        if (coff[i + 1] - cb <= 0) continue;                                              \
        for (int d = 0; d < ratio; ++d) {                                                 \
            int32_t f = fidx[i * ratio + d];                                              \
            int32_t fb = foff[f], fw = foff[f + 1] - foff[f];                             \
            for (int32_t k = 0; k < fw; ++k) fv[fb + k] = cv[cb + k / ratio];             \
        }                                                                                 \
    }                                                                                     \
}
ORC_PROLONG(orc_prolong_field_f32, float)
ORC_PROLONG(orc_prolong_field_f64, double)

/* ratio x ratio block reduction with the sub-row loop outside, the column
 * loop inside, and an early stop at the fine interval's end.  mean = sum *
 * norm.  Restates subsetix_cupy/kernels.py:458-599. */
#define ORC_RESTRICT(NAME, T)                                                             \
void NAME(int64_t intervals, int ratio, int reducer, T norm, const int32_t* coff,        \
          const int32_t* foff, const int32_t* fidx, const T* fv, T* cv)                   \
{                                                                                         \
    _Pragma("omp parallel for schedule(dynamic, 64)")                                     \
    for (int64_t i = 0; i < intervals; ++i) {                                             \
        int32_t cb = coff[i], width = coff[i + 1] - coff[i];                              \
        if (width <= 0) continue;                                                         \
        for (int32_t k = 0; k < width; ++k) {                                             \
            T acc = (T)0, lo = (T)0, hi = (T)0;                                           \
            int have = 0;                                                                 \
            for (int dy = 0; dy < ratio; ++dy) {                                          \
                int32_t f = fidx[i * ratio + dy];                                         \
                int32_t fend = foff[f + 1];                                               \
                int32_t start = foff[f] + k * ratio;                                      \
                for (int dx = 0; dx < ratio; ++dx) {                                      \
                    int32_t idx = start + dx;                                             \
                    if (idx >= fend) break;                                               \
                    T v = fv[idx];                                                        \
                    if (reducer == 2) { if (!have || v < lo) lo = v; }                    \
                    else if (reducer == 3) { if (!have || v > hi) hi = v; }               \
                    else acc += v;                                                        \
                    have = 1;                                                             \
                }                                                                         \
            }                                                                             \
            cv[cb + k] = reducer == 0 ? acc * norm : reducer == 1 ? acc                    \
                       : reducer == 2 ? lo : hi;                                          \
        }                                                                                 \
    }                                                                                     \
}
ORC_RESTRICT(orc_restrict_field_f32, float)
ORC_RESTRICT(orc_restrict_field_f64, double)

/* Value of the cell (row, x), or zero when the cell lies outside the domain
 * or outside the set.  Uses a binary search inside the row
 * (subsetix_cupy/interval_stencil.py:17-57). */
#define ORC_SAMPLE(NAME, T)                                                               \
static T NAME(int row, int x, int height, int width, const int32_t* lookup,              \
              const int32_t* off, const int32_t* b, const int32_t* e,                     \
              const int32_t* coff, const T* v)                                            \
{                                                                                         \
    if (row < 0 || row >= height || x < 0 || x >= width) return (T)0;                     \
    int32_t ord = lookup[row];                                                            \
    if (ord < 0) return (T)0;                                                             \
    int32_t lo = off[ord], hi = off[ord + 1] - 1;                                         \
    while (lo <= hi) {                                                                    \
        int32_t mid = (lo + hi) >> 1;                                                     \
        if (x < b[mid]) hi = mid - 1;                                                     \
        else if (x >= e[mid]) lo = mid + 1;                                               \
        else return v[coff[mid] + (x - b[mid])];                                          \
    }                                                                                     \
    return (T)0;                                                                          \
}
ORC_SAMPLE(orc_sample_f32, float)
ORC_SAMPLE(orc_sample_f64, double)

/* First-order upwind update with zero exterior.  The upwind side is chosen
 * by the sign of each velocity component, and the differences are divided
 * by dx and dy (subsetix_cupy/interval_stencil.py:59-113). */
/* The update c - dt (a du_dx + b du_dy).  Float32 fuses it the way the
 * reference's NVRTC build does (two fmaf, inner first); float64, which has no
 * reference counterpart, rounds each operation once. */
static float orc_update_f32(float c, float ddx, float ddy, float a, float b, float dt)
{
    return fmaf(-dt, fmaf(a, ddx, b * ddy), c);
}
static double orc_update_f64(double c, double ddx, double ddy, double a, double b, double dt)
{
    double t1 = a * ddx;
    double t2 = b * ddy;
    double s = t1 + t2;
    double m = dt * s;
    return c - m;
}

#define ORC_UPWIND(NAME, SAMPLE, T, UPDATE)                                               \
void NAME(int64_t intervals, const int32_t* row_ids, const int32_t* b, const int32_t* e,  \
          const int32_t* off, const int32_t* coff, const int32_t* ordinals,               \
          const int32_t* lookup, const T* v, T* out, int width, int height,               \
          T a, T bb, T dt, T dx, T dy)                                                    \
{                                                                                         \
    _Pragma("omp parallel for schedule(dynamic, 64)")                                     \
    for (int64_t i = 0; i < intervals; ++i) {                                             \
        int row = row_ids[i];                                                             \
        if (ordinals[i] < 0) continue;                                                    \
        int32_t ib = b[i], ie = e[i];                                                     \
        if (ie <= ib) continue;                                                           \
        int32_t base = coff[i];                                                           \
        for (int32_t k = 0; k < ie - ib; ++k) {                                           \
            int x = ib + k;                                                               \
            T c = v[base + k];                                                            \
            T l = SAMPLE(row, x - 1, height, width, lookup, off, b, e, coff, v);          \
            T r = SAMPLE(row, x + 1, height, width, lookup, off, b, e, coff, v);          \
            T d = SAMPLE(row - 1, x, height, width, lookup, off, b, e, coff, v);          \
            T u = SAMPLE(row + 1, x, height, width, lookup, off, b, e, coff, v);          \
            T ddx = (a >= (T)0) ? (c - l) / dx : (r - c) / dx;                            \
            T ddy = (bb >= (T)0) ? (c - d) / dy : (u - c) / dy;                           \
            out[base + k] = UPDATE(c, ddx, ddy, a, bb, dt);                               \
        }                                                                                 \
    }                                                                                     \
}
ORC_UPWIND(orc_upwind_f32, orc_sample_f32, float, orc_update_f32)
ORC_UPWIND(orc_upwind_f64, orc_sample_f64, double, orc_update_f64)

/* Gradient magnitude on a full width x height grid.  Central differences
 * are taken inside, one-sided differences at the borders, with no division
 * by dx (subsetix_amr2/regrid.py:172-223). */
void orc_gradient_f32(const float* data, int width, int height, float* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < (int64_t)width * height; ++idx) {
        int x = (int)(idx % width), y = (int)(idx / width);
        float c = data[idx], gx = 0.0f, gy = 0.0f;
        if (width > 1) {
            if (x == 0) gx = data[idx + 1] - c;
            else if (x == width - 1) gx = c - data[idx - 1];
            else gx = (data[idx + 1] - data[idx - 1]) * 0.5f;
        }
        if (height > 1) {
            if (y == 0) gy = data[idx + width] - c;
            else if (y == height - 1) gy = c - data[idx - width];
            else gy = (data[idx + width] - data[idx - width]) * 0.5f;
        }
        out[idx] = sqrtf(fmaf(gx, gx, gy * gy));  /* fused as in the reference's NVRTC build */
    }
}

/* Run-length encoding of data >= threshold, one row at a time.  This is the
 * ballot RLE of subsetix_amr2/regrid.py:20-124 restated as a scalar scan.
 * A run starts where the predicate turns on and ends where it turns off, or
 * at the width.  When ob is NULL only counts are produced. */
void orc_threshold_rle(const float* data, int width, int height, float threshold,
                       const int32_t* offsets, int32_t* counts, int32_t* ob, int32_t* oe)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int y = 0; y < height; ++y) {
        const float* row = data + (int64_t)y * width;
        int prev = 0, n = 0;
        int64_t w = ob ? offsets[y] : 0;
        for (int x = 0; x < width; ++x) {
            int on = row[x] >= threshold;
            if (on && !prev) { if (ob) ob[w] = x; }
            if (!on && prev) { if (ob) { oe[w] = x; } ++w; ++n; }
            prev = on;
        }
        if (prev) { if (ob) oe[w] = width; ++n; }
        if (counts) counts[y] = n;
    }
}

/* Copy of cells between a subset geometry and a superset geometry with the
 * same coordinates.  dir = 0 gathers super -> subset, dir = 1 scatters
 * subset -> super.  Per subset interval: binary search in the super row,
 * then a walk across super intervals (subsetix_amr2/fields.py:127-294).
 * Values are opaque elements of elem_size bytes. */
void orc_subset_copy(int dir, int64_t intervals, int elem_size,
                     const int32_t* sub_rows, const int32_t* sub_b, const int32_t* sub_e,
                     const int32_t* sub_coff, const int32_t* sup_off, const int32_t* sup_b,
                     const int32_t* sup_e, const int32_t* sup_coff, int32_t super_rows,
                     void* sub_values, void* sup_values)
{
    char* subv = (char*)sub_values;
    char* supv = (char*)sup_values;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < intervals; ++i) {
        int32_t row = sub_rows[i];
        if (row < 0 || row >= super_rows) continue;
        int32_t start = sub_b[i], stop = sub_e[i];
        if (stop <= start) continue;
        int32_t rs = sup_off[row], rt = sup_off[row + 1];
        if (rs >= rt) continue;
        int32_t lo = rs, hi = rt - 1, idx = rs;
        int found = 0;
        while (lo <= hi) {
            int32_t mid = (lo + hi) >> 1;
            if (start < sup_b[mid]) hi = mid - 1;
            else if (start >= sup_e[mid]) lo = mid + 1;
            else { idx = mid; found = 1; break; }
        }
        if (!found) idx = lo;
        if (idx < rs) idx = rs;
        int32_t cur = start, done = 0;
        int32_t sub_base = sub_coff[i];
        while (cur < stop && idx < rt) {
            int32_t b = sup_b[idx], e = sup_e[idx];
            if (cur < b) { cur = b; continue; }
            int32_t stop2 = stop < e ? stop : e;
            int32_t len = stop2 - cur;
            if (len > 0) {
                int64_t sup_pos = (int64_t)sup_coff[idx] + (cur - b);
                int64_t sub_pos = (int64_t)sub_base + done;
                if (dir == 0) memcpy(subv + sub_pos * elem_size, supv + sup_pos * elem_size, (size_t)len * elem_size);
                else memcpy(supv + sup_pos * elem_size, subv + sub_pos * elem_size, (size_t)len * elem_size);
                done += len;
                cur = stop2;
            }
            if (cur >= e) ++idx;
            if (len == 0 && cur < stop) ++cur;
        }
    }
}

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
