// Row sweeps: fused boolean expressions over canonical sets, and run merging
// of widened, row-shifted sets (dilation).
//
// Why one kernel covers a whole expression.  Take canonical sets: inside
// each row, intervals are non-empty, strictly increasing and non-touching.
// On them the reference's union, intersection, difference and xor each
// return the maximal runs of the cell-set result
// (subsetix_cupy/kernels.py:36-113; xor is (A\B) | (B\A),
// expressions.py:380-388).  Maximal runs are canonical again, so any nested
// expression of those ops returns the maximal runs of f(in_1(x), ...,
// in_k(x)), where f is the expression as a boolean function.  MODE_TABLE
// computes exactly that from a truth table of f.
//
// MODE_UNION merges widened intervals ([b - w, e + w)) from k row-shifted
// views of one set.  A run continues while the next begin is <= the running
// end.  This is the merge of subsetix_cupy/kernels.py:292-381 after the
// (row, begin) sort of morphology.py:21-107, which dilation uses
// (morphology.py:211-248).  It needs non-empty intervals with strictly
// increasing begins and ends inside each row.
//
// Layout of the work.  One lane owns one row of the aligned row list, and a
// warp owns a tile of 32 consecutive rows.  A lane sweeps its row as a k-way
// merge of the leaves' boundary streams in coordinate order.  It applies
// every event at a coordinate, then evaluates f once.  A change of f opens
// or closes a run.
//   pass 1   count the row's runs;
//   scan     warp-wide exclusive scan of the counts, then a look-back over
//            tiles for the tile's global base;
//   pass 2   sweep the row again and write its runs.  The row's intervals
//            were read moments before, so this second read is served from
//            L1/L2 and DRAM sees each input about once.
// No shared memory is used.  A row of any length stays on one lane, so
// there is no tile capacity to overflow.
//
// Look-back.  Tiles publish their aggregate and, once known, their
// inclusive prefix (sx_common.cuh).  Groups of 32 consecutive tiles also
// publish a group aggregate (the last member to finish adds it up) and a
// group prefix (posted by the group's last tile).  A tile walks back at
// most 31 tile statuses of its own group, then whole groups, 32 per step.
// The walk stays short even with thousands of tiles in flight.
//
// Inputs outside the contract raise SXF_CONTRACT, and the host then reruns
// the exact reference-order kernels (sx_exact.cu).  All waits are bounded
// (SX_LOOKBACK_SPIN_LIMIT).

#include <climits>

#include "sx_internal.cuh"

#define SX_SWEEP_WARPS 8
#define SX_GROUP 32

enum { MODE_TABLE = 0, MODE_UNION = 1 };

// Look-back state in the workspace: counters[4] | tile status[tiles] |
// group status[groups] | group sum[groups] | group count[groups].
struct SxSweepState {
    unsigned* counters;
    unsigned long long* tile_status;
    unsigned long long* group_status;
    int* group_sum;
    unsigned* group_count;
};

__device__ __forceinline__ unsigned long long sx_ld_status(const unsigned long long* p)
{
    return *((volatile const unsigned long long*)p);
}

// Wait until a status word is published (kind != 0); bounded.
__device__ __forceinline__ unsigned long long sx_wait_status(const unsigned long long* p, bool& timed_out)
{
    unsigned spins = 0;
    while (true) {
        const unsigned long long w = sx_ld_status(p);
        if ((w >> 32) & 3ull) return w;
        if (++spins > SX_LOOKBACK_SPIN_LIMIT) {
            timed_out = true;
            return (SX_KIND_PREFIX << 32);  // treat as a zero prefix so the kernel finishes
        }
        if (spins > 4) __nanosleep(32);
    }
}

__device__ __forceinline__ unsigned long long sx_word(unsigned long long kind, int value)
{
    return (kind << 32) | (unsigned long long)(unsigned)value;
}

// Returns the exclusive prefix of `tile` (whole warp participates).
__device__ __forceinline__ int sx_hier_lookback(const SxSweepState& st, int tile, int tiles, int aggregate,
                                                unsigned& flags)
{
    const int lane = threadIdx.x & 31;
    const int group = tile / SX_GROUP;
    const int gfirst = group * SX_GROUP;
    const int gsize = min(SX_GROUP, tiles - gfirst);
    bool timed_out = false;
    int exclusive = 0;
    if (tile == 0) {
        if (lane == 0) atomicExch(&st.tile_status[0], sx_word(SX_KIND_PREFIX, aggregate));
    } else {
        if (lane == 0) atomicExch(&st.tile_status[tile], sx_word(SX_KIND_AGG, aggregate));
    }
    // group aggregate: the last member to add publishes it (never over a prefix)
    if (lane == 0) {
        atomicAdd(&st.group_sum[group], aggregate);
        __threadfence();
        const unsigned done = atomicAdd(&st.group_count[group], 1u);
        if (done == (unsigned)gsize - 1u) {
            __threadfence();
            const int gsum = atomicAdd(&st.group_sum[group], 0);
            atomicCAS(&st.group_status[group], 0ull, sx_word(SX_KIND_AGG, gsum));
        }
    }
    if (tile > 0) {
        // 1. tiles of the own group before this one (at most 31)
        bool found = false;
        {
            const int t = tile - 1 - lane;
            unsigned long long w = sx_word(SX_KIND_AGG, 0);
            if (t >= gfirst) w = sx_wait_status(&st.tile_status[t], timed_out);
            const bool is_prefix = (t >= gfirst) && (((w >> 32) & 3ull) == SX_KIND_PREFIX);
            const unsigned pm = __ballot_sync(0xFFFFFFFFu, is_prefix);
            const int stop = pm ? __ffs(pm) - 1 : 32;
            int v = (t >= gfirst && lane <= stop) ? (int)(unsigned)(w & 0xFFFFFFFFull) : 0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            exclusive = v;
            found = pm != 0u;
        }
        // 2. whole groups before the own group, 32 per step
        int g = group - 1;
        while (!found && g >= 0) {
            const int gg = g - lane;
            unsigned long long w = sx_word(SX_KIND_PREFIX, 0);
            if (gg >= 0) w = sx_wait_status(&st.group_status[gg], timed_out);
            const bool is_prefix = ((w >> 32) & 3ull) == SX_KIND_PREFIX;
            const unsigned pm = __ballot_sync(0xFFFFFFFFu, is_prefix);
            const int stop = pm ? __ffs(pm) - 1 : 32;
            int v = (gg >= 0 && lane <= stop) ? (int)(unsigned)(w & 0xFFFFFFFFull) : 0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            exclusive += v;
            found = pm != 0u;
            g -= 32;
        }
        if (lane == 0) atomicExch(&st.tile_status[tile], sx_word(SX_KIND_PREFIX, exclusive + aggregate));
    }
    if (lane == 0 && tile == gfirst + gsize - 1)
        atomicExch(&st.group_status[group], sx_word(SX_KIND_PREFIX, exclusive + aggregate));
    if (__any_sync(0xFFFFFFFFu, timed_out)) flags |= SXF_TIMEOUT;
    return exclusive;
}

__device__ __forceinline__ bool sx_table(const SxBoolArgs& A, unsigned state)
{
    return (A.table[state >> 5] >> (state & 31u)) & 1u;
}

// One row, canonical leaves, truth-table function.  Returns the run count;
// writes runs at out_begin/out_end + pos when WRITE.
template <int K, bool WRITE>
__device__ __forceinline__ int sx_sweep_table(const SxBoolArgs& A, const int* s, const int* lim, int* out_b, int* out_e,
                                              long long pos, bool& bad, bool& over)
{
    int q[K], h[K];
    int rem = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        q[l] = 0;
        h[l] = lim[l] > 0 ? __ldg(A.leaf[l].begin + s[l]) : INT_MAX;
        rem += lim[l];
    }
    unsigned state = 0u;
    bool fprev = false;
    int run_start = 0;
    int n = 0;
    while (rem > 0) {
        int c = INT_MAX;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (q[l] < lim[l]) c = min(c, h[l]);
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (q[l] < lim[l] && h[l] == c) {
                state ^= 1u << l;
                const int qn = q[l] + 1;
                q[l] = qn;
                --rem;
                if (qn < lim[l]) {
                    const int i = s[l] + (qn >> 1);
                    const int v = (qn & 1) ? __ldg(A.leaf[l].end + i) : __ldg(A.leaf[l].begin + i);
                    if (v <= c) bad = true;  // boundaries must rise strictly: non-empty, non-touching
                    h[l] = v;
                }
            }
        }
        const bool fn = sx_table(A, state);
        if (fn != fprev) {
            if (fn) {
                run_start = c;
            } else {
                if (WRITE) {
                    const long long o = pos + n;
                    if (o < A.capacity) {
                        out_b[o] = run_start;
                        out_e[o] = c;
                    } else {
                        over = true;
                    }
                }
                ++n;
            }
            fprev = fn;
        }
        if (c == INT_MAX) break;  // only reachable with malformed input
    }
    return n;
}

// Begin/end of one interval after the leaf's coordinate transform: widened
// by `widen` ([b - w, e + w)), or coarsened by `scale` ([floor(b/r), ceil(e/r))).
__device__ __forceinline__ int sx_floordiv(int a, int r) { return a >= 0 ? a / r : -((-a + r - 1) / r); }

__device__ __forceinline__ int sx_tb(const SxLeafDev& L, int i)
{
    const int b = __ldg(L.begin + i);
    return L.scale > 1 ? sx_floordiv(b, L.scale) : b - L.widen;
}

__device__ __forceinline__ int sx_te(const SxLeafDev& L, int i)
{
    const int e = __ldg(L.end + i);
    return L.scale > 1 ? -sx_floordiv(-e, L.scale) : e + L.widen;
}

// One row, K views of interval sets (row-shifted, widened or coarsened):
// their union with the reference's merge semantics (touching runs join).
// Begins and ends of a view must each be non-decreasing; every event at a
// coordinate is applied before the run state is examined.
template <int K, bool WRITE>
__device__ __forceinline__ int sx_sweep_union(const SxBoolArgs& A, const int* s, const int* cnt, int* out_b, int* out_e,
                                              long long pos, bool& bad, bool& over)
{
    int qb[K], qe[K], hb[K], he[K];
    int rem = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        qb[l] = 0;
        qe[l] = 0;
        hb[l] = cnt[l] > 0 ? sx_tb(A.leaf[l], s[l]) : INT_MAX;
        he[l] = cnt[l] > 0 ? sx_te(A.leaf[l], s[l]) : INT_MAX;
        rem += 2 * cnt[l];
    }
    int active = 0;
    int run_start = 0;
    int n = 0;
    while (rem > 0) {
        int c = INT_MAX;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (qb[l] < cnt[l]) c = min(c, hb[l]);
            if (qe[l] < cnt[l]) c = min(c, he[l]);
        }
        const bool was = active > 0;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            // ends before begins: an element whose begin has not been taken at
            // an earlier coordinate is empty (or reversed) and breaks the contract
            while (qe[l] < cnt[l] && he[l] == c) {
                --active;
                --rem;
                if (qe[l] >= qb[l]) bad = true;
                const int qn = ++qe[l];
                if (qn < cnt[l]) {
                    const int v = sx_te(A.leaf[l], s[l] + qn);
                    if (v < c) bad = true;
                    he[l] = v;
                }
            }
            while (qb[l] < cnt[l] && hb[l] == c) {
                ++active;
                --rem;
                const int qn = ++qb[l];
                if (qn < cnt[l]) {
                    const int v = sx_tb(A.leaf[l], s[l] + qn);
                    if (v < c) bad = true;
                    hb[l] = v;
                }
            }
        }
        const bool now = active > 0;
        if (now != was) {
            if (now) {
                run_start = c;
            } else {
                if (WRITE) {
                    const long long o = pos + n;
                    if (o < A.capacity) {
                        out_b[o] = run_start;
                        out_e[o] = c;
                    } else {
                        over = true;
                    }
                }
                ++n;
            }
        }
        if (active < 0) bad = true;
        if (c == INT_MAX) break;
    }
    return n;
}

template <int K, int MODE>
__global__ void __launch_bounds__(32 * SX_SWEEP_WARPS) sx_sweep_kernel(SxBoolArgs A, SxSweepState st, int tiles)
{
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    if (blockIdx.x * SX_SWEEP_WARPS + wid >= tiles) return;  // exactly `tiles` warps take tickets

    int tile = 0;
    if (lane == 0) tile = (int)atomicAdd(&st.counters[0], 1u);
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);

    const int row = tile * 32 + lane;
    const bool active = row < A.rows;
    int s[K], lim[K];
#pragma unroll
    for (int l = 0; l < K; ++l) {
        const int a = active ? A.leaf[l].off[row] : 0;
        const int b = active ? (A.leaf[l].off_end ? A.leaf[l].off_end[row] : A.leaf[l].off[row + 1]) : 0;
        s[l] = a;
        lim[l] = MODE == MODE_TABLE ? 2 * (b - a) : (b - a);
    }
    bool bad = false, over = false;
    int count = 0;
    if (active) {
        count = MODE == MODE_TABLE ? sx_sweep_table<K, false>(A, s, lim, nullptr, nullptr, 0, bad, over)
                                   : sx_sweep_union<K, false>(A, s, lim, nullptr, nullptr, 0, bad, over);
    }
    int incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    unsigned flags = __any_sync(0xFFFFFFFFu, bad) ? SXF_CONTRACT : 0u;
    const int base = sx_hier_lookback(st, tile, tiles, total, flags);
    if (active) {
        const long long pos = (long long)base + incl - count;
        if (count > 0) {
            bool bad2 = false;
            if (MODE == MODE_TABLE)
                sx_sweep_table<K, true>(A, s, lim, A.out_begin, A.out_end, pos, bad2, over);
            else
                sx_sweep_union<K, true>(A, s, lim, A.out_begin, A.out_end, pos, bad2, over);
        }
        A.out_off[row + 1] = base + incl;
        if (row == 0) A.out_off[0] = 0;
    }
    if (__any_sync(0xFFFFFFFFu, over)) flags |= SXF_CAPACITY;
    if (lane == 0) {
        // retire: the last tile publishes the total and the flags
        if (flags) atomicOr(&st.counters[3], flags);
        __threadfence();
        const unsigned prev = atomicAdd(&st.counters[1], 1u);
        if (prev == (unsigned)tiles - 1u) {
            __threadfence();
            const unsigned long long last = sx_ld_status(&st.tile_status[tiles - 1]);
            const unsigned f = atomicExch(&st.counters[3], 0u);
            A.result[0] = (int)(unsigned)(last & 0xFFFFFFFFull);
            A.result[1] = (int)f;
        }
    }
}

// ---------------------------------------------------------------------------
// Shared-memory form of the table sweep (a tuning option, sx_tuning kernel 2).
//
// The warp stages its 32-row tile with coalesced loads.  Each leaf's
// segment is stored interleaved, [b0, e0, b1, e1, ...], so a lane's
// boundary stream for one leaf is contiguous.  The lane then sweeps its row
// from shared memory in one pass.  Its runs go to a provisional slice of
// the output staging area (a row never yields more runs than it has
// elements).  After the warp scan and the look-back, the warp copies the
// runs out to global memory with coalesced stores.  Tiles larger than the
// staging capacity use the global-memory sweep above.
// ---------------------------------------------------------------------------

#define SX_SMEM_WARPS 4

__host__ __device__ inline int sx_smem_warp_ints(int ecap) { return 4 * ecap + 8 + 64; }

template <int K>
__device__ __forceinline__ int sx_smem_sweep_table(const SxBoolArgs& A, const int* __restrict__ S, const int* qs,
                                                   const int* qend, int* __restrict__ ob, int* __restrict__ oe,
                                                   bool& bad)
{
    int q[K], h[K];
#pragma unroll
    for (int l = 0; l < K; ++l) {
        q[l] = qs[l];
        h[l] = q[l] < qend[l] ? S[q[l]] : INT_MAX;
    }
    unsigned state = 0u;
    bool fprev = false;
    int run_start = 0;
    int n = 0;
    while (true) {
        int c = h[0];
#pragma unroll
        for (int l = 1; l < K; ++l) c = min(c, h[l]);
        if (c == INT_MAX) break;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (h[l] == c) {
                state ^= 1u << l;
                const int qn = q[l] + 1;
                q[l] = qn;
                const int v = S[qn];  // one slot of slack after the staged data
                if (qn < qend[l]) {
                    if (v <= c) bad = true;
                    h[l] = v;
                } else {
                    h[l] = INT_MAX;
                }
            }
        }
        const bool fn = sx_table(A, state);
        if (fn != fprev) {
            if (fn) {
                run_start = c;
            } else {
                ob[n] = run_start;
                oe[n] = c;
                ++n;
            }
            fprev = fn;
        }
    }
    return n;
}

template <int K>
__global__ void __launch_bounds__(32 * SX_SMEM_WARPS) sx_sweep_smem_kernel(SxBoolArgs A, SxSweepState st, int tiles,
                                                                          int ecap)
{
    extern __shared__ int smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    if (blockIdx.x * SX_SMEM_WARPS + wid >= tiles) return;  // exactly `tiles` warps take tickets
    int* S = smem_raw + wid * sx_smem_warp_ints(ecap);
    int* Ob = S + 2 * ecap + 8;
    int* Oe = Ob + ecap;
    int* X = Oe + ecap;  // [32] exclusive run counts, [32] provisional starts

    int tile = 0;
    if (lane == 0) tile = (int)atomicAdd(&st.counters[0], 1u);
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
    const int lo = tile * 32;
    const int hi = min(A.rows, lo + 32);
    const int row = lo + lane;
    const bool active = row < A.rows;

    // tile range of every leaf
    int g0v = 0, g1v = 0;
    if (lane < K) {
        g0v = A.leaf[lane].off[lo];
        g1v = A.leaf[lane].off[hi];
    }
    int g0[K], g1[K], lb2[K];
    int E = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        g0[l] = __shfl_sync(0xFFFFFFFFu, g0v, l);
        g1[l] = __shfl_sync(0xFFFFFFFFu, g1v, l);
        lb2[l] = 2 * E;
        E += g1[l] - g0[l];
    }
    // this lane's row range in every leaf
    int qs[K], qend[K], s[K], lim[K];
    int nrow = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        const int a = active ? A.leaf[l].off[row] : g1[l];
        const int b = active ? A.leaf[l].off[row + 1] : g1[l];
        qs[l] = lb2[l] + 2 * (a - g0[l]);
        qend[l] = lb2[l] + 2 * (b - g0[l]);
        s[l] = a;
        lim[l] = 2 * (b - a);
        nrow += b - a;
    }
    int prov = nrow;  // provisional start of this lane's runs (exclusive scan of row elements)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, prov, o);
        if (lane >= o) prov += y;
    }
    prov -= nrow;

    const bool staged = E <= ecap;
    bool bad = false, over = false;
    int count = 0;
    if (staged) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int cnt = g1[l] - g0[l];
            const int* gb = A.leaf[l].begin + g0[l];
            const int* ge = A.leaf[l].end + g0[l];
            for (int j = lane; j < cnt; j += 32) {
                const int b = __ldg(gb + j);
                const int e = __ldg(ge + j);
                if (b == INT_MAX || e == INT_MAX) bad = true;  // reserved as the stream sentinel
                S[lb2[l] + 2 * j] = b;
                S[lb2[l] + 2 * j + 1] = e;
            }
        }
        if (lane == 0) S[2 * E] = INT_MAX;
        __syncwarp();
        if (active) count = sx_smem_sweep_table<K>(A, S, qs, qend, Ob + prov, Oe + prov, bad);
    } else if (active) {
        count = sx_sweep_table<K, false>(A, s, lim, nullptr, nullptr, 0, bad, over);
    }

    int incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const int excl = incl - count;
    unsigned flags = __any_sync(0xFFFFFFFFu, bad) ? SXF_CONTRACT : 0u;
    const int base = sx_hier_lookback(st, tile, tiles, total, flags);

    if (staged) {
        X[lane] = excl;
        X[32 + lane] = prov;
        __syncwarp();
        for (int i = lane; i < total; i += 32) {
            int lo2 = 0, hi2 = 31;  // owner: last lane with excl <= i
            while (lo2 < hi2) {
                const int mid = (lo2 + hi2 + 1) >> 1;
                if (X[mid] <= i) lo2 = mid; else hi2 = mid - 1;
            }
            const int src = X[32 + lo2] + (i - X[lo2]);
            const long long o = (long long)base + i;
            if (o < A.capacity) {
                A.out_begin[o] = Ob[src];
                A.out_end[o] = Oe[src];
            } else {
                over = true;
            }
        }
    } else if (active && count > 0) {
        bool bad2 = false;
        sx_sweep_table<K, true>(A, s, lim, A.out_begin, A.out_end, (long long)base + excl, bad2, over);
    }
    if (active) {
        A.out_off[row + 1] = base + incl;
        if (row == 0) A.out_off[0] = 0;
    }
    if (__any_sync(0xFFFFFFFFu, over)) flags |= SXF_CAPACITY;
    if (lane == 0) {
        if (flags) atomicOr(&st.counters[3], flags);
        __threadfence();
        const unsigned prev = atomicAdd(&st.counters[1], 1u);
        if (prev == (unsigned)tiles - 1u) {
            __threadfence();
            const unsigned long long last = sx_ld_status(&st.tile_status[tiles - 1]);
            const unsigned f = atomicExch(&st.counters[3], 0u);
            A.result[0] = (int)(unsigned)(last & 0xFFFFFFFFull);
            A.result[1] = (int)f;
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// Merge-path form of the table sweep (a tuning option, sx_tuning kernel 3).
//
// A block of SXM_THREADS threads owns one tile of 32 aligned rows.  Every
// boundary of every leaf in the tile becomes a key (row, x, leaf) in shared
// memory: 32 bits (row << 27 | (x - xmin) << 3 | leaf) when the tile's
// coordinates span less than 2^24, else 64 bits (row << 40 | (x + 2^31) << 8
// | leaf).  Each leaf's keys are already sorted (rows are consecutive and,
// on canonical leaves, boundaries rise inside a row), so the tile's keys are
// merged pairwise with balanced merge paths: every thread merges the same
// number of keys, whatever the row lengths.  An exclusive XOR-scan of
// (1 << leaf) over the merged keys gives the membership state after each
// boundary.  At the last key of each (row, x) group, f(state) is compared
// with f before the group; a change is an output boundary.  Output
// boundaries alternate begin/end and never cross rows (every row ends with
// all leaves outside, and f(0) = 0).
//
// One pass over the inputs: the output boundaries are kept in shared memory
// while the block scans their count and the tile's global base comes from
// the look-back, then they are written out.
//
// Contract: each leaf's boundaries must rise strictly inside a row
// (non-empty, non-touching, sorted intervals); otherwise SXF_CONTRACT.  A
// tile whose keys do not fit in shared memory is swept by its first warp
// with the one-lane-per-row sweep above (same results, slower).
// ---------------------------------------------------------------------------
#define SXM_THREADS 256
#define SXM_WARPS (SXM_THREADS / 32)
#define SXM_TR 32

template <typename KeyT>
struct SxmKey;

template <>
struct SxmKey<unsigned> {
    static constexpr unsigned MAX = 0xFFFFFFFFu;
    __device__ static unsigned make(int r, int x, int l, int xmin)
    {
        return ((unsigned)r << 27) | ((unsigned)(x - xmin) << 3) | (unsigned)l;
    }
    __device__ static unsigned group(unsigned k) { return k >> 3; }
    __device__ static int row(unsigned k) { return (int)(k >> 27); }
    __device__ static int x(unsigned k, int xmin) { return xmin + (int)((k >> 3) & 0xFFFFFFu); }
    __device__ static unsigned tag(unsigned k) { return k & 7u; }
};

template <>
struct SxmKey<unsigned long long> {
    static constexpr unsigned long long MAX = 0xFFFFFFFFFFFFFFFFull;
    __device__ static unsigned long long make(int r, int x, int l, int)
    {
        return ((unsigned long long)r << 40) | ((unsigned long long)((unsigned)x ^ 0x80000000u) << 8) |
               (unsigned long long)l;
    }
    __device__ static unsigned long long group(unsigned long long k) { return k >> 8; }
    __device__ static int row(unsigned long long k) { return (int)(k >> 40); }
    __device__ static int x(unsigned long long k, int) { return (int)((unsigned)(k >> 8) ^ 0x80000000u); }
    __device__ static unsigned tag(unsigned long long k) { return (unsigned)(k & 7ull); }
};

// Block-wide exclusive sum (all SXM_THREADS threads call it).
__device__ __forceinline__ int sxm_block_excl_sum(int v, int* s_warp, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int w = lane < SXM_WARPS ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < SXM_WARPS) s_warp[lane] = wi - w;
        if (lane == SXM_WARPS - 1) s_warp[SXM_WARPS] = wi;
    }
    __syncthreads();
    const int r = s_warp[wid] + incl - v;
    *total = s_warp[SXM_WARPS];
    __syncthreads();
    return r;
}

// Block-wide exclusive XOR scan.
__device__ __forceinline__ unsigned sxm_block_excl_xor(unsigned v, int* s_warp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl ^= y;
    }
    if (lane == 31) s_warp[wid] = (int)incl;
    __syncthreads();
    if (wid == 0) {
        const unsigned w = lane < SXM_WARPS ? (unsigned)s_warp[lane] : 0u;
        unsigned wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi ^= y;
        }
        if (lane < SXM_WARPS) s_warp[lane] = (int)(wi ^ w);
    }
    __syncthreads();
    const unsigned r = (unsigned)s_warp[wid] ^ incl ^ v;
    __syncthreads();
    return r;
}

struct SxmTile {
    int off[SX_TABLE_MAX_LEAVES][SXM_TR + 1];
    const int* lb[SX_TABLE_MAX_LEAVES];
    const int* le[SX_TABLE_MAX_LEAVES];
    int ls[SX_TABLE_MAX_LEAVES], ll[SX_TABLE_MAX_LEAVES], lbuf[SX_TABLE_MAX_LEAVES];
    int nl;
    int warp[SXM_WARPS + 1];
    unsigned tab[8];
    int rowcnt[SXM_TR];
    int xmin, xmax;
    int tile, base;
    unsigned flags;
};

// Keys, merges and output boundaries of one tile with key type KeyT.
// Returns the number of output boundaries of this thread; they are left in
// `emits` (this thread's slots [c0, c0 + n)); *excl receives this thread's
// exclusive position among the tile's output boundaries and *total the
// tile's count.  All threads of the block call it.
// Key buffers per tile: two, or three for K = 3, 6, 7, where the merge tree
// (odd lists stay in place) would otherwise read and write one buffer.
template <int K>
struct SxmBuffers {
    static constexpr int n = (K == 3 || K == 6 || K == 7) ? 3 : 2;
};

template <int K, typename KeyT>
__device__ __forceinline__ int sxm_tile(SxmTile& S, unsigned char* smem, int cap_bytes, int nrows, int T,
                                        const int* start, const int* len, unsigned& bad, KeyT*& emits, int& c0,
                                        int* excl, int* total)
{
    using Key = SxmKey<KeyT>;
    constexpr int NB = SxmBuffers<K>::n;
    const int tid = threadIdx.x;
    const int capk = cap_bytes / (NB * (int)sizeof(KeyT));
    KeyT* buf[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) buf[q] = (KeyT*)smem + q * capk;
    const int xmin = S.xmin;
    const int nint = T >> 1;
    // 1a. row of every interval of the tile, one byte each (in buffer 1)
    unsigned char* rowmap = (unsigned char*)buf[1];
    for (int t = tid; t < K * nrows; t += SXM_THREADS) {
        const int l = t / nrows, r = t - l * nrows;
        int sl = 0;
#pragma unroll
        for (int q = 1; q < K; ++q)
            if (l == q) sl = start[q];
        const int o0 = S.off[l][0];
        for (int g = S.off[l][r]; g < S.off[l][r + 1]; ++g) rowmap[(sl >> 1) + g - o0] = (unsigned char)r;
    }
    __syncthreads();
    // 1b. keys, one thread per interval: list l's keys sit at [start[l], start[l] + len[l])
    for (int e = tid; e < nint; e += SXM_THREADS) {
        int l = 0, sl = 0, el = len[0];
#pragma unroll
        for (int q = 1; q < K; ++q)
            if (2 * e >= start[q]) {
                l = q;
                sl = start[q];
                el = start[q] + len[q];
            }
        const int g = S.off[l][0] + e - (sl >> 1);
        const int r = rowmap[e];
        const int b = __ldg(S.lb[l] + g), en = __ldg(S.le[l] + g);
        bool ok = b < en;
        if (2 * e + 2 < el && rowmap[e + 1] == r) ok = ok && en < __ldg(S.lb[l] + g + 1);
        if (!ok) bad = 1u;
        buf[0][2 * e] = Key::make(r, b, l, xmin);
        buf[0][2 * e + 1] = Key::make(r, en, l, xmin);
    }
    if (tid == 0) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            S.ls[l] = start[l];
            S.ll[l] = len[l];
            S.lbuf[l] = 0;
        }
        S.nl = K;
    }
    __syncthreads();
    // 2. pairwise merges; a list without a partner stays where it is
    c0 = (int)(((long long)T * tid) / SXM_THREADS);
    const int c1 = (int)(((long long)T * (tid + 1)) / SXM_THREADS);
    unsigned xacc = 0u;  // XOR of (1 << leaf) over this thread's last merged range
    const bool single = S.nl == 1;
    while (S.nl > 1) {
        xacc = 0u;
        const int nl = S.nl;
        const int np = nl >> 1;  // merged pairs; list nl-1 waits when nl is odd
        const int M = S.ls[2 * np - 1] + S.ll[2 * np - 1];  // pairs cover [0, M)
        const int m0 = (int)(((long long)M * tid) / SXM_THREADS);
        const int m1 = (int)(((long long)M * (tid + 1)) / SXM_THREADS);
        int k = m0;
        int p = 0;
        while (k < m1) {
            while (p + 1 < np && k >= S.ls[2 * (p + 1)]) ++p;
            const int a0 = S.ls[2 * p], la = S.ll[2 * p], lb = S.ll[2 * p + 1];
            const int ba = S.lbuf[2 * p], bb = S.lbuf[2 * p + 1];
            const int bo = (ba != 0 && bb != 0) ? 0 : ((ba != 1 && bb != 1) ? 1 : 2);
            const KeyT* A_ = buf[0];
            const KeyT* B_ = buf[0];
            KeyT* D_ = buf[0];
#pragma unroll
            for (int q = 1; q < NB; ++q) {
                if (ba == q) A_ = buf[q];
                if (bb == q) B_ = buf[q];
                if (bo == q) D_ = buf[q];
            }
            const int b0 = a0 + la;
            const int pend = min(m1, a0 + la + lb);
            const int d = k - a0;
            int lo = max(0, d - lb), hi = min(d, la);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (A_[a0 + mid] < B_[b0 + d - 1 - mid]) lo = mid + 1; else hi = mid;
            }
            int i = lo, j = d - lo;
            KeyT ka = i < la ? A_[a0 + i] : Key::MAX;
            KeyT kb = j < lb ? B_[b0 + j] : Key::MAX;
            for (; k < pend; ++k) {
                const bool ta = ka < kb;
                const KeyT kk = ta ? ka : kb;
                D_[k] = kk;
                xacc ^= 1u << Key::tag(kk);
                if (ta) {
                    ++i;
                    ka = i < la ? A_[a0 + i] : Key::MAX;
                } else {
                    ++j;
                    kb = j < lb ? B_[b0 + j] : Key::MAX;
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            for (int q = 0; q < np; ++q) {
                const int ba = S.lbuf[2 * q], bb = S.lbuf[2 * q + 1];
                S.ls[q] = S.ls[2 * q];
                S.ll[q] = S.ll[2 * q] + S.ll[2 * q + 1];
                S.lbuf[q] = (ba != 0 && bb != 0) ? 0 : ((ba != 1 && bb != 1) ? 1 : 2);
            }
            if (nl & 1) {
                S.ls[np] = S.ls[nl - 1];
                S.ll[np] = S.ll[nl - 1];
                S.lbuf[np] = S.lbuf[nl - 1];
            }
            S.nl = np + (nl & 1);
        }
        __syncthreads();
    }
    const int mb = S.lbuf[0];
    const KeyT* m = buf[0];
    emits = buf[1];
#pragma unroll
    for (int q = 1; q < NB; ++q)
        if (mb == q) m = buf[q];
    if (mb == 1) emits = buf[0];
    // 3. states: XOR of (1 << leaf) before this thread's chunk.  The last
    // merge round covered all T keys with the same split as [c0, c1).
    if (single)
        for (int i = c0; i < c1; ++i) xacc ^= 1u << Key::tag(m[i]);
    unsigned s = sxm_block_excl_xor(xacc, S.warp);
    // 4. output boundaries of the chunk, kept in `emits` at [c0, c0 + n)
    int n = 0;
    if (c0 < c1) {
        unsigned gstate = s;  // state before the (row, x) group holding c0
        {
            const KeyT g = Key::group(m[c0]);
            int gs = c0;
            while (gs > 0 && Key::group(m[gs - 1]) == g) {
                --gs;
                gstate ^= 1u << Key::tag(m[gs]);
            }
        }
        const unsigned tab0 = S.tab[0];
        bool fprev = K <= 5 ? ((tab0 >> gstate) & 1u) : ((S.tab[gstate >> 5] >> (gstate & 31u)) & 1u);
        KeyT cur = m[c0];
        for (int i = c0; i < c1; ++i) {
            const KeyT nxt = (i + 1 < T) ? m[i + 1] : Key::MAX;
            s ^= 1u << Key::tag(cur);
            if (Key::group(nxt) != Key::group(cur)) {
                const bool fa = K <= 5 ? ((tab0 >> s) & 1u) : ((S.tab[s >> 5] >> (s & 31u)) & 1u);
                if (fa != fprev) {
                    emits[c0 + n] = cur;
                    ++n;
                    if (fa) atomicAdd(&S.rowcnt[Key::row(cur)], 1);
                    fprev = fa;
                }
            }
            cur = nxt;
        }
    }
    *excl = sxm_block_excl_sum(n, S.warp, total);
    return n;
}

template <int K, typename KeyT>
__device__ __forceinline__ void sxm_write(const SxBoolArgs& A, const SxmTile& S, const KeyT* emits, int c0, int n,
                                          int excl, int base, bool& over)
{
    using Key = SxmKey<KeyT>;
    const long long cap = A.capacity;
    for (int q = 0; q < n; ++q) {
        const KeyT key = emits[c0 + q];
        const int p = excl + q;
        const long long o = (long long)base + (p >> 1);
        if (o < cap) {
            if (p & 1) A.out_end[o] = Key::x(key, S.xmin); else A.out_begin[o] = Key::x(key, S.xmin);
        } else {
            over = true;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(SXM_THREADS) sx_merge_kernel(SxBoolArgs A, SxSweepState st, int tiles,
                                                                 int cap_bytes)
{
    extern __shared__ __align__(16) unsigned char sxm_smem[];
    __shared__ SxmTile S;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) {
        S.tile = (int)atomicAdd(&st.counters[0], 1u);
        S.flags = 0u;
        S.xmin = INT_MAX;
        S.xmax = INT_MIN;
    }
    if (tid < 8) S.tab[tid] = A.table[tid];
    if (tid < SXM_TR) S.rowcnt[tid] = 0;
    if (tid < K) {
        S.lb[tid] = A.leaf[tid].begin;
        S.le[tid] = A.leaf[tid].end;
    }
    __syncthreads();
    const int tile = S.tile;
    const int r0 = tile * SXM_TR;
    const int nrows = min(SXM_TR, A.rows - r0);
    for (int t = tid; t < K * (nrows + 1); t += SXM_THREADS) {
        const int l = t / (nrows + 1), r = t - l * (nrows + 1);
        S.off[l][r] = A.leaf[l].off[r0 + r];
    }
    __syncthreads();
    // coordinate span of the tile: first begin and last end of every leaf row
    for (int t = tid; t < K * nrows; t += SXM_THREADS) {
        const int l = t / nrows, r = t - l * nrows;
        const int g0 = S.off[l][r], g1 = S.off[l][r + 1];
        if (g1 > g0) {
            atomicMin(&S.xmin, min(__ldg(S.lb[l] + g0), __ldg(S.le[l] + g0)));
            atomicMax(&S.xmax, max(__ldg(S.le[l] + g1 - 1), __ldg(S.lb[l] + g1 - 1)));
        }
    }
    int len[K], start[K];
    int T = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        len[l] = 2 * (S.off[l][nrows] - S.off[l][0]);
        start[l] = T;
        T += len[l];
    }
    __syncthreads();
    const bool narrow = (long long)S.xmax - (long long)S.xmin < (1ll << 24);
    constexpr int NB = SxmBuffers<K>::n;
    const int mode = (narrow && 4ll * NB * T <= cap_bytes) ? 1 : ((8ll * NB * T <= cap_bytes) ? 2 : 0);
    unsigned bad = 0u;
    int count = 0, n = 0, excl = 0, c0 = 0;
    unsigned* e32 = nullptr;
    unsigned long long* e64 = nullptr;
    if (mode == 1) {
        int total;
        n = sxm_tile<K, unsigned>(S, sxm_smem, cap_bytes, nrows, T, start, len, bad, e32, c0, &excl, &total);
        count = total >> 1;
    } else if (mode == 2) {
        int total;
        n = sxm_tile<K, unsigned long long>(S, sxm_smem, cap_bytes, nrows, T, start, len, bad, e64, c0, &excl, &total);
        count = total >> 1;
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0) S.flags |= SXF_CONTRACT;
    }
    // fallback tile: one lane per row over global memory
    int lane_count = 0;
    int s_row[K], lim_row[K];
    if (mode == 0 && wid == 0) {
        const bool act = lane < nrows;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int a = act ? S.off[l][lane] : 0;
            const int b = act ? S.off[l][lane + 1] : 0;
            s_row[l] = a;
            lim_row[l] = 2 * (b - a);
        }
        bool fb_bad = false, fb_over = false;
        if (act) lane_count = sx_sweep_table<K, false>(A, s_row, lim_row, nullptr, nullptr, 0, fb_bad, fb_over);
        if (__any_sync(0xFFFFFFFFu, fb_bad) && lane == 0) S.flags |= SXF_CONTRACT;
        int tot = lane_count;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
        count = tot;
    }
    // look-back for the tile's base
    if (wid == 0) {
        unsigned f = 0u;
        const int base = sx_hier_lookback(st, tile, tiles, count, f);
        if (lane == 0) {
            S.base = base;
            if (f) S.flags |= f;
        }
    }
    __syncthreads();
    const int base = S.base;
    bool over = false;
    if (mode != 0) {
        if (mode == 1) sxm_write<K, unsigned>(A, S, e32, c0, n, excl, base, over);
        else sxm_write<K, unsigned long long>(A, S, e64, c0, n, excl, base, over);
        if (wid == 0) {
            const int c = lane < nrows ? S.rowcnt[lane] : 0;
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < nrows) A.out_off[r0 + lane + 1] = base + incl;
            if (tile == 0 && lane == 0) A.out_off[0] = 0;
        }
    } else if (wid == 0) {
        int incl = lane_count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nrows) {
            bool fb_bad = false;
            if (lane_count > 0)
                sx_sweep_table<K, true>(A, s_row, lim_row, A.out_begin, A.out_end, (long long)base + incl - lane_count,
                                        fb_bad, over);
            A.out_off[r0 + lane + 1] = base + incl;
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    }
    if (__syncthreads_or(over)) {
        if (tid == 0) S.flags |= SXF_CAPACITY;
    }
    if (tid == 0) {
        const unsigned flags = S.flags;
        if (flags) atomicOr(&st.counters[3], flags);
        __threadfence();
        const unsigned prev = atomicAdd(&st.counters[1], 1u);
        if (prev == (unsigned)tiles - 1u) {
            __threadfence();
            const unsigned long long last = sx_ld_status(&st.tile_status[tiles - 1]);
            const unsigned fl = atomicExch(&st.counters[3], 0u);
            A.result[0] = (int)(unsigned)(last & 0xFFFFFFFFull);
            A.result[1] = (int)fl;
        }
    }
}

// ---------------------------------------------------------------------------
// Segmented sweep in block tiles (sx_tuning kernel 4; the automatic choice
// for skewed rows).  The warp-tile forms below (kernels 5 and 6) share its
// algorithm and are the automatic choice for even rows.
//
// A block owns one tile of 32 aligned rows, as in the merge-path kernel.
// Thread 0 copies every leaf's begin and end ranges of the tile into shared
// memory with bulk asynchronous copies (one round trip for the whole tile,
// completion counted on an mbarrier); meanwhile the warps build, per leaf,
// a bitmap of row starts.  Every boundary then becomes a 32-bit key
// (row << 26 | (x - xmin)) in its leaf's list; the row of an interval is
// the rank of its row start (a prefix popcount) mapped through the list of
// the leaf's non-empty rows.  Each list is sorted (rows are consecutive
// and, on canonical leaves, boundaries rise strictly inside a row) and ends
// with the sentinel 0xFFFFFFFF.
//
// Each thread then sweeps one piece of the tile by itself: the keys in
// [p_t, p_t+1), where the pivots p_t are the keys of the longest list at
// positions t/L of it (L threads).  The piece starts in every list at the
// first key not below p_t (binary searches, interleaved over the lists);
// the membership state there is the parity of that position, because every
// interval contributes a begin and an end.  The sweep takes the smallest
// head, toggles the state bit of every leaf holding it and compares f(state)
// with f before; a change is an output boundary.  A piece never splits a
// (row, x) group, so f is evaluated exactly where the truth-table semantics
// require it.  Output boundaries alternate begin/end and never cross rows
// (every row ends with all leaves outside, and f(0) = 0).  A thread's output
// boundaries are at most its keys, so each thread writes them to its own
// slice of an output area (the space of the copies, dead by then); a block
// scan of the counts packs them into the key area while the look-back gives
// the tile's global base, and the tile is written with coalesced stores.
//
// Inputs are read once, outputs written once.  Per boundary the sweep
// costs a few instructions per leaf plus the min and the table lookup.
//
// Contract: each leaf's boundaries must rise strictly inside a row
// (non-empty, non-touching, sorted intervals); otherwise SXF_CONTRACT and
// the tile writes no intervals.  A tile whose lists exceed the shared-memory
// capacity or whose coordinates span 2^26 or more is swept by its first
// warp with the one-lane-per-row sweep (same results, slower).  Every wait
// is bounded.
// ---------------------------------------------------------------------------
#define SXS_XBITS 26
#define SXS_XMASK ((1u << SXS_XBITS) - 1u)
#define SXS_MAX_THREADS 256
#define SXS_SENTINEL 0xFFFFFFFFu
#define SXS_WAIT_LIMIT (1u << 16)
#define SXS_WAIT_HINT_NS 20000

struct SxsTile {
    int off[SX_TABLE_MAX_LEAVES][SXM_TR + 1];
    int rowtab[SX_TABLE_MAX_LEAVES][SXM_TR];  // rank among the leaf's non-empty rows -> row
    int rawb[SX_TABLE_MAX_LEAVES];            // word index of the tile's first begin in the copy area
    int rawe[SX_TABLE_MAX_LEAVES];            // same for the ends
    unsigned tab[8];
    int warp[SXS_MAX_THREADS / 32 + 1];
    int xmin, xmax;
    int tile, base;
    unsigned flags;
    unsigned long long bar;
};

__device__ __forceinline__ unsigned sxs_saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void sxs_bar_init(unsigned long long* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sxs_saddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The single arrival of the barrier's phase 0, announcing `bytes` of copies.
__device__ __forceinline__ void sxs_bar_expect(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sxs_saddr(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy of `bytes` (a multiple of 16) between 16-byte aligned addresses,
// global to this block's shared memory, counted on `bar`.
__device__ __forceinline__ void sxs_bulk_copy(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sxs_saddr(dst)),
                 "l"(src), "r"(bytes), "r"(sxs_saddr(bar))
                 : "memory");
}

// Bounded wait for phase 0 of `bar`; false if it did not complete.  Each
// try_wait may suspend the thread for up to SXS_WAIT_HINT_NS (it resumes as
// soon as the phase completes), so waiting warps take no issue slots; the
// whole wait is bounded by SXS_WAIT_LIMIT tries.
__device__ __forceinline__ bool sxs_bar_wait(unsigned long long* bar)
{
    const unsigned a = sxs_saddr(bar);
    for (unsigned i = 0; i < SXS_WAIT_LIMIT; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "n"(SXS_WAIT_HINT_NS)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Wait until a tile status word is published, backing off from 32 ns to
// 512 ns between polls so that waiting warps leave the issue slots to the
// warps that sweep; bounded by SX_LOOKBACK_SPIN_LIMIT polls.
__device__ __forceinline__ unsigned long long sxs_wait_status(const unsigned long long* p, bool& timed_out,
                                                             unsigned limit)
{
    unsigned sleep = 32;
    for (unsigned spins = 0;; ++spins) {
        const unsigned long long w = sx_ld_status(p);
        if ((w >> 32) & 3ull) return w;
        if (spins > limit) {
            timed_out = true;
            return (SX_KIND_PREFIX << 32);  // treat as a zero prefix so the kernel finishes
        }
        __nanosleep(sleep);
        if (sleep < 512) sleep <<= 1;
    }
}

// Single-level decoupled look-back for the segmented sweeps (whole warp).
// Status word of a tile: bits 0-31 the value, bits 32-33 the kind (1 tile
// aggregate, 2 inclusive prefix), bits 34-37 the OR of the SXF_* flags of
// the tiles the value covers.  The tile publishes its aggregate, then reads
// its 32 nearest predecessors at once (each wait bounded) and adds values up
// to the nearest inclusive prefix, 32 tiles per step.  Returns the exclusive
// prefix; `flags` comes back as the OR over this tile and all before it.
// A.wait_limit (when set) bounds every wait instead of SX_LOOKBACK_SPIN_LIMIT,
// and the tile A.withhold_tile - 1 publishes nothing: both exist only so that
// tests can make the waits give up.
__device__ __forceinline__ int sxs_lookback(const SxBoolArgs& A, const SxSweepState& st, int tile, int aggregate,
                                            unsigned& flags)
{
    const int lane = threadIdx.x & 31;
    const unsigned limit = A.wait_limit ? A.wait_limit : SX_LOOKBACK_SPIN_LIMIT;
    const bool publish = A.withhold_tile != tile + 1;
    const unsigned long long own = ((unsigned long long)(flags & 15u) << 34) | (unsigned long long)(unsigned)aggregate;
    if (tile == 0) {
        if (lane == 0 && publish) atomicExch(&st.tile_status[0], own | (SX_KIND_PREFIX << 32));
        return 0;
    }
    if (lane == 0 && publish) atomicExch(&st.tile_status[tile], own | (SX_KIND_AGG << 32));
    int exclusive = 0;
    unsigned fl = flags;
    bool timed_out = false;
    for (int pos = tile - 1;; pos -= 32) {
        const int t = pos - lane;
        unsigned long long w = SX_KIND_PREFIX << 32;  // before tile 0: an empty prefix
        if (t >= 0) w = sxs_wait_status(&st.tile_status[t], timed_out, limit);
        const unsigned pm = __ballot_sync(0xFFFFFFFFu, ((w >> 32) & 3ull) == SX_KIND_PREFIX);
        const int stop = pm ? __ffs(pm) - 1 : 32;
        int v = lane <= stop ? (int)(unsigned)(w & 0xFFFFFFFFull) : 0;
        unsigned f = lane <= stop ? (unsigned)(w >> 34) & 15u : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            f |= __shfl_xor_sync(0xFFFFFFFFu, f, o);
        }
        exclusive += v;
        fl |= f;
        if (pm) break;
    }
    if (__any_sync(0xFFFFFFFFu, timed_out)) fl |= SXF_TIMEOUT;
    if (lane == 0 && publish)
        atomicExch(&st.tile_status[tile], ((unsigned long long)(fl & 15u) << 34) | (SX_KIND_PREFIX << 32) |
                                              (unsigned long long)(unsigned)(exclusive + aggregate));
    flags = fl;
    return exclusive;
}

// The last tile in ticket order reports the grand total and the flags of
// every tile; an output beyond the capacity shows as a total above it.
__device__ __forceinline__ void sxs_report(const SxBoolArgs& A, int tile, int tiles, int base, int aggregate,
                                           unsigned flags)
{
    if (tile == tiles - 1 && (threadIdx.x & 31) == 0) {
        const long long total = (long long)base + aggregate;
        A.result[0] = (int)total;
        A.result[1] = (int)(flags | (total > A.capacity ? SXF_CAPACITY : 0u));
    }
}

// Block-wide exclusive sum for any block of whole warps (up to 256 threads).
__device__ __forceinline__ int sxs_block_excl_sum(int v, int* s_warp, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int w = lane < nw ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < nw) s_warp[lane] = wi - w;
        if (lane == nw - 1) s_warp[SXS_MAX_THREADS / 32] = wi;
    }
    __syncthreads();
    const int r = s_warp[wid] + incl - v;
    *total = s_warp[SXS_MAX_THREADS / 32];
    __syncthreads();
    return r;
}

// First position in the sorted list k[0, n) whose key is not below v.
__device__ __forceinline__ int sxs_lower_bound(const unsigned* k, int n, unsigned v)
{
    int pos = 0;
    while (n > 0) {
        const int half = n >> 1;
        if (k[pos + half] < v) {
            pos += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return pos;
}

// One leaf of a sweep step: if the head h equals the step's key c, toggle
// the leaf's state bit and load the next key from shared-memory byte
// address pa + 4.  Predicated, so lanes that take different leaves do not
// diverge.
__device__ __forceinline__ void sxs_advance(unsigned& h, unsigned& pa, unsigned& state, unsigned c, unsigned bit)
{
    asm volatile(
        "{\n .reg .pred q;\n setp.eq.u32 q, %0, %3;\n @q add.u32 %1, %1, 4;\n @q xor.b32 %2, %2, %4;\n"
        " @q ld.shared.u32 %0, [%1];\n}\n"
        : "+r"(h), "+r"(pa), "+r"(state)
        : "r"(c), "r"(bit));
}

// Store c at shared-memory byte address oa and advance oa when f != fprev.
__device__ __forceinline__ void sxs_emit(unsigned& oa, unsigned f, unsigned fprev, unsigned c)
{
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %1, %2;\n @q st.shared.u32 [%0], %3;\n @q add.u32 %0, %0, 4;\n}\n"
                 : "+r"(oa)
                 : "r"(f), "r"(fprev), "r"(c)
                 : "memory");
}

template <int K>
__device__ __forceinline__ unsigned sxs_f(const SxsTile& S, unsigned tab0, unsigned state)
{
    if (K <= 5) return (tab0 >> state) & 1u;
    return (S.tab[state >> 5] >> (state & 31u)) & 1u;
}

template <int K>
__global__ void __launch_bounds__(SXS_MAX_THREADS) sx_seg_kernel(SxBoolArgs A, SxSweepState st, int tiles,
                                                                  int cap_keys, int tr)
{
    extern __shared__ __align__(16) unsigned sxs_smem[];
    __shared__ SxsTile S;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int L = blockDim.x, NW = L >> 5;
    if (tid == 0) {
        S.tile = (int)atomicAdd(&st.counters[0], 1u);
        S.flags = 0u;
        S.xmin = INT_MAX;
        S.xmax = INT_MIN;
        sxs_bar_init(&S.bar);
    }
    if (tid < 8) S.tab[tid] = A.table[tid];
    __syncthreads();
    const int tile = S.tile;
    const int r0 = tile * tr;  // tr <= 32 rows per tile
    const int nrows = min(tr, A.rows - r0);
    for (int r = tid; r <= nrows; r += L) {
#pragma unroll
        for (int l = 0; l < K; ++l) S.off[l][r] = A.leaf[l].off[r0 + r];
    }
    __syncthreads();
    // Shared memory, in 32-bit words: key lists [0, KS) (leaf l at ks[l],
    // 2 n_l keys and two sentinels); copies of the begins and ends, later the
    // output boundaries, [RO, RO + RN); row-start bitmaps and their prefix
    // popcounts [BO, BO + BN).
    int n[K], ks[K];
    long long KSl = 0, El = 0, RNl = 0, BNl = 0;
    int big = 0, nbig = -1, ksbig = 0;
    bool ok = true;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        n[l] = S.off[l][nrows] - S.off[l][0];
        ok = ok && n[l] >= 0;
        ks[l] = (int)KSl;
        if (n[l] > nbig) {
            big = l;
            nbig = n[l];
            ksbig = (int)KSl;
        }
        KSl += 2ll * n[l] + 2;
        El += 2ll * n[l];
        RNl += 2ll * ((n[l] + 11) & ~3);  // two copies of at most n + 6 words, 16-byte aligned
        BNl += 2ll * ((n[l] + 31) >> 5);
    }
    KSl = (KSl + 3) & ~3ll;
    if (RNl < El + 1) RNl = El + 1;  // output boundaries, plus one slot a finished sweep may store into
    const bool fits = ok && KSl + RNl + BNl <= (long long)cap_keys;
    const int E = fits ? (int)El : 0, RO = (int)KSl, BO = (int)(KSl + RNl);
    unsigned* keys = sxs_smem;
    unsigned* raw = sxs_smem + RO;  // copies, then output boundaries
    // 1. bulk copies of every leaf's begins and ends (thread 0)
    if (fits && wid == 0) {
        // lane q < 2K copies leaf q/2's begins (q even) or ends (q odd)
        const int q = lane < 2 * K ? lane : 0;
        const int l = q >> 1;
        int nl = 0, g0 = 0;
        const int* arr = nullptr;
#pragma unroll
        for (int m = 0; m < K; ++m)
            if (m == l) {
                nl = n[m];
                g0 = S.off[m][0];
                arr = (q & 1) ? A.leaf[m].end : A.leaf[m].begin;
            }
        const int* g = arr + g0;
        const uintptr_t a0 = (uintptr_t)g & ~(uintptr_t)15;
        const unsigned len =
            (lane < 2 * K && nl > 0) ? (unsigned)((((uintptr_t)(g + nl) + 15) & ~(uintptr_t)15) - a0) : 0u;
        int incl = (int)(len >> 2);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const int words = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const int pos = incl - (int)(len >> 2);
        if (lane < 2 * K) {
            const int first = pos + (int)(((uintptr_t)g & 15) >> 2);
            if (q & 1) S.rawe[l] = first; else S.rawb[l] = first;
        }
        __syncwarp();  // orders the lanes' writes before lane 0's release on the barrier
        if (lane == 0) sxs_bar_expect(&S.bar, 4u * (unsigned)words);
        __syncwarp();
        if (len > 0u) sxs_bulk_copy(raw + pos, (const void*)a0, len, &S.bar);
    }
    // 2. per leaf (one warp each): row-start bitmap and rank -> row table
    //    (offsets only, so it overlaps the copies)
    if (fits) {
        int bs = BO;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int W = (n[l] + 31) >> 5;
            if (l % NW == wid && n[l] > 0) {
                unsigned* bm = sxs_smem + bs;
                int* wp = (int*)(sxs_smem + bs + W);
                const int g0 = S.off[l][0];
                for (int w = lane; w < W; w += 32) bm[w] = 0u;
                __syncwarp();
                const bool act = lane < nrows;
                const int a = act ? S.off[l][lane] - g0 : 0;
                const int b = act ? S.off[l][lane + 1] - g0 : 0;
                const bool ne = act && a >= 0 && a < b && b <= n[l];
                const unsigned bal = __ballot_sync(0xFFFFFFFFu, ne);
                if (ne) {
                    S.rowtab[l][__popc(bal & ((1u << lane) - 1u))] = lane;
                    atomicOr(&bm[a >> 5], 1u << (a & 31));
                }
                __syncwarp();
                int carry = 0;
                for (int w0 = 0; w0 < W; w0 += 32) {
                    const int w = w0 + lane;
                    const int c = w < W ? __popc(bm[w]) : 0;
                    int incl = c;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                        if (lane >= o) incl += y;
                    }
                    if (w < W) wp[w] = carry + incl - c;
                    carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
                }
            }
            bs += 2 * W;
        }
    }
    // 3. wait for the copies, then the coordinate span (first begin, last end of every row)
    bool copied = true;
    if (fits) copied = sxs_bar_wait(&S.bar);
    if (fits && copied) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (l % NW == wid && n[l] > 0) {
                const int g0 = S.off[l][0];
                const bool act = lane < nrows;
                const int a = act ? S.off[l][lane] - g0 : 0;
                const int b = act ? S.off[l][lane + 1] - g0 : 0;
                int lo = INT_MAX, hi = INT_MIN;
                if (act && a >= 0 && a < b && b <= n[l]) {
                    lo = (int)raw[S.rawb[l] + a];
                    hi = (int)raw[S.rawe[l] + b - 1];
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
                    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
                }
                if (lane == 0) {
                    atomicMin(&S.xmin, lo);
                    atomicMax(&S.xmax, hi);
                }
            }
        }
    }
    if (__syncthreads_or(!copied)) {
        copied = false;
        if (tid == 0) S.flags |= SXF_TIMEOUT;
    }
    const int xmin = S.xmin;
    const bool staged =
        fits && copied && (E == 0 || (long long)S.xmax - (long long)xmin < (1ll << SXS_XBITS));
    unsigned bad = 0u;
    // 4. keys, and the contract checked on the raw coordinates
    if (staged) {
        const unsigned le_mask = 0xFFFFFFFFu >> (31 - lane);  // lanes 0..lane
        int bs = BO;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int W = (n[l] + 31) >> 5;
            const unsigned* bm = sxs_smem + bs;
            const int* wp = (const int*)(sxs_smem + bs + W);
            const unsigned* rb = raw + S.rawb[l];
            const unsigned* re = raw + S.rawe[l];
            unsigned* kk = keys + ks[l];
            for (int j = tid; j < n[l]; j += L) {  // j & 31 == lane
                const int b = (int)rb[j], e = (int)re[j];
                const unsigned word = bm[j >> 5];
                const int rank = wp[j >> 5] + __popc(word & le_mask) - 1;  // < 0 only for disordered offsets
                const unsigned rk = (unsigned)S.rowtab[l][max(rank, 0)] << SXS_XBITS;
                const bool first = (word >> lane) & 1u;
                if (!(b < e) || (!first && !((int)re[j - 1] < b)) || rank < 0) bad = 1u;
                *(uint2*)(kk + 2 * j) =
                    make_uint2(rk | ((unsigned)(b - xmin) & SXS_XMASK), rk | ((unsigned)(e - xmin) & SXS_XMASK));
            }
            if (tid == 0) {
                kk[2 * n[l]] = SXS_SENTINEL;
                kk[2 * n[l] + 1] = SXS_SENTINEL;
            }
            bs += 2 * W;
        }
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0) S.flags |= SXF_CONTRACT;
        bad = 1u;
    }
    const bool sweep = staged && !bad && E > 0;
    unsigned* outk = raw;
    int count = 0, total = 0, excl = 0, prov = 0;
    if (sweep) {
        // 5. this thread's piece [klo, khi) and where it starts in every list
        const int nb2 = 2 * nbig;
        unsigned klo = 0u, khi = SXS_SENTINEL;
        if (tid > 0) klo = keys[ksbig + (int)(((long long)tid * nb2) / L)];
        if (tid + 1 < L) khi = keys[ksbig + (int)(((long long)(tid + 1) * nb2) / L)];
        // lists below the pivot's row lie wholly before it, rows above wholly after
        int pos[K];
        const int rp = (int)(klo >> SXS_XBITS);
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (tid == 0) {
                pos[l] = 0;
            } else if (l == big) {
                pos[l] = (int)(((long long)tid * nb2) / L);
            } else {
                const int lo = 2 * (S.off[l][rp] - S.off[l][0]);
                const int hi = 2 * (S.off[l][rp + 1] - S.off[l][0]);
                pos[l] = lo + sxs_lower_bound(keys + ks[l] + lo, hi - lo, klo);
            }
        }
        unsigned pa[K];
        unsigned h[K];
        unsigned state = 0u;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            pa[l] = sxs_saddr(keys + ks[l] + pos[l]);
            h[l] = keys[ks[l] + pos[l]];
            state |= (unsigned)(pos[l] & 1) << l;
            prov += pos[l];
        }
        // 6. the sweep: smallest head, toggle every leaf holding it, compare f
        const unsigned tab0 = S.tab[0];
        unsigned fprev = sxs_f<K>(S, tab0, state);
        const unsigned o0 = sxs_saddr(outk + prov), oend = sxs_saddr(outk + E);
        unsigned oa = o0;
        while (true) {
            unsigned c = h[0];
#pragma unroll
            for (int l = 1; l < K; ++l) c = min(c, h[l]);
            if (c >= khi) break;
#pragma unroll
            for (int l = 0; l < K; ++l) sxs_advance(h[l], pa[l], state, c, 1u << l);
            const unsigned f = sxs_f<K>(S, tab0, state);
            sxs_emit(oa, f, fprev, c);
            oa = min(oa, oend);
            fprev = f;
        }
        const int o = prov + (int)((oa - o0) >> 2);
        count = max(0, min(o, E) - prov);
        excl = sxs_block_excl_sum(count, S.warp, &total);  // `sweep` is uniform over the block
        total = min(total, E);
    }
    // fallback tile: one lane per row over global memory
    int lane_count = 0;
    int s_row[K], lim_row[K];
    if (!staged && wid == 0) {
        const bool act = lane < nrows;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int a = act ? S.off[l][lane] : 0;
            const int b = act ? S.off[l][lane + 1] : 0;
            s_row[l] = a;
            lim_row[l] = 2 * (b - a);
        }
        bool fb_bad = false, fb_over = false;
        if (act) lane_count = sx_sweep_table<K, false>(A, s_row, lim_row, nullptr, nullptr, 0, fb_bad, fb_over);
        if (__any_sync(0xFFFFFFFFu, fb_bad) && lane == 0) S.flags |= SXF_CONTRACT;
        int tot = lane_count;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
        total = 2 * tot;
    }
    // 7. look-back for the tile's base (warp 0); meanwhile every thread packs
    //    its output boundaries from the output area into the key area
    if (wid == 0) {
        unsigned f = S.flags;
        const int base = sxs_lookback(A, st, tile, total >> 1, f);
        if (lane == 0) {
            S.base = base;
            S.flags = f;
        }
    }
    if (sweep) {
        const int m = min(count, E - excl);
        for (int i = 0; i < m; ++i) keys[excl + i] = outk[prov + i];
    }
    __syncthreads();
    const int base = S.base;
    bool over = false;
    if (staged) {
        // 8. coalesced output and the tile's row offsets
        const int nint = total >> 1;
        for (int i = tid; i < nint; i += L) {
            const uint2 kv = *(const uint2*)(keys + 2 * i);
            const long long o = (long long)base + i;
            if (o < A.capacity) {
                A.out_begin[o] = xmin + (int)(kv.x & SXS_XMASK);
                A.out_end[o] = xmin + (int)(kv.y & SXS_XMASK);
            } else {
                over = true;
            }
        }
        for (int r = tid; r < nrows; r += L) {
            const int pos = sxs_lower_bound(keys, total, (unsigned)(r + 1) << SXS_XBITS);
            A.out_off[r0 + r + 1] = base + (pos >> 1);
        }
        if (tile == 0 && tid == 0) A.out_off[0] = 0;
    } else if (wid == 0) {
        int incl = lane_count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nrows) {
            bool fb_bad = false;
            if (lane_count > 0)
                sx_sweep_table<K, true>(A, s_row, lim_row, A.out_begin, A.out_end, (long long)base + incl - lane_count,
                                        fb_bad, over);
            A.out_off[r0 + lane + 1] = base + incl;
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    }
    (void)over;  // an output beyond the capacity shows in the reported total
    if (wid == 0) sxs_report(A, tile, tiles, base, total >> 1, S.flags);
}

// ---------------------------------------------------------------------------
// Warp-tile segmented sweep.
//
// The same algorithm as the block kernel above, with one warp per tile of
// `tr` rows (at most 32) and no block-wide barrier: each warp takes its own
// tile ticket, has its own slice of shared memory and its own mbarrier, and
// runs its own look-back.  A block holds several independent warps.  Small
// tiles and independent warps keep many tiles in flight per SM, so one
// warp's waits (copies, look-back) are covered by the others' sweeps.
//
// The row of each staged interval is found by walking the tile's row ends
// (a lane starts from the row of the previous chunk's last interval), which
// needs no bitmap.
// ---------------------------------------------------------------------------

// Per-warp header at the start of the warp's slice, in 32-bit words:
// [0, 2) mbarrier, then the tile's row offsets (tr + 1 per leaf), then the
// begin and end copy positions (K each).
__host__ __device__ inline int sxw_hdr_words(int k, int tr) { return (2 + (tr + 1) * k + 2 * k + 3) & ~3; }
__host__ __device__ inline size_t sxw_slice_bytes(int k, int tr, int cap_words)
{
    return 4u * (size_t)(sxw_hdr_words(k, tr) + ((cap_words + 3) & ~3));
}

template <int K>
__global__ void __launch_bounds__(256) sx_wseg_kernel(SxBoolArgs A, SxSweepState st, int tiles, int cap_words, int tr)
{
    extern __shared__ __align__(16) unsigned char sxw_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
    if (blockIdx.x * NW + wid >= tiles) return;  // exactly `tiles` warps take tickets
    unsigned* base_w = (unsigned*)(sxw_smem + (size_t)wid * sxw_slice_bytes(K, tr, cap_words));
    unsigned long long* bar = (unsigned long long*)base_w;
    const int os = tr + 1;                // row offsets of leaf l: off[l * os + r], r in [0, nrows]
    int* off = (int*)base_w + 2;
    int* rawb = off + os * K;             // [K]
    int* rawe = rawb + K;                 // [K]
    unsigned* Wd = base_w + sxw_hdr_words(K, tr);

    int tile = 0;
    if (lane == 0) {
        tile = (int)atomicAdd(&st.counters[0], 1u);
        sxs_bar_init(bar);
    }
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
    const int r0 = tile * tr;
    const int nrows = min(tr, A.rows - r0);
    for (int r = lane; r <= nrows; r += 32) {
#pragma unroll
        for (int l = 0; l < K; ++l) off[l * os + r] = A.leaf[l].off[r0 + r];
    }
    __syncwarp();
    // layout (words): copies, later output boundaries, [0, RN); key lists [RN, RN + KS)
    int n[K], ks[K];
    long long KSl = 0, El = 0, RNl = 0;
    int big = 0, nbig = -1, ksbig = 0;
    bool ok = true;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        n[l] = off[l * os + nrows] - off[l * os];
        ok = ok && n[l] >= 0;
        RNl += 2ll * ((n[l] + 11) & ~3);  // two copies of at most n + 6 words, 16-byte aligned
        El += 2ll * n[l];
    }
    if (RNl < El + 1) RNl = El + 1;
    RNl = (RNl + 3) & ~3ll;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        ks[l] = (int)(RNl + KSl);
        if (n[l] > nbig) {
            big = l;
            nbig = n[l];
            ksbig = ks[l];
        }
        KSl += 2ll * n[l] + 2;
    }
    const bool fits = ok && RNl + KSl <= (long long)cap_words;
    const int E = fits ? (int)El : 0;
    unsigned* raw = Wd;  // copies, then output boundaries
    unsigned* keys = Wd;  // key lists at absolute word positions ks[l]
    // 1. bulk copies: lane q < 2K copies leaf q/2's begins (q even) or ends (q odd)
    if (fits) {
        const int q = lane < 2 * K ? lane : 0;
        const int l = q >> 1;
        int nl = 0, g0 = 0;
        const int* arr = nullptr;
#pragma unroll
        for (int m = 0; m < K; ++m)
            if (m == l) {
                nl = n[m];
                g0 = off[m * os];
                arr = (q & 1) ? A.leaf[m].end : A.leaf[m].begin;
            }
        const int* g = arr + g0;
        const uintptr_t a0 = (uintptr_t)g & ~(uintptr_t)15;
        const unsigned len =
            (lane < 2 * K && nl > 0) ? (unsigned)((((uintptr_t)(g + nl) + 15) & ~(uintptr_t)15) - a0) : 0u;
        int incl = (int)(len >> 2);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const int words = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const int pos = incl - (int)(len >> 2);
        if (lane < 2 * K) {
            const int first = pos + (int)(((uintptr_t)g & 15) >> 2);
            if (q & 1) rawe[l] = first; else rawb[l] = first;
        }
        __syncwarp();  // orders the lanes' writes before lane 0's release on the barrier
        if (lane == 0) sxs_bar_expect(bar, 4u * (unsigned)words);
        __syncwarp();
        if (len > 0u) sxs_bulk_copy(raw + pos, (const void*)a0, len, bar);
    }
    bool copied = true;
    if (fits) copied = __all_sync(0xFFFFFFFFu, sxs_bar_wait(bar));
    unsigned flags = (fits && !copied) ? SXF_TIMEOUT : 0u;
    // 2. coordinate span: first begin and last end of every leaf row
    int xmin = INT_MAX, xmax = INT_MIN;
    if (fits && copied) {
        if (lane < nrows) {
#pragma unroll
            for (int l = 0; l < K; ++l) {
                const int a = off[l * os + lane] - off[l * os], b = off[l * os + lane + 1] - off[l * os];
                if (a >= 0 && a < b && b <= n[l]) {
                    xmin = min(xmin, (int)raw[rawb[l] + a]);
                    xmax = max(xmax, (int)raw[rawe[l] + b - 1]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xFFFFFFFFu, xmin, o));
            xmax = max(xmax, __shfl_xor_sync(0xFFFFFFFFu, xmax, o));
        }
    }
    const bool staged = fits && copied && (E == 0 || (long long)xmax - (long long)xmin < (1ll << SXS_XBITS));
    bool bad = false;
    // 3. keys: the row of interval j is found by walking the row ends from
    //    the previous chunk's row; the contract is checked on the raw values
    if (staged) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int* o = off + l * os;
            const int g0 = o[0];
            const unsigned* rb = raw + rawb[l];
            const unsigned* re = raw + rawe[l];
            unsigned* kk = keys + ks[l];
            int rc = 0;
            for (int j0 = 0; j0 < n[l]; j0 += 32) {
                const int j = j0 + lane;
                int r = rc;
                if (j < n[l]) {
                    while (r + 1 < nrows && o[r + 1] - g0 <= j) ++r;
                    const int b = (int)rb[j], e = (int)re[j];
                    const bool first = j == o[r] - g0;
                    if (!(b < e) || (!first && !((int)re[j - 1] < b)) || o[r] - g0 > j) bad = true;
                    const unsigned rk = (unsigned)r << SXS_XBITS;
                    *(uint2*)(kk + 2 * j) =
                        make_uint2(rk | ((unsigned)(b - xmin) & SXS_XMASK), rk | ((unsigned)(e - xmin) & SXS_XMASK));
                }
                rc = __shfl_sync(0xFFFFFFFFu, r, 31);
            }
            if (lane == 0) {
                kk[2 * n[l]] = SXS_SENTINEL;
                kk[2 * n[l] + 1] = SXS_SENTINEL;
            }
        }
    }
    bad = __any_sync(0xFFFFFFFFu, bad);
    __syncwarp();
    if (bad) flags |= SXF_CONTRACT;
    const bool sweep = staged && !bad && E > 0;
    unsigned* outk = raw;
    int count = 0, total = 0, excl = 0, prov = 0;
    if (sweep) {
        // 4. this lane's piece [klo, khi) and where it starts in every list
        const int nb2 = 2 * nbig;
        unsigned klo = 0u, khi = SXS_SENTINEL;
        if (lane > 0) klo = keys[ksbig + (lane * nb2) / 32];
        if (lane < 31) khi = keys[ksbig + ((lane + 1) * nb2) / 32];
        const int rp = (int)(klo >> SXS_XBITS);
        int pos[K];
#pragma unroll
        for (int l = 0; l < K; ++l) {
            if (lane == 0) {
                pos[l] = 0;
            } else if (l == big) {
                pos[l] = (lane * nb2) / 32;
            } else {
                const int lo = 2 * (off[l * os + rp] - off[l * os]);
                const int hi = 2 * (off[l * os + rp + 1] - off[l * os]);
                pos[l] = lo + sxs_lower_bound(keys + ks[l] + lo, hi - lo, klo);
            }
        }
        unsigned pa[K];
        unsigned h[K];
        unsigned state = 0u;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            pa[l] = sxs_saddr(keys + ks[l] + pos[l]);
            h[l] = keys[ks[l] + pos[l]];
            state |= (unsigned)(pos[l] & 1) << l;
            prov += pos[l];
        }
        // 5. the sweep
        const unsigned tab0 = A.table[0];
        unsigned fprev = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
        const unsigned o0 = sxs_saddr(outk + prov), oend = sxs_saddr(outk + E);
        unsigned oa = o0;
        while (true) {
            unsigned c = h[0];
#pragma unroll
            for (int l = 1; l < K; ++l) c = min(c, h[l]);
            if (c >= khi) break;
#pragma unroll
            for (int l = 0; l < K; ++l) sxs_advance(h[l], pa[l], state, c, 1u << l);
            const unsigned f = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
            sxs_emit(oa, f, fprev, c);
            oa = min(oa, oend);
            fprev = f;
        }
        count = (int)((oa - o0) >> 2);
        int incl = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        excl = incl - count;
        total = min(__shfl_sync(0xFFFFFFFFu, incl, 31), E);
    }
    // fallback tile: one lane per row over global memory
    int lane_count = 0;
    int s_row[K], lim_row[K];
    if (!staged) {
        const bool act = lane < nrows;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int a = act ? off[l * os + lane] : 0;
            const int b = act ? off[l * os + lane + 1] : 0;
            s_row[l] = a;
            lim_row[l] = 2 * (b - a);
        }
        bool fb_bad = false, fb_over = false;
        if (act) lane_count = sx_sweep_table<K, false>(A, s_row, lim_row, nullptr, nullptr, 0, fb_bad, fb_over);
        if (__any_sync(0xFFFFFFFFu, fb_bad)) flags |= SXF_CONTRACT;
        int tot = lane_count;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
        total = 2 * tot;
    }
    // 6. look-back, then pack the output boundaries into the key area
    const int base = sxs_lookback(A, st, tile, total >> 1, flags);
    bool over = false;
    if (staged) {
        unsigned* packed = Wd + (int)RNl;  // the key lists are dead after the sweep
        __syncwarp();
        if (sweep) {
            const int m = min(count, E - excl);
            for (int i = 0; i < m; ++i) packed[excl + i] = outk[prov + i];
        }
        __syncwarp();
        // 7. coalesced output and the tile's row offsets
        const int nint = total >> 1;
        for (int i = lane; i < nint; i += 32) {
            const uint2 kv = *(const uint2*)(packed + 2 * i);
            const long long o = (long long)base + i;
            if (o < A.capacity) {
                A.out_begin[o] = xmin + (int)(kv.x & SXS_XMASK);
                A.out_end[o] = xmin + (int)(kv.y & SXS_XMASK);
            } else {
                over = true;
            }
        }
        for (int r = lane; r < nrows; r += 32) {
            const int pos = sxs_lower_bound(packed, total, (unsigned)(r + 1) << SXS_XBITS);
            A.out_off[r0 + r + 1] = base + (pos >> 1);
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    } else {
        int incl = lane_count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nrows) {
            bool fb_bad = false;
            if (lane_count > 0)
                sx_sweep_table<K, true>(A, s_row, lim_row, A.out_begin, A.out_end, (long long)base + incl - lane_count,
                                        fb_bad, over);
            A.out_off[r0 + lane + 1] = base + incl;
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    }
    (void)over;  // an output beyond the capacity shows in the reported total
    sxs_report(A, tile, tiles, base, total >> 1, flags);
}

// ---------------------------------------------------------------------------
// Warp-tile segmented sweep with 16-bit keys.
//
// In a tile of at most 8 rows whose coordinates span at most 8190, a key
// (row << 13 | (x - xmin)) fits in 16 bits.  The begins of all leaves are
// staged first and the ends after them.  Interval j's key pair is then
// written in place over its staged begin (one 32-bit word holds both keys),
// the staged ends, once checked, become the output area, and the dead key
// lists take the packed output.  A tile so needs 4 bytes of shared memory
// per boundary instead of 8, and twice as many tiles are in flight per SM.
// Everything else is the 32-bit warp kernel above.
// ---------------------------------------------------------------------------
#define SXW16_XBITS 13
#define SXW16_XMASK ((1u << SXW16_XBITS) - 1u)
#define SXW16_SPAN 8190
#define SXW16_SENTINEL 0xFFFFu

// The 16-bit form of sxs_advance: keys are halfwords, pa a byte address.
__device__ __forceinline__ void sxs_advance16(unsigned& h, unsigned& pa, unsigned& state, unsigned c, unsigned bit)
{
    asm volatile(
        "{\n .reg .pred q;\n setp.eq.u32 q, %0, %3;\n @q add.u32 %1, %1, 2;\n"
        " @q xor.b32 %2, %2, %4;\n @q ld.shared.u16 %0, [%1];\n}\n"
        : "+r"(h), "+r"(pa), "+r"(state)
        : "r"(c), "r"(bit));
}

__device__ __forceinline__ void sxs_emit16(unsigned& oa, unsigned f, unsigned fprev, unsigned c)
{
    asm volatile(
        "{\n .reg .pred q;\n setp.ne.u32 q, %1, %2;\n @q st.shared.u16 [%0], %3;\n @q add.u32 %0, %0, 2;\n}\n"
        : "+r"(oa)
        : "r"(f), "r"(fprev), "r"(c)
        : "memory");
}

__device__ __forceinline__ int sxs_lower_bound16(const unsigned short* k, int n, unsigned v)
{
    int pos = 0;
    while (n > 0) {
        const int half = n >> 1;
        if ((unsigned)k[pos + half] < v) {
            pos += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return pos;
}

template <int K>
__global__ void __launch_bounds__(256, K <= 5 ? 5 : 4) sx_wseg16_kernel(SxBoolArgs A, SxSweepState st, int tiles, int cap_words,
                                                        int tr)
{
    extern __shared__ __align__(16) unsigned char sxw_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
    if (blockIdx.x * NW + wid >= tiles) return;  // exactly `tiles` warps take tickets
    unsigned* base_w = (unsigned*)(sxw_smem + (size_t)wid * sxw_slice_bytes(K, tr, cap_words));
    unsigned long long* bar = (unsigned long long*)base_w;
    const int os = tr + 1;
    int* off = (int*)base_w + 2;
    int* rawb = off + os * K;
    int* rawe = rawb + K;
    unsigned* Wd = base_w + sxw_hdr_words(K, tr);

    int tile = 0;
    if (lane == 0) {
        tile = (int)atomicAdd(&st.counters[0], 1u);
        sxs_bar_init(bar);
    }
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
    const int r0 = tile * tr;
    const int nrows = min(tr, A.rows - r0);
    for (int r = lane; r <= nrows; r += 32) {
#pragma unroll
        for (int l = 0; l < K; ++l) off[l * os + r] = A.leaf[l].off[r0 + r];
    }
    __syncwarp();
    // layout (words): the begins of every leaf [0, RB), then the ends [RB, 2 RB)
    int n[K];
    long long RBl = 0, El = 0;
    int big = 0, nbig = -1;
    bool ok = tr <= 8;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        n[l] = off[l * os + nrows] - off[l * os];
        ok = ok && n[l] >= 0;
        RBl += (n[l] + 11) & ~3;  // a copy of at most n + 6 words, 16-byte aligned, then the list's sentinel
        El += 2ll * n[l];
        if (n[l] > nbig) {
            big = l;
            nbig = n[l];
        }
    }
    const bool fits = ok && 2 * RBl <= (long long)cap_words;
    const int E = fits ? (int)El : 0, RB = (int)RBl;
    unsigned* raw = Wd;
    unsigned short* const h16 = (unsigned short*)Wd;  // halfword view of the slice
    // 1. bulk copies: lane q < K copies leaf q's begins, lane K + q its ends
    if (fits) {
        const int q = lane < 2 * K ? lane : 0;
        const bool ends = q >= K;
        const int l = ends ? q - K : q;
        int nl = 0, g0 = 0;
        const int* arr = nullptr;
#pragma unroll
        for (int m = 0; m < K; ++m)
            if (m == l) {
                nl = n[m];
                g0 = off[m * os];
                arr = ends ? A.leaf[m].end : A.leaf[m].begin;
            }
        const int* g = arr + g0;
        const uintptr_t a0 = (uintptr_t)g & ~(uintptr_t)15;
        const unsigned len =
            (lane < 2 * K && nl > 0) ? (unsigned)((((uintptr_t)(g + nl) + 15) & ~(uintptr_t)15) - a0) : 0u;
        // region of this copy: the begins' regions first, then the ends'
        int region = lane < 2 * K ? ((nl + 11) & ~3) : 0;
        int incl = region;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const int pos = incl - region;
        int bytes = (int)len;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xFFFFFFFFu, bytes, o);
        if (lane < 2 * K) {
            const int first = pos + (int)(((uintptr_t)g & 15) >> 2);
            if (ends) rawe[l] = first; else rawb[l] = first;
        }
        __syncwarp();  // orders the lanes' writes before lane 0's release on the barrier
        if (lane == 0) sxs_bar_expect(bar, (unsigned)bytes);
        __syncwarp();
        if (len > 0u) sxs_bulk_copy(raw + pos, (const void*)a0, len, bar);
    }
    bool copied = true;
    if (fits) copied = __all_sync(0xFFFFFFFFu, sxs_bar_wait(bar));
    unsigned flags = (fits && !copied) ? SXF_TIMEOUT : 0u;
    // 2. coordinate span: first begin and last end of every leaf row
    int xmin = INT_MAX, xmax = INT_MIN;
    if (fits && copied) {
        if (lane < nrows) {
#pragma unroll
            for (int l = 0; l < K; ++l) {
                const int a = off[l * os + lane] - off[l * os], b = off[l * os + lane + 1] - off[l * os];
                if (a >= 0 && a < b && b <= n[l]) {
                    xmin = min(xmin, (int)raw[rawb[l] + a]);
                    xmax = max(xmax, (int)raw[rawe[l] + b - 1]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xFFFFFFFFu, xmin, o));
            xmax = max(xmax, __shfl_xor_sync(0xFFFFFFFFu, xmax, o));
        }
    }
    __syncwarp();  // the begins read above are overwritten below
    const bool staged = fits && copied && (E == 0 || (long long)xmax - (long long)xmin <= SXW16_SPAN);
    bool bad = false;
    // 3. keys in place: begin word j becomes interval j's key pair.  The row
    //    of interval j counts the leaf's row starts at or below j (seven
    //    compares against registers, no branch); j starts a row when its row
    //    differs from interval j - 1's (taken from the lane below, or carried
    //    over from the previous chunk).
    if (staged) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int* o = off + l * os;
            const int g0 = o[0];
            int rs[7];
#pragma unroll
            for (int i = 0; i < 7; ++i) rs[i] = i + 1 < nrows ? o[i + 1] - g0 : INT_MAX;
            bool disordered = false;  // row offsets must rise from 0 to n[l]
#pragma unroll
            for (int i = 0; i < 7; ++i)
                disordered = disordered || rs[i] < 0 || (rs[i] != INT_MAX && rs[i] > n[l]) ||
                             (i < 6 && rs[i] > rs[i + 1]);
            if (disordered) bad = true;
            unsigned* rb = raw + rawb[l];
            const unsigned* re = raw + rawe[l];
            int carry_r = -1, carry_e = 0;
            for (int j0 = 0; j0 < n[l]; j0 += 32) {
                const int j = j0 + lane;
                const bool in = j < n[l];
                const int b = in ? (int)rb[j] : 0, e = in ? (int)re[j] : 0;
                int r = 0;
#pragma unroll
                for (int i = 0; i < 7; ++i) r += j >= rs[i] ? 1 : 0;
                int rprev = __shfl_up_sync(0xFFFFFFFFu, r, 1);
                int eprev = __shfl_up_sync(0xFFFFFFFFu, e, 1);
                if (lane == 0) {
                    rprev = carry_r;
                    eprev = carry_e;
                }
                const bool first = r != rprev;
                if (in && (!(b < e) || (!first && !(eprev < b)))) bad = true;
                if (in) {
                    const unsigned rk = (unsigned)r << SXW16_XBITS;
                    rb[j] = (rk | ((unsigned)(b - xmin) & SXW16_XMASK)) |
                            ((rk | ((unsigned)(e - xmin) & SXW16_XMASK)) << 16);
                }
                carry_r = __shfl_sync(0xFFFFFFFFu, r, 31);
                carry_e = __shfl_sync(0xFFFFFFFFu, e, 31);
            }
            if (lane == 0) rb[n[l]] = 0xFFFFFFFFu;  // the list's sentinel
        }
    }
    bad = __any_sync(0xFFFFFFFFu, bad);
    __syncwarp();
    if (bad) flags |= SXF_CONTRACT;
    const bool sweep = staged && !bad && E > 0;
    unsigned short* out16 = h16 + 2 * RB;  // the staged ends, dead after the check
    int count = 0, total = 0, excl = 0, prov = 0;
    if (sweep) {
        // 4. this lane's piece [klo, khi) and where it starts in every list
        const int nb2 = 2 * nbig;
        int bigw = 0;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (l == big) bigw = rawb[l];
        const unsigned short* Lb = h16 + 2 * bigw;
        const unsigned klo = lane > 0 ? (unsigned)Lb[(lane * nb2) / 32] : 0u;
        const unsigned khi = lane < 31 ? (unsigned)Lb[((lane + 1) * nb2) / 32] : SXW16_SENTINEL;
        const int rp = (int)(klo >> SXW16_XBITS);
        unsigned pa[K];
        unsigned h[K];
        unsigned state = 0u;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const unsigned short* Ll = h16 + 2 * rawb[l];
            int pos;
            if (lane == 0) {
                pos = 0;
            } else if (l == big) {
                pos = (lane * nb2) / 32;
            } else {
                const int lo = 2 * (off[l * os + rp] - off[l * os]);
                const int hi = 2 * (off[l * os + rp + 1] - off[l * os]);
                pos = lo + sxs_lower_bound16(Ll + lo, hi - lo, klo);
            }
            pa[l] = sxs_saddr(Ll + pos);
            h[l] = Ll[pos];
            state |= (unsigned)(pos & 1) << l;
            prov += pos;
        }
        // 5. the sweep
        const unsigned tab0 = A.table[0];
        unsigned fprev = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
        const unsigned o0 = sxs_saddr(out16 + prov), oend = sxs_saddr(out16 + E);
        unsigned oa = o0;
        while (true) {
            unsigned c = h[0];
#pragma unroll
            for (int l = 1; l < K; ++l) c = min(c, h[l]);
            if (c >= khi) break;
#pragma unroll
            for (int l = 0; l < K; ++l) sxs_advance16(h[l], pa[l], state, c, 1u << l);
            const unsigned f = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
            sxs_emit16(oa, f, fprev, c);
            oa = min(oa, oend);
            fprev = f;
        }
        count = (int)((oa - o0) >> 1);
        int incl = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        excl = incl - count;
        total = min(__shfl_sync(0xFFFFFFFFu, incl, 31), E);
    }
    // fallback tile: one lane per row over global memory
    int lane_count = 0;
    int s_row[K], lim_row[K];
    if (!staged) {
        const bool act = lane < nrows;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const int a = act ? off[l * os + lane] : 0;
            const int b = act ? off[l * os + lane + 1] : 0;
            s_row[l] = a;
            lim_row[l] = 2 * (b - a);
        }
        bool fb_bad = false, fb_over = false;
        if (act) lane_count = sx_sweep_table<K, false>(A, s_row, lim_row, nullptr, nullptr, 0, fb_bad, fb_over);
        if (__any_sync(0xFFFFFFFFu, fb_bad)) flags |= SXF_CONTRACT;
        int tot = lane_count;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
        total = 2 * tot;
    }
    // 6. look-back, then pack the output boundaries over the dead key lists
    const int base = sxs_lookback(A, st, tile, total >> 1, flags);
    bool over = false;
    if (staged) {
        unsigned short* packed = h16;
        __syncwarp();
        if (sweep) {
            const int m = min(count, E - excl);
            for (int i = 0; i < m; ++i) packed[excl + i] = out16[prov + i];
        }
        __syncwarp();
        // 7. coalesced output and the tile's row offsets
        const int nint = total >> 1;
        const unsigned* pw = (const unsigned*)packed;
        for (int i = lane; i < nint; i += 32) {
            const unsigned kv = pw[i];
            const long long o = (long long)base + i;
            if (o < A.capacity) {
                A.out_begin[o] = xmin + (int)(kv & SXW16_XMASK);
                A.out_end[o] = xmin + (int)((kv >> 16) & SXW16_XMASK);
            } else {
                over = true;
            }
        }
        for (int r = lane; r < nrows; r += 32) {
            const int pos = sxs_lower_bound16(packed, total, (unsigned)(r + 1) << SXW16_XBITS);
            A.out_off[r0 + r + 1] = base + (pos >> 1);
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    } else {
        int incl = lane_count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nrows) {
            bool fb_bad = false;
            if (lane_count > 0)
                sx_sweep_table<K, true>(A, s_row, lim_row, A.out_begin, A.out_end, (long long)base + incl - lane_count,
                                        fb_bad, over);
            A.out_off[r0 + lane + 1] = base + incl;
        }
        if (tile == 0 && lane == 0) A.out_off[0] = 0;
    }
    (void)over;  // an output beyond the capacity shows in the reported total
    sxs_report(A, tile, tiles, base, total >> 1, flags);
}

// ---------------------------------------------------------------------------
// Row-lane sweep with 16-bit coordinates (sx_tuning kernel 7).
//
// A warp owns a tile of 32 aligned rows and lane r sweeps row r, so a step
// needs no combined (row, x) keys, no piece search and no search for the
// row offsets of the output.
//
// Staging.  One bulk copy per leaf array (begins, ends) into the warp's
// slice of shared memory, above a gap; then interval j of leaf l becomes the
// word (b - xmin) | (e - xmin) << 16 in leaf l's pair list, which holds one
// spare word after every non-empty row: word j of row q-th non-empty row
// goes to j + q.  The spare word holds 0xFFFF in its low half, so a lane's
// walk (b0 e0 b1 e1 ... as halfwords) stops at its row's end with no
// per-step limit test, and rows whose lengths are multiples of 32 words
// (a 64-pixel checkerboard on 4096 columns) no longer put every lane of a
// step on the same shared-memory bank.  The pair lists grow into the gap
// while the raw copies above are read: a pair is written at most 31 + 25 l
// words above its own raw begin's distance from the slice start, below every
// raw word not yet read.  xmin is the tile's smallest first begin and xmax
// its largest last end; a tile with xmax - xmin > 65534 takes the
// global-memory sweep, and a coordinate outside [xmin, xmin + 65534] in a
// narrower tile breaks the contract (on canonical rows every coordinate lies
// between its row's first begin and last end).
//
// Step: the smallest head c; each leaf whose head equals c toggles its state
// bit and loads its next halfword (predicated, no divergence); f(state) from
// the truth table; a change of f stores c.  On canonical rows successive c
// rise strictly, so one compare per step checks the contract (non-empty,
// sorted, non-touching intervals).  Row r's output halfwords go to an area
// as large as its input plus one word (the dead raw copies).  A scan of the
// per-row counts gives the row offsets, the look-back the tile's base; the
// lanes pack their output words over the dead pair lists and the warp writes
// them out coalesced.  Every wait is bounded.
// ---------------------------------------------------------------------------
#define SXR_TR 32
#define SXR_SPAN 65534
#define SXR_SENTINEL 0xFFFFu
#define SXR_HDR_WORDS 4

// Words below the raw copies into which the padded pair lists grow, for k
// leaves and tiles of tr rows.  Leaf l's list starts at most l (tr - 7) words
// further from the slice than its raw begins (each list holds its n pairs
// plus tr + 1 spare words, each raw region at least n + 8 words), and a pair
// lands at most tr - 1 words above its own index: (k - 1)(tr - 7) + tr
// keeps every pair below the raw words not yet read.  The output areas
// (n + tr words in all, after the lists) must also end inside the raw
// region's 2 (n + 8 k) words: k (tr + 1) + tr - 16 k.
__host__ __device__ inline int sxr_gap_words(int k, int tr)
{
    const int lists = (k - 1) * (tr - 7) + tr;
    const int outputs = k * (tr + 1) + tr - 16 * k;
    return ((lists > outputs ? lists : outputs) + 4 + 3) & ~3;
}

__host__ __device__ inline size_t sxr_slice_bytes(int cap_words)
{
    return 4u * (size_t)(SXR_HDR_WORDS + ((cap_words + 3) & ~3));
}

// One leaf of a row-lane step: when the head h equals the step's key c, load
// the next halfword from pa + 2 (the load does not wait for the address
// update), advance pa and toggle the leaf's state bit.  Predicated.
__device__ __forceinline__ void sxr_advance16(unsigned& h, unsigned& pa, unsigned& state, unsigned c, unsigned bit)
{
    asm volatile(
        "{\n .reg .pred q;\n setp.eq.u32 q, %0, %3;\n @q ld.shared.u16 %0, [%1+2];\n @q add.u32 %1, %1, 2;\n"
        " @q xor.b32 %2, %2, %4;\n}\n"
        : "+r"(h), "+r"(pa), "+r"(state)
        : "r"(c), "r"(bit));
}

template <int K>
__device__ __forceinline__ unsigned sxr_min_head(const unsigned* h)
{
    unsigned c = h[0];
    int l = 1;
#pragma unroll
    for (; l + 1 < K; l += 2) c = __vimin3_u32(c, h[l], h[l + 1]);
#pragma unroll
    for (; l < K; ++l) c = min(c, h[l]);
    return c;
}

// A tile of 32 / LPR rows: lanes LPR r .. LPR r + LPR - 1 sweep row r in
// pieces [p_i, p_{i+1}) of its keys, the pivots p_i being halfwords of the
// row's longest leaf at positions i m / LPR (m its boundaries).  A piece
// starts in every other leaf at the first key not below p_i (a binary search
// within the row) with the parity of that position as the leaf's state bit,
// and writes at most as many outputs as it reads inputs, so piece i's output
// area starts where the inputs of the pieces before it end.  Consecutive
// pieces must meet: each piece's end positions are checked against the next
// piece's start positions (with the per-piece rising keys, that checks the
// contract across pieces).
template <int K, int LPR>
__global__ void __launch_bounds__(256) sx_rlane16_kernel(SxBoolArgs A, SxSweepState st, int tiles, int cap_words)
{
    extern __shared__ __align__(16) unsigned char sxr_smem[];
    constexpr int TR = SXR_TR / LPR;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
    if (blockIdx.x * NW + wid >= tiles) return;  // exactly `tiles` warps take tickets
    unsigned* base_w = (unsigned*)(sxr_smem + (size_t)wid * sxr_slice_bytes(cap_words));
    unsigned long long* bar = (unsigned long long*)base_w;
    unsigned* const W = base_w + SXR_HDR_WORDS;  // pair lists, then the output areas
    unsigned short* const h16 = (unsigned short*)W;
    const int gap = sxr_gap_words(K, TR);
    unsigned* const raw = W + gap;  // the bulk copies
    const int row = lane / LPR, piece = lane % LPR;
    const int first_lane = row * LPR;

    int tile = 0;
    if (lane == 0) {
        tile = (int)atomicAdd(&st.counters[0], 1u);
        sxs_bar_init(bar);
    }
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
    const int r0 = tile * TR;
    const int nrows = min(TR, A.rows - r0);
    const bool act = row < nrows;
    // this lane's row in every leaf, relative to the tile's first interval
    int lo[K], hi[K], n[K], g0[K];
    bool ok = true;
    long long RBl = 0, PBl = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        const int a = A.leaf[l].off[r0 + min(row, nrows)];
        const int b = A.leaf[l].off[r0 + min(row + 1, nrows)];
        g0[l] = __shfl_sync(0xFFFFFFFFu, a, 0);
        n[l] = __shfl_sync(0xFFFFFFFFu, b, (nrows - 1) * LPR) - g0[l];
        lo[l] = act ? a - g0[l] : n[l];
        hi[l] = act ? b - g0[l] : n[l];
        ok = ok && lo[l] >= 0 && lo[l] <= hi[l] && hi[l] <= n[l];
        RBl += (long long)((n[l] + 11) & ~3);
        PBl += (long long)n[l] + TR + 1;
    }
    ok = __all_sync(0xFFFFFFFFu, ok);  // row offsets must rise through the tile
    const bool fits = ok && gap + 2 * RBl <= (long long)cap_words;
    const int OA = (int)PBl;  // output areas start after the pair lists
    unsigned flags = ok ? 0u : SXF_CONTRACT;
    // 1. bulk copies: lane q < K copies leaf q's begins, lane K + q its ends
    int rb[K], re[K];
#pragma unroll
    for (int l = 0; l < K; ++l) rb[l] = re[l] = 0;
    bool copied = true;
    if (fits) {
        const int q = lane < 2 * K ? lane : 0;
        const bool ends = q >= K;
        const int lq = ends ? q - K : q;
        int nl = 0, gq = 0;
        const int* arr = nullptr;
#pragma unroll
        for (int m = 0; m < K; ++m)
            if (m == lq) {
                nl = n[m];
                gq = g0[m];
                arr = ends ? A.leaf[m].end : A.leaf[m].begin;
            }
        const int* g = arr + gq;
        const uintptr_t a0 = (uintptr_t)g & ~(uintptr_t)15;
        const unsigned len =
            (lane < 2 * K && nl > 0) ? (unsigned)((((uintptr_t)(g + nl) + 15) & ~(uintptr_t)15) - a0) : 0u;
        const int region = lane < 2 * K ? ((nl + 11) & ~3) : 0;  // at most n + 6 copied words
        int incl = region;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const int pos = incl - region;
        int bytes = (int)len;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xFFFFFFFFu, bytes, o);
        const int first = pos + (int)(((uintptr_t)g & 15) >> 2);
#pragma unroll
        for (int l = 0; l < K; ++l) {
            rb[l] = __shfl_sync(0xFFFFFFFFu, first, l);
            re[l] = __shfl_sync(0xFFFFFFFFu, first, K + l);
        }
        __syncwarp();
        if (lane == 0) sxs_bar_expect(bar, (unsigned)bytes);
        __syncwarp();
        if (len > 0u) sxs_bulk_copy(raw + pos, (const void*)a0, len, bar);
        copied = __all_sync(0xFFFFFFFFu, sxs_bar_wait(bar));
        if (!copied) flags |= SXF_TIMEOUT;
    }
    // 2. the tile's coordinate range: first begin and last end of every row
    int xmin = INT_MAX, xmax = INT_MIN;
    if (fits && copied) {
        if (act && piece == 0) {
#pragma unroll
            for (int l = 0; l < K; ++l)
                if (lo[l] < hi[l]) {
                    xmin = min(xmin, (int)raw[rb[l] + lo[l]]);
                    xmax = max(xmax, (int)raw[re[l] + hi[l] - 1]);
                }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xFFFFFFFFu, xmin, o));
            xmax = max(xmax, __shfl_xor_sync(0xFFFFFFFFu, xmax, o));
        }
    }
    const bool staged = fits && copied && (xmin > xmax || (long long)xmax - (long long)xmin <= SXR_SPAN);
    bool bad = false;
    // 3. padded pair lists, leaf by leaf; qr[l] is this row's rank among the leaf's non-empty rows
    int qr[K], pb[K];
    {
        int p = 0;
        const unsigned below = (1u << first_lane) - 1u;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const bool ne = act && piece == 0 && lo[l] < hi[l];
            qr[l] = __popc(__ballot_sync(0xFFFFFFFFu, ne) & below);
            pb[l] = p;
            p += n[l] + TR + 1;
        }
    }
    if (staged) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const unsigned* src_b = raw + rb[l];
            const unsigned* src_e = raw + re[l];
            unsigned* dst = W + pb[l];
            const bool ne = act && piece == 0 && lo[l] < hi[l];
            int qbase = 0;  // non-empty rows starting before the chunk
            for (int j0 = 0; j0 < n[l]; j0 += 32) {
                const int j = j0 + lane;
                const unsigned d = (unsigned)(lo[l] - j0);
                const unsigned starts = __reduce_or_sync(0xFFFFFFFFu, (ne && d < 32u) ? 1u << d : 0u);
                const int q = qbase + __popc(starts & (0xFFFFFFFFu >> (31 - lane))) - 1;
                unsigned word = 0u;
                if (j < n[l]) {
                    const unsigned ub = src_b[j] - (unsigned)xmin, ue = src_e[j] - (unsigned)xmin;
                    if (max(ub, ue) > (unsigned)SXR_SPAN) bad = true;
                    word = __byte_perm(ub, ue, 0x5410);
                }
                __syncwarp();  // the chunk's raw words are read before any pair lands on them
                if (j < n[l]) dst[j + q] = word;
                qbase += __popc(starts);
            }
        }
    }
    __syncwarp();
    if (staged && act && piece == 0) {
#pragma unroll
        for (int l = 0; l < K; ++l)  // the row's spare word
            if (lo[l] < hi[l]) h16[2 * (pb[l] + hi[l] + qr[l])] = (unsigned short)SXR_SENTINEL;
    }
    __syncwarp();
    // this row's output area: as much as its input, plus one word
    int cap_r = 0;
#pragma unroll
    for (int l = 0; l < K; ++l) cap_r += hi[l] - lo[l];
    int cap_excl = piece == 0 ? cap_r : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, cap_excl, o);
        if (lane >= o) cap_excl += y;
    }
    cap_excl = cap_excl - (piece == 0 ? cap_r : 0) + row;
    cap_excl = __shfl_sync(0xFFFFFFFFu, cap_excl, first_lane);
    int khw = 0, prov = 0;  // output halfwords of this piece; inputs of the row's earlier pieces
    unsigned sa[K], pa[K], h[K];
#pragma unroll
    for (int l = 0; l < K; ++l) sa[l] = pa[l] = h[l] = 0u;
    if (staged && act) {
        // 4. this piece's start in every leaf
        int big = 0, nbig = -1;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (hi[l] - lo[l] > nbig) {
                big = l;
                nbig = hi[l] - lo[l];
            }
        const int m = 2 * nbig;
        int bigw = 0;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (l == big) bigw = pb[l] + lo[l] + qr[l];
        const unsigned short* Lb = h16 + 2 * bigw;
        unsigned klo = 0u, khi = SXR_SENTINEL;
        if (LPR > 1) {
            klo = piece == 0 ? 0u : (m > 0 ? (unsigned)Lb[(piece * m) / LPR] : SXR_SENTINEL);
            khi = piece == LPR - 1 ? SXR_SENTINEL : (m > 0 ? (unsigned)Lb[((piece + 1) * m) / LPR] : SXR_SENTINEL);
        }
        unsigned state = 0u;
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const unsigned short* Ll = h16 + 2 * (pb[l] + lo[l] + qr[l]);
            const int cnt = 2 * (hi[l] - lo[l]);
            int pos = 0;
            if (LPR > 1 && piece > 0) pos = l == big ? (piece * m) / LPR : sxs_lower_bound16(Ll, cnt, klo);
            if (cnt == 0) pos = 0;
            sa[l] = pa[l] = sxs_saddr(Ll + pos);
            h[l] = pos < cnt ? (unsigned)Ll[pos] : SXR_SENTINEL;
            state |= (unsigned)(pos & 1) << l;
            prov += pos;
        }
        // 5. the sweep of this piece
        const unsigned tab0 = A.table[0];
        unsigned fprev = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
        int cprev = -1;
        const unsigned o0 = sxs_saddr(h16 + 2 * (OA + cap_excl) + prov);
        unsigned oa = o0;
        unsigned c = sxr_min_head<K>(h);
        while (c < khi) {
            bad = bad || (int)c <= cprev;
            cprev = (int)c;
#pragma unroll
            for (int l = 0; l < K; ++l) sxr_advance16(h[l], pa[l], state, c, 1u << l);
            const unsigned f = K <= 5 ? (tab0 >> state) & 1u : (A.table[state >> 5] >> (state & 31u)) & 1u;
            sxs_emit16(oa, f, fprev, c);
            fprev = f;
            c = sxr_min_head<K>(h);
        }
        khw = (int)((oa - o0) >> 1);
    }
    if (LPR > 1) {
        // consecutive pieces of a row meet: this piece ends where the next one starts
#pragma unroll
        for (int l = 0; l < K; ++l) {
            const unsigned nxt = __shfl_down_sync(0xFFFFFFFFu, sa[l], 1);
            if (staged && act && piece < LPR - 1 && pa[l] != nxt) bad = true;
        }
    }
    if (__any_sync(0xFFFFFFFFu, bad)) {
        flags |= SXF_CONTRACT;
        khw = 0;  // pieces may overlap on such input: the tile writes nothing
    }
    // fallback tile: one lane per row over global memory
    int s_row[K], lim_row[K];
    int nint = 0;
    if (ok && !staged) {
#pragma unroll
        for (int l = 0; l < K; ++l) {
            s_row[l] = g0[l] + lo[l];
            lim_row[l] = 2 * (hi[l] - lo[l]);
        }
        bool fb_bad = false, fb_over = false;
        if (act && piece == 0) nint = sx_sweep_table<K, false>(A, s_row, lim_row, nullptr, nullptr, 0, fb_bad, fb_over);
        if (__any_sync(0xFFFFFFFFu, fb_bad)) flags |= SXF_CONTRACT;
        khw = 2 * nint;
    }
    int incl = khw;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - khw;  // halfwords of the pieces before this one
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31) >> 1;
    // 6. look-back, then pack the output halfwords over the dead pair lists
    const int base = sxs_lookback(A, st, tile, total, flags);
    bool over = false;
    if (staged) {
        __syncwarp();  // every lane's sweep has read its pairs
        if (act) {
            const unsigned short* src = h16 + 2 * (OA + cap_excl) + prov;
            for (int i = 0; i < khw; ++i) h16[excl + i] = src[i];
        }
        __syncwarp();
        const unsigned* pw = W;
        for (int i = lane; i < total; i += 32) {
            const unsigned kv = pw[i];
            const long long o = (long long)base + i;
            if (o < A.capacity) {
                A.out_begin[o] = xmin + (int)(kv & 0xFFFFu);
                A.out_end[o] = xmin + (int)(kv >> 16);
            } else {
                over = true;
            }
        }
    } else if (ok && act && piece == 0 && nint > 0) {
        bool fb_bad = false;
        sx_sweep_table<K, true>(A, s_row, lim_row, A.out_begin, A.out_end, (long long)base + (excl >> 1), fb_bad, over);
    }
    if (act && piece == LPR - 1) A.out_off[r0 + row + 1] = base + (incl >> 1);
    if (tile == 0 && lane == 0) A.out_off[0] = 0;
    (void)over;  // an output beyond the capacity shows in the reported total
    sxs_report(A, tile, tiles, base, total, flags);
}

size_t sx_sweep_state_bytes(long long tiles)
{
    const long long groups = (tiles + SX_GROUP - 1) / SX_GROUP;
    return a256(16) + a256((size_t)tiles * 8) + a256((size_t)groups * 8) + a256((size_t)groups * 4) +
           a256((size_t)groups * 4);
}

long long sx_sweep_tiles(int rows) { return ((long long)rows + 31) / 32; }

static SxSweepState sx_sweep_state(void* ws, long long tiles)
{
    const long long groups = (tiles + SX_GROUP - 1) / SX_GROUP;
    char* p = (char*)ws;
    SxSweepState st;
    st.counters = (unsigned*)p;
    p += a256(16);
    st.tile_status = (unsigned long long*)p;
    p += a256((size_t)tiles * 8);
    st.group_status = (unsigned long long*)p;
    p += a256((size_t)groups * 8);
    st.group_sum = (int*)p;
    p += a256((size_t)groups * 4);
    st.group_count = (unsigned*)p;
    return st;
}

template <int K, int MODE>
static cudaError_t sx_sweep_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, cudaStream_t stream)
{
    // Residency cap through unused dynamic shared memory.  Fewer resident
    // rows keep every lane's boundary streams inside L1.
    int pad = 0;
    if (A.tune_blocks_per_sm > 0) {
        pad = 233472 / A.tune_blocks_per_sm - 1024 - 256;
        if (pad > 232448) pad = 232448;
        if (pad < 0) pad = 0;
        static int configured = 0;
        if (pad > configured) {
            cudaError_t err = cudaFuncSetAttribute(sx_sweep_kernel<K, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   pad);
            if (err != cudaSuccess) return err;
            configured = pad;
        }
    }
    const int blocks = (tiles + SX_SWEEP_WARPS - 1) / SX_SWEEP_WARPS;
    sx_sweep_kernel<K, MODE><<<blocks, 32 * SX_SWEEP_WARPS, pad, stream>>>(A, st, tiles);
    return cudaGetLastError();
}

template <int K>
static cudaError_t sx_sweep_smem_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int ecap,
                                          cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    const int smem = SX_SMEM_WARPS * sx_smem_warp_ints(ecap) * (int)sizeof(int);
    if (smem > configured) {
        cudaError_t err = cudaFuncSetAttribute(sx_sweep_smem_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (err != cudaSuccess) return err;
        configured = smem;
    }
    const int blocks = (tiles + SX_SMEM_WARPS - 1) / SX_SMEM_WARPS;
    sx_sweep_smem_kernel<K><<<blocks, 32 * SX_SMEM_WARPS, smem, stream>>>(A, st, tiles, ecap);
    return cudaGetLastError();
}

// Staging capacity per warp: 1.25x the average tile size, in [256, 3584]
// elements.  Tiles above it take the global-memory sweep.  3584 keeps four
// warps' staging under the 227 KB per-block limit.
static int sx_pick_ecap(long long elems, long long tiles)
{
    long long avg = tiles > 0 ? (elems + tiles - 1) / tiles : 0;
    long long e = (avg * 5) / 4;
    e = (e + 63) / 64 * 64;
    if (e < 256) e = 256;
    if (e > 3584) e = 3584;
    return (int)e;
}


template <int K>
static cudaError_t sx_merge_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_bytes,
                                     cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    if (cap_bytes > configured) {
        cudaError_t err =
            cudaFuncSetAttribute(sx_merge_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap_bytes);
        if (err != cudaSuccess) return err;
        configured = cap_bytes;
    }
    sx_merge_kernel<K><<<tiles, SXM_THREADS, cap_bytes, stream>>>(A, st, tiles, cap_bytes);
    return cudaGetLastError();
}

template <int K>
static cudaError_t sx_seg_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_keys, int threads,
                                   int tr, cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    const int bytes = 4 * cap_keys;
    if (bytes > configured) {
        cudaError_t err = cudaFuncSetAttribute(sx_seg_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (err != cudaSuccess) return err;
        configured = bytes;
    }
    sx_seg_kernel<K><<<tiles, threads, bytes, stream>>>(A, st, tiles, cap_keys, tr);
    return cudaGetLastError();
}

template <int K>
static cudaError_t sx_wseg_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_words, int warps,
                                    int tr, cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    const int bytes = warps * (int)sxw_slice_bytes(K, tr, cap_words);
    if (bytes > configured) {
        cudaError_t err = cudaFuncSetAttribute(sx_wseg_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (err != cudaSuccess) return err;
        configured = bytes;
    }
    const int blocks = (tiles + warps - 1) / warps;
    sx_wseg_kernel<K><<<blocks, 32 * warps, bytes, stream>>>(A, st, tiles, cap_words, tr);
    return cudaGetLastError();
}

template <int K>
static cudaError_t sx_wseg16_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_words,
                                      int warps, int tr, cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    const int bytes = warps * (int)sxw_slice_bytes(K, tr, cap_words);
    if (bytes > configured) {
        cudaError_t err =
            cudaFuncSetAttribute(sx_wseg16_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (err != cudaSuccess) return err;
        configured = bytes;
    }
    const int blocks = (tiles + warps - 1) / warps;
    sx_wseg16_kernel<K><<<blocks, 32 * warps, bytes, stream>>>(A, st, tiles, cap_words, tr);
    return cudaGetLastError();
}

template <int K, int LPR>
static cudaError_t sx_rlane16_launch_kl(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_words,
                                        int warps, cudaStream_t stream)
{
    static int configured = 0;  // largest dynamic shared memory set for this instantiation
    const int bytes = warps * (int)sxr_slice_bytes(cap_words);
    if (bytes > configured) {
        cudaError_t err =
            cudaFuncSetAttribute(sx_rlane16_kernel<K, LPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (err != cudaSuccess) return err;
        configured = bytes;
    }
    const int blocks = (tiles + warps - 1) / warps;
    sx_rlane16_kernel<K, LPR><<<blocks, 32 * warps, bytes, stream>>>(A, st, tiles, cap_words);
    return cudaGetLastError();
}

// Lanes per row from the tile height: 32 rows one lane each, 16 rows two, 8 rows four.
template <int K>
static cudaError_t sx_rlane16_launch_k(const SxBoolArgs& A, const SxSweepState& st, int tiles, int cap_words,
                                       int warps, int tr, cudaStream_t stream)
{
    if (tr == 8) return sx_rlane16_launch_kl<K, 4>(A, st, tiles, cap_words, warps, stream);
    if (tr == 16) return sx_rlane16_launch_kl<K, 2>(A, st, tiles, cap_words, warps, stream);
    return sx_rlane16_launch_kl<K, 1>(A, st, tiles, cap_words, warps, stream);
}

// Segmented sweep shape: `keys` boundaries per tile (0: 1.25x the average
// plus slack), stored twice (lists and output area), at most 200 KiB per
// block; `warps` per block (0: about 48 boundaries per thread).
static void sx_seg_shape(long long leaf_intervals, long long tiles, int keys, int warps, int k, int* cap_keys,
                         int* threads)
{
    const long long avg = tiles > 0 ? (2 * leaf_intervals + tiles - 1) / tiles : 0;
    long long e = keys > 0 ? keys : avg + avg / 4 + 256;
    long long c = 2 * e + e / 32 + 26 * k + 64;
    c = (c + 255) / 256 * 256;
    if (c > 51200) c = 51200;
    *cap_keys = (int)c;
    int w = warps;
    if (w <= 0) {
        w = (int)((avg + 1535) / 1536);
        if (w < 1) w = 1;
    }
    if (w > SXS_MAX_THREADS / 32) w = SXS_MAX_THREADS / 32;
    *threads = 32 * w;
}

// Shared memory per tile: two (or three) key buffers of 32-bit keys with
// room for 1.25x the average tile plus slack, in steps of 2 KiB, between
// 8 KiB and 96 KiB.  `requested` (keys) overrides the average.
static int sx_merge_cap(long long leaf_intervals, long long tiles, int requested, int nbuf)
{
    long long keys;
    if (requested > 0) {
        keys = requested;
    } else {
        const long long avg = tiles > 0 ? (2 * leaf_intervals + tiles - 1) / tiles : 0;
        keys = avg + avg / 4 + 256;
    }
    long long bytes = 4ll * nbuf * keys;
    bytes = (bytes + 2047) / 2048 * 2048;
    if (bytes < 8192) bytes = 8192;
    if (bytes > 98304) bytes = 98304;
    return (int)bytes;
}

cudaError_t sx_sweep_launch(const SxBoolArgs& A, bool union_mode, void* workspace, size_t workspace_bytes,
                            cudaStream_t stream)
{
    if (A.rows <= 0) return cudaSuccess;
    // The segmented sweep takes tiles of 16 rows when the workspace holds
    // their look-back state (smaller tiles keep more blocks resident), else 32.
    const bool seg = !union_mode && (A.tune_kernel == 0 || A.tune_kernel >= 4);
    int tr = 32;
    if (seg) {
        tr = A.tune_tile_rows > 0 ? A.tune_tile_rows : (A.tune_kernel == 4 ? 32 : 8);
        if (A.tune_kernel == 6 && tr > 8) tr = 8;  // 16-bit keys hold 3 row bits
        if (A.tune_kernel == 7) tr = A.tune_tile_rows == 8 || A.tune_tile_rows == 32 ? A.tune_tile_rows : 16;
        if (sx_sweep_state_bytes(((long long)A.rows + tr - 1) / tr) > workspace_bytes) tr = 32;
    }
    const long long tiles = ((long long)A.rows + tr - 1) / tr;
    if (sx_sweep_state_bytes(tiles) > workspace_bytes) return cudaErrorInvalidValue;
    // The look-back state must start cleared; the workspace may hold other scratch.
    cudaError_t err = cudaMemsetAsync(workspace, 0, sx_sweep_state_bytes(tiles), stream);
    if (err != cudaSuccess) return err;
    SxSweepState st = sx_sweep_state(workspace, tiles);
    const int t = (int)tiles;
    if (union_mode) {
        switch (A.k) {
            case 1: return sx_sweep_launch_k<1, MODE_UNION>(A, st, t, stream);
            case 2: return sx_sweep_launch_k<2, MODE_UNION>(A, st, t, stream);
            case 3: return sx_sweep_launch_k<3, MODE_UNION>(A, st, t, stream);
            case 4: return sx_sweep_launch_k<4, MODE_UNION>(A, st, t, stream);
            case 5: return sx_sweep_launch_k<5, MODE_UNION>(A, st, t, stream);
            case 6: return sx_sweep_launch_k<6, MODE_UNION>(A, st, t, stream);
            case 7: return sx_sweep_launch_k<7, MODE_UNION>(A, st, t, stream);
            case 8: return sx_sweep_launch_k<8, MODE_UNION>(A, st, t, stream);
            case 9: return sx_sweep_launch_k<9, MODE_UNION>(A, st, t, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    // Automatic choice: staged sweep for light tiles (it keeps many warps
    // resident), global sweep with a residency cap of 3 blocks per SM for
    // heavy tiles (measured best on the 4096x4096 shape expression).
    SxBoolArgs B = A;
    if (B.tune_kernel == 0) B.tune_kernel = 5;
    if (B.tune_kernel == 7) {
        // words per warp: the staged begins and ends (later pairs and outputs) of the largest tile
        const long long avg = (2 * A.capacity + tiles - 1) / tiles;
        const long long e = A.tune_staging_cap > 0 ? A.tune_staging_cap : avg + avg / 4 + 64;
        long long words = e + 22 * A.k + 8 + sxr_gap_words(A.k, tr);
        const long long slice = 4 * (SXR_HDR_WORDS + words);
        // about 25 KiB per block: small blocks pack the SM's shared memory closely and retire independently
        int warps = A.tune_warps > 0 ? A.tune_warps : (int)((25 * 1024) / slice);
        if (warps > 4 && A.tune_warps <= 0) warps = 4;
        if (warps < 1) warps = 1;
        const long long limit = (200 * 1024) / warps / 4 - SXR_HDR_WORDS;
        if (words > limit) words = limit;
        const int cw = (int)words;
        switch (A.k) {
            case 1: return sx_rlane16_launch_k<1>(A, st, t, cw, warps, tr, stream);
            case 2: return sx_rlane16_launch_k<2>(A, st, t, cw, warps, tr, stream);
            case 3: return sx_rlane16_launch_k<3>(A, st, t, cw, warps, tr, stream);
            case 4: return sx_rlane16_launch_k<4>(A, st, t, cw, warps, tr, stream);
            case 5: return sx_rlane16_launch_k<5>(A, st, t, cw, warps, tr, stream);
            case 6: return sx_rlane16_launch_k<6>(A, st, t, cw, warps, tr, stream);
            case 7: return sx_rlane16_launch_k<7>(A, st, t, cw, warps, tr, stream);
            case 8: return sx_rlane16_launch_k<8>(A, st, t, cw, warps, tr, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (B.tune_kernel == 6 && tr <= 8) {
        // words per warp: the staged begins and ends (later keys and outputs) of the largest tile
        const long long avg = (2 * A.capacity + tiles - 1) / tiles;
        const long long e = A.tune_staging_cap > 0 ? A.tune_staging_cap : avg + avg / 4 + 64;
        long long words = e + 22 * A.k + 8;
        const long long room = (200 * 1024) / 4 - sxw_hdr_words(A.k, tr);
        int warps = A.tune_warps > 0 ? A.tune_warps : (int)(room / (words + sxw_hdr_words(A.k, tr)));
        if (warps > 4 && A.tune_warps <= 0) warps = 4;
        if (warps < 1) warps = 1;
        const long long limit = (200 * 1024) / warps / 4 - sxw_hdr_words(A.k, tr);
        if (words > limit) words = limit;
        const int cw = (int)words;
        switch (A.k) {
            case 1: return sx_wseg16_launch_k<1>(A, st, t, cw, warps, tr, stream);
            case 2: return sx_wseg16_launch_k<2>(A, st, t, cw, warps, tr, stream);
            case 3: return sx_wseg16_launch_k<3>(A, st, t, cw, warps, tr, stream);
            case 4: return sx_wseg16_launch_k<4>(A, st, t, cw, warps, tr, stream);
            case 5: return sx_wseg16_launch_k<5>(A, st, t, cw, warps, tr, stream);
            case 6: return sx_wseg16_launch_k<6>(A, st, t, cw, warps, tr, stream);
            case 7: return sx_wseg16_launch_k<7>(A, st, t, cw, warps, tr, stream);
            case 8: return sx_wseg16_launch_k<8>(A, st, t, cw, warps, tr, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (B.tune_kernel == 6) B.tune_kernel = 5;  // tiles above 8 rows: 32-bit keys
    if (B.tune_kernel == 5) {
        // words per warp: the copies (or outputs) and the key lists of the largest tile
        const long long avg = (2 * A.capacity + tiles - 1) / tiles;
        long long e = A.tune_staging_cap > 0 ? A.tune_staging_cap : avg + avg / 4 + 64;
        long long words = 2 * e + 26 * A.k + 16;
        // four warps per block unless a slice that large allows fewer (200 KiB per block)
        const long long room = (200 * 1024) / 4 - sxw_hdr_words(A.k, tr);
        int warps = A.tune_warps > 0 ? A.tune_warps : (int)(room / (words + sxw_hdr_words(A.k, tr)));
        if (warps > 4 && A.tune_warps <= 0) warps = 4;
        if (warps < 1) warps = 1;
        B.tune_kernel = 5;
        const long long limit = (200 * 1024) / warps / 4 - sxw_hdr_words(A.k, tr);
        if (words > limit) words = limit;
        const int cw = (int)words;
        switch (A.k) {
            case 1: return sx_wseg_launch_k<1>(A, st, t, cw, warps, tr, stream);
            case 2: return sx_wseg_launch_k<2>(A, st, t, cw, warps, tr, stream);
            case 3: return sx_wseg_launch_k<3>(A, st, t, cw, warps, tr, stream);
            case 4: return sx_wseg_launch_k<4>(A, st, t, cw, warps, tr, stream);
            case 5: return sx_wseg_launch_k<5>(A, st, t, cw, warps, tr, stream);
            case 6: return sx_wseg_launch_k<6>(A, st, t, cw, warps, tr, stream);
            case 7: return sx_wseg_launch_k<7>(A, st, t, cw, warps, tr, stream);
            case 8: return sx_wseg_launch_k<8>(A, st, t, cw, warps, tr, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (B.tune_kernel == 4) {
        int cap = 0, threads = 0;
        sx_seg_shape(A.capacity, tiles, A.tune_staging_cap, A.tune_warps, A.k, &cap, &threads);
        switch (A.k) {
            case 1: return sx_seg_launch_k<1>(A, st, t, cap, threads, tr, stream);
            case 2: return sx_seg_launch_k<2>(A, st, t, cap, threads, tr, stream);
            case 3: return sx_seg_launch_k<3>(A, st, t, cap, threads, tr, stream);
            case 4: return sx_seg_launch_k<4>(A, st, t, cap, threads, tr, stream);
            case 5: return sx_seg_launch_k<5>(A, st, t, cap, threads, tr, stream);
            case 6: return sx_seg_launch_k<6>(A, st, t, cap, threads, tr, stream);
            case 7: return sx_seg_launch_k<7>(A, st, t, cap, threads, tr, stream);
            case 8: return sx_seg_launch_k<8>(A, st, t, cap, threads, tr, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (B.tune_kernel == 3) {
        const int nbuf = (A.k == 3 || A.k == 6 || A.k == 7) ? 3 : 2;
        const int cap = sx_merge_cap(A.capacity, tiles, A.tune_staging_cap, nbuf);
        switch (A.k) {
            case 1: return sx_merge_launch_k<1>(A, st, t, cap, stream);
            case 2: return sx_merge_launch_k<2>(A, st, t, cap, stream);
            case 3: return sx_merge_launch_k<3>(A, st, t, cap, stream);
            case 4: return sx_merge_launch_k<4>(A, st, t, cap, stream);
            case 5: return sx_merge_launch_k<5>(A, st, t, cap, stream);
            case 6: return sx_merge_launch_k<6>(A, st, t, cap, stream);
            case 7: return sx_merge_launch_k<7>(A, st, t, cap, stream);
            case 8: return sx_merge_launch_k<8>(A, st, t, cap, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (B.tune_kernel == 1 && B.tune_blocks_per_sm == 0) B.tune_blocks_per_sm = 3;
    if (B.tune_kernel == 1) {
        const SxBoolArgs& A = B;
        switch (A.k) {
            case 1: return sx_sweep_launch_k<1, MODE_TABLE>(A, st, t, stream);
            case 2: return sx_sweep_launch_k<2, MODE_TABLE>(A, st, t, stream);
            case 3: return sx_sweep_launch_k<3, MODE_TABLE>(A, st, t, stream);
            case 4: return sx_sweep_launch_k<4, MODE_TABLE>(A, st, t, stream);
            case 5: return sx_sweep_launch_k<5, MODE_TABLE>(A, st, t, stream);
            case 6: return sx_sweep_launch_k<6, MODE_TABLE>(A, st, t, stream);
            case 7: return sx_sweep_launch_k<7, MODE_TABLE>(A, st, t, stream);
            case 8: return sx_sweep_launch_k<8, MODE_TABLE>(A, st, t, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    int ecap = A.tune_staging_cap > 0 ? A.tune_staging_cap : sx_pick_ecap(A.capacity, tiles);
    if (ecap > 3584) ecap = 3584;
    if (ecap < 64) ecap = 64;
    switch (A.k) {
        case 1: return sx_sweep_smem_launch_k<1>(A, st, t, ecap, stream);
        case 2: return sx_sweep_smem_launch_k<2>(A, st, t, ecap, stream);
        case 3: return sx_sweep_smem_launch_k<3>(A, st, t, ecap, stream);
        case 4: return sx_sweep_smem_launch_k<4>(A, st, t, ecap, stream);
        case 5: return sx_sweep_smem_launch_k<5>(A, st, t, ecap, stream);
        case 6: return sx_sweep_smem_launch_k<6>(A, st, t, ecap, stream);
        case 7: return sx_sweep_smem_launch_k<7>(A, st, t, ecap, stream);
        case 8: return sx_sweep_smem_launch_k<8>(A, st, t, ecap, stream);
        default: return cudaErrorInvalidValue;
    }
}
