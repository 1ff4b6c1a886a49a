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
// Shared-memory form of the table sweep (the main path for set algebra).
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
// Merge-path form of the table sweep (the main path for set algebra).
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

cudaError_t sx_sweep_launch(const SxBoolArgs& A, bool union_mode, void* workspace, cudaStream_t stream)
{
    const long long tiles = sx_sweep_tiles(A.rows);
    if (tiles <= 0) return cudaSuccess;
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
    if (B.tune_kernel == 0) B.tune_kernel = 3;
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
