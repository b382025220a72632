// gsofa_kernels.cu -- sm_100a kernels of the fill-path symbolic factorization.
//
// Fill-path rule (the reference's, SOA symbfact_warp_centric_new_scheduling.cuh
// :842-1001): (s,m), s != m, is an entry of L+U iff A(s,m) != 0 or a path
// s -> v1 -> ... -> m exists in the graph of A whose intermediate vertices are
// all < min(s,m).  The reference finds the entries of row s with one max-id
// label per (source, vertex) in global memory and atomicMin relaxations.
//
// Here the rule is split in its two halves, each a plain reachability search
// with a 1-bit "seen" state:
//   * U row s (m > s): m is adjacent to s or to a vertex reachable from s
//     through vertices < s.  One search from s in A, expanding only ids < s.
//   * L column m (s > m): a path s -> m through ids < m is a path m -> s in
//     A^T through ids < m.  One search from m in A^T, expanding only ids < m.
// Each search visits every vertex at most once (no label re-expansions), and
// its whole state is one bit per vertex, kept in shared memory: n bits =
// 82 KB at n = 659,033, 125 KB at n = 10^6.
//
// A search is direction-optimising (Beamer, Asanovic, Patterson, SC'12):
// top-down levels expand a frontier queue while it is small; once it is
// large, bottom-up sweeps test, for every unseen vertex, whether one of its
// in-neighbours (its row of the other graph) is seen, and a last bottom-up
// pass marks the ids > source adjacent to the seen set.  Only reachability
// is needed, so a sweep tests "seen" rather than "in the last frontier".
//
// The per-source work item of the reference (one slot of a source group,
// :2929-3081) becomes a (matrix, source, direction) work item; persistent CTAs
// take items from a global atomic counter (work stealing), largest sources
// first.  There is no grid barrier (the reference's barrier.cuh spins) and no
// wait on another CTA: each CTA only synchronises with itself.
//
// Graph layout (both A and A^T): padded CSR.  Row v occupies
// cl[rp[v] & ~3, rp[v+1] & ~3): a multiple of 4 entries, 16-byte aligned, so
// rows are read with int4 loads; the last (rp[v+1] & 3) entries repeat v
// itself, which every test below treats as a no-op.
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include "gsofa_internal.h"
#include "../../include/gsofa.h"

namespace gsofa {

#define FULL_MASK 0xffffffffu

// Digest mixing: splitmix64 finaliser (Steele, Lea, Flood 2014).  A U-row
// or L-column digest sums mix64((w << 32) | mask) over the set's non-zero
// 32-id words w; an L-row digest (scattered) sums mix64(id) over its ids.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ int find_matrix(const MatDesc* mats, int nmats, long long item) {
    int lo = 0, hi = nmats - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (mats[mid].item_base <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t ld_vol(const uint32_t* p) {
    return *reinterpret_cast<const volatile uint32_t*>(p);
}

// Loads of matrix data.  CG = false: the read-only path (L1-cached), valid
// because nothing writes a matrix while a launch reads it.  CG = true (the
// serving kernel): L2 only.  A serving launch outlives the matrices it reads;
// their memory is freed and reused for later requests while it runs, so a
// line it once cached in L1 could be stale.
template <bool CG>
__device__ __forceinline__ int ld_i32(const int32_t* p) {
    return CG ? __ldcg(p) : __ldg(p);
}

template <bool CG>
__device__ __forceinline__ int4 ld_row4(const int32_t* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    return CG ? __ldcg(q) : __ldg(q);
}

// Original (unpadded) length of row v of a padded graph.
template <bool CG>
__device__ __forceinline__ int row_degree(const int32_t* rp, int v) {
    const int a = ld_i32<CG>(rp + v), b = ld_i32<CG>(rp + v + 1);
    return (b & ~3) - (a & ~3) - (b & 3);
}

// Ring slot masks: one bit per closure-ring slot (up to 64 slots).
typedef unsigned long long rmask_t;

// Chained starts.  When source s-1 lies in R(s) -- for a U row that is
// L(s, s-1) != 0, for an L column U(s-1, s) != 0 -- the whole closure of s-1
// belongs to the closure of s and every vertex of it is already expanded, so
// the search of s starts from the bitmap s-1 left behind instead of an empty
// one and expands only what is new.  Whether it holds is known before s
// starts: symmetric patterns read it from s-1's own bitmap (bit s), the other
// patterns from the other direction's search of s-1 (MatDesc::link), when
// that one has finished already.  With the old bits in place, a first
// occurrence of an id > s in the source row can no longer be told from a
// fresh bit, so chained starts count the distinct ids of that row through a
// small set in shared memory; only rows of up to kChainMaxRow entries chain.
constexpr int kHsetCap = 256;
constexpr int kChainMaxRow = 128;
// the set, one per CTA (static shared memory of every kernel that uses it)
__shared__ int chain_hset[kHsetCap];

template <int BLOCK>
struct TraverseSmem {
    typedef cub::BlockScan<int, BLOCK> Scan;
    typename Scan::TempStorage scan;
    unsigned long long red[BLOCK / 32][7];
    long long item;
    int cnt[3];
    int grab[3];          // per level (rotating): 32-vertex chunks of the frontier taken
    int redo[3];          // per level (rotating): smallest queue index of a chunk abandoned
                          // when a cached source was reached (INT_MAX: none)
    int abort_level;  // set when a cached source is reached: stop, merge, redo
    int pushed;       // ids a merge appended to the queue
    rmask_t pending;      // cached sources a merge set (slots), for the next decision
    rmask_t reached[3];   // per level (rotating): cached sources first reached
    int mi;               // matrix of the current item
    int skip;             // the current item's matrix failed ingest: count it only
    int cta;              // workspace slot (serving) or block index
    int wlo, whi;         // bitmap words holding the current source's set bits
    int sym;              // the current item's matrix has a symmetric pattern
    int ring_lo[64];      // per ring slot: the words its closure occupies
    int ring_hi[64];
    int chain;            // the next source starts from this source's bitmap
    int premerge;         // else: ring slot of a cached source the next one is known to reach
};

// Bitmap words of a matrix of order n: n bits plus zero padding read by the
// 128-bit L-mask extraction past the last vertex.
__host__ __device__ __forceinline__ long long bitmap_words_for(int32_t n) {
    return (((long long)n + 31) >> 5) + 6;
}

struct Src {
    int32_t src, n;
    int dir;
    const int32_t* __restrict__ rp;   // out-graph (top-down)
    const int32_t* __restrict__ cl;
    const int32_t* __restrict__ irp;  // in-graph (bottom-up)
    const int32_t* __restrict__ icl;
    uint32_t* bm;                     // X: this source's seen bits
    // Ring of the closures of the last `ring` sources this CTA finished in the
    // current chunk: source t lives in slot t & (ring-1).  Sources in
    // [cache_lo, src) are cached; merged_mask has the slots already merged.
    const uint32_t* ring_base;
    const int* ring_lo;               // per slot: first and last word of its closure
    const int* ring_hi;               // (words outside hold stale data from older closures)
    long long words;                  // ring slot stride (the launch's widest bitmap)
    long long mwords;                 // this matrix's bitmap words (what a merge ORs)
    int ring;
    int32_t cache_lo;
    rmask_t merged_mask;
    int top;                          // slot of the largest merged source, -1 if none
    rmask_t pending;                  // cached sources a merge set, not yet merged (slots)
    int* abort_flag;
    rmask_t* reached;                 // slots of cached sources first reached this level
    int qmark;                        // queue entries from here on were queued after the
                                      // last merge: none lies in the top merged closure
    bool chained;                     // started from the previous source's closure
};

// The cached source held in ring slot j.
__device__ __forceinline__ int32_t slot_source(const Src& S, int j) {
    return S.src - 1 - ((S.src - 1 - j) & (S.ring - 1));
}

// v lies in R(t) u {t} for the largest merged cached source t (slot `top`):
// every out-neighbour of v is already in the merged closure, so v needs no
// expansion.  (Ids in (t, src) of t's closure were only touched by t, never
// expanded.)  Only an optimisation: a false "no" costs one needless expansion.
__device__ __forceinline__ bool covered(const Src& S, int top, int32_t v) {
    if (top < 0 || v > slot_source(S, top)) return false;
    const int w = v >> 5;
    if (w < S.ring_lo[top] || w > S.ring_hi[top]) return false;  // no set bit there
    // plain load: the ring is written by this kernel
    const uint32_t* y = S.ring_base + (long long)top * S.words;
    return (y[w] >> (v & 31)) & 1u;
}

// Slot of the largest source in a merged mask, or -1.
__device__ __forceinline__ int top_slot(const Src& S, rmask_t mask) {
    for (int32_t t = S.src - 1; t >= S.cache_lo; t--)
        if ((mask >> (t & (S.ring - 1))) & 1u) return t & (S.ring - 1);
    return -1;
}

// Inserts w (>= 0) into the open-addressing set h of kHsetCap slots (-1 =
// empty); returns 1 when w was not there.  Holds at most kChainMaxRow keys,
// so a free slot or w itself is always found.
__device__ __forceinline__ uint32_t hset_insert(int w) {
    int* const h = chain_hset;
    unsigned k = ((unsigned)w * 0x9E3779B1u) >> 24;  // 8 bits: kHsetCap = 256
    for (int p = 0; p < kHsetCap; p++) {
        const int old = atomicCAS(h + k, -1, w);
        if (old == -1) return 1u;
        if (old == w) return 0u;
        k = (k + 1) & (kHsetCap - 1);
    }
    return 0u;
}

// Warp-aggregated append of up to 4 vertices per lane to the queue.
// BALLOT: one ballot per entry position gives each lane its offsets, and the
// queue takes position 0 of all lanes, then position 1, and so on; otherwise
// an inclusive shuffle scan of the per-lane counts keeps each lane's entries
// together.  The queue's order does not change what a search reaches; the
// ballot form measured faster with 512 threads per source and more (the
// circuit-like n=659,033 matrix: 403 -> 366 ms), the scan with 128 and 256
// (the 512-matrix grid/banded mix, 129 against 156 ms; the 64^3 grid, 5.2
// against 5.4 ms).
template <bool BALLOT>
__device__ __forceinline__ void push4(int32_t* q, long long qcap, long long le, int* cnt,
                                      int32_t* status, int lane, const int4& e, unsigned f) {
    if constexpr (BALLOT) {
        if (!__any_sync(FULL_MASK, f)) return;
        const unsigned b0 = __ballot_sync(FULL_MASK, f & 1u), b1 = __ballot_sync(FULL_MASK, f & 2u);
        const unsigned b2 = __ballot_sync(FULL_MASK, f & 4u), b3 = __ballot_sync(FULL_MASK, f & 8u);
        const int n0 = __popc(b0), n1 = __popc(b1), n2 = __popc(b2), n3 = __popc(b3);
        const int total = n0 + n1 + n2 + n3;
        int base = 0;
        if (lane == 0) base = atomicAdd(cnt, total);
        base = __shfl_sync(FULL_MASK, base, 0);
        const unsigned lt = (1u << lane) - 1u;
        const long long at0 = le + base;
        const int ws[4] = {e.x, e.y, e.z, e.w};
        const unsigned bs[4] = {b0, b1, b2, b3};
        const int off[4] = {0, n0, n0 + n1, n0 + n1 + n2};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (f & (1u << c)) {
                const long long at = at0 + off[c] + __popc(bs[c] & lt);
                if (at < qcap) q[at] = ws[c];
                else atomicOr(status, DEV_ERR_QUEUE);
            }
        }
    } else {
        const int mine = __popc(f);
        if (!__any_sync(FULL_MASK, mine)) return;
        int incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= o) incl += t;
        }
        const int total = __shfl_sync(FULL_MASK, incl, 31);
        int base = 0;
        if (lane == 31) base = atomicAdd(cnt, total);
        base = __shfl_sync(FULL_MASK, base, 31);
        long long at = le + base + (incl - mine);
        const int ws[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (f & (1u << c)) {
                if (at < qcap) q[at] = ws[c];
                else atomicOr(status, DEV_ERR_QUEUE);
                at++;
            }
        }
    }
}

// Top-down visit of edges v -> e.x, e.y, e.z, e.w.  Bit c of the result is
// set when entry c is a new vertex < src to queue.  An entry equal to src
// (also the sentinel of idle lanes and the padding of the source's row) is a
// no-op.  raw / orig count the source row's entries > src (with multiplicity
// / distinct) for the reference's nz_row_U counter.
template <bool PAIRED>
__device__ __forceinline__ unsigned td_edge4(const Src& S, int v, const int4& e, uint32_t& raw,
                                             uint32_t& orig, int& wl, int& wh) {
    // PAIRED: the bitmap accesses are issued four at a time: the four words
    // are read together, then the unset bits are claimed together, so a lane
    // waits for one read and one atomic rather than for four of each in turn.
    // Two entries with the same bit stay correct: a thread's atomics on one
    // word are ordered, and the second sees the first's bit.  Otherwise each
    // entry's read and claim finish before the next entry's start.
    const int ws[4] = {e.x, e.y, e.z, e.w};
    uint32_t cur[4], old[4];
    if constexpr (PAIRED) {
#pragma unroll
        for (int c = 0; c < 4; c++) cur[c] = ws[c] != S.src ? ld_vol(S.bm + (ws[c] >> 5)) : ~0u;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const uint32_t bit = 1u << (ws[c] & 31);
            old[c] = !(cur[c] & bit) ? atomicOr(S.bm + (ws[c] >> 5), bit) : bit;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const uint32_t bit = 1u << (ws[c] & 31);
            cur[c] = ws[c] != S.src ? ld_vol(S.bm + (ws[c] >> 5)) : ~0u;
            old[c] = !(cur[c] & bit) ? atomicOr(S.bm + (ws[c] >> 5), bit) : bit;
        }
    }
    unsigned f = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int w = ws[c];
        if (w == S.src) continue;
        const bool fresh = !(old[c] & (1u << (w & 31)));
        if (fresh) {
            wl = min(wl, w >> 5);
            wh = max(wh, w >> 5);
        }
        if (w > S.src) {
            if (v == S.src) {
                raw++;
                if (S.chained) orig += hset_insert(w);
                else if (fresh) orig++;
            }
            continue;
        }
        if (fresh && w >= S.cache_lo && !((S.merged_mask >> (w & (S.ring - 1))) & 1u)) {
            atomicOr(S.reached, 1ull << (w & (S.ring - 1)));
            *(volatile int*)S.abort_flag = 1;
        }
        if (fresh) f |= 1u << c;
    }
    return f;
}

// One top-down level: expand queue[lb, le), append new vertices after le.
// After a merge, vertices inside the merged closure (and the source itself)
// are skipped: their reach is already in the bitmap.
template <int BLOCK, bool CG>
__device__ __forceinline__ void td_level(const Src& S, int32_t* q, long long qcap, long long lb,
                                         long long le, int* cnt, int* grab, int* redo, int32_t* status,
                                         int heavy_len, uint32_t& raw, uint32_t& orig,
                                         uint32_t& trav, int& wl, int& wh) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int4 idle = make_int4(S.src, S.src, S.src, S.src);
    (void)NW;
    (void)warp;
    // warps take 32-vertex chunks of the frontier as they free up: rows of
    // very uneven length would leave statically assigned warps idle at the
    // level's barrier
    int chunk0 = 0;
    if (lane == 0) chunk0 = atomicAdd(grab, 1);
    long long nbase = lb + 32ll * __shfl_sync(FULL_MASK, chunk0, 0);
    int nv = (nbase + lane < le) ? q[nbase + lane] : S.src;
    for (;;) {
        const long long base = nbase;
        if (base >= le) break;
        const long long i = base + lane;
        int v = nv;
        // take the next chunk and start loading its entries now: the queue
        // round trip overlaps this chunk's work
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(grab, 1);
        nbase = lb + 32ll * __shfl_sync(FULL_MASK, chunk, 0);
        nv = (nbase + lane < le) ? q[nbase + lane] : S.src;
        // stop when a cached source was reached; one value for the whole warp
        const int ab = __shfl_sync(FULL_MASK, *(volatile int*)S.abort_flag, 0);
        if (lb > 0 && ab) {
            // chunks are handed out in increasing order and each is either
            // finished or abandoned: the level is redone from the smallest
            // abandoned one (this chunk; the prefetched next one is larger)
            if (lane == 0) atomicMin(redo, (int)base);
            break;
        }
        int s0 = 0, plen = 0;
        if (i < le) {
            bool skip = false;
            if (S.merged_mask && i < S.qmark) skip = v == S.src || covered(S, S.top, v);
            if (!skip) {
                const int r0 = ld_i32<CG>(S.rp + v), r1 = ld_i32<CG>(S.rp + v + 1);
                s0 = r0 & ~3;
                plen = (r1 & ~3) - s0;
                trav += (uint32_t)plen;
            } else {
                v = S.src;
            }
        }
        // long rows: the whole warp walks one row with coalesced int4 loads
        unsigned heavy = __ballot_sync(FULL_MASK, plen > heavy_len);
        while (heavy) {
            const int l = __ffs(heavy) - 1;
            heavy &= heavy - 1;
            const int hb = __shfl_sync(FULL_MASK, s0, l);
            const int hl = __shfl_sync(FULL_MASK, plen, l);
            const int hv = __shfl_sync(FULL_MASK, v, l);
            // the next 128 entries are loaded before these are processed
            int4 he = 4 * lane < hl ? ld_row4<CG>(S.cl + hb + 4 * lane) : idle;
            for (int k0 = 0; k0 < hl; k0 += 128) {
                const int kn = k0 + 128 + 4 * lane;
                const int4 hn = kn < hl ? ld_row4<CG>(S.cl + hb + kn) : idle;
                const unsigned f = td_edge4<(BLOCK >= 512)>(S, hv, he, raw, orig, wl, wh);
                push4<(BLOCK >= 512)>(q, qcap, le, cnt, status, lane, he, f);
                he = hn;
            }
        }
        if (plen > heavy_len) plen = 0;
        // short rows: one lane per vertex, 4 entries per int4 load
        const int its = plen >> 2;
        const int maxit = __reduce_max_sync(FULL_MASK, its);
        // the next int4 of the row is loaded before this one is processed, so
        // two loads of each lane's chain are in flight
        int4 e = 0 < its ? ld_row4<CG>(S.cl + s0) : idle;
        for (int it = 0; it < maxit; it++) {
            const int4 nx = it + 1 < its ? ld_row4<CG>(S.cl + s0 + 4 * (it + 1)) : idle;
            const unsigned f = td_edge4<(BLOCK >= 512)>(S, v, e, raw, orig, wl, wh);
            push4<(BLOCK >= 512)>(q, qcap, le, cnt, status, lane, e, f);
            e = nx;
        }
    }
}

__device__ __forceinline__ bool seen_le_src(const Src& S, int p) {
    return p <= S.src && ((ld_vol(S.bm + (p >> 5)) >> (p & 31)) & 1u);
}

// Bottom-up sweep.  upper == false: unseen u < src become seen (and queued)
// when an in-neighbour p <= src is seen.  upper == true: unmarked w in
// (src, n) are marked when an in-neighbour p <= src is seen.
template <int BLOCK, bool CG>
__device__ __forceinline__ void bu_sweep(const Src& S, bool upper, int32_t* q, long long qcap,
                                         long long le, int* cnt, int32_t* status, uint32_t& trav) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long lo = upper ? ((long long)S.src + 1) : 0;
    const long long hi = upper ? (long long)S.n : (long long)S.src;
    const long long w0 = lo >> 5, w1 = (hi + 31) >> 5;
    for (long long wd = w0 + warp; wd < w1; wd += NW) {
        const long long u = wd * 32 + lane;
        const bool valid = u >= lo && u < hi;
        const uint32_t bits = ld_vol(S.bm + wd);
        const bool need = valid && !((bits >> lane) & 1u);
        if (!__any_sync(FULL_MASK, need)) continue;
        bool found = false;
        if (need) {
            const int a0 = ld_i32<CG>(S.irp + u), a1 = ld_i32<CG>(S.irp + u + 1);
            const int ib = a0 & ~3, ie = a1 & ~3;
            for (int j = ib; j < ie; j += 4) {
                const int4 p = ld_row4<CG>(S.icl + j);
                trav += 4;
                if (seen_le_src(S, p.x) || seen_le_src(S, p.y) || seen_le_src(S, p.z) ||
                    seen_le_src(S, p.w)) {
                    found = true;
                    break;
                }
            }
        }
        const unsigned bal = __ballot_sync(FULL_MASK, found);
        if (!bal) continue;
        const int leader = __ffs(bal) - 1;
        if (lane == leader) atomicOr(S.bm + wd, bal);
        if (!upper) {
            int base = 0;
            if (lane == leader) base = atomicAdd(cnt, __popc(bal));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (found) {
                const long long at = le + base + __popc(bal & ((1u << lane) - 1u));
                if (at < qcap) q[at] = (int32_t)u;
                else atomicOr(status, DEV_ERR_QUEUE);
                if (u >= S.cache_lo) atomicOr(S.reached, 1ull << ((int)u & (S.ring - 1)));
            }
        }
    }
}

// Merges the closures of the cached sources that the search has reached.
// If t in [cache_lo, src) is reached then t's closure (its R(t), t and its
// entries > t) belongs to src's closure.  Reached sources are taken from the
// largest down; one inside an already merged R(t') u {t'} adds nothing.
// Vertices of (t, src) that only the merge set were never expanded: they are
// appended to the queue at `at` (*pushed gets their number).  Block-wide,
// uniform; returns the new merged mask.
template <int BLOCK>
__device__ __forceinline__ rmask_t merge_reached(const Src& S, rmask_t reached, uint32_t* bm,
                                                  int32_t* q, long long at, long long qcap,
                                                  int* pushed, rmask_t* pending_out,
                                                  int32_t* status, bool& did_merge, int& wl,
                                                  int& wh) {
    // The decision uses only values every thread holds identically: the
    // level's reached mask (stable until two levels later), the pending mask
    // and the ring, never the live bitmap.
    rmask_t add = 0;
    did_merge = false;
    rmask_t mm = S.merged_mask;
    const rmask_t cand = (reached | S.pending) & ~mm;
    if (!cand) return mm;
    // Candidates in decreasing source order, each tested against the largest
    // source marked so far.  After the first candidate is marked that source
    // no longer changes (every later candidate is smaller), and all
    // candidates lie in [cache_lo, src), at most three words: load those
    // words of its closure once and test the rest with register bit tests.
    int32_t t = S.src - 1;
    while (t >= S.cache_lo && !((cand >> (t & (S.ring - 1))) & 1ull)) t--;
    {
        const bool inside = covered(S, top_slot(S, mm), t);
        mm |= 1ull << (t & (S.ring - 1));
        if (!inside) add |= 1ull << (t & (S.ring - 1));
    }
    const int top = top_slot(S, mm);
    const int32_t tsrc = slot_source(S, top);
    const long long wb = S.cache_lo >> 5;
    uint32_t cw[3] = {0u, 0u, 0u};
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const long long w = wb + j;
        if (w <= ((S.src - 1) >> 5) && w >= S.ring_lo[top] && w <= S.ring_hi[top])
            cw[j] = S.ring_base[(long long)top * S.words + w];
    }
    for (t = t - 1; t >= S.cache_lo; t--) {
        const int slot = t & (S.ring - 1);
        if (!((cand >> slot) & 1ull)) continue;
        const int j = (int)((t >> 5) - wb);
        const uint32_t word = j == 0 ? cw[0] : (j == 1 ? cw[1] : cw[2]);
        const bool inside = t <= tsrc && ((word >> (t & 31)) & 1u);
        mm |= 1ull << slot;
        if (!inside) add |= 1ull << slot;
    }
    if (!add) return mm;
    did_merge = true;
    // stream the added closures into L2 at once with the bulk-copy engine;
    // the loads below then hit L2 instead of waiting on DRAM a few lines at
    // a time (16-byte-aligned interior only, so nothing outside the closure
    // is touched)
    if (threadIdx.x == 0) {
        for (rmask_t a = add; a; a &= a - 1) {
            const int sl = __ffsll((long long)a) - 1;
            const uint32_t* p0 = S.ring_base + (long long)sl * S.words + S.ring_lo[sl];
            const uint32_t* p1 = S.ring_base + (long long)sl * S.words + S.ring_hi[sl] + 1;
            const unsigned long long a0 = (reinterpret_cast<unsigned long long>(p0) + 15ull) & ~15ull;
            const unsigned long long a1 = reinterpret_cast<unsigned long long>(p1) & ~15ull;
            if (a1 > a0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0),
                             "r"((unsigned)(a1 - a0))
                             : "memory");
        }
    }
    // ids in (t, src) of an added t's closure were never expanded; with only
    // src-1 added that window is empty and the merge is a plain OR
    int32_t lo = S.src;
    for (rmask_t a = add; a; a &= a - 1) {
        const int32_t t = slot_source(S, __ffsll((long long)a) - 1);
        if (t + 1 < lo) lo = t + 1;
    }
    const bool window = lo < S.src;
    // the window [lo, src) spans at most 63 ids: three words before the merge
    const long long w0 = lo >> 5, w1 = (S.src - 1) >> 5;
    uint32_t b0 = 0, b1 = 0, b2 = 0;
    if (window) {
        b0 = ld_vol(bm + w0);
        if (w0 + 1 <= w1) b1 = ld_vol(bm + w0 + 1);
        if (w0 + 2 <= w1) b2 = ld_vol(bm + w0 + 2);
        __syncthreads();
    }
    // OR the added closures over the words they occupy, four words per
    // thread per pass so that their loads overlap
    int mlo = INT_MAX, mhi = -1;
    for (rmask_t a = add; a; a &= a - 1) {
        const int sl = __ffsll((long long)a) - 1;
        mlo = min(mlo, S.ring_lo[sl]);
        mhi = max(mhi, S.ring_hi[sl]);
    }
    for (long long i0 = (long long)mlo + threadIdx.x; i0 <= mhi; i0 += 4ll * BLOCK) {
        uint32_t y[4] = {0u, 0u, 0u, 0u};
        for (rmask_t a = add; a; a &= a - 1) {
            const int sl = __ffsll((long long)a) - 1;
            const int slo = S.ring_lo[sl], shi = S.ring_hi[sl];
            const uint32_t* src = S.ring_base + (long long)sl * S.words;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const long long i = i0 + (long long)j * BLOCK;
                if (i >= slo && i <= shi) y[j] |= src[i];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const long long i = i0 + (long long)j * BLOCK;
            if (i <= mhi && y[j]) bm[i] |= y[j];
        }
    }
    wl = min(wl, mlo);
    wh = max(wh, mhi);
    if (!window) {
        if (threadIdx.x == 0) {
            *pushed = 0;
            *pending_out = 0ull;
        }
        return mm;  // the caller's barrier completes the merge
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int np = 0;
        rmask_t pend = 0;
        const int top = top_slot(S, mm);
        for (int32_t v = lo; v < S.src; v++) {
            const long long w = v >> 5;
            const uint32_t before = w == w0 ? b0 : (w == w0 + 1 ? b1 : b2);
            const uint32_t bit = 1u << (v & 31);
            if ((before & bit) || !(ld_vol(bm + w) & bit)) continue;  // not set by the merge
            // a cached source set by the merge is reached too: merge it next time
            if (!((mm >> (v & (S.ring - 1))) & 1ull)) pend |= 1ull << (v & (S.ring - 1));
            if (covered(S, top, v)) continue;
            if (at + np < qcap) q[at + np] = v;
            else atomicOr(status, DEV_ERR_QUEUE);
            np++;
        }
        *pushed = np;
        *pending_out = pend;
    }
    return mm;
}

__device__ __forceinline__ unsigned long long ld_vol64(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ int ld_vol_i32(const int32_t* p) {
    return *reinterpret_cast<const volatile int32_t*>(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Called by the 32 lanes of warp 0 when source nx = src + 1 cannot start
// from src's closure: the ring slot of the largest cached source t < src that
// nx is known to reach, or -1.  nx reaches t when the other direction's
// search of t has finished (its link byte is set) and its mask of
// t+1 .. t+128 has bit nx: L(nx, t) != 0 for a U-row search (the L-column
// mask of t), U(t, nx) != 0 for an L-column search (the U-row mask of t).  A
// symmetric pattern reads bit nx of t's own closure in the ring.  Lane k
// tests t = src - 1 - k (and t - 32).
__device__ int premerge_candidate(const Src& S, const MatDesc& M, int32_t src, int32_t s_first,
                                  int dir, bool lfold) {
    const int lane = threadIdx.x & 31;
    const int32_t nx = src + 1;
    const int32_t lo = max(s_first, nx - S.ring);
    for (int k0 = 0; k0 < 64; k0 += 32) {
        const int32_t t = src - 1 - k0 - lane;
        bool ok = false;
        if (t >= lo) {
            const int j = nx - t - 1;  // 1 .. 63: bit of nx in t's mask
            if (lfold) {
                const int slot = t & (S.ring - 1);
                const int w = nx >> 5;
                if (w >= S.ring_lo[slot] && w <= S.ring_hi[slot])
                    ok = (S.ring_base[(long long)slot * S.words + w] >> (nx & 31)) & 1u;
            } else if (M.link) {
                uint32_t lk;
                asm volatile("ld.acquire.gpu.global.u8 %0, [%1];"
                             : "=r"(lk) : "l"(M.link + 2ll * t + (1 - dir)) : "memory");
                const uint32_t* mk = dir == 0 ? M.lmask : M.umask;
                if (lk != 0 && mk) ok = (__ldcg(mk + 4ll * t + (j >> 5)) >> (j & 31)) & 1u;
            }
        }
        const unsigned b = __ballot_sync(FULL_MASK, ok);
        if (b) return (src - 1 - k0 - (__ffs(b) - 1)) & (S.ring - 1);
    }
    return -1;
}

// Serving, called by all 32 lanes of warp 0: claims a work item of any
// published request.  Each lane checks one list entry (rotating start); the
// claimable entry with the fewest unclaimed items is taken with
// compare-and-swap on its claim word.  Returns false (in every
// lane) when the host says to take no more items (ctrl[1]), when nothing is
// claimable and the host asks idle CTAs to exit (ctrl[0]), after idle_ns of
// finding nothing, or after max_idle_polls polls.
__device__ bool serve_claim(const TraverseLaunch& P, int* slot_out, long long* item_out) {
    const ServeLaunch& V = P.serve;
    const int lane = threadIdx.x & 31;
    unsigned ns = 32;
    const unsigned long long t0 = global_ns();
    for (long long polls = 0; polls < V.max_idle_polls; polls++) {
        int c0 = 0, c1 = 0, n = 0;
        unsigned r = 0;
        if (lane == 0) {
            c1 = ld_vol_i32(V.ctrl + 1);
            c0 = ld_vol_i32(V.ctrl);
            n = min(ld_vol_i32(V.ctrl + 2), V.nslots);
            if (!c1 && n > 0) r = atomicAdd(V.rr, 1u);
        }
        c0 = __shfl_sync(FULL_MASK, c0, 0);
        c1 = __shfl_sync(FULL_MASK, c1, 0);
        n = __shfl_sync(FULL_MASK, n, 0);
        r = __shfl_sync(FULL_MASK, r, 0);
        if (c1) return false;
        for (int base = 0; base < n; base += 32) {
            const int k = base + lane;
            bool ok = false;
            int slot = -1;
            unsigned seq = 0;
            unsigned long long v = 0;
            long long nit = 0;
            if (k < n) {
                const unsigned long long e = ld_vol64(V.list + (r + (unsigned)k) % (unsigned)n);
                slot = (int)(e >> 32);
                seq = (unsigned)e;
                if (slot >= 0 && slot < V.nslots) {
                    v = ld_vol64(V.claim + slot);
                    if ((unsigned)(v >> 32) == seq) {
                        __threadfence();  // the descriptor was written before the claim word
                        nit = __ldcg(&V.slots[slot].n_items);
                        ok = (long long)(v & 0xffffffffull) < nit;
                    }
                }
            }
            // shortest remaining work first (fewest unclaimed items), ties in
            // rotation order: small requests overtake large ones item by item
            unsigned rem = 0xffffffffu;
            if (ok) rem = (unsigned)min(nit - (long long)(v & 0xffffffffull), 0xfffffffell);
            for (int round = 0; round < 32; round++) {
                const unsigned best = __reduce_min_sync(FULL_MASK, rem);
                if (best == 0xffffffffu) break;
                const int l = __ffs(__ballot_sync(FULL_MASK, rem == best)) - 1;
                int got = 0;
                long long it = 0;
                if (lane == l) {
                    for (int tries = 0; tries < 256; tries++) {
                        if ((unsigned)(v >> 32) != seq || (long long)(v & 0xffffffffull) >= nit) break;
                        const unsigned long long old = atomicCAS(V.claim + slot, v, v + 1ull);
                        if (old == v) {
                            got = 1;
                            it = (long long)(v & 0xffffffffull);
                            break;
                        }
                        v = old;
                    }
                    rem = 0xffffffffu;  // taken or gone: this entry is done
                }
                if (__shfl_sync(FULL_MASK, got, l)) {
                    *slot_out = __shfl_sync(FULL_MASK, slot, l);
                    *item_out = __shfl_sync(FULL_MASK, it, l);
                    return true;
                }
            }
        }
        if (c0) return false;
        if (global_ns() - t0 > (unsigned long long)V.idle_ns) return false;
        __nanosleep(ns);
        if (ns < 2048) ns <<= 1;
    }
    return false;
}

// Serving: takes a free per-CTA workspace slot, or returns -1.
__device__ int take_cta_slot(const ServeLaunch& V) {
    const int nw = (V.n_cta_slots + 31) >> 5;
    for (int w = 0; w < nw; w++) {
        unsigned v = ld_vol_i32(reinterpret_cast<const int32_t*>(V.cta_slots + w));
        for (int tries = 0; tries < 64 && ~v; tries++) {
            const int b = __ffs(~v) - 1;
            if (w * 32 + b >= V.n_cta_slots) break;
            const unsigned old = atomicOr(V.cta_slots + w, 1u << b);
            if (!(old & (1u << b))) {
                atomicAdd(V.alive, 1);
                __threadfence();
                return w * 32 + b;
            }
            v = old | (1u << b);
        }
    }
    return -1;
}

// Thread 0 copies a matrix descriptor to shared memory (through L2 when it
// may have been rewritten since the launch began).
template <bool CG>
__device__ __forceinline__ void copy_desc(MatDesc* dst, const MatDesc* src) {
    static_assert(sizeof(MatDesc) % 8 == 0, "descriptor copied in 8-byte words");
    const unsigned long long* a = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* b = reinterpret_cast<unsigned long long*>(dst);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(MatDesc) / 8); k++) b[k] = CG ? __ldcg(a + k) : a[k];
}

__device__ __forceinline__ void flush_counters(unsigned long long* c, unsigned long long* acc) {
    atomicAdd(&c[CNT_FILLS], acc[0]);
    atomicAdd(&c[CNT_EDGES_ALG], acc[1]);
    atomicAdd(&c[CNT_VERTS_ALG], acc[2]);
    atomicAdd(&c[CNT_EDGES_TRAV], acc[3]);
    atomicAdd(&c[CNT_NNZ_U], acc[4]);
    atomicAdd(&c[CNT_NNZ_L], acc[5]);
    if (acc[6]) atomicAdd(&c[CNT_CHAINED], acc[6]);
    for (int j = 0; j < 7; j++) acc[j] = 0;
}

// MODE 0: each CTA's bitmap in global memory; 1: in shared memory;
// 2: serving -- items come from the requests the request loop publishes, and an
// item's bitmap sits in shared memory when the matrix fits, else in global
// memory (kept zero between items by the census, zeroed by the host once).
template <int BLOCK, int MODE>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) traverse_kernel(TraverseLaunch P) {
    extern __shared__ uint4 dyn_smem[];
    __shared__ TraverseSmem<BLOCK> SM;
    __shared__ MatDesc SD;  // the current item's matrix
    constexpr bool CG = MODE == 2;
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if constexpr (MODE == 2) {
        if (threadIdx.x == 0) SM.cta = take_cta_slot(P.serve);
        __syncthreads();
        if (SM.cta < 0) return;  // every workspace slot is taken
    } else if (threadIdx.x == 0) {
        SM.cta = blockIdx.x;
    }
    if (threadIdx.x == 0) {
        SM.chain = 0;
        SM.premerge = -1;
    }
    const long long cta = MODE == 2 ? SM.cta : blockIdx.x;
    uint32_t* const sbm = reinterpret_cast<uint32_t*>(dyn_smem);
    uint32_t* const gbm = MODE == 1 ? nullptr : P.gbitmap + cta * P.bitmap_words;
    uint32_t* bm = MODE == 1 ? sbm : gbm;
    uint32_t* ring_base = P.gprev + cta * P.ring * P.bitmap_words;
    int32_t* q = P.queue + cta * P.queue_stride;
    const long long qcap = P.queue_stride;

    if constexpr (MODE == 2) {
        for (long long i = threadIdx.x; i < P.serve.smem_words; i += BLOCK) sbm[i] = 0u;
    } else {
        for (long long i = threadIdx.x; i < P.bitmap_words; i += BLOCK) bm[i] = 0u;
    }

    // thread 0 accumulates per-matrix counters and flushes on matrix change
    // (serving: after every item)
    int acc_mat = -1;
    unsigned long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const long long stride = P.sample_stride > 1 ? P.sample_stride : 1;

    for (;;) {
        if constexpr (MODE == 2) {
            if (warp == 0) {
                int slot = 0;
                long long it = -1;
                const bool got = serve_claim(P, &slot, &it);
                if (lane == 0) {
                    if (got) {
                        copy_desc<true>(&SD, P.serve.slots + slot);
                        SM.skip = __ldcg(P.serve.slot_status + slot) != 0;  // ingest failed
                        SM.sym = SD.asym != nullptr && __ldcg(SD.asym) == 0;
                    }
                    SM.item = got ? it : -1;
                }
            }
        } else {
            // every thread is done with the previous item's descriptor before
            // thread 0 replaces it (an empty item, e.g. the direction-1 half
            // of a symmetric matrix, has no source-loop barrier of its own)
            __syncthreads();
        }
        if (MODE != 2 && threadIdx.x == 0) {
            const unsigned long long c = atomicAdd(P.work_counter, 1ull);
            const long long it = (long long)c < P.total_items ? (long long)c : -1;
            if (it >= 0) {
                SM.mi = find_matrix(P.mats, P.nmats, it * stride);
                copy_desc<false>(&SD, P.mats + SM.mi);
                SM.skip = 0;
                SM.sym = SD.asym != nullptr && *SD.asym == 0;
            }
            SM.item = it;
        }
        __syncthreads();
        if (SM.item < 0) break;
        const MatDesc& M = SD;
        const int mi = MODE == 2 ? 0 : SM.mi;
        const long long item = MODE == 2 ? SM.item : SM.item * stride;
        const int32_t n = M.n;
        const long long clen = MODE == 2 ? (long long)M.chunk : (long long)P.chunk;
        const long long local = item - M.item_base;
        const int dir = (int)(local & 1);
        const long long nchunks = ((long long)n + clen - 1) / clen;
        const long long chunk = nchunks - 1 - (local >> 1);  // largest sources first
        const int32_t s_first = (int32_t)(chunk * clen);
        // symmetric pattern: the direction-0 item of this chunk does both halves
        const bool sym = SM.sym != 0;
        const bool lfold = sym && dir == 0;
        const int32_t s_end = (SM.skip || (sym && dir == 1))
                                  ? s_first
                                  : (int32_t)min((long long)n, (chunk + 1) * clen);
        const long long words = bitmap_words_for(n);
        const long long nwords = ((long long)n + 31) >> 5;
        if constexpr (MODE == 2) bm = words <= P.serve.smem_words ? sbm : gbm;

        Src S;
        S.n = n;
        S.dir = dir;
        S.rp = dir ? M.trowptr : M.rowptr;
        S.cl = dir ? M.tcol : M.col;
        S.irp = dir ? M.rowptr : M.trowptr;
        S.icl = dir ? M.col : M.tcol;
        S.bm = bm;
        S.ring_base = ring_base;
        S.ring_lo = SM.ring_lo;
        S.ring_hi = SM.ring_hi;
        S.words = P.bitmap_words;
        S.mwords = words;
        S.ring = P.ring;
        S.abort_flag = &SM.abort_level;
        const bool digests = M.dig_u != nullptr;
        const bool scatter = (dir == 1 || lfold) && M.nnz_lr != nullptr && !P.pattern_pass;

        for (int32_t src = s_first; src < s_end; src++) {
            S.src = src;
            // cached: the last `ring` sources of this chunk (none without merging)
            S.cache_lo = P.merge ? max(s_first, src - P.ring) : src;
            S.merged_mask = 0ull;
            S.top = -1;
            // a cached source known (from the other direction's search) to be
            // reached: merged right after the source's own row
            S.pending = (P.merge && src > s_first && SM.premerge >= 0) ? (1ull << SM.premerge) : 0ull;
            S.reached = &SM.reached[0];
            S.qmark = 0;
            // the bitmap still holds the closure of src - 1 (decided by its census)
            S.chained = SM.chain != 0;
            if (S.chained)
                for (int i = threadIdx.x; i < kHsetCap; i += BLOCK) chain_hset[i] = -1;
            if (threadIdx.x == 0) {
                bm[src >> 5] |= 1u << (src & 31);
                q[0] = src;
                SM.cnt[0] = 0;
                SM.grab[0] = 0;
                SM.redo[0] = INT_MAX;
                SM.reached[0] = 0ull;
                SM.abort_level = 0;
                if (S.chained) {  // the census range covers the kept bits too
                    SM.wlo = min(SM.wlo, src >> 5);
                    SM.whi = max(SM.whi, src >> 5);
                } else {
                    SM.wlo = SM.whi = src >> 5;
                }
            }
            __syncthreads();
            // this thread's share of the set bits' word range
            int wl = src >> 5, wh = src >> 5;

            uint32_t raw = 0, orig = 0, trav = 0;
            long long lb = 0, le = 1;
            int level = 0;
            bool bottom_up = false, used_bu = false;
            const bool allow_bu = P.bu_alpha > 0 && src >= P.bu_min_src;
            for (;;) {
                if (!bottom_up) {
                    if (lb >= le) break;
                    const long long unseen = (long long)src - (le - 1);
                    if (allow_bu && lb > 0 && (le - lb) * (long long)P.bu_alpha > unseen) {
                        bottom_up = used_bu = true;
                        continue;
                    }
                    if (threadIdx.x == 0) {
                        SM.cnt[(level + 1) % 3] = 0;
                        SM.grab[(level + 1) % 3] = 0;
                        SM.redo[(level + 1) % 3] = INT_MAX;
                        SM.reached[(level + 1) % 3] = 0ull;
                    }
                    S.reached = &SM.reached[level % 3];
                    td_level<BLOCK, CG>(S, q, qcap, lb, le, &SM.cnt[level % 3], &SM.grab[level % 3],
                                        &SM.redo[level % 3], P.status, P.heavy_len, raw, orig, trav, wl, wh);
                    __syncthreads();
                    const int nxt = SM.cnt[level % 3];
                    level++;
                    // a reached cached source's closure is ours: merge it
                    bool did = false;
                    const rmask_t reached = SM.reached[(level - 1) % 3];
                    const rmask_t mm =
                        S.cache_lo < src
                            ? merge_reached<BLOCK>(S, reached, bm, q, le + nxt, qcap, &SM.pushed,
                                                   &SM.pending, P.status, did, wl, wh)
                            : S.merged_mask;
                    if (mm != S.merged_mask) {
                        S.merged_mask = mm;
                        S.top = top_slot(S, mm);
                        if (threadIdx.x == 0) SM.abort_level = 0;
                        __syncthreads();
                        const int np = did ? SM.pushed : 0;
                        S.pending = did ? (SM.pending & ~mm) : (S.pending & ~mm);
                        // redo this level from its first abandoned chunk (every
                        // earlier chunk was expanded; none abandoned: all were)
                        const int rf = SM.redo[(level - 1) % 3];
                        lb = rf < le ? (long long)rf : le;
                        le = le + nxt + np;
                        S.qmark = (int)le;   // later entries are outside the merged closures
                    } else {
                        lb = le;
                        le = le + nxt;
                    }
                    if (le > qcap) le = qcap;  // unreachable: each vertex is queued once
                } else {
                    const long long unseen = (long long)src - (le - 1);
                    if (threadIdx.x == 0) {
                        SM.cnt[(level + 1) % 3] = 0;
                        SM.grab[(level + 1) % 3] = 0;
                        SM.reached[(level + 1) % 3] = 0ull;
                    }
                    S.reached = &SM.reached[level % 3];
                    bu_sweep<BLOCK, CG>(S, false, q, qcap, le, &SM.cnt[level % 3], P.status, trav);
                    __syncthreads();
                    const int found = SM.cnt[level % 3];
                    level++;
                    lb = le;
                    le = le + found;
                    if (le > qcap) le = qcap;
                    bool did = false;
                    const rmask_t reached = SM.reached[(level - 1) % 3];
                    const rmask_t mm =
                        S.cache_lo < src
                            ? merge_reached<BLOCK>(S, reached, bm, q, le, qcap, &SM.pushed,
                                                   &SM.pending, P.status, did, wl, wh)
                            : S.merged_mask;
                    if (mm != S.merged_mask) {
                        S.merged_mask = mm;
                        S.top = top_slot(S, mm);
                        if (threadIdx.x == 0) SM.abort_level = 0;
                        __syncthreads();
                        S.pending = did ? (SM.pending & ~mm) : (S.pending & ~mm);
                        le = le + (did ? SM.pushed : 0);  // merged-in ids become queue entries
                        S.qmark = (int)le;
                        continue;  // sweep again with the merged closure
                    }
                    if (found == 0) break;
                    if ((long long)found * P.bu_beta < unseen) bottom_up = false;  // few new
                }
            }
            if (used_bu) {
                bu_sweep<BLOCK, CG>(S, true, q, qcap, le, nullptr, P.status, trav);
                __syncthreads();
                wl = 0;  // sweeps set bits anywhere
                wh = (int)nwords - 1;
            }
            // the block's word range of set bits
            wl = __reduce_min_sync(FULL_MASK, wl);
            wh = __reduce_max_sync(FULL_MASK, wh);
            if (lane == 0) {
                atomicMin(&SM.wlo, wl);
                atomicMax(&SM.whi, wh);
            }
            if (warp == 0) {
                // Publish, for the other direction's searches, the 128 bits
                // src+1 .. src+128 of this closure (lanes 0-3: the L-column
                // mask of a direction-1 or symmetric search, the U-row mask
                // of a direction-0 one) and then the link byte of src; then
                // decide how src + 1 starts.  The search is over: every bit
                // is final after its last barrier.
                const int32_t nx = src + 1;
                const bool nbit = nx < n && ((ld_vol(bm + (nx >> 5)) >> (nx & 31)) & 1u);
                if (!P.pattern_pass && lane < 4) {
                    const long long p = (long long)src + 1 + 32 * lane;
                    const long long wd = p >> 5;
                    const int off = (int)(p & 31);
                    uint32_t val = bm[wd] >> off;
                    if (off) val |= bm[wd + 1] << (32 - off);
                    if (dir == 1 || lfold) M.lmask[4ll * src + lane] = val;
                    else if (M.umask) M.umask[4ll * src + lane] = val;
                    __threadfence();  // the masks are visible before the link
                }
                __syncwarp();
                if (lane == 0 && M.link && !lfold && !P.pattern_pass)
                    *reinterpret_cast<volatile uint8_t*>(M.link + 2ll * src + dir) = nbit ? 2 : 1;
                int ch = 0, pre = -1;
                if (P.chain && P.bu_alpha <= 0 && nx < s_end) {
                    if (lane == 0) {
                        const int r0 = ld_i32<CG>(S.rp + nx), r1 = ld_i32<CG>(S.rp + nx + 1);
                        if ((r1 & ~3) - (r0 & ~3) <= kChainMaxRow) {
                            if (lfold) {
                                ch = nbit;  // symmetric: U(src, src+1) = L(src+1, src)
                            } else if (M.link) {
                                const volatile uint8_t* lk = M.link + 2ll * src + (1 - dir);
                                uint8_t v = *lk;
                                // the other direction's search of this chunk has
                                // finished src - 1 and is on src: wait a bounded
                                // time for it rather than start src + 1 cold
                                if (v == 0 && P.chain_wait_ns > 0 && src > s_first &&
                                    *(const volatile uint8_t*)(M.link + 2ll * (src - 1) + (1 - dir)) != 0) {
                                    const unsigned long long t0 = global_ns();
                                    while ((v = *lk) == 0 &&
                                           global_ns() - t0 < (unsigned long long)P.chain_wait_ns)
                                        __nanosleep(64);
                                }
                                ch = v == 2;
                            }
                        }
                    }
                    ch = __shfl_sync(FULL_MASK, ch, 0);
                    if (!ch && P.merge) pre = premerge_candidate(S, M, src, s_first, dir, lfold);
                }
                if (lane == 0) {
                    SM.chain = ch;
                    SM.premerge = pre;
                }
            }
            __syncthreads();
            const long long wlo = SM.wlo, whi = SM.whi;
            const bool chain_next = SM.chain != 0;

            if (P.pattern_pass) {
                // sorted ids of the set bits > src: U row (dir 0) or L column (dir 1)
                int32_t* out = dir == 0 ? M.ucols : M.lrows;
                const long long obase = dir == 0 ? M.uptr[src] : M.lptr[src];
                int32_t* out2 = lfold ? M.lrows : nullptr;  // the same ids: L column src
                const long long obase2 = lfold ? M.lptr[src] : 0;
                long long wpos = ((long long)src + 1) >> 5;
                long long written = 0;
                for (; wpos < nwords; wpos += BLOCK) {
                    const long long wi = wpos + threadIdx.x;
                    uint32_t word = 0;
                    if (wi < nwords) {
                        word = bm[wi];
                        const long long first = wi << 5;
                        if (first <= src) {  // drop bits <= src
                            const int keep_from = (int)(src - first) + 1;
                            word = keep_from >= 32 ? 0u : (word & (~0u << keep_from));
                        }
                    }
                    int cntw = __popc(word), ex = 0, tot = 0;
                    typename TraverseSmem<BLOCK>::Scan(SM.scan).ExclusiveSum(cntw, ex, tot);
                    long long o = obase + written + ex;
                    long long o2 = obase2 + written + ex;
                    while (word) {
                        const int bpos = __ffs(word) - 1;
                        word &= word - 1;
                        out[o++] = (int32_t)((wi << 5) + bpos);
                        if (out2) out2[o2++] = (int32_t)((wi << 5) + bpos);
                    }
                    written += tot;
                    __syncthreads();  // scan storage reuse
                }
            }
            __syncthreads();

            // ---- census of the closure: counts and digests from the bitmap; the
            // bitmap moves to the CTA's previous-closure buffer and is cleared
            unsigned long long c_gt = 0, c_v = 0, c_e = 0, c_dig = 0;
            const bool keep = P.merge && src + 1 < s_end;
            uint32_t* keep_slot = ring_base + (long long)(src & (P.ring - 1)) * P.bitmap_words;
            if (keep && threadIdx.x == 0) {
                SM.ring_lo[src & (P.ring - 1)] = (int)wlo;
                SM.ring_hi[src & (P.ring - 1)] = (int)whi;
            }
            // every set bit lies in words [wlo, whi]: the rest of the bitmap is zero
            for (long long w = wlo + threadIdx.x; w <= whi; w += BLOCK) {
                const uint32_t x = bm[w];
                if (!chain_next) bm[w] = 0u;
                if (keep) keep_slot[w] = x;
                if (!x || w >= nwords) continue;
                const long long base = w << 5;
                uint32_t lo_m, hi_m;
                if (base + 31 < src) { lo_m = ~0u; hi_m = 0u; }
                else if (base > src) { lo_m = 0u; hi_m = ~0u; }
                else {
                    const int b = (int)(src - base);  // 0..31: bit of src
                    lo_m = b ? ((1u << b) - 1u) : 0u;
                    hi_m = b == 31 ? 0u : (~0u << (b + 1));
                }
                const uint32_t xl = x & lo_m, xh = x & hi_m;
                c_v += __popc(xl);
                if (dir == 0 && xl) {
                    if (xl == ~0u) {
                        c_e += (unsigned long long)ld_i32<CG>(M.wdeg + w);
                    } else if (BLOCK >= 256 && lo_m == ~0u && __popc(xl) >= 28) {
                        // a nearly full word (dense closures): its sum minus
                        // the degrees of its at most four clear bits, every
                        // load issued together, instead of three rounds of
                        // bit-plane loads.  Not compiled into 128-thread CTAs
                        // (small matrices, sparse closures), which measured
                        // slower with it.
                        uint32_t t = ~xl;
                        int ra[4], rb[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const int v = t ? (int)(base + __ffs(t) - 1) : -1;
                            t &= t - 1;
                            ra[j] = v >= 0 ? ld_i32<CG>(M.rowptr + v) : 0;
                            rb[j] = v >= 0 ? ld_i32<CG>(M.rowptr + v + 1) : 0;
                        }
                        int d = ld_i32<CG>(M.wdeg + w);
#pragma unroll
                        for (int j = 0; j < 4; j++) d -= (rb[j] & ~3) - (ra[j] & ~3) - (rb[j] & 3);
                        c_e += (unsigned long long)d;
                    } else if (__popc(xl) <= 2 || M.dplanes == nullptr) {
                        uint32_t t = xl;
                        while (t) {
                            const int bp = __ffs(t) - 1;
                            t &= t - 1;
                            c_e += (unsigned long long)row_degree<CG>(M.rowptr, (int)(base + bp));
                        }
                    } else {
                        // degree sum from the bit-planes: coalesced loads, four
                        // issued before any is used
                        const int32_t* pl = reinterpret_cast<const int32_t*>(M.dplanes) + w;
                        const int np = M.nplanes;
                        for (int k = 0; k < np; k += 4) {
                            uint32_t p4[4];
#pragma unroll
                            for (int j = 0; j < 4; j++)
                                p4[j] = k + j < np ? (uint32_t)ld_i32<CG>(pl + (k + j) * nwords) : 0u;
#pragma unroll
                            for (int j = 0; j < 4; j++)
                                c_e += (unsigned long long)__popc(xl & p4[j]) << (k + j);
                        }
                    }
                }
                c_gt += __popc(xh);
                // U-row / L-column digest: one term per non-zero word
                if (digests && xh) c_dig += mix64(((uint64_t)w << 32) | xh);
                if (scatter && xh) {
                    const unsigned long long ds = mix64((uint64_t)src);
                    uint32_t t = xh;
                    while (t) {
                        const int bp = __ffs(t) - 1;
                        t &= t - 1;
                        const int wv = (int)(base + bp);
                        atomicAdd(&M.nnz_lr[wv], 1);
                        atomicAdd((unsigned long long*)&M.dig_lr[wv], ds);
                    }
                }
            }
            unsigned long long vals[7] = {c_gt, raw, orig, c_v, c_e, c_dig, trav};
#pragma unroll
            for (int j = 0; j < 7; j++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) vals[j] += __shfl_xor_sync(FULL_MASK, vals[j], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 7; j++) SM.red[warp][j] = vals[j];
            }
            __syncthreads();
            if (threadIdx.x == 0 && !P.pattern_pass) {
                unsigned long long r[7] = {0, 0, 0, 0, 0, 0, 0};
                for (int wi = 0; wi < NW; wi++)
                    for (int j = 0; j < 7; j++) r[j] += SM.red[wi][j];
                const unsigned long long gt = r[0], rw = r[1], og = r[2], vv = r[3], ee = r[4];
                if (dir == 0) {
                    M.nnz_u[src] = (int32_t)gt;
                    M.nz_row_u[src] = (int32_t)(rw + gt - og);
                    if (digests) M.dig_u[src] = r[5];
                }
                if (dir == 1 || lfold) {
                    M.nnz_lc[src] = (int32_t)gt;
                    if (digests) M.dig_lc[src] = r[5];
                }
                if (MODE != 2 && acc_mat != mi) {
                    if (acc_mat >= 0) flush_counters(P.mats[acc_mat].counters, acc);
                    acc_mat = mi;
                }
                acc[0] += (gt - og) * (lfold ? 2 : 1);  // symmetric: L fills = U fills
                acc[3] += r[6];
                if (dir == 0) {
                    acc[1] += ee;
                    acc[2] += vv;
                    acc[4] += gt;
                }
                if (dir == 1 || lfold) acc[5] += gt;
                acc[6] += S.chained ? 1 : 0;
            }
            __syncthreads();
        }
        if constexpr (MODE == 2) {
            // publish this item's results, then count it; the CTA that
            // finishes the request's last item tells the host
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                flush_counters(M.counters, acc);
                __threadfence();
                const unsigned long long d = atomicAdd(P.serve.items_done + M.slot, 1ull) + 1ull;
                if (d == (unsigned long long)M.n_items) {
                    __threadfence_system();
                    *reinterpret_cast<volatile unsigned long long*>(P.serve.done_flags + M.slot) =
                        M.seq;
                }
            }
        }
    }
    if (MODE != 2 && threadIdx.x == 0 && acc_mat >= 0) flush_counters(P.mats[acc_mat].counters, acc);
    if constexpr (MODE == 2) {
        __syncthreads();  // the workspace is no longer in use
        if (threadIdx.x == 0) {
            __threadfence();
            atomicSub(P.serve.alive, 1);
            atomicAnd(P.serve.cta_slots + (SM.cta >> 5), ~(1u << (SM.cta & 31)));
        }
    }
}

template <int BLOCK, int MODE>
static cudaError_t launch_one(const TraverseLaunch& L, int grid, size_t smem, cudaStream_t st) {
    auto k = traverse_kernel<BLOCK, MODE>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(MODE == 0 ? 0 : smem));
    if (e != cudaSuccess) return e;
    k<<<grid, BLOCK, MODE == 0 ? 0 : smem, st>>>(L);
    return cudaGetLastError();
}

template <int BLOCK, int MODE>
static int occ_one(size_t smem) {
    auto k = traverse_kernel<BLOCK, MODE>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(MODE == 0 ? 0 : smem)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, BLOCK, MODE == 0 ? 0 : smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

int traverse_block_sizes(int* sizes, int max_sizes) {
    static const int s[] = {128, 256, 512, 1024};
    int k = 0;
    for (int i = 0; i < 4 && k < max_sizes; i++) sizes[k++] = s[i];
    return k;
}

int traverse_occupancy(int block, bool smem_bitmap, size_t smem) {
#define OCC_CASE(B) \
    case B: return smem_bitmap ? occ_one<B, 1>(smem) : occ_one<B, 0>(smem);
    switch (block) {
        OCC_CASE(128)
        OCC_CASE(256)
        OCC_CASE(512)
        OCC_CASE(1024)
        default: return 0;
    }
#undef OCC_CASE
}

cudaError_t launch_traverse(const TraverseLaunch& L, int block, int grid, bool smem_bitmap,
                            size_t smem, cudaStream_t st) {
#define LAUNCH_CASE(B) \
    case B: return smem_bitmap ? launch_one<B, 1>(L, grid, smem, st) \
                               : launch_one<B, 0>(L, grid, smem, st);
    switch (block) {
        LAUNCH_CASE(128)
        LAUNCH_CASE(256)
        LAUNCH_CASE(512)
        LAUNCH_CASE(1024)
        default: return cudaErrorInvalidValue;
    }
#undef LAUNCH_CASE
}

int serve_occupancy(int block, size_t smem) {
    switch (block) {
        case 256: return occ_one<256, 2>(smem);
        case 512: return occ_one<512, 2>(smem);
        case 1024: return occ_one<1024, 2>(smem);
        default: return 0;
    }
}

cudaError_t launch_serve(const TraverseLaunch& L, int block, int grid, size_t smem,
                         cudaStream_t st) {
    switch (block) {
        case 256: return launch_one<256, 2>(L, grid, smem, st);
        case 512: return launch_one<512, 2>(L, grid, smem, st);
        case 1024: return launch_one<1024, 2>(L, grid, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

// ---- ingest: padded CSR of A and of A^T --------------------------------------
//
// The host computes A's padded row pointers (pad counts in the low 2 bits).
// One warp per row copies the row into its padded slot, writes the padding
// (the row's own id) and counts the entries per column for A^T.

__global__ void gather_rows_kernel(int32_t n, long long nnz_in, const int32_t* __restrict__ beg,
                                   const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ col_in, int32_t* __restrict__ col_out,
                                   int32_t* __restrict__ tcount, int32_t* status) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gw; v < n; v += nwarps) {
        const long long b = beg[v];
        const int r0 = rp[v], r1 = rp[v + 1];
        const long long o = r0 & ~3;
        const long long plen = (long long)(r1 & ~3) - o;
        const long long d = plen - (r1 & 3);
        for (long long j = lane; j < plen; j += 32) {
            if (j >= d) {
                col_out[o + j] = (int32_t)v;
                continue;
            }
            const long long src = b + j;
            // invalid entries become self loops so A^T stays consistent; the
            // status word makes the load fail afterwards
            if (src < 0 || src >= nnz_in) {
                atomicOr(status, DEV_ERR_ROW_RANGE);
                col_out[o + j] = (int32_t)v;
                atomicAdd(&tcount[v], 1);
                continue;
            }
            const int32_t c = col_in[src];
            if (c < 0 || c >= n) {
                atomicOr(status, DEV_ERR_COL_RANGE);
                col_out[o + j] = (int32_t)v;
                atomicAdd(&tcount[v], 1);
                continue;
            }
            col_out[o + j] = c;
            atomicAdd(&tcount[c], 1);
        }
    }
}

// tpad[c] = count rounded up to a multiple of 4 (tpad[n] = 0 for the scan).
__global__ void pad_counts_kernel(int32_t n, const int32_t* __restrict__ tcount,
                                  int32_t* __restrict__ tpad) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c <= n;
         c += (long long)gridDim.x * blockDim.x)
        tpad[c] = c < n ? ((tcount[c] + 3) & ~3) : 0;
}

// After the exclusive scan of tpad into trp: store each row's pad count in
// the low bits of the next row pointer.
__global__ void encode_pads_kernel(int32_t n, const int32_t* __restrict__ tcount,
                                   const int32_t* __restrict__ tpad, int32_t* __restrict__ trp) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        trp[c + 1] |= tpad[c] - tcount[c];
}

__global__ void transpose_scatter_kernel(int32_t n, const int32_t* __restrict__ rp,
                                         const int32_t* __restrict__ col,
                                         const int32_t* __restrict__ trp,
                                         int32_t* __restrict__ tfill, int32_t* __restrict__ tcol) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gw; v < n; v += nwarps) {
        const int r0 = rp[v], r1 = rp[v + 1];
        const int b = r0 & ~3, e = (r1 & ~3) - (r1 & 3);
        for (int j = b + lane; j < e; j += 32) {
            const int c = col[j];
            const int pos = atomicAdd(&tfill[c], 1);
            tcol[(trp[c] & ~3) + pos] = (int32_t)v;
        }
    }
}

// wdeg[w] = total length of A's rows 32w .. 32w+31 (census of full words),
// and the degree bit-planes: bit j of planes[k * nw + w] is bit k of the
// length of row 32w + j, so the degree sum over any set x of word w's
// vertices is sum_k 2^k popc(x & planes[k * nw + w]).
__global__ void word_degree_kernel(int32_t n, const int32_t* __restrict__ rp,
                                   int32_t* __restrict__ wdeg, uint32_t* __restrict__ planes,
                                   int nplanes) {
    const long long nw = ((long long)n + 31) >> 5;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (long long w = gw; w < nw; w += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long v = (w << 5) + lane;
        int d = 0;
        if (v < n) {
            const int r0 = rp[v], r1 = rp[v + 1];
            d = (r1 & ~3) - (r0 & ~3) - (r1 & 3);
        }
        for (int k = 0; k < nplanes; k++) {
            const unsigned b = __ballot_sync(FULL_MASK, (d >> k) & 1);
            if (lane == 0) planes[(long long)k * nw + w] = b;
        }
        int sum = d;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL_MASK, sum, o);
        if (lane == 0) wdeg[w] = sum;
    }
}

// Pattern symmetry check, one warp per row: *asym becomes non-zero as soon
// as an off-diagonal entry (v, w) has no (w, v).  Rows are unsorted, so each
// lane scans row w; the caller skips the check (and marks the matrix
// unsymmetric) when some row is longer than 8192 entries.
__global__ void symmetry_kernel(int32_t n, const int32_t* __restrict__ rp,
                                const int32_t* __restrict__ col, int32_t* asym) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gw; v < n; v += nwarps) {
        if (*reinterpret_cast<volatile int32_t*>(asym)) return;
        const int b = rp[v] & ~3, e = rp[v + 1] & ~3;  // padding entries repeat v
        for (int k = b + lane; k < e; k += 32) {
            const int w = col[k];
            if (w == (int)v) continue;
            const int wb = rp[w] & ~3, we = rp[w + 1] & ~3;
            bool found = false;
            for (int j = wb; j < we && !found; j++) found = col[j] == (int)v;
            if (!found) atomicOr(asym, 1);
        }
    }
}

__global__ void transpose_pad_kernel(int32_t n, const int32_t* __restrict__ tcount,
                                     const int32_t* __restrict__ trp, int32_t* __restrict__ tcol) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int b = trp[c] & ~3, e = trp[c + 1] & ~3;
        for (int j = b + tcount[c]; j < e; j++) tcol[j] = (int32_t)c;
    }
}

// One warp per row: the sum of |v - c| over the row's entries (padding
// entries repeat v and add nothing).
__global__ void index_distance_kernel(int32_t n, const int32_t* __restrict__ rp,
                                      const int32_t* __restrict__ col,
                                      unsigned long long* sum) {
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long acc = 0;
    for (long long v = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int b = rp[v] & ~3, e = rp[v + 1] & ~3;
        for (int j = b + lane; j < e; j += 32) {
            const long long d = (long long)col[j] - v;
            acc += (unsigned long long)(d < 0 ? -d : d);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL_MASK, acc, o);
    if (lane == 0 && acc) atomicAdd(sum, acc);
}

cudaError_t launch_index_distance(int32_t n, const int32_t* rp, const int32_t* col,
                                  unsigned long long* sum, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    long long g = ((long long)n * 32 + 255) / 256;
    index_distance_kernel<<<(int)(g > 148 * 16 ? 148 * 16 : g), 256, 0, stream>>>(n, rp, col, sum);
    return cudaGetLastError();
}

size_t canonicalize_scan_bytes(int32_t n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int32_t*)nullptr, (int32_t*)nullptr,
                                  (int)n + 1);
    return bytes;
}

// rp (A, n+1, encoded) is on the device.  tcount/tfill/tpad: n+1 zeroed ints.
// col_in may equal col_out only when no row moves and no row is padded.
cudaError_t launch_canonicalize(int32_t n, long long nnz_in, const int32_t* beg,
                                const int32_t* col_in, const int32_t* rp, int32_t* col_out,
                                int32_t* tcount, int32_t* tpad, int32_t* trp, int32_t* tcol,
                                int32_t* tfill, int32_t* wdeg, uint32_t* dplanes, int nplanes,
                                int32_t* asym, int check_symmetry, void* scan_tmp,
                                size_t scan_tmp_bytes, int32_t* status, cudaStream_t st) {
    cudaError_t e0 = cudaMemsetAsync(asym, check_symmetry ? 0 : 1, 4, st);
    if (e0 != cudaSuccess) return e0;
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    long long grid_w = ((long long)n * 32 + threads - 1) / threads;
    int grid = (int)(grid_w > 148 * 64 ? 148 * 64 : grid_w);
    long long grid_t = ((long long)n + threads) / threads;
    int gridt = (int)(grid_t > 148 * 16 ? 148 * 16 : grid_t);
    gather_rows_kernel<<<grid, threads, 0, st>>>(n, nnz_in, beg, rp, col_in, col_out, tcount, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pad_counts_kernel<<<gridt, threads, 0, st>>>(n, tcount, tpad);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t bytes = scan_tmp_bytes;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, bytes, tpad, trp, (int)n + 1, st);
    if (e != cudaSuccess) return e;
    encode_pads_kernel<<<gridt, threads, 0, st>>>(n, tcount, tpad, trp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    transpose_scatter_kernel<<<grid, threads, 0, st>>>(n, rp, col_out, trp, tfill, tcol);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    transpose_pad_kernel<<<gridt, threads, 0, st>>>(n, tcount, trp, tcol);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    word_degree_kernel<<<gridt, threads, 0, st>>>(n, rp, wdeg, dplanes, nplanes);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (check_symmetry) {
        symmetry_kernel<<<grid, threads, 0, st>>>(n, rp, col_out, asym);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

// ---- supernodes: segmented compare-and-scan ---------------------------------
//
// Reference rule (SOA :1833-2052, one 128-thread block per group): inside the
// chunk [c*mss, (c+1)*mss) a row r starts a supernode when its offset is a
// multiple of 128 or nz_row_U[r-1] - nz_row_U[r] != 1; any other row extends
// the current start f if L(r,f) != 0 and otherwise adds one supernode while f
// stays the first row.  Segments (runs between forced starts) hold <= 128
// rows, so one warp handles one segment: 4 rows per lane, a warp max-scan
// finds each row's start f, and the L-mask of column f answers L(r,f).
// Inputs are read through L2: in serving they come from a traversal kernel
// that is still running when this one starts.
// One segment (<= 128 rows between forced starts) of one matrix, one warp.
// Returns this lane's count of supernode starts and splits.
__device__ __forceinline__ unsigned long long supernode_segment(
    long long sg, int32_t n, int32_t mss, const int32_t* __restrict__ nzu,
    const uint32_t* __restrict__ lmask, int8_t* __restrict__ flags) {
    const int lane = threadIdx.x & 31;
    const long long segs_per_chunk = ((long long)mss + 127) / 128;
    const long long c = sg / segs_per_chunk;
    const long long k = sg % segs_per_chunk;
    const long long start = c * mss + 128 * k;
    long long stop = start + 128;
    if (stop > (c + 1) * mss) stop = (c + 1) * mss;
    if (stop > n) stop = n;
    if (start >= stop) return 0;
    unsigned long long count = 0;
    int head[4];
    long long last = -1;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const long long r = start + 4 * lane + j;
        head[j] = 0;
        if (r < stop) {
            head[j] = (r == start) || (__ldcg(nzu + r - 1) - __ldcg(nzu + r) != 1);
            if (head[j]) last = r;
        }
    }
    // exclusive max-scan of `last` over lanes
    long long incl = last;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long t = __shfl_up_sync(FULL_MASK, incl, o);
        if (lane >= o && t > incl) incl = t;
    }
    long long f = __shfl_up_sync(FULL_MASK, incl, 1);
    if (lane == 0) f = -1;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const long long r = start + 4 * lane + j;
        if (r >= stop) continue;
        int8_t fl;
        if (head[j]) {
            f = r;
            fl = 1;
            count++;
        } else {
            const long long bit = r - f - 1;  // 0..126
            const uint32_t wv = __ldcg(lmask + 4 * f + (bit >> 5));
            const bool in_l = (wv >> (bit & 31)) & 1u;
            fl = in_l ? 0 : 2;
            if (!in_l) count++;
        }
        if (flags) flags[r] = fl;
    }
    return count;
}

__device__ __forceinline__ long long supernode_segments(int32_t n, int32_t mss) {
    return n <= 0 ? 0 : (((long long)n + mss - 1) / mss) * (((long long)mss + 127) / 128);
}

__global__ void supernode_kernel(int32_t n, int32_t mss, const int32_t* __restrict__ nzu,
                                 const uint32_t* __restrict__ lmask, int8_t* __restrict__ flags,
                                 unsigned long long* counters) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nseg = supernode_segments(n, mss);
    unsigned long long count = 0;
    for (long long sg = gw; sg < nseg; sg += ((long long)gridDim.x * blockDim.x) >> 5)
        count += supernode_segment(sg, n, mss, nzu, lmask, flags);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(FULL_MASK, count, o);
    if (lane == 0 && count) atomicAdd(&counters[CNT_NSUP], count);
}

// All matrices of a batch in one launch: a global segment index is split
// into (matrix, segment) by the per-matrix segment prefix seg_base[].
__global__ void supernode_batch_kernel(const MatDesc* __restrict__ mats, int nmats, int32_t mss,
                                       const long long* __restrict__ seg_base) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long total = seg_base[nmats];
    for (long long g = gw; g < total; g += ((long long)gridDim.x * blockDim.x) >> 5) {
        int lo = 0, hi = nmats - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (seg_base[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const MatDesc& M = mats[lo];
        unsigned long long count =
            supernode_segment(g - seg_base[lo], M.n, mss, M.nz_row_u, M.lmask, M.sflags);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(FULL_MASK, count, o);
        if (lane == 0 && count) atomicAdd(&M.counters[CNT_NSUP], count);
    }
}

// Zeroes the per-matrix counters (and the optional per-row L scatter
// targets) of a batch before its traversal.
__global__ void batch_reset_kernel(const MatDesc* __restrict__ mats, int nmats) {
    for (int mi = blockIdx.x; mi < nmats; mi += gridDim.x) {
        const MatDesc& M = mats[mi];
        if (threadIdx.x < CNT_SLOTS) M.counters[threadIdx.x] = 0ull;
        if (M.nnz_lr) {
            for (long long i = threadIdx.x; i < M.n; i += blockDim.x) {
                M.nnz_lr[i] = 0;
                M.dig_lr[i] = 0ull;
            }
        }
    }
}

cudaError_t launch_batch_reset(const MatDesc* mats, int nmats, cudaStream_t st) {
    if (nmats <= 0) return cudaSuccess;
    batch_reset_kernel<<<nmats < 148 * 8 ? nmats : 148 * 8, 256, 0, st>>>(mats, nmats);
    return cudaGetLastError();
}

cudaError_t launch_supernodes_batch(const MatDesc* mats, int nmats, int32_t mss,
                                    const long long* seg_base, long long total_segments,
                                    cudaStream_t st) {
    if (nmats <= 0 || total_segments <= 0) return cudaSuccess;
    const int threads = 256;
    long long grid = (total_segments * 32 + threads - 1) / threads;
    if (grid > 148 * 32) grid = 148 * 32;
    supernode_batch_kernel<<<(int)grid, threads, 0, st>>>(mats, nmats, mss, seg_base);
    return cudaGetLastError();
}

long long supernode_segment_count(int32_t n, int32_t mss) {
    return n <= 0 ? 0 : (((long long)n + mss - 1) / mss) * (((long long)mss + 127) / 128);
}

cudaError_t launch_supernodes(int32_t n, int32_t mss, const int32_t* nzu, const uint32_t* lmask,
                              int8_t* flags, unsigned long long* counters, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const long long segs = (((long long)n + mss - 1) / mss) * (((long long)mss + 127) / 128);
    const int threads = 256;
    long long grid = (segs * 32 + threads - 1) / threads;
    if (grid > 148 * 32) grid = 148 * 32;
    supernode_kernel<<<(int)grid, threads, 0, st>>>(n, mss, nzu, lmask, flags, counters);
    return cudaGetLastError();
}

// ---- pattern pointers -------------------------------------------------------
__global__ void widen_kernel(int32_t n, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                             int64_t* __restrict__ wa, int64_t* __restrict__ wb) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        wa[i] = i < n ? (int64_t)a[i] : 0;
        wb[i] = i < n ? (int64_t)b[i] : 0;
    }
}

size_t pattern_scan_bytes(int32_t n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int64_t*)nullptr, (int64_t*)nullptr,
                                  (int)n + 1);
    return bytes + 2 * sizeof(int64_t) * ((size_t)n + 1) + 256;
}

cudaError_t launch_pattern_ptrs(int32_t n, const int32_t* nnz_u, const int32_t* nnz_lc,
                                int64_t* uptr, int64_t* lptr, void* scan_tmp,
                                size_t scan_tmp_bytes, cudaStream_t st) {
    int64_t* wa = reinterpret_cast<int64_t*>(scan_tmp);
    int64_t* wb = wa + (n + 1);
    char* tmp = reinterpret_cast<char*>(wb + (n + 1));
    tmp = reinterpret_cast<char*>(((uintptr_t)tmp + 255) & ~(uintptr_t)255);
    size_t bytes = scan_tmp_bytes - (size_t)(tmp - reinterpret_cast<char*>(scan_tmp));
    widen_kernel<<<148 * 4, 256, 0, st>>>(n, nnz_u, nnz_lc, wa, wb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t b1 = bytes;
    e = cub::DeviceScan::ExclusiveSum(tmp, b1, wa, uptr, (int)n + 1, st);
    if (e != cudaSuccess) return e;
    size_t b2 = bytes;
    return cub::DeviceScan::ExclusiveSum(tmp, b2, wb, lptr, (int)n + 1, st);
}

}  // namespace gsofa
