// gsofa_order.cu -- fill-reducing ordering on the device (gsofa_order_nd)
// and the symmetric permutation of a loaded matrix (gsofa_matrix_permute).
//
// The reference receives its matrices already permuted by SuperLU_DIST
// (gSoFaTPDS README.md:27-33) and contains no ordering code.  The ordering
// here is level-set nested dissection of the structure of A + A^T (George,
// SIAM J. Numer. Anal. 10, 1973; George and Liu, "Computer Solution of Large
// Sparse Positive Definite Systems", 1981, ch. 8), fixed to one
// deterministic rule so that its result does not depend on thread timing:
//
//   Every vertex is either placed in a group (a range of final positions
//   holding its members in increasing id order) or active in a part (a
//   vertex set with a range start lo).  Round r, while a vertex is active:
//   1. each part splits into the connected components of the subgraph it
//      induces; a component's root is its smallest id; the components of a
//      part take consecutive ranges from the part's lo in root order;
//   2. a component of at most `leaf` vertices (any component in the last
//      round) is placed as a group at its range start;
//   3. every other component c: BFS from its root; r1 = the smallest id at
//      the largest distance; BFS from r1 gives distances d, eccentricity e
//      and level sizes N_l; m = the smallest l with 2 (N_0+..+N_l) >= |c|,
//      capped at e - 1; the separator S = the level-m vertices with a
//      neighbour at level m + 1 in c; A = the rest of levels <= m, B =
//      levels > m.  S is placed last in c's range, A and B become parts.
//
// Device mapping.  The graph is read where the matrix already keeps it: row
// v of A plus row v of A^T (both padded CSR; padding repeats v).  All parts
// of a round are processed together:
//   components  union-find with hooking of the larger root under the smaller
//               by compare-and-swap and path halving (the ECL-CC scheme:
//               Jaiganesh and Burtscher, HPDC 2018); a tree's root is then
//               its smallest id, whatever order the hooks ran in;
//   ranges      roots keyed (part, root), radix-sorted, sizes exclusive-
//               scanned, each part's first key found by binary search;
//   BFS         parts above 2048 vertices: one cooperative launch per
//               search, all their searches level-synchronous together: warp
//               per frontier vertex, compare-and-swap on the distance,
//               block-local queue flushed with one atomic per block per
//               level, a grid barrier whose wait is bounded (GSOFA_ERR_TIMEOUT
//               past 2 s); smaller parts: the whole search inside one CTA
//               (block barriers only), queued in the part's own slice;
//   levels      per part, level sizes are counted into the part's own slice
//               of a histogram (lo + level < lo + |part|), one warp per part
//               scans it for m and e;
//   final       group keys (lo << 32 | v) radix-sorted give perm.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <vector>

#include "gsofa_host.h"
#include "gsofa_order_ml.h"

using namespace gsofa;
using namespace gsofa::host;

namespace {

#define FULL_MASK 0xffffffffu

constexpr int kThreads = 256;
constexpr int kBfsThreads = 512;
constexpr int kBfsBlocksPerSm = 2;
constexpr int kBlockQueue = 2048;                         // block-local BFS queue entries
constexpr unsigned long long kBarrierLimitNs = 2000000000ull;  // one grid barrier wait
constexpr int kLocalThreads = 512;
constexpr int32_t kLocalMax = 2048;  // parts up to this size search inside one CTA
constexpr int32_t kDefaultLeaf = 32;
constexpr int32_t kDefaultMaxRounds = 512;

struct Graph {
    const int32_t* rp;
    const int32_t* col;
    const int32_t* trp;
    const int32_t* tcol;
};

int grid_for(long long items, int threads) {
    long long g = (items + threads - 1) / threads;
    return (int)std::max(1ll, std::min(g, 148ll * 32));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int warp_sum(int x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
    return x;
}

// ---- connected components ---------------------------------------------------

// Root of x's tree.  Parents only ever point to smaller ids, so the loop
// stops at the root; skipping a node (path halving) keeps every pointer on
// an ancestor, so concurrent finds and hooks stay consistent.
__device__ __forceinline__ int uf_find(int32_t* parent, int x) {
    volatile int32_t* P = parent;
    int cur = P[x];
    if (cur != x) {
        int prev = x, next;
        while (cur > (next = P[cur])) {
            P[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__device__ void uf_union(int32_t* parent, int a, int b) {
    int ra = uf_find(parent, a), rb = uf_find(parent, b);
    while (ra != rb) {
        if (ra < rb) {
            const int t = ra;
            ra = rb;
            rb = t;
        }
        const int old = atomicCAS(parent + ra, ra, rb);  // hook the larger root
        if (old == ra) return;
        ra = uf_find(parent, old);
        rb = uf_find(parent, rb);
    }
}

__global__ void cc_init_kernel(int32_t n, const int32_t* __restrict__ part,
                               int32_t* __restrict__ parent) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (long long)gridDim.x * blockDim.x)
        if (part[v] >= 0) parent[v] = (int32_t)v;
}

// One warp per vertex: every edge {v, w} with w < v inside v's part.
__global__ void cc_hook_kernel(Graph g, int32_t n, const int32_t* __restrict__ part,
                               int32_t* parent) {
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long vv = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; vv < n; vv += nw) {
        const int v = (int)vv;
        const int p = __ldg(part + v);
        if (p < 0) continue;
        for (int side = 0; side < 2; side++) {
            const int32_t* rp = side ? g.trp : g.rp;
            const int32_t* cl = side ? g.tcol : g.col;
            const int b = __ldg(rp + v) & ~3, e = __ldg(rp + v + 1) & ~3;
            for (int j = b + lane; j < e; j += 32) {
                const int w = __ldg(cl + j);
                if (w < v && __ldg(part + w) == p) uf_union(parent, v, w);
            }
        }
    }
}

// root_of[v], component sizes, and one key (part << 32 | root) per root.
__global__ void cc_roots_kernel(int32_t n, const int32_t* __restrict__ part, int32_t* parent,
                                int32_t* __restrict__ root_of, int32_t* __restrict__ csize,
                                unsigned long long* __restrict__ keys, int32_t* nroots) {
    for (long long vv = (long long)blockIdx.x * blockDim.x + threadIdx.x; vv < n;
         vv += (long long)gridDim.x * blockDim.x) {
        const int v = (int)vv;
        const int p = part[v];
        if (p < 0) continue;
        const int r = uf_find(parent, v);
        root_of[v] = r;
        atomicAdd(csize + r, 1);
        if (r == v)
            keys[atomicAdd(nroots, 1)] = ((unsigned long long)(uint32_t)p << 32) | (uint32_t)v;
    }
}

__global__ void comp_sizes_kernel(int R, const unsigned long long* __restrict__ sorted,
                                  const int32_t* __restrict__ csize, int32_t* __restrict__ s) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < R;
         k += (long long)gridDim.x * blockDim.x)
        s[k] = csize[(uint32_t)sorted[k]];
}

// New part k = the k-th root in (old part, root) order; its range starts at
// the old part's lo plus the sizes of the old part's earlier components.
__global__ void new_parts_kernel(int R, const unsigned long long* __restrict__ sorted,
                                 const int32_t* __restrict__ s, const int32_t* __restrict__ excl,
                                 const int32_t* __restrict__ plo_old, int32_t* __restrict__ plo,
                                 int32_t* __restrict__ psize, int32_t* __restrict__ proot,
                                 int32_t* __restrict__ pr1, int32_t* __restrict__ rootidx) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < R;
         k += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = sorted[k];
        const uint32_t p = (uint32_t)(key >> 32);
        const unsigned long long first = (unsigned long long)p << 32;
        long long lo = 0, hi = k;  // first index whose key is >= (p << 32)
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (sorted[mid] < first) lo = mid + 1;
            else hi = mid;
        }
        const int root = (int)(uint32_t)key;
        plo[k] = plo_old[p] + excl[k] - excl[lo];
        psize[k] = s[k];
        proot[k] = root;
        pr1[k] = INT_MAX;
        rootidx[root] = (int32_t)k;
    }
}

// Components of at most `leaf` vertices are placed; the others' vertices
// take their new part id and an unset distance.
__global__ void relabel_kernel(int32_t n, int32_t* __restrict__ part,
                               const int32_t* __restrict__ root_of,
                               const int32_t* __restrict__ rootidx, const int32_t* __restrict__ plo,
                               const int32_t* __restrict__ psize, int32_t leaf,
                               unsigned long long* __restrict__ fkey, int32_t* __restrict__ dist) {
    for (long long vv = (long long)blockIdx.x * blockDim.x + threadIdx.x; vv < n;
         vv += (long long)gridDim.x * blockDim.x) {
        const int v = (int)vv;
        if (part[v] < 0) continue;
        const int k = rootidx[root_of[v]];
        if (psize[k] <= leaf) {
            fkey[v] = ((unsigned long long)(uint32_t)plo[k] << 32) | (uint32_t)v;
            part[v] = -1;
        } else {
            part[v] = k;
            dist[v] = -1;
        }
    }
}

// ---- breadth-first search -----------------------------------------------------

// A source outside [0, n) can only follow a search that gave up (the round
// is then abandoned): it is recorded, not used.
// Seeds the grid-wide search with the parts above max(leaf, local_max).
__global__ void bfs_seed_kernel(int R, int32_t n, const int32_t* __restrict__ psize, int32_t leaf,
                                int32_t local_max, const int32_t* __restrict__ src,
                                const int32_t* __restrict__ plo, int32_t* __restrict__ dist,
                                int32_t* __restrict__ q0, int32_t* lcnt, int32_t* __restrict__ H,
                                int32_t* err) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < R;
         k += (long long)gridDim.x * blockDim.x) {
        if (psize[k] <= leaf || psize[k] <= local_max) continue;
        const int s = src[k];
        if (s < 0 || s >= n) {
            atomicOr(err, 2);
            continue;
        }
        dist[s] = 0;
        q0[atomicAdd(lcnt, 1)] = s;
        H[plo[k]] = 1;
    }
}

struct BfsArgs {
    Graph g;
    const int32_t* part;
    const int32_t* plo;
    int32_t* dist;
    int32_t* q0;
    int32_t* q1;
    int32_t* lcnt;  // frontier size per level (level 0 set by the seed kernel)
    int32_t* H;     // level sizes, part k's level l at plo[k] + l
    unsigned* bar;  // [0] arrivals, [1] generation
    int32_t* err;
    int32_t max_levels;
    unsigned arrivals;             // blocks the barrier waits for (gridDim.x; more only
                                   // in gsofa_order_wait_selftest, so that the wait runs out)
    unsigned long long limit_ns;   // one barrier wait gives up after this
};

// Grid-wide barrier of a cooperative launch (every block is resident) over
// `arrivals` blocks.  The wait gives up after limit_ns or once another block
// has given up; then it sets *err and returns false, and the caller returns.
__device__ bool grid_barrier(unsigned* bar, int32_t* err, unsigned arrivals,
                             unsigned long long limit_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == arrivals - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*gen == g0) {
                if (*reinterpret_cast<volatile int32_t*>(err) || global_ns() - t0 > limit_ns) {
                    atomicOr(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Level-synchronous BFS of every part at once, each inside its own part.
__global__ void __launch_bounds__(kBfsThreads) bfs_kernel(BfsArgs a) {
    __shared__ int32_t sq[kBlockQueue];
    __shared__ int sq_n, sq_base;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    if (threadIdx.x == 0) sq_n = 0;
    __syncthreads();
    for (int L = 0; L < a.max_levels; L++) {
        const int cnt = __ldcg(a.lcnt + L);
        if (cnt == 0) break;
        const int32_t* qin = (L & 1) ? a.q1 : a.q0;
        int32_t* qout = (L & 1) ? a.q0 : a.q1;
        for (long long i = gw; i < cnt; i += nw) {
            const int u = __ldcg(qin + i);
            const int p = __ldg(a.part + u);
            int found = 0;
            for (int side = 0; side < 2; side++) {
                const int32_t* rp = side ? a.g.trp : a.g.rp;
                const int32_t* cl = side ? a.g.tcol : a.g.col;
                const int b = __ldg(rp + u) & ~3, e = __ldg(rp + u + 1) & ~3;
                for (int j = b + lane; j < e; j += 32) {
                    const int w = __ldg(cl + j);
                    if (w == u || __ldg(a.part + w) != p || __ldcg(a.dist + w) >= 0) continue;
                    if (atomicCAS(a.dist + w, -1, L + 1) != -1) continue;
                    found++;
                    const int pos = atomicAdd(&sq_n, 1);
                    if (pos < kBlockQueue) sq[pos] = w;
                    else qout[atomicAdd(a.lcnt + L + 1, 1)] = w;
                }
            }
            found = warp_sum(found);
            if (lane == 0 && found) atomicAdd(a.H + __ldg(a.plo + p) + L + 1, found);
        }
        __syncthreads();
        const int ns = min(sq_n, kBlockQueue);
        if (threadIdx.x == 0 && ns > 0) sq_base = atomicAdd(a.lcnt + L + 1, ns);
        __syncthreads();
        for (int t = threadIdx.x; t < ns; t += blockDim.x) qout[sq_base + t] = sq[t];
        __syncthreads();
        if (threadIdx.x == 0) sq_n = 0;
        if (!grid_barrier(a.bar, a.err, a.arrivals, a.limit_ns)) return;
    }
}

// The search of each part of (leaf, local_max] vertices inside one CTA: no
// grid barrier, one block barrier per level.  The queue is the part's own
// slice q[plo .. plo + size) (parts are disjoint), level sizes go to
// H[plo + level] as in the grid-wide search.
__global__ void __launch_bounds__(kLocalThreads) bfs_local_kernel(
    Graph g, int R, int32_t n, const int32_t* __restrict__ psize, int32_t leaf, int32_t local_max,
    const int32_t* __restrict__ src, const int32_t* __restrict__ plo,
    const int32_t* __restrict__ part, int32_t* dist, int32_t* q, int32_t* __restrict__ H,
    int32_t* err) {
    __shared__ int found;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    constexpr int NW = kLocalThreads / 32;
    for (int k = blockIdx.x; k < R; k += gridDim.x) {
        const int size = psize[k];
        if (size <= leaf || size > local_max) continue;
        const int base = plo[k];
        const int s0 = src[k];
        if (s0 < 0 || s0 >= n) {  // only after a search that gave up
            if (threadIdx.x == 0) atomicOr(err, 2);
            continue;
        }
        if (threadIdx.x == 0) {
            dist[s0] = 0;
            q[base] = s0;
            H[base] = 1;
            found = 0;
        }
        __syncthreads();
        int lb = 0, le = 1;
        for (int L = 0; lb < le; L++) {
            for (int i = lb + warp; i < le; i += NW) {
                const int u = q[base + i];
                for (int side = 0; side < 2; side++) {
                    const int32_t* rp = side ? g.trp : g.rp;
                    const int32_t* cl = side ? g.tcol : g.col;
                    const int b = __ldg(rp + u) & ~3, e = __ldg(rp + u + 1) & ~3;
                    for (int j = b + lane; j < e; j += 32) {
                        const int w = __ldg(cl + j);
                        if (w == u || __ldg(part + w) != k || dist[w] >= 0) continue;
                        if (atomicCAS(dist + w, -1, L + 1) != -1) continue;
                        const int pos = le + atomicAdd(&found, 1);
                        if (pos < size) q[base + pos] = w;
                        else atomicOr(err, 4);  // a part holds at most `size` vertices
                    }
                }
            }
            __syncthreads();
            const int nxt = found;
            __syncthreads();
            if (threadIdx.x == 0) {
                found = 0;
                if (nxt > 0 && le < size) H[base + L + 1] = nxt;
            }
            lb = le;
            le = min(le + nxt, size);
            __syncthreads();
        }
    }
}

// One warp per split part: e = the level where the running count reaches
// |part|; with `second`, also m (first level where twice the running count
// reaches |part|, capped at e - 1), the vertices on levels < m and N_m.
__global__ void level_scan_kernel(int R, const int32_t* __restrict__ psize, int32_t leaf,
                                  const int32_t* __restrict__ plo, const int32_t* __restrict__ H,
                                  int second, int32_t* __restrict__ pecc, int32_t* __restrict__ pm,
                                  int32_t* __restrict__ pa0, int32_t* __restrict__ pnm,
                                  int32_t* err) {
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < R; k += nw) {
        const int size = psize[k];
        if (size <= leaf) continue;
        const int base = plo[k];
        long long carry = 0;
        int m0 = -1, e = -1;
        for (int l0 = 0; e < 0 && l0 < size; l0 += 32) {
            const int l = l0 + lane;
            int x = l < size ? H[base + l] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL_MASK, x, o);
                if (lane >= o) x += y;
            }
            const long long cum = carry + x;
            if (m0 < 0) {
                const unsigned bm = __ballot_sync(FULL_MASK, 2 * cum >= size);
                if (bm) m0 = l0 + __ffs(bm) - 1;
            }
            const unsigned be = __ballot_sync(FULL_MASK, cum == size && l < size);
            if (be) e = l0 + __ffs(be) - 1;
            carry += __shfl_sync(FULL_MASK, x, 31);
        }
        // a connected part of two or more vertices has e >= 1 and m0 >= 0;
        // anything else follows a search that gave up (recorded, not used)
        if (e < 1 || m0 < 0) {
            if (lane == 0) {
                atomicOr(err, 2);
                pecc[k] = 0;
                pm[k] = 0;
                pa0[k] = 0;
                pnm[k] = 0;
            }
            continue;
        }
        if (!second) {
            if (lane == 0) pecc[k] = e;
            continue;
        }
        const int m = min(m0, e - 1);
        int a = 0;
        for (int l = lane; l < m; l += 32) a += H[base + l];
        a = warp_sum(a);
        if (lane == 0) {
            pecc[k] = e;
            pm[k] = m;
            pa0[k] = a;
            pnm[k] = H[base + m];
        }
    }
}

// r1 of each split part (smallest id at the largest distance of the first
// search); distances are cleared for the second search.
__global__ void far_min_kernel(int32_t n, const int32_t* __restrict__ part,
                               int32_t* __restrict__ dist, const int32_t* __restrict__ pecc,
                               int32_t* pr1) {
    for (long long vv = (long long)blockIdx.x * blockDim.x + threadIdx.x; vv < n;
         vv += (long long)gridDim.x * blockDim.x) {
        const int v = (int)vv;
        const int k = part[v];
        if (k < 0) continue;
        if (dist[v] == pecc[k]) atomicMin(pr1 + k, v);
        dist[v] = -1;
    }
}

// One warp per vertex on its part's level m: is it next to level m + 1?
__global__ void separator_kernel(Graph g, int32_t n, const int32_t* __restrict__ part,
                                 const int32_t* __restrict__ dist, const int32_t* __restrict__ pm,
                                 int32_t* __restrict__ sflag, int32_t* pcnts) {
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long vv = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; vv < n; vv += nw) {
        const int v = (int)vv;
        const int k = part[v];
        if (k < 0) continue;
        const int m = pm[k];
        if (dist[v] != m) continue;
        bool any = false;
        for (int side = 0; side < 2 && !any; side++) {
            const int32_t* rp = side ? g.trp : g.rp;
            const int32_t* cl = side ? g.tcol : g.col;
            const int b = __ldg(rp + v) & ~3, e = __ldg(rp + v + 1) & ~3;
            for (int j0 = b; j0 < e && !any; j0 += 32) {
                const int j = j0 + lane;
                bool hit = false;
                if (j < e) {
                    const int w = __ldg(cl + j);
                    hit = part[w] == k && dist[w] == m + 1;
                }
                any = __any_sync(FULL_MASK, hit);
            }
        }
        if (lane == 0) {
            sflag[v] = any ? 1 : 0;
            if (any) atomicAdd(pcnts + k, 1);
        }
    }
}

// The hybrid rule's choice per part (pml[k] = 1: the multilevel split).  A
// multilevel split is used when its separator is smaller than the level-set
// one and leaves both sides non-empty.
__global__ void choose_kernel(int R, const int32_t* __restrict__ psize, int32_t leaf,
                              const int32_t* __restrict__ pcnts, const int32_t* __restrict__ pns,
                              const int32_t* __restrict__ pna, const int32_t* __restrict__ pnb,
                              int32_t* __restrict__ pml) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < R;
         k += (long long)gridDim.x * blockDim.x)
        pml[k] = psize[k] > leaf && pns[k] < pcnts[k] && pna[k] > 0 && pnb[k] > 0 ? 1 : 0;
}

// The split of each part: S placed last in its range, A and B become parts 2k
// and 2k + 1 of the next round.  Level-set split: S = the separator flags on
// level m, A = the rest of levels <= m; multilevel (pml[k]): S = msep, A and B
// by mside.
__global__ void assign_kernel(int32_t n, int32_t* __restrict__ part,
                              const int32_t* __restrict__ dist, const int32_t* __restrict__ pm,
                              const int32_t* __restrict__ sflag, const int32_t* __restrict__ plo,
                              const int32_t* __restrict__ psize, const int32_t* __restrict__ pcnts,
                              unsigned long long* __restrict__ fkey, const int32_t* __restrict__ pml,
                              const int32_t* __restrict__ mside, const int32_t* __restrict__ msep,
                              const int32_t* __restrict__ pns) {
    for (long long vv = (long long)blockIdx.x * blockDim.x + threadIdx.x; vv < n;
         vv += (long long)gridDim.x * blockDim.x) {
        const int v = (int)vv;
        const int k = part[v];
        if (k < 0) continue;
        if (pml && pml[k]) {
            if (msep[v]) {
                const int slo = plo[k] + psize[k] - pns[k];
                fkey[v] = ((unsigned long long)(uint32_t)slo << 32) | (uint32_t)v;
                part[v] = -1;
            } else {
                part[v] = 2 * k + mside[v];
            }
            continue;
        }
        const int d = dist[v], m = pm[k];
        if (d == m && sflag[v]) {
            const int slo = plo[k] + psize[k] - pcnts[k];
            fkey[v] = ((unsigned long long)(uint32_t)slo << 32) | (uint32_t)v;
            part[v] = -1;
        } else {
            part[v] = 2 * k + (d > m ? 1 : 0);
        }
    }
}

// Ranges of the two sides (parts 2k and 2k+1 of the next round) and the
// round's totals: [0] vertices still active, [1] splits, [2] separator
// vertices, [3] largest separator.
__global__ void next_parts_kernel(int R, const int32_t* __restrict__ psize, int32_t leaf,
                                  const int32_t* __restrict__ plo, const int32_t* __restrict__ pa0,
                                  const int32_t* __restrict__ pnm,
                                  const int32_t* __restrict__ pcnts, int32_t* __restrict__ plo_next,
                                  unsigned long long* tot, const int32_t* __restrict__ pml,
                                  const int32_t* __restrict__ pns, const int32_t* __restrict__ pna) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < R;
         k += (long long)gridDim.x * blockDim.x) {
        const int size = psize[k];
        if (size <= leaf) continue;
        const bool ml = pml && pml[k];
        const int s = ml ? pns[k] : pcnts[k];
        const int a = ml ? pna[k] : pa0[k] + pnm[k] - s;
        plo_next[2 * k] = plo[k];
        plo_next[2 * k + 1] = plo[k] + a;
        atomicAdd(tot + 0, (unsigned long long)(size - s));
        atomicAdd(tot + 1, 1ull);
        atomicAdd(tot + 2, (unsigned long long)s);
        atomicMax(tot + 3, (unsigned long long)s);
    }
}

__global__ void low_word_kernel(int32_t n, const unsigned long long* __restrict__ keys,
                                int32_t* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (int32_t)(uint32_t)keys[i];
}

// ---- permutation ----------------------------------------------------------------

__global__ void inverse_kernel(int32_t n, const int32_t* __restrict__ perm,
                               int32_t* __restrict__ iperm) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        iperm[perm[k]] = (int32_t)k;
}

// Row k of the result is row perm[k] of the source: its padded length, its
// pad count and where its entries start in the source's column array.
__global__ void permuted_rows_kernel(int32_t n, const int32_t* __restrict__ rp_old,
                                     const int32_t* __restrict__ perm, int32_t* __restrict__ plen,
                                     int32_t* __restrict__ pads, int32_t* __restrict__ beg) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int v = perm[k];
        const int a = rp_old[v], b = rp_old[v + 1];
        plen[k] = (b & ~3) - (a & ~3);
        pads[k] = b & 3;
        beg[k] = a & ~3;
    }
}

__global__ void encode_rows_kernel(int32_t n, const int32_t* __restrict__ incl,
                                   const int32_t* __restrict__ pads, int32_t* __restrict__ rp) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k <= n;
         k += (long long)gridDim.x * blockDim.x)
        rp[k] = k == 0 ? 0 : (incl[k - 1] | pads[k - 1]);
}

__global__ void rename_kernel(long long count, const int32_t* __restrict__ col,
                              const int32_t* __restrict__ iperm, int32_t* __restrict__ out) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < count;
         j += (long long)gridDim.x * blockDim.x)
        out[j] = iperm[col[j]];
}

int bits_for(long long x) {  // bits to hold values 0..x
    int b = 1;
    while (b < 32 && (1ll << b) <= x) b++;
    return b;
}

int order_impl(gsofa_ctx* ctx, const gsofa_matrix* mat, int32_t leaf, int32_t max_rounds,
               bool hybrid, int32_t* perm, gsofa_order_stats* stats) {
    const int32_t n = mat->n;
    cudaStream_t st = ctx->stream;
    DeviceScratch S(ctx);
    const size_t N = (size_t)n;
    auto i32 = [&](size_t count) { return static_cast<int32_t*>(S.get(4 * count)); };
    auto u64 = [&](size_t count) { return static_cast<unsigned long long*>(S.get(8 * count)); };
    int32_t* part = i32(N);
    int32_t* parent = i32(N);
    int32_t* root_of = i32(N);
    int32_t* csize = i32(N);
    int32_t* rootidx = i32(N);
    int32_t* dist = i32(N);
    int32_t* H = i32(N);
    int32_t* q0 = i32(N);
    int32_t* q1 = i32(N);
    int32_t* lcnt = i32(N + 2);
    int32_t* sflag = i32(N);
    int32_t* s = i32(N);
    int32_t* excl = i32(N);
    int32_t* plo = i32(N);
    int32_t* psize = i32(N);
    int32_t* proot = i32(N);
    int32_t* pr1 = i32(N);
    int32_t* pecc = i32(N);
    int32_t* pm = i32(N);
    int32_t* pa0 = i32(N);
    int32_t* pnm = i32(N);
    int32_t* pcnts = i32(N);
    int32_t* plo_a = i32(2 * N);
    int32_t* plo_b = i32(2 * N);
    int32_t* dperm = i32(N);
    unsigned long long* keys = u64(N);
    unsigned long long* sorted = u64(N);
    unsigned long long* fkey = u64(N);
    // small words: [0] root count, [8..15] barrier + error, [16..] round totals
    int32_t* small = i32(64);
    size_t sort_b = 0, scan_b = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_b, keys, sorted, (int)n, 0, 64, st);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_b, s, excl, (int)n, st);
    void* tmp = S.get(std::max(sort_b, scan_b));
    if (!part || !parent || !root_of || !csize || !rootidx || !dist || !H || !q0 || !q1 || !lcnt ||
        !sflag || !s || !excl || !plo || !psize || !proot || !pr1 || !pecc || !pm || !pa0 ||
        !pnm || !pcnts || !plo_a || !plo_b || !dperm || !keys || !sorted || !fkey || !small || !tmp)
        return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "ordering workspace exceeds the budget");
    // the hybrid rule's multilevel splits (gsofa_order_ml.cu)
    SymGraph Hg;
    int32_t *mside = nullptr, *msep = nullptr, *pns = nullptr, *pna = nullptr, *pnb = nullptr,
            *pml = nullptr;
    if (hybrid) {
        mside = i32(N);
        msep = i32(N);
        pns = i32(N);
        pna = i32(N);
        pnb = i32(N);
        pml = i32(N);
        if (!mside || !msep || !pns || !pna || !pnb || !pml)
            return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "ordering workspace exceeds the budget");
        int rc = sym_graph_build(ctx, S, n, mat->rowptr, mat->col, mat->trowptr, mat->tcol, &Hg);
        if (rc) return rc;
    }
    int32_t* nroots = small;
    unsigned* bar = reinterpret_cast<unsigned*>(small + 8);
    int32_t* err = small + 10;
    unsigned long long* tot = reinterpret_cast<unsigned long long*>(small + 16);
    Graph g{mat->rowptr, mat->col, mat->trowptr, mat->tcol};

    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bfs_kernel, kBfsThreads, 0) !=
            cudaSuccess || occ <= 0)
        return set_err(ctx, GSOFA_ERR_CUDA, "ordering: BFS kernel cannot be resident");
    const int bfs_grid = ctx->sm_count * std::min(occ, kBfsBlocksPerSm);

    cudaEventRecord(ctx->ev0, st);
    cudaMemsetAsync(part, 0, 4 * N, st);
    cudaMemsetAsync(plo_a, 0, 4, st);
    int32_t* plo_old = plo_a;
    int32_t* plo_next = plo_b;
    long long nold = 1;  // part ids of this round are < nold
    long long active = n, rounds = 0, splits = 0, sepv = 0, sepmax = 0;
    const int G = grid_for(n, kThreads);
    const int GW = grid_for(32ll * n, kThreads);
    auto bfs = [&](const int32_t* src, int R, int32_t leaf_eff) -> int {
        cudaMemsetAsync(lcnt, 0, 4 * (N + 2), st);
        cudaMemsetAsync(H, 0, 4 * N, st);
        cudaMemsetAsync(bar, 0, 8, st);
        bfs_seed_kernel<<<grid_for(R, kThreads), kThreads, 0, st>>>(
            R, n, psize, leaf_eff, kLocalMax, src, plo, dist, q0, lcnt, H, err);
        BfsArgs a{g, part, plo, dist, q0, q1, lcnt, H, bar, err, n + 1, (unsigned)bfs_grid,
                  kBarrierLimitNs};
        void* args[] = {&a};
        cudaError_t e = cudaLaunchCooperativeKernel((const void*)bfs_kernel, dim3(bfs_grid),
                                                    dim3(kBfsThreads), args, 0, st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "ordering BFS launch");
        // the smaller parts, one CTA each; q0 is free once the grid-wide search ended
        bfs_local_kernel<<<std::max(1, std::min(R, ctx->sm_count * 4)), kLocalThreads, 0, st>>>(
            g, R, n, psize, leaf_eff, kLocalMax, src, plo, part, dist, q0, H, err);
        return GSOFA_OK;
    };
    cudaMemsetAsync(err, 0, 4, st);
    for (int r = 0; active > 0; r++) {
        // the last permitted round places every component, so active reaches
        // 0 by then; anything else is a failure reported here, not a loop
        if (r >= max_rounds)
            return set_err(ctx, GSOFA_ERR_CUDA, "ordering: vertices left after round %d", r);
        rounds++;
        const int32_t leaf_eff = r == max_rounds - 1 ? INT32_MAX : leaf;
        // 1. components of every part
        cc_init_kernel<<<G, kThreads, 0, st>>>(n, part, parent);
        cc_hook_kernel<<<GW, kThreads, 0, st>>>(g, n, part, parent);
        cudaMemsetAsync(csize, 0, 4 * N, st);
        cudaMemsetAsync(nroots, 0, 4, st);
        cc_roots_kernel<<<G, kThreads, 0, st>>>(n, part, parent, root_of, csize, keys, nroots);
        int32_t hR = 0;
        if (cudaMemcpyAsync(&hR, nroots, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return set_err(ctx, GSOFA_ERR_CUDA, "ordering: component count read-back");
        const int R = hR;
        // 2. ranges of the components
        cub::DeviceRadixSort::SortKeys(tmp, sort_b, keys, sorted, R, 0, 32 + bits_for(nold - 1),
                                       st);
        comp_sizes_kernel<<<grid_for(R, kThreads), kThreads, 0, st>>>(R, sorted, csize, s);
        cub::DeviceScan::ExclusiveSum(tmp, scan_b, s, excl, R, st);
        new_parts_kernel<<<grid_for(R, kThreads), kThreads, 0, st>>>(
            R, sorted, s, excl, plo_old, plo, psize, proot, pr1, rootidx);
        relabel_kernel<<<G, kThreads, 0, st>>>(n, part, root_of, rootidx, plo, psize, leaf_eff,
                                               fkey, dist);
        // 3. split the larger components
        int rc = bfs(proot, R, leaf_eff);
        if (rc) return rc;
        const int GR = grid_for(32ll * R, kThreads);
        level_scan_kernel<<<GR, kThreads, 0, st>>>(R, psize, leaf_eff, plo, H, 0, pecc, pm, pa0,
                                                   pnm, err);
        far_min_kernel<<<G, kThreads, 0, st>>>(n, part, dist, pecc, pr1);
        rc = bfs(pr1, R, leaf_eff);
        if (rc) return rc;
        level_scan_kernel<<<GR, kThreads, 0, st>>>(R, psize, leaf_eff, plo, H, 1, pecc, pm, pa0,
                                                   pnm, err);
        cudaMemsetAsync(pcnts, 0, 4 * (size_t)std::max(R, 1), st);
        separator_kernel<<<GW, kThreads, 0, st>>>(g, n, part, dist, pm, sflag, pcnts);
        if (hybrid) {
            rc = ml_round(ctx, Hg, n, part, R, psize, leaf_eff, mside, msep, pns, pna, pnb);
            if (rc) return rc;
            choose_kernel<<<grid_for(R, kThreads), kThreads, 0, st>>>(R, psize, leaf_eff, pcnts,
                                                                      pns, pna, pnb, pml);
        }
        assign_kernel<<<G, kThreads, 0, st>>>(n, part, dist, pm, sflag, plo, psize, pcnts, fkey,
                                              pml, mside, msep, pns);
        cudaMemsetAsync(tot, 0, 32, st);
        next_parts_kernel<<<grid_for(R, kThreads), kThreads, 0, st>>>(
            R, psize, leaf_eff, plo, pa0, pnm, pcnts, plo_next, tot, pml, pns, pna);
        unsigned long long ht[4] = {0, 0, 0, 0};
        int32_t herr = 0;
        cudaError_t e = cudaGetLastError();  // launch errors of this round
        if (e == cudaSuccess) e = cudaMemcpyAsync(ht, tot, 32, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "ordering round");
        if (herr)
            return set_err(ctx, GSOFA_ERR_TIMEOUT,
                           "ordering: a BFS grid barrier wait gave up (flags %d)", herr);
        active = (long long)ht[0];
        splits += (long long)ht[1];
        sepv += (long long)ht[2];
        sepmax = std::max(sepmax, (long long)ht[3]);
        std::swap(plo_old, plo_next);
        nold = 2ll * R;
    }
    // final positions: group keys in order
    cub::DeviceRadixSort::SortKeys(tmp, sort_b, fkey, sorted, (int)n, 0, 32 + bits_for(n), st);
    low_word_kernel<<<G, kThreads, 0, st>>>(n, sorted, dperm);
    cudaEventRecord(ctx->ev1, st);
    cudaError_t e = cudaMemcpyAsync(perm, dperm, 4 * N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ordering");
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->rounds = (int32_t)rounds;
        stats->splits = (int32_t)splits;
        stats->separator_vertices = sepv;
        stats->max_separator = (int32_t)sepmax;
        stats->reserved = 0;
        stats->ms = ms;
    }
    return GSOFA_OK;
}

}  // namespace

extern "C" int gsofa_order_nd(gsofa_ctx* ctx, const gsofa_matrix* mat, int32_t leaf_size,
                              int32_t max_rounds, int32_t* perm, gsofa_order_stats* stats) {
    if (!ctx || !mat || (mat->n > 0 && !perm)) return GSOFA_ERR_ARG;
    if (mat->ctx != ctx) return set_err(ctx, GSOFA_ERR_ARG, "matrix belongs to another context");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    if (stats) *stats = gsofa_order_stats{};
    if (mat->n == 0) return GSOFA_OK;
    return order_impl(ctx, mat, leaf_size > 0 ? leaf_size : kDefaultLeaf,
                      max_rounds > 0 ? max_rounds : kDefaultMaxRounds, false, perm, stats);
}

extern "C" int gsofa_order_hybrid(gsofa_ctx* ctx, const gsofa_matrix* mat, int32_t leaf_size,
                                  int32_t* perm, gsofa_order_stats* stats) {
    if (!ctx || !mat || (mat->n > 0 && !perm)) return GSOFA_ERR_ARG;
    if (mat->ctx != ctx) return set_err(ctx, GSOFA_ERR_ARG, "matrix belongs to another context");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    if (stats) *stats = gsofa_order_stats{};
    if (mat->n == 0) return GSOFA_OK;
    // no round cap: every round places at least one separator vertex
    return order_impl(ctx, mat, leaf_size > 0 ? leaf_size : kDefaultLeaf, mat->n + 2, true, perm,
                      stats);
}

extern "C" int gsofa_matrix_permute(gsofa_ctx* ctx, const gsofa_matrix* mat, const int32_t* perm,
                                    gsofa_matrix** out) {
    if (!ctx || !mat || !out || (mat->n > 0 && !perm)) return GSOFA_ERR_ARG;
    *out = nullptr;
    if (mat->ctx != ctx) return set_err(ctx, GSOFA_ERR_ARG, "matrix belongs to another context");
    const int32_t n = mat->n;
    {
        std::vector<char> seen((size_t)n, 0);
        for (int32_t k = 0; k < n; k++) {
            const int32_t v = perm[k];
            if (v < 0 || v >= n || seen[(size_t)v])
                return set_err(ctx, GSOFA_ERR_ARG, "perm is not a permutation (entry %d = %d)",
                               k, v);
            seen[(size_t)v] = 1;
        }
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    int32_t rpn = 0;
    if (cudaMemcpyAsync(&rpn, mat->rowptr + n, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "permute: row pointer read-back");
    const int64_t padded = rpn & ~3;
    gsofa_matrix* m = nullptr;
    int rc = matrix_alloc(ctx, st, n, mat->nnz, padded, mat->nplanes, &m);
    if (rc) return rc;
    unsigned long long* wc = nullptr;
    int32_t* dstatus = work_counter_status(ctx, &wc);
    {
        DeviceScratch S(ctx);
        const size_t N = (size_t)std::max(n, 1);
        int32_t* dperm = static_cast<int32_t*>(S.get(4 * N));
        int32_t* iperm = static_cast<int32_t*>(S.get(4 * N));
        int32_t* plen = static_cast<int32_t*>(S.get(4 * N));
        int32_t* pads = static_cast<int32_t*>(S.get(4 * N));
        int32_t* incl = static_cast<int32_t*>(S.get(4 * N));
        int32_t* dbeg = static_cast<int32_t*>(S.get(4 * N));
        int32_t* cols = static_cast<int32_t*>(S.get(4 * (size_t)std::max<int64_t>(padded, 1)));
        size_t scan_b = 0;
        cub::DeviceScan::InclusiveSum(nullptr, scan_b, plen, incl, (int)n, st);
        void* tmp = S.get(scan_b);
        if (!dperm || !iperm || !plen || !pads || !incl || !dbeg || !cols || !tmp) {
            matrix_free_on(m, st);
            return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "permute workspace exceeds the budget");
        }
        cudaError_t e = cudaMemsetAsync(ctx->small, 0, 128, st);
        if (e == cudaSuccess && n > 0)
            e = cudaMemcpyAsync(dperm, perm, 4 * (size_t)n, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            matrix_free_on(m, st);
            return cuda_fail(ctx, e, "permute upload");
        }
        const int G = grid_for(n, kThreads);
        if (n > 0) {
            inverse_kernel<<<G, kThreads, 0, st>>>(n, dperm, iperm);
            permuted_rows_kernel<<<G, kThreads, 0, st>>>(n, mat->rowptr, dperm, plen, pads, dbeg);
            cub::DeviceScan::InclusiveSum(tmp, scan_b, plen, incl, (int)n, st);
            rename_kernel<<<grid_for(padded, kThreads), kThreads, 0, st>>>(padded, mat->col, iperm,
                                                                           cols);
        }
        encode_rows_kernel<<<grid_for((long long)n + 1, kThreads), kThreads, 0, st>>>(n, incl, pads,
                                                                                      m->rowptr);
        rc = matrix_build(ctx, st, dstatus, m, padded, dbeg, cols, 0);
        if (rc) {
            matrix_free_on(m, st);
            return rc;
        }
        // P A P^T is symmetric exactly when A is
        e = cudaMemcpyAsync(m->asym, mat->asym, 4, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->h_status, dstatus, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            matrix_free_on(m, st);
            return cuda_fail(ctx, e, "permute");
        }
    }
    rc = check_status(ctx);
    if (rc) {
        matrix_free_on(m, st);
        return rc;
    }
    *out = m;
    return GSOFA_OK;
}

// The grid barrier's bounded wait, exercised on the device: the BFS kernel
// runs on a two-vertex graph with no edges, waiting at its first barrier for
// one block more than the launch has.  Every block's wait runs out after
// limit_ms; the kernel returns and GSOFA_ERR_TIMEOUT is reported, and the
// context stays usable.
extern "C" int gsofa_order_wait_selftest(gsofa_ctx* ctx, double limit_ms) {
    if (!ctx || !(limit_ms > 0.0) || limit_ms > 2000.0) return GSOFA_ERR_ARG;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    DeviceScratch S(ctx);
    // rp, trp: 3 zeros (two empty rows); col: 4 ints; part, dist, q0, q1, plo,
    // H: 2 each; lcnt 4; bar 2 words; err 1
    int32_t* w = static_cast<int32_t*>(S.get(4 * 64));
    if (!w) return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "self-test workspace");
    int32_t h[64];
    for (int i = 0; i < 64; i++) h[i] = 0;
    int32_t *rp = w, *col = w + 4, *part = w + 8, *dist = w + 12, *q0 = w + 16, *q1 = w + 20,
            *plo = w + 24, *H = w + 28, *lcnt = w + 32, *err = w + 40;
    unsigned* bar = reinterpret_cast<unsigned*>(w + 44);
    h[12] = 0;   // dist[0] = 0 (the source)
    h[13] = -1;  // dist[1] unseen
    h[32] = 1;   // lcnt[0]: one frontier vertex, q0[0] = 0
    cudaError_t e = cudaMemcpyAsync(w, h, sizeof(h), cudaMemcpyHostToDevice, st);
    int occ = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bfs_kernel, kBfsThreads, 0);
    if (e != cudaSuccess || occ <= 0) return set_err(ctx, GSOFA_ERR_CUDA, "self-test setup");
    const int grid = ctx->sm_count * std::min(occ, kBfsBlocksPerSm);
    Graph g{rp, col, rp, col};
    BfsArgs a{g, part, plo, dist, q0, q1, lcnt, H, bar, err, 3, (unsigned)grid + 1u,
              (unsigned long long)(limit_ms * 1e6)};
    void* args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void*)bfs_kernel, dim3(grid), dim3(kBfsThreads), args,
                                    0, st);
    int32_t herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "self-test");
    if (herr) return set_err(ctx, GSOFA_ERR_TIMEOUT, "grid barrier wait gave up (as intended)");
    return GSOFA_OK;
}
