// gsofa_order_ml.cu -- the multilevel bisection of the hybrid ordering
// (gsofa_order_hybrid), for every part of one nested-dissection round at once.
//
// The hybrid rule is level-set nested dissection (gsofa_order.cu) with one
// change at each split: a second, multilevel separator is computed for the
// component, and the smaller of the two is used (ties: the level-set one).
// Every step is fixed so that the result does not depend on thread timing,
// and the CPU oracle (oracle/gsofa_order_hybrid_oracle.c, or_order_hybrid)
// restates the same steps one component at a time:
//
//   graph      the component's subgraph of A + A^T: distinct neighbours,
//              sorted by id, unit edge and vertex weights; local ids follow
//              increasing global id.
//   coarsen    while the graph has more than 200 vertices: three rounds of
//              mutual proposals (every unmatched vertex proposes to its
//              unmatched neighbour of largest edge weight, ties the largest
//              id; a pair matches when its two proposals meet); coarse ids
//              in increasing order of each pair's smaller member; edge and
//              vertex weights summed, neighbours sorted by coarse id.  Stop
//              when a level keeps more than 95 % of its vertices.
//   bisect     the coarsest graph by BFS growth: from the last vertex of a
//              BFS started at the last vertex of a BFS from vertex 0,
//              vertices join side 0 in BFS order (neighbours in id order)
//              until it holds half the weight.
//   refine     at every level (the coarsest included, then after each
//              projection): up to 10 passes; gain = (edge weight to the
//              other side) - (to its own side); a vertex with positive gain
//              larger than every neighbour's (ties: the smaller id wins) is
//              a candidate; candidates are taken in increasing id, each
//              moved only if side 0's weight stays within 40..60 % of the
//              total (the others are skipped).
//   separator  the boundary vertices (with a neighbour on the other side) of
//              the side that has fewer of them (ties: side 0).
//
// Device mapping.  The parts of a round are laid out one after another in a
// level-0 index space (a part's vertices in increasing id); every level keeps
// that layout for the parts still present, so a part is a contiguous range
// and per-part work is a segmented scan, sort or reduction:
//   matching     one thread per vertex per proposal round;
//   coarse ids   an exclusive scan of the "pair's smaller member" flags;
//   contraction  64-bit (coarse u, coarse w) keys radix-sorted with their
//                weights and reduced by key: the coarse CSR, rows sorted;
//   BFS order    parts of up to 256 vertices: one thread each, a plain
//                sequential BFS; larger parts: one CTA each, level by level
//                with block barriers, each new vertex appended by its first
//                parent in queue order (the smallest queue position among its
//                frontier neighbours) at an offset from a block scan, in
//                adjacency order: exactly the queue order of a sequential BFS
//                that visits neighbours in id order;
//   refinement   gains and candidates one thread per vertex; candidates
//                compacted in increasing id; then one thread per part
//                accepts them in order against the balance bounds (the one
//                sequential step; a pass has few candidates).
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "gsofa_host.h"
#include "gsofa_order_ml.h"

using namespace gsofa;
using namespace gsofa::host;

namespace {

constexpr int kT = 256;
constexpr int32_t kCoarsenMin = 200;   // graphs of at most this many vertices are not coarsened
constexpr int kMatchRounds = 3;
constexpr int kRefinePasses = 10;
constexpr unsigned long long kNoKey = ~0ull;
// parts of at most this many vertices are searched by one thread each (a
// plain sequential BFS, all such parts at once); larger ones by one CTA each
constexpr int32_t kSeqBfsMax = 256;
constexpr int kCtaBfsThreads = 1024;

int blocks_for(long long items) {
    long long g = (items + kT - 1) / kT;
    return (int)std::max(1ll, std::min(g, 148ll * 64));
}

#define GRID_LOOP(i, count) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (count); \
         i += (long long)gridDim.x * blockDim.x)

// ---- A + A^T: distinct sorted neighbours, no self loops -------------------------

// keys (v << 32 | w) for the entries of row v of A and of A^T, w != v;
// padding (which repeats v) and loops become kNoKey
__global__ void sym_keys_kernel(int32_t n, const int32_t* __restrict__ rp,
                                const int32_t* __restrict__ col, const int32_t* __restrict__ trp,
                                const int32_t* __restrict__ tcol, long long tbase,
                                unsigned long long* __restrict__ keys) {
    GRID_LOOP(vv, n) {
        const int v = (int)vv;
        for (int side = 0; side < 2; side++) {
            const int32_t* r = side ? trp : rp;
            const int32_t* c = side ? tcol : col;
            const long long off = side ? tbase : 0;
            const int b = r[v] & ~3, e = r[v + 1] & ~3;
            for (int j = b; j < e; j++) {
                const int w = c[j];
                keys[off + j] = w == v ? kNoKey : (((unsigned long long)(uint32_t)v << 32) | (uint32_t)w);
            }
        }
    }
}

// first occurrence of each valid key: flag 1
__global__ void unique_flags_kernel(long long m, const unsigned long long* __restrict__ s,
                                    int32_t* __restrict__ flag, int32_t* __restrict__ deg) {
    GRID_LOOP(i, m) {
        const unsigned long long k = s[i];
        const int f = k != kNoKey && (i == 0 || s[i - 1] != k);
        flag[i] = f;
        if (f) atomicAdd(deg + (int)(k >> 32), 1);
    }
}

__global__ void unique_scatter_kernel(long long m, const unsigned long long* __restrict__ s,
                                      const int32_t* __restrict__ flag,
                                      const int32_t* __restrict__ pos, int32_t* __restrict__ adj) {
    GRID_LOOP(i, m) {
        if (flag[i]) adj[pos[i]] = (int32_t)(uint32_t)s[i];
    }
}

// ---- level 0: the parts' induced subgraphs ---------------------------------------

// the active vertices (part >= 0) keyed (part << 32 | v)
__global__ void active_keys_kernel(int32_t n, const int32_t* __restrict__ part,
                                   unsigned long long* __restrict__ keys, int32_t* cnt) {
    GRID_LOOP(vv, n) {
        const int v = (int)vv;
        const int k = part[v];
        if (k >= 0) keys[atomicAdd(cnt, 1)] = ((unsigned long long)(uint32_t)k << 32) | (uint32_t)v;
    }
}

__global__ void level0_ids_kernel(long long V, const unsigned long long* __restrict__ sorted,
                                  int32_t* __restrict__ xid, int32_t* __restrict__ lidx,
                                  int32_t* __restrict__ vpart, int32_t* __restrict__ vw) {
    GRID_LOOP(x, V) {
        const unsigned long long k = sorted[x];
        const int v = (int)(uint32_t)k;
        xid[x] = v;
        lidx[v] = (int32_t)x;
        vpart[x] = (int32_t)(k >> 32);
        vw[x] = 1;
    }
}

// neighbours of xid[x] inside its part (pass 0: count; pass 1: write)
__global__ void level0_adj_kernel(long long V, const int32_t* __restrict__ hrp,
                                  const int32_t* __restrict__ hadj, const int32_t* __restrict__ part,
                                  const int32_t* __restrict__ xid, const int32_t* __restrict__ lidx,
                                  int32_t* __restrict__ deg, const int32_t* __restrict__ xadj,
                                  int32_t* __restrict__ adj, int32_t* __restrict__ ew) {
    GRID_LOOP(x, V) {
        const int v = xid[x];
        const int k = part[v];
        int c = 0;
        const int b = hrp[v], e = hrp[v + 1];
        const int o = xadj ? xadj[x] : 0;
        for (int j = b; j < e; j++) {
            const int w = hadj[j];
            if (part[w] != k) continue;
            if (xadj) {
                adj[o + c] = lidx[w];
                ew[o + c] = 1;
            }
            c++;
        }
        if (!xadj) deg[x] = c;
    }
}

// ---- coarsening -------------------------------------------------------------------

__global__ void propose_kernel(long long V, const int32_t* __restrict__ xadj,
                               const int32_t* __restrict__ adj, const int32_t* __restrict__ ew,
                               const int32_t* __restrict__ vpart, const int32_t* __restrict__ pn,
                               const int32_t* __restrict__ match, int32_t* __restrict__ prop) {
    GRID_LOOP(x, V) {
        int best = -1, bw = -1;
        if (match[x] < 0 && pn[vpart[x]] > kCoarsenMin) {
            for (int j = xadj[x]; j < xadj[x + 1]; j++) {
                const int y = adj[j];
                if (match[y] >= 0) continue;
                const int w = ew[j];
                if (w > bw || (w == bw && y > best)) {
                    bw = w;
                    best = y;
                }
            }
        }
        prop[x] = best;
    }
}

__global__ void resolve_kernel(long long V, const int32_t* __restrict__ prop, int32_t* match) {
    GRID_LOOP(x, V) {
        const int y = prop[x];
        if (y > x && prop[y] == (int)x) {
            match[x] = y;
            match[y] = (int32_t)x;
        }
    }
}

// rep[x] = 1 when x keeps a coarse vertex of its own (unmatched, or the
// smaller member of its pair); parts that are not coarsened count nothing
__global__ void rep_kernel(long long V, const int32_t* __restrict__ match,
                           const int32_t* __restrict__ vpart, const int32_t* __restrict__ pn,
                           int32_t* __restrict__ rep) {
    GRID_LOOP(x, V) {
        const int m = match[x];
        rep[x] = pn[vpart[x]] > kCoarsenMin && (m < 0 || m > x) ? 1 : 0;
    }
}

// per part: coarse vertices nc, whether it goes on (cont), its coarsest level
__global__ void coarsen_decide_kernel(int R, const int32_t* __restrict__ pb,
                                      const int32_t* __restrict__ pn,
                                      const int32_t* __restrict__ rscan, int level,
                                      int32_t* __restrict__ pn_next, int32_t* __restrict__ clev) {
    GRID_LOOP(k, R) {
        const int size = pn[k];
        int next = 0;
        if (size > 0) {
            const int nc = rscan[pb[k] + size] - rscan[pb[k]];
            if (size > kCoarsenMin && (long long)nc * 100 <= (long long)size * 95) next = nc;
            else clev[k] = level;
        }
        pn_next[k] = next;
    }
}

__global__ void cmap_kernel(long long V, const int32_t* __restrict__ match,
                            const int32_t* __restrict__ vpart, const int32_t* __restrict__ pb,
                            const int32_t* __restrict__ pn_next, const int32_t* __restrict__ pb_next,
                            const int32_t* __restrict__ rscan, const int32_t* __restrict__ vw,
                            int32_t* __restrict__ cmap, int32_t* __restrict__ vw_next,
                            int32_t* __restrict__ vpart_next) {
    GRID_LOOP(x, V) {
        const int k = vpart[x];
        if (pn_next[k] == 0) {
            cmap[x] = -1;
            continue;
        }
        const int m = match[x];
        const int r = (m >= 0 && m < x) ? m : (int)x;  // the pair's smaller member
        const int c = pb_next[k] + rscan[r] - rscan[pb[k]];
        cmap[x] = c;
        if (r == x) {
            vw_next[c] = vw[x] + (m > x ? vw[m] : 0);
            vpart_next[c] = k;
        }
    }
}

__global__ void coarse_keys_kernel(long long V, const int32_t* __restrict__ xadj,
                                   const int32_t* __restrict__ adj, const int32_t* __restrict__ ew,
                                   const int32_t* __restrict__ cmap,
                                   unsigned long long* __restrict__ keys, int32_t* __restrict__ vals) {
    GRID_LOOP(x, V) {
        const int cx = cmap[x];
        for (int j = xadj[x]; j < xadj[x + 1]; j++) {
            const int cy = cx >= 0 ? cmap[adj[j]] : cx;
            if (cx < 0 || cy == cx) {
                keys[j] = kNoKey;
                vals[j] = 0;
            } else {
                keys[j] = ((unsigned long long)(uint32_t)cx << 32) | (uint32_t)cy;
                vals[j] = ew[j];
            }
        }
    }
}

__global__ void coarse_rows_kernel(long long m, const unsigned long long* __restrict__ ukeys,
                                   int32_t* __restrict__ deg, int32_t* __restrict__ adj) {
    GRID_LOOP(i, m) {
        const unsigned long long k = ukeys[i];
        atomicAdd(deg + (int)(k >> 32), 1);
        adj[i] = (int32_t)(uint32_t)k;
    }
}

// ---- breadth-first search in exact queue order ---------------------------------

// one thread per part: the sequential BFS from start[k], its queue in qord
__global__ void seq_bfs_kernel(int R, const int32_t* __restrict__ on,
                               const int32_t* __restrict__ start, const int32_t* __restrict__ pb,
                               const int32_t* __restrict__ pn, const int32_t* __restrict__ xadj,
                               const int32_t* __restrict__ adj, int32_t* __restrict__ lev,
                               int32_t* __restrict__ qord, int32_t* __restrict__ cnt) {
    GRID_LOOP(k, R) {
        if (!on[k]) continue;
        const int base = pb[k], size = pn[k];
        for (int i = base; i < base + size; i++) lev[i] = -1;
        const int s = start[k];
        qord[base] = s;
        lev[s] = 0;
        int h = 0, t = 1;
        while (h < t) {
            const int u = qord[base + h++];
            for (int j = xadj[u]; j < xadj[u + 1]; j++) {
                const int y = adj[j];
                if (lev[y] == -1 && t < size) {
                    lev[y] = 0;
                    qord[base + t++] = y;
                }
            }
        }
        cnt[k] = t;
    }
}

// One CTA per part: the BFS from start[k] with its queue (qord) in exactly
// the order a sequential BFS visiting neighbours in id order produces.  Per
// level, every unvisited neighbour of the frontier keeps the smallest queue
// position of a frontier vertex next to it (its first parent); each frontier
// vertex counts the neighbours it won, a block scan over the frontier in
// queue order gives each its offset, and it appends them in adjacency order.
// Block barriers only; the loop ends when a level adds nothing.
__global__ void __launch_bounds__(kCtaBfsThreads) cta_bfs_kernel(
    int R, const int32_t* __restrict__ on, const int32_t* __restrict__ start,
    const int32_t* __restrict__ pb, const int32_t* __restrict__ pn,
    const int32_t* __restrict__ xadj, const int32_t* __restrict__ adj, int32_t* lev,
    int32_t* par, int32_t* __restrict__ qord, int32_t* __restrict__ cnt) {
    typedef cub::BlockScan<int, kCtaBfsThreads> Scan;
    __shared__ typename Scan::TempStorage scan;
    for (int k = blockIdx.x; k < R; k += gridDim.x) {
        if (!on[k]) continue;
        const int base = pb[k], size = pn[k];
        for (int i = base + threadIdx.x; i < base + size; i += blockDim.x) {
            lev[i] = -1;
            par[i] = INT_MAX;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int s = start[k];
            qord[base] = s;
            lev[s] = 0;
        }
        __syncthreads();
        int h = 0, t = 1, level = 0;
        while (h < t) {
            for (int i = h + threadIdx.x; i < t; i += blockDim.x) {
                const int u = qord[base + i];
                for (int j = xadj[u]; j < xadj[u + 1]; j++) {
                    const int y = adj[j];
                    if (lev[y] == -1) atomicMin(par + y, i);
                }
            }
            __syncthreads();
            int tt = t;
            for (int c0 = h; c0 < t; c0 += blockDim.x) {
                const int i = c0 + threadIdx.x;
                int mine = 0;
                if (i < t) {
                    const int u = qord[base + i];
                    for (int j = xadj[u]; j < xadj[u + 1]; j++) {
                        const int y = adj[j];
                        mine += lev[y] == -1 && par[y] == i;
                    }
                }
                int off = 0, total = 0;
                Scan(scan).ExclusiveSum(mine, off, total);
                if (i < t && mine) {
                    const int u = qord[base + i];
                    int o = tt + off;
                    for (int j = xadj[u]; j < xadj[u + 1]; j++) {
                        const int y = adj[j];
                        if (lev[y] == -1 && par[y] == i && o < size) {
                            qord[base + o++] = y;
                            lev[y] = level + 1;
                        }
                    }
                }
                tt += total;
                __syncthreads();  // scan storage reuse; this chunk's marks are visible
            }
            h = t;
            t = tt < size ? tt : size;
            level++;
        }
        if (threadIdx.x == 0) cnt[k] = t;
        __syncthreads();
    }
}

// a searched part whose queue did not reach every vertex (never for the
// connected parts this file is given): recorded
__global__ void bfs_check_kernel(int R, const int32_t* __restrict__ on,
                                 const int32_t* __restrict__ pn, const int32_t* __restrict__ cnt,
                                 int32_t* err) {
    GRID_LOOP(k, R) {
        if (on[k] && cnt[k] != pn[k]) atomicOr(err, 1);
    }
}

__global__ void last_of_queue_kernel(int R, const int32_t* __restrict__ on,
                                     const int32_t* __restrict__ pb, const int32_t* __restrict__ pn,
                                     const int32_t* __restrict__ qord, int32_t* __restrict__ start) {
    GRID_LOOP(k, R) {
        if (on[k]) start[k] = qord[pb[k] + pn[k] - 1];
    }
}

__global__ void first_of_part_kernel(int R, const int32_t* __restrict__ on,
                                     const int32_t* __restrict__ pb, int32_t* __restrict__ start) {
    GRID_LOOP(k, R) {
        if (on[k]) start[k] = pb[k];
    }
}

// weights in queue order (for the growth's prefix sums)
__global__ void queue_weights_kernel(long long V, const int32_t* __restrict__ vpart,
                                     const int32_t* __restrict__ on, const int32_t* __restrict__ qord,
                                     const int32_t* __restrict__ pb, const int32_t* __restrict__ vw,
                                     long long* __restrict__ wq) {
    GRID_LOOP(i, V) {
        // position i belongs to the part whose range holds it; qord[i] is a
        // vertex of that part when the part was searched
        const int k = vpart[i];  // parts are contiguous: vertex i and position i share a part
        wq[i] = on[k] ? (long long)vw[qord[i]] : 0;
    }
}

// side 0 = the queue prefix popped while 2 * (weight so far) < total
__global__ void growth_side_kernel(long long V, const int32_t* __restrict__ vpart,
                                   const int32_t* __restrict__ on, const int32_t* __restrict__ pb,
                                   const int32_t* __restrict__ qord,
                                   const long long* __restrict__ wscan,
                                   const long long* __restrict__ ptotal, int32_t* __restrict__ side) {
    GRID_LOOP(i, V) {
        const int k = vpart[i];
        if (!on[k]) continue;
        const long long before = wscan[i] - wscan[pb[k]];
        side[qord[i]] = 2 * before < ptotal[k] ? 0 : 1;
    }
}

// ---- refinement -------------------------------------------------------------------

__global__ void part_weights_kernel(long long V, const int32_t* __restrict__ vpart,
                                    const int32_t* __restrict__ vw, const int32_t* __restrict__ side,
                                    long long* __restrict__ ptotal, long long* __restrict__ pw0) {
    GRID_LOOP(x, V) {
        const int k = vpart[x];
        atomicAdd(reinterpret_cast<unsigned long long*>(ptotal + k), (unsigned long long)vw[x]);
        if (side && side[x] == 0)
            atomicAdd(reinterpret_cast<unsigned long long*>(pw0 + k), (unsigned long long)vw[x]);
    }
}

__global__ void gain_kernel(long long V, const int32_t* __restrict__ xadj,
                            const int32_t* __restrict__ adj, const int32_t* __restrict__ ew,
                            const int32_t* __restrict__ vpart, const int32_t* __restrict__ done,
                            const int32_t* __restrict__ side, int32_t* __restrict__ gain) {
    GRID_LOOP(x, V) {
        if (done[vpart[x]]) continue;
        const int s = side[x];
        int g = 0;
        for (int j = xadj[x]; j < xadj[x + 1]; j++) g += side[adj[j]] != s ? ew[j] : -ew[j];
        gain[x] = g;
    }
}

__global__ void cand_kernel(long long V, const int32_t* __restrict__ xadj,
                            const int32_t* __restrict__ adj, const int32_t* __restrict__ vpart,
                            const int32_t* __restrict__ done, const int32_t* __restrict__ gain,
                            int32_t* __restrict__ cand, int32_t* __restrict__ ccount) {
    GRID_LOOP(x, V) {
        const int k = vpart[x];
        int c = 0;
        if (!done[k]) {
            const int g = gain[x];
            if (g > 0) {
                c = 1;
                for (int j = xadj[x]; j < xadj[x + 1] && c; j++) {
                    const int y = adj[j];
                    const int gy = gain[y];
                    if (gy > g || (gy == g && y < x)) c = 0;
                }
            }
        }
        cand[x] = c;
        if (c) atomicAdd(ccount + k, 1);
    }
}

// one thread per part: its candidates in increasing id, each moved when
// side 0's weight stays within 40..60 % of the total
__global__ void accept_kernel(int R, const int32_t* __restrict__ cstart,
                              const int32_t* __restrict__ ccount, const int32_t* __restrict__ clist,
                              const int32_t* __restrict__ vw, const long long* __restrict__ ptotal,
                              long long* __restrict__ pw0, int32_t* __restrict__ side,
                              int32_t* __restrict__ done, int32_t* any_moved) {
    GRID_LOOP(k, R) {
        if (done[k]) continue;
        const long long total = ptotal[k];
        long long w0 = pw0[k];
        int moved = 0;
        const int b = cstart[k], e = b + ccount[k];
        for (int i = b; i < e; i++) {
            const int x = clist[i];
            const long long nw0 = side[x] ? w0 + vw[x] : w0 - vw[x];
            if (nw0 * 100 < total * 40 || nw0 * 100 > total * 60) continue;
            side[x] ^= 1;
            w0 = nw0;
            moved++;
        }
        pw0[k] = w0;
        if (!moved) done[k] = 1;
        else *any_moved = 1;
    }
}

__global__ void project_kernel(long long V, const int32_t* __restrict__ cmap,
                               const int32_t* __restrict__ side_next, int32_t* __restrict__ side) {
    GRID_LOOP(x, V) {
        const int c = cmap[x];
        if (c >= 0) side[x] = side_next[c];
    }
}

// ---- the separator ------------------------------------------------------------------

__global__ void boundary_kernel(long long V, const int32_t* __restrict__ xadj,
                                const int32_t* __restrict__ adj, const int32_t* __restrict__ vpart,
                                const int32_t* __restrict__ side, int32_t* __restrict__ isb,
                                int32_t* __restrict__ bnd) {
    GRID_LOOP(x, V) {
        const int s = side[x];
        int b = 0;
        for (int j = xadj[x]; j < xadj[x + 1] && !b; j++) b = side[adj[j]] != s;
        isb[x] = b;
        if (b) atomicAdd(bnd + 2 * vpart[x] + s, 1);
    }
}

__global__ void ml_result_kernel(long long V, const int32_t* __restrict__ xid,
                                 const int32_t* __restrict__ vpart, const int32_t* __restrict__ side,
                                 const int32_t* __restrict__ isb, const int32_t* __restrict__ bnd,
                                 int32_t* __restrict__ mside, int32_t* __restrict__ msep,
                                 int32_t* __restrict__ pna, int32_t* __restrict__ pnb) {
    GRID_LOOP(x, V) {
        const int k = vpart[x];
        const int small = bnd[2 * k] <= bnd[2 * k + 1] ? 0 : 1;
        const int s = side[x];
        const int sep = isb[x] && s == small;
        const int v = xid[x];
        mside[v] = s;
        msep[v] = sep;
        if (!sep) atomicAdd(s ? pnb + k : pna + k, 1);
    }
}

__global__ void ml_sizes_kernel(int R, const int32_t* __restrict__ bnd, int32_t* __restrict__ pns) {
    GRID_LOOP(k, R) {
        const int b0 = bnd[2 * k], b1 = bnd[2 * k + 1];
        pns[k] = b0 <= b1 ? b0 : b1;
    }
}

// ---- host helpers ---------------------------------------------------------------------

struct Level {
    long long V = 0;
    long long E = 0;
    int32_t* xadj = nullptr;
    int32_t* adj = nullptr;
    int32_t* ew = nullptr;
    int32_t* vw = nullptr;
    int32_t* vpart = nullptr;
    int32_t* pb = nullptr;   // per part: first vertex at this level
    int32_t* pn = nullptr;   // per part: vertices at this level (0 = absent)
    int32_t* cmap = nullptr; // to the next level (-1: the part stops here)
    int32_t* side = nullptr;
};

// cub temporary storage that grows on demand (stream-ordered frees)
struct Temp {
    DeviceScratch* S;
    void* p = nullptr;
    size_t bytes = 0;
    void* need(size_t b) {
        if (b <= bytes) return p;
        p = S->get(b);
        bytes = p ? b : 0;
        return p;
    }
};

int fail(gsofa_ctx* ctx, const char* what) {
    return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "hybrid ordering workspace: %s", what);
}

}  // namespace

namespace gsofa {
namespace host {

int sym_graph_build(gsofa_ctx* ctx, DeviceScratch& S, int32_t n, const int32_t* rp,
                    const int32_t* col, const int32_t* trp, const int32_t* tcol, SymGraph* out) {
    cudaStream_t st = ctx->stream;
    int32_t h[2] = {0, 0};
    if (cudaMemcpyAsync(&h[0], rp + n, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&h[1], trp + n, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "hybrid ordering: row pointer read-back");
    const long long pa = h[0] & ~3, pt = h[1] & ~3, m = pa + pt;
    auto* keys = static_cast<unsigned long long*>(S.get(8 * (size_t)std::max(m, 1ll)));
    auto* sorted = static_cast<unsigned long long*>(S.get(8 * (size_t)std::max(m, 1ll)));
    auto* flag = static_cast<int32_t*>(S.get(4 * (size_t)std::max(m, 1ll)));
    auto* fpos = static_cast<int32_t*>(S.get(4 * (size_t)std::max(m, 1ll)));
    auto* hdeg = static_cast<int32_t*>(S.get(4 * ((size_t)n + 1)));
    auto* hrp = static_cast<int32_t*>(S.get(4 * ((size_t)n + 1)));
    if (!keys || !sorted || !flag || !fpos || !hdeg || !hrp) return fail(ctx, "A + A^T keys");
    Temp T{&S};
    size_t b1 = 0, b2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, b1, keys, sorted, (int)m, 0, 64, st);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, flag, fpos, (int)m, st);
    if (!T.need(std::max(b1, b2))) return fail(ctx, "sort storage");
    sym_keys_kernel<<<blocks_for(n), kT, 0, st>>>(n, rp, col, trp, tcol, pa, keys);
    size_t tb = T.bytes;
    cub::DeviceRadixSort::SortKeys(T.p, tb, keys, sorted, (int)m, 0, 64, st);
    cudaMemsetAsync(hdeg, 0, 4 * ((size_t)n + 1), st);
    unique_flags_kernel<<<blocks_for(m), kT, 0, st>>>(m, sorted, flag, hdeg + 1);
    tb = T.bytes;
    cub::DeviceScan::ExclusiveSum(T.p, tb, flag, fpos, (int)m, st);
    int32_t lastf = 0, lastp = 0;
    if (m > 0) {
        cudaMemcpyAsync(&lastf, flag + m - 1, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&lastp, fpos + m - 1, 4, cudaMemcpyDeviceToHost, st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "hybrid ordering: A + A^T build");
    const long long E = (long long)lastp + lastf;
    auto* adj = static_cast<int32_t*>(S.get(4 * (size_t)std::max(E, 1ll)));
    if (!adj) return fail(ctx, "A + A^T adjacency");
    unique_scatter_kernel<<<blocks_for(m), kT, 0, st>>>(m, sorted, flag, fpos, adj);
    // row pointers: hdeg[v + 1] holds deg(v), hdeg[0] = 0
    size_t b3 = 0;
    cub::DeviceScan::InclusiveSum(nullptr, b3, hdeg, hrp, n + 1, st);
    if (!T.need(b3)) return fail(ctx, "scan storage");
    tb = T.bytes;
    cub::DeviceScan::InclusiveSum(T.p, tb, hdeg, hrp, n + 1, st);
    out->rp = hrp;
    out->adj = adj;
    out->E = E;
    return cudaGetLastError() == cudaSuccess ? GSOFA_OK
                                             : set_err(ctx, GSOFA_ERR_CUDA, "hybrid ordering: A + A^T");
}

int ml_round(gsofa_ctx* ctx, const SymGraph& H, int32_t n, const int32_t* part, int R,
             const int32_t* psize, int32_t leaf, int32_t* mside, int32_t* msep, int32_t* pns,
             int32_t* pna, int32_t* pnb) {
    cudaStream_t st = ctx->stream;
    DeviceScratch S(ctx);
    Temp T{&S};
    auto i32 = [&](size_t c) { return static_cast<int32_t*>(S.get(4 * std::max<size_t>(c, 1))); };
    auto i64 = [&](size_t c) { return static_cast<long long*>(S.get(8 * std::max<size_t>(c, 1))); };
    auto u64 = [&](size_t c) {
        return static_cast<unsigned long long*>(S.get(8 * std::max<size_t>(c, 1)));
    };
    auto sync = [&](const char* what) -> int {
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? GSOFA_OK : cuda_fail(ctx, e, what);
    };
    auto excl_scan_i32 = [&](const int32_t* in, int32_t* out, int count) -> bool {
        size_t b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, in, out, count, st);
        if (!T.need(b)) return false;
        b = T.bytes;
        cub::DeviceScan::ExclusiveSum(T.p, b, in, out, count, st);
        return true;
    };

    // ---- level 0: the split parts' vertices in (part, id) order
    int32_t* cnt = i32(1);
    unsigned long long* vkeys = u64(n);
    unsigned long long* vsorted = u64(n);
    int32_t* lidx = i32(n);
    if (!cnt || !vkeys || !vsorted || !lidx) return fail(ctx, "level 0");
    cudaMemsetAsync(cnt, 0, 4, st);
    active_keys_kernel<<<blocks_for(n), kT, 0, st>>>(n, part, vkeys, cnt);
    int32_t hV = 0;
    cudaMemcpyAsync(&hV, cnt, 4, cudaMemcpyDeviceToHost, st);
    if (int rc = sync("hybrid ordering: active vertices")) return rc;
    cudaMemsetAsync(pns, 0, 4 * (size_t)std::max(R, 1), st);
    cudaMemsetAsync(pna, 0, 4 * (size_t)std::max(R, 1), st);
    cudaMemsetAsync(pnb, 0, 4 * (size_t)std::max(R, 1), st);
    if (hV == 0) return sync("hybrid ordering");
    const long long V0 = hV;
    {
        size_t b = 0;
        int bits = 32;
        while (bits < 64 && (1ll << (bits - 32)) <= (long long)R) bits++;
        cub::DeviceRadixSort::SortKeys(nullptr, b, vkeys, vsorted, (int)V0, 0, bits, st);
        if (!T.need(b)) return fail(ctx, "sort storage");
        b = T.bytes;
        cub::DeviceRadixSort::SortKeys(T.p, b, vkeys, vsorted, (int)V0, 0, bits, st);
    }
    std::vector<Level> L(1);  // L[0]'s pointers are copied out before L grows
    Level& l0 = L[0];
    l0.V = V0;
    int32_t* xid = i32(V0);
    l0.vpart = i32(V0);
    l0.vw = i32(V0);
    int32_t* deg = i32(V0 + 1);
    l0.xadj = i32(V0 + 1);
    l0.pb = i32(R + 1);
    l0.pn = i32(R);
    if (!xid || !l0.vpart || !l0.vw || !deg || !l0.xadj || !l0.pb || !l0.pn)
        return fail(ctx, "level 0");
    level0_ids_kernel<<<blocks_for(V0), kT, 0, st>>>(V0, vsorted, xid, lidx, l0.vpart, l0.vw);
    // part sizes at level 0: the split parts' sizes (0 for the placed ones)
    {
        std::vector<int32_t> hs((size_t)R);
        cudaMemcpyAsync(hs.data(), psize, 4 * (size_t)R, cudaMemcpyDeviceToHost, st);
        if (int rc = sync("hybrid ordering: part sizes")) return rc;
        for (auto& x : hs) x = x > leaf ? x : 0;
        cudaMemcpyAsync(l0.pn, hs.data(), 4 * (size_t)R, cudaMemcpyHostToDevice, st);
        if (int rc = sync("hybrid ordering: part sizes")) return rc;
    }
    if (!excl_scan_i32(l0.pn, l0.pb, R)) return fail(ctx, "scan storage");
    level0_adj_kernel<<<blocks_for(V0), kT, 0, st>>>(V0, H.rp, H.adj, part, xid, lidx, deg,
                                                     nullptr, nullptr, nullptr);
    cudaMemsetAsync(deg + V0, 0, 4, st);
    if (!excl_scan_i32(deg, l0.xadj, (int)V0 + 1)) return fail(ctx, "scan storage");
    {
        int32_t hE = 0;
        cudaMemcpyAsync(&hE, l0.xadj + V0, 4, cudaMemcpyDeviceToHost, st);
        if (int rc = sync("hybrid ordering: level 0")) return rc;
        l0.E = hE;
    }
    l0.adj = i32(l0.E);
    l0.ew = i32(l0.E);
    if (!l0.adj || !l0.ew) return fail(ctx, "level 0 adjacency");
    level0_adj_kernel<<<blocks_for(V0), kT, 0, st>>>(V0, H.rp, H.adj, part, xid, lidx, deg,
                                                     l0.xadj, l0.adj, l0.ew);

    // ---- coarsening
    int32_t* clev = i32(R);
    int32_t* match = i32(V0);
    int32_t* prop = i32(V0);
    int32_t* rep = i32(V0 + 1);
    int32_t* rscan = i32(V0 + 1);
    if (!clev || !match || !prop || !rep || !rscan) return fail(ctx, "coarsening");
    cudaMemsetAsync(clev, 0xff, 4 * (size_t)R, st);
    for (int lv = 0;; lv++) {
        Level& c = L[(size_t)lv];
        const long long V = c.V;
        cudaMemsetAsync(match, 0xff, 4 * (size_t)V, st);
        for (int r = 0; r < kMatchRounds; r++) {
            propose_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.xadj, c.adj, c.ew, c.vpart, c.pn,
                                                         match, prop);
            resolve_kernel<<<blocks_for(V), kT, 0, st>>>(V, prop, match);
        }
        rep_kernel<<<blocks_for(V), kT, 0, st>>>(V, match, c.vpart, c.pn, rep);
        cudaMemsetAsync(rep + V, 0, 4, st);
        if (!excl_scan_i32(rep, rscan, (int)V + 1)) return fail(ctx, "scan storage");
        Level nx;
        nx.pn = i32(R + 1);  // a trailing 0: the scan's last entry is the total
        nx.pb = i32(R + 1);
        if (!nx.pn || !nx.pb) return fail(ctx, "coarsening");
        coarsen_decide_kernel<<<blocks_for(R), kT, 0, st>>>(R, c.pb, c.pn, rscan, lv, nx.pn, clev);
        cudaMemsetAsync(nx.pn + R, 0, 4, st);
        if (!excl_scan_i32(nx.pn, nx.pb, R + 1)) return fail(ctx, "scan storage");
        int32_t hVn = 0;
        cudaMemcpyAsync(&hVn, nx.pb + R, 4, cudaMemcpyDeviceToHost, st);
        if (int rc = sync("hybrid ordering: coarsening")) return rc;
        if (hVn == 0) break;
        nx.V = hVn;
        c.cmap = i32(V);
        nx.vw = i32(nx.V);
        nx.vpart = i32(nx.V);
        unsigned long long* ekeys = u64(c.E);
        unsigned long long* esorted = u64(c.E);
        int32_t* evals = i32(c.E);
        int32_t* esv = i32(c.E);
        unsigned long long* ukeys = u64(c.E);
        int32_t* uvals = i32(c.E);
        int32_t* nruns = i32(1);
        if (!c.cmap || !nx.vw || !nx.vpart || !ekeys || !esorted || !evals || !esv || !ukeys ||
            !uvals || !nruns)
            return fail(ctx, "contraction");
        cmap_kernel<<<blocks_for(V), kT, 0, st>>>(V, match, c.vpart, c.pb, nx.pn, nx.pb, rscan,
                                                  c.vw, c.cmap, nx.vw, nx.vpart);
        coarse_keys_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.xadj, c.adj, c.ew, c.cmap, ekeys,
                                                         evals);
        {
            size_t b1 = 0, b2 = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, b1, ekeys, esorted, evals, esv, (int)c.E, 0,
                                            64, st);
            cub::DeviceReduce::ReduceByKey(nullptr, b2, esorted, ukeys, esv, uvals, nruns,
                                           cub::Sum(), (int)c.E, st);
            if (!T.need(std::max(b1, b2))) return fail(ctx, "sort storage");
            size_t b = T.bytes;
            cub::DeviceRadixSort::SortPairs(T.p, b, ekeys, esorted, evals, esv, (int)c.E, 0, 64,
                                            st);
            b = T.bytes;
            cub::DeviceReduce::ReduceByKey(T.p, b, esorted, ukeys, esv, uvals, nruns, cub::Sum(),
                                           (int)c.E, st);
        }
        int32_t hruns = 0;
        unsigned long long hlast = 0;
        cudaMemcpyAsync(&hruns, nruns, 4, cudaMemcpyDeviceToHost, st);
        if (int rc = sync("hybrid ordering: contraction")) return rc;
        if (hruns > 0) {
            cudaMemcpyAsync(&hlast, ukeys + hruns - 1, 8, cudaMemcpyDeviceToHost, st);
            if (int rc = sync("hybrid ordering: contraction")) return rc;
        }
        nx.E = hruns - (hruns > 0 && hlast == kNoKey ? 1 : 0);
        int32_t* ndeg = i32(nx.V + 1);
        nx.xadj = i32(nx.V + 1);
        nx.adj = i32(nx.E);
        if (!ndeg || !nx.xadj || !nx.adj) return fail(ctx, "contraction");
        nx.ew = uvals;
        cudaMemsetAsync(ndeg, 0, 4 * ((size_t)nx.V + 1), st);
        coarse_rows_kernel<<<blocks_for(nx.E), kT, 0, st>>>(nx.E, ukeys, ndeg, nx.adj);
        if (!excl_scan_i32(ndeg, nx.xadj, (int)nx.V + 1)) return fail(ctx, "scan storage");
        L.push_back(nx);
    }

    // ---- bisection at each part's coarsest level, refinement on the way up
    int32_t* start = i32(R);
    int32_t* on = i32(R);
    int32_t* on_small = i32(R);
    int32_t* on_big = i32(R);
    int32_t* bcnt = i32(R);
    int32_t* done = i32(R);
    int32_t* ccount = i32(R + 1);
    int32_t* cstart = i32(R + 1);
    int32_t* err = i32(2);
    long long* ptotal = i64(R);
    long long* pw0 = i64(R);
    int32_t* lev = i32(V0);
    int32_t* par = i32(V0);
    int32_t* qord = i32(V0);
    int32_t* gain = i32(V0);
    int32_t* cand = i32(V0);
    int32_t* clist = i32(V0);
    int32_t* nsel = i32(1);
    long long* wq = i64(V0 + 1);
    long long* wscan = i64(V0 + 1);
    if (!start || !on || !on_small || !on_big || !bcnt || !done || !ccount || !cstart || !err ||
        !ptotal || !pw0 || !lev || !par || !qord || !gain || !cand || !clist || !nsel || !wq ||
        !wscan)
        return fail(ctx, "bisection");
    cudaMemsetAsync(err, 0, 8, st);
    // queue slots of a part are all written by a search that covers it; the
    // zeros keep any other slot a valid vertex index
    cudaMemsetAsync(qord, 0, 4 * (size_t)V0, st);
    std::vector<int32_t> hclev((size_t)R);
    cudaMemcpyAsync(hclev.data(), clev, 4 * (size_t)R, cudaMemcpyDeviceToHost, st);
    if (int rc = sync("hybrid ordering: coarsest levels")) return rc;

    // one exact-order search of the parts flagged in `on` at level c, from
    // start[]: the small ones (on_small) one thread each, the others (on_big)
    // one CTA each
    auto bfs = [&](Level& c, int nbig) -> int {
        seq_bfs_kernel<<<blocks_for(R), kT, 0, st>>>(R, on_small, start, c.pb, c.pn, c.xadj, c.adj,
                                                     lev, qord, bcnt);
        if (nbig > 0)
            cta_bfs_kernel<<<std::min(nbig, 2 * ctx->sm_count), kCtaBfsThreads, 0, st>>>(
                R, on_big, start, c.pb, c.pn, c.xadj, c.adj, lev, par, qord, bcnt);
        bfs_check_kernel<<<blocks_for(R), kT, 0, st>>>(R, on, c.pn, bcnt, err);
        return GSOFA_OK;
    };

    const int top = (int)L.size() - 1;
    std::vector<int32_t> hon((size_t)R), hsmall((size_t)R), hbig((size_t)R), hpn((size_t)R);
    for (int lv = top; lv >= 0; lv--) {
        Level& c = L[(size_t)lv];
        const long long V = c.V;
        c.side = i32(V);
        if (!c.side) return fail(ctx, "bisection");
        if (lv < top) project_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.cmap, L[(size_t)lv + 1].side, c.side);
        // parts whose coarsest level is this one: BFS growth
        cudaMemcpyAsync(hpn.data(), c.pn, 4 * (size_t)R, cudaMemcpyDeviceToHost, st);
        if (int rc = sync("hybrid ordering: part sizes")) return rc;
        bool any = false;
        int nbig = 0;
        for (int k = 0; k < R; k++) {
            const size_t i = (size_t)k;
            hon[i] = hclev[i] == lv ? 1 : 0;
            hsmall[i] = hon[i] && hpn[i] <= kSeqBfsMax ? 1 : 0;
            hbig[i] = hon[i] && !hsmall[i] ? 1 : 0;
            any |= hon[i] != 0;
            nbig += hbig[i];
        }
        cudaMemsetAsync(ptotal, 0, 8 * (size_t)R, st);
        part_weights_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.vpart, c.vw, nullptr, ptotal, nullptr);
        if (any) {
            cudaMemcpyAsync(on, hon.data(), 4 * (size_t)R, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(on_small, hsmall.data(), 4 * (size_t)R, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(on_big, hbig.data(), 4 * (size_t)R, cudaMemcpyHostToDevice, st);
            first_of_part_kernel<<<blocks_for(R), kT, 0, st>>>(R, on, c.pb, start);
            for (int rep_i = 0; rep_i < 3; rep_i++) {
                if (int rc = bfs(c, nbig)) return rc;
                if (rep_i < 2) last_of_queue_kernel<<<blocks_for(R), kT, 0, st>>>(R, on, c.pb, c.pn, qord, start);
            }
            queue_weights_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.vpart, on, qord, c.pb, c.vw, wq);
            cudaMemsetAsync(wq + V, 0, 8, st);
            size_t b = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, b, wq, wscan, (int)V + 1, st);
            if (!T.need(b)) return fail(ctx, "scan storage");
            b = T.bytes;
            cub::DeviceScan::ExclusiveSum(T.p, b, wq, wscan, (int)V + 1, st);
            growth_side_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.vpart, on, c.pb, qord, wscan,
                                                             ptotal, c.side);
        }
        // refinement of every part present at this level
        cudaMemsetAsync(pw0, 0, 8 * (size_t)R, st);
        cudaMemsetAsync(ptotal, 0, 8 * (size_t)R, st);
        part_weights_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.vpart, c.vw, c.side, ptotal, pw0);
        cudaMemsetAsync(done, 0, 4 * (size_t)R, st);
        for (int pass = 0; pass < kRefinePasses; pass++) {
            gain_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.xadj, c.adj, c.ew, c.vpart, done, c.side,
                                                      gain);
            cudaMemsetAsync(ccount, 0, 4 * ((size_t)R + 1), st);
            cand_kernel<<<blocks_for(V), kT, 0, st>>>(V, c.xadj, c.adj, c.vpart, done, gain, cand,
                                                      ccount);
            if (!excl_scan_i32(ccount, cstart, R + 1)) return fail(ctx, "scan storage");
            size_t b = 0;
            cub::DeviceSelect::Flagged(nullptr, b, thrust::counting_iterator<int32_t>(0), cand,
                                       clist, nsel, (int)V, st);
            if (!T.need(b)) return fail(ctx, "select storage");
            b = T.bytes;
            cub::DeviceSelect::Flagged(T.p, b, thrust::counting_iterator<int32_t>(0), cand, clist,
                                       nsel, (int)V, st);
            // parts that moved nothing are done and skip later passes; the
            // host looks every other pass whether any part is left
            if (pass % 2 == 0) cudaMemsetAsync(err + 1, 0, 4, st);
            accept_kernel<<<blocks_for(R), kT, 0, st>>>(R, cstart, ccount, clist, c.vw, ptotal, pw0,
                                                        c.side, done, err + 1);
            if (pass % 2 == 1) {
                int32_t moved = 0;
                cudaMemcpyAsync(&moved, err + 1, 4, cudaMemcpyDeviceToHost, st);
                if (int rc = sync("hybrid ordering: refinement")) return rc;
                if (!moved) break;
            }
        }
    }

    // ---- level 0: boundaries, the smaller side's as separator
    const Level& f = L[0];
    int32_t* isb = i32(V0);
    int32_t* bnd = i32(2 * (size_t)R);
    if (!isb || !bnd) return fail(ctx, "separator");
    cudaMemsetAsync(bnd, 0, 8 * (size_t)R, st);
    boundary_kernel<<<blocks_for(V0), kT, 0, st>>>(V0, f.xadj, f.adj, f.vpart, f.side, isb, bnd);
    ml_result_kernel<<<blocks_for(V0), kT, 0, st>>>(V0, xid, f.vpart, f.side, isb, bnd, mside,
                                                    msep, pna, pnb);
    ml_sizes_kernel<<<blocks_for(R), kT, 0, st>>>(R, bnd, pns);
    int32_t herr = 0;
    cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st);
    if (int rc = sync("hybrid ordering: separator")) return rc;
    if (herr) return set_err(ctx, GSOFA_ERR_CUDA, "hybrid ordering: a search missed part of a component");
    return GSOFA_OK;
}

}  // namespace host
}  // namespace gsofa
