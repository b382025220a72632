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
//     through vertices < s.  One BFS from s in A, expanding only ids < s.
//   * L column m (s > m): a path s -> m through ids < m is a path m -> s in
//     A^T through ids < m.  One BFS from m in A^T, expanding only ids < m.
// Each BFS expands every vertex at most once (no label re-expansions), and
// its whole state is one bit per vertex, kept in shared memory: n bits =
// 82 KB at n = 659,033, 125 KB at n = 10^6.
//
// The per-source work item of the reference (one slot of a source group,
// :2929-3081) becomes a (matrix, source, direction) work item; persistent CTAs
// take items from a global atomic counter (work stealing), largest sources
// first.  There is no grid barrier (the reference's barrier.cuh spins) and no
// wait on another CTA: each CTA only synchronises with itself.
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include "gsofa_internal.h"
#include "../../include/gsofa.h"

namespace gsofa {

#define FULL_MASK 0xffffffffu

// Column-set digest term: splitmix64 finaliser (Steele, Lea, Flood 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
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

template <int BLOCK>
struct TraverseSmem {
    typedef cub::BlockScan<int, BLOCK> Scan;
    typename Scan::TempStorage scan;
    unsigned long long red[BLOCK / 32][5];
    long long item;
    int cnt[3];
};

// Bitmap words of a matrix of order n: n bits plus zero padding read by the
// 128-bit L-mask extraction past the last vertex.
__host__ __device__ __forceinline__ long long bitmap_words_for(int32_t n) {
    return (((long long)n + 31) >> 5) + 6;
}

template <int BLOCK, bool SMEM_BM>
__global__ void __launch_bounds__(BLOCK) traverse_kernel(TraverseLaunch P) {
    extern __shared__ uint4 dyn_smem[];
    __shared__ TraverseSmem<BLOCK> S;
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint32_t* bm = SMEM_BM ? reinterpret_cast<uint32_t*>(dyn_smem)
                           : P.gbitmap + (long long)blockIdx.x * P.bitmap_words;
    int32_t* q = P.queue + (long long)blockIdx.x * P.queue_stride;
    const long long qcap = P.queue_stride;

    for (long long i = threadIdx.x; i < P.bitmap_words; i += BLOCK) bm[i] = 0u;

    // thread 0 accumulates per-matrix counters and flushes on matrix change
    int acc_mat = -1;
    unsigned long long acc[7] = {0, 0, 0, 0, 0, 0, 0};

    for (;;) {
        if (threadIdx.x == 0) S.item = (long long)atomicAdd(P.work_counter, 1ull);
        __syncthreads();
        const long long item = S.item;
        if (item >= P.total_items) break;
        const int mi = find_matrix(P.mats, P.nmats, item);
        const MatDesc& M = P.mats[mi];
        const int32_t n = M.n;
        const long long local = item - M.item_base;
        const int32_t src = n - 1 - (int32_t)(local >> 1);
        const int dir = (int)(local & 1);
        const int32_t* __restrict__ rp = dir ? M.trowptr : M.rowptr;
        const int32_t* __restrict__ cl = dir ? M.tcol : M.col;
        const bool scatter = dir == 1 && M.nnz_lr != nullptr && !P.pattern_pass;
        const bool digests = M.dig_u != nullptr;

        if (threadIdx.x == 0) {
            bm[src >> 5] |= 1u << (src & 31);
            q[0] = src;
            S.cnt[0] = 0;
        }
        __syncthreads();

        unsigned long long t_gt = 0, t_orig = 0, t_raw = 0, t_edges = 0, t_dig = 0;
        long long lb = 0, le = 1;
        int level = 0;
        while (lb < le) {
            if (threadIdx.x == 0) S.cnt[(level + 1) % 3] = 0;
            int* cnt = &S.cnt[level % 3];
            for (long long base = lb + warp * 32; base < le; base += NW * 32) {
                const long long i = base + lane;
                int v = -1, b = 0, deg = 0;
                if (i < le) {
                    v = q[i];
                    b = rp[v];
                    deg = rp[v + 1] - b;
                }
                t_edges += (unsigned long long)deg;
                int incl = deg;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int t = __shfl_up_sync(FULL_MASK, incl, o);
                    if (lane >= o) incl += t;
                }
                const int total = __shfl_sync(FULL_MASK, incl, 31);
                const int excl = incl - deg;
                for (int k0 = 0; k0 < total; k0 += 32) {
                    const int k = k0 + lane;
                    // owner lane: the last lane whose exclusive offset <= k
                    int lo = 0;
#pragma unroll
                    for (int st = 16; st > 0; st >>= 1) {
                        int c = lo + st;
                        int ex = __shfl_sync(FULL_MASK, excl, c);
                        if (ex <= k) lo = c;
                    }
                    const int ob = __shfl_sync(FULL_MASK, b, lo);
                    const int oex = __shfl_sync(FULL_MASK, excl, lo);
                    const int ov = __shfl_sync(FULL_MASK, v, lo);
                    bool push = false;
                    int w = -1;
                    if (k < total) {
                        w = cl[ob + (k - oex)];
                        if (w != src) {
                            const uint32_t bit = 1u << (w & 31);
                            uint32_t* word = bm + (w >> 5);
                            bool fresh = false;
                            if (!(*(volatile uint32_t*)word & bit))
                                fresh = !(atomicOr(word, bit) & bit);
                            if (w > src) {
                                if (ov == src) t_raw++;
                                if (fresh) {
                                    t_gt++;
                                    if (ov == src) t_orig++;
                                    if (digests) t_dig += mix64((uint64_t)w);
                                    if (scatter) {
                                        atomicAdd(&M.nnz_lr[w], 1);
                                        atomicAdd((unsigned long long*)&M.dig_lr[w],
                                                  (unsigned long long)mix64((uint64_t)src));
                                    }
                                }
                            } else if (fresh) {
                                push = true;
                            }
                        }
                    }
                    const unsigned bal = __ballot_sync(FULL_MASK, push);
                    if (bal) {
                        const int leader = __ffs(bal) - 1;
                        int pos = 0;
                        if (lane == leader) pos = atomicAdd(cnt, __popc(bal));
                        pos = __shfl_sync(FULL_MASK, pos, leader);
                        if (push) {
                            const long long at = le + pos + __popc(bal & ((1u << lane) - 1u));
                            if (at < qcap) q[at] = w;
                            else atomicOr(P.status, DEV_ERR_QUEUE);
                        }
                    }
                }
            }
            __syncthreads();
            const int nxt = *cnt;
            lb = le;
            le = le + nxt;
            if (le > qcap) le = qcap;  // unreachable: at most n vertices are queued
            level++;
        }

        // ---- per-source reduction
        unsigned long long vals[5] = {t_gt, t_orig, t_raw, t_edges, t_dig};
#pragma unroll
        for (int j = 0; j < 5; j++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) vals[j] += __shfl_xor_sync(FULL_MASK, vals[j], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < 5; j++) S.red[warp][j] = vals[j];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long r[5] = {0, 0, 0, 0, 0};
            for (int wi = 0; wi < NW; wi++)
                for (int j = 0; j < 5; j++) r[j] += S.red[wi][j];
            const unsigned long long gt = r[0], orig = r[1], raw = r[2], edges = r[3];
            const unsigned long long dig = r[4];
            const long long src_deg = (long long)rp[src + 1] - rp[src];
            if (!P.pattern_pass) {
                if (dir == 0) {
                    M.nnz_u[src] = (int32_t)gt;
                    M.nz_row_u[src] = (int32_t)(raw + gt - orig);
                    if (digests) M.dig_u[src] = dig;
                } else {
                    M.nnz_lc[src] = (int32_t)gt;
                    if (digests) M.dig_lc[src] = dig;
                }
                if (acc_mat != mi) {
                    if (acc_mat >= 0) {
                        unsigned long long* c = P.mats[acc_mat].counters;
                        atomicAdd(&c[CNT_FILLS], acc[0]);
                        atomicAdd(&c[CNT_EDGES_ALG], acc[1]);
                        atomicAdd(&c[CNT_VERTS_ALG], acc[2]);
                        atomicAdd(&c[CNT_EDGES_TRAV], acc[3]);
                        atomicAdd(&c[CNT_NNZ_U], acc[4]);
                        atomicAdd(&c[CNT_NNZ_L], acc[5]);
                    }
                    acc_mat = mi;
                    for (int j = 0; j < 7; j++) acc[j] = 0;
                }
                acc[0] += gt - orig;
                acc[3] += edges;
                if (dir == 0) {
                    acc[1] += edges - (unsigned long long)src_deg;
                    acc[2] += (unsigned long long)(le - 1);
                    acc[4] += gt;
                } else {
                    acc[5] += gt;
                }
            }
        }
        if (dir == 1 && !P.pattern_pass && threadIdx.x < 4) {
            // 128-bit mask of rows f+1 .. f+128 in L column f (supernode test)
            const long long p = (long long)src + 1 + 32 * threadIdx.x;
            const long long wd = p >> 5;
            const int off = (int)(p & 31);
            uint32_t val = bm[wd] >> off;
            if (off) val |= bm[wd + 1] << (32 - off);
            M.lmask[4ll * src + threadIdx.x] = val;
        }
        if (P.pattern_pass) {
            // sorted ids of the set bits > src: U row (dir 0) or L column (dir 1)
            int32_t* out = dir == 0 ? M.ucols : M.lrows;
            const long long obase = dir == 0 ? M.uptr[src] : M.lptr[src];
            const long long nw = ((long long)n + 31) >> 5;
            long long wpos = ((long long)src + 1) >> 5;
            long long written = 0;
            for (; wpos < nw; wpos += BLOCK) {
                const long long wi = wpos + threadIdx.x;
                uint32_t word = 0;
                if (wi < nw) {
                    word = bm[wi];
                    const long long first = wi << 5;
                    if (first <= src) {  // drop bits <= src
                        const int keep_from = (int)(src - first) + 1;
                        word = keep_from >= 32 ? 0u : (word & (~0u << keep_from));
                    }
                }
                int cntw = __popc(word), ex = 0, tot = 0;
                typename TraverseSmem<BLOCK>::Scan(S.scan).ExclusiveSum(cntw, ex, tot);
                long long o = obase + written + ex;
                while (word) {
                    const int bpos = __ffs(word) - 1;
                    word &= word - 1;
                    out[o++] = (int32_t)((wi << 5) + bpos);
                }
                written += tot;
                __syncthreads();  // scan storage reuse
            }
        }
        __syncthreads();
        const long long words = bitmap_words_for(n);
        for (long long i = threadIdx.x; i < words; i += BLOCK) bm[i] = 0u;
        __syncthreads();
    }
    if (threadIdx.x == 0 && acc_mat >= 0) {
        unsigned long long* c = P.mats[acc_mat].counters;
        atomicAdd(&c[CNT_FILLS], acc[0]);
        atomicAdd(&c[CNT_EDGES_ALG], acc[1]);
        atomicAdd(&c[CNT_VERTS_ALG], acc[2]);
        atomicAdd(&c[CNT_EDGES_TRAV], acc[3]);
        atomicAdd(&c[CNT_NNZ_U], acc[4]);
        atomicAdd(&c[CNT_NNZ_L], acc[5]);
    }
}

template <int BLOCK, bool SMEM_BM>
static cudaError_t launch_one(const TraverseLaunch& L, int grid, size_t smem, cudaStream_t st) {
    auto k = traverse_kernel<BLOCK, SMEM_BM>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(SMEM_BM ? smem : 0));
    if (e != cudaSuccess) return e;
    k<<<grid, BLOCK, SMEM_BM ? smem : 0, st>>>(L);
    return cudaGetLastError();
}

template <int BLOCK, bool SMEM_BM>
static int occ_one(size_t smem) {
    auto k = traverse_kernel<BLOCK, SMEM_BM>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(SMEM_BM ? smem : 0)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, BLOCK, SMEM_BM ? smem : 0) !=
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
    case B: return smem_bitmap ? occ_one<B, true>(smem) : occ_one<B, false>(smem);
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
    case B: return smem_bitmap ? launch_one<B, true>(L, grid, smem, st) \
                               : launch_one<B, false>(L, grid, smem, st);
    switch (block) {
        LAUNCH_CASE(128)
        LAUNCH_CASE(256)
        LAUNCH_CASE(512)
        LAUNCH_CASE(1024)
        default: return cudaErrorInvalidValue;
    }
#undef LAUNCH_CASE
}

// ---- ingest: gather rows into contiguous CSR and build A^T ------------------

// One warp per row: copy the row's entries and count them per column.
__global__ void gather_rows_kernel(int32_t n, long long nnz_in, const int32_t* __restrict__ beg,
                                   const int32_t* __restrict__ rowptr,
                                   const int32_t* __restrict__ col_in, int32_t* __restrict__ col_out,
                                   int32_t* __restrict__ tcount, int32_t* status) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gw; v < n; v += nwarps) {
        const long long b = beg[v];
        const long long o = rowptr[v];
        const long long d = (long long)rowptr[v + 1] - o;
        for (long long j = lane; j < d; j += 32) {
            const long long src = b + j;
            if (src < 0 || src >= nnz_in) {
                atomicOr(status, DEV_ERR_ROW_RANGE);
                continue;
            }
            const int32_t c = col_in[src];
            if (c < 0 || c >= n) {
                atomicOr(status, DEV_ERR_COL_RANGE);
                col_out[o + j] = (int32_t)v;  // keep the structure in range
                atomicAdd(&tcount[v], 1);
                continue;
            }
            col_out[o + j] = c;
            atomicAdd(&tcount[c], 1);
        }
    }
}

__global__ void transpose_scatter_kernel(int32_t n, const int32_t* __restrict__ rowptr,
                                         const int32_t* __restrict__ col,
                                         const int32_t* __restrict__ trowptr,
                                         int32_t* __restrict__ tfill, int32_t* __restrict__ tcol) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gw; v < n; v += nwarps) {
        const int b = rowptr[v], e = rowptr[v + 1];
        for (int j = b + lane; j < e; j += 32) {
            const int c = col[j];
            const int pos = atomicAdd(&tfill[c], 1);
            tcol[trowptr[c] + pos] = (int32_t)v;
        }
    }
}

size_t canonicalize_scan_bytes(int32_t n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int32_t*)nullptr, (int32_t*)nullptr,
                                  (int)n + 1);
    return bytes;
}

// rowptr (n+1) is already on the device (computed on the host from beg/end).
// tcount and tfill: n+1 zeroed ints.  col_in may equal col_out when the rows
// are already contiguous in order (then only validation + counting happens).
cudaError_t launch_canonicalize(int32_t n, long long nnz_in, const int32_t* beg, const int32_t* /*end*/,
                                const int32_t* col_in, int32_t* rowptr, int32_t* col_out,
                                int32_t* tcount, int32_t* trowptr, int32_t* tcol, int32_t* tfill,
                                void* scan_tmp, size_t scan_tmp_bytes, int32_t* status,
                                cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    long long warps_needed = n;
    int grid = (int)((warps_needed * 32 + threads - 1) / threads);
    if (grid > 148 * 64) grid = 148 * 64;
    gather_rows_kernel<<<grid, threads, 0, st>>>(n, nnz_in, beg, rowptr, col_in, col_out, tcount,
                                                 status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t bytes = scan_tmp_bytes;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, bytes, tcount, trowptr, (int)n + 1, st);
    if (e != cudaSuccess) return e;
    transpose_scatter_kernel<<<grid, threads, 0, st>>>(n, rowptr, col_out, trowptr, tfill, tcol);
    return cudaGetLastError();
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
__global__ void supernode_kernel(int32_t n, int32_t mss, const int32_t* __restrict__ nzu,
                                 const uint32_t* __restrict__ lmask, int8_t* __restrict__ flags,
                                 unsigned long long* counters) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long segs_per_chunk = ((long long)mss + 127) / 128;
    const long long nchunks = ((long long)n + mss - 1) / mss;
    const long long nseg = nchunks * segs_per_chunk;
    unsigned long long count = 0;
    for (long long sg = gw; sg < nseg; sg += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long c = sg / segs_per_chunk;
        const long long k = sg % segs_per_chunk;
        const long long start = c * mss + 128 * k;
        long long stop = start + 128;
        if (stop > (c + 1) * mss) stop = (c + 1) * mss;
        if (stop > n) stop = n;
        if (start >= stop) continue;
        int head[4];
        long long last = -1;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const long long r = start + 4 * lane + j;
            head[j] = 0;
            if (r < stop) {
                head[j] = (r == start) || (nzu[r - 1] - nzu[r] != 1);
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
                const uint32_t wv = lmask[4 * f + (bit >> 5)];
                const bool in_l = (wv >> (bit & 31)) & 1u;
                fl = in_l ? 0 : 2;
                if (!in_l) count++;
            }
            if (flags) flags[r] = fl;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(FULL_MASK, count, o);
    if (lane == 0 && count) atomicAdd(&counters[CNT_NSUP], count);
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
