// Internal structures shared by the host library and the CUDA kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gsofa.h"

namespace gsofa {

// Device-side error word bits (read back by the host after every launch).
enum : int32_t {
    DEV_ERR_COL_RANGE = 1,   // a column id outside [0, n)
    DEV_ERR_ROW_RANGE = 2,   // a row interval outside [0, nnz) or begin > end
    DEV_ERR_QUEUE = 4,       // a traversal queue write past its bound
};

// The status code a device error word stands for: row or column ids out of
// range are the caller's input (GSOFA_ERR_ARG), a queue write past its bound
// is GSOFA_ERR_OVERFLOW; no bit set is GSOFA_OK.
inline int device_status_code(int32_t s) {
    if (s & (DEV_ERR_COL_RANGE | DEV_ERR_ROW_RANGE)) return GSOFA_ERR_ARG;
    if (s & DEV_ERR_QUEUE) return GSOFA_ERR_OVERFLOW;
    return GSOFA_OK;
}

// Counter slots of MatOut::counters.
enum : int {
    CNT_FILLS = 0,
    CNT_EDGES_ALG = 1,
    CNT_VERTS_ALG = 2,
    CNT_EDGES_TRAV = 3,
    CNT_NSUP = 4,
    CNT_NNZ_U = 5,
    CNT_NNZ_L = 6,
    CNT_CHAINED = 7,   // source searches that started from the previous source's closure
    CNT_SLOTS = 8,
};

// One matrix as the traversal sees it: A by rows and A^T by rows, both with
// contiguous rows, plus the per-row outputs.
struct MatDesc {
    int32_t n;
    int32_t flags;              // GSOFA_* bits
    const int32_t* rowptr;      // n+1
    const int32_t* col;
    const int32_t* trowptr;     // n+1 (A^T)
    const int32_t* tcol;
    const int32_t* wdeg;        // ceil(n/32): sum of A's row lengths per 32-vertex word
    const uint32_t* dplanes;    // nplanes * ceil(n/32): degree bit-planes of A's rows
    int32_t nplanes;            // bits of A's largest row length
    int32_t pad0;
    // 0 when A's pattern equals A^T's (set by the ingest's check): the L
    // column searches in A^T then repeat the U row searches in A, and the
    // direction-0 census writes both halves
    const int32_t* asym;
    int32_t* nnz_u;             // n: |U row|
    int32_t* nz_row_u;          // n: reference nz_row_U counter
    uint64_t* dig_u;            // n (or null)
    int32_t* nnz_lc;            // n: |L column|
    uint64_t* dig_lc;           // n (or null)
    uint32_t* lmask;            // 4n: L(f+1+j, f) bits
    uint32_t* umask;            // 4n or null: U(f, f+1+j) bits (read by chained starts)
    int8_t* sflags;             // n: supernode flags (batched supernode kernel)
    int32_t* nnz_lr;            // n or null (L row scatter)
    uint64_t* dig_lr;           // n or null
    unsigned long long* counters;  // CNT_SLOTS
    const int64_t* uptr;        // pattern pass: U row pointers (n+1) or null
    int32_t* ucols;
    const int64_t* lptr;        // pattern pass: L column pointers (n+1) or null
    int32_t* lrows;
    // 2n bytes or null: link[2 s + d] is 0 until the direction-d search of
    // source s has finished, then 1 + (s+1 is in its closure): for d = 0 that
    // bit is U(s, s+1), for d = 1 it is L(s+1, s).  The search of source s+1
    // in the other direction reads it (see traverse_kernel: chained starts)
    uint8_t* link;
    long long item_base;        // first work item of this matrix
    // serving only (zero elsewhere)
    long long n_items;          // work items of this request
    unsigned long long seq;     // request number (claim word tag, done flag value)
    int32_t chunk;              // consecutive sources per work item
    int32_t slot;               // slot of the serving tables
};

// The serving kernel's view of the request loop.  Each admitted request
// owns a slot: its descriptor, a claim word (request number << 32 | items
// claimed) and a finished-items counter.  The host publishes a request by
// writing its claim word (request number, 0) with a stream-ordered copy after
// the request's build and descriptor, and lists (slot, request number) in a
// device table it rewrites with small copies.  A CTA picks the listed request
// with the fewest unclaimed items and claims one with compare-and-swap; a
// claim only succeeds while the word still carries the entry's request
// number, so stale or torn list entries are harmless.  The CTA that finishes
// a request's last item writes the request number to done_flags[slot]
// (mapped host memory, the one place the kernel touches host memory).
// Every wait is bounded: a CTA that finds nothing to claim for idle_ns (or
// max_idle_polls polls) exits, which also returns its SM to other work.
struct ServeLaunch {
    unsigned long long* claim;            // per slot
    const unsigned long long* list;       // (slot << 32) | request number
    const int32_t* ctrl;                  // [0] exit when idle, [1] take no more items, [2] list entries
    unsigned int* rr;                     // rotating start of the list scan (tie order)
    const MatDesc* slots;                 // one descriptor per slot
    unsigned long long* items_done;       // per slot: finished items
    const int32_t* slot_status;           // per slot: ingest error word
    unsigned long long* done_flags;       // mapped host memory, per slot
    int32_t nslots;
    long long smem_words;                 // bitmap words that fit in shared memory
    long long max_idle_polls;
    long long idle_ns;
    // per-CTA workspace slots (queue, closure ring, global bitmap): several
    // launches may run at once, so a CTA takes a free slot when it starts
    // (bit set in cta_slots) instead of using its block index, and returns
    // it when it exits; a CTA that finds none exits at once
    unsigned int* cta_slots;
    int32_t n_cta_slots;
    int* alive;                           // CTAs holding a slot
};

struct TraverseLaunch {
    const MatDesc* mats;        // device array
    int32_t nmats;
    long long total_items;
    unsigned long long* work_counter;  // device, zeroed before launch
    int32_t* queue;             // grid * queue_stride ints
    long long queue_stride;
    uint32_t* gbitmap;          // grid * bitmap_words (global-bitmap variant) or null
    uint32_t* gprev;            // grid * ring * bitmap_words: each CTA's recent closures
    int chunk;                  // consecutive sources per work item
    int merge;                  // 1: reuse the closures of reached cached sources
    int chain;                  // 1: start a source from the previous source's closure when it is known to hold
    long long chain_wait_ns;    // wait this long for the other direction's result when it is one source behind
    int ring;                   // cached closures per CTA (power of 2, <= 64)
    long long sample_stride;    // > 1: process only every stride-th item (autotuner timing)
    long long bitmap_words;     // words per bitmap (covers max n + padding)
    int32_t* status;            // device error word
    int pattern_pass;           // 1: write patterns instead of counting
    int bu_alpha;               // top-down -> bottom-up when frontier*alpha > unseen (0: never)
    int bu_beta;                // bottom-up -> top-down when found*beta < unseen
    int bu_min_src;             // sources below this id stay top-down
    int heavy_len;              // padded rows longer than this are walked by a whole warp
    ServeLaunch serve;          // serving kernel only
};

// Launch helpers (gsofa_kernels.cu).  All asynchronous on `stream`.
int traverse_block_sizes(int* sizes, int max_sizes);
// Returns the resident CTAs per SM for the given configuration (0 = cannot run).
int traverse_occupancy(int block, bool smem_bitmap, size_t smem_bytes);
cudaError_t launch_traverse(const TraverseLaunch& L, int block, int grid, bool smem_bitmap,
                            size_t smem_bytes, cudaStream_t stream);
// The serving kernel: bitmaps of up to L.serve.smem_words words in shared
// memory (smem_bytes), wider ones in L.gbitmap.
int serve_occupancy(int block, size_t smem_bytes);
cudaError_t launch_serve(const TraverseLaunch& L, int block, int grid, size_t smem_bytes,
                         cudaStream_t stream);

// Builds the padded CSR of A (row pointers rp precomputed on the host, with
// pad counts in their low 2 bits) and of A^T.
cudaError_t launch_canonicalize(int32_t n, long long nnz_in, const int32_t* beg,
                                const int32_t* col_in, const int32_t* rp, int32_t* col_out,
                                int32_t* tcount, int32_t* tpad, int32_t* trp, int32_t* tcol,
                                int32_t* tfill, int32_t* wdeg, uint32_t* dplanes, int nplanes,
                                int32_t* asym, int check_symmetry, void* scan_tmp,
                                size_t scan_tmp_bytes, int32_t* status, cudaStream_t stream);
size_t canonicalize_scan_bytes(int32_t n);
// *sum (zeroed by the caller) += sum over A's entries (v, c) of |v - c|.
cudaError_t launch_index_distance(int32_t n, const int32_t* rp, const int32_t* col,
                                  unsigned long long* sum, cudaStream_t stream);
cudaError_t launch_supernodes(int32_t n, int32_t mss, const int32_t* nz_row_u,
                              const uint32_t* lmask, int8_t* flags,
                              unsigned long long* counters, cudaStream_t stream);
cudaError_t launch_batch_reset(const MatDesc* mats, int nmats, cudaStream_t stream);
cudaError_t launch_supernodes_batch(const MatDesc* mats, int nmats, int32_t mss,
                                    const long long* seg_base, long long total_segments,
                                    cudaStream_t stream);
long long supernode_segment_count(int32_t n, int32_t mss);
cudaError_t launch_pattern_ptrs(int32_t n, const int32_t* nnz_u, const int32_t* nnz_lc,
                                int64_t* uptr, int64_t* lptr, void* scan_tmp,
                                size_t scan_tmp_bytes, cudaStream_t stream);
size_t pattern_scan_bytes(int32_t n);

// Device-resident view of a loaded matrix (gsofa_capi.cpp), for entry points
// that live in other translation units.
struct MatrixView {
    int device;
    int32_t n;
    const int32_t* rowptr;
    const int32_t* col;
    const int32_t* trowptr;
    const int32_t* tcol;
    const int32_t* wdeg;
    const uint32_t* dplanes;
    int32_t nplanes;
    const int32_t* asym;
};
bool matrix_view(const void* mat, MatrixView* out);

}  // namespace gsofa
