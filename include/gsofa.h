/*
 * gsofa.h -- C-ABI of the B200 symbolic-LU ("fill-path") engine.
 *
 * The reference (gSoFaTPDS) is an executable, not a library: its entry is
 *   void symbfact_min_id(int argc, char** argv, int rank, ull_t& fill_count,
 *                        double& time, int& N_supernodes, ull_t& TEPS)
 *   (gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh:2529;
 *    SpaceOptimization/symbfact.cuh:1553 has the same call without the last two)
 * called from main() (gSoFa_SOAComparison/main.cu:20-64).  This header splits
 * that monolith into handles so a caller (CLI, test harness, benchmark,
 * serving loop, or another language through its FFI) can load a matrix once,
 * keep it device-resident and factor it repeatedly.  Every function returns a
 * status code; none of them exits or aborts the process (the reference's
 * H_ERR macro calls exit(EXIT_FAILURE), barrier.cuh:11-20).
 *
 * Plain C types only: no CUDA or torch types appear in the signatures.
 */
#ifndef GSOFA_H
#define GSOFA_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define GSOFA_OK 0
#define GSOFA_ERR_ARG 1          /* invalid argument or malformed CSR        */
#define GSOFA_ERR_IO 2           /* file missing or unparsable               */
#define GSOFA_ERR_OOM_BUDGET 3   /* would exceed the context's memory budget */
#define GSOFA_ERR_TIMEOUT 4      /* a bounded device wait gave up            */
#define GSOFA_ERR_OVERFLOW 5     /* a device queue bound was exceeded        */
#define GSOFA_ERR_CUDA 6         /* CUDA runtime error (message in last_error) */
#define GSOFA_ERR_UNSUPPORTED 7  /* size or option outside what is built     */
#define GSOFA_ERR_BUSY 8         /* serving queue full / ticket not finished */
#define GSOFA_ERR_SCRATCH 9      /* problem larger than the no-allocation scratch area */

typedef struct gsofa_ctx gsofa_ctx;
typedef struct gsofa_matrix gsofa_matrix;
typedef struct gsofa_result gsofa_result;
typedef struct gsofa_batch gsofa_batch;

/* ---- options -------------------------------------------------------------- */
#define GSOFA_SUPERNODES (1u << 0)  /* detect supernodes (reference SOA :1790-2123) */
#define GSOFA_L_ROW_STATS (1u << 1) /* also per-row L counts + digests (scatter)     */
#define GSOFA_PATTERN (1u << 2)     /* materialise L (by columns) and U (by rows)    */
#define GSOFA_DIGESTS (1u << 3)     /* per-row/column 64-bit column-set digests      */
/* Diagnostic: keep the traversal's seen-bitmap in global memory even when
 * it fits in shared memory (the variant used for orders above ~1.8M). */
#define GSOFA_FORCE_GLOBAL_BITMAP (1u << 30)
/* Diagnostic: never reuse the previous source's closure (every source is
 * searched from scratch). */
#define GSOFA_NO_MERGE (1u << 29)
/* Fault injection: each CTA's frontier queue holds only 64 entries, so any
 * search that queues more reports GSOFA_ERR_OVERFLOW (every queue access is
 * bounds-checked; nothing is written past the bound).  gsofa_factor_symbolic
 * and gsofa_factor_symbolic_noalloc. */
#define GSOFA_DEBUG_QUEUE_CAP (1u << 28)
/* Diagnostic: never start a source's search from the previous source's
 * closure (the start the traversal takes when the other direction's search
 * has shown that the previous source is reachable); merges stay on. */
#define GSOFA_NO_CHAIN (1u << 27)

typedef struct gsofa_opts {
    /* rows per supernode chunk; the reference's max_supernode_size, argv[5]
     * of the SOA command line (symbfact_warp_centric_new_scheduling.cuh:2540) */
    int32_t max_supernode_size;
    /* threads cooperating on one source traversal (CTA size: 128..1024,
     * multiple of 32); 0 = autotuned */
    int32_t threads_per_source;
    /* concurrent source traversals (CTAs); 0 = as many as fit on the GPU.
     * The reference's N_src_group (Compute_Src_group, :1031-1048) */
    int32_t sources_in_flight;
    uint32_t flags; /* GSOFA_* option bits */
    /* traversal direction switch: a search turns from top-down to bottom-up
     * sweeps when frontier * bu_alpha exceeds its unseen vertices, and back
     * when a sweep finds fewer than unseen / bu_beta; 0 = defaults,
     * bu_alpha < 0 = top-down only */
    int32_t bu_alpha;
    int32_t bu_beta;
    /* rows longer than this many entries are walked by a whole warp instead
     * of one lane; 0 = default (16) */
    int32_t heavy_row;
    /* sources with a smaller id always stay top-down; 0 = default (2048) */
    int32_t bu_min_source;
    /* consecutive sources one CTA takes as a work item (the previous source's
     * closure is reused inside a chunk); 0 = default */
    int32_t chunk_sources;
    /* closures of recently finished sources each CTA keeps for reuse
     * (rounded down to a power of 2, at most 64); 0 = default */
    int32_t cached_closures;
    /* how long (microseconds) a source search may wait, when the search of
     * the same chunk in the other direction is one source behind, for the
     * result that lets it start from the previous source's closure; 0 =
     * default, < 0 = never wait */
    int32_t chain_wait_us;
    int32_t reserved;
} gsofa_opts;

/* Defaults: max_supernode_size 128, autotuned CTA size, GPU-filling
 * concurrency, flags = GSOFA_SUPERNODES | GSOFA_DIGESTS. */
int gsofa_opts_default(gsofa_opts* opts);

/* ---- context -------------------------------------------------------------- */
/* One context per device.  budget_bytes bounds every device allocation the
 * context makes (matrices, workspace, results); 0 = 90% of free memory.
 * Replaces the reference's cudaSetDevice + per-GPU allocation
 * (Allocate_Initialize, :2296-2472; SPO pool, symbfact.cuh:1683-1687). */
int gsofa_create(int device, size_t budget_bytes, gsofa_ctx** out);
int gsofa_destroy(gsofa_ctx* ctx);
/* Message for the last failing call on this context (never NULL). */
const char* gsofa_last_error(const gsofa_ctx* ctx);
const char* gsofa_status_string(int status);
/* Launch on this CUDA stream (a cudaStream_t passed as void*); NULL = the
 * context's own stream. */
int gsofa_set_stream(gsofa_ctx* ctx, void* cuda_stream);
/* Device bytes currently held by the context. */
int gsofa_memory_used(const gsofa_ctx* ctx, size_t* bytes);

/* ---- matrices (replaces the ASCII ingest, :2567-2616 / symbfact.cuh:1591-1640) */
/* Row v of A is col[row_begin[v] .. row_end[v]).  Rows may be stored in any
 * order and need not be contiguous or sorted (the reference's BC input is
 * neither).  Host pointers; the matrix is copied to the device. */
int gsofa_load_csr(gsofa_ctx* ctx, int32_t n, int64_t nnz, const int32_t* row_begin,
                   const int32_t* row_end, const int32_t* col, gsofa_matrix** out);
/* The reference's three ASCII files: csr = "E N" then E column ids,
 * beg / end = n ids each. */
int gsofa_load_csr_files(gsofa_ctx* ctx, const char* beg_file, const char* end_file,
                         const char* csr_file, gsofa_matrix** out);
/* Binary CSR files: the parsed form of the three ASCII files, read at disk
 * speed instead of being parsed again (the reference reads the ASCII files
 * with fscanf on every run, :2567-2616).  Little-endian: "GSOFACSR", version,
 * n, nnz, a payload checksum, then beg[n], end[n], col[nnz] as int32 exactly
 * as in the .dat files.  Writing and reading need no GPU; a truncated or
 * corrupted file is GSOFA_ERR_IO. */
int gsofa_write_csr_binary(const char* path, int32_t n, int64_t nnz, const int32_t* row_begin,
                           const int32_t* row_end, const int32_t* col);
/* With all three arrays NULL, only *n and *nnz are returned (size query). */
int gsofa_read_csr_binary(const char* path, int32_t* n, int64_t* nnz, int32_t* row_begin,
                          int32_t* row_end, int32_t* col);
int gsofa_convert_dat_to_binary(const char* beg_file, const char* end_file, const char* csr_file,
                                const char* out_path);
int gsofa_load_csr_binary(gsofa_ctx* ctx, const char* path, gsofa_matrix** out);
int gsofa_matrix_info(const gsofa_matrix* mat, int32_t* n, int64_t* nnz);
int gsofa_matrix_destroy(gsofa_matrix* mat);

/* ---- fill-reducing ordering (the step before the reference: its inputs are
 * already permuted by SuperLU_DIST, README.md:27-33; no counterpart in its
 * code) */
typedef struct gsofa_order_stats {
    int32_t rounds;              /* dissection rounds run                      */
    int32_t splits;              /* components cut by a separator              */
    int64_t separator_vertices;  /* vertices placed in separators              */
    int32_t max_separator;       /* largest separator                          */
    int32_t reserved;
    double ms;                   /* device time of the ordering                */
} gsofa_order_stats;
/* Level-set nested dissection of the structure of A + A^T, on the device:
 * every round splits each part into its connected components, places the
 * components of at most leaf_size vertices (ids ascending), and cuts each
 * larger one at the middle level of a BFS from a pseudo-peripheral vertex
 * (the separator trimmed to the vertices adjacent to the next level; George
 * 1973, George and Liu 1981 ch. 8), the two sides first and the separator
 * last.  Deterministic: the same matrix always gives the same perm.
 * perm (host, n entries): new index k holds old index perm[k].
 * leaf_size <= 0 means 32; max_rounds <= 0 means 512 (the last round places
 * every remaining component whole).  stats may be NULL. */
int gsofa_order_nd(gsofa_ctx* ctx, const gsofa_matrix* mat, int32_t leaf_size, int32_t max_rounds,
                   int32_t* perm, gsofa_order_stats* stats);
/* Hybrid nested dissection, on the device: gsofa_order_nd's rounds (no round
 * cap), where every component to be cut also gets a multilevel bisection --
 * coarsening by mutual heavy-edge proposals, BFS growth on the coarsest
 * graph, boundary refinement at every level within 40..60 % balance -- and
 * the boundary of its side with fewer boundary vertices is used as the
 * separator when it is smaller than the level-set one and leaves both sides
 * non-empty.  On small-world graphs (circuit-like patterns) level sets give
 * very large separators and the multilevel ones cut the fill; on grids the
 * level-set separator wins and is kept.  Deterministic: the same matrix
 * always gives the same perm.  Arguments as gsofa_order_nd. */
int gsofa_order_hybrid(gsofa_ctx* ctx, const gsofa_matrix* mat, int32_t leaf_size, int32_t* perm,
                       gsofa_order_stats* stats);
/* The symmetrically permuted matrix P A P^T built on the device: row k of
 * *out is row perm[k] of mat with every column id c renamed to the k' with
 * perm[k'] = c.  perm: host, n entries, a permutation of 0..n-1 (else
 * GSOFA_ERR_ARG). */
int gsofa_matrix_permute(gsofa_ctx* ctx, const gsofa_matrix* mat, const int32_t* perm,
                         gsofa_matrix** out);
/* Failure-path self-test of the ordering's grid barrier, whose every wait is
 * bounded: the BFS kernel is launched waiting for one block more than it
 * has, each wait gives up after limit_ms (0 < limit_ms <= 2000), and the
 * call returns GSOFA_ERR_TIMEOUT with the context still usable. */
int gsofa_order_wait_selftest(gsofa_ctx* ctx, double limit_ms);

/* ---- factorization (replaces the group loop :2965-3218 and its kernels) --- */
/* Synchronous: returns when the result is complete on the device. */
int gsofa_factor_symbolic(gsofa_ctx* ctx, const gsofa_matrix* mat, const gsofa_opts* opts,
                          gsofa_result** out);
/* Autotuner: times candidate launch shapes (threads_per_source,
 * chunk_sources, cached_closures, heavy_row) for this matrix on a sample of its work
 * and writes the fastest into *opts (other fields are left as given).
 * Results never depend on these settings.  Choices are cached in the
 * context per class (log2 n, mean row length, and half-octaves of the mean
 * distance |i - j| of the entries from the diagonal over n, one device pass),
 * so later calls for similar matrices return at once.  Replaces the reference's fixed sizing
 * (Compute_Src_group, :1031-1048; SPO :1101-1119, :1465-1507). */
int gsofa_autotune(gsofa_ctx* ctx, const gsofa_matrix* mat, gsofa_opts* opts);
/* The same search for a batch: each candidate is timed as one persistent
 * launch over all `count` matrices (what gsofa_factor_batch and
 * gsofa_batch_create run), so the shape suits the mix rather than its
 * largest member.  Not cached. */
int gsofa_autotune_batch(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                         gsofa_opts* opts);
/* Many matrices of uneven size in one persistent launch; results[i] is the
 * result of mats[i] (identical to factoring it alone). */
int gsofa_factor_batch(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                       const gsofa_opts* opts, gsofa_result** results);

/* A prepared batch: many matrices of uneven size in one persistent launch
 * captured in a CUDA graph (reset, traversal over every matrix's work items,
 * supernode detection of all of them, read-back of the totals), so each run
 * is a single graph launch.  The batch owns its results (read them with
 * gsofa_batch_result and the gsofa_result_* getters; do not destroy them) and
 * a private workspace.  Matrices must stay alive while the batch exists.
 * GSOFA_PATTERN is not available in a batch.  The reference factors one
 * matrix per run (SOA :2965-3218); this has no counterpart there. */
int gsofa_batch_create(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                       const gsofa_opts* opts, gsofa_batch** out);
/* Runs the captured graph; synchronous.  Results reflect the latest run;
 * every run gives the same results. */
int gsofa_batch_run(gsofa_batch* batch);
int gsofa_batch_result(const gsofa_batch* batch, int32_t i, gsofa_result** res);
int gsofa_batch_destroy(gsofa_batch* batch);

typedef struct gsofa_counts {
    int32_t n;
    int32_t reserved;
    uint64_t fill_count;      /* reference "Number of fill-ins detected"        */
    uint64_t nnz_l;           /* strictly-lower entries of L+U (A's + fills)     */
    uint64_t nnz_u;           /* strictly-upper entries of L+U                   */
    uint64_t nnz_lu;          /* nnz_l + nnz_u + n (full diagonal)               */
    int64_t n_supernodes;     /* reference's printed count (detected + 1), -1 if off */
    uint64_t edges_alg;       /* sum over sources s of the degrees of the vertices
                               * < s reachable from s through vertices < s      */
    uint64_t vertices_alg;    /* number of such (source, vertex) pairs          */
    uint64_t edges_traversed; /* edge inspections this engine made (A and A^T)  */
    double ms_device;         /* device time of the factorization (CUDA events) */
    double ms_traverse;       /* device time of the traversal kernel alone      */
    uint64_t sources_chained; /* source searches (U rows and L columns) that
                               * started from the previous source's closure    */
} gsofa_counts;
int gsofa_result_counts(const gsofa_result* res, gsofa_counts* out);

/* Per-row / per-column counts (host buffers of n entries; any may be NULL):
 *   nnz_u_row[v]  distinct strictly-upper entries of row v of U
 *   nz_row_u[v]   the reference's nz_row_U counter (SOA :895-903, :985-992)
 *   nnz_l_col[v]  distinct strictly-lower entries of column v of L
 *   nnz_l_row[v]  distinct strictly-lower entries of row v (needs GSOFA_L_ROW_STATS) */
int gsofa_result_row_counts(const gsofa_result* res, int32_t* nnz_u_row, int32_t* nz_row_u,
                            int32_t* nnz_l_col, int32_t* nnz_l_row);
/* Column-set digests (mod 2^64 sums of the splitmix64 finaliser): for U rows
 * and L columns, sum over the set's non-zero 32-id words w of
 * splitmix64((w << 32) | mask_w) (bit j of mask_w: id 32w + j in the set);
 * for L rows (GSOFA_L_ROW_STATS), sum of splitmix64(column id). */
int gsofa_result_digests(const gsofa_result* res, uint64_t* dig_u_row, uint64_t* dig_l_col,
                         uint64_t* dig_l_row);
/* Supernode partition: flags[v] (n bytes) = 1 row starts a supernode, 2 a
 * supernode is counted at this row without moving the first row (the
 * reference's split rule, SOA :2043-2052), 0 row extends the current one.
 * boundaries: rows with a non-zero flag, ascending, up to cap entries;
 * *count gets the total.  Any pointer may be NULL. */
int gsofa_result_supernodes(const gsofa_result* res, int8_t* flags, int32_t* boundaries,
                            int64_t cap, int64_t* count);
/* 128-bit masks per column f: bit j of word j/32 set iff L(f+1+j, f) != 0. */
int gsofa_result_lmask(const gsofa_result* res, uint32_t* mask4n);
/* Materialised pattern (needs GSOFA_PATTERN).  U by rows: ptr[n+1] and the
 * sorted column ids of each row; L by columns: ptr[n+1] and the sorted row
 * ids of each column.  cap = capacity of the id buffer; pass ids = NULL to
 * get ptr only. */
int gsofa_result_pattern_u(const gsofa_result* res, int64_t* ptr, int32_t* cols, int64_t cap);
int gsofa_result_pattern_l(const gsofa_result* res, int64_t* ptr, int32_t* rows, int64_t cap);
/* The symbolic-to-numeric handoff (needs GSOFA_PATTERN and GSOFA_SUPERNODES):
 * L and U in supernodal block form, what a supernodal numeric LU allocates
 * from.  Block k is the run of columns [block_start[k], block_start[k+1]),
 * a new block starting at every row with a non-zero supernode flag.  With
 * l = block_start[k+1]:
 *   lrows[lptr[k] .. lptr[k+1])  sorted rows r >= l with L(r, c) != 0 for
 *                                some column c of the block;
 *   ucols[uptr[k] .. uptr[k+1])  sorted columns c >= l with U(r, c) != 0 for
 *                                some row r of the block;
 * the diagonal block is dense and implicit.  Call with NULL arrays to get
 * the sizes (*nblocks, *nl, *nu); buffers then need nblocks + 1, nl and nu
 * entries.  Built on the device on the first call and kept with the result.
 * No counterpart in the reference, which stops at counts (its consumer,
 * SuperLU_DIST, recomputes the structure). */
int gsofa_result_supernodal(const gsofa_result* res, int64_t* nblocks, int64_t* nl, int64_t* nu,
                            int32_t* block_start, int64_t* lptr, int32_t* lrows, int64_t* uptr,
                            int32_t* ucols);
int gsofa_result_destroy(gsofa_result* res);

/* ---- serving: a request loop with continuous batching ------------------------ */
/* No counterpart in the reference, which factors one matrix per run.  A server
 * owns a host thread, three streams and a persistent traversal kernel that
 * stays on the device while published work is waiting.  Each submitted matrix is a
 * request; the loop admits requests in arrival order as slots and memory free
 * up (its workspace footprint -- the padded CSR of A and A^T and its result
 * arrays -- must fit the budget next to the requests already admitted),
 * uploads and builds the matrix on a side stream, then publishes its work
 * items to the running kernel.  The kernel's CTAs take items of every admitted
 * request as they free up, so requests that arrive while others run share the
 * device.  When a request's last item is done the loop runs its supernode
 * detection and hands out a result identical to gsofa_factor_symbolic's
 * (gsofa_result_* getters; the caller destroys it).
 *
 * opts: max_supernode_size and flags (GSOFA_SUPERNODES, GSOFA_DIGESTS,
 * GSOFA_L_ROW_STATS; GSOFA_PATTERN is not served), threads_per_source (256,
 * 512 or 1024; 0 = chosen from max_n), sources_in_flight (CTA cap),
 * chunk_sources (0 = per request), cached_closures, heavy_row.  max_n is the
 * largest order served (it sizes the per-CTA queues, closure rings and global
 * bitmaps); budget_bytes bounds all device memory the server holds
 * (0 = 40 GB). */
typedef struct gsofa_server gsofa_server;
int gsofa_server_create(gsofa_ctx* ctx, const gsofa_opts* opts, int32_t max_n,
                        size_t budget_bytes, gsofa_server** out);
/* Queues a request and returns at once with its ticket.  The arrays are read
 * when the request is admitted: they must stay valid and unchanged until the
 * ticket completes.  GSOFA_ERR_UNSUPPORTED if n > max_n, GSOFA_ERR_OOM_BUDGET
 * if the request alone exceeds the budget, GSOFA_ERR_ARG after destroy began. */
int gsofa_server_submit(gsofa_server* srv, int32_t n, int64_t nnz, const int32_t* row_begin,
                        const int32_t* row_end, const int32_t* col, uint64_t* ticket);
/* GSOFA_OK and *res once the ticket is complete (the result is handed out
 * once; later calls return GSOFA_ERR_ARG), GSOFA_ERR_BUSY while it is queued
 * or running, or the request's own error (malformed CSR: GSOFA_ERR_ARG). */
int gsofa_server_poll(gsofa_server* srv, uint64_t ticket, gsofa_result** res);
/* As poll, blocking up to timeout_ms (< 0: no limit); GSOFA_ERR_TIMEOUT when
 * the time runs out first. */
int gsofa_server_wait(gsofa_server* srv, uint64_t ticket, double timeout_ms, gsofa_result** res);
typedef struct gsofa_ticket_info {
    double t_submit_ms;   /* host clock, ms since the server was created      */
    double t_admit_ms;    /* memory reserved, upload queued                   */
    double t_publish_ms;  /* built on the device, work items claimable         */
    double t_done_ms;     /* result complete (supernodes and totals read back) */
    uint64_t footprint_bytes;
    int32_t status;       /* GSOFA_OK, GSOFA_ERR_BUSY (not finished), or the error */
    int32_t n;
} gsofa_ticket_info;
int gsofa_server_ticket_info(gsofa_server* srv, uint64_t ticket, gsofa_ticket_info* info);
typedef struct gsofa_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t kernel_launches;   /* persistent kernel (re)launches          */
    uint64_t items_published;
    uint64_t bytes_in_use;      /* workspace + admitted requests            */
    uint64_t peak_bytes;
    uint64_t fixed_bytes;       /* per-CTA queues, rings, bitmaps, tables   */
    int32_t grid, block;        /* the kernel's CTAs and threads per CTA     */
    int32_t max_in_flight;      /* most requests admitted at once           */
    int32_t reserved;
} gsofa_server_stats;
int gsofa_server_get_stats(gsofa_server* srv, gsofa_server_stats* out);
/* Finishes every queued request, stops the kernel and frees the server.
 * Results already handed out stay valid; unclaimed ones are destroyed. */
int gsofa_server_destroy(gsofa_server* srv);
/* Message of the server's last internal error ("" if none). */
const char* gsofa_server_last_error(const gsofa_server* srv);

/* ---- factorization without device allocation --------------------------------- */
/* No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc at factorization time (a host framework that owns all device
 * memory through its own pool, or a loop that must not allocate after its
 * set-up).  The matrix is loaded beforehand with gsofa_load_csr; the results
 * go to caller-owned device buffers; the kernel's scratch (work counter,
 * status, descriptor, per-CTA queues and closure rings) comes from one static
 * __device__ array of GSOFA_NOALLOC_SCRATCH_BYTES that every GPU loading this
 * library holds until exit.  Nothing is allocated: no cudaMalloc, cudaFree or
 * allocating library call.
 *   - Size limit: a matrix of order n needs 4n bytes of queue plus
 *     cached_closures * (n/8 + 24) bytes of closure ring per CTA (plus n/8
 *     bytes of bitmap when n > ~1.8M); the grid shrinks to what fits and
 *     GSOFA_ERR_SCRATCH is returned when not even one CTA fits (n above
 *     roughly 12M with the default 8 cached closures).  Other launch
 *     defaults are those of gsofa_factor_symbolic; the ring defaults to 8
 *     slots (not 64) so that more CTAs fit the fixed array.
 *   - Every call looks up the array's device address (cudaGetSymbolAddress)
 *     with the matrix's device current; no address is kept between calls.
 *   - Every call shares the array and leaves its contents behind; the work
 *     counter and status word are cleared by each call.  Calls that overlap
 *     on the GPU (other streams, other threads) race on the array.
 *   - Outputs (device pointers, n entries each unless noted): d_nnz_u_row,
 *     d_nz_row_u, d_nnz_l_col as in gsofa_result_row_counts; d_lmask 4n words
 *     as gsofa_result_lmask; d_supernode_flags n bytes (needed only with
 *     GSOFA_SUPERNODES); d_counters 8 entries: fills, edges_alg,
 *     vertices_alg, edges_traversed, supernodes detected (printed count - 1),
 *     nnz_u, nnz_l, sources chained.
 *   - GSOFA_L_ROW_STATS and GSOFA_PATTERN are not available here; digests are
 *     not computed.  Errors map as in gsofa_factor_symbolic (a queue bound
 *     exceeded, e.g. under GSOFA_DEBUG_QUEUE_CAP: GSOFA_ERR_OVERFLOW).
 *   - Synchronous: returns after the work queued on cuda_stream (NULL =
 *     legacy stream) has finished. */
#define GSOFA_NOALLOC_SCRATCH_BYTES (64u << 20)
int gsofa_factor_symbolic_noalloc(const gsofa_matrix* mat, const gsofa_opts* opts,
                                  void* cuda_stream, int32_t* d_nnz_u_row, int32_t* d_nz_row_u,
                                  int32_t* d_nnz_l_col, uint32_t* d_lmask,
                                  int8_t* d_supernode_flags, uint64_t* d_counters);

/* ---- reference-shaped entry point ------------------------------------------ */
/* Same argument layouts as the reference executables:
 *   SOA: exe beg end csr num_process max_supernode_size percent_cat0
 *        percent_cat2 N_blocks_source_cat2 N_GPU_Node N_src_group  (argc == 11)
 *   SPO: exe beg end csr N_virtualGPU total_memory_GB              (argc == 6)
 * Outputs mirror symbfact_min_id's reference parameters; teps_edges gets
 * edges_alg.  Process/GPU counts are accepted and folded onto one device. */
int gsofa_symbfact_min_id(int argc, char** argv, int rank, uint64_t* fill_count,
                          double* time_ms, int32_t* n_supernodes, uint64_t* teps_edges);

#ifdef __cplusplus
}
#endif
#endif /* GSOFA_H */
