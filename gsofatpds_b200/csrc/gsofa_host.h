// Host-side handle structures and helpers shared by the translation units
// of libgsofa.so (gsofa_capi.cpp: the C-ABI; gsofa_server.cpp: the request
// loop).  Not installed.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/gsofa.h"
#include "gsofa_internal.h"

struct gsofa_ctx {
    int device = 0;
    int sm_count = 0;
    int smem_optin = 0;
    int smem_per_sm = 0;
    size_t budget = 0;
    size_t used = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evt = nullptr;
    std::recursive_mutex mu;
    std::string err;
    // autotuner choices per class (log2 n, mean row length, locality: half-
    // octaves of the mean |i - j| of the entries over n)
    std::map<std::tuple<int, int, int>, gsofa_opts> tuned;
    // pinned staging
    unsigned long long* h_counters = nullptr;  // CNT_SLOTS
    int32_t* h_status = nullptr;
    // grown workspace
    void* queue = nullptr;
    size_t queue_bytes = 0;
    void* gbitmap = nullptr;
    size_t gbitmap_bytes = 0;
    void* gprev = nullptr;
    size_t gprev_bytes = 0;
    void* small = nullptr;  // work counter (8 B) + status (4 B)
    void* scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
};

struct gsofa_matrix {
    gsofa_ctx* ctx = nullptr;
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t* rowptr = nullptr;
    int32_t* col = nullptr;
    int32_t* trowptr = nullptr;
    int32_t* tcol = nullptr;
    int32_t* wdeg = nullptr;
    uint32_t* dplanes = nullptr;
    int32_t nplanes = 0;
    int32_t* asym = nullptr;  // device word: 0 iff the pattern is symmetric
    size_t bytes = 0;
    mutable int host_sym = -1;  // the device word read back once (-1: not yet)
};

struct gsofa_result {
    gsofa_ctx* ctx = nullptr;
    int32_t n = 0;
    uint32_t flags = 0;
    int32_t mss = 128;
    void* arena = nullptr;  // one device block holding every array below
    size_t bytes = 0;
    int32_t* nnz_u = nullptr;
    int32_t* nz_row_u = nullptr;
    uint64_t* dig_u = nullptr;
    int32_t* nnz_lc = nullptr;
    uint64_t* dig_lc = nullptr;
    uint32_t* lmask = nullptr;
    int32_t* nnz_lr = nullptr;
    uint64_t* dig_lr = nullptr;
    int8_t* sflags = nullptr;
    unsigned long long* counters = nullptr;
    uint8_t* link = nullptr;  // 2n: chained-start links between the directions
    uint32_t* umask = nullptr;  // 4n: U(f, f+1+j) bits, read by chained starts
    // pattern (separate allocation, only with GSOFA_PATTERN)
    void* parena = nullptr;
    size_t pbytes = 0;
    int64_t* uptr = nullptr;
    int32_t* ucols = nullptr;
    int64_t* lptr = nullptr;
    int32_t* lrows = nullptr;
    // supernodal block form (gsofa_result_supernodal), built on first request
    bool sn_built = false;
    long long sn_nblocks = 0, sn_nl = 0, sn_nu = 0;
    int32_t* sn_start = nullptr;
    int64_t* sn_lptr = nullptr;
    int32_t* sn_lrows = nullptr;
    int64_t* sn_uptr = nullptr;
    int32_t* sn_ucols = nullptr;
    gsofa_counts counts{};
    bool batch_owned = false;  // lives inside a gsofa_batch: not destroyed alone
};

struct gsofa_batch {
    gsofa_ctx* ctx = nullptr;
    int32_t count = 0;
    gsofa_opts opts{};
    std::vector<gsofa_result*> res;
    void* ws = nullptr;  // private workspace (graph holds raw pointers into it)
    size_t ws_bytes = 0;
    unsigned long long* h_counters = nullptr;  // pinned, count * CNT_SLOTS
    int32_t* h_status = nullptr;               // pinned
    cudaEvent_t e0 = nullptr, et = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long items = 0;
};

namespace gsofa {
namespace host {

int set_err(gsofa_ctx* ctx, int status, const char* fmt, ...);
// The reference's three ASCII files into host arrays (ctx may be null).
int parse_dat_files(gsofa_ctx* ctx, const char* beg_file, const char* end_file,
                    const char* csr_file, int32_t* n, int64_t* nnz, std::vector<int32_t>* beg,
                    std::vector<int32_t>* end, std::vector<int32_t>* col);
int cuda_fail(gsofa_ctx* ctx, cudaError_t e, const char* where);
// The context's device status word (DEV_ERR_*) and work counter; the
// status is read back into ctx->h_status and turned into a code by
// check_status.
int32_t* work_counter_status(gsofa_ctx* ctx, unsigned long long** wc);
int check_status(gsofa_ctx* ctx);
// Pool allocation with budget accounting, ordered on `stream`; the caller
// holds ctx->mu.
int dev_alloc_on(gsofa_ctx* ctx, size_t bytes, void** p, cudaStream_t stream);
void dev_free_on(gsofa_ctx* ctx, void* p, size_t bytes, cudaStream_t stream);
size_t align256(size_t x);
long long default_chunk(long long total_sources, int grid);
// m's share in the default chunk length: 2n for an unsymmetric pattern (a
// U-row and an L-column search per source), n/4 for a symmetric one (the
// U-row searches fill both halves, and its costly sources cluster in the top
// separators of a nested-dissection order, which shorter chunks spread over
// more CTAs).  Reads the ingest's symmetry word back once (synchronous on
// ctx->stream) and keeps it with m.
long long chunk_weight(gsofa_ctx* ctx, const gsofa_matrix* m);
int default_block(int32_t nmax, int smem_per_sm);
// Result arrays of an n-row matrix, zero-initialised on `stream`.
int result_alloc_on(gsofa_ctx* ctx, int32_t n, uint32_t flags, int32_t mss, cudaStream_t stream,
                    gsofa_result** out);
void result_free(gsofa_result* r);
void supernodal_free(gsofa_result* r);  // caller holds ctx->mu
MatDesc make_desc(const gsofa_matrix* m, const gsofa_result* r, long long base);
// Uploads from pageable host memory through a few pinned buffers: the host
// copies the next piece into one buffer while the previous piece's DMA
// runs, and no upload waits for the stream's earlier work to finish (a
// pageable cudaMemcpyAsync synchronises its stream first).  One caller at a
// time; upload() returns once the source may be reused.
struct PinnedStager {
    static constexpr int kBufs = 4;
    static constexpr size_t kPiece = 8u << 20;
    void* buf[kBufs] = {};
    cudaEvent_t ev[kBufs] = {};
    int next = 0;
    cudaError_t init();
    void release();
    cudaError_t upload(void* dst, const void* src, size_t bytes, cudaStream_t stream);
};
// Validates the row intervals on the host, then queues the upload and the
// padded-CSR build of A and A^T on `stream` without waiting.  Column ids
// outside [0, n) are reported in *dstatus (DEV_ERR_COL_RANGE) when the
// stream reaches the build.  The caller holds ctx->mu.  With `stager` the
// host arrays are uploaded through it (see PinnedStager), else directly.
int ingest_csr(gsofa_ctx* ctx, cudaStream_t stream, int32_t* dstatus, int32_t n, int64_t nnz,
               const int32_t* row_begin, const int32_t* row_end, const int32_t* col,
               gsofa_matrix** out, PinnedStager* stager = nullptr);
// A matrix handle and its device block for n rows, `real` entries and
// `padded` padded entries of A (rows rounded up to multiples of 4).
int matrix_alloc(gsofa_ctx* ctx, cudaStream_t stream, int32_t n, int64_t real, int64_t padded,
                 int nplanes, gsofa_matrix** out);
void matrix_free_on(gsofa_matrix* m, cudaStream_t stream);
// Queues the padded-CSR build of A and A^T on `stream`: m->rowptr (encoded)
// must already be on the device (or queued); row v of the input is
// dcol_in[dbeg[v] ...] with the length m->rowptr gives it.
int matrix_build(gsofa_ctx* ctx, cudaStream_t stream, int32_t* dstatus, gsofa_matrix* m,
                 int64_t nnz_in, const int32_t* dbeg, const int32_t* dcol_in, int check_symmetry);
// Device bytes ingest_csr holds for a matrix (kept) and while it runs (staging).
void ingest_bytes(int32_t n, int64_t nnz, size_t* kept, size_t* staging);
size_t result_bytes(int32_t n, uint32_t flags);

// Device blocks from the context's pool, released (stream-ordered on the
// context's stream) when the object goes out of scope.  get() returns null
// when the budget is exceeded.
struct DeviceScratch {
    gsofa_ctx* ctx;
    std::vector<std::pair<void*, size_t>> blocks;
    explicit DeviceScratch(gsofa_ctx* c) : ctx(c) {}
    DeviceScratch(const DeviceScratch&) = delete;
    DeviceScratch& operator=(const DeviceScratch&) = delete;
    void* get(size_t bytes) {
        const size_t b = bytes < 16 ? 16 : bytes;
        void* p = nullptr;
        if (dev_alloc_on(ctx, b, &p, ctx->stream)) return nullptr;
        blocks.emplace_back(p, b);
        return p;
    }
    ~DeviceScratch() {
        for (auto& b : blocks) dev_free_on(ctx, b.first, b.second, ctx->stream);
    }
};

constexpr int kDefaultBuAlpha = 0;  // top-down only unless a caller asks
constexpr int kDefaultBuBeta = 24;
constexpr int kBuMinSource = 2048;
constexpr int kDefaultHeavyRow = 16;  // padded rows above it are walked by a whole warp
constexpr int kDefaultRing = 64;
constexpr int kMaxRing = 64;  // the kernel's ring masks hold 64 slots
// a source search waits up to this long for the other direction's result
// when that search is one source behind (chained starts)
constexpr int kDefaultChainWaitUs = 300;
inline long long chain_wait_ns(const gsofa_opts& o) {
    const int us = o.chain_wait_us > 0 ? o.chain_wait_us : (o.chain_wait_us < 0 ? 0 : kDefaultChainWaitUs);
    return 1000ll * us;
}
// rows longer than this skip the ingest's symmetry check (its cost grows with
// the product of row lengths); such matrices are treated as unsymmetric
constexpr int64_t kSymmetryCheckMaxRow = 8192;

}  // namespace host
}  // namespace gsofa
