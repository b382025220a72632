// gsofa_capi.cpp -- host side of libgsofa.so: the C-ABI declared in
// include/gsofa.h.  Owns device memory (a dedicated stream-ordered pool with
// budget accounting), device-resident matrices and results, the launch
// configuration of the traversal kernel, and the reference-shaped entry point.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <cerrno>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gsofa_host.h"

using namespace gsofa;
using namespace gsofa::host;

// ---------------------------------------------------------------------------
namespace gsofa {
namespace host {

int set_err(gsofa_ctx* ctx, int status, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return status;
}

int cuda_fail(gsofa_ctx* ctx, cudaError_t e, const char* where) {
    return set_err(ctx, GSOFA_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define CK(call)                                          \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

int dev_alloc_on(gsofa_ctx* ctx, size_t bytes, void** p, cudaStream_t stream) {
    *p = nullptr;
    if (bytes == 0) return GSOFA_OK;
    bytes = (bytes + 255) & ~(size_t)255;
    if (ctx->used + bytes > ctx->budget)
        return set_err(ctx, GSOFA_ERR_OOM_BUDGET,
                       "allocation of %zu bytes exceeds the budget (%zu of %zu bytes in use)",
                       bytes, ctx->used, ctx->budget);
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(ctx, e, "cudaMallocFromPoolAsync");
    }
    ctx->used += bytes;
    return GSOFA_OK;
}

void dev_free_on(gsofa_ctx* ctx, void* p, size_t bytes, cudaStream_t stream) {
    if (!p) return;
    bytes = (bytes + 255) & ~(size_t)255;
    cudaFreeAsync(p, stream);
    ctx->used -= std::min(ctx->used, bytes);
}

int dev_alloc(gsofa_ctx* ctx, size_t bytes, void** p) {
    return dev_alloc_on(ctx, bytes, p, ctx->stream);
}

void dev_free(gsofa_ctx* ctx, void* p, size_t bytes) { dev_free_on(ctx, p, bytes, ctx->stream); }

// Grow-only workspace buffer.
int ensure(gsofa_ctx* ctx, void** p, size_t* have, size_t need) {
    if (*have >= need) return GSOFA_OK;
    dev_free(ctx, *p, *have);
    *p = nullptr;
    *have = 0;
    int rc = dev_alloc(ctx, need, p);
    if (rc) return rc;
    *have = (need + 255) & ~(size_t)255;
    return GSOFA_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

long long bitmap_words(int32_t n) { return (((long long)n + 31) >> 5) + 6; }

// Default chunk (consecutive sources per work item): total / grid, a power
// of 2 between 16 and 512 sources, where total weighs each matrix by
// chunk_weight -- about one item per CTA for unsymmetric patterns.  Each
// chunk's first source starts cold (nothing to reuse), while later ones
// mostly start from their predecessor's closure, so long chunks pay; the
// autotuner tries shorter and longer ones.
long long default_chunk(long long total_sources, int grid) {
    long long c = total_sources / (grid > 0 ? grid : 1);
    long long p = 16;
    while (p * 2 <= c && p < 512) p *= 2;
    return p;
}

// Launch order of a batch's matrices: most entries first (longest processing
// time first), so that the persistent kernel's last items are small ones and
// no large matrix starts when the rest of the batch is almost done.
std::vector<int32_t> batch_order(const gsofa_matrix* const* mats, int32_t count) {
    std::vector<int32_t> order((size_t)count);
    for (int32_t i = 0; i < count; i++) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return mats[a]->nnz > mats[b]->nnz; });
    return order;
}

long long chunk_weight(gsofa_ctx* ctx, const gsofa_matrix* m) {
    if (m->host_sym < 0) {
        int sym = 0;
        if (m->n > 0 &&
            cudaMemcpyAsync(ctx->h_status + 1, m->asym, 4, cudaMemcpyDeviceToHost, ctx->stream) ==
                cudaSuccess &&
            cudaStreamSynchronize(ctx->stream) == cudaSuccess)
            sym = ctx->h_status[1] == 0;
        else
            cudaGetLastError();
        m->host_sym = sym;
    }
    return m->host_sym ? m->n / 4 : 2ll * m->n;
}

// Default CTA size: about 1024 resident threads per SM (the kernel is held
// to 64 registers), given how many shared-memory bitmaps fit per SM.
// Measured on B200: 256-thread CTAs are fastest whenever 4 fit, else fewer,
// larger CTAs.
int default_block(int32_t nmax, int smem_per_sm) {
    const long long words = (((long long)nmax + 31) >> 5) + 6;
    const long long per_cta = ((words * 4 + 15) & ~15ll) + 8 * 1024;
    long long fit = smem_per_sm / per_cta;
    if (fit >= 4) return 256;
    if (fit >= 2) return 512;
    return 1024;
}

struct LaunchCfg {
    int block = 512;
    int grid = 0;
    bool smem_bitmap = true;
    size_t smem = 0;
    long long words = 0;
};

int plan_launch(gsofa_ctx* ctx, int32_t nmax, const gsofa_opts* o, LaunchCfg* c) {
    c->block = o->threads_per_source > 0 ? o->threads_per_source
                                         : default_block(nmax, ctx->smem_per_sm);
    if (c->block != 128 && c->block != 256 && c->block != 512 && c->block != 1024)
        return set_err(ctx, GSOFA_ERR_ARG, "threads_per_source must be 128, 256, 512 or 1024");
    c->words = bitmap_words(nmax);
    size_t bytes = (size_t)c->words * 4;
    bytes = (bytes + 15) & ~(size_t)15;
    // leave room for the kernel's static shared memory (reduction + scan)
    c->smem_bitmap = bytes + 12 * 1024 <= (size_t)ctx->smem_optin &&
                     !(o->flags & GSOFA_FORCE_GLOBAL_BITMAP);
    c->smem = c->smem_bitmap ? bytes : 0;
    int occ = traverse_occupancy(c->block, c->smem_bitmap, c->smem);
    if (occ <= 0)
        return set_err(ctx, GSOFA_ERR_UNSUPPORTED,
                       "traversal kernel cannot be resident (block %d, %zu B shared)", c->block,
                       c->smem);
    c->grid = occ * ctx->sm_count;
    if (o->sources_in_flight > 0) c->grid = std::min(c->grid, o->sources_in_flight);
    return GSOFA_OK;
}

int check_status(gsofa_ctx* ctx) {
    const int32_t s = *ctx->h_status;
    const int code = device_status_code(s);
    if (code == GSOFA_OK) return GSOFA_OK;
    if (s & DEV_ERR_COL_RANGE) return set_err(ctx, code, "column id outside [0, n)");
    if (s & DEV_ERR_ROW_RANGE) return set_err(ctx, code, "row interval outside [0, nnz)");
    return set_err(ctx, code, "traversal queue bound exceeded");
}

int32_t* work_counter_status(gsofa_ctx* ctx, unsigned long long** wc) {
    *wc = reinterpret_cast<unsigned long long*>(ctx->small);
    return reinterpret_cast<int32_t*>(reinterpret_cast<char*>(ctx->small) + 64);
}

void result_free(gsofa_result* r) {
    if (!r) return;
    if (r->ctx) {
        std::lock_guard<std::recursive_mutex> g(r->ctx->mu);
        dev_free(r->ctx, r->arena, r->bytes);
        dev_free(r->ctx, r->parena, r->pbytes);
        supernodal_free(r);
    }
    delete r;
}

// Layout of a result arena: the per-row arrays of an n-row matrix.
static size_t result_layout(int32_t n, uint32_t flags, size_t off[12]) {
    const size_t N = (size_t)std::max(n, 1);
    const bool dig = flags & GSOFA_DIGESTS;
    const bool lrow = flags & GSOFA_L_ROW_STATS;
    size_t sz[12];
    sz[0] = 4 * N;                       // nnz_u
    sz[1] = 4 * N;                       // nz_row_u
    sz[2] = dig ? 8 * N : 0;             // dig_u
    sz[3] = 4 * N;                       // nnz_lc
    sz[4] = dig ? 8 * N : 0;             // dig_lc
    sz[5] = 16 * N;                      // lmask
    sz[6] = lrow ? 4 * N : 0;            // nnz_lr
    sz[7] = lrow ? 8 * N : 0;            // dig_lr
    sz[8] = N;                           // supernode flags
    sz[9] = 8 * CNT_SLOTS;               // counters
    sz[10] = 2 * N;                      // link (chained starts)
    sz[11] = 16 * N;                     // umask (chained starts)
    size_t total = 0;
    for (int i = 0; i < 12; i++) {
        off[i] = total;
        total += align256(sz[i]);
    }
    return total;
}

size_t result_bytes(int32_t n, uint32_t flags) {
    size_t off[12];
    return result_layout(n, flags, off);
}

// Carve the per-row result arrays out of one arena.
int result_alloc_on(gsofa_ctx* ctx, int32_t n, uint32_t flags, int32_t mss, cudaStream_t stream,
                    gsofa_result** out) {
    gsofa_result* r = new (std::nothrow) gsofa_result();
    if (!r) return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "host allocation failed");
    r->ctx = ctx;
    r->n = n;
    r->flags = flags;
    r->mss = mss;
    const size_t N = (size_t)std::max(n, 1);
    const bool dig = flags & GSOFA_DIGESTS;
    const bool lrow = flags & GSOFA_L_ROW_STATS;
    size_t off[12];
    const size_t total = result_layout(n, flags, off);
    int rc = dev_alloc_on(ctx, total, &r->arena, stream);
    if (rc) {
        delete r;
        return rc;
    }
    r->bytes = total;
    char* b = reinterpret_cast<char*>(r->arena);
    r->nnz_u = reinterpret_cast<int32_t*>(b + off[0]);
    r->nz_row_u = reinterpret_cast<int32_t*>(b + off[1]);
    r->dig_u = dig ? reinterpret_cast<uint64_t*>(b + off[2]) : nullptr;
    r->nnz_lc = reinterpret_cast<int32_t*>(b + off[3]);
    r->dig_lc = dig ? reinterpret_cast<uint64_t*>(b + off[4]) : nullptr;
    r->lmask = reinterpret_cast<uint32_t*>(b + off[5]);
    r->nnz_lr = lrow ? reinterpret_cast<int32_t*>(b + off[6]) : nullptr;
    r->dig_lr = lrow ? reinterpret_cast<uint64_t*>(b + off[7]) : nullptr;
    r->sflags = reinterpret_cast<int8_t*>(b + off[8]);
    r->counters = reinterpret_cast<unsigned long long*>(b + off[9]);
    r->link = reinterpret_cast<uint8_t*>(b + off[10]);
    r->umask = reinterpret_cast<uint32_t*>(b + off[11]);
    // zero the scatter targets, the counters and the flags
    cudaError_t e = cudaSuccess;
    if (lrow) {
        e = cudaMemsetAsync(r->nnz_lr, 0, 4 * N, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(r->dig_lr, 0, 8 * N, stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(r->counters, 0, 8 * CNT_SLOTS, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(r->sflags, 0, N, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(r->link, 0, 2 * N, stream);
    if (e != cudaSuccess) {
        dev_free_on(ctx, r->arena, r->bytes, stream);
        delete r;
        return cuda_fail(ctx, e, "result init");
    }
    *out = r;
    return GSOFA_OK;
}

int result_alloc(gsofa_ctx* ctx, int32_t n, uint32_t flags, int32_t mss, gsofa_result** out) {
    return result_alloc_on(ctx, n, flags, mss, ctx->stream, out);
}

MatDesc make_desc(const gsofa_matrix* m, const gsofa_result* r, long long base) {
    MatDesc d{};
    d.n = m->n;
    d.flags = (int32_t)r->flags;
    d.rowptr = m->rowptr;
    d.col = m->col;
    d.trowptr = m->trowptr;
    d.tcol = m->tcol;
    d.wdeg = m->wdeg;
    d.dplanes = m->dplanes;
    d.nplanes = m->nplanes;
    d.asym = m->asym;
    d.nnz_u = r->nnz_u;
    d.nz_row_u = r->nz_row_u;
    d.dig_u = r->dig_u;
    d.nnz_lc = r->nnz_lc;
    d.dig_lc = r->dig_lc;
    d.lmask = r->lmask;
    d.sflags = r->sflags;
    d.nnz_lr = r->nnz_lr;
    d.dig_lr = r->dig_lr;
    d.counters = r->counters;
    d.uptr = r->uptr;
    d.ucols = r->ucols;
    d.lptr = r->lptr;
    d.lrows = r->lrows;
    d.link = r->link;
    d.umask = r->umask;
    d.item_base = base;
    return d;
}

// Runs the traversal (and optionally supernodes / pattern) for `count`
// matrices in one persistent launch.  results[i] must be freshly allocated.
int run_factor(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
               const gsofa_opts* o, gsofa_result** res, long long sample_stride = 1) {
    int32_t nmax = 0;
    long long items = 0;
    long long total_sources = 0;
    for (int32_t i = 0; i < count; i++) {
        nmax = std::max(nmax, mats[i]->n);
        total_sources += chunk_weight(ctx, mats[i]);
    }
    LaunchCfg cfg;
    int rc = plan_launch(ctx, std::max(nmax, 1), o, &cfg);
    if (rc) return rc;
    // So few sources that each can have a CTA of its own: chunks of one source
    // run them all at once (a 115-row matrix: 0.06 instead of 0.23 ms); with
    // more, chunks share closures between consecutive sources.
    long long one_each = 0;
    for (int32_t i = 0; i < count; i++) one_each += 2ll * mats[i]->n;
    const long long chunk = o->chunk_sources > 0 ? o->chunk_sources
                            : one_each <= cfg.grid ? 1
                                                   : default_chunk(total_sources, cfg.grid);
    for (int32_t i = 0; i < count; i++) items += 2ll * ((mats[i]->n + chunk - 1) / chunk);
    rc = ensure(ctx, &ctx->queue, &ctx->queue_bytes, (size_t)cfg.grid * (size_t)std::max(nmax, 1) * 4);
    if (rc) return rc;
    if (!cfg.smem_bitmap) {
        rc = ensure(ctx, &ctx->gbitmap, &ctx->gbitmap_bytes, (size_t)cfg.grid * (size_t)cfg.words * 4);
        if (rc) return rc;
    }
    const bool merge = !(o->flags & GSOFA_NO_MERGE);
    int ring = o->cached_closures > 0 ? o->cached_closures : kDefaultRing;
    if (ring > kMaxRing) ring = kMaxRing;
    while (ring & (ring - 1)) ring &= ring - 1;  // power of 2
    if (merge) {
        rc = ensure(ctx, &ctx->gprev, &ctx->gprev_bytes,
                    (size_t)cfg.grid * (size_t)ring * (size_t)cfg.words * 4);
        if (rc) return rc;
    }
    // matrix descriptors, largest matrices first
    const std::vector<int32_t> order = batch_order(mats, count);
    std::vector<MatDesc> descs((size_t)count);
    long long base = 0;
    for (int32_t k = 0; k < count; k++) {
        const int32_t i = order[(size_t)k];
        descs[(size_t)k] = make_desc(mats[i], res[i], base);
        base += 2ll * ((mats[i]->n + chunk - 1) / chunk);
    }
    void* ddesc = nullptr;
    rc = dev_alloc(ctx, sizeof(MatDesc) * (size_t)count, &ddesc);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ddesc, descs.data(), sizeof(MatDesc) * (size_t)count, cudaMemcpyHostToDevice,
                       ctx->stream));
    unsigned long long* wc = nullptr;
    int32_t* dstatus = work_counter_status(ctx, &wc);
    CK(cudaMemsetAsync(ctx->small, 0, 128, ctx->stream));

    TraverseLaunch L{};
    L.mats = reinterpret_cast<const MatDesc*>(ddesc);
    L.nmats = count;
    L.total_items = sample_stride > 1 ? (items + sample_stride - 1) / sample_stride : items;
    L.sample_stride = sample_stride > 1 ? sample_stride : 1;
    L.work_counter = wc;
    L.queue = reinterpret_cast<int32_t*>(ctx->queue);
    L.queue_stride = std::max(nmax, 1);
    if (o->flags & GSOFA_DEBUG_QUEUE_CAP) L.queue_stride = std::min<long long>(L.queue_stride, 64);
    L.gbitmap = reinterpret_cast<uint32_t*>(ctx->gbitmap);
    L.bitmap_words = cfg.words;
    L.status = dstatus;
    L.pattern_pass = 0;
    L.bu_alpha = o->bu_alpha > 0 ? o->bu_alpha : (o->bu_alpha < 0 ? 0 : kDefaultBuAlpha);
    L.bu_beta = o->bu_beta > 0 ? o->bu_beta : kDefaultBuBeta;
    L.bu_min_src = o->bu_min_source > 0 ? o->bu_min_source : kBuMinSource;
    L.gprev = reinterpret_cast<uint32_t*>(ctx->gprev);
    L.merge = merge ? 1 : 0;
    L.chain = merge && !(o->flags & GSOFA_NO_CHAIN) ? 1 : 0;
    L.chain_wait_ns = chain_wait_ns(*o);
    L.ring = ring;
    L.chunk = (int)chunk;
    L.heavy_len = o->heavy_row > 0 ? ((o->heavy_row + 3) & ~3) : kDefaultHeavyRow;

    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (items > 0) CK(launch_traverse(L, cfg.block, cfg.grid, cfg.smem_bitmap, cfg.smem, ctx->stream));
    CK(cudaEventRecord(ctx->evt, ctx->stream));
    for (int32_t i = 0; i < count; i++) {
        if ((o->flags & GSOFA_SUPERNODES) && mats[i]->n > 0)
            CK(launch_supernodes(mats[i]->n, o->max_supernode_size, res[i]->nz_row_u, res[i]->lmask,
                                 res[i]->sflags, res[i]->counters, ctx->stream));
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_status, dstatus, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    rc = check_status(ctx);
    if (rc) {
        dev_free(ctx, ddesc, sizeof(MatDesc) * (size_t)count);
        return rc;
    }
    float ms = 0.f, ms_trav = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    CK(cudaEventElapsedTime(&ms_trav, ctx->ev0, ctx->evt));

    // pattern pass (second traversal writing sorted ids)
    if (o->flags & GSOFA_PATTERN) {
        for (int32_t k = 0; k < count; k++) {
            const int32_t i = order[(size_t)k];
            gsofa_result* r = res[i];
            CK(cudaMemcpyAsync(ctx->h_counters, r->counters, 8 * CNT_SLOTS, cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            const size_t N = (size_t)r->n + 1;
            const size_t nu = ctx->h_counters[CNT_NNZ_U], nl = ctx->h_counters[CNT_NNZ_L];
            size_t total = align256(8 * N) * 2 + align256(4 * std::max<size_t>(nu, 1)) +
                           align256(4 * std::max<size_t>(nl, 1));
            rc = dev_alloc(ctx, total, &r->parena);
            if (rc) return rc;
            r->pbytes = total;
            char* b = reinterpret_cast<char*>(r->parena);
            r->uptr = reinterpret_cast<int64_t*>(b);
            r->lptr = reinterpret_cast<int64_t*>(b + align256(8 * N));
            r->ucols = reinterpret_cast<int32_t*>(b + 2 * align256(8 * N));
            r->lrows = reinterpret_cast<int32_t*>(b + 2 * align256(8 * N) +
                                                  align256(4 * std::max<size_t>(nu, 1)));
            rc = ensure(ctx, &ctx->scan_tmp, &ctx->scan_tmp_bytes, pattern_scan_bytes(r->n));
            if (rc) return rc;
            CK(launch_pattern_ptrs(r->n, r->nnz_u, r->nnz_lc, r->uptr, r->lptr, ctx->scan_tmp,
                                   ctx->scan_tmp_bytes, ctx->stream));
            descs[(size_t)k] = make_desc(mats[i], r, descs[(size_t)k].item_base);
        }
        CK(cudaMemcpyAsync(ddesc, descs.data(), sizeof(MatDesc) * (size_t)count,
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(ctx->small, 0, 128, ctx->stream));
        L.pattern_pass = 1;
        if (items > 0)
            CK(launch_traverse(L, cfg.block, cfg.grid, cfg.smem_bitmap, cfg.smem, ctx->stream));
        CK(cudaMemcpyAsync(ctx->h_status, dstatus, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        rc = check_status(ctx);
        if (rc) {
            dev_free(ctx, ddesc, sizeof(MatDesc) * (size_t)count);
            return rc;
        }
    }
    dev_free(ctx, ddesc, sizeof(MatDesc) * (size_t)count);

    for (int32_t i = 0; i < count; i++) {
        gsofa_result* r = res[i];
        CK(cudaMemcpyAsync(ctx->h_counters, r->counters, 8 * CNT_SLOTS, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const unsigned long long* c = ctx->h_counters;
        gsofa_counts& k = r->counts;
        k.n = r->n;
        k.fill_count = c[CNT_FILLS];
        k.nnz_l = c[CNT_NNZ_L];
        k.nnz_u = c[CNT_NNZ_U];
        k.nnz_lu = c[CNT_NNZ_L] + c[CNT_NNZ_U] + (uint64_t)r->n;
        k.n_supernodes = (o->flags & GSOFA_SUPERNODES) ? (int64_t)c[CNT_NSUP] + 1 : -1;
        k.edges_alg = c[CNT_EDGES_ALG];
        k.vertices_alg = c[CNT_VERTS_ALG];
        k.edges_traversed = c[CNT_EDGES_TRAV];
        k.sources_chained = c[CNT_CHAINED];
        k.ms_device = (double)ms;  // for a batch: the whole launch
        k.ms_traverse = (double)ms_trav;
    }
    return GSOFA_OK;
}

int validate_opts(gsofa_ctx* ctx, const gsofa_opts* o) {
    if (o->max_supernode_size <= 0)
        return set_err(ctx, GSOFA_ERR_ARG, "max_supernode_size must be positive");
    if (o->threads_per_source < 0 || o->sources_in_flight < 0 || o->chunk_sources < 0 ||
        o->cached_closures < 0)
        return set_err(ctx, GSOFA_ERR_ARG, "negative launch option");
    return GSOFA_OK;
}

// ---- fast ASCII reader --------------------------------------------------------
int read_file(const char* path, std::string* out) {
    FILE* f = fopen(path, "rb");
    if (!f) return -1;
    if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return -1; }
    long sz = ftell(f);
    if (sz < 0) { fclose(f); return -1; }
    rewind(f);
    out->resize((size_t)sz);
    size_t got = sz ? fread(&(*out)[0], 1, (size_t)sz, f) : 0;
    fclose(f);
    return got == (size_t)sz ? 0 : -1;
}

// Parses up to `count` whitespace-separated integers; returns how many.
int64_t parse_ints(const std::string& s, size_t* pos, int64_t count, int32_t* out, bool* bad) {
    const char* p = s.data() + *pos;
    const char* e = s.data() + s.size();
    int64_t i = 0;
    while (i < count) {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
        if (p >= e) break;
        bool neg = false;
        if (*p == '-') { neg = true; p++; }
        if (p >= e || *p < '0' || *p > '9') { *bad = true; break; }
        int64_t v = 0;
        while (p < e && *p >= '0' && *p <= '9') { v = v * 10 + (*p - '0'); p++; if (v > 4294967295ll) { *bad = true; break; } }
        out[i++] = (int32_t)(neg ? -v : v);
    }
    *pos = (size_t)(p - s.data());
    return i;
}

// The reference's three ASCII files (csr = "E N" then E column ids, beg /
// end = n ids each) into host arrays.  ctx may be null (no message kept).
int parse_dat_files(gsofa_ctx* ctx, const char* beg_file, const char* end_file,
                    const char* csr_file, int32_t* n_out, int64_t* nnz_out,
                    std::vector<int32_t>* beg, std::vector<int32_t>* end,
                    std::vector<int32_t>* col) {
    std::string sc, sb, se;
    if (read_file(csr_file, &sc)) return set_err(ctx, GSOFA_ERR_IO, "cannot read %s", csr_file);
    size_t pos = 0;
    bool bad = false;
    int32_t hdr[2];
    if (parse_ints(sc, &pos, 2, hdr, &bad) != 2 || bad || hdr[0] < 0 || hdr[1] < 0)
        return set_err(ctx, GSOFA_ERR_IO, "%s: bad header (expected E N)", csr_file);
    const int64_t E = hdr[0];
    const int32_t n = hdr[1];
    col->assign((size_t)std::max<int64_t>(E, 1), 0);
    beg->assign((size_t)n + 1, 0);
    end->assign((size_t)n + 1, 0);
    if (parse_ints(sc, &pos, E, col->data(), &bad) != E || bad)
        return set_err(ctx, GSOFA_ERR_IO, "%s: expected %lld column ids", csr_file, (long long)E);
    if (read_file(beg_file, &sb)) return set_err(ctx, GSOFA_ERR_IO, "cannot read %s", beg_file);
    if (read_file(end_file, &se)) return set_err(ctx, GSOFA_ERR_IO, "cannot read %s", end_file);
    pos = 0;
    if (parse_ints(sb, &pos, n, beg->data(), &bad) != n || bad)
        return set_err(ctx, GSOFA_ERR_IO, "%s: expected %d row starts", beg_file, n);
    pos = 0;
    if (parse_ints(se, &pos, n, end->data(), &bad) != n || bad)
        return set_err(ctx, GSOFA_ERR_IO, "%s: expected %d row ends", end_file, n);
    *n_out = n;
    *nnz_out = E;
    return GSOFA_OK;
}

}  // namespace host
}  // namespace gsofa

bool gsofa::matrix_view(const void* mat, MatrixView* out) {
    const gsofa_matrix* m = static_cast<const gsofa_matrix*>(mat);
    if (!m || !out || !m->ctx) return false;
    out->device = m->ctx->device;
    out->n = m->n;
    out->rowptr = m->rowptr;
    out->col = m->col;
    out->trowptr = m->trowptr;
    out->tcol = m->tcol;
    out->wdeg = m->wdeg;
    out->dplanes = m->dplanes;
    out->nplanes = m->nplanes;
    out->asym = m->asym;
    return true;
}

void gsofa::host::ingest_bytes(int32_t n, int64_t nnz, size_t* kept, size_t* staging) {
    // padded A: each row rounded up to 4 entries (at most 3n pads); A^T: the same bound
    const size_t N1 = (size_t)n + 1;
    const size_t PT = (size_t)std::max<int64_t>(nnz + 3ll * n, 4);
    const size_t NW = (size_t)(((int64_t)n + 31) >> 5) + 1;
    *kept = align256(4 * N1) * 2 + align256(4 * PT) * 2 + align256(4 * NW) * 32 + 256;
    const size_t Nin = (size_t)std::max<int64_t>(nnz, 1);
    *staging = align256(4 * N1) + align256(4 * Nin) + align256(4 * N1) * 3 +
               align256(canonicalize_scan_bytes(n)) + 256;
}

cudaError_t gsofa::host::PinnedStager::init() {
    for (int k = 0; k < kBufs; k++) {
        cudaError_t e = cudaHostAlloc(&buf[k], kPiece, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void gsofa::host::PinnedStager::release() {
    for (int k = 0; k < kBufs; k++) {
        if (ev[k]) cudaEventSynchronize(ev[k]);
        if (buf[k]) cudaFreeHost(buf[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
        buf[k] = nullptr;
        ev[k] = nullptr;
    }
}

cudaError_t gsofa::host::PinnedStager::upload(void* dst, const void* src, size_t bytes,
                                              cudaStream_t stream) {
    const char* p = static_cast<const char*>(src);
    char* d = static_cast<char*>(dst);
    while (bytes > 0) {
        const size_t k = std::min(bytes, kPiece);
        // the buffer's previous DMA is complete before it is refilled
        cudaError_t e = cudaEventSynchronize(ev[next]);
        if (e != cudaSuccess) return e;
        std::memcpy(buf[next], p, k);
        e = cudaMemcpyAsync(d, buf[next], k, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[next], stream);
        if (e != cudaSuccess) return e;
        next = (next + 1) % kBufs;
        p += k;
        d += k;
        bytes -= k;
    }
    return cudaSuccess;
}

int gsofa::host::ingest_csr(gsofa_ctx* ctx, cudaStream_t stream, int32_t* dstatus, int32_t n,
                            int64_t nnz, const int32_t* row_begin, const int32_t* row_end,
                            const int32_t* col, gsofa_matrix** out, PinnedStager* stager) {
    *out = nullptr;
    if (n < 0 || nnz < 0) return set_err(ctx, GSOFA_ERR_ARG, "negative n or nnz");
    if (n > 0 && (!row_begin || !row_end)) return set_err(ctx, GSOFA_ERR_ARG, "null row arrays");
    if (nnz > 0 && !col) return set_err(ctx, GSOFA_ERR_ARG, "null column array");
    if (nnz > INT32_MAX) return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "nnz above 2^31-1");
    // host: padded row pointers of A.  Row v gets a multiple of 4 slots; the
    // number of padding slots of row v sits in the low 2 bits of rp[v+1].
    std::vector<int32_t> rp((size_t)n + 1);
    int64_t acc = 0, real = 0, maxd = 0;
    rp[0] = 0;
    for (int32_t v = 0; v < n; v++) {
        const int64_t b = row_begin[v], e = row_end[v];
        if (b < 0 || e < b || e > nnz)
            return set_err(ctx, GSOFA_ERR_ARG, "row %d interval [%lld,%lld) outside [0,%lld)", v,
                           (long long)b, (long long)e, (long long)nnz);
        const int64_t d = e - b, pd = (d + 3) & ~(int64_t)3;
        real += d;
        if (d > maxd) maxd = d;
        acc += pd;
        if (acc > INT32_MAX - 4 || real + 3ll * n > INT32_MAX - 4)
            return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "padded nnz above 2^31");
        rp[(size_t)v + 1] = (int32_t)(acc | (pd - d));
    }
    const int64_t padded = acc;
    int nplanes = 0;
    while (nplanes < 32 && (maxd >> nplanes) != 0) nplanes++;
    gsofa_matrix* m = nullptr;
    int rc = matrix_alloc(ctx, stream, n, real, padded, nplanes, &m);
    if (rc) return rc;
    // staging: the raw input (row starts, column ids)
    const size_t N1 = (size_t)n + 1;
    const size_t Nin = (size_t)std::max<int64_t>(nnz, 1);
    const size_t stage = align256(4 * N1) + align256(4 * Nin);
    void* sblk = nullptr;
    rc = dev_alloc_on(ctx, stage, &sblk, stream);
    if (rc) { matrix_free_on(m, stream); return rc; }
    int32_t* dbeg = reinterpret_cast<int32_t*>(sblk);
    int32_t* dcol_in = reinterpret_cast<int32_t*>(reinterpret_cast<char*>(sblk) + align256(4 * N1));
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return stager ? stager->upload(dst, src, bytes, stream)
                      : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    };
    cudaError_t e = up(m->rowptr, rp.data(), 4 * N1);
    if (e == cudaSuccess && n > 0) e = up(dbeg, row_begin, 4 * (size_t)n);
    if (e == cudaSuccess && nnz > 0) e = up(dcol_in, col, 4 * (size_t)nnz);
    if (e != cudaSuccess) {
        dev_free_on(ctx, sblk, stage, stream);
        matrix_free_on(m, stream);
        return cuda_fail(ctx, e, "ingest upload");
    }
    rc = matrix_build(ctx, stream, dstatus, m, nnz, dbeg, dcol_in,
                      maxd <= kSymmetryCheckMaxRow ? 1 : 0);
    dev_free_on(ctx, sblk, stage, stream);  // stream-ordered: after the build
    if (rc) { matrix_free_on(m, stream); return rc; }
    *out = m;
    return GSOFA_OK;
}

int gsofa::host::matrix_alloc(gsofa_ctx* ctx, cudaStream_t stream, int32_t n, int64_t real,
                              int64_t padded, int nplanes, gsofa_matrix** out) {
    *out = nullptr;
    gsofa_matrix* m = new (std::nothrow) gsofa_matrix();
    if (!m) return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "host allocation failed");
    m->ctx = ctx;
    m->n = n;
    m->nnz = real;
    m->nplanes = nplanes;
    const size_t N1 = (size_t)n + 1;
    const size_t PA = (size_t)std::max<int64_t>(padded, 4);
    const size_t PT = (size_t)std::max<int64_t>(real + 3ll * n, 4);  // bound for A^T
    const size_t NW = (size_t)(((int64_t)n + 31) >> 5) + 1;
    size_t total = align256(4 * N1) * 2 + align256(4 * PA) + align256(4 * PT) + align256(4 * NW) +
                   align256(4 * NW * (size_t)std::max(nplanes, 1)) + 256;
    void* blk = nullptr;
    int rc = dev_alloc_on(ctx, total, &blk, stream);
    if (rc) { delete m; return rc; }
    m->bytes = total;
    char* b = reinterpret_cast<char*>(blk);
    m->rowptr = reinterpret_cast<int32_t*>(b);
    m->trowptr = reinterpret_cast<int32_t*>(b + align256(4 * N1));
    m->col = reinterpret_cast<int32_t*>(b + 2 * align256(4 * N1));
    m->tcol = reinterpret_cast<int32_t*>(b + 2 * align256(4 * N1) + align256(4 * PA));
    m->wdeg = reinterpret_cast<int32_t*>(b + 2 * align256(4 * N1) + align256(4 * PA) +
                                         align256(4 * PT));
    m->dplanes = reinterpret_cast<uint32_t*>(b + 2 * align256(4 * N1) + align256(4 * PA) +
                                             align256(4 * PT) + align256(4 * NW));
    m->asym = reinterpret_cast<int32_t*>(b + total - 256);
    *out = m;
    return GSOFA_OK;
}

void gsofa::host::matrix_free_on(gsofa_matrix* m, cudaStream_t stream) {
    if (!m) return;
    dev_free_on(m->ctx, m->rowptr, m->bytes, stream);
    delete m;
}

int gsofa::host::matrix_build(gsofa_ctx* ctx, cudaStream_t stream, int32_t* dstatus,
                              gsofa_matrix* m, int64_t nnz_in, const int32_t* dbeg,
                              const int32_t* dcol_in, int check_symmetry) {
    const int32_t n = m->n;
    const size_t N1 = (size_t)n + 1;
    size_t scan_bytes = canonicalize_scan_bytes(n);
    const size_t stage = align256(4 * N1) * 3 + align256(scan_bytes) + 256;
    void* sblk = nullptr;
    int rc = dev_alloc_on(ctx, stage, &sblk, stream);
    if (rc) return rc;
    char* s = reinterpret_cast<char*>(sblk);
    int32_t* tcount = reinterpret_cast<int32_t*>(s);
    s += align256(4 * N1);
    int32_t* tfill = reinterpret_cast<int32_t*>(s);
    s += align256(4 * N1);
    int32_t* tpad = reinterpret_cast<int32_t*>(s);
    s += align256(4 * N1);
    void* scan_tmp = s;
    cudaError_t e = cudaSuccess;
    if (n == 0) e = cudaMemsetAsync(m->trowptr, 0, 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(tcount, 0, 4 * N1, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(tfill, 0, 4 * N1, stream);
    if (e == cudaSuccess)
        e = launch_canonicalize(n, nnz_in, dbeg, dcol_in, m->rowptr, m->col, tcount, tpad,
                                m->trowptr, m->tcol, tfill, m->wdeg, m->dplanes, m->nplanes,
                                m->asym, check_symmetry, scan_tmp, scan_bytes, dstatus, stream);
    dev_free_on(ctx, sblk, stage, stream);  // stream-ordered: after the build
    return e == cudaSuccess ? GSOFA_OK : cuda_fail(ctx, e, "matrix build");
}

// ============================================================================
extern "C" {

const char* gsofa_status_string(int s) {
    switch (s) {
        case GSOFA_OK: return "ok";
        case GSOFA_ERR_ARG: return "invalid argument";
        case GSOFA_ERR_IO: return "i/o error";
        case GSOFA_ERR_OOM_BUDGET: return "memory budget exceeded";
        case GSOFA_ERR_TIMEOUT: return "device wait timed out";
        case GSOFA_ERR_OVERFLOW: return "queue bound exceeded";
        case GSOFA_ERR_CUDA: return "cuda error";
        case GSOFA_ERR_UNSUPPORTED: return "unsupported size or option";
        case GSOFA_ERR_BUSY: return "busy";
        default: return "unknown status";
    }
}

int gsofa_opts_default(gsofa_opts* o) {
    if (!o) return GSOFA_ERR_ARG;
    o->max_supernode_size = 128;
    o->threads_per_source = 0;
    o->sources_in_flight = 0;
    o->flags = GSOFA_SUPERNODES | GSOFA_DIGESTS;
    o->bu_alpha = 0;
    o->bu_beta = 0;
    o->heavy_row = 0;
    o->bu_min_source = 0;
    o->chunk_sources = 0;
    o->cached_closures = 0;
    o->chain_wait_us = 0;
    o->reserved = 0;
    return GSOFA_OK;
}

int gsofa_create(int device, size_t budget_bytes, gsofa_ctx** out) {
    if (!out) return GSOFA_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GSOFA_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return GSOFA_ERR_ARG;
    gsofa_ctx* ctx = new (std::nothrow) gsofa_ctx();
    if (!ctx) return GSOFA_ERR_OOM_BUDGET;
    ctx->device = device;
    auto fail = [&](cudaError_t e) {
        (void)e;
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        if (ctx->ev0) cudaEventDestroy(ctx->ev0);
        if (ctx->ev1) cudaEventDestroy(ctx->ev1);
        if (ctx->evt) cudaEventDestroy(ctx->evt);
        if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
        if (ctx->h_status) cudaFreeHost(ctx->h_status);
        if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
        delete ctx;
        return GSOFA_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&ctx->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    cudaDeviceGetAttribute(&ctx->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    size_t fr = 0, tot = 0;
    if ((e = cudaMemGetInfo(&fr, &tot)) != cudaSuccess) return fail(e);
    ctx->budget = budget_bytes ? budget_bytes : (size_t)(0.9 * (double)fr);
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e);
    ctx->stream = ctx->own_stream;
    if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&ctx->evt)) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost((void**)&ctx->h_counters, 8 * CNT_SLOTS)) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost((void**)&ctx->h_status, 64)) != cudaSuccess) return fail(e);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) return fail(e);
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (dev_alloc(ctx, 256, &ctx->small) != GSOFA_OK) return fail(cudaErrorMemoryAllocation);
    *out = ctx;
    return GSOFA_OK;
}

int gsofa_destroy(gsofa_ctx* ctx) {
    if (!ctx) return GSOFA_ERR_ARG;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        dev_free(ctx, ctx->queue, ctx->queue_bytes);
        dev_free(ctx, ctx->gbitmap, ctx->gbitmap_bytes);
        dev_free(ctx, ctx->gprev, ctx->gprev_bytes);
        dev_free(ctx, ctx->scan_tmp, ctx->scan_tmp_bytes);
        dev_free(ctx, ctx->small, 256);
        cudaStreamSynchronize(ctx->stream);
        cudaStreamSynchronize(ctx->own_stream);
        cudaStreamDestroy(ctx->own_stream);
        cudaEventDestroy(ctx->ev0);
        cudaEventDestroy(ctx->ev1);
        cudaEventDestroy(ctx->evt);
        cudaFreeHost(ctx->h_counters);
        cudaFreeHost(ctx->h_status);
        cudaMemPoolDestroy(ctx->pool);
    }
    delete ctx;
    return GSOFA_OK;
}

const char* gsofa_last_error(const gsofa_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

int gsofa_set_stream(gsofa_ctx* ctx, void* s) {
    if (!ctx) return GSOFA_ERR_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    // drain work queued on the previous stream before switching
    cudaStreamSynchronize(ctx->stream);
    ctx->stream = s ? reinterpret_cast<cudaStream_t>(s) : ctx->own_stream;
    return GSOFA_OK;
}

int gsofa_memory_used(const gsofa_ctx* ctx, size_t* bytes) {
    if (!ctx || !bytes) return GSOFA_ERR_ARG;
    *bytes = ctx->used;
    return GSOFA_OK;
}

int gsofa_load_csr(gsofa_ctx* ctx, int32_t n, int64_t nnz, const int32_t* row_begin,
                   const int32_t* row_end, const int32_t* col, gsofa_matrix** out) {
    if (!ctx || !out) return GSOFA_ERR_ARG;
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    unsigned long long* wc = nullptr;
    int32_t* dstatus = work_counter_status(ctx, &wc);
    CK(cudaMemsetAsync(ctx->small, 0, 128, ctx->stream));
    gsofa_matrix* m = nullptr;
    int rc = ingest_csr(ctx, ctx->stream, dstatus, n, nnz, row_begin, row_end, col, &m);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(ctx->h_status, dstatus, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    rc = e != cudaSuccess ? cuda_fail(ctx, e, "load") : check_status(ctx);
    if (rc) {
        dev_free(ctx, m->rowptr, m->bytes);
        delete m;
        return rc;
    }
    *out = m;
    return GSOFA_OK;
}

int gsofa_load_csr_files(gsofa_ctx* ctx, const char* beg_file, const char* end_file,
                         const char* csr_file, gsofa_matrix** out) {
    if (!ctx || !out || !beg_file || !end_file || !csr_file) return GSOFA_ERR_ARG;
    int32_t n = 0;
    int64_t E = 0;
    std::vector<int32_t> beg, end, col;
    int rc = parse_dat_files(ctx, beg_file, end_file, csr_file, &n, &E, &beg, &end, &col);
    if (rc) return rc;
    return gsofa_load_csr(ctx, n, E, beg.data(), end.data(), col.data(), out);
}

int gsofa_matrix_info(const gsofa_matrix* m, int32_t* n, int64_t* nnz) {
    if (!m) return GSOFA_ERR_ARG;
    if (n) *n = m->n;
    if (nnz) *nnz = m->nnz;
    return GSOFA_OK;
}

int gsofa_matrix_destroy(gsofa_matrix* m) {
    if (!m) return GSOFA_ERR_ARG;
    {
        std::lock_guard<std::recursive_mutex> g(m->ctx->mu);
        dev_free(m->ctx, m->rowptr, m->bytes);
    }
    delete m;
    return GSOFA_OK;
}

int gsofa_factor_batch(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                       const gsofa_opts* opts, gsofa_result** results) {
    if (!ctx || count < 0 || (count > 0 && (!mats || !results))) return GSOFA_ERR_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    gsofa_opts o;
    if (opts) o = *opts; else gsofa_opts_default(&o);
    int rc = validate_opts(ctx, &o);
    if (rc) return rc;
    for (int32_t i = 0; i < count; i++) {
        results[i] = nullptr;
        if (!mats[i] || mats[i]->ctx != ctx)
            return set_err(ctx, GSOFA_ERR_ARG, "matrix %d is null or from another context", i);
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    std::vector<gsofa_result*> res((size_t)count, nullptr);
    for (int32_t i = 0; i < count; i++) {
        rc = result_alloc(ctx, mats[i]->n, o.flags, o.max_supernode_size, &res[i]);
        if (rc) {
            for (auto* r : res) result_free(r);
            return rc;
        }
    }
    rc = run_factor(ctx, mats, count, &o, res.data());
    if (rc) {
        for (auto* r : res) result_free(r);
        return rc;
    }
    for (int32_t i = 0; i < count; i++) results[i] = res[i];
    return GSOFA_OK;
}

// Times candidate launch shapes on an evenly spread sample of the matrix's
// work items (large matrices) or on the whole matrix (small ones) and keeps
// the fastest.  The candidates differ only in speed: every setting gives the
// same results.  Choices are cached per size class in the context.
// Coordinate descent over the launch shape (CTA size, closure ring, chunk,
// warp-walked row threshold), each candidate timed on the device as one
// persistent launch over all `count` matrices.  Writes the best into *opts.
static int autotune_impl(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                         gsofa_opts* opts) {
    int rc = GSOFA_OK;
    int32_t nmax = 0;
    long long total_sources = 0;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    for (int32_t i = 0; i < count; i++) {
        nmax = std::max(nmax, mats[i]->n);
        total_sources += chunk_weight(ctx, mats[i]);
    }
    gsofa_opts base = *opts;
    base.flags &= ~(uint32_t)(GSOFA_SUPERNODES | GSOFA_PATTERN | GSOFA_L_ROW_STATS);
    // reference timing with the defaults picks the sampling rate
    std::vector<gsofa_result*> rr((size_t)count, nullptr);
    auto free_all = [&]() {
        for (gsofa_result* x : rr) result_free(x);
    };
    for (int32_t i = 0; i < count; i++) {
        rc = result_alloc(ctx, mats[i]->n, base.flags, base.max_supernode_size, &rr[(size_t)i]);
        if (rc) { free_all(); return rc; }
    }
    rc = run_factor(ctx, mats, count, &base, rr.data());
    if (rc) { free_all(); return rc; }
    const double full_ms = rr[0]->counts.ms_traverse;  // the launch's time
    // Full runs while they are short; above 2 s time every stride-th work
    // item, keeping at least 16 items per CTA so the tail does not dominate.
    long long stride = 1;
    if (full_ms > 2000.0) {
        LaunchCfg c0;
        if (plan_launch(ctx, nmax, &base, &c0) == GSOFA_OK) {
            const long long items = total_sources / 16 + 2ll * count;
            stride = (long long)(full_ms / 1000.0);
            while (stride > 1 && items / stride < 16ll * c0.grid) stride--;
        }
    }
    auto time_opts = [&](const gsofa_opts& p, double* ms) -> int {
        LaunchCfg c;
        if (plan_launch(ctx, nmax, &p, &c) != GSOFA_OK) {
            ctx->err.clear();
            *ms = 1e300;
            return GSOFA_OK;
        }
        int e = run_factor(ctx, mats, count, &p, rr.data(), stride);
        *ms = e ? 1e300 : rr[0]->counts.ms_traverse;
        if (e) {
            const std::string prev = ctx->err;
            set_err(ctx, e, "%s; timing threads %d, ring %d, chunk %d, heavy row %d", prev.c_str(),
                    c.block, p.cached_closures, p.chunk_sources, p.heavy_row);
        }
        return e;
    };
    // coordinate descent from the defaults: CTA size, closure ring, chunk,
    // warp-walked row threshold
    gsofa_opts best = base;
    double best_ms = 0;
    rc = time_opts(best, &best_ms);
    if (rc) { free_all(); return rc; }
    {
        LaunchCfg c0;
        if (plan_launch(ctx, nmax, &base, &c0) == GSOFA_OK) best.threads_per_source = c0.block;
        ctx->err.clear();
    }
    const int tps_c[] = {128, 256, 512, 1024};
    for (int tps : tps_c) {
        if (tps == best.threads_per_source) continue;
        gsofa_opts p = best;
        p.threads_per_source = tps;
        double ms;
        if ((rc = time_opts(p, &ms))) { free_all(); return rc; }
        if (ms < best_ms) { best_ms = ms; best = p; }
    }
    const int ring_c[] = {1, 8, 32, 64};
    const int ring_now = best.cached_closures > 0 ? best.cached_closures : kDefaultRing;
    best.cached_closures = ring_now;
    for (int ring : ring_c) {
        if (ring == ring_now) continue;
        gsofa_opts p = best;
        p.cached_closures = ring;
        double ms;
        if ((rc = time_opts(p, &ms))) { free_all(); return rc; }
        if (ms < best_ms) { best_ms = ms; best = p; }
    }
    {
        LaunchCfg c;
        long long auto_chunk = 64;
        if (plan_launch(ctx, nmax, &best, &c) == GSOFA_OK) auto_chunk = default_chunk(total_sources, c.grid);
        ctx->err.clear();
        if (best.chunk_sources <= 0) best.chunk_sources = (int32_t)auto_chunk;
        const long long cands[] = {auto_chunk / 8, auto_chunk / 4, auto_chunk / 2, auto_chunk * 2};
        for (long long ch : cands) {
            if (ch < 16 || ch > 1024 || ch == best.chunk_sources) continue;
            gsofa_opts p = best;
            p.chunk_sources = (int32_t)ch;
            double ms;
            if ((rc = time_opts(p, &ms))) { free_all(); return rc; }
            if (ms < best_ms) { best_ms = ms; best = p; }
        }
    }
    // rows longer than this are walked by a whole warp
    const int heavy_now = best.heavy_row > 0 ? best.heavy_row : kDefaultHeavyRow;
    best.heavy_row = heavy_now;
    for (int hr : {32, 64}) {
        if (hr == heavy_now) continue;
        gsofa_opts p = best;
        p.heavy_row = hr;
        double ms;
        if ((rc = time_opts(p, &ms))) { free_all(); return rc; }
        if (ms < best_ms) { best_ms = ms; best = p; }
    }
    (void)best_ms;
    free_all();
    opts->threads_per_source = best.threads_per_source;
    opts->chunk_sources = best.chunk_sources;
    opts->cached_closures = best.cached_closures;
    opts->heavy_row = best.heavy_row;
    return GSOFA_OK;
}

int gsofa_autotune(gsofa_ctx* ctx, const gsofa_matrix* mat, gsofa_opts* opts) {
    if (!ctx || !mat || !opts || mat->ctx != ctx) return GSOFA_ERR_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    int rc = validate_opts(ctx, opts);
    if (rc) return rc;
    if (mat->n <= 0) return GSOFA_OK;
    int lg = 0;
    while ((1ll << (lg + 1)) <= (long long)mat->n) lg++;
    const int deg = (int)((mat->nnz + mat->n / 2) / mat->n);
    // locality: matrices of one size but different orderings want different
    // shapes (a renumbered grid is not its banded original)
    unsigned long long* dsum = reinterpret_cast<unsigned long long*>(
        reinterpret_cast<char*>(ctx->small) + 96);
    unsigned long long hsum = 0;
    cudaError_t ce = cudaMemsetAsync(dsum, 0, 8, ctx->stream);
    if (ce == cudaSuccess) ce = launch_index_distance(mat->n, mat->rowptr, mat->col, dsum, ctx->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&hsum, dsum, 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "autotune locality");
    const double rel = mat->nnz > 0 ? (double)hsum / (double)mat->nnz / (double)mat->n : 0.0;
    const int loc = rel > 1e-9 ? std::max(-60, (int)std::floor(2.0 * std::log2(rel))) : -61;
    const std::tuple<int, int, int> key(lg, deg, loc);
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end()) {
        opts->threads_per_source = it->second.threads_per_source;
        opts->chunk_sources = it->second.chunk_sources;
        opts->cached_closures = it->second.cached_closures;
        opts->heavy_row = it->second.heavy_row;
        return GSOFA_OK;
    }
    const gsofa_matrix* const mats[1] = {mat};
    rc = autotune_impl(ctx, mats, 1, opts);
    if (rc == GSOFA_OK) ctx->tuned[key] = *opts;
    return rc;
}

int gsofa_autotune_batch(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                         gsofa_opts* opts) {
    if (!ctx || !opts || count < 0 || (count > 0 && !mats)) return GSOFA_ERR_ARG;
    for (int32_t i = 0; i < count; i++)
        if (!mats[i] || mats[i]->ctx != ctx) return GSOFA_ERR_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    int rc = validate_opts(ctx, opts);
    if (rc) return rc;
    bool any = false;
    for (int32_t i = 0; i < count; i++) any |= mats[i]->n > 0;
    if (!any) return GSOFA_OK;
    return autotune_impl(ctx, mats, count, opts);
}

int gsofa_factor_symbolic(gsofa_ctx* ctx, const gsofa_matrix* mat, const gsofa_opts* opts,
                          gsofa_result** out) {
    if (!out) return GSOFA_ERR_ARG;
    return gsofa_factor_batch(ctx, &mat, 1, opts, out);
}

static void batch_free(gsofa_batch* b) {
    if (!b) return;
    gsofa_ctx* ctx = b->ctx;
    if (ctx) {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        for (gsofa_result* r : b->res) {
            if (!r) continue;
            r->batch_owned = false;
            result_free(r);
        }
        dev_free(ctx, b->ws, b->ws_bytes);
        cudaStreamSynchronize(ctx->stream);
        if (b->h_counters) cudaFreeHost(b->h_counters);
        if (b->h_status) cudaFreeHost(b->h_status);
        if (b->e0) cudaEventDestroy(b->e0);
        if (b->et) cudaEventDestroy(b->et);
        if (b->e1) cudaEventDestroy(b->e1);
    }
    delete b;
}

int gsofa_batch_create(gsofa_ctx* ctx, const gsofa_matrix* const* mats, int32_t count,
                       const gsofa_opts* opts, gsofa_batch** out) {
    if (!ctx || !out || count <= 0 || !mats) return GSOFA_ERR_ARG;
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    gsofa_opts o;
    if (opts) o = *opts; else gsofa_opts_default(&o);
    int rc = validate_opts(ctx, &o);
    if (rc) return rc;
    if (o.flags & GSOFA_PATTERN)
        return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "a captured batch cannot materialise patterns");
    int32_t nmax = 1;
    long long total_sources = 0;
    for (int32_t i = 0; i < count; i++) {
        if (!mats[i] || mats[i]->ctx != ctx)
            return set_err(ctx, GSOFA_ERR_ARG, "matrix %d is null or from another context", i);
        nmax = std::max(nmax, mats[i]->n);
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    for (int32_t i = 0; i < count; i++) total_sources += chunk_weight(ctx, mats[i]);
    gsofa_batch* b = new (std::nothrow) gsofa_batch();
    if (!b) return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "host allocation failed");
    b->ctx = ctx;
    b->count = count;
    b->opts = o;
    b->res.assign((size_t)count, nullptr);
    auto fail = [&](int code) {
        batch_free(b);
        return code;
    };
    for (int32_t i = 0; i < count; i++) {
        rc = result_alloc(ctx, mats[i]->n, o.flags, o.max_supernode_size, &b->res[(size_t)i]);
        if (rc) return fail(rc);
        b->res[(size_t)i]->batch_owned = true;
    }
    LaunchCfg cfg;
    rc = plan_launch(ctx, nmax, &o, &cfg);
    if (rc) return fail(rc);
    const long long chunk =
        o.chunk_sources > 0 ? o.chunk_sources : default_chunk(total_sources, cfg.grid);
    const bool merge = !(o.flags & GSOFA_NO_MERGE);
    int ring = o.cached_closures > 0 ? o.cached_closures : kDefaultRing;
    if (ring > kMaxRing) ring = kMaxRing;
    while (ring & (ring - 1)) ring &= ring - 1;
    // descriptors, segment prefix, counters, workspace: one private block
    std::vector<MatDesc> descs((size_t)count);
    std::vector<long long> seg((size_t)count + 1, 0);
    long long base = 0;
    const std::vector<int32_t> order = batch_order(mats, count);  // largest first
    for (int32_t k = 0; k < count; k++) {
        const int32_t i = order[(size_t)k];
        descs[(size_t)k] = make_desc(mats[i], b->res[(size_t)i], base);
        base += 2ll * ((mats[i]->n + chunk - 1) / chunk);
        seg[(size_t)k + 1] = seg[(size_t)k] + supernode_segment_count(mats[i]->n, o.max_supernode_size);
    }
    b->items = base;
    const size_t sz_small = 256;
    const size_t sz_desc = align256(sizeof(MatDesc) * (size_t)count);
    const size_t sz_seg = align256(sizeof(long long) * ((size_t)count + 1));
    const size_t sz_cnt = align256(8ull * CNT_SLOTS * (size_t)count);
    const size_t sz_q = align256((size_t)cfg.grid * (size_t)nmax * 4);
    const size_t sz_ring = merge ? align256((size_t)cfg.grid * (size_t)ring * (size_t)cfg.words * 4) : 0;
    const size_t sz_gbm = cfg.smem_bitmap ? 0 : align256((size_t)cfg.grid * (size_t)cfg.words * 4);
    b->ws_bytes = sz_small + sz_desc + sz_seg + sz_cnt + sz_q + sz_ring + sz_gbm;
    rc = dev_alloc(ctx, b->ws_bytes, &b->ws);
    if (rc) return fail(rc);
    char* p = reinterpret_cast<char*>(b->ws);
    unsigned long long* wc = reinterpret_cast<unsigned long long*>(p);
    int32_t* dstatus = reinterpret_cast<int32_t*>(p + 64);
    p += sz_small;
    MatDesc* ddesc = reinterpret_cast<MatDesc*>(p);
    p += sz_desc;
    long long* dseg = reinterpret_cast<long long*>(p);
    p += sz_seg;
    unsigned long long* dcnt = reinterpret_cast<unsigned long long*>(p);
    p += sz_cnt;
    int32_t* dq = reinterpret_cast<int32_t*>(p);
    p += sz_q;
    uint32_t* dring = merge ? reinterpret_cast<uint32_t*>(p) : nullptr;
    p += sz_ring;
    uint32_t* dgbm = cfg.smem_bitmap ? nullptr : reinterpret_cast<uint32_t*>(p);
    for (int32_t k = 0; k < count; k++)  // matrix i's counters at slot i, whatever its launch order
        descs[(size_t)k].counters = dcnt + (size_t)order[(size_t)k] * CNT_SLOTS;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(ddesc, descs.data(), sizeof(MatDesc) * (size_t)count,
                             cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dseg, seg.data(), sizeof(long long) * ((size_t)count + 1),
                             cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&b->h_counters, 8ull * CNT_SLOTS * (size_t)count)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&b->h_status, 64)) != cudaSuccess ||
        (e = cudaEventCreate(&b->e0)) != cudaSuccess || (e = cudaEventCreate(&b->et)) != cudaSuccess ||
        (e = cudaEventCreate(&b->e1)) != cudaSuccess)
        return fail(cuda_fail(ctx, e, "batch set-up"));

    TraverseLaunch L{};
    L.mats = ddesc;
    L.nmats = count;
    L.total_items = b->items;
    L.work_counter = wc;
    L.queue = dq;
    L.queue_stride = nmax;
    L.gbitmap = dgbm;
    L.bitmap_words = cfg.words;
    L.status = dstatus;
    L.pattern_pass = 0;
    L.bu_alpha = o.bu_alpha > 0 ? o.bu_alpha : (o.bu_alpha < 0 ? 0 : kDefaultBuAlpha);
    L.bu_beta = o.bu_beta > 0 ? o.bu_beta : kDefaultBuBeta;
    L.bu_min_src = o.bu_min_source > 0 ? o.bu_min_source : kBuMinSource;
    L.heavy_len = o.heavy_row > 0 ? ((o.heavy_row + 3) & ~3) : kDefaultHeavyRow;
    L.gprev = dring;
    L.chunk = (int)chunk;
    L.merge = merge ? 1 : 0;
    L.chain = merge && !(o.flags & GSOFA_NO_CHAIN) ? 1 : 0;
    L.chain_wait_ns = chain_wait_ns(o);
    L.ring = ring;
    L.sample_stride = 1;

    // capture: reset -> traversal -> supernodes -> read-back
    if ((e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed)) != cudaSuccess)
        return fail(cuda_fail(ctx, e, "cudaStreamBeginCapture"));
    e = cudaMemsetAsync(b->ws, 0, 128, ctx->stream);
    if (e == cudaSuccess) e = launch_batch_reset(ddesc, count, ctx->stream);
    if (e == cudaSuccess && b->items > 0)
        e = launch_traverse(L, cfg.block, cfg.grid, cfg.smem_bitmap, cfg.smem, ctx->stream);
    if (e == cudaSuccess && (o.flags & GSOFA_SUPERNODES))
        e = launch_supernodes_batch(ddesc, count, o.max_supernode_size, dseg, seg[(size_t)count],
                                    ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_counters, dcnt, 8ull * CNT_SLOTS * (size_t)count,
                            cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_status, dstatus, 4, cudaMemcpyDeviceToHost, ctx->stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(cuda_fail(ctx, e != cudaSuccess ? e : e2, "batch capture"));
    }
    b->graph = graph;
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
        return fail(cuda_fail(ctx, e, "cudaGraphInstantiate"));
    *out = b;
    return GSOFA_OK;
}

int gsofa_batch_run(gsofa_batch* b) {
    if (!b) return GSOFA_ERR_ARG;
    gsofa_ctx* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    // events around the graph launch: the whole batch's device time
    CK(cudaEventRecord(b->e0, ctx->stream));
    CK(cudaGraphLaunch(b->exec, ctx->stream));
    CK(cudaEventRecord(b->e1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *ctx->h_status = *b->h_status;
    int rc = check_status(ctx);
    if (rc) return rc;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, b->e0, b->e1));
    for (int32_t i = 0; i < b->count; i++) {
        gsofa_result* r = b->res[(size_t)i];
        const unsigned long long* c = b->h_counters + (size_t)i * CNT_SLOTS;
        gsofa_counts& k = r->counts;
        k.n = r->n;
        k.fill_count = c[CNT_FILLS];
        k.nnz_l = c[CNT_NNZ_L];
        k.nnz_u = c[CNT_NNZ_U];
        k.nnz_lu = c[CNT_NNZ_L] + c[CNT_NNZ_U] + (uint64_t)r->n;
        k.n_supernodes = (b->opts.flags & GSOFA_SUPERNODES) ? (int64_t)c[CNT_NSUP] + 1 : -1;
        k.edges_alg = c[CNT_EDGES_ALG];
        k.vertices_alg = c[CNT_VERTS_ALG];
        k.edges_traversed = c[CNT_EDGES_TRAV];
        k.sources_chained = c[CNT_CHAINED];
        k.ms_device = (double)ms;  // the whole batch (one graph launch)
        k.ms_traverse = (double)ms;
    }
    return GSOFA_OK;
}

int gsofa_batch_result(const gsofa_batch* b, int32_t i, gsofa_result** res) {
    if (!b || !res || i < 0 || i >= b->count) return GSOFA_ERR_ARG;
    *res = b->res[(size_t)i];
    return GSOFA_OK;
}

int gsofa_batch_destroy(gsofa_batch* b) {
    if (!b) return GSOFA_ERR_ARG;
    batch_free(b);
    return GSOFA_OK;
}

int gsofa_result_counts(const gsofa_result* r, gsofa_counts* out) {
    if (!r || !out) return GSOFA_ERR_ARG;
    *out = r->counts;
    return GSOFA_OK;
}

static int fetch(const gsofa_result* r, void* dst, const void* src, size_t bytes) {
    if (!dst) return GSOFA_OK;
    if (!src) return set_err(r->ctx, GSOFA_ERR_ARG, "requested array was not computed (option off)");
    std::lock_guard<std::recursive_mutex> g(r->ctx->mu);
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, r->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(r->ctx, e, "result fetch");
    return GSOFA_OK;
}

int gsofa_result_row_counts(const gsofa_result* r, int32_t* nnz_u_row, int32_t* nz_row_u,
                            int32_t* nnz_l_col, int32_t* nnz_l_row) {
    if (!r) return GSOFA_ERR_ARG;
    const size_t b = 4 * (size_t)r->n;
    int rc;
    if ((rc = fetch(r, nnz_u_row, r->nnz_u, b))) return rc;
    if ((rc = fetch(r, nz_row_u, r->nz_row_u, b))) return rc;
    if ((rc = fetch(r, nnz_l_col, r->nnz_lc, b))) return rc;
    return fetch(r, nnz_l_row, r->nnz_lr, b);
}

int gsofa_result_digests(const gsofa_result* r, uint64_t* du, uint64_t* dlc, uint64_t* dlr) {
    if (!r) return GSOFA_ERR_ARG;
    const size_t b = 8 * (size_t)r->n;
    int rc;
    if ((rc = fetch(r, du, r->dig_u, b))) return rc;
    if ((rc = fetch(r, dlc, r->dig_lc, b))) return rc;
    return fetch(r, dlr, r->dig_lr, b);
}

int gsofa_result_lmask(const gsofa_result* r, uint32_t* mask4n) {
    if (!r) return GSOFA_ERR_ARG;
    return fetch(r, mask4n, r->lmask, 16 * (size_t)r->n);
}

int gsofa_result_supernodes(const gsofa_result* r, int8_t* flags, int32_t* boundaries, int64_t cap,
                            int64_t* count) {
    if (!r) return GSOFA_ERR_ARG;
    if (!(r->flags & GSOFA_SUPERNODES))
        return set_err(r->ctx, GSOFA_ERR_ARG, "supernode detection was not requested");
    std::vector<int8_t> f((size_t)r->n);
    int rc = fetch(r, f.data(), r->sflags, (size_t)r->n);
    if (rc) return rc;
    if (flags) memcpy(flags, f.data(), (size_t)r->n);
    int64_t k = 0;
    for (int32_t v = 0; v < r->n; v++) {
        if (f[v]) {
            if (boundaries && k < cap) boundaries[k] = v;
            k++;
        }
    }
    if (count) *count = k;
    return GSOFA_OK;
}

static int fetch_pattern(const gsofa_result* r, const int64_t* dptr, const int32_t* dids,
                         int64_t* ptr, int32_t* ids, int64_t cap) {
    if (!(r->flags & GSOFA_PATTERN) || !dptr)
        return set_err(r->ctx, GSOFA_ERR_ARG, "pattern was not requested (GSOFA_PATTERN)");
    std::vector<int64_t> p((size_t)r->n + 1);
    int rc = fetch(r, p.data(), dptr, 8 * ((size_t)r->n + 1));
    if (rc) return rc;
    if (ptr) memcpy(ptr, p.data(), 8 * ((size_t)r->n + 1));
    if (ids) {
        if (cap < p[(size_t)r->n])
            return set_err(r->ctx, GSOFA_ERR_ARG, "id buffer holds %lld, needs %lld", (long long)cap,
                           (long long)p[(size_t)r->n]);
        if (p[(size_t)r->n] > 0) rc = fetch(r, ids, dids, 4 * (size_t)p[(size_t)r->n]);
    }
    return rc;
}

int gsofa_result_pattern_u(const gsofa_result* r, int64_t* ptr, int32_t* cols, int64_t cap) {
    if (!r) return GSOFA_ERR_ARG;
    return fetch_pattern(r, r->uptr, r->ucols, ptr, cols, cap);
}

int gsofa_result_pattern_l(const gsofa_result* r, int64_t* ptr, int32_t* rows, int64_t cap) {
    if (!r) return GSOFA_ERR_ARG;
    return fetch_pattern(r, r->lptr, r->lrows, ptr, rows, cap);
}

int gsofa_result_destroy(gsofa_result* r) {
    if (!r) return GSOFA_ERR_ARG;
    if (r->batch_owned) return set_err(r->ctx, GSOFA_ERR_ARG, "result belongs to a batch");
    result_free(r);
    return GSOFA_OK;
}

// The reference's two command lines (SOA argc == 11, :2532-2545; SPO argc == 6,
// symbfact.cuh:1557-1571), folded onto one device.
int gsofa_symbfact_min_id(int argc, char** argv, int rank, uint64_t* fill_count, double* time_ms,
                          int32_t* n_supernodes, uint64_t* teps_edges) {
    if (!argv || (argc != 11 && argc != 6)) return GSOFA_ERR_ARG;
    gsofa_opts o;
    gsofa_opts_default(&o);
    size_t budget = 0;
    if (argc == 11) {
        int mss = atoi(argv[5]);
        if (mss <= 0) return GSOFA_ERR_ARG;
        o.max_supernode_size = mss;
    } else {
        double gb = atof(argv[5]);
        if (gb < 0) return GSOFA_ERR_ARG;
        // the reference's pool holds its 6 work arrays; here the budget bounds
        // everything the context allocates (matrix, workspace, results)
        budget = gb > 0 ? (size_t)(gb * 1024.0 * 1024.0 * 1024.0) : 0;
        o.flags &= ~(uint32_t)GSOFA_SUPERNODES;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return GSOFA_ERR_CUDA;
    gsofa_ctx* ctx = nullptr;
    int rc = gsofa_create(rank % ndev, budget, &ctx);
    if (rc) return rc;
    gsofa_matrix* m = nullptr;
    rc = gsofa_load_csr_files(ctx, argv[1], argv[2], argv[3], &m);
    if (rc) {
        fprintf(stderr, "gsofa: %s\n", gsofa_last_error(ctx));
        gsofa_destroy(ctx);
        return rc;
    }
    gsofa_result* r = nullptr;
    rc = gsofa_factor_symbolic(ctx, m, &o, &r);
    if (rc) {
        fprintf(stderr, "gsofa: %s\n", gsofa_last_error(ctx));
        gsofa_matrix_destroy(m);
        gsofa_destroy(ctx);
        return rc;
    }
    gsofa_counts c;
    gsofa_result_counts(r, &c);
    if (fill_count) *fill_count = c.fill_count;
    if (time_ms) *time_ms = c.ms_device;
    if (n_supernodes) *n_supernodes = (int32_t)c.n_supernodes;
    if (teps_edges) *teps_edges = c.edges_alg;
    gsofa_result_destroy(r);
    gsofa_matrix_destroy(m);
    gsofa_destroy(ctx);
    return GSOFA_OK;
}

}  // extern "C"
