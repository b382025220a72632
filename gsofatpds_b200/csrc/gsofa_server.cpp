// gsofa_server.cpp -- the serving request loop (continuous batching).
//
// One host thread per server drives:
//   * a persistent traversal kernel (traverse_kernel, serving mode) on the
//     kernel stream.  Its CTAs claim work items of every published request;
//     it stays on the device while published work is waiting and ends by
//     itself when its CTAs have found nothing to claim for a short while;
//   * a side stream for everything else: the upload and padded-CSR build of
//     each admitted request, its descriptor, the copy that publishes it (its
//     claim word), and, once the kernel reports the request finished, its
//     supernode detection and the read-back of its totals;
//   * a control stream for the small table the kernel polls (the list of live
//     requests the CTAs pick from, the "exit when idle" and "take no more
//     items" controls): the host keeps the master copy in pinned memory and
//     pushes it whole, synchronously, after each change;
//   * mapped host memory for the kernel's per-slot "request done" flags, its
//     only writes to host memory.  Nothing the kernel polls lives in host
//     memory: hundreds of idle CTAs polling across PCIe would compete with
//     the uploads of the requests they wait for.
//
// Admission is first come, first served: the request at the head of the
// queue is admitted when a slot is free and its footprint (padded CSR of A
// and A^T, staging, result arrays) fits the budget beside the workspace and
// the requests in flight.  A request never waits for the kernel: it joins the
// running launch, and a CTA takes its next item from the live request with
// the fewest unclaimed items, so a small request that arrives behind a large
// one is not queued behind the large one's items.  The kernel leaves four SMs' worth of CTAs free,
// and the side stream has the higher priority, so uploads and builds run
// beside it.
//
// Nothing here waits on the device without a bound: a CTA's idle polling
// ends after kIdleNs, and the host waits only for streams whose work is
// already queued.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gsofa_host.h"

using namespace gsofa;
using namespace gsofa::host;

namespace {

enum ReqState { R_QUEUED, R_RUNNING, R_FINISHING, R_DONE, R_FAILED };

struct Request {
    uint64_t ticket = 0;
    int32_t n = 0;
    int64_t nnz = 0;
    const int32_t* beg = nullptr;
    const int32_t* end = nullptr;
    const int32_t* col = nullptr;
    int state = R_QUEUED;
    int status = GSOFA_ERR_BUSY;
    int slot = -1;
    long long item_base = 0;
    long long n_items = 0;
    unsigned long long seq = 0;
    size_t footprint = 0;
    gsofa_matrix* mat = nullptr;
    gsofa_result* res = nullptr;
    bool handed_out = false;
    double t_submit = 0, t_admit = 0, t_publish = 0, t_done = 0;
    bool published = false;  // the claim word copy has executed
};

constexpr int kSlots = 256;
constexpr int kKernelStreams = 4;  // serving launches that may run at once
constexpr int kReserveSms = 4;
constexpr long long kMaxIdlePolls = 1000000;  // a cap far above idle_ns worth of polls
constexpr long long kIdleNs = 300000;         // a CTA with nothing to claim for 0.3 ms exits
constexpr double kTopUpCheckMs = 0.5;         // how often a partial launch is topped up
constexpr double kAdmitSliceMs = 1.0;         // admissions per loop pass stop after this long
constexpr size_t kDefaultBudget = 40ull << 30;
constexpr double kShutdownGraceMs = 120000.0;  // destroy waits this long for queued work

}  // namespace

struct gsofa_server {
    gsofa_ctx* ctx = nullptr;
    gsofa_opts opts{};
    int32_t max_n = 0;
    size_t budget = 0;
    int block = 256, grid = 0, occ = 0;
    size_t smem = 0;
    long long smem_words = 0, words = 0;
    int ring = 32;
    bool merge = true;
    cudaStream_t ks[kKernelStreams] = {};  // serving launches (low priority)
    cudaEvent_t kdone[kKernelStreams] = {};
    bool krun[kKernelStreams] = {};
    cudaStream_t as = nullptr, cs = nullptr, fs = nullptr;
    std::vector<cudaEvent_t> slot_ev;  // per slot: read-back done
    std::vector<cudaEvent_t> pub_ev;   // per slot: claim word written
    // device workspace (one block)
    void* ws = nullptr;
    size_t ws_bytes = 0;
    int32_t* queue = nullptr;
    uint32_t* rings = nullptr;
    uint32_t* gbm = nullptr;
    MatDesc* d_slots = nullptr;
    unsigned long long* d_claim = nullptr;
    unsigned long long* d_items_done = nullptr;
    int32_t* d_slot_status = nullptr;
    unsigned int* d_rr = nullptr;
    unsigned int* d_cta_slots = nullptr;
    int* d_alive = nullptr;
    int* h_alive = nullptr;  // pinned read-back of *d_alive
    double alive_checked = -1.0;
    unsigned long long* d_work = nullptr;
    int32_t* d_status = nullptr;
    // control table: int32 ctrl[4] ([0] exit when idle, [1] take no more
    // items, [2] list entries), then u64 list[kSlots] = (slot << 32) | request
    // number.  Master copy in pinned host memory, pushed whole.
    void* d_ctl = nullptr;
    void* h_ctl = nullptr;
    // mapped host memory
    unsigned long long* h_done = nullptr;
    unsigned long long* d_done = nullptr;
    // pinned staging, per slot
    MatDesc* h_desc = nullptr;
    unsigned long long* h_claim = nullptr;
    unsigned long long* h_cnt = nullptr;
    int32_t* h_sstat = nullptr;
    // uploads of the submitted (pageable) host arrays
    gsofa::host::PinnedStager stager;
    // host state (mu guards everything a caller thread touches)
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread th;
    bool shutdown = false;
    uint64_t next_ticket = 1;
    std::deque<std::shared_ptr<Request>> queued;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> tickets;
    std::vector<std::shared_ptr<Request>> slot_req;
    std::vector<int> free_slots;
    // loop-thread state
    unsigned long long seq = 0;
    int nlist = 0;
    bool kernel_running = false;
    bool launch_failed = false;
    int live = 0;
    // accounting
    size_t fixed = 0, in_use = 0, peak = 0;
    gsofa_server_stats st{};
    std::string err;
    std::chrono::steady_clock::time_point t0;
};

namespace {

double now_ms(const gsofa_server* s) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s->t0)
        .count();
}

void server_err(gsofa_server* s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> g(s->mu);
    s->err = buf;
}

size_t request_footprint(const gsofa_server* s, int32_t n, int64_t nnz) {
    size_t kept = 0, staging = 0;
    ingest_bytes(n, nnz, &kept, &staging);
    return kept + staging + result_bytes(n, s->opts.flags);
}

// Consecutive sources per work item: about four items per CTA for this
// order and grid (requests share the CTAs, so items stay shorter than the
// plain path's), capped so that chunk * n stays near 2^28 -- one item of a
// large request then holds its CTA for a bounded time, not for a large part
// of the request, and a request that arrives meanwhile finds CTAs soon.  The
// cap is no tighter because every item's first source starts cold.
int request_chunk(const gsofa_server* s, int32_t n) {
    if (s->opts.chunk_sources > 0) return s->opts.chunk_sources;
    long long cap = 512;
    while (cap > 16 && cap * (long long)std::max(n, 1) > (1ll << 28)) cap >>= 1;
    return (int)std::min<long long>(default_chunk(2ll * n, 4 * s->grid), cap);
}

// Marks a request finished (done or failed) and releases its slot and memory.
void finish(gsofa_server* s, const std::shared_ptr<Request>& r, int status) {
    gsofa_ctx* ctx = s->ctx;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        if (r->mat) {
            dev_free_on(ctx, r->mat->rowptr, r->mat->bytes, s->as);
            delete r->mat;
            r->mat = nullptr;
        }
        if (status != GSOFA_OK && r->res) {
            dev_free_on(ctx, r->res->arena, r->res->bytes, s->as);
            delete r->res;
            r->res = nullptr;
        }
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (r->slot >= 0) {
        s->slot_req[(size_t)r->slot].reset();
        s->free_slots.push_back(r->slot);
        r->slot = -1;
        s->live--;
    }
    s->in_use -= std::min(s->in_use, r->footprint);
    r->t_done = now_ms(s);
    r->status = status;
    r->state = status == GSOFA_OK ? R_DONE : R_FAILED;
    if (status == GSOFA_OK) s->st.completed++;
    else s->st.failed++;
    s->cv_done.notify_all();
}

constexpr size_t kCtlBytes = 16 + 8 * (size_t)kSlots;

int32_t* ctl_flags(gsofa_server* s) { return static_cast<int32_t*>(s->h_ctl); }
unsigned long long* ctl_list(gsofa_server* s) {
    return reinterpret_cast<unsigned long long*>(static_cast<char*>(s->h_ctl) + 16);
}

// Copies the control table to the device and waits for the copy (tens of
// microseconds), so the master copy can change again at once.
void push_control(gsofa_server* s) {
    cudaError_t e = cudaMemcpyAsync(s->d_ctl, s->h_ctl, kCtlBytes, cudaMemcpyHostToDevice, s->cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->cs);
    if (e != cudaSuccess) server_err(s, "control table update: %s", cudaGetErrorString(e));
}

// The live-request list.  A CTA that reads a stale, duplicated or half
// copied entry fails the claim word's request-number check.
void list_add(gsofa_server* s, int slot, unsigned long long seq) {
    ctl_list(s)[s->nlist++] = ((unsigned long long)slot << 32) | (seq & 0xffffffffull);
    ctl_flags(s)[2] = s->nlist;
    push_control(s);
}

void list_remove(gsofa_server* s, int slot) {
    unsigned long long* L = ctl_list(s);
    for (int i = 0; i < s->nlist; i++) {
        if ((int)(L[i] >> 32) != slot) continue;
        L[i] = L[s->nlist - 1];
        L[--s->nlist] = ~0ull;
        ctl_flags(s)[2] = s->nlist;
        push_control(s);
        return;
    }
}

void set_control(gsofa_server* s, int which, int32_t value) {
    ctl_flags(s)[which] = value;
    push_control(s);
}

// Admits the request at the head of the queue if it fits; queues its upload,
// build, table writes and publication on the side stream.
bool admit_one(gsofa_server* s) {
    std::shared_ptr<Request> r;
    int slot = -1;
    long long items = 0;
    int chunk = 0;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->queued.empty() || s->free_slots.empty()) return false;
        r = s->queued.front();
        if (s->in_use + r->footprint > s->budget) return false;
        chunk = request_chunk(s, r->n);
        items = 2ll * (((long long)r->n + chunk - 1) / chunk);
        s->queued.pop_front();
        slot = s->free_slots.back();
        s->free_slots.pop_back();
        s->slot_req[(size_t)slot] = r;
        s->live++;
        s->st.max_in_flight = std::max(s->st.max_in_flight, s->live);
        s->in_use += r->footprint;
        s->peak = std::max(s->peak, s->in_use);
        r->slot = slot;
        r->state = R_RUNNING;
        r->t_admit = now_ms(s);
    }
    gsofa_ctx* ctx = s->ctx;
    const uint32_t flags = s->opts.flags & (GSOFA_SUPERNODES | GSOFA_DIGESTS | GSOFA_L_ROW_STATS);
    int rc = GSOFA_OK;
    cudaError_t e = cudaMemsetAsync(s->d_slot_status + slot, 0, 4, s->as);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_items_done + slot, 0, 8, s->as);
    if (e != cudaSuccess) rc = GSOFA_ERR_CUDA;
    std::string why;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        if (rc == GSOFA_OK)
            rc = ingest_csr(ctx, s->as, s->d_slot_status + slot, r->n, r->nnz, r->beg, r->end,
                            r->col, &r->mat, &s->stager);
        if (rc == GSOFA_OK)
            rc = result_alloc_on(ctx, r->n, flags, s->opts.max_supernode_size, s->as, &r->res);
        if (rc != GSOFA_OK) why = ctx->err;
    }
    if (rc != GSOFA_OK) {
        server_err(s, "ticket %llu: %s", (unsigned long long)r->ticket, why.c_str());
        finish(s, r, rc);
        return true;
    }
    r->item_base = 0;
    r->n_items = items;
    r->seq = ++s->seq;
    MatDesc d = make_desc(r->mat, r->res, 0);
    d.n_items = items;
    d.seq = r->seq;
    d.chunk = chunk;
    d.slot = slot;
    s->h_desc[slot] = d;
    s->h_done[slot] = 0ull;
    s->h_claim[slot] = (r->seq & 0xffffffffull) << 32;
    e = cudaMemcpyAsync(s->d_slots + slot, s->h_desc + slot, sizeof(MatDesc),
                        cudaMemcpyHostToDevice, s->as);
    // the publication: the claim word (request number, 0 claimed), ordered
    // after the build and the descriptor
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d_claim + slot, s->h_claim + slot, 8, cudaMemcpyHostToDevice,
                            s->as);
    if (e == cudaSuccess) e = cudaEventRecord(s->pub_ev[(size_t)slot], s->as);
    if (e != cudaSuccess) {
        // not published: no CTA will claim these items
        server_err(s, "ticket %llu: %s", (unsigned long long)r->ticket, cudaGetErrorString(e));
        finish(s, r, GSOFA_ERR_CUDA);
        return true;
    }
    if (items > 0) list_add(s, slot, r->seq);
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->st.items_published += (uint64_t)items;
    }
    if (items == 0) {
        // nothing for the kernel: read back at once
        std::lock_guard<std::mutex> g(s->mu);
        r->published = true;
        r->t_publish = now_ms(s);
        s->h_done[slot] = r->seq;
    }
    return true;
}

bool launch_kernel(gsofa_server* s, int k, int grid) {
    TraverseLaunch L{};
    L.work_counter = s->d_work;
    L.queue = s->queue;
    L.queue_stride = std::max(s->max_n, 1);
    L.gbitmap = s->gbm;
    L.gprev = s->rings;
    L.chunk = 1;
    L.merge = s->merge ? 1 : 0;
    L.chain = s->merge && !(s->opts.flags & GSOFA_NO_CHAIN) ? 1 : 0;
    L.chain_wait_ns = chain_wait_ns(s->opts);
    L.ring = s->ring;
    L.sample_stride = 1;
    L.bitmap_words = s->words;
    L.status = s->d_status;
    L.pattern_pass = 0;
    const gsofa_opts& o = s->opts;
    L.bu_alpha = o.bu_alpha > 0 ? o.bu_alpha : 0;
    L.bu_beta = o.bu_beta > 0 ? o.bu_beta : kDefaultBuBeta;
    L.bu_min_src = o.bu_min_source > 0 ? o.bu_min_source : kBuMinSource;
    L.heavy_len = o.heavy_row > 0 ? ((o.heavy_row + 3) & ~3) : kDefaultHeavyRow;
    ServeLaunch& V = L.serve;
    V.claim = s->d_claim;
    V.list = reinterpret_cast<const unsigned long long*>(static_cast<char*>(s->d_ctl) + 16);
    V.ctrl = static_cast<const int32_t*>(s->d_ctl);
    V.rr = s->d_rr;
    V.nslots = kSlots;
    V.slots = s->d_slots;
    V.items_done = s->d_items_done;
    V.slot_status = s->d_slot_status;
    V.done_flags = s->d_done;
    V.smem_words = s->smem_words;
    V.max_idle_polls = kMaxIdlePolls;
    V.idle_ns = kIdleNs;
    V.cta_slots = s->d_cta_slots;
    V.n_cta_slots = s->grid;
    V.alive = s->d_alive;
    cudaError_t e = launch_serve(L, s->block, grid, s->smem, s->ks[k]);
    if (e == cudaSuccess) e = cudaEventRecord(s->kdone[k], s->ks[k]);
    if (e != cudaSuccess) {
        server_err(s, "serving kernel launch: %s", cudaGetErrorString(e));
        s->launch_failed = true;
        return false;
    }
    s->krun[k] = true;
    s->kernel_running = true;
    std::lock_guard<std::mutex> g(s->mu);
    s->st.kernel_launches++;
    return true;
}

// CTAs currently holding a workspace slot (a short synchronous read).
int alive_ctas(gsofa_server* s) {
    cudaError_t e = cudaMemcpyAsync(s->h_alive, s->d_alive, 4, cudaMemcpyDeviceToHost, s->cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->cs);
    return e == cudaSuccess ? *s->h_alive : s->grid;
}

// Keeps CTAs on the device while published work is waiting.  A CTA leaves
// once it has found nothing to claim for kIdleNs, which hands its SM back to
// the side stream (uploads and builds of later requests).  When work is
// waiting and fewer CTAs than workspace slots are alive -- none at all, or
// the rest left during a large request's last items -- another launch of
// the missing CTAs goes out on a free kernel stream (CTAs that find no free
// slot exit at once, so a stale count costs nothing).
bool manage_kernel(gsofa_server* s, bool claimable) {
    bool progress = false;
    bool any = false;
    int free_k = -1;
    for (int k = 0; k < kKernelStreams; k++) {
        if (s->krun[k] && cudaEventQuery(s->kdone[k]) == cudaSuccess) {
            s->krun[k] = false;
            progress = true;
        }
        if (s->krun[k]) any = true;
        else if (free_k < 0) free_k = k;
    }
    s->kernel_running = any;
    if (!claimable || free_k < 0) return progress;
    if (!any) return launch_kernel(s, free_k, s->grid) || progress;
    const double t = now_ms(s);
    if (t - s->alive_checked < kTopUpCheckMs) return progress;
    s->alive_checked = t;
    const int missing = s->grid - alive_ctas(s);
    if (missing >= std::max(8, s->grid / 16)) progress |= launch_kernel(s, free_k, missing);
    return progress;
}

// Requests whose last item is done: supernodes + read-back on the side
// stream; then, when that is complete, hand out the result.
bool reap(gsofa_server* s) {
    bool progress = false;
    std::vector<std::shared_ptr<Request>> act;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (auto& r : s->slot_req)
            if (r && (r->state == R_RUNNING || r->state == R_FINISHING)) act.push_back(r);
    }
    for (auto& r : act) {
        const int slot = r->slot;
        if (r->state == R_RUNNING) {
            const unsigned long long f =
                reinterpret_cast<volatile unsigned long long*>(s->h_done)[slot];
            if (f != r->seq) continue;
            if (r->n_items > 0) list_remove(s, slot);
            cudaError_t e = cudaSuccess;
            if ((s->opts.flags & GSOFA_SUPERNODES) && r->n > 0)
                e = launch_supernodes(r->n, s->opts.max_supernode_size, r->res->nz_row_u,
                                      r->res->lmask, r->res->sflags, r->res->counters, s->fs);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->h_cnt + (size_t)slot * CNT_SLOTS, r->res->counters,
                                    8 * CNT_SLOTS, cudaMemcpyDeviceToHost, s->fs);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->h_sstat + slot, s->d_slot_status + slot, 4,
                                    cudaMemcpyDeviceToHost, s->fs);
            if (e == cudaSuccess) e = cudaEventRecord(s->slot_ev[(size_t)slot], s->fs);
            if (e != cudaSuccess) {
                server_err(s, "ticket %llu: %s", (unsigned long long)r->ticket,
                           cudaGetErrorString(e));
                finish(s, r, GSOFA_ERR_CUDA);
                progress = true;
                continue;
            }
            std::lock_guard<std::mutex> g(s->mu);
            r->state = R_FINISHING;
            progress = true;
        } else {
            cudaError_t q = cudaEventQuery(s->slot_ev[(size_t)slot]);
            if (q == cudaErrorNotReady) continue;
            progress = true;
            if (q != cudaSuccess) {
                server_err(s, "ticket %llu: %s", (unsigned long long)r->ticket,
                           cudaGetErrorString(q));
                finish(s, r, GSOFA_ERR_CUDA);
                continue;
            }
            if (s->h_sstat[slot] != 0) {
                server_err(s, "ticket %llu: %s", (unsigned long long)r->ticket,
                           (s->h_sstat[slot] & DEV_ERR_COL_RANGE) ? "column id outside [0, n)"
                                                                  : "malformed CSR");
                finish(s, r, GSOFA_ERR_ARG);
                continue;
            }
            const unsigned long long* c = s->h_cnt + (size_t)slot * CNT_SLOTS;
            gsofa_counts& k = r->res->counts;
            k.n = r->n;
            k.fill_count = c[CNT_FILLS];
            k.nnz_l = c[CNT_NNZ_L];
            k.nnz_u = c[CNT_NNZ_U];
            k.nnz_lu = c[CNT_NNZ_L] + c[CNT_NNZ_U] + (uint64_t)r->n;
            k.n_supernodes = (s->opts.flags & GSOFA_SUPERNODES) ? (int64_t)c[CNT_NSUP] + 1 : -1;
            k.edges_alg = c[CNT_EDGES_ALG];
            k.vertices_alg = c[CNT_VERTS_ALG];
            k.edges_traversed = c[CNT_EDGES_TRAV];
            k.sources_chained = c[CNT_CHAINED];
            const double t = now_ms(s);
            k.ms_device = t - r->t_publish;  // host clock: publication to completion
            k.ms_traverse = k.ms_device;
            finish(s, r, GSOFA_OK);
        }
    }
    return progress;
}

// Fails every admitted request (the kernel is not running).
void fail_live(gsofa_server* s, int status) {
    std::vector<std::shared_ptr<Request>> act;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (auto& r : s->slot_req)
            if (r) act.push_back(r);
    }
    for (auto& r : act) {
        if (r->n_items > 0 && r->state == R_RUNNING) list_remove(s, r->slot);
        finish(s, r, status);
    }
}

void loop(gsofa_server* s) {
    cudaSetDevice(s->ctx->device);
    int idle_spins = 0;
    double shutdown_at = -1.0;
    for (;;) {
        bool progress = false;
        // admit in slices, so that publication, the kernel launch and the
        // read-back of finished requests are not held up behind the uploads
        // of a long queue
        const double t_adm = now_ms(s);
        while (admit_one(s)) {
            progress = true;
            if (now_ms(s) - t_adm > kAdmitSliceMs) break;
        }
        // requests whose claim word is on the device and whose items are not
        // all finished
        bool claimable = false;
        {
            std::lock_guard<std::mutex> g(s->mu);
            for (auto& r : s->slot_req) {
                if (!r || r->state != R_RUNNING || r->n_items == 0) continue;
                if (!r->published &&
                    cudaEventQuery(s->pub_ev[(size_t)r->slot]) == cudaSuccess) {
                    r->published = true;
                    r->t_publish = now_ms(s);
                }
                if (r->published) claimable = true;
            }
        }
        progress |= manage_kernel(s, claimable);
        if (s->launch_failed) {
            // no kernel can run: nothing admitted can finish
            fail_live(s, GSOFA_ERR_CUDA);
            s->launch_failed = false;
        }
        progress |= reap(s);
        std::unique_lock<std::mutex> lk(s->mu);
        const bool idle = s->queued.empty() && s->live == 0;
        if (s->shutdown && idle && !s->kernel_running) break;
        if (s->shutdown && idle && s->kernel_running && ctl_flags(s)[0] == 0) {
            lk.unlock();
            set_control(s, 0, 1);  // idle CTAs leave at once
            continue;
        }
        if (s->shutdown && shutdown_at < 0) shutdown_at = now_ms(s);
        if (s->shutdown && now_ms(s) - shutdown_at > kShutdownGraceMs) {
            // still busy long after destroy began: stop taking items, let the
            // CTAs finish the ones they hold, and fail whatever is left
            lk.unlock();
            set_control(s, 1, 1);
            for (int k = 0; k < kKernelStreams; k++)
                if (s->krun[k]) cudaEventSynchronize(s->kdone[k]);
            s->kernel_running = false;
            reap(s);
            fail_live(s, GSOFA_ERR_TIMEOUT);
            std::lock_guard<std::mutex> g(s->mu);
            for (auto& r : s->queued) {
                r->state = R_FAILED;
                r->status = GSOFA_ERR_TIMEOUT;
            }
            s->queued.clear();
            s->cv_done.notify_all();
            break;
        }
        if (progress) {
            idle_spins = 0;
            continue;
        }
        if (idle && !s->kernel_running) {
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
        } else {
            lk.unlock();
            // poll the device signals: spin briefly, then back off
            if (++idle_spins < 200) std::this_thread::yield();
            else std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

void release(gsofa_server* s) {
    gsofa_ctx* ctx = s->ctx;
    cudaSetDevice(ctx->device);
    if (s->ws) {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        dev_free_on(ctx, s->ws, s->ws_bytes, s->as ? s->as : ctx->stream);
    }
    if (s->as) cudaStreamSynchronize(s->as);
    for (int k = 0; k < kKernelStreams; k++)
        if (s->ks[k]) cudaStreamSynchronize(s->ks[k]);
    if (s->cs) cudaStreamSynchronize(s->cs);
    if (s->fs) cudaStreamSynchronize(s->fs);
    for (cudaEvent_t e : s->slot_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : s->pub_ev)
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < kKernelStreams; k++)
        if (s->kdone[k]) cudaEventDestroy(s->kdone[k]);
    if (s->as) cudaStreamDestroy(s->as);
    for (int k = 0; k < kKernelStreams; k++)
        if (s->ks[k]) cudaStreamDestroy(s->ks[k]);
    if (s->h_alive) cudaFreeHost(s->h_alive);
    if (s->cs) cudaStreamDestroy(s->cs);
    if (s->fs) cudaStreamDestroy(s->fs);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_desc) cudaFreeHost(s->h_desc);
    if (s->h_claim) cudaFreeHost(s->h_claim);
    if (s->h_cnt) cudaFreeHost(s->h_cnt);
    if (s->h_sstat) cudaFreeHost(s->h_sstat);
    s->stager.release();
}

}  // namespace

extern "C" {

int gsofa_server_create(gsofa_ctx* ctx, const gsofa_opts* opts, int32_t max_n,
                        size_t budget_bytes, gsofa_server** out) {
    if (!ctx || !out || max_n <= 0) return GSOFA_ERR_ARG;
    *out = nullptr;
    gsofa_opts o;
    if (opts) o = *opts;
    else gsofa_opts_default(&o);
    if (o.max_supernode_size <= 0 || o.threads_per_source < 0 || o.sources_in_flight < 0 ||
        o.chunk_sources < 0 || o.cached_closures < 0)
        return set_err(ctx, GSOFA_ERR_ARG, "invalid serving options");
    if (o.flags & GSOFA_PATTERN)
        return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "GSOFA_PATTERN is not served");
    // default CTA size: the plain path's for the largest order served (the
    // widest bitmap then fits in shared memory up to n of about 1.8M)
    const int block = o.threads_per_source > 0 ? o.threads_per_source
                                                : std::max(256, default_block(max_n, ctx->smem_per_sm));
    if (block != 256 && block != 512 && block != 1024)
        return set_err(ctx, GSOFA_ERR_ARG, "serving threads_per_source must be 256, 512 or 1024");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");

    gsofa_server* s = new (std::nothrow) gsofa_server();
    if (!s) return set_err(ctx, GSOFA_ERR_OOM_BUDGET, "host allocation failed");
    s->ctx = ctx;
    s->opts = o;
    s->max_n = max_n;
    s->budget = budget_bytes ? budget_bytes : kDefaultBudget;
    s->block = block;
    s->merge = !(o.flags & GSOFA_NO_MERGE);
    s->ring = o.cached_closures > 0 ? std::min(o.cached_closures, kMaxRing) : kDefaultRing;
    while (s->ring & (s->ring - 1)) s->ring &= s->ring - 1;
    s->t0 = std::chrono::steady_clock::now();
    auto fail = [&](int rc, const char* what, cudaError_t e) {
        if (e != cudaSuccess) set_err(ctx, rc, "%s: %s", what, cudaGetErrorString(e));
        else set_err(ctx, rc, "%s", what);
        release(s);
        delete s;
        return rc;
    };

    // shared-memory bitmap: the widest that keeps the block's full residency
    // (none with the diagnostic GSOFA_FORCE_GLOBAL_BITMAP)
    const int occ_target = 1024 / block;
    size_t smem = 0;
    if (!(o.flags & GSOFA_FORCE_GLOBAL_BITMAP)) {
        smem = (size_t)std::min(ctx->smem_optin, ctx->smem_per_sm / occ_target - 8 * 1024);
        smem &= ~(size_t)1023;
        while (smem >= 4096 && serve_occupancy(block, smem) < occ_target) smem -= 1024;
        if (smem < 4096) smem = 0;
    }
    if (serve_occupancy(block, smem) <= 0)
        return fail(GSOFA_ERR_UNSUPPORTED, "serving kernel cannot be resident", cudaSuccess);
    s->smem = smem;
    s->smem_words = (long long)(smem / 4);
    s->occ = serve_occupancy(block, smem);
    s->words = (((long long)max_n + 31) >> 5) + 6;
    s->grid = s->occ * std::max(1, ctx->sm_count - kReserveSms);
    if (o.sources_in_flight > 0) s->grid = std::min(s->grid, o.sources_in_flight);

    // the side and control streams outrank the kernel stream: when an SM
    // frees up, their pending blocks are placed first
    cudaError_t e;
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    for (int k = 0; k < kKernelStreams; k++)
        if ((e = cudaStreamCreateWithPriority(&s->ks[k], cudaStreamNonBlocking, prio_low)) !=
            cudaSuccess)
            return fail(GSOFA_ERR_CUDA, "stream", e);
    if ((e = cudaStreamCreateWithPriority(&s->as, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "stream", e);
    if ((e = cudaStreamCreateWithPriority(&s->cs, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "stream", e);
    if ((e = cudaStreamCreateWithPriority(&s->fs, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "stream", e);
    for (int k = 0; k < kKernelStreams; k++)
        if ((e = cudaEventCreateWithFlags(&s->kdone[k], cudaEventDisableTiming)) != cudaSuccess)
            return fail(GSOFA_ERR_CUDA, "event", e);
    s->slot_ev.assign(kSlots, nullptr);
    s->pub_ev.assign(kSlots, nullptr);
    for (auto& ev : s->slot_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
            return fail(GSOFA_ERR_CUDA, "event", e);
    for (auto& ev : s->pub_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
            return fail(GSOFA_ERR_CUDA, "event", e);
    if ((e = cudaHostAlloc((void**)&s->h_done, 8 * kSlots, cudaHostAllocMapped)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "mapped host memory", e);
    memset(s->h_done, 0, 8 * kSlots);
    if ((e = cudaHostGetDevicePointer((void**)&s->d_done, s->h_done, 0)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "mapped host memory", e);
    if ((e = cudaMallocHost(&s->h_ctl, kCtlBytes)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&s->h_alive, 64)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "pinned host memory", e);
    memset(s->h_ctl, 0, 16);
    memset(static_cast<char*>(s->h_ctl) + 16, 0xff, kCtlBytes - 16);
    if ((e = cudaMallocHost((void**)&s->h_desc, sizeof(MatDesc) * kSlots)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&s->h_claim, 8 * kSlots)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&s->h_cnt, 8 * CNT_SLOTS * kSlots)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&s->h_sstat, 4 * kSlots)) != cudaSuccess ||
        (e = s->stager.init()) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "pinned host memory", e);

    // device workspace: per-CTA queues, closure rings and global bitmaps
    // (only when max_n's bitmap exceeds shared memory), then the tables
    const bool need_gbm = s->words > s->smem_words;
    const size_t G = (size_t)s->grid;
    const size_t qb = align256(G * (size_t)max_n * 4);
    const size_t rb = s->merge ? align256(G * (size_t)s->ring * (size_t)s->words * 4) : 0;
    const size_t gb = need_gbm ? align256(G * (size_t)s->words * 4) : 0;
    const size_t tb = align256(sizeof(MatDesc) * kSlots) + align256(8 * kSlots) * 2 +
                      align256(4 * kSlots) + 256 + align256(4 * (size_t)((s->grid + 31) / 32)) +
                      align256(kCtlBytes);
    s->ws_bytes = qb + rb + gb + tb;
    if (s->ws_bytes > s->budget)
        return fail(GSOFA_ERR_OOM_BUDGET, "serving workspace exceeds the budget", cudaSuccess);
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        int rc = dev_alloc_on(ctx, s->ws_bytes, &s->ws, s->as);
        if (rc) {
            s->ws = nullptr;
            release(s);
            delete s;
            return rc;
        }
    }
    char* b = static_cast<char*>(s->ws);
    s->queue = reinterpret_cast<int32_t*>(b);
    b += qb;
    s->rings = s->merge ? reinterpret_cast<uint32_t*>(b) : nullptr;
    b += rb;
    s->gbm = need_gbm ? reinterpret_cast<uint32_t*>(b) : nullptr;
    b += gb;
    s->d_slots = reinterpret_cast<MatDesc*>(b);
    b += align256(sizeof(MatDesc) * kSlots);
    s->d_claim = reinterpret_cast<unsigned long long*>(b);
    b += align256(8 * kSlots);
    s->d_items_done = reinterpret_cast<unsigned long long*>(b);
    b += align256(8 * kSlots);
    s->d_slot_status = reinterpret_cast<int32_t*>(b);
    b += align256(4 * kSlots);
    s->d_work = reinterpret_cast<unsigned long long*>(b);
    s->d_rr = reinterpret_cast<unsigned int*>(s->d_work + 1);
    s->d_status = reinterpret_cast<int32_t*>(s->d_work + 2);
    s->d_alive = reinterpret_cast<int*>(s->d_work + 3);
    b += 256;
    s->d_cta_slots = reinterpret_cast<unsigned int*>(b);
    b += align256(4 * (size_t)((s->grid + 31) / 32));
    s->d_ctl = b;
    if (need_gbm && (e = cudaMemsetAsync(s->gbm, 0, gb, s->as)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "workspace init", e);
    // claim words start at request number 0 (never used): nothing claimable
    if ((e = cudaMemsetAsync(s->d_claim, 0, 8 * kSlots, s->as)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->d_work, 0, 256, s->as)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->d_cta_slots, 0, 4 * (size_t)((s->grid + 31) / 32), s->as)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(s->d_ctl, s->h_ctl, kCtlBytes, cudaMemcpyHostToDevice, s->as)) !=
            cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "workspace init", e);
    if ((e = cudaStreamSynchronize(s->as)) != cudaSuccess)
        return fail(GSOFA_ERR_CUDA, "workspace init", e);
    s->fixed = s->ws_bytes;
    s->in_use = s->peak = s->fixed;
    s->slot_req.assign(kSlots, nullptr);
    for (int i = kSlots - 1; i >= 0; i--) s->free_slots.push_back(i);
    s->st.grid = s->grid;
    s->st.block = s->block;
    try {
        s->th = std::thread(loop, s);
    } catch (...) {
        return fail(GSOFA_ERR_UNSUPPORTED, "cannot start the serving thread", cudaSuccess);
    }
    *out = s;
    return GSOFA_OK;
}

int gsofa_server_submit(gsofa_server* s, int32_t n, int64_t nnz, const int32_t* row_begin,
                        const int32_t* row_end, const int32_t* col, uint64_t* ticket) {
    if (!s || !ticket) return GSOFA_ERR_ARG;
    *ticket = 0;
    if (n < 0 || nnz < 0 || (n > 0 && (!row_begin || !row_end)) || (nnz > 0 && !col))
        return GSOFA_ERR_ARG;
    if (n > s->max_n) return GSOFA_ERR_UNSUPPORTED;
    auto r = std::make_shared<Request>();
    r->n = n;
    r->nnz = nnz;
    r->beg = row_begin;
    r->end = row_end;
    r->col = col;
    r->footprint = request_footprint(s, n, nnz);
    if (r->footprint + s->fixed > s->budget) return GSOFA_ERR_OOM_BUDGET;
    std::lock_guard<std::mutex> g(s->mu);
    if (s->shutdown) return GSOFA_ERR_ARG;
    r->ticket = s->next_ticket++;
    r->t_submit = now_ms(s);
    s->queued.push_back(r);
    s->tickets[r->ticket] = r;
    s->st.submitted++;
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return GSOFA_OK;
}

// Hands out a finished request's result (once).  With res == NULL the result
// is returned in *drop for the caller to destroy outside the server's lock.
static int take_result(Request& r, gsofa_result** res, gsofa_result** drop) {
    if (r.state == R_FAILED) return r.status;
    if (r.state != R_DONE) return GSOFA_ERR_BUSY;
    if (r.handed_out || !r.res) return GSOFA_ERR_ARG;
    r.handed_out = true;
    if (res) *res = r.res;
    else *drop = r.res;
    r.res = nullptr;
    return GSOFA_OK;
}

int gsofa_server_poll(gsofa_server* s, uint64_t ticket, gsofa_result** res) {
    if (!s) return GSOFA_ERR_ARG;
    if (res) *res = nullptr;
    gsofa_result* drop = nullptr;
    int rc;
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) return GSOFA_ERR_ARG;
        rc = take_result(*it->second, res, &drop);
    }
    if (drop) result_free(drop);
    return rc;
}

int gsofa_server_wait(gsofa_server* s, uint64_t ticket, double timeout_ms, gsofa_result** res) {
    if (!s) return GSOFA_ERR_ARG;
    if (res) *res = nullptr;
    gsofa_result* drop = nullptr;
    int rc;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) return GSOFA_ERR_ARG;
        std::shared_ptr<Request> r = it->second;
        auto done = [&] { return r->state == R_DONE || r->state == R_FAILED; };
        if (timeout_ms < 0) {
            s->cv_done.wait(lk, done);
        } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                        done)) {
            return GSOFA_ERR_TIMEOUT;
        }
        rc = take_result(*r, res, &drop);
    }
    if (drop) result_free(drop);
    return rc;
}

int gsofa_server_ticket_info(gsofa_server* s, uint64_t ticket, gsofa_ticket_info* info) {
    if (!s || !info) return GSOFA_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return GSOFA_ERR_ARG;
    const Request& r = *it->second;
    info->t_submit_ms = r.t_submit;
    info->t_admit_ms = r.t_admit;
    info->t_publish_ms = r.t_publish;
    info->t_done_ms = r.t_done;
    info->footprint_bytes = r.footprint;
    info->status = (r.state == R_DONE || r.state == R_FAILED) ? r.status : GSOFA_ERR_BUSY;
    info->n = r.n;
    return GSOFA_OK;
}

int gsofa_server_get_stats(gsofa_server* s, gsofa_server_stats* out) {
    if (!s || !out) return GSOFA_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    *out = s->st;
    out->bytes_in_use = s->in_use;
    out->peak_bytes = s->peak;
    out->fixed_bytes = s->fixed;
    return GSOFA_OK;
}

const char* gsofa_server_last_error(const gsofa_server* s) {
    if (!s) return "null server";
    return s->err.c_str();
}

int gsofa_server_destroy(gsofa_server* s) {
    if (!s) return GSOFA_ERR_ARG;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->shutdown = true;
        s->cv_work.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    // the loop has finished every request and the kernel has exited
    for (auto& kv : s->tickets) {
        Request& r = *kv.second;
        if (r.res) {
            result_free(r.res);
            r.res = nullptr;
        }
    }
    release(s);
    delete s;
    return GSOFA_OK;
}

}  // extern "C"
