// gsofa_noalloc.cu -- symbolic factorization for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- inside a
// host framework that owns every byte of device memory through its own pool,
// or in a latency-critical loop that was set up once and must not allocate
// again.  Such a caller loads its matrix at set-up time (gsofa_load_csr,
// which does allocate) and later factors it with caller-owned output
// buffers.  Everything else the traversal kernel needs -- its work counter,
// status word, matrix descriptor, per-CTA frontier queues and the per-CTA
// ring of recent closures -- is carved from the one static array below.
//
// The array is a file-scope __device__ object: every GPU that loads this
// library holds GSOFA_NOALLOC_SCRATCH_BYTES for it until the process exits.
// Host code cannot use the symbol itself as a device address (on the host it
// names a stand-in); every call looks the address up with
// cudaGetSymbolAddress, with the matrix's device current, so no address is
// kept across calls (a context reset between calls leaves nothing stale).
// Calls share the array: the work counter and the status word are cleared
// on every call, and two calls that overlap on the GPU race on it.
//
// Launch shape: the main entry point's defaults (gsofa_host.h) except the
// closure ring, which defaults to kNoallocRing slots instead of kDefaultRing:
// every CTA's queue and ring come out of the one fixed array, and a 64-deep
// ring (8n bytes per CTA) would leave about a quarter of the CTAs that the
// 8-deep one leaves at n ~ 600k.
#include <cuda_runtime.h>

#include "../../include/gsofa.h"
#include "gsofa_host.h"
#include "gsofa_internal.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GSOFA_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocRing = 8;

// Device address of the scratch array on the current device.
cudaError_t scratch_address(void** out) {
    return cudaGetSymbolAddress(out, g_noalloc_scratch);
}

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

// Restores the caller's current device on every return path.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int gsofa_factor_symbolic_noalloc(const gsofa_matrix* mat, const gsofa_opts* opts,
                                             void* cuda_stream, int32_t* d_nnz_u_row,
                                             int32_t* d_nz_row_u, int32_t* d_nnz_l_col,
                                             uint32_t* d_lmask, int8_t* d_supernode_flags,
                                             uint64_t* d_counters) {
    using namespace gsofa;
    MatrixView mv;
    if (!matrix_view(mat, &mv)) return GSOFA_ERR_ARG;
    if (!d_nnz_u_row || !d_nz_row_u || !d_nnz_l_col || !d_lmask || !d_counters) return GSOFA_ERR_ARG;
    gsofa_opts o;
    if (opts) {
        o = *opts;
    } else {
        gsofa_opts_default(&o);
    }
    if (o.max_supernode_size <= 0 || o.threads_per_source < 0 || o.sources_in_flight < 0 ||
        o.chunk_sources < 0 || o.cached_closures < 0)
        return GSOFA_ERR_ARG;
    // digests, per-row L scatter and materialised patterns need result
    // storage this entry point does not have
    if (o.flags & (GSOFA_L_ROW_STATS | GSOFA_PATTERN)) return GSOFA_ERR_UNSUPPORTED;
    if ((o.flags & GSOFA_SUPERNODES) && !d_supernode_flags) return GSOFA_ERR_ARG;

    DeviceGuard guard(mv.device);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
    void* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return GSOFA_ERR_CUDA;

    const int32_t n = mv.n;
    const long long words = (((long long)n + 31) >> 5) + 6;
    int sm_count = 0, smem_optin = 0, smem_per_sm = 0;
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, mv.device);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, mv.device);
    cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, mv.device);
    size_t bm_bytes = ((size_t)words * 4 + 15) & ~(size_t)15;
    const bool smem_bitmap = bm_bytes + 12 * 1024 <= (size_t)smem_optin &&
                             !(o.flags & GSOFA_FORCE_GLOBAL_BITMAP);
    int block = o.threads_per_source;
    if (block == 0) {
        const long long fit = smem_per_sm / (long long)(bm_bytes + 8 * 1024);
        block = fit >= 4 ? 256 : (fit >= 2 ? 512 : 1024);
    }
    if (block != 128 && block != 256 && block != 512 && block != 1024) return GSOFA_ERR_ARG;
    const int occ = traverse_occupancy(block, smem_bitmap, smem_bitmap ? bm_bytes : 0);
    if (occ <= 0) return GSOFA_ERR_UNSUPPORTED;

    const bool merge = !(o.flags & GSOFA_NO_MERGE);
    int ring = o.cached_closures > 0 ? o.cached_closures : kNoallocRing;
    if (ring > host::kMaxRing) ring = host::kMaxRing;
    while (ring & (ring - 1)) ring &= ring - 1;

    // scratch layout: [counter+status 256 B][descriptor][per-CTA queues]
    // [per-CTA closure rings][per-CTA global bitmaps when shared memory is too small]
    const size_t head = 256 + round256(sizeof(MatDesc));
    const size_t per_cta = round256((size_t)(n > 0 ? n : 1) * 4) +
                           (merge ? round256((size_t)ring * words * 4) : 0) +
                           (smem_bitmap ? 0 : round256((size_t)words * 4));
    if (head + per_cta > (size_t)GSOFA_NOALLOC_SCRATCH_BYTES) return GSOFA_ERR_SCRATCH;
    long long grid = (long long)occ * sm_count;
    const long long fit = (long long)(((size_t)GSOFA_NOALLOC_SCRATCH_BYTES - head) / per_cta);
    if (grid > fit) grid = fit;
    if (o.sources_in_flight > 0 && grid > o.sources_in_flight) grid = o.sources_in_flight;
    const long long chunk = o.chunk_sources > 0 ? o.chunk_sources
                                                : host::default_chunk(2ll * n, (int)grid);

    unsigned char* b = static_cast<unsigned char*>(base);
    unsigned long long* work_counter = reinterpret_cast<unsigned long long*>(b);
    int32_t* status = reinterpret_cast<int32_t*>(b + 64);
    MatDesc* ddesc = reinterpret_cast<MatDesc*>(b + 256);
    unsigned char* p = b + head;
    int32_t* queue = reinterpret_cast<int32_t*>(p);
    p += (size_t)grid * round256((size_t)(n > 0 ? n : 1) * 4);
    uint32_t* rings = merge ? reinterpret_cast<uint32_t*>(p) : nullptr;
    if (merge) p += (size_t)grid * round256((size_t)ring * words * 4);
    uint32_t* gbm = smem_bitmap ? nullptr : reinterpret_cast<uint32_t*>(p);

    MatDesc d{};
    d.n = n;
    d.flags = (int32_t)o.flags;
    d.rowptr = mv.rowptr;
    d.col = mv.col;
    d.trowptr = mv.trowptr;
    d.tcol = mv.tcol;
    d.wdeg = mv.wdeg;
    d.dplanes = mv.dplanes;
    d.nplanes = mv.nplanes;
    d.asym = mv.asym;
    d.nnz_u = d_nnz_u_row;
    d.nz_row_u = d_nz_row_u;
    d.nnz_lc = d_nnz_l_col;
    d.lmask = d_lmask;
    d.counters = reinterpret_cast<unsigned long long*>(d_counters);
    d.item_base = 0;

    cudaError_t e = cudaMemsetAsync(b, 0, 256, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counters, 0, 8 * CNT_SLOTS, st);
    if (e == cudaSuccess && d_supernode_flags && n > 0)
        e = cudaMemsetAsync(d_supernode_flags, 0, (size_t)n, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ddesc, &d, sizeof(d), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return GSOFA_ERR_CUDA;

    TraverseLaunch L{};
    L.mats = ddesc;
    L.nmats = 1;
    L.total_items = 2ll * (((long long)n + chunk - 1) / chunk);
    L.work_counter = work_counter;
    L.queue = queue;
    L.queue_stride = (long long)(round256((size_t)(n > 0 ? n : 1) * 4) / 4);
    if (o.flags & GSOFA_DEBUG_QUEUE_CAP) L.queue_stride = L.queue_stride < 64 ? L.queue_stride : 64;
    L.gbitmap = gbm;
    L.bitmap_words = words;
    L.status = status;
    L.pattern_pass = 0;
    L.bu_alpha = o.bu_alpha > 0 ? o.bu_alpha : (o.bu_alpha < 0 ? 0 : host::kDefaultBuAlpha);
    L.bu_beta = o.bu_beta > 0 ? o.bu_beta : host::kDefaultBuBeta;
    L.bu_min_src = o.bu_min_source > 0 ? o.bu_min_source : host::kBuMinSource;
    L.heavy_len = o.heavy_row > 0 ? ((o.heavy_row + 3) & ~3) : host::kDefaultHeavyRow;
    L.gprev = rings;
    L.chunk = (int)chunk;
    L.merge = merge ? 1 : 0;
    // chained starts of symmetric patterns only: the links between the two
    // directions of unsymmetric ones would need result storage (d.link stays null)
    L.chain = merge && !(o.flags & GSOFA_NO_CHAIN) ? 1 : 0;
    L.ring = ring;
    if (L.total_items > 0) {
        e = launch_traverse(L, block, (int)grid, smem_bitmap, smem_bitmap ? bm_bytes : 0, st);
        if (e != cudaSuccess) return GSOFA_ERR_CUDA;
    }
    if ((o.flags & GSOFA_SUPERNODES) && n > 0) {
        e = launch_supernodes(n, o.max_supernode_size, d_nz_row_u, d_lmask, d_supernode_flags,
                              reinterpret_cast<unsigned long long*>(d_counters), st);
        if (e != cudaSuccess) return GSOFA_ERR_CUDA;
    }
    int32_t h_status = 0;
    e = cudaMemcpyAsync(&h_status, status, sizeof(h_status), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GSOFA_ERR_CUDA;
    return device_status_code(h_status);
}
