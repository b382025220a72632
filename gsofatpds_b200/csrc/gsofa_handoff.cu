// gsofa_handoff.cu -- the symbolic-to-numeric handoff: the structure of L
// and U in supernodal block form, the input a supernodal numeric LU
// (SuperLU-style) allocates and factors from.
//
// Blocks are the supernode partition's runs of consecutive columns: block k
// is [start[k], start[k+1]), a new block beginning at every row whose
// supernode flag is set.  For block k with end l = start[k+1]:
//   L rows  = { r >= l : L(r, c) != 0 for some column c of the block }
//   U cols  = { c >= l : U(r, c) != 0 for some row r of the block }
// both sorted; the diagonal block itself is dense and implicit.  They are
// built from the materialised pattern (L by columns, U by rows) with no
// per-block bitmaps: every (block, index) pair is emitted as one 64-bit key,
// radix-sorted and made unique, and each block's range is found by binary
// search on the block id.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>

#include "gsofa_host.h"

using namespace gsofa;
using namespace gsofa::host;

namespace {

__global__ void nonzero_kernel(int32_t n, const int8_t* __restrict__ flags, int32_t* __restrict__ f) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        f[c] = flags[c] != 0;
}

__global__ void minus_one_kernel(int32_t n, int32_t* __restrict__ a) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        a[c] -= 1;
}

// blk[c] = inclusive count of flagged rows up to c, minus one: c's block.
__global__ void block_start_kernel(int32_t n, const int8_t* __restrict__ flags,
                                   const int32_t* __restrict__ blk, int32_t* __restrict__ start) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        if (flags[c]) start[blk[c]] = (int32_t)c;
}

__device__ __forceinline__ long long lower_bound_i32(const int32_t* a, long long lo, long long hi,
                                                     int32_t x) {
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// cnt[c] = entries of list c (sorted) at or beyond the end of c's block
__global__ void count_kernel(int32_t n, const int64_t* __restrict__ ptr,
                             const int32_t* __restrict__ idx, const int32_t* __restrict__ blk,
                             const int32_t* __restrict__ start, long long* __restrict__ cnt) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int32_t l = start[blk[c] + 1];
        const long long b = ptr[c], e = ptr[c + 1];
        cnt[c] = e - lower_bound_i32(idx, b, e, l);
    }
}

__global__ void emit_kernel(int32_t n, const int64_t* __restrict__ ptr,
                            const int32_t* __restrict__ idx, const int32_t* __restrict__ blk,
                            const int32_t* __restrict__ start, const long long* __restrict__ off,
                            unsigned long long* __restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = gw; c < n; c += nwarps) {  // a warp per list
        const int32_t l = start[blk[c] + 1];
        const long long b = ptr[c], e = ptr[c + 1];
        const long long first = lower_bound_i32(idx, b, e, l);
        const unsigned long long hi = (unsigned long long)(uint32_t)blk[c] << 32;
        for (long long j = first + lane; j < e; j += 32)
            keys[off[c] + (j - first)] = hi | (uint32_t)idx[j];
    }
}

// out_ptr[k] = first unique key of block k (binary search); out_idx = low words
__global__ void block_ptr_kernel(long long nblocks, const unsigned long long* __restrict__ ukeys,
                                 long long nu, int64_t* __restrict__ out_ptr) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k <= nblocks;
         k += (long long)gridDim.x * blockDim.x) {
        const unsigned long long x = (unsigned long long)k << 32;
        long long lo = 0, hi = nu;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (ukeys[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        out_ptr[k] = lo;
    }
}

__global__ void low_word_kernel(long long count, const unsigned long long* __restrict__ ukeys,
                                int32_t* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (int32_t)(uint32_t)ukeys[i];
}

int grid_for(long long items, int threads) {
    long long g = (items + threads - 1) / threads;
    return (int)std::max(1ll, std::min(g, 148ll * 32));
}

// Unique sorted (block, index) pairs of one side; returns their count and
// leaves ptr (nblocks + 1) and idx on the device in *ptr_out / *idx_out,
// allocated from the result's arena by the caller-supplied allocator.
int one_side(gsofa_ctx* ctx, DeviceScratch& S, int32_t n, long long nblocks, const int64_t* ptr,
             const int32_t* idx, const int32_t* blk, const int32_t* start, int64_t* out_ptr,
             int32_t** out_idx, long long* out_count) {
    cudaStream_t st = ctx->stream;
    long long* cnt = static_cast<long long*>(S.get(8 * ((size_t)n + 1)));
    long long* off = static_cast<long long*>(S.get(8 * ((size_t)n + 1)));
    if (!cnt || !off) return GSOFA_ERR_OOM_BUDGET;
    cudaMemsetAsync(cnt + n, 0, 8, st);
    count_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, ptr, idx, blk, start, cnt);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)n + 1, st);
    void* tmp = S.get(tb);
    if (!tmp) return GSOFA_ERR_OOM_BUDGET;
    cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, (int)n + 1, st);
    long long total = 0;
    if (cudaMemcpyAsync(&total, off + n, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form: count read-back");
    if (total > INT32_MAX)
        return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "supernodal form: more than 2^31 entries");
    const int items = (int)total;
    unsigned long long* keys = static_cast<unsigned long long*>(S.get(8 * (size_t)items));
    unsigned long long* sorted = static_cast<unsigned long long*>(S.get(8 * (size_t)items));
    unsigned long long* uniq = static_cast<unsigned long long*>(S.get(8 * (size_t)items));
    int* nsel = static_cast<int*>(S.get(16));
    if (!keys || !sorted || !uniq || !nsel) return GSOFA_ERR_OOM_BUDGET;
    emit_kernel<<<grid_for(32ll * n, 256), 256, 0, st>>>(n, ptr, idx, blk, start, off, keys);
    int end_bit = 32;
    while (end_bit < 64 && (1ll << (end_bit - 32)) <= nblocks) end_bit++;
    size_t sb = 0, ub = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sb, keys, sorted, items, 0, end_bit, st);
    cub::DeviceSelect::Unique(nullptr, ub, sorted, uniq, nsel, items, st);
    void* tmp2 = S.get(std::max(sb, ub));
    if (!tmp2) return GSOFA_ERR_OOM_BUDGET;
    cub::DeviceRadixSort::SortKeys(tmp2, sb, keys, sorted, items, 0, end_bit, st);
    cub::DeviceSelect::Unique(tmp2, ub, sorted, uniq, nsel, items, st);
    int nu = 0;
    if (cudaMemcpyAsync(&nu, nsel, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form: unique count read-back");
    block_ptr_kernel<<<grid_for(nblocks + 1, 256), 256, 0, st>>>(nblocks, uniq, nu, out_ptr);
    int32_t* dst = nullptr;
    if (dev_alloc_on(ctx, 4 * (size_t)std::max(nu, 1), (void**)&dst, st)) return GSOFA_ERR_OOM_BUDGET;
    low_word_kernel<<<grid_for(nu, 256), 256, 0, st>>>(nu, uniq, dst);
    *out_idx = dst;
    *out_count = nu;
    return cudaGetLastError() == cudaSuccess ? GSOFA_OK
                                              : set_err(ctx, GSOFA_ERR_CUDA, "supernodal form");
}

// Builds and caches the supernodal form in the result.
int build(gsofa_result* r) {
    gsofa_ctx* ctx = r->ctx;
    if (!(r->flags & GSOFA_PATTERN) || !r->uptr || !(r->flags & GSOFA_SUPERNODES))
        return set_err(ctx, GSOFA_ERR_ARG,
                       "supernodal form needs GSOFA_PATTERN and GSOFA_SUPERNODES");
    const int32_t n = r->n;
    cudaStream_t st = ctx->stream;
    DeviceScratch S(ctx);
    int32_t* f01 = static_cast<int32_t*>(S.get(4 * ((size_t)n + 1)));
    int32_t* blk = static_cast<int32_t*>(S.get(4 * ((size_t)n + 1)));
    if (!f01 || !blk) return GSOFA_ERR_OOM_BUDGET;
    nonzero_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, r->sflags, f01);
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, f01, blk, (int)n, st);
    void* tmp = S.get(tb);
    if (!tmp) return GSOFA_ERR_OOM_BUDGET;
    cub::DeviceScan::InclusiveSum(tmp, tb, f01, blk, (int)n, st);
    int32_t nb = 0;
    if (cudaMemcpyAsync(&nb, blk + n - 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form: block count read-back");
    // row 0 always starts a block, so the inclusive counts are >= 1
    minus_one_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, blk);
    int32_t* start = nullptr;
    int64_t* lp = nullptr;
    int64_t* up = nullptr;
    if (dev_alloc_on(ctx, 4 * ((size_t)nb + 1), (void**)&start, st)) return GSOFA_ERR_OOM_BUDGET;
    if (dev_alloc_on(ctx, 8 * ((size_t)nb + 1), (void**)&lp, st)) {
        dev_free_on(ctx, start, 4 * ((size_t)nb + 1), st);
        return GSOFA_ERR_OOM_BUDGET;
    }
    if (dev_alloc_on(ctx, 8 * ((size_t)nb + 1), (void**)&up, st)) {
        dev_free_on(ctx, start, 4 * ((size_t)nb + 1), st);
        dev_free_on(ctx, lp, 8 * ((size_t)nb + 1), st);
        return GSOFA_ERR_OOM_BUDGET;
    }
    r->sn_start = start;
    r->sn_lptr = lp;
    r->sn_uptr = up;
    r->sn_nblocks = nb;
    block_start_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, r->sflags, blk, start);
    cudaMemcpyAsync(start + nb, &n, 4, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);  // the copy's source is on this stack frame
    // L: rows of each column; U: columns of each row
    long long nl = 0, nu = 0;
    int rc = one_side(ctx, S, n, nb, r->lptr, r->lrows, blk, start, lp, &r->sn_lrows, &nl);
    if (rc) return rc;
    rc = one_side(ctx, S, n, nb, r->uptr, r->ucols, blk, start, up, &r->sn_ucols, &nu);
    if (rc) return rc;
    r->sn_nl = nl;
    r->sn_nu = nu;
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form");
    r->sn_built = true;
    return GSOFA_OK;
}

}  // namespace

// Frees a result's supernodal form (called by result_free with ctx->mu held).
void gsofa::host::supernodal_free(gsofa_result* r) {
    gsofa_ctx* ctx = r->ctx;
    const size_t nb = (size_t)std::max<long long>(r->sn_nblocks, 0) + 1;
    dev_free_on(ctx, r->sn_start, 4 * nb, ctx->stream);
    dev_free_on(ctx, r->sn_lptr, 8 * nb, ctx->stream);
    dev_free_on(ctx, r->sn_uptr, 8 * nb, ctx->stream);
    dev_free_on(ctx, r->sn_lrows, 4 * (size_t)std::max<long long>(r->sn_nl, 1), ctx->stream);
    dev_free_on(ctx, r->sn_ucols, 4 * (size_t)std::max<long long>(r->sn_nu, 1), ctx->stream);
    r->sn_start = nullptr;
    r->sn_lptr = r->sn_uptr = nullptr;
    r->sn_lrows = r->sn_ucols = nullptr;
    r->sn_built = false;
}

extern "C" int gsofa_result_supernodal(const gsofa_result* res, int64_t* nblocks, int64_t* nl,
                                       int64_t* nu, int32_t* block_start, int64_t* lptr,
                                       int32_t* lrows, int64_t* uptr, int32_t* ucols) {
    if (!res) return GSOFA_ERR_ARG;
    gsofa_result* r = const_cast<gsofa_result*>(res);  // the form is built once and cached
    gsofa_ctx* ctx = r->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "cudaSetDevice");
    if (!r->sn_built) {
        const int rc = build(r);
        if (rc) {
            supernodal_free(r);
            return rc;
        }
    }
    if (nblocks) *nblocks = r->sn_nblocks;
    if (nl) *nl = r->sn_nl;
    if (nu) *nu = r->sn_nu;
    const size_t nb = (size_t)r->sn_nblocks + 1;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (block_start) e = cudaMemcpyAsync(block_start, r->sn_start, 4 * nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && lptr) e = cudaMemcpyAsync(lptr, r->sn_lptr, 8 * nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && uptr) e = cudaMemcpyAsync(uptr, r->sn_uptr, 8 * nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && lrows && r->sn_nl > 0)
        e = cudaMemcpyAsync(lrows, r->sn_lrows, 4 * (size_t)r->sn_nl, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && ucols && r->sn_nu > 0)
        e = cudaMemcpyAsync(ucols, r->sn_ucols, 4 * (size_t)r->sn_nu, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form: %s", cudaGetErrorString(e));
    return GSOFA_OK;
}
