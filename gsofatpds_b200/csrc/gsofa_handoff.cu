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
// per-block bitmaps.  The ids at or past each list's block end are emitted
// list after list, so every block's ids form one contiguous segment; a
// segmented sort of the 32-bit ids, a head flag per new value (the first of
// a segment, or one that differs from its predecessor) and a scan of the
// flags give each block's sorted union and its offset.
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

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
                            int32_t* __restrict__ ids) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = gw; c < n; c += nwarps) {  // a warp per list
        const int32_t l = start[blk[c] + 1];
        const long long b = ptr[c], e = ptr[c + 1];
        const long long first = lower_bound_i32(idx, b, e, l);
        for (long long j = first + lane; j < e; j += 32) ids[off[c] + (j - first)] = idx[j];
    }
}

// seg[k] = where block k's ids start (its first list's offset); seg[nb] = total
__global__ void segment_kernel(long long nblocks, const int32_t* __restrict__ start,
                               const long long* __restrict__ off, int32_t* __restrict__ seg) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k <= nblocks;
         k += (long long)gridDim.x * blockDim.x)
        seg[k] = (int32_t)off[start[k]];
}

// flag[i] = 1 when sorted[i] opens a segment or differs from sorted[i-1]
// (head[i] marks segment starts)
__global__ void new_value_kernel(long long count, const int32_t* __restrict__ sorted,
                                 const int8_t* __restrict__ head, int32_t* __restrict__ flag) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || head[i] || sorted[i] != sorted[i - 1]) ? 1 : 0;
}

__global__ void head_kernel(long long nblocks, const int32_t* __restrict__ seg,
                            int8_t* __restrict__ head) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nblocks;
         k += (long long)gridDim.x * blockDim.x)
        if (seg[k] < seg[k + 1]) head[seg[k]] = 1;
}

// out[pos[i]] = sorted[i] for flagged i; out_ptr[k] = pos at block k's start
__global__ void compact_kernel(long long count, const int32_t* __restrict__ sorted,
                               const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                               int32_t* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = sorted[i];
}

__global__ void block_ptr_kernel(long long nblocks, const int32_t* __restrict__ seg,
                                 const int32_t* __restrict__ pos, int64_t* __restrict__ out_ptr) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k <= nblocks;
         k += (long long)gridDim.x * blockDim.x)
        out_ptr[k] = pos[seg[k]];
}

int grid_for(long long items, int threads) {
    long long g = (items + threads - 1) / threads;
    return (int)std::max(1ll, std::min(g, 148ll * 32));
}

// Sorted union per block of one side's lists past the block end: fills
// out_ptr (nblocks + 1) and allocates *out_idx (*out_count ids).
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
    if (total >= INT32_MAX)
        return set_err(ctx, GSOFA_ERR_UNSUPPORTED, "supernodal form: 2^31 entries or more");
    const int items = (int)total;
    const size_t I = (size_t)std::max(items, 1);
    int32_t* ids = static_cast<int32_t*>(S.get(4 * I));
    int32_t* sorted = static_cast<int32_t*>(S.get(4 * I));
    int32_t* flag = static_cast<int32_t*>(S.get(4 * (I + 1)));
    int32_t* pos = static_cast<int32_t*>(S.get(4 * (I + 1)));
    int8_t* head = static_cast<int8_t*>(S.get(I));
    int32_t* seg = static_cast<int32_t*>(S.get(4 * ((size_t)nblocks + 1)));
    if (!ids || !sorted || !flag || !pos || !head || !seg) return GSOFA_ERR_OOM_BUDGET;
    emit_kernel<<<grid_for(32ll * n, 256), 256, 0, st>>>(n, ptr, idx, blk, start, off, ids);
    segment_kernel<<<grid_for(nblocks + 1, 256), 256, 0, st>>>(nblocks, start, off, seg);
    size_t sb = 0, pb = 0;
    cub::DeviceSegmentedSort::SortKeys(nullptr, sb, ids, sorted, items, (int)nblocks, seg, seg + 1,
                                       st);
    cub::DeviceScan::ExclusiveSum(nullptr, pb, flag, pos, items + 1, st);
    void* tmp2 = S.get(std::max(sb, pb));
    if (!tmp2) return GSOFA_ERR_OOM_BUDGET;
    cub::DeviceSegmentedSort::SortKeys(tmp2, sb, ids, sorted, items, (int)nblocks, seg, seg + 1,
                                       st);
    cudaMemsetAsync(head, 0, I, st);
    head_kernel<<<grid_for(nblocks, 256), 256, 0, st>>>(nblocks, seg, head);
    cudaMemsetAsync(flag + items, 0, 4, st);
    new_value_kernel<<<grid_for(items, 256), 256, 0, st>>>(items, sorted, head, flag);
    cub::DeviceScan::ExclusiveSum(tmp2, pb, flag, pos, items + 1, st);
    int nu = 0;
    if (cudaMemcpyAsync(&nu, pos + items, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(ctx, GSOFA_ERR_CUDA, "supernodal form: unique count read-back");
    block_ptr_kernel<<<grid_for(nblocks + 1, 256), 256, 0, st>>>(nblocks, seg, pos, out_ptr);
    int32_t* dst = nullptr;
    if (dev_alloc_on(ctx, 4 * (size_t)std::max(nu, 1), (void**)&dst, st)) return GSOFA_ERR_OOM_BUDGET;
    compact_kernel<<<grid_for(items, 256), 256, 0, st>>>(items, sorted, flag, pos, dst);
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
    r->sn_nl = nl;  // recorded at once: a failure below frees it with its size
    rc = one_side(ctx, S, n, nb, r->uptr, r->ucols, blk, start, up, &r->sn_ucols, &nu);
    if (rc) return rc;
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
