// ref_soa_supernodes.cu -- runs the reference's own supernode kernel,
// warpcentric_local_detection_test (gSoFa_SOAComparison/
// symbfact_warp_centric_new_scheduling.cuh:1790-2123), on given inputs.
// TEST INFRASTRUCTURE ONLY (oracle/ref_soa.py drives it); the product never
// uses it.  Built by oracle/Makefile's `ref` target against the reference's
// unmodified header, with oracle/ref_stub/mpi.h standing in for MPI.
//
// The reference launches the kernel <<<1,128>>> per source group
// (DetectSuperNodes_parallel_test, :2169-2205) with each group's nz_row_U
// counters and fill markers (fill_in[slot][m] == source when (source, m) is
// an entry).  Here one launch covers one chunk of max_supernode_size rows,
// as one group of one chunk on one GPU of one node (N_GPU_Node = 1), which
// is how the kernel reads a chunk: only the chunk's own rows and the markers
// L(r, f) with f in the chunk.  The markers are scattered into a zeroed
// mss x n array before the launch and cleared after it.  The running
// supernode counter carries over from launch to launch, and the kernel
// indexes its supernode records with it, so those hold one entry per row.
//
// Input (binary, little-endian): int32 n, int32 mss, int32 nz_row_U[n],
// int64 lptr[n+1], int32 lcols[lptr[n]] (the strictly-lower columns of each
// row).  Output: "chunk_starts <c> <k>" per chunk (the kernel's
// Nsup_per_chunk), then "Nsup_detected <N>" (its Nsup counter; the reference
// prints N + 1).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "mpi.h"
#include "symbfact_warp_centric_new_scheduling.cuh"

#define CK(x)                                                                      \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),    \
                    __FILE__, __LINE__);                                           \
            return 2;                                                              \
        }                                                                          \
    } while (0)

// markers[idx[k]] = val[k]
__global__ void scatter_markers(int* markers, const long long* idx, const int* val, long long k) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < k;
         i += (long long)gridDim.x * blockDim.x)
        markers[idx[i]] = val[i];
}

int main(int argc, char** argv) {
    if (argc != 2) {
        fprintf(stderr, "usage: %s input.bin\n", argv[0]);
        return 1;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 1;
    int n = 0, mss = 0;
    if (fread(&n, 4, 1, f) != 1 || fread(&mss, 4, 1, f) != 1 || n <= 0 || mss <= 0 ||
        mss > 1024) {
        fprintf(stderr, "bad header\n");
        return 1;
    }
    std::vector<int> nz(n);
    std::vector<long long> lptr((size_t)n + 1);
    if (fread(nz.data(), 4, n, f) != (size_t)n ||
        fread(lptr.data(), 8, (size_t)n + 1, f) != (size_t)n + 1 || lptr[0] != 0) {
        fprintf(stderr, "bad arrays\n");
        return 1;
    }
    std::vector<int> lcols((size_t)lptr[n] > 0 ? (size_t)lptr[n] : 1);
    if (lptr[n] > 0 && fread(lcols.data(), 4, (size_t)lptr[n], f) != (size_t)lptr[n]) {
        fprintf(stderr, "bad columns\n");
        return 1;
    }
    fclose(f);
    const int n_chunks = (n + mss - 1) / mss;

    // device buffers: one chunk's counters, markers (mss x n), flags, outputs
    int *d_nz, *d_markers, *d_flags, *d_chunks, *d_nsup, *d_per_chunk, *d_dummy;
    Super* d_super;
    CK(cudaMalloc(&d_nz, sizeof(int) * mss));
    CK(cudaMalloc(&d_markers, sizeof(int) * (size_t)mss * n));
    CK(cudaMemset(d_markers, 0, sizeof(int) * (size_t)mss * n));
    CK(cudaMalloc(&d_flags, sizeof(int) * mss));
    CK(cudaMalloc(&d_chunks, sizeof(int)));
    CK(cudaMalloc(&d_nsup, sizeof(int)));
    CK(cudaMemset(d_nsup, 0, sizeof(int)));
    CK(cudaMalloc(&d_per_chunk, sizeof(int) * n_chunks));
    CK(cudaMemset(d_per_chunk, 0, sizeof(int) * n_chunks));
    CK(cudaMalloc(&d_dummy, sizeof(int) * 16));
    CK(cudaMemset(d_dummy, 0, sizeof(int) * 16));
    // the kernel stores supernode i at superObj_d[i], i from its running Nsup
    // counter, which every launch continues: at most one per row in total
    CK(cudaMalloc(&d_super, sizeof(Super) * ((size_t)n + 1)));
    long long cap = 1;
    long long *d_idx = nullptr;
    int* d_val = nullptr;
    CK(cudaMalloc(&d_idx, sizeof(long long) * cap));
    CK(cudaMalloc(&d_val, sizeof(int) * cap));

    std::vector<int> h_nz(mss);
    std::vector<long long> h_idx;
    std::vector<int> h_val, h_zero;
    for (int c = 0; c < n_chunks; c++) {
        const int r0 = c * mss;
        for (int j = 0; j < mss; j++) h_nz[j] = r0 + j < n ? nz[r0 + j] : 0;
        h_idx.clear();
        h_val.clear();
        for (int j = 0; j < mss && r0 + j < n; j++) {
            const int r = r0 + j;
            for (long long k = lptr[r]; k < lptr[r + 1]; k++) {
                const int m = lcols[k];
                if (m >= r0 && m < r) {  // L(r, m) with m in the chunk
                    h_idx.push_back((long long)j * n + m);
                    h_val.push_back(r);
                }
            }
        }
        const long long k = (long long)h_idx.size();
        if (k > cap) {
            cudaFree(d_idx);
            cudaFree(d_val);
            cap = k;
            CK(cudaMalloc(&d_idx, sizeof(long long) * cap));
            CK(cudaMalloc(&d_val, sizeof(int) * cap));
        }
        CK(cudaMemcpy(d_nz, h_nz.data(), sizeof(int) * mss, cudaMemcpyHostToDevice));
        CK(cudaMemset(d_flags, 0, sizeof(int) * mss));
        CK(cudaMemcpy(d_chunks, &c, sizeof(int), cudaMemcpyHostToDevice));
        if (k > 0) {
            CK(cudaMemcpy(d_idx, h_idx.data(), sizeof(long long) * k, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d_val, h_val.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
            scatter_markers<<<64, 256>>>(d_markers, d_idx, d_val, k);
            CK(cudaGetLastError());
        }
        // the reference's own launch shape (:2198): one block of 128 threads,
        // (mss + 1) ints of shared memory
        warpcentric_local_detection_test<<<1, 128, sizeof(int_t) * (mss + 1)>>>(
            d_nz, d_nz, d_nz, d_nz, d_nz, d_nz, /*N_src_group*/ mss, mss, /*N_gpu*/ 1,
            /*global_gpu_id*/ 0, d_super, n, /*group*/ 0, n_chunks, d_per_chunk, d_nsup,
            d_markers, d_markers, d_markers, d_markers, d_markers, d_markers,
            /*source_d*/ d_dummy, /*my_supernode_d*/ d_dummy, /*new_col_ed_d*/ d_dummy,
            /*col_ed_d*/ d_dummy, /*csr_d*/ d_dummy, /*col_st_d*/ d_dummy, /*local_gpu_id*/ 0,
            /*N_GPU_Node*/ 1, /*count*/ d_dummy, d_flags, d_chunks, /*chunks*/ 1);
        CK(cudaGetLastError());
        if (k > 0) {
            h_zero.assign((size_t)k, 0);
            CK(cudaMemcpy(d_val, h_zero.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
            scatter_markers<<<64, 256>>>(d_markers, d_idx, d_val, k);
            CK(cudaGetLastError());
        }
    }
    CK(cudaDeviceSynchronize());
    std::vector<int> per(n_chunks);
    int nsup = 0;
    CK(cudaMemcpy(per.data(), d_per_chunk, sizeof(int) * n_chunks, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&nsup, d_nsup, sizeof(int), cudaMemcpyDeviceToHost));
    for (int c = 0; c < n_chunks; c++) printf("chunk_starts %d %d\n", c, per[c]);
    printf("Nsup_detected %d\n", nsup);
    return 0;
}
