// gsofa_cli -- command-line front end accepting the reference's two argument
// layouts and printing its "Final ..." summary lines
// (gSoFa_SOAComparison/main.cu:49-61, SpaceOptimization/main.cu:38-47).
//   SOA: gsofa_cli beg end csr num_process max_supernode_size percent_cat0
//        percent_cat2 N_blocks_source_cat2 N_GPU_Node N_src_group
//   SPO: gsofa_cli beg end csr N_virtualGPU total_memory_GB
// Two more modes for the binary CSR files of include/gsofa.h:
//   gsofa_cli --convert beg end csr out.gsofacsr   (parse once, no GPU)
//   gsofa_cli --binary file.gsofacsr max_supernode_size
// and two that order the matrix on the device first (gsofa_order_nd or
// gsofa_order_hybrid, then gsofa_matrix_permute) and factor the permuted
// matrix:
//   gsofa_cli --order file.gsofacsr max_supernode_size
//   gsofa_cli --order-hybrid file.gsofacsr max_supernode_size
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/gsofa.h"

// order: 0 = none, 1 = level-set nested dissection, 2 = hybrid
static int run_binary(const char* path, int mss, int order) {
    gsofa_ctx* ctx = nullptr;
    int rc = gsofa_create(0, 0, &ctx);
    if (rc) {
        fprintf(stderr, "gsofa_cli: %s\n", gsofa_status_string(rc));
        return 2;
    }
    gsofa_matrix* m = nullptr;
    gsofa_result* r = nullptr;
    gsofa_opts o;
    gsofa_opts_default(&o);
    o.max_supernode_size = mss;
    rc = gsofa_load_csr_binary(ctx, path, &m);
    if (rc == GSOFA_OK && order) {
        int32_t n = 0;
        int64_t nnz = 0;
        gsofa_matrix_info(m, &n, &nnz);
        std::vector<int32_t> perm((size_t)n);
        gsofa_order_stats st;
        gsofa_matrix* pm = nullptr;
        rc = order == 2 ? gsofa_order_hybrid(ctx, m, 0, perm.data(), &st)
                        : gsofa_order_nd(ctx, m, 0, 0, perm.data(), &st);
        if (rc == GSOFA_OK) rc = gsofa_matrix_permute(ctx, m, perm.data(), &pm);
        if (rc == GSOFA_OK) {
            printf("Ordering (%s nested dissection on the device): %g ms, %d rounds, %lld separator "
                   "vertices\n",
                   order == 2 ? "hybrid" : "level-set", st.ms, st.rounds,
                   (long long)st.separator_vertices);
            gsofa_matrix_destroy(m);
            m = pm;
        }
    }
    if (rc == GSOFA_OK) rc = gsofa_factor_symbolic(ctx, m, &o, &r);
    if (rc != GSOFA_OK) {
        fprintf(stderr, "gsofa_cli: %s (%s)\n", gsofa_status_string(rc), gsofa_last_error(ctx));
        gsofa_destroy(ctx);
        return 2;
    }
    gsofa_counts c;
    gsofa_result_counts(r, &c);
    printf("Final Number of fill-ins detected: %llu\n", (unsigned long long)c.fill_count);
    printf("Final Number of Supernodes detected: %lld\n", (long long)c.n_supernodes);
    printf("Final Maximum time reported among the processes: %g ms\n", c.ms_device);
    printf("Final TEPS according to slowest process: %g\n",
           c.ms_device > 0 ? c.edges_traversed / (c.ms_device / 1000.0) : 0.0);
    gsofa_result_destroy(r);
    gsofa_matrix_destroy(m);
    gsofa_destroy(ctx);
    return 0;
}

int main(int argc, char** argv) {
    if (argc == 6 && strcmp(argv[1], "--convert") == 0) {
        const int rc = gsofa_convert_dat_to_binary(argv[2], argv[3], argv[4], argv[5]);
        if (rc != GSOFA_OK) {
            fprintf(stderr, "gsofa_cli: %s\n", gsofa_status_string(rc));
            return 2;
        }
        return 0;
    }
    if (argc == 4 && strcmp(argv[1], "--binary") == 0) return run_binary(argv[2], atoi(argv[3]), 0);
    if (argc == 4 && strcmp(argv[1], "--order") == 0) return run_binary(argv[2], atoi(argv[3]), 1);
    if (argc == 4 && strcmp(argv[1], "--order-hybrid") == 0)
        return run_binary(argv[2], atoi(argv[3]), 2);
    if (argc != 11 && argc != 6) {
        fprintf(stderr,
                "usage: %s beg end csr #Processes max_supernode_size percent_cat0 percent_cat2 "
                "N_blocks_source_cat2 N_GPU_Node N_src_group\n"
                "   or: %s beg end csr N_virtualGPU total_memory_GB\n"
                "   or: %s --convert beg end csr out.gsofacsr\n"
                "   or: %s --binary file.gsofacsr max_supernode_size\n"
                "   or: %s --order file.gsofacsr max_supernode_size\n"
                "   or: %s --order-hybrid file.gsofacsr max_supernode_size\n",
                argv[0], argv[0], argv[0], argv[0], argv[0], argv[0]);
        return 1;
    }
    printf("Number of Processes: %s\n", argv[4]);
    uint64_t fills = 0, edges = 0;
    double ms = 0;
    int32_t nsup = -1;
    int rc = gsofa_symbfact_min_id(argc, argv, 0, &fills, &ms, &nsup, &edges);
    if (rc != GSOFA_OK) {
        fprintf(stderr, "gsofa_cli: %s\n", gsofa_status_string(rc));
        return 2;
    }
    printf("Final Number of fill-ins detected: %llu\n", (unsigned long long)fills);
    if (argc == 11) printf("Final Number of Supernodes detected: %d\n", nsup);
    printf("Final Maximum time reported among the processes: %g ms\n", ms);
    printf("Final Minimum time reported among the processes: %g ms\n", ms);
    printf("Final TEPS according to slowest process: %g\n", ms > 0 ? edges / (ms / 1000.0) : 0.0);
    return 0;
}
