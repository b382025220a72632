// gsofa_cli -- command-line front end accepting the reference's two argument
// layouts and printing its "Final ..." summary lines
// (gSoFa_SOAComparison/main.cu:49-61, SpaceOptimization/main.cu:38-47).
//   SOA: gsofa_cli beg end csr num_process max_supernode_size percent_cat0
//        percent_cat2 N_blocks_source_cat2 N_GPU_Node N_src_group
//   SPO: gsofa_cli beg end csr N_virtualGPU total_memory_GB
#include <cstdio>
#include <cstdlib>

#include "../../include/gsofa.h"

int main(int argc, char** argv) {
    if (argc != 11 && argc != 6) {
        fprintf(stderr,
                "usage: %s beg end csr #Processes max_supernode_size percent_cat0 percent_cat2 "
                "N_blocks_source_cat2 N_GPU_Node N_src_group\n"
                "   or: %s beg end csr N_virtualGPU total_memory_GB\n",
                argv[0], argv[0]);
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
