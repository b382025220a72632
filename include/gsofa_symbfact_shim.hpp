// gsofa_symbfact_shim.hpp -- the reference-side binding: a drop-in
// symbfact_min_id over the C-ABI.  A maintainer who keeps the reference's
// main.cu includes this header in place of
// "symbfact_warp_centric_new_scheduling.cuh" and links -lgsofa.
#pragma once
#include <cstdio>
#include <cstdlib>
#include "gsofa.h"
typedef unsigned long long ull_t;

// Same signature and outputs as the reference (SOA :2529).
inline void symbfact_min_id(int argc, char** argv, int rank, ull_t& fill_count, double& time,
                            int& N_supernodes, ull_t& TEPS) {
    uint64_t fills = 0, edges = 0;
    double ms = 0;
    int32_t nsup = 0;
    int rc = gsofa_symbfact_min_id(argc, argv, rank, &fills, &ms, &nsup, &edges);
    if (rc != GSOFA_OK) {  // the reference exits on any error (barrier.cuh:11-20)
        fprintf(stderr, "gsofa: %s\n", gsofa_status_string(rc));
        exit(EXIT_FAILURE);
    }
    fill_count = fills;
    time = ms;
    N_supernodes = nsup;
    TEPS = edges;  // traversed edges, the numerator of "Final TEPS"
}
