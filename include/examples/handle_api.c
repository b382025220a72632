/* The handle API: load a matrix once, factor it, read the counts.
 * Build: gcc -std=c11 -I include handle_api.c -L gsofatpds_b200 -lgsofa
 * Run:   ./a.out colbeg.dat colend.dat csr.dat */
#include <stdio.h>
#include <stdlib.h>

#include "gsofa.h"

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s colbeg.dat colend.dat csr.dat\n", argv[0]);
        return 2;
    }
    gsofa_ctx* ctx;       if (gsofa_create(0, 0 /* budget: 90% of free */, &ctx)) return 1;
    gsofa_matrix* A;      if (gsofa_load_csr_files(ctx, argv[1], argv[2], argv[3], &A)) {
                              puts(gsofa_last_error(ctx)); return 1; }
                          /* or gsofa_load_csr(ctx, n, nnz, row_begin, row_end, col, &A) */
    gsofa_opts o;         gsofa_opts_default(&o); o.max_supernode_size = 128;
    gsofa_result* r;      if (gsofa_factor_symbolic(ctx, A, &o, &r)) { puts(gsofa_last_error(ctx)); return 1; }
    gsofa_counts c;       gsofa_result_counts(r, &c);        /* c.fill_count, c.n_supernodes, ... */
    int32_t *u = malloc(4 * (size_t)c.n), *z = malloc(4 * (size_t)c.n), *l = malloc(4 * (size_t)c.n);
    gsofa_result_row_counts(r, u, z, l, NULL);                /* |U row|, nz_row_U, |L col| */
    printf("fills %llu supernodes %lld\n", (unsigned long long)c.fill_count, (long long)c.n_supernodes);
    free(u); free(z); free(l);
    gsofa_result_destroy(r); gsofa_matrix_destroy(A); gsofa_destroy(ctx);
    return 0;
}
