/* The serving request loop: submit host CSR matrices, wait for results.
 * Build: gcc -std=c11 -I include serving.c -L gsofatpds_b200 -lgsofa
 * The example serves one small tridiagonal matrix. */
#include <stdio.h>
#include <stdlib.h>

#include "gsofa.h"

int main(void) {
    enum { n = 1000 };
    static int32_t row_begin[n], row_end[n], col[3 * n];
    int64_t nnz = 0;
    for (int i = 0; i < n; i++) {
        row_begin[i] = (int32_t)nnz;
        for (int j = i - 1; j <= i + 1; j++)
            if (j >= 0 && j < n) col[nnz++] = j;
        row_end[i] = (int32_t)nnz;
    }
    gsofa_ctx* ctx;     if (gsofa_create(0, 0, &ctx)) return 1;
    gsofa_opts o;       gsofa_opts_default(&o);
    gsofa_server* srv;  gsofa_server_create(ctx, &o, /*max_n*/ 1000000, /*budget*/ 40ull << 30, &srv);
    uint64_t t;         gsofa_server_submit(srv, n, nnz, row_begin, row_end, col, &t);  /* returns at once */
    gsofa_result* r;    gsofa_server_wait(srv, t, -1.0, &r);   /* or gsofa_server_poll: GSOFA_ERR_BUSY until done */
    gsofa_ticket_info i; gsofa_server_ticket_info(srv, t, &i); /* submit / admit / publish / done times */
    gsofa_counts c;     gsofa_result_counts(r, &c);
    printf("fills %llu in %.3f ms\n", (unsigned long long)c.fill_count, i.t_done_ms - i.t_submit_ms);
    gsofa_result_destroy(r); gsofa_server_destroy(srv); gsofa_destroy(ctx);
    return 0;
}
