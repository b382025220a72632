/*
 * gsofa_oracle.c -- CPU oracle (test infrastructure only; see gsofa_oracle.h).
 *
 * Per source row s the reference keeps a max-id label per vertex
 * (cost_array_d, SOA symbfact_warp_centric_new_scheduling.cuh:842-1001):
 *   - seeding (:842-906): label[s] = offset, and every column w of row s gets
 *     label[w] = offset (no intermediate vertex), w < s is queued;
 *   - relaxation (:950-1001): expanding a queued vertex v passes
 *     cost = max(v, label[v]) to every column m of row v; a smaller cost
 *     lowers label[m] (atomicMin) and re-queues m when m < s;
 *   - a column m becomes an entry of row s when its final label says every
 *     intermediate vertex is < m (for m > s that holds for any reached m).
 * The reference's label-correcting queue reaches the unique minimal labels in
 * any order; here the same labels are computed with a monotone bucket queue
 * (keys = cost values 1..s), which expands every reachable vertex once.
 *
 * Label encoding used here: 0 = reached directly from s, k+1 = the largest
 * intermediate vertex id on the best path is k, UINT32_MAX = unreached.
 */
#include "gsofa_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <ctype.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_INF 0xFFFFFFFFu

uint64_t or_mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

typedef struct {
    uint32_t* lab;     /* n labels, OR_INF when untouched */
    uint8_t* done;     /* n expanded flags */
    int32_t* bhead;    /* n+2 bucket heads, -1 = empty */
    int32_t* touched;  /* list of vertices whose label was set */
    int64_t ntouched;
    int32_t* pv;       /* bucket pool: vertex */
    int32_t* pnext;    /* bucket pool: next index */
    int64_t pcap, plen;
    int32_t* tmp;      /* sort scratch for pattern output */
    uint32_t* wmask;   /* (n+31)/32 word masks of the U column set, kept zero */
    int32_t* wlist;    /* words with a non-zero mask */
} or_ws;

static int ws_init(or_ws* w, int32_t n) {
    memset(w, 0, sizeof(*w));
    w->lab = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n + 1));
    w->done = (uint8_t*)calloc((size_t)n + 1, 1);
    w->bhead = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 2));
    w->touched = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    w->tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    w->wmask = (uint32_t*)calloc((size_t)n / 32 + 2, sizeof(uint32_t));
    w->wlist = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n / 32 + 2));
    w->pcap = 1024;
    w->pv = (int32_t*)malloc(sizeof(int32_t) * (size_t)w->pcap);
    w->pnext = (int32_t*)malloc(sizeof(int32_t) * (size_t)w->pcap);
    if (!w->lab || !w->done || !w->bhead || !w->touched || !w->tmp || !w->pv || !w->pnext ||
        !w->wmask || !w->wlist)
        return -1;
    for (int64_t i = 0; i <= n; i++) w->lab[i] = OR_INF;
    for (int64_t i = 0; i < (int64_t)n + 2; i++) w->bhead[i] = -1;
    return 0;
}

static void ws_free(or_ws* w) {
    free(w->lab); free(w->done); free(w->bhead); free(w->touched);
    free(w->tmp); free(w->pv); free(w->pnext); free(w->wmask); free(w->wlist);
}

static int push(or_ws* w, int32_t v, uint32_t key) {
    if (w->plen == w->pcap) {
        int64_t nc = w->pcap * 2;
        int32_t* a = (int32_t*)realloc(w->pv, sizeof(int32_t) * (size_t)nc);
        if (!a) return -1;
        w->pv = a;
        int32_t* b = (int32_t*)realloc(w->pnext, sizeof(int32_t) * (size_t)nc);
        if (!b) return -1;
        w->pnext = b;
        w->pcap = nc;
    }
    int64_t e = w->plen++;
    w->pv[e] = v;
    w->pnext[e] = w->bhead[key];
    w->bhead[key] = (int32_t)e;
    return 0;
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* One source row s.  Returns 0 or -1 (allocation failure). */
static int one_row(or_ws* w, int32_t n, const int32_t* beg, const int32_t* end,
                   const int32_t* col, int32_t s, int64_t i,
                   int32_t* nnzL, int32_t* nnzU, int32_t* nzU_ref,
                   uint64_t* digL, uint64_t* digU, uint64_t* fills,
                   uint64_t* e_alg, uint64_t* v_alg, uint32_t* lback,
                   const int64_t* Loff, int32_t* Lcols,
                   const int64_t* Uoff, int32_t* Ucols) {
    (void)n;  /* the workspace was sized for n by ws_init */
    uint32_t* lab = w->lab;
    w->ntouched = 0;
    w->plen = 0;
    /* seeding (SOA :842-906): the source and every column of its row get the
     * "no intermediate" label; columns < s are queued with key w+1. */
    lab[s] = 0;
    w->touched[w->ntouched++] = s;
    int64_t rawU = 0, origU = 0, origL = 0;
    for (int64_t k = beg[s]; k < end[s]; k++) {
        int32_t c = col[k];
        if (c == s) continue;
        if (c > s) rawU++;
        if (lab[c] == OR_INF) {
            w->touched[w->ntouched++] = c;
            if (c > s) origU++; else origL++;
        }
        if (lab[c] != 0) {
            lab[c] = 0;
            if (c < s && push(w, c, (uint32_t)c + 1)) return -1;
        }
    }
    /* relaxation in increasing cost order (SOA :950-1001). */
    uint64_t E = 0, V = 0;
    for (uint32_t key = 1; key <= (uint32_t)s; key++) {
        /* entries pushed into `key` while it is scanned are consumed here too */
        while (w->bhead[key] >= 0) {
            int32_t e = w->bhead[key];
            w->bhead[key] = w->pnext[e];
            int32_t v = w->pv[e];
            if (w->done[v]) continue;
            uint32_t kv = lab[v] > (uint32_t)v + 1 ? lab[v] : (uint32_t)v + 1;
            if (kv != key) continue; /* stale entry */
            w->done[v] = 1;
            V++;
            E += (uint64_t)(end[v] - beg[v]);
            for (int64_t k = beg[v]; k < end[v]; k++) {
                int32_t m = col[k];
                if (key < lab[m]) {
                    if (lab[m] == OR_INF) w->touched[w->ntouched++] = m;
                    lab[m] = key;
                    if (m < s && !w->done[m]) {
                        /* cost passed on never decreases: m's key is >= key */
                        uint32_t km = key > (uint32_t)m + 1 ? key : (uint32_t)m + 1;
                        if (push(w, m, km)) return -1;
                    }
                }
            }
        }
    }
    /* collect results from the final labels */
    int64_t cL = 0, cU = 0, nwl = 0;
    uint64_t dL = 0, dU = 0;
    uint32_t lb[4] = {0, 0, 0, 0};
    for (int64_t t = 0; t < w->ntouched; t++) {
        int32_t v = w->touched[t];
        if (v == s) continue;
        if (v < s) {
            if (lab[v] <= (uint32_t)v) {
                cL++;
                dL += or_mix64((uint64_t)v);
                int32_t j = s - 1 - v;
                if (j < 128) lb[j >> 5] |= 1u << (j & 31);
            }
        } else {
            cU++;
            uint32_t* m = &w->wmask[v >> 5];
            if (!*m) w->wlist[nwl++] = v >> 5;
            *m |= 1u << (v & 31);
        }
    }
    /* U digest: one term per non-zero 32-column word (word index, mask) */
    for (int64_t k = 0; k < nwl; k++) {
        const int32_t wd = w->wlist[k];
        dU += or_mix64(((uint64_t)(uint32_t)wd << 32) | w->wmask[wd]);
        w->wmask[wd] = 0;
    }
    if (nnzL) nnzL[i] = (int32_t)cL;
    if (nnzU) nnzU[i] = (int32_t)cU;
    if (nzU_ref) nzU_ref[i] = (int32_t)(rawU + (cU - origU));
    if (digL) digL[i] = dL;
    if (digU) digU[i] = dU;
    if (fills) fills[i] = (uint64_t)((cL - origL) + (cU - origU));
    if (e_alg) e_alg[i] = E;
    if (v_alg) v_alg[i] = V;
    if (lback) memcpy(lback + 4 * i, lb, sizeof(lb));
    if ((Loff && Lcols) || (Uoff && Ucols)) {
        int64_t nl = 0, nu = 0;
        for (int64_t t = 0; t < w->ntouched; t++) {
            int32_t v = w->touched[t];
            if (v < s && lab[v] <= (uint32_t)v) w->tmp[nl++] = v;
        }
        qsort(w->tmp, (size_t)nl, sizeof(int32_t), cmp_i32);
        if (Loff && Lcols) memcpy(Lcols + Loff[i], w->tmp, sizeof(int32_t) * (size_t)nl);
        for (int64_t t = 0; t < w->ntouched; t++) {
            int32_t v = w->touched[t];
            if (v > s) w->tmp[nu++] = v;
        }
        qsort(w->tmp, (size_t)nu, sizeof(int32_t), cmp_i32);
        if (Uoff && Ucols) memcpy(Ucols + Uoff[i], w->tmp, sizeof(int32_t) * (size_t)nu);
    }
    /* reset the touched state */
    for (int64_t t = 0; t < w->ntouched; t++) {
        int32_t v = w->touched[t];
        lab[v] = OR_INF;
        w->done[v] = 0;
    }
    return 0;
}

int or_rows(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
            const int32_t* rows, int64_t nrows, int nthreads,
            int32_t* nnzL, int32_t* nnzU, int32_t* nzU_ref,
            uint64_t* digL, uint64_t* digU, uint64_t* fills,
            uint64_t* e_alg, uint64_t* v_alg, uint32_t* lback,
            const int64_t* Loff, int32_t* Lcols,
            const int64_t* Uoff, int32_t* Ucols) {
    if (n < 0 || nrows < 0 || (!rows && nrows != n)) return -1;
    for (int32_t v = 0; v < n; v++) {
        if (beg[v] > end[v]) return -1;
        for (int64_t k = beg[v]; k < end[v]; k++)
            if (col[k] < 0 || col[k] >= n) return -1;
    }
    if (rows)
        for (int64_t i = 0; i < nrows; i++)
            if (rows[i] < 0 || rows[i] >= n) return -1;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(| : err)
#endif
    {
        or_ws w;
        if (ws_init(&w, n)) {
            err = 1;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t i = 0; i < nrows; i++) {
                int32_t s = rows ? rows[i] : (int32_t)i;
                if (one_row(&w, n, beg, end, col, s, i, nnzL, nnzU, nzU_ref, digL, digU,
                            fills, e_alg, v_alg, lback, Loff, Lcols, Uoff, Ucols))
                    err = 1;
            }
        }
        ws_free(&w);
    }
    (void)nthreads;
    return err ? -1 : 0;
}

/* Supernodes, following the reference kernel's two phases literally
 * (SOA symbfact_warp_centric_new_scheduling.cuh:1833-1950 phase 1,
 * :1959-2111 phase 2). */
int64_t or_supernodes(int32_t n, const int32_t* nzU, const uint32_t* lback,
                      int32_t mss, int8_t* flags) {
    if (mss <= 0 || n < 0) return -1;
    int64_t nsup = 0;
    int64_t nchunks = ((int64_t)n + mss - 1) / mss;
    int32_t* starts = (int32_t*)malloc(sizeof(int32_t) * (size_t)mss);
    uint8_t* pass = (uint8_t*)calloc((size_t)mss + 1, 1);
    if (!starts || !pass) { free(starts); free(pass); return -1; }
    for (int64_t c = 0; c < nchunks; c++) {
        int64_t first = c * mss;
        int32_t ns = 0;
        memset(pass, 0, (size_t)mss + 1);
        /* phase 1: the block's thread t handles offsets t, t+128, ...; thread 0
         * always records a start; others compare adjacent nz_row_U counts. */
        for (int32_t j = 0; j < mss; j++) {
            int64_t src = first + j;
            if (src >= n) break;
            if (j % 128 == 0) {
                starts[ns++] = (int32_t)src;
            } else if (nzU[src - 1] - nzU[src] != 1) {
                starts[ns++] = (int32_t)src;
            } else {
                pass[j] = 1;
            }
        }
        /* phase 2: one walk per start; the first row of the supernode never
         * moves, a failed L(r,f) test only adds a supernode (:2043-2052). */
        for (int32_t t = 0; t < ns; t++) {
            int32_t f = starts[t];
            nsup++;
            if (flags) flags[f] = 1;
            int64_t r = (int64_t)f + 1;
            while (r < n && (r - first) < mss && pass[r - first]) {
                int32_t j = (int32_t)(r - 1 - f);
                int in_l = j < 128 && ((lback[4 * r + (j >> 5)] >> (j & 31)) & 1u);
                if (!in_l) nsup++;
                if (flags) flags[r] = in_l ? 0 : 2;
                r++;
            }
        }
    }
    free(starts);
    free(pass);
    return nsup;
}

/* ---- ASCII reader (same file layout the reference reads, SOA :2567-2616) -- */
static int read_ints(FILE* f, int64_t count, int32_t* out, int64_t* got) {
    int64_t i = 0;
    int c = fgetc(f);
    while (i < count) {
        while (c != EOF && isspace(c)) c = fgetc(f);
        if (c == EOF) break;
        int neg = 0;
        if (c == '-') { neg = 1; c = fgetc(f); }
        if (!isdigit(c)) return -1;
        int64_t v = 0;
        while (c != EOF && isdigit(c)) { v = v * 10 + (c - '0'); c = fgetc(f); }
        out[i++] = (int32_t)(neg ? -v : v);
    }
    *got = i;
    return 0;
}

int or_read_dat(const char* beg_file, const char* end_file, const char* csr_file,
                int32_t* n_out, int64_t* nnz_out, int32_t** beg, int32_t** end, int32_t** col) {
    FILE* f = fopen(csr_file, "r");
    if (!f) return -1;
    int32_t hdr[2];
    int64_t got = 0;
    if (read_ints(f, 2, hdr, &got) || got != 2 || hdr[0] < 0 || hdr[1] < 0) { fclose(f); return -1; }
    int64_t E = hdr[0];
    int32_t n = hdr[1];
    /* the header was consumed with one byte of lookahead: rewind and skip it */
    rewind(f);
    int32_t* c = (int32_t*)malloc(sizeof(int32_t) * (size_t)(E + 2));
    if (!c) { fclose(f); return -1; }
    if (read_ints(f, E + 2, c, &got) || got != E + 2) { free(c); fclose(f); return -1; }
    fclose(f);
    memmove(c, c + 2, sizeof(int32_t) * (size_t)E);
    int32_t* b = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t* e = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    if (!b || !e) { free(c); free(b); free(e); return -1; }
    f = fopen(beg_file, "r");
    if (!f || read_ints(f, n, b, &got) || got != n) { if (f) fclose(f); free(c); free(b); free(e); return -1; }
    fclose(f);
    f = fopen(end_file, "r");
    if (!f || read_ints(f, n, e, &got) || got != n) { if (f) fclose(f); free(c); free(b); free(e); return -1; }
    fclose(f);
    *n_out = n;
    *nnz_out = E;
    *beg = b;
    *end = e;
    *col = c;
    return 0;
}

void or_free(void* p) { free(p); }
