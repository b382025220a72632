/*
 * gsofa_order_oracle.c -- CPU oracle of the fill-reducing ordering
 * (TEST INFRASTRUCTURE ONLY: the test-suite and bench.py's CPU-baseline leg
 * call it as the checker; libgsofa.so never links or calls it).
 *
 * The reference has no ordering code: its inputs arrive already permuted by
 * SuperLU_DIST (gSoFaTPDS README.md:27-33), which is not part of the
 * project.  The ordering restated here is the published level-set nested
 * dissection (A. George, "Nested dissection of a regular finite element
 * mesh", SIAM J. Numer. Anal. 10, 1973; A. George and J. W. H. Liu,
 * "Computer Solution of Large Sparse Positive Definite Systems", 1981,
 * ch. 8: pseudo-peripheral root, middle level of the rooted level structure
 * as separator, trimmed to the vertices adjacent to the next level), made
 * deterministic so that the device implementation must match it exactly:
 *
 * Graph: vertices 0..n-1, an edge {u, w} (u != w) wherever A(u,w) or A(w,u)
 * is stored.  Every vertex is either placed in a group (a range of final
 * positions, its members in increasing id order) or active in a part (a set
 * with a range start lo).  Initially one part holds every vertex, lo = 0.
 * Round r = 0, 1, ... while a vertex is active:
 *   1. every part splits into the connected components of the subgraph it
 *      induces; component c has root min(c), and the components of a part
 *      take consecutive ranges from the part's lo in increasing root order;
 *   2. a component with |c| <= leaf (or any component in round
 *      max_rounds - 1) is placed as a group at its range start;
 *   3. every other component c:
 *      a. BFS inside c from min(c); r1 = the smallest id at the largest
 *         distance;
 *      b. BFS inside c from r1: distance d(v), eccentricity e >= 1, level
 *         sizes N_l;
 *      c. m = the smallest l with 2 (N_0 + ... + N_l) >= |c|, then
 *         m = min(m, e - 1);
 *      d. S = { v : d(v) = m and some neighbour w in c has d(w) = m + 1 },
 *         A = { d < m } + { d = m, not in S },  B = { d > m };
 *      e. S is placed as a group at lo_c + |c| - |S| (last), A becomes a
 *         part at lo_c, B a part at lo_c + |A|.
 * perm[k] is the vertex at final position k (new index k <- old perm[k]).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gsofa_oracle.h"

static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y;
}

typedef struct {
    int64_t* ptr;  /* n + 1 */
    int32_t* adj;  /* A + A^T without self loops, duplicates kept */
} sym_graph;

static int build_sym(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                     sym_graph* g) {
    g->ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    if (!g->ptr) return -1;
    int64_t total = 0;
    for (int32_t v = 0; v < n; v++)
        for (int64_t j = beg[v]; j < end[v]; j++) {
            const int32_t w = col[j];
            if (w < 0 || w >= n) return -1;
            if (w == v) continue;
            g->ptr[v + 1]++;
            g->ptr[w + 1]++;
            total += 2;
        }
    for (int32_t v = 0; v < n; v++) g->ptr[v + 1] += g->ptr[v];
    g->adj = (int32_t*)malloc((size_t)(total > 0 ? total : 1) * sizeof(int32_t));
    int64_t* fill = (int64_t*)malloc(((size_t)n + 1) * sizeof(int64_t));
    if (!g->adj || !fill) { free(fill); return -1; }
    memcpy(fill, g->ptr, ((size_t)n + 1) * sizeof(int64_t));
    for (int32_t v = 0; v < n; v++)
        for (int64_t j = beg[v]; j < end[v]; j++) {
            const int32_t w = col[j];
            if (w == v) continue;
            g->adj[fill[v]++] = w;
            g->adj[fill[w]++] = v;
        }
    free(fill);
    return 0;
}

/* BFS inside the active part `p` from `src`; returns the eccentricity and
 * leaves distances in dist (vertices of the part only) and the visit order
 * in q (its length in *qn). */
static int32_t bfs(const sym_graph* g, const int32_t* part, int32_t p, int32_t src, int32_t* dist,
                   int32_t* q, int64_t* qn) {
    int64_t head = 0, tail = 0;
    dist[src] = 0;
    q[tail++] = src;
    int32_t ecc = 0;
    while (head < tail) {
        const int32_t u = q[head++];
        const int32_t du = dist[u];
        if (du > ecc) ecc = du;
        for (int64_t j = g->ptr[u]; j < g->ptr[u + 1]; j++) {
            const int32_t w = g->adj[j];
            if (part[w] == p && dist[w] < 0) {
                dist[w] = du + 1;
                q[tail++] = w;
            }
        }
    }
    *qn = tail;
    return ecc;
}

int or_order_nd(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                int32_t leaf, int32_t max_rounds, int32_t* perm, int64_t* stats) {
    if (n < 0 || leaf < 1 || max_rounds < 1 || (n > 0 && (!beg || !end || !perm))) return -1;
    if (stats) memset(stats, 0, 4 * sizeof(int64_t));
    if (n == 0) return 0;
    sym_graph g = {0, 0};
    int rc = -1;
    int32_t *part = 0, *comp = 0, *dist = 0, *q = 0, *newpart = 0, *cnt = 0;
    int64_t *plo = 0, *plo_next = 0, *running = 0;
    uint64_t* key = 0;
    if (build_sym(n, beg, end, col, &g)) goto done;
    const size_t N = (size_t)n;
    part = (int32_t*)malloc(N * 4);
    comp = (int32_t*)malloc(N * 4);
    dist = (int32_t*)malloc(N * 4);
    q = (int32_t*)malloc(N * 4);
    newpart = (int32_t*)malloc(N * 4);
    cnt = (int32_t*)malloc((N + 1) * 4);
    plo = (int64_t*)malloc(2 * N * 8);
    plo_next = (int64_t*)malloc(2 * N * 8);
    running = (int64_t*)malloc(2 * N * 8);
    key = (uint64_t*)malloc(N * 8);
    if (!part || !comp || !dist || !q || !newpart || !cnt || !plo || !plo_next || !running || !key)
        goto done;
    for (size_t v = 0; v < N; v++) part[v] = 0;
    plo[0] = 0;
    int64_t nparts = 1, active = n;
    int64_t rounds = 0, nsep = 0, sepv = 0, sepmax = 0;
    for (int32_t r = 0; active > 0; r++) {
        rounds++;
        const int32_t leaf_eff = r == max_rounds - 1 ? INT32_MAX : leaf;
        for (int64_t p = 0; p < nparts; p++) running[p] = 0;
        for (size_t v = 0; v < N; v++) comp[v] = -1;
        int64_t next_parts = 0;
        active = 0;
        /* roots are met in increasing id order, so a part's components are
         * laid out in increasing root order */
        for (int32_t root = 0; root < n; root++) {
            if (part[root] < 0 || comp[root] >= 0) continue;
            const int32_t p = part[root];
            int64_t head = 0, tail = 0;
            comp[root] = root;
            q[tail++] = root;
            while (head < tail) {
                const int32_t u = q[head++];
                for (int64_t j = g.ptr[u]; j < g.ptr[u + 1]; j++) {
                    const int32_t w = g.adj[j];
                    if (part[w] == p && comp[w] < 0) {
                        comp[w] = root;
                        q[tail++] = w;
                    }
                }
            }
            const int64_t size = tail;
            const int64_t lo = plo[p] + running[p];
            running[p] += size;
            if (size <= leaf_eff) {
                for (int64_t i = 0; i < size; i++) key[q[i]] = ((uint64_t)lo << 32) | (uint32_t)q[i];
                for (int64_t i = 0; i < size; i++) newpart[q[i]] = -1;
                continue;
            }
            /* the component, under a private part id for its BFS */
            const int32_t cid = -2 - root;
            for (int64_t i = 0; i < size; i++) part[q[i]] = cid;
            for (int64_t i = 0; i < size; i++) dist[q[i]] = -1;
            int64_t qn = 0;
            const int32_t e1 = bfs(&g, part, cid, root, dist, q, &qn);
            int32_t r1 = INT32_MAX;
            for (int64_t i = 0; i < qn; i++)
                if (dist[q[i]] == e1 && q[i] < r1) r1 = q[i];
            for (int64_t i = 0; i < qn; i++) dist[q[i]] = -1;
            const int32_t e = bfs(&g, part, cid, r1, dist, q, &qn);
            for (int32_t l = 0; l <= e; l++) cnt[l] = 0;
            for (int64_t i = 0; i < qn; i++) cnt[dist[q[i]]]++;
            int32_t m = 0;
            int64_t cum = 0;
            for (m = 0; m <= e; m++) {
                cum += cnt[m];
                if (2 * cum >= size) break;
            }
            if (m > e - 1) m = e - 1;
            int64_t na = 0, ns = 0;
            for (int64_t i = 0; i < qn; i++) {
                const int32_t v = q[i];
                const int32_t d = dist[v];
                int sep = 0;
                if (d == m)
                    for (int64_t j = g.ptr[v]; j < g.ptr[v + 1] && !sep; j++) {
                        const int32_t w = g.adj[j];
                        sep = part[w] == cid && dist[w] == m + 1;
                    }
                if (d < m || (d == m && !sep)) na++;
                if (sep) ns++;
                /* 0: A, 1: B, -1: separator (decided before any part id changes) */
                newpart[v] = sep ? -1 : (d <= m ? 0 : 1);
            }
            const int64_t slo = lo + size - ns;
            const int64_t ida = next_parts++, idb = next_parts++;
            plo_next[ida] = lo;
            plo_next[idb] = lo + na;
            for (int64_t i = 0; i < qn; i++) {
                const int32_t v = q[i];
                if (newpart[v] < 0) {
                    key[v] = ((uint64_t)slo << 32) | (uint32_t)v;
                } else {
                    newpart[v] = newpart[v] == 0 ? (int32_t)ida : (int32_t)idb;
                    active++;
                }
            }
            nsep++;
            sepv += ns;
            if (ns > sepmax) sepmax = ns;
        }
        for (size_t v = 0; v < N; v++)
            if (part[v] != -1) part[v] = newpart[v];
        int64_t* t = plo;
        plo = plo_next;
        plo_next = t;
        nparts = next_parts;
    }
    qsort(key, N, sizeof(uint64_t), cmp_u64);
    for (size_t k = 0; k < N; k++) perm[k] = (int32_t)(uint32_t)key[k];
    if (stats) {
        stats[0] = rounds;
        stats[1] = nsep;
        stats[2] = sepv;
        stats[3] = sepmax;
    }
    rc = 0;
done:
    free(g.ptr);
    free(g.adj);
    free(part);
    free(comp);
    free(dist);
    free(q);
    free(newpart);
    free(cnt);
    free(plo);
    free(plo_next);
    free(running);
    free(key);
    return rc;
}
