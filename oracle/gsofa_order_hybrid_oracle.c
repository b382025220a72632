/*
 * gsofa_order_hybrid_oracle.c -- CPU oracle of the hybrid nested-dissection
 * rule (TEST INFRASTRUCTURE ONLY: the checker of gsofa_order_hybrid, whose
 * device implementation is gsofatpds_b200/csrc/gsofa_order.cu and
 * gsofa_order_ml.cu; libgsofa.so never links or calls this file).
 *
 * The hybrid rule is or_order_nd's (gsofa_order_oracle.c) with one change at
 * each split: a second, multilevel separator is computed for the component,
 * and the smaller of the two is used (ties: the level-set one).  Every step
 * is fixed so that a parallel implementation can reproduce it exactly:
 *
 *   graph      the component's subgraph of A + A^T: distinct neighbours,
 *              sorted by id, unit edge and vertex weights; local ids follow
 *              increasing global id.
 *   coarsen    while the graph has more than 200 vertices: three rounds of
 *              mutual proposals (every unmatched vertex proposes to its
 *              unmatched neighbour of largest edge weight, ties the largest
 *              id; a pair matches when its two proposals meet); coarse ids
 *              in increasing order of each pair's smaller member; edge and
 *              vertex weights summed, neighbours sorted by coarse id.  Stop
 *              when a level keeps more than 95 % of its vertices.
 *   bisect     the coarsest graph by BFS growth: from the last vertex of a
 *              BFS started at the last vertex of a BFS from vertex 0,
 *              vertices join side 0 in BFS order (neighbours in id order)
 *              until it holds half the weight; an exhausted search goes on
 *              from the smallest vertex not yet queued.
 *   refine     at every level (the coarsest included, then after each
 *              projection): up to 10 passes; gain = (edge weight to the
 *              other side) - (to its own side); a vertex with positive gain
 *              larger than every neighbour's (ties: the smaller id wins) is
 *              a candidate; candidates are taken in increasing id, each
 *              moved only if side 0's weight stays within 40..60 % of the
 *              total (the others are skipped).
 *   separator  the boundary vertices (with a neighbour on the other side) of
 *              the side that has fewer of them (ties: side 0); A = side 0
 *              minus S, B = side 1 minus S.
 * The component's range is laid out [A | B | S] as in or_order_nd; a split
 * that leaves A or B empty keeps the level-set split.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gsofa_oracle.h"

typedef struct {
    int n;
    int64_t* ptr;
    int* adj;
    int* ew;
    int* vw;
} hg;

static void hg_free(hg* g) {
    free(g->ptr);
    free(g->adj);
    free(g->ew);
    free(g->vw);
}

static int cmp_i(const void* a, const void* b) {
    const int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* sort each row's (neighbour, weight) pairs by neighbour id */
static void sort_rows(hg* g) {
    for (int v = 0; v < g->n; v++) {
        const int64_t b = g->ptr[v], e = g->ptr[v + 1];
        for (int64_t i = b + 1; i < e; i++) {  /* insertion sort: rows are short */
            const int a = g->adj[i], w = g->ew[i];
            int64_t j = i - 1;
            while (j >= b && g->adj[j] > a) {
                g->adj[j + 1] = g->adj[j];
                g->ew[j + 1] = g->ew[j];
                j--;
            }
            g->adj[j + 1] = a;
            g->ew[j + 1] = w;
        }
    }
}

/* BFS levels of g from src; d[v] (-1 unreached); returns eccentricity and
 * the number reached; q receives the visit order */
static int hg_bfs(const hg* g, int src, int* d, int* q, int* reached) {
    for (int v = 0; v < g->n; v++) d[v] = -1;
    int h = 0, t = 0, e = 0;
    d[src] = 0;
    q[t++] = src;
    while (h < t) {
        const int u = q[h++];
        if (d[u] > e) e = d[u];
        for (int64_t j = g->ptr[u]; j < g->ptr[u + 1]; j++)
            if (d[g->adj[j]] < 0) {
                d[g->adj[j]] = d[u] + 1;
                q[t++] = g->adj[j];
            }
    }
    *reached = t;
    return e;
}

/* or_order_nd's split on g (connected or not), from its vertex 0:
 * cls 0 = A, 1 = B, 2 = S.  Returns |S|, or -1 when no split exists. */
static int hg_levelset(const hg* g, int* cls) {
    const int n = g->n;
    int* d = malloc(sizeof(int) * n);
    int* q = malloc(sizeof(int) * n);
    int reached = 0;
    const int e1 = hg_bfs(g, 0, d, q, &reached);
    int r1 = n;
    for (int i = 0; i < reached; i++)
        if (d[q[i]] == e1 && q[i] < r1) r1 = q[i];
    const int e = hg_bfs(g, r1, d, q, &reached);
    if (e < 1) {
        free(d);
        free(q);
        return -1;
    }
    int* cnt = calloc((size_t)e + 2, sizeof(int));
    for (int i = 0; i < reached; i++) cnt[d[q[i]]]++;
    int m = 0;
    int64_t cum = 0;
    for (m = 0; m <= e; m++) {
        cum += cnt[m];
        if (2 * cum >= reached) break;
    }
    if (m > e - 1) m = e - 1;
    int ns = 0;
    for (int v = 0; v < n; v++) {
        if (d[v] < 0 || d[v] > m) {
            cls[v] = 1;
        } else if (d[v] < m) {
            cls[v] = 0;
        } else {
            int sep = 0;
            for (int64_t j = g->ptr[v]; j < g->ptr[v + 1] && !sep; j++) sep = d[g->adj[j]] == m + 1;
            cls[v] = sep ? 2 : 0;
            ns += sep;
        }
    }
    free(d);
    free(q);
    free(cnt);
    return ns;
}

/* one coarsening level; returns 0 when the level keeps > 95 % */
static int hg_coarsen(const hg* g, hg* c, int* cmap) {
    const int n = g->n;
    int* match = malloc(sizeof(int) * n);
    int* prop = malloc(sizeof(int) * n);
    for (int v = 0; v < n; v++) match[v] = -1;
    for (int round = 0; round < 3; round++) {
        for (int v = 0; v < n; v++) {
            prop[v] = -1;
            if (match[v] >= 0) continue;
            int best = -1, bw = -1;
            for (int64_t j = g->ptr[v]; j < g->ptr[v + 1]; j++) {
                const int w = g->adj[j];
                if (match[w] >= 0) continue;
                if (g->ew[j] > bw || (g->ew[j] == bw && w > best)) {
                    bw = g->ew[j];
                    best = w;
                }
            }
            prop[v] = best;
        }
        for (int v = 0; v < n; v++)
            if (prop[v] > v && prop[prop[v]] == v) {
                match[v] = prop[v];
                match[prop[v]] = v;
            }
    }
    int nc = 0;
    for (int v = 0; v < n; v++) {
        if (match[v] >= 0 && match[v] < v) continue;
        cmap[v] = nc;
        if (match[v] > v) cmap[match[v]] = nc;
        nc++;
    }
    free(prop);
    if ((int64_t)nc * 100 > (int64_t)n * 95) {
        free(match);
        return 0;
    }
    c->n = nc;
    c->ptr = calloc((size_t)nc + 1, sizeof(int64_t));
    c->vw = calloc((size_t)nc, sizeof(int));
    c->adj = malloc(sizeof(int) * (size_t)(g->ptr[n] + 1));
    c->ew = malloc(sizeof(int) * (size_t)(g->ptr[n] + 1));
    int* mark = malloc(sizeof(int) * nc);
    int* pos = malloc(sizeof(int) * nc);
    for (int i = 0; i < nc; i++) mark[i] = -1;
    int64_t m = 0;
    for (int v = 0; v < n; v++) {  /* coarse vertices in increasing order */
        if (match[v] >= 0 && match[v] < v) continue;
        const int cv = cmap[v];
        c->ptr[cv] = m;
        for (int s = 0; s < 2; s++) {
            const int u = s == 0 ? v : (match[v] > v ? match[v] : -1);
            if (u < 0) continue;
            c->vw[cv] += g->vw[u];
            for (int64_t j = g->ptr[u]; j < g->ptr[u + 1]; j++) {
                const int cw = cmap[g->adj[j]];
                if (cw == cv) continue;
                if (mark[cw] != cv) {
                    mark[cw] = cv;
                    pos[cw] = (int)m;
                    c->adj[m] = cw;
                    c->ew[m] = g->ew[j];
                    m++;
                } else {
                    c->ew[pos[cw]] += g->ew[j];
                }
            }
        }
    }
    c->ptr[nc] = m;
    sort_rows(c);
    free(match);
    free(mark);
    free(pos);
    return 1;
}

static void hg_refine(const hg* g, int* side) {
    const int n = g->n;
    int64_t total = 0, w0 = 0;
    for (int v = 0; v < n; v++) {
        total += g->vw[v];
        if (!side[v]) w0 += g->vw[v];
    }
    int64_t* gain = malloc(sizeof(int64_t) * (size_t)n);
    for (int pass = 0; pass < 10; pass++) {
        for (int v = 0; v < n; v++) {
            int64_t in = 0, out = 0;
            for (int64_t j = g->ptr[v]; j < g->ptr[v + 1]; j++) {
                if (side[g->adj[j]] == side[v]) in += g->ew[j];
                else out += g->ew[j];
            }
            gain[v] = out - in;
        }
        int moved = 0;
        for (int v = 0; v < n; v++) {
            if (gain[v] <= 0) continue;
            int best = 1;
            for (int64_t j = g->ptr[v]; j < g->ptr[v + 1] && best; j++) {
                const int w = g->adj[j];
                if (gain[w] > gain[v] || (gain[w] == gain[v] && w < v)) best = 0;
            }
            if (!best) continue;
            const int64_t nw0 = side[v] ? w0 + g->vw[v] : w0 - g->vw[v];
            if (nw0 * 100 < total * 40 || nw0 * 100 > total * 60) continue;
            side[v] ^= 1;
            w0 = nw0;
            moved++;
        }
        if (!moved) break;
    }
    free(gain);
}

/* multilevel bisection of g into side[] */
static void hg_bisect(const hg* g, int* side) {
    hg c;
    int* cmap = malloc(sizeof(int) * (size_t)g->n);
    if (g->n > 200 && hg_coarsen(g, &c, cmap)) {
        int* cs = malloc(sizeof(int) * (size_t)c.n);
        hg_bisect(&c, cs);
        for (int v = 0; v < g->n; v++) side[v] = cs[cmap[v]];
        free(cs);
        hg_free(&c);
    } else {
        /* BFS growth to half the weight from a pseudo-peripheral vertex (the
         * last of a BFS from the last of a BFS from vertex 0); an exhausted
         * search continues from the smallest unvisited vertex */
        const int n = g->n;
        int* d = malloc(sizeof(int) * (size_t)n);
        int* q = malloc(sizeof(int) * (size_t)n);
        int reached = 0, start = 0;
        for (int rep = 0; rep < 2; rep++) {
            hg_bfs(g, start, d, q, &reached);
            start = q[reached - 1];
        }
        int64_t total = 0, got = 0;
        for (int v = 0; v < n; v++) {
            total += g->vw[v];
            side[v] = 1;
            d[v] = 0;  /* reused as "queued" */
        }
        int h = 0, t = 0, next = 0;
        q[t++] = start;
        d[start] = 1;
        while (got * 2 < total) {
            if (h == t) {
                while (next < n && d[next]) next++;
                if (next == n) break;
                q[t++] = next;
                d[next] = 1;
            }
            const int u = q[h++];
            side[u] = 0;
            got += g->vw[u];
            for (int64_t j = g->ptr[u]; j < g->ptr[u + 1]; j++)
                if (!d[g->adj[j]]) {
                    d[g->adj[j]] = 1;
                    q[t++] = g->adj[j];
                }
        }
        free(d);
        free(q);
    }
    free(cmap);
    hg_refine(g, side);
}

/* ---- the ordering --------------------------------------------------------- */

typedef struct {
    int64_t* ptr;
    int* adj;
    int32_t n;
    int32_t leaf;
    int32_t* perm;
    int* loc;   /* local ids inside split(), -1 elsewhere */
    int* mark;  /* component walk of solve() */
    int64_t stats[4];
    int32_t* trace;  /* or_order_hybrid_trace: kTraceFields per split, or NULL */
    int64_t trace_cap, trace_n;
} hctx;

/* one split as traced: range start, component size, |A|, |B|, |S|, rule
 * (0 level-set, 1 multilevel), and the level-set separator's size */
enum { kTraceFields = 7 };

static void place(hctx* H, int* vs, int k, int lo) {
    qsort(vs, (size_t)k, sizeof(int), cmp_i);
    for (int i = 0; i < k; i++) H->perm[lo + i] = vs[i];
}

static void solve(hctx* H, int* vs, int k, int lo, int depth);

/* split one connected component (vs sorted ascending) */
static void split(hctx* H, int* vs, int k, int lo, int depth) {
    hg g;
    g.n = k;
    g.ptr = malloc(sizeof(int64_t) * ((size_t)k + 1));
    for (int i = 0; i < k; i++) H->loc[vs[i]] = i;
    int64_t m = 0;
    g.ptr[0] = 0;
    for (int i = 0; i < k; i++) {
        for (int64_t j = H->ptr[vs[i]]; j < H->ptr[vs[i] + 1]; j++)
            if (H->loc[H->adj[j]] >= 0) m++;
        g.ptr[i + 1] = m;
    }
    g.adj = malloc(sizeof(int) * (size_t)(m + 1));
    g.ew = malloc(sizeof(int) * (size_t)(m + 1));
    g.vw = malloc(sizeof(int) * (size_t)k);
    m = 0;
    for (int i = 0; i < k; i++) {
        g.vw[i] = 1;
        for (int64_t j = H->ptr[vs[i]]; j < H->ptr[vs[i] + 1]; j++) {
            const int l = H->loc[H->adj[j]];
            if (l >= 0) {
                g.adj[m] = l;
                g.ew[m] = 1;
                m++;
            }
        }
    }
    for (int i = 0; i < k; i++) H->loc[vs[i]] = -1;
    /* the global adjacency is sorted and distinct, so local rows are too */
    int* cls = malloc(sizeof(int) * (size_t)k);
    int nls = hg_levelset(&g, cls);
    const int nls_levelset = nls;
    int ml_won = 0;
    int* side = malloc(sizeof(int) * (size_t)k);
    hg_bisect(&g, side);
    int bnd[2] = {0, 0};
    int* isb = calloc((size_t)k, sizeof(int));
    for (int v = 0; v < k; v++)
        for (int64_t j = g.ptr[v]; j < g.ptr[v + 1]; j++)
            if (side[g.adj[j]] != side[v]) {
                isb[v] = 1;
                bnd[side[v]]++;
                break;
            }
    const int small = bnd[0] <= bnd[1] ? 0 : 1;
    int nml = bnd[small], na_ml = 0, nb_ml = 0;
    for (int v = 0; v < k; v++) {
        if (isb[v] && side[v] == small) continue;
        if (side[v] == 0) na_ml++;
        else nb_ml++;
    }
    if (nml < nls && na_ml > 0 && nb_ml > 0) {
        for (int v = 0; v < k; v++) cls[v] = (isb[v] && side[v] == small) ? 2 : side[v];
        nls = nml;
        ml_won = 1;
    }
    int* A = malloc(sizeof(int) * (size_t)k);
    int* B = malloc(sizeof(int) * (size_t)k);
    int* S = malloc(sizeof(int) * (size_t)k);
    int na = 0, nb = 0, ns = 0;
    for (int v = 0; v < k; v++) {
        if (cls[v] == 2) S[ns++] = vs[v];
        else if (cls[v] == 0) A[na++] = vs[v];
        else B[nb++] = vs[v];
    }
    hg_free(&g);
    free(cls);
    free(side);
    free(isb);
    H->stats[1]++;
    H->stats[2] += ns;
    if (ns > H->stats[3]) H->stats[3] = ns;
    if (H->trace && H->trace_n < H->trace_cap) {
        int32_t* t = H->trace + kTraceFields * H->trace_n;
        t[0] = lo;
        t[1] = k;
        t[2] = na;
        t[3] = nb;
        t[4] = ns;
        t[5] = ml_won;
        t[6] = nls_levelset;
    }
    if (H->trace) H->trace_n++;
    place(H, S, ns, lo + k - ns);
    if (na) solve(H, A, na, lo, depth + 1);
    if (nb) solve(H, B, nb, lo + na, depth + 1);
    free(A);
    free(B);
    free(S);
}

/* components of vs (in root order), each placed or split.  mark: 1 = member
 * not yet visited, 2 = visited, 0 = not a member (a child call only marks
 * vertices its parent has already visited, so the parent's scan is safe). */
static void solve(hctx* H, int* vs, int k, int lo, int depth) {
    if (depth + 1 > H->stats[0]) H->stats[0] = depth + 1;
    qsort(vs, (size_t)k, sizeof(int), cmp_i);
    for (int i = 0; i < k; i++) H->mark[vs[i]] = 1;
    int* comp = malloc(sizeof(int) * (size_t)k);
    int off = lo;
    for (int r = 0; r < k; r++) {
        if (H->mark[vs[r]] != 1) continue;
        int h = 0, t = 0;
        comp[t++] = vs[r];
        H->mark[vs[r]] = 2;
        while (h < t) {
            const int u = comp[h++];
            for (int64_t j = H->ptr[u]; j < H->ptr[u + 1]; j++)
                if (H->mark[H->adj[j]] == 1) {
                    H->mark[H->adj[j]] = 2;
                    comp[t++] = H->adj[j];
                }
        }
        int* c = malloc(sizeof(int) * (size_t)t);
        memcpy(c, comp, sizeof(int) * (size_t)t);
        qsort(c, (size_t)t, sizeof(int), cmp_i);
        if (t <= H->leaf) place(H, c, t, off);
        else split(H, c, t, off, depth);
        off += t;
        free(c);
    }
    for (int i = 0; i < k; i++) H->mark[vs[i]] = 0;
    free(comp);
}

static int order_hybrid(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                        int32_t leaf, int32_t* perm, int64_t* stats, int32_t* trace,
                        int64_t trace_cap, int64_t* trace_n) {
    if (n < 0 || leaf < 1 || (n > 0 && (!beg || !end || !perm))) return -1;
    if (stats) memset(stats, 0, 4 * sizeof(int64_t));
    if (n == 0) return 0;
    /* A + A^T, distinct neighbours sorted by id */
    int64_t* ptr = calloc((size_t)n + 1, sizeof(int64_t));
    for (int32_t v = 0; v < n; v++)
        for (int64_t j = beg[v]; j < end[v]; j++) {
            if (col[j] < 0 || col[j] >= n) { free(ptr); return -1; }
            if (col[j] != v) { ptr[v + 1]++; ptr[col[j] + 1]++; }
        }
    for (int32_t v = 0; v < n; v++) ptr[v + 1] += ptr[v];
    int* adj = malloc(sizeof(int) * (size_t)(ptr[n] + 1));
    int64_t* fill = malloc(sizeof(int64_t) * ((size_t)n + 1));
    memcpy(fill, ptr, sizeof(int64_t) * ((size_t)n + 1));
    for (int32_t v = 0; v < n; v++)
        for (int64_t j = beg[v]; j < end[v]; j++)
            if (col[j] != v) {
                adj[fill[v]++] = col[j];
                adj[fill[col[j]]++] = v;
            }
    int64_t w = 0;  /* sort and deduplicate rows, compacting in place */
    for (int32_t v = 0; v < n; v++) {
        const int64_t b = ptr[v], e = ptr[v + 1];
        qsort(adj + b, (size_t)(e - b), sizeof(int), cmp_i);
        ptr[v] = w;
        for (int64_t j = b; j < e; j++)
            if (j == b || adj[j] != adj[j - 1]) adj[w++] = adj[j];
    }
    ptr[n] = w;
    free(fill);
    hctx H;
    H.ptr = ptr;
    H.adj = adj;
    H.n = n;
    H.leaf = leaf;
    H.perm = perm;
    H.loc = malloc(sizeof(int) * (size_t)n);
    H.mark = calloc((size_t)n, sizeof(int));
    memset(H.stats, 0, sizeof(H.stats));
    H.trace = trace;
    H.trace_cap = trace_cap;
    H.trace_n = 0;
    for (int32_t v = 0; v < n; v++) H.loc[v] = -1;
    int* all = malloc(sizeof(int) * (size_t)n);
    for (int32_t v = 0; v < n; v++) all[v] = v;
    solve(&H, all, n, 0, 0);
    if (stats) memcpy(stats, H.stats, sizeof(H.stats));
    if (trace_n) *trace_n = H.trace_n;
    free(all);
    free(H.loc);
    free(H.mark);
    free(ptr);
    free(adj);
    return 0;
}

int or_order_hybrid(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                    int32_t leaf, int32_t* perm, int64_t* stats) {
    return order_hybrid(n, beg, end, col, leaf, perm, stats, NULL, 0, NULL);
}

int or_order_hybrid_trace(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                          int32_t leaf, int32_t* perm, int64_t* stats, int32_t* trace,
                          int64_t trace_cap, int64_t* trace_n) {
    if (trace_cap < 0 || (trace_cap > 0 && !trace) || !trace_n) return -1;
    return order_hybrid(n, beg, end, col, leaf, perm, stats, trace, trace_cap, trace_n);
}
