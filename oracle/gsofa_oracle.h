/*
 * gsofa_oracle.h -- CPU oracle for the gSoFa fill-path symbolic factorization.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C (OpenMP) restatement of the
 * reference's per-source max-id label algorithm, used by the test-suite, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product library (libgsofa.so) never links or calls it.
 *
 * Reference algorithm followed (paths relative to the gSoFaTPDS project):
 *   - seeding of a source row:  gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh:842-906
 *   - relaxation / fill test:   same file :950-1001; SpaceOptimization/symbfact.cuh:989-1067
 *   - per-row U counter nz_row_U (original entries > src counted per CSR entry,
 *     fills > src counted once):  same SOA file :895-903, :985-992
 *   - supernode detection rule: same SOA file :1833-2052 (kernel launched <<<1,128>>>, :2198)
 *   - reported supernode count = detected + 1: same SOA file :3549
 *
 * Parity pin: on the reference's bundled BC matrix (n=11,948, nnz=149,090)
 * the oracle's total fill count must equal the reference's logged 980,136
 * (SpaceOptimization/with_supernodes/space_optimization_log_1_264_GPU_warp_centric.dat:2).
 */
#ifndef GSOFA_ORACLE_H
#define GSOFA_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* splitmix64 finaliser (Steele/Lea/Flood 2014), the digest mixing function.
 * A U-row digest is the sum (mod 2^64) of or_mix64((w << 32) | mask_w) over
 * the non-zero 32-column words w of the row's column set (mask_w: bit j set
 * iff column 32w + j is in the set); an L-row digest is the sum of
 * or_mix64(column id) over the set. */
uint64_t or_mix64(uint64_t x);

/*
 * Per-source max-id label search for the rows listed in `rows` (NULL = all
 * rows 0..n-1, then nrows must be n).  Row v of A is col[beg[v] .. end[v]).
 * Every output array is indexed by position in `rows` and may be NULL.
 *
 *   nnzL[i], nnzU[i]  distinct strictly-lower / strictly-upper entries of row
 *                     rows[i] in L+U (originals + fills)
 *   nzU_ref[i]        the reference's nz_row_U counter (CSR entries > row with
 *                     multiplicity, plus fills > row)
 *   digL[i], digU[i]  digests of the L column set (per column) and of the U
 *                     column set (per 32-column word), see or_mix64
 *   fills[i]          fill entries of the row (not in A, off-diagonal)
 *   e_alg[i], v_alg[i] edges inspected / vertices expanded by an ideal search
 *                     (vertices v < row reachable through vertices < row)
 *   lback[4*i .. 4*i+3]  128-bit mask, bit j set iff column (row-1-j) is in L
 *
 * Pattern output: if Loff/Lcols (Uoff/Ucols) are non-NULL, the sorted L (U)
 * column ids of row rows[i] are written to Lcols[Loff[i] ...] (capacity is
 * the caller's responsibility: call once without them to get the counts).
 * Returns 0, or -1 on allocation failure / bad arguments.
 */
int or_rows(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
            const int32_t* rows, int64_t nrows, int nthreads,
            int32_t* nnzL, int32_t* nnzU, int32_t* nzU_ref,
            uint64_t* digL, uint64_t* digU, uint64_t* fills,
            uint64_t* e_alg, uint64_t* v_alg, uint32_t* lback,
            const int64_t* Loff, int32_t* Lcols,
            const int64_t* Uoff, int32_t* Ucols);

/*
 * Supernode detection exactly as the reference kernel does it, for all rows:
 * chunks of `mss` rows; inside a chunk a row starts a supernode when its
 * offset is a multiple of 128 (the kernel's thread 0 of a 128-thread block
 * handles those offsets) or nzU[r-1]-nzU[r] != 1; every other row is a
 * pass-through row that extends the current start f when L(r,f) != 0 and
 * otherwise counts one more supernode WITHOUT moving f.
 * nzU: the reference nz_row_U of every row; lback: 4 words per row (or_rows).
 * flags (optional, n bytes): 0 pass-through extended, 1 start, 2 split.
 * Returns the detected count (the reference prints this + 1).
 */
int64_t or_supernodes(int32_t n, const int32_t* nzU, const uint32_t* lback,
                      int32_t mss, int8_t* flags);

/* Fill-reducing ordering by level-set nested dissection of A + A^T (the
 * rule is stated in gsofa_order_oracle.c).  perm (n entries): new index k
 * holds old index perm[k].  leaf >= 1: components of at most `leaf`
 * vertices are not split; round max_rounds - 1 places every component.
 * stats (optional, 4 entries): rounds, splits, separator vertices, largest
 * separator.  Returns 0, or -1 on bad arguments / allocation failure. */
int or_order_nd(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                int32_t leaf, int32_t max_rounds, int32_t* perm, int64_t* stats);

/* The hybrid rule (gsofa_order_hybrid_oracle.c): or_order_nd with, at every
 * split, a deterministic multilevel separator computed too and the smaller
 * of the two used.  Same outputs as or_order_nd (no round cap). */
int or_order_hybrid(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                    int32_t leaf, int32_t* perm, int64_t* stats);
/* or_order_hybrid, also recording every split in trace (7 int32 per split:
 * range start, component size, |A|, |B|, |S|, rule 0 level-set / 1
 * multilevel, the level-set separator's size), at most trace_cap splits;
 * *trace_n gets the number of splits (which may exceed trace_cap). */
int or_order_hybrid_trace(int32_t n, const int32_t* beg, const int32_t* end, const int32_t* col,
                          int32_t leaf, int32_t* perm, int64_t* stats, int32_t* trace,
                          int64_t trace_cap, int64_t* trace_n);

/* Parse the reference's ASCII files (csr: "E N" then E ids; beg/end: n ids).
 * Allocates *beg,*end,*col with malloc; caller frees with or_free.
 * Returns 0 or -1. */
int or_read_dat(const char* beg_file, const char* end_file, const char* csr_file,
                int32_t* n, int64_t* nnz, int32_t** beg, int32_t** end, int32_t** col);
void or_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
