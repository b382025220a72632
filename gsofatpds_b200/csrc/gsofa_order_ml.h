// gsofa_order_ml.h -- the multilevel half of the hybrid ordering
// (gsofa_order_ml.cu), called by the nested-dissection rounds of
// gsofa_order.cu.
#pragma once

#include <cstdint>

#include "gsofa_host.h"

namespace gsofa {
namespace host {

// The structure of A + A^T: row v holds v's distinct neighbours (no v itself)
// in increasing id.
struct SymGraph {
    const int32_t* rp = nullptr;   // n + 1 row starts
    const int32_t* adj = nullptr;  // rp[n] neighbour ids
    long long E = 0;
};

// Builds the structure of A + A^T from the padded CSR of A (rp, col) and of
// A^T (trp, tcol) into memory held by S.  Synchronous on ctx->stream.
int sym_graph_build(gsofa_ctx* ctx, DeviceScratch& S, int32_t n, const int32_t* rp,
                    const int32_t* col, const int32_t* trp, const int32_t* tcol, SymGraph* out);

// The multilevel bisection of every part of one round: part[v] (device, n
// entries) is v's part in [0, R) or -1; parts with psize[k] > leaf (device,
// R entries) are bisected.  Outputs (device): per vertex of those parts,
// mside[v] (0/1) and msep[v] (1: in the separator, the boundary of the side
// with fewer boundary vertices); per part, pns[k] (separator size), pna[k]
// and pnb[k] (vertices of sides 0 and 1 outside the separator; all three 0
// for parts not bisected).  Synchronous on ctx->stream.
int ml_round(gsofa_ctx* ctx, const SymGraph& H, int32_t n, const int32_t* part, int R,
             const int32_t* psize, int32_t leaf, int32_t* mside, int32_t* msep, int32_t* pns,
             int32_t* pna, int32_t* pnb);

}  // namespace host
}  // namespace gsofa
