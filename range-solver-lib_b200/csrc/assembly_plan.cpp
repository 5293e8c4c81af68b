// Assembly plan builder (host, C++17 + OpenMP).
//
// The reference builds its sparse pattern implicitly through
// RSparseMatrix::addValue under a critical section (src/rsolverheat.cpp:802-819,
// src/rsolverstress.cpp:1742-1771); its fluid solver precomputes the pattern
// and per-element matrix positions once (RSolverFluid::buildSparseMatrixPattern,
// src/rsolverfluid.cpp:2305-2397).  This follows the latter: the pattern of the
// free-DOF system is derived from node adjacency once, together with a map
// from every (node, adjacent tet) pair to the column offsets of the tet's
// nodes inside that node's rows.  The GPU then assembles values with one
// thread per row and no atomics.
#include "assembly_plan.h"

#include <omp.h>

#include <algorithm>
#include <cstring>

namespace rsg {

namespace {
const uint32_t kEod = 0xffffffffu;

inline int popc(uint8_t m) { return __builtin_popcount(unsigned(m)); }

// Sorted unique neighbours of node a that own at least one free component.
void neighbours(const AsmPlanHost &P, const uint32_t *tets, uint32_t a, std::vector<uint32_t> &nb)
{
    nb.clear();
    for (uint32_t t = P.adj_ptr[a]; t < P.adj_ptr[a + 1]; t++) {
        const uint32_t *tv = tets + 4 * size_t(P.adj_elem[t]);
        for (int k = 0; k < 4; k++)
            if (P.node_mask[tv[k]]) nb.push_back(tv[k]);
    }
    std::sort(nb.begin(), nb.end());
    nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
}
}  // namespace

bool build_assembly_plan(uint32_t n_nodes, uint32_t n_tets, const uint32_t *tets, uint32_t n_tris,
                         const uint32_t *tris, const uint32_t *book, uint32_t dofs, uint32_t n_free,
                         AsmPlanHost &P, std::string &err)
{
    if (dofs != 1 && dofs != 3) {
        err = "dofs per node must be 1 or 3";
        return false;
    }
    P = AsmPlanHost();
    P.n_nodes = n_nodes;
    P.n_tets = n_tets;
    P.n_tris = n_tris;
    P.dofs = dofs;
    P.n_free = n_free;

    // node book: free positions must be 0..n_free-1, increasing with the DOF index
    // (the numbering RSolverGeneric::rebuildNodeBook produces, src/rsolvergeneric.cpp:565-582)
    P.node_mask.assign(n_nodes, 0);
    P.row_node.resize(n_free);
    P.row_comp.resize(n_free);
    uint32_t next = 0;
    for (uint32_t a = 0; a < n_nodes; a++)
        for (uint32_t j = 0; j < dofs; j++) {
            const uint32_t pos = book[size_t(a) * dofs + j];
            if (pos == kEod) continue;
            if (pos != next) {
                err = "node book must number free DOFs consecutively in DOF order";
                return false;
            }
            P.node_mask[a] |= uint8_t(1u << j);
            P.row_node[next] = a;
            P.row_comp[next] = uint8_t(j);
            next++;
        }
    if (next != n_free) {
        err = "n_free does not match the node book";
        return false;
    }
    for (size_t i = 0; i < size_t(n_tets) * 4; i++)
        if (tets[i] >= n_nodes) {
            err = "tet node index out of range";
            return false;
        }
    for (size_t i = 0; i < size_t(n_tris) * 3; i++)
        if (tris[i] >= n_nodes) {
            err = "triangle node index out of range";
            return false;
        }

    // node -> tet adjacency, ascending tet order
    P.adj_ptr.assign(size_t(n_nodes) + 1, 0);
    for (size_t i = 0; i < size_t(n_tets) * 4; i++) P.adj_ptr[tets[i] + 1]++;
    for (uint32_t a = 0; a < n_nodes; a++) P.adj_ptr[a + 1] += P.adj_ptr[a];
    P.adj_elem.resize(size_t(n_tets) * 4);
    P.adj_loc.resize(size_t(n_tets) * 4);
    {
        std::vector<uint32_t> fill(P.adj_ptr.begin(), P.adj_ptr.end() - 1);
        for (uint32_t e = 0; e < n_tets; e++)
            for (int k = 0; k < 4; k++) {
                const uint32_t a = tets[4 * size_t(e) + k];
                const uint32_t t = fill[a]++;
                P.adj_elem[t] = e;
                P.adj_loc[t] = uint8_t(k);
            }
    }
    // node -> triangle adjacency (traction RHS)
    P.tadj_ptr.assign(size_t(n_nodes) + 1, 0);
    for (size_t i = 0; i < size_t(n_tris) * 3; i++) P.tadj_ptr[tris[i] + 1]++;
    for (uint32_t a = 0; a < n_nodes; a++) P.tadj_ptr[a + 1] += P.tadj_ptr[a];
    P.tadj_tri.resize(size_t(n_tris) * 3);
    {
        std::vector<uint32_t> fill(P.tadj_ptr.begin(), P.tadj_ptr.end() - 1);
        for (uint32_t f = 0; f < n_tris; f++)
            for (int k = 0; k < 3; k++) P.tadj_tri[fill[tris[3 * size_t(f) + k]]++] = f;
    }

    // pass 1: row lengths (columns of a node's rows = free comps of its neighbours)
    std::vector<uint32_t> node_len(n_nodes, 0);
    bool too_long = false;
#pragma omp parallel
    {
        std::vector<uint32_t> nb;
#pragma omp for schedule(dynamic, 1024) reduction(|| : too_long)
        for (int64_t a = 0; a < int64_t(n_nodes); a++) {
            if (!P.node_mask[a]) continue;
            neighbours(P, tets, uint32_t(a), nb);
            uint32_t len = 0;
            for (uint32_t b : nb) len += popc(P.node_mask[b]);
            node_len[a] = len;
            if (len >= 0xffffu) too_long = true;
        }
    }
    if (too_long) {
        err = "a row has more than 65534 entries";
        return false;
    }
    P.rp.assign(size_t(n_free) + 1, 0);
    for (uint32_t r = 0; r < n_free; r++) {
        const uint64_t e = uint64_t(P.rp[r]) + node_len[P.row_node[r]];
        if (e > 0xffffffffull) {
            err = "more than 2^32-1 nonzeros";
            return false;
        }
        P.rp[r + 1] = uint32_t(e);
    }
    P.ci.resize(P.rp[n_free]);
    P.adj_off.assign(size_t(n_tets) * 4 * 4, 0xffffu);

    // pass 2: columns and the scatter map
    std::vector<uint32_t> first_row(n_nodes, kEod);
    for (uint32_t r = n_free; r-- > 0;) first_row[P.row_node[r]] = r;
#pragma omp parallel
    {
        std::vector<uint32_t> nb, off;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t a = 0; a < int64_t(n_nodes); a++) {
            if (!P.node_mask[a]) continue;
            neighbours(P, tets, uint32_t(a), nb);
            off.resize(nb.size());
            uint32_t o = 0;
            for (size_t k = 0; k < nb.size(); k++) {
                off[k] = o;
                o += popc(P.node_mask[nb[k]]);
            }
            // every row of node a has the same columns
            for (uint32_t r = first_row[a]; r < n_free && P.row_node[r] == uint32_t(a); r++) {
                uint32_t c = P.rp[r];
                for (uint32_t b : nb)
                    for (uint32_t j = 0; j < dofs; j++)
                        if (P.node_mask[b] & (1u << j)) P.ci[c++] = book[size_t(b) * dofs + j];
            }
            for (uint32_t t = P.adj_ptr[a]; t < P.adj_ptr[a + 1]; t++) {
                const uint32_t *tv = tets + 4 * size_t(P.adj_elem[t]);
                for (int k = 0; k < 4; k++) {
                    if (!P.node_mask[tv[k]]) continue;
                    const size_t idx = std::lower_bound(nb.begin(), nb.end(), tv[k]) - nb.begin();
                    P.adj_off[size_t(t) * 4 + k] = uint16_t(off[idx]);
                }
            }
        }
    }
    return true;
}

}  // namespace rsg
