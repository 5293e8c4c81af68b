// Host-side assembly plan: sparsity pattern of the free-DOF system and the
// element-to-nonzero scatter map (plain C++; built once per mesh + node book).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace rsg {

struct AsmPlanHost {
    uint32_t n_nodes = 0, n_tets = 0, n_tris = 0, dofs = 1, n_free = 0;
    std::vector<uint32_t> row_node;   // node of each free row
    std::vector<uint8_t> row_comp;    // component of each free row
    std::vector<uint32_t> rp, ci;     // CSR pattern (sorted columns)
    // node -> tets adjacency in ascending tet order
    std::vector<uint32_t> adj_ptr, adj_elem;
    std::vector<uint8_t> adj_loc;     // local index of the node in the tet
    std::vector<uint16_t> adj_off;    // 4 per entry: offset of each tet node's column block in the row (0xffff: none)
    // node -> traction triangles adjacency (elasticity only)
    std::vector<uint32_t> tadj_ptr, tadj_tri;
    std::vector<uint8_t> node_mask;   // bit j set when component j of the node is free
};

// book has n_nodes * dofs entries (free position or 0xffffffff).  Returns false and sets err on bad input.
bool build_assembly_plan(uint32_t n_nodes, uint32_t n_tets, const uint32_t *tets, uint32_t n_tris,
                         const uint32_t *tris, const uint32_t *book, uint32_t dofs, uint32_t n_free,
                         AsmPlanHost &plan, std::string &err);

}  // namespace rsg
