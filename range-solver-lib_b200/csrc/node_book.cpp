// Node books: the numbering of free degrees of freedom (host, C++17 + OpenMP).
//
// The reference numbers DOFs once per prepare():
//   * RSolverGeneric::generateNodeBook (src/rsolvergeneric.cpp:498-561) disables
//     every node of an element group that carries an explicit boundary condition
//     of the problem type and every node that no computable element touches;
//     rebuildNodeBook (:565-582) then numbers the remaining nodes consecutively
//     in node order (disabled nodes get RConstants::eod);
//   * RSolverStress::generateNodeBook (src/rsolverstress.cpp:1564-1652) does the
//     same on 3 interleaved components per node (position 3 node + c): a
//     displacement or normal-displacement condition disables all three, a roller
//     on a line group the y and z components, a roller on any other group the x
//     component.
// Here the marking pass runs in parallel over the groups' elements (every write
// stores the same value 1, so the order of the writes does not matter) and the
// numbering is a two-pass blocked prefix sum; the result is the reference's
// numbering exactly.  Everything is host memory; no GPU is involved.
#include <omp.h>

#include <algorithm>
#include <vector>

#include "../../include/rsg.h"

namespace {

constexpr uint32_t kEod = 0xffffffffu;

// Checks the CSR-like element and group arrays of the model description.
bool valid_model(const rsg_model_groups *m)
{
    if (!m || m->n_nodes == 0 || !m->elem_begin || (m->n_groups && (!m->group_begin || !m->group_elems)))
        return false;
    if (m->elem_begin[0] != 0) return false;
    for (uint32_t e = 0; e < m->n_elements; e++)
        if (m->elem_begin[e + 1] < m->elem_begin[e]) return false;
    if (m->elem_begin[m->n_elements] > 0 && !m->elem_nodes) return false;
    for (uint32_t j = 0; j < m->elem_begin[m->n_elements]; j++)
        if (m->elem_nodes[j] >= m->n_nodes) return false;
    if (m->n_groups) {
        if (m->group_begin[0] != 0) return false;
        for (uint32_t g = 0; g < m->n_groups; g++)
            if (m->group_begin[g + 1] < m->group_begin[g]) return false;
        for (uint32_t j = 0; j < m->group_begin[m->n_groups]; j++)
            if (m->group_elems[j] >= m->n_elements) return false;
    }
    return true;
}

// Sets mark[stride * node + c] for every c in `comps` (bit mask) and every node of the group's elements.
void mark_group(const rsg_model_groups *m, uint32_t g, uint32_t stride, uint32_t comps, uint8_t *mark)
{
    const int64_t e0 = m->group_begin[g], e1 = m->group_begin[g + 1];
#pragma omp parallel for schedule(static)
    for (int64_t j = e0; j < e1; j++) {
        const uint32_t e = m->group_elems[j];
        for (uint32_t k = m->elem_begin[e]; k < m->elem_begin[e + 1]; k++) {
            const size_t base = size_t(stride) * m->elem_nodes[k];
            for (uint32_t c = 0; c < stride; c++)
                if (comps & (1u << c)) {
#pragma omp atomic write
                    mark[base + c] = uint8_t(1);
                }
        }
    }
}

// Disables (stride components of) every node that no computable element touches.
void mark_not_computable(const rsg_model_groups *m, uint32_t stride, uint8_t *mark)
{
    std::vector<uint8_t> touched(m->n_nodes, 0);
    const int64_t ne = m->n_elements;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < ne; e++) {
        if (m->computable && !m->computable[e]) continue;
        for (uint32_t k = m->elem_begin[e]; k < m->elem_begin[e + 1]; k++) {
#pragma omp atomic write
            touched[m->elem_nodes[k]] = uint8_t(1);
        }
    }
    const int64_t nn = m->n_nodes;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nn; i++)
        if (!touched[i])
            for (uint32_t c = 0; c < stride; c++) mark[size_t(stride) * i + c] = 1;
}

// rebuildNodeBook: consecutive positions for the unmarked entries in index order, kEod for the others.
uint32_t number_positions(const uint8_t *mark, size_t n, uint32_t *book)
{
    const int nb = std::max(1, std::min<int>(omp_get_max_threads(), int(n / 65536) + 1));
    std::vector<uint64_t> count(size_t(nb) + 1, 0);
    auto range = [&](int t, size_t &lo, size_t &hi) {
        lo = n * size_t(t) / size_t(nb);
        hi = n * size_t(t + 1) / size_t(nb);
    };
#pragma omp parallel for num_threads(nb) schedule(static, 1)
    for (int t = 0; t < nb; t++) {
        size_t lo, hi;
        range(t, lo, hi);
        uint64_t c = 0;
        for (size_t i = lo; i < hi; i++) c += mark[i] ? 0 : 1;
        count[size_t(t) + 1] = c;
    }
    for (int t = 0; t < nb; t++) count[size_t(t) + 1] += count[size_t(t)];
#pragma omp parallel for num_threads(nb) schedule(static, 1)
    for (int t = 0; t < nb; t++) {
        size_t lo, hi;
        range(t, lo, hi);
        uint32_t next = uint32_t(count[size_t(t)]);
        for (size_t i = lo; i < hi; i++) book[i] = mark[i] ? kEod : next++;
    }
    return uint32_t(count[size_t(nb)]);
}

}  // namespace

extern "C" {

rsg_status rsg_node_book_generic(const rsg_model_groups *model, const uint8_t *group_explicit_bc, uint32_t *book,
                                 uint32_t *n_free)
{
    if (!valid_model(model) || !book || !n_free || (model->n_groups && !group_explicit_bc)) return RSG_ERR_INVALID_ARG;
    try {
        std::vector<uint8_t> mark(model->n_nodes, 0);
        for (uint32_t g = 0; g < model->n_groups; g++)
            if (group_explicit_bc[g]) mark_group(model, g, 1, 1u, mark.data());
        mark_not_computable(model, 1, mark.data());
        *n_free = number_positions(mark.data(), mark.size(), book);
    } catch (...) {
        return RSG_ERR_OUT_OF_MEMORY;
    }
    return RSG_OK;
}

rsg_status rsg_node_book_stress(const rsg_model_groups *model, const uint8_t *group_bc, const uint8_t *group_is_line,
                                uint32_t *book, uint32_t *n_free)
{
    if (!valid_model(model) || !book || !n_free || (model->n_groups && (!group_bc || !group_is_line)))
        return RSG_ERR_INVALID_ARG;
    try {
        std::vector<uint8_t> mark(size_t(model->n_nodes) * 3, 0);
        for (uint32_t g = 0; g < model->n_groups; g++) {
            uint32_t comps = 0;
            if (group_bc[g] & (RSG_BC_DISPLACEMENT | RSG_BC_DISPLACEMENT_NORMAL)) comps |= 7u;
            if (group_bc[g] & RSG_BC_DISPLACEMENT_ROLLER) comps |= group_is_line[g] ? 6u : 1u;
            if (comps) mark_group(model, g, 3, comps, mark.data());
        }
        mark_not_computable(model, 3, mark.data());
        *n_free = number_positions(mark.data(), mark.size(), book);
    } catch (...) {
        return RSG_ERR_OUT_OF_MEMORY;
    }
    return RSG_OK;
}

}  // extern "C"
