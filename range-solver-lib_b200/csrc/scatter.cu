// Pattern-cached assembly of caller-computed element matrices: RSolverFluid::buildSparseMatrixPattern
// and assemblyMatrix (src/rsolverfluid.cpp:2305-2419) on the GPU.
//
// The reference builds, once per pattern, the sparse pattern of every active element's enabled DOFs
// (RSparseMatrix::addValue(row, column, 0.0)) and each element's map from local (row, column) to the
// entry's position, then adds every element matrix into the matrix through that map in element
// order (serially).  Here the plan (host, once) stores the inverse of that map: for every stored
// entry the list of (element, local entry) contributions in element order, and likewise for the
// right-hand side.  The numeric assembly is then one thread per entry gathering its contributions
// from the concatenated element matrices and adding them in element order starting from zero --
// the reference's sum, bit for bit, without atomics.
#include "csr.cuh"

#include <algorithm>
#include <numeric>
#include <vector>

struct rsg_scatter_plan {
    uint32_t d = 0, n_free = 0, n_elements = 0;
    uint64_t ae_values = 0, fe_values = 0, nnz = 0;
    std::vector<uint32_t> rp, ci;  // the pattern (host copy, for creating A)
    uint32_t *entry_ptr = nullptr;  // nnz + 1 (device)
    uint64_t *entry_src = nullptr;  // contributions: indexes into the concatenated element matrices
    uint32_t *row_ptr = nullptr;    // n_free + 1
    uint64_t *row_src = nullptr;    // contributions to b: indexes into the concatenated element vectors
    double *stage = nullptr;        // device copies of host element matrices / vectors (grow-only)
    size_t stage_cap = 0;
};

namespace rsg {
namespace {

__global__ void k_scatter_entries(uint64_t nnz, const uint32_t *__restrict__ ptr, const uint64_t *__restrict__ src,
                                  const double *__restrict__ ae, double *__restrict__ val)
{
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < nnz; e += uint64_t(gridDim.x) * blockDim.x) {
        double v = 0.0;
        for (uint32_t k = ptr[e]; k < ptr[e + 1]; k++) v += ae[src[k]];
        val[e] = v;
    }
}

__global__ void k_scatter_rhs(uint32_t n, const uint32_t *__restrict__ ptr, const uint64_t *__restrict__ src,
                              const double *__restrict__ fe, double *__restrict__ b)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (uint32_t k = ptr[i]; k < ptr[i + 1]; k++) v += fe[src[k]];
        b[i] = v;
    }
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_scatter_plan_create(rsg_context *ctx, uint32_t d, uint32_t ne, const uint32_t *elem_begin,
                                   const uint32_t *elem_nodes, const uint8_t *elem_active, uint32_t n_nodes,
                                   const uint32_t *book, uint32_t n_free, rsg_scatter_plan **out)
{
    if (!ctx || !out || !elem_begin || (ne && !elem_nodes) || !book || d == 0 || n_free == 0)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_plan_create: bad arguments");
    *out = nullptr;
    constexpr uint32_t kOff = 0xffffffffu;
    for (uint64_t k = 0; k < uint64_t(n_nodes) * d; k++)
        if (book[k] != kOff && book[k] >= n_free)
            return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_plan_create: book entry %llu out of range",
                             (unsigned long long)k);
    // 1. each active element's enabled local DOFs (node slot m, component i in order) and their rows
    std::vector<uint32_t> act_begin(size_t(ne) + 1, 0), act_local, act_row;
    std::vector<uint64_t> ae_off(ne, 0), fe_off(ne, 0);
    std::vector<uint32_t> ndofs(ne, 0);
    uint64_t ae_total = 0, fe_total = 0;
    for (uint32_t e = 0; e < ne; e++) {
        act_begin[e] = uint32_t(act_local.size());
        if (elem_begin[e + 1] < elem_begin[e])
            return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_plan_create: elem_begin not ascending");
        if (!elem_active || elem_active[e]) {
            const uint32_t size = elem_begin[e + 1] - elem_begin[e];
            ndofs[e] = size * d;
            ae_off[e] = ae_total;
            fe_off[e] = fe_total;
            ae_total += uint64_t(ndofs[e]) * ndofs[e];
            fe_total += ndofs[e];
            for (uint32_t m = 0; m < size; m++) {
                const uint32_t node = elem_nodes[elem_begin[e] + m];
                if (node >= n_nodes) return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_plan_create: node out of range");
                for (uint32_t i = 0; i < d; i++) {
                    const uint32_t mp = book[size_t(node) * d + i];
                    if (mp == kOff) continue;
                    act_local.push_back(m * d + i);
                    act_row.push_back(mp);
                }
            }
        }
    }
    act_begin[ne] = uint32_t(act_local.size());
    // 2. the pattern: every (row, column) pair of every active element, rows sorted and unique
    std::vector<std::vector<uint32_t>> cols(n_free);
    for (uint32_t e = 0; e < ne; e++)
        for (uint32_t a = act_begin[e]; a < act_begin[e + 1]; a++)
            for (uint32_t c = act_begin[e]; c < act_begin[e + 1]; c++) cols[act_row[a]].push_back(act_row[c]);
    auto *P = new rsg_scatter_plan;
    P->d = d;
    P->n_free = n_free;
    P->n_elements = ne;
    P->ae_values = ae_total;
    P->fe_values = fe_total;
    P->rp.assign(size_t(n_free) + 1, 0);
    for (uint32_t r = 0; r < n_free; r++) {
        auto &c = cols[r];
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        P->rp[r + 1] = P->rp[r] + uint32_t(c.size());
    }
    P->nnz = P->rp[n_free];
    P->ci.reserve(P->nnz);
    for (uint32_t r = 0; r < n_free; r++) P->ci.insert(P->ci.end(), cols[r].begin(), cols[r].end());
    std::vector<std::vector<uint32_t>>().swap(cols);
    // 3. contributions per entry and per right-hand-side row, in element order (counting sort)
    auto position = [&](uint32_t row, uint32_t col) {
        const uint32_t *b = P->ci.data() + P->rp[row], *e = P->ci.data() + P->rp[row + 1];
        return uint32_t(std::lower_bound(b, e, col) - P->ci.data());
    };
    std::vector<uint32_t> eptr(P->nnz + 1, 0), rptr(size_t(n_free) + 1, 0);
    for (uint32_t e = 0; e < ne; e++)
        for (uint32_t a = act_begin[e]; a < act_begin[e + 1]; a++) {
            rptr[act_row[a] + 1]++;
            for (uint32_t c = act_begin[e]; c < act_begin[e + 1]; c++) eptr[position(act_row[a], act_row[c]) + 1]++;
        }
    for (uint64_t k = 0; k < P->nnz; k++) eptr[k + 1] += eptr[k];
    for (uint32_t r = 0; r < n_free; r++) rptr[r + 1] += rptr[r];
    std::vector<uint64_t> esrc(eptr[P->nnz]), rsrc(rptr[n_free]);
    std::vector<uint32_t> efill(eptr.begin(), eptr.end() - 1), rfill(rptr.begin(), rptr.end() - 1);
    for (uint32_t e = 0; e < ne; e++)
        for (uint32_t a = act_begin[e]; a < act_begin[e + 1]; a++) {
            const uint32_t la = act_local[a];
            rsrc[rfill[act_row[a]]++] = fe_off[e] + la;
            for (uint32_t c = act_begin[e]; c < act_begin[e + 1]; c++)
                esrc[efill[position(act_row[a], act_row[c])]++] = ae_off[e] + uint64_t(la) * ndofs[e] + act_local[c];
        }
    // 4. device copies
    auto fail = [&](rsg_status s) {
        rsg_scatter_plan_destroy(ctx, P);
        return s;
    };
    if (cudaMalloc(&P->entry_ptr, eptr.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&P->entry_src, std::max<size_t>(esrc.size(), 1) * sizeof(uint64_t)) != cudaSuccess ||
        cudaMalloc(&P->row_ptr, rptr.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&P->row_src, std::max<size_t>(rsrc.size(), 1) * sizeof(uint64_t)) != cudaSuccess)
        return fail(set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "scatter_plan_create: device maps"));
    if (cudaMemcpy(P->entry_ptr, eptr.data(), eptr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P->entry_src, esrc.data(), esrc.size() * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P->row_ptr, rptr.data(), rptr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(P->row_src, rsrc.data(), rsrc.size() * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_error(ctx, RSG_ERR_CUDA, "scatter_plan_create: upload"));
    *out = P;
    return RSG_OK;
}

rsg_status rsg_scatter_plan_info(const rsg_scatter_plan *P, uint64_t *ae_values, uint64_t *fe_values, uint64_t *nnz)
{
    if (!P) return RSG_ERR_INVALID_ARG;
    if (ae_values) *ae_values = P->ae_values;
    if (fe_values) *fe_values = P->fe_values;
    if (nnz) *nnz = P->nnz;
    return RSG_OK;
}

rsg_status rsg_scatter_assemble(rsg_context *ctx, rsg_scatter_plan *P, const double *Ae, const double *fe,
                                int32_t memory, rsg_csr **A, double *b)
{
    if (!ctx || !P || !A || (P->ae_values && !Ae) || (b && P->fe_values && !fe))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_assemble: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    if (*A && ((*A)->n != P->n_free || (*A)->nnz != P->nnz))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "scatter_assemble: A does not have the plan's pattern");
    if (!*A) {
        std::vector<double> zero(P->nnz, 0.0);
        RSG_TRY(rsg_csr_create(ctx, P->n_free, P->rp.data(), P->ci.data(), zero.data(), RSG_MEM_HOST, A));
    }
    const double *ae = Ae, *fv = fe;
    if (memory == RSG_MEM_HOST) {
        const size_t need = size_t(P->ae_values) + (b ? size_t(P->fe_values) : 0);
        if (need > P->stage_cap) {
            if (P->stage) cudaFree(P->stage);
            P->stage = nullptr;
            P->stage_cap = 0;
            if (cudaMalloc(&P->stage, std::max<size_t>(need, 1) * sizeof(double)) != cudaSuccess)
                return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "scatter_assemble: staging");
            P->stage_cap = need;
        }
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(P->stage, Ae, P->ae_values * sizeof(double), cudaMemcpyHostToDevice,
                                            ctx->stream));
        if (b)
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(P->stage + P->ae_values, fe, P->fe_values * sizeof(double),
                                                cudaMemcpyHostToDevice, ctx->stream));
        ae = P->stage;
        fv = P->stage + P->ae_values;
    }
    rsg_csr *M = *A;
    const int ge = std::max(1, int(std::min<uint64_t>((P->nnz + kBlock - 1) / kBlock, uint64_t(ctx->num_sms) * 16)));
    k_scatter_entries<<<ge, kBlock, 0, ctx->stream>>>(P->nnz, P->entry_ptr, P->entry_src, ae, M->val);
    if (b) {
        const int gr = std::max(1, int(std::min<uint64_t>((P->n_free + kBlock - 1) / kBlock, uint64_t(ctx->num_sms) * 16)));
        k_scatter_rhs<<<gr, kBlock, 0, ctx->stream>>>(P->n_free, P->row_ptr, P->row_src, fv, b);
    }
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return csr_refresh(ctx, M);
}

void rsg_scatter_plan_destroy(rsg_context *ctx, rsg_scatter_plan *P)
{
    if (!P) return;
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(P->entry_ptr);
    cudaFree(P->entry_src);
    cudaFree(P->row_ptr);
    cudaFree(P->row_src);
    if (P->stage) cudaFree(P->stage);
    delete P;
}

}  // extern "C"
