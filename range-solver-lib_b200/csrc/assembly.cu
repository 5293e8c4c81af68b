// GPU stiffness assembly for linear tetrahedra (heat: 1 DOF/node, elasticity:
// 3 DOFs/node), deterministic and atomic-free.
//
// One thread owns one free row.  It walks its node's adjacent tets in
// ascending tet order (traction triangles first for elasticity, as the
// reference assembles surfaces before volumes), recomputes the tet's element
// row it needs (constant-gradient P1 element: B = grad N, V = |det J| / 6),
// applies the theta scheme and the Dirichlet lifting of
// RSolverHeat/RSolverStress::assemblyMatrix, and adds the row into its own CSR
// entries through the plan's scatter offsets.  Every entry therefore sums its
// element contributions in the same order as the reference's sequential
// element loop, and repeated assemblies are bitwise identical.
//
// Reference lines restated: heat element src/rsolverheat.cpp:397-435, heat
// assembly :755-820; elasticity element src/rsolverstress.cpp:613-693,
// traction :498-507, assembly :1654-1772.
#include "assembly_plan.h"
#include "csr.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>

struct rsg_assembly {
    uint32_t n_nodes = 0, n_tets = 0, n_tris = 0, dofs = 1, n_free = 0;
    uint64_t nnz = 0;
    double *xyz = nullptr;
    uint32_t *tets = nullptr, *tris = nullptr, *book = nullptr;
    uint32_t *row_node = nullptr;
    uint8_t *row_comp = nullptr;
    uint32_t *rp = nullptr, *ci = nullptr;
    uint32_t *adj_ptr = nullptr, *adj_elem = nullptr;
    uint8_t *adj_loc = nullptr;
    uint16_t *adj_off = nullptr;
    uint32_t *tadj_ptr = nullptr, *tadj_tri = nullptr;
    uint8_t *node_mask = nullptr;
    double *stage = nullptr;   // host inputs staged on the device
    size_t stage_cap = 0;
    uint32_t max_row = 0;      // longest row of the pattern (the thread-local kernels take short rows)
    int kind = 0;              // rsg::kPlanHeat / kPlanStress / kPlanMagnetostatics
};

namespace rsg {

enum { kPlanHeat = 1, kPlanStress = 2, kPlanMagnetostatics = 3 };

namespace {

__device__ __forceinline__ double tet_geometry(const double *__restrict__ xyz, const uint4 t, double G[4][3])
{
    double X0[3], a[3], b[3], c[3];
    for (int k = 0; k < 3; k++) X0[k] = xyz[3 * size_t(t.x) + k];
    for (int k = 0; k < 3; k++) {
        a[k] = xyz[3 * size_t(t.y) + k] - X0[k];
        b[k] = xyz[3 * size_t(t.z) + k] - X0[k];
        c[k] = xyz[3 * size_t(t.w) + k] - X0[k];
    }
    const double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    const double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    const double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    const double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
    for (int k = 0; k < 3; k++) {
        G[1][k] = bc[k] / det;
        G[2][k] = ca[k] / det;
        G[3][k] = ab[k] / det;
        G[0][k] = -(G[1][k] + G[2][k] + G[3][k]);
    }
    return fabs(det) / 6.0;
}

// Row m of the gradient matrix selected without indexing G by a run-time m (which would put G
// in local memory).
__device__ __forceinline__ void grad_row(const double G[4][3], int m, double gm[3])
{
    for (int c = 0; c < 3; c++) gm[c] = m == 0 ? G[0][c] : m == 1 ? G[1][c] : m == 2 ? G[2][c] : G[3][c];
}

__device__ __forceinline__ uint32_t node_of(const uint4 t, int k)
{
    return k == 0 ? t.x : k == 1 ? t.y : k == 2 ? t.z : t.w;
}

// Contribution of one (row node, adjacent tet) pair to the row: Ar[n] for the tet's
// 4 nodes (theta scheme applied when transient) and the right-hand side part be
// (source, transient history, Dirichlet lifting).
__device__ __forceinline__ void heat_adj(uint32_t t, const uint32_t *__restrict__ adj_elem,
                                         const uint8_t *__restrict__ adj_loc, const double *__restrict__ xyz,
                                         const uint4 *__restrict__ tets, const uint32_t *__restrict__ book,
                                         const double *__restrict__ k_e, const double *__restrict__ q_e,
                                         const double *__restrict__ rhoc_e, const double *__restrict__ node_t,
                                         int transient, double alpha, double dt, double (&Ar)[4], double &be)
{
    const uint32_t e = adj_elem[t];
    const int m = adj_loc[t];
    const uint4 tv = tets[e];
    double G[4][3];
    const double V = tet_geometry(xyz, tv, G);
    const double k = k_e[e];
    double gm[3];
    grad_row(G, m, gm);
    for (int n = 0; n < 4; n++) Ar[n] = (gm[0] * G[n][0] + gm[1] * G[n][1] + gm[2] * G[n][2]) * k * V;
    const double fe = q_e[e] * V / 4.0;
    if (transient) {
        const double rc = rhoc_e[e];
        be = dt * fe;
        for (int n = 0; n < 4; n++) {
            const double Me = rc * V * (m == n ? 2.0 : 1.0) / 20.0;
            const double Ke = Ar[n];
            Ar[n] = Me + alpha * dt * Ke;
            be += (Me - (1.0 - alpha) * dt * Ke) * node_t[node_of(tv, n)];
        }
    } else {
        be = fe;
    }
    for (int n = 0; n < 4; n++) {
        const uint32_t nd = node_of(tv, n);
        if (book[nd] == RSG_EOD) be -= Ar[n] * node_t[nd];
    }
}

// Rows accumulated in global memory (any row length).
__global__ void __launch_bounds__(kBlock) k_asm_heat(
    uint32_t n_free, const uint32_t *__restrict__ row_node, const uint32_t *__restrict__ rp,
    const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem, const uint8_t *__restrict__ adj_loc,
    const ushort4 *__restrict__ adj_off, const double *__restrict__ xyz, const uint4 *__restrict__ tets,
    const uint32_t *__restrict__ book, const double *__restrict__ k_e, const double *__restrict__ q_e,
    const double *__restrict__ rhoc_e, const double *__restrict__ node_t, int transient, double alpha, double dt,
    double *__restrict__ val, double *__restrict__ b)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_free; r += gridDim.x * blockDim.x) {
        const uint32_t a = row_node[r], start = rp[r], end = rp[r + 1];
        for (uint32_t j = start; j < end; j++) val[j] = 0.0;
        double bs = 0.0;
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            double Ar[4], be;
            heat_adj(t, adj_elem, adj_loc, xyz, tets, book, k_e, q_e, rhoc_e, node_t, transient, alpha, dt, Ar, be);
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            bs += be;
            for (int n = 0; n < 4; n++)
                if (off[n] != 0xffffu) val[start + off[n]] += Ar[n];
        }
        b[r] = bs;
    }
}

// One thread per row with the row accumulated in shared memory (rows of up to kLocalRowMax
// entries, the launch sizes it for the plan's longest row; entry j of a thread at
// acc_s[j * blockDim.x + threadIdx.x]): the same per-entry order
// as k_asm_heat without read-modify-write round trips through global memory.  A thread-local
// array indexed by the column offset cannot stay in registers: it went through local memory,
// 515 MB of DRAM writes per launch at 100^3 against 127 MB of results.
constexpr uint32_t kLocalRowMax = 32;
constexpr size_t kHeatLocalSmem = size_t(kLocalRowMax) * kBlock * sizeof(double);

__global__ void __launch_bounds__(kBlock) k_asm_heat_local(
    uint32_t n_free, const uint32_t *__restrict__ row_node, const uint32_t *__restrict__ rp,
    const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem, const uint8_t *__restrict__ adj_loc,
    const ushort4 *__restrict__ adj_off, const double *__restrict__ xyz, const uint4 *__restrict__ tets,
    const uint32_t *__restrict__ book, const double *__restrict__ k_e, const double *__restrict__ q_e,
    const double *__restrict__ rhoc_e, const double *__restrict__ node_t, int transient, double alpha, double dt,
    double *__restrict__ val, double *__restrict__ b)
{
    extern __shared__ double acc_s[];
    double *acc = acc_s + threadIdx.x;
    const uint32_t stride = blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_free; r += gridDim.x * blockDim.x) {
        const uint32_t a = row_node[r], start = rp[r], len = min(rp[r + 1] - start, kLocalRowMax);
        for (uint32_t j = 0; j < len; j++) acc[j * stride] = 0.0;
        double bs = 0.0;
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            double Ar[4], be;
            heat_adj(t, adj_elem, adj_loc, xyz, tets, book, k_e, q_e, rhoc_e, node_t, transient, alpha, dt, Ar, be);
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            bs += be;
            for (int n = 0; n < 4; n++)
                if (off[n] < len) acc[off[n] * stride] += Ar[n];
        }
        for (uint32_t j = 0; j < len; j++) val[start + j] = acc[j * stride];
        b[r] = bs;
    }
}

// Row (3n+j) of the 12x6 strain-displacement matrix Be (strain order xx yy zz yz xz xy).
__device__ __forceinline__ void be_row(const double g[3], int j, double out[6])
{
    for (int k = 0; k < 6; k++) out[k] = 0.0;
    if (j == 0) {
        out[0] = g[0];
        out[4] = g[2];
        out[5] = g[1];
    } else if (j == 1) {
        out[1] = g[1];
        out[3] = g[2];
        out[5] = g[0];
    } else {
        out[2] = g[2];
        out[3] = g[1];
        out[4] = g[0];
    }
}

// Right-hand side of one traction triangle for component i (thickness 0: no stiffness).
__device__ __forceinline__ double traction_fe(uint32_t f, int i, const double *__restrict__ xyz,
                                              const uint32_t *__restrict__ tris, const double *__restrict__ traction,
                                              int transient, double dt)
{
    const uint32_t v0 = tris[3 * size_t(f)], v1 = tris[3 * size_t(f) + 1], v2 = tris[3 * size_t(f) + 2];
    double p[3], q[3];
    for (int k = 0; k < 3; k++) {
        p[k] = xyz[3 * size_t(v1) + k] - xyz[3 * size_t(v0) + k];
        q[k] = xyz[3 * size_t(v2) + k] - xyz[3 * size_t(v0) + k];
    }
    const double cr[3] = {p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]};
    const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    const double fe = traction[3 * size_t(f) + i] * area / 3.0;
    return transient ? dt * fe : fe;
}

// Contribution of one (row node a, component i, adjacent tet) triple: Ar[3n+j] for the
// tet's 4 nodes x 3 components (theta scheme applied when transient) and its be.
__device__ __forceinline__ void stress_adj(uint32_t t, int i, const uint32_t *__restrict__ adj_elem,
                                           const uint8_t *__restrict__ adj_loc, const double *__restrict__ xyz,
                                           const uint4 *__restrict__ tets, const uint32_t *__restrict__ book,
                                           const double *__restrict__ e_mod, const double *__restrict__ nu,
                                           const double *__restrict__ rho_e, const double *__restrict__ gravity,
                                           const double *__restrict__ texp_e, const double *__restrict__ dtemp_e,
                                           const double *__restrict__ node_u, int transient, double alpha, double dt,
                                           double (&Ar)[12], double &be, uint4 &tv)
{
    const uint32_t e = adj_elem[t];
    const int m = adj_loc[t];
    tv = tets[e];
    double G[4][3];
    const double V = tet_geometry(xyz, tv, G);
    const double E = e_mod[e], v = nu[e];
    const double f = E / ((1.0 + v) * (1.0 - 2.0 * v));
    double De[6][6];
    for (int p = 0; p < 6; p++)
        for (int q = 0; q < 6; q++) De[p][q] = 0.0;
    De[0][0] = 1.0 - v; De[0][1] = v;       De[0][2] = v;
    De[1][0] = v;       De[1][1] = 1.0 - v; De[1][2] = v;
    De[2][0] = v;       De[2][1] = v;       De[2][2] = 1.0 - v;
    De[3][3] = De[4][4] = De[5][5] = (1.0 - 2.0 * v) / 2.0;
    for (int p = 0; p < 6; p++)
        for (int q = 0; q < 6; q++) De[p][q] *= f;
    double Bm[6], BD[6];
    double gm[3];
    grad_row(G, m, gm);
    be_row(gm, i, Bm);
    for (int q = 0; q < 6; q++) {
        double s = 0.0;
        for (int k = 0; k < 6; k++) s += Bm[k] * De[k][q];
        BD[q] = s;
    }
    for (int n = 0; n < 4; n++)
        for (int j = 0; j < 3; j++) {
            double Bn[6];
            be_row(G[n], j, Bn);
            double s = 0.0;
            for (int k = 0; k < 6; k++) s += BD[k] * Bn[k];
            Ar[3 * n + j] = s * V;
        }
    double fe = gravity[i] * rho_e[e] * V / 4.0;
    for (int k = 0; k < 3; k++) fe += texp_e[e] * dtemp_e[e] * BD[k] * V;
    if (transient) {
        be = dt * fe;
        const double mv = rho_e[e] * V;
        for (int n = 0; n < 4; n++)
            for (int j = 0; j < 3; j++) {
                const double Me = (j == i) ? mv * (m == n ? 2.0 : 1.0) / 20.0 : 0.0;
                const double Ke = Ar[3 * n + j];
                Ar[3 * n + j] = Me + alpha * dt * Ke;
                be += (Me - (1.0 - alpha) * dt * Ke) * node_u[3 * size_t(node_of(tv, n)) + j];
            }
    } else {
        be = fe;
    }
    for (int n = 0; n < 4; n++) {
        const uint32_t nd = node_of(tv, n);
        for (int j = 0; j < 3; j++)
            if (book[3 * size_t(nd) + j] == RSG_EOD) be -= Ar[3 * n + j] * node_u[3 * size_t(nd) + j];
    }
}

// Rows accumulated in global memory (any row length).
__global__ void __launch_bounds__(128) k_asm_stress(
    uint32_t n_free, const uint32_t *__restrict__ row_node, const uint8_t *__restrict__ row_comp,
    const uint32_t *__restrict__ rp, const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem,
    const uint8_t *__restrict__ adj_loc, const ushort4 *__restrict__ adj_off, const uint32_t *__restrict__ tadj_ptr,
    const uint32_t *__restrict__ tadj_tri, const uint8_t *__restrict__ node_mask, const double *__restrict__ xyz,
    const uint4 *__restrict__ tets, const uint32_t *__restrict__ tris, const uint32_t *__restrict__ book,
    const double *__restrict__ e_mod, const double *__restrict__ nu, const double *__restrict__ rho_e,
    const double *__restrict__ gravity, const double *__restrict__ texp_e, const double *__restrict__ dtemp_e,
    const double *__restrict__ traction, const double *__restrict__ node_u, int transient, double alpha, double dt,
    double *__restrict__ val, double *__restrict__ b)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_free; r += gridDim.x * blockDim.x) {
        const uint32_t a = row_node[r], start = rp[r], end = rp[r + 1];
        const int i = row_comp[r];
        for (uint32_t j = start; j < end; j++) val[j] = 0.0;
        double bs = 0.0;
        for (uint32_t t = tadj_ptr[a]; t < tadj_ptr[a + 1]; t++)
            bs += traction_fe(tadj_tri[t], i, xyz, tris, traction, transient, dt);
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            double Ar[12], be;
            uint4 tv;
            stress_adj(t, i, adj_elem, adj_loc, xyz, tets, book, e_mod, nu, rho_e, gravity, texp_e, dtemp_e, node_u,
                       transient, alpha, dt, Ar, be, tv);
            bs += be;
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            for (int n = 0; n < 4; n++) {
                if (off[n] == 0xffffu) continue;
                const uint8_t mask = node_mask[node_of(tv, n)];
                uint32_t rank = 0;
                for (int j = 0; j < 3; j++)
                    if (mask & (1u << j)) val[start + off[n] + rank++] += Ar[3 * n + j];
            }
        }
        b[r] = bs;
    }
}

// One thread per row with the row accumulated in shared memory (rows of up to
// kLocalStressRowMax entries, the launch sizes it for the plan's longest row), as k_asm_heat_local.
constexpr uint32_t kLocalStressRowMax = 96;
constexpr int kStressBlock = 128;
constexpr size_t kStressLocalSmemMax = size_t(kLocalStressRowMax) * kStressBlock * sizeof(double);

__global__ void __launch_bounds__(128) k_asm_stress_local(
    uint32_t n_free, const uint32_t *__restrict__ row_node, const uint8_t *__restrict__ row_comp,
    const uint32_t *__restrict__ rp, const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem,
    const uint8_t *__restrict__ adj_loc, const ushort4 *__restrict__ adj_off, const uint32_t *__restrict__ tadj_ptr,
    const uint32_t *__restrict__ tadj_tri, const uint8_t *__restrict__ node_mask, const double *__restrict__ xyz,
    const uint4 *__restrict__ tets, const uint32_t *__restrict__ tris, const uint32_t *__restrict__ book,
    const double *__restrict__ e_mod, const double *__restrict__ nu, const double *__restrict__ rho_e,
    const double *__restrict__ gravity, const double *__restrict__ texp_e, const double *__restrict__ dtemp_e,
    const double *__restrict__ traction, const double *__restrict__ node_u, int transient, double alpha, double dt,
    double *__restrict__ val, double *__restrict__ b)
{
    extern __shared__ double acc_s[];
    double *acc = acc_s + threadIdx.x;
    const uint32_t stride = blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_free; r += gridDim.x * blockDim.x) {
        const uint32_t a = row_node[r], start = rp[r], len = min(rp[r + 1] - start, kLocalStressRowMax);
        const int i = row_comp[r];
        for (uint32_t j = 0; j < len; j++) acc[j * stride] = 0.0;
        double bs = 0.0;
        for (uint32_t t = tadj_ptr[a]; t < tadj_ptr[a + 1]; t++)
            bs += traction_fe(tadj_tri[t], i, xyz, tris, traction, transient, dt);
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            double Ar[12], be;
            uint4 tv;
            stress_adj(t, i, adj_elem, adj_loc, xyz, tets, book, e_mod, nu, rho_e, gravity, texp_e, dtemp_e, node_u,
                       transient, alpha, dt, Ar, be, tv);
            bs += be;
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            for (int n = 0; n < 4; n++) {
                if (off[n] == 0xffffu) continue;
                const uint8_t mask = node_mask[node_of(tv, n)];
                uint32_t rank = 0;
                for (int j = 0; j < 3; j++)
                    if (mask & (1u << j)) {
                        const uint32_t pos = off[n] + rank++;
                        if (pos < len) acc[pos * stride] += Ar[3 * n + j];
                    }
            }
        }
        for (uint32_t j = 0; j < len; j++) val[start + j] = acc[j * stride];
        b[r] = bs;
    }
}

// vacuum permittivity, RSolverGeneric::e0 (src/rsolvergeneric.cpp:13)
constexpr double kE0 = 8.854187817e-12;

// Contribution of one (row node, component i, adjacent tet) triple to a magnetostatic row
// (src/rsolvermagnetostatics.cpp:94-119, lifting :240-254): Ar[3n+j] = -(grad N_m . grad N_n) V
// on the component diagonal (j == i) and an explicit 0 elsewhere, be = e0 V/4 (grad N_m x J)_i
// with J the row node's current density, minus the lifting by disabled nodes' potentials.
__device__ __forceinline__ void magneto_adj(uint32_t t, int i, const uint32_t *__restrict__ adj_elem,
                                            const uint8_t *__restrict__ adj_loc, const double *__restrict__ xyz,
                                            const uint4 *__restrict__ tets, const uint32_t *__restrict__ book,
                                            const double *__restrict__ J, const double *__restrict__ node_a,
                                            double (&Ar)[12], double &be, uint4 &tv)
{
    const uint32_t e = adj_elem[t];
    const int m = adj_loc[t];
    tv = tets[e];
    double G[4][3];
    const double V = tet_geometry(xyz, tv, G);
    double gm[3];
    grad_row(G, m, gm);
    for (int n = 0; n < 4; n++) {
        const double v = (gm[0] * G[n][0] + gm[1] * G[n][1] + gm[2] * G[n][2]) * V;
        for (int j = 0; j < 3; j++) Ar[3 * n + j] = j == i ? 0.0 - v : 0.0;
    }
    const double js = i == 0 ? -gm[2] * J[1] + gm[1] * J[2]
                    : i == 1 ? gm[2] * J[0] - gm[0] * J[2]
                             : -gm[1] * J[0] + gm[0] * J[1];
    be = V / 4.0 * kE0 * js;
    for (int n = 0; n < 4; n++) {
        const uint32_t nd = node_of(tv, n);
        if (book[3 * size_t(nd)] == RSG_EOD)
            for (int j = 0; j < 3; j++) be -= Ar[3 * n + j] * node_a[3 * size_t(nd) + j];
    }
}

// One thread per row, the row accumulated in global memory (any row length).
__global__ void __launch_bounds__(128) k_asm_magneto(
    uint32_t n_free, const uint32_t *__restrict__ row_node, const uint8_t *__restrict__ row_comp,
    const uint32_t *__restrict__ rp, const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem,
    const uint8_t *__restrict__ adj_loc, const ushort4 *__restrict__ adj_off, const uint8_t *__restrict__ node_mask,
    const double *__restrict__ xyz, const uint4 *__restrict__ tets, const uint32_t *__restrict__ book,
    const double *__restrict__ node_j, const double *__restrict__ node_a, double *__restrict__ val,
    double *__restrict__ b)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_free; r += gridDim.x * blockDim.x) {
        const uint32_t a = row_node[r], start = rp[r], len = rp[r + 1] - start;
        const int i = row_comp[r];
        for (uint32_t j = 0; j < len; j++) val[start + j] = 0.0;
        const double J[3] = {node_j[3 * size_t(a)], node_j[3 * size_t(a) + 1], node_j[3 * size_t(a) + 2]};
        double bs = 0.0;
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            double Ar[12], be;
            uint4 tv;
            magneto_adj(t, i, adj_elem, adj_loc, xyz, tets, book, J, node_a, Ar, be, tv);
            bs += be;
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            for (int n = 0; n < 4; n++) {
                if (off[n] == 0xffffu) continue;
                const uint8_t mask = node_mask[node_of(tv, n)];
                uint32_t rank = 0;
                for (int j = 0; j < 3; j++)
                    if (mask & (1u << j)) val[start + off[n] + rank++] += Ar[3 * n + j];
            }
        }
        b[r] = bs;
    }
}

// One thread per free node.  Its three component rows (3p, 3p+1, 3p+2: a node's components are
// enabled or disabled together, checked when the plan is made) share the column pattern, the
// element geometry and the -(grad N_m . grad N_n) V values of the diagonal blocks, so each
// adjacent tet's geometry is computed once for the three rows, and one shared-memory slot per
// neighbour node accumulates the diagonal-block value.  Entry (n, j) of row i is that sum when
// j == i and an exact +0.0 otherwise; the right-hand side of each row follows magneto_adj's
// sequence.  The bits equal the row kernel's (tests compare them).
__global__ void __launch_bounds__(128) k_asm_magneto_node(
    uint32_t n_free_nodes, const uint32_t *__restrict__ row_node, const uint32_t *__restrict__ rp,
    const uint32_t *__restrict__ adj_ptr, const uint32_t *__restrict__ adj_elem, const uint8_t *__restrict__ adj_loc,
    const ushort4 *__restrict__ adj_off, const double *__restrict__ xyz, const uint4 *__restrict__ tets,
    const uint32_t *__restrict__ book, const double *__restrict__ node_j, const double *__restrict__ node_a,
    double *__restrict__ val, double *__restrict__ b)
{
    extern __shared__ double acc_s[];
    double *acc = acc_s + threadIdx.x;
    const uint32_t stride = blockDim.x;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_free_nodes; q += gridDim.x * blockDim.x) {
        const uint32_t r0 = 3 * q, a = row_node[r0], len = rp[r0 + 1] - rp[r0];
        const uint32_t slots = min(len / 3, kLocalStressRowMax / 3);
        for (uint32_t s = 0; s < slots; s++) acc[s * stride] = 0.0;
        const double J[3] = {node_j[3 * size_t(a)], node_j[3 * size_t(a) + 1], node_j[3 * size_t(a) + 2]};
        double bs[3] = {0.0, 0.0, 0.0};
        for (uint32_t t = adj_ptr[a]; t < adj_ptr[a + 1]; t++) {
            const uint32_t e = adj_elem[t];
            const int m = adj_loc[t];
            const uint4 tv = tets[e];
            double G[4][3];
            const double V = tet_geometry(xyz, tv, G);
            double gm[3];
            grad_row(G, m, gm);
            double dv[4];  // diagonal-block value of the pair (m, n)
            for (int n = 0; n < 4; n++) dv[n] = 0.0 - (gm[0] * G[n][0] + gm[1] * G[n][1] + gm[2] * G[n][2]) * V;
            const double js[3] = {-gm[2] * J[1] + gm[1] * J[2], gm[2] * J[0] - gm[0] * J[2],
                                  -gm[1] * J[0] + gm[0] * J[1]};
            double be[3];
            for (int i = 0; i < 3; i++) be[i] = V / 4.0 * kE0 * js[i];
            for (int n = 0; n < 4; n++) {
                const uint32_t nd = node_of(tv, n);
                if (book[3 * size_t(nd)] == RSG_EOD)
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) be[i] -= (j == i ? dv[n] : 0.0) * node_a[3 * size_t(nd) + j];
            }
            for (int i = 0; i < 3; i++) bs[i] += be[i];
            const ushort4 off4 = adj_off[t];
            const uint16_t off[4] = {off4.x, off4.y, off4.z, off4.w};
            for (int n = 0; n < 4; n++)
                if (off[n] != 0xffffu && off[n] / 3u < slots) acc[(off[n] / 3u) * stride] += dv[n];
        }
        for (int i = 0; i < 3; i++) {
            const uint32_t start = rp[r0 + i];
            for (uint32_t s = 0; s < slots; s++) {
                const double d = acc[s * stride];
                for (int j = 0; j < 3; j++) val[start + 3 * s + j] = j == i ? d : 0.0;
            }
            b[r0 + i] = bs[i];
        }
    }
}

// node_values[node * dofs + c] = x[book[node * dofs + c]] for every free DOF (the
// Dirichlet values stay): the solution back into the nodal field, e.g. the
// previous-step temperatures of the next transient assembly.
__global__ void k_asm_scatter(uint32_t n_entries, const uint32_t *__restrict__ book, const double *__restrict__ x,
                              double *__restrict__ node_values)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_entries; i += gridDim.x * blockDim.x) {
        const uint32_t pos = book[i];
        if (pos != RSG_EOD) node_values[i] = x[pos];
    }
}

// RSG_ASM_ROW_THREADS=1 selects the kernels that accumulate in global memory (tests compare the two)
bool row_threads_forced()
{
    const char *v = std::getenv("RSG_ASM_ROW_THREADS");
    return v && v[0] == '1';
}

template <typename T>
rsg_status upload(rsg_context *ctx, T **dst, const T *src, size_t count)
{
    if (count == 0) count = 1;
    RSG_CHECK_CUDA(ctx, cudaMalloc(dst, count * sizeof(T)));
    if (src) RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return RSG_OK;
}

void free_plan(rsg_assembly *p)
{
    if (!p) return;
    void *ptrs[] = {p->xyz, p->tets, p->tris, p->book, p->row_node, p->row_comp, p->rp, p->ci, p->adj_ptr,
                    p->adj_elem, p->adj_loc, p->adj_off, p->tadj_ptr, p->tadj_tri, p->node_mask, p->stage};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    delete p;
}

rsg_status create_plan(rsg_context *ctx, uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                       uint32_t n_tris, const uint32_t *tris, const uint32_t *book, uint32_t dofs, uint32_t n_free,
                       rsg_assembly **out)
{
    if (!ctx || !out || !xyz || !tets || !book || n_nodes == 0 || n_tets == 0 || n_free == 0 ||
        (n_tris && !tris))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assembly_create: bad arguments");
    *out = nullptr;
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    AsmPlanHost H;
    std::string err;
    if (!build_assembly_plan(n_nodes, n_tets, tets, n_tris, tris, book, dofs, n_free, H, err))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assembly_create: %s", err.c_str());
    auto *p = new rsg_assembly;
    p->n_nodes = n_nodes;
    p->n_tets = n_tets;
    p->n_tris = n_tris;
    p->dofs = dofs;
    p->n_free = n_free;
    p->nnz = H.ci.size();
    for (size_t r = 0; r + 1 < H.rp.size(); r++) p->max_row = std::max(p->max_row, H.rp[r + 1] - H.rp[r]);
    rsg_status s = RSG_OK;
    auto chk = [&](rsg_status r) {
        if (s == RSG_OK) s = r;
    };
    chk(upload(ctx, &p->xyz, xyz, size_t(n_nodes) * 3));
    chk(upload(ctx, &p->tets, tets, size_t(n_tets) * 4));
    chk(upload(ctx, &p->tris, n_tris ? tris : nullptr, size_t(n_tris) * 3));
    chk(upload(ctx, &p->book, book, size_t(n_nodes) * dofs));
    chk(upload(ctx, &p->row_node, H.row_node.data(), H.row_node.size()));
    chk(upload(ctx, &p->row_comp, H.row_comp.data(), H.row_comp.size()));
    chk(upload(ctx, &p->rp, H.rp.data(), H.rp.size()));
    chk(upload(ctx, &p->ci, H.ci.data(), H.ci.size()));
    chk(upload(ctx, &p->adj_ptr, H.adj_ptr.data(), H.adj_ptr.size()));
    chk(upload(ctx, &p->adj_elem, H.adj_elem.data(), H.adj_elem.size()));
    chk(upload(ctx, &p->adj_loc, H.adj_loc.data(), H.adj_loc.size()));
    chk(upload(ctx, &p->adj_off, H.adj_off.data(), H.adj_off.size()));
    chk(upload(ctx, &p->tadj_ptr, H.tadj_ptr.data(), H.tadj_ptr.size()));
    chk(upload(ctx, &p->tadj_tri, H.tadj_tri.empty() ? nullptr : H.tadj_tri.data(), H.tadj_tri.size()));
    chk(upload(ctx, &p->node_mask, H.node_mask.data(), H.node_mask.size()));
    if (s == RSG_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) s = set_error(ctx, RSG_ERR_CUDA, "assembly upload: %s", cudaGetErrorString(e));
    }
    if (s != RSG_OK) {
        free_plan(p);
        return s;
    }
    *out = p;
    return RSG_OK;
}

// Stage host arrays on the device; returns device pointers in the same order.
rsg_status stage_inputs(rsg_context *ctx, rsg_assembly *p, int32_t memory, std::initializer_list<size_t> counts,
                        std::initializer_list<const double *> srcs, const double **dst)
{
    if (memory == RSG_MEM_DEVICE) {
        size_t k = 0;
        for (const double *s : srcs) dst[k++] = s;
        return RSG_OK;
    }
    size_t total = 0;
    for (size_t c : counts) total += (c + 31) & ~size_t(31);
    if (total > p->stage_cap) {
        if (p->stage) {
            RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(p->stage);
        }
        p->stage = nullptr;
        RSG_CHECK_CUDA(ctx, cudaMalloc(&p->stage, total * sizeof(double)));
        p->stage_cap = total;
    }
    size_t o = 0, k = 0;
    auto ci = counts.begin();
    for (const double *s : srcs) {
        const size_t c = *ci++;
        if (s) {
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(p->stage + o, s, c * sizeof(double), cudaMemcpyHostToDevice,
                                                ctx->stream));
            dst[k] = p->stage + o;
        } else {
            dst[k] = nullptr;
        }
        k++;
        o += (c + 31) & ~size_t(31);
    }
    return RSG_OK;
}

// Create *A from the plan pattern on the first call; afterwards write into its values.
template <class Launch>
rsg_status assemble_into(rsg_context *ctx, rsg_assembly *p, rsg_csr **A, Launch launch)
{
    if (*A) {
        if ((*A)->n != p->n_free || (*A)->nnz != p->nnz)
            return set_error(ctx, RSG_ERR_INVALID_ARG, "assemble: matrix does not match the plan's pattern");
        launch((*A)->val);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        return csr_refresh(ctx, *A);
    }
    double *tmp = nullptr;
    RSG_CHECK_CUDA(ctx, cudaMalloc(&tmp, std::max<size_t>(p->nnz, 1) * sizeof(double)));
    launch(tmp);
    cudaError_t e = cudaGetLastError();
    rsg_status s = e == cudaSuccess ? RSG_OK : set_error(ctx, RSG_ERR_CUDA, "assemble: %s", cudaGetErrorString(e));
    if (s == RSG_OK) s = rsg_csr_create(ctx, p->n_free, p->rp, p->ci, tmp, RSG_MEM_DEVICE, A);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(tmp);
    return s;
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_assembly_create_heat(rsg_context *ctx, uint32_t n_nodes, const double *xyz, uint32_t n_tets,
                                    const uint32_t *tets, const uint32_t *book, uint32_t n_free, rsg_assembly **out)
{
    const rsg_status s = create_plan(ctx, n_nodes, xyz, n_tets, tets, 0, nullptr, book, 1, n_free, out);
    if (s == RSG_OK) (*out)->kind = kPlanHeat;
    return s;
}

rsg_status rsg_assembly_create_stress(rsg_context *ctx, uint32_t n_nodes, const double *xyz, uint32_t n_tets,
                                      const uint32_t *tets, uint32_t n_tris, const uint32_t *tris,
                                      const uint32_t *book, uint32_t n_free, rsg_assembly **out)
{
    const rsg_status s = create_plan(ctx, n_nodes, xyz, n_tets, tets, n_tris, tris, book, 3, n_free, out);
    if (s == RSG_OK) (*out)->kind = kPlanStress;
    return s;
}

rsg_status rsg_assembly_create_magnetostatics(rsg_context *ctx, uint32_t n_nodes, const double *xyz,
                                              uint32_t n_tets, const uint32_t *tets, const uint32_t *book,
                                              uint32_t n_free, rsg_assembly **out)
{
    if (!ctx || !book || !out) return set_error(ctx, RSG_ERR_INVALID_ARG, "assembly_create_magnetostatics: bad arguments");
    // one node book position per node (src/rsolvermagnetostatics.cpp:245, :261): the three
    // potential components of a node are enabled or disabled together, at 3 * position + c
    for (uint32_t nd = 0; nd < n_nodes; nd++) {
        const int eod = int(book[3 * size_t(nd)] == RSG_EOD) + int(book[3 * size_t(nd) + 1] == RSG_EOD) +
                        int(book[3 * size_t(nd) + 2] == RSG_EOD);
        if (eod != 0 && eod != 3)
            return set_error(ctx, RSG_ERR_INVALID_ARG,
                             "assembly_create_magnetostatics: node %u has some but not all components disabled", nd);
        const uint32_t p0 = book[3 * size_t(nd)];
        if (eod == 0 && (p0 % 3 != 0 || book[3 * size_t(nd) + 1] != p0 + 1 || book[3 * size_t(nd) + 2] != p0 + 2))
            return set_error(ctx, RSG_ERR_INVALID_ARG,
                             "assembly_create_magnetostatics: node %u: components must sit at 3*position + c", nd);
    }
    const rsg_status s = create_plan(ctx, n_nodes, xyz, n_tets, tets, 0, nullptr, book, 3, n_free, out);
    if (s == RSG_OK) (*out)->kind = kPlanMagnetostatics;
    return s;
}

void rsg_assembly_destroy(rsg_context *ctx, rsg_assembly *plan)
{
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    free_plan(plan);
}

rsg_status rsg_assembly_info(const rsg_assembly *plan, uint32_t *n_free, uint64_t *nnz)
{
    if (!plan) return RSG_ERR_INVALID_ARG;
    if (n_free) *n_free = plan->n_free;
    if (nnz) *nnz = plan->nnz;
    return RSG_OK;
}

rsg_status rsg_assemble_heat(rsg_context *ctx, rsg_assembly *p, const double *k_e, const double *q_e,
                             const double *rhoc_e, const double *node_t, const rsg_time *time, int32_t memory,
                             rsg_csr **A, double *b_device)
{
    if (!ctx || !p || !k_e || !q_e || !node_t || !A || !b_device || p->kind != kPlanHeat)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assemble_heat: bad arguments");
    const bool transient = time && time->transient;
    if (transient && !rhoc_e) return set_error(ctx, RSG_ERR_INVALID_ARG, "assemble_heat: transient needs rhoc_e");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const double *d[4];
    RSG_TRY(stage_inputs(ctx, p, memory, {p->n_tets, p->n_tets, p->n_tets, p->n_nodes},
                         {k_e, q_e, transient ? rhoc_e : nullptr, node_t}, d));
    const double alpha = time ? time->alpha : 1.0, dt = time ? time->dt : 0.0;
    const bool local = p->max_row <= kLocalRowMax && !row_threads_forced();
    auto kern = local ? k_asm_heat_local : k_asm_heat;
    // shared memory for the plan's longest row only (15 entries on tet meshes of structured hexes)
    const size_t smem = local ? size_t(std::max<uint32_t>(p->max_row, 1)) * kBlock * sizeof(double) : 0;
    if (local)
        RSG_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_asm_heat_local, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(kHeatLocalSmem)));
    const int grid = std::min(grid_for(ctx, (const void *)kern, kBlock, smem, p->n_free), kMaxGrid * 4);
    return assemble_into(ctx, p, A, [&](double *val) {
        kern<<<grid, kBlock, smem, ctx->stream>>>(p->n_free, p->row_node, p->rp, p->adj_ptr, p->adj_elem, p->adj_loc,
                                              reinterpret_cast<const ushort4 *>(p->adj_off), p->xyz,
                                              reinterpret_cast<const uint4 *>(p->tets), p->book, d[0], d[1], d[2],
                                              d[3], transient ? 1 : 0, alpha, dt, val, b_device);
    });
}

rsg_status rsg_assemble_stress(rsg_context *ctx, rsg_assembly *p, const double *e_mod, const double *nu,
                               const double *rho_e, const double *gravity, const double *texp_e,
                               const double *dtemp_e, const double *traction, const double *node_u,
                               const rsg_time *time, int32_t memory, rsg_csr **A, double *b_device)
{
    if (!ctx || !p || !e_mod || !nu || !rho_e || !gravity || !texp_e || !dtemp_e || !node_u || !A || !b_device ||
        p->kind != kPlanStress || (p->n_tris && !traction))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assemble_stress: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const bool transient = time && time->transient;
    const double *d[8];
    RSG_TRY(stage_inputs(ctx, p, memory,
                         {p->n_tets, p->n_tets, p->n_tets, 3, p->n_tets, p->n_tets, size_t(p->n_tris) * 3,
                          size_t(p->n_nodes) * 3},
                         {e_mod, nu, rho_e, gravity, texp_e, dtemp_e, p->n_tris ? traction : nullptr, node_u}, d));
    const double alpha = time ? time->alpha : 1.0, dt = time ? time->dt : 0.0;
    const bool local = p->max_row <= kLocalStressRowMax && !row_threads_forced();
    auto kern = local ? k_asm_stress_local : k_asm_stress;
    const int block = kStressBlock;
    const size_t smem = local ? size_t(std::max<uint32_t>(p->max_row, 1)) * block * sizeof(double) : 0;
    if (local)
        RSG_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_asm_stress_local, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(kStressLocalSmemMax)));
    const int grid = std::min(grid_for(ctx, (const void *)kern, block, smem, p->n_free), kMaxGrid * 4);
    return assemble_into(ctx, p, A, [&](double *val) {
        kern<<<grid, block, smem, ctx->stream>>>(
            p->n_free, p->row_node, p->row_comp, p->rp, p->adj_ptr, p->adj_elem, p->adj_loc,
            reinterpret_cast<const ushort4 *>(p->adj_off), p->tadj_ptr, p->tadj_tri, p->node_mask, p->xyz,
            reinterpret_cast<const uint4 *>(p->tets), p->tris, p->book, d[0], d[1], d[2], d[3], d[4], d[5], d[6],
            d[7], transient ? 1 : 0, alpha, dt, val, b_device);
    });
}

rsg_status rsg_assemble_magnetostatics(rsg_context *ctx, rsg_assembly *p, const double *node_j,
                                       const double *node_a, int32_t memory, rsg_csr **A, double *b_device)
{
    if (!ctx || !p || !node_j || !node_a || !A || !b_device || p->kind != kPlanMagnetostatics)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assemble_magnetostatics: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const double *d[2];
    RSG_TRY(stage_inputs(ctx, p, memory, {size_t(p->n_nodes) * 3, size_t(p->n_nodes) * 3}, {node_j, node_a}, d));
    const int block = kStressBlock;
    if (p->max_row <= kLocalStressRowMax && !row_threads_forced()) {
        const uint32_t nodes = p->n_free / 3;
        const size_t smem = size_t(std::max<uint32_t>(p->max_row / 3, 1)) * block * sizeof(double);
        const int grid = std::min(grid_for(ctx, (const void *)k_asm_magneto_node, block, smem, nodes), kMaxGrid * 4);
        return assemble_into(ctx, p, A, [&](double *val) {
            k_asm_magneto_node<<<grid, block, smem, ctx->stream>>>(
                nodes, p->row_node, p->rp, p->adj_ptr, p->adj_elem, p->adj_loc,
                reinterpret_cast<const ushort4 *>(p->adj_off), p->xyz, reinterpret_cast<const uint4 *>(p->tets),
                p->book, d[0], d[1], val, b_device);
        });
    }
    const int grid = std::min(grid_for(ctx, (const void *)k_asm_magneto, block, 0, p->n_free), kMaxGrid * 4);
    return assemble_into(ctx, p, A, [&](double *val) {
        k_asm_magneto<<<grid, block, 0, ctx->stream>>>(p->n_free, p->row_node, p->row_comp, p->rp, p->adj_ptr,
                                                       p->adj_elem, p->adj_loc,
                                                       reinterpret_cast<const ushort4 *>(p->adj_off), p->node_mask,
                                                       p->xyz, reinterpret_cast<const uint4 *>(p->tets), p->book,
                                                       d[0], d[1], val, b_device);
    });
}

rsg_status rsg_assembly_scatter(rsg_context *ctx, const rsg_assembly *p, const double *x_device,
                                double *node_values_device)
{
    if (!ctx || !p || !x_device || !node_values_device)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "assembly_scatter: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t ne = p->n_nodes * p->dofs;
    const int grid = std::min(grid_for(ctx, (const void *)k_asm_scatter, kBlock, 0, ne), kMaxGrid);
    k_asm_scatter<<<grid, kBlock, 0, ctx->stream>>>(ne, p->book, x_device, node_values_device);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

}  // extern "C"
