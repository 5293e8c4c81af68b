// Eigenvalue drivers of the pencil (M, K): REigenValueSolver's Lanczos, Arnoldi and Rayleigh
// quotient methods (src/reigenvaluesolver.cpp:40-110, 119-392, 420-592) on the GPU.
//
// Each method is a short sequence of solves with K (or a shifted matrix) and vector operations; the
// solves are rsg_solve with the caller's configuration and Jacobi, every vector stays on the device,
// and only the handful of scalars each step produces (a dot product, a norm) cross to the host,
// where the reference's scalar recurrences run unchanged.  Vector updates use separately rounded
// multiplies and adds (no fused multiply-add), as the reference's loops compute them; dot products
// and norms are reduced in a fixed order (deterministic, not the reference's serial order, so they
// agree to rounding).
//
// What the reference does and this file keeps:
// - Lanczos (:119-210): K w = M v - e_i K v_old, d_i = w.v, w -= d_i v, e_{i+1} = |w|, v = w / e_{i+1};
//   then qlDecomposition (:420-497), whose split test always ends the sweep before any rotation
//   (m starts at l, and the loop leaves when m >= l), so d is returned as the Lanczos diagonal;
// - Arnoldi (:211-294): K q = M q_{i-1}, modified Gram-Schmidt against the stored basis, Hessenberg H;
//   then the unshifted QR iteration of qrDecomposition (:499-592) and ev = (Q_a Q_qr)^T;
// - Rayleigh (:295-392): (M + mu K) c = (mu K) b, b <- M^{-1} (mu K b / |c|), K d = M b,
//   mu = d.b / b.b until |mu - mu_old| < cvg; the shifted matrix is updated in place by adding and
//   then subtracting mu K, as the reference does;
// - the post-processing of solve (:90-110) for more than one value: d_i <- |1 / d_i|, the first two
//   swapped, then sorted ascending with the eigenvectors reordered alike.
#include "krylov.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace rsg {
namespace {

constexpr int kEigBlock = 256;
constexpr int kEigPartials = 1024;

__global__ void k_eig_copy_scaled(uint32_t n, const double *__restrict__ x, double s, int divide,
                                  double *__restrict__ y)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = divide ? __ddiv_rn(x[i], s) : __dmul_rn(x[i], s);
}

// y_i = y_i - a x_i (the product rounded, then the difference)
__global__ void k_eig_axmy(uint32_t n, double a, const double *__restrict__ x, double *__restrict__ y)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(a, x[i]));
}

// y_i = y_i - (x_i a) (the reference scales a temporary vector, then subtracts it)
__global__ void k_eig_sub_scaled(uint32_t n, const double *__restrict__ x, double a, double *__restrict__ y)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = __dsub_rn(y[i], __dmul_rn(x[i], a));
}

// partial[b] = sum of x_i y_i over block b's grid-stride share, tree-reduced in a fixed order
__global__ void __launch_bounds__(kEigBlock) k_eig_dot_partial(uint32_t n, const double *__restrict__ x,
                                                               const double *__restrict__ y,
                                                               double *__restrict__ partial)
{
    __shared__ double s[kEigBlock];
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc = __dadd_rn(acc, __dmul_rn(x[i], y[i]));
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kEigBlock / 2; o > 0; o >>= 1) {
        if (int(threadIdx.x) < o) s[threadIdx.x] = __dadd_rn(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kEigBlock) k_eig_dot_final(int m, const double *__restrict__ partial,
                                                             double *__restrict__ out)
{
    __shared__ double s[kEigBlock];
    double acc = 0.0;
    for (int i = threadIdx.x; i < m; i += kEigBlock) acc = __dadd_rn(acc, partial[i]);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kEigBlock / 2; o > 0; o >>= 1) {
        if (int(threadIdx.x) < o) s[threadIdx.x] = __dadd_rn(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// Rayleigh: f_i = sum over row i of (k_ij mu) b_j (column order, products and sums rounded apart;
// mu = 1 uses the values as they are)
__global__ void k_eig_scaled_rowsum(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                                    const double *__restrict__ val, double mu, const double *__restrict__ b,
                                    double *__restrict__ f)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            const double v = mu == 1.0 ? val[j] : __dmul_rn(val[j], mu);
            acc = __dadd_rn(acc, __dmul_rn(v, b[ci[j]]));
        }
        f[i] = acc;
    }
}

// Rayleigh: m2_j += sign * (k_j mu) where that value is not zero
__global__ void k_eig_shift(uint64_t nnz, const double *__restrict__ kval, double mu, double sign,
                            double *__restrict__ m2)
{
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < nnz; j += uint64_t(gridDim.x) * blockDim.x) {
        const double v = __dmul_rn(__dmul_rn(sign, kval[j]), mu);
        if (v != 0.0) m2[j] = __dadd_rn(m2[j], v);
    }
}

// out (n x m, column-major) = Q (n x m, column-major) x R (m x m, row-major): the eigenvectors of
// the Arnoldi basis, sums over the m columns in index order
__global__ void k_eig_basis_mul(uint32_t n, uint32_t m, const double *__restrict__ Q, const double *__restrict__ R,
                                double *__restrict__ out)
{
    const uint64_t total = uint64_t(n) * m;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t i = uint32_t(t % n), c = uint32_t(t / n);
        double acc = 0.0;
        for (uint32_t k = 0; k < m; k++) acc = __dadd_rn(acc, __dmul_rn(Q[size_t(k) * n + i], R[size_t(k) * m + c]));
        out[size_t(c) * n + i] = acc;
    }
}

int vec_grid(const rsg_context *ctx, uint64_t n)
{
    return int(std::max<uint64_t>(1, std::min<uint64_t>((n + kEigBlock - 1) / kEigBlock, uint64_t(ctx->num_sms) * 8)));
}

// Device scratch of the drivers, freed on every exit path.
struct EigWork {
    std::vector<double *> bufs;
    ~EigWork()
    {
        for (double *p : bufs) cudaFree(p);
    }
    double *take(size_t count)
    {
        double *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(double)) != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return p;
    }
};

struct Eig {
    rsg_context *ctx;
    uint32_t n;
    double *partial, *scalar, *scalar_h;
    uint32_t solves = 0;
    uint64_t iterations = 0;

    rsg_status dot(const double *x, const double *y, double *out)
    {
        const int g = std::min(vec_grid(ctx, n), kEigPartials);
        k_eig_dot_partial<<<g, kEigBlock, 0, ctx->stream>>>(n, x, y, partial);
        k_eig_dot_final<<<1, kEigBlock, 0, ctx->stream>>>(g, partial, scalar);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(scalar_h, scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *out = *scalar_h;
        return RSG_OK;
    }
    rsg_status norm(const double *x, double *out)
    {
        double s = 0.0;
        RSG_TRY(dot(x, x, &s));
        *out = std::sqrt(s);
        return RSG_OK;
    }
    void scale(const double *x, double s, bool divide, double *y)
    {
        k_eig_copy_scaled<<<vec_grid(ctx, n), kEigBlock, 0, ctx->stream>>>(n, x, s, divide ? 1 : 0, y);
    }
    void axmy(double a, const double *x, double *y)
    {
        k_eig_axmy<<<vec_grid(ctx, n), kEigBlock, 0, ctx->stream>>>(n, a, x, y);
    }
    rsg_status solve(rsg_csr *A, const rsg_solver_conf *conf, const double *b, double *x)
    {
        rsg_stats st{};
        RSG_TRY(rsg_solve(ctx, A, conf, RSG_PREC_JACOBI, 1, b, x, RSG_MEM_DEVICE, &st));
        solves++;
        iterations += st.iterations;
        return RSG_OK;
    }
};

// The unshifted QR iteration of an m x m matrix by Gram-Schmidt (qrDecomposition,
// src/reigenvaluesolver.cpp:499-592): A_{k+1} = R_k Q_k, V = Q_0 Q_1 ..., until every subdiagonal
// entry is at most cvg or n_iterations sweeps ran; d = diag(A).  Row-major dense arrays.
rsg_status qr_iteration(rsg_context *ctx, uint32_t m, std::vector<double> A, uint32_t n_iterations, double cvg,
                        std::vector<double> &d, std::vector<double> &V)
{
    std::vector<double> Q(size_t(m) * m, 0.0), R(size_t(m) * m, 0.0), T(size_t(m) * m), a(m), e(m), u(m);
    V.assign(size_t(m) * m, 0.0);
    auto at = [m](std::vector<double> &X, uint32_t r, uint32_t c) -> double & { return X[size_t(r) * m + c]; };
    auto dotv = [m](const std::vector<double> &x, const std::vector<double> &y) {
        double s = 0.0;
        for (uint32_t k = 0; k < m; k++) s += x[k] * y[k];
        return s;
    };
    auto mul = [&](std::vector<double> &X, std::vector<double> &Y, std::vector<double> &Z) {  // Z = X Y
        for (uint32_t r = 0; r < m; r++)
            for (uint32_t c = 0; c < m; c++) {
                double s = 0.0;
                for (uint32_t k = 0; k < m; k++) s += at(X, r, k) * at(Y, k, c);
                at(Z, r, c) = s;
            }
    };
    for (uint32_t it = 0; it < n_iterations; it++) {
        for (uint32_t i = 0; i < m; i++) {  // Q: orthonormalised columns of A (classical Gram-Schmidt)
            for (uint32_t j = 0; j < m; j++) a[j] = at(A, j, i);
            u = a;
            for (uint32_t j = 0; j < i; j++) {
                for (uint32_t k = 0; k < m; k++) e[k] = at(Q, k, j);
                const double p = dotv(a, e);
                for (uint32_t k = 0; k < m; k++) u[k] -= p * e[k];
            }
            double nu = 0.0;
            for (uint32_t k = 0; k < m; k++) nu += u[k] * u[k];
            nu = std::sqrt(nu);
            if (nu == 0.0) return set_error(ctx, RSG_ERR_SINGULAR, "eigen: QR iteration met a dependent column");
            for (uint32_t k = 0; k < m; k++) at(Q, k, i) = u[k] * (1.0 / nu);
        }
        for (uint32_t i = 0; i < m; i++) {  // R = Q^T A, upper triangle
            for (uint32_t j = 0; j < m; j++) e[j] = at(Q, j, i);
            for (uint32_t j = i; j < m; j++) {
                for (uint32_t k = 0; k < m; k++) a[k] = at(A, k, j);
                at(R, i, j) = dotv(a, e);
            }
        }
        mul(R, Q, A);
        if (it == 0) {
            V = Q;
        } else {
            mul(V, Q, T);
            V = T;
        }
        bool done = true;
        for (uint32_t i = 1; i < m; i++)
            if (std::fabs(at(A, i, i - 1)) > cvg) done = false;
        if (done) break;
    }
    d.resize(m);
    for (uint32_t i = 0; i < m; i++) d[i] = at(A, i, i);
    return RSG_OK;
}

// solve()'s post-processing for more than one value (src/reigenvaluesolver.cpp:90-110): |1 / d_i|,
// the first two swapped, sorted ascending (ties keep their order); order receives the permutation.
void invert_and_sort(std::vector<double> &d, std::vector<uint32_t> &order)
{
    for (double &v : d) v = std::fabs(1.0 / v);
    std::swap(d[0], d[1]);
    order.resize(d.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return d[a] < d[b]; });
    std::vector<double> s(d.size());
    for (size_t i = 0; i < d.size(); i++) s[i] = d[order[i]];
    d = s;
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" rsg_status rsg_eigen_solve(rsg_context *ctx, const rsg_csr *M, rsg_csr *K, const rsg_eigen_conf *ec,
                                      const rsg_solver_conf *conf, const double *start, double *values,
                                      double *vectors, rsg_eigen_stats *stats)
{
    if (!ctx || !M || !K || !ec || !conf || !start || !values)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "eigen_solve: bad arguments");
    if (M->n != K->n) return set_error(ctx, RSG_ERR_INVALID_ARG, "eigen_solve: M and K differ in size");
    const uint32_t n = K->n;
    const int method = ec->method;
    if (method != RSG_EIGEN_LANCZOS && method != RSG_EIGEN_ARNOLDI && method != RSG_EIGEN_RAYLEIGH)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "eigen_solve: unknown method %d", method);
    const uint32_t ne = method == RSG_EIGEN_RAYLEIGH ? 1u : std::min(ec->n_eigen, n);
    if (ne == 0) return set_error(ctx, RSG_ERR_INVALID_ARG, "eigen_solve: no eigenvalue asked for");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    EigWork W;
    Eig E{ctx, n, W.take(kEigPartials), W.take(1), nullptr};
    double scalar_h = 0.0;
    E.scalar_h = &scalar_h;
    const size_t vb = size_t(n);
    double *v = W.take(vb), *vo = W.take(vb), *w = W.take(vb), *b = W.take(vb), *t = W.take(vb);
    if (!E.partial || !E.scalar || !v || !vo || !w || !b || !t)
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "eigen_solve: vectors");
    cudaStream_t s = ctx->stream;
    const int gv = vec_grid(ctx, n);
    // the start vector, normalised (v / |v|)
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(t, start, vb * sizeof(double), cudaMemcpyHostToDevice, s));
    double nv = 0.0;
    RSG_TRY(E.norm(t, &nv));
    if (nv == 0.0) return set_error(ctx, RSG_ERR_INVALID_ARG, "eigen_solve: zero start vector");
    E.scale(t, nv, true, v);
    std::vector<double> d, vec;  // vec: ne x n eigenvectors (row-major), when the method has them

    if (method == RSG_EIGEN_LANCZOS) {
        std::vector<double> e(ne + 1, 0.0);
        d.assign(ne, 0.0);
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(vo, 0, vb * sizeof(double), s));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(w, 0, vb * sizeof(double), s));
        for (uint32_t i = 0; i < ne; i++) {
            RSG_TRY(rsg_spmv(ctx, M, v, b));  // b = M v
            if (i > 0) {                      // b -= e_i (K v_old)
                RSG_TRY(rsg_spmv(ctx, K, vo, t));
                k_eig_sub_scaled<<<gv, kEigBlock, 0, s>>>(n, t, e[i], b);
            }
            RSG_TRY(E.solve(K, conf, b, w));  // K w = b, from the previous w
            RSG_TRY(E.dot(w, v, &d[i]));
            if (i + 1 < ne) {
                E.axmy(d[i], v, w);
                RSG_TRY(E.norm(w, &e[i + 1]));
                if (e[i + 1] == 0.0) return set_error(ctx, RSG_ERR_SINGULAR, "eigen: Lanczos breakdown at step %u", i);
                RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(vo, v, vb * sizeof(double), cudaMemcpyDeviceToDevice, s));
                E.scale(w, e[i + 1], true, v);
            }
        }
        // qlDecomposition leaves d as it is (its split test ends every sweep before a rotation)
    } else if (method == RSG_EIGEN_ARNOLDI) {
        double *Qa = W.take(vb * ne), *Qq = W.take(size_t(ne) * ne), *ev = W.take(vb * ne);
        if (!Qa || !Qq || !ev) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "eigen_solve: Arnoldi basis");
        std::vector<double> H(size_t(ne) * ne, 0.0);
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(Qa, v, vb * sizeof(double), cudaMemcpyDeviceToDevice, s));
        double *q = v;  // the start vector is the first solve's initial guess, as in the reference
        for (uint32_t i = 1; i <= ne; i++) {
            RSG_TRY(rsg_spmv(ctx, M, Qa + size_t(i - 1) * n, b));  // f = M q_{i-1}
            RSG_TRY(E.solve(K, conf, b, q));                         // K q = f
            for (uint32_t j = 0; j < i; j++) {                        // modified Gram-Schmidt
                double h = 0.0;
                RSG_TRY(E.dot(Qa + size_t(j) * n, q, &h));
                H[size_t(j) * ne + (i - 1)] = h;
                E.axmy(h, Qa + size_t(j) * n, q);
            }
            if (i < ne) {
                double h = 0.0;
                RSG_TRY(E.norm(q, &h));
                if (h == 0.0) return set_error(ctx, RSG_ERR_SINGULAR, "eigen: Arnoldi breakdown at step %u", i);
                H[size_t(i) * ne + (i - 1)] = h;
                E.scale(q, h, true, Qa + size_t(i) * n);
            }
        }
        std::vector<double> V;
        RSG_TRY(qr_iteration(ctx, ne, H, ec->n_iterations, ec->cvg, d, V));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(Qq, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        k_eig_basis_mul<<<vec_grid(ctx, uint64_t(n) * ne), kEigBlock, 0, s>>>(n, ne, Qa, Qq, ev);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        vec.resize(vb * ne);  // column c of (Qa Qq) is eigenvector row c after the transpose
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(vec.data(), ev, vec.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    } else {  // Rayleigh quotient iteration
        if (M->nnz != K->nnz) return set_error(ctx, RSG_ERR_UNSUPPORTED, "eigen: Rayleigh needs M and K on one pattern");
        {
            std::vector<uint32_t> rm(size_t(n) + 1), rk(size_t(n) + 1), cm(M->nnz), ck(K->nnz);
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(rm.data(), M->rp, rm.size() * 4, cudaMemcpyDeviceToHost, s));
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(rk.data(), K->rp, rk.size() * 4, cudaMemcpyDeviceToHost, s));
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(cm.data(), M->ci, cm.size() * 4, cudaMemcpyDeviceToHost, s));
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ck.data(), K->ci, ck.size() * 4, cudaMemcpyDeviceToHost, s));
            RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
            if (rm != rk || cm != ck)
                return set_error(ctx, RSG_ERR_UNSUPPORTED, "eigen: Rayleigh needs M and K on one pattern");
        }
        rsg_csr *M2 = nullptr;  // M + mu K, updated in place
        RSG_TRY(rsg_csr_create(ctx, n, M->rp, M->ci, M->val, RSG_MEM_DEVICE, &M2));
        struct Drop {
            rsg_context *c;
            rsg_csr *a;
            ~Drop() { rsg_csr_destroy(c, a); }
        } drop{ctx, M2};
        double *m2 = W.take(M->nnz), *c = W.take(vb), *dd = W.take(vb), *f = W.take(vb);
        if (!m2 || !c || !dd || !f) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "eigen_solve: Rayleigh vectors");
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(m2, M->val, size_t(M->nnz) * sizeof(double), cudaMemcpyDeviceToDevice, s));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(c, 0, vb * sizeof(double), s));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(dd, 0, vb * sizeof(double), s));
        double *bb = v;  // b: the normalised start vector
        double mu = ec->mu0;
        const int ge = vec_grid(ctx, M->nnz);
        for (uint32_t it = 0; it < ec->n_iterations; it++) {
            const double muo = mu;
            k_eig_shift<<<ge, kEigBlock, 0, s>>>(M->nnz, K->val, mu, 1.0, m2);  // M2 += mu K
            k_eig_scaled_rowsum<<<gv, kEigBlock, 0, s>>>(n, K->rp, K->ci, K->val, mu, bb, f);
            RSG_TRY(rsg_csr_update_values(ctx, M2, m2, RSG_MEM_DEVICE));
            RSG_TRY(E.solve(M2, conf, f, c));  // (M + mu K) c = mu K b
            double nc = 0.0;
            RSG_TRY(E.norm(c, &nc));
            if (nc == 0.0) return set_error(ctx, RSG_ERR_SINGULAR, "eigen: Rayleigh iterate vanished");
            E.scale(f, 1.0 / nc, false, f);
            RSG_TRY(E.solve(const_cast<rsg_csr *>(M), conf, f, bb));  // M b = f / |c|
            k_eig_shift<<<ge, kEigBlock, 0, s>>>(M->nnz, K->val, mu, -1.0, m2);  // M2 -= mu K
            k_eig_scaled_rowsum<<<gv, kEigBlock, 0, s>>>(n, M->rp, M->ci, m2, 1.0, bb, f);  // f = M2 b
            RSG_CHECK_CUDA(ctx, cudaGetLastError());
            RSG_TRY(E.solve(K, conf, f, dd));  // K d = f
            double bdb = 0.0, ddb = 0.0;
            RSG_TRY(E.dot(bb, bb, &bdb));
            if (bdb == 0.0) return set_error(ctx, RSG_ERR_SINGULAR, "eigen: Rayleigh iterate vanished");
            RSG_TRY(E.dot(dd, bb, &ddb));
            mu = ddb / bdb;
            if (it > 0 && std::fabs(muo - mu) < ec->cvg) break;
        }
        d.assign(1, mu);
        vec.resize(vb);
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(vec.data(), bb, vb * sizeof(double), cudaMemcpyDeviceToHost, s));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    }
    RSG_CHECK_CUDA(ctx, cudaGetLastError());

    std::vector<uint32_t> order(d.size());
    std::iota(order.begin(), order.end(), 0u);
    if (d.size() > 1) invert_and_sort(d, order);
    std::copy(d.begin(), d.end(), values);
    if (vectors && !vec.empty()) {
        // eigenvector r (row r of the transposed basis product) in the sorted order
        for (size_t r = 0; r < d.size(); r++)
            std::copy(vec.begin() + order[r] * vb, vec.begin() + (order[r] + 1) * vb, vectors + r * vb);
    }
    if (stats) {
        stats->n_values = uint32_t(d.size());
        stats->solves = E.solves;
        stats->iterations = E.iterations;
    }
    return RSG_OK;
}
