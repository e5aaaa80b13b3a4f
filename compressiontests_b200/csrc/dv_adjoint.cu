// Adjoint sensitivities of a density-parametrised hexahedral cantilever.
//
// Model: on an ne[0] x ne[1] x ne[2] grid of unit cubes (x = 0 face clamped)
// element e has modulus E_e = E0 rho_e^penal, so K(rho) = sum_e rho_e^penal Ke
// with Ke the unit-cube stiffness at modulus E0.  For J(u) with u = K^-1 f:
//
//   dJ/drho_e = -lambda_e^T (dK_e/drho_e) u_e = -penal rho_e^(penal-1) lambda_e^T Ke u_e,
//   K lambda = dJ/du   (K is symmetric, so the adjoint system is the forward one).
//
// Forward builds K(rho), a Galerkin hierarchy of the vertex factor-2
// coarsening and the MG-PCG solver, and solves K u = f.  Backward reuses that
// solver for K lambda = dJ/du (a fresh solve: nothing of the forward
// iterations is stored) and runs the element kernel over the connectivity.
// The reference has no adjoint; the element gradient follows the oracle's
// or_adjoint_element_gradient (same local node order and summation order).
#include "dv_mgpcg.cuh"

#include <cmath>
#include <cstdlib>
#include <vector>

namespace {

// One thread per element.  Ke (24 x 24, VTK corner order) is staged in shared
// memory; the 24 values of u and lambda at the element's dofs are gathered
// (0 at the clamped x = 0 nodes).  s = sum_i lam_i (sum_j Ke_ij u_j) with each
// product rounded before it is added, in the oracle's order.
__global__ void __launch_bounds__(128) k_element_gradient(const double *__restrict__ ke_g, int32_t ne0, int32_t ne1,
                                                          int32_t ne2, const double *__restrict__ rho, double penal,
                                                          int ipenal, const double *__restrict__ u,
                                                          const double *__restrict__ lam, double *__restrict__ grad) {
    __shared__ double ke[576];
    for (int i = threadIdx.x; i < 576; i += blockDim.x) ke[i] = ke_g[i];
    __syncthreads();
    const int64_t nel = (int64_t)ne0 * ne1 * ne2;
    const int32_t nx = ne0 + 1, ny = ne1 + 1;
    const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = (int32_t)(e % ne0), b = (int32_t)((e / ne0) % ne1), c = (int32_t)(e / ((int64_t)ne0 * ne1));
        double ue[24], le[24];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int32_t i = a + off[q][0], j = b + off[q][1], k = c + off[q][2];
            const int64_t f = 3 * ((int64_t)(i - 1) + (int64_t)(nx - 1) * (j + (int64_t)ny * k));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ue[3 * q + d] = i == 0 ? 0.0 : __ldg(u + f + d);
                le[3 * q + d] = i == 0 ? 0.0 : __ldg(lam + f + d);
            }
        }
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 24; ++i) {
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 24; ++j) t = __dadd_rn(t, __dmul_rn(ke[i * 24 + j], ue[j]));
            s = __dadd_rn(s, __dmul_rn(le[i], t));
        }
        const double r = rho[e];
        double g = -penal;
        if (ipenal > 0) {   // integral exponent: (-penal) rho ... rho, one rounding per product
            for (int t = 1; t < ipenal; ++t) g = g * r;
        } else {
            g = g * pow(r, penal - 1.0);
        }
        grad[e] = g * s;
    }
}

int integral_penal(double penal) {
    return (penal >= 1.0 && penal <= 16.0 && penal == std::floor(penal)) ? (int)penal : 0;
}

void launch_element_gradient(dv_context *ctx, const int32_t *ne, const double *d_ke, const double *d_rho, double penal,
                             const double *d_u, const double *d_lam, double *d_grad) {
    const int64_t nel = (int64_t)ne[0] * ne[1] * ne[2];
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nel + 127) / 128, (int64_t)ctx->num_sms * 16));
    k_element_gradient<<<grid, 128, 0, ctx->stream>>>(d_ke, ne[0], ne[1], ne[2], d_rho, penal, integral_penal(penal),
                                                       d_u, d_lam, d_grad);
    DV_CUDA(cudaGetLastError());
    ctx->count();
}

void check_mesh(const int32_t *ne) {
    DV_REQUIRE(ne && ne[0] >= 1 && ne[1] >= 1 && ne[2] >= 1, DV_ERR_ARG, "element counts must be >= 1");
    DV_REQUIRE((int64_t)ne[0] * ne[1] * ne[2] < INT32_MAX, DV_ERR_ARG, "too many elements");
}

struct HostCsrOwned {
    std::vector<int32_t> rp, ci;
    std::vector<double> va;
    int32_t nr = 0, nc = 0;
    dv_csr_host view() const { return dv_csr_host{nr, nc, rp.data(), ci.data(), va.data()}; }
};

}  // namespace

struct dv_adjoint {
    dv_context *ctx = nullptr;
    int32_t ne[3] = {0, 0, 0};
    int64_t nel = 0;
    int32_t n = 0;
    double penal = 3.0;
    dv_mgpcg *solver = nullptr;
    DevMem rho, ke, u, lam, grad, f;
    bool have_u = false;
    bool matrix_free = false;   // finest operator applied element by element (DV_FORMAT_HEX)
    ~dv_adjoint() {
        if (solver) dv_mgpcg_destroy(solver);
    }
};

extern "C" DV_API int dv_hex_element_gradient(dv_context *ctx, const int32_t *ne, const double *d_rho, double penal,
                                              double E0, double nu, const double *d_u, const double *d_lambda,
                                              double *d_grad) {
    return dv_guard([&] {
        DV_REQUIRE(ctx && d_rho && d_u && d_lambda && d_grad, DV_ERR_ARG, "null argument");
        check_mesh(ne);
        dv_ctx_check(ctx);
        std::vector<double> ke(576);
        dv_hex_ke(E0, nu, ke.data());
        DevMem dke(8 * 576);
        DV_CUDA(cudaMemcpyAsync(dke.p, ke.data(), 8 * 576, cudaMemcpyHostToDevice, ctx->stream));
        launch_element_gradient(ctx, ne, dke.as<double>(), d_rho, penal, d_u, d_lambda, d_grad);
        DV_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" DV_API int dv_adjoint_create(dv_context *ctx, const int32_t *ne, const double *rho, double penal, double E0,
                                        double nu, int32_t max_coarse_dofs, const dv_mgpcg_config *cfg,
                                        dv_adjoint **out) {
    return dv_guard([&] {
        DV_REQUIRE(ctx && rho && cfg && out, DV_ERR_ARG, "null argument");
        check_mesh(ne);
        DV_REQUIRE(penal >= 1.0 && E0 > 0 && max_coarse_dofs >= 1, DV_ERR_ARG, "bad material or hierarchy parameters");
        dv_ctx_check(ctx);
        auto s = std::make_unique<dv_adjoint>();
        s->ctx = ctx;
        for (int d = 0; d < 3; ++d) s->ne[d] = ne[d];
        s->nel = (int64_t)ne[0] * ne[1] * ne[2];
        s->penal = penal;
        for (int64_t e = 0; e < s->nel; ++e) DV_REQUIRE(rho[e] > 0.0, DV_ERR_ARG, "densities must be positive");
        // fine stiffness K = sum_e (rho_e^penal) Ke(E0)
        std::vector<double> scale_e(s->nel);
        const int ip = integral_penal(penal);
        for (int64_t e = 0; e < s->nel; ++e) {
            double pw = 1.0;
            if (ip > 0)
                for (int t = 0; t < ip; ++t) pw = pw * rho[e];
            else
                pw = std::pow(rho[e], penal);
            scale_e[e] = pw;
        }
        std::vector<HostCsrOwned> A(1), P;
        {
            int32_t nr;
            int64_t nnz;
            int st = dv_hex_csr_size(ne, &nr, &nnz);
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            A[0].nr = A[0].nc = nr;
            A[0].rp.resize((size_t)nr + 1);
            A[0].ci.resize(nnz);
            A[0].va.resize(nnz);
            st = dv_hex_assemble(ne, scale_e.data(), 1.0, E0, nu, A[0].rp.data(), A[0].ci.data(), A[0].va.data());
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
        }
        s->n = A[0].nr;
        // Galerkin hierarchy of the vertex factor-2 coarsening
        int32_t cur[3] = {ne[0], ne[1], ne[2]};
        while (A.back().nr > max_coarse_dofs && std::max(cur[0], std::max(cur[1], cur[2])) > 1) {
            HostCsrOwned p;
            int32_t nr, nc;
            int64_t nnz;
            int st = dv_hex_trilinear_size(cur, &nr, &nc, &nnz);
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            p.nr = nr;
            p.nc = nc;
            p.rp.resize((size_t)nr + 1);
            p.ci.resize(nnz);
            p.va.resize(nnz);
            st = dv_hex_trilinear(cur, p.rp.data(), p.ci.data(), p.va.data());
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            const dv_csr_host av = A.back().view(), pv = p.view();
            HostCsrOwned g;
            int32_t gn;
            int64_t gnnz;
            st = dv_galerkin_size(&av, &pv, &gn, &gnnz);
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            g.nr = g.nc = gn;
            g.rp.resize((size_t)gn + 1);
            g.ci.resize(gnnz);
            g.va.resize(gnnz);
            st = dv_galerkin(&av, &pv, g.rp.data(), g.ci.data(), g.va.data());
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            P.push_back(std::move(p));
            A.push_back(std::move(g));
            for (int d = 0; d < 3; ++d) cur[d] = (cur[d] + 1) / 2;
        }
        DV_REQUIRE(A.size() >= 2, DV_ERR_ARG, "mesh too small for a hierarchy (raise it or lower max_coarse_dofs)");
        std::vector<dv_csr_host> av, pv;
        for (auto &a : A) av.push_back(a.view());
        for (auto &p : P) pv.push_back(p.view());
        int st = dv_mgpcg_create(ctx, (int32_t)av.size(), av.data(), pv.data(), cfg, &s->solver);
        DV_REQUIRE(st == DV_OK, st, dv_last_error());
        // The finest operator K(rho) has a factor per element and no repeating rows: the solver
        // applies it matrix-free (element kernel) in the outer FP64 loop and in the finest level
        // of the Jacobi V-cycle; the coarse Galerkin levels stay assembled.  DV_MATRIX_FREE=0
        // keeps the assembled operator (A/B comparisons).
        const char *mf = getenv("DV_MATRIX_FREE");
        if (!(mf && mf[0] == '0') && cfg->smoother == DV_SMOOTHER_JACOBI) {
            dv_mgpcg *m = s->solver;
            dv_matrix *h64 = nullptr;
            st = dv_matrix_create_hex(ctx, ne, scale_e.data(), 1.0, E0, nu, DV_F64, &h64);
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            m->Aout.reset(h64);
            if (m->v32) {
                dv_matrix *h32 = nullptr;
                st = dv_matrix_create_hex(ctx, ne, scale_e.data(), 1.0, E0, nu, DV_F32, &h32);
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                m->v32->lv[0].A.reset(h32);
            } else {
                dv_matrix *h = nullptr;
                st = dv_matrix_create_hex(ctx, ne, scale_e.data(), 1.0, E0, nu, DV_F64, &h);
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                m->v64->lv[0].A.reset(h);
            }
            s->matrix_free = true;
        }
        // device copies
        cudaStream_t stream = ctx->stream;
        std::vector<double> ke(576);
        dv_hex_ke(E0, nu, ke.data());
        s->ke.alloc(8 * 576);
        s->rho.alloc(8 * (size_t)s->nel);
        s->u.alloc(8 * (size_t)s->n);
        s->lam.alloc(8 * (size_t)s->n);
        s->f.alloc(8 * (size_t)s->n);
        s->grad.alloc(8 * (size_t)s->nel);
        DV_CUDA(cudaMemcpyAsync(s->ke.p, ke.data(), 8 * 576, cudaMemcpyHostToDevice, stream));
        DV_CUDA(cudaMemcpyAsync(s->rho.p, rho, 8 * (size_t)s->nel, cudaMemcpyHostToDevice, stream));
        DV_CUDA(cudaStreamSynchronize(stream));
        *out = s.release();
    });
}

extern "C" DV_API int dv_adjoint_info(const dv_adjoint *s, int32_t *n_dofs, int64_t *n_elements) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "adjoint problem not created");
        if (n_dofs) *n_dofs = s->n;
        if (n_elements) *n_elements = s->nel;
    });
}

extern "C" DV_API int dv_adjoint_forward(dv_adjoint *s, const double *f, double *u, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "adjoint problem not created");
        DV_REQUIRE(f && u, DV_ERR_ARG, "null argument");
        dv_ctx_check(s->ctx);
        cudaStream_t st = s->ctx->stream;
        const size_t nb = 8 * (size_t)s->n;
        DV_CUDA(cudaMemcpyAsync(s->f.p, f, nb, cudaMemcpyHostToDevice, st));
        int rc = dv_mgpcg_solve_device(s->solver, s->f.as<double>(), s->u.as<double>(), stats);
        DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
        DV_CUDA(cudaMemcpyAsync(u, s->u.p, nb, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
        s->have_u = true;
    });
}

extern "C" DV_API int dv_adjoint_backward(dv_adjoint *s, const double *dJdu, double *dJdrho, double *lambda,
                                          dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "adjoint problem not created");
        DV_REQUIRE(s->have_u, DV_ERR_NOT_INITIALIZED, "call dv_adjoint_forward first");
        DV_REQUIRE(dJdu && dJdrho, DV_ERR_ARG, "null argument");
        dv_ctx_check(s->ctx);
        cudaStream_t st = s->ctx->stream;
        const size_t nb = 8 * (size_t)s->n;
        DV_CUDA(cudaMemcpyAsync(s->f.p, dJdu, nb, cudaMemcpyHostToDevice, st));
        int rc = dv_mgpcg_solve_device(s->solver, s->f.as<double>(), s->lam.as<double>(), stats);
        DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
        launch_element_gradient(s->ctx, s->ne, s->ke.as<double>(), s->rho.as<double>(), s->penal, s->u.as<double>(),
                                s->lam.as<double>(), s->grad.as<double>());
        DV_CUDA(cudaMemcpyAsync(dJdrho, s->grad.p, 8 * (size_t)s->nel, cudaMemcpyDeviceToHost, st));
        if (lambda) DV_CUDA(cudaMemcpyAsync(lambda, s->lam.p, nb, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" DV_API int dv_adjoint_destroy(dv_adjoint *s) {
    return dv_guard([&] {
        if (!s) return;
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
        delete s;
    });
}
