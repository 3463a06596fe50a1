// dfea_newton.cu -- the Newton-Krylov solve driven from C++: load continuation with cut-backs, inexact
// Newton with the Eisenstat-Walker forcing term, Armijo backtracking (the control flow of the reference's
// newton_krylov.py:94-264), over the device kernels of this library.  One call solves one problem; the
// host reads back one scalar per residual evaluation and (status, iterations) per linear solve, and holds
// no interpreter lock while the solve runs, so host threads serving different requests run side by side.
//
// Host arithmetic follows the Python driver of this package operation for operation (pow(x, 0.5) where it
// writes x ** 0.5), so both drivers produce the same iterates bit for bit.
#include <cmath>
#include <cstdio>
#include <utility>

#include "dfea_common.cuh"

namespace dfea {

int validate_mesh(const dfea_mesh_view* mv, bool need_grad32);

// w = fixed ? lf * u_D : u0 per DOF (u_D NULL: zero), the prescribed displacements of a load level
__global__ void k_newton_start(int64_t n_nodes, const uint8_t* __restrict__ node_fix, const double* __restrict__ u_D,
                               double lf, const double* __restrict__ u0, double* __restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const bool fixed = (node_fix[i >> 1] >> (i & 1)) & 1;
        w[i] = fixed ? lf * (u_D ? u_D[i] : 0.0) : u0[i];
    }
}

__global__ void k_negate(int64_t n, const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = -x[i];
}

namespace {

struct Driver {
    const dfea_newton* nw;
    cudaStream_t s;
    int64_t n;          // 2N
    double* R;          // residual of the current iterate
    double* Rc;         // residual of the line-search trial
    double* w;          // the Newton iterate at this load level
    double* uc;         // the line-search trial

    int residual(const double* u, double lf, double* out, double* rn) {
        int rc = dfea_residual_mat(nw->mesh, u, nw->theta, &nw->material, nw->f, lf, out, nw->scal, nullptr,
                                   nw->reduce_work, s);
        if (rc) return rc;
        if ((rc = check_cuda(cudaMemcpyAsync(nw->scal_host, nw->scal, sizeof(double), cudaMemcpyDeviceToHost, s),
                             "cudaMemcpyAsync")) ||
            (rc = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
            return rc;
        *rn = std::pow(nw->scal_host[0], 0.5);
        return DFEA_OK;
    }

    int linearize(const double* u) {
        int rc = dfea_qp_moduli_mat(nw->mesh, u, nw->theta, &nw->material, nw->moduli, nw->moduli_dtype, nw->diag,
                                    nw->blocks, s);
        if (rc || !nw->mg) return rc;
        return dfea_mg_setup(nw->mesh, nw->mg, nw->moduli, nw->moduli_dtype, nw->diag, s);
    }

    // du = PCG(A, -R) to relative tolerance rtol
    int solve(double rtol, int max_iter, int32_t* iters, int32_t* status) {
        k_negate<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(n, R, nw->b);
        note_launches(1);
        int rc = launch_check("dfea_newton_solve: -R");
        if (rc) return rc;
        if (nw->mg)
            return dfea_mg_pcg(nw->mesh, nw->mg, nw->moduli, nw->moduli_dtype, nw->b, nw->du, rtol, max_iter, iters,
                               status, s);
        return dfea_pcg_solve(nw->pcg, rtol, max_iter, iters, status, s);
    }

    // newton_at_load: returns the outcome in *ok; the iterate stays in w
    int at_load(const double* u0, double lf, double tol, int max_newton, int pcg_max_iter, int step_id, bool* ok,
                dfea_newton_info* info, dfea_newton_record* records, int max_records) {
        *ok = false;
        k_newton_start<<<grid_for(n / 2, kThreads, 8), kThreads, 0, s>>>(n / 2, nw->mesh->node_fix, nw->u_D, lf, u0, w);
        note_launches(1);
        int rc = launch_check("dfea_newton_solve: load level");
        double rn;
        if (rc || (rc = residual(w, lf, R, &rn))) return rc;
        const double r0 = rn;
        for (int it = 0; it < max_newton + 1; ++it) {
            if (rn < tol) {
                *ok = true;
                return DFEA_OK;
            }
            if (it == max_newton) break;
            const double eta = std::fmin(0.5, std::pow(rn / (r0 + 1e-14), 0.5));
            const double rtol = nw->min_rtol > 0.0 ? std::fmax(eta, nw->min_rtol) : eta;
            int32_t cg = 0, status = 0;
            if ((rc = linearize(w)) || (rc = solve(rtol, pcg_max_iter, &cg, &status))) return rc;
            // Armijo backtracking: alpha = 1, 1/2, ... >= 2^-5, c1 = 1e-4; NaN rejects the step
            double alpha = 1.0, rn_new = rn;
            bool accepted = false;
            while (alpha >= 0.03125) {
                if ((rc = dfea_add_scaled(n, w, alpha, nw->du, uc, s))) return rc;
                double rn_c;
                if ((rc = residual(uc, lf, Rc, &rn_c))) return rc;
                if (rn_c < (1.0 - 1e-4 * alpha) * rn) {
                    std::swap(R, Rc);
                    std::swap(w, uc);
                    rn_new = rn_c;
                    accepted = true;
                    break;
                }
                alpha *= 0.5;
            }
            rn = rn_new;
            if (info->n_records < max_records && records) {
                dfea_newton_record& r = records[info->n_records];
                r.step = step_id;
                r.iteration = it;
                r.cg_iters = cg;
                r.pcg_status = status;
                r.load_factor = lf;
                r.residual = rn;
                r.alpha = alpha;
                info->n_records++;
            }
            info->total_newton++;
            info->total_cg += cg;
            if (!accepted) return DFEA_OK;
        }
        return DFEA_OK;
    }
};

int validate_newton(const dfea_newton* nw) {
    if (!nw) return set_error(DFEA_ERR_INVALID, "dfea_newton_solve: NULL description");
    int rc = validate_mesh(nw->mesh, false);
    if (rc) return rc;
    if ((nw->pcg == nullptr) == (nw->mg == nullptr))
        return set_error(DFEA_ERR_INVALID, "dfea_newton_solve: give exactly one linear solver (pcg or mg)");
    const void* need[] = {nw->theta, nw->f, nw->u, nw->R, nw->Rc, nw->uc, nw->w, nw->du, nw->b, nw->diag, nw->moduli,
                          nw->reduce_work, nw->scal, nw->scal_host};
    for (const void* p : need)
        if (!p) return set_error(DFEA_ERR_INVALID, "dfea_newton_solve: NULL buffer");
    if (!(nw->min_rtol >= 0.0)) return set_error(DFEA_ERR_INVALID, "dfea_newton_solve: min_rtol must be >= 0");
    return DFEA_OK;
}

}  // namespace
}  // namespace dfea

using namespace dfea;

extern "C" int dfea_newton_solve(const dfea_newton* nw, int32_t n_load_steps, double tol, int32_t max_newton,
                                 int32_t max_cutbacks, int32_t pcg_max_iter, dfea_newton_info* info,
                                 dfea_newton_record* records, int32_t max_records, void* stream) {
    if (!info || n_load_steps < 1 || max_newton < 0 || max_cutbacks < 0 || pcg_max_iter < 1 || max_records < 0 ||
        (max_records > 0 && !records) || !(tol >= 0.0))
        return set_error(DFEA_ERR_INVALID, "dfea_newton_solve: bad arguments");
    int rc = validate_newton(nw);
    if (rc) return rc;
    *info = dfea_newton_info{};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 2 * nw->mesh->n_nodes;
    Driver d{nw, s, n, nw->R, nw->Rc, nw->w, nw->uc};
    // u holds the last accepted state, starting from zero
    if ((rc = check_cuda(cudaMemsetAsync(nw->u, 0, n * sizeof(double), s), "cudaMemsetAsync"))) return rc;
    const double d_nominal = 1.0 / n_load_steps;
    double d_lf = d_nominal, lf = 0.0;
    int step_id = 0, cutbacks_in_row = 0;
    while (lf < 1.0 - 1e-12) {
        const double lf_try = std::fmin(1.0, lf + d_lf);
        ++step_id;
        bool ok = false;
        if ((rc = d.at_load(nw->u, lf_try, tol, max_newton, pcg_max_iter, step_id, &ok, info, records, max_records)))
            return rc;
        if (ok) {
            if ((rc = check_cuda(cudaMemcpyAsync(nw->u, d.w, n * sizeof(double), cudaMemcpyDeviceToDevice, s),
                                 "cudaMemcpyAsync")))
                return rc;
            lf = lf_try;
            cutbacks_in_row = 0;
            d_lf = std::fmin(d_nominal, 1.5 * d_lf);
        } else {
            ++cutbacks_in_row;
            ++info->n_cutbacks;
            if (cutbacks_in_row > max_cutbacks) {
                info->load_factor = lf;
                return check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            }
            d_lf *= 0.5;
        }
    }
    info->converged = 1;
    info->load_factor = 1.0;
    return check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
}
