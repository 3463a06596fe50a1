// dfea_kernels.cu -- mesh packing, kernel (a) (Gauss-point moduli + Jacobi diagonal), the tangent
// product entry point, the FP64 residual / strain energy, norms, kernel (d) (element sensitivity)
// and small vector helpers.  All entry points are `extern "C"` (include/difffea_b200.h).
#include <cstdio>

#include <type_traits>

#include "dfea_apply.cuh"
#include "dfea_common.cuh"
#include "dfea_material.cuh"

namespace dfea {

// ------------------------------------------------------------------------------------------
// validation shared by the entry points
// ------------------------------------------------------------------------------------------
int validate_mesh(const dfea_mesh_view* mv, bool need_grad32) {
    if (mv == nullptr) return set_error(DFEA_ERR_INVALID, "mesh view is NULL");
    if (mv->n_el < 0 || mv->n_nodes <= 0) return set_error(DFEA_ERR_INVALID, "bad sizes n_el=%lld n_nodes=%lld",
                                                             (long long)mv->n_el, (long long)mv->n_nodes);
    if (mv->stride < mv->n_el || mv->stride % 32 != 0)
        return set_error(DFEA_ERR_INVALID, "stride %lld must be a multiple of 32 and >= n_el %lld",
                         (long long)mv->stride, (long long)mv->n_el);
    if (!dfea_element_supported(mv->nen, mv->n_q))
        return set_error(DFEA_ERR_UNSUPPORTED, "element with nen=%d n_q=%d is not built", mv->nen, mv->n_q);
    if (mv->n_colours < 1 || mv->n_colours > DFEA_MAX_COLOURS)
        return set_error(DFEA_ERR_INVALID, "n_colours %d out of [1, %d]", mv->n_colours, DFEA_MAX_COLOURS);
    if (mv->colour_begin[0] != 0 || mv->colour_begin[mv->n_colours] != mv->n_el)
        return set_error(DFEA_ERR_INVALID, "colour ranges must cover [0, n_el)");
    for (int c = 0; c < mv->n_colours; ++c)
        if (mv->colour_begin[c + 1] < mv->colour_begin[c]) return set_error(DFEA_ERR_INVALID, "colour ranges not sorted");
    if (!mv->conn || !mv->orig || !mv->grad || !mv->wdet || !mv->node_fix)
        return set_error(DFEA_ERR_INVALID, "mesh view has a NULL device pointer");
    if (need_grad32 && !mv->grad32) return set_error(DFEA_ERR_INVALID, "FP32 operator needs mesh->grad32");
    if (mv->n_nodes >= (int64_t(1) << 29)) return set_error(DFEA_ERR_INVALID, "too many nodes for the packed connectivity");
    return DFEA_OK;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int validate_material(const dfea_material* mat) {
    if (mat == nullptr) return set_error(DFEA_ERR_INVALID, "material is NULL");
    const int n = material_n_params(mat->model);
    if (n == 0) return set_error(DFEA_ERR_UNSUPPORTED, "material model %d is not built", mat->model);
    if (mat->scalable >> n) return set_error(DFEA_ERR_INVALID, "scalable mask 0x%x names parameters beyond the %d of model %d",
                                             mat->scalable, n, mat->model);
    return DFEA_OK;
}

// The neo-Hookean material with theta scaling both parameters: the legacy (mu0, lambda0) entry points.
static dfea_material neo_hookean(double mu0, double lambda0) {
    dfea_material mt{};
    mt.model = DFEA_MAT_NEO_HOOKEAN;
    mt.scalable = 0x3u;
    mt.p[0] = mu0;
    mt.p[1] = lambda0;
    return mt;
}

// fn(std::bool_constant<GEN>): GEN = the model is evaluated by forward-mode differentiation of its
// energy; neo-Hookean keeps the closed form.
template <typename Fn>
int dispatch_material(const dfea_material& mat, Fn&& fn) {
    if (mat.model == DFEA_MAT_NEO_HOOKEAN) return fn(std::false_type{});
    return fn(std::true_type{});
}

// ------------------------------------------------------------------------------------------
// mesh packing
// ------------------------------------------------------------------------------------------
__global__ void k_pack(int64_t n_el, int64_t S, int nen, int nq, const int64_t* __restrict__ perm,
                       const int64_t* __restrict__ conn_ref, const double* __restrict__ dN,
                       const double* __restrict__ wd, const double* __restrict__ mask,
                       int32_t* __restrict__ conn, int32_t* __restrict__ orig, double* __restrict__ grad,
                       double* __restrict__ wdet) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n_el; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = perm[s];
        orig[s] = (int32_t)o;
        for (int a = 0; a < nen; ++a) {
            const int64_t node = conn_ref[o * nen + a];
            const int fix = (mask[2 * node] == 0.0 ? 1 : 0) | (mask[2 * node + 1] == 0.0 ? 2 : 0);
            conn[a * S + s] = (int32_t)((node << 2) | fix);
        }
        for (int q = 0; q < nq; ++q) {
            wdet[q * S + s] = wd[o * nq + q];
            for (int a = 0; a < nen; ++a) {
                const double* src = dN + ((o * nq + q) * nen + a) * 2;
                reinterpret_cast<double2*>(grad)[(int64_t)(q * nen + a) * S + s] = make_double2(src[0], src[1]);
            }
        }
    }
}

__global__ void k_node_fix(int64_t n_nodes, const double* __restrict__ mask, uint8_t* __restrict__ node_fix) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_nodes; n += (int64_t)gridDim.x * blockDim.x)
        node_fix[n] = (uint8_t)((mask[2 * n] == 0.0 ? 1 : 0) | (mask[2 * n + 1] == 0.0 ? 2 : 0));
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ x, float* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

__global__ void k_to_f64(int64_t n, const float* __restrict__ x, double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (double)x[i];
}

// ------------------------------------------------------------------------------------------
// kernel (a): moduli + element diagonals, one colour per launch
// ------------------------------------------------------------------------------------------
// REF (with CT = float): store the moduli pulled back to the reference frame (DFEA_F32REF layout).
// GEN: moduli of the material's energy by forward-mode differentiation (dfea_material.cuh), else closed-form
// neo-Hookean.
template <int NEN, int NQ, typename CT, bool REF = false, bool GEN = false>
__global__ void __launch_bounds__(128)
k_moduli(Mesh m, int64_t e0, int64_t e1, const double* __restrict__ u, const double* __restrict__ theta,
         dfea_material mat, CT* __restrict__ Cout, double* __restrict__ diag, double* __restrict__ blocks) {
    const int64_t S = m.stride;
    const double2* u2 = reinterpret_cast<const double2*>(u);
    for (int64_t e = e0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < e1; e += (int64_t)gridDim.x * blockDim.x) {
        int node[NEN];
        double ux[NEN], uy[NEN], dx[NEN], dy[NEN], dxy[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            node[a] = m.conn[a * S + e] >> 2;
            const double2 t = __ldg(u2 + node[a]);
            ux[a] = t.x;
            uy[a] = t.y;
            dx[a] = 0.0;
            dy[a] = 0.0;
            dxy[a] = 0.0;
        }
        double pe[DFEA_MAX_MAT_PARAMS];
        element_params(mat, theta[m.orig[e]], pe);
#pragma unroll(GEN ? 1 : NQ)
        for (int q = 0; q < NQ; ++q) {
            double gx[NEN], gy[NEN];
            double F[4] = {1.0, 0.0, 0.0, 1.0};
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const double2 g = load_grad(m.grad, (int64_t)(q * NEN + a) * S + e);
                gx[a] = g.x;
                gy[a] = g.y;
                F[0] += ux[a] * g.x;
                F[1] += ux[a] * g.y;
                F[2] += uy[a] * g.x;
                F[3] += uy[a] * g.y;
            }
            double Cq[16];
            if constexpr (GEN) {
                gen_moduli(mat.model, F, pe, m.wdet[q * S + e], Cq);
            } else {
                const NHPoint p = nh_point(F);
                nh_moduli(p, pe[0], pe[1], m.wdet[q * S + e], Cq);
            }
            if (Cout != nullptr) {
                if constexpr (REF) {
                    const double2* j2 = reinterpret_cast<const double2*>(m.jinv);
                    const double2 r0 = __ldg(j2 + (int64_t)(q * 2) * S + e), r1 = __ldg(j2 + (int64_t)(q * 2 + 1) * S + e);
                    const double ji[4] = {r0.x, r0.y, r1.x, r1.y};
                    store_moduli_ref(Cout, S, q, e, Cq, ji);
                } else {
                    store_moduli(Cout, S, q, e, Cq);
                }
            }
            if (diag != nullptr) {
                // e_k^T K_e e_k for the unit DOF (a, i): sum_{J,L} C[(iJ),(iL)] dN_aJ dN_aL
#pragma unroll
                for (int a = 0; a < NEN; ++a) {
                    dx[a] += Cq[0] * gx[a] * gx[a] + (Cq[1] + Cq[4]) * gx[a] * gy[a] + Cq[5] * gy[a] * gy[a];
                    dy[a] += Cq[10] * gx[a] * gx[a] + (Cq[11] + Cq[14]) * gx[a] * gy[a] + Cq[15] * gy[a] * gy[a];
                }
                if (blocks != nullptr) {
                    // coupling term of the node's 2x2 block: sum_{J,L} C[(0J),(1L)] dN_aJ dN_aL
#pragma unroll
                    for (int a = 0; a < NEN; ++a)
                        dxy[a] += Cq[2] * gx[a] * gx[a] + (Cq[3] + Cq[6]) * gx[a] * gy[a] + Cq[7] * gy[a] * gy[a];
                }
            }
        }
        if (diag != nullptr) {
            double2* d2 = reinterpret_cast<double2*>(diag);
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                double2 t = d2[node[a]];
                t.x += dx[a];
                t.y += dy[a];
                d2[node[a]] = t;
            }
        }
        if (blocks != nullptr) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) blocks[4 * (int64_t)node[a] + 3] += dxy[a];  // slot 3: raw coupling
        }
    }
}

// Nodal block-Jacobi (operators.py:598-625): B = M B M + (I - M) + 1e-12 I from the raw diagonal (diag) and
// coupling (blocks[4n + 3]); blocks[4n .. 4n+3] := (Binv00, Binv01, Binv11, 0).
__global__ void k_block_finalize(Mesh m, const double* __restrict__ diag, double* __restrict__ blocks) {
    const double2* d2 = reinterpret_cast<const double2*>(diag);
    double2* b2 = reinterpret_cast<double2*>(blocks);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const double2 dn = d2[n];
        const double c = b2[2 * n + 1].y;
        const bool fx = fix & 1, fy = fix & 2;
        const double a00 = (fx ? 1.0 : dn.x) + 1e-12, a11 = (fy ? 1.0 : dn.y) + 1e-12;
        const double a01 = (fx || fy) ? 0.0 : c;
        const double det = a00 * a11 - a01 * a01;
        b2[2 * n] = make_double2(a11 / det, -a01 / det);
        b2[2 * n + 1] = make_double2(a00 / det, 0.0);
    }
}

__global__ void k_zero(int64_t n, double* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = 0.0;
}

// diag = where(m > 0, clamp(diag, min=1e-6), 1)   (operators.py:555-556)
__global__ void k_diag_finalize(Mesh m, double* __restrict__ diag) {
    double2* d2 = reinterpret_cast<double2*>(diag);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        double2 t = d2[n];
        t.x = (fix & 1) ? 1.0 : fmax(t.x, 1e-6);
        t.y = (fix & 2) ? 1.0 : fmax(t.y, 1e-6);
        d2[n] = t;
    }
}

// ------------------------------------------------------------------------------------------
// FP64 residual and strain energy, one colour per launch
// ------------------------------------------------------------------------------------------
// R = -load_factor * f on free DOFs, 0 on fixed DOFs (the colour passes then add R_int).
__global__ void k_residual_init(Mesh m, const double* __restrict__ f, double lf, double* __restrict__ R) {
    const double2* f2 = reinterpret_cast<const double2*>(f);
    double2* R2 = reinterpret_cast<double2*>(R);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const double2 t = f ? f2[n] : make_double2(0.0, 0.0);
        R2[n] = make_double2((fix & 1) ? 0.0 : -lf * t.x, (fix & 2) ? 0.0 : -lf * t.y);
    }
}

// MASK = false: the internal force at every DOF (constrained ones included), for support reactions.
template <int NEN, int NQ, bool ENERGY, bool MASK = true, bool GEN = false>
__global__ void __launch_bounds__(128)
k_residual(Mesh m, int64_t e0, int64_t e1, const double* __restrict__ u, const double* __restrict__ theta,
           dfea_material mat, double* __restrict__ R, RedSite site) {
    const int64_t S = m.stride;
    const double2* u2 = reinterpret_cast<const double2*>(u);
    double2* R2 = reinterpret_cast<double2*>(R);
    double energy = 0.0;
    for (int64_t e = e0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < e1; e += (int64_t)gridDim.x * blockDim.x) {
        int node[NEN], fix[NEN];
        double ux[NEN], uy[NEN], fx[NEN], fy[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const int c = m.conn[a * S + e];
            node[a] = c >> 2;
            fix[a] = c & 3;
            const double2 t = __ldg(u2 + node[a]);
            ux[a] = t.x;
            uy[a] = t.y;
            fx[a] = 0.0;
            fy[a] = 0.0;
        }
        double pe[DFEA_MAX_MAT_PARAMS];
        element_params(mat, theta ? theta[m.orig[e]] : 1.0, pe);
#pragma unroll(GEN ? 1 : NQ)
        for (int q = 0; q < NQ; ++q) {
            double gx[NEN], gy[NEN];
            double F[4] = {1.0, 0.0, 0.0, 1.0};
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const double2 g = load_grad(m.grad, (int64_t)(q * NEN + a) * S + e);
                gx[a] = g.x;
                gy[a] = g.y;
                F[0] += ux[a] * g.x;
                F[1] += ux[a] * g.y;
                F[2] += uy[a] * g.x;
                F[3] += uy[a] * g.y;
            }
            double P[4];
            const double w = m.wdet[q * S + e];
            if constexpr (GEN) {
                const double psi = gen_stress(mat.model, F, pe, P);
                if (ENERGY) energy += w * psi;
            } else {
                const NHPoint p = nh_point(F);
                nh_stress(F, p, pe[0], pe[1], P);
                if (ENERGY) energy += w * nh_energy(F, p, pe[0], pe[1]);
            }
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                fx[a] += w * (P[0] * gx[a] + P[1] * gy[a]);
                fy[a] += w * (P[2] * gx[a] + P[3] * gy[a]);
            }
        }
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            double2 t = R2[node[a]];
            if (!MASK || !(fix[a] & 1)) t.x += fx[a];
            if (!MASK || !(fix[a] & 2)) t.y += fy[a];
            R2[node[a]] = t;
        }
    }
    if (ENERGY) {
        const double vals[1] = {block_sum<128>(energy)};
        double tot[1];
        if (last_block_sum<128, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

// ------------------------------------------------------------------------------------------
// Post-processing (postprocess.py:24-118): per element the quadrature-weighted averages of the
// Gauss-point state [J, sigma_xx, sigma_yy, sigma_xy, sigma_zz, psi] (weights w detJ), the area, and von
// Mises from the averaged components; per node the plain average over the incident elements.  Cauchy
// stress of the plane-strain neo-Hookean energy: sigma = (mu (F F^T - I) + lambda lnJ I) / J in 3D with
// F33 = 1, so sigma_zz = lambda lnJ / J.
// ------------------------------------------------------------------------------------------
constexpr int kNodeFields = 6;  // J, sxx, syy, sxy, mises, psi   ([field][n_nodes])

template <int NEN, int NQ, bool GEN = false>
__global__ void __launch_bounds__(128)
k_element_fields(Mesh m, const double* __restrict__ u, const double* __restrict__ theta, dfea_material mat,
                 double* __restrict__ out) {
    const int64_t S = m.stride, n_el = m.n_el;
    const double2* u2 = reinterpret_cast<const double2*>(u);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_el; e += (int64_t)gridDim.x * blockDim.x) {
        double ux[NEN], uy[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const double2 t = __ldg(u2 + (m.conn[a * S + e] >> 2));
            ux[a] = t.x;
            uy[a] = t.y;
        }
        const int64_t oe = m.orig[e];
        double pe[DFEA_MAX_MAT_PARAMS];
        element_params(mat, theta ? theta[oe] : 1.0, pe);
        double area = 0.0, acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll(GEN ? 1 : NQ)
        for (int q = 0; q < NQ; ++q) {
            double F[4] = {1.0, 0.0, 0.0, 1.0};
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const double2 g = load_grad(m.grad, (int64_t)(q * NEN + a) * S + e);
                F[0] += ux[a] * g.x;
                F[1] += ux[a] * g.y;
                F[2] += uy[a] * g.x;
                F[3] += uy[a] * g.y;
            }
            double J, sxx, syy, sxy, szz, psi;
            if constexpr (GEN) {
                // sigma = P3 F3^T / J (postprocess.py:40-44); P3 is zero in the (i, 3) and (3, i) slots
                double P[5];
                psi = gen_stress3(mat.model, F, pe, P);
                J = F[0] * F[3] - F[1] * F[2];
                const double iJ = 1.0 / J;
                sxx = (P[0] * F[0] + P[1] * F[1]) * iJ;
                syy = (P[2] * F[2] + P[3] * F[3]) * iJ;
                sxy = (P[0] * F[2] + P[1] * F[3]) * iJ;
                szz = P[4] * iJ;
            } else {
                const double mu = pe[0], lam = pe[1];
                const NHPoint pt = nh_point(F);
                const double iJ = 1.0 / pt.J, c = lam * pt.lnJ;
                const double b00 = F[0] * F[0] + F[1] * F[1], b11 = F[2] * F[2] + F[3] * F[3], b01 = F[0] * F[2] + F[1] * F[3];
                J = pt.J;
                sxx = (mu * (b00 - 1.0) + c) * iJ;
                syy = (mu * (b11 - 1.0) + c) * iJ;
                sxy = (mu * b01) * iJ;
                szz = c * iJ;
                psi = nh_energy(F, pt, mu, lam);
            }
            const double w = m.wdet[q * S + e];
            area += w;
            acc[0] += w * J;
            acc[1] += w * sxx;
            acc[2] += w * syy;
            acc[3] += w * sxy;
            acc[4] += w * szz;
            acc[5] += w * psi;
        }
        double mean[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) mean[k] = acc[k] / area;
        const double sxx = mean[1], syy = mean[2], sxy = mean[3], szz = mean[4];
        const double mises = sqrt(0.5 * ((sxx - syy) * (sxx - syy) + (syy - szz) * (syy - szz) + (szz - sxx) * (szz - sxx)) +
                                  3.0 * sxy * sxy);
        out[0 * n_el + oe] = area;
        out[1 * n_el + oe] = mean[0];
        out[2 * n_el + oe] = sxx;
        out[3 * n_el + oe] = syy;
        out[4 * n_el + oe] = sxy;
        out[5 * n_el + oe] = mises;
        out[6 * n_el + oe] = mean[5];
    }
}

// node value = sum over the node's incident elements (incidence order) / their number
__global__ void __launch_bounds__(kThreads)
k_node_fields(Mesh m, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
              const double* __restrict__ elem, double* __restrict__ out) {
    const int64_t S = m.stride, n_el = m.n_el, N = m.n_nodes;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        double acc[kNodeFields] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int j0 = inc_ptr[n], j1 = inc_ptr[n + 1];
        for (int j = j0; j < j1; ++j) {
            const int64_t oe = m.orig[inc[j] % S];
#pragma unroll
            for (int k = 0; k < kNodeFields; ++k) acc[k] += elem[(k + 1) * n_el + oe];
        }
        const double cnt = (j1 > j0) ? (double)(j1 - j0) : 1.0;
#pragma unroll
        for (int k = 0; k < kNodeFields; ++k) out[k * N + n] = acc[k] / cnt;
    }
}

// sum x^2 over 2N entries; the last block also adds up per-colour energies (if any) in colour order.
__global__ void __launch_bounds__(kThreads)
k_norm2(int64_t n, const double* __restrict__ x, RedSite site, double* __restrict__ out,
        const double* __restrict__ colour_energy, int n_colours, double* __restrict__ out_energy) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double t = x[i];
        s += t * t;
    }
    const double vals[1] = {block_sum<kThreads>(s)};
    double tot[1];
    if (last_block_sum<kThreads, 1>(vals, site, tot) && threadIdx.x == 0) {
        if (out) *out = tot[0];
        if (out_energy) {
            double E = 0.0;
            for (int c = 0; c < n_colours; ++c) E += colour_energy[c];
            *out_energy = E;
        }
    }
}

// ------------------------------------------------------------------------------------------
// kernel (d): per-element sensitivity g_e = -lambda_e . f_e(u; p0)
// ------------------------------------------------------------------------------------------
// mat.p holds d p_e / d theta_e: the nominal value of every scalable parameter, 0 for the others (all of
// them prefactors of terms of the energy, so f_e is linear in theta_e with slope f_e(u; mat.p)).
template <int NEN, int NQ, bool GEN = false>
__global__ void __launch_bounds__(128)
k_sensitivity(Mesh m, const double* __restrict__ u, const double* __restrict__ lam_adj, dfea_material mat,
              double* __restrict__ g) {
    const int64_t S = m.stride;
    const double2* u2 = reinterpret_cast<const double2*>(u);
    const double2* l2 = reinterpret_cast<const double2*>(lam_adj);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m.n_el; e += (int64_t)gridDim.x * blockDim.x) {
        double ux[NEN], uy[NEN], lx[NEN], ly[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const int c = m.conn[a * S + e];
            const int node = c >> 2, fix = c & 3;
            const double2 t = __ldg(u2 + node);
            const double2 l = __ldg(l2 + node);
            ux[a] = t.x;
            uy[a] = t.y;
            lx[a] = (fix & 1) ? 0.0 : l.x;
            ly[a] = (fix & 2) ? 0.0 : l.y;
        }
        double ge = 0.0;
#pragma unroll(GEN ? 1 : NQ)
        for (int q = 0; q < NQ; ++q) {
            double gx[NEN], gy[NEN];
            double F[4] = {1.0, 0.0, 0.0, 1.0};
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const double2 gg = load_grad(m.grad, (int64_t)(q * NEN + a) * S + e);
                gx[a] = gg.x;
                gy[a] = gg.y;
                F[0] += ux[a] * gg.x;
                F[1] += ux[a] * gg.y;
                F[2] += uy[a] * gg.x;
                F[3] += uy[a] * gg.y;
            }
            double P[4];
            if constexpr (GEN) {
                gen_stress(mat.model, F, mat.p, P);
            } else {
                const NHPoint p = nh_point(F);
                nh_stress(F, p, mat.p[0], mat.p[1], P);
            }
            const double w = m.wdet[q * S + e];
            // lambda_e : (P dN^T) integrated, i.e. sum_a lambda_a . f_a
            double lgx = 0.0, lgy = 0.0, lgx2 = 0.0, lgy2 = 0.0;
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                lgx += lx[a] * gx[a];
                lgy += lx[a] * gy[a];
                lgx2 += ly[a] * gx[a];
                lgy2 += ly[a] * gy[a];
            }
            ge += w * (P[0] * lgx + P[1] * lgy + P[2] * lgx2 + P[3] * lgy2);
        }
        g[m.orig[e]] = -ge;
    }
}

// ------------------------------------------------------------------------------------------
// small vector kernels
// ------------------------------------------------------------------------------------------
__global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

__global__ void k_add_scaled(int64_t n, const double* __restrict__ a, double alpha, const double* __restrict__ b,
                             double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] + alpha * b[i];
}

// Scratch layout of dfea_residual / dfea_vec_norm2:
//   [0, DFEA_MAX_COLOURS + 1) reduction sites of kMaxBlocks partials, then tickets, then results.
struct ReduceWork {
    double* partials;   // n_sites x kMaxBlocks
    unsigned* tickets;  // kTicketSlots >= n_sites
    double* results;    // n_sites
    static constexpr int n_sites = DFEA_MAX_COLOURS + 1;
    static constexpr int kTicketSlots = 128;
    static int64_t bytes() {
        return (int64_t)n_sites * kMaxBlocks * 8 + kTicketSlots * 4 + (int64_t)n_sites * 8 + 256;
    }
    explicit ReduceWork(void* base) {
        char* p = static_cast<char*>(base);
        partials = reinterpret_cast<double*>(p);
        p += (int64_t)n_sites * kMaxBlocks * 8;
        tickets = reinterpret_cast<unsigned*>(p);
        p += kTicketSlots * 4;
        results = reinterpret_cast<double*>(p);
    }
    RedSite site(int i) const { return RedSite{partials + (int64_t)i * kMaxBlocks, tickets + i, results + i}; }
};

__global__ void k_zero_tickets(unsigned* t, int n, double* results, int nr) {
    // one block of >= max(n, nr) threads; n <= ReduceWork::kTicketSlots
    const int i = threadIdx.x;
    if (i < n) t[i] = 0u;
    if (i < nr) results[i] = 0.0;
}

// ------------------------------------------------------------------------------------------
// Serving requests' problems on the device (dfea_build_rectangle): grid node (i, j) of the rectangle mesher
// is i (gy + 1) + j at (linspace(0, W, gx + 1)[i], linspace(0, H, gy + 1)[j]), with gx = nx (Q4) or 2 nx (Q9)
// lines; element e = I ny + J.
// ------------------------------------------------------------------------------------------
// torch.linspace's value at ind: from the start below the halfway point, from the end above it
__host__ __device__ inline double lin_value(double start, double end, int64_t steps, int64_t ind) {
    const double step = (end - start) / (steps - 1);
    return ind < steps / 2 ? start + step * ind : end - step * (steps - ind - 1);
}

struct RectGrid {
    int64_t gx, gy;
    __host__ __device__ int64_t id(int64_t i, int64_t j) const { return i * (gy + 1) + j; }
};

__host__ __device__ inline RectGrid rect_grid(const dfea_rect_spec& p) {
    const int64_t span = p.nen == 9 ? 2 : 1;
    return RectGrid{span * p.nx, span * p.ny};
}

// grid node id: coordinates, supports (the side x = 0; the next line lies a cell width away), zero load
__host__ __device__ inline void rect_node(const dfea_rect_spec& p, const RectGrid& g, int64_t id, double* nodes,
                                          double* m, uint8_t* fixed, double* u_D, double* f) {
    const int64_t i = id / (g.gy + 1), j = id - i * (g.gy + 1);
    nodes[2 * id] = lin_value(0.0, p.width, g.gx + 1, i);
    nodes[2 * id + 1] = lin_value(0.0, p.height, g.gy + 1, j);
    const bool clamped = i == 0;
    for (int c = 0; c < 2; ++c) {
        fixed[2 * id + c] = clamped ? 1 : 0;
        m[2 * id + c] = clamped ? 0.0 : 1.0;
        u_D[2 * id + c] = 0.0;
        f[2 * id + c] = 0.0;
    }
}

// element e: connectivity in the element library's local order, dN/dX = J^-T dN/dxi and w detJ at its Gauss points
__host__ __device__ inline void rect_element(const dfea_rect_spec& p, const RectGrid& g, int64_t e, int64_t* conn,
                                             double* dN_dX, double* w_detJ) {
    // grid offsets of the nine Q9 nodes in their 2 x 2 block of grid cells; the four Q4 corners
    const int di9[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1}, dj9[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
    const int di4[4] = {0, 1, 1, 0}, dj4[4] = {0, 0, 1, 1};
    const int nen = p.nen, nq = p.n_q;
    const int64_t I = e / p.ny, J = e - I * p.ny;
    double X[DFEA_MAX_NEN][2];
    for (int a = 0; a < nen; ++a) {
        const int64_t i = nen == 9 ? 2 * I + di9[a] : I + di4[a], j = nen == 9 ? 2 * J + dj9[a] : J + dj4[a];
        conn[e * nen + a] = g.id(i, j);
        X[a][0] = lin_value(0.0, p.width, g.gx + 1, i);
        X[a][1] = lin_value(0.0, p.height, g.gy + 1, j);
    }
    for (int q = 0; q < nq; ++q) {
        const double* dNr = p.ref_grad + q * nen * 2;
        double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
        for (int a = 0; a < nen; ++a) {
            J00 += X[a][0] * dNr[2 * a];
            J01 += X[a][0] * dNr[2 * a + 1];
            J10 += X[a][1] * dNr[2 * a];
            J11 += X[a][1] * dNr[2 * a + 1];
        }
        const double det = J00 * J11 - J01 * J10;
        const double i00 = J11 / det, i01 = -J01 / det, i10 = -J10 / det, i11 = J00 / det;
        double* out = dN_dX + (e * nq + q) * nen * 2;
        for (int a = 0; a < nen; ++a) {
            out[2 * a] = dNr[2 * a] * i00 + dNr[2 * a + 1] * i10;
            out[2 * a + 1] = dNr[2 * a] * i01 + dNr[2 * a + 1] * i11;
        }
        w_detJ[e * nq + q] = p.gauss_w[q] * det;
    }
}

// the consistent nodal forces of the uniform traction on x = W: edge J joins grid nodes (gx, k J) and
// (gx, k J + k) (k = 1 for Q4, 2 for Q9 with its mid node at k J + 1); t = load / total edge length
__host__ __device__ inline void edge_shape_at(int order, double s, double (&N)[3], double (&dN)[3]) {
    if (order == 1) {
        N[0] = 0.5 * (1.0 - s); N[1] = 0.5 * (1.0 + s); N[2] = 0.0;
        dN[0] = -0.5; dN[1] = 0.5; dN[2] = 0.0;
    } else {
        N[0] = 0.5 * s * (s - 1.0); N[1] = 0.5 * s * (s + 1.0); N[2] = 1.0 - s * s;
        dN[0] = s - 0.5; dN[1] = s + 0.5; dN[2] = -2.0 * s;
    }
}

__host__ __device__ inline double edge_speed(const dfea_rect_spec& p, const RectGrid& g, int64_t J, int gpt) {
    const int order = p.nen == 9 ? 2 : 1, k = order;
    double N[3], dN[3];
    edge_shape_at(order, p.edge_s[gpt], N, dN);
    const int64_t js[3] = {k * J, k * J + k, k * J + 1};
    double t0 = 0.0, t1 = 0.0;
    for (int a = 0; a <= order; ++a) {
        t0 += dN[a] * lin_value(0.0, p.width, g.gx + 1, g.gx);
        t1 += dN[a] * lin_value(0.0, p.height, g.gy + 1, js[a]);
    }
    return sqrt(t0 * t0 + t1 * t1);
}

__host__ __device__ inline double rect_edge_length(const dfea_rect_spec& p, const RectGrid& g) {
    double L = 0.0;
    for (int64_t J = 0; J < p.ny; ++J)
        for (int gpt = 0; gpt < 3; ++gpt) L += edge_speed(p, g, J, gpt) * p.edge_w[gpt];
    return L;
}

// the load of grid node (gx, j): the contributions of the (at most two) edges that hold it, in edge order
__host__ __device__ inline void rect_load_node(const dfea_rect_spec& p, const RectGrid& g, int64_t j, double tx,
                                               double ty, double* f) {
    const int order = p.nen == 9 ? 2 : 1;
    int64_t edge[2];
    int local[2], n_edges = 0;
    if (order == 1) {
        if (j > 0) { edge[n_edges] = j - 1; local[n_edges++] = 1; }
        if (j < p.ny) { edge[n_edges] = j; local[n_edges++] = 0; }
    } else if (j % 2) {
        edge[n_edges] = (j - 1) / 2; local[n_edges++] = 2;
    } else {
        if (j > 0) { edge[n_edges] = j / 2 - 1; local[n_edges++] = 1; }
        if (j / 2 < p.ny) { edge[n_edges] = j / 2; local[n_edges++] = 0; }
    }
    double fx = 0.0, fy = 0.0;
    for (int k = 0; k < n_edges; ++k) {
        double cx = 0.0, cy = 0.0;
        for (int gpt = 0; gpt < 3; ++gpt) {
            double N[3], dN[3];
            edge_shape_at(order, p.edge_s[gpt], N, dN);
            const double w = p.edge_w[gpt] * N[local[k]] * edge_speed(p, g, edge[k], gpt);
            cx += w * tx;
            cy += w * ty;
        }
        fx += cx;
        fy += cy;
    }
    const int64_t id = g.id(g.gx, j);
    f[2 * id] = fx;
    f[2 * id + 1] = fy;
}

__global__ void k_rect_nodes(dfea_rect_spec p, double* __restrict__ nodes, double* __restrict__ m,
                             uint8_t* __restrict__ fixed, double* __restrict__ u_D, double* __restrict__ f) {
    const RectGrid g = rect_grid(p);
    const int64_t N = (g.gx + 1) * (g.gy + 1);
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < N; id += (int64_t)gridDim.x * blockDim.x)
        rect_node(p, g, id, nodes, m, fixed, u_D, f);
}

__global__ void k_rect_elements(dfea_rect_spec p, int64_t* __restrict__ conn, double* __restrict__ dN_dX,
                                double* __restrict__ w_detJ) {
    const RectGrid g = rect_grid(p);
    const int64_t n_el = (int64_t)p.nx * p.ny;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_el; e += (int64_t)gridDim.x * blockDim.x)
        rect_element(p, g, e, conn, dN_dX, w_detJ);
}

__global__ void __launch_bounds__(256) k_rect_load(dfea_rect_spec p, double* __restrict__ f) {
    const RectGrid g = rect_grid(p);
    __shared__ double length;
    if (threadIdx.x == 0) length = rect_edge_length(p, g);
    __syncthreads();
    const double tx = p.load_x / length, ty = p.load_y / length;
    for (int64_t j = threadIdx.x; j <= g.gy; j += blockDim.x) rect_load_node(p, g, j, tx, ty, f);
}

// Node -> (element, local node) incidence of the gather form, CSR: ptr[n_nodes + 1] and the slots
// a * stride + e of every node in increasing order -- the arrays a stable sort of the slots by node gives.
// Counting with integer atomics, an exclusive scan in one block, a fill at per-node cursors (in any order),
// then each node's few slots sorted ascending: every step is exact, so the result is the same each time.
__global__ void k_inc_count(int64_t n_slots, int64_t n_el, int64_t S, const int32_t* __restrict__ conn,
                            int32_t* __restrict__ count) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_slots; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = t / n_el, e = t - a * n_el;
        atomicAdd(&count[conn[a * S + e] >> 2], 1);
    }
}

constexpr int kIncScanThreads = 1024;

// ptr[i] = sum of count[0..i), ptr[N] = the total; the counts are replaced by the same prefix (the fill's
// cursors).  One block: each thread scans its contiguous chunk, the chunk totals are scanned in shared memory.
__global__ void __launch_bounds__(kIncScanThreads) k_inc_scan(int64_t N, int32_t* __restrict__ count_cursor,
                                                              int32_t* __restrict__ ptr) {
    __shared__ long long part[kIncScanThreads];
    const int tid = threadIdx.x;
    const int64_t chunk = (N + kIncScanThreads - 1) / kIncScanThreads;
    const int64_t lo = tid * chunk, hi = lo + chunk < N ? lo + chunk : N;
    long long s = 0;
    for (int64_t i = lo; i < hi; ++i) s += count_cursor[i];
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < kIncScanThreads; off <<= 1) {
        const long long v = tid >= off ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    long long run = part[tid] - s;
    for (int64_t i = lo; i < hi; ++i) {
        const int32_t c = count_cursor[i];
        ptr[i] = (int32_t)run;
        count_cursor[i] = (int32_t)run;
        run += c;
    }
    if (tid == kIncScanThreads - 1) ptr[N] = (int32_t)part[tid];
}

__global__ void k_inc_fill(int64_t n_slots, int64_t n_el, int64_t S, const int32_t* __restrict__ conn,
                           int32_t* __restrict__ cursor, int32_t* __restrict__ inc) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_slots; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = t / n_el, e = t - a * n_el;
        const int pos = atomicAdd(&cursor[conn[a * S + e] >> 2], 1);
        inc[pos] = (int32_t)(a * S + e);
    }
}

__global__ void k_inc_sort(int64_t N, const int32_t* __restrict__ ptr, int32_t* __restrict__ inc) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        const int b = ptr[n], end = ptr[n + 1];
        for (int i = b + 1; i < end; ++i) {
            const int32_t v = inc[i];
            int j = i - 1;
            while (j >= b && inc[j] > v) {
                inc[j + 1] = inc[j];
                --j;
            }
            inc[j + 1] = v;
        }
    }
}

// Inverse element Jacobians of the reference-frame FP32 operator, packed [q][row][stride] as (col 0, col 1)
// pairs (zeros in the padding slots), from the packed connectivity and the node coordinates:
// J_ij = sum_a X_a,i dN_a/dxi_j, Jinv = J^-1.  check[0] and check[1] receive the largest |Jinv^T dN/dxi -
// dN/dX| and |dN/dX| over every element, Gauss point and node (maxima of non-negative values, combined by
// atomic maxima of their bit patterns: order-independent; a NaN wins, as in a propagating maximum).
__device__ __forceinline__ void nan_max(double& m, double v) {
    if (v > m || v != v) m = (m != m) ? m : v;
}

template <int NEN, int NQ>
__global__ void __launch_bounds__(128) k_ref_frame(Mesh m, RefGrad<NEN, NQ> rg, const double* __restrict__ nodes,
                                                   double* __restrict__ jinv, double* __restrict__ check) {
    const int64_t S = m.stride;
    double2* out = reinterpret_cast<double2*>(jinv);
    const double2* g2 = reinterpret_cast<const double2*>(m.grad);
    double dmax = 0.0, smax = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < S; e += (int64_t)gridDim.x * blockDim.x) {
        if (e >= m.n_el) {
#pragma unroll
            for (int k = 0; k < 2 * NQ; ++k) out[k * S + e] = make_double2(0.0, 0.0);
            continue;
        }
        double X[NEN][2];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const int64_t node = m.conn[a * S + e] >> 2;
            X[a][0] = nodes[2 * node];
            X[a][1] = nodes[2 * node + 1];
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                J00 += X[a][0] * rg.g[q][a][0];
                J01 += X[a][0] * rg.g[q][a][1];
                J10 += X[a][1] * rg.g[q][a][0];
                J11 += X[a][1] * rg.g[q][a][1];
            }
            const double det = J00 * J11 - J01 * J10;
            const double i00 = J11 / det, i01 = -J01 / det, i10 = -J10 / det, i11 = J00 / det;
            out[(2 * q) * S + e] = make_double2(i00, i01);
            out[(2 * q + 1) * S + e] = make_double2(i10, i11);
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const double r0 = rg.g[q][a][0] * i00 + rg.g[q][a][1] * i10;
                const double r1 = rg.g[q][a][0] * i01 + rg.g[q][a][1] * i11;
                const double2 g = g2[(q * NEN + a) * S + e];
                nan_max(dmax, fabs(r0 - g.x));
                nan_max(dmax, fabs(r1 - g.y));
                nan_max(smax, fabs(g.x));
                nan_max(smax, fabs(g.y));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nan_max(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
        nan_max(smax, __shfl_down_sync(0xffffffffu, smax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(reinterpret_cast<unsigned long long*>(check), (unsigned long long)__double_as_longlong(dmax));
        atomicMax(reinterpret_cast<unsigned long long*>(check + 1), (unsigned long long)__double_as_longlong(smax));
    }
}

// Node pass of the gather-form product q = A v on the finite-element level of the multigrid V-cycle, with
// the smoothing arithmetic that follows the product applied at the node (each node's q is complete here and
// the element pass has finished reading v):
//   MG_FE_STEP    (v = d): x += d, r -= q, d = c1 d + c2 r / D (d kept by the last step), coef = (c1, c2);
//   MG_FE_RESTART (v = x): r = b - q, d = s r / D, coef = (s).
// The expressions are those of k_node_gather followed by the multigrid's separate Chebyshev kernels, so the
// iterates are bitwise the same.  d and v alias in MG_FE_STEP (read and written at the thread's own node).
template <int MODE>
__global__ void __launch_bounds__(kThreads)
k_node_gather_cheb(Mesh m, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc, const double* __restrict__ fe,
                   const double* v, double* __restrict__ x, double* __restrict__ r, double* d, const double* __restrict__ b,
                   const double* __restrict__ diag, const double* __restrict__ coef, int last) {
    grid_dependency_wait();
    grid_dependents_launch();
    const double2* fe2 = reinterpret_cast<const double2*>(fe);
    const double c1 = (MODE == MG_FE_RESTART || last) ? 0.0 : coef[0];
    const double c2 = (MODE == MG_FE_RESTART || last) ? 0.0 : coef[1];
    const double sc = MODE == MG_FE_RESTART ? coef[0] : 0.0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const double2 f = node_sum<double>(inc_ptr, inc, fe2, n);
        const double2 vn = reinterpret_cast<const double2*>(v)[n];
        const double q0 = (fix & 1) ? vn.x : f.x, q1 = (fix & 2) ? vn.y : f.y;
        const double2 Dn = reinterpret_cast<const double2*>(diag)[n];
        if (MODE == MG_FE_STEP) {
            const double2 dn = reinterpret_cast<const double2*>(d)[n];
            double2 xn = reinterpret_cast<const double2*>(x)[n];
            xn.x += dn.x;
            xn.y += dn.y;
            reinterpret_cast<double2*>(x)[n] = xn;
            const double2 rn = reinterpret_cast<const double2*>(r)[n];
            const double r0 = rn.x - q0, r1 = rn.y - q1;
            reinterpret_cast<double2*>(r)[n] = make_double2(r0, r1);
            if (!last) reinterpret_cast<double2*>(d)[n] = make_double2(c1 * dn.x + c2 * r0 / Dn.x, c1 * dn.y + c2 * r1 / Dn.y);
        } else {
            const double2 bn = reinterpret_cast<const double2*>(b)[n];
            const double r0 = bn.x - q0, r1 = bn.y - q1;
            reinterpret_cast<double2*>(r)[n] = make_double2(r0, r1);
            reinterpret_cast<double2*>(d)[n] = make_double2(sc * r0 / Dn.x, sc * r1 / Dn.y);
        }
    }
}

}  // namespace dfea

using namespace dfea;

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" int dfea_mesh_pack(int64_t n_el, int64_t stride, int32_t nen, int32_t n_q, int64_t n_nodes,
                              const int64_t* perm, const int64_t* conn_ref, const double* dN_dX,
                              const double* w_detJ, const double* m, int32_t* conn_out, int32_t* orig_out,
                              double* grad_out, double* wdet_out, uint8_t* node_fix_out, void* stream) {
    if (n_el < 0 || n_nodes <= 0 || stride < n_el || stride % 32 != 0)
        return set_error(DFEA_ERR_INVALID, "dfea_mesh_pack: bad sizes");
    if (!dfea_element_supported(nen, n_q))
        return set_error(DFEA_ERR_UNSUPPORTED, "element with nen=%d n_q=%d is not built", nen, n_q);
    if (n_nodes >= (int64_t(1) << 29)) return set_error(DFEA_ERR_INVALID, "too many nodes for the packed connectivity");
    if (!m || !node_fix_out || (n_el > 0 && (!perm || !conn_ref || !dN_dX || !w_detJ || !conn_out || !orig_out ||
                                             !grad_out || !wdet_out)))
        return set_error(DFEA_ERR_INVALID, "dfea_mesh_pack: NULL pointer");
    if (!aligned16(grad_out)) return set_error(DFEA_ERR_INVALID, "dfea_mesh_pack: grad_out must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n_el > 0) {
        k_pack<<<grid_for(n_el, kThreads, 8), kThreads, 0, s>>>(n_el, stride, nen, n_q, perm, conn_ref, dN_dX, w_detJ, m,
                                                                  conn_out, orig_out, grad_out, wdet_out);
        note_launches(1);
    }
    k_node_fix<<<grid_for(n_nodes, kThreads, 8), kThreads, 0, s>>>(n_nodes, m, node_fix_out);
    note_launches(1);
    return launch_check("dfea_mesh_pack");
}

static int validate_rect(const dfea_rect_spec* spec, const char* what) {
    if (!spec) return set_error(DFEA_ERR_INVALID, "%s: NULL spec", what);
    const dfea_rect_spec& p = *spec;
    if (!((p.nen == 4 && p.n_q == 4) || (p.nen == 9 && p.n_q == 9)) || p.nx < 1 || p.ny < 1 || !(p.width > 0.0) ||
        !(p.height > 0.0))
        return set_error(DFEA_ERR_INVALID, "%s: a Q4 or Q9 rectangle of at least one cell", what);
    const int64_t span = p.nen == 9 ? 2 : 1;
    if ((span * p.nx + 1) * (span * p.ny + 1) >= (int64_t(1) << 29)) return set_error(DFEA_ERR_INVALID, "%s: too many nodes", what);
    return DFEA_OK;
}

extern "C" int dfea_build_rectangle_host(const dfea_rect_spec* spec, double* nodes, int64_t* conn, double* dN_dX,
                                         double* w_detJ, double* f, double* m, uint8_t* fixed, double* u_D) {
    int rc = validate_rect(spec, "dfea_build_rectangle_host");
    if (rc) return rc;
    if (!nodes || !conn || !dN_dX || !w_detJ || !f || !m || !fixed || !u_D)
        return set_error(DFEA_ERR_INVALID, "dfea_build_rectangle_host: NULL pointer");
    const dfea_rect_spec& p = *spec;
    const RectGrid g = rect_grid(p);
    const int64_t N = (g.gx + 1) * (g.gy + 1), n_el = (int64_t)p.nx * p.ny;
    for (int64_t id = 0; id < N; ++id) rect_node(p, g, id, nodes, m, fixed, u_D, f);
    for (int64_t e = 0; e < n_el; ++e) rect_element(p, g, e, conn, dN_dX, w_detJ);
    const double L = rect_edge_length(p, g);
    for (int64_t j = 0; j <= g.gy; ++j) rect_load_node(p, g, j, p.load_x / L, p.load_y / L, f);
    return DFEA_OK;
}

extern "C" int dfea_build_rectangle(const dfea_rect_spec* spec, double* nodes, int64_t* conn, double* dN_dX,
                                    double* w_detJ, double* f, double* m, uint8_t* fixed, double* u_D, void* stream) {
    int rc = validate_rect(spec, "dfea_build_rectangle");
    if (rc) return rc;
    const dfea_rect_spec& p = *spec;
    const int64_t span = p.nen == 9 ? 2 : 1;
    const int64_t N = (span * p.nx + 1) * (span * p.ny + 1), n_el = (int64_t)p.nx * p.ny;
    if (!nodes || !conn || !dN_dX || !w_detJ || !f || !m || !fixed || !u_D)
        return set_error(DFEA_ERR_INVALID, "dfea_build_rectangle: NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_rect_nodes<<<grid_for(N, kThreads, 8), kThreads, 0, s>>>(p, nodes, m, fixed, u_D, f);
    k_rect_elements<<<grid_for(n_el, 128, 8), 128, 0, s>>>(p, conn, dN_dX, w_detJ);
    k_rect_load<<<1, 256, 0, s>>>(p, f);
    note_launches(3);
    return launch_check("dfea_build_rectangle");
}

extern "C" int dfea_mesh_node_incidence(const dfea_mesh_view* mesh, int32_t* ptr_out, int32_t* inc_out, int32_t* work,
                                        void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!ptr_out || !inc_out || !work) return set_error(DFEA_ERR_INVALID, "dfea_mesh_node_incidence: NULL pointer");
    if ((int64_t)mesh->nen * mesh->stride >= (int64_t(1) << 31))
        return set_error(DFEA_ERR_INVALID, "dfea_mesh_node_incidence: mesh too large for 32-bit incidence indices");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t N = mesh->n_nodes, n_slots = (int64_t)mesh->nen * mesh->n_el;
    if ((rc = check_cuda(cudaMemsetAsync(work, 0, N * sizeof(int32_t), s), "cudaMemsetAsync"))) return rc;
    if (n_slots > 0)
        k_inc_count<<<grid_for(n_slots, kThreads, 8), kThreads, 0, s>>>(n_slots, mesh->n_el, mesh->stride, mesh->conn, work);
    k_inc_scan<<<1, kIncScanThreads, 0, s>>>(N, work, ptr_out);
    if (n_slots > 0) {
        k_inc_fill<<<grid_for(n_slots, kThreads, 8), kThreads, 0, s>>>(n_slots, mesh->n_el, mesh->stride, mesh->conn, work,
                                                                        inc_out);
        k_inc_sort<<<grid_for(N, kThreads, 8), kThreads, 0, s>>>(N, ptr_out, inc_out);
    }
    note_launches(n_slots > 0 ? 4 : 1);
    return launch_check("dfea_mesh_node_incidence");
}

extern "C" int dfea_mesh_ref_frame(const dfea_mesh_view* mesh, const double* nodes, double* jinv_out, double* check,
                                   void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!nodes || !jinv_out || !check) return set_error(DFEA_ERR_INVALID, "dfea_mesh_ref_frame: NULL pointer");
    if (!aligned16(jinv_out)) return set_error(DFEA_ERR_INVALID, "dfea_mesh_ref_frame: jinv_out must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((rc = check_cuda(cudaMemsetAsync(check, 0, 2 * sizeof(double), s), "cudaMemsetAsync"))) return rc;
    const Mesh m = kernel_mesh(*mesh);
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        k_ref_frame<NEN, NQ><<<grid_for(mesh->stride, 128, 8), 128, 0, s>>>(m, ref_grad_of<NEN, NQ>(*mesh), nodes, jinv_out,
                                                                             check);
        return DFEA_OK;
    });
    if (rc) return rc;
    note_launches(1);
    return launch_check("dfea_mesh_ref_frame");
}

extern "C" int dfea_mesh_grad_to_f32(const dfea_mesh_view* mesh, float* grad32_out, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!grad32_out || !aligned16(grad32_out)) return set_error(DFEA_ERR_INVALID, "grad32_out must be 16-byte aligned");
    const int64_t n = (int64_t)mesh->n_q * mesh->nen * mesh->stride * 2;
    k_to_f32<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, mesh->grad, grad32_out);
    note_launches(1);
    return launch_check("dfea_mesh_grad_to_f32");
}

extern "C" int dfea_qp_moduli(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                              double lambda0, void* moduli, int32_t moduli_dtype, double* diag, void* stream) {
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_qp_moduli_mat(mesh, u, theta, &mat, moduli, moduli_dtype, diag, nullptr, stream);
}

extern "C" int dfea_qp_moduli_block(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                                    double lambda0, void* moduli, int32_t moduli_dtype, double* diag, double* blocks,
                                    void* stream) {
    if (!diag || !blocks) return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli_block: diag and blocks are required");
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_qp_moduli_mat(mesh, u, theta, &mat, moduli, moduli_dtype, diag, blocks, stream);
}

extern "C" int dfea_qp_moduli_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                                  const dfea_material* material, void* moduli, int32_t moduli_dtype, double* diag,
                                  double* blocks, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_material(material))) return rc;
    const dfea_material mat = *material;
    if (blocks && !diag) return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli: blocks need diag");
    if (blocks && !aligned16(blocks)) return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli: blocks must be 16-byte aligned");
    if (!u || !theta || (!moduli && !diag)) return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli: NULL pointer");
    if (!aligned16(u) || (moduli && !aligned16(moduli)) || (diag && !aligned16(diag)))
        return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli: u, moduli and diag must be 16-byte aligned");
    if (moduli_dtype != DFEA_F64 && moduli_dtype != DFEA_F32 && moduli_dtype != DFEA_F32REF)
        return set_error(DFEA_ERR_INVALID, "bad moduli dtype");
    if (moduli_dtype == DFEA_F32REF && moduli && !mesh->jinv)
        return set_error(DFEA_ERR_INVALID, "dfea_qp_moduli: DFEA_F32REF moduli need mesh->jinv");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    if (diag) {
        k_zero<<<grid_for(2 * mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(2 * mesh->n_nodes, diag);
        note_launches(1);
    }
    if (blocks) {
        k_zero<<<grid_for(4 * mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(4 * mesh->n_nodes, blocks);
        note_launches(1);
    }
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        return dispatch_material(mat, [&](auto gen_c) -> int {
            constexpr bool GEN = decltype(gen_c)::value;
            for (int c = 0; c < mesh->n_colours; ++c) {
                const int64_t e0 = mesh->colour_begin[c], e1 = mesh->colour_begin[c + 1];
                if (e1 <= e0) continue;
                const int grid = grid_for(e1 - e0, 128, 12);
                if (moduli_dtype == DFEA_F64)
                    k_moduli<NEN, NQ, double, false, GEN><<<grid, 128, 0, s>>>(m, e0, e1, u, theta, mat,
                                                                               static_cast<double*>(moduli), diag, blocks);
                else if (moduli_dtype == DFEA_F32REF)
                    k_moduli<NEN, NQ, float, true, GEN><<<grid, 128, 0, s>>>(m, e0, e1, u, theta, mat,
                                                                             static_cast<float*>(moduli), diag, blocks);
                else
                    k_moduli<NEN, NQ, float, false, GEN><<<grid, 128, 0, s>>>(m, e0, e1, u, theta, mat,
                                                                              static_cast<float*>(moduli), diag, blocks);
                note_launches(1);
            }
            return DFEA_OK;
        });
    });
    if (rc) return rc;
    if (blocks) {  // from the raw diagonal, before the Jacobi clamp below
        k_block_finalize<<<grid_for(mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(m, diag, blocks);
        note_launches(1);
    }
    if (diag) {
        k_diag_finalize<<<grid_for(mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(m, diag);
        note_launches(1);
    }
    return launch_check("dfea_qp_moduli");
}

extern "C" int dfea_tangent_apply(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype, const void* v,
                                  void* y, int32_t vec_dtype, void* stream) {
    int rc = validate_mesh(mesh, moduli_dtype == DFEA_F32);
    if (rc) return rc;
    if (moduli_dtype == DFEA_F32REF) {
        if (vec_dtype != DFEA_F64) return set_error(DFEA_ERR_INVALID, "DFEA_F32REF moduli apply to f64 vectors");
        if (!moduli || !v || !y) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: NULL pointer");
        if (v == y) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: y must not alias v");
        if (!aligned16(moduli) || !aligned16(v) || !aligned16(y))
            return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: moduli, v and y must be 16-byte aligned");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const Mesh m = kernel_mesh(*mesh);
        const double* vv = static_cast<const double*>(v);
        double* yy = static_cast<double*>(y);
        k_pivot_init<double><<<grid_for(mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(m, vv, yy);
        rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
            constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
            return launch_apply_ref_colours<NEN, NQ, double, false>(*mesh, static_cast<const float*>(moduli), vv, yy,
                                                                   nullptr, nullptr, s);
        });
        if (rc) return rc;
        int nonempty = 0;
        for (int c = 0; c < mesh->n_colours; ++c) nonempty += mesh->colour_begin[c + 1] > mesh->colour_begin[c];
        note_launches(1 + nonempty);
        return DFEA_OK;
    }
    if (!moduli || !v || !y) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: NULL pointer");
    if (v == y) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: y must not alias v");
    if (!aligned16(moduli) || !aligned16(v) || !aligned16(y))
        return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply: moduli, v and y must be 16-byte aligned");
    if (moduli_dtype != DFEA_F64 && moduli_dtype != DFEA_F32) return set_error(DFEA_ERR_INVALID, "bad moduli dtype");
    if (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32) return set_error(DFEA_ERR_INVALID, "bad vector dtype");
    if (vec_dtype == DFEA_F32 && moduli_dtype != DFEA_F32)
        return set_error(DFEA_ERR_INVALID, "FP32 vectors need FP32 moduli");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    const int gn = grid_for(mesh->n_nodes, kThreads, 8);
    return dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        if (vec_dtype == DFEA_F64) {
            const double* vv = static_cast<const double*>(v);
            double* yy = static_cast<double*>(y);
            k_pivot_init<double><<<gn, kThreads, 0, s>>>(m, vv, yy);
            note_launches(1);
            if (moduli_dtype == DFEA_F64)
                return launch_apply_colours<NEN, NQ, double, double, false>(*mesh, static_cast<const double*>(moduli),
                                                                           mesh->grad, vv, yy, nullptr, nullptr, s);
            return launch_apply_colours<NEN, NQ, float, double, false>(*mesh, static_cast<const float*>(moduli),
                                                                      mesh->grad32, vv, yy, nullptr, nullptr, s);
        }
        k_pivot_init<float><<<gn, kThreads, 0, s>>>(m, static_cast<const float*>(v), static_cast<float*>(y));
        note_launches(1);
        return launch_apply_colours<NEN, NQ, float, float, false>(*mesh, static_cast<const float*>(moduli), mesh->grad32,
                                                                 static_cast<const float*>(v), static_cast<float*>(y),
                                                                 nullptr, nullptr, s);
    });
}

extern "C" int64_t dfea_gather_work_bytes(const dfea_mesh_view* mesh, int32_t vec_dtype) {
    if (!mesh || (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32)) return -1;
    return (int64_t)mesh->nen * mesh->stride * 2 * (vec_dtype == DFEA_F64 ? 8 : 4);
}

extern "C" int dfea_tangent_apply_gather(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype,
                                         const void* v, void* y, int32_t vec_dtype, void* fe_work, void* stream) {
    int rc = validate_mesh(mesh, moduli_dtype == DFEA_F32);
    if (rc) return rc;
    if (moduli_dtype == DFEA_F32REF && vec_dtype != DFEA_F64)
        return set_error(DFEA_ERR_INVALID, "DFEA_F32REF moduli apply to f64 vectors");
    if (!mesh->node_elem_ptr || !mesh->node_elem)
        return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply_gather: the mesh has no node incidence");
    if (!moduli || !v || !y || !fe_work) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply_gather: NULL pointer");
    if (v == y) return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply_gather: y must not alias v");
    if (!aligned16(moduli) || !aligned16(v) || !aligned16(y) || !aligned16(fe_work))
        return set_error(DFEA_ERR_INVALID, "dfea_tangent_apply_gather: moduli, v, y and fe_work must be 16-byte aligned");
    if (moduli_dtype != DFEA_F64 && moduli_dtype != DFEA_F32 && moduli_dtype != DFEA_F32REF)
        return set_error(DFEA_ERR_INVALID, "bad moduli dtype");
    if (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32) return set_error(DFEA_ERR_INVALID, "bad vector dtype");
    if (vec_dtype == DFEA_F32 && moduli_dtype != DFEA_F32)
        return set_error(DFEA_ERR_INVALID, "FP32 vectors need FP32 moduli");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    const int gn = grid_for(mesh->n_nodes, kThreads, 4);
    const RedSite none{nullptr, nullptr, nullptr};
    LaunchOpts pdl;
    pdl.pdl = true;
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        if (moduli_dtype == DFEA_F32REF) {
            const double* vv = static_cast<const double*>(v);
            double* fe = static_cast<double*>(fe_work);
            int r = launch_apply_ref_elem<NEN, NQ, double, false>(*mesh, static_cast<const float*>(moduli), vv, fe, none,
                                                                 nullptr, s);
            if (r) return r;
            return launch_kernel(k_node_gather<double>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mesh->node_elem_ptr,
                                 mesh->node_elem, (const double*)fe, vv, static_cast<double*>(y));
        }
        if (vec_dtype == DFEA_F64) {
            const double* vv = static_cast<const double*>(v);
            double* fe = static_cast<double*>(fe_work);
            int r = (moduli_dtype == DFEA_F64)
                        ? launch_apply_elem<NEN, NQ, double, double, false>(*mesh, static_cast<const double*>(moduli),
                                                                           mesh->grad, vv, fe, none, nullptr, s)
                        : launch_apply_elem<NEN, NQ, float, double, false>(*mesh, static_cast<const float*>(moduli),
                                                                          mesh->grad32, vv, fe, none, nullptr, s);
            if (r) return r;
            return launch_kernel(k_node_gather<double>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mesh->node_elem_ptr,
                                 mesh->node_elem, (const double*)fe, vv, static_cast<double*>(y));
        }
        const float* vv = static_cast<const float*>(v);
        float* fe = static_cast<float*>(fe_work);
        int r = launch_apply_elem<NEN, NQ, float, float, false>(*mesh, static_cast<const float*>(moduli), mesh->grad32,
                                                               vv, fe, none, nullptr, s);
        if (r) return r;
        return launch_kernel(k_node_gather<float>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mesh->node_elem_ptr,
                             mesh->node_elem, (const float*)fe, vv, static_cast<float*>(y));
    });
    if (rc) return rc;
    note_launches(2);
    return launch_check("dfea_tangent_apply_gather");
}

int dfea::mg_fe_gather_cheb(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype, void* fe_work, int mode,
                           const double* v, double* x, double* r, double* d, const double* b, const double* diag,
                           const double* coef, int last, cudaStream_t s) {
    int rc = validate_mesh(mesh, moduli_dtype == DFEA_F32);
    if (rc) return rc;
    if (!mesh->node_elem_ptr || !mesh->node_elem) return set_error(DFEA_ERR_INVALID, "multigrid smoothing: no node incidence");
    if (!moduli || !v || !fe_work || !r || !d || !diag || (!last && !coef) || (mode == MG_FE_STEP && !x) ||
        (mode == MG_FE_RESTART && !b))
        return set_error(DFEA_ERR_INVALID, "multigrid smoothing: NULL pointer");
    if (!aligned16(moduli) || !aligned16(v) || !aligned16(fe_work))
        return set_error(DFEA_ERR_INVALID, "multigrid smoothing: moduli, v and fe_work must be 16-byte aligned");
    if (moduli_dtype != DFEA_F64 && moduli_dtype != DFEA_F32 && moduli_dtype != DFEA_F32REF)
        return set_error(DFEA_ERR_INVALID, "bad moduli dtype");
    const Mesh m = kernel_mesh(*mesh);
    const int gn = grid_for(mesh->n_nodes, kThreads, 4);
    const RedSite none{nullptr, nullptr, nullptr};
    LaunchOpts pdl;
    pdl.pdl = true;
    double* fe = static_cast<double*>(fe_work);
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        if (moduli_dtype == DFEA_F32REF)
            return launch_apply_ref_elem<NEN, NQ, double, false>(*mesh, static_cast<const float*>(moduli), v, fe, none,
                                                                nullptr, s);
        if (moduli_dtype == DFEA_F64)
            return launch_apply_elem<NEN, NQ, double, double, false>(*mesh, static_cast<const double*>(moduli), mesh->grad,
                                                                    v, fe, none, nullptr, s);
        return launch_apply_elem<NEN, NQ, float, double, false>(*mesh, static_cast<const float*>(moduli), mesh->grad32, v,
                                                               fe, none, nullptr, s);
    });
    if (rc) return rc;
    rc = mode == MG_FE_STEP
             ? launch_kernel(k_node_gather_cheb<MG_FE_STEP>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mesh->node_elem_ptr,
                             mesh->node_elem, (const double*)fe, v, x, r, d, b, diag, coef, last)
             : launch_kernel(k_node_gather_cheb<MG_FE_RESTART>, dim3(gn), dim3(kThreads), 0, s, pdl, m,
                             mesh->node_elem_ptr, mesh->node_elem, (const double*)fe, v, x, r, d, b, diag, coef, last);
    if (rc) return rc;
    note_launches(2);
    return launch_check("multigrid smoothing");
}

extern "C" int64_t dfea_reduce_work_bytes(const dfea_mesh_view* mesh) {
    (void)mesh;
    return ReduceWork::bytes();
}

extern "C" int dfea_residual(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                             double lambda0, const double* f, double load_factor, double* R, double* out_norm2,
                             double* out_energy, void* work, void* stream) {
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_residual_mat(mesh, u, theta, &mat, f, load_factor, R, out_norm2, out_energy, work, stream);
}

extern "C" int dfea_residual_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                                 const dfea_material* material, const double* f, double load_factor, double* R,
                                 double* out_norm2, double* out_energy, void* work, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_material(material))) return rc;
    const dfea_material mat = *material;
    if (!u || !R) return set_error(DFEA_ERR_INVALID, "dfea_residual: NULL pointer");
    if ((out_norm2 || out_energy) && !work) return set_error(DFEA_ERR_INVALID, "dfea_residual: reductions need work");
    if (!aligned16(u) || !aligned16(R) || (f && !aligned16(f)) || (work && !aligned16(work)))
        return set_error(DFEA_ERR_INVALID, "dfea_residual: vectors must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    ReduceWork w(work);
    if (work) {
        k_zero_tickets<<<1, 128, 0, s>>>(w.tickets, ReduceWork::n_sites, w.results, ReduceWork::n_sites);
        note_launches(1);
    }
    k_residual_init<<<grid_for(mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(m, f, load_factor, R);
    note_launches(1);
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        return dispatch_material(mat, [&](auto gen_c) -> int {
            constexpr bool GEN = decltype(gen_c)::value;
            for (int c = 0; c < mesh->n_colours; ++c) {
                const int64_t e0 = mesh->colour_begin[c], e1 = mesh->colour_begin[c + 1];
                if (e1 <= e0) continue;
                const int grid = grid_for(e1 - e0, 128, 12);
                if (out_energy)
                    k_residual<NEN, NQ, true, true, GEN><<<grid, 128, 0, s>>>(m, e0, e1, u, theta, mat, R, w.site(1 + c));
                else
                    k_residual<NEN, NQ, false, true, GEN><<<grid, 128, 0, s>>>(m, e0, e1, u, theta, mat, R, RedSite{});
                note_launches(1);
            }
            return DFEA_OK;
        });
    });
    if (rc) return rc;
    if (out_norm2 || out_energy) {
        const int64_t n = 2 * mesh->n_nodes;
        k_norm2<<<grid_for(n, kThreads, 4), kThreads, 0, s>>>(n, R, w.site(0), out_norm2, w.results + 1,
                                                             mesh->n_colours, out_energy);
        note_launches(1);
    }
    return launch_check("dfea_residual");
}

extern "C" int dfea_vec_norm2(const dfea_mesh_view* mesh, const double* x, double* out, void* work, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!x || !out || !work) return set_error(DFEA_ERR_INVALID, "dfea_vec_norm2: NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ReduceWork w(work);
    k_zero_tickets<<<1, 128, 0, s>>>(w.tickets, ReduceWork::n_sites, w.results, ReduceWork::n_sites);
    note_launches(1);
    const int64_t n = 2 * mesh->n_nodes;
    k_norm2<<<grid_for(n, kThreads, 4), kThreads, 0, s>>>(n, x, w.site(0), out, nullptr, 0, nullptr);
    note_launches(1);
    return launch_check("dfea_vec_norm2");
}

extern "C" int dfea_element_sensitivity(const dfea_mesh_view* mesh, const double* u, const double* lam, double mu0,
                                        double lambda0, double* g, void* stream) {
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_element_sensitivity_mat(mesh, u, lam, &mat, g, stream);
}

extern "C" int dfea_element_sensitivity_mat(const dfea_mesh_view* mesh, const double* u, const double* lam,
                                            const dfea_material* material, double* g, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_material(material))) return rc;
    const unsigned linear = material_linear_mask(material->model);
    if (material->scalable & ~linear)
        return set_error(DFEA_ERR_UNSUPPORTED, "dfea_element_sensitivity: theta scales a parameter that enters the "
                                               "energy nonlinearly (scalable 0x%x, linear 0x%x)", material->scalable, linear);
    dfea_material slope = *material;  // d p_e / d theta_e
    for (int k = 0; k < DFEA_MAX_MAT_PARAMS; ++k)
        if (((linear >> k) & 1u) && !((material->scalable >> k) & 1u)) slope.p[k] = 0.0;
    if (!u || !lam || !g) return set_error(DFEA_ERR_INVALID, "dfea_element_sensitivity: NULL pointer");
    if (!aligned16(u) || !aligned16(lam)) return set_error(DFEA_ERR_INVALID, "u and lambda must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    if (mesh->n_el == 0) return DFEA_OK;
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        return dispatch_material(slope, [&](auto gen_c) -> int {
            constexpr bool GEN = decltype(gen_c)::value;
            k_sensitivity<NEN, NQ, GEN><<<grid_for(mesh->n_el, 128, 12), 128, 0, s>>>(m, u, lam, slope, g);
            note_launches(1);
            return DFEA_OK;
        });
    });
    if (rc) return rc;
    return launch_check("dfea_element_sensitivity");
}

extern "C" int dfea_axpy(int64_t n, double a, const double* x, double* y, void* stream) {
    if (n < 0 || (n > 0 && (!x || !y))) return set_error(DFEA_ERR_INVALID, "dfea_axpy: bad arguments");
    if (n == 0) return DFEA_OK;
    k_axpy<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, a, x, y);
    note_launches(1);
    return launch_check("dfea_axpy");
}

extern "C" int dfea_add_scaled(int64_t n, const double* a, double alpha, const double* b, double* out, void* stream) {
    if (n < 0 || (n > 0 && (!a || !b || !out))) return set_error(DFEA_ERR_INVALID, "dfea_add_scaled: bad arguments");
    if (n == 0) return DFEA_OK;
    k_add_scaled<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, a, alpha, b, out);
    note_launches(1);
    return launch_check("dfea_add_scaled");
}

extern "C" int dfea_f64_to_f32(int64_t n, const double* x, float* y, void* stream) {
    if (n < 0 || (n > 0 && (!x || !y))) return set_error(DFEA_ERR_INVALID, "dfea_f64_to_f32: bad arguments");
    if (n == 0) return DFEA_OK;
    k_to_f32<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, x, y);
    note_launches(1);
    return launch_check("dfea_f64_to_f32");
}

extern "C" int dfea_f32_to_f64(int64_t n, const float* x, double* y, void* stream) {
    if (n < 0 || (n > 0 && (!x || !y))) return set_error(DFEA_ERR_INVALID, "dfea_f32_to_f64: bad arguments");
    if (n == 0) return DFEA_OK;
    k_to_f64<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, x, y);
    note_launches(1);
    return launch_check("dfea_f32_to_f64");
}

extern "C" int dfea_element_fields(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                                   double lambda0, double* elem_out, void* stream) {
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_element_fields_mat(mesh, u, theta, &mat, elem_out, stream);
}

extern "C" int dfea_element_fields_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                                       const dfea_material* material, double* elem_out, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_material(material))) return rc;
    const dfea_material mat = *material;
    if (!u || !elem_out) return set_error(DFEA_ERR_INVALID, "dfea_element_fields: NULL pointer");
    if (!aligned16(u)) return set_error(DFEA_ERR_INVALID, "dfea_element_fields: u must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    const int grid = grid_for(mesh->n_el, 128, 12);
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        return dispatch_material(mat, [&](auto gen_c) -> int {
            constexpr bool GEN = decltype(gen_c)::value;
            k_element_fields<NEN, NQ, GEN><<<grid, 128, 0, s>>>(m, u, theta, mat, elem_out);
            return DFEA_OK;
        });
    });
    if (rc) return rc;
    note_launches(1);
    return launch_check("dfea_element_fields");
}

extern "C" int dfea_node_fields(const dfea_mesh_view* mesh, const double* elem, double* node_out, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!elem || !node_out) return set_error(DFEA_ERR_INVALID, "dfea_node_fields: NULL pointer");
    if (!mesh->node_elem_ptr || !mesh->node_elem)
        return set_error(DFEA_ERR_INVALID, "dfea_node_fields: the mesh has no node incidence");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_node_fields<<<grid_for(mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(kernel_mesh(*mesh), mesh->node_elem_ptr,
                                                                           mesh->node_elem, elem, node_out);
    note_launches(1);
    return launch_check("dfea_node_fields");
}

extern "C" int dfea_internal_force(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                                   double lambda0, double* R_int, void* stream) {
    const dfea_material mat = neo_hookean(mu0, lambda0);
    return dfea_internal_force_mat(mesh, u, theta, &mat, R_int, stream);
}

extern "C" int dfea_internal_force_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                                       const dfea_material* material, double* R_int, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_material(material))) return rc;
    const dfea_material mat = *material;
    if (!u || !R_int) return set_error(DFEA_ERR_INVALID, "dfea_internal_force: NULL pointer");
    if (!aligned16(u) || !aligned16(R_int)) return set_error(DFEA_ERR_INVALID, "dfea_internal_force: alignment");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Mesh m = kernel_mesh(*mesh);
    k_zero<<<grid_for(2 * mesh->n_nodes, kThreads, 8), kThreads, 0, s>>>(2 * mesh->n_nodes, R_int);
    note_launches(1);
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        return dispatch_material(mat, [&](auto gen_c) -> int {
            constexpr bool GEN = decltype(gen_c)::value;
            for (int c = 0; c < mesh->n_colours; ++c) {
                const int64_t e0 = mesh->colour_begin[c], e1 = mesh->colour_begin[c + 1];
                if (e1 <= e0) continue;
                k_residual<NEN, NQ, false, false, GEN><<<grid_for(e1 - e0, 128, 12), 128, 0, s>>>(m, e0, e1, u, theta, mat,
                                                                                                 R_int, RedSite{});
                note_launches(1);
            }
            return DFEA_OK;
        });
    });
    if (rc) return rc;
    return launch_check("dfea_internal_force");
}
