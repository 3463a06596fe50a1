// dfea_pcg.cu -- kernel (c): Jacobi-preconditioned CG resident on the device.
//
// The reference runs PCG in Python with three host synchronisations per iteration
// (newton_krylov.py:28-88).  Here one iteration is
//     colour passes of k_apply<DOT>   Ap = A p  and  p.Ap (energy form, per colour, fixed order)
//     k_pcg_update1                   alpha = rz / pAp;  x += alpha p;  r -= alpha Ap;
//                                     |r|^2 and r.z with z = r / diag   (z is never stored)
//     k_pcg_update2                   convergence test; beta; p = z + beta p; Ap := (1 - m) p
//                                     (the pivot term of the next product); sum of fixed p^2
//     k_pcg_cond                      sets the condition of the graph's while-loop node
// captured once in a CUDA graph whose conditional WHILE node repeats it on the device, so that a
// whole solve is one graph launch and one read-back.  Scalars (rz, |r|^2, status, k) live in a
// device state block; every reduction is a fixed-order two-level sum (no float atomics).
//
// Termination does not depend on the numerics: k_pcg_update2 stops at max_iter and k_pcg_cond keeps
// an independent execution counter that ends the loop after max_iter + 4 bodies in any case.
#include <cstring>
#include <mutex>
#include <new>
#include <type_traits>

#include "dfea_apply.cuh"
#include "dfea_common.cuh"

namespace dfea {

int validate_mesh(const dfea_mesh_view* mv, bool need_grad32);

struct PcgState {
    double rz;      // r.z of the current iterate
    double rr;      // |r|^2 after the last update   (result[0] of the update-1 site)
    double rz_new;  // r.z after the last update     (result[1] of the update-1 site)
    double norm_b;
    double rtol;
    double pfix;    // sum of p^2 over fixed DOFs (identity rows of A)
    double curv;    // last p.Ap
    double beta;    // fused form: beta of the last update (0 before the first iteration)
    double curv_c[DFEA_MAX_COLOURS];
    int32_t k;
    int32_t max_iter;
    int32_t done;
    int32_t iters;
    int32_t guard;
    int32_t spare_i[3];
    unsigned tickets[DFEA_MAX_COLOURS + 8];
};

// Work buffer: [r | p | Ap] vectors (2N each, 256-byte aligned), partials, state, and for the gather
// form the element results fe (nen * stride pairs) at the end.
struct PcgLayout {
    int64_t off_r, off_p, off_y, off_part, off_state, off_fe, total;
    PcgLayout(int64_t n_nodes, int vec_bytes, int n_colours, int64_t fe_pairs = 0) {
        auto up = [](int64_t x) { return (x + 255) / 256 * 256; };
        const int64_t vb = up(2 * n_nodes * vec_bytes);
        off_r = 0;
        off_p = vb;
        off_y = 2 * vb;
        off_part = 3 * vb;
        const int64_t n_sites = n_colours + 3;
        off_state = off_part + up(n_sites * 3 * (int64_t)kMaxBlocks * 8);
        off_fe = off_state + up(sizeof(PcgState));
        total = off_fe + up(fe_pairs * 2 * vec_bytes);
    }
};

// The preconditioner z = M^-1 r at node n.  BJ = false: point Jacobi, d = diag (2N);  BJ = true: nodal
// block-Jacobi, d = the inverse 2x2 blocks (Binv00, Binv01, Binv11, 0) per node (4N, double vectors only).
template <bool BJ, typename T>
__device__ __forceinline__ v2_t<T> precond(const T* __restrict__ d, int64_t n, v2_t<T> r) {
    if constexpr (BJ) {
        const double2* b2 = reinterpret_cast<const double2*>(d);
        const double2 a = b2[2 * n], b = b2[2 * n + 1];
        return make_v2<T>((T)(a.x * r.x + a.y * r.y), (T)(a.y * r.x + b.x * r.y));
    } else {
        const v2_t<T> dn = reinterpret_cast<const v2_t<T>*>(d)[n];
        return make_v2<T>(r.x / dn.x, r.y / dn.y);
    }
}

__global__ void k_pcg_reset(PcgState* st) {
    const int i = threadIdx.x;
    if (i < DFEA_MAX_COLOURS + 8) st->tickets[i] = 0u;
    if (i < DFEA_MAX_COLOURS) st->curv_c[i] = 0.0;
    if (i == 0) {
        st->done = DFEA_PCG_RUNNING;
        st->k = 0;
        st->iters = 0;
        st->guard = 0;
    }
}

// x = 0, r = b, z = b / d, p = z, Ap := (1 - m) p;  rz = r.z, |b|, pfix.
template <typename T, bool BJ>
__global__ void __launch_bounds__(kThreads)
k_pcg_setup(Mesh m, const T* __restrict__ b, const T* __restrict__ d, T* __restrict__ x, T* __restrict__ r,
            T* __restrict__ p, T* __restrict__ y, PcgState* st, RedSite site, double rtol, int max_iter) {
    using T2 = v2_t<T>;
    double rz = 0.0, bb = 0.0, pf = 0.0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const T2 bn = reinterpret_cast<const T2*>(b)[n];
        const T2 zn = precond<BJ, T>(d, n, bn);
        const T zx = zn.x, zy = zn.y;
        reinterpret_cast<T2*>(x)[n] = make_v2<T>(T(0), T(0));
        reinterpret_cast<T2*>(r)[n] = bn;
        reinterpret_cast<T2*>(p)[n] = make_v2<T>(zx, zy);
        reinterpret_cast<T2*>(y)[n] = make_v2<T>((fix & 1) ? zx : T(0), (fix & 2) ? zy : T(0));
        rz += (double)bn.x * zx + (double)bn.y * zy;
        bb += (double)bn.x * bn.x + (double)bn.y * bn.y;
        if (fix & 1) pf += (double)zx * zx;
        if (fix & 2) pf += (double)zy * zy;
    }
    const double vals[3] = {block_sum<kThreads>(rz), block_sum<kThreads>(bb), block_sum<kThreads>(pf)};
    double tot[3];
    if (last_block_sum<kThreads, 3>(vals, site, tot) && threadIdx.x == 0) {
        st->rz = tot[0];
        st->norm_b = sqrt(tot[1]);
        st->pfix = tot[2];
        st->beta = 0.0;
        st->rtol = rtol;
        st->max_iter = max_iter;
        st->k = 0;
        st->iters = 0;
        st->guard = 0;
        st->done = (st->norm_b == 0.0) ? DFEA_PCG_ZERO_RHS : DFEA_PCG_RUNNING;
    }
}

// GATHER: Ap is not stored; each node sums its elements' results (fe, the element pass of the gather
// form) in the incidence order, and takes p on its fixed DOFs (the identity rows).
// The body of update 1 for block blk of nblk (one launch, or one solve's share of a batched launch).
template <typename T, bool GATHER, bool BJ>
__device__ __forceinline__ void pcg_update1_body(const Mesh& m, int n_colours, const T* __restrict__ p,
                                                 const T* __restrict__ y, const T* __restrict__ d, T* __restrict__ x,
                                                 T* __restrict__ r, PcgState* st, const RedSite& site,
                                                 const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                                                 const T* __restrict__ fe, int64_t blk, int64_t nblk) {
    using T2 = v2_t<T>;
    if (st->done) return;
    double curv = st->pfix;
    for (int c = 0; c < n_colours; ++c) curv += st->curv_c[c];
    const int k = st->k;
    if (curv <= 0.0) {
        // not SPD along p: return z at k = 0 and x otherwise (newton_krylov.py:69-70)
        if (k == 0) {
            for (int64_t n = blk * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)nblk * blockDim.x) {
                const T2 rn = reinterpret_cast<const T2*>(r)[n];
                reinterpret_cast<T2*>(x)[n] = precond<BJ, T>(d, n, rn);
            }
        }
        const double vals[1] = {0.0};
        double tot[1];
        if (last_block_sum_in<kThreads, 1>(vals, site, tot, blk, nblk) && threadIdx.x == 0) {
            st->curv = curv;
            st->iters = k;
            st->done = DFEA_PCG_NEG_CURV;
        }
        return;
    }
    const double alpha = st->rz / curv;
    const T a = (T)alpha;
    double rr = 0.0, rz = 0.0;
    for (int64_t n = blk * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)nblk * blockDim.x) {
        const T2 pn = reinterpret_cast<const T2*>(p)[n];
        T2 yn;
        if constexpr (GATHER) {
            const int fix = m.node_fix[n];
            const T2 f = node_sum<T>(inc_ptr, inc, reinterpret_cast<const T2*>(fe), n);
            yn = make_v2<T>((fix & 1) ? pn.x : f.x, (fix & 2) ? pn.y : f.y);
        } else {
            yn = reinterpret_cast<const T2*>(y)[n];
        }
        T2 xn = reinterpret_cast<const T2*>(x)[n];
        T2 rn = reinterpret_cast<const T2*>(r)[n];
        xn.x += a * pn.x;
        xn.y += a * pn.y;
        rn.x -= a * yn.x;
        rn.y -= a * yn.y;
        reinterpret_cast<T2*>(x)[n] = xn;
        reinterpret_cast<T2*>(r)[n] = rn;
        rr += (double)rn.x * rn.x + (double)rn.y * rn.y;
        const T2 zn = precond<BJ, T>(d, n, rn);
        rz += (double)rn.x * zn.x + (double)rn.y * zn.y;
    }
    const double vals[2] = {block_sum<kThreads>(rr), block_sum<kThreads>(rz)};
    double tot[2];
    if (last_block_sum_in<kThreads, 2>(vals, site, tot, blk, nblk) && threadIdx.x == 0) {
        st->rr = tot[0];
        st->rz_new = tot[1];
        st->curv = curv;
    }
}

template <typename T, bool GATHER, bool BJ>
__global__ void __launch_bounds__(kThreads)
k_pcg_update1(Mesh m, int n_colours, const T* __restrict__ p, const T* __restrict__ y, const T* __restrict__ d,
              T* __restrict__ x, T* __restrict__ r, PcgState* st, RedSite site, const int32_t* __restrict__ inc_ptr,
              const int32_t* __restrict__ inc, const T* __restrict__ fe) {
    grid_dependency_wait();  // launched with PDL: everything below reads the predecessors' results
    grid_dependents_launch();
    pcg_update1_body<T, GATHER, BJ>(m, n_colours, p, y, d, x, r, st, site, inc_ptr, inc, fe, blockIdx.x, gridDim.x);
}

// PIVOT: write Ap := (1 - m) p, the identity rows the colour passes then add to (the colour form).
template <typename T, bool PIVOT, bool BJ>
__device__ __forceinline__ void pcg_update2_body(const Mesh& m, const T* __restrict__ r, const T* __restrict__ d,
                                                 T* __restrict__ p, T* __restrict__ y, PcgState* st,
                                                 const RedSite& site, int64_t blk, int64_t nblk) {
    using T2 = v2_t<T>;
    if (st->done) return;
    const int k = st->k;
    if (sqrt(st->rr) <= st->rtol * st->norm_b) {
        // converged: ||r|| <= rtol ||b||  (newton_krylov.py:77-79)
        const double vals[1] = {0.0};
        double tot[1];
        if (last_block_sum_in<kThreads, 1>(vals, site, tot, blk, nblk) && threadIdx.x == 0) {
            st->iters = k + 1;
            st->done = DFEA_PCG_CONVERGED;
        }
        return;
    }
    const double beta = st->rz_new / st->rz;
    const T bt = (T)beta;
    double pf = 0.0;
    for (int64_t n = blk * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)nblk * blockDim.x) {
        const int fix = m.node_fix[n];
        const T2 rn = reinterpret_cast<const T2*>(r)[n];
        const T2 zn = precond<BJ, T>(d, n, rn);
        T2 pn = reinterpret_cast<const T2*>(p)[n];
        pn.x = zn.x + bt * pn.x;
        pn.y = zn.y + bt * pn.y;
        reinterpret_cast<T2*>(p)[n] = pn;
        if (PIVOT) reinterpret_cast<T2*>(y)[n] = make_v2<T>((fix & 1) ? pn.x : T(0), (fix & 2) ? pn.y : T(0));
        if (fix & 1) pf += (double)pn.x * pn.x;
        if (fix & 2) pf += (double)pn.y * pn.y;
    }
    const double vals[1] = {block_sum<kThreads>(pf)};
    double tot[1];
    if (last_block_sum_in<kThreads, 1>(vals, site, tot, blk, nblk) && threadIdx.x == 0) {
        st->rz = st->rz_new;
        st->pfix = tot[0];
        st->k = k + 1;
        if (k + 1 >= st->max_iter) {
            st->iters = st->max_iter;
            st->done = DFEA_PCG_MAX_ITER;
        }
    }
}

template <typename T, bool PIVOT, bool BJ>
__global__ void __launch_bounds__(kThreads)
k_pcg_update2(Mesh m, const T* __restrict__ r, const T* __restrict__ d, T* __restrict__ p, T* __restrict__ y,
              PcgState* st, RedSite site) {
    grid_dependency_wait();
    grid_dependents_launch();
    pcg_update2_body<T, PIVOT, BJ>(m, r, d, p, y, st, site, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------------------------------------
// Fused gather form: 2 kernels per iteration.  The direction update p_k = M^-1 r_k + beta_{k-1} p_{k-1}
// moves out of the second vector kernel: the element pass computes p_k at the nodes it gathers, and the
// node pass computes it again (same expression, same bits) and stores it.  The node pass also sums the
// element results (Ap), updates x and r, reduces |r|^2 and r.z, and its last block does the scalar step
// (convergence test, beta, k).  The identity rows' part of p.Ap (fixed DOFs) is added by the element
// pass, counted once per node by the node's first incidence slot.
// ------------------------------------------------------------------------------------------------
template <bool BJ, typename T>
__device__ __forceinline__ v2_t<T> next_direction(const T* __restrict__ d, int64_t n, v2_t<T> r, v2_t<T> p, T beta) {
    const v2_t<T> z = precond<BJ, T>(d, n, r);
    return make_v2<T>(z.x + beta * p.x, z.y + beta * p.y);
}

template <typename T, bool BJ, int NEN>
__device__ __forceinline__ void fused_scatter(int64_t e, int64_t S, const int (&node)[NEN], const int (&fix)[NEN],
                                              const T (&fx)[NEN], const T (&fy)[NEN], v2_t<T>* __restrict__ fe2,
                                              const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                                              const T* __restrict__ d, const v2_t<T>* __restrict__ r2,
                                              const v2_t<T>* __restrict__ p2, T beta, double& pfix) {
#pragma unroll
    for (int a = 0; a < NEN; ++a) fe2[(int64_t)a * S + e] = make_v2<T>(fx[a], fy[a]);
#pragma unroll
    for (int a = 0; a < NEN; ++a) {
        if (fix[a] && inc[inc_ptr[node[a]]] == (int32_t)((int64_t)a * S + e)) {
            const v2_t<T> pn = next_direction<BJ, T>(d, node[a], __ldg(r2 + node[a]), __ldg(p2 + node[a]), beta);
            if (fix[a] & 1) pfix += (double)pn.x * pn.x;
            if (fix[a] & 2) pfix += (double)pn.y * pn.y;
        }
    }
}

template <int NEN, int NQ, typename SD, typename T, bool BJ>
__global__ void __launch_bounds__(128)
k_pcg_elem_fused(Mesh m, const SD* __restrict__ C, const SD* __restrict__ G, const T* __restrict__ r,
                 const T* __restrict__ d, const T* __restrict__ p, T* __restrict__ fe, const int32_t* __restrict__ inc_ptr,
                 const int32_t* __restrict__ inc, PcgState* st, RedSite site) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    const T2* r2 = reinterpret_cast<const T2*>(r);
    const T2* p2 = reinterpret_cast<const T2*>(p);
    T2* fe2 = reinterpret_cast<T2*>(fe);
    double curv = 0.0, pfix = 0.0;
    T beta = T(0);
    const bool ran = apply_tiles<NEN, NQ, SD, T, true>(
        m, 0, m.n_el, C, G, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (st->done) return false;
            beta = (T)st->beta;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return next_direction<BJ, T>(d, n, __ldg(r2 + n), __ldg(p2 + n), beta); },
        [&](int64_t e, const int (&node)[NEN], const int (&fix)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
            fused_scatter<T, BJ, NEN>(e, m.stride, node, fix, fx, fy, fe2, inc_ptr, inc, d, r2, p2, beta, pfix);
        });
    if (!ran) return;
    const double vals[1] = {block_sum<128>(curv + pfix)};
    double tot[1];
    if (last_block_sum<128, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
}

template <int NEN, int NQ, typename T, bool BJ>
__global__ void __launch_bounds__(128)
k_pcg_elem_fused_ref(Mesh m, const float* __restrict__ C, const RefGrad<NEN, NQ> rg, const T* __restrict__ r,
                     const T* __restrict__ d, const T* __restrict__ p, T* __restrict__ fe,
                     const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc, PcgState* st, RedSite site) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    const T2* r2 = reinterpret_cast<const T2*>(r);
    const T2* p2 = reinterpret_cast<const T2*>(p);
    T2* fe2 = reinterpret_cast<T2*>(fe);
    double curv = 0.0, pfix = 0.0;
    T beta = T(0);
    const bool ran = apply_tiles_ref<NEN, NQ, T, true>(
        m, 0, m.n_el, C, rg, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (st->done) return false;
            beta = (T)st->beta;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return next_direction<BJ, T>(d, n, __ldg(r2 + n), __ldg(p2 + n), beta); },
        [&](int64_t e, const int (&node)[NEN], const int (&fix)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
            fused_scatter<T, BJ, NEN>(e, m.stride, node, fix, fx, fy, fe2, inc_ptr, inc, d, r2, p2, beta, pfix);
        });
    if (!ran) return;
    const double vals[1] = {block_sum<128>(curv + pfix)};
    double tot[1];
    if (last_block_sum<128, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
}

template <typename T, bool BJ>
__global__ void __launch_bounds__(kThreads)
k_pcg_node_fused(Mesh m, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc, const T* __restrict__ fe,
                 const T* __restrict__ d, T* __restrict__ x, T* __restrict__ r, T* __restrict__ p, PcgState* st,
                 RedSite site) {
    using T2 = v2_t<T>;
    grid_dependency_wait();
    grid_dependents_launch();
    if (st->done) return;
    const double curv = st->curv_c[0];
    const int k = st->k;
    if (curv <= 0.0) {
        // not SPD along p: return z at k = 0 and x otherwise (newton_krylov.py:69-70)
        if (k == 0) {
            for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x)
                reinterpret_cast<T2*>(x)[n] = precond<BJ, T>(d, n, reinterpret_cast<const T2*>(r)[n]);
        }
        const double vals[1] = {0.0};
        double tot[1];
        if (last_block_sum<kThreads, 1>(vals, site, tot) && threadIdx.x == 0) {
            st->curv = curv;
            st->iters = k;
            st->done = DFEA_PCG_NEG_CURV;
        }
        return;
    }
    const T a = (T)(st->rz / curv);
    const T beta = (T)st->beta;
    const T2* fe2 = reinterpret_cast<const T2*>(fe);
    double rr = 0.0, rz = 0.0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        T2 rn = reinterpret_cast<const T2*>(r)[n];
        const T2 pn = next_direction<BJ, T>(d, n, rn, reinterpret_cast<const T2*>(p)[n], beta);
        reinterpret_cast<T2*>(p)[n] = pn;
        const T2 f = node_sum<T>(inc_ptr, inc, fe2, n);
        const T2 yn = make_v2<T>((fix & 1) ? pn.x : f.x, (fix & 2) ? pn.y : f.y);
        T2 xn = reinterpret_cast<const T2*>(x)[n];
        xn.x += a * pn.x;
        xn.y += a * pn.y;
        rn.x -= a * yn.x;
        rn.y -= a * yn.y;
        reinterpret_cast<T2*>(x)[n] = xn;
        reinterpret_cast<T2*>(r)[n] = rn;
        const T2 zn = precond<BJ, T>(d, n, rn);
        rr += (double)rn.x * rn.x + (double)rn.y * rn.y;
        rz += (double)rn.x * zn.x + (double)rn.y * zn.y;
    }
    const double vals[2] = {block_sum<kThreads>(rr), block_sum<kThreads>(rz)};
    double tot[2];
    if (last_block_sum<kThreads, 2>(vals, site, tot) && threadIdx.x == 0) {
        st->rr = tot[0];
        st->curv = curv;
        if (sqrt(tot[0]) <= st->rtol * st->norm_b) {  // newton_krylov.py:77-79
            st->iters = k + 1;
            st->done = DFEA_PCG_CONVERGED;
        } else {
            st->beta = tot[1] / st->rz;
            st->rz = tot[1];
            st->k = k + 1;
            if (k + 1 >= st->max_iter) {
                st->iters = st->max_iter;
                st->done = DFEA_PCG_MAX_ITER;
            }
        }
    }
}

__global__ void k_pcg_cond(PcgState* st, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    const int g = ++st->guard;
    if (st->done == DFEA_PCG_RUNNING && g >= st->max_iter + 4) {
        st->iters = st->max_iter;
        st->done = DFEA_PCG_MAX_ITER;
    }
    cudaGraphSetConditional(h, st->done == DFEA_PCG_RUNNING ? 1u : 0u);
}

}  // namespace dfea

using namespace dfea;

struct dfea_pcg {
    dfea_mesh_view mesh;
    const void* moduli;
    const void* diag;
    const void* b;
    void* x;
    int vec_dtype;
    char* work;
    PcgLayout layout{1, 8, 1};
    int use_graph;
    bool gather = false;             // product in the gather form (element pass + node sums in update 1)
    int grid_cap = 0;                // most blocks per launch (0: as many as the GPU holds)
    bool block = false;              // nodal block-Jacobi: diag holds the inverse 2x2 blocks (4N doubles)
    bool fused = false;              // fused gather form: 2 kernels per iteration
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // [done, iters, bodies]: read after the stream has reached the copy, staged through the library's pool of
    // page-locked blocks (a page-locked allocation per handle cost a device-wide driver call per solve set up).
    int32_t status_buf[4] = {0, 0, 0, 0};
    int32_t* host_status = status_buf;

    PcgState* state() const { return reinterpret_cast<PcgState*>(work + layout.off_state); }
    RedSite site(int i, int k_slot_results) const {
        double* parts = reinterpret_cast<double*>(work + layout.off_part) + (int64_t)i * 3 * kMaxBlocks;
        PcgState* st = state();
        (void)k_slot_results;
        double* res = nullptr;
        if (i < mesh.n_colours) res = st->curv_c + i;          // colour curvature
        else if (i == mesh.n_colours) res = &st->rr;            // update 1: rr, rz_new
        return RedSite{parts, st->tickets + i, res};
    }
};

namespace {

// Kernels of one iteration without the loop condition: the non-empty colour passes and two updates
// (colour form), or the element pass and two updates (gather form).
int kernels_per_iteration(const dfea_pcg& h) {
    if (h.fused) return 2;
    if (h.gather) return 3;
    int nonempty = 0;
    for (int c = 0; c < h.mesh.n_colours; ++c) nonempty += h.mesh.colour_begin[c + 1] > h.mesh.colour_begin[c];
    return nonempty + 2;
}

// S: storage type of moduli and gradients, T: Krylov vector type; REF: DFEA_F32REF moduli (S = float),
// no gradients read.
template <typename S, typename T, bool REF = false, bool BJ = false>
int launch_iteration(const dfea_pcg& h, cudaStream_t s, cudaGraphConditionalHandle cond, bool with_cond) {
    const dfea_mesh_view& mv = h.mesh;
    const Mesh m = kernel_mesh(mv);
    const S* C = static_cast<const S*>(h.moduli);
    const S* G = std::is_same<S, float>::value ? reinterpret_cast<const S*>(mv.grad32) : reinterpret_cast<const S*>(mv.grad);
    T* r = reinterpret_cast<T*>(h.work + h.layout.off_r);
    T* p = reinterpret_cast<T*>(h.work + h.layout.off_p);
    T* y = reinterpret_cast<T*>(h.work + h.layout.off_y);
    const T* d = static_cast<const T*>(h.diag);
    T* x = static_cast<T*>(h.x);
    PcgState* st = h.state();
    const int gn = capped(grid_for(mv.n_nodes, kThreads, 4), h.grid_cap);
    LaunchOpts pdl;
    pdl.pdl = true;
    int rc;
    if (h.fused) {
        T* fe = reinterpret_cast<T*>(h.work + h.layout.off_fe);
        rc = dispatch_element(mv.nen, mv.n_q, [&](auto nen_c, auto nq_c) -> int {
            constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
            long long max_window = 0;
            const long long setaside = persisting_l2_bytes(&max_window);
            LaunchOpts opts;
            opts.pdl = true;
            // r and p (adjacent in the work buffer) are gathered by every element: keep them in L2
            L2Window w = l2_window(r, p, (size_t)(2 * mv.n_nodes) * sizeof(T));
            if ((long long)w.bytes > max_window) w.bytes = (size_t)max_window;
            if (setaside > 0 && w.bytes > 0) {
                opts.win_base = w.base;
                opts.win_bytes = w.bytes;
                opts.hit_ratio = setaside >= (long long)w.bytes ? 1.0f : (float)((double)setaside / (double)w.bytes);
            }
            if constexpr (REF) {
                const int grid = capped(resident_grid<k_pcg_elem_fused_ref<NEN, NQ, T, BJ>, RefApplyCfg<NEN>::SMEM, 128>(mv.n_el),
                                        h.grid_cap);
                return launch_kernel(k_pcg_elem_fused_ref<NEN, NQ, T, BJ>, dim3(grid), dim3(128), RefApplyCfg<NEN>::SMEM,
                                     s, opts, m, reinterpret_cast<const float*>(C), ref_grad_of<NEN, NQ>(mv), (const T*)r,
                                     d, (const T*)p, fe, mv.node_elem_ptr, mv.node_elem, st, h.site(0, 1));
            } else {
                using Cfg = ApplyCfg<NEN, S>;
                const int grid = capped(resident_grid<k_pcg_elem_fused<NEN, NQ, S, T, BJ>, Cfg::SMEM, Cfg::NT>(mv.n_el),
                                        h.grid_cap);
                return launch_kernel(k_pcg_elem_fused<NEN, NQ, S, T, BJ>, dim3(grid), dim3(Cfg::NT), Cfg::SMEM, s, opts,
                                     m, C, G, (const T*)r, d, (const T*)p, fe, mv.node_elem_ptr, mv.node_elem, st,
                                     h.site(0, 1));
            }
        });
        if (rc) return rc;
        if ((rc = launch_kernel(k_pcg_node_fused<T, BJ>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mv.node_elem_ptr,
                                mv.node_elem, (const T*)fe, d, x, r, p, st, h.site(mv.n_colours, 2))))
            return rc;
    } else if (h.gather) {
        // element pass (curvature into site 0, read as colour 0), node sums fused into update 1
        T* fe = reinterpret_cast<T*>(h.work + h.layout.off_fe);
        rc = dispatch_element(mv.nen, mv.n_q, [&](auto nen_c, auto nq_c) -> int {
            constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
            if constexpr (REF)
                return launch_apply_ref_elem<NEN, NQ, T, true>(mv, reinterpret_cast<const float*>(C), p, fe, h.site(0, 1),
                                                               &st->done, s, h.grid_cap);
            else
                return launch_apply_elem<NEN, NQ, S, T, true>(mv, C, G, p, fe, h.site(0, 1), &st->done, s, h.grid_cap);
        });
        if (rc) return rc;
        if ((rc = launch_kernel(k_pcg_update1<T, true, BJ>, dim3(gn), dim3(kThreads), 0, s, pdl, m, 1, p, (const T*)y, d, x,
                                r, st, h.site(mv.n_colours, 2), mv.node_elem_ptr, mv.node_elem, (const T*)fe)))
            return rc;
        if ((rc = launch_kernel(k_pcg_update2<T, false, BJ>, dim3(gn), dim3(kThreads), 0, s, pdl, m, (const T*)r, d, p, y,
                                st, h.site(mv.n_colours + 1, 1))))
            return rc;
    } else {
        RedSite sites[DFEA_MAX_COLOURS];
        for (int c = 0; c < mv.n_colours; ++c) sites[c] = h.site(c, 1);
        rc = dispatch_element(mv.nen, mv.n_q, [&](auto nen_c, auto nq_c) -> int {
            constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
            if constexpr (REF)
                return launch_apply_ref_colours<NEN, NQ, T, true>(mv, reinterpret_cast<const float*>(C), p, y, sites,
                                                                  &st->done, s, h.grid_cap);
            else
                return launch_apply_colours<NEN, NQ, S, T, true>(mv, C, G, p, y, sites, &st->done, s, false,
                                                                 h.grid_cap);
        });
        if (rc) return rc;
        if ((rc = launch_kernel(k_pcg_update1<T, false, BJ>, dim3(gn), dim3(kThreads), 0, s, pdl, m, mv.n_colours, p,
                                (const T*)y, d, x, r, st, h.site(mv.n_colours, 2), (const int32_t*)nullptr,
                                (const int32_t*)nullptr, (const T*)nullptr)))
            return rc;
        if ((rc = launch_kernel(k_pcg_update2<T, true, BJ>, dim3(gn), dim3(kThreads), 0, s, pdl, m, (const T*)r, d, p, y,
                                st, h.site(mv.n_colours + 1, 1))))
            return rc;
    }
    if (with_cond) k_pcg_cond<<<1, 32, 0, s>>>(st, cond);
    else note_launches(kernels_per_iteration(h));  // graph-captured kernels are counted when the solve returns
    return launch_check("pcg iteration");
}

int launch_iteration_any(const dfea_pcg& h, cudaStream_t s, cudaGraphConditionalHandle cond, bool with_cond) {
    if (h.block) {  // block-Jacobi: double vectors only (checked at create)
        if (h.vec_dtype == DFEA_F64) return launch_iteration<double, double, false, true>(h, s, cond, with_cond);
        if (h.vec_dtype == DFEA_MIXED) return launch_iteration<float, double, false, true>(h, s, cond, with_cond);
        return launch_iteration<float, double, true, true>(h, s, cond, with_cond);
    }
    if (h.vec_dtype == DFEA_F64) return launch_iteration<double, double>(h, s, cond, with_cond);
    if (h.vec_dtype == DFEA_MIXED) return launch_iteration<float, double>(h, s, cond, with_cond);
    if (h.vec_dtype == DFEA_F32REF) return launch_iteration<float, double, true>(h, s, cond, with_cond);
    return launch_iteration<float, float>(h, s, cond, with_cond);
}

template <typename T, bool BJ = false>
int launch_setup(const dfea_pcg& h, cudaStream_t s, double rtol, int max_iter) {
    const dfea_mesh_view& mv = h.mesh;
    const Mesh m = kernel_mesh(mv);
    T* r = reinterpret_cast<T*>(h.work + h.layout.off_r);
    T* p = reinterpret_cast<T*>(h.work + h.layout.off_p);
    T* y = reinterpret_cast<T*>(h.work + h.layout.off_y);
    PcgState* st = h.state();
    k_pcg_reset<<<1, 128, 0, s>>>(st);
    k_pcg_setup<T, BJ><<<grid_for(mv.n_nodes, kThreads, 4), kThreads, 0, s>>>(
        m, static_cast<const T*>(h.b), static_cast<const T*>(h.diag), static_cast<T*>(h.x), r, p, y, st,
        h.site(mv.n_colours + 2, 3), rtol, max_iter);
    note_launches(2);
    return launch_check("pcg setup");
}

int build_graph(dfea_pcg* h) {
    int rc;
    if ((rc = check_cuda(cudaGraphCreate(&h->graph, 0), "cudaGraphCreate"))) return rc;
    cudaGraphConditionalHandle cond;
    if ((rc = check_cuda(cudaGraphConditionalHandleCreate(&cond, h->graph, 1u, cudaGraphCondAssignDefault),
                         "cudaGraphConditionalHandleCreate")))
        return rc;
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};  // aggregate init: the rest is zero
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((rc = check_cuda(cudaGraphAddNode(&node, h->graph, nullptr, 0, &cp), "cudaGraphAddNode(while)"))) return rc;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((rc = check_cuda(cudaStreamBeginCaptureToGraph(h->capture_stream, body, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal),
                         "cudaStreamBeginCaptureToGraph")))
        return rc;
    rc = launch_iteration_any(*h, h->capture_stream, cond, true);
    cudaGraph_t captured = body;
    const int rc_end = check_cuda(cudaStreamEndCapture(h->capture_stream, &captured), "cudaStreamEndCapture");
    if (rc) return rc;
    if (rc_end) return rc_end;
    return check_cuda(cudaGraphInstantiate(&h->exec, h->graph, 0), "cudaGraphInstantiate");
}

// Unrolled form: kUnrolled iterations captured back to back in a plain graph (no conditional node),
// replayed by the host until the status word reports an end.  Iterations after the end are no-ops.
constexpr int kUnrolled = 8;

int build_unrolled_graph(dfea_pcg* h) {
    int rc;
    if ((rc = check_cuda(cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal),
                         "cudaStreamBeginCapture")))
        return rc;
    for (int i = 0; i < kUnrolled && rc == DFEA_OK; ++i) rc = launch_iteration_any(*h, h->capture_stream, 0, false);
    cudaGraph_t g = nullptr;
    const int rc_end = check_cuda(cudaStreamEndCapture(h->capture_stream, &g), "cudaStreamEndCapture");
    h->graph = g;
    if (rc) return rc;
    if (rc_end) return rc_end;
    return check_cuda(cudaGraphInstantiate(&h->exec, h->graph, 0), "cudaGraphInstantiate");
}

void release(dfea_pcg* h) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
    delete h;
}

}  // namespace

namespace {
// the layout of a handle: with room for the gather form's element results when the mesh has the
// node incidence that form needs
PcgLayout layout_for(const dfea_mesh_view& mv, int32_t vec_dtype) {
    const int64_t fe_pairs = (mv.node_elem_ptr && mv.node_elem) ? (int64_t)mv.nen * mv.stride : 0;
    return PcgLayout(mv.n_nodes, vec_dtype == DFEA_F32 ? 4 : 8, mv.n_colours, fe_pairs);
}
}  // namespace

extern "C" int64_t dfea_pcg_work_bytes(const dfea_mesh_view* mesh, int32_t vec_dtype) {
    if (!mesh || (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32 && vec_dtype != DFEA_MIXED && vec_dtype != DFEA_F32REF))
        return -1;
    return layout_for(*mesh, vec_dtype).total;
}

extern "C" int dfea_pcg_create(const dfea_mesh_view* mesh, const void* moduli, const void* diag, const void* b,
                               void* x, int32_t vec_dtype, void* work, int32_t use_graph, dfea_pcg** out) {
    if (!out) return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: out is NULL");
    *out = nullptr;
    int rc = validate_mesh(mesh, vec_dtype == DFEA_F32 || vec_dtype == DFEA_MIXED);
    if (rc) return rc;
    if (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32 && vec_dtype != DFEA_MIXED && vec_dtype != DFEA_F32REF)
        return set_error(DFEA_ERR_INVALID, "bad vector dtype");
    if (!moduli || !diag || !b || !x || !work) return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: NULL pointer");
    auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 255u) == 0; };
    auto al16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (!al(work)) return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: work must be 256-byte aligned");
    if (!al16(moduli) || !al16(diag) || !al16(b) || !al16(x))
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: moduli, diag, b and x must be 16-byte aligned");
    if (x == b) return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: x must not alias b");

    dfea_pcg* h = new (std::nothrow) dfea_pcg;
    if (!h) return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: out of host memory");
    h->mesh = *mesh;
    h->moduli = moduli;
    h->diag = diag;
    h->b = b;
    h->x = x;
    h->vec_dtype = vec_dtype;
    h->work = static_cast<char*>(work);
    h->layout = layout_for(*mesh, vec_dtype);
    h->gather = (use_graph & DFEA_PCG_GATHER) != 0;
    h->block = (use_graph & DFEA_PCG_BLOCK_JACOBI) != 0;
    h->fused = (use_graph & DFEA_PCG_FUSED) != 0;
    if (h->fused) h->gather = true;
    h->grid_cap = (int)((uint32_t)use_graph >> 8);
    use_graph &= 0xff & ~(DFEA_PCG_GATHER | DFEA_PCG_BLOCK_JACOBI | DFEA_PCG_FUSED);
    if (h->block && vec_dtype == DFEA_F32) {
        delete h;
        return set_error(DFEA_ERR_UNSUPPORTED, "dfea_pcg_create: block-Jacobi needs f64 Krylov vectors");
    }
    h->use_graph = (use_graph == 2) ? 2 : (use_graph ? 1 : 0);
    if (h->gather && h->layout.off_fe == h->layout.total) {
        delete h;
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_create: the gather form needs the mesh's node incidence");
    }
    // device queries and kernel attributes are set up before any stream capture
    (void)device_sm_count();
    dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        if (vec_dtype == DFEA_F64) prepare_apply<NEN, NQ, double, double>();
        else if (vec_dtype == DFEA_MIXED) prepare_apply<NEN, NQ, float, double>();
        else if (vec_dtype == DFEA_F32REF) prepare_apply_ref<NEN, NQ, double>();
        else prepare_apply<NEN, NQ, float, float>();
        if (h->fused) {  // the fused element pass of this handle's types
            if (vec_dtype == DFEA_F32REF) {
                if (h->block) (void)resident_grid<k_pcg_elem_fused_ref<NEN, NQ, double, true>, RefApplyCfg<NEN>::SMEM, 128>(1);
                else (void)resident_grid<k_pcg_elem_fused_ref<NEN, NQ, double, false>, RefApplyCfg<NEN>::SMEM, 128>(1);
            } else if (vec_dtype == DFEA_F64) {
                using Cfg = ApplyCfg<NEN, double>;
                if (h->block) (void)resident_grid<k_pcg_elem_fused<NEN, NQ, double, double, true>, Cfg::SMEM, Cfg::NT>(1);
                else (void)resident_grid<k_pcg_elem_fused<NEN, NQ, double, double, false>, Cfg::SMEM, Cfg::NT>(1);
            } else if (vec_dtype == DFEA_MIXED) {
                using Cfg = ApplyCfg<NEN, float>;
                if (h->block) (void)resident_grid<k_pcg_elem_fused<NEN, NQ, float, double, true>, Cfg::SMEM, Cfg::NT>(1);
                else (void)resident_grid<k_pcg_elem_fused<NEN, NQ, float, double, false>, Cfg::SMEM, Cfg::NT>(1);
            } else {
                using Cfg = ApplyCfg<NEN, float>;
                (void)resident_grid<k_pcg_elem_fused<NEN, NQ, float, float, false>, Cfg::SMEM, Cfg::NT>(1);
            }
        }
        return DFEA_OK;
    });
    if ((rc = check_cuda(cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking), "cudaStreamCreate"))) {
        release(h);
        return rc;
    }
    // zero the partial sums, tickets and state once (later solves reset what they use)
    if ((rc = check_cuda(cudaMemsetAsync(h->work + h->layout.off_part, 0, h->layout.total - h->layout.off_part,
                                         h->capture_stream), "cudaMemsetAsync")) ||
        (rc = check_cuda(cudaStreamSynchronize(h->capture_stream), "cudaStreamSynchronize"))) {
        release(h);
        return rc;
    }
    if (h->use_graph == 1 && (rc = build_graph(h))) {
        release(h);
        return rc;
    }
    if (h->use_graph == 2 && (rc = build_unrolled_graph(h))) {
        release(h);
        return rc;
    }
    *out = h;
    return DFEA_OK;
}

extern "C" int dfea_pcg_solve(dfea_pcg* h, double rtol, int32_t max_iter, int32_t* iters, int32_t* status,
                              void* stream) {
    if (!h) return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve: NULL handle");
    if (max_iter < 1 || max_iter > 100000000) return set_error(DFEA_ERR_INVALID, "max_iter %d out of [1, 1e8]", max_iter);
    if (!(rtol >= 0.0)) return set_error(DFEA_ERR_INVALID, "rtol must be >= 0");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = (h->vec_dtype == DFEA_F32) ? launch_setup<float>(*h, s, rtol, max_iter)
             : h->block                 ? launch_setup<double, true>(*h, s, rtol, max_iter)
                                        : launch_setup<double>(*h, s, rtol, max_iter);
    if (rc) return rc;
    PcgState* st = h->state();
    if (h->use_graph == 2) {
        int launched = 0;
        h->host_status[0] = DFEA_PCG_RUNNING;
        while (true) {
            if ((rc = check_cuda(cudaGraphLaunch(h->exec, s), "cudaGraphLaunch"))) return rc;
            launched += kUnrolled;
            if ((rc = read_to_host(h->host_status, &st->done, 2 * sizeof(int32_t), s))) return rc;
            if (h->host_status[0] != DFEA_PCG_RUNNING || launched > max_iter + kUnrolled) break;
        }
        note_launches((long long)launched * kernels_per_iteration(*h));
    } else if (h->use_graph) {
        if ((rc = check_cuda(cudaGraphLaunch(h->exec, s), "cudaGraphLaunch"))) return rc;
        if ((rc = read_to_host(h->host_status, &st->done, 3 * sizeof(int32_t), s))) return rc;
        // each executed body ran one iteration's kernels and the loop condition
        note_launches((long long)h->host_status[2] * (kernels_per_iteration(*h) + 1));
    } else {
        // the same kernels launched directly; the host reads the status every 16 iterations
        const int chunk = 16;
        int launched = 0;
        h->host_status[0] = DFEA_PCG_RUNNING;
        while (true) {
            for (int i = 0; i < chunk; ++i) {
                rc = launch_iteration_any(*h, s, 0, false);
                if (rc) return rc;
            }
            launched += chunk;
            if ((rc = read_to_host(h->host_status, &st->done, 2 * sizeof(int32_t), s))) return rc;
            if (h->host_status[0] != DFEA_PCG_RUNNING || launched > max_iter + chunk) break;
        }
    }
    if (h->host_status[0] == DFEA_PCG_RUNNING)
        return set_error(DFEA_ERR_INVALID, "PCG ended without a status (internal error)");
    if (status) *status = h->host_status[0];
    if (iters) *iters = h->host_status[1];
    return DFEA_OK;
}

extern "C" int dfea_pcg_destroy(dfea_pcg* h) {
    if (h) release(h);
    return DFEA_OK;
}

// ------------------------------------------------------------------------------------------------
// Allocation-free PCG: the work area is a file-scope device array instead of a caller buffer.
// ------------------------------------------------------------------------------------------------
// Reserved in each GPU's memory when the library's module is loaded there; kept until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DFEA_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxColours = 16;
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch for the current device.  In host code the symbol itself is a
// host-side stand-in, so the address is looked up once per device, with that device current.
int noalloc_scratch(void** out) {
    int dev = 0;
    int rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if (dev < 0 || dev >= kNoallocMaxDevices) return set_error(DFEA_ERR_INVALID, "device ordinal %d unsupported", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[dev] == nullptr) {
        void* p = nullptr;
        rc = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(g_noalloc_scratch)");
        if (rc) return rc;
        g_noalloc_address[dev] = p;
    }
    *out = g_noalloc_address[dev];
    return DFEA_OK;
}

}  // namespace

extern "C" int dfea_pcg_solve_noalloc(const dfea_mesh_view* mesh, const void* moduli, const void* diag, const void* b,
                                      void* x, int32_t vec_dtype, double rtol, int32_t max_iter, int32_t* iters,
                                      int32_t* status, void* stream) {
    int rc = validate_mesh(mesh, vec_dtype != DFEA_F64);
    if (rc) return rc;
    if (vec_dtype != DFEA_F64 && vec_dtype != DFEA_F32 && vec_dtype != DFEA_MIXED)
        return set_error(DFEA_ERR_INVALID, "bad vector dtype");
    if (!moduli || !diag || !b || !x) return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: NULL pointer");
    auto al16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (!al16(moduli) || !al16(diag) || !al16(b) || !al16(x))
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: moduli, diag, b and x must be 16-byte aligned");
    if (x == b) return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: x must not alias b");
    if (mesh->n_nodes > DFEA_NOALLOC_MAX_NODES)
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: %lld nodes exceed the fixed scratch limit of %d nodes",
                         (long long)mesh->n_nodes, DFEA_NOALLOC_MAX_NODES);
    if (mesh->n_colours > kNoallocMaxColours)
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: %d colours exceed the limit of %d", mesh->n_colours,
                         kNoallocMaxColours);
    if (max_iter < 1 || max_iter > 100000000) return set_error(DFEA_ERR_INVALID, "max_iter %d out of [1, 1e8]", max_iter);
    if (!(rtol >= 0.0)) return set_error(DFEA_ERR_INVALID, "rtol must be >= 0");
    const PcgLayout layout(mesh->n_nodes, vec_dtype == DFEA_F32 ? 4 : 8, mesh->n_colours);
    if (layout.total > DFEA_NOALLOC_SCRATCH_BYTES)
        return set_error(DFEA_ERR_INVALID, "dfea_pcg_solve_noalloc: needs %lld scratch bytes, the fixed array has %d",
                         (long long)layout.total, DFEA_NOALLOC_SCRATCH_BYTES);
    void* scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;

    // A handle on the stack bound to the fixed scratch: no graph, no stream, no pinned buffer.
    dfea_pcg h;
    int32_t host_status[4] = {DFEA_PCG_RUNNING, 0, 0, 0};
    h.mesh = *mesh;
    h.moduli = moduli;
    h.diag = diag;
    h.b = b;
    h.x = x;
    h.vec_dtype = vec_dtype;
    h.work = static_cast<char*>(scratch);
    h.layout = layout;
    h.use_graph = 0;
    h.host_status = host_status;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    (void)device_sm_count();
    // k_pcg_reset (first kernel of the setup) clears the tickets and state the previous call left behind
    rc = (vec_dtype == DFEA_F32) ? launch_setup<float>(h, s, rtol, max_iter) : launch_setup<double>(h, s, rtol, max_iter);
    if (rc) return rc;
    PcgState* st = h.state();
    const int chunk = 16;
    int launched = 0;
    while (true) {
        for (int i = 0; i < chunk; ++i) {
            rc = launch_iteration_any(h, s, 0, false);
            if (rc) return rc;
        }
        launched += chunk;
        if ((rc = check_cuda(cudaMemcpyAsync(host_status, &st->done, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s),
                             "cudaMemcpyAsync")) ||
            (rc = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
            return rc;
        if (host_status[0] != DFEA_PCG_RUNNING || launched > max_iter + chunk) break;
    }
    if (host_status[0] == DFEA_PCG_RUNNING) return set_error(DFEA_ERR_INVALID, "PCG ended without a status (internal error)");
    if (status) *status = host_status[0];
    if (iters) *iters = host_status[1];
    return DFEA_OK;
}

// ------------------------------------------------------------------------------------------------
// Batched PCG: the solves of several handles advance together, one set of launches per iteration for
// all of them (an element pass per element type, one launch of each vector update).  Every block works
// for one solve (a block map gives the solve and the block's number within it); each solve keeps its
// own state, partial sums and tickets.  A solve's blocks are as many, and split its work the same way,
// as when it runs alone with the same block cap, so its iterates are bitwise those of its own handle.
// Supported handles: gather form (not fused), Jacobi, DFEA_F32REF moduli on f64 vectors (the serving
// configuration).
// ------------------------------------------------------------------------------------------------
namespace dfea {

struct BatchSolve {
    Mesh m;
    const int32_t* inc_ptr;
    const int32_t* inc;
    const float* C;
    const double* d;
    double* x;
    double* r;
    double* p;
    double* fe;
    PcgState* st;
    RedSite site_elem, site_u1, site_u2;
    int elem_blocks;
    int node_blocks;
};

template <int NEN, int NQ>
__global__ void __launch_bounds__(128)
k_batch_elem(const BatchSolve* __restrict__ solves, const int2* __restrict__ block_map, const RefGrad<NEN, NQ> rg) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int2 bm = block_map[blockIdx.x];
    const BatchSolve* S = solves + bm.x;
    const Mesh m = S->m;
    PcgState* st = S->st;
    const double2* p2 = reinterpret_cast<const double2*>(S->p);
    double2* fe2 = reinterpret_cast<double2*>(S->fe);
    const int64_t Sd = m.stride;
    double curv = 0.0;
    const bool ran = apply_tiles_ref<NEN, NQ, double, true>(
        m, 0, m.n_el, S->C, rg, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (st->done) return false;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return __ldg(p2 + n); },
        [&](int64_t e, const int (&)[NEN], const int (&)[NEN], const double (&fx)[NEN], const double (&fy)[NEN]) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) fe2[(int64_t)a * Sd + e] = make_double2(fx[a], fy[a]);
        },
        bm.y, S->elem_blocks);
    if (!ran) return;
    const double vals[1] = {block_sum<128>(curv)};
    double tot[1];
    if (last_block_sum_in<128, 1>(vals, S->site_elem, tot, bm.y, S->elem_blocks) && threadIdx.x == 0)
        S->site_elem.result[0] = tot[0];
}

__global__ void __launch_bounds__(kThreads) k_batch_update1(const BatchSolve* __restrict__ solves,
                                                           const int2* __restrict__ block_map) {
    grid_dependency_wait();
    grid_dependents_launch();
    const int2 bm = block_map[blockIdx.x];
    const BatchSolve* S = solves + bm.x;
    pcg_update1_body<double, true, false>(S->m, 1, S->p, S->p, S->d, S->x, S->r, S->st, S->site_u1, S->inc_ptr, S->inc,
                                          S->fe, bm.y, S->node_blocks);
}

__global__ void __launch_bounds__(kThreads) k_batch_update2(const BatchSolve* __restrict__ solves,
                                                           const int2* __restrict__ block_map) {
    grid_dependency_wait();
    grid_dependents_launch();
    const int2 bm = block_map[blockIdx.x];
    const BatchSolve* S = solves + bm.x;
    pcg_update2_body<double, false, false>(S->m, S->r, S->d, S->p, S->p, S->st, S->site_u2, bm.y, S->node_blocks);
}

__global__ void k_batch_status(const BatchSolve* __restrict__ solves, int n, int32_t* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[2 * i] = solves[i].st->done;
        out[2 * i + 1] = solves[i].st->iters;
    }
}

}  // namespace dfea

struct dfea_batch {
    int capacity = 0;
    int max_blocks = 0;
    int n = 0;
    BatchSolve* d_solves = nullptr;
    BatchSolve* h_solves = nullptr;  // pinned
    int2* d_map = nullptr;
    int2* h_map = nullptr;           // pinned: element maps by type, then the node map
    int32_t* d_status = nullptr;
    int32_t* h_status = nullptr;     // pinned
    int map_entries = 0;
    struct TypeRange {
        int nen, nq, first, count;   // element-map entries [first, first + count)
        dfea_mesh_view view;         // a view of this type (for its reference gradients)
    } types[8];
    int n_types = 0;
    int node_first = 0, node_count = 0;
};

namespace {

void batch_release(dfea_batch* b) {
    if (b->d_solves) cudaFree(b->d_solves);
    if (b->d_map) cudaFree(b->d_map);
    if (b->d_status) cudaFree(b->d_status);
    if (b->h_solves) cudaFreeHost(b->h_solves);
    if (b->h_map) cudaFreeHost(b->h_map);
    if (b->h_status) cudaFreeHost(b->h_status);
    delete b;
}

}  // namespace

extern "C" int dfea_batch_create(int32_t capacity, int32_t max_blocks, dfea_batch** out) {
    if (!out) return set_error(DFEA_ERR_INVALID, "dfea_batch_create: out is NULL");
    *out = nullptr;
    if (capacity < 1 || capacity > 4096) return set_error(DFEA_ERR_INVALID, "dfea_batch_create: capacity out of [1, 4096]");
    if (max_blocks < 1 || max_blocks > kMaxBlocks)
        return set_error(DFEA_ERR_INVALID, "dfea_batch_create: max_blocks out of [1, %d]", kMaxBlocks);
    dfea_batch* b = new (std::nothrow) dfea_batch;
    if (!b) return set_error(DFEA_ERR_INVALID, "dfea_batch_create: out of host memory");
    b->capacity = capacity;
    b->max_blocks = max_blocks;
    b->map_entries = 2 * capacity * max_blocks;  // element blocks + node blocks, at most max_blocks each
    int rc;
    if ((rc = check_cuda(cudaMalloc(&b->d_solves, sizeof(BatchSolve) * capacity), "cudaMalloc")) ||
        (rc = check_cuda(cudaMalloc(&b->d_map, sizeof(int2) * b->map_entries), "cudaMalloc")) ||
        (rc = check_cuda(cudaMalloc(&b->d_status, sizeof(int32_t) * 2 * capacity), "cudaMalloc")) ||
        (rc = check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&b->h_solves), sizeof(BatchSolve) * capacity,
                                       cudaHostAllocDefault), "cudaHostAlloc")) ||
        (rc = check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&b->h_map), sizeof(int2) * b->map_entries,
                                       cudaHostAllocDefault), "cudaHostAlloc")) ||
        (rc = check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&b->h_status), sizeof(int32_t) * 2 * capacity,
                                       cudaHostAllocDefault), "cudaHostAlloc"))) {
        batch_release(b);
        return rc;
    }
    *out = b;
    return DFEA_OK;
}

extern "C" int dfea_batch_destroy(dfea_batch* b) {
    if (b) batch_release(b);
    return DFEA_OK;
}

extern "C" int dfea_batch_start(dfea_batch* b, dfea_pcg* h, double rtol, int32_t max_iter, void* stream) {
    if (!b || !h) return set_error(DFEA_ERR_INVALID, "dfea_batch_start: NULL pointer");
    if (!h->gather || h->fused || h->block || h->vec_dtype != DFEA_F32REF)
        return set_error(DFEA_ERR_UNSUPPORTED,
                         "dfea_batch_start: batched solves need the gather form, Jacobi and DFEA_F32REF moduli");
    if (max_iter < 1 || max_iter > 100000000) return set_error(DFEA_ERR_INVALID, "max_iter %d out of [1, 1e8]", max_iter);
    if (!(rtol >= 0.0)) return set_error(DFEA_ERR_INVALID, "rtol must be >= 0");
    return launch_setup<double>(*h, static_cast<cudaStream_t>(stream), rtol, max_iter);
}

extern "C" int dfea_batch_set(dfea_batch* b, dfea_pcg* const* solves, int32_t n, void* stream) {
    if (!b || (n > 0 && !solves)) return set_error(DFEA_ERR_INVALID, "dfea_batch_set: NULL pointer");
    if (n < 0 || n > b->capacity) return set_error(DFEA_ERR_INVALID, "dfea_batch_set: %d solves, capacity %d", n, b->capacity);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the previous table may still be read by launched kernels: wait for them before rewriting it
    int rc = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (rc) return rc;
    b->n = n;
    b->n_types = 0;
    int entries = 0;
    for (int i = 0; i < n; ++i) {
        const dfea_pcg& h = *solves[i];
        if (!h.gather || h.fused || h.block || h.vec_dtype != DFEA_F32REF)
            return set_error(DFEA_ERR_UNSUPPORTED, "dfea_batch_set: solve %d is not in the batched configuration", i);
        const dfea_mesh_view& mv = h.mesh;
        BatchSolve& S = b->h_solves[i];
        S.m = kernel_mesh(mv);
        S.inc_ptr = mv.node_elem_ptr;
        S.inc = mv.node_elem;
        S.C = static_cast<const float*>(h.moduli);
        S.d = static_cast<const double*>(h.diag);
        S.x = static_cast<double*>(h.x);
        S.r = reinterpret_cast<double*>(h.work + h.layout.off_r);
        S.p = reinterpret_cast<double*>(h.work + h.layout.off_p);
        S.fe = reinterpret_cast<double*>(h.work + h.layout.off_fe);
        S.st = h.state();
        S.site_elem = h.site(0, 1);
        S.site_u1 = h.site(mv.n_colours, 2);
        S.site_u2 = h.site(mv.n_colours + 1, 1);
        const int cap = h.grid_cap > 0 ? h.grid_cap : b->max_blocks;
        rc = dispatch_element(mv.nen, mv.n_q, [&](auto nen_c, auto nq_c) -> int {
            constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
            S.elem_blocks = capped(apply_ref_elem_grid<NEN, NQ, double, true>(mv.n_el), cap);
            (void)resident_grid<k_batch_elem<NEN, NQ>, RefApplyCfg<NEN>::SMEM, 128>(1);  // shared-memory attribute
            return DFEA_OK;
        });
        if (rc) return rc;
        S.node_blocks = capped(grid_for(mv.n_nodes, kThreads, 4), cap);
        if (S.elem_blocks > b->max_blocks || S.node_blocks > b->max_blocks)
            return set_error(DFEA_ERR_INVALID, "dfea_batch_set: solve %d needs more blocks than the batch's cap", i);
    }
    // element maps grouped by element type, then the node map
    for (int i = 0; i < n; ++i) {
        const dfea_mesh_view& mv = solves[i]->mesh;
        int t = 0;
        while (t < b->n_types && !(b->types[t].nen == mv.nen && b->types[t].nq == mv.n_q)) ++t;
        if (t == b->n_types) {
            if (b->n_types == 8) return set_error(DFEA_ERR_UNSUPPORTED, "dfea_batch_set: too many element types");
            b->types[t] = {mv.nen, mv.n_q, 0, 0, mv};
            ++b->n_types;
        } else if (std::memcmp(b->types[t].view.ref_grad, mv.ref_grad, sizeof(double) * mv.nen * mv.n_q * 2) != 0) {
            // one launch per element type passes one table of reference gradients
            return set_error(DFEA_ERR_INVALID, "dfea_batch_set: solves of one element type differ in ref_grad");
        }
    }
    for (int t = 0; t < b->n_types; ++t) {
        b->types[t].first = entries;
        for (int i = 0; i < n; ++i) {
            const dfea_mesh_view& mv = solves[i]->mesh;
            if (mv.nen != b->types[t].nen || mv.n_q != b->types[t].nq) continue;
            for (int k = 0; k < b->h_solves[i].elem_blocks; ++k) b->h_map[entries++] = make_int2(i, k);
        }
        b->types[t].count = entries - b->types[t].first;
    }
    b->node_first = entries;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < b->h_solves[i].node_blocks; ++k) b->h_map[entries++] = make_int2(i, k);
    b->node_count = entries - b->node_first;
    if (n == 0) return DFEA_OK;
    if ((rc = check_cuda(cudaMemcpyAsync(b->d_solves, b->h_solves, sizeof(BatchSolve) * n, cudaMemcpyHostToDevice, s),
                         "cudaMemcpyAsync")) ||
        (rc = check_cuda(cudaMemcpyAsync(b->d_map, b->h_map, sizeof(int2) * entries, cudaMemcpyHostToDevice, s),
                         "cudaMemcpyAsync")))
        return rc;
    return DFEA_OK;
}

extern "C" int dfea_batch_iterate(dfea_batch* b, int32_t n_iterations, int32_t* status, int32_t* iters, void* stream) {
    if (!b) return set_error(DFEA_ERR_INVALID, "dfea_batch_iterate: NULL batch");
    if (n_iterations < 0 || n_iterations > 1000000) return set_error(DFEA_ERR_INVALID, "n_iterations out of range");
    if (b->n == 0) return DFEA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    LaunchOpts pdl;
    pdl.pdl = true;
    int rc = DFEA_OK;
    for (int it = 0; it < n_iterations && rc == DFEA_OK; ++it) {
        for (int t = 0; t < b->n_types && rc == DFEA_OK; ++t) {
            const auto& ty = b->types[t];
            rc = dispatch_element(ty.nen, ty.nq, [&](auto nen_c, auto nq_c) -> int {
                constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
                return launch_kernel(k_batch_elem<NEN, NQ>, dim3(ty.count), dim3(128), RefApplyCfg<NEN>::SMEM, s, pdl,
                                     (const BatchSolve*)b->d_solves, (const int2*)(b->d_map + ty.first),
                                     ref_grad_of<NEN, NQ>(ty.view));
            });
        }
        if (rc) break;
        if ((rc = launch_kernel(k_batch_update1, dim3(b->node_count), dim3(kThreads), 0, s, pdl,
                                (const BatchSolve*)b->d_solves, (const int2*)(b->d_map + b->node_first))))
            break;
        rc = launch_kernel(k_batch_update2, dim3(b->node_count), dim3(kThreads), 0, s, pdl, (const BatchSolve*)b->d_solves,
                           (const int2*)(b->d_map + b->node_first));
    }
    if (rc) return rc;
    note_launches((long long)n_iterations * (b->n_types + 2));
    k_batch_status<<<1, 128, 0, s>>>(b->d_solves, b->n, b->d_status);
    if ((rc = launch_check("k_batch_status")) ||
        (rc = check_cuda(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(int32_t) * 2 * b->n, cudaMemcpyDeviceToHost, s),
                         "cudaMemcpyAsync")) ||
        (rc = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
        return rc;
    for (int i = 0; i < b->n; ++i) {
        if (status) status[i] = b->h_status[2 * i];
        if (iters) iters[i] = b->h_status[2 * i + 1];
    }
    return DFEA_OK;
}
