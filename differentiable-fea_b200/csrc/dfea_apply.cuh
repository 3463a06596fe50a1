// dfea_apply.cuh -- kernel (b): the stored-moduli tangent product, one colour per launch.
//
// For every element e of one colour (one thread per element, grid-stride):
//     gather     v_e[a,i] = (m * v)[dof(e,a,i)]                      (fix bits in conn, no mask reads)
//     contract   dgrad_iJ = sum_a v_e[a,i] dN_aJ ;  dP = C_q dgrad ;  f_e[a,i] += sum_J dP_iJ dN_aJ
//     scatter    y[dof] += f_e  on free DOFs                         (read-modify-write, no atomics)
// which is the `qp_ew` product of the reference (operators.py:403-410) element by element.
// Elements of one colour share no node, so the read-modify-write of y is race-free, and the
// colour order fixes the summation order: the result is bit-reproducible.
//
// With DOT the kernel also returns p.Ap restricted to free DOFs in energy form,
//     sum_e sum_q dgrad_q . C_q dgrad_q = (m p)^T J (m p),
// reduced per colour in fixed order: the curvature of PCG fused into the operator epilogue.
//
// Moduli and gradients are read once with streaming (evict-first) loads, so that the DOF vectors
// (a few % of the traffic, gathered ~nen times) stay resident in the 126 MB L2.
#pragma once

#include "dfea_common.cuh"

namespace dfea {

template <int NEN>
__host__ __device__ constexpr int apply_threads() { return NEN <= 4 ? 256 : 128; }

// y = (1 - m) * v : the Dirichlet identity pivot, written before the colour passes add m * J (m v).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pivot_init(Mesh m, const T* __restrict__ v, T* __restrict__ y) {
    using T2 = v2_t<T>;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    T2* y2 = reinterpret_cast<T2*>(y);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const T2 a = v2[n];
        y2[n] = make_v2<T>((fix & 1) ? a.x : T(0), (fix & 2) ? a.y : T(0));
    }
}

template <int NEN, int NQ, typename T, bool DOT>
__global__ void __launch_bounds__(apply_threads<NEN>())
k_apply(Mesh m, int64_t e0, int64_t e1, const T* __restrict__ C, const T* __restrict__ G,
        const T* __restrict__ v, T* __restrict__ y, RedSite site, const int* __restrict__ done) {
    constexpr int NT = apply_threads<NEN>();
    using T2 = v2_t<T>;
    if (DOT && done != nullptr && *done) return;  // solve finished: no-op iteration of the graph

    const int64_t S = m.stride;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    T2* y2 = reinterpret_cast<T2*>(y);
    double curv = 0.0;

    for (int64_t e = e0 + blockIdx.x * (int64_t)NT + threadIdx.x; e < e1; e += (int64_t)gridDim.x * NT) {
        int node[NEN], fix[NEN];
        T vx[NEN], vy[NEN], fx[NEN], fy[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const int c = __ldcs(m.conn + a * S + e);
            node[a] = c >> 2;
            fix[a] = c & 3;
            const T2 t = __ldg(v2 + node[a]);
            vx[a] = (fix[a] & 1) ? T(0) : t.x;
            vy[a] = (fix[a] & 2) ? T(0) : t.y;
            fx[a] = T(0);
            fy[a] = T(0);
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            T gx[NEN], gy[NEN];
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const T2 g = load_grad(G, (int64_t)(q * NEN + a) * S + e);
                gx[a] = g.x;
                gy[a] = g.y;
            }
            T d[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                d[0] += vx[a] * gx[a];
                d[1] += vx[a] * gy[a];
                d[2] += vy[a] * gx[a];
                d[3] += vy[a] * gy[a];
            }
            T dP[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                T row[4];
                load_moduli_row(C, S, q, r, e, row);
                dP[r] = row[0] * d[0] + row[1] * d[1] + row[2] * d[2] + row[3] * d[3];
            }
            if (DOT) curv += (double)(d[0] * dP[0] + d[1] * dP[1] + d[2] * dP[2] + d[3] * dP[3]);
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                fx[a] += dP[0] * gx[a] + dP[1] * gy[a];
                fy[a] += dP[2] * gx[a] + dP[3] * gy[a];
            }
        }
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            T2 t = y2[node[a]];
            if (!(fix[a] & 1)) t.x += fx[a];
            if (!(fix[a] & 2)) t.y += fy[a];
            y2[node[a]] = t;
        }
    }

    if (DOT) {
        const double vals[1] = {block_sum<NT>(curv)};
        double tot[1];
        if (last_block_sum<NT, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

// Launch the colour passes of one product on `stream` (the pivot init is launched by the caller).
// With DOT, colour c reduces into sites[c] (result = curvature of that colour).
template <int NEN, int NQ, typename T, bool DOT>
int launch_apply_colours(const dfea_mesh_view& mv, const T* C, const T* G, const T* v, T* y,
                         const RedSite* sites, const int* done, cudaStream_t stream, bool count = true) {
    constexpr int NT = apply_threads<NEN>();
    const Mesh m = kernel_mesh(mv);
    for (int c = 0; c < mv.n_colours; ++c) {
        const int64_t e0 = mv.colour_begin[c], e1 = mv.colour_begin[c + 1];
        if (e1 <= e0) continue;
        const int grid = grid_for(e1 - e0, NT, NT == 256 ? 8 : 12);
        const RedSite site = DOT ? sites[c] : RedSite{nullptr, nullptr, nullptr};
        k_apply<NEN, NQ, T, DOT><<<grid, NT, 0, stream>>>(m, e0, e1, C, G, v, y, site, done);
        if (count) note_launches(1);
    }
    return launch_check("k_apply");
}

}  // namespace dfea
