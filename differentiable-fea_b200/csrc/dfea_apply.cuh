// dfea_apply.cuh -- kernel (b): the stored-moduli tangent product, one colour per launch.
//
// For every element e of one colour (one thread per element):
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
// Memory pipeline.  The kernel is persistent (a grid of a few blocks per SM walks tiles of 128
// elements) and streams the moduli and gradients through shared memory with cp.async: the unit of
// the pipeline is one (tile, Gauss point) item -- 8 x 16 B of moduli and nen x 16 B of gradients per
// element in FP64 -- and STAGES items are in flight per thread, so each SM keeps ~100 KB of loads
// outstanding without spending registers on them.  Each thread copies and later reads only its own
// element's slots (layout [row][thread], conflict-free), so the pipeline needs no block barrier.
// The copies bypass L1 and stream through L2 once.  The DOF vectors (a few % of the traffic, but
// gathered and scattered once per colour pass) are kept in L2 across the passes by an access-policy
// window on the launch that marks them persisting (see `l2_window`).
#pragma once

#include <mutex>

#include "dfea_common.cuh"

namespace dfea {

// ------------------------------------------------------------------------------------------
// cp.async helpers (asynchronous global -> shared copies)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const size_t g = __cvta_generic_to_global(gmem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const size_t g = __cvta_generic_to_global(gmem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const size_t g = __cvta_generic_to_global(gmem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T> struct ApplyUnits;
template <> struct ApplyUnits<double> {
    using CU = double2;              // one pair of moduli entries
    using GU = double2;              // (dN/dX, dN/dY)
    static constexpr int CROWS = 8;  // CU units per Gauss point
};
template <> struct ApplyUnits<float> {
    using CU = float4;               // one row of the 4x4 moduli
    using GU = float2;
    static constexpr int CROWS = 4;
};

template <int NEN, typename T>
struct ApplyCfg {
    using CU = typename ApplyUnits<T>::CU;
    using GU = typename ApplyUnits<T>::GU;
    static constexpr int NT = 128;
    static constexpr int CROWS = ApplyUnits<T>::CROWS;
    static constexpr int STAGES = (sizeof(T) == 8 && NEN > 4) ? 3 : 4;
    static constexpr int C_BYTES = CROWS * 16 * NT;                 // moduli of one item
    static constexpr int G_BYTES = NEN * (int)sizeof(GU) * NT;      // gradients of one item
    static constexpr int N_BYTES = NEN * 4 * NT;                    // connectivity (tile's first item)
    static constexpr int STAGE_BYTES = C_BYTES + G_BYTES + N_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES;
};

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

// The body of kernel (b) for elements [e0, e1), walked by this block in tiles of 128 (one element per
// thread).  `start()` runs after the prologue's prefetches were issued and before any vector is read;
// returning false abandons the walk (after draining the copies).  `scatter(e, node, fix, fx, fy)`
// receives each element's result f_e.  With DOT the curvature contributions are added to `curv`.
// SD: storage type of the moduli and gradients; T: type of the DOF vectors and of the arithmetic
// (SD = float, T = double is the mixed form: FP32 operator data, FP64 Krylov vectors).
template <int NEN, int NQ, typename SD, typename T, bool DOT, typename Start, typename Gather, typename Scatter>
__device__ __forceinline__ bool apply_tiles(const Mesh& m, int64_t e0, int64_t e1, const SD* __restrict__ C,
                                            const SD* __restrict__ G, unsigned char* smem, double& curv, Start&& start,
                                            Gather&& gather, Scatter&& scatter) {
    using Cfg = ApplyCfg<NEN, SD>;
    using CU = typename Cfg::CU;
    using GU = typename Cfg::GU;
    using T2 = v2_t<T>;
    constexpr int NT = Cfg::NT, ST = Cfg::STAGES, CR = Cfg::CROWS;

    const int tid = threadIdx.x;
    const int64_t S = m.stride;
    const int64_t n_tiles = (e1 - e0 + NT - 1) / NT;
    const int64_t my_tiles = (n_tiles > (int64_t)blockIdx.x) ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t n_items = my_tiles * NQ;
    const CU* Cg = reinterpret_cast<const CU*>(C);
    const GU* Gg = reinterpret_cast<const GU*>(G);

    auto element_of = [&](int64_t item) -> int64_t {
        return e0 + ((int64_t)blockIdx.x + (item / NQ) * (int64_t)gridDim.x) * NT + tid;
    };
    auto c_slot = [&](int s, int k) -> CU* {
        return reinterpret_cast<CU*>(smem + s * Cfg::STAGE_BYTES) + k * NT + tid;
    };
    auto g_slot = [&](int s, int a) -> GU* {
        return reinterpret_cast<GU*>(smem + s * Cfg::STAGE_BYTES + Cfg::C_BYTES) + a * NT + tid;
    };
    auto n_slot = [&](int s, int a) -> int* {
        return reinterpret_cast<int*>(smem + s * Cfg::STAGE_BYTES + Cfg::C_BYTES + Cfg::G_BYTES) + a * NT + tid;
    };
    // prefetch item `it` (its moduli, gradients, and at a tile's first point its connectivity)
    auto issue = [&](int64_t it) {
        if (it < n_items) {
            const int64_t e = element_of(it);
            if (e < e1) {
                const int q = (int)(it % NQ), s = (int)(it % ST);
#pragma unroll
                for (int k = 0; k < CR; ++k) cp_async16(c_slot(s, k), Cg + (int64_t)(q * CR + k) * S + e);
#pragma unroll
                for (int a = 0; a < NEN; ++a) {
                    if (sizeof(GU) == 16) cp_async16(g_slot(s, a), Gg + (int64_t)(q * NEN + a) * S + e);
                    else cp_async8(g_slot(s, a), Gg + (int64_t)(q * NEN + a) * S + e);
                }
                if (q == 0) {
#pragma unroll
                    for (int a = 0; a < NEN; ++a) cp_async4(n_slot(s, a), m.conn + (int64_t)a * S + e);
                }
            }
        }
        cp_async_commit();  // empty groups keep the group count uniform
    };

#pragma unroll
    for (int i = 0; i < ST - 1; ++i) issue(i);  // moduli/gradients/connectivity: no predecessor writes them

    if (!start()) {
        cp_async_wait<0>();
        return false;
    }

    int node[NEN], fix[NEN];
    T vx[NEN], vy[NEN], fx[NEN], fy[NEN];
#pragma unroll
    for (int a = 0; a < NEN; ++a) {
        node[a] = 0;
        fix[a] = 3;
        vx[a] = vy[a] = fx[a] = fy[a] = T(0);
    }

    for (int64_t it = 0; it < n_items; ++it) {
        issue(it + ST - 1);
        cp_async_wait<ST - 1>();  // item `it` has landed (groups complete in order)
        const int64_t e = element_of(it);
        if (e >= e1) continue;
        const int q = (int)(it % NQ), s = (int)(it % ST);
        if (q == 0) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const int c = *n_slot(s, a);
                node[a] = c >> 2;
                fix[a] = c & 3;
            }
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                const T2 t = gather(node[a]);
                vx[a] = (fix[a] & 1) ? T(0) : t.x;
                vy[a] = (fix[a] & 2) ? T(0) : t.y;
                fx[a] = T(0);
                fy[a] = T(0);
            }
        }
        T gx[NEN], gy[NEN];
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            const GU g = *g_slot(s, a);
            gx[a] = (T)g.x;
            gy[a] = (T)g.y;
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
        if constexpr (sizeof(SD) == 8) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double2 a = *reinterpret_cast<const double2*>(c_slot(s, 2 * r));
                const double2 b = *reinterpret_cast<const double2*>(c_slot(s, 2 * r + 1));
                dP[r] = (T)a.x * d[0] + (T)a.y * d[1] + (T)b.x * d[2] + (T)b.y * d[3];
            }
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const float4 a = *reinterpret_cast<const float4*>(c_slot(s, r));
                dP[r] = (T)a.x * d[0] + (T)a.y * d[1] + (T)a.z * d[2] + (T)a.w * d[3];
            }
        }
        if (DOT) curv += (double)(d[0] * dP[0] + d[1] * dP[1] + d[2] * dP[2] + d[3] * dP[3]);
#pragma unroll
        for (int a = 0; a < NEN; ++a) {
            fx[a] += dP[0] * gx[a] + dP[1] * gy[a];
            fy[a] += dP[2] * gx[a] + dP[3] * gy[a];
        }
        if (q == NQ - 1) scatter(e, node, fix, fx, fy);
    }
    cp_async_wait<0>();
    return true;
}

// Colour form: y[dof] += f_e on the free DOFs of the element (read-modify-write; the elements of one
// colour share no node).
template <int NEN, int NQ, typename SD, typename T, bool DOT>
__global__ void __launch_bounds__(128)
k_apply(Mesh m, int64_t e0, int64_t e1, const SD* __restrict__ C, const SD* __restrict__ G,
        const T* __restrict__ v, T* __restrict__ y, RedSite site, const int* __restrict__ done) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T2* y2 = reinterpret_cast<T2*>(y);
    double curv = 0.0;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    const bool ran = apply_tiles<NEN, NQ, SD, T, DOT>(
        m, e0, e1, C, G, smem, curv,
        [&]() -> bool {
            // from here on v, y and the solver state may come from the predecessor (PDL)
            grid_dependency_wait();
            if (DOT && done != nullptr && *done) return false;  // solve finished: no-op iteration of the graph
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return __ldg(v2 + n); },
        [&](int64_t, const int (&node)[NEN], const int (&fix)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                T2 t = y2[node[a]];
                if (!(fix[a] & 1)) t.x += fx[a];
                if (!(fix[a] & 2)) t.y += fy[a];
                y2[node[a]] = t;
            }
        });
    if (!ran) return;
    if (DOT) {
        constexpr int NT = ApplyCfg<NEN, SD>::NT;
        const double vals[1] = {block_sum<NT>(curv)};
        double tot[1];
        if (last_block_sum<NT, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

// Gather form, element pass: all elements in one launch, each element's f_e stored in its own slots,
// fe[a][e] = (f_x, f_y) (coalesced: e runs fastest).  The node pass (k_node_gather, or the PCG's
// update 1) sums them per node in a fixed order.  With DOT the curvature p.Ap (energy form) reduces
// into site.result[0].
template <int NEN, int NQ, typename SD, typename T, bool DOT>
__global__ void __launch_bounds__(128)
k_apply_elem(Mesh m, const SD* __restrict__ C, const SD* __restrict__ G, const T* __restrict__ v,
             T* __restrict__ fe, RedSite site, const int* __restrict__ done) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T2* fe2 = reinterpret_cast<T2*>(fe);
    const int64_t S = m.stride;
    double curv = 0.0;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    const bool ran = apply_tiles<NEN, NQ, SD, T, DOT>(
        m, 0, m.n_el, C, G, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (DOT && done != nullptr && *done) return false;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return __ldg(v2 + n); },
        [&](int64_t e, const int (&)[NEN], const int (&)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) fe2[(int64_t)a * S + e] = make_v2<T>(fx[a], fy[a]);
        });
    if (!ran) return;
    if (DOT) {
        constexpr int NT = ApplyCfg<NEN, SD>::NT;
        const double vals[1] = {block_sum<NT>(curv)};
        double tot[1];
        if (last_block_sum<NT, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

// Sum of the element results at node n: f = sum over the node's (element, local node) slots, in the
// incidence order (fixed, so the sum is reproducible).
template <typename T>
__device__ __forceinline__ v2_t<T> node_sum(const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                                            const v2_t<T>* __restrict__ fe2, int64_t n) {
    T sx = T(0), sy = T(0);
    const int j1 = inc_ptr[n + 1];
    for (int j = inc_ptr[n]; j < j1; ++j) {
        const v2_t<T> f = fe2[inc[j]];
        sx += f.x;
        sy += f.y;
    }
    return make_v2<T>(sx, sy);
}

// Gather form, node pass of a plain product: y = (1 - m) v + m * sum of the element results.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_node_gather(Mesh m, const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc, const T* __restrict__ fe,
              const T* __restrict__ v, T* __restrict__ y) {
    using T2 = v2_t<T>;
    grid_dependency_wait();
    grid_dependents_launch();
    const T2* fe2 = reinterpret_cast<const T2*>(fe);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < m.n_nodes; n += (int64_t)gridDim.x * blockDim.x) {
        const int fix = m.node_fix[n];
        const T2 f = node_sum<T>(inc_ptr, inc, fe2, n);
        const T2 vn = reinterpret_cast<const T2*>(v)[n];
        reinterpret_cast<T2*>(y)[n] = make_v2<T>((fix & 1) ? vn.x : f.x, (fix & 2) ? vn.y : f.y);
    }
}

// ------------------------------------------------------------------------------------------
// Reference-frame form (DFEA_F32REF moduli, FP64 vectors): per Gauss point only the 10 packed FP32
// moduli stream in (40 B); the gradients are the element type's reference gradients, a kernel
// parameter.  With G = sum_a v_a (x) dN_a/dxi the product at a Gauss point is dPhat = Chat G and
// f_a += dPhat . dN_a/dxi -- the same operator as C applied to the physical gradients.
// ------------------------------------------------------------------------------------------
template <int NEN>
struct RefApplyCfg {
    static constexpr int NT = 128;
    static constexpr int STAGES = 6;
    static constexpr int A_BYTES = 16 * NT;   // entries 00 01 02 03
    static constexpr int B_BYTES = 16 * NT;   // entries 11 12 13 22
    static constexpr int D_BYTES = 8 * NT;    // entries 23 33
    static constexpr int N_BYTES = NEN * 4 * NT;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES + D_BYTES + N_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES;
};

template <int NEN, int NQ, typename T, bool DOT, typename Start, typename Gather, typename Scatter>
__device__ __forceinline__ bool apply_tiles_ref(const Mesh& m, int64_t e0, int64_t e1, const float* __restrict__ C,
                                                const RefGrad<NEN, NQ>& rg, unsigned char* smem, double& curv,
                                                Start&& start, Gather&& gather, Scatter&& scatter,
                                                int64_t blk = -1, int64_t nblk = -1) {
    if (blk < 0) {  // the whole launch walks [e0, e1)
        blk = blockIdx.x;
        nblk = gridDim.x;
    }
    using Cfg = RefApplyCfg<NEN>;
    using T2 = v2_t<T>;
    constexpr int NT = Cfg::NT, ST = Cfg::STAGES;

    const int tid = threadIdx.x;
    const int64_t S = m.stride;
    const int64_t n_tiles = (e1 - e0 + NT - 1) / NT;
    const int64_t my_tiles = (n_tiles > blk) ? (n_tiles - 1 - blk) / nblk + 1 : 0;
    const int64_t n_items = my_tiles * NQ;

    auto element_of = [&](int64_t item) -> int64_t {
        return e0 + (blk + (item / NQ) * nblk) * NT + tid;
    };
    auto stage = [&](int s) -> unsigned char* { return smem + s * Cfg::STAGE_BYTES; };
    auto a_slot = [&](int s) -> float4* { return reinterpret_cast<float4*>(stage(s)) + tid; };
    auto b_slot = [&](int s) -> float4* { return reinterpret_cast<float4*>(stage(s) + Cfg::A_BYTES) + tid; };
    auto d_slot = [&](int s) -> float2* {
        return reinterpret_cast<float2*>(stage(s) + Cfg::A_BYTES + Cfg::B_BYTES) + tid;
    };
    auto n_slot = [&](int s, int a) -> int* {
        return reinterpret_cast<int*>(stage(s) + Cfg::A_BYTES + Cfg::B_BYTES + Cfg::D_BYTES) + a * NT + tid;
    };
    auto issue = [&](int64_t it) {
        if (it < n_items) {
            const int64_t e = element_of(it);
            if (e < e1) {
                const int q = (int)(it % NQ), s = (int)(it % ST);
                const float* base = C + (int64_t)q * 10 * S;
                cp_async16(a_slot(s), reinterpret_cast<const float4*>(base) + e);
                cp_async16(b_slot(s), reinterpret_cast<const float4*>(base + 4 * S) + e);
                cp_async8(d_slot(s), reinterpret_cast<const float2*>(base + 8 * S) + e);
                if (q == 0) {
#pragma unroll
                    for (int a = 0; a < NEN; ++a) cp_async4(n_slot(s, a), m.conn + (int64_t)a * S + e);
                }
            }
        }
        cp_async_commit();
    };

#pragma unroll
    for (int i = 0; i < ST - 1; ++i) issue(i);

    if (!start()) {
        cp_async_wait<0>();
        return false;
    }

    int node[NEN], fix[NEN];
    T vx[NEN], vy[NEN], fx[NEN], fy[NEN];
#pragma unroll
    for (int a = 0; a < NEN; ++a) {
        node[a] = 0;
        fix[a] = 3;
        vx[a] = vy[a] = fx[a] = fy[a] = T(0);
    }

    for (int64_t tile = 0; tile < my_tiles; ++tile) {
        const int64_t e = element_of(tile * NQ);
        const bool live = e < e1;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {  // unrolled: the reference gradients of point q are constants
            const int64_t it = tile * NQ + q;
            issue(it + ST - 1);
            cp_async_wait<ST - 1>();
            const int s = (int)(it % ST);
            if (live) {
                if (q == 0) {
#pragma unroll
                    for (int a = 0; a < NEN; ++a) {
                        const int c = *n_slot(s, a);
                        node[a] = c >> 2;
                        fix[a] = c & 3;
                    }
#pragma unroll
                    for (int a = 0; a < NEN; ++a) {
                        const T2 t = gather(node[a]);
                        vx[a] = (fix[a] & 1) ? T(0) : t.x;
                        vy[a] = (fix[a] & 2) ? T(0) : t.y;
                        fx[a] = T(0);
                        fy[a] = T(0);
                    }
                }
                T G[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
                for (int a = 0; a < NEN; ++a) {
                    const T r0 = (T)rg.g[q][a][0], r1 = (T)rg.g[q][a][1];
                    G[0] += vx[a] * r0;
                    G[1] += vx[a] * r1;
                    G[2] += vy[a] * r0;
                    G[3] += vy[a] * r1;
                }
                const float4 A = *a_slot(s), B = *b_slot(s);
                const float2 D = *d_slot(s);
                const T c00 = A.x, c01 = A.y, c02 = A.z, c03 = A.w, c11 = B.x, c12 = B.y, c13 = B.z, c22 = B.w,
                        c23 = D.x, c33 = D.y;
                const T dP0 = c00 * G[0] + c01 * G[1] + c02 * G[2] + c03 * G[3];
                const T dP1 = c01 * G[0] + c11 * G[1] + c12 * G[2] + c13 * G[3];
                const T dP2 = c02 * G[0] + c12 * G[1] + c22 * G[2] + c23 * G[3];
                const T dP3 = c03 * G[0] + c13 * G[1] + c23 * G[2] + c33 * G[3];
                if (DOT) curv += (double)(G[0] * dP0 + G[1] * dP1 + G[2] * dP2 + G[3] * dP3);
#pragma unroll
                for (int a = 0; a < NEN; ++a) {
                    const T r0 = (T)rg.g[q][a][0], r1 = (T)rg.g[q][a][1];
                    fx[a] += dP0 * r0 + dP1 * r1;
                    fy[a] += dP2 * r0 + dP3 * r1;
                }
                if (q == NQ - 1) scatter(e, node, fix, fx, fy);
            }
        }
    }
    cp_async_wait<0>();
    return true;
}

template <int NEN, int NQ, typename T, bool DOT>
__global__ void __launch_bounds__(128)
k_apply_ref(Mesh m, int64_t e0, int64_t e1, const float* __restrict__ C, const RefGrad<NEN, NQ> rg,
            const T* __restrict__ v, T* __restrict__ y, RedSite site, const int* __restrict__ done) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T2* y2 = reinterpret_cast<T2*>(y);
    double curv = 0.0;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    const bool ran = apply_tiles_ref<NEN, NQ, T, DOT>(
        m, e0, e1, C, rg, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (DOT && done != nullptr && *done) return false;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return __ldg(v2 + n); },
        [&](int64_t, const int (&node)[NEN], const int (&fix)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) {
                T2 t = y2[node[a]];
                if (!(fix[a] & 1)) t.x += fx[a];
                if (!(fix[a] & 2)) t.y += fy[a];
                y2[node[a]] = t;
            }
        });
    if (!ran) return;
    if (DOT) {
        const double vals[1] = {block_sum<128>(curv)};
        double tot[1];
        if (last_block_sum<128, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

template <int NEN, int NQ, typename T, bool DOT>
__global__ void __launch_bounds__(128)
k_apply_ref_elem(Mesh m, const float* __restrict__ C, const RefGrad<NEN, NQ> rg, const T* __restrict__ v,
                 T* __restrict__ fe, RedSite site, const int* __restrict__ done) {
    using T2 = v2_t<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T2* fe2 = reinterpret_cast<T2*>(fe);
    const int64_t S = m.stride;
    double curv = 0.0;
    const T2* v2 = reinterpret_cast<const T2*>(v);
    const bool ran = apply_tiles_ref<NEN, NQ, T, DOT>(
        m, 0, m.n_el, C, rg, smem, curv,
        [&]() -> bool {
            grid_dependency_wait();
            if (DOT && done != nullptr && *done) return false;
            grid_dependents_launch();
            return true;
        },
        [&](int n) { return __ldg(v2 + n); },
        [&](int64_t e, const int (&)[NEN], const int (&)[NEN], const T (&fx)[NEN], const T (&fy)[NEN]) {
#pragma unroll
            for (int a = 0; a < NEN; ++a) fe2[(int64_t)a * S + e] = make_v2<T>(fx[a], fy[a]);
        });
    if (!ran) return;
    if (DOT) {
        const double vals[1] = {block_sum<128>(curv)};
        double tot[1];
        if (last_block_sum<128, 1>(vals, site, tot) && threadIdx.x == 0) site.result[0] = tot[0];
    }
}

// Persistent grid for a walk over n_elements: as many blocks as fit on the GPU at once (occupancy of
// the kernel with its shared memory, configured once per device), never more than there are tiles or
// kMaxBlocks.
template <auto Kernel, int SMEM, int NT>
int resident_grid(int64_t n_elements) {
    // the shared-memory opt-in is a property of the function on each device: set once per device ordinal,
    // race-free when several host threads launch their first product at the same time
    static std::once_flag configured[64];
    static int blocks_per_sm[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    std::call_once(configured[dev], [dev] {
        cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, Kernel, NT, SMEM) != cudaSuccess || b < 1) b = 1;
        blocks_per_sm[dev] = b;
    });
    const int64_t tiles = (n_elements + NT - 1) / NT;
    int64_t grid = (int64_t)device_sm_count() * blocks_per_sm[dev];
    if (grid > kMaxBlocks) grid = kMaxBlocks;
    if (grid > tiles) grid = tiles;
    return (int)(grid < 1 ? 1 : grid);
}

// A grid limited to `cap` blocks (0: no limit).  Solves that share the GPU with other streams run
// with fewer, longer-lived blocks per launch, so that launches of different streams fit side by side.
inline int capped(int grid, int cap) { return (cap > 0 && grid > cap) ? cap : grid; }

template <int NEN, int NQ, typename SD, typename T, bool DOT>
int apply_grid(int64_t n_elements) {
    using Cfg = ApplyCfg<NEN, SD>;
    return resident_grid<k_apply<NEN, NQ, SD, T, DOT>, Cfg::SMEM, Cfg::NT>(n_elements);
}

template <int NEN, int NQ, typename SD, typename T, bool DOT>
int apply_elem_grid(int64_t n_elements) {
    using Cfg = ApplyCfg<NEN, SD>;
    return resident_grid<k_apply_elem<NEN, NQ, SD, T, DOT>, Cfg::SMEM, Cfg::NT>(n_elements);
}

template <int NEN, int NQ, typename T, bool DOT>
int apply_ref_grid(int64_t n_elements) {
    return resident_grid<k_apply_ref<NEN, NQ, T, DOT>, RefApplyCfg<NEN>::SMEM, 128>(n_elements);
}

template <int NEN, int NQ, typename T, bool DOT>
int apply_ref_elem_grid(int64_t n_elements) {
    return resident_grid<k_apply_ref_elem<NEN, NQ, T, DOT>, RefApplyCfg<NEN>::SMEM, 128>(n_elements);
}

// The byte range of the DOF vectors a product gathers (v) and scatters (y): both when they are
// adjacent (one allocation, as in the PCG work buffer), else y alone.
struct L2Window {
    const void* base = nullptr;
    size_t bytes = 0;
};
inline L2Window l2_window(const void* v, const void* y, size_t vec_bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(v), b = reinterpret_cast<uintptr_t>(y);
    const uintptr_t lo = a < b ? a : b, hi = (a < b ? b : a) + vec_bytes;
    if (hi - lo <= 2 * vec_bytes + 4096) return L2Window{reinterpret_cast<const void*>(lo), hi - lo};
    return L2Window{y, vec_bytes};
}

// Launch the colour passes of one product on `stream` (the pivot init is launched by the caller).
// With DOT, colour c reduces into sites[c] (result = curvature of that colour).
template <int NEN, int NQ, typename SD, typename T, bool DOT>
int launch_apply_colours(const dfea_mesh_view& mv, const SD* C, const SD* G, const T* v, T* y,
                         const RedSite* sites, const int* done, cudaStream_t stream, bool count = true,
                         int grid_cap = 0) {
    using Cfg = ApplyCfg<NEN, SD>;
    const Mesh m = kernel_mesh(mv);
    long long max_window = 0;
    const long long setaside = persisting_l2_bytes(&max_window);
    L2Window w = l2_window(v, y, (size_t)(2 * mv.n_nodes) * sizeof(T));
    if ((long long)w.bytes > max_window) w.bytes = (size_t)max_window;
    LaunchOpts opts;
    opts.pdl = true;
    if (setaside > 0 && w.bytes > 0) {
        opts.win_base = w.base;
        opts.win_bytes = w.bytes;
        opts.hit_ratio = setaside >= (long long)w.bytes ? 1.0f : (float)((double)setaside / (double)w.bytes);
    }
    for (int c = 0; c < mv.n_colours; ++c) {
        const int64_t e0 = mv.colour_begin[c], e1 = mv.colour_begin[c + 1];
        if (e1 <= e0) continue;
        const int grid = capped(apply_grid<NEN, NQ, SD, T, DOT>(e1 - e0), grid_cap);
        const RedSite site = DOT ? sites[c] : RedSite{nullptr, nullptr, nullptr};
        const int rc = launch_kernel(k_apply<NEN, NQ, SD, T, DOT>, dim3(grid), dim3(Cfg::NT), Cfg::SMEM, stream, opts, m, e0,
                                     e1, C, G, v, y, site, done);
        if (rc) return rc;
        if (count) note_launches(1);
    }
    return launch_check("k_apply");
}

// Gather form: the element pass over all elements (results into fe), launched with PDL and the L2
// window on v.  The node pass is launched by the caller.
template <int NEN, int NQ, typename SD, typename T, bool DOT>
int launch_apply_elem(const dfea_mesh_view& mv, const SD* C, const SD* G, const T* v, T* fe, RedSite site,
                      const int* done, cudaStream_t stream, int grid_cap = 0) {
    using Cfg = ApplyCfg<NEN, SD>;
    const Mesh m = kernel_mesh(mv);
    long long max_window = 0;
    const long long setaside = persisting_l2_bytes(&max_window);
    size_t wb = (size_t)(2 * mv.n_nodes) * sizeof(T);
    if ((long long)wb > max_window) wb = (size_t)max_window;
    LaunchOpts opts;
    opts.pdl = true;
    if (setaside > 0 && wb > 0) {
        opts.win_base = v;
        opts.win_bytes = wb;
        opts.hit_ratio = setaside >= (long long)wb ? 1.0f : (float)((double)setaside / (double)wb);
    }
    const int grid = capped(apply_elem_grid<NEN, NQ, SD, T, DOT>(mv.n_el), grid_cap);
    const int rc = launch_kernel(k_apply_elem<NEN, NQ, SD, T, DOT>, dim3(grid), dim3(Cfg::NT), Cfg::SMEM, stream, opts, m,
                                 C, G, v, fe, site, done);
    if (rc) return rc;
    return launch_check("k_apply_elem");
}

// Reference-frame launches: colour passes (y read-modify-write) or the element pass (results into fe).
template <int NEN, int NQ, typename T, bool DOT>
int launch_apply_ref_colours(const dfea_mesh_view& mv, const float* C, const T* v, T* y, const RedSite* sites,
                             const int* done, cudaStream_t stream, int grid_cap = 0) {
    const Mesh m = kernel_mesh(mv);
    const RefGrad<NEN, NQ> rg = ref_grad_of<NEN, NQ>(mv);
    long long max_window = 0;
    const long long setaside = persisting_l2_bytes(&max_window);
    L2Window w = l2_window(v, y, (size_t)(2 * mv.n_nodes) * sizeof(T));
    if ((long long)w.bytes > max_window) w.bytes = (size_t)max_window;
    LaunchOpts opts;
    opts.pdl = true;
    if (setaside > 0 && w.bytes > 0) {
        opts.win_base = w.base;
        opts.win_bytes = w.bytes;
        opts.hit_ratio = setaside >= (long long)w.bytes ? 1.0f : (float)((double)setaside / (double)w.bytes);
    }
    for (int c = 0; c < mv.n_colours; ++c) {
        const int64_t e0 = mv.colour_begin[c], e1 = mv.colour_begin[c + 1];
        if (e1 <= e0) continue;
        const int grid = capped(apply_ref_grid<NEN, NQ, T, DOT>(e1 - e0), grid_cap);
        const RedSite site = DOT ? sites[c] : RedSite{nullptr, nullptr, nullptr};
        const int rc = launch_kernel(k_apply_ref<NEN, NQ, T, DOT>, dim3(grid), dim3(128), RefApplyCfg<NEN>::SMEM, stream,
                                     opts, m, e0, e1, C, rg, v, y, site, done);
        if (rc) return rc;
    }
    return launch_check("k_apply_ref");
}

template <int NEN, int NQ, typename T, bool DOT>
int launch_apply_ref_elem(const dfea_mesh_view& mv, const float* C, const T* v, T* fe, RedSite site, const int* done,
                          cudaStream_t stream, int grid_cap = 0) {
    const Mesh m = kernel_mesh(mv);
    const RefGrad<NEN, NQ> rg = ref_grad_of<NEN, NQ>(mv);
    long long max_window = 0;
    const long long setaside = persisting_l2_bytes(&max_window);
    size_t wb = (size_t)(2 * mv.n_nodes) * sizeof(T);
    if ((long long)wb > max_window) wb = (size_t)max_window;
    LaunchOpts opts;
    opts.pdl = true;
    if (setaside > 0 && wb > 0) {
        opts.win_base = v;
        opts.win_bytes = wb;
        opts.hit_ratio = setaside >= (long long)wb ? 1.0f : (float)((double)setaside / (double)wb);
    }
    const int grid = capped(apply_ref_elem_grid<NEN, NQ, T, DOT>(mv.n_el), grid_cap);
    const int rc = launch_kernel(k_apply_ref_elem<NEN, NQ, T, DOT>, dim3(grid), dim3(128), RefApplyCfg<NEN>::SMEM, stream,
                                 opts, m, C, rg, v, fe, site, done);
    if (rc) return rc;
    return launch_check("k_apply_ref_elem");
}

// Configure the instantiations a solver launches (shared-memory size, occupancy) before any stream capture.
template <int NEN, int NQ, typename T>
void prepare_apply_ref() {
    (void)apply_ref_grid<NEN, NQ, T, true>(1);
    (void)apply_ref_elem_grid<NEN, NQ, T, true>(1);
    (void)persisting_l2_bytes(nullptr);
}

// Configure the instantiations a solver launches (shared-memory size, occupancy) before any stream capture.
template <int NEN, int NQ, typename SD, typename T>
void prepare_apply() {
    (void)apply_grid<NEN, NQ, SD, T, true>(1);
    (void)apply_grid<NEN, NQ, SD, T, false>(1);
    (void)apply_elem_grid<NEN, NQ, SD, T, true>(1);
    (void)apply_elem_grid<NEN, NQ, SD, T, false>(1);
    (void)persisting_l2_bytes(nullptr);
}

}  // namespace dfea
