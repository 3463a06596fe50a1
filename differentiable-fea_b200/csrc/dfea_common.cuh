// dfea_common.cuh -- shared device code of the difffea_b200 kernels (sm_100a).
//
// Contents
//   * Mesh: the kernel-side copy of dfea_mesh_view (passed by value)
//   * deterministic reductions: warp/block trees of fixed shape and a "last block finalises"
//     two-level sum (per-block partials + an integer ticket), so that every dot product and norm
//     is bit-reproducible for a given mesh and grid, with no float atomics
//   * neo-Hookean plane-strain point math in closed form: P, d2psi/dF2 and psi of
//         psi = mu/2 (I1 - 3 - 2 ln J) + lambda/2 (ln J)^2,   F3 = [[F, 0], [0, 1]]
//     (the energy of materials.py:209-217; the reference differentiates it with torch.func,
//     here the derivatives are written out:  P = mu F + (lambda lnJ - mu) F^-T,
//     dP_iJ/dF_kL = mu d_ik d_JL + lambda F^-T_iJ F^-T_kL + (mu - lambda lnJ) F^-1_Jk F^-1_Li)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "difffea_b200.h"

namespace dfea {

// ------------------------------------------------------------------------------------------
// host-side error helpers (defined in dfea_host.cpp)
// ------------------------------------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int check_cuda(cudaError_t err, const char* what);
int launch_check(const char* what);
void note_launches(long long n);
long long thread_launch_count();  // launches noted by the calling thread (kernels captured into a graph are
                                  // noted while capturing; the capture subtracts them again)
int device_sm_count();
long long persisting_l2_bytes(long long* max_window);
// copy `bytes` from the device to `host` once stream `s` reaches the copy, through a pooled page-locked block
int read_to_host(void* host, const void* dev, size_t bytes, cudaStream_t s);
// gather-form product on the finite-element level of the multigrid V-cycle with the smoothing update in its
// node pass (dfea_kernels.cu): MG_FE_STEP, one Chebyshev step from direction v = d; MG_FE_RESTART, the
// residual r = b - A v and first direction after the coarse-grid correction (v = x)
enum { MG_FE_STEP = 0, MG_FE_RESTART = 1 };
int mg_fe_gather_cheb(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype, void* fe_work, int mode,
                      const double* v, double* x, double* r, double* d, const double* b, const double* diag,
                      const double* coef, int last, cudaStream_t s);

// Partial sums per reduction site; grids of reducing kernels never exceed this many blocks.
constexpr int kMaxBlocks = 2048;
constexpr int kThreads = 256;

struct Mesh {
    int64_t n_el, stride, n_nodes;
    const int32_t* conn;
    const int32_t* orig;
    const double* grad;
    const double* wdet;
    const float* grad32;
    const uint8_t* node_fix;
    const double* jinv;
};

inline Mesh kernel_mesh(const dfea_mesh_view& v) {
    Mesh m;
    m.n_el = v.n_el;
    m.stride = v.stride;
    m.n_nodes = v.n_nodes;
    m.conn = v.conn;
    m.orig = v.orig;
    m.grad = v.grad;
    m.wdet = v.wdet;
    m.grad32 = v.grad32;
    m.node_fix = v.node_fix;
    m.jinv = v.jinv;
    return m;
}

// The reference shape gradients of one element type at its Gauss points, passed by value (kernel
// parameter space: read through the constant cache, broadcast to a warp since all its threads are at
// the same Gauss point).
template <int NEN, int NQ>
struct RefGrad {
    double g[NQ][NEN][2];
};
template <int NEN, int NQ>
inline RefGrad<NEN, NQ> ref_grad_of(const dfea_mesh_view& v) {
    RefGrad<NEN, NQ> r;
    for (int q = 0; q < NQ; ++q)
        for (int a = 0; a < NEN; ++a)
            for (int k = 0; k < 2; ++k) r.g[q][a][k] = v.ref_grad[(q * NEN + a) * 2 + k];
    return r;
}

// One reduction site in scratch memory: kMaxBlocks partials per value, a ticket, the result(s).
struct RedSite {
    double* partials;   // [K][kMaxBlocks]
    unsigned* ticket;
    double* result;     // [K]
};

// Grid size of a grid-stride launch over n items: enough blocks to fill every SM a few times,
// never more than kMaxBlocks (the partial-sum capacity).
inline int grid_for(int64_t n, int threads, int blocks_per_sm) {
    int64_t want = (n + threads - 1) / threads;
    int64_t cap = (int64_t)device_sm_count() * blocks_per_sm;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

// ------------------------------------------------------------------------------------------
// programmatic dependent launch (PDL) and launches with attributes
// ------------------------------------------------------------------------------------------
// A kernel launched with the PDL attribute may start while its predecessor on the stream still
// runs.  It must not touch anything the predecessor writes before grid_dependency_wait(), which
// returns once the predecessor has completed and its memory is visible; every block of every PDL
// kernel calls it before its first dependent access.  Without the attribute both are no-ops.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

struct LaunchOpts {
    bool pdl = false;               // allow this launch to overlap its predecessor's tail
    const void* win_base = nullptr; // L2 access-policy window marked persisting (0 bytes: none)
    size_t win_bytes = 0;
    float hit_ratio = 0.f;
};

template <typename... KArgs, typename... Args>
int launch_kernel(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                  const LaunchOpts& o, Args... args) {
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (o.pdl) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        ++n;
    }
    if (o.win_bytes > 0 && o.hit_ratio > 0.f) {
        attr[n].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[n].val.accessPolicyWindow.base_ptr = const_cast<void*>(o.win_base);
        attr[n].val.accessPolicyWindow.num_bytes = o.win_bytes;
        attr[n].val.accessPolicyWindow.hitRatio = o.hit_ratio;
        attr[n].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[n].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        ++n;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cfg.attrs = n ? attr : nullptr;
    cfg.numAttrs = n;
    return check_cuda(cudaLaunchKernelEx(&cfg, kernel, args...), "cudaLaunchKernelEx");
}

// ------------------------------------------------------------------------------------------
// deterministic reductions
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block; the result is valid in thread 0.  Every thread must call it.
template <int NT>
__device__ __forceinline__ double block_sum(double v) {
    static_assert(NT % 32 == 0 && NT <= 1024, "block size");
    __shared__ double sh[NT / 32];
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < NT / 32) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Two-level sum of K values: every block stores its block sums (valid in thread 0), the last block
// to arrive adds all partials in block order and returns true (in all its threads) with the totals
// in tot[] (valid in thread 0).  It resets the ticket for the next launch.  Every thread of every
// block must call this with the same K.
// The same over a group of blocks [0, nblk) of which this block is number blk (several groups, each
// with its own site, can share one launch).
template <int NT, int K>
__device__ bool last_block_sum_in(const double (&vals)[K], const RedSite& site, double (&tot)[K], int blk, int nblk) {
    __shared__ int am_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) site.partials[k * kMaxBlocks + blk] = vals[k];
        __threadfence();
        const unsigned t = atomicAdd(site.ticket, 1u);
        am_last = (t == (unsigned)nblk - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int i = threadIdx.x; i < nblk; i += NT) s += __ldcg(site.partials + k * kMaxBlocks + i);
        tot[k] = block_sum<NT>(s);
    }
    if (threadIdx.x == 0) *site.ticket = 0u;
    return true;
}

template <int NT, int K>
__device__ bool last_block_sum(const double (&vals)[K], const RedSite& site, double (&tot)[K]) {
    return last_block_sum_in<NT, K>(vals, site, tot, (int)blockIdx.x, (int)gridDim.x);
}

// ------------------------------------------------------------------------------------------
// vector element types
// ------------------------------------------------------------------------------------------
template <typename T> struct V2;
template <> struct V2<double> { using type = double2; };
template <> struct V2<float> { using type = float2; };
template <typename T> using v2_t = typename V2<T>::type;

template <typename T> __device__ __forceinline__ v2_t<T> make_v2(T a, T b);
template <> __device__ __forceinline__ double2 make_v2<double>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 make_v2<float>(float a, float b) { return make_float2(a, b); }

// Streaming (evict-first) load of one (dN/dX, dN/dY) pair of the packed gradients.
__device__ __forceinline__ double2 load_grad(const double* g, int64_t idx) {
    return __ldcs(reinterpret_cast<const double2*>(g) + idx);
}
__device__ __forceinline__ float2 load_grad(const float* g, int64_t idx) {
    return __ldcs(reinterpret_cast<const float2*>(g) + idx);
}

// Row r of the 4x4 moduli of Gauss point q of element e (streaming loads).
//   f64 layout [n_q][8][stride] double2: row r = pairs 2r, 2r+1
//   f32 layout [n_q][4][stride] float4:  row r = one float4
__device__ __forceinline__ void load_moduli_row(const double* C, int64_t S, int q, int r, int64_t e,
                                                double (&row)[4]) {
    const double2* p = reinterpret_cast<const double2*>(C);
    const double2 a = __ldcs(p + (int64_t)(q * 8 + 2 * r) * S + e);
    const double2 b = __ldcs(p + (int64_t)(q * 8 + 2 * r + 1) * S + e);
    row[0] = a.x; row[1] = a.y; row[2] = b.x; row[3] = b.y;
}
__device__ __forceinline__ void load_moduli_row(const float* C, int64_t S, int q, int r, int64_t e,
                                                float (&row)[4]) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(C) + (int64_t)(q * 4 + r) * S + e);
    row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = a.w;
}

__device__ __forceinline__ void store_moduli(double* C, int64_t S, int q, int64_t e, const double (&c)[16]) {
    double2* p = reinterpret_cast<double2*>(C);
#pragma unroll
    for (int k = 0; k < 8; ++k) p[(int64_t)(q * 8 + k) * S + e] = make_double2(c[2 * k], c[2 * k + 1]);
}
// Moduli pulled back to the reference frame, packed symmetric (DFEA_F32REF layout):
//   h_(ia),(kb) = sum_{J,L} Jinv_aJ C_(iJ),(kL) Jinv_bL,  ji[2a+J] = Jinv_aJ.
__device__ __forceinline__ void store_moduli_ref(float* C, int64_t S, int q, int64_t e, const double (&c)[16],
                                                 const double (&ji)[4]) {
    double h[16];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            // t = B Jinv^T with B the (i, k) block of C, then h = Jinv t
            double t[2][2];
#pragma unroll
            for (int J = 0; J < 2; ++J)
#pragma unroll
                for (int b = 0; b < 2; ++b)
                    t[J][b] = c[(2 * i + J) * 4 + 2 * k] * ji[2 * b] + c[(2 * i + J) * 4 + 2 * k + 1] * ji[2 * b + 1];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) h[(2 * i + a) * 4 + 2 * k + b] = ji[2 * a] * t[0][b] + ji[2 * a + 1] * t[1][b];
        }
    const int64_t base = (int64_t)q * 10 * S;
    float4* A = reinterpret_cast<float4*>(C + base);
    float4* B = reinterpret_cast<float4*>(C + base + 4 * S);
    float2* D = reinterpret_cast<float2*>(C + base + 8 * S);
    A[e] = make_float4((float)h[0], (float)h[1], (float)h[2], (float)h[3]);
    B[e] = make_float4((float)h[5], (float)h[6], (float)h[7], (float)h[10]);
    D[e] = make_float2((float)h[11], (float)h[15]);
}

__device__ __forceinline__ void store_moduli(float* C, int64_t S, int q, int64_t e, const double (&c)[16]) {
    float4* p = reinterpret_cast<float4*>(C);
#pragma unroll
    for (int r = 0; r < 4; ++r)
        p[(int64_t)(q * 4 + r) * S + e] =
            make_float4((float)c[4 * r], (float)c[4 * r + 1], (float)c[4 * r + 2], (float)c[4 * r + 3]);
}

// ------------------------------------------------------------------------------------------
// neo-Hookean plane strain, F[2i+J] = F_iJ
// ------------------------------------------------------------------------------------------
struct NHPoint {
    double J, lnJ;
    double FiT[4];  // F^-T, FiT[2i+J] = (F^-1)_Ji
};

__device__ __forceinline__ NHPoint nh_point(const double (&F)[4]) {
    NHPoint p;
    p.J = F[0] * F[3] - F[1] * F[2];
    const double iJ = 1.0 / p.J;
    p.FiT[0] = F[3] * iJ;
    p.FiT[1] = -F[2] * iJ;
    p.FiT[2] = -F[1] * iJ;
    p.FiT[3] = F[0] * iJ;
    p.lnJ = log(p.J);  // NaN for J < 0 (inverted element), as torch.log in the reference
    return p;
}

// First Piola stress P_iJ = mu F_iJ + (lambda lnJ - mu) F^-T_iJ.
__device__ __forceinline__ void nh_stress(const double (&F)[4], const NHPoint& p, double mu, double lam,
                                          double (&P)[4]) {
    const double b = lam * p.lnJ - mu;
#pragma unroll
    for (int r = 0; r < 4; ++r) P[r] = mu * F[r] + b * p.FiT[r];
}

// Energy density psi = mu/2 (|F|^2 + 1 - 3 - 2 lnJ) + lambda/2 lnJ^2.
__device__ __forceinline__ double nh_energy(const double (&F)[4], const NHPoint& p, double mu, double lam) {
    const double I1 = F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3] + 1.0;
    return 0.5 * mu * (I1 - 3.0 - 2.0 * p.lnJ) + 0.5 * lam * p.lnJ * p.lnJ;
}

// w * d2psi/dF_r dF_c, r = 2i+J, c = 2k+L (row-major 4x4, the flattening of operators.py:341).
__device__ __forceinline__ void nh_moduli(const NHPoint& p, double mu, double lam, double w, double (&C)[16]) {
    const double a = mu - lam * p.lnJ;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = r >> 1, J = r & 1, k = c >> 1, L = c & 1;
            double v = lam * p.FiT[r] * p.FiT[c] + a * p.FiT[2 * k + J] * p.FiT[2 * i + L];
            if (r == c) v += mu;
            C[4 * r + c] = w * v;
        }
    }
}

// ------------------------------------------------------------------------------------------
// element-type dispatch: (nen, n_q) -> template instantiation
// ------------------------------------------------------------------------------------------
template <int V> struct IntC { static constexpr int value = V; };

// fn(IntC<NEN>{}, IntC<NQ>{}) for the five element types of the reference's library
// (elements.py:38-58 with the default rules of gauss_quadratures.py); other pairs are rejected.
template <typename Fn>
int dispatch_element(int nen, int nq, Fn&& fn) {
    if (nen == 4 && nq == 4) return fn(IntC<4>{}, IntC<4>{});   // quad4, 2x2 Gauss
    if (nen == 9 && nq == 9) return fn(IntC<9>{}, IntC<9>{});   // quad9, 3x3 Gauss
    if (nen == 3 && nq == 1) return fn(IntC<3>{}, IntC<1>{});   // tri3, centroid rule
    if (nen == 6 && nq == 6) return fn(IntC<6>{}, IntC<6>{});   // tri6, 6-point rule
    if (nen == 8 && nq == 9) return fn(IntC<8>{}, IntC<9>{});   // quad8, 3x3 Gauss
    return set_error(DFEA_ERR_UNSUPPORTED, "element with nen=%d n_q=%d is not built", nen, nq);
}

}  // namespace dfea
