// Hyperelastic material library of the device kernels (the reference's materials.py:60-186).
//
// Every model is one energy psi3(F3, p) of the plane-strain embedding F3 = [[F, 0], [0, F33]] with F33 = 1.
// The neo-Hookean model keeps its closed-form stress and moduli (dfea_common.cuh).  The others are
// written once, as templates over a number type, and differentiated in forward mode: a Jet carries a value,
// its gradient with respect to NV variables and (optionally) the packed upper triangle of its Hessian, so
// one evaluation of psi over Jet<4, true> gives P = dpsi/dF and C = d2psi/dF2 exactly (to rounding), as the
// reference gets them from torch.func.grad / hessian.  Jet<5, false> adds F33 as a variable for the
// out-of-plane stress of the post-processing.
#pragma once

#include "dfea_common.cuh"

namespace dfea {

// ------------------------------------------------------------------------------------------
// forward-mode numbers
// ------------------------------------------------------------------------------------------
template <int NV, bool H>
struct Jet {
    static constexpr int NH = H ? NV * (NV + 1) / 2 : 1;
    double v;
    double g[NV];
    double h[NH];  // h[hidx(i, j)], i <= j (unused when !H)
};

template <int NV>
__host__ __device__ constexpr int hidx(int i, int j) {
    return i * NV - (i * (i - 1)) / 2 + (j - i);
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> jconst(double c) {
    Jet<NV, H> r;
    r.v = c;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = 0.0;
    if constexpr (H) {
#pragma unroll
        for (int k = 0; k < Jet<NV, H>::NH; ++k) r.h[k] = 0.0;
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> jvar(double x, int k) {
    Jet<NV, H> r = jconst<NV, H>(x);
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = (i == k) ? 1.0 : 0.0;
    return r;
}

// f(a) for a scalar function with f(a.v) = f0, f' = f1, f'' = f2
template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> chain(const Jet<NV, H>& a, double f0, double f1, double f2) {
    Jet<NV, H> r;
    r.v = f0;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = f1 * a.g[i];
    if constexpr (H) {
#pragma unroll
        for (int i = 0; i < NV; ++i)
#pragma unroll
            for (int j = i; j < NV; ++j) r.h[hidx<NV>(i, j)] = f1 * a.h[hidx<NV>(i, j)] + f2 * a.g[i] * a.g[j];
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator+(const Jet<NV, H>& a, const Jet<NV, H>& b) {
    Jet<NV, H> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = a.g[i] + b.g[i];
    if constexpr (H) {
#pragma unroll
        for (int k = 0; k < Jet<NV, H>::NH; ++k) r.h[k] = a.h[k] + b.h[k];
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator-(const Jet<NV, H>& a, const Jet<NV, H>& b) {
    Jet<NV, H> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = a.g[i] - b.g[i];
    if constexpr (H) {
#pragma unroll
        for (int k = 0; k < Jet<NV, H>::NH; ++k) r.h[k] = a.h[k] - b.h[k];
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator*(const Jet<NV, H>& a, const Jet<NV, H>& b) {
    Jet<NV, H> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = a.v * b.g[i] + b.v * a.g[i];
    if constexpr (H) {
#pragma unroll
        for (int i = 0; i < NV; ++i)
#pragma unroll
            for (int j = i; j < NV; ++j) {
                const int k = hidx<NV>(i, j);
                r.h[k] = a.v * b.h[k] + b.v * a.h[k] + a.g[i] * b.g[j] + a.g[j] * b.g[i];
            }
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator*(const Jet<NV, H>& a, double c) {
    Jet<NV, H> r;
    r.v = a.v * c;
#pragma unroll
    for (int i = 0; i < NV; ++i) r.g[i] = a.g[i] * c;
    if constexpr (H) {
#pragma unroll
        for (int k = 0; k < Jet<NV, H>::NH; ++k) r.h[k] = a.h[k] * c;
    }
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator*(double c, const Jet<NV, H>& a) { return a * c; }

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator+(const Jet<NV, H>& a, double c) {
    Jet<NV, H> r = a;
    r.v += c;
    return r;
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> operator-(const Jet<NV, H>& a, double c) { return a + (-c); }

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> jlog(const Jet<NV, H>& a) {
    const double iv = 1.0 / a.v;
    return chain(a, log(a.v), iv, -iv * iv);  // NaN for a.v < 0, as torch.log
}

template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> jexp(const Jet<NV, H>& a) {
    const double e = exp(a.v);
    return chain(a, e, e, e);
}

// max(a, 0) with derivative 0 at a = 0 (torch.relu's convention)
template <int NV, bool H>
__device__ __forceinline__ Jet<NV, H> jrelu(const Jet<NV, H>& a) {
    return (a.v > 0.0) ? a : jconst<NV, H>(0.0);
}

__device__ __forceinline__ double jlog(double a) { return log(a); }
__device__ __forceinline__ double jexp(double a) { return exp(a); }
__device__ __forceinline__ double jrelu(double a) { return a > 0.0 ? a : 0.0; }

// ------------------------------------------------------------------------------------------
// parameters
// ------------------------------------------------------------------------------------------
// Number of parameters of each model and the bit mask of those that enter its energy linearly, as a
// prefactor of a term (materials.py:224-236): only those may be scaled by theta for the sensitivity.
__host__ __device__ constexpr int material_n_params(int model) {
    return model == DFEA_MAT_NEO_HOOKEAN ? 2
         : model == DFEA_MAT_MOONEY_RIVLIN ? 3
         : model == DFEA_MAT_SAINT_VENANT ? 2
         : model == DFEA_MAT_DEMIRAY ? 3
         : model == DFEA_MAT_FIBER_REINFORCED ? 7
         : 0;
}

__host__ __device__ constexpr unsigned material_linear_mask(int model) {
    return model == DFEA_MAT_NEO_HOOKEAN ? 0x3u           // mu, lambda
         : model == DFEA_MAT_MOONEY_RIVLIN ? 0x7u         // c10, c01, kappa
         : model == DFEA_MAT_SAINT_VENANT ? 0x3u          // mu, lambda
         : model == DFEA_MAT_DEMIRAY ? 0x5u               // mu, lambda (gamma is inside the exponential)
         : model == DFEA_MAT_FIBER_REINFORCED ? 0x7u      // mu, lambda, k1
         : 0u;
}

// p_e = p0 with the scalable entries multiplied by theta_e (materials.py:239-246)
__device__ __forceinline__ void element_params(const dfea_material& mat, double th, double (&pe)[DFEA_MAX_MAT_PARAMS]) {
#pragma unroll
    for (int k = 0; k < DFEA_MAX_MAT_PARAMS; ++k) pe[k] = ((mat.scalable >> k) & 1u) ? mat.p[k] * th : mat.p[k];
}

// ------------------------------------------------------------------------------------------
// the energies (T = double or a Jet); F = (F00, F01, F10, F11), F22 the out-of-plane stretch
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T psi_neo_hookean3(const T& I1, const T& lnJ, double mu, double lam) {
    return (I1 - 3.0 - 2.0 * lnJ) * (0.5 * mu) + lnJ * lnJ * (0.5 * lam);
}

// materials.py:60-186.  model is warp-uniform (one material per mesh).
template <typename T>
__device__ __forceinline__ T psi_model(int model, const T& f00, const T& f01, const T& f10, const T& f11, const T& f22,
                                       const double (&p)[DFEA_MAX_MAT_PARAMS]) {
    // right Cauchy-Green C = F3^T F3 (C02 = C12 = 0)
    const T C00 = f00 * f00 + f10 * f10, C11 = f01 * f01 + f11 * f11, C01 = f00 * f01 + f10 * f11, C22 = f22 * f22;
    const T I1 = C00 + C11 + C22;
    const T J = (f00 * f11 - f01 * f10) * f22;  // det F3 of the block-diagonal embedding (materials.py:49-52)
    switch (model) {
        case DFEA_MAT_MOONEY_RIVLIN: {
            // c10 (J^-2/3 I1 - 3) + c01 (J^-4/3 I2 - 3) + kappa/2 lnJ^2, I2 = (I1^2 - tr C^2) / 2
            const T lnJ = jlog(J);
            const T trC2 = C00 * C00 + C11 * C11 + C22 * C22 + 2.0 * (C01 * C01);
            const T I2 = (I1 * I1 - trC2) * 0.5;
            const T J23 = jexp(lnJ * (-2.0 / 3.0));
            return (J23 * I1 - 3.0) * p[0] + (J23 * J23 * I2 - 3.0) * p[1] + lnJ * lnJ * (0.5 * p[2]);
        }
        case DFEA_MAT_SAINT_VENANT: {
            // lambda/2 (tr E)^2 + mu tr(E^2), E = (C - I) / 2
            const T E00 = (C00 - 1.0) * 0.5, E11 = (C11 - 1.0) * 0.5, E22 = (C22 - 1.0) * 0.5, E01 = C01 * 0.5;
            const T trE = E00 + E11 + E22;
            const T trE2 = E00 * E00 + E11 * E11 + E22 * E22 + 2.0 * (E01 * E01);
            return trE * trE * (0.5 * p[1]) + trE2 * p[0];
        }
        case DFEA_MAT_DEMIRAY: {
            // mu / (2 gamma) (exp(gamma (I1 - 3)) - 1) - mu lnJ + lambda/2 lnJ^2, p = (mu, gamma, lambda)
            const T lnJ = jlog(J);
            return (jexp((I1 - 3.0) * p[1]) - 1.0) * (p[0] / (2.0 * p[1])) - lnJ * p[0] + lnJ * lnJ * (0.5 * p[2]);
        }
        case DFEA_MAT_FIBER_REINFORCED: {
            // neo-Hookean matrix + k1 / (2 k2) (exp(k2 <E_i>^2) - 1) per fibre family, E_i = d I1 + (1 - 3d) I4_i - 1,
            // I4 = a . C a, a = (cos beta, +-sin beta, 0); p = (mu, lambda, k1, k2, beta_deg, d, second_family)
            const T lnJ = jlog(J);
            T psi = psi_neo_hookean3(I1, lnJ, p[0], p[1]);
            const double beta = p[4] * (3.141592653589793 / 180.0);
            const double cb = cos(beta), sb = sin(beta), d = p[5];
            const double pref = p[2] / (2.0 * p[3]);
#pragma unroll
            for (int fam = 0; fam < 2; ++fam) {
                const double s = fam == 0 ? sb : -sb;
                // (a^T C) a, in the order of the reference's a @ C @ a
                const T I4 = (C00 * cb + C01 * s) * cb + (C01 * cb + C11 * s) * s;
                const T E = I1 * d + I4 * (1.0 - 3.0 * d) - 1.0;
                const T Et = jrelu(E);
                const T fib = (jexp(Et * Et * p[3]) - 1.0) * pref;
                psi = fam == 0 ? psi + fib : psi + fib * p[6];
            }
            return psi;
        }
        default: {  // DFEA_MAT_NEO_HOOKEAN (materials.py:60-73)
            return psi_neo_hookean3(I1, jlog(J), p[0], p[1]);
        }
    }
}

// psi with its gradient and Hessian over (F00, F01, F10, F11) at F33 = 1
template <int NV>
__device__ __forceinline__ Jet<NV, true> psi_hessian(int model, const double (&F)[4], const double (&p)[DFEA_MAX_MAT_PARAMS]) {
    using Jt = Jet<NV, true>;
    return psi_model<Jt>(model, jvar<NV, true>(F[0], 0), jvar<NV, true>(F[1], 1), jvar<NV, true>(F[2], 2),
                         jvar<NV, true>(F[3], 3), jconst<NV, true>(1.0), p);
}

// w * d2psi/dF2, row-major 4x4 over (F00, F01, F10, F11): the flattening of operators.py:341
__device__ __forceinline__ void gen_moduli(int model, const double (&F)[4], const double (&p)[DFEA_MAX_MAT_PARAMS],
                                           double w, double (&C)[16]) {
    const Jet<4, true> t = psi_hessian<4>(model, F, p);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) C[4 * r + c] = w * t.h[r <= c ? hidx<4>(r, c) : hidx<4>(c, r)];
}

// P = dpsi/dF (F00, F01, F10, F11); returns psi
__device__ __forceinline__ double gen_stress(int model, const double (&F)[4], const double (&p)[DFEA_MAX_MAT_PARAMS],
                                             double (&P)[4]) {
    using Jt = Jet<4, false>;
    const Jt t = psi_model<Jt>(model, jvar<4, false>(F[0], 0), jvar<4, false>(F[1], 1), jvar<4, false>(F[2], 2),
                               jvar<4, false>(F[3], 3), jconst<4, false>(1.0), p);
#pragma unroll
    for (int r = 0; r < 4; ++r) P[r] = t.g[r];
    return t.v;
}

// P3 = dpsi3/dF3 with F33 as a fifth variable: P[0..3] in-plane, P[4] = P3_33; returns psi
__device__ __forceinline__ double gen_stress3(int model, const double (&F)[4], const double (&p)[DFEA_MAX_MAT_PARAMS],
                                              double (&P)[5]) {
    using Jt = Jet<5, false>;
    const Jt t = psi_model<Jt>(model, jvar<5, false>(F[0], 0), jvar<5, false>(F[1], 1), jvar<5, false>(F[2], 2),
                               jvar<5, false>(F[3], 3), jvar<5, false>(1.0, 4), p);
#pragma unroll
    for (int r = 0; r < 5; ++r) P[r] = t.g[r];
    return t.v;
}

}  // namespace dfea
