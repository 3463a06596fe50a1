// dfea_mg.cu -- geometric multigrid on structured quadrilateral grids: the kernels of a V-cycle
// preconditioner for the PCG of the Newton-Krylov solve.
//
// Levels.  Level 0 is the finite-element mesh (Q4, or Q9 whose nodes form a grid refined twice); every
// coarser level l >= 1 is a Q4 grid of gx x gy cells with bilinear interpolation between levels, each
// level halving the cell count of the one above it in both directions (a last cell one line wide when
// the count is odd).  Coarse operators are Galerkin products built element by element: level 1 from
// the stored Gauss-point moduli of the fine mesh, K_C = sum_{e in C} sum_q (B_q P~)^T C_q (B_q P~), and
// level l + 1 from level l's 8 x 8 element matrices, K_C = sum P^T K_c P.  P~ zeroes fixed fine DOFs, so
// a coarse DOF whose whole support is fixed has a zero row and becomes an identity row; the coarse
// operator equals P~^T A P~ of A = M K M + (I - M) on the free DOFs.
//
// Everything here is deterministic: node-centric gathers in a fixed order, single-block reductions.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <new>
#include <utility>

#include "dfea_common.cuh"

namespace dfea {

int validate_mesh(const dfea_mesh_view* mv, bool need_grad32);

struct MgGrid {
    int gx, gy;
    const int32_t* line_x;
    const int32_t* line_y;
    const int32_t* cell_x;
    const int32_t* cell_y;
    double* K;
    uint8_t* fix;
};

static MgGrid mg_grid(const dfea_mg_grid& g) {
    return MgGrid{g.gx, g.gy, g.line_x, g.line_y, g.cell_x, g.cell_y, g.K, g.fix};
}

static int validate_grid(const dfea_mg_grid* g, bool coarse, const char* what) {
    if (!g || g->gx < 1 || g->gy < 1) return set_error(DFEA_ERR_INVALID, "%s: bad grid", what);
    if ((int64_t)(g->gx + 1) * (g->gy + 1) >= (int64_t(1) << 30)) return set_error(DFEA_ERR_INVALID, "%s: grid too large", what);
    if (coarse && (!g->line_x || !g->line_y || !g->cell_x || !g->cell_y))
        return set_error(DFEA_ERR_INVALID, "%s: a coarse grid needs its line and cell maps", what);
    return DFEA_OK;
}

// weight of coarse line c (lines X) at finer line i, for i in [X[c-1], X[c+1]]
__device__ __forceinline__ double hat(const int32_t* X, int n_lines, int c, int i) {
    const int xc = X[c];
    if (i == xc) return 1.0;
    if (i < xc) {
        if (c == 0) return 0.0;
        const int xl = X[c - 1];
        return i <= xl ? 0.0 : (double)(i - xl) / (double)(xc - xl);
    }
    if (c == n_lines - 1) return 0.0;
    const int xr = X[c + 1];
    return i >= xr ? 0.0 : (double)(xr - i) / (double)(xr - xc);
}

// ------------------------------------------------------------------------------------------
// level 1 from the finite-element mesh: K_C = sum_e sum_q (B_q P~)^T C_q (B_q P~)
// ------------------------------------------------------------------------------------------
// MOD 0: FP64 physical moduli (16 per Gauss point) with the mesh gradients; 1: FP32 physical moduli; 2: FP32
// reference-frame moduli (10 per Gauss point, DFEA_F32REF) with the reference gradients.
template <int NEN, int NQ, int MOD>
__global__ void __launch_bounds__(128)
k_mg_galerkin_fe(Mesh m, const void* __restrict__ moduli, RefGrad<NEN, NQ> rg, const int32_t* __restrict__ node_ij,
                 const int32_t* __restrict__ cell_slot, int span, int epc, int ncy, MgGrid cg) {
    const int n_cells = cg.gx * cg.gy;
    const int64_t S = m.stride;
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < n_cells; C += gridDim.x * blockDim.x) {
        const int CX = C / cg.gy, CY = C % cg.gy;
        const int x0 = cg.line_x[CX], x1 = cg.line_x[CX + 1], y0 = cg.line_y[CY], y1 = cg.line_y[CY + 1];
        double K[64];
#pragma unroll
        for (int k = 0; k < 64; ++k) K[k] = 0.0;
#pragma unroll 1
        for (int fcx = x0 / span; fcx < x1 / span; ++fcx) {
#pragma unroll 1
            for (int fce = (y0 / span) * epc; fce < (y1 / span) * epc; ++fce) {
                // element fce % epc of the cell (fcx, fce / epc)
                const int64_t s = cell_slot[((int64_t)fcx * ncy + fce / epc) * epc + fce % epc];
                double P[NEN][4];
                int fix[NEN];
#pragma unroll
                for (int a = 0; a < NEN; ++a) {
                    const int c = m.conn[a * S + s];
                    const int n = c >> 2;
                    fix[a] = c & 3;
                    const double wx1 = (double)(node_ij[2 * n] - x0) / (double)(x1 - x0);
                    const double wy1 = (double)(node_ij[2 * n + 1] - y0) / (double)(y1 - y0);
                    const double wx0 = 1.0 - wx1, wy0 = 1.0 - wy1;
                    P[a][0] = wx0 * wy0;
                    P[a][1] = wx1 * wy0;
                    P[a][2] = wx1 * wy1;
                    P[a][3] = wx0 * wy1;
                }
#pragma unroll 1
                for (int q = 0; q < NQ; ++q) {
                    double g[NEN][2], M[16];
                    if constexpr (MOD == 2) {
                        const float* Cf = static_cast<const float*>(moduli);
                        const int64_t base = (int64_t)q * 10 * S;
                        const float4 A = reinterpret_cast<const float4*>(Cf + base)[s];
                        const float4 B = reinterpret_cast<const float4*>(Cf + base + 4 * S)[s];
                        const float2 D = reinterpret_cast<const float2*>(Cf + base + 8 * S)[s];
                        const double h[10] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w, D.x, D.y};
                        // packed upper triangle: (0,0..3) (1,1..3) (2,2..3) (3,3)
                        M[0] = h[0]; M[1] = h[1]; M[2] = h[2]; M[3] = h[3];
                        M[5] = h[4]; M[6] = h[5]; M[7] = h[6];
                        M[10] = h[7]; M[11] = h[8];
                        M[15] = h[9];
                        M[4] = M[1]; M[8] = M[2]; M[12] = M[3]; M[9] = M[6]; M[13] = M[7]; M[14] = M[11];
#pragma unroll
                        for (int a = 0; a < NEN; ++a) {
                            g[a][0] = rg.g[q][a][0];
                            g[a][1] = rg.g[q][a][1];
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            if constexpr (MOD == 0) {
                                double row[4];
                                load_moduli_row(static_cast<const double*>(moduli), S, q, r, s, row);
#pragma unroll
                                for (int c = 0; c < 4; ++c) M[4 * r + c] = row[c];
                            } else {
                                float row[4];
                                load_moduli_row(static_cast<const float*>(moduli), S, q, r, s, row);
#pragma unroll
                                for (int c = 0; c < 4; ++c) M[4 * r + c] = row[c];
                            }
                        }
#pragma unroll
                        for (int a = 0; a < NEN; ++a) {
                            const double2 t = load_grad(m.grad, (int64_t)(q * NEN + a) * S + s);
                            g[a][0] = t.x;
                            g[a][1] = t.y;
                        }
                    }
                    // coarse gradients per component: G[i][b][J] = sum_a P~_(a,i),b dN_a,J
                    double G[2][4][2];
#pragma unroll
                    for (int i = 0; i < 2; ++i)
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            double s0 = 0.0, s1 = 0.0;
#pragma unroll
                            for (int a = 0; a < NEN; ++a) {
                                const double w = (fix[a] >> i) & 1 ? 0.0 : P[a][b];
                                s0 += w * g[a][0];
                                s1 += w * g[a][1];
                            }
                            G[i][b][0] = s0;
                            G[i][b][1] = s1;
                        }
#pragma unroll
                    for (int c = 0; c < 4; ++c)
#pragma unroll
                        for (int k = 0; k < 2; ++k) {
                            double t[4];
#pragma unroll
                            for (int r = 0; r < 4; ++r) t[r] = M[4 * r + 2 * k] * G[k][c][0] + M[4 * r + 2 * k + 1] * G[k][c][1];
#pragma unroll
                            for (int b = 0; b < 4; ++b)
#pragma unroll
                                for (int i = 0; i < 2; ++i)
                                    K[(2 * b + i) * 8 + 2 * c + k] += G[i][b][0] * t[2 * i] + G[i][b][1] * t[2 * i + 1];
                        }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 64; ++k) cg.K[(int64_t)k * n_cells + C] = K[k];
    }
}

// ------------------------------------------------------------------------------------------
// level l + 1 from level l: K_C = sum_{fine cells c in C} P_c^T K_c P_c
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mg_galerkin(MgGrid fg, MgGrid cg) {
    const int n_cells = cg.gx * cg.gy, nf_cells = fg.gx * fg.gy;
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < n_cells; C += gridDim.x * blockDim.x) {
        const int CX = C / cg.gy, CY = C % cg.gy;
        const int x0 = cg.line_x[CX], x1 = cg.line_x[CX + 1], y0 = cg.line_y[CY], y1 = cg.line_y[CY + 1];
        double K[64];
#pragma unroll
        for (int k = 0; k < 64; ++k) K[k] = 0.0;
#pragma unroll 1
        for (int fx = x0; fx < x1; ++fx) {
#pragma unroll 1
            for (int fy = y0; fy < y1; ++fy) {
                const int fc = fx * fg.gy + fy;
                // P[a][b]: weight of coarse corner b at fine corner a (corners (0,0) (1,0) (1,1) (0,1))
                double P[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int i = fx + ((a == 1 || a == 2) ? 1 : 0), j = fy + ((a >= 2) ? 1 : 0);
                    const double wx1 = (double)(i - x0) / (double)(x1 - x0), wy1 = (double)(j - y0) / (double)(y1 - y0);
                    const double wx0 = 1.0 - wx1, wy0 = 1.0 - wy1;
                    P[a][0] = wx0 * wy0;
                    P[a][1] = wx1 * wy0;
                    P[a][2] = wx1 * wy1;
                    P[a][3] = wx0 * wy1;
                }
                // T = K_c P (8 x 8), then K += P^T T; P acts on both components alike
#pragma unroll 1
                for (int col = 0; col < 8; ++col) {
                    const int b = col >> 1, k = col & 1;
                    double t[8];
#pragma unroll
                    for (int row = 0; row < 8; ++row) {
                        double acc = 0.0;
#pragma unroll
                        for (int a = 0; a < 4; ++a) acc += fg.K[(int64_t)(row * 8 + 2 * a + k) * nf_cells + fc] * P[a][b];
                        t[row] = acc;
                    }
#pragma unroll
                    for (int bb = 0; bb < 4; ++bb)
#pragma unroll
                        for (int i = 0; i < 2; ++i) {
                            double acc = 0.0;
#pragma unroll
                            for (int a = 0; a < 4; ++a) acc += P[a][bb] * t[2 * a + i];
                            K[(2 * bb + i) * 8 + col] += acc;
                        }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 64; ++k) cg.K[(int64_t)k * n_cells + C] = K[k];
    }
}

// ------------------------------------------------------------------------------------------
// transfers; gnode maps a grid node of the finer level to its DOF node (level 0: the FE node id, -1 where
// the grid has no node), NULL for the lexicographic numbering of the coarse levels
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int fine_node(const int32_t* gnode, int fgy, int i, int j) {
    const int id = i * (fgy + 1) + j;
    return gnode ? gnode[id] : id;
}

// rc = P~^T r (masked at fixed fine DOFs); with fix_out, also the coarse fix bits (a coarse DOF is fixed
// when every fine DOF it interpolates to is fixed)
// coarse node n of the restriction r_c = P~^T r (and the coarse fixed-DOF bits); the kernels below and the
// one-block tail of the V-cycle share these per-node functions, whose pointers carry no __restrict__ because
// the tail reads in one phase what it wrote in the previous one
__device__ __forceinline__ void mg_restrict_node(const MgGrid& fg, const MgGrid& cg, const int32_t* gnode,
                                                 const uint8_t* ffix, const double* r, double* rc, uint8_t* fix_out,
                                                 int n) {
    const int nx = cg.gx + 1, ny = cg.gy + 1;
    const double2* r2 = reinterpret_cast<const double2*>(r);
    const int I = n / ny, J = n % ny;
    const int ilo = I > 0 ? cg.line_x[I - 1] + 1 : cg.line_x[I], ihi = I < cg.gx ? cg.line_x[I + 1] - 1 : cg.line_x[I];
    const int jlo = J > 0 ? cg.line_y[J - 1] + 1 : cg.line_y[J], jhi = J < cg.gy ? cg.line_y[J + 1] - 1 : cg.line_y[J];
    double ax = 0.0, ay = 0.0;
    int free_bits = 0;
    for (int i = ilo; i <= ihi; ++i) {
        const double wx = hat(cg.line_x, nx, I, i);
        for (int j = jlo; j <= jhi; ++j) {
            const int id = fine_node(gnode, fg.gy, i, j);
            if (id < 0) continue;
            const double w = wx * hat(cg.line_y, ny, J, j);
            const int f = ffix[id];
            if (r) {
                const double2 t = r2[id];
                if (!(f & 1)) ax += w * t.x;
                if (!(f & 2)) ay += w * t.y;
            }
            if (w > 0.0) free_bits |= (~f) & 3;
        }
    }
    if (rc) reinterpret_cast<double2*>(rc)[n] = make_double2(ax, ay);
    if (fix_out) fix_out[n] = (uint8_t)((~free_bits) & 3);
}

__global__ void k_mg_restrict(MgGrid fg, MgGrid cg, const int32_t* __restrict__ gnode, const uint8_t* __restrict__ ffix,
                              const double* __restrict__ r, double* __restrict__ rc, uint8_t* __restrict__ fix_out) {
    const int n_nodes = (cg.gx + 1) * (cg.gy + 1);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x)
        mg_restrict_node(fg, cg, gnode, ffix, r, rc, fix_out, n);
}

// x += P~ ec (x untouched at fixed fine DOFs) at fine grid node n
__device__ __forceinline__ void mg_prolong_node(const MgGrid& fg, const MgGrid& cg, const int32_t* gnode,
                                                const uint8_t* ffix, const double* ec, double* x, int n) {
    const int fny = fg.gy + 1, cny = cg.gy + 1;
    const double2* e2 = reinterpret_cast<const double2*>(ec);
    double2* x2 = reinterpret_cast<double2*>(x);
    const int i = n / fny, j = n % fny;
    const int id = gnode ? gnode[n] : n;
    if (id < 0) return;
    const int f = ffix[id];
    if ((f & 3) == 3) return;
    const int CX = cg.cell_x[i], CY = cg.cell_y[j];
    const int x0 = cg.line_x[CX], x1 = cg.line_x[CX + 1], y0 = cg.line_y[CY], y1 = cg.line_y[CY + 1];
    const double wx1 = (double)(i - x0) / (double)(x1 - x0), wy1 = (double)(j - y0) / (double)(y1 - y0);
    const double wx0 = 1.0 - wx1, wy0 = 1.0 - wy1;
    const double2 e00 = e2[CX * cny + CY], e10 = e2[(CX + 1) * cny + CY];
    const double2 e11 = e2[(CX + 1) * cny + CY + 1], e01 = e2[CX * cny + CY + 1];
    double2 t = x2[id];
    if (!(f & 1)) t.x += wx0 * wy0 * e00.x + wx1 * wy0 * e10.x + wx1 * wy1 * e11.x + wx0 * wy1 * e01.x;
    if (!(f & 2)) t.y += wx0 * wy0 * e00.y + wx1 * wy0 * e10.y + wx1 * wy1 * e11.y + wx0 * wy1 * e01.y;
    x2[id] = t;
}

__global__ void k_mg_prolong_add(MgGrid fg, MgGrid cg, const int32_t* __restrict__ gnode, const uint8_t* __restrict__ ffix,
                                 const double* __restrict__ ec, double* __restrict__ x) {
    const int n_nodes = (fg.gx + 1) * (fg.gy + 1);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x)
        mg_prolong_node(fg, cg, gnode, ffix, ec, x, n);
}

// ------------------------------------------------------------------------------------------
// coarse-level operator: y = K v + (I - M) v (K has zero rows and columns at fixed DOFs); DIAG: diag(A)
// ------------------------------------------------------------------------------------------
// row of node n = I * ny + J (both DOFs); the standalone product and the fused smoothing steps below share it,
// so they compute the same sums in the same order
template <bool DIAG>
__device__ __forceinline__ double2 mg_node_row(const MgGrid& g, const double2* v2, int n) {
    const int ny = g.gy + 1, n_cells = g.gx * g.gy;
    const int I = n / ny, J = n % ny;
    double y0 = 0.0, y1 = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        // cells around the node and the node's corner in each: (I-1,J-1):2 (I,J-1):3 (I,J):0 (I-1,J):1
        const int CX = (k == 0 || k == 3) ? I - 1 : I, CY = (k <= 1) ? J - 1 : J;
        const int b = k == 0 ? 2 : k == 1 ? 3 : k == 2 ? 0 : 1;
        if (CX < 0 || CY < 0 || CX >= g.gx || CY >= g.gy) continue;
        const int c = CX * g.gy + CY;
        if (DIAG) {
            y0 += g.K[(int64_t)((2 * b) * 8 + 2 * b) * n_cells + c];
            y1 += g.K[(int64_t)((2 * b + 1) * 8 + 2 * b + 1) * n_cells + c];
        } else {
            const int cn[4] = {CX * ny + CY, (CX + 1) * ny + CY, (CX + 1) * ny + CY + 1, CX * ny + CY + 1};
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double2 t = v2[cn[a]];
                y0 += g.K[(int64_t)((2 * b) * 8 + 2 * a) * n_cells + c] * t.x +
                      g.K[(int64_t)((2 * b) * 8 + 2 * a + 1) * n_cells + c] * t.y;
                y1 += g.K[(int64_t)((2 * b + 1) * 8 + 2 * a) * n_cells + c] * t.x +
                      g.K[(int64_t)((2 * b + 1) * 8 + 2 * a + 1) * n_cells + c] * t.y;
            }
        }
    }
    const int f = g.fix[n];
    if (DIAG) {
        y0 = (f & 1) ? 1.0 : y0;
        y1 = (f & 2) ? 1.0 : y1;
    } else {
        const double2 t = v2[n];
        if (f & 1) y0 += t.x;
        if (f & 2) y1 += t.y;
    }
    return make_double2(y0, y1);
}

template <bool DIAG>
__global__ void __launch_bounds__(256) k_mg_apply(MgGrid g, const double* __restrict__ v, double* __restrict__ y) {
    const int n_nodes = (g.gx + 1) * (g.gy + 1);
    const double2* v2 = reinterpret_cast<const double2*>(v);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x)
        reinterpret_cast<double2*>(y)[n] = mg_node_row<DIAG>(g, v2, n);
}

// ------------------------------------------------------------------------------------------
// Chebyshev smoothing steps (the Chebyshev iteration, e.g. Saad, Iterative Methods, Alg. 12.1, with the
// Jacobi diagonal as preconditioner)
// ------------------------------------------------------------------------------------------
// the coefficients are read from device memory, so a captured cycle follows them from one linearisation
// to the next
__global__ void k_mg_cheb_start(int64_t n, const double* __restrict__ r, const double* __restrict__ diag,
                                const double* __restrict__ scale, double* __restrict__ d) {
    const double s = *scale;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = s * r[i] / diag[i];
}

__global__ void k_mg_cheb_step(int64_t n, double* __restrict__ x, double* __restrict__ r, double* __restrict__ d,
                               const double* __restrict__ q, const double* __restrict__ diag,
                               const double* __restrict__ c, int last) {
    const double c1 = last ? 0.0 : c[0], c2 = last ? 0.0 : c[1];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double di = d[i];
        x[i] += di;
        const double ri = r[i] - q[i];
        r[i] = ri;
        if (!last) d[i] = c1 * di + c2 * ri / diag[i];
    }
}

// Fused forms used inside a V-cycle; each computes exactly the expressions of the separate kernels it
// replaces (the copy and reset before the pre-smoothing, k_mg_cheb_start, k_mg_apply + k_mg_cheb_step,
// k_mg_apply / the tangent product + r = b - q + k_mg_cheb_start), in one launch instead of two or three.

// start of the pre-smoothing from x = 0: r = b, x = 0, d = s r / D
__global__ void k_mg_cheb_first(int64_t n, const double* __restrict__ b, const double* __restrict__ diag,
                                const double* __restrict__ scale, double* __restrict__ r, double* __restrict__ x,
                                double* __restrict__ d) {
    const double s = *scale;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double bi = b[i];
        r[i] = bi;
        x[i] = 0.0;
        d[i] = s * bi / diag[i];
    }
}

// start of the post-smoothing from the product q = A x in memory: r = b - q, d = s r / D
__global__ void k_mg_cheb_restart(int64_t n, const double* __restrict__ b, const double* __restrict__ q,
                                  const double* __restrict__ diag, const double* __restrict__ scale,
                                  double* __restrict__ r, double* __restrict__ d) {
    const double s = *scale;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = b[i] - q[i];
        r[i] = ri;
        d[i] = s * ri / diag[i];
    }
}

// the same on a coarse level with the product computed at node n: r = b - A x, d = s r / D
__device__ __forceinline__ void mg_residual_restart_node(const MgGrid& g, const double* b, const double* x,
                                                         const double* diag, double s, double* r, double* d, int n) {
    const double2 q = mg_node_row<false>(g, reinterpret_cast<const double2*>(x), n);
    const double2 bn = reinterpret_cast<const double2*>(b)[n], dn = reinterpret_cast<const double2*>(diag)[n];
    const double r0 = bn.x - q.x, r1 = bn.y - q.y;
    reinterpret_cast<double2*>(r)[n] = make_double2(r0, r1);
    reinterpret_cast<double2*>(d)[n] = make_double2(s * r0 / dn.x, s * r1 / dn.y);
}

__global__ void __launch_bounds__(256) k_mg_residual_restart(MgGrid g, const double* __restrict__ b,
                                                             const double* __restrict__ x, const double* __restrict__ diag,
                                                             const double* __restrict__ scale, double* __restrict__ r,
                                                             double* __restrict__ d) {
    const double s = *scale;
    const int n_nodes = (g.gx + 1) * (g.gy + 1);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x)
        mg_residual_restart_node(g, b, x, diag, s, r, d, n);
}

// one Chebyshev step on a coarse level with its product computed at node n: q = A d_in, x += d_in,
// r -= q, d_out = c1 d_in + c2 r / D (not written by the last step).  d is double-buffered because
// neighbouring nodes read d_in.
__device__ __forceinline__ void mg_cheb_apply_step_node(const MgGrid& g, double* x, double* r, const double* d_in,
                                                        double* d_out, const double* diag, double c1, double c2,
                                                        int last, int n) {
    const double2* d2 = reinterpret_cast<const double2*>(d_in);
    const double2 q = mg_node_row<false>(g, d2, n), dn = d2[n];
    double2* x2 = reinterpret_cast<double2*>(x);
    double2* r2 = reinterpret_cast<double2*>(r);
    double2 xn = x2[n];
    xn.x += dn.x;
    xn.y += dn.y;
    x2[n] = xn;
    const double2 rn = r2[n];
    const double r0 = rn.x - q.x, r1 = rn.y - q.y;
    r2[n] = make_double2(r0, r1);
    if (!last) {
        const double2 Dn = reinterpret_cast<const double2*>(diag)[n];
        reinterpret_cast<double2*>(d_out)[n] = make_double2(c1 * dn.x + c2 * r0 / Dn.x, c1 * dn.y + c2 * r1 / Dn.y);
    }
}

__global__ void __launch_bounds__(256) k_mg_cheb_apply_step(MgGrid g, double* __restrict__ x, double* __restrict__ r,
                                                            const double* __restrict__ d_in, double* __restrict__ d_out,
                                                            const double* __restrict__ diag,
                                                            const double* __restrict__ c, int last) {
    const double c1 = last ? 0.0 : c[0], c2 = last ? 0.0 : c[1];
    const int n_nodes = (g.gx + 1) * (g.gy + 1);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x)
        mg_cheb_apply_step_node(g, x, r, d_in, d_out, diag, c1, c2, last, n);
}

// ------------------------------------------------------------------------------------------
// Lanczos by Jacobi-preconditioned CG (the extreme eigenvalue of D^-1 A from the CG coefficients): the
// scalars stay on the device, s = [p.Ap, r.z, -, beta], hist = (alpha_k, beta_k) per step
// ------------------------------------------------------------------------------------------
// Dot products in two fixed-order passes: per-block partial sums (the block count depends on n only), then
// one block adds them in block order.
constexpr int kMgDotBlocks = 296;
constexpr int kMgDotThreads = 256;

__host__ __device__ static int mg_dot_blocks(int64_t n) {
    const int64_t b = (n + 4 * kMgDotThreads - 1) / (4 * kMgDotThreads);
    return (int)(b < 1 ? 1 : (b > kMgDotBlocks ? kMgDotBlocks : b));
}

// The library's own drivers take a dot product in ONE launch: every block stores its partial sum, and the last
// block to arrive (an integer ticket after the partials in dot_work, zeroed at every set-up and reset by that
// block) adds the partials with k_mg_dot_final's tree, so the result is bitwise that of the two-launch form.
constexpr int kMgDotWork = kMgDotBlocks + 32;   // doubles: the partials, then the ticket (256-byte padded)
__host__ __device__ inline unsigned* dot_ticket(double* work) { return reinterpret_cast<unsigned*>(work + kMgDotBlocks); }

__global__ void __launch_bounds__(kMgDotThreads) k_mg_dot_part(int64_t n, const double* __restrict__ x,
                                                                const double* __restrict__ y, double* __restrict__ part) {
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a += x[i] * y[i];
    a = block_sum<kMgDotThreads>(a);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// thread 0 of the block that holds the total: what k_mg_dot_final stores (LANCZOS: the CG step's bookkeeping)
template <bool LANCZOS>
__device__ __forceinline__ void dot_store(double a, double* out, double* hist, int k) {
    if (LANCZOS) {
        const double alpha = out[1] / out[0], beta = a / out[1];
        hist[2 * k] = alpha;
        hist[2 * k + 1] = beta;
        out[1] = a;
        out[3] = beta;
    } else {
        *out = a;
    }
}

// the block partial of a dot handed to the last-block sum; true in the block that stored the total
template <bool LANCZOS>
__device__ __forceinline__ void dot_finish(double a, double* work, double* out, double* hist, int k) {
    const double vals[1] = {block_sum<kMgDotThreads>(a)};
    double tot[1];
    if (last_block_sum<kMgDotThreads, 1>(vals, RedSite{work, dot_ticket(work), nullptr}, tot) && threadIdx.x == 0)
        dot_store<LANCZOS>(tot[0], out, hist, k);
}

// x.y in one launch (grid: mg_dot_blocks(n) blocks of kMgDotThreads)
template <bool LANCZOS>
__global__ void __launch_bounds__(kMgDotThreads) k_mg_dot1(int64_t n, const double* __restrict__ x,
                                                            const double* __restrict__ y, double* __restrict__ work,
                                                            double* __restrict__ out, double* __restrict__ hist, int k) {
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a += x[i] * y[i];
    dot_finish<LANCZOS>(a, work, out, hist, k);
}

// k_mg_lanczos_step and the following r.z in one launch: r -= alpha q, z = r / D with alpha = s[1] / s[0], then
// the CG step's bookkeeping of k_mg_dot_final<true>
__global__ void __launch_bounds__(kMgDotThreads) k_mg_lanczos_step_rz(int64_t n, const double* __restrict__ q,
                                                                       double* __restrict__ r, double* __restrict__ z,
                                                                       const double* __restrict__ diag,
                                                                       double* __restrict__ s, double* __restrict__ work,
                                                                       double* __restrict__ hist, int k) {
    const double alpha = s[1] / s[0];
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double zi = ri / diag[i];
        z[i] = zi;
        a += ri * zi;
    }
    dot_finish<true>(a, work, s, hist, k);
}

// the drivers' dot: x.y into *out in one launch (the ticket in work is zero, as every set-up leaves it)
static int mg_dot1(int64_t n, const double* x, const double* y, double* out, double* work, cudaStream_t s) {
    k_mg_dot1<false><<<mg_dot_blocks(n), kMgDotThreads, 0, s>>>(n, x, y, work, out, nullptr, 0);
    note_launches(1);
    return launch_check("multigrid dot");
}

// x += alpha p, r += neg q (neg = -alpha) and r.r in the grid and accumulation order of the dot: the PCG update
// of dfea_mg_pcg's host-driven loop (two axpys and its r.r) in one launch, with the same expressions, so the
// iterates and the norm are bitwise the same
__global__ void __launch_bounds__(kMgDotThreads) k_mg_update_rr(int64_t n, double alpha, double neg,
                                                                 const double* __restrict__ p, const double* __restrict__ q,
                                                                 double* __restrict__ x, double* __restrict__ r,
                                                                 double* __restrict__ work, double* __restrict__ out) {
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        double ri = r[i];
        ri += neg * q[i];
        r[i] = ri;
        a += ri * ri;
    }
    dot_finish<false>(a, work, out, nullptr, 0);
}

// LANCZOS: the sum is r.z of a CG step: alpha = s[1] / s[0], beta = sum / s[1] into hist, s[1] = sum, s[3] = beta
template <bool LANCZOS>
__global__ void __launch_bounds__(kMgDotThreads) k_mg_dot_final(int nb, const double* __restrict__ part,
                                                                 double* __restrict__ out, double* __restrict__ hist, int k) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) a += part[b];
    a = block_sum<kMgDotThreads>(a);
    if (threadIdx.x == 0) {
        if (LANCZOS) {
            const double alpha = out[1] / out[0], beta = a / out[1];
            hist[2 * k] = alpha;
            hist[2 * k + 1] = beta;
            out[1] = a;
            out[3] = beta;
        } else {
            *out = a;
        }
    }
}

__global__ void k_mg_lanczos_step(int64_t n, const double* __restrict__ q, double* __restrict__ r, double* __restrict__ z,
                                  const double* __restrict__ diag, const double* __restrict__ s) {
    const double alpha = s[1] / s[0];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        z[i] = ri / diag[i];
    }
}

__global__ void k_mg_lanczos_p(int64_t n, double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ s) {
    const double beta = s[3];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// the drivers' Lanczos step: dfea_mg_lanczos_step's arithmetic in three launches instead of six
static int mg_lanczos_step1(int64_t n, double* p, const double* q, double* r, double* z, const double* diag, double* sc,
                            double* hist, int k, double* work, cudaStream_t s) {
    const int nb = mg_dot_blocks(n);
    k_mg_dot1<false><<<nb, kMgDotThreads, 0, s>>>(n, p, q, work, sc, nullptr, 0);
    k_mg_lanczos_step_rz<<<nb, kMgDotThreads, 0, s>>>(n, q, r, z, diag, sc, work, hist, k);
    k_mg_lanczos_p<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(n, p, z, sc);
    note_launches(3);
    return launch_check("multigrid Lanczos step");
}

// ------------------------------------------------------------------------------------------
// Lanczos of the small levels in one block (levels of at most kMgTailNodes nodes, each smoothed level's
// start and all its steps).  The dot products reproduce dfea_mg_dot inside the block: nb = mg_dot_blocks(n)
// virtual blocks of kMgDotThreads threads with the same grid-stride accumulation, the same warp and block
// trees, then the final block's tree over the nb partials, so the coefficients, the bounds and every later
// iterate are bitwise those of the separate launches.
// ------------------------------------------------------------------------------------------
constexpr int kMgTailLanczosThreads = 2 * kMgDotThreads;

struct MgLanczosLevel {
    MgGrid grid;
    int n;                       // DOFs
    const double* diag;
    double *r, *z, *p, *q;       // the level's r, d, x and q buffers
    double* s;                   // [p.Ap, r.z, -, beta]
    double* hist;                // (alpha_k, beta_k) per step
};

struct MgLanczosTail {
    int n_levels, steps;
    MgLanczosLevel lv[DFEA_MG_MAX_LEVELS];
};

// x.y, returned to every thread; every thread of the block calls it
__device__ double tail_dot(int n, const double* x, const double* y) {
    constexpr int NW = kMgDotThreads / 32;
    __shared__ double warp_part[kMgTailLanczosThreads / 32];
    __shared__ double block_part[kMgDotBlocks];
    __shared__ double result;
    const int half = threadIdx.x / kMgDotThreads, vt = threadIdx.x % kMgDotThreads;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nb = mg_dot_blocks(n);
    for (int vb0 = 0; vb0 < nb; vb0 += 2) {
        const int vb = vb0 + half;
        double a = 0.0;
        if (vb < nb)
            for (int64_t i = vb * (int64_t)kMgDotThreads + vt; i < n; i += (int64_t)nb * kMgDotThreads) a += x[i] * y[i];
        a = warp_sum(a);
        if (lane == 0) warp_part[warp] = a;
        __syncthreads();
        if (warp % NW == 0) {
            double r = (lane < NW) ? warp_part[warp + lane] : 0.0;
            r = warp_sum(r);
            if (lane == 0 && vb < nb) block_part[vb] = r;
        }
        __syncthreads();
    }
    if (threadIdx.x < kMgDotThreads) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nb; b += kMgDotThreads) a += block_part[b];
        a = warp_sum(a);
        if (lane == 0) warp_part[warp] = a;
    }
    __syncthreads();
    if (warp == 0) {
        double r = (lane < NW) ? warp_part[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) result = r;
    }
    __syncthreads();
    const double out = result;
    __syncthreads();
    return out;
}

__global__ void __launch_bounds__(kMgTailLanczosThreads) k_mg_tail_lanczos(const __grid_constant__ MgLanczosTail T) {
    for (int l = 0; l < T.n_levels; ++l) {
        const MgLanczosLevel& L = T.lv[l];
        const int n_nodes = L.n / 2;
        // start: r = sin(i + 1), z = r / D, p = z, s[1] = r.z
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            const double ri = sin((double)(i + 1));
            L.r[i] = ri;
            const double zi = ri / L.diag[i];
            L.z[i] = zi;
            L.p[i] = zi;
        }
        __syncthreads();
        double rz = tail_dot(L.n, L.r, L.z);
        if (threadIdx.x == 0) L.s[1] = rz;
        for (int k = 0; k < T.steps; ++k) {
            for (int n = threadIdx.x; n < n_nodes; n += blockDim.x)
                reinterpret_cast<double2*>(L.q)[n] = mg_node_row<false>(L.grid, reinterpret_cast<const double2*>(L.p), n);
            __syncthreads();
            const double pq = tail_dot(L.n, L.p, L.q);
            const double alpha = rz / pq;
            for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
                const double ri = L.r[i] - alpha * L.q[i];
                L.r[i] = ri;
                L.z[i] = ri / L.diag[i];
            }
            __syncthreads();
            const double rz_new = tail_dot(L.n, L.r, L.z);
            const double beta = rz_new / rz;
            if (threadIdx.x == 0) {
                L.hist[2 * k] = alpha;
                L.hist[2 * k + 1] = beta;
                L.s[0] = pq;
                L.s[1] = rz_new;
                L.s[3] = beta;
            }
            rz = rz_new;
            for (int i = threadIdx.x; i < L.n; i += blockDim.x) L.p[i] = L.z[i] + beta * L.p[i];
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------------------------
// coarsest level: dense A (assembled in cell order), inverted by Gauss-Jordan (A is SPD: no pivoting)
// ------------------------------------------------------------------------------------------
constexpr int kMgDenseMax = 256;     // DOFs
constexpr int kMgDenseShared = 112;  // up to this many DOFs A, Ainv and the pivot column live in shared memory

// SHARED: A and Ainv in dynamic shared memory (copied to Ainv_out at the end), else in global memory
template <bool SHARED>
__global__ void __launch_bounds__(1024) k_mg_dense_inverse(MgGrid g, double* __restrict__ A_glob, double* __restrict__ Ainv_out) {
    extern __shared__ double dense_sm[];
    const int ny = g.gy + 1, nn = (g.gx + 1) * ny, n = 2 * nn, n_cells = g.gx * g.gy;
    double* A = SHARED ? dense_sm : A_glob;
    double* Ainv = SHARED ? dense_sm + n * n : Ainv_out;
    double* fcol = SHARED ? dense_sm + 2 * n * n : nullptr;
    __shared__ double fcol_glob[SHARED ? 1 : 2 * kMgDenseMax];
    if (!SHARED) fcol = fcol_glob;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        A[k] = 0.0;
        Ainv[k] = (k / n == k % n) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int c = 0; c < n_cells; ++c) {
        const int CX = c / g.gy, CY = c % g.gy;
        if (threadIdx.x < 64) {
            const int row = threadIdx.x >> 3, col = threadIdx.x & 7;
            const int cn[4] = {CX * ny + CY, (CX + 1) * ny + CY, (CX + 1) * ny + CY + 1, CX * ny + CY + 1};
            const int R = 2 * cn[row >> 1] + (row & 1), Cc = 2 * cn[col >> 1] + (col & 1);
            A[R * n + Cc] += g.K[(int64_t)threadIdx.x * n_cells + c];
        }
        __syncthreads();
    }
    for (int d = threadIdx.x; d < n; d += blockDim.x)
        if ((g.fix[d >> 1] >> (d & 1)) & 1) A[d * n + d] += 1.0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double p = 1.0 / A[k * n + k];
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            A[k * n + j] *= p;
            Ainv[k * n + j] *= p;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = A[r * n + k];
        __syncthreads();
        for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
            const int r = t / n, j = t % n;
            if (r == k) continue;
            const double f = fcol[r];
            A[r * n + j] -= f * A[k * n + j];
            Ainv[r * n + j] -= f * Ainv[k * n + j];
        }
        __syncthreads();
    }
    if (SHARED)
        for (int t = threadIdx.x; t < n * n; t += blockDim.x) Ainv_out[t] = Ainv[t];
}

// x = Ainv b, one warp per row
// row r of x = Ainv b by one warp (lane-strided partial sums, then the warp's butterfly sum)
__device__ __forceinline__ void mg_dense_row(int n, const double* Ainv, const double* b, double* x, int r, int lane) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += Ainv[(int64_t)r * n + j] * b[j];
    s = warp_sum(s);
    if (lane == 0) x[r] = s;
}

__global__ void k_mg_dense_solve(int n, const double* __restrict__ Ainv, const double* __restrict__ b, double* __restrict__ x) {
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5)
        mg_dense_row(n, Ainv, b, x, r, lane);
}

// ------------------------------------------------------------------------------------------
// the coarse tail of a V-cycle in one block: levels t .. L-1 are small enough that a launch per smoothing
// step costs more than the step, so one block runs the restriction from level t - 1, the smoothing of
// every tail level, the coarsest solve and the prolongation back to level t - 1, with a block barrier
// between phases.  Each phase calls the per-node function of the kernel it replaces, so the result is
// bitwise that of the separate launches.
// ------------------------------------------------------------------------------------------
constexpr int kMgTailThreads = 1024;
constexpr int kMgTailNodes = 1536;   // levels of at most this many nodes run in the tail

struct MgTailLevel {
    MgGrid grid;
    int n;                       // DOFs
    const double* diag;
    const double* coef;          // [scale, (c1, c2) per step]
    double *b, *x, *r, *d, *q;
};

struct MgTail {
    MgGrid fine;                 // level t - 1 (the transfers' fine side)
    const int32_t* gnode;
    const uint8_t* ffix;
    const double* r_fine;        // level t - 1's residual, restricted into level t's right-hand side
    double* x_fine;              // level t - 1's iterate, corrected by the prolongation of level t's
    const double* Ainv;
    int n_levels, degree;        // tail levels; the last is the coarsest
    MgTailLevel lv[DFEA_MG_MAX_LEVELS];
};

__device__ __forceinline__ void tail_smooth(const MgTailLevel& L, int degree) {
    const int n_nodes = L.n / 2;
    double *d_in = L.d, *d_out = L.q;
    for (int k = 1; k <= degree; ++k) {
        const int last = k == degree ? 1 : 0;
        const double c1 = last ? 0.0 : L.coef[1 + 2 * (k - 1)], c2 = last ? 0.0 : L.coef[2 + 2 * (k - 1)];
        for (int n = threadIdx.x; n < n_nodes; n += blockDim.x)
            mg_cheb_apply_step_node(L.grid, L.x, L.r, d_in, d_out, L.diag, c1, c2, last, n);
        __syncthreads();
        double* t = d_in;
        d_in = d_out;
        d_out = t;
    }
}

__global__ void __launch_bounds__(kMgTailThreads) k_mg_tail(const __grid_constant__ MgTail T) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    const int last = T.n_levels - 1;
    for (int l = 0; l <= last; ++l) {
        const MgTailLevel& L = T.lv[l];
        const MgGrid& fg = l == 0 ? T.fine : T.lv[l - 1].grid;
        const int32_t* gn = l == 0 ? T.gnode : nullptr;
        const uint8_t* ffix = l == 0 ? T.ffix : T.lv[l - 1].grid.fix;
        const double* r = l == 0 ? T.r_fine : T.lv[l - 1].r;
        for (int n = threadIdx.x; n < L.n / 2; n += blockDim.x) mg_restrict_node(fg, L.grid, gn, ffix, r, L.b, nullptr, n);
        __syncthreads();
        if (l == last) break;
        const double s = L.coef[0];
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            const double bi = L.b[i];
            L.r[i] = bi;
            L.x[i] = 0.0;
            L.d[i] = s * bi / L.diag[i];
        }
        __syncthreads();
        tail_smooth(L, T.degree);
    }
    const MgTailLevel& C = T.lv[last];
    for (int r = warp; r < C.n; r += n_warps) mg_dense_row(C.n, T.Ainv, C.b, C.x, r, lane);
    __syncthreads();
    for (int l = last; l >= 0; --l) {
        const MgTailLevel& L = T.lv[l];
        const MgGrid& fg = l == 0 ? T.fine : T.lv[l - 1].grid;
        const int32_t* gn = l == 0 ? T.gnode : nullptr;
        const uint8_t* ffix = l == 0 ? T.ffix : T.lv[l - 1].grid.fix;
        double* xf = l == 0 ? T.x_fine : T.lv[l - 1].x;
        const int fine_nodes = (fg.gx + 1) * (fg.gy + 1);
        for (int n = threadIdx.x; n < fine_nodes; n += blockDim.x) mg_prolong_node(fg, L.grid, gn, ffix, L.x, xf, n);
        __syncthreads();
        if (l == 0) break;
        const MgTailLevel& F = T.lv[l - 1];
        const double s = F.coef[0];
        for (int n = threadIdx.x; n < F.n / 2; n += blockDim.x) mg_residual_restart_node(F.grid, F.b, F.x, F.diag, s, F.r, F.d, n);
        __syncthreads();
        tail_smooth(F, T.degree);
    }
}

}  // namespace dfea

using namespace dfea;

extern "C" int dfea_mg_galerkin_fe(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype,
                                   const int32_t* node_ij, const int32_t* cell_slot, int32_t span,
                                   const dfea_mg_grid* fine, const dfea_mg_grid* coarse, void* stream) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if ((rc = validate_grid(fine, false, "dfea_mg_galerkin_fe")) || (rc = validate_grid(coarse, true, "dfea_mg_galerkin_fe")))
        return rc;
    if (!moduli || !node_ij || !cell_slot || !coarse->K) return set_error(DFEA_ERR_INVALID, "dfea_mg_galerkin_fe: NULL pointer");
    if (span != 1 && span != 2) return set_error(DFEA_ERR_INVALID, "dfea_mg_galerkin_fe: span must be 1 or 2");
    const int64_t n_cells = (int64_t)(fine->gx / span) * (fine->gy / span);
    const int epc = n_cells > 0 ? (int)(mesh->n_el / n_cells) : 0;   // elements per cell: 1, or 2 triangles
    if (fine->gx % span || fine->gy % span || (epc != 1 && epc != 2) || n_cells * epc != mesh->n_el)
        return set_error(DFEA_ERR_INVALID, "dfea_mg_galerkin_fe: the grid does not match the mesh's element count");
    const Mesh m = kernel_mesh(*mesh);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n_ccells = coarse->gx * coarse->gy;
    const int grid = grid_for(n_ccells, 128, 8);
    const MgGrid cg = mg_grid(*coarse);
    const int ncy = fine->gy / span;
    rc = dispatch_element(mesh->nen, mesh->n_q, [&](auto nen_c, auto nq_c) -> int {
        constexpr int NEN = decltype(nen_c)::value, NQ = decltype(nq_c)::value;
        const RefGrad<NEN, NQ> rg = ref_grad_of<NEN, NQ>(*mesh);
        if (moduli_dtype == DFEA_F64)
            k_mg_galerkin_fe<NEN, NQ, 0><<<grid, 128, 0, s>>>(m, moduli, rg, node_ij, cell_slot, span, epc, ncy, cg);
        else if (moduli_dtype == DFEA_F32)
            k_mg_galerkin_fe<NEN, NQ, 1><<<grid, 128, 0, s>>>(m, moduli, rg, node_ij, cell_slot, span, epc, ncy, cg);
        else if (moduli_dtype == DFEA_F32REF)
            k_mg_galerkin_fe<NEN, NQ, 2><<<grid, 128, 0, s>>>(m, moduli, rg, node_ij, cell_slot, span, epc, ncy, cg);
        else
            return set_error(DFEA_ERR_INVALID, "dfea_mg_galerkin_fe: bad moduli dtype");
        return DFEA_OK;
    });
    if (rc) return rc;
    note_launches(1);
    return launch_check("dfea_mg_galerkin_fe");
}

extern "C" int dfea_mg_galerkin(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, void* stream) {
    int rc;
    if ((rc = validate_grid(fine, true, "dfea_mg_galerkin")) || (rc = validate_grid(coarse, true, "dfea_mg_galerkin")))
        return rc;
    if (!fine->K || !coarse->K) return set_error(DFEA_ERR_INVALID, "dfea_mg_galerkin: NULL element matrices");
    const int n_cells = coarse->gx * coarse->gy;
    k_mg_galerkin<<<grid_for(n_cells, 128, 8), 128, 0, static_cast<cudaStream_t>(stream)>>>(mg_grid(*fine), mg_grid(*coarse));
    note_launches(1);
    return launch_check("dfea_mg_galerkin");
}

extern "C" int dfea_mg_restrict(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, const int32_t* gnode,
                                const uint8_t* fine_fix, const double* r, double* rc_out, uint8_t* coarse_fix_out,
                                void* stream) {
    int rc;
    if ((rc = validate_grid(fine, false, "dfea_mg_restrict")) || (rc = validate_grid(coarse, true, "dfea_mg_restrict")))
        return rc;
    if (!fine_fix || (!rc_out && !coarse_fix_out) || (rc_out && !r))
        return set_error(DFEA_ERR_INVALID, "dfea_mg_restrict: NULL pointer");
    const int n = (coarse->gx + 1) * (coarse->gy + 1);
    k_mg_restrict<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        mg_grid(*fine), mg_grid(*coarse), gnode, fine_fix, r, rc_out, coarse_fix_out);
    note_launches(1);
    return launch_check("dfea_mg_restrict");
}

extern "C" int dfea_mg_prolong_add(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, const int32_t* gnode,
                                   const uint8_t* fine_fix, const double* ec, double* x, void* stream) {
    int rc;
    if ((rc = validate_grid(fine, false, "dfea_mg_prolong_add")) || (rc = validate_grid(coarse, true, "dfea_mg_prolong_add")))
        return rc;
    if (!fine_fix || !ec || !x) return set_error(DFEA_ERR_INVALID, "dfea_mg_prolong_add: NULL pointer");
    const int n = (fine->gx + 1) * (fine->gy + 1);
    k_mg_prolong_add<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        mg_grid(*fine), mg_grid(*coarse), gnode, fine_fix, ec, x);
    note_launches(1);
    return launch_check("dfea_mg_prolong_add");
}

extern "C" int dfea_mg_apply(const dfea_mg_grid* grid, const double* v, double* y, void* stream) {
    int rc = validate_grid(grid, false, "dfea_mg_apply");
    if (rc) return rc;
    if (!grid->K || !grid->fix || !y || (v == nullptr)) return set_error(DFEA_ERR_INVALID, "dfea_mg_apply: NULL pointer");
    const int n = (grid->gx + 1) * (grid->gy + 1);
    k_mg_apply<false><<<grid_for(n, 256, 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(mg_grid(*grid), v, y);
    note_launches(1);
    return launch_check("dfea_mg_apply");
}

extern "C" int dfea_mg_diag(const dfea_mg_grid* grid, double* diag, void* stream) {
    int rc = validate_grid(grid, false, "dfea_mg_diag");
    if (rc) return rc;
    if (!grid->K || !grid->fix || !diag) return set_error(DFEA_ERR_INVALID, "dfea_mg_diag: NULL pointer");
    const int n = (grid->gx + 1) * (grid->gy + 1);
    k_mg_apply<true><<<grid_for(n, 256, 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(mg_grid(*grid), nullptr, diag);
    note_launches(1);
    return launch_check("dfea_mg_diag");
}

extern "C" int dfea_mg_cheb_start(int64_t n, const double* r, const double* diag, const double* scale, double* d,
                                  void* stream) {
    if (n < 0 || (n > 0 && (!r || !diag || !d || !scale))) return set_error(DFEA_ERR_INVALID, "dfea_mg_cheb_start: bad arguments");
    if (n == 0) return DFEA_OK;
    k_mg_cheb_start<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, r, diag, scale, d);
    note_launches(1);
    return launch_check("dfea_mg_cheb_start");
}

extern "C" int dfea_mg_cheb_step(int64_t n, double* x, double* r, double* d, const double* q, const double* diag,
                                 const double* c, int32_t last, void* stream) {
    if (n < 0 || (n > 0 && (!x || !r || !d || !q || !diag || (!last && !c))))
        return set_error(DFEA_ERR_INVALID, "dfea_mg_cheb_step: bad arguments");
    if (n == 0) return DFEA_OK;
    k_mg_cheb_step<<<grid_for(n, kThreads, 8), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, x, r, d, q, diag, c,
                                                                                                    last);
    note_launches(1);
    return launch_check("dfea_mg_cheb_step");
}

extern "C" int64_t dfea_mg_dense_max(void) { return kMgDenseMax; }

extern "C" int dfea_mg_dense_inverse(const dfea_mg_grid* grid, double* work, double* Ainv, void* stream) {
    int rc = validate_grid(grid, false, "dfea_mg_dense_inverse");
    if (rc) return rc;
    const int n = 2 * (grid->gx + 1) * (grid->gy + 1);
    if (n > kMgDenseMax) return set_error(DFEA_ERR_INVALID, "dfea_mg_dense_inverse: %d DOFs exceed %d", n, kMgDenseMax);
    if (!grid->K || !grid->fix || !work || !Ainv) return set_error(DFEA_ERR_INVALID, "dfea_mg_dense_inverse: NULL pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n <= kMgDenseShared) {
        const size_t smem = (size_t)(2 * n * n + n) * sizeof(double);
        // the shared-memory opt-in is a property of the function on each device: set once per device
        // ordinal (a bit per device, set under a mutex so that concurrent first set-ups are safe)
        static std::mutex attr_mutex;
        static unsigned long long attr_set = 0ull;
        int dev = 0;
        if ((rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
        if (dev < 0 || dev >= 64) return set_error(DFEA_ERR_INVALID, "dfea_mg_dense_inverse: device ordinal %d", dev);
        {
            std::lock_guard<std::mutex> lock(attr_mutex);
            if (!(attr_set & (1ull << dev))) {
                rc = check_cuda(cudaFuncSetAttribute(k_mg_dense_inverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)((2 * kMgDenseShared * kMgDenseShared + kMgDenseShared) * sizeof(double))),
                                "cudaFuncSetAttribute");
                if (rc) return rc;
                attr_set |= 1ull << dev;
            }
        }
        k_mg_dense_inverse<true><<<1, 1024, smem, st>>>(mg_grid(*grid), work, Ainv);
    } else {
        k_mg_dense_inverse<false><<<1, 1024, 0, st>>>(mg_grid(*grid), work, Ainv);
    }
    note_launches(1);
    return launch_check("dfea_mg_dense_inverse");
}

extern "C" int dfea_mg_dense_solve(int32_t n, const double* Ainv, const double* b, double* x, void* stream) {
    if (n < 1 || n > kMgDenseMax || !Ainv || !b || !x) return set_error(DFEA_ERR_INVALID, "dfea_mg_dense_solve: bad arguments");
    k_mg_dense_solve<<<(n + 7) / 8, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, Ainv, b, x);
    note_launches(1);
    return launch_check("dfea_mg_dense_solve");
}

extern "C" int64_t dfea_mg_dot_work(void) { return kMgDotWork; }

extern "C" int dfea_mg_dot(int64_t n, const double* x, const double* y, double* out, double* work, void* stream) {
    if (n < 0 || !x || !y || !out || !work) return set_error(DFEA_ERR_INVALID, "dfea_mg_dot: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = mg_dot_blocks(n);
    k_mg_dot_part<<<nb, kMgDotThreads, 0, st>>>(n, x, y, work);
    k_mg_dot_final<false><<<1, kMgDotThreads, 0, st>>>(nb, work, out, nullptr, 0);
    note_launches(2);
    return launch_check("dfea_mg_dot");
}

extern "C" int dfea_mg_lanczos_step(int64_t n, double* p, const double* q, double* r, double* z, const double* diag,
                                    double* s, double* hist, int32_t k, double* work, void* stream) {
    if (n < 1 || !p || !q || !r || !z || !diag || !s || !hist || k < 0 || !work)
        return set_error(DFEA_ERR_INVALID, "dfea_mg_lanczos_step: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = mg_dot_blocks(n);
    k_mg_dot_part<<<nb, kMgDotThreads, 0, st>>>(n, p, q, work);
    k_mg_dot_final<false><<<1, kMgDotThreads, 0, st>>>(nb, work, s, nullptr, 0);
    k_mg_lanczos_step<<<grid_for(n, kThreads, 8), kThreads, 0, st>>>(n, q, r, z, diag, s);
    k_mg_dot_part<<<nb, kMgDotThreads, 0, st>>>(n, r, z, work);
    k_mg_dot_final<true><<<1, kMgDotThreads, 0, st>>>(nb, work, s, hist, k);
    k_mg_lanczos_p<<<grid_for(n, kThreads, 8), kThreads, 0, st>>>(n, p, z, s);
    note_launches(6);
    return launch_check("dfea_mg_lanczos_step");
}

// ------------------------------------------------------------------------------------------
// the C++ driver: set-up, V-cycle, PCG
// ------------------------------------------------------------------------------------------
namespace dfea {

__global__ void k_mg_start(int64_t n, double* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = sin((double)(i + 1));
}

__global__ void k_mg_div(int64_t n, const double* __restrict__ r, const double* __restrict__ diag, double* __restrict__ z) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = r[i] / diag[i];
}

// Largest eigenvalue of the symmetric tridiagonal matrix (diagonal a, off-diagonal e) by bisection on the
// Sturm sequence count (number of eigenvalues below x), from the Gershgorin upper bound.
static double tridiag_max_eig(const double* a, const double* e, int m) {
    double lo = a[0], hi = a[0];
    for (int i = 0; i < m; ++i) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < m ? fabs(e[i]) : 0.0);
        lo = fmin(lo, a[i] - r);
        hi = fmax(hi, a[i] + r);
    }
    auto below = [&](double x) {
        int c = 0;
        double d = 1.0;
        for (int i = 0; i < m; ++i) {
            d = a[i] - x - (i > 0 ? e[i - 1] * e[i - 1] / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) ++c;
        }
        return c;
    };
    for (int it = 0; it < 200 && hi - lo > 1e-14 * fmax(1.0, fabs(hi)); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (below(mid) >= m) hi = mid;   // every eigenvalue is below mid
        else lo = mid;
    }
    return hi;
}

// lambda_max of D^-1 A from Jacobi-CG coefficients (alpha_k, beta_k), over the prefix before a breakdown
static double ritz_max(const double* hist, int steps) {
    double a[64], e[64];
    int m = 0;
    for (; m < steps && m < 64; ++m) {
        const double al = hist[2 * m], be = hist[2 * m + 1];
        if (!(std::isfinite(al) && al > 0.0 && std::isfinite(be) && be >= 0.0)) break;
    }
    if (m == 0) return 2.5;
    for (int k = 0; k < m; ++k) {
        a[k] = 1.0 / hist[2 * k] + (k > 0 ? hist[2 * k - 1] / hist[2 * k - 2] : 0.0);
        if (k + 1 < m) e[k] = sqrt(hist[2 * k + 1]) / hist[2 * k];
    }
    return tridiag_max_eig(a, e, m);
}

static void transfer_args(const dfea_mesh_view* mesh, const dfea_mg* mg, int l, const int32_t** gnode,
                          const uint8_t** ffix) {
    *gnode = l == 0 ? mg->gnode : nullptr;
    *ffix = l == 0 ? mesh->node_fix : mg->level[l].grid.fix;
}

// level 0 in the gather form (the hierarchy was given element-product scratch and the mesh has node incidence)
static bool fe_gather(const dfea_mesh_view* mesh, const dfea_mg* mg) {
    return mg->fe_work && mesh->node_elem_ptr && mesh->node_elem;
}

static int mg_apply(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t code, int l,
                    const double* v, double* y, cudaStream_t s) {
    if (l == 0)
        return fe_gather(mesh, mg)
                   ? dfea_tangent_apply_gather(mesh, moduli, code, v, y, DFEA_F64, mg->fe_work, s)
                   : dfea_tangent_apply(mesh, moduli, code, v, y, DFEA_F64, s);
    return dfea_mg_apply(&mg->level[l].grid, v, y, s);
}

// the Chebyshev steps of one smoothing pass at level l, from the first direction in lv.d; on coarse levels
// each step is one fused launch with d alternating between lv.d and lv.q
static int mg_cheb_steps(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t code, int l,
                         double* x, double* r, cudaStream_t s) {
    const dfea_mg_level& lv = mg->level[l];
    const double* row = mg->coef + (int64_t)l * 2 * DFEA_MG_MAX_DEGREE;
    double *d_in = lv.d, *d_out = lv.q;
    int rc = DFEA_OK;
    for (int k = 1; !rc && k <= mg->degree; ++k) {
        const int last = k == mg->degree ? 1 : 0;
        const double* c = last ? nullptr : row + 1 + 2 * (k - 1);
        if (l == 0 && fe_gather(mesh, mg)) {
            rc = mg_fe_gather_cheb(mesh, moduli, code, mg->fe_work, MG_FE_STEP, lv.d, x, r, lv.d, nullptr, lv.diag, c,
                                   last, s);
            continue;
        }
        if (l == 0) {
            if (!(rc = mg_apply(mesh, mg, moduli, code, 0, lv.d, lv.q, s)))
                rc = dfea_mg_cheb_step(lv.n, x, r, lv.d, lv.q, lv.diag, c, last, s);
            continue;
        }
        const int n_nodes = (lv.grid.gx + 1) * (lv.grid.gy + 1);
        k_mg_cheb_apply_step<<<grid_for(n_nodes, 256, 8), 256, 0, s>>>(mg_grid(lv.grid), x, r, d_in, d_out, lv.diag, c, last);
        note_launches(1);
        rc = launch_check("dfea_mg_vcycle: smoothing step");
        std::swap(d_in, d_out);
    }
    return rc;
}

// first level (>= 1) of the one-block tail: levels shrink, so every level from it on is small enough
static int tail_start(const dfea_mg* mg) {
    for (int l = 1; l < mg->n_levels; ++l)
        if (mg->level[l].n / 2 <= kMgTailNodes) return l;
    return mg->n_levels;
}

// restriction of level l's residual, the cycle of levels l + 1 .. L - 1 and the prolongation into x, in one launch
static int launch_tail(const dfea_mesh_view* mesh, const dfea_mg* mg, int l, double* x, cudaStream_t s) {
    MgTail T = {};
    const dfea_mg_level& lv = mg->level[l];
    T.fine = mg_grid(lv.grid);
    transfer_args(mesh, mg, l, &T.gnode, &T.ffix);
    T.r_fine = lv.r;
    T.x_fine = x;
    T.Ainv = mg->Ainv;
    T.n_levels = mg->n_levels - (l + 1);
    T.degree = mg->degree;
    for (int k = 0; k < T.n_levels; ++k) {
        const dfea_mg_level& c = mg->level[l + 1 + k];
        T.lv[k] = MgTailLevel{mg_grid(c.grid), (int)c.n, c.diag, mg->coef + (int64_t)(l + 1 + k) * 2 * DFEA_MG_MAX_DEGREE,
                              c.b, c.x, c.r, c.d, c.q};
    }
    k_mg_tail<<<1, kMgTailThreads, 0, s>>>(T);
    note_launches(1);
    return launch_check("dfea_mg_vcycle: coarse tail");
}

static int mg_vcycle(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t code, int l,
                     const double* b, double* x, cudaStream_t s) {
    const dfea_mg_level& lv = mg->level[l];
    int rc;
    if (l == mg->n_levels - 1) return dfea_mg_dense_solve((int32_t)lv.n, mg->Ainv, b, x, s);
    const double* scale = mg->coef + (int64_t)l * 2 * DFEA_MG_MAX_DEGREE;
    k_mg_cheb_first<<<grid_for(lv.n, kThreads, 8), kThreads, 0, s>>>(lv.n, b, lv.diag, scale, lv.r, x, lv.d);
    note_launches(1);
    if ((rc = launch_check("dfea_mg_vcycle: smoothing start")) || (rc = mg_cheb_steps(mesh, mg, moduli, code, l, x, lv.r, s)))
        return rc;
    const dfea_mg_level& c = mg->level[l + 1];
    const int32_t* gn;
    const uint8_t* ffix;
    transfer_args(mesh, mg, l, &gn, &ffix);
    if (l + 1 == tail_start(mg)) {
        if ((rc = launch_tail(mesh, mg, l, x, s))) return rc;
    } else if ((rc = dfea_mg_restrict(&lv.grid, &c.grid, gn, ffix, lv.r, c.b, nullptr, s)) ||
               (rc = mg_vcycle(mesh, mg, moduli, code, l + 1, c.b, c.x, s)) ||
               (rc = dfea_mg_prolong_add(&lv.grid, &c.grid, gn, ffix, c.x, x, s))) {
        return rc;
    }
    if (l == 0 && fe_gather(mesh, mg)) {
        if ((rc = mg_fe_gather_cheb(mesh, moduli, code, mg->fe_work, MG_FE_RESTART, x, nullptr, lv.r, lv.d, b, lv.diag,
                                    scale, 0, s)))
            return rc;
        return mg_cheb_steps(mesh, mg, moduli, code, l, x, lv.r, s);
    }
    if (l == 0) {
        if ((rc = mg_apply(mesh, mg, moduli, code, 0, x, lv.q, s))) return rc;
        k_mg_cheb_restart<<<grid_for(lv.n, kThreads, 8), kThreads, 0, s>>>(lv.n, b, lv.q, lv.diag, scale, lv.r, lv.d);
    } else {
        const int n_nodes = (lv.grid.gx + 1) * (lv.grid.gy + 1);
        k_mg_residual_restart<<<grid_for(n_nodes, 256, 8), 256, 0, s>>>(mg_grid(lv.grid), b, x, lv.diag, scale, lv.r, lv.d);
    }
    note_launches(1);
    if ((rc = launch_check("dfea_mg_vcycle: residual"))) return rc;
    return mg_cheb_steps(mesh, mg, moduli, code, l, x, lv.r, s);
}

static int validate_mg(const dfea_mesh_view* mesh, const dfea_mg* mg, const char* what) {
    int rc = validate_mesh(mesh, false);
    if (rc) return rc;
    if (!mg || mg->n_levels < 2 || mg->n_levels > DFEA_MG_MAX_LEVELS || mg->degree < 1 ||
        mg->degree > DFEA_MG_MAX_DEGREE || mg->lanczos_steps < 1 || mg->lanczos_steps > 64 || !(mg->ratio > 1.0))
        return set_error(DFEA_ERR_INVALID, "%s: bad hierarchy parameters", what);
    if (mg->level[0].n != 2 * mesh->n_nodes) return set_error(DFEA_ERR_INVALID, "%s: level 0 is not the mesh", what);
    for (int l = 0; l < mg->n_levels; ++l) {
        const dfea_mg_level& lv = mg->level[l];
        // level 0 holds the mesh's DOFs (a Q8 grid has no nodes at the cell centres), the others their grid's
        if ((l > 0 && lv.n != 2 * (int64_t)(lv.grid.gx + 1) * (lv.grid.gy + 1)) || !lv.diag || !lv.b || !lv.x || !lv.r ||
            !lv.d || !lv.q)
            return set_error(DFEA_ERR_INVALID, "%s: level %d buffers", what, l);
        if (l > 0 && (rc = validate_grid(&lv.grid, true, what))) return rc;
    }
    if (mg->level[mg->n_levels - 1].n > kMgDenseMax) return set_error(DFEA_ERR_INVALID, "%s: coarsest level too large", what);
    if (!mg->node_ij || !mg->gnode || !mg->cell_slot || !mg->Ainv || !mg->dense_work || !mg->coef || !mg->lscal ||
        !mg->lhist || !mg->dot_work || !mg->pcg || !mg->scal)
        return set_error(DFEA_ERR_INVALID, "%s: NULL buffer", what);
    return DFEA_OK;
}

static int read_scalars(double* host, const double* dev, int k, cudaStream_t s) {
    return read_to_host(host, dev, k * sizeof(double), s);
}

}  // namespace dfea

namespace dfea {

// ------------------------------------------------------------------------------------------
// graph-driven mode: the captured set-up and the device-side PCG loop
// ------------------------------------------------------------------------------------------
// State of a device-side PCG solve (mg->pcg_state, 16 doubles).
struct MgPcgState {
    double rz, curv, rr, rz_new, nb2, tol2, rtol2, spare;
    int32_t k, max_iter, status, iters, guard, spare_i[3];
};
static_assert(sizeof(MgPcgState) <= 16 * sizeof(double), "pcg_state holds 16 doubles");

// the graphs of one hierarchy, each bound to the buffers it was captured with
struct MgGraphs {
    cudaStream_t capture = nullptr;
    // set-up: moduli, diag and the mesh arrays the level-0 product reads; with and without the Lanczos bounds
    const void* key_setup[6] = {};
    int32_t code_setup = -1;
    int calls_setup[2] = {0, 0};
    cudaGraphExec_t setup[2] = {nullptr, nullptr};
    long long kernels_setup[2] = {0, 0};
    // PCG: moduli, b, x and the mesh arrays
    const void* key_pcg[7] = {};
    int32_t code_pcg = -1;
    int calls_pcg = 0;
    cudaGraphExec_t start = nullptr, loop = nullptr;
    long long kernels_start = 0, kernels_body = 0;

    void drop_setup() {
        for (int i = 0; i < 2; ++i) {
            if (setup[i]) cudaGraphExecDestroy(setup[i]);
            setup[i] = nullptr;
            calls_setup[i] = 0;
        }
    }
    void drop_pcg() {
        if (start) cudaGraphExecDestroy(start);
        if (loop) cudaGraphExecDestroy(loop);
        start = loop = nullptr;
    }
    ~MgGraphs() {
        drop_setup();
        drop_pcg();
        if (capture) cudaStreamDestroy(capture);
    }
};

static bool same_key(const void* const* a, const void* const* b, int n) {
    for (int i = 0; i < n; ++i)
        if (a[i] != b[i]) return false;
    return true;
}

// the device part of a set-up: coarse operators, coarsest inverse, Lanczos coefficients into mg->lhist
static int setup_device_part(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                             const double* diag, cudaStream_t s, bool lanczos) {
    int rc;
    const int L = mg->n_levels;
    if ((rc = check_cuda(cudaMemsetAsync(dot_ticket(mg->dot_work), 0, sizeof(unsigned), s), "cudaMemsetAsync")) ||
        (rc = check_cuda(cudaMemcpyAsync(mg->level[0].diag, diag, mg->level[0].n * sizeof(double), cudaMemcpyDeviceToDevice, s),
                         "cudaMemcpyAsync")))
        return rc;
    for (int l = 1; l < L; ++l) {
        const int32_t* gn;
        const uint8_t* ffix;
        transfer_args(mesh, mg, l - 1, &gn, &ffix);
        if ((rc = dfea_mg_restrict(&mg->level[l - 1].grid, &mg->level[l].grid, gn, ffix, nullptr, nullptr,
                                   mg->level[l].grid.fix, s)))
            return rc;
        rc = l == 1 ? dfea_mg_galerkin_fe(mesh, moduli, moduli_dtype, mg->node_ij, mg->cell_slot, mg->span,
                                          &mg->level[0].grid, &mg->level[1].grid, s)
                    : dfea_mg_galerkin(&mg->level[l - 1].grid, &mg->level[l].grid, s);
        if (rc || (rc = dfea_mg_diag(&mg->level[l].grid, mg->level[l].diag, s))) return rc;
    }
    if ((rc = dfea_mg_dense_inverse(&mg->level[L - 1].grid, mg->dense_work, mg->Ainv, s))) return rc;
    if (!lanczos) return DFEA_OK;
    // Lanczos on every smoothed level (p in x, z in d): the small levels in one block, the others in lockstep
    const int t = tail_start(mg) < L - 1 ? tail_start(mg) : L - 1;
    if (t < L - 1) {
        MgLanczosTail T = {};
        T.n_levels = L - 1 - t;
        T.steps = mg->lanczos_steps;
        for (int k = 0; k < T.n_levels; ++k) {
            const dfea_mg_level& lv = mg->level[t + k];
            T.lv[k] = MgLanczosLevel{mg_grid(lv.grid), (int)lv.n, lv.diag, lv.r, lv.d, lv.x, lv.q, mg->lscal + 4 * (t + k),
                                     mg->lhist + (int64_t)2 * mg->lanczos_steps * (t + k)};
        }
        k_mg_tail_lanczos<<<1, kMgTailLanczosThreads, 0, s>>>(T);
        note_launches(1);
        if ((rc = launch_check("dfea_mg_setup: Lanczos of the small levels"))) return rc;
    }
    for (int l = 0; l < t; ++l) {
        const dfea_mg_level& lv = mg->level[l];
        k_mg_start<<<grid_for(lv.n, kThreads, 8), kThreads, 0, s>>>(lv.n, lv.r);
        k_mg_div<<<grid_for(lv.n, kThreads, 8), kThreads, 0, s>>>(lv.n, lv.r, lv.diag, lv.d);
        note_launches(2);
        if ((rc = check_cuda(cudaMemcpyAsync(lv.x, lv.d, lv.n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync")) ||
            (rc = mg_dot1(lv.n, lv.r, lv.d, mg->lscal + 4 * l + 1, mg->dot_work, s)))
            return rc;
    }
    for (int k = 0; k < mg->lanczos_steps; ++k)
        for (int l = 0; l < t; ++l) {
            const dfea_mg_level& lv = mg->level[l];
            if ((rc = mg_apply(mesh, mg, moduli, moduli_dtype, l, lv.x, lv.q, s)) ||
                (rc = mg_lanczos_step1(lv.n, lv.x, lv.q, lv.r, lv.d, lv.diag, mg->lscal + 4 * l,
                                       mg->lhist + (int64_t)2 * mg->lanczos_steps * l, k, mg->dot_work, s)))
                return rc;
        }
    return DFEA_OK;
}

// Capture `body(stream)` into a new graph on the hierarchy's capture stream and instantiate it; the kernels
// the body notes while capturing are not launches yet (they are counted per replay instead).
template <typename F>
static int capture_exec(MgGraphs* g, F&& body, cudaGraphExec_t* out, long long* kernels) {
    int rc;
    if (!g->capture && (rc = check_cuda(cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking), "cudaStreamCreate")))
        return rc;
    const long long before = thread_launch_count();
    if ((rc = check_cuda(cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")))
        return rc;
    rc = body(g->capture);
    cudaGraph_t graph = nullptr;
    const int rc_end = check_cuda(cudaStreamEndCapture(g->capture, &graph), "cudaStreamEndCapture");
    *kernels = thread_launch_count() - before;
    note_launches(-*kernels);
    if (!rc && !rc_end) rc = check_cuda(cudaGraphInstantiate(out, graph, 0), "cudaGraphInstantiate");
    if (graph) cudaGraphDestroy(graph);
    return rc ? rc : rc_end;
}

__global__ void k_mgp_init(MgPcgState* st, double rtol, int max_iter) {
    st->rtol2 = rtol * rtol;
    st->max_iter = max_iter;
    st->k = 0;
    st->iters = 0;
    st->guard = 0;
    st->status = DFEA_PCG_RUNNING;
}

// after |b|^2: the tolerance, and the ends that need no iteration
__global__ void k_mgp_check(MgPcgState* st) {
    st->tol2 = st->rtol2 * st->nb2;
    if (st->nb2 == 0.0) {
        st->status = DFEA_PCG_ZERO_RHS;
    } else if (st->max_iter <= 0) {
        st->status = DFEA_PCG_MAX_ITER;
        st->iters = st->max_iter;
    }
}

// x += alpha p, r -= alpha q (alpha = rz / p.q); on p.q <= 0 only x = z at the first iteration
__global__ void k_mgp_update(int64_t n, const MgPcgState* __restrict__ st, double* __restrict__ x, double* __restrict__ r,
                             const double* __restrict__ p, const double* __restrict__ q, const double* __restrict__ z) {
    if (st->status != DFEA_PCG_RUNNING) return;
    const double curv = st->curv;
    if (!(curv > 0.0)) {
        if (st->k == 0)
            for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
                x[i] = z[i];
        return;
    }
    const double alpha = st->rz / curv, neg = -alpha;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        r[i] += neg * q[i];
    }
}

// p = z + (r.z_new / r.z) p while the solve goes on
__global__ void k_mgp_direction(int64_t n, const MgPcgState* __restrict__ st, double* __restrict__ p,
                                const double* __restrict__ z) {
    if (st->status != DFEA_PCG_RUNNING || !(st->curv > 0.0) || st->rr <= st->tol2) return;
    const double beta = st->rz_new / st->rz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// end of an iteration: the status, the counters and the loop condition.  The loop runs at most
// max_iter + 4 bodies whatever the numbers do.
__global__ void k_mgp_end(MgPcgState* st, cudaGraphConditionalHandle cond) {
    st->guard += 1;
    if (st->status == DFEA_PCG_RUNNING) {
        if (!(st->curv > 0.0)) {
            st->status = DFEA_PCG_NEG_CURV;
            st->iters = st->k;
        } else if (st->rr <= st->tol2) {
            st->status = DFEA_PCG_CONVERGED;
            st->iters = st->k + 1;
        } else {
            st->rz = st->rz_new;
            st->k += 1;
            if (st->k >= st->max_iter) {
                st->status = DFEA_PCG_MAX_ITER;
                st->iters = st->max_iter;
            }
        }
    }
    cudaGraphSetConditional(cond, (st->status == DFEA_PCG_RUNNING && st->guard < st->max_iter + 4) ? 1u : 0u);
}

__global__ void k_mgp_begin(const MgPcgState* st, cudaGraphConditionalHandle cond) {
    cudaGraphSetConditional(cond, st->status == DFEA_PCG_RUNNING ? 1u : 0u);
}

// start of a solve: x = 0, r = b, |b|^2, z = V(r), p = z, r.z
static int pcg_start_part(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t code,
                          const double* b, double* x, cudaStream_t s) {
    const int64_t n = mg->level[0].n;
    double *r = mg->pcg, *z = mg->pcg + n, *p = mg->pcg + 2 * n;
    MgPcgState* st = reinterpret_cast<MgPcgState*>(mg->pcg_state);
    int rc;
    if ((rc = check_cuda(cudaMemsetAsync(x, 0, n * sizeof(double), s), "cudaMemsetAsync")) ||
        (rc = check_cuda(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync")) ||
        (rc = mg_dot1(n, b, b, &st->nb2, mg->dot_work, s)))
        return rc;
    k_mgp_check<<<1, 1, 0, s>>>(st);
    note_launches(1);
    if ((rc = launch_check("dfea_mg_pcg: check")) || (rc = mg_vcycle(mesh, mg, moduli, code, 0, r, z, s)) ||
        (rc = check_cuda(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync")))
        return rc;
    return mg_dot1(n, r, z, &st->rz, mg->dot_work, s);
}

// one iteration of the device-side loop
static int pcg_body_part(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t code, double* x,
                         cudaGraphConditionalHandle cond, cudaStream_t s) {
    const int64_t n = mg->level[0].n;
    double *r = mg->pcg, *z = mg->pcg + n, *p = mg->pcg + 2 * n, *q = mg->pcg + 3 * n;
    MgPcgState* st = reinterpret_cast<MgPcgState*>(mg->pcg_state);
    int rc;
    if ((rc = mg_apply(mesh, mg, moduli, code, 0, p, q, s)) || (rc = mg_dot1(n, p, q, &st->curv, mg->dot_work, s)))
        return rc;
    k_mgp_update<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(n, st, x, r, p, q, z);
    note_launches(1);
    if ((rc = launch_check("dfea_mg_pcg: update")) || (rc = mg_dot1(n, r, r, &st->rr, mg->dot_work, s)) ||
        (rc = mg_vcycle(mesh, mg, moduli, code, 0, r, z, s)) || (rc = mg_dot1(n, r, z, &st->rz_new, mg->dot_work, s)))
        return rc;
    k_mgp_direction<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(n, st, p, z);
    k_mgp_end<<<1, 1, 0, s>>>(st, cond);
    note_launches(2);
    return launch_check("dfea_mg_pcg: end");
}

// the loop graph: a node that sets the condition from the status, then a while node around one iteration
static int build_loop_graph(MgGraphs* g, const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli,
                            int32_t code, double* x) {
    int rc;
    if (!g->capture && (rc = check_cuda(cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking), "cudaStreamCreate")))
        return rc;
    cudaGraph_t graph = nullptr;
    if ((rc = check_cuda(cudaGraphCreate(&graph, 0), "cudaGraphCreate"))) return rc;
    auto fail = [&](int code_) {
        cudaGraphDestroy(graph);
        return code_;
    };
    cudaGraphConditionalHandle cond;
    if ((rc = check_cuda(cudaGraphConditionalHandleCreate(&cond, graph, 0u, cudaGraphCondAssignDefault),
                         "cudaGraphConditionalHandleCreate")))
        return fail(rc);
    MgPcgState* st = reinterpret_cast<MgPcgState*>(mg->pcg_state);
    if ((rc = check_cuda(cudaStreamBeginCaptureToGraph(g->capture, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                         "cudaStreamBeginCaptureToGraph")))
        return fail(rc);
    k_mgp_begin<<<1, 1, 0, g->capture>>>(st, cond);
    rc = launch_check("dfea_mg_pcg: begin");
    cudaGraph_t cap = graph;
    int rc_end = check_cuda(cudaStreamEndCapture(g->capture, &cap), "cudaStreamEndCapture");
    if (rc || rc_end) return fail(rc ? rc : rc_end);
    cudaGraphNode_t first = nullptr;
    size_t n_nodes = 1;
    if ((rc = check_cuda(cudaGraphGetNodes(graph, &first, &n_nodes), "cudaGraphGetNodes"))) return fail(rc);
    if (n_nodes != 1) return fail(set_error(DFEA_ERR_CUDA, "dfea_mg_pcg: unexpected loop-graph prologue"));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((rc = check_cuda(cudaGraphAddNode(&node, graph, &first, 1, &cp), "cudaGraphAddNode(while)"))) return fail(rc);
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const long long before = thread_launch_count();
    if ((rc = check_cuda(cudaStreamBeginCaptureToGraph(g->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                         "cudaStreamBeginCaptureToGraph")))
        return fail(rc);
    rc = pcg_body_part(mesh, mg, moduli, code, x, cond, g->capture);
    cudaGraph_t body_cap = body;
    rc_end = check_cuda(cudaStreamEndCapture(g->capture, &body_cap), "cudaStreamEndCapture");
    g->kernels_body = thread_launch_count() - before;
    note_launches(-g->kernels_body);
    if (rc || rc_end) return fail(rc ? rc : rc_end);
    rc = check_cuda(cudaGraphInstantiate(&g->loop, graph, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(graph);
    return rc;
}

// graph-driven PCG: init kernel, start graph, loop graph, one status read
static int pcg_graph_solve(MgGraphs* g, const dfea_mg* mg, double rtol, int32_t max_iter, int32_t* iterations,
                           int32_t* status, cudaStream_t s) {
    MgPcgState* st = reinterpret_cast<MgPcgState*>(mg->pcg_state);
    k_mgp_init<<<1, 1, 0, s>>>(st, rtol, max_iter);
    int rc = launch_check("dfea_mg_pcg: init");
    if (rc || (rc = check_cuda(cudaGraphLaunch(g->start, s), "cudaGraphLaunch")) ||
        (rc = check_cuda(cudaGraphLaunch(g->loop, s), "cudaGraphLaunch")))
        return rc;
    int32_t host[5];  // k, max_iter, status, iters, guard
    if ((rc = read_to_host(host, &st->k, sizeof(host), s))) return rc;
    note_launches(2 + g->kernels_start + (long long)host[4] * g->kernels_body);
    if (host[2] == DFEA_PCG_RUNNING) return set_error(DFEA_ERR_INVALID, "dfea_mg_pcg: the device loop ended without a status");
    *status = host[2];
    *iterations = host[3];
    return DFEA_OK;
}

}  // namespace dfea

extern "C" int dfea_mg_setup(const dfea_mesh_view* mesh, dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                             const double* diag, void* stream) {
    int rc = validate_mg(mesh, mg, "dfea_mg_setup");
    if (rc) return rc;
    if (!moduli || !diag) return set_error(DFEA_ERR_INVALID, "dfea_mg_setup: NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int L = mg->n_levels;
    // the smoother bounds: estimated now, or kept from an earlier set-up of this hierarchy
    const bool lanczos = mg->bounds_every <= 0 || mg->setups <= 0 || (mg->setups % mg->bounds_every) == 0;
    mg->setups = mg->setups < 0 ? 1 : mg->setups + 1;
    if (mg->pcg_state) {
        if (!mg->graphs) {
            MgGraphs* g = new (std::nothrow) MgGraphs;
            if (!g) return set_error(DFEA_ERR_INVALID, "dfea_mg_setup: out of host memory");
            mg->graphs = g;
        }
        MgGraphs* g = static_cast<MgGraphs*>(mg->graphs);
        const void* key[6] = {moduli, diag, mesh->conn, mesh->grad, mesh->grad32, mesh->jinv};
        if (!same_key(key, g->key_setup, 6) || g->code_setup != moduli_dtype) {
            g->drop_setup();
            for (int i = 0; i < 6; ++i) g->key_setup[i] = key[i];
            g->code_setup = moduli_dtype;
        }
        const int v = lanczos ? 1 : 0;
        if (g->calls_setup[v]++ == 0) {
            rc = setup_device_part(mesh, mg, moduli, moduli_dtype, diag, s, lanczos);   // direct, the first time
        } else {
            if (!g->setup[v] &&
                (rc = capture_exec(g, [&](cudaStream_t cs) { return setup_device_part(mesh, mg, moduli, moduli_dtype, diag, cs, lanczos); },
                                   &g->setup[v], &g->kernels_setup[v])))
                return rc;
            rc = check_cuda(cudaGraphLaunch(g->setup[v], s), "cudaGraphLaunch");
            note_launches(g->kernels_setup[v]);
        }
    } else {
        rc = setup_device_part(mesh, mg, moduli, moduli_dtype, diag, s, lanczos);
    }
    if (rc) return rc;
    if (!lanczos) return DFEA_OK;   // bounds, coefficients and lam[] of the last estimate stay in force
    const int nh = 2 * mg->lanczos_steps * (L - 1);
    double hist[2 * 64 * DFEA_MG_MAX_LEVELS];
    if ((rc = read_scalars(hist, mg->lhist, nh, s))) return rc;
    double coef[DFEA_MG_MAX_LEVELS * 2 * DFEA_MG_MAX_DEGREE] = {0.0};
    for (int l = 0; l < L - 1; ++l) {
        const double lam = ritz_max(hist + 2 * mg->lanczos_steps * l, mg->lanczos_steps);
        mg->lam[l] = lam;
        const double hi = 1.1 * lam, lo = hi / mg->ratio;
        const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
        double rho = 1.0 / sigma;
        double* row = coef + l * 2 * DFEA_MG_MAX_DEGREE;
        row[0] = 1.0 / theta;
        for (int k = 1; k < mg->degree; ++k) {
            const double rho_new = 1.0 / (2.0 * sigma - rho);
            row[1 + 2 * (k - 1)] = rho_new * rho;
            row[2 + 2 * (k - 1)] = 2.0 * rho_new / delta;
            rho = rho_new;
        }
    }
    if ((rc = check_cuda(cudaMemcpyAsync(mg->coef, coef, sizeof(double) * 2 * DFEA_MG_MAX_DEGREE * (L - 1),
                                         cudaMemcpyHostToDevice, s), "cudaMemcpyAsync")))
        return rc;
    // the copy reads a stack array: it has completed when the stream has
    return check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
}

extern "C" int dfea_mg_release(dfea_mg* mg) {
    if (mg && mg->graphs) {
        delete static_cast<MgGraphs*>(mg->graphs);
        mg->graphs = nullptr;
    }
    return DFEA_OK;
}

extern "C" double dfea_mg_lanczos_bound(const double* hist, int32_t steps) {
    if (!hist || steps < 1 || steps > 64) return -1.0;
    return ritz_max(hist, steps);
}

extern "C" int dfea_mg_vcycle(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                              const double* r, double* z, void* stream) {
    int rc = validate_mg(mesh, mg, "dfea_mg_vcycle");
    if (rc) return rc;
    if (!moduli || !r || !z) return set_error(DFEA_ERR_INVALID, "dfea_mg_vcycle: NULL pointer");
    return mg_vcycle(mesh, mg, moduli, moduli_dtype, 0, r, z, static_cast<cudaStream_t>(stream));
}

extern "C" int dfea_mg_pcg(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                           const double* b, double* x, double rtol, int32_t max_iter, int32_t* iterations,
                           int32_t* status, void* stream) {
    int rc = validate_mg(mesh, mg, "dfea_mg_pcg");
    if (rc) return rc;
    if (!moduli || !b || !x || !iterations || !status || max_iter < 0)
        return set_error(DFEA_ERR_INVALID, "dfea_mg_pcg: bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mg->pcg_state && mg->graphs) {
        // graph-driven: the second solve with the same buffers captures the loop, later ones replay it
        MgGraphs* g = static_cast<MgGraphs*>(mg->graphs);
        const void* key[7] = {moduli, b, x, mesh->conn, mesh->grad, mesh->grad32, mesh->jinv};
        if (!same_key(key, g->key_pcg, 7) || g->code_pcg != moduli_dtype) {
            g->drop_pcg();
            for (int i = 0; i < 7; ++i) g->key_pcg[i] = key[i];
            g->code_pcg = moduli_dtype;
            g->calls_pcg = 0;
        }
        if (g->calls_pcg++ > 0) {
            if (!g->start) {
                rc = capture_exec(g, [&](cudaStream_t cs) { return pcg_start_part(mesh, mg, moduli, moduli_dtype, b, x, cs); },
                                  &g->start, &g->kernels_start);
                if (!rc) rc = build_loop_graph(g, mesh, mg, moduli, moduli_dtype, x);
                if (rc) {
                    g->drop_pcg();
                    return rc;
                }
            }
            return pcg_graph_solve(g, mg, rtol, max_iter, iterations, status, s);
        }
    }
    const int64_t n = mg->level[0].n;
    double *r = mg->pcg, *z = mg->pcg + n, *p = mg->pcg + 2 * n, *q = mg->pcg + 3 * n;
    double h[1];
    auto dot = [&](const double* u, const double* v, double* out) -> int {
        int e = mg_dot1(n, u, v, mg->scal, mg->dot_work, s);
        return e ? e : read_scalars(out, mg->scal, 1, s);
    };
    *iterations = 0;
    if ((rc = check_cuda(cudaMemsetAsync(x, 0, n * sizeof(double), s), "cudaMemsetAsync")) ||
        (rc = check_cuda(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync")) ||
        (rc = dot(b, b, h)))
        return rc;
    const double nb2 = h[0];
    if (nb2 == 0.0) {
        *status = DFEA_PCG_ZERO_RHS;
        return DFEA_OK;
    }
    const double tol2 = rtol * rtol * nb2;
    if ((rc = mg_vcycle(mesh, mg, moduli, moduli_dtype, 0, r, z, s)) ||
        (rc = check_cuda(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync")) ||
        (rc = dot(r, z, h)))
        return rc;
    double rz = h[0];
    for (int k = 0; k < max_iter; ++k) {
        if ((rc = mg_apply(mesh, mg, moduli, moduli_dtype, 0, p, q, s)) || (rc = dot(p, q, h))) return rc;
        const double curv = h[0];
        if (!(curv > 0.0)) {
            if (k == 0)
                rc = check_cuda(cudaMemcpyAsync(x, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
            *iterations = k;
            *status = DFEA_PCG_NEG_CURV;
            return rc;
        }
        const double alpha = rz / curv;
        const int nb = mg_dot_blocks(n);
        k_mg_update_rr<<<nb, kMgDotThreads, 0, s>>>(n, alpha, -alpha, p, q, x, r, mg->dot_work, mg->scal);
        note_launches(1);
        if ((rc = launch_check("dfea_mg_pcg: update")) || (rc = read_scalars(h, mg->scal, 1, s))) return rc;
        if (h[0] <= tol2) {
            *iterations = k + 1;
            *status = DFEA_PCG_CONVERGED;
            return DFEA_OK;
        }
        if ((rc = mg_vcycle(mesh, mg, moduli, moduli_dtype, 0, r, z, s)) || (rc = dot(r, z, h))) return rc;
        const double rz_new = h[0];
        if ((rc = dfea_add_scaled(n, z, rz_new / rz, p, p, s))) return rc;
        rz = rz_new;
    }
    *iterations = max_iter;
    *status = DFEA_PCG_MAX_ITER;
    return DFEA_OK;
}
