/*
 * difffea_b200.h -- C ABI of the B200 (sm_100a) matrix-free Newton-Krylov kernels.
 *
 * Every entry point takes plain pointers and sizes; device pointers point to memory the caller
 * owns (the Python host layer passes torch tensors from the caching allocator).  Nothing here
 * allocates device memory: scratch space for reductions and Krylov vectors is a caller buffer
 * whose size the matching *_work_bytes query returns.  Streams are passed as `void*`
 * (a cudaStream_t); every launch is asynchronous on that stream unless the comment says otherwise.
 *
 * Return value: DFEA_OK (0) or one of the DFEA_ERR_* codes below; dfea_last_error() gives a
 * human-readable message for the calling thread.
 *
 * Layouts (all "SoA": the element index runs fastest so that a warp reads 32 consecutive elements):
 *   stride             element stride of every per-element row, a multiple of 32 that is >= n_el
 *   conn   int32       [nen][stride]   node << 2 | fix bits (bit 0: x DOF fixed, bit 1: y DOF fixed)
 *   orig   int32       [stride]        original (reference) element id of a colour-sorted slot
 *   grad   f64 (f32)   [n_q][nen][stride][2]  (dN_a/dX, dN_a/dY) at Gauss point q
 *   wdet   f64         [n_q][stride]   Gauss weight * det(dX/dxi)
 *   moduli f64         [n_q][8][stride][2]   entry pair k holds C[2k], C[2k+1] of the row-major 4x4
 *          f32         [n_q][4][stride][4]   row r holds C[4r .. 4r+3]
 *   vectors            (2 * n_nodes) node-major DOF vectors, dof = 2 * node + component,
 *                      as in the reference (boundary_conditions.py:171-179)
 * Elements are stored sorted by colour: no two elements of one colour share a node, so the
 * scatter of one colour needs neither atomics nor a fixed summation order to be deterministic.
 */
#ifndef DIFFFEA_B200_H
#define DIFFFEA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFEA_OK 0
#define DFEA_ERR_INVALID 1     /* a size, pointer or option is out of range */
#define DFEA_ERR_UNSUPPORTED 2 /* (nen, n_q) pair of an element type the library does not build */
#define DFEA_ERR_CUDA 3        /* a CUDA call failed; dfea_last_error() has the CUDA message */
#define DFEA_ERR_COLOURS 4     /* the element graph needs more than DFEA_MAX_COLOURS colours */

#define DFEA_F64 0
#define DFEA_F32 1
#define DFEA_MIXED 2  /* PCG only: FP32 moduli and gradients (the operator), FP64 Krylov vectors */
/* Moduli in the element's reference frame, FP32, symmetric (10 entries per Gauss point):
 * Chat_(i a),(k b) = sum_{J,L} Jinv_aJ C_(iJ),(kL) Jinv_bL with Jinv = (dX/dxi)^-1, so that the product
 * needs the fixed reference shape gradients only (mesh->ref_grad), not the per-element dN/dX.
 * Layout per Gauss point q: float4 [stride] (entries 00 01 02 03), float4 [stride] (11 12 13 22),
 * float2 [stride] (23 33), i.e. 10 * stride floats per q.  As a moduli dtype (dfea_qp_moduli,
 * dfea_tangent_apply[_gather] with f64 vectors) and as a PCG vec_dtype (FP64 Krylov vectors). */
#define DFEA_F32REF 3
#define DFEA_MAX_NEN 9
#define DFEA_MAX_NQ 9

#define DFEA_MAX_COLOURS 64

/* Status words of the device-resident PCG (dfea_pcg_solve). */
#define DFEA_PCG_RUNNING 0
#define DFEA_PCG_CONVERGED 1   /* ||r|| <= rtol ||b||                                  */
#define DFEA_PCG_MAX_ITER 2    /* max_iter iterations without convergence             */
#define DFEA_PCG_NEG_CURV 3    /* p.Ap <= 0: the operator is not SPD along p           */
#define DFEA_PCG_ZERO_RHS 4    /* ||b|| == 0: x = 0 after zero iterations              */

#define DFEA_PCG_GATHER 16     /* dfea_pcg_create flag: gather form of the product     */
#define DFEA_PCG_BLOCK_JACOBI 32 /* dfea_pcg_create flag: nodal block-Jacobi; diag = the
                                  * inverse 2x2 blocks of dfea_qp_moduli_block (4N f64) */
#define DFEA_PCG_FUSED 64      /* dfea_pcg_create flag: fused gather form, 2 kernels per iteration
                                * (implies DFEA_PCG_GATHER) */
/* dfea_pcg_create option: at most n blocks per launch (n < 2^23; 0 = as many as the GPU holds at
 * once).  For solves that share the GPU with solves on other streams. */
#define DFEA_PCG_MAX_BLOCKS(n) ((int32_t)(n) << 8)

/*
 * Material models of the reference's library (materials.py:65-186, MATERIAL_LIBRARY at :164-186), with
 * the parameter order of its param_names.  Every model is an energy psi3(F3, p) of the plane-strain
 * embedding F3 = [[F, 0], [0, 1]]; neo-Hookean is evaluated in closed form, the others by forward-mode
 * differentiation of their energy on the device.
 */
#define DFEA_MAT_NEO_HOOKEAN 0      /* p = (mu, lambda)                                      */
#define DFEA_MAT_MOONEY_RIVLIN 1    /* p = (c10, c01, kappa)                                 */
#define DFEA_MAT_SAINT_VENANT 2     /* p = (mu, lambda)                                      */
#define DFEA_MAT_DEMIRAY 3          /* p = (mu, gamma, lambda)                               */
#define DFEA_MAT_FIBER_REINFORCED 4 /* p = (mu, lambda, k1, k2, beta_deg, d, second_family)  */
#define DFEA_MAX_MAT_PARAMS 8

/* A material (host struct, passed by pointer): the problem's material, mat_p and mat_scalable. */
typedef struct dfea_material {
    int32_t model;                 /* DFEA_MAT_*                                                  */
    uint32_t scalable;             /* bit k set: the design field theta_e scales p[k] per element */
    double p[DFEA_MAX_MAT_PARAMS]; /* nominal parameters p0; entries past the model's count unused */
} dfea_material;

/* A mesh in device memory, colour-sorted.  Sizes are host values, pointers are device pointers. */
typedef struct dfea_mesh_view {
    int64_t n_el;        /* number of elements                                           */
    int64_t stride;      /* element stride of every SoA row (multiple of 32, >= n_el)     */
    int64_t n_nodes;     /* number of nodes N; DOF vectors have 2N entries                */
    int32_t nen;         /* nodes per element                                             */
    int32_t n_q;         /* Gauss points per element                                      */
    int32_t n_colours;   /* number of colour classes                                      */
    int32_t reserved;
    int64_t colour_begin[DFEA_MAX_COLOURS + 1]; /* elements [colour_begin[c], colour_begin[c+1]) */
    const int32_t* conn;     /* [nen][stride]                                              */
    const int32_t* orig;     /* [stride]                                                   */
    const double* grad;      /* [n_q][nen][stride][2]                                      */
    const double* wdet;      /* [n_q][stride]                                              */
    const float* grad32;     /* optional FP32 copy of grad (NULL if not built)              */
    const uint8_t* node_fix; /* [n_nodes] fix bits of every node                           */
    /* Optional node -> element incidence for the gather form of the product (NULL if not built):
     * the slots of node n are node_elem[node_elem_ptr[n] .. node_elem_ptr[n+1]), each the index
     * a * stride + e of local node a of (packed) element e, in increasing order. */
    const int32_t* node_elem_ptr; /* [n_nodes + 1]                                           */
    const int32_t* node_elem;     /* [n_el * nen]                                            */
    /* Optional, for DFEA_F32REF moduli: inverse element Jacobians [n_q][2][stride] (rows of
     * Jinv as f64 pairs, NULL if not built) and the reference shape gradients at the Gauss points,
     * ref_grad[(q * nen + a) * 2 + alpha] = dN_a/dxi_alpha (host values). */
    const double* jinv;
    double ref_grad[DFEA_MAX_NQ * DFEA_MAX_NEN * 2];
} dfea_mesh_view;

/* ---------------------------------------------------------------- library --------------------- */

/* Message of the last error of the calling thread (static storage, never NULL). */
const char* dfea_last_error(void);

/* Library version as major * 10000 + minor * 100 + patch. */
int dfea_version(void);

/* Number of kernels this library has launched in the process so far (kernels run by a captured
 * PCG graph are added when its solve returns).  A diagnostic for benchmarks. */
int64_t dfea_launch_count(void);

/* Blocking synchronisation (cudaDeviceScheduleBlockingSync, on != 0) or the default heuristic (on == 0)
 * for this process's context on `device`: with blocking, host threads waiting for the GPU sleep instead of
 * spinning.  For processes that run many host threads per GPU (the serving engine).  A per-process
 * setting of this process's context, gone with the process. */
int dfea_set_blocking_sync(int32_t device, int32_t on);


/* sizeof of a public struct of this header, by its type name ("dfea_mesh_view", "dfea_material", "dfea_mg_grid",
 * "dfea_mg_level", "dfea_mg", "dfea_newton", "dfea_newton_record", "dfea_newton_info"); -1 for other names.
 * Host function: lets a binding check its mirrors of these structs against the library's layout. */
int64_t dfea_struct_size(const char* name);

/* 1 if the (nen, n_q) pair is built: (3,1) tri3, (6,6) tri6, (4,4) quad4, (8,9) quad8, (9,9) quad9. */
int dfea_element_supported(int32_t nen, int32_t n_q);

/* ---------------------------------------------------------------- mesh set-up ----------------- */

/*
 * Greedy element colouring (host function, host pointers).  conn is the reference connectivity
 * (n_el, nen) int64 (problem.py:180-190 `conn`).  On return colour[e] in [0, *n_colours) and no
 * two elements that share a node have the same colour.  Elements are visited in id order; each
 * takes the smallest colour unused at its nodes, which gives 4 colours on structured Q4/Q8/Q9 grids.
 */
int dfea_colour_elements(const int64_t* conn, int64_t n_el, int32_t nen, int64_t n_nodes,
                         int32_t* colour, int32_t* n_colours);

/*
 * Copy the reference-layout mesh arrays (device pointers) into the colour-sorted SoA layout of a
 * dfea_mesh_view.  perm[s] = original element id stored in slot s (n_el entries).  dN_dX is
 * (n_el, n_q, nen, 2) and w_detJ (n_el, n_q), as precompute_geometry returns them
 * (operators.py:85-120); m is the (2N) Dirichlet mask of 0.0/1.0 entries (operators.py:29).
 * Outputs: conn_out [nen][stride], orig_out [stride], grad_out [n_q][nen][stride][2],
 * wdet_out [n_q][stride], node_fix_out [n_nodes].
 */
int dfea_mesh_pack(int64_t n_el, int64_t stride, int32_t nen, int32_t n_q, int64_t n_nodes,
                   const int64_t* perm, const int64_t* conn_ref, const double* dN_dX,
                   const double* w_detJ, const double* m, int32_t* conn_out, int32_t* orig_out,
                   double* grad_out, double* wdet_out, uint8_t* node_fix_out, void* stream);

/* FP32 copy of the packed gradients (the geometry of the FP32 inner operator). */
int dfea_mesh_grad_to_f32(const dfea_mesh_view* mesh, float* grad32_out, void* stream);

/*
 * Inverse element Jacobians of the reference-frame FP32 operator (DFEA_F32REF), from the packed mesh and
 * the node coordinates nodes (n_nodes, 2) float64 (problem.py `nodes`): jinv_out [n_q][2][stride][2]
 * (row r of Jinv at Gauss point q as an f64 pair; zeros in the padding slots), 16-byte aligned.  check (2
 * doubles) receives the largest |Jinv^T dN/dxi - dN/dX| and the largest |dN/dX| over the mesh: the caller
 * accepts the problem's geometry when the first is within a tolerance of the second (the reference
 * derives dN/dX the same way, operators.py:85-120).  No counterpart function in the reference.
 */
int dfea_mesh_ref_frame(const dfea_mesh_view* mesh, const double* nodes, double* jinv_out, double* check,
                        void* stream);

/*
 * Node incidence of the gather form (the node_elem_ptr / node_elem arrays of dfea_mesh_view): ptr_out
 * [n_nodes + 1] and inc_out [nen * n_el], the slots a * stride + e of each node in increasing order; work is
 * n_nodes int32 of scratch.  Exact (integer counting, a scan and per-node sorts), so the same each time.
 * No counterpart function in the reference (its products scatter through torch index_add, operators.py:385-412).
 */
int dfea_mesh_node_incidence(const dfea_mesh_view* mesh, int32_t* ptr_out, int32_t* inc_out, int32_t* work,
                             void* stream);

/*
 * The problem of a serving request, written on the device: a structured rectangle [0, width] x [0, height]
 * of nx x ny Q4 (nen 4) or Q9 (nen 9) cells, both displacement components fixed on x = 0, a uniform traction
 * of total (load_x, load_y) on x = width -- the arrays problem.build_rectangle_problem builds (the
 * reference's rectangle mesher, boundary conditions and precompute_geometry, problem.py:115-194 and
 * operators.py:85-120): nodes (N, 2), conn (n_el, nen) int64 in the mesher's numbering, dN_dX
 * (n_el, n_q, nen, 2), w_detJ (n_el, n_q), f, m and u_D (2N), fixed (2N bytes 0/1).  The reference gradients,
 * Gauss weights and the 3-point edge rule come from the caller.  No counterpart function in the reference.
 */
typedef struct {
    int32_t nen;                                        /* 4 or 9 */
    int32_t n_q;                                        /* Gauss points per element */
    int32_t nx, ny;                                     /* cells */
    double width, height;
    double load_x, load_y;                              /* total traction force on x = width */
    double ref_grad[DFEA_MAX_NQ * DFEA_MAX_NEN * 2];    /* dN_a/dxi_alpha at the Gauss points, [q][a][alpha] */
    double gauss_w[DFEA_MAX_NQ];                        /* Gauss weights */
    double edge_s[3], edge_w[3];                        /* the edge rule on [-1, 1] */
} dfea_rect_spec;

int dfea_build_rectangle(const dfea_rect_spec* spec, double* nodes, int64_t* conn, double* dN_dX, double* w_detJ,
                         double* f, double* m, uint8_t* fixed, double* u_D, void* stream);

/* The same arrays computed on the host into host memory (a problem submitted from host memory). */
int dfea_build_rectangle_host(const dfea_rect_spec* spec, double* nodes, int64_t* conn, double* dN_dX, double* w_detJ,
                              double* f, double* m, uint8_t* fixed, double* u_D);

/* ---------------------------------------------------------------- kernels (a), (b) ------------ */

/*
 * Kernel (a): Gauss-point tangent moduli and Jacobi diagonal at state u.
 * Replaces `_qp_setup` (operators.py:316-342) and `compute_jacobi_diagonal` (operators.py:477-556):
 *   F = I + sum_a u_a (x) dN_a,  C[(iJ),(kL)] = w detJ d2psi/dF_iJ dF_kL  (neo-Hookean, plane strain,
 *   materials.py:209-217 with mu = mu0 theta_e, lambda = lambda0 theta_e, materials.py:383-390),
 *   diag = where(m > 0, max(sum_e diag(K_e), 1e-6), 1).
 * theta is indexed by ORIGINAL element id.  moduli_dtype selects the moduli layout (DFEA_F64 or
 * DFEA_F32).  diag (2N, f64) is written; it may be NULL to skip the diagonal, and moduli may be NULL
 * to compute the diagonal alone (the Jacobi preconditioner of operators.py:562-570).
 */
int dfea_qp_moduli(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                   double lambda0, void* moduli, int32_t moduli_dtype, double* diag, void* stream);

/*
 * dfea_qp_moduli (and, with blocks != NULL, dfea_qp_moduli_block) for any material of the library:
 * p_e = p0 with the scalable entries times theta_e (materials.py:239-246), C = w detJ d2psi/dF2 of that
 * material's energy.  The (mu0, lambda0) entry points are these with the neo-Hookean material and
 * scalable = 0x3.
 */
int dfea_qp_moduli_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                       const dfea_material* material, void* moduli, int32_t moduli_dtype, double* diag,
                       double* blocks, void* stream);

/*
 * Kernel (b): y = m * J(u) (m * v) + (1 - m) * v from the stored moduli, i.e. the `qp`/`qp_ew`
 * tangent product (operators.py:345-412).  One fused gather-contract-scatter launch per colour;
 * no atomics.  vec_dtype selects f64 or f32 vectors; f32 moduli (with mesh->grad32 set) may be applied
 * to f64 vectors (arithmetic in f64) or f32 vectors; f32 vectors need f32 moduli.  y must not alias v.
 */
int dfea_tangent_apply(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype,
                       const void* v, void* y, int32_t vec_dtype, void* stream);

/* ---------------------------------------------------------------- residual, energy ------------ */

/* Bytes of the element-result buffer of the gather form: nen * stride pairs of vec_dtype. */
int64_t dfea_gather_work_bytes(const dfea_mesh_view* mesh, int32_t vec_dtype);

/*
 * dfea_qp_moduli plus the nodal block-Jacobi preconditioner (operators.py:586-625,
 * make_block_jacobi_preconditioner): blocks (4N f64, 16-byte aligned) receives per node the inverse of
 * B = M B_K M + (I - M) + 1e-12 I, B_K the 2x2 diagonal block of the tangent, as (Binv00, Binv01, Binv11,
 * 0); diag (2N) receives the Jacobi diagonal as in dfea_qp_moduli.  Both are required.
 */
int dfea_qp_moduli_block(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                         double lambda0, void* moduli, int32_t moduli_dtype, double* diag, double* blocks,
                         void* stream);

/*
 * The same product as dfea_tangent_apply in two passes instead of one pass per colour: every element
 * writes its f_e into fe_work (one launch over all elements), then every node sums its elements'
 * results in the fixed incidence order (mesh->node_elem_ptr / node_elem) and takes v on fixed DOFs.
 * Same operator and the same arithmetic per element; the per-node sums are grouped differently from
 * the colour order, so the two forms agree to rounding.  Two launches regardless of the colour count.
 * Replaces the same reference interface as dfea_tangent_apply (operators.py:385-412).
 */
int dfea_tangent_apply_gather(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype,
                              const void* v, void* y, int32_t vec_dtype, void* fe_work, void* stream);

/*
 * Post-processing (postprocess.py:70-118, compute_fields).  dfea_element_fields writes per element, in
 * ORIGINAL element order, 7 rows of n_el doubles: area (sum w detJ), and the w detJ-weighted averages of
 * J, sigma_xx, sigma_yy, sigma_xy, then von Mises from the averaged components (sigma_zz included),
 * then psi.  dfea_node_fields averages rows 1..6 of that output over each node's incident elements
 * (needs node_elem_ptr/node_elem): 6 rows of n_nodes doubles.
 */
int dfea_element_fields(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                        double lambda0, double* elem_out, void* stream);
int dfea_element_fields_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                            const dfea_material* material, double* elem_out, void* stream);
int dfea_node_fields(const dfea_mesh_view* mesh, const double* elem, double* node_out, void* stream);

/* Internal force at every DOF, constrained ones included (the support_reactions evaluation,
 * postprocess.py:121-137): R_int (2N) = sum_e f_e(u, theta). */
int dfea_internal_force(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                        double lambda0, double* R_int, void* stream);
int dfea_internal_force_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                            const dfea_material* material, double* R_int, void* stream);

/* Bytes of scratch that dfea_residual and dfea_vec_norm2 need for their reductions. */
int64_t dfea_reduce_work_bytes(const dfea_mesh_view* mesh);

/*
 * R = m * (R_int(u) - load_factor * f), R_int = scatter(sum_q w detJ P(F) dN)  (global_residual,
 * operators.py:159-220).  If out_norm2 is not NULL, *out_norm2 (device) = sum R^2 (fixed-order,
 * deterministic).  If out_energy is not NULL, *out_energy (device) = sum_e sum_q w detJ psi(F_q),
 * the strain energy of compute_fields (postprocess.py:102).  f may be NULL (zero load).
 * work: dfea_reduce_work_bytes(mesh) bytes of scratch.
 */
int dfea_residual(const dfea_mesh_view* mesh, const double* u, const double* theta, double mu0,
                  double lambda0, const double* f, double load_factor, double* R, double* out_norm2,
                  double* out_energy, void* work, void* stream);
int dfea_residual_mat(const dfea_mesh_view* mesh, const double* u, const double* theta,
                      const dfea_material* material, const double* f, double load_factor, double* R,
                      double* out_norm2, double* out_energy, void* work, void* stream);

/* *out (device) = sum_i x_i^2 over 2N entries, fixed-order reduction.  work as for dfea_residual. */
int dfea_vec_norm2(const dfea_mesh_view* mesh, const double* x, double* out, void* work, void* stream);

/* ---------------------------------------------------------------- kernel (d) ------------------ */

/*
 * Per-element compliance sensitivity, the implicit VJP of adjoint.py:75-106:
 *   g_e = -sum_{a,i} (m * lambda)[dof(e,a,i)] f_e[a,i](u; mu0, lambda0),
 * exact because R_int is linear in theta_e when theta scales every parameter (neo-Hookean mu and
 * lambda, materials.py:308-312).  g has n_el entries in ORIGINAL element order.
 */
int dfea_element_sensitivity(const dfea_mesh_view* mesh, const double* u, const double* lam,
                             double mu0, double lambda0, double* g, void* stream);

/*
 * The same for any material: every energy of the library is linear in each parameter that may be
 * scaled (mu, lambda, c10, c01, kappa, k1: prefactors of its terms), so f_e is linear in theta_e with
 * slope f_e(u; p0 restricted to the scalable entries).  DFEA_ERR_UNSUPPORTED if theta scales a
 * parameter that enters nonlinearly (gamma, k2, beta_deg, d, second_family).
 */
int dfea_element_sensitivity_mat(const dfea_mesh_view* mesh, const double* u, const double* lam,
                                 const dfea_material* material, double* g, void* stream);

/* ---------------------------------------------------------------- multigrid ------------------- */
/*
 * Geometric multigrid on structured quadrilateral grids: the kernels of a V-cycle preconditioner
 * (preconditioner="multigrid"; the reference lists a scalable preconditioner as its main open item,
 * docs/ROADMAP.md:11).  Level 0 is the finite-element mesh, described as a grid of gx x gy node-grid
 * cells (Q4: the element grid; Q9: the element grid refined twice) with node_ij (2N int32, the grid
 * position of every FE node), gnode ((gx+1)(gy+1) int32, the FE node at every grid node) and
 * cell_slot (one int32 per element cell, the element's packed slot; element cell (cx, cy) spans grid
 * nodes [span cx, span cx + span] x [span cy, span cy + span]).  Every coarser level is a Q4 grid whose
 * grid lines sit on lines of the level above (line_x / line_y) with bilinear interpolation between them;
 * its nodes are numbered i * (gy + 1) + j and its cells cx * gy + cy; its operator is stored as one
 * 8 x 8 Galerkin element matrix per cell (K: [64][gx gy], DOF order 2 corner + component, corners
 * (0,0) (1,0) (1,1) (0,1)) plus fix bits per node (identity rows).  All device pointers.
 */
typedef struct dfea_mg_grid {
    int32_t gx, gy;         /* cells; nodes (gx + 1) x (gy + 1)                                     */
    const int32_t* line_x;  /* [gx + 1]: the grid line of the finer level under each line (coarse)  */
    const int32_t* line_y;  /* [gy + 1]                                                              */
    const int32_t* cell_x;  /* [finer gx + 1]: the cell of this level holding each finer line        */
    const int32_t* cell_y;  /* [finer gy + 1]                                                        */
    double* K;              /* [64][gx * gy] element matrices (coarse levels)                        */
    uint8_t* fix;           /* [(gx + 1) (gy + 1)] fix bits (coarse levels)                          */
} dfea_mg_grid;

/* Level 1 from the stored moduli (DFEA_F64, DFEA_F32 or DFEA_F32REF) of the mesh: coarse->K.  Any element
 * type on a grid: one element per cell (Q4, Q8, Q9; span 1 or 2 grid cells) or two triangles per cell (Tri3,
 * Tri6); cell_slot lists the packed slots of the elements of cell c at [c epc .. c epc + epc). */
int dfea_mg_galerkin_fe(const dfea_mesh_view* mesh, const void* moduli, int32_t moduli_dtype,
                        const int32_t* node_ij, const int32_t* cell_slot, int32_t span,
                        const dfea_mg_grid* fine, const dfea_mg_grid* coarse, void* stream);
/* Level l + 1 from level l (l >= 1): coarse->K = sum over fine cells of P^T K P. */
int dfea_mg_galerkin(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, void* stream);
/* rc = P~^T r, P~ the interpolation with fixed fine DOFs zeroed (r, rc may be NULL); coarse_fix_out
 * (optional) receives the coarse fix bits.  gnode: level 0's grid-to-FE-node map, NULL on coarse levels;
 * fine_fix: the fine level's fix bits per DOF node (level 0: the mesh's node_fix). */
int dfea_mg_restrict(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, const int32_t* gnode,
                     const uint8_t* fine_fix, const double* r, double* rc, uint8_t* coarse_fix_out,
                     void* stream);
/* x += P~ ec. */
int dfea_mg_prolong_add(const dfea_mg_grid* fine, const dfea_mg_grid* coarse, const int32_t* gnode,
                        const uint8_t* fine_fix, const double* ec, double* x, void* stream);
/* y = K v + (I - M) v on a coarse level; dfea_mg_diag: its diagonal. */
int dfea_mg_apply(const dfea_mg_grid* grid, const double* v, double* y, void* stream);
int dfea_mg_diag(const dfea_mg_grid* grid, double* diag, void* stream);
/* Chebyshev smoothing (Jacobi-preconditioned Chebyshev iteration): d = (*scale) r / diag; and one step
 * x += d, r -= q (q = A d), then unless last d = c[0] d + c[1] r / diag.  scale and c are device
 * pointers, so a captured CUDA graph of the cycle picks up new coefficients at every linearisation. */
int dfea_mg_cheb_start(int64_t n, const double* r, const double* diag, const double* scale, double* d, void* stream);
int dfea_mg_cheb_step(int64_t n, double* x, double* r, double* d, const double* q, const double* diag,
                      const double* c, int32_t last, void* stream);
/* Lanczos for lambda_max(D^-1 A) by Jacobi-preconditioned CG, scalars on the device: *out = x . y (two
 * fixed-order passes over dfea_mg_dot_work() doubles of caller scratch); and
 * after q = A p, one CG step: s[0] = p.q, alpha = s[1] / s[0], r -= alpha q, z = r / diag,
 * beta = r.z / s[1], p = z + beta p, s[1] = r.z, s[3] = beta, (alpha, beta) into hist[2k], hist[2k+1].
 * Start: r = b, z = r / diag, p = z, s[1] = r.z.  The eigenvalues of the tridiagonal matrix of the
 * coefficients approximate those of D^-1 A (Saad, Iterative Methods, section 6.7). */
int64_t dfea_mg_dot_work(void); /* doubles of the work buffer of dfea_mg_dot, dfea_mg_lanczos_step and
                                   dfea_mg.dot_work (the drivers keep a reduction ticket after the partials;
                                   dfea_mg_setup zeroes it) */
int dfea_mg_dot(int64_t n, const double* x, const double* y, double* out, double* work, void* stream);
int dfea_mg_lanczos_step(int64_t n, double* p, const double* q, double* r, double* z, const double* diag,
                         double* s, double* hist, int32_t k, double* work, void* stream);
/* Coarsest level: the dense inverse of its operator (at most dfea_mg_dense_max() DOFs; work and Ainv
 * hold n x n doubles each), and x = Ainv b. */
int64_t dfea_mg_dense_max(void);
int dfea_mg_dense_inverse(const dfea_mg_grid* grid, double* work, double* Ainv, void* stream);
int dfea_mg_dense_solve(int32_t n, const double* Ainv, const double* b, double* x, void* stream);

/*
 * The whole multigrid preconditioner and its PCG, driven from C++ (one call per set-up, per cycle, per
 * solve; the host reads scalars with stream synchronisations, no other host work between launches).
 * The caller owns every buffer and describes the hierarchy in a dfea_mg (levels[0] is the FE level:
 * only gx, gy and its vectors; coarse levels carry their dfea_mg_grid).  Vectors of a level hold n doubles.
 */
#define DFEA_MG_MAX_LEVELS 24
#define DFEA_MG_MAX_DEGREE 8
typedef struct dfea_mg_level {
    dfea_mg_grid grid;
    int64_t n;                                 /* 2 (gx + 1)(gy + 1); level 0: the mesh's 2N (a Q8 grid has
                                                * no nodes at the cell centres)                        */
    double *diag, *b, *x, *r, *d, *q;          /* device vectors of n doubles                       */
} dfea_mg_level;

typedef struct dfea_mg {
    int32_t n_levels;                          /* including level 0; the last one is solved densely */
    int32_t degree;                            /* Chebyshev steps per smoothing (<= DFEA_MG_MAX_DEGREE) */
    int32_t lanczos_steps;                     /* Jacobi-CG steps of the lambda_max estimate            */
    int32_t span;                              /* FE element span in grid cells: 1 (Q4) or 2 (Q9)    */
    double ratio;                              /* smoothing interval [lambda / ratio, lambda], lambda =
                                                * 1.1 x the Lanczos estimate                            */
    const int32_t* node_ij;                    /* FE node -> grid position (2N)                        */
    const int32_t* gnode;                      /* grid node -> FE node                                 */
    const int32_t* cell_slot;                  /* element cell -> packed element slot                  */
    dfea_mg_level level[DFEA_MG_MAX_LEVELS];
    double* Ainv;                              /* coarsest n x n inverse, and n x n of work            */
    double* dense_work;
    double* coef;                              /* [n_levels][2 DFEA_MG_MAX_DEGREE] Chebyshev coefficients */
    double* lscal;                             /* [n_levels][4] Lanczos scalars                         */
    double* lhist;                             /* [n_levels][2 lanczos_steps] Lanczos coefficients      */
    double* dot_work;                          /* dfea_mg_dot_work() doubles                            */
    double* pcg;                               /* 4 x level[0].n: the PCG's r, z, p, q                  */
    double* scal;                              /* 4 device doubles                                      */
    double lam[DFEA_MG_MAX_LEVELS];            /* out: the lambda_max estimates of the last set-up      */
    /* Graph-driven mode (optional): with pcg_state set, dfea_mg_setup replays its launch sequence as a CUDA
     * graph and dfea_mg_pcg runs its iteration as a device-side loop (scalars on the device, one graph
     * launch and one status read per solve), the same iterates bit for bit as the host-driven loop.  The
     * graphs are captured at the second call with the same buffers (the first runs directly, which also
     * sets up every lazily configured kernel attribute) and are owned by the library through `graphs`
     * (NULL at first; release them with dfea_mg_release).  NULL pcg_state: everything host-driven. */
    double* pcg_state;                         /* 16 device doubles, or NULL                            */
    void* graphs;                              /* library-owned, NULL until the first graph is captured */
    /* Smoother bounds: 0 (or less) estimates lambda_max by Lanczos at every set-up; k > 0 at the first set-up
     * and every k-th one after it, the others keeping the last estimates (and the Chebyshev coefficients
     * on the device): such a set-up rebuilds the coarse operators and the coarsest inverse only, with no
     * host synchronisation.  setups counts the set-ups so far (the library increments it). */
    int32_t bounds_every;
    int32_t setups;
    /* Optional element-result buffer (dfea_gather_work_bytes(mesh, DFEA_F64) bytes): when set and the mesh has
     * its node incidence, every level-0 product of the hierarchy runs in the gather form (an element pass and
     * the node sums: 2 launches) instead of one launch per colour; NULL: the colour form. */
    void* fe_work;
} dfea_mg;

/* Set-up at a linearisation: coarse operators from the moduli, coarsest inverse, Lanczos estimates,
 * Chebyshev coefficients (one host synchronisation). */
int dfea_mg_setup(const dfea_mesh_view* mesh, dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                  const double* diag, void* stream);
/* Host arithmetic of the set-up: the largest eigenvalue of the Lanczos tridiagonal matrix of `steps`
 * Jacobi-CG coefficients hist = (alpha_0, beta_0, alpha_1, ...), over the prefix before a breakdown (2.5 if
 * none), by Sturm-sequence bisection; -1 for bad arguments.  No GPU involved. */
double dfea_mg_lanczos_bound(const double* hist, int32_t steps);
/* z = one V-cycle applied to r (the moduli of the set-up). */
int dfea_mg_vcycle(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                   const double* r, double* z, void* stream);
/* Release the graphs a hierarchy captured in graph-driven mode (mg->graphs); no-op when there are none. */
int dfea_mg_release(dfea_mg* mg);
/* PCG (x0 = 0) for A x = b with the V-cycle as preconditioner; status as dfea_pcg_solve's. */
int dfea_mg_pcg(const dfea_mesh_view* mesh, const dfea_mg* mg, const void* moduli, int32_t moduli_dtype,
                const double* b, double* x, double rtol, int32_t max_iter, int32_t* iterations, int32_t* status,
                void* stream);

/* ---------------------------------------------------------------- kernel (c): PCG ------------- */

typedef struct dfea_pcg dfea_pcg; /* opaque: a captured CUDA graph of one PCG iteration */

/* Bytes of the caller buffer that dfea_pcg_create binds (Krylov vectors, partial sums, state). */
int64_t dfea_pcg_work_bytes(const dfea_mesh_view* mesh, int32_t vec_dtype);

/*
 * Bind a Jacobi-PCG solver to fixed buffers and capture one iteration in a CUDA graph whose
 * while-loop node repeats it on the device until convergence (newton_krylov.py:28-88 semantics:
 * x0 = 0, stop when ||r|| <= rtol ||b|| or at max_iter, early exit on p.Ap <= 0 returning z at
 * k = 0 and x otherwise).  moduli/diag/b/x are device buffers that stay bound to the handle;
 * their CONTENTS may change between solves.  vec_dtype DFEA_F64 needs f64 moduli; DFEA_F32 needs
 * f32 moduli and mesh->grad32, and then diag, b and x are f32; DFEA_MIXED applies f32 moduli and
 * mesh->grad32 to f64 vectors (diag, b, x f64): FP32 operator data, FP64 recurrences; DFEA_F32REF
 * applies reference-frame FP32 moduli (no gradients read) to f64 vectors.  The graph is captured on an internal
 * stream.  use_graph = 1: that graph; 2: 8 iterations captured back to back in a plain graph (no
 * conditional node) replayed by the host until the status word ends, which overlaps better with other
 * streams' work; 0: the same kernels launched directly, host-polled every 16 iterations.
 * OR-ing DFEA_PCG_GATHER into use_graph selects the gather form of the product inside each iteration
 * (one element pass writing every element's result, the per-node sums fused into the first vector
 * update: 3 kernels per iteration instead of n_colours + 2; needs mesh->node_elem_ptr/node_elem, and
 * then dfea_pcg_work_bytes includes the element-result buffer).  Its iterates agree with the colour
 * form's to rounding (the per-node sums are grouped differently); each form is reproducible.
 * DFEA_PCG_FUSED moves the direction update into the next element pass (each element computes
 * p = M^-1 r + beta p at the nodes it gathers; the node pass recomputes and stores it): 2 kernels per
 * iteration, the same recurrences, sums grouped differently.
 * OR-ing DFEA_PCG_MAX_BLOCKS(n) limits every launch of the solve to n blocks (the results agree with
 * the unlimited grid's to rounding: the reductions group their partial sums by block).
 */
int dfea_pcg_create(const dfea_mesh_view* mesh, const void* moduli, const void* diag,
                    const void* b, void* x, int32_t vec_dtype, void* work, int32_t use_graph,
                    dfea_pcg** out);

/*
 * Solve on `stream`.  Blocks the host until the solve ends (it reads back the iteration count);
 * *iters and *status receive the result (DFEA_PCG_* status word).
 */
int dfea_pcg_solve(dfea_pcg* pcg, double rtol, int32_t max_iter, int32_t* iters, int32_t* status,
                   void* stream);

/* Release the graph and the handle (not the bound buffers). */
int dfea_pcg_destroy(dfea_pcg* pcg);

/*
 * Batched PCG (no reference counterpart beyond newton_krylov.py:28-88: it runs several of its solves
 * at once).  The solves of several handles advance together: each iteration is one element-pass launch
 * per element type present plus one launch of each vector update for all of them.  A solve's blocks
 * split its work exactly as its own handle does (same block cap), so its iterates are bitwise those
 * of dfea_pcg_solve.  Handles must be in the serving configuration: gather form (not fused), Jacobi,
 * vec_dtype DFEA_F32REF.  Typical use from one host thread: dfea_batch_start for each new solve (after
 * its right-hand side is ready on `stream`), dfea_batch_set with the solves in flight, then
 * dfea_batch_iterate repeatedly; finished solves (status != DFEA_PCG_RUNNING) are dropped with the
 * next dfea_batch_set and their x is final.
 */
typedef struct dfea_batch dfea_batch;
int dfea_batch_create(int32_t capacity, int32_t max_blocks, dfea_batch** out);
int dfea_batch_destroy(dfea_batch* batch);
/* Reset and set up one handle's solve (x = 0, r = b, ...) on `stream`. */
int dfea_batch_start(dfea_batch* batch, dfea_pcg* pcg, double rtol, int32_t max_iter, void* stream);
/* The solves in flight (at most `capacity`); waits for the stream before replacing the table. */
int dfea_batch_set(dfea_batch* batch, dfea_pcg* const* pcgs, int32_t n, void* stream);
/* n_iterations iterations of every solve in the table (finished ones idle), then status[i], iters[i]
 * of each solve (host arrays of n entries); blocks until they are known. */
int dfea_batch_iterate(dfea_batch* batch, int32_t n_iterations, int32_t* status, int32_t* iters, void* stream);

/*
 * Jacobi-PCG without any device allocation.  This entry point has no counterpart in the reference.
 *
 * It is for callers that cannot allocate GPU memory themselves: a solver embedded in a host
 * application whose memory manager owns the device (a plug-in that must not call cudaMalloc), or a
 * caller on a latency-critical path where cudaMalloc/cudaFree would block or synchronise the device.
 * Such a caller passes only its inputs and outputs (moduli, diag, b, x as in dfea_pcg_create) and
 * gets the same iterates as dfea_pcg_solve with the kernels launched directly.  The Krylov vectors,
 * partial sums and solver state live in one fixed scratch array of DFEA_NOALLOC_SCRATCH_BYTES that
 * the library reserves in every GPU's memory when the library is loaded there, for the life of the
 * process.  Limits: mesh->n_nodes <= DFEA_NOALLOC_MAX_NODES and mesh->n_colours <= 16; larger meshes
 * are rejected with DFEA_ERR_INVALID and a message.  The first call on a device looks up the
 * scratch array's device address once (with that device current); make that first call before any
 * stream capture.  All calls share the one array, so calls that overlap on the GPU (two host threads,
 * two streams) race and must be serialised by the caller.  Blocks the host until the solve ends.
 */
#define DFEA_NOALLOC_SCRATCH_BYTES (8 * 1024 * 1024)
#define DFEA_NOALLOC_MAX_NODES 131072
int dfea_pcg_solve_noalloc(const dfea_mesh_view* mesh, const void* moduli, const void* diag,
                           const void* b, void* x, int32_t vec_dtype, double rtol, int32_t max_iter,
                           int32_t* iters, int32_t* status, void* stream);

/* ---------------------------------------------------------------- Newton-Krylov driver -------- */

/*
 * One complete solve R(u, theta) = 0 driven from C++: load continuation with cut-backs
 * (newton_krylov_solve, newton_krylov.py:185-264), inexact Newton with the Eisenstat-Walker forcing term
 * eta = min(0.5, sqrt(||R|| / ||R_0||)) (newton_at_load, :126-179) and Armijo backtracking from alpha = 1
 * down to 2^-5 with c1 = 1e-4, NaN rejecting a step (armijo_line_search, :94-120).  Each linearisation
 * runs kernel (a) (dfea_qp_moduli_mat) and, with a multigrid hierarchy, dfea_mg_setup; each linear solve
 * negates R into b and runs the bound PCG handle (dfea_pcg_solve, which must be bound to b and du) or
 * dfea_mg_pcg.  The caller owns every buffer (device unless noted).  The host reads one scalar per residual
 * and (status, iterations) per linear solve; nothing here holds a lock of the calling language, so threads
 * solving different problems proceed side by side.  Blocks the host until the solve ends.
 */
typedef struct dfea_newton {
    const dfea_mesh_view* mesh;  /* host pointer                                                     */
    dfea_material material;
    const double* theta;         /* [n_el] design field, ORIGINAL element order                      */
    const double* f;             /* [2N] external load at load factor 1                              */
    const double* u_D;           /* [2N] prescribed displacements at load factor 1, or NULL (zero)   */
    double* u;                   /* [2N] out: the last accepted state (the solution when converged)  */
    double *w, *uc;              /* [2N] scratch: the Newton iterate and the line-search trial       */
    double *R, *Rc;              /* [2N] scratch: their residuals                                    */
    double *du, *b;              /* [2N] the Newton step and -R (the PCG handle's x and b)           */
    double* diag;                /* [2N] Jacobi diagonal (written by kernel (a))                     */
    double* blocks;              /* [4N] inverse 2x2 node blocks for block-Jacobi, or NULL           */
    void* moduli;                /* moduli buffer of moduli_dtype (DFEA_F64, DFEA_F32 or DFEA_F32REF) */
    int32_t moduli_dtype;
    int32_t reserved;
    void* reduce_work;           /* dfea_reduce_work_bytes(mesh) bytes                               */
    double* scal;                /* 4 device doubles                                                 */
    double* scal_host;           /* 4 host doubles (pinned)                                          */
    dfea_pcg* pcg;               /* exactly one of pcg (bound to b, du) and mg                       */
    dfea_mg* mg;
    double min_rtol;             /* floor of the inner tolerance: 0 (FP64 operator) or, for an FP32
                                  * operator, the accuracy it can deliver (1e-5)                     */
} dfea_newton;

typedef struct dfea_newton_record {  /* one Newton iteration, as the reference's history records     */
    int32_t step, iteration, cg_iters, pcg_status;
    double load_factor, residual, alpha;
} dfea_newton_record;

typedef struct dfea_newton_info {
    int32_t converged, total_newton, total_cg, n_cutbacks;
    double load_factor;            /* the load factor reached                                        */
    int32_t n_records;             /* records written (at most max_records; total_newton counts all) */
    int32_t reserved;
} dfea_newton_info;

int dfea_newton_solve(const dfea_newton* nw, int32_t n_load_steps, double tol, int32_t max_newton,
                      int32_t max_cutbacks, int32_t pcg_max_iter, dfea_newton_info* info,
                      dfea_newton_record* records, int32_t max_records, void* stream);

/* ---------------------------------------------------------------- vector helpers -------------- */

/* y = a * x + y  on n entries (f64). */
int dfea_axpy(int64_t n, double a, const double* x, double* y, void* stream);

/* out = a + alpha * b  on n entries (f64): the Newton trial state of the line search. */
int dfea_add_scaled(int64_t n, const double* a, double alpha, const double* b, double* out,
                    void* stream);

/* Element-wise conversions between f64 and f32 vectors (n entries). */
int dfea_f64_to_f32(int64_t n, const double* x, float* y, void* stream);
int dfea_f32_to_f64(int64_t n, const float* x, double* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DIFFFEA_B200_H */
