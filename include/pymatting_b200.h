/*
 * pymatting_b200 — C ABI of the B200 (sm_100a) closed-form alpha solver.
 *
 * Plain C types only: device pointers, sizes and a cudaStream_t passed as
 * void*. Every function returns 0 on success or a negative status
 *   -1  invalid argument         -2  CUDA error         -3  invalid state
 * and pmb_last_error() describes the last failure of the calling thread.
 * The caller owns every device buffer. Objects (pmb_stencil, pmb_csr,
 * pmb_ichol) report the workspace they need; the caller allocates it and
 * binds it. All work is ordered on the caller's stream.
 *
 * Reference interfaces (PyMatting 1.1.15) that these entry points replace
 * are cited per function as file:line.
 *
 * Layout conventions
 *   image   h*w*3 float64, row-major, interleaved RGB (same as the
 *           (h, w, 3) numpy array PyMatting takes).
 *   masks   h*w uint8 (0/1).
 *   vectors contiguous float64, images of a batch concatenated.
 *   planes  the symmetric half stencil of a 25-point pixel-grid operator:
 *           13 planes of h*pitch float64, pitch = pmb_grid_pitch(w);
 *           plane p holds A[i, i+d_p] for d_p = (0,0),(0,1),(0,2),
 *           (1,-2..2),(2,-2..2) (dy, dx). Images of a batch follow each
 *           other (pmb_stencil_plane_offset).
 */
#ifndef PYMATTING_B200_H
#define PYMATTING_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmb_stencil pmb_stencil;
typedef struct pmb_csr pmb_csr;
typedef struct pmb_ichol pmb_ichol;

/* Description of the last failure on the calling thread. */
const char* pmb_last_error(void);
int pmb_version(void);
/* Row pitch (elements) of the pitched grid layout for width w. */
int pmb_grid_pitch(int w);

/* ---- Laplacian assembly ------------------------------------------------ */

/* Replaces cf_laplacian(image, epsilon, radius, is_known)
 * (pymatting/laplacian/cf_laplacian.py:132-177): fills the CSR arrays
 * exactly as the reference does — (4r+1)^2 slots per row, out-of-image
 * slots holding column 0 and value 0 — with bitwise-identical values.
 * is_known may be NULL (no window skipped). radius 1 or 2. */
int pmb_cf_laplacian_ell(const double* image, const uint8_t* is_known, int h, int w,
                         int radius, double epsilon, double* values, int64_t* indices,
                         int64_t* indptr, void* stream);

/* Radius-1 Laplacian as 13 half-stencil planes, plus diag_value on the
 * diagonal where diag_mask is set: with diag_mask = is_known and
 * diag_value = lambda this is make_linear_system's A = L + lambda C
 * (pymatting/laplacian/laplacian.py:46-55). */
int pmb_cf_laplacian_planes(const double* image, const uint8_t* is_known, int h, int w,
                            double epsilon, const uint8_t* diag_mask, double diag_value,
                            double* planes, void* stream);

/* Hard-constraint system of estimate_alpha_cf
 * (pymatting/alpha/estimate_alpha_cf.py:64-74) on the full grid: planes of
 * L_U with identity rows for known pixels, and rhs = -R is_fg (0 on known
 * pixels), pitched. */
int pmb_cf_hard_system(const double* image, const uint8_t* is_known, const uint8_t* is_fg,
                       int h, int w, double epsilon, double* planes, double* rhs, void* stream);

/* ---- Stencil systems: PCG with Jacobi / V-cycle ------------------------- */

/* precision: 0 = FP64; 1 = FP32 inner PCG inside FP64 iterative refinement.
 * preconditioner: 0 none, 1 Jacobi (pymatting/preconditioner/jacobi.py:1-31),
 * 2 V-cycle (pymatting/preconditioner/vcycle.py:103-153, with its
 * num_pre_iter / num_post_iter / omega / direct_solve_size <= 256). */
int pmb_stencil_create(int n_images, const int* h, const int* w, int precision,
                       int preconditioner, int num_pre_iter, int num_post_iter, double omega,
                       int direct_solve_size, pmb_stencil** out);
int64_t pmb_stencil_workspace_bytes(const pmb_stencil* s);
/* Offset (elements) of image k's planes in the level-0 plane buffer, and
 * the buffer's total size in elements. */
int64_t pmb_stencil_plane_offset(const pmb_stencil* s, int image);
int64_t pmb_stencil_plane_elems(const pmb_stencil* s);
/* Number of multigrid levels of image k (1 without a V-cycle). */
int pmb_stencil_levels(const pmb_stencil* s, int image);
int pmb_stencil_bind(pmb_stencil* s, void* workspace, const double* planes64, void* stream);
/* Galerkin coarse operators, dense coarsest inverses, FP32 copies. Run
 * implicitly by the first solve / precondition call when not called. */
int pmb_stencil_setup(pmb_stencil* s, void* stream);
/* Replaces cg(A, b, x0, atol, rtol, maxiter, M=...) (pymatting/solver/cg.py:4-117)
 * for every image of the batch at once. b, x0 (may be NULL) and x_out are
 * concatenated user vectors. inner_rtol / max_outer apply to precision 1. */
int pmb_stencil_solve(pmb_stencil* s, const double* b, const double* x0, double* x_out,
                      double atol, double rtol, int maxiter, int reorthogonalize,
                      double inner_rtol, int max_outer, void* stream);
/* z = M r with the solver's preconditioner (the callable a preconditioner
 * factory returns, e.g. vcycle.py:148-151). FP64 solvers only. */
int pmb_stencil_precondition(pmb_stencil* s, const double* r, double* z, void* stream);
/* y = A x (A.dot(x) of the CSR matrix the planes describe). */
int pmb_stencil_apply(pmb_stencil* s, const double* x, double* y, void* stream);
/* Result of the last solve for image k. status: 1 converged, 2 maxiter,
 * 3 non-finite residual. iters: CG iterations (summed over refinement steps
 * for precision 1); outer_iters: refinement steps. */
int pmb_stencil_stats(pmb_stencil* s, int image, int* iters, int* status, double* norm_r,
                      double* norm_b, int* outer_iters);
/* Kernel launches issued by this object so far (graph replays excluded). */
int64_t pmb_stencil_launch_count(const pmb_stencil* s);
int pmb_stencil_destroy(pmb_stencil* s);

#ifdef __cplusplus
}
#endif

#endif /* PYMATTING_B200_H */
