/*
 * pymatting_b200 — C ABI of the B200 (sm_100a) closed-form alpha solver.
 *
 * Plain C types only: device pointers, sizes and a cudaStream_t passed as
 * void*. Every function returns 0 on success or a negative status
 *   -1  invalid argument         -2  CUDA error         -3  invalid state
 *   -4  division by zero (where the reference raises ZeroDivisionError)
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
 * is_known may be NULL (no window skipped). radius 1 or 2. With diag_mask,
 * diag_value is added to the diagonal slot where the mask is set. */
int pmb_cf_laplacian_ell(const double* image, const uint8_t* is_known, int h, int w,
                         int radius, double epsilon, const uint8_t* diag_mask, double diag_value,
                         double* values, int64_t* indices, int64_t* indptr, void* stream);

/* Radius-1 Laplacian as 13 half-stencil planes, plus diag_value on the
 * diagonal where diag_mask is set: with diag_mask = is_known and
 * diag_value = lambda this is make_linear_system's A = L + lambda C
 * (pymatting/laplacian/laplacian.py:46-55). */
int pmb_cf_laplacian_planes(const double* image, const uint8_t* is_known, int h, int w,
                            double epsilon, const uint8_t* diag_mask, double diag_value,
                            double* planes, void* stream);

/* grad[k] = d(mu' L(image) x) / d image[k] (h*w*3, same layout as image)
 * for the radius-1 Laplacian, with windows skipped where is_known (may be
 * null) covers them, as in cf_laplacian. For the adjoint of a solve through
 * the Laplacian; no counterpart in the reference (it has no gradients). */
int pmb_cf_laplacian_vjp(const double* image, const uint8_t* is_known, int h, int w,
                         double epsilon, const double* x, const double* mu, double* grad,
                         void* stream);

/* ---- Large-kernel matting Laplacian (matrix-free) ---------------------- */

/* Replaces lkm_laplacian(image, epsilon, radius)
 * (pymatting/laplacian/lkm_laplacian.py:6-76). windows: (h-2r)(w-2r)*10
 * doubles (per window V, V mean, 1/|w| + mean' V mean), computed by
 * pmb_lkm_setup; scratch: pmb_lkm_scratch_elems doubles (-1: image not
 * larger than 2 radius). */
int64_t pmb_lkm_scratch_elems(int h, int w, int radius);
int pmb_lkm_setup(const double* image, int h, int w, int radius, double epsilon, double* windows,
                  double* scratch, void* stream);
/* out = L p (+ diag_add * p when diag_add is not null): L_matvec. */
int pmb_lkm_apply(const double* image, int h, int w, int radius, const double* windows,
                  const double* diag_add, const double* p, double* out, double* scratch,
                  void* stream);
/* diag = diag(L) (+ diag_add), inv_diag = 1 / diag if not null: diag_L. */
int pmb_lkm_diagonal(const double* image, int h, int w, int radius, const double* windows,
                     const double* diag_add, double* diag, double* inv_diag, double* scratch,
                     void* stream);

/* ---- Foreground / background estimation -------------------------------- */

/* Replace estimate_foreground_ml(image, alpha, regularization,
 * n_small_iterations, n_big_iterations, small_size, return_background,
 * gradient_weight) (pymatting/foreground/estimate_foreground_ml.py:186-253,
 * kernel _estimate_fb_ml :61-183). image: (h, w, depth) float32, alpha:
 * (h, w) float32, F and B: (h, w, depth) float32 (B may be null), all on the
 * device; depth 1..8. seed: the 2*depth starting colours (F then B) on the
 * device, or null for the mean foreground / background colours of the input
 * (summed in float64; the reference sums in float32, so seeds agree to
 * rounding). With equal seeds F and B are bit-identical to the reference.
 * Asynchronous on `stream`; pmb_fg_status reports a failed sweep.
 * Returns -4 ("division by zero") for a 1x1 image, where the reference
 * raises ZeroDivisionError. */
int64_t pmb_fg_workspace_bytes(int h, int w, int depth);
int pmb_fg_ml(const float* image, const float* alpha, int h, int w, int depth,
              float regularization, int n_small_iterations, int n_big_iterations,
              int small_size, float gradient_weight, const float* seed, float* F, float* B,
              void* workspace, int64_t workspace_bytes, void* stream);
/* Synchronises `stream`; 0 if the last pmb_fg_ml on `workspace` completed. */
int pmb_fg_status(void* workspace, void* stream);
/* Level sizes of estimate_foreground_ml.py:101-105 as (h, w) pairs in hw
 * (host memory); returns the number of levels. */
int pmb_fg_levels(int h, int w, int n_small_iterations, int n_big_iterations, int small_size,
                  int* hw, int max_levels);

/* Replace estimate_foreground_ml_cupy(input_image, input_alpha,
 * regularization, n_small_iterations, n_big_iterations, small_size)
 * (pymatting/foreground/estimate_foreground_ml_cupy.py:110-230, kernels
 * :5-107): the reference's GPU backend, Jacobi iterations in float32 with
 * its buffer handling (seeded with pixel (0, 0), result = the buffer named F
 * after the swaps). image (h, w, 3), alpha (h, w), F and B (h, w, 3)
 * float32 on the device (B may be null). Fused multiply-adds are allowed as
 * in the reference's NVRTC build, so results agree to float32 rounding.
 * Sides up to 65535 and h w 3 < 2^31. Returns -4 for a 1x1 image (the
 * reference divides by zero). */
int64_t pmb_fg_jacobi_workspace_bytes(int h, int w);
int pmb_fg_ml_jacobi(const float* image, const float* alpha, int h, int w, float regularization,
                     int n_small_iterations, int n_big_iterations, int small_size, float* F,
                     float* B, void* workspace, int64_t workspace_bytes, void* stream);

/* Replace uniform_laplacian(image, radius) (mode 0,
 * pymatting/laplacian/uniform_laplacian.py) and rw_laplacian(image, sigma,
 * radius, regularization) (mode 1, pymatting/laplacian/rw_laplacian.py;
 * like the reference, the weights are exp(-900 |z_i - z_j|^2) whatever
 * sigma is), each through weights_to_laplacian (util/util.py:840-875).
 * image: (h, w, 3) float64 (mode 1 only). px: w + 1 and py: h + 1 int64
 * prefix sums of the clamped window width per column and height per row;
 * the result is canonical CSR with rowptr (h w + 1), cols and vals
 * (py[h] * px[w] entries), all on the device. h w < 2^31. */
int pmb_window_laplacian(int mode, const double* image, int h, int w, int radius,
                         double regularization, const int64_t* px, const int64_t* py,
                         int64_t* rowptr, int64_t* cols, double* vals, void* stream);

/* Replace lbdm_laplacian(image, epsilon, radius)
 * (pymatting/laplacian/lbdm_laplacian.py) for radius 1 or 2 and images
 * larger than 2 radius in both directions: per interior window
 * T = (I - F)(I - F)^T with F = (K + eps I)^-1 K, K = X X^T over the
 * window's [colours, 1], summed into canonical CSR. scratch:
 * pmb_lbdm_scratch_elems doubles (-1: unsupported). px / py (w + 1, h + 1
 * int64): prefix sums of the number of columns / rows of pixels that share a
 * window with a pixel of that column / row; cols and vals hold py[h] * px[w]
 * entries. */
int64_t pmb_lbdm_scratch_elems(int h, int w, int radius);
int pmb_lbdm_laplacian(const double* image, int h, int w, int radius, double epsilon,
                       double* scratch, const int64_t* px, const int64_t* py, int64_t* rowptr,
                       int64_t* cols, double* vals, void* stream);

/* Replace knn_laplacian(image, n_neighbors, distance_weights, kernel)
 * (pymatting/laplacian/knn_laplacian.py): per pass p, the n_neighbors[p]
 * nearest pixels in the float32 feature space (r, g, b, dw x, dw y) by an
 * exact search with the distance of pymatting/util/kdtree.py, keeping the k
 * smallest by (distance, index) (the reference resolves equal distances in
 * its tree order);
 * W = sum_p B_p + B_p^T (soft != 0: weights 1 - |f_i - f_j|_1 / 5);
 * L = I - diag(1 / rowsum(W)) W as canonical CSR. Two calls on the same
 * scratch (pmb_knn_scratch_elems int64) and rowptr (h w + 1): the first with
 * cols = vals = null returns the entry count in *nnz; the second fills cols
 * and vals (*nnz entries). image: (h, w, 3) float64 on the device;
 * n_neighbors and distance_weights: host arrays of `passes` (1..4) values. */
int64_t pmb_knn_scratch_elems(int64_t n, int total_neighbors, int passes);
int pmb_knn_laplacian(const double* image, int h, int w, const int* n_neighbors,
                      const double* distance_weights, int passes, int soft, int64_t* scratch,
                      int64_t* rowptr, int64_t* cols, double* vals, int64_t* nnz, void* stream);

/* System matrix of estimate_foreground_cf
 * (pymatting/foreground/estimate_foreground_cf.py) for the default
 * neighbours: A = U^T U + diag(S, S) over 2 h w unknowns (foreground, then
 * background) as canonical CSR. Two calls: with cols = vals = null it writes
 * rowptr (2 h w + 1; the entry count is rowptr[2 h w]); then it fills cols
 * and vals. alpha: (h, w) float64 on the device; scratch:
 * (2 h w + 1023) / 1024 + 2 int64. */
int pmb_fg_cf_system(const double* alpha, int h, int w, double regularization, int64_t* rowptr,
                     int64_t* cols, double* vals, int64_t* scratch, void* stream);

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
/* Kernel launches issued by this object so far (kernels replayed from its
 * CUDA graphs included). */
int64_t pmb_stencil_launch_count(const pmb_stencil* s);
int pmb_stencil_destroy(pmb_stencil* s);
/* Launch-shape knobs of the solver, for the autotuner (no counterpart in the
 * reference): 0 vector width of the CG apply (2 or 4 pixels per thread, 4
 * only for the FP32 inner solve), 1 the same for the prolongation, 2/3/4
 * resident CTAs per SM of the level-0 tile kernels / prolongation /
 * restriction (up to the shared-memory limit), 5 CTAs per SM of the
 * element-wise kernels, 6 CG iterations per graph replay, 7 buffers of the
 * CG apply, restriction and prolongation kernels (1, the default: half the
 * shared memory, so twice the CTAs per SM; 2: a tile in flight per CTA;
 * setting it resets knobs 2, 3 and 4 to the new residency limit). Returns
 * the value applied (after clamping) or a negative status. */
int pmb_stencil_tune(pmb_stencil* s, int knob, int value);
int pmb_stencil_tuning(const pmb_stencil* s, int knob);
/* Average milliseconds of one level-0 operator apply y = A x (inner
 * precision), timed with CUDA events on the solver's stream over `iters`
 * launches. Benchmark hook; no reference counterpart. */
int pmb_stencil_time_apply(pmb_stencil* s, int iters, double* ms, void* stream);
/* Milliseconds per iteration in each kind of launch over `iters` live solve
 * iterations of A x = b (b: concatenated per-image vectors), CUDA events on
 * the solver's stream after every launch. ms_out holds 10 values: CG apply,
 * CG update, mixed-precision refinement, restriction from level 0,
 * restriction from coarser levels, coarse-level tail, direct coarsest
 * solves, prolongation at coarser levels, prolongation at level 0, other.
 * Measurement only: no reference counterpart (it times the loop of
 * pymatting/solver/cg.py:82-113 with vcycle.py:46-100 as M). */
int pmb_stencil_profile(pmb_stencil* s, const double* b, int iters, double* ms_out, void* stream);

/* ---- Sparse-format helpers (device arrays, int64 indices) ---------------- */

/* Scratch elements (int64) the scans below need for n entries. */
int64_t pmb_scan_scratch_elems(int64_t n);
/* Canonical CSR of an assembled ELL (values from pmb_cf_laplacian_ell):
 * in-image slots with a non-zero value, ascending columns — the form scipy
 * gives L + C in make_linear_system (pymatting/laplacian/laplacian.py:50-55).
 * rowptr has n+1 entries; rowptr[n] = nnz. */
int pmb_ell_csr_rowptr(const double* values, int h, int w, int radius, int64_t* rowptr,
                       int64_t* scratch, void* stream);
int pmb_ell_csr_fill(const double* values, int h, int w, int radius, const int64_t* rowptr,
                     int64_t* indices, double* data, void* stream);
/* Canonical CSR of A + diag(c) for a general CSR A of any row length
 * (make_linear_system on a matrix not assembled by this library,
 * pymatting/laplacian/laplacian.py:50-55): columns ascending, duplicates
 * summed in stored order, explicit zeros dropped. *overflow is set to 0 (kept
 * for callers of the earlier row-length limit). */
int pmb_csr_add_diag_rowptr(int64_t n, const int64_t* indptr, const int64_t* indices,
                            const double* data, const double* c, int64_t* rowptr, int* overflow,
                            int64_t* scratch, void* stream);
int pmb_csr_add_diag_fill(int64_t n, const int64_t* indptr, const int64_t* indices,
                          const double* data, const double* c, const int64_t* rowptr,
                          int64_t* out_indices, double* out_data, void* stream);
/* Bounded-wait self-test (no reference counterpart; it tests the failure
 * convention that every device wait of this library ends with an error
 * status instead of spinning, as the reference's solvers end with errors:
 * pymatting/solver/cg.py:115-117, pymatting/preconditioner/ichol.py:259-296).
 * which = 0: the mbarrier wait of the TMA kernels, limit in polls; which = 1:
 * the epoch poll of the foreground sweep, limit in nanoseconds; which = 2:
 * the chunk wait of the streamed ichol solve, limit in polls (a solve whose
 * wait gives up returns NaN). Each waits on a barrier or word that nothing
 * completes; *timed_out = 1 when the wait gave up and reported it.
 * scratch: 64 bytes of device memory. */
int pmb_selftest_wait(int which, int64_t limit, void* scratch, int* timed_out, void* stream);

/* Half-stencil planes (13 x h x pitch doubles, the stencil engine's layout)
 * of an (h w) x (h w) CSR matrix of a pixel grid whose entries lie within
 * the 5x5 neighbourhood of their row's pixel, so that vcycle runs on any
 * such matrix (pymatting/preconditioner/vcycle.py:103-153 accepts any A of
 * shape (h w, h w)). back: 12 x h x pitch doubles of scratch. bad[0] = entries
 * outside the 5x5 neighbourhood, bad[1] = pairs A[i, j] / A[j, i] that differ
 * by more than rel_tol relative (the engine needs a symmetric A). */
int pmb_csr_to_planes(const int64_t* indptr, const int64_t* indices, const double* data, int h,
                      int w, double* planes, double* back, double rel_tol,
                      unsigned long long* bad, void* stream);

/* ---- Trimap and hard-constraint system --------------------------------- */

/* trimap_split (pymatting/util/util.py:510-525): is_fg = t >= fg_threshold,
 * is_known = is_fg | (t <= bg_threshold); counts[0] = #fg, counts[1] = #bg. */
int pmb_trimap_masks(const double* trimap, int64_t n, double fg_threshold, double bg_threshold,
                     uint8_t* is_fg, uint8_t* is_known, unsigned long long* counts, void* stream);
/* Compact index of every unknown pixel (exclusive scan); cidx[n] = #unknown. */
int pmb_unknown_index(const uint8_t* is_known, int64_t n, int64_t* cidx, int64_t* scratch,
                      void* stream);
/* Same result as pmb_unknown_index, but allocates nothing and takes no
 * scratch: for callers that cannot call cudaMalloc (a host program that
 * hands the library only buffers from its own fixed, pre-sized pool, or a
 * binding with no device allocator). No counterpart in the reference. The
 * scan's scratch is a 256 KB array inside the library, present on every
 * device that loads it until the process exits; n is limited to
 * PMB_UNKNOWN_INDEX_STATIC_MAX_N (larger n fails with status -1). The first
 * call on a device looks up the array's device address; make that first
 * call before any stream capture. After a device reset the library is loaded
 * into a new context and the array moves: the first call in the new context
 * looks the address up again (make that call, too, before any capture).
 * Calls share the array, so calls whose work overlaps on the GPU race; order
 * them on one stream. */
#define PMB_UNKNOWN_INDEX_STATIC_MAX_N 33553407
int pmb_unknown_index_static(const uint8_t* is_known, int64_t n, int64_t* cidx, void* stream);
/* L_U = L[U, :][:, U] and b_U = -L[U, :][:, K] is_fg[K] from the ELL of the
 * Laplacian of window radius `radius` assembled with is_known (ELL rows of
 * (4 radius + 1)^2 slots; estimate_alpha_cf.py:55, 64-74). */
int pmb_hard_lu_rowptr(const uint8_t* is_known, int h, int w, int radius, const int64_t* cidx,
                       int64_t n_unknown, int64_t* rowptr, int64_t* scratch, void* stream);
int pmb_hard_lu_fill(const double* ell_values, const uint8_t* is_known, const uint8_t* is_fg,
                     int h, int w, int radius, const int64_t* cidx, const int64_t* rowptr,
                     int64_t* indices, double* data, double* rhs, void* stream);
/* alpha = clip(trimap on known pixels, x_U on unknown ones) to [0, 1]
 * (estimate_alpha_cf.py:72-76). */
int pmb_alpha_compose(const double* trimap, const uint8_t* is_known, const int64_t* cidx,
                      const double* x_unknown, int64_t n, double* alpha, void* stream);
/* out = value * mask (b = lambda * is_fg, laplacian.py:48). */
int pmb_mask_scale(const uint8_t* mask, int64_t n, double value, double* out, void* stream);
/* out = clip(x, 0, 1). */
int pmb_clip01(const double* x, int64_t n, double* out, void* stream);

/* ---- General CSR systems ------------------------------------------------ */

/* One system A x = b with A in CSR (or applied by the caller) solved by
 * cg (pymatting/solver/cg.py:4-117). preconditioner: 0 none, 1 Jacobi (1/diag
 * in the invd row of the vector block), 2 matrix (M.dot, cg.py:58-62),
 * 3 incomplete Cholesky (pmb_ichol), 4 applied by the caller. */
int pmb_csr_create(int64_t n, int64_t nnz, int preconditioner, pmb_csr** out);
int64_t pmb_csr_workspace_bytes(const pmb_csr* c);
/* vectors: 8 n doubles, rows x r z p0 p1 Ap dr invd. indptr/indices/data
 * may be NULL when the caller applies A. */
int pmb_csr_bind(pmb_csr* c, void* workspace, double* vectors, const int64_t* indptr,
                 const int64_t* indices, const double* data);
int pmb_csr_set_matrix_preconditioner(pmb_csr* c, int64_t nnz, const int64_t* indptr,
                                      const int64_t* indices, const double* data, void* stream);
int pmb_csr_set_ichol(pmb_csr* c, pmb_ichol* factor, void* stream);
int pmb_csr_solve(pmb_csr* c, const double* b, const double* x0, double* x_out, double atol,
                  double rtol, int maxiter, int reorthogonalize, void* stream);
/* Step interface for callbacks and caller-applied A or M: begin, then per
 * iteration step(0) (or step(1), caller writes A p into the Ap row,
 * step(2)), stats, and after a caller-applied M finish_precondition. */
int pmb_csr_begin(pmb_csr* c, const double* b, const double* x0, double atol, double rtol,
                  int maxiter, int reorthogonalize, void* stream);
int pmb_csr_step(pmb_csr* c, int mode, void* stream);
int pmb_csr_finish_precondition(pmb_csr* c, void* stream);
/* Row (0 or 1) of the p double-buffer that holds the current direction. */
int pmb_csr_p_index(pmb_csr* c);
int pmb_csr_stats(pmb_csr* c, int* iters, int* status, double* norm_r, double* norm_b);
int pmb_csr_destroy(pmb_csr* c);
/* y = A x; invd = 1 / diag(A) (duplicates summed, jacobi.py:24-26);
 * out = a * b element-wise (the Jacobi apply, jacobi.py:28-29). */
int pmb_csr_spmv(int64_t n, const int64_t* indptr, const int64_t* indices, const double* data,
                 const double* x, double* y, void* stream);
int pmb_csr_inv_diag(int64_t n, const int64_t* indptr, const int64_t* indices,
                     const double* data, double* invd, void* stream);
int pmb_vec_mul(int64_t n, const double* a, const double* b, double* out, void* stream);
/* 1 / diagonal of a radius-1 plane set, in user layout. */
int pmb_planes_inv_diag(const double* planes, int h, int w, double* inv_diag, void* stream);
/* x = A^-1 b for a small square CSR matrix (n <= 4096) by Gaussian
 * elimination with partial pivoting — the direct branch of the V-cycle
 * (vcycle.py:59-60). scratch n*n doubles; x holds b on entry. */
int pmb_dense_solve(int64_t n, const int64_t* indptr, const int64_t* indices, const double* data,
                    double* scratch, double* x, int* singular, void* stream);

/* ---- Thresholded incomplete Cholesky ----------------------------------- */

/* Lower-part profile of a CSC matrix: out[0] = bandwidth, out[1] = envelope
 * (bound on the factor size). scratch: n + 2 uint64. */
int pmb_csc_profile(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                    uint64_t* scratch, uint64_t* out, void* stream);
/* Factor object for ichol(A, discard_threshold, shifts, max_nnz,
 * relative_discard_threshold, diag_keep_discarded)
 * (pymatting/preconditioner/ichol.py:184-301). capacity >= factor nnz. */
int pmb_ichol_create(int64_t n, int64_t bandwidth, int64_t capacity, pmb_ichol** out);
int64_t pmb_ichol_workspace_bytes(const pmb_ichol* f);
int pmb_ichol_bind(pmb_ichol* f, void* workspace);
/* One attempt with a diagonal shift (ichol.py:259-276); *result = factor nnz,
 * -1 (not positive definite) or -2 (more than max_nnz entries). */
int pmb_ichol_factor(pmb_ichol* f, const int64_t* Ap, const int64_t* Ar, const double* Av,
                     double discard_threshold, double shift, int64_t max_nnz,
                     double relative_discard_threshold, int diag_keep_discarded,
                     int64_t* result, void* stream);
/* Dependency levels of the factor (length of the triangular-solve schedule). */
int pmb_ichol_levels(const pmb_ichol* f);
/* CTAs of the cluster that held the factorisation's band front in
 * distributed shared memory in the last pmb_ichol_factor (1..8), 0 when the
 * front was in global memory (bandwidth too wide), -1 before any factor. */
int pmb_ichol_cluster(const pmb_ichol* f);
/* Device time (CUDA events on the factor's stream) of the factorisation
 * kernel in the last pmb_ichol_factor, in milliseconds; -1 before any. */
float pmb_ichol_factor_ms(const pmb_ichol* f);
/* Device pointers of the CSC factor (values, row indices, column pointers). */
int pmb_ichol_factor_arrays(pmb_ichol* f, void** Lv, void** Lr, void** Lp);
/* x = L^-T L^-1 b (CholeskyDecomposition.__call__, ichol.py:175-181). */
int pmb_ichol_apply(pmb_ichol* f, const double* b, double* x, void* stream);
int pmb_ichol_destroy(pmb_ichol* f);

#ifdef __cplusplus
}
#endif

#endif /* PYMATTING_B200_H */
