// Launch interface of the half-stencil kernels (stencil.cu) for the engine.
#pragma once

#include <cuda.h>

#include "pm_common.cuh"

namespace pmb {

enum : int { kPrecNone = 0, kPrecJacobi = 1, kPrecVcycle = 2, kPrecExternal = 3 };

constexpr int kMaxDirect = 256;  // largest coarsest grid solved densely

struct LaunchCfg { int grid; };

// Coarsest grid of one image: dense inverse used in place of a sparse LU.
struct DirectDesc {
    GridDesc g;
    double* inv;        // n x n inverse
    int64_t work_off;   // n x n scratch used while inverting (setup only)
    const double* P;    // FP64 planes of the grid's level (grid at P + g.poff)
};

// Coarse-level tail (one CTA per image, shared-memory resident; k_vc_tail).
constexpr int kTailThreads = 1024;
constexpr int kMaxTailLevels = 16;
constexpr size_t kTailSmem = 212 * 1024;   // planes + 3 vectors of all tail levels (pitched)

template <typename T>
struct TailLevel {
    GridDesc g;
    const T* P;     // planes
    T* b;           // right-hand side (read for the first tail level)
    T* x;           // solution (written for the first tail level)
};

template <typename T>
struct TailDesc {
    int nlev;               // tail levels; the last is solved with `inv`
    int inst;               // image
    int pad_[2];
    const double* inv;      // dense inverse of the last level
    TailLevel<T> lev[kMaxTailLevels];
};

template <typename T>
void launch_vc_tail(const TailDesc<T>* descs, int count, size_t smem, const InstState* st,
                    double omega, int* err, cudaStream_t s);

// Shared memory (bytes) of the TMA-tiled kernels, for launch sizing.
template <typename T> size_t smem_apply();
template <typename T> size_t smem_init();
template <typename T> size_t smem_down(int pre);
template <typename T> size_t smem_up(int pre);
// ... of the register-blocked kernels (default one pre- and one post-sweep).
template <typename T> size_t smem_apply_v(int nst);
// nst: 2 buffers (a tile in flight while one is computed) or 1.
template <typename T> size_t smem_down_v(int nst);
template <typename T> size_t smem_up_v(int nst);
// Resident CTAs per SM of the register-blocked CG apply, restriction and
// prolongation kernels for a vector width and buffer count (occupancy API).
template <typename T> int resident_cg_apply(int vec, int stages);
template <typename T> int resident_down(int stages);
template <typename T> int resident_cg_update(int prec);
template <typename T> int resident_up(int vec, int stages);
// Width of the register-blocked restriction box (its TMA maps).
template <typename T> int down_box_width();

// Raise the dynamic shared-memory limits once (before any graph capture).
void stencil_prepare();

// Self-test: 64 threads wait `polls` polls for an mbarrier that never
// completes; each gives up and adds one to *gave_up.
void launch_selftest_mbar(uint32_t polls, int* gave_up, cudaStream_t s);

template <typename T>
void launch_cg_init(int prec, const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps,
                    const T* P, const T* b, T* x, bool have_x0, T* r, T* z, InstState* st,
                    double* part, double atol, double rtol, int maxiter, int* err, cudaStream_t s);
template <typename T>
void launch_cg_apply(int vec, int stages, const LaunchCfg& L, const WorkList& wl,
                     const CUtensorMap* maps, int zslot, T* p0, T* p1, T* Ap, InstState* st,
                     double* part, int* err, cudaStream_t s);
template <typename T>
void launch_cg_update(int prec, const LaunchCfg& L, const WorkList& wl, const T* P, T* x, T* r,
                      T* z, const T* p0, const T* p1, const T* Ap, T* dr, int reorth, int reliable,
                      int* pending, InstState* st, double* part, cudaStream_t s);
template <typename T>
void launch_cg_rz(const LaunchCfg& L, const WorkList& wl, const T* r, const T* z, const T* dr,
                  int reorth, InstState* st, double* part, cudaStream_t s);
template <typename T>
void launch_vc_down(int pre, int stages, const LaunchCfg& L, const WorkList& wl,
                    const GridDesc* fine, const CUtensorMap* maps, int xs_slot, T* bc,
                    double omega, const InstState* st, int* err, cudaStream_t s);
template <typename T>
void launch_vc_up(int vec, int stages, int pre, int post, const LaunchCfg& L, const WorkList& wl,
                  const GridDesc* coarse, const CUtensorMap* maps, int xs_slot, const T* b,
                  T* xout, double omega, InstState* st, int level0, const T* dr, int reorth,
                  double* part, int* err, cudaStream_t s);
template <typename T>
void launch_vc_smooth(const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps,
                      int xin_slot, const T* P, const T* b, T* xout, double omega,
                      const InstState* st, int* err, cudaStream_t s);
template <typename T>
void launch_vc_direct(const DirectDesc* dd, int count, const T* b, T* x, InstState* st,
                      int rz_level0, cudaStream_t s);
template <typename T>
void launch_apply(const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps, T* y, int* err,
                  cudaStream_t s);
template <typename TS, typename TD>
void launch_pack(const GridDesc* grids, int ngrids, const int64_t* uoff, const TS* src, TD* dst,
                 int64_t total, cudaStream_t s);
template <typename TS, typename TD>
void launch_unpack(const GridDesc* grids, int ngrids, const int64_t* uoff, const TS* src, TD* dst,
                   int64_t total, cudaStream_t s);
// Coarse operators over a list of coarse-grid tiles (8 x 16 coarse pixels);
// `fine` holds each coarse grid's fine grid, whose FP64 planes are read
// through map slot kMapPlG (box kGCols x kGRows x 13).
constexpr int kGalerkinTileY = 8, kGalerkinTileX = 16;
constexpr int kGRows = 2 * kGalerkinTileY + 5;      // 21 fine rows
constexpr int kGCols = 2 * kGalerkinTileX + 10;     // 42 fine columns (even start)
void launch_galerkin_t(const WorkList& wl, const GridDesc* fine, const CUtensorMap* maps,
                       double* Pc, int* err, cudaStream_t s);
void launch_galerkin(const GridDesc* fine_g, const GridDesc* coarse_g, int ngrids, const double* Pf,
                     double* Pc, int64_t total, cudaStream_t s);
// Dense inverses of every coarsest grid in one launch (one CTA per grid).
void launch_dense_inverse(const DirectDesc* dd, int count, double* work, int* status,
                          cudaStream_t s);
void launch_convert_f32(const double* src, float* dst, int64_t n, cudaStream_t s);
void launch_refine_residual(int prec, int first, const LaunchCfg& L, const WorkList& wl,
                            const CUtensorMap* maps, const float* P32, const double* b,
                            float* r32, float* x32, float* z32, InstState* outer,
                            InstState* inner, double* part, double atol, double rtol,
                            double delta, int maxiter, int max_outer, int* err,
                            cudaStream_t s);
// inner != nullptr: images flagged kUpdate; nullptr: every image.
void launch_refine_correct(const LaunchCfg& L, const WorkList& wl, double* x64, float* x32,
                           const InstState* inner, const int* pending, cudaStream_t s);

}  // namespace pmb
