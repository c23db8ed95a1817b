// Shared definitions for the sm_100a kernels of the closed-form alpha path.
//
// Operator layout ("half stencil"). The radius-1 matting Laplacian couples
// pixels at most two apart (pymatting/laplacian/cf_laplacian.py:15-23 writes
// a 5x5 block per row), and so do its Galerkin coarse operators. The matrix
// is symmetric, so only the centre and the 12 "forward" offsets are stored:
// plane p holds A[i, i + d_p] for d_p = (dy, dx) with dy > 0, or dy == 0 and
// dx >= 0. The backward entry A[i, i - d_p] is plane p read at pixel i - d_p.
// Planes are row-pitched 2D arrays, one after the other, so one apply reads
// 13 planes plus x and writes y: 15 values per pixel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pmb {

// Launch helpers return 0 or -2. On -2 they record the CUDA error they saw
// (cudaGetLastError clears it) so that the C ABI can report its text;
// take_launch_error() returns and clears it (cudaSuccess if the helper
// failed an argument check instead).
int launch_status(cudaError_t e);
inline int launch_status() { return launch_status(cudaGetLastError()); }
cudaError_t take_launch_error();

constexpr int kRS = 2;       // stencil radius of the stored operator
constexpr int kNH = 13;      // stored planes (centre + 12 forward offsets)
constexpr int kTX = 64;      // fine tile width
constexpr int kTY = 8;       // fine tile height
constexpr int kThreads = 256;      // element-wise kernels
constexpr int kTileThreads = 512;  // tiled stencil kernels: one pixel per thread
// Elements per tile of the element-wise kernels. 8192 halves the per-chunk
// barriers and directory lookups of the flat loops against 4096 (the FP32 CG
// update: 0.38 -> 0.31 ms per iteration of the 64-image batch).
constexpr int kFlat = 8192;

// Shared-memory boxes loaded by TMA around a fine tile at (x0, y0): origin
// (x0 - kBOX, y0 - 2), kBW x kBH elements. x0 - kBOX keeps the box start
// 16-byte aligned for both precisions.
constexpr int kBOX = 4;
constexpr int kBW = kTX + 2 * kBOX;   // 72
constexpr int kBH = kTY + 4;          // 12
// Plane rows of the register-blocked apply kernels: y0 - 2 .. y0 + 7 (the
// backward entries reach two rows up; no plane is read below the tile).
constexpr int kPH = kTY + 2;          // 10
// Restriction tiles: kCX x CY coarse pixels; the fine box starts at
// (2 X0 - 4, 2 Y0 - 3) and is kBW x (2 CY + 5).
constexpr int kCX = 32;
// Prolongation: coarse box at (x0/2 - 4, y0/2 - 2), kCBW x kCBH.
constexpr int kCBW = 40;
constexpr int kCBH = 8;

#ifndef PMB_CY_FP32
#define PMB_CY_FP32 3
#endif
#ifndef PMB_CY_FP64
#define PMB_CY_FP64 3
#endif
template <typename T> struct Coarse {
    static constexpr int CY = sizeof(T) == 4 ? PMB_CY_FP32 : PMB_CY_FP64;
};

// TMA descriptor slots of one grid (see engine.cu for what each maps).
enum : int {
    kMapPlF = 0,   // planes, fine box (inner precision)
    kMapPlD,       // planes, restriction box
    kMapBF,        // level right-hand side b, fine box (r at level 0)
    kMapBD,        // b, restriction box
    kMapXC,        // level solution x as a coarse operand (z at level 0)
    kMapXF,        // x, fine box
    kMapXAF,       // smoothing ping-pong buffer A, fine box
    kMapXAD,       // buffer A, restriction box
    kMapXBF,       // smoothing ping-pong buffer B, fine box
    kMapXBD,       // buffer B, restriction box
    kMapZF,        // CG z, fine box (level 0)
    kMapP0F,       // CG p parity 0 (also x0 scratch), fine box
    kMapP1F,       // CG p parity 1, fine box
    kMapX64F,      // FP64 refinement iterate, fine box
    kMapP64F,      // FP64 planes, fine box (refinement residual)
    kMapPlS,       // planes, apply box (kPH rows)
    kMapPlDV,      // planes, register-blocked restriction box
    kMapBDV,       // b, register-blocked restriction box
    kMapPlG,       // FP64 planes, Galerkin box (42 x 21 x 13)
    kMapPlD0,      // plane 0, register-blocked restriction box (1 plane)
    kMapPlD1,      // planes 1..12, restriction box two rows shorter (loaded at plane 1)
    kMapPlU0,      // plane 0, prolongation box kBW x kBH (1 plane)
    kMapPlU1,      // planes 1..12, kBW x kPH (loaded at plane 1)
    kMapsPerGrid
};

__host__ __device__ constexpr int half_dy(int p) { return p < 3 ? 0 : (p < 8 ? 1 : 2); }
__host__ __device__ constexpr int half_dx(int p) { return p < 3 ? p : (p < 8 ? p - 5 : p - 10); }
// Plane index of forward offset (dy, dx); -1 if (dy, dx) is not forward.
__host__ __device__ constexpr int half_index(int dy, int dx) {
    return (dy == 0 && dx >= 0 && dx <= 2) ? dx
         : (dy == 1 && dx >= -2 && dx <= 2) ? 5 + dx
         : (dy == 2 && dx >= -2 && dx <= 2) ? 10 + dx : -1;
}

// One grid (an image, or one multigrid level of an image) inside a batch.
struct GridDesc {
    int h, w, pitch, inst;  // inst: index of the image in the batch
    int64_t voff;           // offset of element (0, 0) in the level's vectors
    int64_t poff;           // offset of plane 0 in the level's plane buffer
    int64_t pstride;        // elements between consecutive planes (h * pitch)
    int map_base;           // first TMA descriptor of this grid (kMapsPerGrid each)
    int pad_;
};

// Tiles of one tile shape over the grids of one level. Grid g owns the global
// tiles [tile_start[g], tile_start[g + 1]).
struct WorkList {
    const GridDesc* grids;
    const int* tile_start;
    int ngrids;
    int total;
};

// Per-image solver state, kept on the device so a whole iteration can be
// replayed from a CUDA graph without the host.
struct InstState {
    double rz;        // r . z of the current iterate
    double alpha;     // step length of the current iteration
    double beta;      // p <- z + beta p
    double norm_b;
    double norm_r;
    double tol;       // converged when norm_r < tol (tol = max(atol, rtol*|b|))
    double pap;       // p . Ap
    double aux;       // spare slot (outer residual of the refinement loop)
    int iters;        // completed iterations
    int status;       // kRunning / kConverged / kMaxIter / kNonFinite
    int maxiter;
    int flags;        // kFirst / kUpdate
    unsigned int counter;  // tiles finished in the current reduction
    int pad[3];
};

enum : int { kRunning = 0, kConverged = 1, kMaxIter = 2, kNonFinite = 3, kSkip = 4 };
// flags: kFirst — p = z on the next apply; kUpdate — the FP32 recurrence
// residual of a mixed-precision solve reached its phase tolerance and waits
// for the FP64 residual replacement of this iteration.
enum : int { kFirst = 1, kUpdate = 2 };
// Which images a gated loop visits: running ones, or running ones that
// wait for a residual replacement.
enum : int { kGateRunning = 0, kGateUpdate = 1 };
// Slot of the solver's error words (4 ints) that counts the images waiting
// for a residual replacement (slot 0 is the TMA timeout flag).
constexpr int kPendingSlot = 2;

__device__ __forceinline__ int find_grid(const WorkList& wl, int tile) {
    int lo = 0, hi = wl.ngrids - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (wl.tile_start[mid] <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename T> struct Acc { typedef double type; };

// Block-wide sum of up to 3 doubles; result valid in thread 0. Fixed tree
// order, so results are reproducible run to run.
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ], double* smem /* NQ*32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) smem[q * 32 + warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double t = lane < nwarps ? smem[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            v[q] = t;
        }
    }
}

// Deterministic two-stage reduction across the tiles of one image.
// Each tile stores its partial sums; the block that finishes the image's last
// tile adds all partials in tile order and runs `fin` (thread 0 only).
// Returns true in the block that ran the finaliser.
template <int NQ, typename Fin>
__device__ __forceinline__ bool tile_reduce(double (&v)[NQ], double* partials, int total,
                                            int tile, int t0, int t1, InstState* st,
                                            double* smem, Fin fin) {
    block_sum<NQ>(v, smem);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[(int64_t)q * total + tile] = v[q];
        __threadfence();
        unsigned int done = atomicAdd(&st->counter, 1u);
        last = (done == (unsigned int)(t1 - t0 - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        s[q] = 0.0;
        for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x)
            s[q] += __ldcg(partials + (int64_t)q * total + t);
    }
    block_sum<NQ>(s, smem);
    if (threadIdx.x == 0) {
        st->counter = 0u;
        fin(s);
    }
    __syncthreads();
    return true;
}

// Per-CTA variant for grid-stride tile loops. A CTA walking tiles t, t + G,
// t + 2G, ... (G = gridDim.x) accumulates its sums for one image and calls
// cta_flush once, after its last tile of that image. Partial sums live at
// partials[(inst * 3 + q) * G + cta]; the CTA that completes the image's tile
// count adds the partials of every CTA that owned one of its tiles, in CTA
// order, and runs `fin` (thread 0). Deterministic for a fixed grid size.
template <int NQ, typename Fin>
__device__ __forceinline__ void cta_flush(double (&v)[NQ], double* partials, int inst, int t0,
                                          int t1, unsigned int mine, InstState* st, double* smem,
                                          Fin fin) {
    const int G = gridDim.x;
    block_sum<NQ>(v, smem);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[((int64_t)inst * 3 + q) * G + blockIdx.x] = v[q];
        __threadfence();
        const unsigned int done = atomicAdd(&st->counter, mine);
        last = (done + mine == (unsigned int)(t1 - t0));
    }
    __syncthreads();
    if (last) {
        __threadfence();
        const int n = t1 - t0;
        double s[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            s[q] = 0.0;
            const double* p = partials + ((int64_t)inst * 3 + q) * G;
            if (n >= G) {
                for (int c = threadIdx.x; c < G; c += blockDim.x) s[q] += __ldcg(p + c);
            } else {
                // Fewer tiles than CTAs: tile t0 + k belonged to CTA (t0 + k) % G.
                for (int k = threadIdx.x; k < n; k += blockDim.x) s[q] += __ldcg(p + (t0 + k) % G);
            }
        }
        block_sum<NQ>(s, smem);
        if (threadIdx.x == 0) {
            st->counter = 0u;
            fin(s);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
}

}  // namespace pmb
