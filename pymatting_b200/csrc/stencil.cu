// Matrix-free half-stencil kernels: the soft-constraint system A = L + lambda D,
// the fused preconditioned conjugate-gradient steps, and the geometric
// multigrid V-cycle used as its preconditioner.
//
// Every stencil kernel works on 64 x 8 pixel tiles. One thread of the CTA
// issues TMA loads of the tile plus its halo: a single 3D box holds all 13
// operator planes (72 x 12 x 13), 2D boxes hold the vector operands; the
// hardware zero-fills everything outside the image, which supplies the
// stencil's border terms. The kernels then read operators and operands from
// shared memory only. Element-wise kernels stream kFlat-element chunks.
//
// Every kernel walks a WorkList of tiles over a batch of grids (images of
// different sizes, or the same multigrid level of several images) with a
// grid-stride loop, so one launch serves the whole batch. Per-image scalars
// (alpha, beta, norms, convergence status) live in InstState on the device;
// an image whose status is no longer "running" is skipped tile by tile.
//
// Reference algorithms restated here:
//   cg          pymatting/solver/cg.py:64-117
//   jacobi      pymatting/preconditioner/jacobi.py:24-31
//   V-cycle     pymatting/preconditioner/vcycle.py:6-100 (make_P weights
//               and border mask, jacobi_step, _vcycle_step)
#include "pm_common.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace pmb {

// --------------------------------------------------------------------------
// Tile helpers
// --------------------------------------------------------------------------

// Shared-memory carve-up with 128-byte alignment (TMA destinations).
struct SmemCarve {
    char* p;
    __device__ explicit SmemCarve(char* base) : p(base) {}
    template <typename T>
    __device__ T* take(int count) {
        T* r = reinterpret_cast<T*>(p);
        p += ((size_t)count * sizeof(T) + 127) & ~size_t(127);
        return r;
    }
};

extern __shared__ __align__(128) char g_smem[];

// The two pipeline copies of one shared buffer, addressed by stage index
// without a local-memory pointer array: copy b = p0 + b * d.
template <typename T>
struct Buf2 {
    T* p0;
    ptrdiff_t d;
    __device__ __forceinline__ T* operator[](int b) const { return p0 + b * d; }
};

// V-element vector load / store (8 or 16 bytes, aligned).
template <typename T, int V>
__device__ __forceinline__ void ldv(const T* p, T* o) {
    if constexpr (sizeof(T) == 4 && V == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
    } else if constexpr (sizeof(T) == 4 && V == 2) {
        const float2 q = *reinterpret_cast<const float2*>(p);
        o[0] = q.x; o[1] = q.y;
    } else {
        static_assert(sizeof(T) == 8 && V == 2, "unsupported vector");
        const double2 q = *reinterpret_cast<const double2*>(p);
        o[0] = q.x; o[1] = q.y;
    }
}

template <typename T, int V>
__device__ __forceinline__ void stv(T* p, const T* o) {
    if constexpr (sizeof(T) == 4 && V == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
    } else if constexpr (sizeof(T) == 4 && V == 2) {
        *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
    }
}


// Description of one tile, prepared by thread 0 for the whole CTA.
struct Meta {
    int t, g, y0, x0;     // tile, grid index in the list, tile origin
    int inst, t0, t1;     // image and its tile range in the list
    int run;              // 0: image not running, the tile is skipped
    int par, first;       // CG: iteration parity and first-pass flag
    double beta;          // CG: current beta
};

// Two mbarriers (one per pipeline buffer) and their phase bits.
struct Pipe {
    uint64_t* bar;
    uint32_t phase;
    int* err;
    __device__ void init(uint64_t* b, int* e) {
        bar = b;
        phase = 0;
        err = e;
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
        }
        __syncthreads();
    }
    // Wait for buffer b (bounded). Returns false if this thread gave up; the
    // caller records that and acts on it at its next block barrier.
    __device__ bool wait(int b) {
        const bool ok = mbar_wait(&bar[b], (phase >> b) & 1u);
        phase ^= 1u << b;
        return ok;
    }
    // After a wait that gave up (seen by the whole CTA at a barrier): thread
    // 0 sets the error flag and waits once more, again bounded, for the loads
    // that may still be in flight into buffer b (waited on last) and, if
    // other_issued, into the other buffer, so that the CTA does not exit
    // while a copy into its shared memory is pending.
    __device__ void drain(int b, bool other_issued) {
        if (threadIdx.x != 0) return;
        if (err) atomicExch(err, 1);
        mbar_wait(&bar[b], ((phase >> b) & 1u) ^ 1u);
        if (other_issued) mbar_wait(&bar[b ^ 1], (phase >> (b ^ 1)) & 1u);
    }
};

// Per-CTA directory of a work list in shared memory: tile starts, grid
// descriptors and the fields of each grid's image that the tile loops read
// (gate, CG parity, first-pass flag, beta). Loaded once per launch, so that
// the thread that prepares the next tile does no dependent global loads
// (a binary search over tile_start in global memory costs one L2 round trip
// per level). The image fields are stable for a launch: a kernel's own
// finaliser changes an image's fields only after all of that image's tiles
// are done. Lists of more than kDirGrids grids use global lookups.
constexpr int kDirGrids = 64;
struct TileDir {
    int n;                              // grids held (0: use the global list)
    int start[kDirGrids + 1];
    int run[kDirGrids];
    int par[kDirGrids];
    int first[kDirGrids];
    double beta[kDirGrids];
    GridDesc g[kDirGrids];
};

template <int GATE>
__device__ __forceinline__ void dir_load(TileDir& D, const WorkList& wl, const InstState* st) {
    const bool fits = wl.ngrids <= kDirGrids;
    if (fits) {
        for (int i = threadIdx.x; i <= wl.ngrids; i += blockDim.x) D.start[i] = wl.tile_start[i];
        for (int i = threadIdx.x; i < wl.ngrids; i += blockDim.x) {
            const GridDesc g = wl.grids[i];
            D.g[i] = g;
            int run = 1, par = 0, first = 0;
            double beta = 0.0;
            if (st) {
                const InstState& q = st[g.inst];
                run = q.status == kRunning && (GATE == kGateRunning || (q.flags & kUpdate) != 0);
                par = q.iters & 1;
                first = (q.flags & kFirst) != 0;
                beta = q.beta;
            }
            D.run[i] = run;
            D.par[i] = par;
            D.first[i] = first;
            D.beta[i] = beta;
        }
    }
    if (threadIdx.x == 0) D.n = fits ? wl.ngrids : 0;
    __syncthreads();
}

__device__ __forceinline__ int dir_find(const TileDir& D, int t) {
    int lo = 0, hi = D.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (D.start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ const CUtensorMap* map_of(const CUtensorMap* maps, const GridDesc& g,
                                                     int slot) {
    return maps + (size_t)g.map_base * kMapsPerGrid + slot;
}

// (A x) at the pixel whose box coordinates are (r, c): P is the 13-plane
// box (planes of kBW x ph elements), X the operand box (kBW wide). The
// backward entries A[i, i - d] are plane d at (r - dy, c - dx).
template <typename T>
__device__ __forceinline__ T stencil_at(const T* P, int ph, const T* X, int r, int c) {
    const int ps = ph * kBW;
    const int i = r * kBW + c;
    T acc = P[i] * X[i];
#pragma unroll
    for (int p = 1; p < kNH; ++p) {
        const int d = half_dy(p) * kBW + half_dx(p);
        acc += P[p * ps + i] * X[i + d];
        acc += P[p * ps + i - d] * X[i - d];
    }
    return acc;
}

// The pipelined tile loop shared by the TMA kernels. For every tile the CTA
// owns (t = blockIdx.x, + gridDim.x, ...): thread 0 prepares the meta of the
// next tile and issues its loads into the other buffer, then the CTA waits
// for the current buffer, runs `body`, and (for kernels with reductions)
// flushes its per-image partial sums after its last tile of an image.
//   issue(meta, gd, buf)            thread 0 only
//   body(meta, gd, buf)             all threads; returns nothing
//   flush(meta, mine)               all threads, after an image's last tile
// First tile >= t of this CTA's sequence (t = blockIdx.x mod gridDim.x)
// whose image is running (every image when st is null), or wl.total; *gout
// = its grid. Every tile of an image that is not running is skipped in one
// step per image.
template <int GATE>
__device__ __forceinline__ int next_running_tile(const TileDir& D, const WorkList& wl,
                                                 const InstState* st, int t, int* gout) {
    const int G = gridDim.x;
    while (t < wl.total) {
        int g, nxt;
        bool run;
        if (D.n) {
            g = dir_find(D, t);
            run = D.run[g] != 0;
            nxt = D.start[g + 1];
        } else {
            g = find_grid(wl, t);
            run = true;
            if (st) {
                const InstState& q = st[wl.grids[g].inst];
                run = q.status == kRunning && (GATE == kGateRunning || (q.flags & kUpdate) != 0);
            }
            nxt = wl.tile_start[g + 1];
        }
        if (run) {
            *gout = g;
            return t;
        }
        t += ((nxt - t + G - 1) / G) * G;
    }
    *gout = -1;
    return wl.total;
}

// Meta of tile t of grid g (from the directory when it holds the list).
template <int H, int W>
__device__ __forceinline__ void dir_meta(const TileDir& D, const WorkList& wl, const InstState* st,
                                         int t, int g, Meta& m, GridDesc& gd) {
    m.t = t;
    m.g = g;
    m.run = 1;
    if (D.n) {
        gd = D.g[g];
        m.t0 = D.start[g];
        m.t1 = D.start[g + 1];
        m.par = D.par[g];
        m.first = D.first[g];
        m.beta = D.beta[g];
    } else {
        gd = wl.grids[g];
        m.t0 = wl.tile_start[g];
        m.t1 = wl.tile_start[g + 1];
        m.par = 0;
        m.first = 0;
        m.beta = 0.0;
        if (st) {
            const InstState& q = st[gd.inst];
            m.par = q.iters & 1;
            m.first = (q.flags & kFirst) != 0;
            m.beta = q.beta;
        }
    }
    const int local = t - m.t0;
    const int tiles_x = (gd.w + W - 1) / W;
    const int ty = local / tiles_x;
    m.y0 = ty * H;
    m.x0 = (local - ty * tiles_x) * W;
    m.inst = gd.inst;
}

template <int H, int W, int GATE = kGateRunning, typename Issue, typename Body, typename Flush>
__device__ __forceinline__ void tile_loop(const WorkList& wl, const InstState* st, Pipe& pipe,
                                          Meta* s_m, GridDesc* s_g, Issue issue, Body body,
                                          Flush flush) {
    // Thread 0 walks the CTA's tiles through the directory, skipping every
    // tile of an image that is not running; the tile after the current one
    // is passed through s_t. A wait that gave up is recorded in s_abort and
    // acted on at the barrier that ends the tile.
    __shared__ TileDir D;
    __shared__ int s_t[2], s_abort;
    if (threadIdx.x == 0) s_abort = 0;
    dir_load<GATE>(D, wl, st);
    int b = 0;
    unsigned int mine = 0;
    if (threadIdx.x == 0) {
        int g0;
        const int t0 = next_running_tile<GATE>(D, wl, st, blockIdx.x, &g0);
        s_t[0] = t0;
        if (t0 < wl.total) {
            dir_meta<H, W>(D, wl, st, t0, g0, s_m[0], s_g[0]);
            fence_proxy_async();
            issue(s_m[0], s_g[0], 0);
        }
    }
    __syncthreads();
    int t = s_t[0];
    while (t < wl.total) {
        if (threadIdx.x == 0) {
            int gn;
            const int tn = next_running_tile<GATE>(D, wl, st, t + (int)gridDim.x, &gn);
            s_t[b ^ 1] = tn;
            if (tn < wl.total) {
                dir_meta<H, W>(D, wl, st, tn, gn, s_m[b ^ 1], s_g[b ^ 1]);
                fence_proxy_async();
                issue(s_m[b ^ 1], s_g[b ^ 1], b ^ 1);
            }
        }
        __syncthreads();
        const int tn = s_t[b ^ 1];
        const Meta m = s_m[b];
        if (!pipe.wait(b)) s_abort = 1;
        body(m, s_g[b], b);
        ++mine;
        const bool last_of_image = (tn >= wl.total) || (s_m[b ^ 1].inst != m.inst);
        if (last_of_image) {
            flush(m, mine);
            mine = 0;
        }
        __syncthreads();
        if (s_abort) {
            pipe.drain(b, tn < wl.total);
            return;
        }
        b ^= 1;
        t = tn;
    }
}

// Single-buffer variant of tile_loop: the tile's loads are issued when the
// previous tile is done, so a CTA has at most one tile in flight and needs
// half the shared memory; several CTAs per SM then overlap each other's
// loads and compute.
template <int H, int W, int GATE = kGateRunning, typename Issue, typename Body, typename Flush>
__device__ __forceinline__ void tile_loop1(const WorkList& wl, const InstState* st, Pipe& pipe,
                                           Meta* s_m, GridDesc* s_g, Issue issue, Body body,
                                           Flush flush) {
    __shared__ TileDir D;
    __shared__ int s_tn, s_gn, s_ninst, s_abort;   // the tile after the current one
    if (threadIdx.x == 0) s_abort = 0;
    dir_load<GATE>(D, wl, st);
    unsigned int mine = 0;
    if (threadIdx.x == 0) s_tn = next_running_tile<GATE>(D, wl, st, blockIdx.x, &s_gn);
    __syncthreads();
    int t = s_tn;
    int g = s_gn;
    __syncthreads();
    while (t < wl.total) {
        if (threadIdx.x == 0) {
            dir_meta<H, W>(D, wl, st, t, g, s_m[0], s_g[0]);
            fence_proxy_async();
            issue(s_m[0], s_g[0], 0);
            int gn;
            const int tn = next_running_tile<GATE>(D, wl, st, t + (int)gridDim.x, &gn);
            s_tn = tn;
            s_gn = gn;
            s_ninst = tn < wl.total ? (D.n ? D.g[gn].inst : wl.grids[gn].inst) : -1;
        }
        __syncthreads();
        const Meta m = s_m[0];
        const int tn = s_tn, gn = s_gn, ninst = s_ninst;
        if (!pipe.wait(0)) s_abort = 1;
        body(m, s_g[0], 0);
        ++mine;
        if (ninst != m.inst) {
            flush(m, mine);
            mine = 0;
        }
        __syncthreads();
        if (s_abort) {
            pipe.drain(0, false);
            return;
        }
        t = tn;
        g = gn;
    }
}

struct NoFlush {
    __device__ void operator()(const Meta&, unsigned int) const {}
};

// --------------------------------------------------------------------------
// Conjugate gradient steps (cg.py:64-117)
// --------------------------------------------------------------------------

__device__ __forceinline__ void finish_beta(InstState* st, double rz_new) {
    // First pass after the initial residual: only record r.z (cg.py:78-80).
    if (st->flags & kFirst) {
        st->rz = rz_new;
        return;
    }
    // beta = (1 / rz) * r.z  (cg.py:105-108)
    double beta = 1.0 / st->rz;
    beta *= rz_new;
    st->beta = beta;
    st->rz = rz_new;
}

// beta = ((r - r_old) . z) / rz when reorthogonalising (cg.py:102-104).
__device__ __forceinline__ void finish_beta_reorth(InstState* st, double rz_new, double dz) {
    if (st->flags & kFirst) {
        st->rz = rz_new;
        return;
    }
    st->beta = dz / st->rz;
    st->rz = rz_new;
}

// r = b - A x0 (or r = b), |b|, |r|, and for Jacobi / no preconditioner also
// z and r.z. Finaliser sets norm_b, tol, status (cg.py:64-80). x0 arrives in
// the p-parity-0 buffer (map slot kMapP0F).
template <typename T, int PREC, bool X0>
__global__ void __launch_bounds__(kTileThreads)
k_cg_init(WorkList wl, const CUtensorMap* maps, const T* __restrict__ P, const T* __restrict__ b,
          T* x, T* r, T* z, InstState* st, double* partials, double atol, double rtol,
          int maxiter, int* err) {
    __shared__ double s_red[3 * 32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sX_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = X0 ? sc.take<T>(kNH * kBH * kBW) : nullptr;
        sX_[k] = X0 ? sc.take<T>(kBH * kBW) : nullptr;
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sX{sX_[0], sX_[1] - sX_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    double v[3] = {0.0, 0.0, 0.0};
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        if (!X0) {
            // Nothing to stage: complete the phase with an empty arrival.
            mbar_expect_tx(&pipe.bar[bb], 0);
            return;
        }
        mbar_expect_tx(&pipe.bar[bb], (kNH + 1) * kBH * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlF), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, g, kMapP0F), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        {
            const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
            const int y = m.y0 + ly, xx = m.x0 + lx;
            if (y < g.h && xx < g.w) {
                const int64_t i = g.voff + (int64_t)y * g.pitch + xx;
                const T bi = b[i];
                T ri = bi;
                T d;
                if (X0) {
                    const int q = (ly + 2) * kBW + lx + kBOX;
                    ri = bi - stencil_at<T>(sP[bb], kBH, sX[bb], ly + 2, lx + kBOX);
                    x[i] = sX[bb][q];
                    d = sP[bb][q];
                } else {
                    x[i] = T(0);
                    d = P[g.poff + (int64_t)y * g.pitch + xx];
                }
                r[i] = ri;
                v[0] += (double)bi * (double)bi;
                v[1] += (double)ri * (double)ri;
                if (PREC == kPrecJacobi) {
                    const T zi = ri * (T(1) / d);
                    z[i] = zi;
                    v[2] += (double)ri * (double)zi;
                } else if (PREC == kPrecNone) {
                    v[2] += (double)ri * (double)ri;
                }
            }
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        InstState* s = st + m.inst;
        cta_flush<3>(v, partials, m.inst, m.t0, m.t1, mine, s, s_red, [&](double* sum) {
            s->norm_b = sqrt(sum[0]);
            s->norm_r = sqrt(sum[1]);
            s->tol = fmax(atol, rtol * s->norm_b);
            s->iters = 0;
            s->maxiter = maxiter;
            s->flags = kFirst;
            s->beta = 0.0;
            s->alpha = 0.0;
            if (s->norm_r < atol || s->norm_r < rtol * s->norm_b) s->status = kConverged;
            else if (maxiter <= 0) s->status = kMaxIter;
            else s->status = kRunning;
            if (PREC != kPrecVcycle && PREC != kPrecExternal) s->rz = sum[2];
        });
    };
    // Every image starts from scratch: its tiles run whatever its status.
    tile_loop<kTY, kTX>(wl, nullptr, pipe, s_m, s_g, issue, body, flush);
}

// p_new = z + beta p_old (p_new = z on the first pass), Ap = A p_new and
// p_new . Ap; finaliser: alpha = rz / (p . Ap)   (cg.py:85-90, 111-113).
// p is double-buffered by iteration parity: neighbouring tiles still read
// p_old while this tile writes p_new. zslot selects z (r without a
// preconditioner).
template <typename T>
__global__ void __launch_bounds__(kTileThreads)
k_cg_apply(WorkList wl, const CUtensorMap* maps, int zslot, T* p0, T* p1, T* Ap, InstState* st,
           double* partials, int* err) {
    __shared__ double s_red[32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sZ_[2];
    T* sQ_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<T>(kNH * kBH * kBW);
        sZ_[k] = sc.take<T>(kBH * kBW);
        sQ_[k] = sc.take<T>(kBH * kBW);
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sZ{sZ_[0], sZ_[1] - sZ_[0]};
    const Buf2<T> sQ{sQ_[0], sQ_[1] - sQ_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    double v[1] = {0.0};
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        mbar_expect_tx(&pipe.bar[bb], (kNH + (m.first ? 1 : 2)) * kBH * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlF), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sZ[bb], map_of(maps, g, zslot), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
        if (!m.first)
            tma_load_2d(sQ[bb], map_of(maps, g, m.par ? kMapP1F : kMapP0F), m.x0 - kBOX, m.y0 - 2,
                        &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        T* Z = sZ[bb];
        if (!m.first) {
            const T beta = (T)m.beta;
            const T* Q = sQ[bb];
            for (int q = threadIdx.x; q < kBH * kBW; q += blockDim.x) Z[q] = Z[q] + beta * Q[q];
            __syncthreads();
        }
        T* pnew = m.par ? p0 : p1;
        {
            const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
            const int y = m.y0 + ly, x = m.x0 + lx;
            if (y < g.h && x < g.w) {
                const int64_t i = g.voff + (int64_t)y * g.pitch + x;
                const T pi = Z[(ly + 2) * kBW + lx + kBOX];
                const T api = stencil_at<T>(sP[bb], kBH, Z, ly + 2, lx + kBOX);
                pnew[i] = pi;
                Ap[i] = api;
                v[0] += (double)pi * (double)api;
            }
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        InstState* s = st + m.inst;
        cta_flush<1>(v, partials, m.inst, m.t0, m.t1, mine, s, s_red, [&](double* sum) {
            s->pap = sum[0];
            s->alpha = s->rz / sum[0];
            s->flags &= ~kFirst;
        });
    };
    tile_loop<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
}

// Element-wise loop over a flat work list (kFlat-element chunks) with the same
// per-CTA, per-image flush as the tiled kernels. Chunks cover the pitched
// rows; padding columns are skipped.
template <int GATE = kGateRunning, typename Body, typename Flush>
__device__ __forceinline__ void flat_loop(const WorkList& wl, const InstState* st, Body body,
                                          Flush flush) {
    // Thread 0 walks the CTA's chunks through the list's directory,
    // skipping every chunk of an image that is not running.
    __shared__ TileDir D;
    __shared__ int s_inst[2], s_t0, s_t1, s_next, s_gnext;
    __shared__ GridDesc s_gd;
    dir_load<GATE>(D, wl, st);
    unsigned int mine = 0;
    if (threadIdx.x == 0) s_next = next_running_tile<GATE>(D, wl, st, blockIdx.x, &s_gnext);
    __syncthreads();
    for (int t = s_next; t < wl.total; t = s_next) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int g = s_gnext;
            s_gd = D.n ? D.g[g] : wl.grids[g];
            s_t0 = D.n ? D.start[g] : wl.tile_start[g];
            s_t1 = D.n ? D.start[g + 1] : wl.tile_start[g + 1];
            s_inst[0] = s_gd.inst;
            int gn;
            const int tn = next_running_tile<GATE>(D, wl, st, t + (int)gridDim.x, &gn);
            s_next = tn;
            s_gnext = gn;
            s_inst[1] = tn < wl.total ? (D.n ? D.g[gn].inst : wl.grids[gn].inst) : -1;
        }
        __syncthreads();
        const GridDesc g = s_gd;
        const int64_t n = (int64_t)g.h * g.pitch;
        const int64_t e0 = (int64_t)(t - s_t0) * kFlat;
        const int64_t e1 = min(e0 + kFlat, n);
        body(g, e0, e1);
        ++mine;
        if (s_inst[1] != s_inst[0]) {
            flush(s_inst[0], s_t0, s_t1, mine);
            mine = 0;
        }
        __syncthreads();
    }
}

// x += alpha p; r -= alpha Ap; |r|; convergence test (cg.py:89-99). For the
// Jacobi / identity preconditioners also z = M r and beta (cg.py:101-113).
// With reorthogonalisation the change r - r_old is kept in `dr` (or reduced
// directly against z for Jacobi).
template <typename T, int PREC>
__global__ void __launch_bounds__(kThreads)
k_cg_update(WorkList wl, const T* __restrict__ P, T* x, T* r, T* z, const T* p0, const T* p1,
            const T* __restrict__ Ap, T* dr, int reorth, int reliable, int* pending, InstState* st,
            double* partials) {
    constexpr int VE = 16 / sizeof(T);          // elements per 16-byte vector
    __shared__ double s_red[3 * 32];
    double v[3] = {0.0, 0.0, 0.0};
    auto body = [&](const GridDesc& g, int64_t e0, int64_t e1) {
        const InstState& s = st[g.inst];
        const T a = (T)s.alpha;
        const T* p = (s.iters & 1) ? p0 : p1;   // the buffer k_cg_apply wrote
        // Vectors never straddle rows (the pitch is a multiple of 32); padding
        // lanes keep their values.
#pragma unroll
        for (int k = 0; k < kFlat / (kThreads * VE); ++k) {
            const int64_t e = e0 + (int64_t)(threadIdx.x + k * kThreads) * VE;
            if (e >= e1) break;
            const int col0 = (int)(e % g.pitch);
            if (col0 >= g.w) continue;
            const int64_t i = g.voff + e;
            T xv[VE], rv[VE], pv[VE], av[VE], zv[VE], dv[VE], drv[VE];
            ldv<T, VE>(x + i, xv);
            ldv<T, VE>(r + i, rv);
            ldv<T, VE>(p + i, pv);
            ldv<T, VE>(Ap + i, av);
            if (PREC == kPrecJacobi) {
                const int row = (int)(e / g.pitch);
                ldv<T, VE>(P + g.poff + (int64_t)row * g.pitch + col0, dv);
                ldv<T, VE>(z + i, zv);
            }
            if (PREC == kPrecVcycle && reorth) ldv<T, VE>(dr + i, drv);
#pragma unroll
            for (int u = 0; u < VE; ++u) {
                if (col0 + u >= g.w) continue;
                const T rold = rv[u];
                xv[u] = xv[u] + a * pv[u];
                const T ri = rold - a * av[u];
                rv[u] = ri;
                v[0] += (double)ri * (double)ri;
                if (PREC == kPrecJacobi) {
                    const T zi = ri * (T(1) / dv[u]);
                    zv[u] = zi;
                    v[1] += (double)ri * (double)zi;
                    if (reorth) v[2] += (double)(ri - rold) * (double)zi;
                } else if (PREC == kPrecNone) {
                    v[1] += (double)ri * (double)ri;
                    if (reorth) v[2] += (double)(ri - rold) * (double)ri;
                } else if (reorth) {
                    drv[u] = ri - rold;
                }
            }
            stv<T, VE>(x + i, xv);
            stv<T, VE>(r + i, rv);
            if (PREC == kPrecJacobi) stv<T, VE>(z + i, zv);
            if (PREC == kPrecVcycle && reorth) stv<T, VE>(dr + i, drv);
        }
    };
    auto flush = [&](int inst, int t0, int t1, unsigned int mine) {
        InstState* s = st + inst;
        cta_flush<3>(v, partials, inst, t0, t1, mine, s, s_red, [&](double* sum) {
            const double nr = sqrt(sum[0]);
            s->norm_r = nr;
            s->iters += 1;
            if (!isfinite(nr)) s->status = kNonFinite;
            else if (nr < s->tol) {
                // Mixed precision: the phase ends with an FP64 residual
                // replacement (k_refine_residual, same iteration), which also
                // finishes beta; otherwise the solve has converged.
                if (reliable) {
                    s->flags |= kUpdate;
                    atomicAdd(pending, 1);
                } else {
                    s->status = kConverged;
                }
            } else if (s->iters >= s->maxiter) s->status = kMaxIter;
            if (s->status == kRunning && !(s->flags & kUpdate) &&
                (PREC == kPrecJacobi || PREC == kPrecNone)) {
                if (reorth) finish_beta_reorth(s, sum[1], sum[2]);
                else finish_beta(s, sum[1]);
            }
        });
    };
    flat_loop(wl, st, body, flush);
}

// r . z (and (r - r_old) . z) for preconditioners applied outside the fused
// kernels; finaliser computes beta.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_cg_rz(WorkList wl, const T* __restrict__ r, const T* __restrict__ z, const T* __restrict__ dr,
        int reorth, InstState* st, double* partials) {
    __shared__ double s_red[2 * 32];
    double v[2] = {0.0, 0.0};
    auto body = [&](const GridDesc& g, int64_t e0, int64_t e1) {
#pragma unroll
        for (int k = 0; k < kFlat / kThreads; ++k) {
            const int64_t e = e0 + threadIdx.x + k * kThreads;
            if (e >= e1) break;
            if ((int)(e % g.pitch) >= g.w) continue;
            const int64_t i = g.voff + e;
            v[0] += (double)r[i] * (double)z[i];
            if (reorth) v[1] += (double)dr[i] * (double)z[i];
        }
    };
    auto flush = [&](int inst, int t0, int t1, unsigned int mine) {
        InstState* s = st + inst;
        cta_flush<2>(v, partials, inst, t0, t1, mine, s, s_red, [&](double* sum) {
            if (reorth) finish_beta_reorth(s, sum[0], sum[1]);
            else finish_beta(s, sum[0]);
        });
    };
    flat_loop(wl, st, body, flush);
}

// --------------------------------------------------------------------------
// V-cycle (vcycle.py:46-100)
// --------------------------------------------------------------------------

__device__ __forceinline__ double pw(int a) { return a == 0 ? 2.0 : 1.0; }

// Restriction of the pre-smoothed residual. One tile = kCX x CY coarse
// pixels:
//   x1 = omega b / d         (first Jacobi sweep from zero, vcycle.py:33-36)
//        or x1 = 0 (no pre-smoothing) or x1 = xs (explicit sweeps);
//   res = b - A x1 on the fine pixels under the tile (vcycle.py:77);
//   b_coarse = R res with full-weighting [1 2 1]^2 / 16 (vcycle.py:12-26, 80).
// The fine box starts at (2 X0 - 4, 2 Y0 - 3): rows 2 Y0 - 3 .. 2 Y0 + 2 CY + 1
// cover x1 around the residual rows 2 Y0 - 1 .. 2 Y0 + 2 CY - 1.
template <typename T, int PRE>
__global__ void __launch_bounds__(kTileThreads)
k_vc_down(WorkList wl /* coarse tiles */, const GridDesc* fine, const CUtensorMap* maps,
          int xs_slot, T* bc, double omega, const InstState* st, int* err) {
    constexpr int CY = Coarse<T>::CY;
    constexpr int DH = 2 * CY + 5;                      // box rows
    constexpr int RH = 2 * CY + 1, RW = 2 * kCX + 1;    // residual region
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sB_[2];
    T* sS_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = PRE != 0 ? sc.take<T>(kNH * DH * kBW) : nullptr;
        sB_[k] = sc.take<T>(DH * kBW);
        sS_[k] = PRE > 1 ? sc.take<T>(DH * kBW) : nullptr;
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sB{sB_[0], sB_[1] - sB_[0]};
    const Buf2<T> sS{sS_[0], sS_[1] - sS_[0]};
    T* sX = PRE == 1 ? sc.take<T>(DH * kBW) : nullptr;
    T* sR = sc.take<T>(RH * RW);
    Pipe pipe;
    pipe.init(s_bar, err);
    auto issue = [&](const Meta& m, const GridDesc& gc, int bb) {
        const GridDesc gf = fine[m.g];
        const int bx = 2 * m.x0 - 4, by = 2 * m.y0 - 3;
        const uint32_t nbox = 1 + (PRE != 0 ? kNH : 0) + (PRE > 1 ? 1 : 0);
        mbar_expect_tx(&pipe.bar[bb], nbox * DH * kBW * sizeof(T));
        tma_load_2d(sB[bb], map_of(maps, gf, kMapBD), bx, by, &pipe.bar[bb]);
        if (PRE != 0) tma_load_3d(sP[bb], map_of(maps, gf, kMapPlD), bx, by, 0, &pipe.bar[bb]);
        if (PRE > 1) tma_load_2d(sS[bb], map_of(maps, gf, xs_slot), bx, by, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& gc, int bb) {
        const GridDesc gf = fine[m.g];
        const int bx = 2 * m.x0 - 4, by = 2 * m.y0 - 3;
        const T* B = sB[bb];
        const T* X1 = PRE > 1 ? sS[bb] : sX;
        if (PRE == 1) {
            // x1 = omega b / d inside the image, 0 outside.
            for (int q = threadIdx.x; q < DH * kBW; q += blockDim.x) {
                const int rr = q / kBW, cc = q - rr * kBW;
                const int fy = by + rr, fx = bx + cc;
                T v = T(0);
                if (fy >= 0 && fy < gf.h && fx >= 0 && fx < gf.w) v = (T)omega * B[q] / sP[bb][q];
                sX[q] = v;
            }
            __syncthreads();
        }
        for (int q = threadIdx.x; q < RH * RW; q += blockDim.x) {
            const int rr = q / RW, cc = q - rr * RW;
            const int br = rr + 2, bcol = cc + 3;           // box coordinates
            const int fy = by + br, fx = bx + bcol;
            T v = T(0);
            if (fy >= 0 && fy < gf.h && fx >= 0 && fx < gf.w) {
                v = B[br * kBW + bcol];
                if (PRE != 0) v = v - stencil_at<T>(sP[bb], DH, X1, br, bcol);
            }
            sR[q] = v;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < kCX * CY; q += blockDim.x) {
            const int ly = q / kCX, lx = q - ly * kCX;
            const int Y = m.y0 + ly, X = m.x0 + lx;
            if (Y < gc.h && X < gc.w) {
                T sum = T(0);
#pragma unroll
                for (int ay = -1; ay <= 1; ++ay)
#pragma unroll
                    for (int ax = -1; ax <= 1; ++ax)
                        sum += (T)(pw(ax) * pw(ay) / 16.0) *
                               sR[(2 * ly + 1 + ay) * RW + (2 * lx + 1 + ax)];
                bc[gc.voff + (int64_t)Y * gc.pitch + X] = sum;
            }
        }
    };
    tile_loop<CY, kCX>(wl, st, pipe, s_m, s_g, issue, body, NoFlush());
}

// Prolongation of the coarse correction and the first post-smoothing sweep:
//   x2 = x1 + P xc           (vcycle.py:95; P = R^T)
//   x3 = x2 + omega (b - A x2) / d    (vcycle.py:98, one sweep; POST = 0
//                                       stores x2 unchanged)
// At level 0 (level0 != 0) the CTA also accumulates r . z with r = b, and
// (r - r_old) . z when reorthogonalising, finishing beta.
template <typename T, int PRE, int POST>
__global__ void __launch_bounds__(kTileThreads)
k_vc_up(WorkList wl /* fine tiles */, const GridDesc* coarse, const CUtensorMap* maps,
        int xs_slot, const T* __restrict__ b, T* xout, double omega, InstState* st, int level0,
        const T* __restrict__ dr, int reorth, double* partials, int* err) {
    __shared__ double s_red[2 * 32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sX_[2];
    T* sS_[2];
    T* sC_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<T>(kNH * kBH * kBW);
        sX_[k] = sc.take<T>(kBH * kBW);          // b, then x2 in place
        sS_[k] = PRE > 1 ? sc.take<T>(kBH * kBW) : nullptr;
        sC_[k] = sc.take<T>(kCBH * kCBW);
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sX{sX_[0], sX_[1] - sX_[0]};
    const Buf2<T> sS{sS_[0], sS_[1] - sS_[0]};
    const Buf2<T> sC{sC_[0], sC_[1] - sC_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    double v[2] = {0.0, 0.0};
    auto issue = [&](const Meta& m, const GridDesc& gf, int bb) {
        const GridDesc gc = coarse[m.g];
        const int bx = m.x0 - kBOX, by = m.y0 - 2;
        const int cx0 = (m.x0 >> 1) - 4, cy0 = (m.y0 >> 1) - 2;
        mbar_expect_tx(&pipe.bar[bb], ((kNH + 1 + (PRE > 1 ? 1 : 0)) * kBH * kBW + kCBH * kCBW) *
                                          sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, gf, kMapPlF), bx, by, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, gf, kMapBF), bx, by, &pipe.bar[bb]);
        if (PRE > 1) tma_load_2d(sS[bb], map_of(maps, gf, xs_slot), bx, by, &pipe.bar[bb]);
        tma_load_2d(sC[bb], map_of(maps, gc, kMapXC), cx0, cy0, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& gf, int bb) {
        const GridDesc gc = coarse[m.g];
        const int bx = m.x0 - kBOX, by = m.y0 - 2;
        const int cx0 = (m.x0 >> 1) - 4, cy0 = (m.y0 >> 1) - 2;
        T* X = sX[bb];
        const T* Pl = sP[bb];
        const T* C = sC[bb];
        // Each element is read and rewritten by the same thread: no hazard.
        for (int q = threadIdx.x; q < kBH * kBW; q += blockDim.x) {
            const int rr = q / kBW, cc = q - rr * kBW;
            const int y = by + rr, x = bx + cc;
            T val = T(0);
            if (y >= 0 && y < gf.h && x >= 0 && x < gf.w) {
                T x1 = T(0);
                if (PRE == 1) x1 = (T)omega * X[q] / Pl[q];
                else if (PRE > 1) x1 = sS[bb][q];
                // Coarse pixels whose 3x3 support contains (y, x), in raster
                // order of the coarse grid: an even coordinate has one parent
                // (weight 2), an odd one the two neighbours (weight 1 each);
                // parents outside the coarse grid contribute nothing.
                const int Ya = (y - 1) >> 1, Xa = (x - 1) >> 1;   // first parent candidate
                const bool ey = (y & 1) == 0, ex = (x & 1) == 0;
                T sum = T(0);
#pragma unroll
                for (int jy = 0; jy < 2; ++jy) {
                    const int Y = ey ? (y >> 1) : Ya + jy;
                    if ((ey && jy == 1) || Y >= gc.h) continue;
                    const double wy = ey ? 2.0 : 1.0;
#pragma unroll
                    for (int jx = 0; jx < 2; ++jx) {
                        const int Xc = ex ? (x >> 1) : Xa + jx;
                        if ((ex && jx == 1) || Xc >= gc.w) continue;
                        const double wx = ex ? 2.0 : 1.0;
                        sum += (T)(wx * wy / 16.0) * C[(Y - cy0) * kCBW + (Xc - cx0)];
                    }
                }
                val = x1 + sum;
            }
            X[q] = val;
        }
        __syncthreads();
        {
            const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
            const int y = m.y0 + ly, x = m.x0 + lx;
            if (y < gf.h && x < gf.w) {
                const int64_t i = gf.voff + (int64_t)y * gf.pitch + x;
                const int q = (ly + 2) * kBW + lx + kBOX;
                T x3 = X[q];
                const T bi = b[i];
                if (POST > 0) {
                    const T ax = stencil_at<T>(Pl, kBH, X, ly + 2, lx + kBOX);
                    x3 = x3 + (T)omega * (bi - ax) / Pl[q];
                }
                xout[i] = x3;
                if (level0) {
                    v[0] += (double)bi * (double)x3;
                    if (reorth) v[1] += (double)dr[i] * (double)x3;
                }
            }
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        if (!level0 || !st) return;
        InstState* s = st + m.inst;
        cta_flush<2>(v, partials, m.inst, m.t0, m.t1, mine, s, s_red, [&](double* sum) {
            if (reorth) finish_beta_reorth(s, sum[0], sum[1]);
            else finish_beta(s, sum[0]);
        });
    };
    tile_loop<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
}

// One weighted Jacobi sweep xout = xin + omega (b - A xin) / d, or the first
// sweep from zero xout = omega b / d when xin_slot < 0 (vcycle.py:32-43).
template <typename T>
__global__ void __launch_bounds__(kTileThreads)
k_vc_smooth(WorkList wl, const CUtensorMap* maps, int xin_slot, const T* __restrict__ P,
            const T* __restrict__ b, T* xout, double omega, const InstState* st, int* err) {
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sX_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<T>(kNH * kBH * kBW);
        sX_[k] = sc.take<T>(kBH * kBW);
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sX{sX_[0], sX_[1] - sX_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        if (xin_slot < 0) {
            mbar_expect_tx(&pipe.bar[bb], 0);
            return;
        }
        mbar_expect_tx(&pipe.bar[bb], (kNH + 1) * kBH * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlF), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, g, xin_slot), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        {
            const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
            const int y = m.y0 + ly, x = m.x0 + lx;
            if (y < g.h && x < g.w) {
                const int64_t i = g.voff + (int64_t)y * g.pitch + x;
                T out;
                if (xin_slot >= 0) {
                    const int q = (ly + 2) * kBW + lx + kBOX;
                    const T ax = stencil_at<T>(sP[bb], kBH, sX[bb], ly + 2, lx + kBOX);
                    out = sX[bb][q] + (T)omega * (b[i] - ax) / sP[bb][q];
                } else {
                    out = (T)omega * b[i] / P[g.poff + (int64_t)y * g.pitch + x];
                }
                xout[i] = out;
            }
        }
    };
    tile_loop<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, NoFlush());
}

// Coarsest level: x = A^{-1} b with the inverse precomputed per image
// (replaces scipy.sparse.linalg.spsolve at vcycle.py:59-60). One CTA per
// image; the rz reduction runs when the coarsest level is level 0.
template <typename T>
__global__ void k_vc_direct(const DirectDesc* dd, int count, const T* __restrict__ b, T* x,
                            InstState* st, int rz_level0) {
    if ((int)blockIdx.x >= count) return;
    const DirectDesc d = dd[blockIdx.x];
    InstState* s = st ? st + d.g.inst : nullptr;
    if (s && s->status != kRunning) return;
    const int n = d.g.h * d.g.w;
    __shared__ double s_b[kMaxDirect];
    __shared__ double s_red[32];
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const int yy = q / d.g.w, xx = q - yy * d.g.w;
        s_b[q] = (double)b[d.g.voff + (int64_t)yy * d.g.pitch + xx];
    }
    __syncthreads();
    double v[1] = {0.0};
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const double* row = d.inv + (int64_t)q * n;
        double acc = 0.0;
        for (int j = 0; j < n; ++j) acc += row[j] * s_b[j];
        const int yy = q / d.g.w, xx = q - yy * d.g.w;
        x[d.g.voff + (int64_t)yy * d.g.pitch + xx] = (T)acc;
        if (rz_level0) v[0] += s_b[q] * (double)(T)acc;
    }
    if (rz_level0 && s) {
        block_sum<1>(v, s_red);
        if (threadIdx.x == 0) finish_beta(s, v[0]);
    }
}

// y = A x on pitched vectors (no reductions): used by A.dot(x) and by the
// benchmark's apply timing. x is the level-0 b buffer (map slot kMapBF).
template <typename T>
__global__ void __launch_bounds__(kTileThreads)
k_apply(WorkList wl, const CUtensorMap* maps, T* y, int* err) {
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sX_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<T>(kNH * kBH * kBW);
        sX_[k] = sc.take<T>(kBH * kBW);
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sX{sX_[0], sX_[1] - sX_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        mbar_expect_tx(&pipe.bar[bb], (kNH + 1) * kBH * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlF), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, g, kMapBF), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        {
            const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
            const int yy = m.y0 + ly, xx = m.x0 + lx;
            if (yy < g.h && xx < g.w)
                y[g.voff + (int64_t)yy * g.pitch + xx] =
                    stencil_at<T>(sP[bb], kBH, sX[bb], ly + 2, lx + kBOX);
        }
    };
    tile_loop<kTY, kTX>(wl, nullptr, pipe, s_m, s_g, issue, body, NoFlush());
}

// --------------------------------------------------------------------------
// Setup: Galerkin coarse operator, dense coarsest inverse, precision copies
// --------------------------------------------------------------------------

// Entry A[i, i + e] of a half-stencil operator for any |e| <= 2.
__device__ __forceinline__ double half_entry(const double* Pg, const GridDesc& g, int y, int x,
                                             int ey, int ex) {
    const int yj = y + ey, xj = x + ex;
    if (yj < 0 || yj >= g.h || xj < 0 || xj >= g.w) return 0.0;
    int p = half_index(ey, ex);
    if (p >= 0) return Pg[p * g.pstride + (int64_t)y * g.pitch + x];
    p = half_index(-ey, -ex);
    return Pg[p * g.pstride + (int64_t)yj * g.pitch + xj];
}

// Coarse operator R A P (vcycle.py:65) for one coarse pixel and forward
// offset D: sum over the 3x3 restriction support a of I and b of I + D of
// w_a w_b A[fa, fb]. One thread per (coarse pixel, forward offset).
__global__ void k_galerkin(const GridDesc* fine_g, const GridDesc* coarse_g, int ngrids,
                           const double* __restrict__ Pf, double* Pc, int64_t total) {
    int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int g = 0;
    int64_t base = 0;
    for (; g < ngrids; ++g) {
        const int64_t cnt = (int64_t)coarse_g[g].h * coarse_g[g].w * kNH;
        if (idx < base + cnt) break;
        base += cnt;
    }
    const GridDesc gf = fine_g[g], gc = coarse_g[g];
    const int64_t local = idx - base;
    const int p = (int)(local % kNH);
    const int64_t pix = local / kNH;
    const int Y = (int)(pix / gc.w), X = (int)(pix % gc.w);
    const int DY = half_dy(p), DX = half_dx(p);
    double acc = 0.0;
    const int Y2 = Y + DY, X2 = X + DX;
    if (Y2 >= 0 && Y2 < gc.h && X2 >= 0 && X2 < gc.w) {
        const double* Pg = Pf + gf.poff;
        for (int ay = -1; ay <= 1; ++ay) {
            for (int ax = -1; ax <= 1; ++ax) {
                const int fy = 2 * Y + ay, fx = 2 * X + ax;
                if (fy < 0 || fy >= gf.h || fx < 0 || fx >= gf.w) continue;
                const double wa = pw(ax) * pw(ay) / 16.0;
                for (int by = -1; by <= 1; ++by) {
                    for (int bx = -1; bx <= 1; ++bx) {
                        const int gy = 2 * Y2 + by, gx = 2 * X2 + bx;
                        if (gy < 0 || gy >= gf.h || gx < 0 || gx >= gf.w) continue;
                        const int ey = gy - fy, ex = gx - fx;
                        if (ey < -2 || ey > 2 || ex < -2 || ex > 2) continue;
                        const double wb = pw(bx) * pw(by) / 16.0;
                        acc += wa * half_entry(Pg, gf, fy, fx, ey, ex) * wb;
                    }
                }
            }
        }
    }
    Pc[gc.poff + p * gc.pstride + (int64_t)Y * gc.pitch + X] = acc;
}

// Tiled coarse operator: one CTA per 8x16 tile of coarse pixels, one thread
// per coarse pixel computing its 13 forward entries. One TMA box brings the
// fine planes under the tile (rows 2 Y0 - 1 .. 2 Y0 + 19, columns
// 2 X0 - 6 .. 2 X0 + 35) into shared memory, zero-filled outside the fine
// grid; the zeros stand in for the bounds tests of k_galerkin (entries of A
// that leave the grid are zero in the planes, so the terms they would skip
// add +0). Same terms in the same order as k_galerkin: bit-identical planes.
constexpr int kGTY = kGalerkinTileY, kGTX = kGalerkinTileX;   // coarse tile
constexpr int kGThreads = kGTY * kGTX;

template <int P>
__device__ __forceinline__ double galerkin_entry(const double* s_pl, int ly, int lx) {
    constexpr int DY = half_dy(P), DX = half_dx(P);
    double acc = 0.0;
#pragma unroll
    for (int ay = -1; ay <= 1; ++ay) {
#pragma unroll
        for (int ax = -1; ax <= 1; ++ax) {
            const double wa = pw(ax) * pw(ay) / 16.0;
            const int r = 2 * ly + 1 + ay, c = 2 * lx + 6 + ax;   // a = (2Y + ay, 2X + ax)
#pragma unroll
            for (int by = -1; by <= 1; ++by) {
#pragma unroll
                for (int bx = -1; bx <= 1; ++bx) {
                    const int ey = 2 * DY + by - ay, ex = 2 * DX + bx - ax;
                    if (ey < -2 || ey > 2 || ex < -2 || ex > 2) continue;
                    const double wb = pw(bx) * pw(by) / 16.0;
                    const int pf = half_index(ey, ex);
                    const double v = pf >= 0
                        ? s_pl[(pf * kGRows + r) * kGCols + c]
                        : s_pl[(half_index(-ey, -ex) * kGRows + r + ey) * kGCols + c + ex];
                    acc += wa * v * wb;
                }
            }
        }
    }
    return acc;
}

template <int P>
__device__ __forceinline__ void galerkin_all(const double* s_pl, int ly, int lx, int Y, int X,
                                             const GridDesc& gc, double* Pc) {
    if constexpr (P < kNH) {
        constexpr int DY = half_dy(P), DX = half_dx(P);
        const int Y2 = Y + DY, X2 = X + DX;
        double acc = 0.0;
        if (Y2 >= 0 && Y2 < gc.h && X2 >= 0 && X2 < gc.w) acc = galerkin_entry<P>(s_pl, ly, lx);
        Pc[gc.poff + P * gc.pstride + (int64_t)Y * gc.pitch + X] = acc;
        galerkin_all<P + 1>(s_pl, ly, lx, Y, X, gc, Pc);
    }
}

__global__ void __launch_bounds__(kGThreads)
k_galerkin_t(WorkList wl /* coarse tiles */, const GridDesc* fine, const CUtensorMap* maps,
             double* Pc, int* err) {
    extern __shared__ __align__(128) double s_pl[];      // [kNH][kGRows][kGCols]
    __shared__ __align__(8) uint64_t s_bar;
    const int t = blockIdx.x;
    const int g = find_grid(wl, t);
    const GridDesc gc = wl.grids[g];
    const int local = t - wl.tile_start[g];
    const int tiles_x = (gc.w + kGTX - 1) / kGTX;
    const int Y0 = (local / tiles_x) * kGTY, X0 = (local % tiles_x) * kGTX;
    if (threadIdx.x == 0) {
        const GridDesc gf = fine[g];
        mbar_init(&s_bar, 1);
        mbar_expect_tx(&s_bar, kNH * kGRows * kGCols * sizeof(double));
        tma_load_3d(s_pl, map_of(maps, gf, kMapPlG), 2 * X0 - 6, 2 * Y0 - 1, 0, &s_bar);
    }
    __syncthreads();
    const bool ok = mbar_wait(&s_bar, 0);
    if (__syncthreads_or(!ok)) {
        // Report, and wait (bounded) for the copy still in flight.
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            if (!ok) mbar_wait(&s_bar, 0);
        }
        return;
    }
    const int ly = threadIdx.x / kGTX, lx = threadIdx.x % kGTX;
    const int Y = Y0 + ly, X = X0 + lx;
    if (Y >= gc.h || X >= gc.w) return;
    galerkin_all<0>(s_pl, ly, lx, Y, X, gc, Pc);
}

// Dense inverse of the coarsest operator by Gauss-Jordan elimination with
// partial pivoting. One CTA per image; n <= kMaxDirect. *status is raised to
// 2 on an exactly zero pivot and to 1 on a non-finite one.
__global__ void k_dense_inverse(const DirectDesc* dd, int count, double* work, int* status) {
    if ((int)blockIdx.x >= count) return;
    const DirectDesc d = dd[blockIdx.x];
    const double* __restrict__ Pc = d.P;
    const GridDesc g = d.g;
    const int n = g.h * g.w;
    double* A = work + d.work_off;
    double* Inv = d.inv;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q / n, j = q - i * n;
        const int yi = i / g.w, xi = i - yi * g.w, yj = j / g.w, xj = j - yj * g.w;
        const int ey = yj - yi, ex = xj - xi;
        double v = 0.0;
        if (ey >= -2 && ey <= 2 && ex >= -2 && ex <= 2) v = half_entry(Pc + g.poff, g, yi, xi, ey, ex);
        A[q] = v;
        Inv[q] = (i == j) ? 1.0 : 0.0;
    }
    __shared__ int s_piv;
    __shared__ double s_pval;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            double bv = fabs(A[(int64_t)k * n + k]);
            for (int i = k + 1; i < n; ++i) {
                const double v = fabs(A[(int64_t)i * n + k]);
                if (v > bv) { bv = v; best = i; }
            }
            s_piv = best;
            s_pval = A[(int64_t)best * n + k];
            // 2: exactly singular (fatal for the setup); 1: non-finite
            // entries, which the solve reports per image as kNonFinite.
            if (bv == 0.0) atomicMax(status, 2);
            else if (!isfinite(bv)) atomicMax(status, 1);
        }
        __syncthreads();
        const int pr = s_piv;
        if (pr != k) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double t = A[(int64_t)k * n + j]; A[(int64_t)k * n + j] = A[(int64_t)pr * n + j]; A[(int64_t)pr * n + j] = t;
                t = Inv[(int64_t)k * n + j]; Inv[(int64_t)k * n + j] = Inv[(int64_t)pr * n + j]; Inv[(int64_t)pr * n + j] = t;
            }
        }
        __syncthreads();
        const double piv = s_pval;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            A[(int64_t)k * n + j] /= piv;
            Inv[(int64_t)k * n + j] /= piv;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q / n, j = q - i * n;
            if (i == k || j == k) continue;
            const double f = A[(int64_t)i * n + k];
            A[q] -= f * A[(int64_t)k * n + j];
            Inv[q] -= f * Inv[(int64_t)k * n + j];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if (i == k) continue;
            const double f = A[(int64_t)i * n + k];
            Inv[(int64_t)i * n + k] -= f * Inv[(int64_t)k * n + k];
            A[(int64_t)i * n + k] = 0.0;
        }
        __syncthreads();
    }
}

__global__ void k_convert_f32(const double* __restrict__ src, float* dst, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; i < n; i += (int64_t)gridDim.x * blockDim.x) dst[i] = (float)src[i];
}

// --------------------------------------------------------------------------
// Packing between user layout (contiguous h*w per image) and pitched grids
// --------------------------------------------------------------------------

// Grid g of element idx of the user layout (the last g with off[g] <= idx;
// every grid has at least one element) and idx's position in that grid.
// The offsets come from shared memory when the list has at most kDirGrids
// grids; positions within one image fit 32 bits.
struct PackLoc {
    int g, y, x;
};
__device__ __forceinline__ PackLoc pack_locate(const GridDesc* grids, int ngrids,
                                               const int64_t* off, int64_t idx) {
    int lo = 0, hi = ngrids - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= idx) lo = mid;
        else hi = mid - 1;
    }
    const int w = grids[lo].w;
    const int local = (int)(idx - off[lo]);
    const int y = local / w;
    return PackLoc{lo, y, local - y * w};
}

__device__ __forceinline__ const int64_t* pack_offsets(int64_t* s_off, const int64_t* user_off,
                                                       int ngrids) {
    const bool fits = ngrids <= kDirGrids;
    if (fits)
        for (int i = threadIdx.x; i < ngrids; i += blockDim.x) s_off[i] = user_off[i];
    __syncthreads();
    return fits ? s_off : user_off;
}

template <typename TS, typename TD>
__global__ void k_pack(const GridDesc* grids, int ngrids, const int64_t* user_off,
                       const TS* __restrict__ src, TD* dst, int64_t total) {
    __shared__ int64_t s_off[kDirGrids];
    const int64_t* off = pack_offsets(s_off, user_off, ngrids);
    int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const PackLoc q = pack_locate(grids, ngrids, off, idx);
        const GridDesc& d = grids[q.g];
        dst[d.voff + (int64_t)q.y * d.pitch + q.x] = (TD)src[idx];
    }
}

template <typename TS, typename TD>
__global__ void k_unpack(const GridDesc* grids, int ngrids, const int64_t* user_off,
                         const TS* __restrict__ src, TD* dst, int64_t total) {
    __shared__ int64_t s_off[kDirGrids];
    const int64_t* off = pack_offsets(s_off, user_off, ngrids);
    int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const PackLoc q = pack_locate(grids, ngrids, off, idx);
        const GridDesc& d = grids[q.g];
        dst[idx] = (TD)src[d.voff + (int64_t)q.y * d.pitch + q.x];
    }
}

// --------------------------------------------------------------------------
// Iterative refinement around the FP32 inner solve
// --------------------------------------------------------------------------

// Mixed precision: FP32 PCG with reliable updates (Sleijpen & van der Vorst,
// 1996). The FP64 iterate x64 accumulates; the FP32 CG runs on the
// correction x32 with its own recurrence residual r32. When |r32| has dropped
// by `delta` since the last replacement (or below the FP64 tolerance),
// k_cg_update flags the image (kUpdate) and, in the same iteration,
//   k_refine_correct   x64 += x32, x32 = 0
//   k_refine_residual  r64 = b - A64 x64 (FP64 planes), r32 = (float) r64
// replace the recurrence residual by the true one; CG then continues with the
// same search direction (beta from the new r . z). Convergence is decided on
// the FP64 residual only.
// Phase tolerance floor, x the FP64 tolerance. At 1 the last FP32 phase stops
// where the FP64 solve would: its recurrence residual then tracks the true one
// to far below the tolerance (the phase starts from a replaced residual), so
// the FP32 and FP64 iteration counts agree; a phase that stops short of the
// FP64 test just continues. A floor of 0.5 cost 3 to 8 iterations per image
// (the iterations from the tolerance to half of it).
constexpr double kReliableFloor = 1.0;

// r64 = b - A64 x64 in FP64, r32 = (float) r64. FIRST: the initial residual
// (every image whose outer state runs): sets |b|, the FP64 tolerance and
// starts the FP32 CG with x32 = 0. Otherwise only images flagged kUpdate:
// the residual replacement described above.
template <int PREC, bool FIRST>
__global__ void __launch_bounds__(kTileThreads)
k_refine_residual(WorkList wl, const CUtensorMap* maps, const float* __restrict__ P32,
                  const double* __restrict__ b, float* r32, float* x32, float* z32,
                  InstState* outer, InstState* inner, double* partials, double atol, double rtol,
                  double delta, int maxiter, int max_outer, int* err) {
    // Replacement launches with no image flagged (most iterations) end here:
    // err[kPendingSlot] counts the images k_cg_update flagged.
    if (!FIRST && *(volatile int*)(err + kPendingSlot) == 0) return;
    __shared__ double s_red[3 * 32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    double* sP_[2];
    double* sX_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<double>(kNH * kBH * kBW);
        sX_[k] = sc.take<double>(kBH * kBW);
    }
    const Buf2<double> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<double> sX{sX_[0], sX_[1] - sX_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    double v[3] = {0.0, 0.0, 0.0};
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        mbar_expect_tx(&pipe.bar[bb], (kNH + 1) * kBH * kBW * sizeof(double));
        tma_load_3d(sP[bb], map_of(maps, g, kMapP64F), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, g, kMapX64F), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
        const int y = m.y0 + ly, xx = m.x0 + lx;
        if (y < g.h && xx < g.w) {
            const int64_t i = g.voff + (int64_t)y * g.pitch + xx;
            const double bi = b[i];
            const double ri = bi - stencil_at<double>(sP[bb], kBH, sX[bb], ly + 2, lx + kBOX);
            const float rf = (float)ri;
            r32[i] = rf;
            if (FIRST) x32[i] = 0.0f;
            v[0] += bi * bi;
            v[1] += ri * ri;
            if (PREC == kPrecJacobi) {
                const float zi = rf * (1.0f / P32[g.poff + (int64_t)y * g.pitch + xx]);
                z32[i] = zi;
                v[2] += (double)rf * (double)zi;
            } else if (PREC == kPrecNone) {
                v[2] += (double)rf * (double)rf;
            }
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        InstState* so = outer + m.inst;
        InstState* si = inner + m.inst;
        cta_flush<3>(v, partials, m.inst, m.t0, m.t1, mine, so, s_red, [&](double* sum) {
            const double nr = sqrt(sum[1]);
            if (FIRST) {
                const double nb = sqrt(sum[0]);
                so->norm_b = nb;
                so->tol = fmax(atol, rtol * nb);
                so->iters = 0;
                si->iters = 0;
                si->maxiter = maxiter;
                si->flags = kFirst;
                si->beta = 0.0;
            } else {
                so->iters += 1;
                si->flags &= ~kUpdate;
                atomicSub(err + kPendingSlot, 1);
            }
            so->norm_r = nr;
            int status = kRunning;
            if (!isfinite(nr)) status = kNonFinite;
            else if (nr < atol || nr < so->tol) status = kConverged;
            else if (so->iters >= max_outer) status = kMaxIter;
            else if (!FIRST && si->iters >= si->maxiter) status = kMaxIter;
            so->status = status;
            si->status = status;
            si->norm_r = nr;
            if (status == kRunning) {
                si->norm_b = nr;
                si->tol = fmax(delta * nr, kReliableFloor * so->tol);
                if (PREC != kPrecVcycle) {
                    if (FIRST) si->rz = sum[2];
                    else finish_beta(si, sum[2]);
                }
            }
        });
    };
    if (FIRST) tile_loop<kTY, kTX, kGateRunning>(wl, outer, pipe, s_m, s_g, issue, body, flush);
    else tile_loop<kTY, kTX, kGateUpdate>(wl, inner, pipe, s_m, s_g, issue, body, flush);
}

// x64 += x32, x32 = 0: for images flagged kUpdate (GATE = kGateUpdate), or
// for every image (st == nullptr) at the end of a solve.
template <int GATE>
__global__ void __launch_bounds__(kThreads)
k_refine_correct(WorkList wl, double* x64, float* x32, const InstState* st, const int* pending) {
    if (GATE == kGateUpdate && *(volatile const int*)pending == 0) return;
    auto body = [&](const GridDesc& g, int64_t e0, int64_t e1) {
#pragma unroll
        for (int k = 0; k < kFlat / kThreads; ++k) {
            const int64_t e = e0 + threadIdx.x + k * kThreads;
            if (e >= e1) break;
            if ((int)(e % g.pitch) >= g.w) continue;
            const int64_t i = g.voff + e;
            x64[i] += (double)x32[i];
            x32[i] = 0.0f;
        }
    };
    flat_loop<GATE>(wl, st, body, [](int, int, int, unsigned int) {});
}


// --------------------------------------------------------------------------
// Launchers
// --------------------------------------------------------------------------



// --------------------------------------------------------------------------
// Register-blocked kernels
// --------------------------------------------------------------------------
//
// Each thread computes V adjacent pixels of a row (V = 2 or 4 in FP32, 2 in
// FP64: one 8- or 16-byte shared-memory vector). The operand window of the 25-point
// stencil is held in registers (5 rows x 3 vectors) and every plane is read
// with vector loads, so a pixel costs ~12 (FP32) or ~25 (FP64) shared loads
// instead of 50. The accumulation order per pixel is that of stencil_at, so
// the results are bit-identical to the one-pixel-per-thread kernels.

// Threads of the 64x8-tile kernels: one V-pixel group each.
template <int V> __host__ __device__ constexpr int tile_threads_v() { return kTX / V * kTY; }
// Threads of the restriction kernel (grid-stride over its work items).
constexpr int kDownThreads = 256;

// (A x) for the V pixels at box row r, box columns c0 .. c0 + V - 1 (c0 a
// multiple of V, c0 >= V). P: 13 planes of BW-wide rows, `ps` elements apart,
// row 0 = two rows above the first output row of the tile; loadx(row, col, o)
// loads V operand values at an aligned box position. Needs rows r-2 .. r+2 of
// the operand, r-2 .. r of the planes, columns c0 - V .. c0 + 2V - 1.
// Plane 0 and planes 1..12 may lie in separate boxes with the same first
// row: plane 0 at P0, plane p >= 1 at P1 + (p - 1) ps1 (BW-wide rows).
template <typename T, int V, int BW, typename LoadX>
__device__ __forceinline__ void stencil_split(const T* P0, const T* P1, int ps1, LoadX loadx,
                                              int r, int c0, T (&acc)[V]) {
    T xr[5][3 * V];
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) loadx(r - 2 + k, c0 - V + j * V, &xr[k][j * V]);
    T pc[V];
    ldv<T, V>(P0 + r * BW + c0, pc);
    // FP32: forward and backward terms in two independent chains (half the
    // dependent-FMA latency per pixel). FP64 keeps one chain in the original
    // order, which its iteration-count parity with the reference rests on.
    constexpr bool kSplit = sizeof(T) == 4;
    T accb[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        acc[v] = pc[v] * xr[2][V + v];
        accb[v] = T(0);
    }
#pragma unroll
    for (int p = 1; p < kNH; ++p) {
        const int dy = half_dy(p), dx = half_dx(p);
        const T* Pp = P1 + (p - 1) * ps1;
        T pf[V];
        ldv<T, V>(Pp + r * BW + c0, pf);
        // Backward entries A[i, i - d] = plane p at (r - dy, c - dx): an
        // aligned window of one or two vectors around c0 - dx.
        T pb[2 * V];
        const int cb = dx > 0 ? c0 - V : c0;
        ldv<T, V>(Pp + (r - dy) * BW + cb, pb);
        if (dx != 0) ldv<T, V>(Pp + (r - dy) * BW + cb + V, pb + V);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            acc[v] += pf[v] * xr[2 + dy][V + v + dx];
            if (kSplit) accb[v] += pb[(dx > 0 ? V : 0) + v - dx] * xr[2 - dy][V + v - dx];
            else acc[v] += pb[(dx > 0 ? V : 0) + v - dx] * xr[2 - dy][V + v - dx];
        }
    }
    if (kSplit) {
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] += accb[v];
    }
}

template <typename T, int V, int BW, typename LoadX>
__device__ __forceinline__ void stencil_vec(const T* P, int ps, LoadX loadx, int r, int c0,
                                            T (&acc)[V]) {
    stencil_split<T, V, BW>(P, P + ps, ps, loadx, r, c0, acc);
}

// Division in the smoothing sweeps: IEEE in FP64; __fdividef in FP32, where
// the V-cycle is the inner preconditioner of the mixed solve (convergence is
// judged on the FP64 residual).
template <typename T> __device__ __forceinline__ T smooth_div(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float smooth_div<float>(float a, float b) {
    return __fdividef(a, b);
}

// y = A x (pitched vectors, no reductions). Plane box: rows y0-2 .. y0+7
// (kMapPlS), operand box 72 x 12 (kMapBF).
template <typename T, int V>
__global__ void __launch_bounds__(tile_threads_v<V>())
k_apply_v(WorkList wl, const CUtensorMap* maps, T* y, int* err) {
    constexpr int TPR = kTX / V;
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sX_[2];
    for (int k = 0; k < 2; ++k) {
        sP_[k] = sc.take<T>(kNH * kPH * kBW);
        sX_[k] = sc.take<T>(kBH * kBW);
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sX{sX_[0], sX_[1] - sX_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        mbar_expect_tx(&pipe.bar[bb], (kNH * kPH + kBH) * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlS), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sX[bb], map_of(maps, g, kMapBF), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
        const int yy = m.y0 + ty, xx = m.x0 + V * tx;
        if (yy < g.h && xx < g.w) {
            const T* X = sX[bb];
            T acc[V];
            stencil_vec<T, V, kBW>(sP[bb], kPH * kBW,
                                [&](int rr, int cc, T* o) { ldv<T, V>(X + rr * kBW + cc, o); },
                                ty + 2, kBOX + V * tx, acc);
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (xx + v >= g.w) acc[v] = T(0);
            stv<T, V>(y + g.voff + (int64_t)yy * g.pitch + xx, acc);
        }
    };
    tile_loop<kTY, kTX>(wl, nullptr, pipe, s_m, s_g, issue, body, NoFlush());
}

// p_new = z + beta p_old (z on the first pass), Ap = A p_new, p_new . Ap;
// finaliser alpha = rz / (p . Ap) (cg.py:85-90, 111-113). p_new is formed
// in registers from the z and p_old boxes.
template <typename T, int V, int NST>
__global__ void __launch_bounds__(tile_threads_v<V>())
k_cg_apply_v(WorkList wl, const CUtensorMap* maps, int zslot, T* p0, T* p1, T* Ap, InstState* st,
             double* partials, int* err) {
    constexpr int TPR = kTX / V;
    __shared__ double s_red[32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP_[2];
    T* sZ_[2];
    T* sQ_[2];
    for (int k = 0; k < NST; ++k) {
        sP_[k] = sc.take<T>(kNH * kPH * kBW);
        sZ_[k] = sc.take<T>(kBH * kBW);
        sQ_[k] = sc.take<T>(kBH * kBW);
    }
    if (NST == 1) {
        sP_[1] = sP_[0];
        sZ_[1] = sZ_[0];
        sQ_[1] = sQ_[0];
    }
    const Buf2<T> sP{sP_[0], sP_[1] - sP_[0]};
    const Buf2<T> sZ{sZ_[0], sZ_[1] - sZ_[0]};
    const Buf2<T> sQ{sQ_[0], sQ_[1] - sQ_[0]};
    Pipe pipe;
    pipe.init(s_bar, err);
    double v0[1] = {0.0};
    auto issue = [&](const Meta& m, const GridDesc& g, int bb) {
        mbar_expect_tx(&pipe.bar[bb], (kNH * kPH + (m.first ? 1 : 2) * kBH) * kBW * sizeof(T));
        tma_load_3d(sP[bb], map_of(maps, g, kMapPlS), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_2d(sZ[bb], map_of(maps, g, zslot), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
        if (!m.first)
            tma_load_2d(sQ[bb], map_of(maps, g, m.par ? kMapP1F : kMapP0F), m.x0 - kBOX, m.y0 - 2,
                        &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& g, int bb) {
        const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
        const int yy = m.y0 + ty, xx = m.x0 + V * tx;
        if (yy < g.h && xx < g.w) {
            const T* Z = sZ[bb];
            const T* Q = sQ[bb];
            const bool first = m.first != 0;
            const T beta = (T)m.beta;
            auto loadp = [&](int rr, int cc, T* o) {
                ldv<T, V>(Z + rr * kBW + cc, o);
                if (!first) {
                    T q[V];
                    ldv<T, V>(Q + rr * kBW + cc, q);
#pragma unroll
                    for (int v = 0; v < V; ++v) o[v] = o[v] + beta * q[v];
                }
            };
            T acc[V], pv[V];
            stencil_vec<T, V, kBW>(sP[bb], kPH * kBW, loadp, ty + 2, kBOX + V * tx, acc);
            loadp(ty + 2, kBOX + V * tx, pv);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (xx + v >= g.w) {
                    acc[v] = T(0);
                    pv[v] = T(0);
                }
                v0[0] += (double)pv[v] * (double)acc[v];
            }
            const int64_t i = g.voff + (int64_t)yy * g.pitch + xx;
            stv<T, V>((m.par ? p0 : p1) + i, pv);
            stv<T, V>(Ap + i, acc);
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        InstState* s = st + m.inst;
        cta_flush<1>(v0, partials, m.inst, m.t0, m.t1, mine, s, s_red, [&](double* sum) {
            s->pap = sum[0];
            s->alpha = s->rz / sum[0];
            s->flags &= ~kFirst;
        });
    };
    if (NST == 2) tile_loop<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
    else tile_loop1<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
}

// Restriction box of the register-blocked restriction kernel: fine columns
// from 2 X0 - DOFF, DW wide; rows 2 Y0 - 3 .. 2 Y0 + 2 CY + 1.
template <typename T, int VV> struct DownBox {
    static constexpr int V = VV;
    static constexpr int CY = Coarse<T>::CY;
    static constexpr int DH = 2 * CY + 5;
    static constexpr int DOFF = 2 * V;
    static constexpr int DW = kTX + DOFF + 4;      // 76 (FP32), 72 (FP64)
    static constexpr int RH = 2 * CY + 1;          // residual rows
    static constexpr int RW = kTX + V;             // residual columns from 2 X0 - V
};

// One pre-smoothing sweep from zero, residual and full-weighting restriction
// (vcycle.py:33-36, 77-80; same arithmetic as k_vc_down<T, 1>):
//   x1 = omega b / d on the box, res = b - A x1 on the fine rows
//   2 Y0 - 1 .. 2 Y0 + 2 CY - 1, b_coarse = R res.
// NST: 2 buffers (a tile in flight while the previous one is computed) or 1
// (half the shared memory, twice the CTAs per SM). Plane 0 (the diagonal of
// the sweep over the whole box) is loaded on DH rows, planes 1..12 (only
// the residual rows' backward entries) on DH - 2.
template <typename T, int V, int NST>
__global__ void __launch_bounds__(kDownThreads)
k_vc_down_v(WorkList wl /* coarse tiles */, const GridDesc* fine, const CUtensorMap* maps, T* bc,
            double omega, const InstState* st, int* err) {
    using D = DownBox<T, V>;
    constexpr int DH = D::DH, DW = D::DW, RH = D::RH, RW = D::RW, CY = D::CY;
    constexpr int RV = RW / V, XV = DW / V;
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP0_[2];
    T* sP1_[2];
    T* sB_[2];
    for (int k = 0; k < NST; ++k) {
        sP0_[k] = sc.take<T>(DH * DW);
        sP1_[k] = sc.take<T>((kNH - 1) * (DH - 2) * DW);
        sB_[k] = sc.take<T>(DH * DW);
    }
    if (NST == 1) {
        sP0_[1] = sP0_[0];
        sP1_[1] = sP1_[0];
        sB_[1] = sB_[0];
    }
    const Buf2<T> sP0{sP0_[0], sP0_[1] - sP0_[0]};
    const Buf2<T> sP1{sP1_[0], sP1_[1] - sP1_[0]};
    const Buf2<T> sB{sB_[0], sB_[1] - sB_[0]};
    T* sX = sc.take<T>(DH * DW);
    T* sR = sc.take<T>(RH * RW);
    Pipe pipe;
    pipe.init(s_bar, err);
    auto issue = [&](const Meta& m, const GridDesc& gc, int bb) {
        const GridDesc gf = fine[m.g];
        const int bx = 2 * m.x0 - D::DOFF, by = 2 * m.y0 - 3;
        mbar_expect_tx(&pipe.bar[bb], (2 * DH + (kNH - 1) * (DH - 2)) * DW * sizeof(T));
        tma_load_3d(sP0[bb], map_of(maps, gf, kMapPlD0), bx, by, 0, &pipe.bar[bb]);
        tma_load_3d(sP1[bb], map_of(maps, gf, kMapPlD1), bx, by, 1, &pipe.bar[bb]);
        tma_load_2d(sB[bb], map_of(maps, gf, kMapBDV), bx, by, &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& gc, int bb) {
        const GridDesc gf = fine[m.g];
        const int bx = 2 * m.x0 - D::DOFF, by = 2 * m.y0 - 3;
        const T* B = sB[bb];
        const T* P = sP0[bb];
        const T* P1 = sP1[bb];
        for (int q = threadIdx.x; q < DH * XV; q += kDownThreads) {
            const int rr = q / XV, col = (q - rr * XV) * V;
            const int fy = by + rr;
            T bv[V], dv[V], o[V];
            ldv<T, V>(B + rr * DW + col, bv);
            ldv<T, V>(P + rr * DW + col, dv);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int fx = bx + col + v;
                o[v] = (fy >= 0 && fy < gf.h && fx >= 0 && fx < gf.w)
                           ? smooth_div<T>((T)omega * bv[v], dv[v]) : T(0);
            }
            stv<T, V>(sX + rr * DW + col, o);
        }
        __syncthreads();
        for (int q = threadIdx.x; q < RH * RV; q += kDownThreads) {
            const int rr = q / RV, cv = q - rr * RV;
            const int br = rr + 2, bcol = D::DOFF - V + cv * V;
            const int fy = by + br;
            T acc[V], bv[V], o[V];
            stencil_split<T, V, DW>(P, P1, (DH - 2) * DW,
                                    [&](int r2, int c2, T* out) { ldv<T, V>(sX + r2 * DW + c2, out); },
                                    br, bcol, acc);
            ldv<T, V>(B + br * DW + bcol, bv);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int fx = bx + bcol + v;
                o[v] = (fy >= 0 && fy < gf.h && fx >= 0 && fx < gf.w) ? bv[v] - acc[v] : T(0);
            }
            stv<T, V>(sR + rr * RW + cv * V, o);
        }
        __syncthreads();
        for (int q = threadIdx.x; q < kCX * CY; q += kDownThreads) {
            const int ly = q / kCX, lx = q - ly * kCX;
            const int Y = m.y0 + ly, X = m.x0 + lx;
            if (Y < gc.h && X < gc.w) {
                T sum = T(0);
#pragma unroll
                for (int ay = -1; ay <= 1; ++ay)
#pragma unroll
                    for (int ax = -1; ax <= 1; ++ax)
                        sum += (T)(pw(ax) * pw(ay) / 16.0) *
                               sR[(2 * ly + 1 + ay) * RW + (2 * lx + ax + V)];
                bc[gc.voff + (int64_t)Y * gc.pitch + X] = sum;
            }
        }
    };
    if (NST == 2) tile_loop<CY, kCX>(wl, st, pipe, s_m, s_g, issue, body, NoFlush());
    else tile_loop1<CY, kCX>(wl, st, pipe, s_m, s_g, issue, body, NoFlush());
}

// Prolongation and one post-smoothing sweep (same arithmetic as
// k_vc_up<T, 1, 1>): x2 = x1 + P xc on the 72 x 12 box into shared memory,
// then x3 = x2 + omega (b - A x2) / d for the tile; at level 0 also r . z
// (and (r - r_old) . z) with beta.
// NST as in k_vc_down_v. Plane 0 (the diagonal of the first sweep over the
// whole box) is loaded on kBH rows, planes 1..12 (the post sweep's backward
// entries) on kPH.
template <typename T, int V, int NST>
__global__ void __launch_bounds__(tile_threads_v<V>())
k_vc_up_v(WorkList wl /* fine tiles */, const GridDesc* coarse, const CUtensorMap* maps,
          const T* __restrict__ b, T* xout, double omega, InstState* st, int level0,
          const T* __restrict__ dr, int reorth, double* partials, int* err) {
    constexpr int TPR = kTX / V, NT = tile_threads_v<V>(), XV = kBW / V;
    __shared__ double s_red[2 * 32];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ Meta s_m[2];
    __shared__ GridDesc s_g[2];
    SmemCarve sc(g_smem);
    T* sP0_[2];
    T* sP1_[2];
    T* sB_[2];
    T* sC_[2];
    for (int k = 0; k < NST; ++k) {
        sP0_[k] = sc.take<T>(kBH * kBW);
        sP1_[k] = sc.take<T>((kNH - 1) * kPH * kBW);
        sB_[k] = sc.take<T>(kBH * kBW);
        sC_[k] = sc.take<T>(kCBH * kCBW);
    }
    if (NST == 1) {
        sP0_[1] = sP0_[0];
        sP1_[1] = sP1_[0];
        sB_[1] = sB_[0];
        sC_[1] = sC_[0];
    }
    const Buf2<T> sP0{sP0_[0], sP0_[1] - sP0_[0]};
    const Buf2<T> sP1{sP1_[0], sP1_[1] - sP1_[0]};
    const Buf2<T> sB{sB_[0], sB_[1] - sB_[0]};
    const Buf2<T> sC{sC_[0], sC_[1] - sC_[0]};
    T* sX = sc.take<T>(kBH * kBW);
    Pipe pipe;
    pipe.init(s_bar, err);
    double acc2[2] = {0.0, 0.0};
    auto issue = [&](const Meta& m, const GridDesc& gf, int bb) {
        const GridDesc gc = coarse[m.g];
        mbar_expect_tx(&pipe.bar[bb],
                       ((2 * kBH + (kNH - 1) * kPH) * kBW + kCBH * kCBW) * sizeof(T));
        tma_load_3d(sP0[bb], map_of(maps, gf, kMapPlU0), m.x0 - kBOX, m.y0 - 2, 0, &pipe.bar[bb]);
        tma_load_3d(sP1[bb], map_of(maps, gf, kMapPlU1), m.x0 - kBOX, m.y0 - 2, 1, &pipe.bar[bb]);
        tma_load_2d(sB[bb], map_of(maps, gf, kMapBF), m.x0 - kBOX, m.y0 - 2, &pipe.bar[bb]);
        tma_load_2d(sC[bb], map_of(maps, gc, kMapXC), (m.x0 >> 1) - 4, (m.y0 >> 1) - 2,
                    &pipe.bar[bb]);
    };
    auto body = [&](const Meta& m, const GridDesc& gf, int bb) {
        const int bx = m.x0 - kBOX, by = m.y0 - 2;
        const int cx0 = (m.x0 >> 1) - 4, cy0 = (m.y0 >> 1) - 2;
        const T* P = sP0[bb];
        const T* P1 = sP1[bb];
        const T* B = sB[bb];
        const T* C = sC[bb];
        for (int q = threadIdx.x; q < kBH * XV; q += NT) {
            const int rr = q / XV, col = (q - rr * XV) * V;
            const int y = by + rr;
            T bv[V], dv[V], o[V];
            ldv<T, V>(B + rr * kBW + col, bv);
            ldv<T, V>(P + rr * kBW + col, dv);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int x = bx + col + v;
                T val = T(0);
                if (y >= 0 && y < gf.h && x >= 0 && x < gf.w) {
                    const T x1 = smooth_div<T>((T)omega * bv[v], dv[v]);
                    // Coarse pixels whose 3x3 support holds (y, x), in raster
                    // order: an even coordinate has one parent (weight 2), an
                    // odd one two (weight 1). Written without branches: the
                    // second parent of an even coordinate gets weight 0, and
                    // parents outside the coarse grid read the zeros the TMA
                    // box is filled with there, so both add exactly nothing.
                    const int oy = y & 1, ox = x & 1;
                    const T* c00 = C + (((y - oy) >> 1) - cy0) * kCBW + (((x - ox) >> 1) - cx0);
                    const T wy0 = T(2 - oy), wy1 = T(oy), wx0 = T(2 - ox), wx1 = T(ox);
                    const T s16 = T(0.0625);
                    T sum = T(0);
                    sum += (wx0 * wy0 * s16) * c00[0];
                    sum += (wx1 * wy0 * s16) * c00[ox];
                    sum += (wx0 * wy1 * s16) * c00[oy * kCBW];
                    sum += (wx1 * wy1 * s16) * c00[oy * kCBW + ox];
                    val = x1 + sum;
                }
                o[v] = val;
            }
            stv<T, V>(sX + rr * kBW + col, o);
        }
        __syncthreads();
        const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
        const int yy = m.y0 + ty, xx = m.x0 + V * tx;
        if (yy < gf.h && xx < gf.w) {
            const int r = ty + 2, c0 = kBOX + V * tx;
            T ax[V], x2[V], bv[V], dv[V], x3[V];
            stencil_split<T, V, kBW>(P, P1, kPH * kBW,
                                     [&](int r2, int c2, T* out) { ldv<T, V>(sX + r2 * kBW + c2, out); },
                                     r, c0, ax);
            ldv<T, V>(sX + r * kBW + c0, x2);
            ldv<T, V>(B + r * kBW + c0, bv);
            ldv<T, V>(P + r * kBW + c0, dv);
            const int64_t i = gf.voff + (int64_t)yy * gf.pitch + xx;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (xx + v < gf.w) {
                    x3[v] = x2[v] + smooth_div<T>((T)omega * (bv[v] - ax[v]), dv[v]);
                    if (level0) {
                        acc2[0] += (double)bv[v] * (double)x3[v];
                        if (reorth) acc2[1] += (double)dr[i + v] * (double)x3[v];
                    }
                } else {
                    x3[v] = T(0);
                }
            }
            stv<T, V>(xout + i, x3);
        }
    };
    auto flush = [&](const Meta& m, unsigned int mine) {
        if (!level0 || !st) return;
        InstState* s = st + m.inst;
        cta_flush<2>(acc2, partials, m.inst, m.t0, m.t1, mine, s, s_red, [&](double* sum) {
            if (reorth) finish_beta_reorth(s, sum[0], sum[1]);
            else finish_beta(s, sum[0]);
        });
    };
    if (NST == 2) tile_loop<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
    else tile_loop1<kTY, kTX>(wl, st, pipe, s_m, s_g, issue, body, flush);
}


// --------------------------------------------------------------------------
// Self-test of the bounded mbarrier wait
// --------------------------------------------------------------------------
//
// Thread 0 arms a barrier for 16 bytes of transaction that no copy will ever
// deliver (nothing is issued, so nothing is in flight), then every thread
// waits for it with a limit of `polls`; each thread whose wait gave up adds
// one to *gave_up. Used to show on the device that the waits of the TMA
// kernels end with an error status instead of spinning.
__global__ void k_selftest_mbar(uint32_t polls, int* gave_up) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, 16);
    }
    __syncthreads();
    if (!mbar_wait(&bar, 0, polls)) atomicAdd(gave_up, 1);
}

void launch_selftest_mbar(uint32_t polls, int* gave_up, cudaStream_t s) {
    k_selftest_mbar<<<1, 64, 0, s>>>(polls, gave_up);
}

// --------------------------------------------------------------------------
// Coarse-level tail: one CTA per image, shared-memory resident
// --------------------------------------------------------------------------
//
// The smallest levels of an image (a few thousand pixels in all) cost one
// launch latency each and move almost no data. One CTA per image runs them in
// a single launch: bulk copies bring every tail level's planes and the first
// tail level's right-hand side into shared memory (pitched, as in global
// memory), the CTA walks down (first Jacobi sweep, residual, restriction),
// solves the coarsest grid with its dense inverse, walks back up
// (prolongation, post sweep) with __syncthreads between phases, and writes the
// first tail level's solution back. Same arithmetic as k_vc_down<T, 1> /
// k_vc_up<T, 1, 1> (vcycle.py:74-98). Shared layout per level: 13 planes,
// then b, x, t (t: residual, then the prolonged iterate), each h x pitch.

// A[i, i + e] of a pitched plane set at offset 0 (zero outside the grid).
template <typename T>
__device__ __forceinline__ T tail_entry(const T* P, const GridDesc& g, int y, int x, int ey,
                                        int ex) {
    const int yj = y + ey, xj = x + ex;
    if (yj < 0 || yj >= g.h || xj < 0 || xj >= g.w) return T(0);
    int p = half_index(ey, ex);
    if (p >= 0) return P[p * g.pstride + y * g.pitch + x];
    p = half_index(-ey, -ex);
    return P[p * g.pstride + yj * g.pitch + xj];
}

template <typename T>
__device__ __forceinline__ T tail_val(const T* v, const GridDesc& g, int y, int x) {
    if (y < 0 || y >= g.h || x < 0 || x >= g.w) return T(0);
    return v[y * g.pitch + x];
}

// (A v) at (y, x), accumulated in the order of stencil_at. Pixels at least
// two away from every border take the unchecked path.
template <typename T>
__device__ __forceinline__ T tail_stencil(const T* P, const T* v, const GridDesc& g, int y, int x) {
    const int i = y * g.pitch + x;
    if (y >= 2 && y < g.h - 2 && x >= 2 && x < g.w - 2) {
        T acc = P[i] * v[i];
#pragma unroll
        for (int p = 1; p < kNH; ++p) {
            const int d = half_dy(p) * g.pitch + half_dx(p);
            acc += P[p * g.pstride + i] * v[i + d];
            acc += P[p * g.pstride + i - d] * v[i - d];
        }
        return acc;
    }
    T acc = P[y * g.pitch + x] * v[y * g.pitch + x];
#pragma unroll
    for (int p = 1; p < kNH; ++p) {
        const int dy = half_dy(p), dx = half_dx(p);
        acc += tail_entry<T>(P, g, y, x, dy, dx) * tail_val<T>(v, g, y + dy, x + dx);
        acc += tail_entry<T>(P, g, y, x, -dy, -dx) * tail_val<T>(v, g, y - dy, x - dx);
    }
    return acc;
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads)
k_vc_tail(const TailDesc<T>* __restrict__ descs, const InstState* st, double omega, int* err) {
    __shared__ TailDesc<T> D;
    __shared__ int s_off[kMaxTailLevels + 1];
    __shared__ __align__(8) uint64_t s_bar;
    if (threadIdx.x == 0) D = descs[blockIdx.x];
    __syncthreads();
    if (st && st[D.inst].status != kRunning) return;   // uniform over the CTA
    const int nlev = D.nlev;
    T* sm = reinterpret_cast<T*>(g_smem);
    if (threadIdx.x == 0) {
        int off = 0;
        for (int l = 0; l < nlev; ++l) {
            s_off[l] = off;
            off += (kNH + 3) * D.lev[l].g.h * D.lev[l].g.pitch;
        }
        s_off[nlev] = off;
        mbar_init(&s_bar, 1);
        // Planes of every level (one block each) and the first level's b.
        uint32_t bytes = 0;
        for (int l = 0; l < nlev; ++l) bytes += kNH * D.lev[l].g.pstride * sizeof(T);
        bytes += D.lev[0].g.pstride * sizeof(T);
        mbar_expect_tx(&s_bar, bytes);
        for (int l = 0; l < nlev; ++l) {
            const GridDesc g = D.lev[l].g;
            bulk_load(sm + s_off[l], D.lev[l].P + g.poff,
                      (uint32_t)(kNH * g.pstride * sizeof(T)), &s_bar);
        }
        const GridDesc g0 = D.lev[0].g;
        bulk_load(sm + s_off[0] + kNH * g0.pstride, D.lev[0].b + g0.voff,
                  (uint32_t)(g0.pstride * sizeof(T)), &s_bar);
    }
    __syncthreads();
    const bool ok = mbar_wait(&s_bar, 0);
    if (__syncthreads_or(!ok)) {
        // Report, and wait (bounded) for the copies still in flight.
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            if (!ok) mbar_wait(&s_bar, 0);
        }
        return;
    }
    auto planes = [&](int l) { return sm + s_off[l]; };
    auto vb = [&](int l) { return sm + s_off[l] + kNH * D.lev[l].g.pstride; };
    auto vx = [&](int l) { return vb(l) + D.lev[l].g.pstride; };
    auto vt = [&](int l) { return vx(l) + D.lev[l].g.pstride; };
    const T om = (T)omega;
    // Down.
    for (int l = 0; l + 1 < nlev; ++l) {
        const GridDesc g = D.lev[l].g, gc = D.lev[l + 1].g;
        const int n = g.h * g.w;
        const T* P = planes(l);
        const T* b = vb(l);
        T* x1 = vx(l);
        T* t = vt(l);
        for (int k = threadIdx.x; k < n; k += kTailThreads) {
            const int y = k / g.w, x = k - y * g.w, i = y * g.pitch + x;
            x1[i] = om * b[i] / P[i];
        }
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += kTailThreads) {
            const int y = k / g.w, x = k - y * g.w, i = y * g.pitch + x;
            t[i] = b[i] - tail_stencil<T>(P, x1, g, y, x);
        }
        __syncthreads();
        T* bc = vb(l + 1);
        for (int k = threadIdx.x; k < gc.h * gc.w; k += kTailThreads) {
            const int Y = k / gc.w, X = k - Y * gc.w;
            T sum = T(0);
#pragma unroll
            for (int ay = -1; ay <= 1; ++ay)
#pragma unroll
                for (int ax = -1; ax <= 1; ++ax)
                    sum += (T)(pw(ax) * pw(ay) / 16.0) * tail_val<T>(t, g, 2 * Y + ay, 2 * X + ax);
            bc[Y * gc.pitch + X] = sum;
        }
        __syncthreads();
    }
    // Coarsest: x = inv b, one warp per row.
    {
        const GridDesc g = D.lev[nlev - 1].g;
        const int n = g.h * g.w;
        const T* b = vb(nlev - 1);
        T* x = vx(nlev - 1);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int q = warp; q < n; q += kTailThreads / 32) {
            const double* row = D.inv + (int64_t)q * n;
            double acc = 0.0;
            for (int j = lane; j < n; j += 32) {
                const int yj = j / g.w, xj = j - yj * g.w;
                acc += row[j] * (double)b[yj * g.pitch + xj];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                const int yq = q / g.w, xq = q - yq * g.w;
                x[yq * g.pitch + xq] = (T)acc;
            }
        }
    }
    __syncthreads();
    // Up.
    for (int l = nlev - 2; l >= 0; --l) {
        const GridDesc g = D.lev[l].g, gc = D.lev[l + 1].g;
        const int n = g.h * g.w;
        const T* P = planes(l);
        const T* b = vb(l);
        const T* xc = vx(l + 1);
        T* x = vx(l);
        T* t = vt(l);
        for (int k = threadIdx.x; k < n; k += kTailThreads) {
            const int y = k / g.w, xx = k - y * g.w;
            const int Ya = (y - 1) >> 1, Xa = (xx - 1) >> 1;
            const bool ey = (y & 1) == 0, ex = (xx & 1) == 0;
            T sum = T(0);
#pragma unroll
            for (int jy = 0; jy < 2; ++jy) {
                const int Y = ey ? (y >> 1) : Ya + jy;
                if ((ey && jy == 1) || Y >= gc.h) continue;
                const double wy = ey ? 2.0 : 1.0;
#pragma unroll
                for (int jx = 0; jx < 2; ++jx) {
                    const int Xc = ex ? (xx >> 1) : Xa + jx;
                    if ((ex && jx == 1) || Xc >= gc.w) continue;
                    const double wx = ex ? 2.0 : 1.0;
                    sum += (T)(wx * wy / 16.0) * xc[Y * gc.pitch + Xc];
                }
            }
            const int i = y * g.pitch + xx;
            t[i] = x[i] + sum;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += kTailThreads) {
            const int y = k / g.w, xx = k - y * g.w, i = y * g.pitch + xx;
            const T ax = tail_stencil<T>(P, t, g, y, xx);
            x[i] = t[i] + om * (b[i] - ax) / P[i];
        }
        __syncthreads();
    }
    // Copy out the first level's solution.
    {
        const GridDesc g = D.lev[0].g;
        const T* src = vx(0);
        for (int k = threadIdx.x; k < g.h * g.w; k += kTailThreads) {
            const int y = k / g.w, x = k - y * g.w;
            D.lev[0].x[g.voff + (int64_t)y * g.pitch + x] = src[y * g.pitch + x];
        }
    }
}

template <typename T>
void launch_vc_tail(const TailDesc<T>* descs, int count, size_t smem, const InstState* st,
                    double omega, int* err, cudaStream_t s) {
    if (count > 0) k_vc_tail<T><<<count, kTailThreads, smem, s>>>(descs, st, omega, err);
}

// Shared-memory sizes; they follow the SmemCarve layout of each kernel (two
// pipeline buffers, every piece rounded up to 128 bytes).
static inline size_t rup(size_t b) { return (b + 127) & ~size_t(127); }
template <typename T> size_t smem_apply() {
    return 2 * (rup(kNH * kBH * kBW * sizeof(T)) + 2 * rup(kBH * kBW * sizeof(T))) + 128;
}
template <typename T> size_t smem_init() {
    return 2 * (rup(kNH * kBH * kBW * sizeof(T)) + rup(kBH * kBW * sizeof(T))) + 128;
}
template <typename T> size_t smem_down(int pre) {
    constexpr int CY = Coarse<T>::CY;
    constexpr int DH = 2 * CY + 5;
    size_t per = rup(DH * kBW * sizeof(T));
    if (pre != 0) per += rup(kNH * DH * kBW * sizeof(T));
    if (pre > 1) per += rup(DH * kBW * sizeof(T));
    size_t s = 2 * per + rup((size_t)(2 * CY + 1) * (2 * kCX + 1) * sizeof(T));
    if (pre == 1) s += rup(DH * kBW * sizeof(T));
    return s + 128;
}
template <typename T> size_t smem_up(int pre) {
    size_t per = rup(kNH * kBH * kBW * sizeof(T)) + rup(kBH * kBW * sizeof(T)) +
                 rup(kCBH * kCBW * sizeof(T));
    if (pre > 1) per += rup(kBH * kBW * sizeof(T));
    return 2 * per + 128;
}

template <typename T> size_t smem_apply_v(int nst) {
    return nst * (rup(kNH * kPH * kBW * sizeof(T)) + 2 * rup(kBH * kBW * sizeof(T))) + 128;
}
// Vector widths of the register-blocked kernels, measured on B200 at
// 1920x1080 and 4096x4096: the plain apply is fastest with 4 FP32 pixels per
// thread (128 threads), the solver kernels (more work per tile) with 2
// (256 threads); FP64 uses 2 (one 16-byte vector).
template <typename T> constexpr int kVApply = sizeof(T) == 8 ? 2 : 4;
template <typename T> constexpr int kVSolve = 2;
// Widest vector of the element type (the tuner may pick it for the CG apply
// and the prolongation): 4 in FP32, 2 in FP64.
template <typename T> constexpr int kVWide = sizeof(T) == 8 ? 2 : 4;

template <typename T, int V> static size_t smem_down_vv(int nst) {
    using D = DownBox<T, V>;
    return nst * (rup(D::DH * D::DW * sizeof(T)) +
                  rup((kNH - 1) * (D::DH - 2) * D::DW * sizeof(T)) + rup(D::DH * D::DW * sizeof(T))) +
           rup(D::DH * D::DW * sizeof(T)) + rup(D::RH * D::RW * sizeof(T)) + 128;
}
template <typename T> size_t smem_up_v(int nst) {
    return nst * (rup(kBH * kBW * sizeof(T)) + rup((kNH - 1) * kPH * kBW * sizeof(T)) +
                  rup(kBH * kBW * sizeof(T)) + rup(kCBH * kCBW * sizeof(T))) +
           rup(kBH * kBW * sizeof(T)) + 128;
}
template <typename T> size_t smem_down_v(int nst) { return smem_down_vv<T, kVSolve<T>>(nst); }
template <typename T> int down_box_width() { return DownBox<T, kVSolve<T>>::DW; }

// Raise the dynamic shared-memory limit of a kernel. Done once for every
// instantiation by stencil_prepare(), before any stream capture.
template <typename K>
static void allow_smem(K kernel, size_t bytes) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T>
void launch_cg_init(int prec, const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps,
                    const T* P, const T* b, T* x, bool have_x0, T* r, T* z, InstState* st,
                    double* part, double atol, double rtol, int maxiter, int* err, cudaStream_t s) {
#define PMB_INIT(PK, X0)                                                                        \
    do {                                                                                        \
        const size_t sm = X0 ? smem_init<T>() : 128;                                            \
                                                                                    \
        k_cg_init<T, PK, X0><<<L.grid, kTileThreads, sm, s>>>(wl, maps, P, b, x, r, z, st, part,   \
                                                          atol, rtol, maxiter, err);            \
    } while (0)
    if (have_x0) {
        if (prec == kPrecNone) PMB_INIT(kPrecNone, true);
        else if (prec == kPrecJacobi) PMB_INIT(kPrecJacobi, true);
        else PMB_INIT(kPrecVcycle, true);
    } else {
        if (prec == kPrecNone) PMB_INIT(kPrecNone, false);
        else if (prec == kPrecJacobi) PMB_INIT(kPrecJacobi, false);
        else PMB_INIT(kPrecVcycle, false);
    }
#undef PMB_INIT
}

template <typename T>
void launch_cg_apply(int vec, int stages, const LaunchCfg& L, const WorkList& wl,
                     const CUtensorMap* maps, int zslot, T* p0, T* p1, T* Ap, InstState* st,
                     double* part, int* err, cudaStream_t s) {
    const int ns = stages <= 1 ? 1 : 2;
    const size_t sm = smem_apply_v<T>(ns);
    constexpr int V4 = kVWide<T>;
#define PMB_CGA(VV, NS)                                                                       \
    k_cg_apply_v<T, VV, NS><<<L.grid, tile_threads_v<VV>(), sm, s>>>(wl, maps, zslot, p0, p1, Ap, \
                                                                     st, part, err)
    if (vec == 4 && V4 == 4) {
        if (ns == 1) PMB_CGA(V4, 1);
        else PMB_CGA(V4, 2);
    } else {
        if (ns == 1) PMB_CGA(2, 1);
        else PMB_CGA(2, 2);
    }
#undef PMB_CGA
}

template <typename T>
void launch_cg_update(int prec, const LaunchCfg& L, const WorkList& wl, const T* P, T* x, T* r,
                      T* z, const T* p0, const T* p1, const T* Ap, T* dr, int reorth, int reliable,
                      int* pending, InstState* st, double* part, cudaStream_t s) {
    switch (prec) {
    case kPrecNone: k_cg_update<T, kPrecNone><<<L.grid, kThreads, 0, s>>>(wl, P, x, r, z, p0, p1, Ap, dr, reorth, reliable, pending, st, part); break;
    case kPrecJacobi: k_cg_update<T, kPrecJacobi><<<L.grid, kThreads, 0, s>>>(wl, P, x, r, z, p0, p1, Ap, dr, reorth, reliable, pending, st, part); break;
    default: k_cg_update<T, kPrecVcycle><<<L.grid, kThreads, 0, s>>>(wl, P, x, r, z, p0, p1, Ap, dr, reorth, reliable, pending, st, part); break;
    }
}

template <typename T>
void launch_cg_rz(const LaunchCfg& L, const WorkList& wl, const T* r, const T* z, const T* dr,
                  int reorth, InstState* st, double* part, cudaStream_t s) {
    k_cg_rz<T><<<L.grid, kThreads, 0, s>>>(wl, r, z, dr, reorth, st, part);
}

template <typename T>
void launch_vc_down(int pre, int stages, const LaunchCfg& L, const WorkList& wl,
                    const GridDesc* fine, const CUtensorMap* maps, int xs_slot, T* bc,
                    double omega, const InstState* st, int* err, cudaStream_t s) {
    const int pk = pre > 1 ? 2 : pre;
    if (pk == 1) {
        constexpr int V = kVSolve<T>;
        if (stages == 1)
            k_vc_down_v<T, V, 1><<<L.grid, kDownThreads, smem_down_v<T>(1), s>>>(
                wl, fine, maps, bc, omega, st, err);
        else
            k_vc_down_v<T, V, 2><<<L.grid, kDownThreads, smem_down_v<T>(2), s>>>(
                wl, fine, maps, bc, omega, st, err);
        return;
    }
    const size_t sm = smem_down<T>(pk);
#define PMB_DOWN(PK)                                                                         \
    do {                                                                                     \
                                                                                    \
        k_vc_down<T, PK><<<L.grid, kTileThreads, sm, s>>>(wl, fine, maps, xs_slot, bc, omega, st, err); \
    } while (0)
    if (pk == 0) PMB_DOWN(0);
    else if (pk == 1) PMB_DOWN(1);
    else PMB_DOWN(2);
#undef PMB_DOWN
}

template <typename T>
void launch_vc_up(int vec, int stages, int pre, int post, const LaunchCfg& L, const WorkList& wl,
                  const GridDesc* coarse, const CUtensorMap* maps, int xs_slot, const T* b,
                  T* xout, double omega, InstState* st, int level0, const T* dr, int reorth,
                  double* part, int* err, cudaStream_t s) {
    const int pk = pre > 1 ? 2 : pre;
    const int qk = post > 0 ? 1 : 0;
    if (pk == 1 && qk == 1) {
        constexpr int V4 = kVWide<T>;
#define PMB_UPV(VV, NS)                                                                       \
    k_vc_up_v<T, VV, NS><<<L.grid, tile_threads_v<VV>(), smem_up_v<T>(NS), s>>>(               \
        wl, coarse, maps, b, xout, omega, st, level0, dr, reorth, part, err)
        if (vec == 4 && V4 == 4) {
            if (stages == 1) PMB_UPV(V4, 1);
            else PMB_UPV(V4, 2);
        } else {
            if (stages == 1) PMB_UPV(2, 1);
            else PMB_UPV(2, 2);
        }
#undef PMB_UPV
        return;
    }
    const size_t sm = smem_up<T>(pk);
#define PMB_UP(PK, QK)                                                                       \
    do {                                                                                     \
                                                                                    \
        k_vc_up<T, PK, QK><<<L.grid, kTileThreads, sm, s>>>(wl, coarse, maps, xs_slot, b, xout,   \
                                                        omega, st, level0, dr, reorth, part, err); \
    } while (0)
    if (pk == 0 && qk == 0) PMB_UP(0, 0);
    else if (pk == 0) PMB_UP(0, 1);
    else if (pk == 1 && qk == 0) PMB_UP(1, 0);
    else if (pk == 1) PMB_UP(1, 1);
    else if (qk == 0) PMB_UP(2, 0);
    else PMB_UP(2, 1);
#undef PMB_UP
}

template <typename T>
void launch_vc_smooth(const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps,
                      int xin_slot, const T* P, const T* b, T* xout, double omega,
                      const InstState* st, int* err, cudaStream_t s) {
    const size_t sm = smem_init<T>();
    k_vc_smooth<T><<<L.grid, kTileThreads, sm, s>>>(wl, maps, xin_slot, P, b, xout, omega, st, err);
}

template <typename T>
void launch_vc_direct(const DirectDesc* dd, int count, const T* b, T* x, InstState* st,
                      int rz_level0, cudaStream_t s) {
    if (count > 0) k_vc_direct<T><<<count, 256, 0, s>>>(dd, count, b, x, st, rz_level0);
}

template <typename T>
void launch_apply(const LaunchCfg& L, const WorkList& wl, const CUtensorMap* maps, T* y, int* err,
                  cudaStream_t s) {
    const size_t sm = smem_apply_v<T>(2);
    constexpr int V = kVApply<T>;
    k_apply_v<T, V><<<L.grid, tile_threads_v<V>(), sm, s>>>(wl, maps, y, err);
}

template <typename TS, typename TD>
void launch_pack(const GridDesc* grids, int ngrids, const int64_t* uoff, const TS* src, TD* dst,
                 int64_t total, cudaStream_t s) {
    if (total <= 0) return;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_pack<TS, TD><<<blocks, 256, 0, s>>>(grids, ngrids, uoff, src, dst, total);
}

template <typename TS, typename TD>
void launch_unpack(const GridDesc* grids, int ngrids, const int64_t* uoff, const TS* src, TD* dst,
                   int64_t total, cudaStream_t s) {
    if (total <= 0) return;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_unpack<TS, TD><<<blocks, 256, 0, s>>>(grids, ngrids, uoff, src, dst, total);
}

void launch_galerkin_t(const WorkList& wl, const GridDesc* fine, const CUtensorMap* maps,
                       double* Pc, int* err, cudaStream_t s) {
    if (wl.total > 0)
        k_galerkin_t<<<wl.total, kGThreads, kNH * kGRows * kGCols * sizeof(double), s>>>(
            wl, fine, maps, Pc, err);
}

void launch_galerkin(const GridDesc* fine_g, const GridDesc* coarse_g, int ngrids, const double* Pf,
                     double* Pc, int64_t total, cudaStream_t s) {
    if (total <= 0) return;
    k_galerkin<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(fine_g, coarse_g, ngrids, Pf, Pc, total);
}

void launch_dense_inverse(const DirectDesc* dd, int count, double* work, int* status,
                          cudaStream_t s) {
    if (count > 0) k_dense_inverse<<<count, 256, 0, s>>>(dd, count, work, status);
}

void launch_convert_f32(const double* src, float* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_convert_f32<<<blocks, 256, 0, s>>>(src, dst, n);
}

void launch_refine_residual(int prec, int first, const LaunchCfg& L, const WorkList& wl,
                            const CUtensorMap* maps, const float* P32, const double* b,
                            float* r32, float* x32, float* z32, InstState* outer,
                            InstState* inner, double* part, double atol, double rtol,
                            double delta, int maxiter, int max_outer, int* err,
                            cudaStream_t s) {
    const size_t sm = smem_init<double>();
#define PMB_RR(PK, F)                                                                           \
    k_refine_residual<PK, F><<<L.grid, kTileThreads, sm, s>>>(wl, maps, P32, b, r32, x32, z32,  \
                                                              outer, inner, part, atol, rtol,   \
                                                              delta, maxiter, max_outer, err)
    if (first) {
        if (prec == kPrecNone) PMB_RR(kPrecNone, true);
        else if (prec == kPrecJacobi) PMB_RR(kPrecJacobi, true);
        else PMB_RR(kPrecVcycle, true);
    } else {
        if (prec == kPrecNone) PMB_RR(kPrecNone, false);
        else if (prec == kPrecJacobi) PMB_RR(kPrecJacobi, false);
        else PMB_RR(kPrecVcycle, false);
    }
#undef PMB_RR
}

void launch_refine_correct(const LaunchCfg& L, const WorkList& wl, double* x64, float* x32,
                           const InstState* inner, const int* pending, cudaStream_t s) {
    if (inner) k_refine_correct<kGateUpdate><<<L.grid, kThreads, 0, s>>>(wl, x64, x32, inner, pending);
    else k_refine_correct<kGateRunning><<<L.grid, kThreads, 0, s>>>(wl, x64, x32, nullptr, pending);
}


template <typename T>
static void prepare_type() {
    allow_smem(k_cg_init<T, kPrecNone, true>, smem_init<T>());
    allow_smem(k_cg_init<T, kPrecJacobi, true>, smem_init<T>());
    allow_smem(k_cg_init<T, kPrecVcycle, true>, smem_init<T>());
    allow_smem(k_cg_apply<T>, smem_apply<T>());
    allow_smem(k_vc_down<T, 0>, smem_down<T>(0));
    allow_smem(k_vc_down<T, 1>, smem_down<T>(1));
    allow_smem(k_vc_down<T, 2>, smem_down<T>(2));
    allow_smem(k_vc_up<T, 0, 0>, smem_up<T>(0));
    allow_smem(k_vc_up<T, 0, 1>, smem_up<T>(0));
    allow_smem(k_vc_up<T, 1, 0>, smem_up<T>(1));
    allow_smem(k_vc_up<T, 1, 1>, smem_up<T>(1));
    allow_smem(k_vc_up<T, 2, 0>, smem_up<T>(2));
    allow_smem(k_vc_up<T, 2, 1>, smem_up<T>(2));
    allow_smem(k_vc_smooth<T>, smem_init<T>());
    allow_smem(k_apply<T>, smem_init<T>());
    allow_smem(k_apply_v<T, kVApply<T>>, smem_apply_v<T>(2));
    allow_smem(k_vc_tail<T>, kTailSmem);
    allow_smem(k_cg_apply_v<T, 2, 2>, smem_apply_v<T>(2));
    allow_smem(k_cg_apply_v<T, 2, 1>, smem_apply_v<T>(1));
    allow_smem(k_cg_apply_v<T, kVWide<T>, 2>, smem_apply_v<T>(2));
    allow_smem(k_cg_apply_v<T, kVWide<T>, 1>, smem_apply_v<T>(1));
    allow_smem(k_vc_up_v<T, kVWide<T>, 2>, smem_up_v<T>(2));
    allow_smem(k_vc_up_v<T, kVWide<T>, 1>, smem_up_v<T>(1));
    allow_smem(k_vc_down_v<T, kVSolve<T>, 2>, smem_down_v<T>(2));
    allow_smem(k_vc_down_v<T, kVSolve<T>, 1>, smem_down_v<T>(1));
    allow_smem(k_vc_up_v<T, kVSolve<T>, 2>, smem_up_v<T>(2));
    allow_smem(k_vc_up_v<T, kVSolve<T>, 1>, smem_up_v<T>(1));
}

// Resident CTAs per SM of the register-blocked kernels as the occupancy
// calculator gives them (registers, static and dynamic shared memory,
// threads), at least 1. The shared-memory limits must be raised first
// (stencil_prepare).
template <typename K>
static int occupancy_of(K kernel, int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

template <typename T> int resident_cg_apply(int vec, int stages) {
    stencil_prepare();
    constexpr int V4 = kVWide<T>;
    const int ns = stages <= 1 ? 1 : 2;
    const size_t sm = smem_apply_v<T>(ns);
    if (vec == 4 && V4 == 4)
        return ns == 1 ? occupancy_of(k_cg_apply_v<T, V4, 1>, tile_threads_v<V4>(), sm)
                       : occupancy_of(k_cg_apply_v<T, V4, 2>, tile_threads_v<V4>(), sm);
    return ns == 1 ? occupancy_of(k_cg_apply_v<T, 2, 1>, tile_threads_v<2>(), sm)
                   : occupancy_of(k_cg_apply_v<T, 2, 2>, tile_threads_v<2>(), sm);
}
// Resident CTAs per SM of k_cg_update (a register limit, below the flat
// lists' default of 8: a persistent grid beyond it would run a second, thin
// wave of CTAs after the first).
template <typename T> int resident_cg_update(int prec) {
    static int cached[3] = {0, 0, 0};
    const int k = prec == kPrecNone ? 0 : (prec == kPrecJacobi ? 1 : 2);
    if (!cached[k]) {
        cached[k] = k == 0 ? occupancy_of(k_cg_update<T, kPrecNone>, kThreads, 0)
                  : k == 1 ? occupancy_of(k_cg_update<T, kPrecJacobi>, kThreads, 0)
                           : occupancy_of(k_cg_update<T, kPrecVcycle>, kThreads, 0);
    }
    return cached[k];
}
template <typename T> int resident_down(int stages) {
    stencil_prepare();
    constexpr int V = kVSolve<T>;
    return stages <= 1 ? occupancy_of(k_vc_down_v<T, V, 1>, kDownThreads, smem_down_v<T>(1))
                       : occupancy_of(k_vc_down_v<T, V, 2>, kDownThreads, smem_down_v<T>(2));
}
template <typename T> int resident_up(int vec, int stages) {
    stencil_prepare();
    constexpr int V4 = kVWide<T>;
    const int ns = stages <= 1 ? 1 : 2;
    if (vec == 4 && V4 == 4)
        return ns == 1 ? occupancy_of(k_vc_up_v<T, V4, 1>, tile_threads_v<V4>(), smem_up_v<T>(1))
                       : occupancy_of(k_vc_up_v<T, V4, 2>, tile_threads_v<V4>(), smem_up_v<T>(2));
    return ns == 1 ? occupancy_of(k_vc_up_v<T, 2, 1>, tile_threads_v<2>(), smem_up_v<T>(1))
                   : occupancy_of(k_vc_up_v<T, 2, 2>, tile_threads_v<2>(), smem_up_v<T>(2));
}

void stencil_prepare() {
    static bool done = false;
    if (done) return;
    prepare_type<double>();
    prepare_type<float>();
    allow_smem(k_galerkin_t, kNH * kGRows * kGCols * sizeof(double));
    allow_smem(k_refine_residual<kPrecNone, true>, smem_init<double>());
    allow_smem(k_refine_residual<kPrecJacobi, true>, smem_init<double>());
    allow_smem(k_refine_residual<kPrecVcycle, true>, smem_init<double>());
    allow_smem(k_refine_residual<kPrecNone, false>, smem_init<double>());
    allow_smem(k_refine_residual<kPrecJacobi, false>, smem_init<double>());
    allow_smem(k_refine_residual<kPrecVcycle, false>, smem_init<double>());
    done = true;
}

#define PMB_INST(T)                                                                              \
    template void launch_cg_init<T>(int, const LaunchCfg&, const WorkList&, const CUtensorMap*,   \
                                    const T*, const T*, T*, bool, T*, T*, InstState*, double*,    \
                                    double, double, int, int*, cudaStream_t);                     \
    template void launch_cg_apply<T>(int, int, const LaunchCfg&, const WorkList&,                 \
                                     const CUtensorMap*, int, T*, T*, T*, InstState*, double*,    \
                                     int*, cudaStream_t);                                         \
    template void launch_cg_update<T>(int, const LaunchCfg&, const WorkList&, const T*, T*, T*,   \
                                      T*, const T*, const T*, const T*, T*, int, int, int*,      \
                                      InstState*, double*, cudaStream_t);                        \
    template void launch_cg_rz<T>(const LaunchCfg&, const WorkList&, const T*, const T*,          \
                                  const T*, int, InstState*, double*, cudaStream_t);             \
    template void launch_vc_down<T>(int, int, const LaunchCfg&, const WorkList&, const GridDesc*, \
                                    const CUtensorMap*, int, T*, double, const InstState*, int*, \
                                    cudaStream_t);                                               \
    template void launch_vc_up<T>(int, int, int, int, const LaunchCfg&, const WorkList&,         \
                                  const GridDesc*, const CUtensorMap*, int, const T*, T*, double, \
                                  InstState*, int, const T*, int, double*, int*, cudaStream_t);  \
    template void launch_vc_smooth<T>(const LaunchCfg&, const WorkList&, const CUtensorMap*, int, \
                                      const T*, const T*, T*, double, const InstState*, int*,    \
                                      cudaStream_t);                                             \
    template void launch_vc_direct<T>(const DirectDesc*, int, const T*, T*, InstState*, int,      \
                                      cudaStream_t);                                             \
    template void launch_apply<T>(const LaunchCfg&, const WorkList&, const CUtensorMap*, T*, int*, \
                                  cudaStream_t);                                                 \
    template size_t smem_apply<T>();                                                              \
    template size_t smem_init<T>();                                                               \
    template size_t smem_down<T>(int);                                                            \
    template size_t smem_up<T>(int);                                                              \
    template size_t smem_apply_v<T>(int);                                                         \
    template int resident_cg_apply<T>(int, int);                                                  \
    template int resident_down<T>(int);                                                           \
    template int resident_cg_update<T>(int);                                                      \
    template int resident_up<T>(int, int);                                                        \
    template size_t smem_down_v<T>(int);                                                          \
    template size_t smem_up_v<T>(int);                                                            \
    template int down_box_width<T>();

PMB_INST(double)
PMB_INST(float)
#undef PMB_INST

template void launch_vc_tail<double>(const TailDesc<double>*, int, size_t, const InstState*,
                                     double, int*, cudaStream_t);
template void launch_vc_tail<float>(const TailDesc<float>*, int, size_t, const InstState*, double,
                                    int*, cudaStream_t);
template void launch_pack<double, double>(const GridDesc*, int, const int64_t*, const double*, double*, int64_t, cudaStream_t);
template void launch_pack<double, float>(const GridDesc*, int, const int64_t*, const double*, float*, int64_t, cudaStream_t);
template void launch_pack<float, double>(const GridDesc*, int, const int64_t*, const float*, double*, int64_t, cudaStream_t);
template void launch_unpack<double, double>(const GridDesc*, int, const int64_t*, const double*, double*, int64_t, cudaStream_t);
template void launch_unpack<float, double>(const GridDesc*, int, const int64_t*, const float*, double*, int64_t, cudaStream_t);
template void launch_unpack<double, float>(const GridDesc*, int, const int64_t*, const double*, float*, int64_t, cudaStream_t);

}  // namespace pmb
