// Thresholded incomplete Cholesky factorisation and its triangular solves.
//
// Restates pymatting/preconditioner/ichol.py:
//   _ichol :6-113           column-by-column factorisation with absolute and
//                           relative discard thresholds, diagonal compensation
//                           of discarded entries, failure codes -1 (not
//                           positive definite) / -2 (more than max_nnz);
//   _backsub_L_csc_inplace  :116-129  and  _backsub_LT_csc_inplace :132-145.
//
// The factorisation is inherently sequential over columns (column j needs
// every column k < j that has a kept entry in row j). Instead of the
// reference's left-looking linked lists, one CTA runs it right-looking over
// a dense band "front": when column k is final, its kept entries update the
// pending columns k+1 .. k+B directly (B = bandwidth of A; fill never leaves
// the envelope). Per column, warp 0 does the serial part with warp ballots
// (candidate rows, pivot, thresholding, compaction), then the whole CTA does
// the pair updates while the last warp recycles the column's front slot:
// two block barriers per column. Diagonal
// updates happen in the same column order as the reference; the off-
// diagonal accumulations differ only in summation order.
//
// The factor's dependency levels (level[i] = 1 + max level of the columns
// that update row i) fall out of the factorisation for free and drive the
// level-scheduled triangular solves: one thread per row inside a level,
// rows subtract their terms in the reference's order, levels separated by
// block barriers (single CTA: the systems this preconditioner is used on
// are the compressed unknown regions, tens of thousands of rows).
#include "pm_common.cuh"
#include "ichol.cuh"

namespace pmb {

constexpr int kIcholThreads = 1024;
constexpr int kIcholChunks = 8;      // front columns of up to 256 rows load in one burst
constexpr int64_t kIcholSmemRows = 27 * 1024;   // x of the shared-memory solve: 216 KB

// Per-column statistics of A (lower part, CSC): diagonal (+ shift), sum of
// |A[j:, j]| for the relative threshold, and the largest i - j.
__global__ void k_ichol_init(int64_t n, const int64_t* __restrict__ Ap,
                             const int64_t* __restrict__ Ar, const double* __restrict__ Av,
                             double shift, double* d, double* rsum, int* level,
                             unsigned long long* band) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double dj = shift, rj = 0.0;
    int64_t bmax = 0;
    for (int64_t k = Ap[j]; k < Ap[j + 1]; ++k) {
        const int64_t i = Ar[k];
        if (i == j) dj += Av[k];
        if (i >= j) rj += fabs(Av[k]);
        if (i > j && Av[k] != 0.0 && i - j > bmax) bmax = i - j;
    }
    d[j] = dj;
    rsum[j] = rj;
    level[j] = 0;
    if (bmax > 0) atomicMax(band, (unsigned long long)bmax);
}

// Load column j of A (entries below the diagonal with non-zero value) into
// its front slot. The slot was cleared beforehand.
__device__ __forceinline__ void load_column(int64_t j, int64_t W, const int64_t* __restrict__ Ap,
                                            const int64_t* __restrict__ Ar,
                                            const double* __restrict__ Av, double* F,
                                            uint8_t* pat) {
    const int64_t slot = (j % W) * W;
    for (int64_t k = Ap[j] + threadIdx.x; k < Ap[j + 1]; k += blockDim.x) {
        const int64_t i = Ar[k];
        const double v = Av[k];
        if (i > j && v != 0.0) {
            // Canonical input has one entry per (i, j): no two threads
            // write the same offset.
            F[slot + (i - j)] += v;
            pat[slot + (i - j)] = 1;
        }
    }
}

// The factorisation. One CTA. Front F / pat: W x W (W = B + 1), slot of
// column j = j % W, entry (i, j) at offset i - j. cand / kept: scratch of
// at least W entries each.
__global__ void __launch_bounds__(kIcholThreads)
k_ichol_factor(int64_t n, int64_t W, const int64_t* __restrict__ Ap,
               const int64_t* __restrict__ Ar, const double* __restrict__ Av, double* d,
               const double* __restrict__ rsum, int* level, double* F, uint8_t* pat, int* cand,
               double* keptv, int64_t* kepti, int64_t* Lp, int64_t* Lr, double* Lv,
               int64_t cap, double discard, int64_t max_nnz, double rel_discard, int diag_keep,
               int64_t* result) {
    __shared__ int64_t s_nnz;
    __shared__ int s_m, s_fail;
    __shared__ double s_keptv[kIcholChunks * 32];     // kept entries of the column
    __shared__ int64_t s_kepti[kIcholChunks * 32];

    // Initial front: columns 0 .. W-1.
    for (int64_t j = 0; j < W && j < n; ++j) load_column(j, W, Ap, Ar, Av, F, pat);
    if (threadIdx.x == 0) {
        s_nnz = 0;
        s_fail = 0;
        Lp[0] = 0;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t j = 0; j < n; ++j) {
        const int64_t slot = (j % W) * W;
        // Warp 0: the serial part of column j, warp-synchronous. Offsets
        // o = 1 + lane + 32 k: chunk k, lane order = ascending rows, the
        // order in which the reference sorts its candidates (ichol.py:87-89).
        // The pattern flags and front values of the first kIcholChunks
        // chunks, the pivot and the threshold are loaded in one burst.
        if (warp == 0) {
            bool flag[kIcholChunks];
            double aval[kIcholChunks];
#pragma unroll
            for (int k = 0; k < kIcholChunks; ++k) {
                const int64_t o = 1 + lane + 32 * k;
                flag[k] = o < W && j + o < n && pat[slot + o];
                aval[k] = flag[k] ? F[slot + o] : 0.0;
            }
            const double dj = d[j];
            const double rel = rel_discard * rsum[j];
            int cn = 0;
#pragma unroll
            for (int k = 0; k < kIcholChunks; ++k) cn += __popc(__ballot_sync(0xffffffffu, flag[k]));
            for (int64_t base = 1 + 32 * kIcholChunks; base < W; base += 32) {   // wide bands
                const int64_t o = base + lane;
                cn += __popc(__ballot_sync(0xffffffffu, o < W && j + o < n && pat[slot + o]));
            }
            int fail = 0;
            const int64_t nnz = s_nnz;
            if (!(dj > 0.0)) fail = -1;                                   // ichol.py:80-81
            else if (nnz + 1 + cn > max_nnz || nnz + 1 + cn > cap) fail = -2;   // ichol.py:82-83
            int kept = 0;
            int64_t nnz0 = nnz + 1;
            if (!fail) {
                const double sj = sqrt(dj);
                if (lane == 0) {
                    d[j] = sj;
                    Lv[nnz] = sj;
                    Lr[nnz] = j;
                }
                auto take = [&](bool fl, double a, int64_t o) {
                    bool keep = false;
                    double L = 0.0;
                    const int64_t i = j + o;
                    if (fl) {
                        L = a / sj;
                        if (diag_keep) d[i] -= L * L;
                        keep = fabs(L) > discard && fabs(a) > rel;
                        if (keep && !diag_keep) d[i] -= L * L;
                    }
                    const unsigned mask = __ballot_sync(0xffffffffu, keep);
                    if (keep) {
                        const int pos = kept + __popc(mask & ((1u << lane) - 1u));
                        Lv[nnz0 + pos] = L;
                        Lr[nnz0 + pos] = i;
                        keptv[pos] = L;
                        kepti[pos] = i;
                        if (pos < kIcholChunks * 32) {
                            s_keptv[pos] = L;
                            s_kepti[pos] = i;
                        }
                    }
                    kept += __popc(mask);
                };
#pragma unroll
                for (int k = 0; k < kIcholChunks; ++k) take(flag[k], aval[k], 1 + lane + 32 * k);
                for (int64_t base = 1 + 32 * kIcholChunks; base < W; base += 32) {
                    const int64_t o = base + lane;
                    const bool fl = o < W && j + o < n && pat[slot + o];
                    take(fl, fl ? F[slot + o] : 0.0, o);
                }
            }
            if (lane == 0) {
                s_fail = fail;
                if (!fail) {
                    s_m = kept;
                    s_nnz = nnz0 + kept;
                    Lp[j + 1] = nnz0 + kept;
                }
            }
        }
        __syncthreads();
        if (s_fail) break;
        const int m = s_m;
        // Levels of the rows this column feeds.
        const int lj = level[j] + 1;
        for (int q = threadIdx.x; q < m; q += blockDim.x) {
            const int64_t i = m <= kIcholChunks * 32 ? s_kepti[q] : kepti[q];
            if (level[i] < lj) level[i] = lj;
        }
        // Right-looking update of the pending columns: for kept rows
        // ia > ib, F[ib][ia - ib] -= L_ia L_ib, one pair per thread. Rows ib
        // lie in (j, j + W), so no update touches slot j.
        const bool shared_list = m <= kIcholChunks * 32;
        const double* kv = shared_list ? s_keptv : keptv;
        const int64_t* ki = shared_list ? s_kepti : kepti;
        const int64_t pairs = (int64_t)m * (m - 1) / 2;
        for (int64_t p = threadIdx.x; p < pairs; p += blockDim.x) {
            // Invert p = a (a - 1) / 2 + b with 0 <= b < a.
            int64_t a = (int64_t)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
            while (a * (a - 1) / 2 > p) --a;
            while ((a + 1) * a / 2 <= p) ++a;
            const int64_t b = p - a * (a - 1) / 2;
            const int64_t ia = ki[a], ib = ki[b];
            const int64_t off = ((ib % W) * W) + (ia - ib);
            F[off] -= kv[a] * kv[b];
            pat[off] = 1;
        }
        // Meanwhile the last warp recycles slot j for column j + W (clear,
        // then load; ordered within the warp).
        if (warp == (int)(blockDim.x >> 5) - 1) {
            for (int64_t o = lane; o < W; o += 32) {
                F[slot + o] = 0.0;
                pat[slot + o] = 0;
            }
            __syncwarp();
            if (j + W < n) {
                const int64_t jn = j + W;
                for (int64_t k = Ap[jn] + lane; k < Ap[jn + 1]; k += 32) {
                    const int64_t i = Ar[k];
                    const double v = Av[k];
                    if (i > jn && v != 0.0) {
                        F[slot + (i - jn)] += v;
                        pat[slot + (i - jn)] = 1;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *result = s_fail ? (int64_t)s_fail : s_nnz;
}

// Level histogram / order of rows, and the row (CSR) view of L used by the
// forward solve. All small single-purpose kernels.
__global__ void k_level_count(int64_t n, const int* __restrict__ level, int64_t* cnt,
                              int* maxlevel) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicAdd((unsigned long long*)&cnt[level[i]], 1ull);
    atomicMax(maxlevel, level[i]);
}

__global__ void k_level_scatter(int64_t n, const int* __restrict__ level, int64_t* fill,
                                int* order) {
    // Sequential within one thread per level bucket would be slow; rows are
    // placed with atomics, then each level segment is sorted by row.
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long at = atomicAdd((unsigned long long*)&fill[level[i]], 1ull);
    order[at] = (int)i;
}

// Insertion-sort each level segment so the schedule is deterministic.
__global__ void k_level_sort(const int64_t* __restrict__ lptr, int nlevels, int* order) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlevels) return;
    const int64_t a = lptr[l], b = lptr[l + 1];
    for (int64_t k = a + 1; k < b; ++k) {
        const int v = order[k];
        int64_t q = k - 1;
        while (q >= a && order[q] > v) {
            order[q + 1] = order[q];
            --q;
        }
        order[q + 1] = v;
    }
}

__global__ void k_row_count(int64_t n, const int64_t* __restrict__ Lp, const int64_t* __restrict__ Lr,
                            int64_t* rcnt) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int64_t k = Lp[j] + 1; k < Lp[j + 1]; ++k)
        atomicAdd((unsigned long long*)&rcnt[Lr[k]], 1ull);
}

// Row view entries in ascending column order: column j writes its entry
// of row i at the slot given by the number of columns < j with an entry in
// row i — computed by walking columns in order within one thread per row
// would be quadratic, so entries are appended with atomics and each row is
// sorted afterwards.
__global__ void k_row_fill(int64_t n, const int64_t* __restrict__ Lp, const int64_t* __restrict__ Lr,
                           const double* __restrict__ Lv, int64_t* rfill, int64_t* Rc, double* Rv) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int64_t k = Lp[j] + 1; k < Lp[j + 1]; ++k) {
        const int64_t i = Lr[k];
        const unsigned long long at = atomicAdd((unsigned long long*)&rfill[i], 1ull);
        Rc[at] = j;
        Rv[at] = Lv[k];
    }
}

__global__ void k_row_sort(int64_t n, const int64_t* __restrict__ Rp, int64_t* Rc, double* Rv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int64_t k = Rp[i] + 1; k < Rp[i + 1]; ++k) {
        const int64_t c = Rc[k];
        const double v = Rv[k];
        int64_t q = k - 1;
        while (q >= Rp[i] && Rc[q] > c) {
            Rc[q + 1] = Rc[q];
            Rv[q + 1] = Rv[q];
            --q;
        }
        Rc[q + 1] = c;
        Rv[q + 1] = v;
    }
}

// x = L^-T L^-1 b. Forward: y_i = (b_i - sum_{j<i} L_ij y_j) / L_ii with
// the subtractions in ascending j (the column sweep of
// _backsub_L_csc_inplace applies them in that order); backward: x_i =
// (y_i - sum_{k>i} L_ki x_k) / L_ii over column i in ascending k
// (_backsub_LT_csc_inplace). Levels run forward, then in reverse.
__global__ void __launch_bounds__(kIcholThreads)
k_ichol_solve(int64_t n, int nlevels, const int64_t* __restrict__ lptr, const int* __restrict__ order,
              const int64_t* __restrict__ Lp, const int64_t* __restrict__ Lr,
              const double* __restrict__ Lv, const int64_t* __restrict__ Rp,
              const int64_t* __restrict__ Rc, const double* __restrict__ Rv,
              const double* __restrict__ b, double* x, const InstState* st) {
    if (st && st->status != kRunning) return;
    for (int l = 0; l < nlevels; ++l) {
        for (int64_t q = lptr[l] + threadIdx.x; q < lptr[l + 1]; q += blockDim.x) {
            const int64_t i = order[q];
            double s = b[i];
            for (int64_t k = Rp[i]; k < Rp[i + 1]; ++k) s -= Rv[k] * x[Rc[k]];
            x[i] = s / Lv[Lp[i]];
        }
        __syncthreads();
    }
    for (int l = nlevels - 1; l >= 0; --l) {
        for (int64_t q = lptr[l] + threadIdx.x; q < lptr[l + 1]; q += blockDim.x) {
            const int64_t i = order[q];
            double s = x[i];
            for (int64_t k = Lp[i] + 1; k < Lp[i + 1]; ++k) s -= Lv[k] * x[Lr[k]];
            x[i] = s / Lv[Lp[i]];
        }
        __syncthreads();
    }
}

// The same solves with x in shared memory (n <= kIcholSmemRows) and one warp
// per row: the lanes split the row's dot product (so the subtractions of a
// row are summed in a different order than the reference, a difference of
// rounding only) and each warp loads the index/value data of its first row
// of the next level before the level barrier, so a level costs one shared-
// memory gather, a warp reduction and a barrier.
struct RowPrefetch {
    int64_t i, k0, k1;
    int64_t c;     // first entry of this lane (column / row index)
    double v;
};

template <bool FWD>
__device__ __forceinline__ RowPrefetch prefetch_row(int64_t q, int64_t qend, const int* order,
                                                    const int64_t* Xp, const int64_t* Xi,
                                                    const double* Xv, int lane) {
    RowPrefetch r{-1, 0, 0, 0, 0.0};
    if (q < qend) {
        r.i = order[q];
        r.k0 = Xp[r.i] + (FWD ? 0 : 1);
        r.k1 = Xp[r.i + 1];
        const int64_t k = r.k0 + lane;
        if (k < r.k1) {
            r.c = Xi[k];
            r.v = Xv[k];
        }
    }
    return r;
}

template <bool FWD>
__device__ __forceinline__ void solve_sweep(int nlevels, const int64_t* __restrict__ lptr,
                                            const int* __restrict__ order,
                                            const int64_t* __restrict__ Xp,
                                            const int64_t* __restrict__ Xi,
                                            const double* __restrict__ Xv,
                                            const int64_t* __restrict__ Lp,
                                            const double* __restrict__ Lv, double* sx) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int l = FWD ? 0 : nlevels - 1;
    RowPrefetch pf = prefetch_row<FWD>(lptr[l] + warp, lptr[l + 1], order, Xp, Xi, Xv, lane);
    for (int step = 0; step < nlevels; ++step, l += FWD ? 1 : -1) {
        const int64_t qend = lptr[l + 1];
        int64_t q = lptr[l] + warp;
        RowPrefetch cur = pf;
        // Prefetch this warp's first row of the next level (its data does
        // not depend on x).
        if (step + 1 < nlevels) {
            const int ln = FWD ? l + 1 : l - 1;
            pf = prefetch_row<FWD>(lptr[ln] + warp, lptr[ln + 1], order, Xp, Xi, Xv, lane);
        }
        while (cur.i >= 0) {
            double acc = (cur.k0 + lane < cur.k1) ? cur.v * sx[cur.c] : 0.0;
            for (int64_t k = cur.k0 + 32 + lane; k < cur.k1; k += 32) acc += Xv[k] * sx[Xi[k]];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) sx[cur.i] = (sx[cur.i] - acc) / Lv[Lp[cur.i]];
            q += nw;
            cur = prefetch_row<FWD>(q, qend, order, Xp, Xi, Xv, lane);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kIcholThreads)
k_ichol_solve_smem(int64_t n, int nlevels, const int64_t* __restrict__ lptr,
                   const int* __restrict__ order, const int64_t* __restrict__ Lp,
                   const int64_t* __restrict__ Lr, const double* __restrict__ Lv,
                   const int64_t* __restrict__ Rp, const int64_t* __restrict__ Rc,
                   const double* __restrict__ Rv, const double* __restrict__ b, double* x,
                   const InstState* st) {
    extern __shared__ double s_x[];
    if (st && st->status != kRunning) return;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s_x[i] = b[i];
    __syncthreads();
    if (nlevels > 0) {
        solve_sweep<true>(nlevels, lptr, order, Rp, Rc, Rv, Lp, Lv, s_x);
        solve_sweep<false>(nlevels, lptr, order, Lp, Lr, Lv, Lp, Lv, s_x);
    }
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = s_x[i];
}

// The forward sweep above overwrites x in place: y lives in x. For the
// forward pass to read y_j of earlier levels and b_i of its own row, b and
// x may alias (the reference also works in place on a copy of b).

void ichol_launch_init(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                       double shift, double* d, double* rsum, int* level, unsigned long long* band,
                       cudaStream_t s) {
    if (n > 0) k_ichol_init<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Ap, Ar, Av, shift, d, rsum, level, band);
}

void ichol_launch_factor(int64_t n, int64_t W, const int64_t* Ap, const int64_t* Ar,
                         const double* Av, double* d, const double* rsum, int* level, double* F,
                         uint8_t* pat, int* cand, double* keptv, int64_t* kepti, int64_t* Lp,
                         int64_t* Lr, double* Lv, int64_t cap, double discard, int64_t max_nnz,
                         double rel, int diag_keep, int64_t* result, cudaStream_t s) {
    k_ichol_factor<<<1, kIcholThreads, 0, s>>>(n, W, Ap, Ar, Av, d, rsum, level, F, pat, cand, keptv,
                                               kepti, Lp, Lr, Lv, cap, discard, max_nnz, rel,
                                               diag_keep, result);
}

void ichol_launch_levels(int64_t n, const int* level, int64_t* cnt, int* maxlevel, cudaStream_t s) {
    if (n > 0) k_level_count<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, level, cnt, maxlevel);
}

void ichol_launch_level_scatter(int64_t n, const int* level, int64_t* fill, int* order,
                                const int64_t* lptr, int nlevels, cudaStream_t s) {
    if (n > 0) k_level_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, level, fill, order);
    if (nlevels > 0) k_level_sort<<<(nlevels + 127) / 128, 128, 0, s>>>(lptr, nlevels, order);
}

void ichol_launch_rows(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                       int64_t* rcnt, cudaStream_t s) {
    if (n > 0) k_row_count<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Lp, Lr, rcnt);
}

void ichol_launch_row_fill(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                           int64_t* rfill, int64_t* Rc, double* Rv, const int64_t* Rp,
                           cudaStream_t s) {
    if (n > 0) {
        k_row_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Lp, Lr, Lv, rfill, Rc, Rv);
        k_row_sort<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Rp, Rc, Rv);
    }
}

// Raise the shared-memory limit of the shared-memory solve; called when a
// factor is built, before any solve can be captured.
void ichol_prepare() {
    cudaFuncSetAttribute(k_ichol_solve_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kIcholSmemRows * sizeof(double)));
}

void ichol_launch_solve(int64_t n, int nlevels, const int64_t* lptr, const int* order,
                        const int64_t* Lp, const int64_t* Lr, const double* Lv, const int64_t* Rp,
                        const int64_t* Rc, const double* Rv, const double* b, double* x,
                        const InstState* st, cudaStream_t s) {
    if (n <= kIcholSmemRows) {
        k_ichol_solve_smem<<<1, kIcholThreads, n * sizeof(double), s>>>(
            n, nlevels, lptr, order, Lp, Lr, Lv, Rp, Rc, Rv, b, x, st);
        return;
    }
    k_ichol_solve<<<1, kIcholThreads, 0, s>>>(n, nlevels, lptr, order, Lp, Lr, Lv, Rp, Rc, Rv, b, x, st);
}

}  // namespace pmb
