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
#include <cooperative_groups.h>

#include "pm_common.cuh"
#include "ichol.cuh"
#include "tma.cuh"

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

// ---------------------------------------------------------------------------
// The same factorisation with the front on chip: a cluster of C CTAs keeps the
// W x W front in distributed shared memory, CTA r owning the slots s with
// s mod C = r (at most S = ceil(W / C) of them) with their FP64 values,
// pattern bytes, ring entries of the diagonal d and of the dependency level.
// Per column j:
//
//   phase F  warp 0 of EVERY CTA reads slot j from its owner (one DSMEM round
//            trip) and runs the serial part of the column (pivot, threshold,
//            compaction) on identical data with identical instructions, so all
//            CTAs hold the same kept list and take the same control path; the
//            owner writes the column of L. Meanwhile the last warp recycles the
//            slot of column j - 1 for column j - 1 + W from registers it loaded
//            one column earlier (A's entries) and two columns earlier (A's
//            column pointers), so no global load latency is on the chain.
//   phase P  each CTA applies the pair updates F[ib][ia - ib] -= L_ia L_ib whose
//            target column ib it owns, and the diagonal and level updates of
//            the rows it owns: every write is CTA-local.
//
// One cluster barrier per column orders phase P of column j before phase F of
// column j + 1 in every CTA. Updates land in the same order as in
// k_ichol_factor (column order, one pair per front entry per column), so the
// two kernels produce identical factors.
// ---------------------------------------------------------------------------

constexpr int kClThreads = 512;
constexpr int kClMaxChunks = 14;      // offsets 1 .. W - 1 in chunks of 32: W <= 449
constexpr int kClMaxCluster = 8;      // portable cluster size
constexpr size_t kClSmemLimit = 227 * 1024 - 256;

struct ClLayout {
    int64_t Wp, S;
    size_t o_F, o_d, o_kv, o_cL, o_lev, o_ki, o_ci, o_own, o_pre, o_pat, bytes;
};

__host__ __device__ inline ClLayout cl_layout(int64_t W, int C) {
    ClLayout L;
    L.Wp = (W + 7) & ~(int64_t)7;
    L.S = (W + C - 1) / C;
    size_t o = 0;
    L.o_F = o;   o += (size_t)(L.S * L.Wp) * sizeof(double);
    L.o_d = o;   o += (size_t)L.S * sizeof(double);
    L.o_kv = o;  o += (size_t)W * sizeof(double);
    L.o_cL = o;  o += (size_t)W * sizeof(double);
    L.o_lev = o; o += (size_t)L.S * sizeof(int);
    L.o_ki = o;  o += (size_t)W * sizeof(int);
    L.o_ci = o;  o += (size_t)W * sizeof(int);
    L.o_own = o; o += (size_t)W * sizeof(int);
    L.o_pre = o; o += (size_t)W * sizeof(int);
    L.o_pat = o; o += (size_t)(L.S * L.Wp);
    L.bytes = (o + 15) & ~(size_t)15;
    return L;
}

// Smallest cluster size whose per-CTA share of the front fits in shared
// memory; 0 when none up to the portable limit does (or W is too wide for
// the register chunks of phase F).
int ichol_cluster_size(int64_t W) {
    if (W < 1 || W - 1 > 32 * kClMaxChunks) return 0;
    for (int C = 1; C <= kClMaxCluster; ++C)
        if (cl_layout(W, C).bytes <= kClSmemLimit) return C;
    return 0;
}

// NCH: 32-offset chunks of a front column held in registers by phase F
// (ceil((W - 1) / 32) rounded up to 2, 4, 8 or 14). Slots are tracked
// incrementally in 32-bit arithmetic. Phase F compacts the column's
// candidates first and divides only those, lane-strided: an FP64 division
// costs about 130 cycles of latency (about 300 with a zero numerator), and
// a column has a quarter of its offsets as candidates or fewer.
template <int NCH>
__global__ void __launch_bounds__(kClThreads, 1)
k_ichol_factor_cluster(int64_t n, int W, int C, const int64_t* __restrict__ Ap,
                       const int64_t* __restrict__ Ar, const double* __restrict__ Av,
                       const double* __restrict__ d0, const double* __restrict__ rsum,
                       int* level, int64_t* Lp, int64_t* Lr, double* Lv, int64_t cap,
                       double discard, int64_t max_nnz, double rel_discard, int diag_keep,
                       int64_t* result) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char cl_smem[];
    __shared__ int64_t s_nnz;
    __shared__ int s_cn, s_nown, s_np, s_levj, s_kept, s_owner, s_fail;
    __shared__ double s_sj;
    const ClLayout Ly = cl_layout(W, C);
    const int S = (int)Ly.S, Wp = (int)Ly.Wp;
    double* F = reinterpret_cast<double*>(cl_smem + Ly.o_F);
    double* dl = reinterpret_cast<double*>(cl_smem + Ly.o_d);
    double* kv = reinterpret_cast<double*>(cl_smem + Ly.o_kv);
    double* cL = reinterpret_cast<double*>(cl_smem + Ly.o_cL);
    int* lev = reinterpret_cast<int*>(cl_smem + Ly.o_lev);
    int* ki = reinterpret_cast<int*>(cl_smem + Ly.o_ki);
    int* ci = reinterpret_cast<int*>(cl_smem + Ly.o_ci);
    int* own = reinterpret_cast<int*>(cl_smem + Ly.o_own);
    int* pre = reinterpret_cast<int*>(cl_smem + Ly.o_pre);
    uint8_t* pat = cl_smem + Ly.o_pat;
    const int r = (int)cluster.block_rank();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    // Slot s belongs to CTA s mod C at local index s / C (interleaved, so the
    // heavy targets just below the pivot spread over the cluster). s < 449
    // and C <= 8: (s * mC) >> 16 with mC = ceil(65536 / C) is s / C exactly.
    const int mC = (65536 + C - 1) / C;
    auto divC = [mC](int v) { return (v * mC) >> 16; };

    // Initial front: columns 0 .. min(W, n) - 1 sit in slots 0 .. W - 1.
    for (int q = threadIdx.x; q < S * Wp; q += blockDim.x) {
        F[q] = 0.0;
        pat[q] = 0;
    }
    __syncthreads();
    for (int ls = warp; r + ls * C < W; ls += nw) {
        const int64_t c = r + ls * C;
        if (c >= n) continue;
        for (int64_t k = Ap[c] + lane; k < Ap[c + 1]; k += 32) {
            const int64_t i = Ar[k];
            const double v = Av[k];
            if (i > c && v != 0.0) {
                F[ls * Wp + (int)(i - c)] = v;
                pat[ls * Wp + (int)(i - c)] = 1;
            }
        }
        if (lane == 0) {
            dl[ls] = d0[c];
            lev[ls] = 0;
        }
    }
    if (threadIdx.x == 0) {
        s_nnz = 0;
        s_fail = 0;
        if (r == 0) Lp[0] = 0;
    }
    cluster.sync();

    // Last warp: A's column pointers of column j + W (loaded a column ahead)
    // and entries of column j - 1 + W (loaded at the previous column).
    int64_t pk0 = 0, pk1 = 0, ebeg = 0, eend = 0;
    int64_t ei[2] = {-1, -1};
    double ev[2] = {0.0, 0.0}, ed0 = 0.0;
    if (warp == nw - 1 && W < n) {
        pk0 = Ap[W];
        pk1 = Ap[W + 1];
    }
    double rs_next = (warp == 0) ? rsum[0] : 0.0;
    int slot = 0, pslot = W - 1;      // j % W and (j - 1) % W

    for (int64_t j = 0; j < n; ++j) {
        if (warp == 0) {
            const int lsj = divC(slot), f = slot - lsj * C;
            const double rs = rs_next;
            if (j + 1 < n) rs_next = rsum[j + 1];
            const double* Fj = cluster.map_shared_rank(F, f) + lsj * Wp;
            const uint8_t* Pj = cluster.map_shared_rank(pat, f) + lsj * Wp;
            const double dj = cluster.map_shared_rank(dl, f)[lsj];
            const int levj = cluster.map_shared_rank(lev, f)[lsj];
            // Offsets o = 1 + lane + 32 k: lane order is ascending rows, the
            // order in which the reference sorts its candidates (ichol.py:87-89).
            double a[NCH];
            bool flag[NCH];
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                const int o = 1 + lane + 32 * k;
                const bool in = o < W && j + o < n;
                a[k] = in ? Fj[o] : 0.0;
                flag[k] = in && Pj[o] != 0;
            }
            unsigned fm[NCH];
            int cn = 0;
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                fm[k] = __ballot_sync(0xffffffffu, flag[k]);
                cn += __popc(fm[k]);
            }
            const int64_t nnz = s_nnz;
            int fail = 0;
            if (!(dj > 0.0)) fail = -1;                                         // ichol.py:80-81
            else if (nnz + 1 + cn > max_nnz || nnz + 1 + cn > cap) fail = -2;   // ichol.py:82-83
            const bool owner = f == r;
            const int64_t nnz0 = nnz + 1;
            // Candidates in ascending rows: value and offset, compacted.
            int cpos = 0;
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                if (flag[k]) {
                    const int q = cpos + __popc(fm[k] & lt);
                    cL[q] = a[k];
                    ci[q] = 1 + lane + 32 * k;
                }
                cpos += __popc(fm[k]);
            }
            __syncwarp();
            int kept = 0, nown = 0;
            if (!fail) {
                const double sj = sqrt(dj);
                const double rel = rel_discard * rs;
                if (lane == 0) s_sj = sj;
                // One quotient per candidate, lane-strided (the candidates
                // of a column are a quarter of its offsets or fewer).
                for (int t0 = 0; t0 < cn; t0 += 32) {
                    const int t = t0 + lane;
                    double L = 0.0;
                    bool keep = false, mine = false;
                    int o = 0;
                    if (t < cn) {
                        const double av = cL[t];
                        o = ci[t];
                        L = av / sj;
                        keep = fabs(L) > discard && fabs(av) > rel;
                        int sl = slot + o;
                        if (sl >= W) sl -= W;
                        mine = keep && sl - divC(sl) * C == r;
                        cL[t] = L;
                        ci[t] = keep ? o : -o;
                    }
                    const unsigned km = __ballot_sync(0xffffffffu, keep);
                    const unsigned om = __ballot_sync(0xffffffffu, mine);
                    if (keep) {
                        const int pos = kept + __popc(km & lt);
                        kv[pos] = L;
                        ki[pos] = o;
                        if (mine) own[nown + __popc(om & lt)] = pos;
                    }
                    kept += __popc(km);
                    nown += __popc(om);
                }
            }
            // Exclusive prefix of the owned targets' pair counts (kept - 1 -
            // pb pairs for the target at kept index pb).
            int np = 0;
            for (int t0 = 0; t0 < nown; t0 += 32) {
                const int t = t0 + lane;
                const int cnt = t < nown ? kept - 1 - own[t] : 0;
                int incl = cnt;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += v;
                }
                if (t < nown) pre[t] = np + incl - cnt;
                np += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) {
                s_fail = fail;
                if (!fail) {
                    s_cn = cn;
                    s_nown = nown;
                    s_np = np;
                    s_levj = levj;
                    s_kept = kept;
                    s_owner = owner;
                    s_nnz = nnz0 + kept;
                }
            }
        } else if (warp == nw - 1) {
            // Recycle slot (j - 1) % W for column c = j - 1 + W (its readers
            // all passed the barrier of column j - 1).
            const int64_t c = j - 1 + W;
            const int pls = divC(pslot);
            if (j >= 1 && c < n && pslot - pls * C == r) {
                double* Fc = F + pls * Wp;
                uint8_t* Pc = pat + pls * Wp;
                for (int o = lane; o < W; o += 32) {
                    Fc[o] = 0.0;
                    Pc[o] = 0;
                }
                __syncwarp();
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t k = ebeg + lane + 32 * e;
                    if (k < eend && ei[e] > c && ev[e] != 0.0) {
                        Fc[ei[e] - c] = ev[e];
                        Pc[ei[e] - c] = 1;
                    }
                }
                for (int64_t k = ebeg + 64 + lane; k < eend; k += 32) {   // rows longer than 64
                    const int64_t i = Ar[k];
                    const double v = Av[k];
                    if (i > c && v != 0.0) {
                        Fc[i - c] = v;
                        Pc[i - c] = 1;
                    }
                }
                if (lane == 0) {
                    dl[pls] = ed0;
                    lev[pls] = 0;
                }
            }
            // Entries of column j + W for the next column's recycle.
            if (j + W < n) {
                ebeg = pk0;
                eend = pk1;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t k = pk0 + lane + 32 * e;
                    ei[e] = k < pk1 ? Ar[k] : -1;
                    ev[e] = k < pk1 ? Av[k] : 0.0;
                }
                ed0 = d0[j + W];
            }
            // Column pointers of column j + 1 + W.
            if (j + 1 + W < n) {
                pk0 = Ap[j + 1 + W];
                pk1 = Ap[j + 2 + W];
            }
        }
        __syncthreads();
        if (s_fail) break;
        // Phase P: CTA-local updates of the rows and front columns owned here.
        // Pairs are spread evenly over the threads (target found by binary
        // search of the prefix); the diagonal and level updates go to the
        // threads with the fewest pairs.
        const int nown = s_nown, cn = s_cn, np = s_np, lj = s_levj + 1;
        // The owner of slot j writes column j of L from the kept list
        // (threads 128.., which have the fewest pairs besides the diagonal
        // and level updates).
        if (s_owner) {
            const int kept = s_kept;
            const int64_t end = s_nnz, nnz = end - kept - 1;
            for (int q = (int)((threadIdx.x + blockDim.x - 128) % blockDim.x); q <= kept;
                 q += blockDim.x) {
                if (q == 0) {
                    Lv[nnz] = s_sj;
                    Lr[nnz] = j;
                    level[j] = s_levj;
                    Lp[j + 1] = end;
                } else {
                    Lv[nnz + q] = kv[q - 1];
                    Lr[nnz + q] = j + ki[q - 1];
                }
            }
        }
        for (int p = threadIdx.x; p < np; p += blockDim.x) {
            int tl = 0, th = nown - 1;
            while (tl < th) {
                const int mid = (tl + th + 1) >> 1;
                if (pre[mid] <= p) tl = mid;
                else th = mid - 1;
            }
            const int pb = own[tl];
            const int q = pb + 1 + (p - pre[tl]);
            const int ob = ki[pb];
            int sl = slot + ob;
            if (sl >= W) sl -= W;
            const int o = ki[q] - ob;
            F[divC(sl) * Wp + o] -= kv[q] * kv[pb];
            pat[divC(sl) * Wp + o] = 1;
        }
        for (int q = (int)blockDim.x - 1 - (int)threadIdx.x; q < cn; q += blockDim.x) {
            const int code = ci[q];
            int sl = slot + (code < 0 ? -code : code);
            if (sl >= W) sl -= W;
            const int ls = divC(sl);
            if (sl - ls * C != r || (!diag_keep && code < 0)) continue;
            dl[ls] -= cL[q] * cL[q];
        }
        for (int t = (int)(threadIdx.x ^ (blockDim.x >> 1)); t < nown; t += blockDim.x) {
            int sl = slot + ki[own[t]];
            if (sl >= W) sl -= W;
            const int ls = divC(sl);
            if (lev[ls] < lj) lev[ls] = lj;
        }
        pslot = slot;
        slot = slot + 1 == W ? 0 : slot + 1;
        cluster.sync();
    }
    // No CTA leaves while another may still read its shared memory.
    cluster.sync();
    if (r == 0 && threadIdx.x == 0) *result = s_fail ? (int64_t)s_fail : s_nnz;
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

// Rows of up to kRowSortMax entries: one warp per row, entries in registers
// (8 a lane); each entry's place is the number of smaller column indices in
// its row (the indices of a row are distinct), counted by broadcasting every
// key through the warp.
constexpr int kRowSortMax = 256;

__global__ void k_row_sort_warp(int64_t n, const int64_t* __restrict__ Rp, int64_t* Rc, double* Rv) {
    const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int64_t b = Rp[i];
    const int64_t len = Rp[i + 1] - b;
    if (len <= 1 || len > kRowSortMax) return;
    int64_t c[8];
    double v[8];
    int rank[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int k = lane + 32 * u;
        c[u] = k < len ? Rc[b + k] : INT64_MAX;
        v[u] = k < len ? Rv[b + k] : 0.0;
        rank[u] = 0;
    }
    const int U = (int)((len + 31) >> 5);
#pragma unroll
    for (int u2 = 0; u2 < 8; ++u2) {
        if (u2 < U) {
            for (int src = 0; src < 32; ++src) {
                const int64_t key = __shfl_sync(0xffffffffu, c[u2], src);
#pragma unroll
                for (int u = 0; u < 8; ++u) rank[u] += key < c[u] ? 1 : 0;
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int k = lane + 32 * u;
        if (k < len) {
            Rc[b + rank[u]] = c[u];
            Rv[b + rank[u]] = v[u];
        }
    }
}

// Longer rows: insertion sort by one thread.
__global__ void k_row_sort(int64_t n, const int64_t* __restrict__ Rp, int64_t* Rc, double* Rv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (Rp[i + 1] - Rp[i] <= kRowSortMax) return;
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

// ---------------------------------------------------------------------------
// Streamed level-scheduled solves (n <= kStreamMaxRows). Both sweeps run in
// one CTA with x in shared memory. The rows of each sweep, in level order,
// are packed at factorisation time into chunks (one level, or a part of a
// level, of at most kStreamRowsMax rows and kStreamEntsMax entries), each a
// contiguous 16-byte-aligned block:
//
//   StreamHead   own row and entry counts, and the offset / size of the
//                block kStreamStages chunks later (the next one to fetch
//                into this stage)
//   StreamRow[rows]   row index, first entry, entry count, diagonal
//   double[ents]      L values of the row terms
//   int[ents]         their x indices       (ents padded to a multiple of 4)
//
// One thread keeps kStreamStages chunks in flight with bulk copies into a
// shared-memory ring (completion on one mbarrier per stage); every chunk
// ends with the block barrier that separates levels and frees the stage.
// The data of a chunk never depends on x, so the copies run ahead of the
// dependency chain and no global-load latency sits on it. Within a row the
// terms are summed lane-strided and reduced across the warp, as in
// k_ichol_solve_smem, and x_i = (x_i - sum) / L_ii as the reference's
// back substitutions (ichol.py:116-145).
// ---------------------------------------------------------------------------

constexpr int kStreamThreads = 256;
constexpr size_t kStreamStageBytes =
    sizeof(StreamHead) + kStreamRowsMax * sizeof(StreamRow) + kStreamEntsMax * 12;
static_assert(kStreamStageBytes % 16 == 0, "stages are 16-byte aligned");

size_t ichol_stream_smem(int64_t n) {
    return kStreamStages * kStreamStageBytes + (size_t)n * sizeof(double);
}

__global__ void __launch_bounds__(kStreamThreads)
k_ichol_solve_stream(int64_t n, int total, StreamFirst first, const unsigned char* __restrict__ blob,
                     const double* __restrict__ b, double* x, const InstState* st, uint32_t limit) {
    extern __shared__ __align__(16) unsigned char ss_smem[];
    __shared__ uint64_t full[kStreamStages];
    __shared__ int s_bad;
    if (st && st->status != kRunning) return;
    double* sx = reinterpret_cast<double*>(ss_smem + kStreamStages * kStreamStageBytes);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        s_bad = 0;
        for (int q = 0; q < kStreamStages; ++q) mbar_init(&full[q], 1);
        for (int q = 0; q < kStreamStages && q < total; ++q) {
            if (first.bytes[q] <= 0) continue;
            mbar_expect_tx(&full[q], (uint32_t)first.bytes[q]);
            bulk_load(ss_smem + q * kStreamStageBytes, blob + first.off[q], (uint32_t)first.bytes[q],
                      &full[q]);
        }
    }
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) sx[i] = b[i];
    __syncthreads();
    int c = 0;
    for (; c < total; ++c) {
        const int q = c % kStreamStages;
        unsigned char* stage = ss_smem + q * kStreamStageBytes;
        if (!mbar_wait(&full[q], (uint32_t)(c / kStreamStages) & 1u, limit)) {
            s_bad = 1;
        } else {
            const StreamHead* h = reinterpret_cast<const StreamHead*>(stage);
            const StreamRow* rec = reinterpret_cast<const StreamRow*>(stage + sizeof(StreamHead));
            const int rows = h->rows, ents = h->ents;
            const double* val = reinterpret_cast<const double*>(stage + sizeof(StreamHead) +
                                                                rows * sizeof(StreamRow));
            const int* col = reinterpret_cast<const int*>(val + ents);
            for (int k = warp; k < rows; k += nw) {
                const StreamRow rw = rec[k];
                const double* rv = val + rw.start;
                const int* rc = col + rw.start;
                double acc = 0.0;
                int e = lane;
                for (; e + 32 < rw.count; e += 64) {     // two terms' loads in flight
                    const double v0 = rv[e], v1 = rv[e + 32];
                    const int c0 = rc[e], c1 = rc[e + 32];
                    const double x0 = sx[c0], x1 = sx[c1];
                    acc += v0 * x0;
                    acc += v1 * x1;
                }
                if (e < rw.count) acc += rv[e] * sx[rc[e]];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) sx[rw.row] = (sx[rw.row] - acc) / rw.diag;
            }
        }
        __syncthreads();          // level barrier; the stage is free again
        if (s_bad) break;
        // The last warp refills the stage: rows go to warps in order, so it
        // only has rows of its own in chunks of more than nw - 1 rows.
        if (threadIdx.x == blockDim.x - 32) {
            const StreamHead* h = reinterpret_cast<const StreamHead*>(stage);
            const int64_t off = h->next_off;
            const int bytes = h->next_bytes;
            if (bytes > 0) {
                fence_proxy_async();
                mbar_expect_tx(&full[q], (uint32_t)bytes);
                bulk_load(stage, blob + off, (uint32_t)bytes, &full[q]);
            }
        }
    }
    if (s_bad) {
        // A copy did not complete: the result is NaN, and copies still in
        // flight are waited for (bounded) before the CTA leaves.
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = __longlong_as_double(0x7ff8000000000000ll);
        if (threadIdx.x == blockDim.x - 32) {
            for (int k = c; k < c + kStreamStages && k < total; ++k)
                mbar_wait(&full[k % kStreamStages], (uint32_t)(k / kStreamStages) & 1u, limit);
        }
        __syncthreads();
        return;
    }
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = sx[i];
}

// Pack the chunk blocks of both sweeps. One warp per row record: its entries
// (x indices narrowed to int) and its record; one thread per chunk writes the
// head and zeroes the entry padding.
__global__ void k_stream_pack_rows(int nrec, const StreamPackRow* __restrict__ recs,
                                   const int64_t* __restrict__ Rc, const double* __restrict__ Rv,
                                   const int64_t* __restrict__ Lr, const double* __restrict__ Lv,
                                   const int64_t* __restrict__ Lp, unsigned char* blob) {
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= nrec) return;
    const StreamPackRow R = recs[w];
    unsigned char* chunk = blob + R.chunk_off;
    StreamRow* rec = reinterpret_cast<StreamRow*>(chunk + sizeof(StreamHead)) + R.slot;
    double* val = reinterpret_cast<double*>(chunk + sizeof(StreamHead) + R.rows * sizeof(StreamRow));
    int* col = reinterpret_cast<int*>(val + R.ents);
    const int64_t* ci = R.backward ? Lr : Rc;
    const double* cv = R.backward ? Lv : Rv;
    for (int e = lane; e < R.count; e += 32) {
        val[R.start + e] = cv[R.src + e];
        col[R.start + e] = (int)ci[R.src + e];
    }
    if (lane == 0) {
        StreamRow rw;
        rw.row = R.row;
        rw.start = R.start;
        rw.count = R.count;
        rw.pad = 0;
        rw.diag = Lv[Lp[R.row]];
        rw.pad2 = 0.0;
        *rec = rw;
    }
}

__global__ void k_stream_pack_heads(int nchunks, const StreamPackChunk* __restrict__ ch,
                                    unsigned char* blob) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const StreamPackChunk C = ch[c];
    StreamHead h;
    h.next_off = c + kStreamStages < nchunks ? ch[c + kStreamStages].off : 0;
    h.next_bytes = c + kStreamStages < nchunks ? ch[c + kStreamStages].bytes : 0;
    h.rows = C.rows;
    h.ents = C.ents;
    h.pad[0] = h.pad[1] = h.pad[2] = 0;
    *reinterpret_cast<StreamHead*>(blob + C.off) = h;
    double* val = reinterpret_cast<double*>(blob + C.off + sizeof(StreamHead) + C.rows * sizeof(StreamRow));
    int* col = reinterpret_cast<int*>(val + C.ents);
    for (int e = C.used; e < C.ents; ++e) {
        val[e] = 0.0;
        col[e] = 0;
    }
}

void ichol_launch_stream_pack(int nrec, const StreamPackRow* recs, int nchunks,
                              const StreamPackChunk* chunks, const int64_t* Rc, const double* Rv,
                              const int64_t* Lr, const double* Lv, const int64_t* Lp,
                              unsigned char* blob, cudaStream_t s) {
    if (nrec > 0)
        k_stream_pack_rows<<<(unsigned)((nrec * 32 + 255) / 256), 256, 0, s>>>(nrec, recs, Rc, Rv, Lr,
                                                                               Lv, Lp, blob);
    if (nchunks > 0)
        k_stream_pack_heads<<<(unsigned)((nchunks + 127) / 128), 128, 0, s>>>(nchunks, chunks, blob);
}

void ichol_launch_solve_stream(int64_t n, int total, const StreamFirst& first,
                               const unsigned char* blob, const double* b, double* x,
                               const InstState* st, uint32_t limit, cudaStream_t s) {
    k_ichol_solve_stream<<<1, kStreamThreads, ichol_stream_smem(n), s>>>(n, total, first, blob, b, x,
                                                                         st, limit);
}

// The forward sweep above overwrites x in place: y lives in x. For the
// forward pass to read y_j of earlier levels and b_i of its own row, b and
// x may alias (the reference also works in place on a copy of b).

void ichol_launch_init(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                       double shift, double* d, double* rsum, int* level, unsigned long long* band,
                       cudaStream_t s) {
    if (n > 0) k_ichol_init<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Ap, Ar, Av, shift, d, rsum, level, band);
}

int ichol_launch_factor(int64_t n, int64_t W, const int64_t* Ap, const int64_t* Ar,
                        const double* Av, double* d, const double* rsum, int* level, double* F,
                        uint8_t* pat, int* cand, double* keptv, int64_t* kepti, int64_t* Lp,
                        int64_t* Lr, double* Lv, int64_t cap, double discard, int64_t max_nnz,
                        double rel, int diag_keep, int64_t* result, cudaStream_t s) {
    // Front on chip when a cluster of at most 8 CTAs holds it and such a
    // cluster can be resident; otherwise the front lives in global memory.
    const int C = ichol_cluster_size(W);
    if (C > 0) {
        const ClLayout L = cl_layout(W, C);
        const int chunks = (int)((W - 1 + 31) / 32);
        auto kern = chunks <= 2 ? k_ichol_factor_cluster<2>
                  : chunks <= 4 ? k_ichol_factor_cluster<4>
                  : chunks <= 8 ? k_ichol_factor_cluster<8> : k_ichol_factor_cluster<kClMaxChunks>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)C);
        cfg.blockDim = dim3(kClThreads);
        cfg.dynamicSmemBytes = L.bytes;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) == cudaSuccess && clusters >= 1) {
            if (cudaLaunchKernelEx(&cfg, kern, n, (int)W, C, Ap, Ar, Av, (const double*)d, rsum,
                                   level, Lp, Lr, Lv, cap, discard, max_nnz, rel, diag_keep,
                                   result) == cudaSuccess)
                return C;
        }
        cudaGetLastError();
    }
    k_ichol_factor<<<1, kIcholThreads, 0, s>>>(n, W, Ap, Ar, Av, d, rsum, level, F, pat, cand, keptv,
                                               kepti, Lp, Lr, Lv, cap, discard, max_nnz, rel,
                                               diag_keep, result);
    return 0;
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
        k_row_sort_warp<<<(unsigned)((n * 32 + 255) / 256), 256, 0, s>>>(n, Rp, Rc, Rv);
        k_row_sort<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Rp, Rc, Rv);
    }
}

// Raise the shared-memory limit of the shared-memory solve; called when a
// factor is built, before any solve can be captured.
void ichol_prepare() {
    cudaFuncSetAttribute(k_ichol_solve_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kIcholSmemRows * sizeof(double)));
    cudaFuncSetAttribute(k_ichol_solve_stream, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)ichol_stream_smem(kStreamMaxRows));
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
