// Window Laplacians assembled on the device as canonical CSR:
// uniform_laplacian (pymatting/laplacian/uniform_laplacian.py) and
// rw_laplacian (pymatting/laplacian/rw_laplacian.py), both passed through
// weights_to_laplacian (pymatting/util/util.py:840-875).
//
// W has one entry per pixel and window offset, with the neighbour clamped
// to the image, so border rows repeat columns. Those repeats carry equal
// values and are summed. Row i of the result is L_i = d_i e_i - W'_i with
// W' = diag(1 / rowsum(W)) W and d_i = regularization + rowsum(W'_i). Each
// row is one thread; its sums follow the reference's operation order:
// rowsum(W) in ascending column order, and rowsum(W') in descending column
// order (the order scipy's sparse product leaves the row in).

#include <cuda_runtime.h>

#include "pm_common.cuh"
#include <math.h>
#include <stdint.h>

namespace pmb {
namespace wl {

enum : int { kUniform = 0, kRandomWalk = 1 };

struct Args {
    const double* image;  // (h, w, 3); unused for kUniform
    int h, w, r;
    double reg;
    const int64_t* px;  // prefix over x of the per-column window width (w + 1)
    const int64_t* py;  // prefix over y of the per-row window height (h + 1)
    int64_t* rowptr;
    int64_t* cols;
    double* vals;
};

// Value of W_ij: `count` equal weights summed one after another.
template <int MODE>
__device__ __forceinline__ double weight(const Args& A, int i, int j, int count) {
    double wv = 1.0;
    if (MODE == kRandomWalk) {
        const double* zi = A.image + (long long)i * 3;
        const double* zj = A.image + (long long)j * 3;
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double d = __dsub_rn(zi[c], zj[c]);
            s = __dadd_rn(s, __dmul_rn(d, d));
        }
        const double nrm = sqrt(s);
        wv = exp(__dmul_rn(-900.0, __dmul_rn(nrm, nrm)));
    }
    double v = wv;
    for (int k = 1; k < count; ++k) v = __dadd_rn(v, wv);
    return v;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_window_laplacian(Args A) {
    const long long n = (long long)A.h * A.w;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int y = (int)(i / A.w), x = (int)(i % A.w);
    const int x0 = max(x - A.r, 0), x1 = min(x + A.r, A.w - 1);
    const int y0 = max(y - A.r, 0), y1 = min(y + A.r, A.h - 1);
    // number of window offsets that clamp onto column x2 / row y2
    auto cnt_x = [&](int x2) {
        int c = 1;
        if (x2 == 0) c += max(A.r - x, 0);
        if (x2 == A.w - 1) c += max(x + A.r - (A.w - 1), 0);
        return c;
    };
    auto cnt_y = [&](int y2) {
        int c = 1;
        if (y2 == 0) c += max(A.r - y, 0);
        if (y2 == A.h - 1) c += max(y + A.r - (A.h - 1), 0);
        return c;
    };
    const int nx = x1 - x0 + 1;
    const long long base = A.py[y] * A.px[A.w] + (long long)(y1 - y0 + 1) * A.px[x];
    if (i == n - 1) A.rowptr[n] = A.py[A.h] * A.px[A.w];
    A.rowptr[i] = base;
    // rowsum(W), ascending columns
    double s1 = 0.0;
    for (int y2 = y0; y2 <= y1; ++y2)
        for (int x2 = x0; x2 <= x1; ++x2) {
            const int j = x2 + y2 * A.w;
            s1 = __dadd_rn(s1, weight<MODE>(A, (int)i, j, cnt_x(x2) * cnt_y(y2)));
        }
    const double f = __ddiv_rn(1.0, s1);
    // rowsum(W'), descending columns
    double s2 = 0.0;
    for (int y2 = y1; y2 >= y0; --y2)
        for (int x2 = x1; x2 >= x0; --x2) {
            const int j = x2 + y2 * A.w;
            s2 = __dadd_rn(s2, __dmul_rn(f, weight<MODE>(A, (int)i, j, cnt_x(x2) * cnt_y(y2))));
        }
    const double d = __dadd_rn(A.reg, s2);
    long long o = base;
    for (int y2 = y0; y2 <= y1; ++y2)
        for (int x2 = x0; x2 <= x1; ++x2, ++o) {
            const int j = x2 + y2 * A.w;
            const double wp = __dmul_rn(f, weight<MODE>(A, (int)i, j, cnt_x(x2) * cnt_y(y2)));
            A.cols[o] = j;
            A.vals[o] = (j == i) ? __dsub_rn(d, wp) : -wp;
        }
    (void)nx;
}

}  // namespace wl
}  // namespace pmb

using namespace pmb::wl;

// mode 0: uniform, 1: random walk. px (w + 1), py (h + 1) int64 prefixes of
// the clamped window extents; rowptr (n + 1), cols / vals (py[h] * px[w]).
int pmb_launch_window_laplacian(int mode, const double* image, int h, int w, int r, double reg,
                                const int64_t* px, const int64_t* py, int64_t* rowptr,
                                int64_t* cols, double* vals, cudaStream_t st) {
    if (h <= 0 || w <= 0 || r < 0 || !px || !py || !rowptr || !cols || !vals) return -2;
    if ((long long)h * w >= (1LL << 31)) return -2;  // pixel indices are 32-bit in the kernel
    if (mode == kRandomWalk && !image) return -2;
    Args A{image, h, w, r, reg, px, py, rowptr, cols, vals};
    const long long n = (long long)h * w;
    const int blocks = (int)((n + 255) / 256);
    if (mode == kUniform) k_window_laplacian<kUniform><<<blocks, 256, 0, st>>>(A);
    else if (mode == kRandomWalk) k_window_laplacian<kRandomWalk><<<blocks, 256, 0, st>>>(A);
    else return -2;
    return pmb::launch_status() ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Learning-based digital matting Laplacian (lbdm_laplacian,
// pymatting/laplacian/lbdm_laplacian.py). Each interior window c of
// (2r+1)^2 pixels gives T_c = (I - F)(I - F)^T with
// F = (K + eps I)^-1 K, K = X X^T, X = [colours, 1] of the window's pixels.
// L_pq sums T_c[a(p), b(q)] over the windows holding both pixels. Pass 1
// stores T_c per window (one thread per window: Gaussian elimination with
// partial pivoting in local memory); pass 2 gathers every row in ascending
// column order, windows in raster order (deterministic).
// ---------------------------------------------------------------------------

namespace pmb {
namespace lbdm {

template <int R>
__global__ void __launch_bounds__(128) k_lbdm_windows(const double* __restrict__ image, int h,
                                                      int w, double eps, double* __restrict__ T) {
    constexpr int S = 2 * R + 1, N = S * S;
    const int ww = w - 2 * R;
    const long long nwin = (long long)(h - 2 * R) * ww;
    const long long wi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (wi >= nwin) return;
    const int cy = (int)(wi / ww) + R, cx = (int)(wi % ww) + R;
    double X[N][4];
    for (int k = 0; k < N; ++k) {
        const int y2 = cy - R + k / S, x2 = cx - R + k % S;
        const double* z = image + ((long long)y2 * w + x2) * 3;
        X[k][0] = z[0];
        X[k][1] = z[1];
        X[k][2] = z[2];
        X[k][3] = 1.0;
    }
    double A[N][N], B[N][N];
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b) {
            double s = 0.0;
            for (int c = 0; c < 4; ++c) s = __dadd_rn(s, __dmul_rn(X[a][c], X[b][c]));
            B[a][b] = s;
            A[a][b] = (a == b) ? __dadd_rn(s, eps) : s;
        }
    // A F = B by elimination with partial pivoting (first maximum wins)
    for (int k = 0; k < N; ++k) {
        int p = k;
        double best = fabs(A[k][k]);
        for (int i = k + 1; i < N; ++i)
            if (fabs(A[i][k]) > best) {
                best = fabs(A[i][k]);
                p = i;
            }
        if (p != k) {
            for (int j = 0; j < N; ++j) {
                double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t;
                t = B[k][j]; B[k][j] = B[p][j]; B[p][j] = t;
            }
        }
        const double inv = __ddiv_rn(1.0, A[k][k]);
        for (int i = k + 1; i < N; ++i) {
            const double l = __dmul_rn(A[i][k], inv);
            for (int j = k + 1; j < N; ++j) A[i][j] = __dsub_rn(A[i][j], __dmul_rn(l, A[k][j]));
            for (int j = 0; j < N; ++j) B[i][j] = __dsub_rn(B[i][j], __dmul_rn(l, B[k][j]));
        }
    }
    for (int i = N - 1; i >= 0; --i)
        for (int j = 0; j < N; ++j) {
            double s = B[i][j];
            for (int k = i + 1; k < N; ++k) s = __dsub_rn(s, __dmul_rn(A[i][k], B[k][j]));
            B[i][j] = __ddiv_rn(s, A[i][i]);  // B now holds F
        }
    // T = (I - F)(I - F)^T, reusing A for I - F
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b) A[a][b] = (a == b) ? __dsub_rn(1.0, B[a][b]) : -B[a][b];
    double* out = T + wi * (N * N);
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b) {
            double s = 0.0;
            for (int k = 0; k < N; ++k) s = __dadd_rn(s, __dmul_rn(A[a][k], A[b][k]));
            out[a * N + b] = s;
        }
}

// Window centres holding pixel coordinate v: [max(R, v - R), min(n - 1 - R, v + R)].
template <int R>
__global__ void __launch_bounds__(256) k_lbdm_rows(int h, int w, const double* __restrict__ T,
                                                   const int64_t* __restrict__ px,
                                                   const int64_t* __restrict__ py,
                                                   int64_t* __restrict__ rowptr,
                                                   int64_t* __restrict__ cols,
                                                   double* __restrict__ vals) {
    constexpr int S = 2 * R + 1, N = S * S;
    const long long n = (long long)h * w;
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int y = (int)(p / w), x = (int)(p % w);
    const int cy0 = max(R, y - R), cy1 = min(h - 1 - R, y + R);
    const int cx0 = max(R, x - R), cx1 = min(w - 1 - R, x + R);
    const int ny = cy1 - cy0 + 2 * R + 1;
    const long long base = py[y] * px[w] + (long long)ny * px[x];
    rowptr[p] = base;
    if (p == n - 1) rowptr[n] = py[h] * px[w];
    const int ww = w - 2 * R;
    long long o = base;
    for (int qy = cy0 - R; qy <= cy1 + R; ++qy)
        for (int qx = cx0 - R; qx <= cx1 + R; ++qx, ++o) {
            double s = 0.0;
            const int dy0 = max(cy0, qy - R), dy1 = min(cy1, qy + R);
            const int dx0 = max(cx0, qx - R), dx1 = min(cx1, qx + R);
            for (int cy = dy0; cy <= dy1; ++cy)
                for (int cx = dx0; cx <= dx1; ++cx) {
                    const long long wi = (long long)(cy - R) * ww + (cx - R);
                    const int a = (y - cy + R) * S + (x - cx + R);
                    const int b = (qy - cy + R) * S + (qx - cx + R);
                    s = __dadd_rn(s, T[wi * (N * N) + a * N + b]);
                }
            cols[o] = (long long)qy * w + qx;
            vals[o] = s;
        }
}

}  // namespace lbdm
}  // namespace pmb

// radius 1 or 2; h, w > 2 radius. T: (h - 2r)(w - 2r) (2r+1)^4 doubles of
// scratch. px / py: prefix sums of the per-column / per-row count of pixels
// sharing a window with the pixel (w + 1, h + 1 int64).
int pmb_launch_lbdm_laplacian(const double* image, int h, int w, int r, double eps, double* T,
                              const int64_t* px, const int64_t* py, int64_t* rowptr,
                              int64_t* cols, double* vals, cudaStream_t st) {
    if (!image || !T || !px || !py || !rowptr || !cols || !vals || (r != 1 && r != 2) ||
        h <= 2 * r || w <= 2 * r)
        return -2;
    const long long nwin = (long long)(h - 2 * r) * (w - 2 * r);
    const long long n = (long long)h * w;
    const int wb = (int)((nwin + 127) / 128), rb = (int)((n + 255) / 256);
    if (r == 1) {
        pmb::lbdm::k_lbdm_windows<1><<<wb, 128, 0, st>>>(image, h, w, eps, T);
        pmb::lbdm::k_lbdm_rows<1><<<rb, 256, 0, st>>>(h, w, T, px, py, rowptr, cols, vals);
    } else {
        pmb::lbdm::k_lbdm_windows<2><<<wb, 128, 0, st>>>(image, h, w, eps, T);
        pmb::lbdm::k_lbdm_rows<2><<<rb, 256, 0, st>>>(h, w, T, px, py, rowptr, cols, vals);
    }
    return pmb::launch_status() ? 1 : 0;
}

// ---------------------------------------------------------------------------
// System of estimate_foreground_cf (pymatting/foreground/estimate_foreground_cf.py)
// for the default neighbours (-1,0), (1,0), (0,-1), (0,1):
// A = U^T U + diag(S, S), U = [diag(a), diag(1 - a)],
// S = sum_d D_d^T diag(reg + |D_d a|) D_d. For unit offsets every pair of
// 4-neighbours p, q enters S twice (once from each direction) with weight
// reg + |a_p - a_q|. Row p (foreground unknowns) holds its neighbours, p and
// n + p; row n + p (background) holds p, then n + its neighbours and n + p.
// ---------------------------------------------------------------------------

namespace pmb {
namespace fgcf {

__device__ __forceinline__ int nbr_count(int y, int x, int h, int w) {
    return (x > 0) + (x < w - 1) + (y > 0) + (y < h - 1);
}

// The coupling entry a (1 - a) of rows p and n + p exists only when it is
// non-zero: the reference builds U from diags(a) and diags(1 - a), whose
// zero entries scipy drops.
__device__ __forceinline__ bool has_coupling(double ap) { return ap != 0.0 && ap != 1.0; }

// rowptr[r] before the scan: entries of row r (r < n: F rows, r >= n: B rows).
__global__ void k_fgcf_count(const double* __restrict__ a, int h, int w, int64_t* rowcnt) {
    const long long n = (long long)h * w;
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= 2 * n) return;
    const long long p = r < n ? r : r - n;
    const int y = (int)(p / w), x = (int)(p % w);
    rowcnt[r] = nbr_count(y, x, h, w) + 1 + (has_coupling(a[p]) ? 1 : 0);
}

__global__ void k_fgcf_fill(const double* __restrict__ a, int h, int w, double reg,
                            const int64_t* __restrict__ rowptr, int64_t* __restrict__ cols,
                            double* __restrict__ vals) {
    const long long n = (long long)h * w;
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= 2 * n) return;
    const bool brow = r >= n;
    const long long p = brow ? r - n : r;
    const int y = (int)(p / w), x = (int)(p % w);
    const double ap = a[p];
    // neighbours in ascending index order: up, left, right, down
    long long q[4];
    double wq[4];
    int m = 0;
    if (y > 0) { q[m] = p - w; ++m; }
    if (x > 0) { q[m] = p - 1; ++m; }
    if (x < w - 1) { q[m] = p + 1; ++m; }
    if (y < h - 1) { q[m] = p + w; ++m; }
    double spp = 0.0;
    for (int t = 0; t < m; ++t) {
        const double wt = __dadd_rn(reg, fabs(__dsub_rn(ap, a[q[t]])));
        wq[t] = __dadd_rn(wt, wt);  // both directions of the pair
        spp = __dadd_rn(spp, wq[t]);
    }
    const double a1 = __dsub_rn(1.0, ap);
    long long o = rowptr[r];
    if (!brow) {
        int t = 0;
        for (; t < m && q[t] < p; ++t, ++o) { cols[o] = q[t]; vals[o] = -wq[t]; }
        cols[o] = p; vals[o] = __dadd_rn(__dmul_rn(ap, ap), spp); ++o;
        for (; t < m; ++t, ++o) { cols[o] = q[t]; vals[o] = -wq[t]; }
        if (has_coupling(ap)) { cols[o] = n + p; vals[o] = __dmul_rn(ap, a1); }
    } else {
        if (has_coupling(ap)) { cols[o] = p; vals[o] = __dmul_rn(ap, a1); ++o; }
        int t = 0;
        for (; t < m && q[t] < p; ++t, ++o) { cols[o] = n + q[t]; vals[o] = -wq[t]; }
        cols[o] = n + p; vals[o] = __dadd_rn(__dmul_rn(a1, a1), spp); ++o;
        for (; t < m; ++t, ++o) { cols[o] = n + q[t]; vals[o] = -wq[t]; }
    }
}

}  // namespace fgcf
}  // namespace pmb

int pmb_scan_exclusive(int64_t* v, int64_t n, int64_t* chunk_scratch, int64_t* total,
                       cudaStream_t s);

// rowptr: 2 h w + 1; cols / vals: rowptr[2 h w] entries (written by the
// first call); scratch: (2 h w + 1023) / 1024 + 2.
int pmb_launch_fg_cf_system(const double* alpha, int h, int w, double reg, int64_t* rowptr,
                            int64_t* cols, double* vals, int64_t* scratch, cudaStream_t st) {
    if (!alpha || !rowptr || h <= 0 || w <= 0) return -2;
    const long long n2 = 2LL * h * w;
    const int blocks = (int)((n2 + 255) / 256);
    if (!cols || !vals) {
        pmb::fgcf::k_fgcf_count<<<blocks, 256, 0, st>>>(alpha, h, w, rowptr);
        if (pmb_scan_exclusive(rowptr, n2, scratch, rowptr + n2, st)) return 1;
        return pmb::launch_status() ? 1 : 0;
    }
    pmb::fgcf::k_fgcf_fill<<<blocks, 256, 0, st>>>(alpha, h, w, reg, rowptr, cols, vals);
    return pmb::launch_status() ? 1 : 0;
}
