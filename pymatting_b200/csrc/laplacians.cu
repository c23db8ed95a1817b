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
    if (mode == kRandomWalk && !image) return -2;
    Args A{image, h, w, r, reg, px, py, rowptr, cols, vals};
    const long long n = (long long)h * w;
    const int blocks = (int)((n + 255) / 256);
    if (mode == kUniform) k_window_laplacian<kUniform><<<blocks, 256, 0, st>>>(A);
    else if (mode == kRandomWalk) k_window_laplacian<kRandomWalk><<<blocks, 256, 0, st>>>(A);
    else return -2;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
