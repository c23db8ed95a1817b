// Large-kernel matting Laplacian (He et al. 2010), matrix-free.
//
// Restates pymatting/laplacian/lkm_laplacian.py:6-76 on the device: every
// quantity is a box filter over (2r+1)^2 windows of the image or of products
// with the operand, so the operator is never formed.
//   setup    means, covariances -> per valid window V = (cov + eps/|w| I)^-1
//            / |w| (3x3 symmetric), Vm = V mean, mVm = 1/|w| + mean' Vm
//   apply    sums of p and p*I over windows (valid box), per window
//            t3 = p_sum Vm - V pI_sum, t1 = p_sum mVm - pI_sum . Vm, back to
//            pixels (full box), L p = c p + I . B(t3) - B(t1), c = number of
//            windows covering the pixel
//   diagonal B(1 - mVm) + I . (2 B(Vm) - B(V) I)
// Box filters are separable: a row pass then a column pass, each a running
// sum over segments of kSeg outputs per thread (the reference runs one sum
// along each whole row; the sums differ only in rounding order). Layouts are
// row-major with interleaved channels, as the reference's numpy arrays.
// "valid" maps n inputs to n - 2r outputs (window inside), "full" maps n
// inputs to n + 2r outputs (zeros outside), boxfilter.py:6-82.

#include <stdint.h>

#include <cuda_runtime.h>

#include "pm_common.cuh"

namespace pmb {

constexpr int kSeg = 64;         // outputs per thread of a box pass
constexpr int kBoxThreads = 256;

// Sliding sum along one axis. Input lines of n_in samples, K channels
// interleaved; `stride` = distance (elements) between consecutive samples of
// a line; lines are `nlines` apart by `line_in` / `line_out` elements and the
// channel index varies fastest inside a sample. out[o] = sum_{i=o+lo}^{o+lo+2r}
// in[i] with lo = 0 (valid) or -2r (full), zero outside the line.
template <int K>
__global__ void __launch_bounds__(kBoxThreads)
k_box_pass(const double* __restrict__ src, double* __restrict__ dst, int nlines, int n_in,
           int n_out, int64_t line_in, int64_t line_out, int64_t stride_in, int64_t stride_out,
           int r, int lo) {
    const int segs = (n_out + kSeg - 1) / kSeg;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)nlines * segs * K;
    if (idx >= total) return;
    // Channel fastest, then line, then segment: adjacent threads of a column
    // pass read adjacent columns.
    const int k = (int)(idx % K);
    const int64_t rest = idx / K;
    const int line = (int)(rest % nlines);
    const int seg = (int)(rest / nlines);
    const double* in = src + line * line_in + k;
    double* out = dst + line * line_out + k;
    const int o0 = seg * kSeg, o1 = min(o0 + kSeg, n_out);
    double s = 0.0;
    const int a0 = o0 + lo;
    for (int i = max(a0, 0); i <= min(a0 + 2 * r, n_in - 1); ++i) s += in[i * stride_in];
    out[o0 * stride_out] = s;
    for (int o = o0 + 1; o < o1; ++o) {
        const int drop = o - 1 + lo, add = o + lo + 2 * r;
        if (drop >= 0 && drop < n_in) s -= in[drop * stride_in];
        if (add >= 0 && add < n_in) s += in[add * stride_in];
        out[o * stride_out] = s;
    }
}

template <int K>
static int box_pass(const double* src, double* dst, int nlines, int n_in, int n_out,
                    int64_t line_in, int64_t line_out, int64_t stride_in, int64_t stride_out,
                    int r, int lo, cudaStream_t s) {
    const int segs = (n_out + kSeg - 1) / kSeg;
    const int64_t total = (int64_t)nlines * segs * K;
    if (total <= 0) return 0;
    k_box_pass<K><<<(unsigned)((total + kBoxThreads - 1) / kBoxThreads), kBoxThreads, 0, s>>>(
        src, dst, nlines, n_in, n_out, line_in, line_out, stride_in, stride_out, r, lo);
    return pmb::launch_status();
}

// 2-D box filter of an (h, w, K) array: rows then columns.
//   valid: (h, w) -> (h - 2r, w - 2r); full: (h, w) -> (h + 2r, w + 2r).
// tmp holds the row pass: h x w_out x K.
template <int K>
static int box2d(const double* src, double* tmp, double* dst, int h, int w, int r, bool full,
                 cudaStream_t s) {
    const int lo = full ? -2 * r : 0;
    const int wo = full ? w + 2 * r : w - 2 * r;
    const int ho = full ? h + 2 * r : h - 2 * r;
    if (int rc = box_pass<K>(src, tmp, h, w, wo, (int64_t)w * K, (int64_t)wo * K, K, K, r, lo, s))
        return rc;
    // Column pass: one line per output column, samples one row apart.
    return box_pass<K>(tmp, dst, wo, h, ho, K, K, (int64_t)wo * K, (int64_t)wo * K, r, lo, s);
}

// q = [p, p I0, p I1, p I2] per pixel.
__global__ void k_lkm_rhs(const double* __restrict__ image, const double* __restrict__ p, int64_t n,
                          double* q) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = p[i];
    q[i * 4 + 0] = v;
    q[i * 4 + 1] = v * image[i * 3 + 0];
    q[i * 4 + 2] = v * image[i * 3 + 1];
    q[i * 4 + 3] = v * image[i * 3 + 2];
}

// Per valid window: V (6: 00 01 02 11 12 22), Vm (3), mVm (1) from the box
// sums of I (3) and of I I' (6). Inverse by the adjugate.
__global__ void k_lkm_windows(const double* __restrict__ s1, const double* __restrict__ s2,
                              int64_t nw, double area, double eps, double* win) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nw) return;
    const double m0 = s1[i * 3 + 0] / area, m1 = s1[i * 3 + 1] / area, m2 = s1[i * 3 + 2] / area;
    const double e = eps / area;
    const double c00 = s2[i * 6 + 0] / area - m0 * m0 + e;
    const double c01 = s2[i * 6 + 1] / area - m0 * m1;
    const double c02 = s2[i * 6 + 2] / area - m0 * m2;
    const double c11 = s2[i * 6 + 3] / area - m1 * m1 + e;
    const double c12 = s2[i * 6 + 4] / area - m1 * m2;
    const double c22 = s2[i * 6 + 5] / area - m2 * m2 + e;
    const double a00 = c11 * c22 - c12 * c12;
    const double a01 = c02 * c12 - c01 * c22;
    const double a02 = c01 * c12 - c02 * c11;
    const double a11 = c00 * c22 - c02 * c02;
    const double a12 = c01 * c02 - c00 * c12;
    const double a22 = c00 * c11 - c01 * c01;
    const double det = c00 * a00 + c01 * a01 + c02 * a02;
    const double f = 1.0 / (det * area);
    const double v00 = a00 * f, v01 = a01 * f, v02 = a02 * f;
    const double v11 = a11 * f, v12 = a12 * f, v22 = a22 * f;
    const double vm0 = v00 * m0 + v01 * m1 + v02 * m2;
    const double vm1 = v01 * m0 + v11 * m1 + v12 * m2;
    const double vm2 = v02 * m0 + v12 * m1 + v22 * m2;
    double* o = win + i * 10;
    o[0] = v00; o[1] = v01; o[2] = v02; o[3] = v11; o[4] = v12; o[5] = v22;
    o[6] = vm0; o[7] = vm1; o[8] = vm2;
    o[9] = 1.0 / area + (m0 * vm0 + m1 * vm1 + m2 * vm2);
}

// Image products I I' (6 channels) for the covariance sums.
__global__ void k_lkm_outer(const double* __restrict__ image, int64_t n, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = image[i * 3 + 0], b = image[i * 3 + 1], c = image[i * 3 + 2];
    double* o = out + i * 6;
    o[0] = a * a; o[1] = a * b; o[2] = a * c; o[3] = b * b; o[4] = b * c; o[5] = c * c;
}

// Per window: t = [t3 (3), t1] from the window sums [p_sum, pI_sum (3)].
__global__ void k_lkm_window_apply(const double* __restrict__ sums, const double* __restrict__ win,
                                   int64_t nw, double* t) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nw) return;
    const double* o = win + i * 10;
    const double ps = sums[i * 4 + 0], q0 = sums[i * 4 + 1], q1 = sums[i * 4 + 2],
                 q2 = sums[i * 4 + 3];
    t[i * 4 + 0] = ps * o[6] - (o[0] * q0 + o[1] * q1 + o[2] * q2);
    t[i * 4 + 1] = ps * o[7] - (o[1] * q0 + o[3] * q1 + o[4] * q2);
    t[i * 4 + 2] = ps * o[8] - (o[2] * q0 + o[4] * q1 + o[5] * q2);
    t[i * 4 + 3] = ps * o[9] - (q0 * o[6] + q1 * o[7] + q2 * o[8]);
}

// Number of valid windows covering pixel (y, x): product of the per-axis
// counts of window origins in [max(0, x - 2r), min(x, nv - 1)].
__device__ __forceinline__ double lkm_count(int y, int x, int hv, int wv, int r) {
    const int cy = min(y, hv - 1) - max(0, y - 2 * r) + 1;
    const int cx = min(x, wv - 1) - max(0, x - 2 * r) + 1;
    return (double)(max(cy, 0) * max(cx, 0));
}

// out = c p + I . B3 - B1, B = full box of t (4 channels: B3, B1).
__global__ void k_lkm_finish(const double* __restrict__ image, const double* __restrict__ p,
                             const double* __restrict__ B, const double* __restrict__ add, int h,
                             int w, int r, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w) return;
    const int y = (int)(i / w), x = (int)(i % w);
    const double c = lkm_count(y, x, h - 2 * r, w - 2 * r, r);
    double v = c * p[i];
    v += image[i * 3 + 0] * B[i * 4 + 0] + image[i * 3 + 1] * B[i * 4 + 1] +
         image[i * 3 + 2] * B[i * 4 + 2];
    v -= B[i * 4 + 3];
    if (add) v += add[i] * p[i];
    out[i] = v;
}

// Diagonal from the full box of [1 - mVm, Vm (3), V (6)].
__global__ void k_lkm_diag_src(const double* __restrict__ win, int64_t nw, double* d10) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nw) return;
    const double* o = win + i * 10;
    double* d = d10 + i * 10;
    d[0] = 1.0 - o[9];
    d[1] = o[6]; d[2] = o[7]; d[3] = o[8];
    for (int k = 0; k < 6; ++k) d[4 + k] = o[k];
}

__global__ void k_lkm_diag(const double* __restrict__ image, const double* __restrict__ B, int64_t n,
                           const double* __restrict__ add, double* diag, double* inv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* b = B + i * 10;
    const double I0 = image[i * 3 + 0], I1 = image[i * 3 + 1], I2 = image[i * 3 + 2];
    // B(V) I with B(V) symmetric (00 01 02 11 12 22 at b[4..9]).
    const double VI0 = b[4] * I0 + b[5] * I1 + b[6] * I2;
    const double VI1 = b[5] * I0 + b[7] * I1 + b[8] * I2;
    const double VI2 = b[6] * I0 + b[8] * I1 + b[9] * I2;
    double dv = b[0] + I0 * (2.0 * b[1] - VI0) + I1 * (2.0 * b[2] - VI1) + I2 * (2.0 * b[3] - VI2);
    if (add) dv += add[i];
    diag[i] = dv;
    if (inv) inv[i] = 1.0 / dv;
}

static unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace pmb

using namespace pmb;

// Scratch (doubles) of the setup / apply / diagonal for an h x w image.
int64_t pmb_launch_lkm_scratch(int h, int w, int r) {
    const int64_t hv = h - 2 * r, wv = w - 2 * r;
    const int64_t big = (int64_t)h * w * 10 + (int64_t)h * (w + 2 * r) * 10;
    return big + hv * wv * 10 + 64;
}

int pmb_launch_lkm_setup(const double* image, int h, int w, int r, double eps, double* win,
                         double* scratch, cudaStream_t s) {
    const int hv = h - 2 * r, wv = w - 2 * r;
    const int64_t n = (int64_t)h * w, nw = (int64_t)hv * wv;
    double* outer = scratch;                       // n * 6
    double* tmp = outer + n * 6;                   // h * wv * 6
    double* s1 = tmp + (int64_t)h * wv * 6;        // nw * 3
    double* s2 = s1 + nw * 3;                      // nw * 6
    if (int rc = box2d<3>(image, tmp, s1, h, w, r, false, s)) return rc;
    k_lkm_outer<<<blocks(n), 256, 0, s>>>(image, n, outer);
    if (int rc = box2d<6>(outer, tmp, s2, h, w, r, false, s)) return rc;
    k_lkm_windows<<<blocks(nw), 256, 0, s>>>(s1, s2, nw, (double)((2 * r + 1) * (2 * r + 1)), eps,
                                              win);
    return pmb::launch_status();
}

int pmb_launch_lkm_apply(const double* image, int h, int w, int r, const double* win,
                         const double* add, const double* p, double* out, double* scratch,
                         cudaStream_t s) {
    const int hv = h - 2 * r, wv = w - 2 * r;
    const int64_t n = (int64_t)h * w, nw = (int64_t)hv * wv;
    double* q = scratch;                           // n * 4
    double* tmp = q + n * 4;                       // max(h * wv, hv * w) * 4
    double* sums = tmp + (int64_t)h * w * 4;       // nw * 4
    double* t = sums + nw * 4;                     // nw * 4
    double* B = t + nw * 4;                        // n * 4
    k_lkm_rhs<<<blocks(n), 256, 0, s>>>(image, p, n, q);
    if (int rc = box2d<4>(q, tmp, sums, h, w, r, false, s)) return rc;
    k_lkm_window_apply<<<blocks(nw), 256, 0, s>>>(sums, win, nw, t);
    if (int rc = box2d<4>(t, tmp, B, hv, wv, r, true, s)) return rc;
    k_lkm_finish<<<blocks(n), 256, 0, s>>>(image, p, B, add, h, w, r, out);
    return pmb::launch_status();
}

int pmb_launch_lkm_diag(const double* image, int h, int w, int r, const double* win,
                        const double* add, double* diag, double* inv, double* scratch,
                        cudaStream_t s) {
    const int hv = h - 2 * r, wv = w - 2 * r;
    const int64_t n = (int64_t)h * w, nw = (int64_t)hv * wv;
    double* d10 = scratch;                         // nw * 10
    double* tmp = d10 + nw * 10;                   // hv * w * 10
    double* B = tmp + (int64_t)hv * w * 10;        // n * 10
    k_lkm_diag_src<<<blocks(nw), 256, 0, s>>>(win, nw, d10);
    if (int rc = box2d<10>(d10, tmp, B, hv, wv, r, true, s)) return rc;
    k_lkm_diag<<<blocks(n), 256, 0, s>>>(image, B, n, add, diag, inv);
    return pmb::launch_status();
}
