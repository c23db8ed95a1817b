// Jacobi foreground / background estimation: the algorithm of PyMatting's
// GPU backend estimate_foreground_ml_cupy
// (pymatting/foreground/estimate_foreground_ml_cupy.py:5-230), on sm_100a.
//
// The reference runs one NVRTC kernel launch per Jacobi iteration and a
// separate resize launch per buffer and level. Here one kernel resizes all
// four buffers of a level, large levels run one kernel per iteration, and
// levels of at most kSmallPixels pixels run all their iterations inside a
// single CTA with a barrier between iterations. The buffer handling is the
// reference's: flat buffers F, F_prev, B, B_prev swapped after every
// iteration, F and B seeded with the colour of pixel (0, 0), each level
// resized from the buffer named F, and F returned. This file is compiled
// with fused multiply-adds allowed, as NVRTC compiles the reference's
// kernel by default; the per-pixel expressions keep the reference's order.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

namespace pmb {
namespace fgj {

constexpr int kSmallThreads = 1024;
constexpr int kSmallPixels = 8192;  // levels this small run in one CTA
constexpr int kMaxLevels = 40;

// One Jacobi update of pixel (x, y): estimate_foreground_ml_cupy.py:34-107.
__device__ __forceinline__ void jacobi_pixel(int x, int y, int w, int h, float reg,
                                             const float* __restrict__ img,
                                             const float* __restrict__ al,
                                             const float* __restrict__ Fp,
                                             const float* __restrict__ Bp, float* __restrict__ F,
                                             float* __restrict__ B) {
    const int i = x + y * w;
    const float a0 = al[i];
    const float a1 = 1.0f - a0;
    float b00 = a0 * img[i * 3 + 0];
    float b01 = a0 * img[i * 3 + 1];
    float b02 = a0 * img[i * 3 + 2];
    float b10 = a1 * img[i * 3 + 0];
    float b11 = a1 * img[i * 3 + 1];
    float b12 = a1 * img[i * 3 + 2];
    const int js[4] = {max(0, x - 1) + y * w, min(w - 1, x + 1) + y * w,
                       x + max(0, y - 1) * w, x + min(h - 1, y + 1) * w};
    float a_sum = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int j = js[d];
        const float da = reg + fabsf(a0 - al[j]);
        a_sum += da;
        b00 += da * Fp[j * 3 + 0];
        b01 += da * Fp[j * 3 + 1];
        b02 += da * Fp[j * 3 + 2];
        b10 += da * Bp[j * 3 + 0];
        b11 += da * Bp[j * 3 + 1];
        b12 += da * Bp[j * 3 + 2];
    }
    const float a00 = a0 * a0 + a_sum;
    const float a11 = a1 * a1 + a_sum;
    const float a01 = a0 * a1;
    const float inv_det = 1.0f / (a00 * a11 - a01 * a01);
    F[i * 3 + 0] = fmaxf(0.0f, fminf(1.0f, inv_det * (a11 * b00 - a01 * b10)));
    F[i * 3 + 1] = fmaxf(0.0f, fminf(1.0f, inv_det * (a11 * b01 - a01 * b11)));
    F[i * 3 + 2] = fmaxf(0.0f, fminf(1.0f, inv_det * (a11 * b02 - a01 * b12)));
    B[i * 3 + 0] = fmaxf(0.0f, fminf(1.0f, inv_det * (a00 * b10 - a01 * b00)));
    B[i * 3 + 1] = fmaxf(0.0f, fminf(1.0f, inv_det * (a00 * b11 - a01 * b01)));
    B[i * 3 + 2] = fmaxf(0.0f, fminf(1.0f, inv_det * (a00 * b12 - a01 * b02)));
}

__device__ __forceinline__ int src_of(int v, int n_src, int n_dst) {
    return min((int)((unsigned)v * (unsigned)n_src / (unsigned)n_dst), n_src - 1);
}

struct ResizeArgs {
    const float* image;  // (h0, w0, 3)
    const float* alpha;  // (h0, w0)
    int h0, w0;
    const float* F;  // read as (hp, wp, 3)
    const float* B;
    int hp, wp;
    float* image_level;  // (h, w, 3)
    float* alpha_level;  // (h, w)
    float* F_prev;
    float* B_prev;
    int h, w;
};

// The four nearest-neighbour resizes of one level (estimate_foreground_ml_cupy.py:5-32,
// x_src = min(x w_src / w_dst, w_src - 1)).
__device__ __forceinline__ void resize_pixel(const ResizeArgs& A, int x, int y) {
    const int i = x + y * A.w;
    const int s0 = src_of(x, A.w0, A.w) + src_of(y, A.h0, A.h) * A.w0;
    const int sp = src_of(x, A.wp, A.w) + src_of(y, A.hp, A.h) * A.wp;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        A.image_level[i * 3 + c] = A.image[s0 * 3 + c];
        A.F_prev[i * 3 + c] = A.F[sp * 3 + c];
        A.B_prev[i * 3 + c] = A.B[sp * 3 + c];
    }
    A.alpha_level[i] = A.alpha[s0];
}

__global__ void __launch_bounds__(256) k_fgj_resize(ResizeArgs A) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= A.w || y >= A.h) return;
    resize_pixel(A, x, y);
}

struct IterArgs {
    const float* image_level;
    const float* alpha_level;
    const float* F_prev;
    const float* B_prev;
    float* F;
    float* B;
    int h, w;
    float reg;
};

__global__ void __launch_bounds__(256) k_fgj_iter(IterArgs A) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= A.w || y >= A.h) return;
    jacobi_pixel(x, y, A.w, A.h, A.reg, A.image_level, A.alpha_level, A.F_prev, A.B_prev, A.F,
                 A.B);
}

// A whole small level in one CTA: the resizes, then n_iter iterations with
// the reference's swaps (buffers p[0] = F, p[1] = F_prev, q[0] = B,
// q[1] = B_prev as the level starts).
__global__ void __launch_bounds__(kSmallThreads) k_fgj_small(ResizeArgs R, float* F, float* F_prev,
                                                             float* B, float* B_prev, int n_iter,
                                                             float reg) {
    const int m = R.h * R.w;
    for (int p = threadIdx.x; p < m; p += blockDim.x) resize_pixel(R, p % R.w, p / R.w);
    __syncthreads();
    for (int it = 0; it < n_iter; ++it) {
        for (int p = threadIdx.x; p < m; p += blockDim.x)
            jacobi_pixel(p % R.w, p / R.w, R.w, R.h, reg, R.image_level, R.alpha_level, F_prev,
                         B_prev, F, B);
        __syncthreads();
        float* t = F;
        F = F_prev;
        F_prev = t;
        t = B;
        B = B_prev;
        B_prev = t;
    }
}

__global__ void k_fgj_seed(const float* __restrict__ image, float* F, float* B) {
    if (threadIdx.x < 3) {
        F[threadIdx.x] = image[threadIdx.x];
        B[threadIdx.x] = image[threadIdx.x];
    }
}

static long long align256(long long v) { return (v + 255) & ~255LL; }

}  // namespace fgj
}  // namespace pmb

using namespace pmb::fgj;

int64_t pmb_launch_fgj_workspace(int h, int w) {
    if (h <= 0 || w <= 0) return -1;
    const long long n = (long long)h * w * 3;
    return 5 * align256(n * 4) + align256((long long)h * w * 4);
}

// Returns 0, -1 (1x1 image: the reference divides by zero), -2 (bad
// arguments), -3 (workspace too small) or a positive CUDA error code.
int pmb_launch_fgj(const float* image, const float* alpha, int h0, int w0, float reg, int n_small,
                   int n_big, int small_size, float* outF, float* outB, void* workspace,
                   int64_t ws_bytes, cudaStream_t st) {
    // pixel and value indices are 32-bit in the kernels
    if (!image || !alpha || !outF || !workspace || h0 <= 0 || w0 <= 0 || h0 > 65535 ||
        w0 > 65535 || (long long)h0 * w0 * 3 >= (1LL << 31) || n_small < 0 || n_big < 0)
        return -2;
    const int m0 = std::max(w0, h0) - 1;
    int n_levels = 0;
    while ((m0 >> n_levels) != 0) ++n_levels;  // (max(w0, h0) - 1).bit_length()
    if (n_levels == 0) return -1;
    if (n_levels + 1 > kMaxLevels) return -2;
    if (ws_bytes < pmb_launch_fgj_workspace(h0, w0)) return -3;
    const long long n = (long long)h0 * w0 * 3;
    unsigned char* ws = (unsigned char*)workspace;
    float* bufs[5];
    for (int k = 0; k < 5; ++k) bufs[k] = (float*)(ws + k * align256(n * 4));
    float* alpha_level = (float*)(ws + 5 * align256(n * 4));
    float *F = bufs[0], *F_prev = bufs[1], *B = bufs[2], *B_prev = bufs[3];
    float* image_level = bufs[4];
    // the reference allocates its buffers with cp.zeros
    cudaError_t e = cudaMemsetAsync(workspace, 0, pmb_launch_fgj_workspace(h0, w0), st);
    if (e != cudaSuccess) return (int)e;
    k_fgj_seed<<<1, 32, 0, st>>>(image, F, B);
    int hp = 1, wp = 1;
    for (int lv = 0; lv <= n_levels; ++lv) {
        const double ex = (double)lv / (double)n_levels;
        const int w = (int)std::nearbyint(std::pow((double)w0, ex));
        const int h = (int)std::nearbyint(std::pow((double)h0, ex));
        const int n_iter = std::min(w, h) <= small_size ? n_small : n_big;
        ResizeArgs R{image, alpha, h0, w0, F, B, hp, wp, image_level, alpha_level, F_prev, B_prev,
                     h, w};
        if ((long long)h * w <= kSmallPixels) {
            k_fgj_small<<<1, kSmallThreads, 0, st>>>(R, F, F_prev, B, B_prev, n_iter, reg);
            if (n_iter & 1) {
                std::swap(F, F_prev);
                std::swap(B, B_prev);
            }
        } else {
            const dim3 grid((w + 31) / 32, (h + 7) / 8);
            k_fgj_resize<<<grid, 256, 0, st>>>(R);
            for (int it = 0; it < n_iter; ++it) {
                IterArgs I{image_level, alpha_level, F_prev, B_prev, F, B, h, w, reg};
                k_fgj_iter<<<grid, 256, 0, st>>>(I);
                std::swap(F, F_prev);
                std::swap(B, B_prev);
            }
        }
        hp = h;
        wp = w;
    }
    e = cudaMemcpyAsync(outF, F, n * 4, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && outB) e = cudaMemcpyAsync(outB, B, n * 4, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
