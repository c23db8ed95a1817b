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
// resized from the buffer named F, and F returned. The per-pixel update is
// this file's own formulation of the 2x2 normal equations (below); it
// agrees with the reference's to float32 rounding, and the tests pin it
// against the oracle's restatement of the reference.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

namespace pmb {
namespace fgj {

constexpr int kSmallThreads = 1024;
constexpr int kSmallPixels = 8192;  // levels this small run in one CTA
constexpr int kMaxLevels = 40;

// Per pixel, the cost (a F + (1 - a) B - I)^2 + sum_j w_j (|F - F_j|^2 +
// |B - B_j|^2) over the four neighbours j (clamped at the border), with
// w_j = reg + |a - a_j|, is minimised channel by channel with the
// neighbours' previous F_j, B_j held fixed (a Jacobi step;
// estimate_foreground_ml_cupy.py:34-107 is the reference's kernel). With
// S = sum_j w_j the normal equations are
//   [a^2 + S   a(1-a)  ] [F]   [a I + sum_j w_j F_j    ]
//   [a(1-a)    (1-a)^2+S] [B] = [(1-a) I + sum_j w_j B_j],
// solved by Cramer's rule and clamped to [0, 1]. The right-hand sides are
// accumulated from the data term on, neighbour by neighbour.
struct FBSums {
    float S;         // sum of the weights
    float f[3];      // a I + sum of w_j F_j per channel
    float b[3];      // (1 - a) I + sum of w_j B_j per channel
};

__device__ __forceinline__ FBSums fb_start(float a, const float* I) {
    const float na = 1.0f - a;
    return FBSums{0.0f, {a * I[0], a * I[1], a * I[2]}, {na * I[0], na * I[1], na * I[2]}};
}

__device__ __forceinline__ void fb_add(FBSums& q, float a, float aj, float reg, const float* Fj,
                                       const float* Bj, int stride) {
    const float wj = reg + fabsf(a - aj);
    q.S += wj;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        q.f[c] += wj * Fj[c * stride];
        q.b[c] += wj * Bj[c * stride];
    }
}

__device__ __forceinline__ void fb_solve(const FBSums& q, float a, float* F, float* B) {
    const float na = 1.0f - a;
    const float pF = a * a + q.S;      // F-F entry
    const float pB = na * na + q.S;    // B-B entry
    const float m = a * na;            // coupling
    const float inv = 1.0f / (pF * pB - m * m);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        // min first: a NaN (S = 0, only with reg = 0) clamps to 1, as in
        // the reference
        F[c] = fmaxf(fminf((pB * q.f[c] - m * q.b[c]) * inv, 1.0f), 0.0f);
        B[c] = fmaxf(fminf((pF * q.b[c] - m * q.f[c]) * inv, 1.0f), 0.0f);
    }
}

// One pixel read straight from global memory (the one-CTA small levels).
__device__ __forceinline__ void jacobi_global(int x, int y, int w, int h, float reg,
                                              const float* __restrict__ img,
                                              const float* __restrict__ al,
                                              const float* __restrict__ Fp,
                                              const float* __restrict__ Bp, float* __restrict__ F,
                                              float* __restrict__ B) {
    const int i = x + y * w;
    const float a = al[i];
    const float I[3] = {img[3 * i], img[3 * i + 1], img[3 * i + 2]};
    FBSums q = fb_start(a, I);
    const int nb[4] = {max(x - 1, 0) + y * w, min(x + 1, w - 1) + y * w,
                       x + max(y - 1, 0) * w, x + min(y + 1, h - 1) * w};
#pragma unroll
    for (int k = 0; k < 4; ++k) fb_add(q, a, al[nb[k]], reg, Fp + 3 * nb[k], Bp + 3 * nb[k], 1);
    float f[3], b[3];
    fb_solve(q, a, f, b);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        F[3 * i + c] = f[c];
        B[3 * i + c] = b[c];
    }
}

// Tiles of the large levels: kJX x kJY pixels per CTA, one per thread. The
// tile's alpha and previous F / B with a one-pixel halo (coordinates clamped
// to the image, which makes the halo hold exactly the neighbours the border
// pixels use) are staged in shared memory, F and B split into channel
// planes; rows of the interleaved global arrays are read contiguously.
constexpr int kJX = 32, kJY = 8;
constexpr int kHX = kJX + 2, kHY = kJY + 2;

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

__global__ void __launch_bounds__(kJX * kJY) k_fgj_iter(IterArgs A) {
    __shared__ float s_a[kHY][kHX];
    __shared__ float s_f[3][kHY][kHX];
    __shared__ float s_b[3][kHY][kHX];
    const int x0 = blockIdx.x * kJX, y0 = blockIdx.y * kJY;
    // Stage: halo row r is image row clamp(y0 - 1 + r); element e of that row
    // is channel e % 3 of column clamp(x0 - 1 + e / 3).
    for (int q = threadIdx.x; q < kHY * kHX * 3; q += kJX * kJY) {
        const int r = q / (kHX * 3), e = q - r * (kHX * 3);
        const int hx = e / 3, c = e - hx * 3;
        const int y = min(max(y0 - 1 + r, 0), A.h - 1);
        const int x = min(max(x0 - 1 + hx, 0), A.w - 1);
        const int g = (y * A.w + x) * 3 + c;
        s_f[c][r][hx] = A.F_prev[g];
        s_b[c][r][hx] = A.B_prev[g];
        if (c == 0) s_a[r][hx] = A.alpha_level[y * A.w + x];
    }
    __syncthreads();
    const int tx = threadIdx.x % kJX, ty = threadIdx.x / kJX;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= A.w || y >= A.h) return;
    const int cx = tx + 1, cy = ty + 1;
    const float a = s_a[cy][cx];
    const int i = y * A.w + x;
    const float I[3] = {A.image_level[3 * i], A.image_level[3 * i + 1],
                        A.image_level[3 * i + 2]};
    FBSums q = fb_start(a, I);
    constexpr int ps = kHY * kHX;   // channel-plane stride
    // Neighbours left, right, up, down (the halo already holds the clamp).
    fb_add(q, a, s_a[cy][cx - 1], A.reg, &s_f[0][cy][cx - 1], &s_b[0][cy][cx - 1], ps);
    fb_add(q, a, s_a[cy][cx + 1], A.reg, &s_f[0][cy][cx + 1], &s_b[0][cy][cx + 1], ps);
    fb_add(q, a, s_a[cy - 1][cx], A.reg, &s_f[0][cy - 1][cx], &s_b[0][cy - 1][cx], ps);
    fb_add(q, a, s_a[cy + 1][cx], A.reg, &s_f[0][cy + 1][cx], &s_b[0][cy + 1][cx], ps);
    float f[3], b[3];
    fb_solve(q, a, f, b);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        A.F[3 * i + c] = f[c];
        A.B[3 * i + c] = b[c];
    }
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
            jacobi_global(p % R.w, p / R.w, R.w, R.h, reg, R.image_level, R.alpha_level, F_prev,
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
            const dim3 tiles((w + kJX - 1) / kJX, (h + kJY - 1) / kJY);
            for (int it = 0; it < n_iter; ++it) {
                IterArgs I{image_level, alpha_level, F_prev, B_prev, F, B, h, w, reg};
                k_fgj_iter<<<tiles, kJX * kJY, 0, st>>>(I);
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
