/* ORACLE — test infrastructure, not product code.
 *
 * Plain-C restatement of PyMatting's multi-level foreground/background
 * estimation, pymatting/foreground/estimate_foreground_ml.py:61-183
 * (_estimate_fb_ml) with the nearest-neighbour resizes of :5-55.
 *
 * The reference runs under numba without parallel=True, so its prange loops
 * are ordinary loops and every level is an in-place Gauss-Seidel sweep in
 * raster order. The arithmetic types follow numba's typing of that source:
 * a0, a00, da, gradient and the right-hand side b are float32; a1, a01, a11,
 * the determinant, its inverse and the 2x2 inverse entries are float64; F and
 * B are stored as float32. Built with -ffp-contract=off so that no product
 * and sum are fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int64_t clampi(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* estimate_foreground_ml.py:5-29 (and :32-55 for one channel) */
static void resize_nearest(float* dst, int64_t hd, int64_t wd, const float* src, int64_t hs,
                           int64_t ws, int depth) {
    for (int64_t y = 0; y < hd; ++y)
        for (int64_t x = 0; x < wd; ++x) {
            int64_t xs = clampi(x * ws / wd, 0, ws - 1);
            int64_t ys = clampi(y * hs / hd, 0, hs - 1);
            for (int c = 0; c < depth; ++c) dst[(y * wd + x) * depth + c] = src[(ys * ws + xs) * depth + c];
        }
}

/* estimate_foreground_ml.py:79-95: running float32 sums in raster order, then
 * division by (count + 1e-5) in float64 and storage as float32. */
void oracle_fg_mean_colors(const float* image, const float* alpha, int64_t h0, int64_t w0,
                           int depth, float* seed /* F[depth], B[depth] */) {
    float fs[8] = {0}, bs[8] = {0};
    int64_t fc = 0, bc = 0;
    for (int64_t p = 0; p < h0 * w0; ++p) {
        if (alpha[p] > 0.9f) {
            for (int c = 0; c < depth; ++c) fs[c] += image[p * depth + c];
            ++fc;
        }
        if (alpha[p] < 0.1f) {
            for (int c = 0; c < depth; ++c) bs[c] += image[p * depth + c];
            ++bc;
        }
    }
    for (int c = 0; c < depth; ++c) {
        seed[c] = (float)((double)fs[c] / ((double)fc + 1e-5));
        seed[depth + c] = (float)((double)bs[c] / ((double)bc + 1e-5));
    }
}

/* Level sizes of estimate_foreground_ml.py:101-105. Returns the number of
 * levels (n_levels + 1), or -1 where the reference divides by zero (a 1x1
 * image). */
int oracle_fg_levels(int64_t h0, int64_t w0, int64_t* hs, int64_t* ws, int max_levels) {
    int64_t m = w0 > h0 ? w0 : h0;
    int n = (int)ceil(log2((double)m));
    if (n == 0) return -1;
    if (n + 1 > max_levels) return -2;
    for (int i = 0; i <= n; ++i) {
        double e = (double)i / (double)n;
        ws[i] = (int64_t)nearbyint(pow((double)w0, e));
        hs[i] = (int64_t)nearbyint(pow((double)h0, e));
    }
    return n + 1;
}

/* estimate_foreground_ml.py:61-183. seed: the 2 depth mean colours (F then
 * B); NULL computes them as the reference does. F_out/B_out: (h0, w0, depth),
 * depth <= 8. */
int oracle_fg_ml(const float* input_image, const float* input_alpha, int64_t h0, int64_t w0,
                 int depth, float regularization, int n_small_iterations, int n_big_iterations,
                 int small_size, float gradient_weight, const float* seed, float* F_out,
                 float* B_out) {
    float mean[16];
    if (depth < 1 || depth > 8) return -3;
    if (seed) memcpy(mean, seed, sizeof(float) * 2 * depth);
    else oracle_fg_mean_colors(input_image, input_alpha, h0, w0, depth, mean);
    int64_t hs[64], ws[64];
    int nl = oracle_fg_levels(h0, w0, hs, ws, 64);
    if (nl < 0) return nl;

    int64_t hp = 1, wp = 1;
    float* Fp = (float*)malloc(sizeof(float) * depth);
    float* Bp = (float*)malloc(sizeof(float) * depth);
    for (int c = 0; c < depth; ++c) { Fp[c] = mean[c]; Bp[c] = mean[depth + c]; }

    static const int dx[4] = {-1, 1, 0, 0};
    static const int dy[4] = {0, 0, -1, 1};
    for (int lv = 0; lv < nl; ++lv) {
        int64_t h = hs[lv], w = ws[lv];
        float* image = (float*)malloc(sizeof(float) * h * w * depth);
        float* alpha = (float*)malloc(sizeof(float) * h * w);
        float* F = (float*)malloc(sizeof(float) * h * w * depth);
        float* B = (float*)malloc(sizeof(float) * h * w * depth);
        resize_nearest(image, h, w, input_image, h0, w0, depth);
        resize_nearest(alpha, h, w, input_alpha, h0, w0, 1);
        resize_nearest(F, h, w, Fp, hp, wp, depth);
        resize_nearest(B, h, w, Bp, hp, wp, depth);
        int n_iter = (w <= small_size && h <= small_size) ? n_small_iterations : n_big_iterations;
        float b[2][8];
        for (int it = 0; it < n_iter; ++it)
            for (int64_t y = 0; y < h; ++y)
                for (int64_t x = 0; x < w; ++x) {
                    float a0 = alpha[y * w + x];
                    double a1 = 1.0 - (double)a0;
                    float a00 = a0 * a0;
                    double a01 = (double)a0 * a1;
                    double a11 = a1 * a1;
                    for (int c = 0; c < depth; ++c) {
                        b[0][c] = a0 * image[(y * w + x) * depth + c];
                        b[1][c] = (float)(a1 * (double)image[(y * w + x) * depth + c]);
                    }
                    for (int d = 0; d < 4; ++d) {
                        int64_t x2 = clampi(x + dx[d], 0, w - 1);
                        int64_t y2 = clampi(y + dy[d], 0, h - 1);
                        float gradient = fabsf(a0 - alpha[y2 * w + x2]);
                        float da = regularization + gradient_weight * gradient;
                        a00 += da;
                        a11 += (double)da;
                        for (int c = 0; c < depth; ++c) {
                            b[0][c] += da * F[(y2 * w + x2) * depth + c];
                            b[1][c] += da * B[(y2 * w + x2) * depth + c];
                        }
                    }
                    double determinant = (double)a00 * a11 - a01 * a01;
                    double inv_det = 1.0 / determinant;
                    double b00 = inv_det * a11;
                    double b01 = inv_det * -a01;
                    double b11 = inv_det * (double)a00;
                    for (int c = 0; c < depth; ++c) {
                        double F_c = b00 * (double)b[0][c] + b01 * (double)b[1][c];
                        double B_c = b01 * (double)b[0][c] + b11 * (double)b[1][c];
                        /* max(0.0, min(1.0, v)) with Python's argument order */
                        F_c = F_c < 1.0 ? F_c : 1.0;
                        F_c = F_c > 0.0 ? F_c : 0.0;
                        B_c = B_c < 1.0 ? B_c : 1.0;
                        B_c = B_c > 0.0 ? B_c : 0.0;
                        F[(y * w + x) * depth + c] = (float)F_c;
                        B[(y * w + x) * depth + c] = (float)B_c;
                    }
                }
        free(image);
        free(alpha);
        free(Fp);
        free(Bp);
        Fp = F;
        Bp = B;
        hp = h;
        wp = w;
    }
    memcpy(F_out, Fp, sizeof(float) * h0 * w0 * depth);
    memcpy(B_out, Bp, sizeof(float) * h0 * w0 * depth);
    free(Fp);
    free(Bp);
    return 0;
}
