// Multi-level foreground / background estimation (PyMatting's
// estimate_foreground_ml, pymatting/foreground/estimate_foreground_ml.py:61-183)
// on sm_100a.
//
// The reference sweeps every level with an in-place Gauss-Seidel pass in
// raster order: pixel (y, x) of iteration i reads the NEW values of (y, x-1)
// and (y-1, x) and the OLD values of (y, x+1) and (y+1, x). This file
// reproduces that order exactly, so the results are bit-identical for the same
// seed colours:
//
// * Rows are cut into strips of 32; a warp sweeps one strip for one colour
//   channel with lane j on row 32k+j, lane j handling column s-j at step s.
//   The new value of the row above comes from lane j-1's previous step by a
//   shuffle, the old value of the row below from lane j+1's current load.
//   Lane 0 reads the strip above, lane 31 the strip below, through global
//   memory.
// * Every (iteration, strip) pair is a unit. Units are claimed from a ticket
//   counter in order, so a unit only ever waits on units that running CTAs
//   already hold. Iteration i+1 of strip k runs behind iteration i of strip
//   k+1, so all iterations of a level are in flight at once.
// * F and B live in a diagonal layout [channel][strip][step][lane], so each
//   warp's per-step loads and stores are one contiguous 512-byte row. Every
//   value is stored as {float value, uint32 epoch} in one 64-bit word. The
//   epoch is 0 for the level's starting values and i+1 for iteration i's
//   output. A reader polls until the epoch it needs appears. A 64-bit
//   relaxed store is single-copy atomic, so no fences or progress counters are
//   needed. Every wait is bounded (2 s on %globaltimer); a timeout sets an
//   error word and the kernel drains without waiting further.
// * The per-pixel terms that depend only on alpha (the four neighbour weights
//   and the inverse of the 2x2 system) are computed once per level by a
//   parallel prep kernel. They are stored per (strip, 32-step chunk) as one
//   contiguous record that the sweep brings into shared memory with bulk
//   async copies, two chunks in flight. The F/B rows a step reads are copied
//   into a per-warp shared-memory ring kDist steps ahead (cp.async groups),
//   so each step waits only for its own rows.
//
// Arithmetic follows numba's typing of the reference (a00, da and the
// right-hand side in float32; a1, a01, a11, the determinant and the inverse
// in float64) with explicitly rounded intrinsics, so nothing is contracted
// into fused multiply-adds.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "tma.cuh"

namespace pmb {
namespace fg {

constexpr int kLanes = 32;
constexpr int kChunk = 32;  // diagonal steps per staged coefficient chunk
constexpr int kMaxDepth = 8;
constexpr int kMaxLevels = 40;
constexpr int kGroupMax = 4;   // colour channels (warps) per sweep CTA
constexpr int kRingSlots = 8;  // shared-memory slots of F/B rows per warp
constexpr int kDist = 2;       // steps between a row's copy and its use (measured best)
constexpr unsigned long long kTimeoutNs = 2000000000ull;
constexpr int kMeanBlocks = 1184;
constexpr int kMeanThreads = 256;
constexpr int kMaxSide = 65535;
enum : int { kErrTimeout = 1, kErrStage = 2 };

// Coefficient record of one (strip, chunk): 32 steps x 32 lanes of
//   float4 da             (weights of the left, right, upper, lower neighbour)
//   double2 {b00, b01}, double b11  (inverse of the 2x2 system)
//   float2 pI[depth]      (a0 * I_c, float32(a1 * I_c))
constexpr int kOffDa = 0;
constexpr int kOffB0 = kChunk * kLanes * 16;
constexpr int kOffB11 = kOffB0 + kChunk * kLanes * 16;
constexpr int kOffPI = kOffB11 + kChunk * kLanes * 8;
constexpr int kPIBytes = kChunk * kLanes * 8;
constexpr int kBaseBytes = kOffPI;  // da and the 2x2 inverse, shared by all channels
__host__ __device__ constexpr int rec_bytes(int depth) { return kOffPI + depth * kPIBytes; }
// Shared memory of one staged chunk for a CTA of `cpg` channels.
__host__ __device__ constexpr int stage_bytes(int cpg) { return kBaseBytes + cpg * kPIBytes; }
// Per-warp ring: kRingSlots x (32 right-hand values + 32 neighbour-strip
// values, of which lanes 0 and 31 use theirs).
constexpr int kRingRow = 2 * kLanes;
constexpr int kWarpRingBytes = kRingSlots * kRingRow * 16;

struct Level {
    int h, w;    // level size
    int S, Q;    // strips, 32-step chunks per strip
    int Sp;      // steps per strip row in the diagonal layout (32 Q >= w + 31)
    int n_iter;  // Gauss-Seidel sweeps on this level
};

__device__ __forceinline__ uint64_t pack(float v, uint32_t epoch) {
    return ((uint64_t)epoch << 32) | (uint64_t)__float_as_uint(v);
}
__device__ __forceinline__ float value_of(uint64_t u) { return __uint_as_float((uint32_t)u); }
__device__ __forceinline__ uint32_t epoch_of(uint64_t u) { return (uint32_t)(u >> 32); }

__device__ __forceinline__ ulonglong2 ld_fb(const ulonglong2* p) {
    ulonglong2 v;
    asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];"
                 : "=l"(v.x), "=l"(v.y)
                 : "l"(p));
    return v;
}
__device__ __forceinline__ void st_fb(ulonglong2* p, uint64_t a, uint64_t b) {
    asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b)
                 : "memory");
}
__device__ __forceinline__ int ld_err(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Poll until both words of *p carry `want` and return them. Bounded: gives
// up (returning the last read) when the error word is set or after
// kTimeoutNs, which it reports.
__device__ __noinline__ ulonglong2 poll_epoch(const ulonglong2* p, uint32_t want, int* err,
                                              unsigned long long timeout_ns = kTimeoutNs) {
    unsigned long long t0 = 0;
    ulonglong2 v = make_ulonglong2(0, 0);
    for (uint32_t n = 0;; ++n) {
        if ((n & 63) == 0) {
            if (ld_err(err)) return v;
            if (n == 0) {
                t0 = now_ns();
            } else if (now_ns() - t0 > timeout_ns) {
                atomicCAS(err, 0, kErrTimeout);
                return v;
            }
        }
        v = ld_fb(p);
        if (epoch_of(v.x) == want && epoch_of(v.y) == want) return v;
    }
}

__device__ __forceinline__ bool has_epoch(ulonglong2 v, uint32_t want) {
    return epoch_of(v.x) == want && epoch_of(v.y) == want;
}

// 16-byte global -> shared copy cached in L2 only, tracked by commit groups.
// With n = 0 nothing is read and the 16 bytes are zero-filled.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t n) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Named barrier 1 over the CTA's `nthreads` threads.
__device__ __forceinline__ void bar_sync1(int nthreads) {
    asm volatile("barrier.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// ---------------------------------------------------------------------------
// Seed colours: mean image colour over alpha > 0.9 (foreground) and
// alpha < 0.1 (background), estimate_foreground_ml.py:79-95. Sums are taken
// in float64 in a fixed order (deterministic); the reference accumulates a
// running float32 sum, so the seeds agree to float32 rounding, not bitwise.
// ---------------------------------------------------------------------------

constexpr int kMeanValues = 2 * kMaxDepth + 2;  // F sums, B sums, F count, B count

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kMeanThreads) k_fg_mean_partial(const float* __restrict__ image,
                                                                  const float* __restrict__ alpha,
                                                                  long long n, int depth,
                                                                  double* __restrict__ part) {
    double acc[kMeanValues];
#pragma unroll
    for (int v = 0; v < kMeanValues; ++v) acc[v] = 0.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const float a = alpha[p];
        if (a > 0.9f) {
#pragma unroll
            for (int c = 0; c < kMaxDepth; ++c)
                if (c < depth) acc[c] += (double)image[p * depth + c];
            acc[2 * kMaxDepth] += 1.0;
        } else if (a < 0.1f) {
#pragma unroll
            for (int c = 0; c < kMaxDepth; ++c)
                if (c < depth) acc[kMaxDepth + c] += (double)image[p * depth + c];
            acc[2 * kMaxDepth + 1] += 1.0;
        }
    }
    __shared__ double red[kMeanThreads / 32][kMeanValues];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int v = 0; v < kMeanValues; ++v) {
        const double t = warp_sum(acc[v]);
        if (lane == 0) red[warp][v] = t;
    }
    __syncthreads();
    if (threadIdx.x < kMeanValues) {
        double t = 0.0;
        for (int wv = 0; wv < kMeanThreads / 32; ++wv) t += red[wv][threadIdx.x];
        part[(long long)blockIdx.x * kMeanValues + threadIdx.x] = t;
    }
}

// One warp per summed value, fixed order: deterministic.
__global__ void __launch_bounds__(32 * kMeanValues) k_fg_mean_final(const double* __restrict__ part,
                                                                    int nblocks, int depth,
                                                                    float* __restrict__ seed) {
    __shared__ double tot[kMeanValues];
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double a = 0.0;
    for (int b = lane; b < nblocks; b += 32) a += part[(long long)b * kMeanValues + v];
    a = warp_sum(a);
    if (lane == 0) tot[v] = a;
    __syncthreads();
    if (threadIdx.x < depth) {
        const int c = threadIdx.x;
        seed[c] = (float)(tot[c] / (tot[2 * kMaxDepth] + 1e-5));
        seed[depth + c] = (float)(tot[kMaxDepth + c] / (tot[2 * kMaxDepth + 1] + 1e-5));
    }
}

// ---------------------------------------------------------------------------
// Prep: coefficients of one level and its starting F/B (epoch 0), both in
// the diagonal layout. The level's image and alpha are the nearest-neighbour
// resize of the input (estimate_foreground_ml.py:5-55, x_src = x w_src / w),
// the starting F/B the nearest-neighbour resize of the previous level's
// result (or the seed colours for the 1x1 level).
// ---------------------------------------------------------------------------

struct PrepArgs {
    const float* image;  // (h0, w0, depth)
    const float* alpha;  // (h0, w0)
    int h0, w0, depth;
    float reg, gw;
    Level L, P;                 // this level and the previous one (P.h == 0: seed)
    const ulonglong2* fb_prev;  // previous level, diagonal layout
    const float* seed;          // F[depth], B[depth]
    unsigned char* rec;
    ulonglong2* fb;
};

// x_src = x * n_src / n_dst (sides <= 65535, so the product fits 32 bits).
__device__ __forceinline__ int src_index(int v, int n_dst, int n_src) {
    if (n_dst == n_src) return v;
    const unsigned s = (unsigned)v * (unsigned)n_src / (unsigned)n_dst;
    return (int)min(s, (unsigned)(n_src - 1));
}

// grid: (ceil(Sp * 32 / 256), S); one thread per diagonal entry (k, s, j).
__global__ void __launch_bounds__(256) k_fg_prep(PrepArgs A) {
    const Level L = A.L;
    const long long plane = (long long)L.S * L.Sp * kLanes;
    const int rb = rec_bytes(A.depth);
    {
        const int e_strip = blockIdx.x * blockDim.x + threadIdx.x;
        if (e_strip >= L.Sp * kLanes) return;
        const int j = e_strip & 31;
        const int s = e_strip >> 5;
        const int k = blockIdx.y;
        const long long idx = (long long)k * L.Sp * kLanes + e_strip;
        const int y = kLanes * k + j, x = s - j;
        const bool valid = y < L.h && x >= 0 && x < L.w;
        unsigned char* R = A.rec + ((long long)k * L.Q + (s >> 5)) * rb;
        const int e = ((s & 31) << 5) | j;  // entry within the record
        float4 da = make_float4(0.f, 0.f, 0.f, 0.f);
        double b00 = 0.0, b01 = 0.0, b11 = 0.0;
        if (valid) {
            const int yc = src_index(y, L.h, A.h0), xc = src_index(x, L.w, A.w0);
            const int ym = src_index(max(y - 1, 0), L.h, A.h0);
            const int yp = src_index(min(y + 1, L.h - 1), L.h, A.h0);
            const int xm = src_index(max(x - 1, 0), L.w, A.w0);
            const int xp = src_index(min(x + 1, L.w - 1), L.w, A.w0);
            const long long pc = (long long)yc * A.w0 + xc;
            const float a0 = A.alpha[pc];
            const float an[4] = {A.alpha[(long long)yc * A.w0 + xm], A.alpha[(long long)yc * A.w0 + xp],
                                 A.alpha[(long long)ym * A.w0 + xc], A.alpha[(long long)yp * A.w0 + xc]};
            const double a1 = __dsub_rn(1.0, (double)a0);
            float a00 = __fmul_rn(a0, a0);
            const double a01 = __dmul_rn((double)a0, a1);
            double a11 = __dmul_rn(a1, a1);
            float d[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float g = fabsf(__fsub_rn(a0, an[q]));
                d[q] = __fadd_rn(A.reg, __fmul_rn(A.gw, g));
                a00 = __fadd_rn(a00, d[q]);
                a11 = __dadd_rn(a11, (double)d[q]);
            }
            const double det = __dsub_rn(__dmul_rn((double)a00, a11), __dmul_rn(a01, a01));
            const double inv = __ddiv_rn(1.0, det);
            b00 = __dmul_rn(inv, a11);
            b01 = __dmul_rn(inv, -a01);
            b11 = __dmul_rn(inv, (double)a00);
            da = make_float4(d[0], d[1], d[2], d[3]);
            for (int c = 0; c < A.depth; ++c) {
                const float I = A.image[pc * A.depth + c];
                *(float2*)(R + kOffPI + c * kPIBytes + e * 8) =
                    make_float2(__fmul_rn(a0, I), __double2float_rn(__dmul_rn(a1, (double)I)));
            }
        } else {
            for (int c = 0; c < A.depth; ++c)
                *(float2*)(R + kOffPI + c * kPIBytes + e * 8) = make_float2(0.f, 0.f);
        }
        *(float4*)(R + kOffDa + e * 16) = da;
        *(double2*)(R + kOffB0 + e * 16) = make_double2(b00, b01);
        *(double*)(R + kOffB11 + e * 8) = b11;

        // starting values (epoch 0)
        long long src = -1;
        if (valid && A.P.h > 0) {
            const int yq = src_index(y, L.h, A.P.h), xq = src_index(x, L.w, A.P.w);
            src = ((long long)(yq >> 5) * A.P.Sp + (xq + (yq & 31))) * kLanes + (yq & 31);
        }
        const long long pplane = (long long)A.P.S * A.P.Sp * kLanes;
        for (int c = 0; c < A.depth; ++c) {
            float Fv = 0.f, Bv = 0.f;
            if (valid) {
                if (src >= 0) {
                    const ulonglong2 v = A.fb_prev[c * pplane + src];
                    Fv = value_of(v.x);
                    Bv = value_of(v.y);
                } else {
                    Fv = A.seed[c];
                    Bv = A.seed[A.depth + c];
                }
            }
            A.fb[c * plane + idx] = make_ulonglong2(pack(Fv, 0u), pack(Bv, 0u));
        }
    }
}

// ---------------------------------------------------------------------------
// Sweep: all iterations of one level. A CTA holds one warp per colour channel
// of a channel group (at most kGroupMax channels) and works on one unit
// (iteration it, strip k, channel group g) at a time.
// ---------------------------------------------------------------------------

struct SweepArgs {
    Level L;
    int depth, groups, cpg;  // channels, channel groups, channels per group
    const unsigned char* rec;
    ulonglong2* fb;
    float* outF;  // last level only: the final iteration also writes (h, w, depth)
    float* outB;
    int* ticket;
    int* err;
};

__global__ void __launch_bounds__(kLanes * kGroupMax, 1) k_fg_sweep(SweepArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_unit;
    const Level L = A.L;
    const int tid = threadIdx.x, w = tid >> 5, j = tid & 31;
    const int rb = rec_bytes(A.depth);
    const int sbytes = stage_bytes(A.cpg);
    ulonglong2* ring = (ulonglong2*)(smem + 2 * sbytes + w * kWarpRingBytes);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
    }
    __syncthreads();
    uint32_t phase0 = 0, phase1 = 0;
    const int units = L.n_iter * L.S * A.groups;
    const long long plane = (long long)L.S * L.Sp * kLanes;
    const long long strip = (long long)L.Sp * kLanes;

    for (;;) {
        if (tid == 0) {
            const int u = atomicAdd(A.ticket, 1);
            s_unit = ld_err(A.err) ? units : u;
        }
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= units) break;
        const int g = u % A.groups, ik = u / A.groups;
        const int it = ik / L.S, k = ik - it * L.S;
        const int c0 = g * A.cpg, ng = min(A.cpg, A.depth - c0);
        const unsigned char* rec_k = A.rec + (long long)k * L.Q * rb;
        const uint32_t stage_tx = kBaseBytes + ng * kPIBytes;
        auto stage = [&](int buf, int q) {
            const unsigned char* r = rec_k + (long long)q * rb;
            mbar_expect_tx(&bars[buf], stage_tx);
            bulk_load(smem + buf * sbytes, r, kBaseBytes, &bars[buf]);
            bulk_load(smem + buf * sbytes + kBaseBytes, r + kOffPI + c0 * kPIBytes, ng * kPIBytes,
                      &bars[buf]);
        };
        if (tid == 0) {
            fence_proxy_async();
            for (int b = 0; b < 2 && b < L.Q; ++b) stage(b, b);
        }
        if (w >= ng) {
            // no channel for this warp in this group: keep the phase parities
            // in step with the warps that wait on every chunk
            phase0 ^= (uint32_t)(((L.Q + 1) >> 1) & 1);
            phase1 ^= (uint32_t)((L.Q >> 1) & 1);
            continue;
        }
        const int c = c0 + w;
        ulonglong2* fbc = A.fb + c * plane;
        const int y0 = kLanes * k, y = y0 + j;
        const bool rowv = y < L.h;
        const uint32_t e_old = it, e_new = it + 1;
        const bool has_up = j == 0 && k > 0;
        const bool has_dn = j == 31 && y0 + kLanes < L.h;
        const bool last_out = A.outF != nullptr && it == L.n_iter - 1;
        ulonglong2* row_self = fbc + k * strip + j;
        const ulonglong2* row_up = fbc + (k - 1) * strip + 31;  // used only if has_up
        const ulonglong2* row_dn = fbc + (k + 1) * strip;       // used only if has_dn
        const bool has_aux = has_up || has_dn;
        const uint32_t want_aux = has_up ? e_new : e_old;
        // Step s reads [k][s+1][j] (right-hand value), [k-1][s+31][31] (lane 0)
        // and [k+1][s-31][0] (lane 31): three arithmetic sequences in s.
        const ulonglong2* gR = row_self + kLanes;
        const ulonglong2* gA = has_up ? row_up + 31 * kLanes : (has_dn ? row_dn - 31 * kLanes : row_self);
        const uint32_t ring_lane = smem_addr(ring) + j * 16;

        // Copy the rows step s needs into ring slot s % kRingSlots (zero-filled
        // where the lane has nothing to read). One commit group per step.
        auto issue = [&](int s) {
            const uint32_t slot = ring_lane + (uint32_t)((s & (kRingSlots - 1)) * kRingRow * 16);
            const bool cR = rowv && (unsigned)(s + 1 - j) < (unsigned)L.w;
            const bool cA = has_aux && (unsigned)(s - j) < (unsigned)L.w;
            cp_async16(slot, cR ? gR + (long long)s * kLanes : row_self, cR ? 16u : 0u);
            cp_async16(slot + kLanes * 16, cA ? gA + (long long)s * kLanes : row_self, cA ? 16u : 0u);
            cp_async_commit();
        };
        for (int r = 0; r < kDist; ++r) issue(r);

        float myF = 0.f, myB = 0.f;  // this lane's value from the previous step
        float pF = 0.f, pB = 0.f;    // old value of this lane's current column
        // Lane j first meets its column 0 as the right-hand value of step j-1;
        // for lane 0 that step would be -1, so its column 0 is read here.
        if (j == 0 && rowv) {
            ulonglong2 v = ld_fb(row_self);
            if (!has_epoch(v, e_old)) v = poll_epoch(row_self, e_old, A.err);
            pF = value_of(v.x);
            pB = value_of(v.y);
        }
        const int nthr = kLanes * ng;
        for (int q = 0; q < L.Q; ++q) {
            uint64_t* bar = &bars[q & 1];
            const uint32_t ph = (q & 1) ? phase1 : phase0;
            if (!mbar_wait(bar, ph)) atomicCAS(A.err, 0, kErrStage);
            if (q & 1) phase1 ^= 1u; else phase0 ^= 1u;
            const unsigned char* cb = smem + (q & 1) * sbytes;
            // the last step with work is w + 30 (lane 31 at column w - 1)
            const int t_end = min(kChunk, L.w + kLanes - 1 - kChunk * q);
// not unrolled: the rolled loop measured 33 % faster than unroll 4
#pragma unroll 1
            for (int t = 0; t < t_end; ++t) {
                const int s = kChunk * q + t;
                const int cur = s - j;
                cp_async_wait<kDist - 1>();
                const ulonglong2* slot = ring + (s & (kRingSlots - 1)) * kRingRow;
                ulonglong2 Rv = slot[j];
                ulonglong2 Av = slot[kLanes + j];
                // the slot refilled now was read at step s - 1
                issue(s + kDist);
                const bool inCol = (unsigned)cur < (unsigned)L.w;
                const bool needR = rowv && (unsigned)(cur + 1) < (unsigned)L.w;
                const bool needA = has_aux && inCol;
                const bool okR = !needR || has_epoch(Rv, e_old);
                const bool okA = !needA || has_epoch(Av, want_aux);
                if (!__all_sync(0xffffffffu, okR && okA)) {
                    if (!okR) Rv = poll_epoch(gR + (long long)s * kLanes, e_old, A.err);
                    if (!okA) Av = poll_epoch(gA + (long long)s * kLanes, want_aux, A.err);
                }
                const float rF = value_of(Rv.x), rB = value_of(Rv.y);
                const float aF = value_of(Av.x), aB = value_of(Av.y);
                const float uF = __shfl_up_sync(0xffffffffu, myF, 1);
                const float uB = __shfl_up_sync(0xffffffffu, myB, 1);
                const float dF = __shfl_down_sync(0xffffffffu, rF, 1);
                const float dB = __shfl_down_sync(0xffffffffu, rB, 1);
                const bool first = cur == 0, rin = cur + 1 < L.w;
                const bool top = y == 0, bottom = y == L.h - 1;
                const float Fl = first ? pF : myF, Bl = first ? pB : myB;
                const float Fr = rin ? rF : pF, Br = rin ? rB : pB;
                const float Fu = top ? pF : (j == 0 ? aF : uF);
                const float Bu = top ? pB : (j == 0 ? aB : uB);
                const float Fd = bottom ? pF : (j == 31 ? aF : dF);
                const float Bd = bottom ? pB : (j == 31 ? aB : dB);
                const int e = (t << 5) | j;
                const float4 da = *(const float4*)(cb + kOffDa + e * 16);
                const double2 b0 = *(const double2*)(cb + kOffB0 + e * 16);
                const double b11 = *(const double*)(cb + kOffB11 + e * 8);
                const float2 pI = *(const float2*)(cb + kOffPI + w * kPIBytes + e * 8);
                float f0 = pI.x, f1 = pI.y;
                f0 = __fadd_rn(f0, __fmul_rn(da.x, Fl));
                f1 = __fadd_rn(f1, __fmul_rn(da.x, Bl));
                f0 = __fadd_rn(f0, __fmul_rn(da.y, Fr));
                f1 = __fadd_rn(f1, __fmul_rn(da.y, Br));
                f0 = __fadd_rn(f0, __fmul_rn(da.z, Fu));
                f1 = __fadd_rn(f1, __fmul_rn(da.z, Bu));
                f0 = __fadd_rn(f0, __fmul_rn(da.w, Fd));
                f1 = __fadd_rn(f1, __fmul_rn(da.w, Bd));
                double Fc = __dadd_rn(__dmul_rn(b0.x, (double)f0), __dmul_rn(b0.y, (double)f1));
                double Bc = __dadd_rn(__dmul_rn(b0.y, (double)f0), __dmul_rn(b11, (double)f1));
                // max(0.0, min(1.0, v)) with Python's argument order
                Fc = Fc < 1.0 ? Fc : 1.0;
                Fc = Fc > 0.0 ? Fc : 0.0;
                Bc = Bc < 1.0 ? Bc : 1.0;
                Bc = Bc > 0.0 ? Bc : 0.0;
                const float nF = __double2float_rn(Fc), nB = __double2float_rn(Bc);
                if (rowv && inCol) {
                    st_fb(row_self + (long long)s * kLanes, pack(nF, e_new), pack(nB, e_new));
                    if (last_out) {
                        const long long o = ((long long)y * L.w + cur) * A.depth + c;
                        A.outF[o] = nF;
                        if (A.outB) A.outB[o] = nB;
                    }
                }
                // (garbage in lanes outside the image; nothing reads it there)
                myF = nF;
                myB = nB;
                pF = rF;
                pB = rB;
            }
            // every active warp is done with this buffer: refill it with chunk q + 2
            bar_sync1(nthr);
            if (tid == 0 && q + 2 < L.Q) {
                fence_proxy_async();
                stage(q & 1, q + 2);
            }
        }
        cp_async_wait<0>();
    }
}

// Final values when the last level runs no sweep (n_iter == 0): gather the
// level's starting values out of the diagonal layout.
__global__ void __launch_bounds__(256) k_fg_output(Level L, int depth, const ulonglong2* __restrict__ fb,
                                                   float* __restrict__ outF, float* __restrict__ outB) {
    const long long n = (long long)L.h * L.w;
    const long long plane = (long long)L.S * L.Sp * kLanes;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(p / L.w), x = (int)(p % L.w);
        const long long d = ((long long)(y >> 5) * L.Sp + (x + (y & 31))) * kLanes + (y & 31);
        for (int c = 0; c < depth; ++c) {
            const ulonglong2 v = fb[c * plane + d];
            outF[p * depth + c] = value_of(v.x);
            if (outB) outB[p * depth + c] = value_of(v.y);
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// Level sizes of estimate_foreground_ml.py:101-105 (glibc pow and log2, ties
// of round() to even). Returns the level count, or -1 for a 1x1 image (the
// reference divides by zero there).
static int plan_levels(int h0, int w0, int n_small, int n_big, int small_size, Level* out) {
    const int m = std::max(h0, w0);
    const int n = (int)std::ceil(std::log2((double)m));
    if (n == 0) return -1;
    if (n + 1 > kMaxLevels) return -2;
    for (int i = 0; i <= n; ++i) {
        const double e = (double)i / (double)n;
        Level& L = out[i];
        L.w = (int)std::nearbyint(std::pow((double)w0, e));
        L.h = (int)std::nearbyint(std::pow((double)h0, e));
        L.S = (L.h + kLanes - 1) / kLanes;
        L.Q = (L.w + kLanes - 1 + kChunk - 1) / kChunk;
        L.Sp = L.Q * kChunk;
        L.n_iter = (L.w <= small_size && L.h <= small_size) ? n_small : n_big;
    }
    return n + 1;
}

static long long align256(long long v) { return (v + 255) & ~255LL; }

struct Layout {
    long long hdr, part, seed, fb0, fb1, rec, total;
};

static Layout layout(int h0, int w0, int depth) {
    const int S = (h0 + kLanes - 1) / kLanes;
    const int Q = (w0 + kLanes - 1 + kChunk - 1) / kChunk;
    const long long fb = (long long)depth * S * Q * kChunk * kLanes * 16;
    Layout l;
    l.hdr = 0;
    l.part = 1024;
    l.seed = l.part + align256((long long)kMeanBlocks * kMeanValues * 8);
    l.fb0 = l.seed + 256;
    l.fb1 = l.fb0 + align256(fb);
    l.rec = l.fb1 + align256(fb);
    l.total = l.rec + align256((long long)S * Q * rec_bytes(depth));
    return l;
}

// Self-test of the bounded poll: one thread waits with poll_epoch for epoch
// 1 in a word that holds epoch 0 and that nothing writes, with a deadline of
// timeout_ns. The poll must give up and leave kErrTimeout in *err.
__global__ void k_selftest_poll(const ulonglong2* word, int* err, unsigned long long timeout_ns) {
    if (threadIdx.x == 0 && blockIdx.x == 0) (void)poll_epoch(word, 1u, err, timeout_ns);
}

}  // namespace fg
}  // namespace pmb

using namespace pmb::fg;

// scratch: 64 bytes of device memory. Returns 0 and sets *timed_out (1 if
// the poll gave up and reported it), or a CUDA error code.
int pmb_launch_selftest_poll(void* scratch, unsigned long long timeout_ns, int* timed_out,
                             cudaStream_t st) {
    ulonglong2* word = static_cast<ulonglong2*>(scratch);
    int* err = reinterpret_cast<int*>(static_cast<char*>(scratch) + 32);
    cudaError_t e = cudaMemsetAsync(scratch, 0, 64, st);
    if (e != cudaSuccess) return (int)e;
    k_selftest_poll<<<1, 32, 0, st>>>(word, err, timeout_ns);
    int h = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    *timed_out = h == kErrTimeout ? 1 : 0;
    return 0;
}

int64_t pmb_launch_fg_workspace(int h, int w, int depth) {
    if (h <= 0 || w <= 0 || depth < 1 || depth > kMaxDepth) return -1;
    return layout(h, w, depth).total;
}

int pmb_launch_fg_levels(int h, int w, int n_small, int n_big, int small_size, int* hw, int max_levels) {
    Level lv[kMaxLevels];
    const int n = plan_levels(h, w, n_small, n_big, small_size, lv);
    if (n < 0) return n;
    for (int i = 0; i < n && i < max_levels; ++i) {
        hw[2 * i] = lv[i].h;
        hw[2 * i + 1] = lv[i].w;
    }
    return n;
}

// Returns 0, -1 (1x1 image), -2 (bad arguments), -3 (workspace too small) or
// a positive CUDA error code.
int pmb_launch_fg(const float* image, const float* alpha, int h0, int w0, int depth, float reg,
                  int n_small, int n_big, int small_size, float gw, const float* seed_in,
                  float* outF, float* outB, void* workspace, int64_t ws_bytes, cudaStream_t st) {
    if (!image || !alpha || !outF || !workspace || h0 <= 0 || w0 <= 0 || h0 > kMaxSide ||
        w0 > kMaxSide || depth < 1 || depth > kMaxDepth || n_small < 0 || n_big < 0)
        return -2;
    Level lv[kMaxLevels];
    const int nl = plan_levels(h0, w0, n_small, n_big, small_size, lv);
    if (nl == -1) return -1;
    if (nl < 0) return -2;
    const Layout l = layout(h0, w0, depth);
    if (ws_bytes < l.total) return -3;
    unsigned char* ws = (unsigned char*)workspace;
    int* hdr = (int*)(ws + l.hdr);  // [0] error word, [1 + level] ticket counters
    double* part = (double*)(ws + l.part);
    float* seed = (float*)(ws + l.seed);
    ulonglong2* fbs[2] = {(ulonglong2*)(ws + l.fb0), (ulonglong2*)(ws + l.fb1)};
    unsigned char* rec = ws + l.rec;

    int dev = 0, num_sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (num_sms <= 0) num_sms = 148;
    const int groups = (depth + kGroupMax - 1) / kGroupMax;
    const int cpg = (depth + groups - 1) / groups;
    const int sweep_smem = 2 * stage_bytes(cpg) + cpg * kWarpRingBytes;
    cudaError_t e = cudaFuncSetAttribute(k_fg_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         2 * stage_bytes(kGroupMax) + kGroupMax * kWarpRingBytes);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemsetAsync(hdr, 0, 1024, st);
    if (e != cudaSuccess) return (int)e;
    if (!seed_in) {
        const long long n = (long long)h0 * w0;
        k_fg_mean_partial<<<kMeanBlocks, kMeanThreads, 0, st>>>(image, alpha, n, depth, part);
        k_fg_mean_final<<<1, 32 * kMeanValues, 0, st>>>(part, kMeanBlocks, depth, seed);
        seed_in = seed;
    }
    Level none{};
    for (int i = 0; i < nl; ++i) {
        const Level& L = lv[i];
        PrepArgs P;
        P.image = image;
        P.alpha = alpha;
        P.h0 = h0;
        P.w0 = w0;
        P.depth = depth;
        P.reg = reg;
        P.gw = gw;
        P.L = L;
        P.P = i > 0 ? lv[i - 1] : none;
        P.fb_prev = fbs[(i + 1) & 1];
        P.seed = seed_in;
        P.rec = rec;
        P.fb = fbs[i & 1];
        const dim3 pgrid((L.Sp * kLanes + 255) / 256, L.S);
        k_fg_prep<<<pgrid, 256, 0, st>>>(P);
        const bool last = i == nl - 1;
        if (L.n_iter > 0) {
            SweepArgs S;
            S.L = L;
            S.depth = depth;
            S.groups = groups;
            S.cpg = cpg;
            S.rec = rec;
            S.fb = fbs[i & 1];
            S.outF = last ? outF : nullptr;
            S.outB = last ? outB : nullptr;
            S.ticket = hdr + 1 + i;
            S.err = hdr;
            const int units = L.n_iter * L.S * groups;
            const int grid = std::min(units, num_sms);
            k_fg_sweep<<<grid, kLanes * cpg, sweep_smem, st>>>(S);
        } else if (last) {
            const long long n = (long long)L.h * L.w;
            const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)num_sms * 16);
            k_fg_output<<<blocks, 256, 0, st>>>(L, depth, fbs[i & 1], outF, outB);
        }
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

// Error word of the last run in `workspace` (synchronises the stream).
int pmb_launch_fg_status(void* workspace, cudaStream_t st, int* status) {
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, workspace, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    *status = v;
    return 0;
}
