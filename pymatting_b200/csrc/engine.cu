// Host-side engine and C-ABI of the closed-form alpha solver.
//
// Objects (all opaque to callers, declared in include/pymatting_b200.h):
//   pmb_stencil  batch of pixel-grid systems (L + lambda D) sharing one
//                preconditioner choice: none / Jacobi / V-cycle, FP64 or
//                FP32-inner with FP64 iterative refinement;
//   pmb_csr      one general CSR system (hard-constraint L_U, user matrices)
//                with none / Jacobi / matrix / incomplete-Cholesky M.
// The caller owns every device buffer: each object reports the workspace
// size it needs and carves it up at bind time. The only things an object
// allocates itself are a stream, two events, CUDA graphs and a small pinned
// status buffer, all released by its destroy call.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "csr.cuh"
#include "ichol.cuh"
#include "pm_common.cuh"
#include "stencil.cuh"

#define PMB_API extern "C" __attribute__((visibility("default")))

int pmb_launch_cf_ell(const double*, const uint8_t*, int, int, int, double, const uint8_t*,
                      double, double*, int64_t*, int64_t*, cudaStream_t);
int pmb_scan_exclusive(int64_t*, int64_t, int64_t*, int64_t*, cudaStream_t);
int pmb_launch_ell_count(const double*, int, int, int, int64_t*, cudaStream_t);
int pmb_launch_ell_fill(const double*, int, int, int, const int64_t*, int64_t*, double*,
                        cudaStream_t);
int pmb_launch_flag_unknown(const uint8_t*, int64_t, int64_t*, cudaStream_t);
int pmb_launch_lu_count(const uint8_t*, int, int, int, int64_t*, const int64_t*, cudaStream_t);
int pmb_launch_lu_fill(const double*, const uint8_t*, const uint8_t*, int, int, int,
                       const int64_t*, const int64_t*, int64_t*, double*, double*, cudaStream_t);
int pmb_launch_alpha_compose(const double*, const uint8_t*, const int64_t*, const double*, int64_t,
                             double*, cudaStream_t);
int pmb_launch_trimap_masks(const double*, int64_t, double, double, uint8_t*, uint8_t*,
                            unsigned long long*, cudaStream_t);
int pmb_launch_cf_half(const double*, const uint8_t*, int, int, double, double*, int,
                       const uint8_t*, double, cudaStream_t);
int pmb_launch_cf_hard(const double*, const uint8_t*, const uint8_t*, int, int, double, double*,
                       int, double*, cudaStream_t);

namespace pmb {

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define PMB_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(-2, std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)

enum : int { kErrArg = -1, kErrCuda = -2, kErrState = -3, kErrZeroDiv = -4 };

static thread_local cudaError_t t_launch_error = cudaSuccess;
int launch_status(cudaError_t e) {
    if (e == cudaSuccess) return 0;
    t_launch_error = e;
    return -2;
}
cudaError_t take_launch_error() {
    const cudaError_t e = t_launch_error;
    t_launch_error = cudaSuccess;
    return e;
}

// Text of the CUDA error behind a failed launch helper (the error the helper
// recorded, else the pending one; "bad arguments or sizes" if there is none).
static const char* launch_error_text() {
    cudaError_t e = take_launch_error();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e != cudaSuccess ? cudaGetErrorString(e) : "bad arguments or sizes";
}

static inline int pitch_for(int w) { return ((w + 31) / 32) * 32; }

// Aligned sub-allocation inside the caller's workspace.
struct Carve {
    size_t off = 0;
    template <typename T>
    size_t take(int64_t count) {
        off = (off + 255) & ~size_t(255);
        size_t at = off;
        off += sizeof(T) * (size_t)std::max<int64_t>(count, 1);
        return at;
    }
};

static int tiles_of(int h, int w, int th, int tw) { return ((h + th - 1) / th) * ((w + tw - 1) / tw); }


// --------------------------------------------------------------------------
// Stencil batch solver
// --------------------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

struct HostList {
    std::vector<GridDesc> grids;     // descriptors of this list
    std::vector<GridDesc> partner;   // matching grid on the other level (or empty)
    std::vector<int> starts;         // tile starts, size ngrids + 1
    size_t d_grids = 0, d_partner = 0, d_starts = 0;  // workspace offsets
    WorkList wl{};                   // device view, filled at bind
    const GridDesc* partner_dev = nullptr;
    int per_sm = 8;                  // resident CTAs per SM of the kernels using it
};

struct Level {
    int ngrids = 0;
    std::vector<GridDesc> grids;     // grids of images that own this level
    std::vector<int> image;          // image index per grid
    int64_t vec_elems = 0;           // elements of one level vector
    int64_t plane_elems = 0;         // elements of the level's planes
    // device offsets (levels >= 1 only, level 0 uses the solver vectors)
    size_t b64 = 0, x64 = 0, xa64 = 0, xb64 = 0, P64 = 0;
    size_t b32 = 0, x32 = 0, xa32 = 0, xb32 = 0, P32 = 0;
    HostList fine;    // 64x8 tiles of level-l grids that have a level l+1
    HostList coarse;  // restriction tiles of the level l+1 grids of the same images
    HostList flat;    // element chunks of the same level-l grids
    HostList gal;     // 8x16 tiles of every level-(l+1) grid (Galerkin setup), tails included
};

struct Stencil {
    int nimg = 0;
    std::vector<int> h, w;
    int precision = 0;   // 0: FP64, 1: FP32 inner + FP64 refinement
    int precond = 0;     // kPrecNone / kPrecJacobi / kPrecVcycle
    // Launch shapes (pmb_stencil_tune): vector width of the CG apply and of
    // the prolongation, resident CTAs per SM of each list family (limit:
    // shared memory), CG iterations per graph replay.
    int vec_apply = 2, vec_up = 2, chunk = 4;
    int max_fine = 1, max_up = 1, max_down = 1;
    int pre = 1, post = 1;
    // Buffers of the CG apply, restriction and prolongation kernels: 1 (the
    // default: half the shared memory, twice the CTAs per SM, measured 14-20 %
    // faster per solve than 2 on the 64-image batch) or 2 (a tile in flight
    // per CTA while another is computed).
    int stages = 1;
    double omega = 0.8;
    int direct = 64;
    int cy = 3;                      // restriction tile height (inner precision)
    std::vector<int> coarsest;      // per image: index of the level solved directly
    std::vector<Level> levels;      // level 0 .. L
    HostList fine0;                 // 64x8 tiles of every image's level-0 grid
    HostList flat0;                 // element chunks of every level-0 grid
    std::vector<int64_t> user_off;  // offset of image k in user vectors
    int64_t user_total = 0;
    int nmaps = 0;                  // grids with a TMA descriptor block
    std::vector<DirectDesc> direct64, direct32;
    // Coarse-level tail: image k runs levels tail_start[k] .. coarsest[k] in
    // k_vc_tail (-1: no tail): the deepest levels whose planes and vectors fit
    // in kTailSmem bytes of shared memory together.
    std::vector<int> tail_start;
    size_t tail_smem = 0;
    std::vector<int> tail_images;   // images with a tail, in descriptor order
    size_t o_tail = 0;
    std::vector<int64_t> direct_inv_off;   // per direct desc: inverse offset (doubles)
    int64_t direct_doubles = 0;
    // workspace offsets
    size_t ws_bytes = 0;
    size_t o_state = 0, o_outer = 0, o_part = 0, o_uoff = 0, o_direct64 = 0, o_direct32 = 0;
    size_t o_inv = 0, o_invwork = 0, o_status = 0, o_err = 0, o_maps = 0;
    size_t o_b64 = 0, o_x64 = 0, o_r64 = 0, o_z64 = 0, o_p064 = 0, o_p164 = 0, o_ap64 = 0, o_dr64 = 0;
    size_t o_P032 = 0;
    size_t o_r32 = 0, o_z32 = 0, o_p032 = 0, o_p132 = 0, o_ap32 = 0, o_dr32 = 0, o_xin32 = 0;
    int64_t partials_count = 0;
    // bound state
    char* ws = nullptr;
    const double* P0 = nullptr;     // caller-owned level-0 FP64 planes
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    InstState* h_state = nullptr;   // pinned copy of the per-image state
    InstState* h_outer = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    int graph_reorth = -1;
    double graph_delta = -1.0;
    int graph_max_outer = -1;
    double delta = 1e-4;            // mixed: FP32 phase reduction before a residual replacement
    int max_outer = 50;             // mixed: most residual replacements
    int64_t graph_kernels = 0;      // kernel nodes of one graph replay
    bool bound = false, setup_done = false;
    // last solve
    int64_t launches = 0;
    // Kernel profile (pmb_stencil_profile): when set, every launch of an
    // iteration is followed by an event tagged with the launch's kind.
    std::vector<std::pair<int, cudaEvent_t>>* prof = nullptr;

    template <typename T> T* at(size_t off) const { return reinterpret_cast<T*>(ws + off); }
    InstState* state() const { return at<InstState>(o_state); }
    InstState* outer() const { return at<InstState>(o_outer); }
    double* partials() const { return at<double>(o_part); }
    int* err() const { return at<int>(o_err); }
    const CUtensorMap* maps() const { return at<CUtensorMap>(o_maps); }
};

// Resident CTAs per SM of a tile kernel using `smem` bytes of dynamic shared
// memory (plus about 6 KB of static shared memory and the per-CTA reserve).
static int blocks_per_sm(size_t smem) {
    const size_t usable = 227 * 1024;
    int b = (int)(usable / (smem + 7 * 1024));
    return std::max(1, std::min(4, b));
}

constexpr int kMaxCtasPerSm = 16;   // bound of every list's per_sm (tile kernels: 4)

// Grid of a launch over list L by a kernel whose CTAs use `smem` bytes of
// dynamic shared memory (its own residency, not the list's).
static int grid_for(const HostList& L, size_t smem) {
    return std::max(1, std::min(L.wl.total, 148 * blocks_per_sm(smem)));
}

static int persistent_grid(const HostList& L) {
    return std::max(1, std::min(L.wl.total, 148 * std::min(L.per_sm, kMaxCtasPerSm)));
}

static void build_list(HostList& L, const std::vector<GridDesc>& grids,
                       const std::vector<GridDesc>& partner, int th, int tw) {
    L.grids = grids;
    L.partner = partner;
    L.starts.assign(grids.size() + 1, 0);
    for (size_t g = 0; g < grids.size(); ++g)
        L.starts[g + 1] = L.starts[g] + tiles_of(grids[g].h, grids[g].w, th, tw);
}

static void build_flat(HostList& L, const std::vector<GridDesc>& grids) {
    L.grids = grids;
    L.partner.clear();
    L.starts.assign(grids.size() + 1, 0);
    for (size_t g = 0; g < grids.size(); ++g) {
        const int64_t n = (int64_t)grids[g].h * grids[g].pitch;
        L.starts[g + 1] = L.starts[g] + (int)((n + kFlat - 1) / kFlat);
    }
}

static void carve_list(Carve& c, HostList& L) {
    L.d_grids = c.take<GridDesc>((int64_t)L.grids.size());
    L.d_partner = c.take<GridDesc>((int64_t)L.partner.size());
    L.d_starts = c.take<int>((int64_t)L.starts.size());
}

static int plan_stencil(Stencil& S) {
    const int n = S.nimg;
    const bool mixed = S.precision == 1;
    S.cy = mixed ? Coarse<float>::CY : Coarse<double>::CY;
    S.coarsest.assign(n, 0);
    // Level shapes per image: h // 2^l, w // 2^l until h*w <= direct size
    // (vcycle.py:59, :83-86). With no V-cycle only level 0 exists.
    std::vector<std::vector<std::pair<int, int>>> shapes(n);
    int L = 0;
    for (int k = 0; k < n; ++k) {
        int hh = S.h[k], ww = S.w[k];
        shapes[k].push_back({hh, ww});
        if (S.precond == kPrecVcycle) {
            while ((int64_t)hh * ww > S.direct) {
                hh /= 2;
                ww /= 2;
                shapes[k].push_back({hh, ww});
            }
            S.coarsest[k] = (int)shapes[k].size() - 1;
            const int64_t nc = (int64_t)hh * ww;
            if (nc > kMaxDirect) return fail(kErrArg, "coarsest grid larger than the dense solve limit");
        }
        L = std::max(L, (int)shapes[k].size());
    }
    // Tails: only the default cycle (one pre- and one post-sweep) has one.
    S.tail_start.assign(n, -1);
    S.tail_images.clear();
    S.tail_smem = 0;
    if (S.precond == kPrecVcycle && S.pre == 1 && S.post == 1) {
        const size_t es = S.precision == 1 ? sizeof(float) : sizeof(double);
        for (int k = 0; k < n; ++k) {
            size_t bytes = 0;
            int start = -1;
            for (int l = S.coarsest[k]; l >= 1 && S.coarsest[k] - l + 1 <= kMaxTailLevels; --l) {
                const size_t add = (size_t)(kNH + 3) * shapes[k][l].first *
                                   pitch_for(std::max(shapes[k][l].second, 1)) * es;
                if (bytes + add > kTailSmem) break;
                bytes += add;
                start = l;
            }
            if (start >= 1) {
                S.tail_start[k] = start;
                S.tail_images.push_back(k);
                S.tail_smem = std::max(S.tail_smem, bytes);
            }
        }
    }
    S.levels.assign(L, Level());
    S.user_off.assign(n + 1, 0);
    for (int k = 0; k < n; ++k) S.user_off[k + 1] = S.user_off[k] + (int64_t)S.h[k] * S.w[k];
    S.user_total = S.user_off[n];
    int map_base = 0;
    for (int l = 0; l < L; ++l) {
        Level& lv = S.levels[l];
        int64_t voff = 0, poff = 0;
        for (int k = 0; k < n; ++k) {
            if ((int)shapes[k].size() <= l) continue;
            GridDesc g{};
            g.h = shapes[k][l].first;
            g.w = shapes[k][l].second;
            g.pitch = pitch_for(std::max(g.w, 1));
            g.inst = k;
            g.voff = voff;
            g.poff = poff;
            g.pstride = (int64_t)g.h * g.pitch;
            g.map_base = map_base++;
            voff += (int64_t)g.h * g.pitch;
            poff += (int64_t)kNH * g.h * g.pitch;
            lv.grids.push_back(g);
            lv.image.push_back(k);
        }
        lv.ngrids = (int)lv.grids.size();
        lv.vec_elems = voff;
        lv.plane_elems = poff;
    }
    S.nmaps = map_base;
    // Work lists and the residency of the kernels that walk them.
    const bool vec_up = S.pre == 1 && S.post == 1, vec_down = S.pre == 1;
    const int per_fine = mixed ? resident_cg_apply<float>(S.vec_apply, S.stages)
                               : resident_cg_apply<double>(S.vec_apply, S.stages);
    const int per_up =
        vec_up ? (mixed ? resident_up<float>(S.vec_up, S.stages)
                        : resident_up<double>(S.vec_up, S.stages))
               : blocks_per_sm(mixed ? smem_up<float>(S.pre) : smem_up<double>(S.pre));
    const int per_down =
        vec_down ? (mixed ? resident_down<float>(S.stages) : resident_down<double>(S.stages))
                 : blocks_per_sm(mixed ? smem_down<float>(S.pre) : smem_down<double>(S.pre));
    S.max_fine = per_fine;
    S.max_up = per_up;
    S.max_down = per_down;
    build_list(S.fine0, S.levels[0].grids, {}, kTY, kTX);
    S.fine0.per_sm = per_fine;
    build_flat(S.flat0, S.levels[0].grids);
    S.flat0.per_sm = 8;
    for (int l = 0; l + 1 < L; ++l) {
        Level& lv = S.levels[l];
        Level& nx = S.levels[l + 1];
        std::vector<GridDesc> f, c, gf, gc;
        for (int gi = 0; gi < lv.ngrids; ++gi) {
            const int k = lv.image[gi];
            if (S.coarsest[k] <= l) continue;
            const auto it = std::find(nx.image.begin(), nx.image.end(), k);
            gf.push_back(lv.grids[gi]);
            gc.push_back(nx.grids[it - nx.image.begin()]);
            if (S.tail_start[k] >= 0 && l >= S.tail_start[k]) continue;   // in the tail
            f.push_back(lv.grids[gi]);
            c.push_back(nx.grids[it - nx.image.begin()]);
        }
        build_list(lv.gal, gc, gf, kGalerkinTileY, kGalerkinTileX);   // coarse tiles
        build_list(lv.fine, f, c, kTY, kTX);
        lv.fine.per_sm = per_up;
        build_list(lv.coarse, c, f, S.cy, kCX);
        lv.coarse.per_sm = per_down;
        build_flat(lv.flat, f);
        lv.flat.per_sm = 8;
    }
    // Dense coarsest solves.
    S.direct64.clear();
    S.direct_inv_off.clear();
    S.direct_doubles = 0;
    if (S.precond == kPrecVcycle) {
        for (int k = 0; k < n; ++k) {
            const int l = S.coarsest[k];
            const Level& lv = S.levels[l];
            const auto it = std::find(lv.image.begin(), lv.image.end(), k);
            DirectDesc d{};
            d.g = lv.grids[it - lv.image.begin()];
            const int64_t nn = (int64_t)d.g.h * d.g.w;
            S.direct_inv_off.push_back(S.direct_doubles);
            d.work_off = S.direct_doubles;
            S.direct_doubles += nn * nn;
            S.direct64.push_back(d);
        }
    }
    // Workspace layout.
    Carve c;
    const int64_t v0 = S.levels[0].vec_elems;
    S.o_state = c.take<InstState>(n);
    S.o_outer = c.take<InstState>(n);
    int64_t maxt = std::max(S.fine0.starts.back(), S.flat0.starts.back());
    for (auto& lv : S.levels) {
        if (!lv.fine.starts.empty()) maxt = std::max<int64_t>(maxt, lv.fine.starts.back());
        if (!lv.flat.starts.empty()) maxt = std::max<int64_t>(maxt, lv.flat.starts.back());
    }
    // Per-CTA partial sums: partials[(image * 3 + q) * G + cta] for the
    // largest persistent grid G of any list (148 SMs x kMaxCtasPerSm, the
    // largest CTAs-per-SM value any list can be given).
    const int64_t gmax = std::min<int64_t>(maxt, 148 * kMaxCtasPerSm);
    S.partials_count = std::max<int64_t>(maxt, (int64_t)n * gmax);
    S.o_part = c.take<double>(3 * S.partials_count);
    S.o_uoff = c.take<int64_t>(n + 1);
    S.o_status = c.take<int>(4);
    S.o_err = c.take<int>(4);
    S.o_maps = c.take<CUtensorMap>((int64_t)S.nmaps * kMapsPerGrid);
    carve_list(c, S.fine0);
    carve_list(c, S.flat0);
    for (auto& lv : S.levels) {
        carve_list(c, lv.fine);
        carve_list(c, lv.coarse);
        carve_list(c, lv.flat);
        carve_list(c, lv.gal);
    }
    S.o_tail = c.take<TailDesc<double>>((int64_t)S.tail_images.size());
    S.o_direct64 = c.take<DirectDesc>((int64_t)S.direct64.size());
    S.o_direct32 = c.take<DirectDesc>((int64_t)S.direct64.size());
    S.o_inv = c.take<double>(S.direct_doubles);
    S.o_invwork = c.take<double>(S.direct_doubles);
    // Level-0 vectors. FP64 always holds b and x (the refinement iterate in
    // mixed mode); the CG vectors take the inner precision.
    S.o_b64 = c.take<double>(v0);
    S.o_x64 = c.take<double>(v0);
    if (!mixed) {
        S.o_r64 = c.take<double>(v0);
        S.o_z64 = c.take<double>(v0);
        S.o_p064 = c.take<double>(v0);
        S.o_p164 = c.take<double>(v0);
        S.o_ap64 = c.take<double>(v0);
        S.o_dr64 = c.take<double>(v0);
    } else {
        S.o_P032 = c.take<float>((int64_t)kNH * v0);
        S.o_r32 = c.take<float>(v0);
        S.o_z32 = c.take<float>(v0);
        S.o_p032 = c.take<float>(v0);
        S.o_p132 = c.take<float>(v0);
        S.o_ap32 = c.take<float>(v0);
        S.o_dr32 = c.take<float>(v0);
        S.o_xin32 = c.take<float>(v0);
    }
    for (int l = 0; l < L; ++l) {
        Level& lv = S.levels[l];
        if (l >= 1) {
            lv.P64 = c.take<double>(lv.plane_elems);
            if (!mixed) {
                lv.b64 = c.take<double>(lv.vec_elems);
                lv.x64 = c.take<double>(lv.vec_elems);
            } else {
                lv.P32 = c.take<float>(lv.plane_elems);
                lv.b32 = c.take<float>(lv.vec_elems);
                lv.x32 = c.take<float>(lv.vec_elems);
            }
        }
        // Ping-pong buffers for extra smoothing sweeps.
        if (S.precond == kPrecVcycle && (S.pre > 1 || S.post > 1)) {
            if (!mixed) {
                lv.xa64 = c.take<double>(lv.vec_elems);
                lv.xb64 = c.take<double>(lv.vec_elems);
            } else {
                lv.xa32 = c.take<float>(lv.vec_elems);
                lv.xb32 = c.take<float>(lv.vec_elems);
            }
        }
    }
    S.ws_bytes = c.off + 256;
    return 0;
}

static void list_view(Stencil& S, HostList& L) {
    L.wl.grids = S.at<GridDesc>(L.d_grids);
    L.wl.tile_start = S.at<int>(L.d_starts);
    L.wl.ngrids = (int)L.grids.size();
    L.wl.total = L.starts.empty() ? 0 : L.starts.back();
    L.partner_dev = S.at<GridDesc>(L.d_partner);
}

static int upload_list(Stencil& S, HostList& L) {
    if (!L.grids.empty())
        PMB_CUDA(cudaMemcpyAsync(S.ws + L.d_grids, L.grids.data(), sizeof(GridDesc) * L.grids.size(),
                                 cudaMemcpyHostToDevice, S.stream));
    if (!L.partner.empty())
        PMB_CUDA(cudaMemcpyAsync(S.ws + L.d_partner, L.partner.data(),
                                 sizeof(GridDesc) * L.partner.size(), cudaMemcpyHostToDevice, S.stream));
    PMB_CUDA(cudaMemcpyAsync(S.ws + L.d_starts, L.starts.data(), sizeof(int) * L.starts.size(),
                             cudaMemcpyHostToDevice, S.stream));
    list_view(S, L);
    return 0;
}

// Run `fn` on the solver's own stream, ordered after everything already
// queued on the caller's stream and before anything queued there later.
template <typename Fn>
static int on_stream(Stencil& S, cudaStream_t caller, Fn fn) {
    PMB_CUDA(cudaEventRecord(S.ev_in, caller));
    PMB_CUDA(cudaStreamWaitEvent(S.stream, S.ev_in, 0));
    int rc = fn();
    PMB_CUDA(cudaEventRecord(S.ev_out, S.stream));
    PMB_CUDA(cudaStreamWaitEvent(caller, S.ev_out, 0));
    return rc;
}

// Plane base pointer of level l (FP64 / FP32).
static const double* planes64(const Stencil& S, int l) {
    return l == 0 ? S.P0 : S.at<double>(S.levels[l].P64);
}
static const float* planes32(const Stencil& S, int l) {
    return l == 0 ? S.at<float>(S.o_P032) : S.at<float>(S.levels[l].P32);
}

// Encode one tiled TMA descriptor of a pitched 2D vector or of the 13-plane
// 3D operator block of grid g.
static int encode_map(CUtensorMap* out, const void* base, const GridDesc& g, bool planes,
                      bool fp32, int box_w, int box_h, int box_d = kNH) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return fail(kErrCuda, "cuTensorMapEncodeTiled is not available");
    const size_t es = fp32 ? 4 : 8;
    const CUtensorMapDataType dt = fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    cuuint64_t dims[3] = {(cuuint64_t)g.w, (cuuint64_t)g.h, (cuuint64_t)kNH};
    cuuint64_t strides[2] = {(cuuint64_t)g.pitch * es, (cuuint64_t)g.pitch * g.h * es};
    cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, (cuuint32_t)box_d};
    cuuint32_t estr[3] = {1, 1, 1};
    const char* ptr = static_cast<const char*>(base) + (planes ? g.poff : g.voff) * es;
    CUresult r = enc(out, dt, planes ? 3 : 2, const_cast<char*>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(kErrCuda, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return 0;
}

// Fill every grid's descriptor block. Slots that a configuration never
// reads are left zero.
// Descriptors of one grid of level l (the block at g.map_base).
static int encode_grid_maps(Stencil& S, int l, const GridDesc& g, CUtensorMap* m) {
    const bool mixed = S.precision == 1;
    const int DH = 2 * S.cy + 5;
    const int DWV = mixed ? down_box_width<float>() : down_box_width<double>();
    Level& lv = S.levels[l];
    const void* P = mixed ? (const void*)planes32(S, l) : (const void*)planes64(S, l);
    const void* B; const void* X; const void* XA = nullptr; const void* XB = nullptr;
    if (l == 0) {
        B = mixed ? (const void*)S.at<float>(S.o_r32) : (const void*)S.at<double>(S.o_r64);
        X = mixed ? (const void*)S.at<float>(S.o_z32) : (const void*)S.at<double>(S.o_z64);
    } else {
        B = mixed ? (const void*)S.at<float>(lv.b32) : (const void*)S.at<double>(lv.b64);
        X = mixed ? (const void*)S.at<float>(lv.x32) : (const void*)S.at<double>(lv.x64);
    }
    if (S.precond == kPrecVcycle && (S.pre > 1 || S.post > 1)) {
        XA = mixed ? (const void*)S.at<float>(lv.xa32) : (const void*)S.at<double>(lv.xa64);
        XB = mixed ? (const void*)S.at<float>(lv.xb32) : (const void*)S.at<double>(lv.xb64);
    }
    int rc = 0;
    rc |= encode_map(m + kMapPlF, P, g, true, mixed, kBW, kBH);
    rc |= encode_map(m + kMapPlD, P, g, true, mixed, kBW, DH);
    rc |= encode_map(m + kMapBF, B, g, false, mixed, kBW, kBH);
    rc |= encode_map(m + kMapBD, B, g, false, mixed, kBW, DH);
    rc |= encode_map(m + kMapXC, X, g, false, mixed, kCBW, kCBH);
    rc |= encode_map(m + kMapXF, X, g, false, mixed, kBW, kBH);
    rc |= encode_map(m + kMapPlS, P, g, true, mixed, kBW, kPH);
    rc |= encode_map(m + kMapPlDV, P, g, true, mixed, DWV, DH);
    rc |= encode_map(m + kMapBDV, B, g, false, mixed, DWV, DH);
    rc |= encode_map(m + kMapPlG, planes64(S, l), g, true, false, kGCols, kGRows);
    rc |= encode_map(m + kMapPlD0, P, g, true, mixed, DWV, DH, 1);
    rc |= encode_map(m + kMapPlD1, P, g, true, mixed, DWV, DH - 2, kNH - 1);
    rc |= encode_map(m + kMapPlU0, P, g, true, mixed, kBW, kBH, 1);
    rc |= encode_map(m + kMapPlU1, P, g, true, mixed, kBW, kPH, kNH - 1);
    if (XA) {
        rc |= encode_map(m + kMapXAF, XA, g, false, mixed, kBW, kBH);
        rc |= encode_map(m + kMapXAD, XA, g, false, mixed, kBW, DH);
        rc |= encode_map(m + kMapXBF, XB, g, false, mixed, kBW, kBH);
        rc |= encode_map(m + kMapXBD, XB, g, false, mixed, kBW, DH);
    }
    if (l == 0) {
        const void* Z = X;
        const void* Q0 = mixed ? (const void*)S.at<float>(S.o_p032) : (const void*)S.at<double>(S.o_p064);
        const void* Q1 = mixed ? (const void*)S.at<float>(S.o_p132) : (const void*)S.at<double>(S.o_p164);
        rc |= encode_map(m + kMapZF, Z, g, false, mixed, kBW, kBH);
        rc |= encode_map(m + kMapP0F, Q0, g, false, mixed, kBW, kBH);
        rc |= encode_map(m + kMapP1F, Q1, g, false, mixed, kBW, kBH);
        if (mixed) {
            rc |= encode_map(m + kMapX64F, S.at<double>(S.o_x64), g, false, false, kBW, kBH);
            rc |= encode_map(m + kMapP64F, S.P0, g, true, false, kBW, kBH);
        }
    }
    return rc;
}

// Fill every grid's descriptor block (host work: thousands of descriptors
// for a large batch), spread over up to 8 host threads. Slots that a
// configuration never reads are left zero.
static int encode_maps(Stencil& S, std::vector<CUtensorMap>& maps) {
    maps.assign((size_t)S.nmaps * kMapsPerGrid, CUtensorMap{});
    if (!encode_fn()) return fail(kErrCuda, "cuTensorMapEncodeTiled is not available");
    std::vector<std::pair<int, GridDesc>> work;
    for (int l = 0; l < (int)S.levels.size(); ++l)
        for (const GridDesc& g : S.levels[l].grids)
            if (g.w > 0 && g.h > 0) work.push_back({l, g});
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<size_t>({(size_t)8, (size_t)hw, (work.size() + 63) / 64});
    std::atomic<int> bad{0};
    int device = 0;
    PMB_CUDA(cudaGetDevice(&device));
    auto run = [&](int k) {
        // The encoder needs the caller's context current in this thread.
        if (k > 0 && cudaSetDevice(device) != cudaSuccess) {
            bad.store(1);
            return;
        }
        for (size_t q = (size_t)k; q < work.size(); q += (size_t)std::max(nt, 1)) {
            const GridDesc& g = work[q].second;
            if (encode_grid_maps(S, work[q].first, g, &maps[(size_t)g.map_base * kMapsPerGrid]))
                bad.store(1);
        }
    };
    // Share 0 on the calling thread (its context is current), the others on
    // helper threads.
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(run, k);
    run(0);
    for (auto& t : th) t.join();
    if (bad.load()) return fail(kErrCuda, "cuTensorMapEncodeTiled failed");
    return 0;
}

static int upload_tail(Stencil& S);

static int bind_stencil(Stencil& S, void* ws, const double* P0) {
    S.ws = reinterpret_cast<char*>(ws);
    S.P0 = P0;
    stencil_prepare();
    if (int rc = upload_list(S, S.fine0)) return rc;
    if (int rc = upload_list(S, S.flat0)) return rc;
    for (auto& lv : S.levels) {
        if (int rc = upload_list(S, lv.fine)) return rc;
        if (int rc = upload_list(S, lv.coarse)) return rc;
        if (int rc = upload_list(S, lv.flat)) return rc;
        if (int rc = upload_list(S, lv.gal)) return rc;
    }
    PMB_CUDA(cudaMemcpyAsync(S.ws + S.o_uoff, S.user_off.data(), sizeof(int64_t) * S.user_off.size(),
                             cudaMemcpyHostToDevice, S.stream));
    std::vector<CUtensorMap> maps;
    if (int rc = encode_maps(S, maps)) return rc;
    if (!maps.empty())
        PMB_CUDA(cudaMemcpyAsync(S.ws + S.o_maps, maps.data(), sizeof(CUtensorMap) * maps.size(),
                                 cudaMemcpyHostToDevice, S.stream));
    // Direct descriptors: the inverse pointers are absolute.
    S.direct32 = S.direct64;
    for (size_t i = 0; i < S.direct64.size(); ++i) {
        S.direct64[i].inv = S.at<double>(S.o_inv) + S.direct_inv_off[i];
        S.direct64[i].P = planes64(S, S.coarsest[S.direct64[i].g.inst]);
        S.direct32[i].inv = S.direct64[i].inv;
        S.direct32[i].P = S.direct64[i].P;
    }
    if (!S.direct64.empty()) {
        PMB_CUDA(cudaMemcpyAsync(S.ws + S.o_direct64, S.direct64.data(),
                                 sizeof(DirectDesc) * S.direct64.size(), cudaMemcpyHostToDevice, S.stream));
        PMB_CUDA(cudaMemcpyAsync(S.ws + S.o_direct32, S.direct32.data(),
                                 sizeof(DirectDesc) * S.direct32.size(), cudaMemcpyHostToDevice, S.stream));
    }
    if (int rc = upload_tail(S)) return rc;
    PMB_CUDA(cudaMemsetAsync(S.ws + S.o_state, 0, sizeof(InstState) * S.nimg, S.stream));
    PMB_CUDA(cudaMemsetAsync(S.ws + S.o_outer, 0, sizeof(InstState) * S.nimg, S.stream));
    PMB_CUDA(cudaMemsetAsync(S.ws + S.o_err, 0, sizeof(int) * 4, S.stream));
    PMB_CUDA(cudaStreamSynchronize(S.stream));
    if (S.graph) {
        cudaGraphExecDestroy(S.graph);
        S.graph = nullptr;
    }
    S.bound = true;
    S.setup_done = false;
    return 0;
}

static int check_err(Stencil& S) {
    int e = 0;
    PMB_CUDA(cudaMemcpyAsync(&e, S.err(), sizeof(int), cudaMemcpyDeviceToHost, S.stream));
    PMB_CUDA(cudaStreamSynchronize(S.stream));
    if (e) return fail(kErrState, "a TMA transfer did not complete in time");
    return 0;
}

static int setup_stencil(Stencil& S) {
    cudaStream_t s = S.stream;
    const int L = (int)S.levels.size();
    for (int l = 0; l + 1 < L; ++l) {
        Level& lv = S.levels[l];
        HostList& f = lv.gal;
        if (f.grids.empty()) continue;
        launch_galerkin_t(f.wl, f.partner_dev, S.maps(), S.at<double>(S.levels[l + 1].P64),
                          S.err(), s);
        ++S.launches;
    }
    PMB_CUDA(cudaMemsetAsync(S.ws + S.o_status, 0, sizeof(int), s));
    if (!S.direct64.empty()) {
        launch_dense_inverse(S.at<DirectDesc>(S.o_direct64), (int)S.direct64.size(),
                             S.at<double>(S.o_invwork), S.at<int>(S.o_status), s);
        ++S.launches;
    }
    if (S.precision == 1) {
        launch_convert_f32(S.P0, S.at<float>(S.o_P032), (int64_t)kNH * S.levels[0].vec_elems, s);
        for (int l = 1; l < L; ++l)
            launch_convert_f32(S.at<double>(S.levels[l].P64), S.at<float>(S.levels[l].P32),
                               S.levels[l].plane_elems, s);
    }
    PMB_CUDA(cudaGetLastError());
    int status = 0;
    PMB_CUDA(cudaMemcpyAsync(&status, S.ws + S.o_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    // A non-finite operator (non-finite image data) is not fatal here: the
    // solve stops that image alone with status kNonFinite.
    if (status == 2) return fail(kErrState, "coarsest multigrid operator is singular");
    S.setup_done = true;
    return 0;
}

// Pointers of the inner-precision CG vectors at level 0.
template <typename T>
struct CgVecs {
    T *x, *r, *z, *p0, *p1, *ap, *dr;
    const T* P;
};

template <typename T> static CgVecs<T> cg_vecs(Stencil& S);
template <> CgVecs<double> cg_vecs<double>(Stencil& S) {
    return {S.at<double>(S.o_x64), S.at<double>(S.o_r64), S.at<double>(S.o_z64),
            S.at<double>(S.o_p064), S.at<double>(S.o_p164), S.at<double>(S.o_ap64),
            S.at<double>(S.o_dr64), S.P0};
}
template <> CgVecs<float> cg_vecs<float>(Stencil& S) {
    return {S.at<float>(S.o_xin32), S.at<float>(S.o_r32), S.at<float>(S.o_z32),
            S.at<float>(S.o_p032), S.at<float>(S.o_p132), S.at<float>(S.o_ap32),
            S.at<float>(S.o_dr32), S.at<float>(S.o_P032)};
}

template <typename T> static T* lvl_b(Stencil& S, int l);
template <typename T> static T* lvl_x(Stencil& S, int l);
template <typename T> static T* lvl_xa(Stencil& S, int l);
template <typename T> static T* lvl_xb(Stencil& S, int l);
template <typename T> static const T* lvl_P(Stencil& S, int l);
template <> double* lvl_b<double>(Stencil& S, int l) { return S.at<double>(S.levels[l].b64); }
template <> double* lvl_x<double>(Stencil& S, int l) { return S.at<double>(S.levels[l].x64); }
template <> double* lvl_xa<double>(Stencil& S, int l) { return S.at<double>(S.levels[l].xa64); }
template <> double* lvl_xb<double>(Stencil& S, int l) { return S.at<double>(S.levels[l].xb64); }
template <> const double* lvl_P<double>(Stencil& S, int l) { return planes64(S, l); }
template <> float* lvl_b<float>(Stencil& S, int l) { return S.at<float>(S.levels[l].b32); }
template <> float* lvl_x<float>(Stencil& S, int l) { return S.at<float>(S.levels[l].x32); }
template <> float* lvl_xa<float>(Stencil& S, int l) { return S.at<float>(S.levels[l].xa32); }
template <> float* lvl_xb<float>(Stencil& S, int l) { return S.at<float>(S.levels[l].xb32); }
template <> const float* lvl_P<float>(Stencil& S, int l) { return planes32(S, l); }

// Tail descriptors with absolute pointers (after the direct inverses are placed).
template <typename T>
static int upload_tail_t(Stencil& S) {
    std::vector<TailDesc<T>> d(S.tail_images.size());
    for (size_t j = 0; j < S.tail_images.size(); ++j) {
        const int k = S.tail_images[j];
        TailDesc<T>& t = d[j];
        std::memset(&t, 0, sizeof(t));
        t.inst = k;
        t.nlev = S.coarsest[k] - S.tail_start[k] + 1;
        for (int q = 0; q < t.nlev; ++q) {
            const int l = S.tail_start[k] + q;
            const Level& lv = S.levels[l];
            const auto it = std::find(lv.image.begin(), lv.image.end(), k);
            t.lev[q].g = lv.grids[it - lv.image.begin()];
            t.lev[q].P = lvl_P<T>(S, l);
            t.lev[q].b = lvl_b<T>(S, l);
            t.lev[q].x = lvl_x<T>(S, l);
        }
        t.inv = S.direct64[k].inv;
    }
    if (!d.empty())
        PMB_CUDA(cudaMemcpyAsync(S.ws + S.o_tail, d.data(), sizeof(TailDesc<T>) * d.size(),
                                 cudaMemcpyHostToDevice, S.stream));
    return 0;
}

static int upload_tail(Stencil& S) {
    if (S.tail_images.empty()) return 0;
    return S.precision == 1 ? upload_tail_t<float>(S) : upload_tail_t<double>(S);
}

template <typename T> static const DirectDesc* direct_dev(Stencil& S);
template <> const DirectDesc* direct_dev<double>(Stencil& S) { return S.at<DirectDesc>(S.o_direct64); }
template <> const DirectDesc* direct_dev<float>(Stencil& S) { return S.at<DirectDesc>(S.o_direct32); }

// Kinds of launches told apart by pmb_stencil_profile (index into its output).
enum : int {
    kPkApply = 0,   // CG apply p = z + beta p, Ap, p.Ap
    kPkUpdate,      // CG vector update x, r, |r|
    kPkRefine,      // mixed: FP64 correction and residual replacement
    kPkDown0,       // V-cycle restriction from level 0
    kPkDown,        // restriction from levels >= 1
    kPkTail,        // shared-memory tail of the small levels
    kPkDirect,      // dense coarsest solves outside a tail
    kPkUp,          // prolongation + post sweep at levels >= 1
    kPkUp0,         // prolongation + post sweep at level 0 (z, r.z, beta)
    kPkOther,       // extra smoothing sweeps, separate r.z
    kPkCount
};

static void prof_mark(Stencil& S, int kind) {
    if (!S.prof) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, S.stream);
    S.prof->push_back({kind, e});
}

// V-cycle z = M r (vcycle.py:46-100) at level 0 with r = b0 (the level-0 b
// buffer) and z = z0 (the level-0 x buffer). With st != null the level-0
// pass also reduces r . z and finishes beta.
template <typename T>
static void run_vcycle(Stencil& S, const T* b0, T* z0, InstState* st, const T* dr, int reorth) {
    cudaStream_t s = S.stream;
    const int L = (int)S.levels.size();
    const double om = S.omega;
    const int pre = S.pre, post = S.post;
    auto B = [&](int l) -> T* { return l == 0 ? const_cast<T*>(b0) : lvl_b<T>(S, l); };
    auto X = [&](int l) -> T* { return l == 0 ? z0 : lvl_x<T>(S, l); };
    // Map slot of each level's pre-smoothed iterate (pre > 1).
    std::vector<int> xs_slot_f(L, -1), xs_slot_d(L, -1);
    for (int l = 0; l + 1 < L; ++l) {
        HostList& f = S.levels[l].fine;
        HostList& c = S.levels[l].coarse;
        if (f.wl.total == 0) continue;
        if (pre > 1) {
            // Sweeps alternate A / B; the first writes A (from zero).
            T* a = lvl_xa<T>(S, l);
            T* bb = lvl_xb<T>(S, l);
            launch_vc_smooth<T>(LaunchCfg{persistent_grid(f)}, f.wl, S.maps(), -1, lvl_P<T>(S, l),
                                B(l), a, om, st, S.err(), s);
            ++S.launches;
            prof_mark(S, kPkOther);
            bool in_a = true;
            for (int k = 1; k < pre; ++k) {
                launch_vc_smooth<T>(LaunchCfg{persistent_grid(f)}, f.wl, S.maps(),
                                    in_a ? kMapXAF : kMapXBF, lvl_P<T>(S, l), B(l), in_a ? bb : a,
                                    om, st, S.err(), s);
                ++S.launches;
                prof_mark(S, kPkOther);
                in_a = !in_a;
            }
            xs_slot_f[l] = in_a ? kMapXAF : kMapXBF;
            xs_slot_d[l] = in_a ? kMapXAD : kMapXBD;
        }
        launch_vc_down<T>(pre, S.stages, LaunchCfg{persistent_grid(c)}, c.wl, c.partner_dev, S.maps(),
                          xs_slot_d[l], B(l + 1), om, st, S.err(), s);
        ++S.launches;
        prof_mark(S, l == 0 ? kPkDown0 : kPkDown);
    }
    // Small levels of the images that have a tail, in one clustered launch.
    if (!S.tail_images.empty()) {
        launch_vc_tail<T>(S.at<TailDesc<T>>(S.o_tail), (int)S.tail_images.size(), S.tail_smem, st,
                          om, S.err(), s);
        ++S.launches;
        prof_mark(S, kPkTail);
    }
    // Coarsest solves of the other images, whatever their depth.
    for (size_t i = 0; i < S.direct64.size(); ++i) {
        const int k = S.direct64[i].g.inst;
        if (S.tail_start[k] >= 0) continue;
        const int l = S.coarsest[k];
        const bool z_out = (l == 0);
        launch_vc_direct<T>(direct_dev<T>(S) + i, 1, B(l), X(l), st, z_out && st != nullptr, s);
        ++S.launches;
        prof_mark(S, kPkDirect);
    }
    for (int l = L - 2; l >= 0; --l) {
        HostList& f = S.levels[l].fine;
        if (f.wl.total == 0) continue;
        LaunchCfg Lf{persistent_grid(f)};
        const int extra = post > 1 ? post - 1 : 0;
        // Sweeps alternate buffers so that the last one lands in X(l).
        const bool first_in_x = (extra % 2 == 0);
        T* first_out = first_in_x ? X(l) : lvl_xa<T>(S, l);
        const bool reduce_here = (l == 0) && st && extra == 0;
        launch_vc_up<T>(S.vec_up, S.stages, pre, post, Lf, f.wl, f.partner_dev, S.maps(), xs_slot_f[l], B(l),
                        first_out, om, st, reduce_here ? 1 : 0, dr, reorth, S.partials(), S.err(),
                        s);
        ++S.launches;
        prof_mark(S, l == 0 ? kPkUp0 : kPkUp);
        bool cur_x = first_in_x;
        for (int k = 0; k < extra; ++k) {
            T* nxt = cur_x ? lvl_xa<T>(S, l) : X(l);
            launch_vc_smooth<T>(Lf, f.wl, S.maps(), cur_x ? kMapXF : kMapXAF, lvl_P<T>(S, l), B(l),
                                nxt, om, st, S.err(), s);
            ++S.launches;
            prof_mark(S, kPkOther);
            cur_x = !cur_x;
        }
        if (l == 0 && st && extra > 0) {
            // r . z for the images that own coarser levels (the others were
            // reduced by their direct solve).
            launch_cg_rz<T>(LaunchCfg{persistent_grid(S.levels[0].flat)}, S.levels[0].flat.wl, b0,
                            z0, dr, reorth, st, S.partials(), s);
            ++S.launches;
            prof_mark(S, kPkOther);
        }
    }
}

// One preconditioned CG iteration on the inner-precision vectors.
template <typename T>
static void cg_iteration(Stencil& S, int reorth) {
    cudaStream_t s = S.stream;
    CgVecs<T> v = cg_vecs<T>(S);
    InstState* st = S.state();
    // Without a preconditioner z is r itself (cg.py:53-55).
    const int zslot = S.precond == kPrecNone ? kMapBF : kMapZF;
    launch_cg_apply<T>(S.vec_apply, S.stages, LaunchCfg{persistent_grid(S.fine0)}, S.fine0.wl,
                       S.maps(), zslot,
                       v.p0, v.p1, v.ap, st, S.partials(), S.err(), s);
    prof_mark(S, kPkApply);
    const bool mixed = S.precision == 1;
    const int upd_grid = std::min(persistent_grid(S.flat0), 148 * resident_cg_update<T>(S.precond));
    launch_cg_update<T>(S.precond, LaunchCfg{upd_grid}, S.flat0.wl, v.P, v.x, v.r,
                        v.z, v.p0, v.p1, v.ap, v.dr, reorth, mixed ? 1 : 0, S.err() + kPendingSlot, st,
                        S.partials(), s);
    prof_mark(S, kPkUpdate);
    S.launches += 2;
    if (mixed) {
        // Residual replacement for the images whose FP32 phase just ended.
        HostList& a = S.fine0;
        launch_refine_correct(LaunchCfg{persistent_grid(S.flat0)}, S.flat0.wl,
                              S.at<double>(S.o_x64), S.at<float>(S.o_xin32), st,
                              S.err() + kPendingSlot, s);
        launch_refine_residual(S.precond, 0, LaunchCfg{grid_for(a, smem_init<double>())}, a.wl,
                               S.maps(),
                               S.at<float>(S.o_P032), S.at<double>(S.o_b64), S.at<float>(S.o_r32),
                               S.at<float>(S.o_xin32), S.at<float>(S.o_z32), S.outer(), st,
                               S.partials(), 0.0, 0.0, S.delta, 0, S.max_outer, S.err(), s);
        S.launches += 2;
        prof_mark(S, kPkRefine);
    }
    if (S.precond == kPrecVcycle) run_vcycle<T>(S, v.r, v.z, st, v.dr, reorth);
}

static int read_states(Stencil& S, bool outer) {
    PMB_CUDA(cudaMemcpyAsync(S.h_state, S.state(), sizeof(InstState) * S.nimg,
                             cudaMemcpyDeviceToHost, S.stream));
    if (outer)
        PMB_CUDA(cudaMemcpyAsync(S.h_outer, S.outer(), sizeof(InstState) * S.nimg,
                                 cudaMemcpyDeviceToHost, S.stream));
    PMB_CUDA(cudaStreamSynchronize(S.stream));
    return 0;
}

static bool any_running(const InstState* st, int n) {
    for (int k = 0; k < n; ++k)
        if (st[k].status == kRunning) return true;
    return false;
}

// Iterate until every image has left the running state. Iterations are
// replayed from a CUDA graph of `chunk` iterations; images that finish early
// turn the remaining kernels of the chunk into no-ops.
template <typename T>
static int iterate(Stencil& S, int reorth, int maxiter) {
    const int chunk = S.chunk;
    if (!S.graph || S.graph_reorth != reorth || S.graph_iters != chunk ||
        S.graph_delta != S.delta || S.graph_max_outer != S.max_outer) {
        if (S.graph) {
            cudaGraphExecDestroy(S.graph);
            S.graph = nullptr;
        }
        cudaGraph_t g;
        PMB_CUDA(cudaStreamBeginCapture(S.stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < chunk; ++i) cg_iteration<T>(S, reorth);
        PMB_CUDA(cudaStreamEndCapture(S.stream, &g));
        size_t nodes = 0;
        PMB_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
        PMB_CUDA(cudaGraphInstantiate(&S.graph, g, 0));
        cudaGraphDestroy(g);
        S.graph_iters = chunk;
        S.graph_reorth = reorth;
        S.graph_delta = S.delta;
        S.graph_max_outer = S.max_outer;
        S.graph_kernels = (int64_t)nodes;
        // Capture only recorded the launches; they did not run.
        S.launches -= (int64_t)nodes;
    }
    int done_iters = 0;
    for (;;) {
        if (int rc = read_states(S, false)) return rc;
        if (!any_running(S.h_state, S.nimg)) break;
        if (done_iters > maxiter + chunk) return fail(kErrState, "iteration control lost");
        PMB_CUDA(cudaGraphLaunch(S.graph, S.stream));
        S.launches += S.graph_kernels;
        done_iters += chunk;
    }
    return check_err(S);
}

// Initial residual and first preconditioner apply of an FP64 solve.
static void start_fp64(Stencil& S, const double* x0, double atol, double rtol, int maxiter) {
    cudaStream_t s = S.stream;
    CgVecs<double> v = cg_vecs<double>(S);
    HostList& a = S.fine0;
    if (x0)
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), x0, v.p0,
                                    S.user_total, s);
    launch_cg_init<double>(S.precond, LaunchCfg{grid_for(a, smem_init<double>())}, a.wl, S.maps(), v.P,
                           S.at<double>(S.o_b64), v.x, x0 != nullptr, v.r, v.z, S.state(),
                           S.partials(), atol, rtol, maxiter, S.err(), s);
    S.launches += 1;
    if (S.precond == kPrecVcycle) run_vcycle<double>(S, v.r, v.z, S.state(), v.dr, 0);
}

static int solve_fp64(Stencil& S, const double* x0, double atol, double rtol, int maxiter,
                      int reorth) {
    start_fp64(S, x0, atol, rtol, maxiter);
    return iterate<double>(S, reorth, maxiter);
}

// First FP64 residual, outer state and first preconditioner apply of a
// mixed-precision solve.
static int start_mixed(Stencil& S, const double* x0, double atol, double rtol, int maxiter,
                       double inner_rtol, int max_outer) {
    cudaStream_t s = S.stream;
    CgVecs<float> v = cg_vecs<float>(S);
    HostList& a = S.fine0;
    double* x64 = S.at<double>(S.o_x64);
    if (x0)
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), x0, x64,
                                    S.user_total, s);
    else
        PMB_CUDA(cudaMemsetAsync(x64, 0, sizeof(double) * S.levels[0].vec_elems, s));
    S.delta = inner_rtol;
    S.max_outer = max_outer;
    PMB_CUDA(cudaMemsetAsync(S.err() + kPendingSlot, 0, sizeof(int), s));
    // Outer state: every image starts running; its first FP64 residual sets
    // |b|, the tolerance and the first FP32 phase.
    std::vector<InstState> init(S.nimg);
    for (auto& o : init) {
        std::memset(&o, 0, sizeof(o));
        o.status = kRunning;
    }
    PMB_CUDA(cudaMemcpyAsync(S.outer(), init.data(), sizeof(InstState) * S.nimg,
                             cudaMemcpyHostToDevice, s));
    launch_refine_residual(S.precond, 1, LaunchCfg{grid_for(a, smem_init<double>())}, a.wl, S.maps(), v.P,
                           S.at<double>(S.o_b64), v.r, v.x, v.z, S.outer(), S.state(),
                           S.partials(), atol, rtol, inner_rtol, maxiter, max_outer, S.err(), s);
    S.launches += 1;
    if (S.precond == kPrecVcycle) run_vcycle<float>(S, v.r, v.z, S.state(), v.dr, 0);
    return 0;
}

static int solve_mixed(Stencil& S, const double* x0, double atol, double rtol, int maxiter,
                       int reorth, double inner_rtol, int max_outer) {
    CgVecs<float> v = cg_vecs<float>(S);
    double* x64 = S.at<double>(S.o_x64);
    if (int rc = start_mixed(S, x0, atol, rtol, maxiter, inner_rtol, max_outer)) return rc;
    if (int rc = iterate<float>(S, reorth, maxiter)) return rc;
    // Fold the last FP32 correction into x64 (zero for converged images).
    launch_refine_correct(LaunchCfg{persistent_grid(S.flat0)}, S.flat0.wl, x64, v.x, nullptr,
                          S.err() + kPendingSlot, S.stream);
    S.launches += 1;
    if (int rc = read_states(S, true)) return rc;
    return check_err(S);
}

}  // namespace pmb

using namespace pmb;

struct pmb_stencil { Stencil S; };
struct pmb_csr;

// --------------------------------------------------------------------------
// C-ABI
// --------------------------------------------------------------------------

PMB_API const char* pmb_last_error(void) { return g_last_error.c_str(); }

PMB_API int pmb_version(void) { return 1; }

PMB_API int pmb_grid_pitch(int w) { return pitch_for(w); }

PMB_API int pmb_cf_laplacian_ell(const double* image, const uint8_t* is_known, int h, int w,
                                 int radius, double epsilon, const uint8_t* diag_mask,
                                 double diag_value, double* values, int64_t* indices,
                                 int64_t* indptr, void* stream) {
    if (!image || !values || !indices || !indptr || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_cf_laplacian_ell: bad arguments");
    int rc = pmb_launch_cf_ell(image, is_known, h, w, radius, epsilon, diag_mask, diag_value,
                               values, indices, indptr, (cudaStream_t)stream);
    if (rc == -1) return fail(kErrArg, "pmb_cf_laplacian_ell: radius must be 1 or 2");
    if (rc) return fail(kErrCuda, std::string("cf_laplacian launch: ") + launch_error_text());
    return 0;
}

PMB_API int pmb_cf_laplacian_planes(const double* image, const uint8_t* is_known, int h, int w,
                                    double epsilon, const uint8_t* diag_mask, double diag_value,
                                    double* planes, void* stream) {
    if (!image || !planes || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_cf_laplacian_planes: bad arguments");
    if (pmb_launch_cf_half(image, is_known, h, w, epsilon, planes, pitch_for(w), diag_mask,
                           diag_value, (cudaStream_t)stream))
        return fail(kErrCuda, std::string("cf planes launch: ") + launch_error_text());
    return 0;
}

int64_t pmb_launch_lkm_scratch(int, int, int);
int pmb_launch_lkm_setup(const double*, int, int, int, double, double*, double*, cudaStream_t);
int pmb_launch_lkm_apply(const double*, int, int, int, const double*, const double*, const double*,
                         double*, double*, cudaStream_t);
int pmb_launch_lkm_diag(const double*, int, int, int, const double*, const double*, double*,
                        double*, double*, cudaStream_t);

PMB_API int64_t pmb_lkm_scratch_elems(int h, int w, int radius) {
    if (h <= 2 * radius || w <= 2 * radius || radius < 0) return -1;
    return pmb_launch_lkm_scratch(h, w, radius);
}

PMB_API int pmb_lkm_setup(const double* image, int h, int w, int radius, double epsilon,
                          double* windows, double* scratch, void* stream) {
    if (!image || !windows || !scratch || radius < 0 || h <= 2 * radius || w <= 2 * radius)
        return fail(kErrArg, "pmb_lkm_setup: bad arguments (the image must exceed 2 radius)");
    if (pmb_launch_lkm_setup(image, h, w, radius, epsilon, windows, scratch, (cudaStream_t)stream))
        return fail(kErrCuda, std::string("lkm setup: ") + launch_error_text());
    return 0;
}

PMB_API int pmb_lkm_apply(const double* image, int h, int w, int radius, const double* windows,
                          const double* diag_add, const double* p, double* out, double* scratch,
                          void* stream) {
    if (!image || !windows || !p || !out || !scratch || radius < 0 || h <= 2 * radius ||
        w <= 2 * radius)
        return fail(kErrArg, "pmb_lkm_apply: bad arguments");
    if (pmb_launch_lkm_apply(image, h, w, radius, windows, diag_add, p, out, scratch,
                             (cudaStream_t)stream))
        return fail(kErrCuda, std::string("lkm apply: ") + launch_error_text());
    return 0;
}

PMB_API int pmb_lkm_diagonal(const double* image, int h, int w, int radius, const double* windows,
                             const double* diag_add, double* diag, double* inv_diag,
                             double* scratch, void* stream) {
    if (!image || !windows || !diag || !scratch || radius < 0 || h <= 2 * radius ||
        w <= 2 * radius)
        return fail(kErrArg, "pmb_lkm_diagonal: bad arguments");
    if (pmb_launch_lkm_diag(image, h, w, radius, windows, diag_add, diag, inv_diag, scratch,
                            (cudaStream_t)stream))
        return fail(kErrCuda, std::string("lkm diagonal: ") + launch_error_text());
    return 0;
}

int pmb_launch_cf_vjp(const double*, const uint8_t*, int, int, double, const double*,
                      const double*, double*, cudaStream_t);

PMB_API int pmb_cf_laplacian_vjp(const double* image, const uint8_t* is_known, int h, int w,
                                 double epsilon, const double* x, const double* mu, double* grad,
                                 void* stream) {
    if (!image || !x || !mu || !grad || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_cf_laplacian_vjp: bad arguments");
    if (pmb_launch_cf_vjp(image, is_known, h, w, epsilon, x, mu, grad, (cudaStream_t)stream))
        return fail(kErrCuda, std::string("cf_laplacian_vjp launch: ") +
                                  launch_error_text());
    return 0;
}

int64_t pmb_launch_fg_workspace(int, int, int);
int pmb_launch_fg_levels(int, int, int, int, int, int*, int);
int pmb_launch_fg(const float*, const float*, int, int, int, float, int, int, int, float,
                  const float*, float*, float*, void*, int64_t, cudaStream_t);
int pmb_launch_fg_status(void*, cudaStream_t, int*);

PMB_API int64_t pmb_fg_workspace_bytes(int h, int w, int depth) {
    return pmb_launch_fg_workspace(h, w, depth);
}

PMB_API int pmb_fg_levels(int h, int w, int n_small, int n_big, int small_size, int* hw,
                          int max_levels) {
    if (h <= 0 || w <= 0 || !hw || max_levels <= 0) return fail(kErrArg, "pmb_fg_levels: bad arguments");
    const int n = pmb_launch_fg_levels(h, w, n_small, n_big, small_size, hw, max_levels);
    if (n == -1) return fail(kErrZeroDiv, "division by zero");
    if (n < 0) return fail(kErrArg, "pmb_fg_levels: too many levels");
    return n;
}

PMB_API int pmb_fg_ml(const float* image, const float* alpha, int h, int w, int depth,
                      float regularization, int n_small_iterations, int n_big_iterations,
                      int small_size, float gradient_weight, const float* seed, float* F,
                      float* B, void* workspace, int64_t workspace_bytes, void* stream) {
    const int rc = pmb_launch_fg(image, alpha, h, w, depth, regularization, n_small_iterations,
                                 n_big_iterations, small_size, gradient_weight, seed, F, B,
                                 workspace, workspace_bytes, (cudaStream_t)stream);
    if (rc == 0) return 0;
    if (rc == -1) return fail(kErrZeroDiv, "division by zero");
    if (rc == -2) return fail(kErrArg, "pmb_fg_ml: bad arguments");
    if (rc == -3) return fail(kErrArg, "pmb_fg_ml: workspace smaller than pmb_fg_workspace_bytes");
    return fail(kErrCuda, std::string("pmb_fg_ml launch: ") + cudaGetErrorString((cudaError_t)rc));
}

PMB_API int pmb_fg_status(void* workspace, void* stream) {
    if (!workspace) return fail(kErrArg, "pmb_fg_status: bad arguments");
    int v = 0;
    const int rc = pmb_launch_fg_status(workspace, (cudaStream_t)stream, &v);
    if (rc) return fail(kErrCuda, std::string("pmb_fg_status: ") + cudaGetErrorString((cudaError_t)rc));
    if (v == 1) return fail(kErrState, "foreground sweep: a wait for a neighbouring strip timed out");
    if (v == 2) return fail(kErrState, "foreground sweep: a coefficient copy did not complete");
    if (v) return fail(kErrState, "foreground sweep failed (" + std::to_string(v) + ")");
    return 0;
}

int64_t pmb_launch_fgj_workspace(int, int);
int pmb_launch_fgj(const float*, const float*, int, int, float, int, int, int, float*, float*,
                   void*, int64_t, cudaStream_t);

PMB_API int64_t pmb_fg_jacobi_workspace_bytes(int h, int w) { return pmb_launch_fgj_workspace(h, w); }

PMB_API int pmb_fg_ml_jacobi(const float* image, const float* alpha, int h, int w,
                             float regularization, int n_small_iterations, int n_big_iterations,
                             int small_size, float* F, float* B, void* workspace,
                             int64_t workspace_bytes, void* stream) {
    const int rc = pmb_launch_fgj(image, alpha, h, w, regularization, n_small_iterations,
                                  n_big_iterations, small_size, F, B, workspace, workspace_bytes,
                                  (cudaStream_t)stream);
    if (rc == 0) return 0;
    if (rc == -1) return fail(kErrZeroDiv, "division by zero");
    if (rc == -2) return fail(kErrArg, "pmb_fg_ml_jacobi: bad arguments");
    if (rc == -3) return fail(kErrArg, "pmb_fg_ml_jacobi: workspace smaller than pmb_fg_jacobi_workspace_bytes");
    return fail(kErrCuda, std::string("pmb_fg_ml_jacobi launch: ") + cudaGetErrorString((cudaError_t)rc));
}

int pmb_launch_window_laplacian(int, const double*, int, int, int, double, const int64_t*,
                                const int64_t*, int64_t*, int64_t*, double*, cudaStream_t);

PMB_API int pmb_window_laplacian(int mode, const double* image, int h, int w, int radius,
                                 double regularization, const int64_t* px, const int64_t* py,
                                 int64_t* rowptr, int64_t* cols, double* vals, void* stream) {
    const int rc = pmb_launch_window_laplacian(mode, image, h, w, radius, regularization, px, py,
                                               rowptr, cols, vals, (cudaStream_t)stream);
    if (rc == -2) return fail(kErrArg, "pmb_window_laplacian: bad arguments");
    if (rc) return fail(kErrCuda, std::string("pmb_window_laplacian launch: ") +
                                      launch_error_text());
    return 0;
}

int pmb_launch_lbdm_laplacian(const double*, int, int, int, double, double*, const int64_t*,
                              const int64_t*, int64_t*, int64_t*, double*, cudaStream_t);

PMB_API int64_t pmb_lbdm_scratch_elems(int h, int w, int radius) {
    if ((radius != 1 && radius != 2) || h <= 2 * radius || w <= 2 * radius) return -1;
    const int64_t s = 2 * radius + 1;
    return (int64_t)(h - 2 * radius) * (w - 2 * radius) * s * s * s * s;
}

PMB_API int pmb_lbdm_laplacian(const double* image, int h, int w, int radius, double epsilon,
                               double* scratch, const int64_t* px, const int64_t* py,
                               int64_t* rowptr, int64_t* cols, double* vals, void* stream) {
    const int rc = pmb_launch_lbdm_laplacian(image, h, w, radius, epsilon, scratch, px, py, rowptr,
                                             cols, vals, (cudaStream_t)stream);
    if (rc == -2) return fail(kErrArg, "pmb_lbdm_laplacian: bad arguments (radius 1 or 2, image larger than 2 radius)");
    if (rc) return fail(kErrCuda, std::string("pmb_lbdm_laplacian launch: ") +
                                      launch_error_text());
    return 0;
}

int64_t pmb_launch_knn_scratch(long long, int, int);
int pmb_launch_knn(const double*, int, int, const int*, const double*, int, int, int64_t*,
                   int64_t*, int64_t*, double*, int64_t*, cudaStream_t);

PMB_API int64_t pmb_knn_scratch_elems(int64_t n, int total_neighbors, int passes) {
    return pmb_launch_knn_scratch((long long)n, total_neighbors, passes);
}

PMB_API int pmb_knn_laplacian(const double* image, int h, int w, const int* n_neighbors,
                              const double* distance_weights, int passes, int soft,
                              int64_t* scratch, int64_t* rowptr, int64_t* cols, double* vals,
                              int64_t* nnz, void* stream) {
    const int rc = pmb_launch_knn(image, h, w, n_neighbors, distance_weights, passes, soft, scratch,
                                  rowptr, cols, vals, nnz, (cudaStream_t)stream);
    if (rc == -2) return fail(kErrArg, "pmb_knn_laplacian: bad arguments (1 to 4 passes of 1 to 64 neighbours, at most the pixel count)");
    if (rc) return fail(kErrCuda, std::string("pmb_knn_laplacian: ") + launch_error_text());
    return 0;
}

int pmb_launch_fg_cf_system(const double*, int, int, double, int64_t*, int64_t*, double*,
                            int64_t*, cudaStream_t);

PMB_API int pmb_fg_cf_system(const double* alpha, int h, int w, double regularization,
                             int64_t* rowptr, int64_t* cols, double* vals, int64_t* scratch,
                             void* stream) {
    const int rc = pmb_launch_fg_cf_system(alpha, h, w, regularization, rowptr, cols, vals,
                                           scratch, (cudaStream_t)stream);
    if (rc == -2) return fail(kErrArg, "pmb_fg_cf_system: bad arguments");
    if (rc) return fail(kErrCuda, std::string("pmb_fg_cf_system: ") + launch_error_text());
    return 0;
}

PMB_API int pmb_cf_hard_system(const double* image, const uint8_t* is_known, const uint8_t* is_fg,
                               int h, int w, double epsilon, double* planes, double* rhs,
                               void* stream) {
    if (!image || !is_known || !is_fg || !planes || !rhs || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_cf_hard_system: bad arguments");
    if (pmb_launch_cf_hard(image, is_known, is_fg, h, w, epsilon, planes, pitch_for(w), rhs,
                           (cudaStream_t)stream))
        return fail(kErrCuda, std::string("cf hard launch: ") + launch_error_text());
    return 0;
}

PMB_API int64_t pmb_scan_scratch_elems(int64_t n) { return (n + 1023) / 1024 + 2; }

#define PMB_LAUNCHED(expr, what)                                                      \
    do {                                                                              \
        if ((expr) != 0)                                                              \
            return fail(kErrCuda, std::string(what) + ": " + launch_error_text());   \
    } while (0)

PMB_API int pmb_ell_csr_rowptr(const double* values, int h, int w, int radius, int64_t* rowptr,
                               int64_t* scratch, void* stream) {
    if (!values || !rowptr || !scratch || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_ell_csr_rowptr: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = (int64_t)h * w;
    PMB_CUDA(cudaMemsetAsync(rowptr + n, 0, sizeof(int64_t), s));
    PMB_LAUNCHED(pmb_launch_ell_count(values, h, w, radius, rowptr, s), "ell count");
    PMB_LAUNCHED(pmb_scan_exclusive(rowptr, n + 1, scratch, scratch + (n + 1023) / 1024 + 1, s),
                 "scan");
    return 0;
}

PMB_API int pmb_ell_csr_fill(const double* values, int h, int w, int radius,
                             const int64_t* rowptr, int64_t* indices, double* data, void* stream) {
    if (!values || !rowptr || h <= 0 || w <= 0) return fail(kErrArg, "pmb_ell_csr_fill: bad arguments");
    PMB_LAUNCHED(pmb_launch_ell_fill(values, h, w, radius, rowptr, indices, data,
                                     (cudaStream_t)stream), "ell fill");
    return 0;
}

PMB_API int pmb_trimap_masks(const double* trimap, int64_t n, double fg_threshold,
                             double bg_threshold, uint8_t* is_fg, uint8_t* is_known,
                             unsigned long long* counts, void* stream) {
    if (!trimap || !is_fg || !is_known || !counts || n <= 0)
        return fail(kErrArg, "pmb_trimap_masks: bad arguments");
    PMB_LAUNCHED(pmb_launch_trimap_masks(trimap, n, fg_threshold, bg_threshold, is_fg, is_known,
                                         counts, (cudaStream_t)stream), "trimap masks");
    return 0;
}

PMB_API int pmb_unknown_index(const uint8_t* is_known, int64_t n, int64_t* cidx, int64_t* scratch,
                              void* stream) {
    if (!is_known || !cidx || !scratch || n <= 0) return fail(kErrArg, "pmb_unknown_index: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    PMB_CUDA(cudaMemsetAsync(cidx + n, 0, sizeof(int64_t), s));
    PMB_LAUNCHED(pmb_launch_flag_unknown(is_known, n, cidx, s), "unknown flags");
    PMB_LAUNCHED(pmb_scan_exclusive(cidx, n + 1, scratch, scratch + (n + 1023) / 1024 + 1, s), "scan");
    return 0;
}

int64_t pmb_static_scan_max_n();
int pmb_launch_unknown_index_static(const uint8_t*, int64_t, int64_t*, cudaStream_t);

// pmb_unknown_index for callers that cannot allocate device memory: the
// scan's scratch is a fixed array inside the library (cf_assemble.cu).
PMB_API int pmb_unknown_index_static(const uint8_t* is_known, int64_t n, int64_t* cidx,
                                     void* stream) {
    if (!is_known || !cidx || n <= 0) return fail(kErrArg, "pmb_unknown_index_static: bad arguments");
    if (n > pmb_static_scan_max_n())
        return fail(kErrArg, "pmb_unknown_index_static: n = " + std::to_string(n) +
                                 " exceeds the built-in scratch limit of " +
                                 std::to_string(pmb_static_scan_max_n()) +
                                 " pixels; use pmb_unknown_index with caller scratch");
    const int rc = pmb_launch_unknown_index_static(is_known, n, cidx, (cudaStream_t)stream);
    if (rc == -3) return fail(kErrCuda, "pmb_unknown_index_static: scratch address lookup failed");
    if (rc) return fail(kErrCuda, std::string("pmb_unknown_index_static: ") +
                                      launch_error_text());
    return 0;
}

PMB_API int pmb_hard_lu_rowptr(const uint8_t* is_known, int h, int w, int radius,
                               const int64_t* cidx, int64_t n_unknown, int64_t* rowptr,
                               int64_t* scratch, void* stream) {
    if (!is_known || !cidx || !rowptr || !scratch || h <= 0 || w <= 0 || radius < 1)
        return fail(kErrArg, "pmb_hard_lu_rowptr: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    PMB_CUDA(cudaMemsetAsync(rowptr, 0, sizeof(int64_t) * (n_unknown + 1), s));
    PMB_LAUNCHED(pmb_launch_lu_count(is_known, h, w, radius, rowptr, cidx, s), "L_U count");
    PMB_LAUNCHED(pmb_scan_exclusive(rowptr, n_unknown + 1, scratch,
                                    scratch + (n_unknown + 1023) / 1024 + 1, s), "scan");
    return 0;
}

PMB_API int pmb_hard_lu_fill(const double* ell_values, const uint8_t* is_known,
                             const uint8_t* is_fg, int h, int w, int radius, const int64_t* cidx,
                             const int64_t* rowptr, int64_t* indices, double* data, double* rhs,
                             void* stream) {
    if (!ell_values || !is_known || !is_fg || !cidx || !rowptr || !rhs || radius < 1)
        return fail(kErrArg, "pmb_hard_lu_fill: bad arguments");
    PMB_LAUNCHED(pmb_launch_lu_fill(ell_values, is_known, is_fg, h, w, radius, cidx, rowptr,
                                    indices, data, rhs, (cudaStream_t)stream), "L_U fill");
    return 0;
}

PMB_API int pmb_alpha_compose(const double* trimap, const uint8_t* is_known, const int64_t* cidx,
                              const double* x_unknown, int64_t n, double* alpha, void* stream) {
    if (!trimap || !is_known || !cidx || !alpha || n <= 0)
        return fail(kErrArg, "pmb_alpha_compose: bad arguments");
    PMB_LAUNCHED(pmb_launch_alpha_compose(trimap, is_known, cidx, x_unknown, n, alpha,
                                          (cudaStream_t)stream), "alpha compose");
    return 0;
}

PMB_API int pmb_stencil_create(int n_images, const int* h, const int* w, int precision,
                               int preconditioner, int num_pre_iter, int num_post_iter,
                               double omega, int direct_solve_size, pmb_stencil** out) {
    if (!out || n_images <= 0 || !h || !w) return fail(kErrArg, "pmb_stencil_create: bad arguments");
    if (precision < 0 || precision > 1) return fail(kErrArg, "precision must be 0 (fp64) or 1 (mixed)");
    if (preconditioner < 0 || preconditioner > 2) return fail(kErrArg, "unknown preconditioner");
    if (num_pre_iter < 0 || num_post_iter < 0) return fail(kErrArg, "negative smoothing count");
    if (direct_solve_size < 0 || direct_solve_size > kMaxDirect)
        return fail(kErrArg, "direct_solve_size must be in [0, 256]");
    pmb_stencil* p = new pmb_stencil();
    Stencil& S = p->S;
    S.nimg = n_images;
    for (int k = 0; k < n_images; ++k) {
        if (h[k] <= 0 || w[k] <= 0) {
            delete p;
            return fail(kErrArg, "image sizes must be positive");
        }
        S.h.push_back(h[k]);
        S.w.push_back(w[k]);
    }
    S.precision = precision;
    S.precond = preconditioner;
    S.pre = num_pre_iter;
    S.post = num_post_iter;
    S.omega = omega;
    S.direct = direct_solve_size;
    if (int rc = plan_stencil(S)) {
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

PMB_API int64_t pmb_stencil_workspace_bytes(const pmb_stencil* p) {
    return p ? (int64_t)p->S.ws_bytes : -1;
}

PMB_API int64_t pmb_stencil_plane_offset(const pmb_stencil* p, int image) {
    if (!p || image < 0 || image >= p->S.nimg) return -1;
    return p->S.levels[0].grids[image].poff;
}

PMB_API int64_t pmb_stencil_plane_elems(const pmb_stencil* p) {
    return p ? p->S.levels[0].plane_elems : -1;
}

PMB_API int pmb_stencil_levels(const pmb_stencil* p, int image) {
    if (!p || image < 0 || image >= p->S.nimg) return -1;
    return p->S.coarsest[image] + 1;
}

PMB_API int pmb_stencil_bind(pmb_stencil* p, void* workspace, const double* planes64,
                             void* stream) {
    if (!p || !workspace || !planes64) return fail(kErrArg, "pmb_stencil_bind: bad arguments");
    Stencil& S = p->S;
    if (!S.stream) {
        PMB_CUDA(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking));
        PMB_CUDA(cudaEventCreateWithFlags(&S.ev_in, cudaEventDisableTiming));
        PMB_CUDA(cudaEventCreateWithFlags(&S.ev_out, cudaEventDisableTiming));
        PMB_CUDA(cudaHostAlloc((void**)&S.h_state, sizeof(InstState) * 2 * S.nimg, cudaHostAllocDefault));
        S.h_outer = S.h_state + S.nimg;
    }
    return on_stream(S, (cudaStream_t)stream, [&]() { return bind_stencil(S, workspace, planes64); });
}

PMB_API int pmb_stencil_setup(pmb_stencil* p, void* stream) {
    if (!p || !p->S.bound) return fail(kErrState, "pmb_stencil_setup: not bound");
    Stencil& S = p->S;
    return on_stream(S, (cudaStream_t)stream, [&]() { return setup_stencil(S); });
}

PMB_API int pmb_stencil_solve(pmb_stencil* p, const double* b, const double* x0, double* x_out,
                              double atol, double rtol, int maxiter, int reorthogonalize,
                              double inner_rtol, int max_outer, void* stream) {
    if (!p || !b || !x_out) return fail(kErrArg, "pmb_stencil_solve: bad arguments");
    Stencil& S = p->S;
    if (!S.bound) return fail(kErrState, "pmb_stencil_solve: not bound");
    return on_stream(S, (cudaStream_t)stream, [&]() -> int {
        if (!S.setup_done) {
            if (int rc = setup_stencil(S)) return rc;
        }
        HostList& a = S.fine0;
        cudaStream_t s = S.stream;
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), b,
                                    S.at<double>(S.o_b64), S.user_total, s);
        int rc;
        if (S.precision == 0) rc = solve_fp64(S, x0, atol, rtol, maxiter, reorthogonalize);
        else rc = solve_mixed(S, x0, atol, rtol, maxiter, reorthogonalize, inner_rtol, max_outer);
        if (rc) return rc;
        launch_unpack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff),
                                      S.at<double>(S.o_x64), x_out, S.user_total, s);
        PMB_CUDA(cudaGetLastError());
        return 0;
    });
}

PMB_API int pmb_stencil_precondition(pmb_stencil* p, const double* r, double* z, void* stream) {
    if (!p || !r || !z) return fail(kErrArg, "pmb_stencil_precondition: bad arguments");
    Stencil& S = p->S;
    if (!S.bound) return fail(kErrState, "pmb_stencil_precondition: not bound");
    if (S.precision != 0) return fail(kErrArg, "standalone preconditioner needs the fp64 solver");
    return on_stream(S, (cudaStream_t)stream, [&]() -> int {
        if (!S.setup_done) {
            if (int rc = setup_stencil(S)) return rc;
        }
        HostList& a = S.fine0;
        cudaStream_t s = S.stream;
        CgVecs<double> v = cg_vecs<double>(S);
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), r, v.r,
                                    S.user_total, s);
        if (S.precond == kPrecVcycle) {
            run_vcycle<double>(S, v.r, v.z, nullptr, nullptr, 0);
        } else if (S.precond == kPrecJacobi) {
            // z = r / diag: the first Jacobi sweep from zero with omega = 1.
            launch_vc_smooth<double>(LaunchCfg{grid_for(a, smem_init<double>())}, a.wl, S.maps(), -1, S.P0, v.r,
                                     v.z, 1.0, nullptr, S.err(), s);
        } else {
            PMB_CUDA(cudaMemcpyAsync(v.z, v.r, sizeof(double) * S.levels[0].vec_elems,
                                     cudaMemcpyDeviceToDevice, s));
        }
        launch_unpack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), v.z, z,
                                      S.user_total, s);
        PMB_CUDA(cudaGetLastError());
        return check_err(S);
    });
}

PMB_API int pmb_stencil_apply(pmb_stencil* p, const double* x, double* y, void* stream) {
    if (!p || !x || !y) return fail(kErrArg, "pmb_stencil_apply: bad arguments");
    Stencil& S = p->S;
    if (!S.bound) return fail(kErrState, "pmb_stencil_apply: not bound");
    if (S.precision != 0) return fail(kErrArg, "pmb_stencil_apply needs the fp64 solver");
    return on_stream(S, (cudaStream_t)stream, [&]() -> int {
        HostList& a = S.fine0;
        cudaStream_t s = S.stream;
        double* tx = S.at<double>(S.o_r64);   // level-0 b buffer: map slot kMapBF
        double* ty = S.at<double>(S.o_ap64);
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), x, tx,
                                    S.user_total, s);
        launch_apply<double>(LaunchCfg{grid_for(a, smem_apply_v<double>(2))}, a.wl, S.maps(), ty,
                             S.err(), s);
        launch_unpack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), ty, y,
                                      S.user_total, s);
        PMB_CUDA(cudaGetLastError());
        return check_err(S);
    });
}

// Per-image result of the last solve: iterations (inner iterations of the
// last refinement step in mixed mode), status, |r|, |b| and refinement steps.
PMB_API int pmb_stencil_stats(pmb_stencil* p, int image, int* iters, int* status, double* norm_r,
                              double* norm_b, int* outer_iters) {
    if (!p || image < 0 || image >= p->S.nimg) return fail(kErrArg, "pmb_stencil_stats: bad image");
    Stencil& S = p->S;
    if (int rc = read_states(S, true)) return rc;
    // Mixed precision: the FP32 state carries the final status (convergence
    // is only declared on an FP64 residual); the norms are the FP64 ones.
    const InstState& st = S.precision == 1 ? S.h_outer[image] : S.h_state[image];
    if (iters) *iters = S.h_state[image].iters;
    if (status) *status = S.h_state[image].status;
    if (norm_r) *norm_r = st.norm_r;
    if (norm_b) *norm_b = st.norm_b;
    if (outer_iters) *outer_iters = S.precision == 1 ? S.h_outer[image].iters : 0;
    return 0;
}

PMB_API int64_t pmb_stencil_launch_count(const pmb_stencil* p) { return p ? p->S.launches : -1; }

// Launch-shape knobs for the autotuner. Values are clamped to what the
// kernels support; the applied value is returned. Changing a knob drops the
// captured iteration graph (it is captured again on the next solve).
PMB_API int pmb_stencil_tune(pmb_stencil* p, int knob, int value) {
    if (!p) return fail(kErrArg, "pmb_stencil_tune: null solver");
    Stencil& S = p->S;
    const int wide = S.precision == 1 ? 4 : 2;
    auto clampi = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
    int applied;
    switch (knob) {
    case 0:
        applied = S.vec_apply = (value >= 4 ? wide : 2);
        S.max_fine = S.precision == 1 ? resident_cg_apply<float>(S.vec_apply, S.stages)
                                      : resident_cg_apply<double>(S.vec_apply, S.stages);
        S.fine0.per_sm = std::min(S.fine0.per_sm, S.max_fine);
        break;
    case 1:
        applied = S.vec_up = (value >= 4 ? wide : 2);
        if (S.pre == 1 && S.post == 1) {
            S.max_up = S.precision == 1 ? resident_up<float>(S.vec_up, S.stages)
                                        : resident_up<double>(S.vec_up, S.stages);
            for (auto& lv : S.levels) lv.fine.per_sm = std::min(lv.fine.per_sm, S.max_up);
        }
        break;
    case 2:
        applied = clampi(value, 1, S.max_fine);
        S.fine0.per_sm = applied;
        break;
    case 3:
        applied = clampi(value, 1, S.max_up);
        for (auto& lv : S.levels) lv.fine.per_sm = applied;
        break;
    case 4:
        applied = clampi(value, 1, S.max_down);
        for (auto& lv : S.levels) lv.coarse.per_sm = applied;
        break;
    case 5:
        applied = clampi(value, 1, kMaxCtasPerSm);
        S.flat0.per_sm = applied;
        for (auto& lv : S.levels) lv.flat.per_sm = applied;
        break;
    case 6: applied = S.chunk = clampi(value, 1, 16); break;
    case 7: {
        // Buffers of the restriction / prolongation kernels; their CTAs per
        // SM follow the shared memory of the choice.
        applied = S.stages = value <= 1 ? 1 : 2;
        const bool mixed = S.precision == 1;
        S.max_fine = mixed ? resident_cg_apply<float>(S.vec_apply, S.stages)
                           : resident_cg_apply<double>(S.vec_apply, S.stages);
        S.fine0.per_sm = S.max_fine;
        if (S.pre == 1 && S.post == 1) {
            S.max_up = mixed ? resident_up<float>(S.vec_up, S.stages)
                             : resident_up<double>(S.vec_up, S.stages);
            S.max_down = mixed ? resident_down<float>(S.stages) : resident_down<double>(S.stages);
            for (auto& lv : S.levels) {
                lv.fine.per_sm = S.max_up;
                lv.coarse.per_sm = S.max_down;
            }
        }
        break;
    }
    default: return fail(kErrArg, "pmb_stencil_tune: unknown knob");
    }
    if (S.graph) {
        cudaGraphExecDestroy(S.graph);
        S.graph = nullptr;
    }
    return applied;
}

PMB_API int pmb_stencil_tuning(const pmb_stencil* p, int knob) {
    if (!p) return fail(kErrArg, "pmb_stencil_tuning: null solver");
    const Stencil& S = p->S;
    switch (knob) {
    case 0: return S.vec_apply;
    case 1: return S.vec_up;
    case 2: return S.fine0.per_sm;
    case 3: return S.levels.empty() ? 0 : S.levels[0].fine.per_sm;
    case 4: return S.levels.empty() ? 0 : S.levels[0].coarse.per_sm;
    case 5: return S.flat0.per_sm;
    case 6: return S.chunk;
    case 7: return S.stages;
    default: return fail(kErrArg, "pmb_stencil_tuning: unknown knob");
    }
}

PMB_API int pmb_stencil_destroy(pmb_stencil* p) {
    if (!p) return 0;
    Stencil& S = p->S;
    if (S.graph) cudaGraphExecDestroy(S.graph);
    if (S.stream) {
        cudaStreamSynchronize(S.stream);
        cudaStreamDestroy(S.stream);
    }
    if (S.ev_in) cudaEventDestroy(S.ev_in);
    if (S.ev_out) cudaEventDestroy(S.ev_out);
    if (S.h_state) cudaFreeHost(S.h_state);
    delete p;
    return 0;
}

// --------------------------------------------------------------------------
// Incomplete Cholesky object
// --------------------------------------------------------------------------

int pmb_scan_exclusive(int64_t*, int64_t, int64_t*, int64_t*, cudaStream_t);

namespace pmb {

struct Ichol {
    int64_t n = 0, band = 0, W = 0, cap = 0;
    size_t ws_bytes = 0;
    size_t o_d, o_rsum, o_level, o_band, o_F, o_pat, o_cand, o_keptv, o_kepti, o_result, o_Lp,
        o_Lr, o_Lv, o_lcnt, o_lfill, o_order, o_maxl, o_Rp, o_rfill, o_Rc, o_Rv, o_scan;
    char* ws = nullptr;
    int64_t nnz = -1;
    int nlevels = 0;
    int cluster = -1;     // CTAs holding the front in the last factorisation (0: global memory)
    cudaEvent_t ev_f0 = nullptr, ev_f1 = nullptr;   // around the factor kernel
    float factor_ms = -1.0f;
    // Streamed solves (n <= kStreamMaxRows): chunk blocks of both sweeps.
    size_t o_blob = 0, o_prow = 0, o_pch = 0, blob_cap = 0;
    int stream_total = 0;  // chunks of both sweeps; 0: level-barrier solves
    StreamFirst first{};
    template <typename T> T* at(size_t off) const { return reinterpret_cast<T*>(ws + off); }
};

static void plan_ichol(Ichol& I) {
    Carve c;
    const int64_t n = I.n, W = I.W, cap = I.cap;
    I.o_d = c.take<double>(n);
    I.o_rsum = c.take<double>(n);
    I.o_level = c.take<int>(n);
    I.o_band = c.take<unsigned long long>(1);
    I.o_F = c.take<double>(W * W);
    I.o_pat = c.take<uint8_t>(W * W);
    I.o_cand = c.take<int>(W);
    I.o_keptv = c.take<double>(W);
    I.o_kepti = c.take<int64_t>(W);
    I.o_result = c.take<int64_t>(1);
    I.o_Lp = c.take<int64_t>(n + 1);
    I.o_Lr = c.take<int64_t>(cap);
    I.o_Lv = c.take<double>(cap);
    I.o_lcnt = c.take<int64_t>(n + 2);
    I.o_lfill = c.take<int64_t>(n + 2);
    I.o_order = c.take<int>(n);
    I.o_maxl = c.take<int>(1);
    I.o_Rp = c.take<int64_t>(n + 1);
    I.o_rfill = c.take<int64_t>(n + 1);
    I.o_Rc = c.take<int64_t>(cap);
    I.o_Rv = c.take<double>(cap);
    I.o_scan = c.take<int64_t>((n + 2 + 1023) / 1024 + 4);
    if (n <= kStreamMaxRows) {
        // At most one chunk per row and sweep; entries of both sweeps are the
        // factor's off-diagonal entries, padded to 4 per chunk.
        I.blob_cap = (size_t)(200 * n + 24 * cap);
        I.o_blob = c.take<unsigned char>((int64_t)I.blob_cap);
        I.o_prow = c.take<StreamPackRow>(2 * n);
        I.o_pch = c.take<StreamPackChunk>(2 * n);
    }
    I.ws_bytes = c.off + 256;
}

// Chunk plan of the streamed solves (ichol.cu), built on the host from the
// level schedule and the row / column pointers, then packed on the device.
// Leaves stream_total = 0 (level-barrier solves) when a row has more entries
// than a chunk holds.
static int build_stream(Ichol& I, cudaStream_t s) {
    I.stream_total = 0;
    if (!I.o_blob) return 0;
    const int64_t n = I.n;
    const int nl = I.nlevels;
    std::vector<int> order(n);
    std::vector<int64_t> lptr(nl + 1), Rp(n + 1), Lp(n + 1);
    PMB_CUDA(cudaMemcpyAsync(order.data(), I.ws + I.o_order, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaMemcpyAsync(lptr.data(), I.ws + I.o_lcnt, sizeof(int64_t) * (nl + 1),
                             cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaMemcpyAsync(Rp.data(), I.ws + I.o_Rp, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaMemcpyAsync(Lp.data(), I.ws + I.o_Lp, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    std::vector<StreamPackRow> recs;
    std::vector<StreamPackChunk> chunks;
    recs.reserve(2 * n);
    int64_t off = 0;
    for (int sweep = 0; sweep < 2; ++sweep) {
        const bool bwd = sweep == 1;
        for (int li = 0; li < nl; ++li) {
            const int l = bwd ? nl - 1 - li : li;
            int64_t q = lptr[l];
            while (q < lptr[l + 1]) {
                const size_t first_rec = recs.size();
                int used = 0, rows = 0;
                while (q < lptr[l + 1] && rows < kStreamRowsMax) {
                    const int i = order[q];
                    const int64_t src = bwd ? Lp[i] + 1 : Rp[i];
                    const int64_t cnt = bwd ? Lp[i + 1] - Lp[i] - 1 : Rp[i + 1] - Rp[i];
                    if (cnt > kStreamEntsMax) return 0;
                    if (used + cnt > kStreamEntsMax) break;
                    recs.push_back(StreamPackRow{off, src, i, rows, used, (int)cnt, 0, 0, bwd ? 1 : 0, 0});
                    used += (int)cnt;
                    ++rows;
                    ++q;
                }
                const int ents = (used + 3) & ~3;
                const int bytes = (int)(sizeof(StreamHead) + rows * sizeof(StreamRow)) + 12 * ents;
                for (size_t k = first_rec; k < recs.size(); ++k) {
                    recs[k].rows = rows;
                    recs[k].ents = ents;
                }
                chunks.push_back(StreamPackChunk{off, bytes, rows, ents, used});
                off += bytes;
            }
        }
    }
    if ((size_t)off > I.blob_cap || (int64_t)chunks.size() > 2 * n) return 0;
    PMB_CUDA(cudaMemcpyAsync(I.ws + I.o_prow, recs.data(), sizeof(StreamPackRow) * recs.size(),
                             cudaMemcpyHostToDevice, s));
    PMB_CUDA(cudaMemcpyAsync(I.ws + I.o_pch, chunks.data(), sizeof(StreamPackChunk) * chunks.size(),
                             cudaMemcpyHostToDevice, s));
    ichol_launch_stream_pack((int)recs.size(), I.at<StreamPackRow>(I.o_prow), (int)chunks.size(),
                             I.at<StreamPackChunk>(I.o_pch), I.at<int64_t>(I.o_Rc), I.at<double>(I.o_Rv),
                             I.at<int64_t>(I.o_Lr), I.at<double>(I.o_Lv), I.at<int64_t>(I.o_Lp),
                             I.at<unsigned char>(I.o_blob), s);
    PMB_CUDA(cudaGetLastError());
    PMB_CUDA(cudaStreamSynchronize(s));    // the host plan arrays are released on return
    for (int q = 0; q < kStreamStages; ++q) {
        I.first.off[q] = q < (int)chunks.size() ? chunks[q].off : 0;
        I.first.bytes[q] = q < (int)chunks.size() ? chunks[q].bytes : 0;
    }
    I.stream_total = (int)chunks.size();
    return 0;
}

// Row profile of a CSC matrix's lower part: bandwidth max(i - j) over
// non-zero entries below the diagonal, and the envelope sum_i (i - f_i + 1)
// with f_i the first column of row i. The envelope bounds the factor size.
__global__ void k_csc_first(int64_t n, const int64_t* __restrict__ Ap, const int64_t* __restrict__ Ar,
                            const double* __restrict__ Av, unsigned long long* first,
                            unsigned long long* band) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    int64_t bmax = 0;
    for (int64_t k = Ap[j]; k < Ap[j + 1]; ++k) {
        const int64_t i = Ar[k];
        if (i < j || i >= n) continue;
        if (i > j && Av[k] == 0.0) continue;
        atomicMin(first + i, (unsigned long long)j);
        if (i - j > bmax) bmax = i - j;
    }
    if (bmax) atomicMax(band, (unsigned long long)bmax);
}

__global__ void k_csc_envelope(int64_t n, const unsigned long long* __restrict__ first,
                               unsigned long long* env) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned long long v = 0;
    if (i < n) {
        const unsigned long long f = first[i] > (unsigned long long)i ? (unsigned long long)i : first[i];
        v = (unsigned long long)i - f + 1;
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(env, v);
}

__global__ void k_fill_u64(unsigned long long* p, int64_t n, unsigned long long v) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace pmb

struct pmb_ichol { Ichol I; };

// out[0] = bandwidth, out[1] = envelope; scratch: n + 2 uint64.
PMB_API int pmb_csc_profile(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                            uint64_t* scratch, uint64_t* out, void* stream) {
    if (n <= 0 || !Ap || !scratch || !out) return fail(kErrArg, "pmb_csc_profile: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* first = (unsigned long long*)scratch;
    unsigned long long* o = (unsigned long long*)out;
    k_fill_u64<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(first, n, ~0ull);
    PMB_CUDA(cudaMemsetAsync(o, 0, 2 * sizeof(unsigned long long), s));
    k_csc_first<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, Ap, Ar, Av, first, o);
    k_csc_envelope<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, first, o + 1);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

PMB_API int pmb_ichol_create(int64_t n, int64_t bandwidth, int64_t capacity, pmb_ichol** out) {
    if (!out || n <= 0 || bandwidth < 0 || capacity < n) return fail(kErrArg, "pmb_ichol_create: bad arguments");
    const int64_t W = bandwidth + 1;
    if (W > (int64_t)1 << 16) return fail(kErrArg, "ichol: bandwidth above 65535 is not supported");
    pmb_ichol* p = new pmb_ichol();
    p->I.n = n;
    p->I.band = bandwidth;
    p->I.W = W;
    p->I.cap = capacity;
    plan_ichol(p->I);
    *out = p;
    return 0;
}

PMB_API int64_t pmb_ichol_workspace_bytes(const pmb_ichol* p) { return p ? (int64_t)p->I.ws_bytes : -1; }

PMB_API int pmb_ichol_bind(pmb_ichol* p, void* workspace) {
    if (!p || !workspace) return fail(kErrArg, "pmb_ichol_bind: bad arguments");
    p->I.ws = (char*)workspace;
    return 0;
}

// One factorisation attempt with a given diagonal shift (ichol.py:259-276).
// *result: factor nnz, -1 (not positive definite), -2 (more than max_nnz).
// On success the level schedule and row view for the solves are built.
PMB_API int pmb_ichol_factor(pmb_ichol* p, const int64_t* Ap, const int64_t* Ar, const double* Av,
                             double discard_threshold, double shift, int64_t max_nnz,
                             double relative_discard_threshold, int diag_keep_discarded,
                             int64_t* result, void* stream) {
    if (!p || !p->I.ws || !Ap || !Ar || !Av || !result) return fail(kErrArg, "pmb_ichol_factor: bad arguments");
    Ichol& I = p->I;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = I.n, W = I.W;
    ichol_prepare();
    PMB_CUDA(cudaMemsetAsync(I.ws + I.o_F, 0, sizeof(double) * W * W, s));
    PMB_CUDA(cudaMemsetAsync(I.ws + I.o_pat, 0, (size_t)(W * W), s));
    ichol_launch_init(n, Ap, Ar, Av, shift, I.at<double>(I.o_d), I.at<double>(I.o_rsum),
                      I.at<int>(I.o_level), I.at<unsigned long long>(I.o_band), s);
    if (!I.ev_f0) {
        PMB_CUDA(cudaEventCreate(&I.ev_f0));
        PMB_CUDA(cudaEventCreate(&I.ev_f1));
    }
    PMB_CUDA(cudaEventRecord(I.ev_f0, s));
    I.cluster = ichol_launch_factor(n, W, Ap, Ar, Av, I.at<double>(I.o_d), I.at<double>(I.o_rsum),
                        I.at<int>(I.o_level), I.at<double>(I.o_F), I.at<uint8_t>(I.o_pat),
                        I.at<int>(I.o_cand), I.at<double>(I.o_keptv), I.at<int64_t>(I.o_kepti),
                        I.at<int64_t>(I.o_Lp), I.at<int64_t>(I.o_Lr), I.at<double>(I.o_Lv), I.cap,
                        discard_threshold, max_nnz, relative_discard_threshold, diag_keep_discarded,
                        I.at<int64_t>(I.o_result), s);
    PMB_CUDA(cudaGetLastError());
    PMB_CUDA(cudaEventRecord(I.ev_f1, s));
    int64_t res = 0;
    PMB_CUDA(cudaMemcpyAsync(&res, I.ws + I.o_result, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    PMB_CUDA(cudaEventElapsedTime(&I.factor_ms, I.ev_f0, I.ev_f1));
    *result = res;
    I.nnz = res;
    if (res < 0) return 0;
    // Level schedule.
    PMB_CUDA(cudaMemsetAsync(I.ws + I.o_lcnt, 0, sizeof(int64_t) * (n + 2), s));
    PMB_CUDA(cudaMemsetAsync(I.ws + I.o_maxl, 0, sizeof(int), s));
    ichol_launch_levels(n, I.at<int>(I.o_level), I.at<int64_t>(I.o_lcnt), I.at<int>(I.o_maxl), s);
    int maxl = 0;
    PMB_CUDA(cudaMemcpyAsync(&maxl, I.ws + I.o_maxl, sizeof(int), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    I.nlevels = maxl + 1;
    if (pmb_scan_exclusive(I.at<int64_t>(I.o_lcnt), I.nlevels + 1, I.at<int64_t>(I.o_scan),
                           I.at<int64_t>(I.o_scan) + (I.nlevels + 1 + 1023) / 1024 + 1, s))
        return fail(kErrCuda, "ichol level scan");
    PMB_CUDA(cudaMemcpyAsync(I.ws + I.o_lfill, I.ws + I.o_lcnt, sizeof(int64_t) * (I.nlevels + 1),
                             cudaMemcpyDeviceToDevice, s));
    ichol_launch_level_scatter(n, I.at<int>(I.o_level), I.at<int64_t>(I.o_lfill), I.at<int>(I.o_order),
                               I.at<int64_t>(I.o_lcnt), I.nlevels, s);
    // Row view of the strictly lower part.
    PMB_CUDA(cudaMemsetAsync(I.ws + I.o_Rp, 0, sizeof(int64_t) * (n + 1), s));
    ichol_launch_rows(n, I.at<int64_t>(I.o_Lp), I.at<int64_t>(I.o_Lr), I.at<double>(I.o_Lv),
                      I.at<int64_t>(I.o_Rp), s);
    if (pmb_scan_exclusive(I.at<int64_t>(I.o_Rp), n + 1, I.at<int64_t>(I.o_scan),
                           I.at<int64_t>(I.o_scan) + (n + 1 + 1023) / 1024 + 1, s))
        return fail(kErrCuda, "ichol row scan");
    PMB_CUDA(cudaMemcpyAsync(I.ws + I.o_rfill, I.ws + I.o_Rp, sizeof(int64_t) * (n + 1),
                             cudaMemcpyDeviceToDevice, s));
    ichol_launch_row_fill(n, I.at<int64_t>(I.o_Lp), I.at<int64_t>(I.o_Lr), I.at<double>(I.o_Lv),
                          I.at<int64_t>(I.o_rfill), I.at<int64_t>(I.o_Rc), I.at<double>(I.o_Rv),
                          I.at<int64_t>(I.o_Rp), s);
    PMB_CUDA(cudaGetLastError());
    return build_stream(I, s);
}

PMB_API int pmb_ichol_levels(const pmb_ichol* p) { return p ? p->I.nlevels : -1; }

PMB_API int pmb_ichol_cluster(const pmb_ichol* p) { return p ? p->I.cluster : -1; }

PMB_API float pmb_ichol_factor_ms(const pmb_ichol* p) { return p ? p->I.factor_ms : -1.0f; }

PMB_API int pmb_ichol_factor_arrays(pmb_ichol* p, void** Lv, void** Lr, void** Lp) {
    if (!p || !p->I.ws || p->I.nnz < 0) return fail(kErrState, "pmb_ichol_factor_arrays: no factor");
    if (Lv) *Lv = p->I.ws + p->I.o_Lv;
    if (Lr) *Lr = p->I.ws + p->I.o_Lr;
    if (Lp) *Lp = p->I.ws + p->I.o_Lp;
    return 0;
}

static int ichol_apply(Ichol& I, const double* b, double* x, const InstState* st, cudaStream_t s) {
    if (I.stream_total > 0) {
        ichol_launch_solve_stream(I.n, I.stream_total, I.first, I.at<unsigned char>(I.o_blob), b, x, st,
                                  kStreamSpinLimit, s);
        return 0;
    }
    ichol_launch_solve(I.n, I.nlevels, I.at<int64_t>(I.o_lcnt), I.at<int>(I.o_order),
                       I.at<int64_t>(I.o_Lp), I.at<int64_t>(I.o_Lr), I.at<double>(I.o_Lv),
                       I.at<int64_t>(I.o_Rp), I.at<int64_t>(I.o_Rc), I.at<double>(I.o_Rv), b, x, st, s);
    return 0;
}

// x = L^-T L^-1 b (CholeskyDecomposition.__call__, ichol.py:175-181).
PMB_API int pmb_ichol_apply(pmb_ichol* p, const double* b, double* x, void* stream) {
    if (!p || !p->I.ws || p->I.nnz < 0 || !b || !x) return fail(kErrArg, "pmb_ichol_apply: bad arguments");
    ichol_apply(p->I, b, x, nullptr, (cudaStream_t)stream);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

PMB_API int pmb_ichol_destroy(pmb_ichol* p) {
    if (p && p->I.ev_f0) {
        cudaEventDestroy(p->I.ev_f0);
        cudaEventDestroy(p->I.ev_f1);
    }
    delete p;
    return 0;
}

// --------------------------------------------------------------------------
// General CSR solver
// --------------------------------------------------------------------------

namespace pmb {

enum : int { kMNone = 0, kMJacobi = 1, kMMatrix = 2, kMIchol = 3, kMExternal = 4 };

struct Csr {
    int64_t n = 0;
    int mkind = 0;
    CsrMat A{}, M{};
    Ichol* ich = nullptr;
    double* vec = nullptr;       // caller block: x r z p0 p1 ap dr invd (8 n)
    const double* invd = nullptr;
    char* ws = nullptr;
    size_t ws_bytes = 0, o_state = 0, o_part = 0;
    int nparts = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    InstState* h_state = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_reorth = -1;
    int reorth = 0;
    double* v(int k) const { return vec + (int64_t)k * n; }
    InstState* state() const { return reinterpret_cast<InstState*>(ws + o_state); }
    double* partials() const { return reinterpret_cast<double*>(ws + o_part); }
};

enum { kVx = 0, kVr, kVz, kVp0, kVp1, kVap, kVdr, kVinvd };

static int csr_prec_kind(const Csr& C) {
    return C.mkind == kMNone ? kCsrPrecNone : (C.mkind == kMJacobi ? kCsrPrecJacobi : kCsrPrecOther);
}

// Internal preconditioners (matrix / ichol): z = M r then r . z -> beta.
static void csr_internal_precond(Csr& C, cudaStream_t s) {
    if (C.mkind == kMMatrix) {
        csr_launch_spmv(C.M, C.n, C.v(kVr), C.v(kVz), C.state(), s);
        csr_launch_rz(C.n, C.v(kVr), C.v(kVz), C.v(kVdr), C.reorth, C.state(), C.partials(), s);
    } else if (C.mkind == kMIchol) {
        ichol_apply(*C.ich, C.v(kVr), C.v(kVz), C.state(), s);
        csr_launch_rz(C.n, C.v(kVr), C.v(kVz), C.v(kVdr), C.reorth, C.state(), C.partials(), s);
    }
}

// Without a preconditioner z is r itself (cg.py:53-55).
static double* csr_z(Csr& C) { return C.mkind == kMNone ? C.v(kVr) : C.v(kVz); }

static void csr_iteration(Csr& C, cudaStream_t s) {
    csr_launch_iteration_head(C.A, C.n, csr_z(C), C.v(kVp0), C.v(kVp1), C.v(kVap), C.state(),
                              C.partials(), s);
    csr_launch_update(csr_prec_kind(C), C.n, C.v(kVx), C.v(kVr), C.v(kVz), C.v(kVp0), C.v(kVp1),
                      C.v(kVap), C.invd, C.v(kVdr), C.reorth, C.state(), C.partials(), s);
    csr_internal_precond(C, s);
}

template <typename Fn>
static int csr_on_stream(Csr& C, cudaStream_t caller, Fn fn) {
    PMB_CUDA(cudaEventRecord(C.ev_in, caller));
    PMB_CUDA(cudaStreamWaitEvent(C.stream, C.ev_in, 0));
    int rc = fn();
    PMB_CUDA(cudaEventRecord(C.ev_out, C.stream));
    PMB_CUDA(cudaStreamWaitEvent(caller, C.ev_out, 0));
    return rc;
}

static int csr_read_state(Csr& C) {
    PMB_CUDA(cudaMemcpyAsync(C.h_state, C.state(), sizeof(InstState), cudaMemcpyDeviceToHost, C.stream));
    PMB_CUDA(cudaStreamSynchronize(C.stream));
    return 0;
}

static int csr_begin(Csr& C, const double* b, const double* x0, double atol, double rtol,
                     int maxiter, int reorth) {
    C.reorth = reorth;
    cudaStream_t s = C.stream;
    csr_launch_init(csr_prec_kind(C), C.A, C.n, b, x0, C.v(kVx), C.v(kVr), C.v(kVz), C.invd,
                    C.state(), C.partials(), atol, rtol, maxiter, s);
    csr_internal_precond(C, s);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace pmb

struct pmb_csr { Csr C; };

PMB_API int pmb_csr_create(int64_t n, int64_t nnz, int preconditioner, pmb_csr** out) {
    if (!out || n <= 0 || preconditioner < 0 || preconditioner > 4)
        return fail(kErrArg, "pmb_csr_create: bad arguments");
    (void)nnz;
    pmb_csr* p = new pmb_csr();
    Csr& C = p->C;
    C.n = n;
    C.mkind = preconditioner;
    C.nparts = csr_partials_count(n);
    Carve c;
    C.o_state = c.take<InstState>(1);
    C.o_part = c.take<double>(3 * (int64_t)C.nparts);
    C.ws_bytes = c.off + 256;
    *out = p;
    return 0;
}

PMB_API int64_t pmb_csr_workspace_bytes(const pmb_csr* p) { return p ? (int64_t)p->C.ws_bytes : -1; }

// vectors: caller block of 8 n doubles (x r z p0 p1 Ap dr invd); the Jacobi
// inverse diagonal, when used, is expected in the invd row. indptr /
// indices / data may be NULL when A is applied by the caller.
PMB_API int pmb_csr_bind(pmb_csr* p, void* workspace, double* vectors, const int64_t* indptr,
                         const int64_t* indices, const double* data) {
    if (!p || !workspace || !vectors) return fail(kErrArg, "pmb_csr_bind: bad arguments");
    Csr& C = p->C;
    C.ws = (char*)workspace;
    C.vec = vectors;
    C.invd = C.v(kVinvd);
    C.A = CsrMat{indptr, indices, data};
    if (!C.stream) {
        PMB_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
        PMB_CUDA(cudaEventCreateWithFlags(&C.ev_in, cudaEventDisableTiming));
        PMB_CUDA(cudaEventCreateWithFlags(&C.ev_out, cudaEventDisableTiming));
        PMB_CUDA(cudaHostAlloc((void**)&C.h_state, sizeof(InstState), cudaHostAllocDefault));
    }
    if (C.graph) {
        cudaGraphExecDestroy(C.graph);
        C.graph = nullptr;
    }
    // Reduction counters must start at zero.
    PMB_CUDA(cudaMemsetAsync(C.ws + C.o_state, 0, sizeof(InstState), C.stream));
    PMB_CUDA(cudaStreamSynchronize(C.stream));
    return 0;
}

PMB_API int pmb_csr_set_matrix_preconditioner(pmb_csr* p, int64_t nnz, const int64_t* indptr,
                                              const int64_t* indices, const double* data,
                                              void* stream) {
    if (!p || !indptr) return fail(kErrArg, "pmb_csr_set_matrix_preconditioner: bad arguments");
    (void)nnz;
    (void)stream;
    p->C.M = CsrMat{indptr, indices, data};
    return 0;
}

PMB_API int pmb_csr_set_ichol(pmb_csr* p, pmb_ichol* f, void* stream) {
    if (!p || !f || f->I.n != p->C.n) return fail(kErrArg, "pmb_csr_set_ichol: size mismatch");
    (void)stream;
    p->C.ich = &f->I;
    return 0;
}

// Full solve on the device (A as a matrix, preconditioner none / Jacobi /
// matrix / ichol). Iterations replay a CUDA graph of 4 iterations.
PMB_API int pmb_csr_solve(pmb_csr* p, const double* b, const double* x0, double* x_out, double atol,
                          double rtol, int maxiter, int reorthogonalize, void* stream) {
    if (!p || !b || !x_out) return fail(kErrArg, "pmb_csr_solve: bad arguments");
    Csr& C = p->C;
    if (!C.A.indptr) return fail(kErrState, "pmb_csr_solve: no matrix bound");
    if (C.mkind == kMExternal) return fail(kErrState, "pmb_csr_solve: external preconditioner needs the step API");
    return csr_on_stream(C, (cudaStream_t)stream, [&]() -> int {
        if (int rc = csr_begin(C, b, x0, atol, rtol, maxiter, reorthogonalize)) return rc;
        const int chunk = 4;
        if (!C.graph || C.graph_reorth != reorthogonalize) {
            if (C.graph) cudaGraphExecDestroy(C.graph);
            C.graph = nullptr;
            cudaGraph_t g;
            PMB_CUDA(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < chunk; ++i) csr_iteration(C, C.stream);
            PMB_CUDA(cudaStreamEndCapture(C.stream, &g));
            PMB_CUDA(cudaGraphInstantiate(&C.graph, g, 0));
            cudaGraphDestroy(g);
            C.graph_reorth = reorthogonalize;
        }
        int done = 0;
        for (;;) {
            if (int rc = csr_read_state(C)) return rc;
            if (C.h_state->status != kRunning) break;
            if (done > maxiter + chunk) return fail(kErrState, "iteration control lost");
            PMB_CUDA(cudaGraphLaunch(C.graph, C.stream));
            done += chunk;
        }
        PMB_CUDA(cudaMemcpyAsync(x_out, C.v(kVx), sizeof(double) * C.n, cudaMemcpyDeviceToDevice, C.stream));
        return 0;
    });
}

// Step interface for callers that apply A or M themselves (Python
// callables): begin / step / finish_precondition; the vectors are the rows
// of the caller's block.
PMB_API int pmb_csr_begin(pmb_csr* p, const double* b, const double* x0, double atol, double rtol,
                          int maxiter, int reorthogonalize, void* stream) {
    if (!p || !b) return fail(kErrArg, "pmb_csr_begin: bad arguments");
    Csr& C = p->C;
    return csr_on_stream(C, (cudaStream_t)stream, [&]() -> int {
        if (!C.A.indptr) {
            // x0 is applied by the caller: r = b - A x0 arrives as b.
            CsrMat none{};
            csr_launch_init(csr_prec_kind(C), none, C.n, b, nullptr, C.v(kVx), C.v(kVr), C.v(kVz),
                            C.invd, C.state(), C.partials(), atol, rtol, maxiter, C.stream);
            C.reorth = reorthogonalize;
            csr_internal_precond(C, C.stream);
            if (x0)
                PMB_CUDA(cudaMemcpyAsync(C.v(kVx), x0, sizeof(double) * C.n, cudaMemcpyDeviceToDevice, C.stream));
            return 0;
        }
        return csr_begin(C, b, x0, atol, rtol, maxiter, reorthogonalize);
    });
}

// mode 0: full iteration with the bound matrix; 1: build p only (caller
// then writes A p into the Ap row); 2: finish after an external A p.
PMB_API int pmb_csr_step(pmb_csr* p, int mode, void* stream) {
    if (!p) return fail(kErrArg, "pmb_csr_step: bad arguments");
    Csr& C = p->C;
    return csr_on_stream(C, (cudaStream_t)stream, [&]() -> int {
        cudaStream_t s = C.stream;
        if (mode == 0) {
            csr_iteration(C, s);
        } else if (mode == 1) {
            csr_launch_pupdate(C.n, csr_z(C), C.v(kVp0), C.v(kVp1), C.state(), s);
        } else {
            csr_launch_pap(C.n, C.v(kVp0), C.v(kVp1), C.v(kVap), C.state(), C.partials(), s);
            csr_launch_update(csr_prec_kind(C), C.n, C.v(kVx), C.v(kVr), C.v(kVz), C.v(kVp0),
                              C.v(kVp1), C.v(kVap), C.invd, C.v(kVdr), C.reorth, C.state(),
                              C.partials(), s);
            csr_internal_precond(C, s);
        }
        PMB_CUDA(cudaGetLastError());
        return 0;
    });
}

// After the caller wrote z = M r into the z row: r . z and beta.
PMB_API int pmb_csr_finish_precondition(pmb_csr* p, void* stream) {
    if (!p) return fail(kErrArg, "pmb_csr_finish_precondition: bad arguments");
    Csr& C = p->C;
    return csr_on_stream(C, (cudaStream_t)stream, [&]() -> int {
        csr_launch_rz(C.n, C.v(kVr), C.v(kVz), C.v(kVdr), C.reorth, C.state(), C.partials(), C.stream);
        PMB_CUDA(cudaGetLastError());
        return 0;
    });
}

// Which parity buffer holds the current search direction p.
PMB_API int pmb_csr_p_index(pmb_csr* p) {
    if (!p) return -1;
    if (int rc = csr_read_state(p->C)) return rc;
    // After pupdate at iteration k the new p sits in buffer (k & 1) ^ 1.
    return ((p->C.h_state->iters & 1) ^ 1);
}

PMB_API int pmb_csr_stats(pmb_csr* p, int* iters, int* status, double* norm_r, double* norm_b) {
    if (!p) return fail(kErrArg, "pmb_csr_stats: bad arguments");
    Csr& C = p->C;
    if (int rc = csr_read_state(C)) return rc;
    if (iters) *iters = C.h_state->iters;
    if (status) *status = C.h_state->status;
    if (norm_r) *norm_r = C.h_state->norm_r;
    if (norm_b) *norm_b = C.h_state->norm_b;
    return 0;
}

PMB_API int pmb_csr_destroy(pmb_csr* p) {
    if (!p) return 0;
    Csr& C = p->C;
    if (C.graph) cudaGraphExecDestroy(C.graph);
    if (C.stream) {
        cudaStreamSynchronize(C.stream);
        cudaStreamDestroy(C.stream);
    }
    if (C.ev_in) cudaEventDestroy(C.ev_in);
    if (C.ev_out) cudaEventDestroy(C.ev_out);
    if (C.h_state) cudaFreeHost(C.h_state);
    delete p;
    return 0;
}

PMB_API int pmb_csr_spmv(int64_t n, const int64_t* indptr, const int64_t* indices,
                         const double* data, const double* x, double* y, void* stream) {
    if (n <= 0 || !indptr || !x || !y) return fail(kErrArg, "pmb_csr_spmv: bad arguments");
    csr_launch_spmv(CsrMat{indptr, indices, data}, n, x, y, nullptr, (cudaStream_t)stream);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

PMB_API int pmb_csr_inv_diag(int64_t n, const int64_t* indptr, const int64_t* indices,
                             const double* data, double* invd, void* stream) {
    if (n <= 0 || !indptr || !invd) return fail(kErrArg, "pmb_csr_inv_diag: bad arguments");
    csr_launch_inv_diag(CsrMat{indptr, indices, data}, n, invd, (cudaStream_t)stream);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

PMB_API int pmb_vec_mul(int64_t n, const double* a, const double* b, double* out, void* stream) {
    if (n <= 0 || !a || !b || !out) return fail(kErrArg, "pmb_vec_mul: bad arguments");
    csr_launch_vec_mul(n, a, b, out, (cudaStream_t)stream);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

// 1 / diagonal of a half-stencil operator, in user layout (jacobi.py:24-26).
namespace pmb {
__global__ void k_planes_inv_diag(const double* __restrict__ P, int h, int w, int pitch, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w) return;
    const int y = (int)(i / w), x = (int)(i % w);
    out[i] = 1.0 / P[(int64_t)y * pitch + x];
}
}  // namespace pmb

PMB_API int pmb_planes_inv_diag(const double* planes, int h, int w, double* inv_diag, void* stream) {
    if (!planes || !inv_diag || h <= 0 || w <= 0) return fail(kErrArg, "pmb_planes_inv_diag: bad arguments");
    const int64_t n = (int64_t)h * w;
    k_planes_inv_diag<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(planes, h, w, pitch_for(w), inv_diag);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

// Canonical CSR of A + diag(c) (rows of at most 64 stored entries):
// rowptr (n+1) and an overflow flag first, then the entries.
PMB_API int pmb_csr_add_diag_rowptr(int64_t n, const int64_t* indptr, const int64_t* indices,
                                    const double* data, const double* c, int64_t* rowptr,
                                    int* overflow, int64_t* scratch, void* stream) {
    if (n <= 0 || !indptr || !c || !rowptr || !overflow || !scratch)
        return fail(kErrArg, "pmb_csr_add_diag_rowptr: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    PMB_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), s));
    PMB_CUDA(cudaMemsetAsync(rowptr + n, 0, sizeof(int64_t), s));
    csr_launch_add_diag_count(CsrMat{indptr, indices, data}, n, c, rowptr, overflow, s);
    if (pmb_scan_exclusive(rowptr, n + 1, scratch, scratch + (n + 1 + 1023) / 1024 + 1, s))
        return fail(kErrCuda, "scan");
    PMB_CUDA(cudaGetLastError());
    return 0;
}

PMB_API int pmb_csr_add_diag_fill(int64_t n, const int64_t* indptr, const int64_t* indices,
                                  const double* data, const double* c, const int64_t* rowptr,
                                  int64_t* out_indices, double* out_data, void* stream) {
    if (n <= 0 || !indptr || !c || !rowptr) return fail(kErrArg, "pmb_csr_add_diag_fill: bad arguments");
    csr_launch_add_diag_fill(CsrMat{indptr, indices, data}, n, c, rowptr, out_indices, out_data,
                             (cudaStream_t)stream);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

int pmb_launch_selftest_poll(void*, unsigned long long, int*, cudaStream_t);

// Bounded-wait self-test: which = 0 runs the mbarrier wait of the TMA
// kernels with a limit of `limit` polls, which = 1 the epoch poll of the
// foreground sweep with a deadline of `limit` nanoseconds, which = 2 the
// chunk wait of the streamed ichol solve (`limit` polls) on a chunk whose
// copy is never issued; each waits on a barrier or word that nothing
// completes. *timed_out = 1 when the wait gave up and reported it (every
// waiting thread, for the mbarrier; a NaN result, for the solve). scratch:
// 64 bytes of device memory.
PMB_API int pmb_selftest_wait(int which, int64_t limit, void* scratch, int* timed_out,
                              void* stream) {
    if (!scratch || !timed_out || limit <= 0 || which < 0 || which > 2)
        return fail(kErrArg, "pmb_selftest_wait: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    *timed_out = 0;
    if (which == 2) {
        if (limit > 0x7fffffff) return fail(kErrArg, "pmb_selftest_wait: poll limit too large");
        ichol_prepare();
        double* v = static_cast<double*>(scratch);
        PMB_CUDA(cudaMemsetAsync(v, 0, 8 * sizeof(double), s));
        StreamFirst first{};    // one chunk, never fetched
        ichol_launch_solve_stream(4, 1, first, static_cast<const unsigned char*>(scratch), v, v + 4,
                                  nullptr, (uint32_t)limit, s);
        PMB_CUDA(cudaGetLastError());
        double h = 0.0;
        PMB_CUDA(cudaMemcpyAsync(&h, v + 4, sizeof(double), cudaMemcpyDeviceToHost, s));
        PMB_CUDA(cudaStreamSynchronize(s));
        *timed_out = std::isnan(h) ? 1 : 0;
        return 0;
    }
    if (which == 1) {
        const int rc = pmb_launch_selftest_poll(scratch, (unsigned long long)limit, timed_out, s);
        if (rc) return fail(kErrCuda, std::string("poll self-test: ") +
                                          cudaGetErrorString((cudaError_t)rc));
        return 0;
    }
    if (limit > 0x7fffffff) return fail(kErrArg, "pmb_selftest_wait: poll limit too large");
    int* gave_up = static_cast<int*>(scratch);
    PMB_CUDA(cudaMemsetAsync(gave_up, 0, sizeof(int), s));
    launch_selftest_mbar((uint32_t)limit, gave_up, s);
    PMB_CUDA(cudaGetLastError());
    int h = 0;
    PMB_CUDA(cudaMemcpyAsync(&h, gave_up, sizeof(int), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    *timed_out = h == 64 ? 1 : 0;
    return 0;
}

// Half-stencil planes of an (h w) x (h w) CSR matrix of a pixel grid (the
// form vcycle needs, pymatting/preconditioner/vcycle.py:103-153 takes any A
// of that shape). planes: 13 h pitch doubles, back: 12 h pitch doubles of
// scratch; bad[0] counts entries outside the 5x5 neighbourhood, bad[1] the
// forward/backward pairs that differ by more than rel_tol (relative).
PMB_API int pmb_csr_to_planes(const int64_t* indptr, const int64_t* indices, const double* data,
                              int h, int w, double* planes, double* back, double rel_tol,
                              unsigned long long* bad, void* stream) {
    if (!indptr || !planes || !back || !bad || h <= 0 || w <= 0)
        return fail(kErrArg, "pmb_csr_to_planes: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t ps = (int64_t)h * pitch_for(w);
    PMB_CUDA(cudaMemsetAsync(planes, 0, sizeof(double) * kNH * ps, s));
    PMB_CUDA(cudaMemsetAsync(back, 0, sizeof(double) * (kNH - 1) * ps, s));
    PMB_CUDA(cudaMemsetAsync(bad, 0, 2 * sizeof(unsigned long long), s));
    csr_launch_to_planes(CsrMat{indptr, indices, data}, h, w, pitch_for(w), planes, back, rel_tol,
                         bad, s);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

// x = A^-1 b for a small square CSR matrix (n <= 4096). scratch: n*n
// doubles; x holds b on entry; *singular set to 1 for a zero pivot.
PMB_API int pmb_dense_solve(int64_t n, const int64_t* indptr, const int64_t* indices,
                            const double* data, double* scratch, double* x, int* singular,
                            void* stream) {
    if (n <= 0 || n > 4096 || !indptr || !scratch || !x || !singular)
        return fail(kErrArg, "pmb_dense_solve: bad arguments (n must be in [1, 4096])");
    cudaStream_t s = (cudaStream_t)stream;
    PMB_CUDA(cudaMemsetAsync(singular, 0, sizeof(int), s));
    csr_launch_dense_solve(CsrMat{indptr, indices, data}, n, scratch, x, singular, s);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

namespace pmb {
__global__ void k_mask_scale(const uint8_t* __restrict__ m, int64_t n, double v, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = m[i] ? v : 0.0;
}
__global__ void k_clip01(const double* __restrict__ x, int64_t n, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        const double v = x[i];
        out[i] = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    }
}
}  // namespace pmb

// out = value * mask (b = lambda * is_fg of laplacian.py:48).
PMB_API int pmb_mask_scale(const uint8_t* mask, int64_t n, double value, double* out, void* stream) {
    if (!mask || !out || n <= 0) return fail(kErrArg, "pmb_mask_scale: bad arguments");
    k_mask_scale<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(mask, n, value, out);
    PMB_CUDA(cudaGetLastError());
    return 0;
}

// out = clip(x, 0, 1) (estimate_alpha_cf.py:76).
PMB_API int pmb_clip01(const double* x, int64_t n, double* out, void* stream) {
    if (!x || !out || n <= 0) return fail(kErrArg, "pmb_clip01: bad arguments");
    k_clip01<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, n, out);
    PMB_CUDA(cudaGetLastError());
    return 0;
}


// Average duration (ms) of the level-0 operator apply y = A x over `iters`
// back-to-back launches on the solver's stream, timed with CUDA events on
// that stream. The solver's inner precision decides FP64 or FP32. Used by
// the benchmark to relate the Laplacian apply to the HBM roofline.
// Milliseconds per iteration spent in each kind of launch (kPkCount values:
// CG apply, CG update, refinement, restriction from level 0, restriction
// from coarser levels, tail, direct solves, prolongation at coarser levels,
// prolongation at level 0, other), over `iters` live iterations of a solve
// of A x = b. Each launch is followed by an event on the solver's stream and
// charged with the time since the previous event. The iterations run one by
// one (not from the captured graph), so launch gaps are included; images
// that converge within `iters` make later launches cheaper. Leaves the
// solver mid-solve (the next solve starts afresh).
PMB_API int pmb_stencil_profile(pmb_stencil* p, const double* b, int iters, double* ms_out,
                                void* stream) {
    if (!p || !b || !ms_out || iters <= 0) return fail(kErrArg, "pmb_stencil_profile: bad arguments");
    Stencil& S = p->S;
    if (!S.bound) return fail(kErrState, "pmb_stencil_profile: not bound");
    return on_stream(S, (cudaStream_t)stream, [&]() -> int {
        if (!S.setup_done) {
            if (int rc = setup_stencil(S)) return rc;
        }
        HostList& a = S.fine0;
        cudaStream_t s = S.stream;
        launch_pack<double, double>(a.wl.grids, a.wl.ngrids, S.at<int64_t>(S.o_uoff), b,
                                    S.at<double>(S.o_b64), S.user_total, s);
        if (S.precision == 0) start_fp64(S, nullptr, 0.0, 1e-30, 1 << 30);
        else if (int rc = start_mixed(S, nullptr, 0.0, 1e-30, 1 << 30, 1e-4, 1 << 20)) return rc;
        std::vector<std::pair<int, cudaEvent_t>> marks;
        S.prof = &marks;
        prof_mark(S, -1);
        for (int i = 0; i < iters; ++i) {
            if (S.precision == 0) cg_iteration<double>(S, 0);
            else cg_iteration<float>(S, 0);
        }
        S.prof = nullptr;
        cudaError_t e = cudaStreamSynchronize(s);
        for (int k = 0; k < kPkCount; ++k) ms_out[k] = 0.0;
        for (size_t i = 1; i < marks.size() && e == cudaSuccess; ++i) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, marks[i - 1].second, marks[i].second) == cudaSuccess)
                ms_out[marks[i].first] += (double)t / iters;
        }
        for (auto& m : marks) cudaEventDestroy(m.second);
        PMB_CUDA(e);
        PMB_CUDA(cudaGetLastError());
        return check_err(S);
    });
}

PMB_API int pmb_stencil_time_apply(pmb_stencil* p, int iters, double* ms, void* stream) {
    if (!p || iters <= 0 || !ms) return fail(kErrArg, "pmb_stencil_time_apply: bad arguments");
    Stencil& S = p->S;
    if (!S.bound) return fail(kErrState, "pmb_stencil_time_apply: not bound");
    return on_stream(S, (cudaStream_t)stream, [&]() -> int {
        if (!S.setup_done) {
            if (int rc = setup_stencil(S)) return rc;
        }
        cudaEvent_t e0, e1;
        PMB_CUDA(cudaEventCreate(&e0));
        PMB_CUDA(cudaEventCreate(&e1));
        HostList& a = S.fine0;
        const LaunchCfg L{grid_for(a, S.precision == 0 ? smem_apply_v<double>(2)
                                                      : smem_apply_v<float>(2))};
        auto launch = [&]() {
            if (S.precision == 0)
                launch_apply<double>(L, a.wl, S.maps(), S.at<double>(S.o_ap64), S.err(), S.stream);
            else
                launch_apply<float>(L, a.wl, S.maps(), S.at<float>(S.o_ap32), S.err(), S.stream);
        };
        launch();
        PMB_CUDA(cudaEventRecord(e0, S.stream));
        for (int i = 0; i < iters; ++i) launch();
        PMB_CUDA(cudaEventRecord(e1, S.stream));
        PMB_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        PMB_CUDA(cudaEventElapsedTime(&t, e0, e1));
        *ms = (double)t / iters;
        S.launches += iters + 1;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        PMB_CUDA(cudaGetLastError());
        return check_err(S);
    });
}
