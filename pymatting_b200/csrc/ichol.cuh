// Launch interface of the incomplete-Cholesky kernels (ichol.cu).
#pragma once

#include "pm_common.cuh"

namespace pmb {

// Streamed solves: chunk limits, stages in flight and the largest system
// whose x fits in shared memory beside the stages.
constexpr int kStreamRowsMax = 64;
constexpr int kStreamEntsMax = 512;
constexpr int kStreamStages = 8;
constexpr int64_t kStreamMaxRows = 20000;
constexpr uint32_t kStreamSpinLimit = 1u << 24;

// Records of a chunk block: its head, then one per row.
struct StreamHead {
    int64_t next_off;      // byte offset of the chunk kStreamStages later
    int next_bytes;        // its size (0: none)
    int rows, ents;        // this chunk
    int pad[3];
};
struct StreamRow {
    int row, start, count, pad;
    double diag, pad2;
};
static_assert(sizeof(StreamHead) == 32 && sizeof(StreamRow) == 32, "chunk records are 32 bytes");

// Offsets and sizes of the first kStreamStages chunk blocks (later ones are
// named by the block kStreamStages before them).
struct StreamFirst {
    int64_t off[kStreamStages];
    int bytes[kStreamStages];
};
// Host-built packing plan: one record per row of each sweep, one per chunk.
struct StreamPackRow {
    int64_t chunk_off;   // byte offset of the row's chunk block
    int64_t src;         // first entry in the row view (forward) or column of L (backward)
    int row, slot, start, count;
    int rows, ents;      // of the row's chunk
    int backward, pad;
};
struct StreamPackChunk {
    int64_t off;
    int bytes, rows, ents, used;   // used: entries before padding
};

size_t ichol_stream_smem(int64_t n);
void ichol_launch_stream_pack(int nrec, const StreamPackRow* recs, int nchunks,
                              const StreamPackChunk* chunks, const int64_t* Rc, const double* Rv,
                              const int64_t* Lr, const double* Lv, const int64_t* Lp,
                              unsigned char* blob, cudaStream_t s);
void ichol_launch_solve_stream(int64_t n, int total, const StreamFirst& first,
                               const unsigned char* blob, const double* b, double* x,
                               const InstState* st, uint32_t limit, cudaStream_t s);

void ichol_launch_init(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                       double shift, double* d, double* rsum, int* level, unsigned long long* band,
                       cudaStream_t s);
// Returns the cluster size of the kernel launched (0: the global-front kernel).
int ichol_launch_factor(int64_t n, int64_t W, const int64_t* Ap, const int64_t* Ar,
                        const double* Av, double* d, const double* rsum, int* level, double* F,
                        uint8_t* pat, int* cand, double* keptv, int64_t* kepti, int64_t* Lp,
                        int64_t* Lr, double* Lv, int64_t cap, double discard, int64_t max_nnz,
                        double rel, int diag_keep, int64_t* result, cudaStream_t s);
void ichol_launch_levels(int64_t n, const int* level, int64_t* cnt, int* maxlevel, cudaStream_t s);
void ichol_launch_level_scatter(int64_t n, const int* level, int64_t* fill, int* order,
                                const int64_t* lptr, int nlevels, cudaStream_t s);
void ichol_launch_rows(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                       int64_t* rcnt, cudaStream_t s);
void ichol_launch_row_fill(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                           int64_t* rfill, int64_t* Rc, double* Rv, const int64_t* Rp,
                           cudaStream_t s);
// Cluster size of the on-chip factorisation for bandwidth W - 1; 0 = global front.
int ichol_cluster_size(int64_t W);
void ichol_prepare();
void ichol_launch_solve(int64_t n, int nlevels, const int64_t* lptr, const int* order,
                        const int64_t* Lp, const int64_t* Lr, const double* Lv, const int64_t* Rp,
                        const int64_t* Rc, const double* Rv, const double* b, double* x,
                        const InstState* st, cudaStream_t s);

}  // namespace pmb
