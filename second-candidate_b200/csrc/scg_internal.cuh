// Internal declarations shared by the CUDA translation units of libscgpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "scg.h"

namespace scg {

// ---------------------------------------------------------------------------
// Host-side error plumbing

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define SCG_CUDA(call)                                         \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return ::scg::cuda_fail(_e, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// Device helpers

// Order-preserving map of a float onto uint32 (negative zero maps as zero).
__device__ __forceinline__ uint32_t f2o(float f) {
    uint32_t u = __float_as_uint(f);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(u);
}

// Status word bits written by kernels (never a trap).
enum : int {
    ST_OK = 0,
    ST_CELL_BUDGET = 1,   // a query enumerated more cells than the budget
    ST_TIE_OVERFLOW = 2,  // more exact key ties at the cut than the tie buffer
    ST_ITER_CAP = 4,      // an iteration cap was reached
    ST_BAD_ARG = 8,
    ST_TC_TIMEOUT = 16,   // a tensor-core completion wait expired
    ST_POOL = 32,         // the split kernels' visited-list pool ran out (the batch reruns fused)
};

// ---------------------------------------------------------------------------
// Kernel launch wrappers (defined in the .cu files)

struct TablesArgs {
    int dim, mc, kc, mp, kp, nq;
    const float *Q;        // [nq][dim]
    const float *cq, *pq;  // codebooks
    const float *norm_c, *norm_r;
    float *dqc;            // [nq][mc*kc]
    float *dqr;            // [nq][mp*kp]
    float *qn;             // [nq][2] half norms (IMI) or [nq][2] = {q_sum, 0}
    float *qsum;           // [nq]
    int lut_only;          // 1: dqr holds -2<q,r> (the fast form keeps ||r||^2 per vector)
    int *status;           // optional status word (ST_* bits)
    int segs;              // tensor-core tables: 0 or 3 both, 1 coarse parts only, 2 PQ subspaces only
};

void launch_precompute1(int dim, int mc, int kc, int mp, int kp, const float *cq, const float *pq,
                        float *norm_c, float *norm_r, float *dot_cr, cudaStream_t s);
void launch_tables_exact(const TablesArgs &a, cudaStream_t s);
// Tensor-core tables: nsplit 3 (hi/lo split, FP32-accurate) or 1; fmt 1 = bf16, 0 = f16.
void launch_tables_tc(const TablesArgs &a, int nsplit, int fmt, cudaStream_t s);
void launch_query_norms(const TablesArgs &a, cudaStream_t s);
void launch_vterm(int mode, int kc, int mp, int kp, int mc, uint64_t ncells, int64_t N, const uint32_t *off,
                  const uint8_t *codes, const float *norm_r, const float *dot_cr, float *vterm, cudaStream_t s);

// One query's visited-cell list as the selection kernel leaves it.
struct QMeta {
    uint32_t off;   // start of the list in the pool
    int nvis;       // visited non-empty cells
    uint32_t svis;  // their candidates
    int err;        // the selection failed (outputs void)
};

struct SearchArgs {
    int mode, dim, mc, kc, mp, kp, nq, R, w, T;
    int precision;
    int rot;                // the fast form's rotated, bank-private LUT (kp == 256, mp in {8, 16, 32})
    int upl;                // candidates per lane per scan chunk: 2, 4 or 8
    int shortlist;          // 1: the R best feed the exact re-rank, which orders them itself
    const int *Tq;          // optional per-query T
    int rank_limit;         // IMI / second candidate: walk ranks < rank_limit of each list (0: all)
    const uint64_t *slist;  // optional coarse-list prefixes sorted ahead: [nq][lists][slist_w]
    const uint32_t *smeta;  // their lengths and next high words: [nq][lists][2]
    int slist_w;
    const float *dqc, *dqr, *qn, *qsum;
    const uint32_t *off;    // [ncells+1] exclusive offsets
    const int *pid;
    const uint8_t *codes;
    const float *dot_cr;
    const float *vterm;     // per-vector term of the fast form (may be null)
    // exact-distance scan (the real_dist branch for every candidate):
    // raw_dim > 0 scores each candidate against its raw row instead of ADC
    const float *Q;         // [nq][raw_dim] queries
    const void *raw;        // [N][raw_dim] raw rows by id, float or uint8
    int raw_u8, raw_dim;
    uint64_t ncells;
    int64_t N;
    // per-CTA scratch slots
    uint32_t *rec_key, *rec_rank, *rec_cnt;  // [slots][cap_rec]
    uint32_t *vis_cell, *vis_pre;            // [slots][cap_rec + 1]
    int cap_rec;
    uint64_t *pend;                          // [slots][pcap] scan survivors
    uint32_t pcap;
    // optional hand-off to the merge kernel (scan-only kernel): a query with
    // at most surv_cap survivors copies them to surv[q] and sets surv_n[q];
    // surv_n[q] = -1: the scan kernel merged and wrote the outputs itself
    uint64_t *surv;                          // [nq][surv_cap]
    int *surv_n;                             // [nq]
    int surv_cap;
    // selection -> scan hand-off of the split kernels (parts 1 and 2)
    QMeta *qmeta;                            // [nq]
    uint32_t *pool_cell, *pool_pre;          // [nq * pool_stride + pool_over_cap] visited lists
    uint32_t pool_stride;                    // each query's own region
    uint32_t *pool_over;                     // allocation counter of the overflow area
    uint32_t pool_over_cap;
    int *qcounter;                           // dynamic query counter
    const int *qlist;                        // optional: qlist[0] queries qlist[1..] instead of 0..nq-1
    // outputs
    int *out_ids;
    float *out_d;
    int *out_sum, *out_nvis, *out_empty;
    int *status;
    long long *phase_cycles;  // optional [16] counters
    unsigned long long *dens_acc;  // optional: adds each query's (candidates, cells)
};

// part 0: fused selection + scan; 1: selection only; 2: scan only.  rot:
// the scan uses the fast form's rotated LUT (search_rot_form).
// qdim > 0: the exact-distance scan over raw rows of qdim floats.
size_t search_smem_bytes(int mode, int kc, int mp, int kp, int part, int rot, int qdim);
int search_launch(const SearchArgs &a, int part, int grid, cudaStream_t s);
int search_max_blocks_per_sm(int mode, int kc, int mp, int kp, int upl, int part, int rot, int qdim = 0);
// Whether searches in `precision` on this shape use the rotated LUT.
bool search_rot_form(int precision, int mp, int kp);
// Warp-per-query cell selection (part 1) for IVFADC, IMI and the
// second-candidate walk with coarse prefixes sorted ahead: whether it serves
// the shape, its launch (queries it cannot finish are appended to
// defer[1..], defer[0] counting them) and its resident CTAs per SM.
bool select_warp_serves(int mode, int kc);
// Top-R of the survivors handed over by the scan-only kernel, one warp per
// query (R <= 256, outputs in (distance, id) order).
constexpr int SURV_CAP = 1024;
void merge_warp_launch(const uint64_t *surv, const int *surv_n, int cap, const int *pid, int nq, int R,
                       int *out_ids, float *out_d, int nsm, cudaStream_t s);
int select_warp_launch(const SearchArgs &a, int *defer, int grid, cudaStream_t s);
int select_warp_blocks_per_sm();

struct EncodeArgs {
    int dim, mc, kc, mp, kp, nc;  // nc = 0: IVF/IMI encoder; nc >= 2: SC encoder
    int64_t n;
    const float *X, *cq, *pq;
    uint16_t *cid;
    uint8_t *codes;
};
void launch_encode(const EncodeArgs &a, cudaStream_t s);
// Shared memory of the exact encoder's block for this shape (must be <= 227 KB).
size_t encode_smem_bytes(int dim, int mcp);
// ||c||^2 of `rows` vectors of length len (the reference's float order).
void launch_norms(const float *C, int rows, int len, float *out, cudaStream_t s);

// Nearest centroid(s) per (row, segment) from a tensor-core distance table,
// re-checked exactly: every centroid whose table value is within the
// table's error margin of the nbest-th smallest is scored with the
// reference's double arithmetic and the nbest smallest (distance, id) win.
struct PickArgs {
    const float *X;        // [n][dim] rows (or residuals)
    int64_t n;
    int dim, nseg, kseg, len;  // segments per row, centroids per segment, dims per segment
    const float *C;        // [nseg][kseg][len]
    const float *tab;      // [n][nseg * kseg]: ||c||^2 - 2<x_seg, c>
    const float *segmax;   // [nseg] largest ||c||^2 of the segment
    uint16_t *cid;         // [n][nseg] (coarse) or null
    uint8_t *code;         // [n][nseg] (PQ) or null
    float *resid;          // [n][dim] x - c for the chosen c (coarse), or null
    int *status;
    int nbest = 1;         // centroids kept per (row, segment), 1..3 (cid holds [n][nseg][nbest])
    int fcmp = 0;          // compare float-rounded distances (the second-candidate encoder)
};
void launch_pick(const PickArgs &a, cudaStream_t s);
void launch_segmax(const float *norms, int nseg, int kseg, float *out, cudaStream_t s);

// Sorted coarse-list prefixes of a batch, ahead of the fused search
// (kc <= 1024; width = coarse_sort_width(kc), 0 when kc is larger).
struct CoarseArgs {
    const float *dqc, *qn, *qsum;
    int nq, kc, mc, imi;
    const int *Tq;       // optional per-query T
    int T;
    double avg_density;  // N / cells, for the prefix length rule
    const unsigned long long *dens_acc;  // optional: candidates, cells seen so far
    int max_prefix;
    int fixed_prefix;    // > 0: this prefix length instead of the density rule
    int width;           // stride of a list in out
    uint64_t *out;       // [nq][lists][width] sorted prefix keys
    uint32_t *meta;      // [nq][lists][2]: prefix length, smallest high word after it
};
int coarse_sort_width(int kc);
void launch_coarse_prefix(const CoarseArgs &a, cudaStream_t s);

// Index build (build_index.cu): rows ordered by cell, CSR offsets.
size_t build_work_bytes(int64_t n, int64_t ncells);
void launch_build_csr(const uint16_t *cid, const uint8_t *codes, int64_t n, int parts, int kc, int mp,
                      int64_t ncells, unsigned char *work, uint32_t *off, int *pid, uint8_t *codes_out, cudaStream_t s);

// Codebook training (train.cu).
size_t kmeans_work_bytes(int64_t n, int nseg, int k, int len, int64_t chunk);
int kmeans_segments(const float *X, int64_t n, int dim, int nseg, int k, int iters, uint64_t seed, float *C,
                    unsigned char *work, int64_t chunk, int *status, int *asg_out, cudaStream_t s);
void launch_residual(const float *X, int64_t n, int dim, int nseg, int k, const float *C, const int *asg, float *R,
                     cudaStream_t s);

// Exact nearest neighbour (gt.cu).
size_t exact_nn_work_bytes(int nq, int64_t chunk);
int exact_nn(const float *X, int64_t n, const float *Q, int nq, int dim, int *ids, float *dists, unsigned char *work,
             int64_t chunk, int *status, cudaStream_t s);

size_t rerank_smem_bytes(int L, int dim);
int launch_rerank(const float *Q, int nq, int dim, const void *raw, int raw_u8, int64_t N, const int *sl_ids, int L,
                  int R, int *out_ids, float *out_d, int *status, cudaStream_t s);

}  // namespace scg
