// Host-side state of the library: the index handle, per-stream search
// workspaces, and the internal entry points shared by api.cu (the C ABI) and
// server.cu (the request loop).
#pragma once

#include <atomic>
#include <mutex>
#include <string>

#include "scg_internal.cuh"

namespace scg {

// cudaMalloc calls made for the library's own device buffers in this
// process (scg_device_allocations).
inline std::atomic<long long> g_device_allocs{0};

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes) {
        if (bytes <= n) return SCG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        g_device_allocs.fetch_add(1, std::memory_order_relaxed);
        n = bytes;
        return SCG_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T>
    T *as() const {
        return (T *)p;
    }
};

// Everything one in-flight batched search writes besides its outputs: the
// per-CTA traversal slots, the status word, the query counter, and (unless
// the caller supplies them) the per-query tables.  One per stream of work.
struct Workspace {
    DevBuf dqc, dqr, qn, qsum, nvis, empty, status, counter;
    DevBuf rec_key, rec_rank, rec_cnt, vis_cell, vis_pre, pend, phase, sl_ids, sl_d, slist, smeta;
    DevBuf qmeta, pool_cell, pool_pre;  // selection -> scan hand-off of the split kernels
    DevBuf defer;  // queries the warp-wide selection left to the block-wide one: [0] count, [1..nq]
    DevBuf surv, surv_n;  // survivors the scan kernel hands to the merge kernel: [nq][SURV_CAP], [nq]
    int *h_status = nullptr;  // pinned copy of the status word
    // events: before tables, after tables, after selection + scan, after
    // re-rank, between the selection and scan kernels (split launches)
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool last_split = false;
    int last_launches = 0;  // kernels the last run_search on this workspace launched
    int last_nq = 0;
    bool phase_on = false;
    int init();
    void release();
};

// Per-request buffers carved by a caller (the request loop's arena); when
// given, run_search uses them instead of growing the workspace.
struct ReqBufs {
    float *dqc, *dqr, *qn, *qsum;
    int *nvis, *empty;
    int *sl_ids;   // [nq][L] when re-ranking
    float *sl_d;
    uint64_t *slist;  // [nq][lists][width] sorted coarse-list prefixes (kc <= 1024)
    uint32_t *smeta;  // [nq][lists][2] their lengths and next high words
};

// Device bytes of the ReqBufs of one request.
size_t req_bytes(int nq, int dim, int mc, int kc, int mp, int kp, int R, int rerank);
// Carves ReqBufs for nq queries from base (256-byte aligned pieces).
ReqBufs carve_req(unsigned char *base, int nq, int mc, int kc, int mp, int kp, int rerank);

}  // namespace scg

struct scg_index {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    int dim = 0, mc = 0, kc = 0, mp = 0, kp = 0;
    int64_t N = 0;
    int64_t ncells = 0;
    bool have_codebooks = false, have_csr = false, precomputed = false;
    int cap_rec = 131072;
    const int *d_Tq = nullptr;
    int rank_limit = 0;  // scg_set_rank_limit: walk ranks < M of each coarse list (0: all)
    int prefix_len = 0;  // sorted coarse-prefix length (0: the density rule; scg_autotune_ex)
    scg::DevBuf cq, pq, norm_c, norm_r, dot_cr, off, pid, codes, raw, vterm;
    // candidates and cells seen by the selection so far (u64 x 2): the
    // coarse prefix length rule uses their ratio instead of N / cells
    scg::DevBuf dens;
    bool have_vterm = false;
    int64_t raw_rows = 0;   // rows of raw vectors loaded (0: none)
    bool raw_u8 = false;    // raw vectors held as uint8
    int tuned_upl[2] = {2, 2};  // scan candidates per lane, per scan form (exact, fast)
    bool split = true;          // selection and scan as two kernels where possible
    // tensor-core encoder (IVF/IMI codes): norms, per-segment maxima, chunk buffers
    int encoder = 1;            // SCG_ENC_TENSOR or SCG_ENC_EXACT
    bool enc_ready = false;
    scg::DevBuf enc_nc, enc_nr, enc_cmax, enc_rmax, enc_tab, enc_res, enc_status;
    scg::Workspace ws;      // the workspace of the index's own entry points
    // scg_search (host buffers) pipelines a batch in chunks over two streams
    cudaStream_t stream2 = nullptr;
    scg::Workspace ws2;
    int *h_chunk_status = nullptr;  // pinned [8]
    scg::DevBuf q, ids, dists, sums, reqbuf;  // device staging of scg_search
    // scg_search_graph: the captured launch sequence and the arguments it holds
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    std::string graph_key;
    std::mutex mu;
};

namespace scg {

int set_device(scg_index *h);
int check_ready(scg_index *h);
int check_params(scg_index *h, const scg_search_params *p, int nq);
// Builds the fast form's per-vector term once (on stream s).
int ensure_vterm(scg_index *h, cudaStream_t s);
// Enqueues tables, search and re-rank of nq device queries on stream s.
// wait = true: synchronises and returns the status; false: returns after
// enqueueing, the status word lands in ws->h_status when the stream reaches
// it and is read by status_result(ws).
// h_stat (optional): pinned int that receives the status word instead of
// ws->h_status.
// allow_split = false forces the fused kernel.  With wait = true a batch
// whose visited lists outgrew the split kernels' pool is searched again fused.
int run_search(scg_index *h, Workspace *ws, const ReqBufs *rb, const scg_search_params *p, const float *dQ, int nq,
               int *d_ids, float *d_d, int *d_sums, cudaStream_t s, bool wait, int *h_stat = nullptr,
               bool allow_split = true);
// Sizes a workspace's visited-list pool for batches of nq queries.
int reserve_pool(scg_index *h, Workspace *ws, int nq);
int status_result(int st);
// Grows a workspace to a search grid of `grid` CTAs (<= 0: a full grid).
int reserve_search(scg_index *h, Workspace *ws, int mode, int grid);
// The search mode the index's shape implies (IMI, IVFADC or SC).
int index_mode(const scg_index *h);
// The scan form of an arithmetic precision: SCG_FP32_EXACT or SCG_FAST.
int scan_form(int precision);

}  // namespace scg
